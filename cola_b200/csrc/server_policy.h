// The serving loop's scheduling, free of CUDA so that it can be tested on its
// own: the admission policy (which pending requests form the next group), the
// wake condition, and the scheduler loop itself over device hooks.
//
// FIFO: the oldest pending request (the head) opens a group when the budget
// has room for it next to what is already in flight.  Later pending requests
// with the head's key (feature width and dtypes) join in queue order while
//   * the group has fewer than max_group requests,
//   * the group's copy bytes are below group_bytes when the request is
//     considered, and stay within group_bytes with it (a group always takes
//     its head, however large),
//   * the budget has room for the group with the request.
// A request that does not fit is skipped, not dropped: it stays pending.
//
// Size classes (pick_admission): a request whose host<->device copies are at
// most small_bytes is small, the others large.  A group holds one class only.
// Small groups may take any free slot; large groups leave the last
// small_slots slots to small ones.  When the head is large and no slot a large
// group may take is free, the oldest small request opens a small group
// instead, so that small requests are not held behind large copies; the
// memory the head needs stays free for it (a small group passes only if the
// head still fits beside it), so the head cannot be starved.  A head that
// waits for memory is passed by nothing (memory is granted in queue order).
#pragma once
#include <algorithm>
#include <condition_variable>
#include <cstddef>
#include <cstdint>
#include <mutex>
#include <type_traits>
#include <vector>

namespace cola {

// Life of a request: pending (queued) -> running (admitted in a group) ->
// done | failed, or pending -> cancelled.
enum ReqState { kPending = 0, kRunning = 1, kDone = 2, kCancelled = 3, kFailed = 4 };

// A group: requests admitted together into one slot.
template <typename Req>
struct SchedGroup {
    std::vector<Req *> reqs;
    int slot = 0;
    int64_t bytes = 0;
    bool completed = false;
    bool small = false;  // opened by a small request (size classes)
    bool by_sms = false;  // its copies run as kernels (the server's small groups)
    bool timed = false;
    float ms[3] = {0, 0, 0};  // copy-in, launch, copy-out (read when retired)
};

// The group opened by pending[first]: it and the later requests with its key
// and, when small_bytes > 0, its size class, in queue order, under the count,
// copy-byte and budget caps above.  Empty when pending[first] does not fit in
// the budget.
template <typename Seq>
std::vector<size_t> scan_group(const Seq &pending, size_t first, int64_t used, int64_t budget, int32_t max_group,
                               int64_t group_bytes, int64_t small_bytes)
{
    std::vector<size_t> out;
    if (first >= pending.size())
        return out;
    const auto &head = *pending[first];
    if (used + head.bytes > budget)
        return out;
    const bool head_small = head.copy_bytes <= small_bytes;
    int64_t bytes = 0, copy = 0;
    for (size_t i = first; i < pending.size() && (int32_t)out.size() < max_group && copy < group_bytes; i++) {
        const auto &r = *pending[i];
        if (r.K == head.K && r.xdt == head.xdt && r.ydt == head.ydt && used + bytes + r.bytes <= budget &&
            (out.empty() || copy + r.copy_bytes <= group_bytes) &&
            (small_bytes <= 0 || (r.copy_bytes <= small_bytes) == head_small)) {
            out.push_back(i);
            bytes += r.bytes;
            copy += r.copy_bytes;
        }
    }
    return out;
}

// R: any type with fields K, xdt, ydt (compared for equality), bytes (device
// bytes while in flight) and copy_bytes (host <-> device bytes).  Returns the
// chosen positions of `pending` in increasing order; empty when the head does
// not fit in the budget (or nothing is pending).
template <typename Seq>
std::vector<size_t> pick_group(const Seq &pending, int64_t used, int64_t budget, int32_t max_group,
                               int64_t group_bytes)
{
    return scan_group(pending, 0, used, budget, max_group, group_bytes, 0);
}

struct Admission {
    std::vector<size_t> pick;  // positions in `pending`, increasing
    bool small = false;        // a small group (opened by a small request)
};

// The next group to admit under the size classes (header comment), or none.
// slot_free: some slot is free; large_slot_free: a slot that a large group may
// take is free.  small_bytes <= 0 turns the classes off (pick_group alone).
template <typename Seq>
Admission pick_admission(const Seq &pending, int64_t used, int64_t budget, int32_t max_group, int64_t group_bytes,
                         int64_t small_bytes, bool slot_free, bool large_slot_free)
{
    Admission a;
    if (pending.empty() || !slot_free)
        return a;
    const auto &head = *pending[0];
    if (used + head.bytes > budget)
        return a;  // the head waits for memory; nothing passes it
    const bool head_small = small_bytes > 0 && head.copy_bytes <= small_bytes;
    if (head_small || large_slot_free || small_bytes <= 0) {
        a.pick = scan_group(pending, 0, used, budget, max_group, group_bytes, small_bytes);
        a.small = head_small;
        return a;
    }
    // a large head waits for a slot: the oldest small request opens a small
    // group in the memory left beside the head's
    for (size_t i = 1; i < pending.size(); i++)
        if (pending[i]->copy_bytes <= small_bytes) {
            a.pick = scan_group(pending, i, used + head.bytes, budget, max_group, group_bytes, small_bytes);
            a.small = !a.pick.empty();
            return a;
        }
    return a;
}

// Whether the scheduler thread has work: a finished group to retire, shutdown
// with nothing in flight, or a group that pick_admission would admit now
// (`admissible`).  Requests that cannot be admitted are not work: the
// scheduler sleeps until a retire frees a slot or memory (were they to count,
// the thread would spin holding the lock that the completion callback needs to
// report the retire).
inline bool scheduler_has_work(bool finished, bool stop, int32_t inflight, bool admissible)
{
    return finished || (stop && inflight == 0) || admissible;
}

// Free slots for pick_admission: any free slot, and a free slot a large group
// may take (large groups in flight fewer than slots - small_slots).
template <typename Srv>
void free_slots(const Srv *S, bool &slot_free, bool &large_slot_free)
{
    int32_t busy = 0, large = 0;
    for (const auto &sl : S->slots)
        if (sl.busy) {
            busy++;
            large += sl.busy->small ? 0 : 1;
        }
    const int32_t n = (int32_t)S->slots.size();
    const int32_t reserved = S->small_bytes > 0 ? std::min(S->small_slots, n - 1) : 0;
    slot_free = busy < n;
    large_slot_free = slot_free && large < n - reserved;
}

template <typename Srv>
Admission next_admission(const Srv *S)
{
    bool slot_free = false, large_slot_free = false;
    free_slots(S, slot_free, large_slot_free);
    return pick_admission(S->pending, S->used, S->budget, S->max_group, S->group_bytes, S->small_bytes, slot_free,
                          large_slot_free);
}

// Reports a group's device work as complete: called once per launched group,
// from any thread (the CUDA driver's callback thread in the server), never
// with S->mu held.
template <typename Srv, typename Group>
void group_finished(Srv *S, Group *G, double t)
{
    {
        std::lock_guard<std::mutex> lk(S->mu);
        for (auto *r : G->reqs)
            r->t_done = t;
        G->completed = true;
        S->finished.push_back(G);
    }
    S->cv_sched.notify_all();
}

// The scheduler thread: retire finished groups (return their memory to the
// budget, wake waiters), then admit pending requests into free slots, a group
// at a time as pick_group chooses; sleep while scheduler_has_work says there
// is nothing to do; end once stopped with nothing in flight.  Srv holds the
// server's state (mu, cv_sched, cv_done, pending, finished, slots[].busy,
// used, budget, inflight, stop, the group caps and the statistics).  B holds
// the device hooks, none of them called with S->mu held:
//   B::launch(S, G)          queue the group's work (0 = queued); the work's
//                            completion must call group_finished(S, G, t)
//   B::read_timings(S, G)    fill G->timed and G->ms for a finished group
//   B::release_failed(S, G)  free what a launch that failed had queued
//   B::now()                 seconds
template <typename Srv, typename B>
void run_scheduler(Srv *S)
{
    using Group = typename std::remove_pointer<typename decltype(S->finished)::value_type>::type;
    std::unique_lock<std::mutex> lk(S->mu);
    while (true) {
        S->cv_sched.wait(lk, [&] {
            return scheduler_has_work(!S->finished.empty(), S->stop, S->inflight,
                                      !S->finished.empty() || !next_admission(S).pick.empty());
        });
        // retire (the timings are read without the lock; a finished group's
        // slot stays busy until it is retired, so its timing state is not
        // reused meanwhile)
        std::vector<Group *> done;
        done.swap(S->finished);
        if (!done.empty()) {
            lk.unlock();
            for (Group *G : done)
                B::read_timings(S, G);
            lk.lock();
        }
        for (Group *G : done) {
            if (G->reqs.front()->t_submit >= S->t_window && G->timed) {
                S->copy_in_ms_sum += G->ms[0];
                S->kernel_ms_sum += G->ms[1];
                S->copy_out_ms_sum += G->ms[2];
                S->timed_groups++;
            }
            S->slots[(size_t)G->slot].busy = nullptr;
            S->used -= G->bytes;
            S->inflight -= (int32_t)G->reqs.size();
            for (auto *r : G->reqs) {
                r->state = kDone;
                if (r->t_submit >= S->t_window) {
                    S->completed++;
                    S->lat_ms.push_back((r->t_done - r->t_submit) * 1e3);
                    S->queue_ms_sum += (r->t_launch - r->t_submit) * 1e3;
                    S->t_last = std::max(S->t_last, r->t_done);
                }
            }
            delete G;
        }
        if (!done.empty())
            S->cv_done.notify_all();
        if (S->stop && S->pending.empty() && S->inflight == 0)
            break;
        // admit
        while (!S->pending.empty()) {
            const Admission adm = next_admission(S);
            if (adm.pick.empty())
                break;  // no slot for the classes waiting, or no memory
            const std::vector<size_t> &pick = adm.pick;
            int slot = -1;
            for (size_t i = 0; i < S->slots.size(); i++)
                if (!S->slots[i].busy) {
                    slot = (int)i;
                    break;
                }
            Group *G = new Group();
            G->slot = slot;
            G->small = adm.small;
            for (size_t i : pick) {
                auto *r = S->pending[i];
                G->reqs.push_back(r);
                G->bytes += r->bytes;
                r->state = kRunning;
            }
            for (size_t k = pick.size(); k-- > 0;)  // back to front: earlier positions stay valid
                S->pending.erase(S->pending.begin() + (std::ptrdiff_t)pick[k]);
            S->used += G->bytes;
            S->peak_used = std::max(S->peak_used, S->used);
            S->inflight += (int32_t)G->reqs.size();
            S->max_inflight = std::max(S->max_inflight, S->inflight);
            S->max_group_seen = std::max(S->max_group_seen, (int32_t)G->reqs.size());
            S->groups_launched++;
            S->slots[(size_t)slot].busy = G;
            const double t_launch = B::now();
            for (auto *r : G->reqs)
                r->t_launch = t_launch;
            // launch without the lock: the completion of earlier groups must
            // be able to report meanwhile
            lk.unlock();
            const auto st = B::launch(S, G);
            if (st != 0)
                B::release_failed(S, G);  // it never reaches group_finished
            lk.lock();
            if (st != 0) {
                S->slots[(size_t)slot].busy = nullptr;
                S->used -= G->bytes;
                S->inflight -= (int32_t)G->reqs.size();
                for (auto *r : G->reqs) {
                    r->state = kFailed;
                    r->status = st;
                    S->failed++;
                }
                delete G;
                S->cv_done.notify_all();
            }
        }
    }
}

}  // namespace cola
