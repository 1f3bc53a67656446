// Admission policy of the serving loop, free of CUDA so that it can be tested
// on its own: which pending requests form the next group.
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
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>

namespace cola {

// R: any type with fields K, xdt, ydt (compared for equality), bytes (device
// bytes while in flight) and copy_bytes (host <-> device bytes).  Returns the
// chosen positions of `pending` in increasing order; empty when the head does
// not fit in the budget (or nothing is pending).
template <typename Seq>
std::vector<size_t> pick_group(const Seq &pending, int64_t used, int64_t budget, int32_t max_group,
                               int64_t group_bytes)
{
    std::vector<size_t> out;
    if (pending.empty())
        return out;
    const auto &head = *pending[0];
    if (used + head.bytes > budget)
        return out;
    int64_t bytes = 0, copy = 0;
    for (size_t i = 0; i < pending.size() && (int32_t)out.size() < max_group && copy < group_bytes; i++) {
        const auto &r = *pending[i];
        if (r.K == head.K && r.xdt == head.xdt && r.ydt == head.ydt && used + bytes + r.bytes <= budget &&
            (out.empty() || copy + r.copy_bytes <= group_bytes)) {
            out.push_back(i);
            bytes += r.bytes;
            copy += r.copy_bytes;
        }
    }
    return out;
}

// Whether the scheduler thread has work: a finished group to retire, shutdown
// with nothing in flight, or a head of the queue that can be admitted now (a
// free slot and room in the budget).  A head that does not fit in the budget
// is not work: the scheduler sleeps until a retire frees memory (were it to
// count, the thread would spin holding the lock that the completion callback
// needs to report the retire).
inline bool scheduler_has_work(bool finished, bool stop, int32_t inflight, bool pending, int64_t head_bytes,
                               int64_t used, int64_t budget, bool free_slot)
{
    if (finished || (stop && inflight == 0))
        return true;
    if (!pending || used + head_bytes > budget)
        return false;
    return free_slot;
}

}  // namespace cola
