// Runs the serving loop's scheduler (run_scheduler in
// cola_b200/csrc/server_policy.h, the loop the server's thread runs) against a
// fake device on the CPU, for tests/test_server_policy.py: a "device" thread
// completes each launched group after a short random delay and reports it
// through group_finished, as the CUDA driver's callback does in the server.
//
//   server_sched_main <scenario> <seed>
//
// Scenarios: budget (the budget admits one request at a time, requests
// submitted while others run), mix (large budget, mixed keys, bursts), fail
// (some launches fail), stop (shutdown with work queued), sizes / sizes_fifo
// (four requests with 20 ms of copies each arrive first, then a small request
// every millisecond; the fake device serves its queue round robin in 0.5 ms
// turns, as the copy engine takes the pieces of chunked copies; with size
// classes on, and off).  Every wait has a
// deadline; a missed deadline prints STALL and exits 1 (a scheduler that spins
// holding its lock stalls the program instead: the caller's timeout catches
// that).  Prints one "ok ..." line with the counters on success.
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <mutex>
#include <random>
#include <thread>
#include <vector>

#include "server_policy.h"

namespace {

double now_s()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Req {
    uint64_t id = 0;
    int K = 0, xdt = 0, ydt = 0;
    int64_t bytes = 0, copy_bytes = 0;
    double t_submit = 0, t_launch = 0, t_done = 0;
    int state = cola::kPending;
    int status = 0;
};

using Group = cola::SchedGroup<Req>;

struct Slot {
    Group *busy = nullptr;
};

struct FakeServer {
    std::mutex mu;
    std::condition_variable cv_sched, cv_done;
    std::deque<Req *> pending;
    std::vector<Group *> finished;
    std::vector<Slot> slots;
    int64_t budget = 0, used = 0, peak_used = 0;
    int32_t max_group = 16;
    int64_t group_bytes = 32 << 20;
    int64_t small_bytes = 0;  // size classes off unless a scenario sets them
    int32_t small_slots = 1;
    bool stop = false;
    int32_t inflight = 0, max_inflight = 0, groups_launched = 0, max_group_seen = 0;
    int64_t completed = 0, failed = 0;
    std::vector<double> lat_ms;
    double queue_ms_sum = 0, copy_in_ms_sum = 0, kernel_ms_sum = 0, copy_out_ms_sum = 0;
    int64_t timed_groups = 0;
    double t_last = 0, t_window = 0;
    // the fake device
    std::mutex dev_mu;
    std::condition_variable dev_cv;
    std::deque<std::pair<Group *, int>> dev_queue;  // group, microseconds of "work"
    bool dev_stop = false;
    int chunk_us = 1 << 30;     // the device serves queued groups round robin, this long a turn
    int us_per_copy_byte = 0;   // > 0: a group's work is its copy bytes times this (the host link)
    int fail_every = 0;  // > 0: launches whose head id % fail_every == 1 fail
    std::mt19937_64 rng{1};
};

struct FakeDevice {
    static int launch(FakeServer *S, Group *G)
    {
        if (S->fail_every > 0 && G->reqs.front()->id % (uint64_t)S->fail_every == 1)
            return 2;  // as a CUDA error would
        std::lock_guard<std::mutex> lk(S->dev_mu);
        int us = (int)(S->rng() % 400);
        if (S->us_per_copy_byte > 0) {
            int64_t copy = 0;
            for (const Req *r : G->reqs)
                copy += r->copy_bytes;
            us = (int)(copy * S->us_per_copy_byte);
        }
        S->dev_queue.emplace_back(G, us);
        S->dev_cv.notify_all();
        return 0;
    }
    static void read_timings(FakeServer *, Group *G)
    {
        G->timed = true;
        G->ms[0] = G->ms[1] = G->ms[2] = 0.1f;
    }
    static void release_failed(FakeServer *, Group *) {}
    static double now() { return now_s(); }
};

void device_thread(FakeServer *S)
{
    std::unique_lock<std::mutex> lk(S->dev_mu);
    while (true) {
        S->dev_cv.wait(lk, [&] { return S->dev_stop || !S->dev_queue.empty(); });
        if (S->dev_queue.empty() && S->dev_stop)
            return;
        auto job = S->dev_queue.front();
        S->dev_queue.pop_front();
        const int turn = std::min(job.second, S->chunk_us);
        lk.unlock();
        std::this_thread::sleep_for(std::chrono::microseconds(turn));
        if (turn < job.second) {  // the rest of this group's work waits for its next turn
            lk.lock();
            S->dev_queue.emplace_back(job.first, job.second - turn);
            continue;
        }
        cola::group_finished(S, job.first, now_s());  // no lock of the server held here
        lk.lock();
    }
}

int fail_stall(const char *what)
{
    std::printf("STALL %s\n", what);
    std::fflush(stdout);
    std::_Exit(1);  // threads may be stuck: do not join them
}

}  // namespace

int main(int argc, char **argv)
{
    if (argc < 3)
        return 2;
    const char *scen = argv[1];
    const uint64_t seed = std::strtoull(argv[2], nullptr, 10);
    FakeServer S;
    S.rng.seed(seed);
    std::mt19937_64 rng(seed * 7 + 1);
    const bool budget_case = !std::strcmp(scen, "budget");
    const bool sizes_case = !std::strncmp(scen, "sizes", 5);
    const int nlarge = 4;
    const int nreq = !std::strcmp(scen, "stop") ? 300 : (sizes_case ? nlarge + 60 : 400);
    S.slots.resize(4);
    S.max_group = 8;
    S.group_bytes = 3000;
    S.budget = budget_case ? 1500 : 1000000;  // budget: one request (1000 bytes) at a time
    S.fail_every = !std::strcmp(scen, "fail") ? 5 : 0;
    if (sizes_case) {
        S.us_per_copy_byte = 1;
        S.chunk_us = 500;
        S.small_bytes = !std::strcmp(scen, "sizes") ? 100 : 0;
    }
    std::thread dev(device_thread, &S);
    std::thread sched([&] { cola::run_scheduler<FakeServer, FakeDevice>(&S); });

    std::vector<Req *> reqs;
    for (int i = 0; i < nreq; i++) {
        Req *r = new Req();
        r->id = (uint64_t)i + 1;
        r->K = budget_case ? 64 : (int)(16 << (rng() % 3));
        r->xdt = budget_case ? 0 : (int)(rng() % 2);
        r->bytes = budget_case ? 1000 : 100 + (int64_t)(rng() % 900);
        r->copy_bytes = 50 + (int64_t)(rng() % 1000);
        if (sizes_case) {
            r->K = 64;
            r->xdt = 0;
            r->bytes = 1000;
            r->copy_bytes = i < nlarge ? 20000 : 20;  // 20 ms and 20 us of copies
        }
        {
            std::lock_guard<std::mutex> lk(S.mu);
            r->t_submit = now_s();
            S.pending.push_back(r);
        }
        S.cv_sched.notify_all();
        reqs.push_back(r);
        if (sizes_case) {
            if (i >= nlarge - 1)
                std::this_thread::sleep_for(std::chrono::milliseconds(1));
        } else if (rng() % 4 == 0) {  // bursts, with requests arriving while others run
            std::this_thread::sleep_for(std::chrono::microseconds(rng() % 300));
        }
    }
    const auto deadline = std::chrono::steady_clock::now() + std::chrono::seconds(30);
    if (!std::strcmp(scen, "stop")) {
        // shutdown with work queued: pending requests are cancelled, running ones finish
        {
            std::lock_guard<std::mutex> lk(S.mu);  // a scheduler spinning on the lock stalls here (the caller's timeout)
            S.stop = true;
            for (Req *r : S.pending)
                r->state = cola::kCancelled;
            S.pending.clear();
        }
        S.cv_sched.notify_all();
    } else {
        std::unique_lock<std::mutex> lk(S.mu);
        const bool all = S.cv_done.wait_until(lk, deadline, [&] {
            for (Req *r : reqs)
                if (r->state < cola::kDone)
                    return false;
            return true;
        });
        if (!all)
            fail_stall("requests not finished by the deadline");
        S.stop = true;
        lk.unlock();
        S.cv_sched.notify_all();
    }
    // the scheduler must end once nothing is in flight
    for (int i = 0; i < 3000; i++) {
        {
            std::lock_guard<std::mutex> lk(S.mu);
            if (S.stop && S.inflight == 0 && S.pending.empty() && S.finished.empty())
                break;
        }
        std::this_thread::sleep_for(std::chrono::milliseconds(10));
    }
    std::atomic<bool> ended{false};
    std::thread joiner([&] {
        sched.join();
        ended = true;
    });
    for (int i = 0; i < 1000 && !ended; i++)
        std::this_thread::sleep_for(std::chrono::milliseconds(10));
    if (!ended)
        fail_stall("scheduler did not end");
    joiner.join();
    {
        std::lock_guard<std::mutex> lk(S.dev_mu);
        S.dev_stop = true;
    }
    S.dev_cv.notify_all();
    dev.join();

    int64_t done = 0, failed = 0, cancelled = 0, other = 0;
    for (Req *r : reqs) {
        if (r->state == cola::kDone)
            done++;
        else if (r->state == cola::kFailed)
            failed++;
        else if (r->state == cola::kCancelled)
            cancelled++;
        else
            other++;
    }
    // latency (submission to completion) of the small and the large requests, in microseconds
    int64_t small_max = 0, large_min = -1;
    for (size_t i = 0; i < reqs.size(); i++) {
        const int64_t us = (int64_t)((reqs[i]->t_done - reqs[i]->t_submit) * 1e6);
        if (sizes_case && (int)i >= nlarge)
            small_max = std::max(small_max, us);
        else if (sizes_case)
            large_min = large_min < 0 ? us : std::min(large_min, us);
    }
    std::printf("ok done=%lld failed=%lld cancelled=%lld other=%lld used=%lld peak=%lld budget=%lld "
                "max_inflight=%d max_group=%d groups=%d completed=%lld sfailed=%lld small_max_us=%lld "
                "large_min_us=%lld\n",
                (long long)done, (long long)failed, (long long)cancelled, (long long)other, (long long)S.used,
                (long long)S.peak_used, (long long)S.budget, S.max_inflight, S.max_group_seen, S.groups_launched,
                (long long)S.completed, (long long)S.failed, (long long)small_max, (long long)large_min);
    for (Req *r : reqs)
        delete r;
    return 0;
}
