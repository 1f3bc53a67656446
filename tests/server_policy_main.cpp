// Runs the serving loop's admission policy (cola_b200/csrc/server_policy.h) on
// scenarios read from stdin, for tests/test_server_policy.py.
//
// Default mode, pick_group: T, then per scenario "used budget max_group
// group_bytes n" and n lines "K xdt ydt bytes copy_bytes".  Output: one line
// per scenario, the chosen positions separated by spaces ("-" for none).
//
// Mode "wake", scheduler_has_work: T lines "finished stop inflight
// admissible"; output one 0/1 line each.
//
// Mode "admit", pick_admission: T, then per scenario "used budget max_group
// group_bytes small_bytes slot_free large_slot_free n" and n request lines as
// above.  Output: "S" (small group) or "L", then the chosen positions ("-" for
// none).
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <deque>

#include "server_policy.h"

struct Req {
    int K, xdt, ydt;
    int64_t bytes, copy_bytes;
};

static int wake_mode()
{
    int T = 0;
    if (std::scanf("%d", &T) != 1)
        return 2;
    for (int t = 0; t < T; t++) {
        int finished, stop, inflight, admissible;
        if (std::scanf("%d %d %d %d", &finished, &stop, &inflight, &admissible) != 4)
            return 2;
        std::printf("%d\n", cola::scheduler_has_work(finished != 0, stop != 0, inflight, admissible != 0) ? 1 : 0);
    }
    return 0;
}

static bool read_reqs(int n, std::deque<Req> &store)
{
    for (int i = 0; i < n; i++) {
        Req r;
        long long b, c;
        if (std::scanf("%d %d %d %lld %lld", &r.K, &r.xdt, &r.ydt, &b, &c) != 5)
            return false;
        r.bytes = b;
        r.copy_bytes = c;
        store.push_back(r);
    }
    return true;
}

static int admit_mode()
{
    int T = 0;
    if (std::scanf("%d", &T) != 1)
        return 2;
    for (int t = 0; t < T; t++) {
        long long used, budget, group_bytes, small_bytes;
        int max_group, slot_free, large_free, n;
        if (std::scanf("%lld %lld %d %lld %lld %d %d %d", &used, &budget, &max_group, &group_bytes, &small_bytes,
                       &slot_free, &large_free, &n) != 8)
            return 2;
        std::deque<Req> store;
        if (!read_reqs(n, store))
            return 2;
        std::deque<Req *> pending;
        for (Req &r : store)
            pending.push_back(&r);
        const cola::Admission a = cola::pick_admission(pending, used, budget, max_group, group_bytes, small_bytes,
                                                       slot_free != 0, large_free != 0);
        std::printf("%s", a.small ? "S" : "L");
        if (a.pick.empty())
            std::printf(" -");
        for (size_t k : a.pick)
            std::printf(" %zu", k);
        std::printf("\n");
    }
    return 0;
}

int main(int argc, char **argv)
{
    if (argc > 1 && std::strcmp(argv[1], "wake") == 0)
        return wake_mode();
    if (argc > 1 && std::strcmp(argv[1], "admit") == 0)
        return admit_mode();
    int T = 0;
    if (std::scanf("%d", &T) != 1)
        return 2;
    for (int t = 0; t < T; t++) {
        long long used, budget, group_bytes;
        int max_group, n;
        if (std::scanf("%lld %lld %d %lld %d", &used, &budget, &max_group, &group_bytes, &n) != 5)
            return 2;
        std::deque<Req> store;
        std::deque<Req *> pending;
        if (!read_reqs(n, store))
            return 2;
        for (Req &r : store)
            pending.push_back(&r);
        const std::vector<size_t> pick = cola::pick_group(pending, used, budget, max_group, group_bytes);
        if (pick.empty())
            std::printf("-\n");
        for (size_t k = 0; k < pick.size(); k++)
            std::printf(k + 1 < pick.size() ? "%zu " : "%zu\n", pick[k]);
    }
    return 0;
}
