"""The serving loop's admission policy (cola_b200/csrc/server_policy.h, the
functions the scheduler thread calls), compiled on the CPU.  pick_group is
checked on seeded random queues against the properties it promises: FIFO head
first, one (K, dtypes) key per group, the request-count, copy-byte and
memory-budget caps, and no request left out that would have fitted when it was
considered.  scheduler_has_work is checked over its whole truth table; in
particular a head that does not fit in the budget must not count as work (the
scheduler would spin holding the lock the completion callback needs).  And the
scheduler loop itself (run_scheduler) runs against a fake device on CPU threads:
every request ends, the budget and caps hold, failed launches and shutdown with
work queued end cleanly, all within a deadline."""
import os
import subprocess

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def policy_exe(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("policy") / "server_policy_main")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-Wall", "-Wextra", "-Werror",
                           "-I", os.path.join(REPO, "cola_b200", "csrc"),
                           os.path.join(REPO, "tests", "server_policy_main.cpp"), "-o", exe])
    return exe


def scenarios(seed, count):
    rng = np.random.Generator(np.random.Philox(seed))
    out = []
    for _ in range(count):
        n = int(rng.integers(0, 40))
        keys = [(int(k), int(x), int(y)) for k, x, y in
                zip(rng.choice([16, 64, 256], n), rng.integers(0, 2, n), rng.integers(0, 2, n))]
        if n and rng.random() < 0.5:  # often one key dominates
            keys = [keys[0] if rng.random() < 0.8 else k for k in keys]
        bytes_ = rng.integers(1, 1000, n).astype(np.int64)
        copy = rng.integers(1, 800, n).astype(np.int64)
        used = int(rng.integers(0, 2000))
        budget = used + int(rng.integers(0, 6000))
        max_group = int(rng.integers(1, 17))
        group_bytes = int(rng.integers(1, 4000))
        reqs = [(k[0], k[1], k[2], int(b), int(c)) for k, b, c in zip(keys, bytes_, copy)]
        out.append((used, budget, max_group, group_bytes, reqs))
    return out


def run(exe, cases):
    lines = [str(len(cases))]
    for used, budget, max_group, group_bytes, reqs in cases:
        lines.append("{} {} {} {} {}".format(used, budget, max_group, group_bytes, len(reqs)))
        lines += ["{} {} {} {} {}".format(*r) for r in reqs]
    res = subprocess.run([exe], input="\n".join(lines) + "\n", capture_output=True, text=True, check=True)
    picks = []
    for line in res.stdout.splitlines():
        picks.append([] if line.strip() == "-" else [int(v) for v in line.split()])
    assert len(picks) == len(cases)
    return picks


def check(case, pick):
    used, budget, max_group, group_bytes, reqs = case
    if not reqs or used + reqs[0][3] > budget:
        assert pick == []  # nothing pending, or the head waits for memory
        return
    assert pick and pick[0] == 0  # FIFO: the head opens the group
    assert pick == sorted(set(pick))
    key = reqs[0][:3]
    assert all(reqs[i][:3] == key for i in pick)
    assert len(pick) <= max_group
    assert used + sum(reqs[i][3] for i in pick) <= budget
    assert len(pick) == 1 or sum(reqs[i][4] for i in pick) <= group_bytes
    # nothing left out that fitted when the scan reached it
    chosen = set(pick)
    n_in, b_in, c_in = 0, 0, 0
    for i, r in enumerate(reqs):
        if n_in >= max_group or c_in >= group_bytes:
            break  # the scan stops here
        fits = (r[:3] == key and used + b_in + r[3] <= budget and (n_in == 0 or c_in + r[4] <= group_bytes))
        assert fits == (i in chosen), (i, r, pick)
        if fits:
            n_in, b_in, c_in = n_in + 1, b_in + r[3], c_in + r[4]
    assert n_in == len(pick)


def test_policy_properties_on_random_queues(policy_exe):
    cases = scenarios(seed=11, count=3000)
    for case, pick in zip(cases, run(policy_exe, cases)):
        check(case, pick)


def test_policy_edge_cases(policy_exe):
    big = (64, 0, 0, 10 ** 12, 10 ** 12)
    small = (64, 0, 0, 10, 10)
    cases = [
        (0, 100, 4, 100, []),                                   # nothing pending
        (0, 100, 4, 100, [(64, 0, 0, 101, 1)]),                 # the head cannot fit yet
        (0, 10 ** 13, 4, 100, [big, small, small]),             # a huge head still gets a group of its own
        (0, 100, 1, 10 ** 6, [small, small, small]),            # max_group 1
        (0, 35, 8, 10 ** 6, [small, small, small, small]),      # the budget admits three
        (0, 10 ** 6, 8, 25, [small, small, small, small]),      # the copy cap admits two
        (0, 10 ** 6, 8, 10 ** 6, [small, (16, 0, 0, 1, 1), small, (64, 1, 0, 1, 1), small]),  # keys
    ]
    picks = run(policy_exe, cases)
    assert picks == [[], [], [0], [0], [0, 1, 2], [0, 1], [0, 2, 4]]
    for case, pick in zip(cases, picks):
        check(case, pick)


def test_scheduler_wake_condition(policy_exe):
    import itertools
    rows, want = [], []
    for finished, stop, inflight, admissible in itertools.product([0, 1], [0, 1], [0, 2], [0, 1]):
        rows.append("{} {} {} {}".format(finished, stop, inflight, admissible))
        want.append(int(bool(finished) or (bool(stop) and inflight == 0) or bool(admissible)))
    res = subprocess.run([policy_exe, "wake"], input="{}\n{}\n".format(len(rows), "\n".join(rows)),
                         capture_output=True, text=True, check=True)
    got = [int(v) for v in res.stdout.split()]
    assert got == want
    # the stall this rules out: requests queued behind a head that waits for
    # memory, a slot free, nothing finished yet -> nothing is admissible, so
    # the scheduler must sleep
    assert admit(policy_exe, [(500, 1000, 8, 10 ** 6, 0, 1, 1, [(64, 0, 0, 600, 1), (64, 0, 0, 100, 1)])]) == \
        [("L", [])]


def admit(exe, cases):
    lines = [str(len(cases))]
    for used, budget, max_group, group_bytes, small, slot_free, large_free, reqs in cases:
        lines.append("{} {} {} {} {} {} {} {}".format(used, budget, max_group, group_bytes, small, slot_free,
                                                        large_free, len(reqs)))
        lines += ["{} {} {} {} {}".format(*r) for r in reqs]
    res = subprocess.run([exe, "admit"], input="\n".join(lines) + "\n", capture_output=True, text=True,
                         check=True)
    out = []
    for line in res.stdout.splitlines():
        f = line.split()
        out.append((f[0], [] if f[1:] == ["-"] else [int(v) for v in f[1:]]))
    assert len(out) == len(cases)
    return out


def test_size_classes_admission(policy_exe):
    """pick_admission: a small request (copies at most small_bytes) passes a
    large head that waits for a slot, in the memory left beside the head's; a
    head that waits for memory is passed by nothing; a group holds one size
    class; with the classes off it is pick_group."""
    L = (64, 0, 0, 100, 10 ** 6)     # large: 1 MB of copies in these units
    Sm = (64, 0, 0, 10, 5)           # small
    S16 = (16, 0, 0, 10, 5)          # small, another key
    big = 10 ** 9
    cases = [
        (0, big, 8, 10 ** 7, 100, 1, 1, [L, Sm, Sm]),      # a large slot is free: FIFO, the large head alone
        (0, big, 8, 10 ** 7, 100, 1, 0, [L, Sm, L, Sm]),   # no large slot: the small ones pass, only small join
        (0, big, 8, 10 ** 7, 100, 1, 0, [L, S16, Sm, S16]),  # the first small opens; its key only
        (0, big, 8, 10 ** 7, 100, 0, 0, [L, Sm]),          # no slot at all: nothing
        (0, 150, 8, 10 ** 7, 100, 1, 1, [L, Sm, Sm]),      # room for the head: it goes, alone (one class)
        (60, 150, 8, 10 ** 7, 100, 1, 0, [L, Sm, Sm, Sm]),  # the head waits for memory: nothing passes
        (20, 140, 8, 10 ** 7, 100, 1, 0, [L, Sm, Sm, Sm]),  # 120 with the head's 100 kept: two smalls fit
        (0, big, 8, 10 ** 7, 100, 1, 0, [Sm, L, Sm]),      # small head: a small group, the large one skipped
        (0, big, 8, 10 ** 7, 0, 1, 0, [L, Sm, Sm]),        # classes off: plain FIFO whatever the slots
        (0, big, 2, 10 ** 7, 100, 1, 0, [L, Sm, Sm, Sm]),  # max_group caps the small group
    ]
    got = admit(policy_exe, cases)
    assert got == [("L", [0]), ("S", [1, 3]), ("S", [1, 3]), ("L", []), ("L", [0]), ("L", []), ("S", [1, 2]),
                   ("S", [0, 2]), ("L", [0, 1, 2]), ("S", [1, 2])]


def test_size_classes_random_queues_never_starve_the_head(policy_exe):
    """On random queues: whatever pick_admission admits fits the budget and
    holds one size class; a head that waits for memory is passed by nothing;
    a small group passing a large head leaves the head's bytes free; with a
    slot its class may take and room for it, the head is admitted first."""
    rng = np.random.Generator(np.random.Philox(21))
    cases = []
    for _ in range(2000):
        n = int(rng.integers(1, 20))
        reqs = [(64, 0, 0, int(rng.integers(1, 500)), int(rng.choice([5, 50, 5000]))) for _ in range(n)]
        used = int(rng.integers(0, 1000))
        cases.append((used, used + int(rng.integers(0, 2000)), int(rng.integers(1, 9)), 10 ** 6, 100,
                      int(rng.integers(0, 2)), int(rng.integers(0, 2)), reqs))
    for case, (cls, pick) in zip(cases, admit(policy_exe, cases)):
        used, budget, max_group, _, small, slot_free, large_free, reqs = case
        head = reqs[0]
        if not slot_free:
            assert pick == []
            continue
        assert used + sum(reqs[i][3] for i in pick) <= budget and len(pick) <= max_group
        assert len({reqs[i][4] <= small for i in pick}) <= 1
        if used + head[3] > budget:
            assert pick == []
        elif head[4] <= small or large_free:
            assert pick and pick[0] == 0 and cls == ("S" if head[4] <= small else "L")
        elif pick:
            assert cls == "S" and pick[0] > 0 and all(reqs[i][4] <= small for i in pick)
            assert used + head[3] + sum(reqs[i][3] for i in pick) <= budget


@pytest.fixture(scope="module")
def sched_exe(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("sched") / "server_sched_main")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-pthread",
                           "-I", os.path.join(REPO, "cola_b200", "csrc"),
                           os.path.join(REPO, "tests", "server_sched_main.cpp"), "-o", exe])
    return exe


def run_sched(exe, scenario, seed):
    # a scheduler that spins holding its lock never returns: the timeout ends it
    res = subprocess.run([exe, scenario, str(seed)], capture_output=True, text=True, timeout=90)
    assert res.returncode == 0, res.stdout + res.stderr
    line = res.stdout.strip().splitlines()[-1]
    assert line.startswith("ok "), line
    return {k: int(v) for k, v in (kv.split("=") for kv in line.split()[1:])}


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_scheduler_loop_budget_one_at_a_time(sched_exe, seed):
    c = run_sched(sched_exe, "budget", seed)
    assert c["done"] == 400 and c["other"] == 0
    assert c["max_inflight"] == 1 and c["peak"] <= c["budget"]
    assert c["used"] == 0 and c["completed"] == 400


@pytest.mark.parametrize("seed", [1, 2])
def test_scheduler_loop_mixed_keys(sched_exe, seed):
    c = run_sched(sched_exe, "mix", seed)
    assert c["done"] == 400 and c["other"] == 0 and c["used"] == 0
    assert c["max_inflight"] > 1 and c["max_group"] > 1 and c["groups"] < 400
    assert c["max_group"] <= 8 and c["peak"] <= c["budget"]


def test_scheduler_loop_failed_launches(sched_exe):
    c = run_sched(sched_exe, "fail", 4)
    assert c["failed"] > 0 and c["done"] + c["failed"] == 400 and c["other"] == 0
    assert c["sfailed"] == c["failed"] and c["used"] == 0


def test_scheduler_loop_shutdown_with_work_queued(sched_exe):
    c = run_sched(sched_exe, "stop", 5)
    assert c["done"] + c["cancelled"] == 300 and c["other"] == 0 and c["used"] == 0


def test_scheduler_loop_has_no_data_race(tmp_path):
    """The same runs under ThreadSanitizer: no data race between the scheduler,
    the submitting thread and the completion reports."""
    exe = str(tmp_path / "server_sched_tsan")
    build = subprocess.run(["g++", "-O1", "-g", "-std=c++17", "-fsanitize=thread", "-pthread",
                            "-I", os.path.join(REPO, "cola_b200", "csrc"),
                            os.path.join(REPO, "tests", "server_sched_main.cpp"), "-o", exe],
                           capture_output=True, text=True)
    if build.returncode != 0:
        pytest.skip("ThreadSanitizer unavailable: " + build.stderr.strip().splitlines()[-1])
    for scenario in ("budget", "fail", "stop"):
        res = subprocess.run([exe, scenario, "9"], capture_output=True, text=True, timeout=300)
        assert "ThreadSanitizer" not in res.stderr, res.stderr[:4000]
        assert res.returncode == 0 and res.stdout.startswith("ok "), res.stdout + res.stderr[:2000]


def test_small_requests_are_not_held_behind_large_copies(sched_exe):
    """Four requests with 20 ms of copies each arrive first, then a small
    request every millisecond, on a fake device that serves its queue round
    robin in 0.5 ms turns (chunked copies).  Plain FIFO: the large requests
    take every slot and each small one waits for one of them to finish.  With
    size classes one slot stays free for small requests, which finish within a
    few turns while the large copies are still running."""
    on = run_sched(sched_exe, "sizes", 3)
    off = run_sched(sched_exe, "sizes_fifo", 3)
    for c in (on, off):
        assert c["done"] == 64 and c["other"] == 0 and c["used"] == 0
    assert on["small_max_us"] < 10000 < on["large_min_us"]
    assert off["small_max_us"] > 15000
