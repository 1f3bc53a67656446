"""The row-major view behind the default schedule (build_row_view in
cola_b200/csrc/prep.cpp, which cola_graph_upload runs), built on the CPU from
the partition arrays and checked against the oracle: the merged view must be
the global CSR (the reference's A.tocsr(), prep_torch_par.py:93-101, with
duplicates summed in input order), hub rows must be cut into fixed segments,
and the other rows packed into tasks by the greedy rule."""
import os
import subprocess

import numpy as np
import pytest

import cola_b200 as cb
from oracle import oracle

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def row_view_exe(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("rowview") / "row_view_main")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-fopenmp", "-I", os.path.join(REPO, "include"),
                           "-I", os.path.join(REPO, "cola_b200", "csrc"), "-I", "/usr/local/cuda/include",
                           os.path.join(REPO, "tests", "row_view_main.cpp"),
                           os.path.join(REPO, "cola_b200", "csrc", "prep.cpp"), "-o", exe])
    return exe


def build(exe, tmp_path, n, row, col, val, P, thr, seg, te):
    inp, out = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    with open(inp, "wb") as f:
        np.array([n, P], np.int32).tofile(f)
        np.array([len(row), thr, seg, te], np.int64).tofile(f)
        np.asarray(row, np.int32).tofile(f)
        np.asarray(col, np.int32).tofile(f)
        np.asarray(val, np.float32).tofile(f)
    subprocess.run([exe, inp, out], check=True, timeout=120)
    arrays = []
    with open(out, "rb") as f:
        for dt in (np.int64, np.int32, np.float32, np.int32, np.int64, np.int32, np.int64, np.int32, np.int32):
            cnt = int(np.fromfile(f, np.int64, 1)[0])
            arrays.append(np.fromfile(f, dt, cnt))
    return dict(zip(("ptr", "col", "val", "seg_row", "seg_beg", "hub_row", "hub_seg", "task_rb", "task_re"), arrays))


def expected_segments_and_tasks(ptr, thr, seg, te):
    """Hub rows (more than thr entries) cut into seg-entry segments; every other
    row packed greedily: a task takes rows while its cost (entries + 2 per row)
    stays below te, closes at the row that reaches te, and never spans a hub."""
    n = len(ptr) - 1
    lens = np.diff(ptr)
    seg_row, seg_beg, hub_row, hub_seg = [], [], [], []
    for r in range(n):
        if lens[r] > thr:
            hub_row.append(r)
            hub_seg.append(len(seg_row))
            for q in range(int(ptr[r]), int(ptr[r + 1]), seg):
                seg_row.append(r)
                seg_beg.append(q)
    hub_seg.append(len(seg_row))
    rb, re_ = [], []
    start, cost = None, 0
    for r in range(n):
        if lens[r] > thr:
            if start is not None:
                rb.append(start)
                re_.append(r)
            start, cost = None, 0
            continue
        if start is None:
            start = r
        cost += int(lens[r]) + 2
        if cost >= te:
            rb.append(start)
            re_.append(r + 1)
            start, cost = None, 0
    if start is not None:
        rb.append(start)
        re_.append(n)
    return seg_row, seg_beg, hub_row, hub_seg, rb, re_


def random_coo(n, nnz, seed):
    rng = np.random.Generator(np.random.Philox(seed))
    row = rng.integers(0, n, nnz).astype(np.int32)
    col = rng.integers(0, n, nnz).astype(np.int32)
    row[: nnz // 10] = 3  # a hub row, with duplicates
    val = rng.standard_normal(nnz).astype(np.float32)
    return row, col, val


CASES = [
    # (graph, P, hub_threshold, hub_segment, task_entries)
    ("rmat12", 4, 256, 256, 128),
    ("rmat12", 8, 16, 8, 64),
    ("rmat12", 3, 1, 1, 1),
    ("random", 5, 40, 16, 100),
    ("random", 1, 10 ** 6, 256, 128),
    ("empty_rows", 4, 4, 2, 16),
]


@pytest.mark.parametrize("graph,P,thr,seg,te", CASES)
def test_row_view_matches_oracle(row_view_exe, tmp_path, graph, P, thr, seg, te):
    if graph == "rmat12":
        n, row, col, val = cb.rmat(12, 16, seed=5)
    elif graph == "random":
        n = 3001
        row, col, val = random_coo(n, 40000, seed=6)
    else:  # most rows empty, the last partition short
        n = 1001
        row, col, val = random_coo(n, 300, seed=7)
    rv = build(row_view_exe, tmp_path, n, row, col, val, P, thr, seg, te)
    rp, ci, vv = oracle.global_csr(n, row, col, val)
    np.testing.assert_array_equal(rv["ptr"], rp.astype(np.int64))
    np.testing.assert_array_equal(rv["col"], ci)
    np.testing.assert_array_equal(rv["val"], vv)  # same additions in the same order: same bits
    seg_row, seg_beg, hub_row, hub_seg, rb, re_ = expected_segments_and_tasks(rv["ptr"], thr, seg, te)
    np.testing.assert_array_equal(rv["seg_row"], np.asarray(seg_row, np.int32))
    np.testing.assert_array_equal(rv["seg_beg"], np.asarray(seg_beg, np.int64))
    np.testing.assert_array_equal(rv["hub_row"], np.asarray(hub_row, np.int32))
    np.testing.assert_array_equal(rv["hub_seg"], np.asarray(hub_seg, np.int64))
    np.testing.assert_array_equal(rv["task_rb"], np.asarray(rb, np.int32))
    np.testing.assert_array_equal(rv["task_re"], np.asarray(re_, np.int32))
    # every non-hub row in exactly one task, tasks in order and disjoint
    covered = np.zeros(n, np.int32)
    for b, e in zip(rb, re_):
        covered[b:e] += 1
    lens = np.diff(rp)
    np.testing.assert_array_equal(covered, (lens <= thr).astype(np.int32))


def test_row_view_rejects_bad_options(row_view_exe, tmp_path):
    n, row, col, val = cb.rmat(9, 8, seed=1)
    with pytest.raises(subprocess.CalledProcessError) as e:
        build(row_view_exe, tmp_path, n, row, col, val, 2, 0, 256, 128)
    assert e.value.returncode == 4


def test_host_builders_clean_under_address_and_ub_sanitizers(tmp_path):
    """The partition build and the row view (host C++ with OpenMP) run clean
    under AddressSanitizer and UndefinedBehaviorSanitizer on power-law, random
    and mostly-empty inputs."""
    exe = str(tmp_path / "row_view_asan")
    build_cmd = ["g++", "-O1", "-g", "-std=c++17", "-fopenmp", "-fsanitize=address,undefined",
                 "-fno-omit-frame-pointer", "-I", os.path.join(REPO, "include"),
                 "-I", os.path.join(REPO, "cola_b200", "csrc"), "-I", "/usr/local/cuda/include",
                 os.path.join(REPO, "tests", "row_view_main.cpp"),
                 os.path.join(REPO, "cola_b200", "csrc", "prep.cpp"), "-o", exe]
    res = subprocess.run(build_cmd, capture_output=True, text=True)
    if res.returncode != 0:
        pytest.skip("sanitizers unavailable: " + res.stderr.strip().splitlines()[-1])
    n1, r1, c1, v1 = cb.rmat(11, 16, seed=5)
    r2, c2, v2 = random_coo(1001, 300, seed=7)
    for (n, row, col, val), P, thr, seg, te in (((n1, r1, c1, v1), 4, 256, 256, 128),
                                                  ((n1, r1, c1, v1), 3, 1, 1, 1),
                                                  ((1001, r2, c2, v2), 8, 4, 2, 16)):
        inp, out = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
        with open(inp, "wb") as f:
            np.array([n, P], np.int32).tofile(f)
            np.array([len(row), thr, seg, te], np.int64).tofile(f)
            np.asarray(row, np.int32).tofile(f)
            np.asarray(col, np.int32).tofile(f)
            np.asarray(val, np.float32).tofile(f)
        run = subprocess.run([exe, inp, out], capture_output=True, text=True, timeout=300,
                             env=dict(os.environ, ASAN_OPTIONS="detect_leaks=1", UBSAN_OPTIONS="halt_on_error=1"))
        assert run.returncode == 0 and "runtime error" not in run.stderr and "ERROR" not in run.stderr, \
            run.stderr[:4000]
