"""Benchmark of the partitioned SpMM on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload bf16|fp32|...]

Default workload (the precision form): R-MAT scale 21 (2,097,152 nodes), avg
degree 48, symmetrised, values D^-1/2 A D^-1/2, P = 8 virtual row partitions,
X 2,097,152 x 256 stored BF16 (rounded from FP32 ~N(0,1), Philox seed 3), FP32
accumulation, BF16 output.  A step is one Y = A X over all partitions, inputs
resident in HBM (default schedule: the row-major view, one writer per output
row).  The metric is algorithmic HBM GB/s:
    B = nnz*(4 + s_v + K*s_x) + (M+1)*4 + M*K*s_y   (s_v = 4)
per step divided by the step time.  Inputs (X and Y 1 GiB each) are larger than
L2, so no L2 flush runs between timed steps.  At one GPU the same line also
carries the plain FP32 path on the identical graph (fp32_same_graph, with the
BF16 speed-up), configuration 2 (R-MAT scale 20, K = 128, FP32) beside the
reference's own CUDA kernels (fp32_config2), and the serving loop's p50/p99
(serving).  roofline.frac is physical: DRAM bytes per SpMM from the committed
ncu summary of the same build, over the kernels' time (alg_frac beside it is
the per-nonzero model above).

Multi-GPU (torchrun): every rank runs an independent replica of the workload
on its own GPU (replicas only: the single-GPU path has no exchange between
GPUs); value = all ranks' bytes / the slowest rank's time.

--impl reference times the reference's own CPU SpMM (SAG_reference_host of
include/utils.cuh, compiled from the reference tree into oracle/_ref) on the
host cores, on a bounded row sample per step.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
# a serving request not back within this long is an error, not an endless wait
WAIT_MS = 600_000
sys.path.insert(0, REPO)

WORKLOADS = {
    # name: (scale, avg_degree, K, nparts, x dtype, y dtype, seed)
    "fp32": dict(scale=20, deg=32, K=128, P=8, xdt="fp32", ydt="fp32", seed=2,
                 desc="R-MAT scale 20 (1,048,576 nodes), avg degree 32, D^-1/2 A D^-1/2; X 1,048,576x128 FP32; "
                      "P=8 virtual row partitions"),
    "bf16": dict(scale=21, deg=48, K=256, P=8, xdt="bf16", ydt="bf16", seed=3,
                 desc="R-MAT scale 21 (2,097,152 nodes), avg degree 48, D^-1/2 A D^-1/2; X 2,097,152x256 BF16 "
                      "(from FP32 N(0,1)), FP32 accumulation, BF16 output; P=8 virtual row partitions"),
    "fp32-k256": dict(scale=21, deg=48, K=256, P=8, xdt="fp32", ydt="fp32", seed=3,
                      desc="R-MAT scale 21 (2,097,152 nodes), avg degree 48, D^-1/2 A D^-1/2; X 2,097,152x256 "
                           "FP32; P=8 virtual row partitions (the plain FP32 path of the precision form)"),
}
BATCHED_DESC = ("512 R-MAT graphs, node counts log-uniform in [1e3, 2e5] (R-MAT at the next power of two, "
                "induced on the first N nodes), avg degree uniform in [4, 64], row-normalised FP32 values, K from "
                "{32, 64, 128} FP32, P=4 partitions each; one persistent launch per step, captured in a CUDA graph, "
                "launch parameters autotuned")
SERVING_DESC = ("64 resident R-MAT graphs (scale uniform in 12..20, avg degree uniform in [8, 48], D^-1/2 A D^-1/2, "
                "P=8) registered once; Poisson arrivals, each request picks a graph uniformly, K from {16, 64, 256, "
                "512}, half BF16 and half FP32 (X and Y), X ~N(0,1) in pinned host memory; admission by a 120 GiB "
                "device budget, 4 slots, requests grouped by (K, dtype) into one launch")
METRIC = "SpMM HBM GB/s (algorithmic bytes / step time)"
PREP_METRIC = "partition build throughput (COO entries / s)"
PREP_DESC = ("partition build of R-MAT scale 20, avg degree 32 (33.5 M COO entries, D^-1/2 A D^-1/2 values), "
             "P=8: local CSR + compacted remote CSC per partition, duplicates merged, as prep_torch_par.py:24-79")


def alg_bytes(nnz, M, K, s_x, s_y, s_v=4):
    return nnz * (4 + s_v + K * s_x) + (M + 1) * 4 + M * K * s_y


def world_reduce(x, dev, op="max"):
    """x reduced over the ranks of the default process group (max or sum);
    x itself when there is one rank."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return x
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def world_barrier():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ---------------------------------------------------------------------------
# clocks sampler (nvidia-smi during the timed region)
# ---------------------------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None
        self.lo = self.hi = 0
        self.t0 = self.t1 = 0.0

    def _lines(self):
        try:
            with open(self.path) as f:
                return sum(1 for line in f if line.endswith("\n"))
        except (OSError, TypeError):
            return 0

    def start(self):
        """Starts nvidia-smi sampling every 200 ms and returns once its first
        sample is written, so that the samples after it cover the load."""
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        t = time.time()
        while time.time() - t < 5.0 and self._lines() == 0 and self.proc.poll() is None:
            time.sleep(0.02)
        self.lo = self._lines()
        self.t0 = time.time()

    def hold(self, step=None, min_s=1.2):
        """Ends the sampled load window.  A timed region shorter than two
        sampling periods would leave nvidia-smi nothing to see, so the same
        work (`step`, untimed) keeps running until the window is min_s long;
        the samples between start() and here are the ones reported."""
        if self.proc is None:
            return
        if step is not None:
            import torch
            while time.time() - self.t0 < min_s:
                step()
                torch.cuda.synchronize()
        self.t1 = time.time()
        self.hi = self._lines()

    def stop(self):
        if self.proc is None:
            return None
        if self.hi == 0:
            self.hold()
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for line in f:
                p = [x.strip() for x in line.split(",")]
                if len(p) >= 9:
                    rows.append(p)
        os.unlink(self.path)
        if self.hi > self.lo:
            rows = rows[self.lo:self.hi]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows), "window_s": round(self.t1 - self.t0, 3),
                "window": "the timed region, then the same work untimed until the window is 1.2 s"}


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------
def make_graph(w):
    import cola_b200 as cb
    n, row, col, val = cb.rmat(w["scale"], w["deg"], w["seed"])
    if w.get("reorder") == "community":
        # the reference's reordering step before partitioning (rabbit_order_write.py:48-55)
        mapping, _ = cb.community_order(n, row, col)
        row, col = cb.relabel_edges(n, row, col, mapping)
        order = np.lexsort((col, row))  # sorted by (row, col) again, as the accuracy check reads it
        row, col, val = row[order], col[order], val[order]
    return n, row, col, val


def dense_x(n, K, seed):
    g = np.random.Generator(np.random.Philox(seed))
    return g.standard_normal((n, K), dtype=np.float32)


def fp64_error(n, row, col, val, Xh, Y, dev, samples=4096, longest=64):
    """Relative Frobenius error of Y on a row sample (evenly spaced rows plus
    the `longest` rows with the most entries, where a power-law graph's hubs
    are) against Y = A X computed in FP64 on the GPU from the FP32 features --
    FP64 is used only in this validation reduction.  Returns (error, rows
    sampled, entries of the longest sampled row)."""
    import torch
    counts = np.bincount(row, minlength=n)
    rowptr = np.zeros(n + 1, np.int64)
    np.cumsum(counts, out=rowptr[1:])
    pick = np.unique(np.concatenate([np.linspace(0, n - 1, samples).astype(np.int64),
                                     np.argsort(counts, kind="stable")[-longest:].astype(np.int64)]))
    crow = [0]
    cols, vals = [], []
    for r in pick:
        a, b = rowptr[r], rowptr[r + 1]
        cols.append(col[a:b])
        vals.append(val[a:b])
        crow.append(crow[-1] + (b - a))
    import warnings
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")  # torch marks sparse CSR as beta
        A = torch.sparse_csr_tensor(torch.tensor(crow, dtype=torch.int64),
                                    torch.from_numpy(np.concatenate(cols).astype(np.int64)),
                                    torch.from_numpy(np.concatenate(vals).astype(np.float64)), size=(len(pick), n),
                                    device=dev, check_invariants=False)
    X64 = torch.from_numpy(Xh).to(dev).double()
    ref = (A @ X64)
    got = Y[torch.from_numpy(pick).to(dev)].double()
    err = float(torch.linalg.norm(got - ref) / torch.linalg.norm(ref))
    del X64
    return err, int(len(pick)), int(counts.max())


PROFILE_FILES = {"fp32": "spmm_dram_rmat20_k128_fp32.md", "bf16": "spmm_dram_rmat21_k256_bf16.md",
                 "fp32-k256": "spmm_dram_rmat21_k256_fp32.md"}


def read_profile(name):
    """The `key = value` lines of a committed ncu summary under profiles/."""
    p = os.path.join(REPO, "profiles", name)
    out = {}
    if not os.path.exists(p):
        return out
    with open(p) as f:
        for line in f:
            t = line.strip()
            if "=" in t and not t.startswith(("|", "#", "ncu", "python")):
                k, v = t.split("=", 1)
                out[k.strip()] = v.strip().split()[0] if v.strip() else ""
    return out


def profiled_traffic(workload, opts_key):
    """DRAM bytes (ncu dram__bytes_read.sum + dram__bytes_write.sum) of one
    SpMM (both of its launches) from the committed summary of this workload,
    when that summary was taken on the native sources built now and with the
    same launch options; else None.  Returns (bytes or None, why)."""
    from cola_b200 import _build
    name = PROFILE_FILES.get(workload)
    if name is None:
        return None, "no profile for this workload"
    prof = read_profile(name)
    if "traffic_bytes_per_spmm" not in prof:
        return None, "profiles/{} absent".format(name)
    have = _build.source_hash()
    if prof.get("build_source_hash") != have:
        return None, "profiles/{} was taken on sources {}, built now: {}".format(
            name, prof.get("build_source_hash"), have)
    if prof.get("launch_options", "") != opts_key:
        return None, "profiles/{} was taken with options {}, this run: {}".format(
            name, prof.get("launch_options"), opts_key)
    return int(float(prof["traffic_bytes_per_spmm"])), "profiles/{} (sources {})".format(name, have)


def measured_peak():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs, burst copy)"
    return 6650.0, "fallback (MEASURED_PEAKS.json absent: the earlier copy measurement on these B200s)"


# ---------------------------------------------------------------------------
# CPU baseline: the reference's own SAG_reference_host on host threads
# ---------------------------------------------------------------------------
def cpu_sample(rp, ci, X, K, nthreads, target_s, rows_hint=None):
    """Runs the reference CPU SpMM over `nthreads` disjoint row blocks spread
    over the matrix.  Returns (seconds, rows, nnz, kind)."""
    from oracle import oracle
    n = len(rp) - 1
    kind = "reference" if oracle.ref_available() else "port"
    rows_per = rows_hint or max(1, min(n // nthreads, 2048))
    blocks = []
    for t in range(nthreads):
        lb = (n // nthreads) * t
        ub = min(n, lb + rows_per)
        blocks.append((lb, ub))
    outs = [np.zeros(((ub - lb), K), np.float32) for lb, ub in blocks]
    if kind == "reference":
        R = oracle.ref()

        def work(i):
            lb, ub = blocks[i]
            R.ref_sag_reference_host(lb, ub, K, rp.ctypes.data, ci.ctypes.data, X.ctypes.data,
                                     outs[i].ctypes.data, 0)
    else:
        L = oracle.lib()

        def work(i):
            lb, ub = blocks[i]
            Yd = np.zeros((ub - lb, K), np.float64)
            sub = np.ascontiguousarray(rp[lb:ub + 1] - rp[lb], np.int32)
            L.orc_spmm_csr_f64(ub - lb, sub.ctypes.data, ci[rp[lb]:].ctypes.data, None, X.ctypes.data, K, K,
                               Yd.ctypes.data, K)
    t0 = time.perf_counter()
    th = [threading.Thread(target=work, args=(i,)) for i in range(nthreads)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    dt = time.perf_counter() - t0
    rows = sum(ub - lb for lb, ub in blocks)
    nnz = int(sum(rp[ub] - rp[lb] for lb, ub in blocks))
    return dt, rows, nnz, kind


def calibrated_cpu(rp, ci, X, K, nthreads, target_s):
    """Grow the per-thread row block until one sample takes ~target_s."""
    n = len(rp) - 1
    rows = 256
    while True:
        dt, r, nnz, kind = cpu_sample(rp, ci, X, K, nthreads, target_s, rows)
        if dt >= target_s * 0.5 or rows >= n // nthreads:
            return dt, r, nnz, kind, rows
        rows = min(n // nthreads, int(rows * max(2.0, target_s / max(dt, 1e-3))))


# ---------------------------------------------------------------------------
def run_reference(args, w):
    from oracle import oracle
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    # the oracle's restatement of the generator: the same graph, bit for bit, with
    # nothing of the product loaded in this process
    n, row, col, val = oracle.rmat(w["scale"], w["deg"], w["seed"])
    rp, ci, _ = oracle.global_csr(n, row, col, val)
    K = w["K"]
    X = dense_x(n, K, w["seed"])
    nth = host_threads()
    dt, rows, nnz, kind, rows_per = calibrated_cpu(rp, ci, X, K, nth, target_s=1.0)
    for _ in range(max(args.warmup - 1, 0)):
        cpu_sample(rp, ci, X, K, nth, 1.0, rows_per)
    times = []
    for _ in range(args.steps):
        dt, rows, nnz, kind = cpu_sample(rp, ci, X, K, nth, 1.0, rows_per)[:4]
        times.append(dt)
    t = sum(times) / len(times)
    s = 4 if w["xdt"] == "fp32" else 2
    B = alg_bytes(nnz, rows, K, 4, 4)  # the bytes the reference moves: it computes in FP32
    v = B / t / 1e9
    sample = "{} threads x {} rows (rows spread over the matrix), {} of {} rows, {} nnz per step".format(
        nth, rows_per, rows, n, nnz)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "GB/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": w["desc"], "nnz": len(row), "K": K, "parallelism": "host threads",
                       "x_storage": w["xdt"] if s == 4 else "fp32 (reference has no BF16 path)"},
            "cpu_baseline": {"value": v, "unit": "GB/s", "cores": nth, "kind": kind, "sample": sample},
            "e2e": {"value": v, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def gather_ceilings(stream):
    """Measured row-gather ceilings of this GPU (cola_probe_gather): 512-byte
    rows at random indices from a 16 MiB table (L2-resident) and from a 4 GiB
    table (DRAM), GB/s."""
    import ctypes

    import cola_b200 as cb
    out = {}
    for name, tb in (("l2", 16 << 20), ("dram", 4 << 30)):
        v = ctypes.c_double()
        rc = cb.lib().cola_probe_gather(tb, 512, 1 << 25, 5, ctypes.c_void_p(stream.cuda_stream), ctypes.byref(v))
        out[name] = v.value if rc == 0 else None
    return out


def spmm_kw(args):
    """Launch options of the row-major schedule given on the command line."""
    return dict(unroll=args.unroll, min_blocks=args.min_blocks, k_tile=args.k_tile)


def opts_key(args):
    return "unroll={},min_blocks={},k_tile={}".format(args.unroll, args.min_blocks, args.k_tile)


def time_steps(step, steps, warmup, stream):
    """Average device time of `steps` calls of step() between two CUDA events
    on `stream`, after `warmup` untimed calls, synchronised on both sides."""
    import torch
    for _ in range(max(warmup, 3)):
        step()
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record(stream)
    for _ in range(steps):
        step()
    ev[1].record(stream)
    torch.cuda.synchronize()
    return ev[0].elapsed_time(ev[1]) / steps


def time_each(step, runs, stream):
    """Device time of each of `runs` calls (CUDA events around every call)."""
    import torch
    kev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(runs)]
    for a, b in kev:
        a.record(stream)
        step()
        b.record(stream)
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in kev]


def run_ours(args, w):
    import torch
    import torch.distributed as dist

    import cola_b200 as cb
    from cola_b200 import spmm as S

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if not torch.cuda.is_available():
        raise RuntimeError("bench.py needs a CUDA device")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", device_id=dev)

    t0 = time.time()
    n, row, col, val = make_graph(w)
    ps = cb.PartitionSet.from_coo(n, row, col, val, w["P"])
    K = w["K"]
    Xh = dense_x(n, K, w["seed"])
    t_prep = time.time() - t0
    stream = torch.cuda.current_stream()
    g = S.Graph(ps, hub_threshold=args.hub_threshold, hub_segment=args.hub_segment, task_entries=args.task_entries,
                stream=stream)
    info = g.info
    xdt = torch.float32 if w["xdt"] == "fp32" else torch.bfloat16
    ydt = torch.float32 if w["ydt"] == "fp32" else torch.bfloat16
    s_x = 4 if xdt == torch.float32 else 2
    s_y = 4 if ydt == torch.float32 else 2
    X = torch.from_numpy(Xh).to(dev).to(xdt)
    Y = torch.empty((n, K), dtype=ydt, device=dev)
    sched = {"auto": S.SCHEDULE_AUTO, "fused": S.SCHEDULE_FUSED, "buffer": S.SCHEDULE_BUFFER,
             "rows": S.SCHEDULE_ROWS}[args.schedule]
    eff = S.SCHEDULE_ROWS if sched == S.SCHEDULE_AUTO else sched
    B = alg_bytes(int(info.nnz), n, K, s_x, s_y)
    kw = spmm_kw(args)

    def step():
        g.spmm(X, Y, schedule=sched, stream=stream, **kw)

    def max_over_ranks(x):
        return world_reduce(x, dev, "max")

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    world_barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record(stream)
    for _ in range(args.steps):
        step()
    ev[1].record(stream)
    torch.cuda.synchronize()
    world_barrier()
    torch.cuda.synchronize()
    ms = ev[0].elapsed_time(ev[1]) / args.steps
    ms = max_over_ranks(ms)

    # the SpMM kernels alone: for the fused schedule in accumulate mode (the same
    # launch without the Y zeroing); the row-major schedule has no zeroing
    Yacc = torch.zeros((n, K), dtype=torch.float32, device=dev) if eff == S.SCHEDULE_FUSED else Y
    # at least 50 launches, so that the median is taken over 50 or more runs
    k_list = time_each(lambda: g.spmm(X, Yacc, accumulate=(eff == S.SCHEDULE_FUSED), schedule=sched, stream=stream,
                                      **kw), max(args.steps, 50), stream)
    k_ms = max_over_ranks(sum(k_list) / len(k_list))
    k_med = max_over_ranks(statistics.median(k_list))
    clocks.hold(step)
    clk = clocks.stop()
    del Yacc

    # end to end through the public API: pinned host X -> device, SpMM, Y -> pinned host.
    # Serial: one stream, copy in, multiply, copy out.  Pipelined (the e2e figure): a
    # stream of feature matrices through the resident graph, two steps in flight on
    # double buffers, step i+1's upload overlapping step i's download (PCIe is full
    # duplex); events order every buffer reuse.
    # end to end through the C ABI's host-buffer call (cola_spmm_host): pinned host X in,
    # SpMM, Y out to pinned host memory, every step.  Serial: one call, then wait for it.
    # Pipelined (the e2e figure): a stream of feature matrices through the resident graph,
    # the library overlapping call i+1's upload with call i's download (two staging sets,
    # its own copy streams); the timed region ends when the last Y is in host memory.
    e2e_ms = e2e_serial_ms = None
    if not args.no_e2e:
        Xpin = [torch.from_numpy(Xh).to(xdt).pin_memory() for _ in range(2)]
        Ypin = [torch.empty((n, K), dtype=ydt).pin_memory() for _ in range(2)]
        e2e_steps = max(1, min(args.steps, 30))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

        def host_steps(k, serial):
            e0.record(stream)
            for i in range(k):
                g.spmm_host(Xpin[i % 2], Ypin[i % 2], schedule=sched, stream=stream)
                if serial:
                    g.sync_host()  # the result in host memory before the next call
            g.join_host(stream)
            e1.record(stream)
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / k

        host_steps(2, True)
        world_barrier()
        e2e_serial_ms = max_over_ranks(host_steps(max(1, min(e2e_steps, 10)), True))
        host_steps(2, False)
        world_barrier()
        e2e_ms = max_over_ranks(host_steps(e2e_steps, False))
        world_barrier()
        # the pipelined results are the product too
        Ylast = Ypin[(e2e_steps - 1) % 2]
        g.spmm(X, Y, schedule=sched, stream=stream, **kw)
        torch.cuda.synchronize()
        if not torch.equal(Ylast, Y.cpu()):
            raise RuntimeError("host-buffer e2e: host Y differs from the device result")
        del Xpin, Ypin

    err, nsamp, longest = fp64_error(n, row, col, val, Xh, Y, dev)
    peak, peak_kind = measured_peak()
    compulsory = int(info.nnz) * 8 + n * K * (s_x + s_y)
    overridden = args.scale is not None or args.K is not None or args.reorder != "none"
    if eff == S.SCHEDULE_ROWS and not overridden:
        traffic, traffic_src = profiled_traffic(args.workload, opts_key(args))
    else:
        traffic, traffic_src = None, "no profile for this schedule or size"
    k_s = k_ms * 1e-3
    # physical: DRAM bytes ncu counted for this build / the kernels' time; without a
    # profile of this build, the compulsory bytes (a lower bound of the traffic)
    phys = traffic if traffic is not None else compulsory
    achieved = phys / k_s / 1e9
    alg_achieved = B / k_s / 1e9
    ceil = gather_ceilings(stream) if not (overridden or args.no_extras) else {"l2": None, "dram": None}
    pattern = {"gbps": None, "ms": None}
    if eff == S.SCHEDULE_ROWS and not args.no_extras:
        import ctypes
        v, t = ctypes.c_double(), ctypes.c_float()
        if cb.lib().cola_probe_graph_gather(g._h, ctypes.c_void_p(X.data_ptr()), X.stride(0) * s_x, K * s_x, 5,
                                            ctypes.c_void_p(stream.cuda_stream), ctypes.byref(v),
                                            ctypes.byref(t)) == 0:
            pattern = {"gbps": v.value, "ms": t.value}
    gather_bytes = int(info.nnz) * K * s_x  # the X rows the entries name (the gathers)
    launches_per_step = int(g.get_info().last_launches)  # counted by the library
    line = {
        "metric": METRIC, "value": B * world / (ms * 1e-3) / 1e9, "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32" if xdt == torch.float32 else "bf16-storage/f32-accum",
        "data": "synthetic",
        "config": {"workload": w["desc"], "nodes": n, "nnz": int(info.nnz), "nnz_local": int(info.nnz_local),
                   "nnz_remote": int(info.nnz_remote), "K": K, "nparts": w["P"], "local_chunks": int(info.local_chunks),
                   "remote_chunks": int(info.remote_chunks), "parallelism": "replicas x{}".format(world),
                   "schedule": {S.SCHEDULE_ROWS: "rows", S.SCHEDULE_FUSED: "fused",
                                S.SCHEDULE_BUFFER: "buffer"}.get(eff, args.schedule),
                   "hub_rows": int(info.hub_rows), "hub_segments": int(info.hub_segments),
                   "launch_options": opts_key(args), "row_tasks": int(info.row_tasks),
                   "alg_bytes_per_step": B,
                   "l2": "inputs larger than L2 (X {:.0f} MiB, Y {:.0f} MiB); no flush".format(
                       n * K * s_x / 2 ** 20, n * K * s_y / 2 ** 20),
                   "prep_seconds": round(t_prep, 1)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic,
                     "frac_basis": ("DRAM bytes per SpMM counted by ncu on this build ({}) / the SpMM kernels' "
                                    "time".format(traffic_src)) if traffic is not None else
                                   ("compulsory bytes (indices and values once, X and Y once: a lower bound of the "
                                    "DRAM traffic) / the SpMM kernels' time; traffic null: {}".format(traffic_src)),
                     "peak_source": peak_kind,
                     "kernel_ms": k_ms, "kernel_ms_median": k_med, "kernel_runs": len(k_list),
                     "compulsory_bytes": compulsory,
                     "traffic_over_compulsory": None if traffic is None else traffic / float(compulsory),
                     # the per-nonzero row-gather model: one X row per entry, most of them L2 hits
                     "alg_bytes": B, "alg_achieved": alg_achieved, "alg_frac": alg_achieved / peak,
                     "alg_frac_of_8TBs": alg_achieved / 8000.0,
                     # what bounds the kernel: its X-row gathers against this GPU's own measured
                     # gather ceilings (512-byte rows at random indices, cola_probe_gather)
                     "gather": {"bytes": gather_bytes, "achieved": gather_bytes / k_s / 1e9,
                                "l2_ceiling": ceil["l2"], "dram_ceiling": ceil["dram"],
                                "frac_of_l2_ceiling": None if not ceil["l2"] else
                                gather_bytes / k_s / 1e9 / ceil["l2"],
                                # the same gathers in the same order with no arithmetic and no writes
                                "pattern_ceiling": pattern["gbps"], "pattern_ms": pattern["ms"],
                                "frac_of_pattern_ceiling": None if not pattern["gbps"] else
                                gather_bytes / k_s / 1e9 / pattern["gbps"],
                                "unit": "GB/s",
                                "note": "ceilings: 512-byte rows at random indices from a 16 MiB table (L2) and "
                                        "a 4 GiB table (DRAM), 4 rows in flight per warp, one full wave; "
                                        "pattern: this graph's own entries in order (cola_probe_graph_gather)"}},
        "e2e": None if e2e_ms is None else {
            "value": B * world / (e2e_ms * 1e-3) / 1e9, "unit": "GB/s", "h2d_bytes_per_step": n * K * s_x,
            "d2h_bytes_per_step": n * K * s_y, "ms_per_step": e2e_ms,
            "mode": "cola_spmm_host (C ABI, pinned host X and Y) called once per step; the library pipelines "
                    "consecutive calls, step i+1's X upload overlapping step i's Y download",
            "steps": max(1, min(args.steps, 30)),
            "serial_ms_per_step": e2e_serial_ms,
            "serial_value": B * world / (e2e_serial_ms * 1e-3) / 1e9},
        "accuracy": {"rel_frobenius_vs_fp64": err, "rows_sampled": nsamp, "longest_row_entries": longest,
                     "bound": 1e-5 if (xdt == torch.float32 and ydt == torch.float32) else 1e-2,
                     "reference": "FP64 on the GPU from the FP32 features, 4,096 evenly spaced rows and the 64 "
                                  "longest"},
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clk,
    }
    extras = world == 1 and not args.no_extras and not overridden
    if extras and eff == S.SCHEDULE_ROWS:
        # the project's autotuner on these operands: its choice among the launch options
        # (every candidate gives the same bits), beside the default launch's time
        opts_t, ms_t, _ = g.autotune(X, Y, reps=3, stream=stream)
        line["autotuned"] = {"choice": {k: v for k, v in opts_t.items() if k != "gather_batch_rows"},
                             "ms": ms_t, "default_kernel_ms_median": k_med,
                             "searched": "feature tile per pass x loads in flight x resident blocks per SM "
                                         "(cola_spmm_autotune)"}
    if extras and xdt == torch.bfloat16:
        # the plain FP32 path on the identical graph and features
        X32 = torch.from_numpy(Xh).to(dev)
        Y32 = torch.empty((n, K), dtype=torch.float32, device=dev)

        def step32():
            g.spmm(X32, Y32, schedule=sched, stream=stream, **kw)

        ms32 = time_steps(step32, args.steps, args.warmup, stream)
        k32 = time_each(step32, max(args.steps, 50), stream)
        err32, _, _ = fp64_error(n, row, col, val, Xh, Y32, dev)
        B32 = alg_bytes(int(info.nnz), n, K, 4, 4)
        line["fp32_same_graph"] = {
            "ms_per_step": ms32, "kernel_ms": sum(k32) / len(k32), "value": B32 / (ms32 * 1e-3) / 1e9,
            "unit": "GB/s", "rel_frobenius_vs_fp64": err32, "bound": 1e-5,
            "bf16_speedup": ms32 / ms, "bf16_kernel_speedup": (sum(k32) / len(k32)) / k_ms,
            "note": "same graph, same X (FP32 features, FP32 output); bf16_speedup = FP32 step time / BF16 step "
                    "time"}
        del X32, Y32
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle
        rp, ci, vv = oracle.global_csr(n, row, col, val)
        nth = host_threads()
        dt, rows, nnz, kind, rows_per = calibrated_cpu(rp, ci, Xh, K, nth, target_s=2.0)
        reps = 3
        tt = []
        for _ in range(reps):
            tt.append(cpu_sample(rp, ci, Xh, K, nth, 2.0, rows_per)[0])
        dt = statistics.median(tt)
        Bc = alg_bytes(nnz, rows, K, 4, 4)
        line["cpu_baseline"] = {"value": Bc / dt / 1e9, "unit": "GB/s", "cores": nth, "kind": kind,
                                "sample": "SAG_reference_host (include/utils.cuh:45-69) over {} threads x {} rows "
                                          "spread over the matrix ({} nnz), FP32 X, median of {}".format(
                                              nth, rows_per, nnz, reps)}
        # beside it, torch.sparse.mm on the host over the whole global CSR (FP32)
        try:
            import warnings
            with warnings.catch_warnings():
                warnings.simplefilter("ignore")  # torch marks sparse CSR as beta
                A = torch.sparse_csr_tensor(torch.from_numpy(rp.astype(np.int64)),
                                            torch.from_numpy(ci.astype(np.int64)), torch.from_numpy(vv),
                                            size=(n, n), check_invariants=False)
            Xc = torch.from_numpy(Xh if Xh.dtype == np.float32 else Xh.astype(np.float32))
            torch.set_num_threads(nth)
            torch.sparse.mm(A, Xc[:, :8])
            tt = []
            for _ in range(3):
                t0 = time.perf_counter()
                torch.sparse.mm(A, Xc)
                tt.append(time.perf_counter() - t0)
            line["cpu_baseline"]["torch_sparse_mm"] = {
                "value": alg_bytes(len(ci), n, K, 4, 4) / statistics.median(tt) / 1e9, "unit": "GB/s",
                "cores": nth, "sample": "the whole matrix, FP32, median of 3"}
            del A, Xc
        except (RuntimeError, MemoryError) as e:
            line["cpu_baseline"]["torch_sparse_mm"] = {"unavailable": str(e)[:200]}
        # and an OpenMP loop over the same P partitions (local CSR + remote CSC chunks)
        line["cpu_baseline"]["openmp_partitions"] = openmp_partitions_baseline(ps, Xh, K, w["P"], nth)
        # the reference's own CUDA kernels on this GPU (FP32 only, as the reference)
        if xdt == torch.float32 and ydt == torch.float32:
            line["reference_gpu_kernels"] = reference_kernels_baseline(g, X, n, K, w["P"], B, k_ms, stream)
    g.close()
    del X, Y, g, ps
    torch.cuda.empty_cache()
    if extras and args.workload == "bf16":
        # the FP32 configuration the reference's kernels run (and the serving loop) in the same line
        line["fp32_config2"] = fp32_config2_leg(args, stream)
        torch.cuda.empty_cache()
        if not args.no_serving:
            line["serving"] = serving_leg(args, seconds=args.serve_seconds_default)[0]
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def fp32_config2_leg(args, stream):
    """Configuration 2 (R-MAT scale 20, degree 32, K = 128, FP32, P = 8) on this
    GPU: our step time, its FP64 error, and the reference's own CUDA kernels
    on the same split blocks."""
    import torch

    import cola_b200 as cb
    from cola_b200 import spmm as S
    w = WORKLOADS["fp32"]
    dev = torch.device("cuda", torch.cuda.current_device())
    n, row, col, val = make_graph(w)
    ps = cb.PartitionSet.from_coo(n, row, col, val, w["P"])
    K = w["K"]
    Xh = dense_x(n, K, w["seed"])
    g = S.Graph(ps, stream=stream)
    X = torch.from_numpy(Xh).to(dev)
    Y = torch.empty((n, K), device=dev)
    kw = spmm_kw(args)

    def step():
        g.spmm(X, Y, stream=stream, **kw)

    ms = time_steps(step, args.steps, args.warmup, stream)
    kl = time_each(step, max(args.steps, 50), stream)
    k_ms = sum(kl) / len(kl)
    err, nsamp, _ = fp64_error(n, row, col, val, Xh, Y, dev)
    B = alg_bytes(int(g.info.nnz), n, K, 4, 4)
    compulsory = int(g.info.nnz) * 8 + n * K * 8
    traffic, src = profiled_traffic("fp32", opts_key(args))
    peak, _ = measured_peak()
    out = {"workload": w["desc"], "nnz": int(g.info.nnz), "ms_per_step": ms, "kernel_ms": k_ms,
           "value": B / (ms * 1e-3) / 1e9, "unit": "GB/s", "rel_frobenius_vs_fp64": err, "bound": 1e-5,
           "rows_sampled": nsamp, "traffic": traffic, "traffic_source": src,
           "frac": (traffic if traffic is not None else compulsory) / (k_ms * 1e-3) / 1e9 / peak,
           "alg_frac": B / (k_ms * 1e-3) / 1e9 / peak}
    if not args.no_cpu_baseline:
        out["reference_gpu_kernels"] = reference_kernels_baseline(g, X, n, K, w["P"], B, k_ms, stream)
    g.close()
    del X, Y
    return out


def openmp_partitions_baseline(ps, Xh, K, P, nthreads):
    """The oracle's OpenMP FP32 loop over the P partitions (their split local
    CSR and remote CSC chunks, one thread per partition), whole matrix, median
    of 3."""
    from oracle import oracle
    parts = [ps.part(r) for r in range(P)]
    run = oracle.partitions_f32_omp(parts, ps.nodes_per_part, Xh)
    nt = min(P, nthreads)
    run(nt)
    tt = []
    for _ in range(3):
        t0 = time.perf_counter()
        run(nt)
        tt.append(time.perf_counter() - t0)
    nnz = sum(len(p["csr_colIdx_l"]) + len(p["csc_rowIdx_r"]) for p in parts)
    return {"value": alg_bytes(nnz, Xh.shape[0], K, 4, 4) / statistics.median(tt) / 1e9, "unit": "GB/s",
            "cores": nt, "sample": "the whole matrix, FP32, one OpenMP thread per partition (the oracle's "
                                   "orc_spmm_partitions_f32_omp), median of 3"}


def reference_kernels_baseline(g, X, n, K, P, B, k_ms, stream, steps=10):
    """The reference's own ppl0_batch_SpMM<ceil(K/32), K%32 != 0> (compiled for
    sm_100a through the NVSHMEM shim), launched once per virtual partition on
    this graph's split blocks; the sum of the P kernel durations (CUDA events)
    per SpMM, averaged over `steps` SpMMs after warm-up."""
    import ctypes

    import torch
    from oracle import oracle
    if not oracle.ref_available():
        return {"unavailable": "the reference's kernels are not built (oracle/_ref)"}
    R = oracle.ref()
    CF, res = (K + 31) // 32, 1 if K & 31 else 0
    if CF not in (1, 2, 3, 4, 8, 16):
        return {"unavailable": "no reference instantiation for K={}".format(K)}
    npp = g.nodes_per_part
    Xr = torch.zeros((P * npp, K), device=X.device)
    Xr[:n] = X.float()
    Yr = torch.zeros((P * npp, K), device=X.device)
    zips = [g.zip_view(p) for p in range(P)]
    sh = ctypes.c_void_p(stream.cuda_stream)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(P)]

    import cola_b200 as cb
    L = cb.lib()

    def spmm(ours=False):
        total = 0.0
        for p, z in enumerate(zips):
            if not ours and R.ref_set_pe(p, npp * K, sh) != 0:
                raise RuntimeError("ref_set_pe failed")
            args = [ctypes.c_void_p(Yr[p * npp:].data_ptr()), ctypes.c_void_p(Xr[p * npp:].data_ptr()),
                    z.csr_rowPtr, z.csr_colIdx, z.csr_rowIdx_zip, z.csr_val, z.csc_colPtr, z.csc_rowIdx,
                    z.csc_colIdx_zip, z.csc_val, 0, 0, z.local_chunks, z.remote_chunks, K, npp, p, sh]
            a, b = evs[p]
            a.record(stream)
            rc = L.cola_ppl0_batch_spmm(*args) if ours else R.ref_ppl0_batch_spmm(CF, res, *args)
            b.record(stream)
            if rc != 0:
                raise RuntimeError("kernel launch failed")
        torch.cuda.synchronize()
        for a, b in evs:
            total += a.elapsed_time(b)
        return total
    # the row view of each PE's zip arrays, built once (what compat.h's
    # ppl0_batch_SpMM keeps per d_csr_zip / d_csc_zip pair), then one call per PE
    views = []
    for p, z in enumerate(zips):
        h = ctypes.c_void_p()
        args = [z.csr_rowPtr, z.csr_colIdx, z.csr_rowIdx_zip, z.csr_val, z.csc_colPtr, z.csc_rowIdx,
                z.csc_colIdx_zip, z.csc_val]
        args = [a if a is None or isinstance(a, ctypes.c_void_p) else ctypes.c_void_p(a) for a in args]
        if L.cola_zip_rows_create(*args, 0, 0, z.local_chunks, z.remote_chunks, npp, p, sh, ctypes.byref(h)) != 0:
            raise RuntimeError("cola_zip_rows_create failed")
        views.append(h)

    def spmm_views():
        total = 0.0
        for p, h in enumerate(views):
            a, b = evs[p]
            a.record(stream)
            rc = L.cola_zip_rows_spmm(h, ctypes.c_void_p(Yr[p * npp:].data_ptr()),
                                      ctypes.c_void_p(Xr[p * npp:].data_ptr()), K, sh)
            b.record(stream)
            if rc != 0:
                raise RuntimeError("cola_zip_rows_spmm failed")
        torch.cuda.synchronize()
        for a, b in evs:
            total += a.elapsed_time(b)
        return total

    # one row view of every PE's chunks (what compat.h's distSpMM_ppl_batch_all keeps for
    # a single stage): one call per SpMM
    parts = (cb._lib.ZipPart * P)()
    for p, z in enumerate(zips):
        q = parts[p]
        q.csr_rowPtr_l, q.csr_colIdx_l, q.csr_rowIdx_zip_l, q.csr_val_l = (z.csr_rowPtr, z.csr_colIdx,
                                                                           z.csr_rowIdx_zip, z.csr_val)
        q.csc_colPtr_r, q.csc_rowIdx_r, q.csc_colIdx_zip_r, q.csc_val_r = (z.csc_colPtr, z.csc_rowIdx,
                                                                           z.csc_colIdx_zip, z.csc_val)
        q.local_row_lb, q.remote_col_lb, q.local_row_num, q.remote_col_num = 0, 0, z.local_chunks, z.remote_chunks
    hall = ctypes.c_void_p()
    if L.cola_zip_rows_create_all(parts, P, npp, sh, ctypes.byref(hall)) != 0:
        raise RuntimeError("cola_zip_rows_create_all failed")
    ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def spmm_all():
        ea.record(stream)
        rc = L.cola_zip_rows_spmm(hall, ctypes.c_void_p(Yr.data_ptr()), ctypes.c_void_p(Xr.data_ptr()), K, sh)
        eb.record(stream)
        if rc != 0:
            raise RuntimeError("cola_zip_rows_spmm failed")
        torch.cuda.synchronize()
        return ea.elapsed_time(eb)

    for _ in range(3):
        spmm()
        spmm(True)
        spmm_views()
        spmm_all()
    ms = sum(spmm() for _ in range(steps)) / steps
    ours_kl = sum(spmm(True) for _ in range(steps)) / steps
    ours_rv = sum(spmm_views() for _ in range(steps)) / steps
    ours_all = sum(spmm_all() for _ in range(steps)) / steps
    for h in views:
        L.cola_zip_rows_free(h)
    L.cola_zip_rows_free(hall)
    del Xr, Yr
    return {"ms_per_spmm": ms, "value": B / (ms * 1e-3) / 1e9, "unit": "GB/s",
            "kernel": "ppl0_batch_SpMM<{}, {}> per virtual partition (include/dist_spmm_ppl_batch.cuh:76-245), "
                      "sum of the {} kernel durations".format(CF, "true" if res else "false", P),
            "ours_speedup": ms / k_ms,
            # the same launches through our kernel-level drop-in (cola_ppl0_batch_spmm, the
            # reference's data layout and arguments, chunk kernel)
            "ours_kernel_level_ms_per_spmm": ours_kl, "ours_kernel_level_speedup": ms / ours_kl,
            # the same per-PE calls on the row view of each PE's zip arrays (built once), as
            # compat.h's ppl0_batch_SpMM / distSpMM_ppl_batch_wrapper run them
            "ours_row_view_ms_per_spmm": ours_rv, "ours_row_view_speedup": ms / ours_rv,
            # all PEs' chunks in one row view (compat.h distSpMM_ppl_batch_all, single stage)
            "ours_all_pes_row_view_ms_per_spmm": ours_all, "ours_all_pes_row_view_speedup": ms / ours_all}


def make_batched(count, seed):
    """The batched workload: per graph (N, row, col, val, K)."""
    import cola_b200 as cb
    rng = np.random.Generator(np.random.Philox(seed))
    out = []
    for i in range(count):
        n = int(round(float(np.exp(rng.uniform(np.log(1e3), np.log(2e5))))))
        deg = float(rng.uniform(4, 64))
        K = int(rng.choice([32, 64, 128]))
        scale = int(np.ceil(np.log2(n)))
        # deg*n/2 draws at the next power of two, then the subgraph induced on
        # the first n nodes (R-MAT puts most edges there)
        _, row, col, _ = cb.rmat(scale, deg * n / float(1 << scale), seed=seed * 100000 + i,
                                 values=cb.prep.VALUES_NONE)
        m = (row < n) & (col < n)
        row, col = row[m], col[m]
        d = np.bincount(row, minlength=n).astype(np.float64)
        d[d == 0] = 1.0
        val = (1.0 / d[row]).astype(np.float32)
        out.append((n, row, col, val, K))
    return out


def run_batched(args):
    import torch

    import cola_b200 as cb
    from cola_b200.batch import Batch

    if not torch.cuda.is_available():
        raise RuntimeError("bench.py needs a CUDA device")
    local = int(os.environ.get("LOCAL_RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", device_id=dev)
    t0 = time.time()
    graphs = make_batched(args.batch_graphs, seed=4)
    from cola_b200 import spmm as S
    gobjs = [S.Graph(cb.PartitionSet.from_coo(n, r, c, v, 4)) for (n, r, c, v, K) in graphs]
    b = Batch.from_graphs(gobjs)
    # every graph's X (and Y) is a view of one contiguous buffer, so the e2e
    # leg moves each direction in one copy
    sizes = [n * K for (n, r, c, v, K) in graphs]
    offs = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    X_all = torch.empty(int(offs[-1]), device=dev)
    Y_all = torch.empty(int(offs[-1]), device=dev)
    Xs, Ys, B = [], [], 0
    xh = []
    for i, (n, r, c, v, K) in enumerate(graphs):
        X = dense_x(n, K, 4000 + i)
        xh.append(X)
        Xs.append(X_all[offs[i]:offs[i + 1]].view(n, K))
        Xs[-1].copy_(torch.from_numpy(X))
        Ys.append(Y_all[offs[i]:offs[i + 1]].view(n, K))
        B += alg_bytes(len(r), n, K, 4, 4)
    nnz = sum(len(g[1]) for g in graphs)
    nodes = sum(g[0] for g in graphs)
    t_prep = time.time() - t0
    b.bind(Xs, Ys)
    stream = torch.cuda.current_stream()
    tuned_ms = b.autotune(reps=3, cache=args.tune_cache)
    cap = torch.cuda.Stream()
    b.capture(stream=cap)
    torch.cuda.synchronize()
    for _ in range(max(args.warmup, 3)):
        b.replay(stream)
    torch.cuda.synchronize()
    world_barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        b.replay(stream)
    e1.record(stream)
    torch.cuda.synchronize()
    clocks.hold(lambda: b.replay(stream))
    clk = clocks.stop()
    ms = world_reduce(e0.elapsed_time(e1) / args.steps, dev, "max")
    # e2e: per graph pinned X -> device, the captured launch, Y -> pinned host;
    # two steps in flight on two operand sets (a second batch over the same
    # graphs, launched on the same stream as the first, so their kernels never
    # overlap), uploads of step i+1 overlapping downloads of step i
    e2e_ms = e2e_serial_ms = None
    if not args.no_e2e:
        Xp = torch.empty(X_all.numel(), dtype=torch.float32).pin_memory()
        Yp = torch.empty(Y_all.numel(), dtype=torch.float32).pin_memory()
        Xp.copy_(X_all)
        X_all2, Y_all2 = torch.empty_like(X_all), torch.empty_like(Y_all)
        Xs2 = [X_all2[offs[i]:offs[i + 1]].view(x.shape) for i, x in enumerate(Xs)]
        Ys2 = [Y_all2[offs[i]:offs[i + 1]].view(y.shape) for i, y in enumerate(Ys)]
        b2 = Batch.from_graphs(gobjs)
        b2.bind(Xs2, Ys2)
        bi = b.info
        b2.set_params(unroll=bi.unroll, grid_pct=bi.grid_pct, blocks_per_sm=bi.blocks_per_sm)
        b2.capture(stream=cap)
        torch.cuda.synchronize()
        sets = [(b, X_all, Y_all, Ys), (b2, X_all2, Y_all2, Ys2)]

        def serial_step():
            X_all.copy_(Xp, non_blocking=True)
            b.replay(stream)
            Yp.copy_(Y_all, non_blocking=True)

        s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
        ev = {k: [torch.cuda.Event() for _ in range(2)] for k in ("x_ready", "x_free", "y_ready", "y_free")}
        for k in ev:
            for e in ev[k]:
                e.record(stream)

        def pipelined_step(i):
            k = i % 2
            bk, Xk, Yk, _ = sets[k]
            s_in.wait_event(ev["x_free"][k])
            with torch.cuda.stream(s_in):
                Xk.copy_(Xp, non_blocking=True)
                ev["x_ready"][k].record(s_in)
            stream.wait_event(ev["x_ready"][k])
            stream.wait_event(ev["y_free"][k])
            bk.replay(stream)
            ev["x_free"][k].record(stream)
            ev["y_ready"][k].record(stream)
            s_out.wait_event(ev["y_ready"][k])
            with torch.cuda.stream(s_out):
                Yp.copy_(Yk, non_blocking=True)
                ev["y_free"][k].record(s_out)

        steps = max(1, min(args.steps, 5))
        serial_step()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(steps):
            serial_step()
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_serial_ms = world_reduce(e0.elapsed_time(e1) / steps, dev, "max")
        for i in range(2):
            pipelined_step(i)
        torch.cuda.synchronize()
        e0.record(stream)
        for i in range(steps):
            pipelined_step(i)
        stream.wait_event(ev["y_free"][(steps - 1) % 2])
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = world_reduce(e0.elapsed_time(e1) / steps, dev, "max")
        # the pipelined results are the product too: the last step's set equals the first set's
        last = sets[(steps - 1) % 2][3]
        if not all(torch.equal(a, c) for a, c in zip(last, Ys)):
            raise RuntimeError("batched pipelined e2e: results differ between the two operand sets")
        if not torch.equal(Yp.to(dev), sets[(steps - 1) % 2][2]):
            raise RuntimeError("batched pipelined e2e: host Y differs from the device result")
        b2.close()
        del Xs2, Ys2, X_all2, Y_all2
    # accuracy on three graphs (the largest, a middle one, the smallest)
    order = np.argsort([g[0] for g in graphs])
    errs = []
    for gi in (order[-1], order[len(order) // 2], order[0]):
        n, r, c, v, K = graphs[gi]
        errs.append(fp64_error(n, r, c, v, xh[gi], Ys[gi], dev, samples=1024)[0])
    info = b.info
    peak, peak_kind = measured_peak()
    achieved = B / (ms * 1e-3) / 1e9
    line = {"metric": METRIC, "value": B * world / (ms * 1e-3) / 1e9, "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": BATCHED_DESC, "graphs": len(graphs), "nodes": nodes, "nnz": nnz,
                       "batched_graphs": int(info.batched_graphs), "alg_bytes_per_step": B,
                       "autotuned": {"unroll": int(info.unroll), "grid_pct": int(info.grid_pct),
                                     "blocks_per_sm": int(info.blocks_per_sm),
                                     "from_cache": bool(b.tuned_from_cache),
                                     "best_ms": tuned_ms},
                       "parallelism": "replicas x{}".format(world),
                       "l2": "inputs larger than L2; no flush", "prep_seconds": round(t_prep, 1)},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None, "peak_source": peak_kind,
                         "kernel_ms": ms, "frac_of_8TBs": achieved / 8000.0},
            "e2e": None if e2e_ms is None else {
                "value": B * world / (e2e_ms * 1e-3) / 1e9, "unit": "GB/s",
                "h2d_bytes_per_step": int(sum(x.numel() * 4 for x in Xs)),
                "d2h_bytes_per_step": int(sum(y.numel() * 4 for y in Ys)), "ms_per_step": e2e_ms,
                "mode": "pipelined: two steps in flight on two operand sets, uploads overlapping downloads",
                "serial_ms_per_step": e2e_serial_ms, "serial_value": B * world / (e2e_serial_ms * 1e-3) / 1e9},
            "accuracy": {"rel_frobenius_vs_fp64_max": max(errs), "graphs_checked": 3, "bound": 1e-5},
            "gpu_launches": int(info.last_launches) * args.steps, "clocks": clk}
    if rank == 0:
        print(json.dumps(line), flush=True)
    b.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def serving_leg(args, seconds):
    """The serving workload: 64 resident graphs, a saturation burst, then an
    open loop of Poisson arrivals at args.serve_load of the saturation rate for
    `seconds`.  Returns the `serving` object of the bench line plus the served
    bytes, wall time, request count and clocks."""
    import torch

    import cola_b200 as cb
    from cola_b200.serving import Server

    local = int(os.environ.get("LOCAL_RANK", "0"))
    t0 = time.time()
    rng = np.random.Generator(np.random.Philox(5))
    srv = Server(memory_budget=120 << 30, slots=4, max_group=16, small_mib=args.serve_small_mib,
                 copy_chunk_mib=args.serve_chunk_mib, copy_engines_only=args.serve_copy_engines_only)
    gn, gnnz = [], []
    for i in range(args.serve_graphs):
        scale = int(rng.integers(12, 21))
        deg = float(rng.uniform(8, 48))
        n, row, col, val = cb.rmat(scale, deg, seed=5000 + i)
        ps = cb.PartitionSet.from_coo(n, row, col, val, 8)
        srv.register(ps)
        gn.append(n)
        gnnz.append(len(row))
        del ps, row, col, val
    max_n = max(gn)
    Ks = (16, 64, 256, 512)
    xin, yout = {}, {}
    for K in Ks:
        xf = torch.from_numpy(dense_x(max_n, K, 600 + K)).pin_memory()
        xin[(K, torch.float32)] = xf
        xin[(K, torch.bfloat16)] = xf.to(torch.bfloat16).pin_memory()
        # results are not read back by the benchmark: requests of one (K, dtype)
        # share an output area (the correctness of every result is a test)
        yout[(K, torch.float32)] = torch.empty((max_n, K), dtype=torch.float32).pin_memory()
        yout[(K, torch.bfloat16)] = torch.empty((max_n, K), dtype=torch.bfloat16).pin_memory()
    t_prep = time.time() - t0

    def draw():
        g = int(rng.integers(0, len(gn)))
        K = int(rng.choice(Ks))
        dt = torch.float32 if rng.random() < 0.5 else torch.bfloat16
        return g, K, dt

    def submit(g, K, dt):
        n = gn[g]
        return srv.submit(g, xin[(K, dt)][:n], out_dtype=dt, Y=yout[(K, dt)][:n])

    def req_bytes(g, K, dt):
        sz = 4 if dt == torch.float32 else 2
        return alg_bytes(gnnz[g], gn[g], K, sz, sz)

    def copy_bytes(g, K, dt):
        return 2 * gn[g] * K * (4 if dt == torch.float32 else 2)

    # warm-up (single requests, then one untimed burst, which also grows the
    # server's memory pool to its working size), then the saturation rate: a
    # burst submitted at once
    for _ in range(max(args.warmup, 3)):
        submit(*draw()).wait(timeout_ms=WAIT_MS)
    for r in [submit(*draw()) for _ in range(args.serve_burst)]:
        r.wait(timeout_ms=WAIT_MS)
    world_barrier()
    burst = [draw() for _ in range(args.serve_burst)]
    tb = time.perf_counter()
    reqs = [submit(*d) for d in burst]
    for r in reqs:
        r.wait(timeout_ms=WAIT_MS)
    cap = len(burst) / (time.perf_counter() - tb)
    # open loop: Poisson arrivals at a fraction of the saturation rate
    rate = args.serve_load * cap
    nreq = max(args.serve_min_requests, int(rate * seconds))
    srv.reset_stats()
    clocks = Clocks(local)
    clocks.start()
    plan = [draw() for _ in range(nreq)]
    gaps = rng.exponential(1.0 / rate, nreq)
    # per size class: latency from submission to the result in host memory,
    # taken by a waiter thread per request as its wait returns (the server's
    # own statistics cover all requests together)
    import concurrent.futures as cf
    lat = [0.0] * nreq

    def waiter(i, r, t0):
        r.wait(timeout_ms=WAIT_MS)
        lat[i] = (time.perf_counter() - t0) * 1e3

    futs = []
    ts = time.perf_counter()
    t_next = ts
    with cf.ThreadPoolExecutor(max_workers=64) as pool:
        for i, (d, gap) in enumerate(zip(plan, gaps)):
            t_next += gap
            delay = t_next - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            t0 = time.perf_counter()
            futs.append(pool.submit(waiter, i, submit(*d), t0))
        for f in futs:
            f.result()
    wall = time.perf_counter() - ts
    clk = clocks.stop()
    st = srv.stats()
    B = sum(req_bytes(*d) for d in plan)
    h2d = sum(gn[g] * K * (4 if dt == torch.float32 else 2) for g, K, dt in plan) / nreq
    classes = {}
    for (gi, K, dt), ms_ in zip(plan, lat):
        mb = copy_bytes(gi, K, dt) / 2 ** 20
        c = "small (<16 MiB of copies)" if mb < 16 else ("medium (16-256 MiB)" if mb < 256 else "large (>=256 MiB)")
        classes.setdefault(c, []).append(ms_)
    per_class = {c: {"requests": len(v), "p50_ms": float(np.percentile(v, 50)), "p99_ms": float(np.percentile(v, 99))}
                 for c, v in sorted(classes.items())}
    srv.close()
    return {"workload": SERVING_DESC, "graphs": len(gn), "nodes": int(sum(gn)), "nnz": int(sum(gnnz)),
            "offered_req_per_s": rate, "saturation_req_per_s": cap, "achieved_req_per_s": st["req_per_s"],
            "sustained": st["req_per_s"] >= 0.95 * rate,
            "completed": st["completed"], "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"],
            "max_ms": st["max_ms"], "mean_ms": st["mean_ms"], "max_inflight": st["max_inflight"],
            "groups_launched": st["groups_launched"], "max_group": st["max_group"],
            "queue_ms_mean": st["queue_ms_mean"], "copy_in_ms_mean": st["copy_in_ms_mean"],
            "kernel_ms_mean": st["kernel_ms_mean"], "copy_out_ms_mean": st["copy_out_ms_mean"],
            "peak_device_bytes": st["peak_bytes"], "budget_bytes": st["budget"],
            "per_size_class": per_class, "open_loop_seconds": round(wall, 2),
            "small_mib": args.serve_small_mib or 16, "copy_chunk_mib": args.serve_chunk_mib or 32,
            "small_groups_copied_by": "copy engines" if args.serve_copy_engines_only else
            "SM kernels on the pinned host buffers",
            "served_GBps": B / wall / 1e9, "prep_seconds": round(t_prep, 1),
            "latency": "submit to result in pinned host memory"}, B, wall, nreq, h2d, clk


def run_serving(args):
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("bench.py needs a CUDA device")
    local = int(os.environ.get("LOCAL_RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", device_id=dev)
    serving, B, wall, nreq, h2d, clk = serving_leg(args, args.serve_seconds)
    value = world_reduce(B / wall / 1e9, dev, "sum")
    peak, peak_kind = measured_peak()
    line = {"metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": nreq,
            "warmup": max(args.warmup, 3), "ms_per_step": wall * 1e3 / nreq, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 and bf16-storage/f32-accum", "data": "synthetic",
            "config": {"workload": SERVING_DESC, "graphs": serving["graphs"], "nodes": serving["nodes"],
                       "nnz": serving["nnz"], "parallelism": "replicas x{}".format(world),
                       "prep_seconds": serving["prep_seconds"]},
            "serving": serving,
            "roofline": {"bound": "hbm", "achieved": value / world, "peak": peak, "unit": "GB/s",
                         "frac": value / world / peak, "traffic": None,
                         "peak_source": peak_kind,
                         "note": "served rate, PCIe copies of X and Y included"},
            "e2e": {"value": value, "unit": "GB/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(h2d)},
            "gpu_launches": None, "clocks": clk}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def prep_case(oracle_gen=False):
    if oracle_gen:  # the reference leg loads nothing of the product
        from oracle import oracle
        return oracle.rmat(20, 32, 2), 8
    import cola_b200 as cb
    return cb.rmat(20, 32, seed=2), 8


def oracle_partitions(n, row, col, val, P, nthreads):
    """The oracle's row_partition for every partition, partitions spread over
    host threads (the C calls release the GIL).  Returns seconds."""
    import concurrent.futures as cf

    from oracle import oracle
    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(max_workers=nthreads) as ex:
        list(ex.map(lambda r: oracle.row_partition(n, row, col, P, r, val), range(P)))
    return time.perf_counter() - t0


def prep_sort_passes(n, P):
    npp = (n + P - 1) // P
    bits = (max(npp - 1, 0)).bit_length() + (max(n - 1, 0)).bit_length() + (2 * P - 1).bit_length()
    return (bits + 7) // 8


def run_prep_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    (n, row, col, val), P = prep_case(oracle_gen=True)
    nth = min(host_threads(), P)
    for _ in range(max(args.warmup - 1, 0)):
        oracle_partitions(n, row, col, val, P, nth)
    times = [oracle_partitions(n, row, col, val, P, nth) for _ in range(args.steps)]
    t = sum(times) / len(times)
    v = len(row) / t / 1e6
    line = {"impl": "reference", "metric": PREP_METRIC, "value": v, "unit": "M entries/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": PREP_DESC, "nnz": len(row), "parallelism": "host threads"},
            "cpu_baseline": {"value": v, "unit": "M entries/s", "cores": nth, "kind": "port",
                             "sample": "the whole workload: the oracle's row_partition (a C restatement of "
                                       "prep_torch_par.py:24-79; the reference's own is Python/scipy) for all {} "
                                       "partitions on {} threads".format(P, nth)},
            "e2e": {"value": v, "unit": "M entries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_prep(args):
    import torch

    import cola_b200 as cb

    if not torch.cuda.is_available():
        raise RuntimeError("bench.py needs a CUDA device")
    local = int(os.environ.get("LOCAL_RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", device_id=dev)
    (n, row, col, val), P = prep_case()
    nnz = len(row)
    rh = torch.from_numpy(row).pin_memory()
    ch = torch.from_numpy(col).pin_memory()
    vh = torch.from_numpy(val).pin_memory()
    rd, cd, vd = rh.to(dev), ch.to(dev), vh.to(dev)
    stream = torch.cuda.current_stream()

    def build(r, c, v):
        return cb.PartitionSet.from_coo_device(n, r, c, v, P)

    for _ in range(max(args.warmup, 3)):
        build(rd, cd, vd).close()
    torch.cuda.synchronize()
    world_barrier()
    clocks = Clocks(local)
    clocks.start()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record(stream)
    for _ in range(args.steps):
        build(rd, cd, vd).close()
    ev[1].record(stream)
    torch.cuda.synchronize()
    clocks.hold(lambda: build(rd, cd, vd).close())
    clk = clocks.stop()
    ms = world_reduce(ev[0].elapsed_time(ev[1]) / args.steps, dev, "max")
    # end to end: pinned host COO -> device, build, partitions in host memory
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2e_steps = max(1, min(args.steps, 5))
    e0.record(stream)
    for _ in range(e2e_steps):
        ps = build(rh.to(dev, non_blocking=True), ch.to(dev, non_blocking=True), vh.to(dev, non_blocking=True))
        d2h = 0
        for r in range(P):
            v = ps.part_view(r)
            d2h += 4 * (v.n_rowPtr_l + 2 * v.nnz_l + v.n_rows_l + v.n_colPtr_r + 2 * v.nnz_r + v.n_cols_r)
        ps.close()
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / e2e_steps
    # the whole graph on the device (row view, hubs, tasks): COO -> ready to multiply
    from cola_b200 import spmm as S
    for _ in range(2):
        S.Graph.from_coo_device(n, rd, cd, vd, P).close()
    torch.cuda.synchronize()
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g0.record(stream)
    gsteps = max(1, min(args.steps, 10))
    for _ in range(gsteps):
        S.Graph.from_coo_device(n, rd, cd, vd, P).close()
    g1.record(stream)
    torch.cuda.synchronize()
    graph_ms = g0.elapsed_time(g1) / gsteps
    th = time.perf_counter()
    gh = S.Graph(cb.PartitionSet.from_coo(n, row, col, val, P))
    torch.cuda.synchronize()
    host_graph_ms = (time.perf_counter() - th) * 1e3
    # full-size parity of the two graphs: the same SpMM bits (K = 128, FP32)
    gd = S.Graph.from_coo_device(n, rd, cd, vd, P)
    Xg = torch.from_numpy(dense_x(n, 128, 2)).to(dev)
    graph_same = bool(torch.equal(gd.spmm(Xg), gh.spmm(Xg, schedule=S.SCHEDULE_ROWS)))
    gd.close()
    gh.close()
    del Xg
    # parity of this very workload against the product's host build
    ref = cb.PartitionSet.from_coo(n, row, col, val, P)
    got = build(rd, cd, vd)
    same = all(np.array_equal(got.part(r)[k], ref.part(r)[k]) for r in range(P) for k in
               ("csr_rowPtr_l", "csr_colIdx_l", "csr_rowIdx_l", "csc_colPtr_r", "csc_rowIdx_r", "csc_colIdx_r",
                "csr_val_l", "csc_val_r"))
    passes = prep_sort_passes(n, P)
    sort_bytes = 32 * passes * nnz
    peak, peak_kind = measured_peak()
    achieved = sort_bytes / (ms * 1e-3) / 1e9
    line = {"metric": PREP_METRIC, "value": nnz * world / (ms * 1e-3) / 1e6, "unit": "M entries/s", "n_gpus": world,
            "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32 (+ f32 value sums)", "data": "synthetic",
            "config": {"workload": PREP_DESC, "nnz": nnz, "nparts": P, "radix_passes": passes,
                       "parallelism": "replicas x{}".format(world),
                       "l2": "inputs larger than L2 (sort buffers {:.0f} MiB); no flush".format(24 * nnz / 2 ** 20)},
            "parity": {"identical_to_host_build": bool(same)},
            "graph_build": {"device_ms": graph_ms, "host_partition_and_upload_ms": host_graph_ms,
                            "spmm_identical_to_host_graph": graph_same,
                            "note": "COO in device memory -> graph ready for the row-major SpMM, built on the GPU "
                                    "(cola_graph_build_device), against the host partitioning + upload"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None, "peak_source": peak_kind,
                         "note": "radix sort bytes (32 B per entry per 8-bit pass) over the whole build's time"},
            "e2e": {"value": nnz * world / (e2e_ms * 1e-3) / 1e6, "unit": "M entries/s",
                    "h2d_bytes_per_step": 12 * nnz, "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_ms},
            # per build: range check, keys, 5 per radix pass (counts, 3-launch scan, scatter),
            # 2 x (scan + pass) for duplicates and rows, group bounds, 3 output launches
            "gpu_launches": (14 + 5 * passes) * args.steps, "clocks": clk}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        t = oracle_partitions(n, row, col, val, P, 1)
        line["cpu_baseline"] = {"value": nnz / t / 1e6, "unit": "M entries/s", "cores": 1, "kind": "port",
                                "sample": "the whole workload once: the oracle's row_partition (C restatement of "
                                          "prep_torch_par.py:24-79) for all {} partitions, one thread".format(P)}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0 if same and graph_same else 1


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="bf16", choices=sorted(WORKLOADS) + ["batched", "serving", "prep"])
    ap.add_argument("--serve-graphs", type=int, default=64)
    ap.add_argument("--serve-burst", type=int, default=64, help="serving: requests of the saturation burst")
    ap.add_argument("--serve-load", type=float, default=0.7, help="serving: offered rate / saturation rate")
    ap.add_argument("--serve-seconds", type=float, default=20.0, help="serving: length of the open-loop phase")
    ap.add_argument("--serve-min-requests", type=int, default=100)
    ap.add_argument("--serve-small-mib", type=int, default=0,
                    help="serving: size-class threshold in MiB of copies (0 = library default 16, -1 = FIFO)")
    ap.add_argument("--serve-chunk-mib", type=int, default=0, help="serving: copy piece size (0 = library default)")
    ap.add_argument("--serve-copy-engines-only", action="store_true",
                    help="serving: small groups copy with the copy engines too (no SM copies)")
    ap.add_argument("--batch-graphs", type=int, default=512, help="batched workload: number of graphs")
    ap.add_argument("--tune-cache", default=None, help="batched workload: autotuner cache file (tuned once per shape)")
    ap.add_argument("--schedule", default="auto", choices=["auto", "fused", "buffer", "rows"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling runs)")
    ap.add_argument("--hub-threshold", type=int, default=0, help="row-major schedule: hub split threshold")
    ap.add_argument("--hub-segment", type=int, default=0, help="row-major schedule: hub segment length")
    ap.add_argument("--unroll", type=int, default=0, help="row-major schedule: loads in flight per lane group")
    ap.add_argument("--task-entries", type=int, default=0, help="row-major schedule: entries per row-block task")
    ap.add_argument("--min-blocks", type=int, default=0, help="row-major schedule: resident blocks per SM")
    ap.add_argument("--k-tile", type=int, default=0, help="row-major schedule: features per pass (0 = library's)")
    ap.add_argument("--no-extras", action="store_true",
                    help="default workload: skip the FP32 same-graph, configuration-2 and serving legs")
    ap.add_argument("--no-serving", action="store_true", help="default workload: skip the serving leg")
    ap.add_argument("--serve-seconds-default", type=float, default=10.0,
                    help="default workload: open-loop length of its serving leg")
    ap.add_argument("--scale", type=int, default=None, help="override the R-MAT scale (profiling runs)")
    ap.add_argument("--K", type=int, default=None, help="override the feature width (exploration runs)")
    ap.add_argument("--reorder", default="none", choices=["none", "community"],
                    help="relabel the graph by cola_community_order before partitioning (exploration runs)")
    args = ap.parse_args()
    if args.workload == "prep":
        return run_prep_reference(args) if args.impl == "reference" else run_prep(args)
    if args.workload in ("batched", "serving"):
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no {} form".format(
                "batched multi-graph" if args.workload == "batched" else "serving")}))
            return 0
        return run_batched(args) if args.workload == "batched" else run_serving(args)
    w = dict(WORKLOADS[args.workload])
    if args.scale is not None:
        w["scale"] = args.scale
        w["desc"] = "{} [scale overridden to {}]".format(w["desc"], args.scale)
    if args.K is not None:
        w["K"] = args.K
        w["desc"] = "{} [K overridden to {}]".format(w["desc"], args.K)
    if args.reorder != "none":
        w["reorder"] = args.reorder
        w["desc"] = "{} [vertices in community order]".format(w["desc"])
    if args.impl == "reference":
        return run_reference(args, w)
    return run_ours(args, w)


if __name__ == "__main__":
    sys.exit(main())
