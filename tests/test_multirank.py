"""The multi-rank plumbing of bench.py, on CPU: world_size-2 gloo ranks for
the cross-rank reductions and barrier, and the reference arm launched under
torchrun with two ranks (rank 0 alone measures and prints one line, the other
rank exits 0 without work).  The path has no exchange between GPUs (replicas
only), so these are all the collectives it has."""
import datetime
import json
import os
import socket
import subprocess
import sys

import torch
import torch.distributed as dist
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    sys.path.insert(0, REPO)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    cpu = torch.device("cpu")
    res = {"max": bench.world_reduce(1.5 + rank, cpu, "max"), "sum": bench.world_reduce(1.5 + rank, cpu, "sum")}
    bench.world_barrier()
    with open(os.path.join(out_dir, "rank{}.json".format(rank)), "w") as f:
        json.dump(res, f)
    dist.destroy_process_group()


def test_world_reduce_over_two_gloo_ranks(tmp_path):
    mp.spawn(_rank_main, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    for r in range(2):
        with open(tmp_path / "rank{}.json".format(r)) as f:
            res = json.load(f)
        assert res == {"max": 2.5, "sum": 4.0}


def test_world_reduce_single_process_is_identity():
    sys.path.insert(0, REPO)
    import bench
    assert not dist.is_initialized()
    assert bench.world_reduce(3.25, torch.device("cpu"), "max") == 3.25
    bench.world_barrier()  # no process group: nothing to wait for


def test_reference_arm_under_torchrun_two_ranks():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(_free_port()), "bench.py", "--impl", "reference", "--workload", "prep",
           "--steps", "1", "--warmup", "1"]
    r = subprocess.run(cmd, cwd=REPO, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["cpu_baseline"]["kind"] == "port"
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
