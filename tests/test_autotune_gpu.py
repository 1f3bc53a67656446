"""The single-graph autotuner (cola_spmm_autotune) and the launch options it
searches.  Row-major schedule, K >= 128 (FP32 X) or >= 256 (BF16 X): every
(k_tile, unroll, min_blocks) candidate gives the same bits, so the tuned run
is the untuned run; the tuner's choice is one of them, and a cache file
returns it again without timing.  Buffer schedule: the remote-row gather batch
(the reference's staging granularity, include/dist_spmm_ppl_batch.cuh:373-417)
is chosen from 1,024 to 16,384 rows and every batch size is within 1e-5 of
FP64."""
import numpy as np
import pytest
import torch

from cola_b200 import spmm as S

from gpu_util import TOL_F32, dense_x, fp64_reference, graph_case, rel

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def candidates(xdt, K):
    e16 = 4 if xdt == torch.float32 else 8
    out = []
    for kt in (64, 128, 256, 512, 1024):
        if (xdt == torch.float32 and kt == 1024) or (kt > 64 and kt // 2 >= K):
            continue
        narrow = kt * (4 if xdt == torch.float32 else 2) < 512
        V = kt // e16
        if narrow:
            out += [(kt, u, mb) for u in (4, 8) for mb in (4, 6, 8)]
        elif V == 32:
            out += [(kt, 2, 0)] + [(kt, 4, mb) for mb in (3, 4, 5, 6)] + [(kt, 6, 0), (kt, 8, 0)]
        elif V == 64:
            out += [(kt, 2, 0), (kt, 4, 0)]
        else:
            out += [(kt, 0, 0)]
    return out


@pytest.fixture(scope="module")
def case13():
    n, row, col, val, ps = graph_case(13, 24, seed=8, nparts=8)
    return n, row, col, val, S.Graph(ps, hub_threshold=64, hub_segment=32)


@pytest.mark.parametrize("K,xdt,ydt", [(128, torch.float32, torch.float32), (256, torch.float32, torch.bfloat16),
                                       (256, torch.bfloat16, torch.bfloat16), (512, torch.bfloat16, torch.float32)])
def test_every_rows_candidate_same_bits_and_tuned_choice(case13, tmp_path, K, xdt, ydt):
    n, row, col, val, g = case13
    X = torch.from_numpy(dense_x(n, K, seed=K)).to(DEV).to(xdt)
    base = g.spmm(X, out_dtype=ydt)
    cands = candidates(xdt, K)
    assert len(cands) >= 8
    for kt, u, mb in cands:
        y = g.spmm(X, out_dtype=ydt, k_tile=kt, unroll=u, min_blocks=mb)
        assert torch.equal(y.view(torch.int16) if ydt == torch.bfloat16 else y.view(torch.int32),
                           base.view(torch.int16) if ydt == torch.bfloat16 else base.view(torch.int32)), (kt, u, mb)
    cache = tmp_path / "tune.txt"
    opts, ms, hit = g.autotune(X, out_dtype=ydt, reps=2, cache_path=cache)
    assert not hit and ms > 0
    assert (opts["k_tile"], opts["unroll"], opts["min_blocks"]) in cands
    again, ms2, hit2 = g.autotune(X, out_dtype=ydt, reps=2, cache_path=cache)
    assert hit2 and again == opts and abs(ms2 - ms) < 1e-3
    y = g.spmm(X, out_dtype=ydt, **{k: v for k, v in opts.items() if k != "gather_batch_rows"})
    assert torch.equal(y.float(), base.float())
    if xdt == torch.float32 and ydt == torch.float32:
        assert rel(y.cpu().numpy(), fp64_reference(n, row, col, val, X.cpu().numpy())) <= TOL_F32


def test_narrow_k_single_geometry(case13):
    n, row, col, val, g = case13
    X = torch.from_numpy(dense_x(n, 32, seed=1)).to(DEV)
    opts, ms, hit = g.autotune(X, reps=1)
    assert (opts["k_tile"], opts["unroll"], opts["min_blocks"]) == (0, 0, 0) and ms > 0 and not hit
    # k_tile is ignored below the one-warp-per-tile widths
    assert torch.equal(g.spmm(X, k_tile=64), g.spmm(X))


def test_buffer_gather_batch_tuned(case13):
    n, row, col, val, g = case13
    K = 64
    Xh = dense_x(n, K, seed=3)
    X = torch.from_numpy(Xh).to(DEV)
    ref = fp64_reference(n, row, col, val, Xh)
    opts, ms, _ = g.autotune(X, schedule=S.SCHEDULE_BUFFER, reps=2)
    assert opts["schedule"] == S.SCHEDULE_BUFFER and opts["gather_batch_rows"] in (1024, 2048, 4096, 8192, 16384)
    for b in (1024, 2048, 4096, 8192, 16384):
        y = g.spmm(X, schedule=S.SCHEDULE_BUFFER, gather_batch_rows=b)
        assert rel(y.cpu().numpy(), ref) <= TOL_F32
