"""GPU parity of the batched form (cola_batch_*): every graph of a mixed batch
against the FP64 oracle, through the direct launch, a captured CUDA graph and
the autotuner."""
import numpy as np
import pytest
import torch

import cola_b200 as cb
from cola_b200.batch import Batch
from oracle import oracle

from gpu_util import TOL_BF16, TOL_F32, bf16_bits, dense_x, fp64_reference, rel

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def make_graphs(count, seed):
    rng = np.random.Generator(np.random.Philox(seed))
    out = []
    for i in range(count):
        scale = int(rng.integers(8, 13))
        deg = float(rng.uniform(4, 40))
        n, row, col, val = cb.rmat(scale, deg, seed=seed * 1000 + i)
        keep = n - int(rng.integers(0, n // 4))  # node counts that are not powers of two
        m = (row < keep) & (col < keep)
        row, col = row[m], col[m]
        deg_r = np.bincount(row, minlength=keep).astype(np.float64)
        val = (1.0 / deg_r[row]).astype(np.float32)  # row-normalised
        out.append((keep, row, col, val, cb.PartitionSet.from_coo(keep, row, col, val, 4)))
    return out


@pytest.fixture(scope="module")
def graphs():
    return make_graphs(12, seed=3)


KS = [32, 64, 128, 512, 33, 16, 96, 64, 128, 32, 256, 8]


def test_batch_fp32_matches_fp64(graphs):
    b = Batch([g[4] for g in graphs], hub_threshold=64, hub_segment=32)
    Xs, Ys, refs = [], [], []
    for (n, row, col, val, _), K in zip(graphs, KS):
        X = dense_x(n, K, seed=K + n)
        Xs.append(torch.from_numpy(X).to(DEV))
        Ys.append(torch.full((n, K), float("nan"), device=DEV))
        refs.append(fp64_reference(n, row, col, val, X))
    b.bind(Xs, Ys)
    info = b.info
    assert info.batched_graphs == 11  # K = 33 is not a 16-byte vector width: it runs on its own
    b.run()
    torch.cuda.synchronize()
    assert b.info.last_launches >= 2
    for Y, ref in zip(Ys, refs):
        assert rel(Y.cpu().numpy(), ref) <= TOL_F32


def test_batch_capture_replay_and_autotune(graphs):
    b = Batch([g[4] for g in graphs])
    Xs = [torch.from_numpy(dense_x(g[0], 64, seed=i)).to(DEV) for i, g in enumerate(graphs)]
    Ys = [torch.zeros((g[0], 64), device=DEV) for g in graphs]
    b.bind(Xs, Ys)
    ms = b.autotune(reps=2)
    assert ms > 0
    b.capture()
    for trial in range(2):
        new = [dense_x(g[0], 64, seed=100 * trial + i) for i, g in enumerate(graphs)]
        for x, h in zip(Xs, new):
            x.copy_(torch.from_numpy(h))  # same buffers, new contents
        b.replay()
        torch.cuda.synchronize()
        for (n, row, col, val, _), Y, h in zip(graphs, Ys, new):
            assert rel(Y.cpu().numpy(), fp64_reference(n, row, col, val, h)) <= TOL_F32


def test_batch_launch_params_do_not_change_results(graphs):
    # every (blocks per SM, unroll, grid) candidate of the autotuner sums each
    # row in the same order: bit-identical outputs
    b = Batch([g[4] for g in graphs])
    Xs = [torch.from_numpy(dense_x(g[0], K, seed=i)).to(DEV) for i, (g, K) in
          enumerate(zip(graphs, [16, 32, 64, 128, 256, 64, 32, 128, 16, 64, 128, 32]))]
    Ys = [torch.zeros((X.shape[0], X.shape[1]), device=DEV) for X in Xs]
    b.bind(Xs, Ys)
    outs = []
    for occ in (3, 4):
        for unroll in (2, 4):
            for grid in (50, 100):
                b.set_params(unroll=unroll, grid_pct=grid, blocks_per_sm=occ)
                b.run()
                torch.cuda.synchronize()
                outs.append([y.clone() for y in Ys])
                assert b.info.blocks_per_sm == occ and b.info.unroll == unroll
    for o in outs[1:]:
        assert all(torch.equal(a, c) for a, c in zip(outs[0], o))
    for (n, row, col, val, _), Y, X in zip(graphs, outs[0], Xs):
        assert rel(Y.cpu().numpy(), fp64_reference(n, row, col, val, X.cpu().numpy())) <= TOL_F32
    with pytest.raises(cb.ColaError):
        b.set_params(unroll=4, grid_pct=100, blocks_per_sm=5)


def test_batch_bf16(graphs):
    b = Batch([g[4] for g in graphs[:6]])
    Xs, Ys, refs = [], [], []
    for (n, row, col, val, _), K in zip(graphs[:6], [32, 64, 128, 256, 16, 64]):
        X = dense_x(n, K, seed=7 * K)
        Xb = bf16_bits(X)
        Xs.append(torch.from_numpy(Xb.view(np.int16)).view(torch.bfloat16).to(DEV))
        Ys.append(torch.zeros((n, K), dtype=torch.bfloat16, device=DEV))
        refs.append(fp64_reference(n, row, col, val, X))
    b.bind(Xs, Ys)
    b.run()
    torch.cuda.synchronize()
    for Y, ref in zip(Ys, refs):
        assert rel(Y.float().cpu().numpy(), ref) <= TOL_BF16


def test_batch_matches_single_graph_calls(graphs):
    """The batched launch gives the same numbers as one cola_spmm per graph."""
    from cola_b200 import spmm as S
    b = Batch([g[4] for g in graphs[:5]])
    Xs = [torch.from_numpy(dense_x(g[0], 128, seed=i)).to(DEV) for i, g in enumerate(graphs[:5])]
    Ys = [torch.zeros((g[0], 128), device=DEV) for g in graphs[:5]]
    b.bind(Xs, Ys)
    b.run()
    for g, X, Y in zip(graphs[:5], Xs, Ys):
        single = S.Graph(g[4]).spmm(X)
        torch.cuda.synchronize()
        assert rel(Y.cpu().numpy(), single.cpu().numpy().astype(np.float64)) <= TOL_F32


def test_batch_rejects_bad_binding(graphs):
    b = Batch([g[4] for g in graphs[:2]])
    with pytest.raises(ValueError):
        b.bind([torch.zeros((1, 8), device=DEV)] * 2, [torch.zeros((1, 8), device=DEV)] * 2)
    with pytest.raises(cb.ColaError):
        b.run()  # nothing bound


def test_batch_from_existing_graphs_device_built(graphs):
    # graphs built on the device, batched without another upload: each result
    # within the bound of FP64, and the same bits as the graph's own SpMM where
    # both use full 32-lane row tiles (K >= 128 FP32); narrower rows are cut
    # into lane groups of other widths by the two kernels (8 lanes minimum in
    # the batched form), which changes the order of the float sums
    from cola_b200 import spmm as S
    gs = [S.Graph.from_coo_device(n, torch.from_numpy(row).to(DEV), torch.from_numpy(col).to(DEV),
                                  torch.from_numpy(val).to(DEV), 4) for n, row, col, val, _ in graphs[:5]]
    b = Batch.from_graphs(gs)
    Ks = [16, 64, 128, 32, 256]
    Xs = [torch.from_numpy(dense_x(g.num_nodes, K, seed=K)).to(DEV) for g, K in zip(gs, Ks)]
    Ys = [torch.zeros((g.num_nodes, K), device=DEV) for g, K in zip(gs, Ks)]
    b.bind(Xs, Ys)
    b.run()
    torch.cuda.synchronize()
    for g, X, Y, (n, row, col, val, _) in zip(gs, Xs, Ys, graphs[:5]):
        alone = g.spmm(X)
        torch.cuda.synchronize()
        if X.shape[1] >= 128:
            assert torch.equal(Y, alone)
        assert rel(Y.cpu().numpy(), fp64_reference(n, row, col, val, X.cpu().numpy())) <= TOL_F32
    b.close()
    del gs


def test_batch_autotune_cache_file(graphs, tmp_path):
    """The tuning cache: a batch tuned once is tuned from the file the next
    time (same parameters, no timing); another shape is tuned anew and gets
    its own line; lines that do not parse are ignored."""
    cache = tmp_path / "tune.txt"
    cache.write_text("garbage line\n" + "x 9 9 9 1.0\n")

    def bound(K):
        b = Batch([g[4] for g in graphs[:4]])
        b.bind([torch.from_numpy(dense_x(g[0], K, seed=1)).to(DEV) for g in graphs[:4]],
               [torch.zeros((g[0], K), device=DEV) for g in graphs[:4]])
        return b
    b1 = bound(64)
    b1.autotune(reps=1, cache=str(cache))
    assert not b1.tuned_from_cache
    p1 = (b1.info.unroll, b1.info.grid_pct, b1.info.blocks_per_sm)
    b2 = bound(64)
    b2.set_params(unroll=2 if p1[0] == 4 else 4, grid_pct=50, blocks_per_sm=3 if p1[2] == 4 else 4)
    b2.autotune(reps=1, cache=str(cache))
    assert b2.tuned_from_cache
    assert (b2.info.unroll, b2.info.grid_pct, b2.info.blocks_per_sm) == p1
    b3 = bound(128)
    b3.autotune(reps=1, cache=str(cache))
    assert not b3.tuned_from_cache
    lines = [l for l in cache.read_text().splitlines() if l.strip()]
    assert len(lines) == 4 and all(len(l.split()) == 5 for l in lines[2:])
    b2.run()
    torch.cuda.synchronize()
