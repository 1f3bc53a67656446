"""GPU tests of the serving loop (cola_server_*): every result is the same
alone and in a concurrent mix, requests overlap and are grouped by width,
admission respects the memory budget, cancellation, timeouts and shutdown."""
import numpy as np
import pytest
import torch

import cola_b200 as cb
from cola_b200.serving import Server

from gpu_util import TOL_BF16, TOL_F32, dense_x, fp64_reference, rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def graphs():
    out = []
    for i, (scale, deg) in enumerate([(10, 8), (11, 16), (12, 24), (10, 40), (13, 12), (9, 30)]):
        n, row, col, val = cb.rmat(scale, deg, seed=50 + i)
        out.append((n, row, col, val, cb.PartitionSet.from_coo(n, row, col, val, 4)))
    return out


def host_x(n, K, seed, dtype=torch.float32):
    return torch.from_numpy(dense_x(n, K, seed)).to(dtype).pin_memory()


def test_alone_equals_mix(graphs):
    srv = Server(slots=3, max_group=4)
    gids = [srv.register(g[4], hub_threshold=64, hub_segment=32) for g in graphs]
    graph_bytes = srv.stats()["bytes_in_use"]
    combos = [(0, 16, torch.float32), (1, 64, torch.float32), (2, 256, torch.bfloat16), (3, 64, torch.bfloat16),
              (4, 512, torch.float32), (5, 16, torch.bfloat16)]
    xs = {c: host_x(graphs[c[0]][0], c[1], seed=c[1] + c[0], dtype=c[2]) for c in combos}
    alone = {}
    for c in combos:
        alone[c] = srv.submit(gids[c[0]], xs[c], out_dtype=c[2]).wait().clone()
    # the mix: every combo several times, interleaved with other traffic
    rng = np.random.Generator(np.random.Philox(9))
    reqs = []
    for rep in range(4):
        for c in [combos[i] for i in rng.permutation(len(combos))]:
            reqs.append((c, srv.submit(gids[c[0]], xs[c], out_dtype=c[2])))
            g2 = int(rng.integers(0, len(graphs)))
            K2 = int(rng.choice([16, 64, 256]))
            reqs.append((None, srv.submit(gids[g2], host_x(graphs[g2][0], K2, seed=rep * 7 + g2), out_dtype=torch.float32)))
    for c, r in reqs:
        y = r.wait(timeout_ms=120000)
        if c is not None:
            assert torch.equal(y, alone[c])  # deterministic kernels: bitwise the same in the mix
    for c in combos:
        n, row, col, val, _ = graphs[c[0]]
        ref = fp64_reference(n, row, col, val, xs[c].float().numpy())
        tol = TOL_F32 if c[2] == torch.float32 else TOL_BF16
        assert rel(alone[c].float().numpy(), ref) <= tol
    st = srv.stats()
    assert st["completed"] == len(combos) + len(reqs)
    assert st["max_inflight"] > 1          # requests overlapped on the device
    assert st["groups_launched"] < st["completed"] and st["max_group"] > 1  # grouped by width
    assert st["p99_ms"] >= st["p50_ms"] > 0
    assert st["bytes_in_use"] == graph_bytes  # every request's memory returned to the budget
    srv.close()


def test_budget_admission_and_rejection(graphs):
    from cola_b200 import spmm as S
    n, row, col, val, ps = graphs[4]
    info = S.Graph(ps).info  # the same upload the server makes
    graph_bytes = info.device_bytes
    one_req = n * 64 * 8 + info.hub_segments * 64 * 4  # X + Y in FP32 at K=64 plus the hub partials
    budget = graph_bytes + one_req + one_req // 2  # one request fits, two do not
    srv = Server(memory_budget=budget, slots=4, max_group=8)
    gid = srv.register(ps)
    reqs = [srv.submit(gid, host_x(n, 64, seed=s)) for s in range(6)]
    for r in reqs:
        r.wait(timeout_ms=120000)
    st = srv.stats()
    assert st["peak_bytes"] <= budget
    assert st["max_inflight"] == 1  # the budget admits one request at a time
    with pytest.raises(cb.ColaError) as e:
        srv.submit(gid, host_x(n, 512, seed=1))  # could never fit
    assert e.value.status == 6
    assert srv.stats()["rejected"] == 1
    srv.close()


def test_cancel_timeout_and_shutdown(graphs):
    n, row, col, val, ps = graphs[4]
    srv = Server(slots=1, max_group=1)
    gid = srv.register(ps)
    reqs = [srv.submit(gid, host_x(n, 512, seed=s)) for s in range(8)]
    last = reqs[-1]
    try:
        last.cancel()
        cancelled = True
    except cb.ColaError as e:  # already admitted: too late to cancel
        assert e.status == 8
        cancelled = False
    if cancelled:
        with pytest.raises(cb.ColaError) as e:
            last.wait()
        assert e.value.status == 9
    try:
        reqs[-2].wait(timeout_ms=0)
    except cb.ColaError as e:
        assert e.status == 7  # still queued or running
    for r in reqs[:-1]:
        r.wait(timeout_ms=120000)
    srv.reset_stats()
    st = srv.stats()
    assert st["completed"] == 0 and st["submitted"] == 0 and st["p50_ms"] == 0
    # shutdown with work still queued: pending requests are cancelled, no hang
    extra = [srv.submit(gid, host_x(n, 512, seed=100 + s)) for s in range(6)]
    srv.close()
    assert len(extra) == 6


def test_bad_requests(graphs):
    n, row, col, val, ps = graphs[0]
    srv = Server()
    gid = srv.register(ps)
    with pytest.raises(cb.ColaError):
        srv.submit(gid, host_x(n, 6, seed=1))  # K not a multiple of 4
    with pytest.raises(ValueError):
        srv.submit(gid, host_x(n + 1, 16, seed=1))
    with pytest.raises(ValueError):
        srv.submit(gid + 5, host_x(n, 16, seed=1))
    srv.close()


def test_register_device_built_graph(graphs):
    from cola_b200 import spmm as S
    n, row, col, val, ps = graphs[0]
    dev = [torch.from_numpy(a).cuda() for a in (row, col, val)]
    srv = Server()
    gid_dev = srv.register_graph(S.Graph.from_coo_device(n, *dev, ps.nparts))
    gid_up = srv.register(ps)
    X = host_x(n, 64, seed=5)
    y_dev = srv.submit(gid_dev, X).wait()
    y_up = srv.submit(gid_up, X).wait()
    assert torch.equal(y_dev, y_up)  # same graph, same bits
    assert rel(y_dev.numpy(), fp64_reference(n, row, col, val, X.numpy())) <= TOL_F32
    # a graph without its row view is refused (and freed)
    g = S.Graph(ps, row_view=False)
    with pytest.raises(cb.ColaError):
        srv.register_graph(g)
    assert g.handle is None
    srv.close()


def test_small_requests_copied_by_sms_equal_copy_engines(graphs):
    """Small groups move their bytes with a kernel on the pinned host buffers
    (not queued behind other slots' copies in the copy engines): the results
    are the bits the copy-engine path gives, in a mix with a large request,
    and pageable host buffers still work (they take the copy engines)."""
    n, row, col, val, ps = graphs[4]
    big_n, _, _, _, big_ps = graphs[2]
    results = []
    for engines_only in (False, True):
        srv = Server(slots=3, max_group=4, small_mib=16, copy_engines_only=engines_only)
        gid = srv.register(ps)
        gbig = srv.register(big_ps)
        xs = [host_x(n, K, seed=K) for K in (16, 64, 128)]
        big = srv.submit(gbig, host_x(big_n, 512, seed=3), out_dtype=torch.float32)
        reqs = [srv.submit(gid, x) for x in xs]
        pageable = torch.from_numpy(dense_x(n, 32, 11))  # not pinned
        rp = srv.submit(gid, pageable)
        results.append([r.wait(timeout_ms=120000).clone() for r in reqs] + [rp.wait(timeout_ms=120000).clone()])
        big.wait(timeout_ms=120000)
        srv.close()
    for a, b in zip(results[0], results[1]):
        assert torch.equal(a, b)
    ref = fp64_reference(n, row, col, val, dense_x(n, 64, 64))
    assert rel(results[0][1].numpy(), ref) <= TOL_F32
