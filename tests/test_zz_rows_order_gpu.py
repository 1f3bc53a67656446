"""The row-major schedule's output, bit for bit: for row tiles of one warp
(32 lanes x 16-byte vectors: K = 128 or 256 with FP32 X, K = 256 with BF16 X)
every output element is summed in one documented order -- fused multiply-adds
in column order per row, hub rows as fixed segments whose partials a binary
counter adds -- and the oracle restates that order on the CPU
(orc_spmm_rows_f32_ordered).  The GPU result must equal it exactly, hub
settings included."""
import numpy as np
import pytest
import torch

import cola_b200 as cb
from cola_b200 import spmm as S
from oracle import oracle

from gpu_util import dense_x

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


@pytest.fixture(scope="module")
def case13():
    n, row, col, val = cb.rmat(13, 24, seed=21)
    return n, row, col, val, cb.PartitionSet.from_coo(n, row, col, val, 4)


@pytest.mark.parametrize("K,xdt", [(128, torch.float32), (256, torch.float32), (256, torch.bfloat16)])
@pytest.mark.parametrize("thr,seg", [(256, 256), (16, 8), (1, 1)])
def test_rows_equal_cpu_restatement_bitwise(case13, K, xdt, thr, seg):
    n, row, col, val, ps = case13
    g = S.Graph(ps, hub_threshold=thr, hub_segment=seg)
    X32 = dense_x(n, K, seed=K + thr)
    Xd = torch.from_numpy(X32).to(DEV).to(xdt)
    Y = g.spmm(Xd, out_dtype=torch.float32, schedule=S.SCHEDULE_ROWS)
    torch.cuda.synchronize()
    rp, ci, vv = oracle.global_csr(n, row, col, val)
    Xc = Xd.float().cpu().numpy()  # BF16 widened exactly, as the kernel does
    ref = oracle.spmm_rows_f32_ordered(rp, ci, vv, Xc, hub_threshold=thr, hub_segment=seg)
    got = Y.cpu().numpy()
    mismatch = int(np.count_nonzero(got.view(np.uint32) != ref.view(np.uint32)))
    assert mismatch == 0, "{} of {} elements differ".format(mismatch, got.size)
