"""include/cola/compat.h builds a reference-style host program that links the
library and reproduces the reference's nnz_split on its own .bin files (CPU)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import cola_b200 as cb
from cola_b200 import _lib
from conftest import load_golden

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_compat_header_program(tmp_path):
    exe = str(tmp_path / "compat_main")
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    subprocess.check_call([cxx, "-std=c++17", "-O1", "-I", os.path.join(REPO, "include"), "-I",
                           "/usr/local/cuda/include", os.path.join(REPO, "tests", "compat_main.cpp"), "-o", exe,
                           "-L", os.path.dirname(_lib.LIB_PATH), "-lcola_b200", "-L", "/usr/local/cuda/lib64",
                           "-lcudart", "-Wl,-rpath," + os.path.dirname(_lib.LIB_PATH)])
    fx = load_golden("rmat12")
    d = tmp_path / "g"
    P = 4
    (d / "GPU4").mkdir(parents=True)
    for nm in ("csr_rowPtr_l", "csr_colIdx_l", "csr_rowIdx_l"):
        fx["P4_r2_" + nm].tofile(str(d / "GPU4" / "{}_4_2.bin".format(nm)))
    out = subprocess.run([exe, str(d / "GPU4") + "/", str(P), "2"], capture_output=True, text=True,
                         check=True).stdout.splitlines()
    t = np.array([int(x) for x in [l for l in out if l.startswith("T")][0].split()[1:]], np.int32)
    p = np.array([int(x) for x in [l for l in out if l.startswith("P ")][0].split()[1:]], np.int32)
    np.testing.assert_array_equal(t, fx["P4_r2_lsplit_target"])
    np.testing.assert_array_equal(p, fx["P4_r2_lsplit_ptr"])
    assert "E {}".format(5) in out  # COLA_ERROR_IO, thrown instead of exit()


@pytest.mark.gpu
@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
@pytest.mark.parametrize("P,dim", [(4, 32), (8, 128), (3, 100)])
def test_compat_reference_main_on_gpu(tmp_path, P, dim):
    """A host program written like the reference's main (bin2vec the partition
    files, nnz_split both blocks, d_csr_zip / d_csc_zip, run_distSpMM_ppl_batch
    with validation against SAG_reference_host and a timed loop), built against
    compat.h, passes its own validation on the GPU for every virtual PE; and
    the same holders in one distSpMM_ppl_batch_all call (single stage: one row
    view of all PEs) give the same product."""
    import scipy.sparse as sp
    exe = str(tmp_path / "compat_gpu_main")
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    subprocess.check_call([cxx, "-std=c++17", "-O2", "-I", os.path.join(REPO, "include"), "-I",
                           "/usr/local/cuda/include", os.path.join(REPO, "tests", "compat_gpu_main.cpp"), "-o", exe,
                           "-L", os.path.dirname(_lib.LIB_PATH), "-lcola_b200", "-L", "/usr/local/cuda/lib64",
                           "-lcudart", "-Wl,-rpath," + os.path.dirname(_lib.LIB_PATH)])
    n, row, col, _ = cb.rmat(11, 12, seed=P + dim)
    n = n - 3  # not a multiple of P
    m = (row < n) & (col < n)
    coo = sp.coo_matrix((np.ones(int(m.sum()), np.float32), (row[m], col[m])), shape=(n, n))
    cb.serialize(coo, "g", str(tmp_path), [P])
    r = subprocess.run([exe, str(tmp_path / "g"), str(n), str(P), str(dim)], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    out = r.stdout.splitlines()
    for p in range(P):
        assert "PEid-{} passed".format(p) in out
        assert any(l.startswith("PE {} ms ".format(p)) and float(l.split()[-1]) > 0 for l in out)
    # distSpMM_ppl_batch_all, single stage: one row view of every PE's chunks
    rel_all = [float(l.split()[-1]) for l in out if l.startswith("ALL rel ")]
    assert rel_all and rel_all[0] <= 1e-5
