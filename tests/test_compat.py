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
