"""The C-ABI library loads and exports every entry point include/*.h declares.
No compute is called (CPU only)."""
import ctypes
import os
import re
import subprocess
import sys

import cola_b200
from cola_b200 import _lib

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    inc = os.path.join(REPO, "include")
    for f in os.listdir(inc):
        if f.endswith(".h"):
            src = open(os.path.join(inc, f)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names.update(re.findall(r"\b(cola_[a-z0-9_]+)\s*\(", src))
    return names


def test_library_exports_every_declared_symbol():
    names = declared_symbols()
    assert len(names) >= 25
    L = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (cola_[a-z0-9_]+)$", out, flags=re.M))
    assert names <= exported, sorted(names - exported)


def test_python_binding_covers_the_abi():
    assert declared_symbols() <= set(_lib.SIGNATURES)


def test_status_strings_and_version():
    L = cola_b200.lib()
    assert L.cola_status_string(0) == b"success"
    assert L.cola_status_string(6) == b"over memory budget"
    assert b"sm_100a" in L.cola_version()


def test_missing_library_fails_loudly(tmp_path):
    """Without the native library every entry point raises: there is no CPU
    fallback behind the package."""
    import os
    import sys
    code = ("import cola_b200._lib as L\n"
            "L.LIB_PATH = {!r}\n"
            "import cola_b200 as cb\n"
            "try:\n"
            "    cb.PartitionSet.from_coo(4, [0, 1], [1, 2], [1.0, 1.0], 2)\n"
            "except RuntimeError as e:\n"
            "    print('raised:', e)\n").format(str(tmp_path / "absent.so"))
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    res = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, cwd=repo, timeout=300)
    assert res.returncode == 0, res.stderr
    assert "raised: cola_b200 native library missing" in res.stdout
