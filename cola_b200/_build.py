"""Builds the in-tree shared library cola_b200/lib/libcola_b200.so (sm_100a).

    python -m cola_b200._build [--force]

The host preprocessing (csrc/prep.cpp) is compiled by g++ with OpenMP; the
kernels and launchers (csrc/*.cu) by nvcc for sm_100a only.  Objects go to
cola_b200/_build/ and are rebuilt when a source or header is newer.
"""
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libcola_b200.so")
INCLUDE = os.path.join(REPO, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc():
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def _cxx():
    # the system g++ (the image's CC/CXX may point at a toolchain without libgomp)
    for c in ("/usr/bin/g++", shutil.which("g++")):
        if c and os.path.exists(c):
            return c
    return "g++"


def _headers():
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))


def source_hash():
    """16 hex digits identifying the native sources (csrc/ and include/): a
    profile of the kernels records it, so a reader can tell whether the
    profile was taken on the code that is built now."""
    import hashlib
    h = hashlib.sha256()
    files = sorted(glob.glob(os.path.join(CSRC, "*")) + glob.glob(os.path.join(INCLUDE, "*.h")) +
                   glob.glob(os.path.join(INCLUDE, "cola", "*.h")))
    for f in files:
        if os.path.isfile(f):
            h.update(os.path.relpath(f, REPO).encode())
            with open(f, "rb") as fh:
                h.update(fh.read())
    return h.hexdigest()[:16]


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout)
    return r.stdout


def build(force=False, verbose=False):
    """Compile every source and link the library; returns its path."""
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    hdr = _headers()
    jobs = []
    objs = []
    ccbin = _cxx()
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu"))):
        obj = os.path.join(OBJ, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + hdr):
            jobs.append([_nvcc(), "-ccbin", ccbin] + ARCH + [
                "-lineinfo", "-O3", "-std=c++17", "--expt-relaxed-constexpr",
                "-Xcompiler", "-fPIC,-fopenmp", "-Xptxas", "-v" if verbose else "-O3",
                "-I", INCLUDE, "-I", CSRC, "-c", src, "-o", obj])
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cpp"))):
        obj = os.path.join(OBJ, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + hdr):
            jobs.append([ccbin, "-O3", "-std=c++17", "-fPIC", "-fopenmp", "-Wall",
                         "-I", INCLUDE, "-I", CSRC, "-I", "/usr/local/cuda/include", "-c", src, "-o", obj])
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            outs = list(ex.map(_run, jobs))
        if verbose:
            for o in outs:
                sys.stdout.write(o)
    if force or jobs or _stale(LIB, objs):
        _run([_nvcc(), "-ccbin", ccbin] + ARCH + ["-shared", "-o", LIB] + objs +
             ["-Xcompiler", "-fopenmp", "-lgomp", "-lcudart"])
    return LIB


if __name__ == "__main__":
    if "--hash" in sys.argv:
        print(source_hash())
    else:
        print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
