"""Build libgauge_higgs_b200.so in-tree (gauge_higgs_b200/lib/) for sm_100a.

    python gauge_higgs_b200/build.py [--force] [-j N]

(run by path: importing the package first would load the previous library)

Each CUDA translation unit is compiled by nvcc with
`-gencode arch=compute_100a,code=sm_100a -lineinfo -O3`; the host-only rep
builder by g++; everything is linked into one shared library with the CUDA
runtime linked statically, so the library only needs the driver at run time.
Objects are rebuilt when a source or any header changed.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import hashlib
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libgauge_higgs_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
                     "-Xptxas", "-warn-spills", "-I" + os.path.join(ROOT, "include")]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall", "-I" + os.path.join(ROOT, "include")]


def _nvcc():
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _headers():
    hs = [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC)) if f.endswith((".cuh", ".h", ".hpp"))]
    hs.append(os.path.join(ROOT, "include", "gauge_higgs_b200.h"))
    return hs


def _digest(src, flags):
    h = hashlib.sha256()
    for p in [src] + _headers():
        with open(p, "rb") as f:
            h.update(f.read())
    h.update(" ".join(flags).encode())
    return h.hexdigest()[:16]


def _compile(src, force):
    os.makedirs(OBJ, exist_ok=True)
    base = os.path.splitext(os.path.basename(src))[0]
    is_cu = src.endswith(".cu")
    flags = NVCC_FLAGS if is_cu else CXX_FLAGS
    dig = _digest(src, flags)
    obj = os.path.join(OBJ, f"{base}.{dig}.o")
    if os.path.exists(obj) and not force:
        return obj, None
    cmd = ([_nvcc()] + flags + ["-c", src, "-o", obj]) if is_cu else (["g++"] + flags + ["-c", src, "-o", obj])
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj, (r.stderr.strip() or None)


def build(force=False, jobs=None, verbose=False):
    srcs = [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC)) if f.endswith((".cu", ".cpp"))]
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(jobs) as ex:
        results = list(ex.map(lambda s: _compile(s, force), srcs))
    objs = [o for o, _ in results]
    if verbose:
        for o, msg in results:
            if msg:
                print(os.path.basename(o), msg, file=sys.stderr)
    os.makedirs(LIBDIR, exist_ok=True)
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        tmp = LIB + ".tmp"
        cmd = [_nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", tmp] + objs + ["-lstdc++"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB)
    build_drivers(force)
    # drop stale objects of earlier source versions
    keep = set(os.path.basename(o) for o in objs)
    for f in os.listdir(OBJ):
        if f.endswith(".o") and f not in keep:
            os.remove(os.path.join(OBJ, f))
    return LIB


DRIVERS = [("hmc_higgs", 4, 2), ("hmc_higgs_su3", 4, 3), ("gh_hmc", 4, 2), ("gh_hmc_su3", 4, 3),
           ("hmc_higgs_multi", 4, 2), ("hmc_higgs_multi_su3", 4, 3)]


def build_drivers(force=False):
    """The C++ drivers (drop-in for the reference's hmc_higgs / gh_hmc), one binary per
    compile-time (NDIM, NCOL) as in the reference build, linked to the library by rpath."""
    bindir = os.path.join(PKG, "bin")
    os.makedirs(bindir, exist_ok=True)
    for name, D, N in DRIVERS:
        src = os.path.join(PKG, "drivers", name.replace("_su3", "") + ".cpp")
        out = os.path.join(bindir, name)
        deps = [src, os.path.join(ROOT, "include", "gauge_higgs_b200.hpp"), LIB]
        if not force and os.path.exists(out) and os.path.getmtime(out) >= max(os.path.getmtime(d) for d in deps):
            continue
        cmd = ["g++", "-O2", "-std=c++17", f"-DNDIM={D}", f"-DNCOL={N}", "-I" + os.path.join(ROOT, "include"), src,
               "-o", out, "-L" + LIBDIR, "-lgauge_higgs_b200", "-Wl,-rpath,$ORIGIN/../lib"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"driver build failed: {' '.join(cmd)}\n{r.stderr}")


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.j, a.v))
