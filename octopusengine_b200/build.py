"""Builds liboctb.so (the C-ABI library: host runtime + sm_100a kernels) in-tree.

    python -m octopusengine_b200.build            # or build() from Python

Every source is compiled by nvcc for sm_100a only; objects go to octopusengine_b200/_build
and the shared library to octopusengine_b200/liboctb.so (both git-ignored).  A source
whose object is newer than it and than every header is not recompiled.
"""
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "liboctb.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-Xcompiler", "-Wall", "-I", os.path.join(ROOT, "include"), "-I", CSRC]
EXTRA = os.environ.get("OCTB_NVCC_FLAGS", "").split()


def _sources():
    srcs = glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp"))
    return sorted(s for s in srcs if not s.endswith("gen_tables.cpp"))


def _gen_tables():
    """Compiles and runs gen_tables.cpp (host only) to write csrc/shape_tables.inc."""
    out = os.path.join(CSRC, "shape_tables.inc")
    deps = [os.path.join(CSRC, f) for f in ("gen_tables.cpp", "shape.cpp", "host.hpp")]
    if os.path.exists(out) and os.path.getmtime(out) >= max(os.path.getmtime(d) for d in deps):
        return
    exe = os.path.join(BUILD, "gen_tables")
    subprocess.check_call([os.environ.get("CXX", "g++"), "-O1", "-std=c++17", "-I", CSRC, deps[0], deps[1], "-o", exe])
    txt = subprocess.check_output([exe], text=True)
    with open(out, "w") as f:
        f.write(txt)


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.hpp")) + \
        glob.glob(os.path.join(CSRC, "*.inc")) + glob.glob(os.path.join(ROOT, "include", "*.h"))


def _compile(src, verbose=False):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    newest = max([os.path.getmtime(src)] + [os.path.getmtime(h) for h in _headers()])
    if os.path.exists(obj) and os.path.getmtime(obj) >= newest:
        return obj
    lang = [] if src.endswith(".cu") else ["-x", "cu"]
    cmd = [NVCC] + ARCH + FLAGS + EXTRA + lang + ["-c", src, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed on %s:\n%s\n%s" % (src, r.stdout, r.stderr))
    if verbose:
        sys.stderr.write(r.stderr)
    return obj


def build(verbose=False, jobs=None):
    os.makedirs(BUILD, exist_ok=True)
    _gen_tables()
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(o) for o in objs):
        return LIB
    cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart_static", "-lrt", "-lpthread", "-ldl"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n%s\n%s" % (r.stdout, r.stderr))
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
