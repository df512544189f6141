#!/usr/bin/env python3
"""Build libqphix_b200.so in-tree for sm_100a with nvcc.

The body and face kernels are instantiated once per (storage type, SOALEN)
from csrc/qb200_inst.cu so that the objects compile in parallel; the C-ABI
layer is csrc/qb200_api.cu.  Objects go to qphix-codegen_b200/_build/, the
library to qphix-codegen_b200/qphix_b200/libqphix_b200.so.
Usage: python qphix-codegen_b200/build.py [-j N] [--force]
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "qphix_b200", "libqphix_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
           "-Xptxas", "-v", "--expt-relaxed-constexpr", "-I" + CSRC, "-I" + INCLUDE]

FTYPES = {"f32": "float", "f64": "double", "f16": "__half", "f16n": "half_norm", "bf16": "__nv_bfloat16"}
SOALENS = [1, 2, 4, 8, 16]
WIDE_ONLY = ("f16n", "bf16")   # built for SOALEN 4, 8, 16
MRHS = ("f32", "f16")           # multi-RHS kernels, SOALEN 4, 8, 16


def nvcc():
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(p):
        raise RuntimeError("nvcc not found")
    return p


def units():
    """(object path, extra flags, source) for every translation unit."""
    out = [(os.path.join(BUILD, "qb200_api.o"), [], os.path.join(CSRC, "qb200_api.cu")),
           (os.path.join(BUILD, "qb200_solver.o"), [], os.path.join(CSRC, "qb200_solver.cu")),
           (os.path.join(BUILD, "qb200_mrhs.o"), [], os.path.join(CSRC, "qb200_mrhs.cu")),
           (os.path.join(BUILD, "qb200_force.o"), [], os.path.join(CSRC, "qb200_force.cu")),
           (os.path.join(BUILD, "qb200_batch.o"), [], os.path.join(CSRC, "qb200_batch.cu")),
           (os.path.join(BUILD, "qb200_convert.o"), [], os.path.join(CSRC, "qb200_convert.cu")),
           (os.path.join(BUILD, "qb200_qphix_tiles.o"), [], os.path.join(CSRC, "qb200_qphix_tiles.cu"))]
    for tag, ft in FTYPES.items():
        for s in SOALENS:
            if tag in WIDE_ONLY and s < 4:
                continue
            mr = 1 if (tag in MRHS and s >= 4) else 0
            out.append((os.path.join(BUILD, "inst_%s_s%d.o" % (tag, s)),
                        ["-DQB_FT=%s" % ft, "-DQB_S=%d" % s, "-DQB_MRHS=%d" % mr],
                        os.path.join(CSRC, "qb200_inst.cu")))
    return out


def newest_source():
    return max(os.path.getmtime(os.path.join(d, f))
               for d in (CSRC, INCLUDE) for f in os.listdir(d))


def newest_header():
    return max(os.path.getmtime(os.path.join(d, f))
               for d in (CSRC, INCLUDE) for f in os.listdir(d) if not f.endswith(".cu"))


def deps_of(obj, extra, src):
    """Files the unit was compiled from, read from the dependency file nvcc
    wrote beside the object.  An object built without one is checked against
    every header of csrc/ and include/; when it is newer than all of them its
    dependency file is written now (nvcc -M, preprocessing only)."""
    dfile = obj + ".d"
    if not os.path.exists(dfile) and os.path.getmtime(obj) >= max(newest_header(), os.path.getmtime(src)):
        subprocess.run([nvcc()] + ARCH + NVFLAGS + extra + ["-M", "-MT", obj, "-MF", dfile, src],
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    if os.path.exists(dfile):
        with open(dfile) as f:
            text = f.read().replace("\\\n", " ")
        _, _, rhs = text.partition(":")
        files = [p for p in rhs.split() if os.path.exists(p)]
        if files:
            return files
    return [src] + [os.path.join(d, f) for d in (CSRC, INCLUDE) for f in os.listdir(d) if not f.endswith(".cu")]


def compile_one(obj, extra, src, log):
    cmd = [nvcc()] + ARCH + NVFLAGS + extra + ["-MD", "-MF", obj + ".d", "-c", src, "-o", obj]
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    with open(log, "w") as f:
        f.write(" ".join(cmd) + "\n" + r.stdout)
    if r.returncode:
        raise RuntimeError("nvcc failed for %s:\n%s" % (obj, r.stdout[-6000:]))
    return obj


def build(jobs=None, force=False, verbose=True):
    os.makedirs(BUILD, exist_ok=True)
    src_t = newest_source()
    if (not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= src_t
            and all(os.path.exists(u[0]) and os.path.getmtime(u[0]) <= os.path.getmtime(LIB) for u in units())):
        return LIB
    jobs = jobs or max(1, os.cpu_count() or 1)
    todo = []
    for obj, extra, src in units():
        # a unit depends on its source and the headers it included
        if not force and os.path.exists(obj):
            dep_t = max(os.path.getmtime(p) for p in deps_of(obj, extra, src))
        if force or not os.path.exists(obj) or os.path.getmtime(obj) < dep_t:
            todo.append((obj, extra, src, obj + ".log"))
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        futs = [ex.submit(compile_one, *t) for t in todo]
        for fu in cf.as_completed(futs):
            o = fu.result()
            if verbose:
                print("built", os.path.relpath(o, HERE), flush=True)
    objs = [u[0] for u in units()]
    cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode:
        raise RuntimeError("link failed:\n" + r.stdout[-4000:])
    return LIB


if __name__ == "__main__":
    j = None
    if "-j" in sys.argv:
        j = int(sys.argv[sys.argv.index("-j") + 1])
    print(build(jobs=j, force="--force" in sys.argv))
