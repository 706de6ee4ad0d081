"""Build the tracker library and CLI for sm_100a, in-tree.

Outputs (git-ignored, shipped with the tree):
  libghc_b200.so   the C-ABI library declared in include/ghc.h
  ghc-main         the command-line solver (``ghc-main -p <problem>``)

Each translation unit is compiled by nvcc (-gencode arch=compute_100a,code=sm_100a,
-fmad=false so only explicit fma() calls fuse) in parallel into _build/, then
linked.  Rebuilds only when a source, header or flag changed.
"""
import concurrent.futures as cf
import hashlib
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libghc_b200.so")
CLI = os.path.join(HERE, "ghc-main")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
         "-I", os.path.join(REPO, "include")]
LIB_SOURCES = ["tracker.cu", "tracker_fp64.cu", "tracker_fp64_v1.cu", "tracker_fp32.cu", "tracker_fp32_v1.cu", "tracker_mixed.cu", "tracker_mixed_v1.cu", "p2c.cu", "results.cu", "abi.cu",
               "peak.cu", "no_alloc.cu", "linsolve.cu", "mix.cu", "problem.cpp"]
HEADERS = ["ghc_internal.h", "tracker.cuh", "tracker_launch.cuh", "problem.h", "abi_internal.h"]


def _digest(paths, extra):
    h = hashlib.sha1()
    for p in paths:
        with open(p, "rb") as f:
            h.update(f.read())
    h.update(" ".join(extra).encode())
    return h.hexdigest()


def _compile(src, verbose):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    dep = [src] + [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(REPO, "include", "ghc.h")]
    stamp = obj + ".sha"
    d = _digest(dep, ARCH + FLAGS)
    if os.path.exists(obj) and os.path.exists(stamp) and open(stamp).read() == d:
        return obj
    lang = ["-x", "cu"] if src.endswith(".cu") else ["-x", "c++"]
    cmd = [NVCC] + ARCH + FLAGS + lang + ["-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    with open(stamp, "w") as f:
        f.write(d)
    return obj


def build(verbose=False, jobs=None):
    os.makedirs(BUILD, exist_ok=True)
    srcs = [os.path.join(CSRC, s) for s in LIB_SOURCES]
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    link_digest = _digest(objs, ["lib"])
    stamp = LIB + ".sha"
    if not (os.path.exists(LIB) and os.path.exists(stamp) and open(stamp).read() == link_digest):
        tmp = LIB + ".tmp%d" % os.getpid()
        cmd = [NVCC] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
        os.replace(tmp, LIB)
        with open(stamp, "w") as f:
            f.write(link_digest)
    # command-line solver, linked against the library
    main_obj = _compile(os.path.join(CSRC, "main.cpp"), verbose)
    cli_digest = _digest([main_obj, LIB], ["cli"])
    stamp = CLI + ".sha"
    if not (os.path.exists(CLI) and os.path.exists(stamp) and open(stamp).read() == cli_digest):
        cmd = [NVCC] + ARCH + ["-o", CLI, main_obj, "-L", HERE, "-lghc_b200", "-Xlinker", "-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
        with open(stamp, "w") as f:
            f.write(cli_digest)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
