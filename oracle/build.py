"""Build recipe for the CPU oracle (test infrastructure).

Compiles oracle/hc_oracle.c into oracle/_build/libhc_oracle.so with
-ffp-contract=off (only explicit fma() calls fuse) and OpenMP.  When the
host CPU has FMA3 the library is built with -mfma so fma() is one
instruction; the arithmetic result is the same either way.

When the reference tree is present, also builds oracle/_ref/ (see
oracle/ref/build_ref.py): the reference's own P2C coefficient builders
compiled from their sources in place.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "libhc_oracle.so")


def _cpu_has_fma():
    try:
        with open("/proc/cpuinfo") as f:
            return " fma " in f.read().replace("\n", " ")
    except OSError:
        return False


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    src = [os.path.join(HERE, "hc_oracle.c")]
    deps = src + [os.path.join(HERE, "hc_oracle_body.h"), __file__]
    if (not force) and os.path.exists(LIB):
        if all(os.path.getmtime(LIB) >= os.path.getmtime(d) for d in deps):
            return LIB
    flags = ["-O2", "-std=c11", "-fPIC", "-shared", "-ffp-contract=off", "-fopenmp", "-Wall"]
    if _cpu_has_fma():
        flags.append("-mfma")
    tmp = LIB + ".tmp%d" % os.getpid()
    cmd = ["gcc"] + flags + src + ["-o", tmp, "-lm"]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
