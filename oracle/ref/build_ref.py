"""Compile the reference's P2C coefficient builders and H / H_x / H_t evaluators into oracle/_ref/.

TEST INFRASTRUCTURE ONLY.  The reference's host-side P2C functions
(GPU-HC/magmaHC/PHC_Coeffs/p2c-<problem>.h, namespace magmaHCWrapper) are
plain C++ over MAGMA's complex type.  They are compiled here from their own
sources, where they lie in the reference tree, against the stand-in header in
oracle/ref/shim/ (a small complex struct), once in double and once in float.

Output: oracle/_ref/libp2c_ref.so with, per problem <p>,
    void ref_p2c_<p>_d(const double* tgt, const double* start, double* hx, double* ht)
    void ref_p2c_<p>_f(const float*  tgt, const float*  start, float*  hx, float*  ht)
(complex arrays interleaved re, im; tgt/start hold P+1 entries, hx
(M+1)(K+1), ht (M+1)K).

The reference's evaluator templates (GPU-HC/magmaHC/gpu-idx-evals/
dev-eval-indxing-<problem>.cuh: eval_Jacobian_Hx, eval_Jacobian_Ht,
eval_Homotopy) are device functions over MAGMA's complex type; with the same
stand-in header (in double) and empty stand-ins for MAGMA's device headers they
compile as host code.  Output: oracle/_ref/libeval_ref.so with, per P2C problem,
    void ref_eval_<p>(const double* x, const double* c, const double* cp,
                      const int* hx_idx, const int* ht_idx,
                      double* Hx, double* Ht, double* H)
x [N+1] (slot N = 1), c / cp [M+1] the coefficients c_k(t) / c'_k(t) (PH problems:
p(t) and p1 - p0 [P+1], slot P of p(t) = 1), the index
tables as read from dHdx_indx.txt / dHdt_indx.txt; out: Hx [N][N], Ht [N] (the
predictor's right-hand side -H_t, as the reference computes it), H [N]: row tx of
each is what the reference's thread tx computes.  The reference's tracker
kernels themselves need MAGMA's internal device headers, which are not part of
the reference tree, so they are not buildable here.
"""
import glob
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE = os.path.dirname(HERE)
OUT = os.path.join(ORACLE, "_ref")
LIB = os.path.join(OUT, "libp2c_ref.so")
EVAL_LIB = os.path.join(OUT, "libeval_ref.so")
CUDA_INCLUDE = "/usr/local/cuda/include"

EVAL_HEAD = """// generated by oracle/ref/build_ref.py -- wrappers around the reference evaluators
#include <cstdio>
#include <iostream>
#include <iomanip>
#include <cstring>
#include <cuda_runtime.h>
#define REF_REAL double
#define ref_cx ref_cx_eval
#include "magma_v2.h"
#include "magma_lapack.h"
#include "magma_internal.h"
#include "magma_templates.h"
#include "sync.cuh"
#include "shuffle.cuh"
#include "batched_kernel_param.h"
"""

EVAL_FN = """namespace refns_%(name)s {
#include "%(hdr)s"
}
extern "C" void ref_eval_%(name)s(const double* x, const double* c, const double* cp, const int* hx_idx,
                                  const int* ht_idx, double* Hx, double* Ht, double* H) {
  const int N = %(N)d, Mc = %(Mc)d;
  ref_cx X[N + 1], C[Mc], CP[Mc], A[N], b;
  for (int i = 0; i <= N; ++i) X[i] = ref_cx(x[2 * i], x[2 * i + 1]);
  for (int k = 0; k < Mc; ++k) { C[k] = ref_cx(c[2 * k], c[2 * k + 1]); CP[k] = ref_cx(cp[2 * k], cp[2 * k + 1]); }
  for (int tx = 0; tx < N; ++tx) {
    refns_%(name)s::eval_Jacobian_Hx<%(N)d, %(Tx)d, %(Px)d, %(Tx)d * %(Px)d, %(N)d * %(Tx)d * %(Px)d>(tx, X, A, hx_idx, C);
    for (int i = 0; i < N; ++i) { Hx[2 * (tx * N + i)] = A[i].x; Hx[2 * (tx * N + i) + 1] = A[i].y; }
    refns_%(name)s::eval_Jacobian_Ht<%(Tt)d, %(Pt)d, %(Tt)d * %(Pt)d>(tx, X, b, ht_idx, CP);
    Ht[2 * tx] = b.x; Ht[2 * tx + 1] = b.y;
    refns_%(name)s::eval_Homotopy<%(Tt)d, %(Pt)d, %(Tt)d * %(Pt)d>(tx, X, b, ht_idx, C);
    H[2 * tx] = b.x; H[2 * tx + 1] = b.y;
  }
}
"""
def reference_root():
    """The reference checkout: $GHC_REFERENCE_ROOT, else a checkout named "reference" beside this
    repository; None when neither holds GPU-HC/ (the GPU box has no reference tree)."""
    for root in (os.environ.get("GHC_REFERENCE_ROOT"),
                 os.path.join(os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))),
                              "..", "reference")):
        if root and os.path.isdir(os.path.join(root, "GPU-HC")):
            return os.path.normpath(root)
    return None


DEFAULT_ROOT = reference_root()

WRAP_HEAD = """// generated by oracle/ref/build_ref.py -- wrappers around the reference P2C builders
#include <cstddef>
#include <stdio.h>
#include <stdlib.h>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <iomanip>
#include <cstring>
#include <chrono>
#define REF_REAL %(real)s
#define ref_cx ref_cx_%(tag)s
#include "magma_v2.h"
namespace ref_%(tag)s {
%(includes)s
}
namespace {
template <int Dummy>
struct Buf {
  static void load(const REF_REAL* s, ref_cx* d, int n) { for (int i = 0; i < n; ++i) d[i] = ref_cx(s[2*i], s[2*i+1]); }
  static void store(const ref_cx* s, REF_REAL* d, int n) { for (int i = 0; i < n; ++i) { d[2*i] = s[i].x; d[2*i+1] = s[i].y; } }
};
}
"""

WRAP_NUM_FN = """extern "C" void ref_p2c_%(name)s_%(tag)s(const REF_REAL* tgt, const REF_REAL* st, REF_REAL* hx, REF_REAL* ht) {
  // this problem's reference builder is numerical: the tables of its shipped parameters only
  static const int NP = 4096;
  ref_cx HX[NP], HT[NP];
  (void)tgt;
  (void)st;
  ref_%(tag)s::magmaHCWrapper::p2c_numerical_%(name)s(HX, HT);
  Buf<0>::store(HX, hx, %(nhx)d); Buf<0>::store(HT, ht, %(nht)d);
}
"""

WRAP_FN = """extern "C" void ref_p2c_%(name)s_%(tag)s(const REF_REAL* tgt, const REF_REAL* st, REF_REAL* hx, REF_REAL* ht) {
  static const int NP = 4096;
  ref_cx T[NP], S[NP], HX[NP], HT[NP];
  Buf<0>::load(tgt, T, %(np)d); Buf<0>::load(st, S, %(np)d);
  ref_%(tag)s::magmaHCWrapper::p2c_%(name)s(T, S, HX, HT);
  Buf<0>::store(HX, hx, %(nhx)d); Buf<0>::store(HT, ht, %(nht)d);
}
"""


def _yaml(path):
    d = {}
    for line in open(path):
        line = line.split("#", 1)[0]
        m = re.match(r"\s*(\w+)\s*:\s*(\S+)", line)
        if m:
            d[m.group(1)] = m.group(2)
    return d


PKG_PROBLEMS = os.path.join(os.path.dirname(ORACLE), "homotopy-continuation-tracker-on-gpu_b200", "problems")


def problems_with_p2c(root):
    """P2C problems of the reference that this package imports: (name, builder header, P, M, K,
    numeric), numeric when the reference's builder is a fixed table of the shipped parameters
    (p2c-numerical_<name>.h)."""
    wanted = set(os.listdir(PKG_PROBLEMS)) if os.path.isdir(PKG_PROBLEMS) else None
    out = []
    for hdr in sorted(glob.glob(os.path.join(root, "GPU-HC/magmaHC/PHC_Coeffs/p2c-*.h"))):
        name = os.path.basename(hdr)[4:-2]
        numeric = name.startswith("numerical_")
        if numeric:
            name = name[len("numerical_"):]
        if wanted is not None and name not in wanted:
            continue
        ydir = os.path.join(root, "GPU-HC/problems", name)
        if not os.path.isdir(ydir):
            continue
        y = _yaml(os.path.join(ydir, "gpuhc_settings.yaml"))
        if y.get("GPUHC_Type") != "P2C":
            continue
        P, M, K = int(y["Num_Of_Params"]), int(y["Num_Of_Coeffs_From_Params"]), int(y["Max_Order_Of_T"])
        out.append((name, hdr, P, M, K, numeric))
    return out


EVAL_PH_FN = """namespace refns_%(name)s {
#include "%(hdr)s"
}
extern "C" void ref_eval_%(name)s(const double* x, const double* ph, const double* dp, const int* hx_idx,
                                  const int* ht_idx, double* Hx, double* Ht, double* H) {
  const int N = %(N)d, Pc = %(Pc)d;
  ref_cx X[N + 1], PH[Pc], DP[Pc], A[N], b;
  for (int i = 0; i <= N; ++i) X[i] = ref_cx(x[2 * i], x[2 * i + 1]);
  for (int k = 0; k < Pc; ++k) { PH[k] = ref_cx(ph[2 * k], ph[2 * k + 1]); DP[k] = ref_cx(dp[2 * k], dp[2 * k + 1]); }
  for (int tx = 0; tx < N; ++tx) {
    refns_%(name)s::eval_Jacobian_Hx<int, %(N)d, %(Tx)d, %(Px)d, %(Tx)d * %(Px)d, %(N)d * %(N)d * %(Tx)d * %(Px)d>(
        tx, A, X, PH, PH, PH, hx_idx);
    for (int i = 0; i < N; ++i) { Hx[2 * (tx * N + i)] = A[i].x; Hx[2 * (tx * N + i) + 1] = A[i].y; }
    refns_%(name)s::eval_Jacobian_Ht<int, %(N)d, %(Tt)d, %(Pt)d, %(N)d * %(Tt)d * %(Pt)d>(tx, b, X, PH, PH, PH, ht_idx, DP);
    Ht[2 * tx] = b.x; Ht[2 * tx + 1] = b.y;
    refns_%(name)s::eval_Homotopy<int, %(N)d, %(Tt)d, %(Pt)d, %(N)d * %(Tt)d * %(Pt)d>(tx, b, X, PH, PH, PH, ht_idx);
    H[2 * tx] = b.x; H[2 * tx + 1] = b.y;
  }
}
"""


def build_eval(root=DEFAULT_ROOT, force=False, verbose=False):
    """libeval_ref.so from the reference's evaluator headers (P2C problems this package imports)."""
    if not os.path.isdir(os.path.join(root, "GPU-HC")) or not os.path.isdir(CUDA_INCLUDE):
        return None
    os.makedirs(OUT, exist_ok=True)
    probs = []
    for name, _, P, M, K, _ in problems_with_p2c(root):
        hdr = os.path.join(root, "GPU-HC/magmaHC/gpu-idx-evals/dev-eval-indxing-%s.cuh" % name)
        if not os.path.exists(hdr):
            continue
        y = _yaml(os.path.join(root, "GPU-HC/problems", name, "gpuhc_settings.yaml"))
        probs.append(dict(name=name, hdr=hdr, N=int(y["Num_Of_Vars"]), Mc=M + 1, Tx=int(y["dHdx_Max_Terms"]),
                          Px=int(y["dHdx_Max_Parts"]), Tt=int(y["dHdt_Max_Terms"]), Pt=int(y["dHdt_Max_Parts"])))
    wanted = set(os.listdir(PKG_PROBLEMS)) if os.path.isdir(PKG_PROBLEMS) else set()
    for ydir in sorted(glob.glob(os.path.join(root, "GPU-HC/problems/*"))):
        name = os.path.basename(ydir)
        hdr = os.path.join(root, "GPU-HC/magmaHC/gpu-idx-evals/dev-eval-indxing-%s.cuh" % name)
        yp = os.path.join(ydir, "gpuhc_settings.yaml")
        if name not in wanted or not os.path.exists(hdr) or not os.path.exists(yp):
            continue
        y = _yaml(yp)
        if y.get("GPUHC_Type") != "PH":
            continue
        probs.append(dict(name=name, hdr=hdr, ph=True, N=int(y["Num_Of_Vars"]), Pc=int(y["Num_Of_Params"]) + 1,
                          Tx=int(y["dHdx_Max_Terms"]), Px=int(y["dHdx_Max_Parts"]), Tt=int(y["dHdt_Max_Terms"]),
                          Pt=int(y["dHdt_Max_Parts"])))
    if (not force) and os.path.exists(EVAL_LIB):
        newest = max([os.path.getmtime(__file__)] + [os.path.getmtime(p["hdr"]) for p in probs])
        if os.path.getmtime(EVAL_LIB) >= newest:
            return EVAL_LIB
    src = EVAL_HEAD + "".join((EVAL_PH_FN if p.get("ph") else EVAL_FN) % p for p in probs)
    cpp = os.path.join(OUT, "eval_ref.cpp")
    with open(cpp, "w") as f:
        f.write(src)
    tmp = EVAL_LIB + ".tmp%d" % os.getpid()
    cmd = ["g++", "-O0", "-std=c++14", "-fPIC", "-w", "-shared", "-I", os.path.join(HERE, "shim"), "-I", CUDA_INCLUDE,
           cpp, "-o", tmp]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    os.replace(tmp, EVAL_LIB)
    with open(os.path.join(OUT, "eval_problems.txt"), "w") as f:
        for p in probs:
            f.write("%s\n" % p["name"])
    return EVAL_LIB


def build(root=DEFAULT_ROOT, force=False, verbose=False):
    if not os.path.isdir(os.path.join(root, "GPU-HC")):
        return None
    os.makedirs(OUT, exist_ok=True)
    probs = problems_with_p2c(root)
    if (not force) and os.path.exists(LIB):
        newest = max([os.path.getmtime(__file__)] + [os.path.getmtime(p[1]) for p in probs])
        if os.path.getmtime(LIB) >= newest:
            return LIB
    objs = []
    for real, tag in (("double", "d"), ("float", "f")):
        includes = "\n".join('#include "%s"' % p[1] for p in probs)
        src = WRAP_HEAD % dict(real=real, tag=tag, includes=includes)
        for name, _, P, M, K, numeric in probs:
            src += (WRAP_NUM_FN if numeric else WRAP_FN) % dict(name=name, tag=tag, np=P + 1, nhx=(M + 1) * (K + 1),
                                                                nht=(M + 1) * K)
        cpp = os.path.join(OUT, "p2c_ref_%s.cpp" % tag)
        with open(cpp, "w") as f:
            f.write(src)
        obj = cpp[:-4] + ".o"
        cmd = ["g++", "-O0", "-std=c++14", "-fPIC", "-w", "-I", os.path.join(HERE, "shim"),
               "-c", cpp, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
        objs.append(obj)
    tmp = LIB + ".tmp%d" % os.getpid()
    subprocess.check_call(["g++", "-shared", "-o", tmp] + objs)
    os.replace(tmp, LIB)
    with open(os.path.join(OUT, "problems.txt"), "w") as f:
        for name, _, P, M, K, numeric in probs:
            f.write("%s %d %d %d %d\n" % (name, P, M, K, numeric))
    return LIB


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 and not sys.argv[1].startswith("-") else DEFAULT_ROOT
    print(build(root, force="--force" in sys.argv, verbose=True))
    print(build_eval(root, force="--force" in sys.argv, verbose=True))
