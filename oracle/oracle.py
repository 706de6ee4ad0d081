"""CPU oracle of the homotopy path tracker -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, and only as the checker.  It restates:

* the problem-data readers   GPU-HC/magmaHC/Data_Reader.cpp:91-225
  (start/target params, start solutions, dH/dx and dH/dt index tables) and
  the YAML keys of GPU-HC/magmaHC/GPU_HC_Solver.cpp:44-66;
* the P2C coefficient tables (GPU-HC/magmaHC/PHC_Coeffs/p2c-*.h semantics):
  c_k(t) = c_k(q + t (p - q)) expanded in t, plus the constant-1 sentinel;
* the tracker (ctypes to oracle/_build/libhc_oracle.so, hc_oracle_body.h);
* the result counts   GPU-HC/magmaHC/Evaluations.cpp:88-176.

When oracle/_ref/libp2c_ref.so exists (the reference's own P2C builders
compiled from its sources), ``ref_p2c`` exposes them for pinning.
"""
import ctypes
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
PKG_PROBLEMS = os.path.join(REPO, "homotopy-continuation-tracker-on-gpu_b200", "problems")

P2C, PH = 0, 1
CONVERGED, DIVERGED, STEP_CAP, NONFINITE, SINGULAR = 0, 1, 2, 3, 4

# Evaluations tolerances (GPU-HC/magmaHC/definitions.hpp:24-26)
DUPLICATE_SOL_DIFF_TOL = 1e-4
ZERO_IMAG_PART_TOL_FOR_SP = 1e-4
ZERO_IMAG_PART_TOL_FOR_DP = 1e-8


# ----------------------------------------------------------------------------
# problem data (Data_Reader.cpp restated)
# ----------------------------------------------------------------------------

def read_yaml(path):
    d = {}
    for line in open(path):
        line = line.split("#", 1)[0]
        m = re.match(r"\s*([A-Za-z_]\w*)\s*:\s*(\S+)", line)
        if m:
            d[m.group(1)] = m.group(2)
    return d


def _read_pairs(path, dtype):
    # whitespace "re im" pairs read as the reference reads them (operator>> pairs)
    vals = np.array(open(path).read().split(), dtype=dtype)
    n = vals.size // 2
    return vals[:2 * n].reshape(n, 2)


class Problem:
    """A problem folder in the reference layout."""

    def __init__(self, name, root=PKG_PROBLEMS, dtype=np.float64):
        self.name = name
        self.dir = os.path.join(root, name)
        y = read_yaml(os.path.join(self.dir, "gpuhc_settings.yaml"))
        self.yaml = y
        self.kind = P2C if y["GPUHC_Type"] == "P2C" else PH
        self.max_steps = int(y["GPUHC_Max_Steps"])
        self.max_corr = int(y["GPUHC_Max_Correction_Steps"])
        self.incr = int(y["GPUHC_Num_Of_Steps_to_Increase_Delta_t"])
        self.N = int(y["Num_Of_Vars"])
        self.P = int(y["Num_Of_Params"])
        self.paths = int(y["Num_Of_Tracks"])
        self.Tx, self.Px = int(y["dHdx_Max_Terms"]), int(y["dHdx_Max_Parts"])
        self.Tt, self.Pt = int(y["dHdt_Max_Terms"]), int(y["dHdt_Max_Parts"])
        self.K = int(y["Max_Order_Of_T"])
        self.M = int(y["Num_Of_Coeffs_From_Params"]) if self.kind == P2C else 0
        self.hx_idx = np.array(open(os.path.join(self.dir, "dHdx_indx.txt")).read().split(), dtype=np.int32)
        self.ht_idx = np.array(open(os.path.join(self.dir, "dHdt_indx.txt")).read().split(), dtype=np.int32)
        assert self.hx_idx.size == self.N * self.N * self.Tx * self.Px, "dHdx size"
        assert self.ht_idx.size == self.N * self.Tt * self.Pt, "dHdt size"
        # params: P values, slot P == 1 (Data_Reader.cpp:161-183)
        self.start_params = self._params("start_params.txt", dtype)
        self.target_params = self._params("target_params.txt", dtype)
        sols = _read_pairs(os.path.join(self.dir, "start_sols.txt"), dtype)
        z = sols[:, 0] + 1j * sols[:, 1]
        self.start_sols = z[: self.paths * self.N].reshape(self.paths, self.N)
        self.terms = None
        tp = os.path.join(self.dir, "p2c_terms.txt")
        if os.path.exists(tp):
            self.terms = read_p2c_terms(tp)

    def _params(self, fname, dtype):
        pr = _read_pairs(os.path.join(self.dir, fname), dtype)
        v = np.zeros(self.P + 1, dtype=np.complex128)
        n = min(self.P, pr.shape[0])
        v[:n] = pr[:n, 0] + 1j * pr[:n, 1]
        v[self.P] = 1.0
        return v


def read_p2c_terms(path):
    rows = [l.split() for l in open(path) if l.strip() and not l.startswith("#")]
    M, K, P = (int(v) for v in rows[0])
    terms = [[] for _ in range(M)]
    for r in rows[1:]:
        k, num, den, nf = int(r[0]), int(r[1]), int(r[2]), int(r[3])
        terms[k].append((num / den, [int(j) for j in r[4:4 + nf]]))
    return dict(M=M, K=K, P=P, terms=terms)


def p2c_tables(terms, start, target, exact_ht=False):
    """Coefficient tables c_k(t) for one hypothesis (numpy restatement).

    Hx[k*(K+1) + j] = coefficient of t^j in c_k(q + t(p - q)),
    Ht[k*K + j]     = (j+1) Hx[k*(K+1) + j+1],
    sentinel k = M: Hx = [1, 0, ..], Ht = [1, 0, ..] (reference,
    createUnivPoly4Coeffs.m:227/333) or Ht = 0 with exact_ht.
    """
    M, K = terms["M"], terms["K"]
    q = np.asarray(start, dtype=np.complex128)
    d = np.asarray(target, dtype=np.complex128) - q
    hx = np.zeros((M + 1, K + 1), dtype=np.complex128)
    for k in range(M):
        acc = np.zeros(K + 1, dtype=np.complex128)
        for c, fac in terms["terms"][k]:
            poly = np.zeros(K + 1, dtype=np.complex128)
            poly[0] = c
            for j in fac:
                nxt = poly * q[j]
                nxt[1:] += poly[:-1] * d[j]
                poly = nxt
            acc += poly
        hx[k] = acc
    hx[M, 0] = 1.0
    ht = np.zeros((M + 1, K), dtype=np.complex128)
    for j in range(K):
        ht[:, j] = (j + 1) * hx[:, j + 1]
    ht[M, :] = 0.0
    if not exact_ht:
        ht[M, 0] = 1.0
    return hx.reshape(-1), ht.reshape(-1)


# ----------------------------------------------------------------------------
# reference P2C builders compiled from the reference sources (oracle/_ref)
# ----------------------------------------------------------------------------

_REF = None


def ref_p2c_available():
    return os.path.exists(os.path.join(HERE, "_ref", "libp2c_ref.so"))


def ref_p2c(pb, start, target, precision="d"):
    global _REF
    if _REF is None:
        _REF = ctypes.CDLL(os.path.join(HERE, "_ref", "libp2c_ref.so"))
    rt = np.float64 if precision == "d" else np.float32
    fn = getattr(_REF, "ref_p2c_%s_%s" % (pb.name, precision))
    t = np.ascontiguousarray(np.stack([np.real(target), np.imag(target)], -1).astype(rt))
    s = np.ascontiguousarray(np.stack([np.real(start), np.imag(start)], -1).astype(rt))
    hx = np.zeros(2 * (pb.M + 1) * (pb.K + 1), dtype=rt)
    ht = np.zeros(2 * (pb.M + 1) * pb.K, dtype=rt)
    p = ctypes.c_void_p
    fn.argtypes = [p, p, p, p]
    fn(t.ctypes.data, s.ctypes.data, hx.ctypes.data, ht.ctypes.data)
    return (hx[0::2] + 1j * hx[1::2]).astype(np.complex128), (ht[0::2] + 1j * ht[1::2]).astype(np.complex128)


_REF_EVAL = None


def ref_eval_available(name):
    f = os.path.join(HERE, "_ref", "eval_problems.txt")
    return os.path.exists(os.path.join(HERE, "_ref", "libeval_ref.so")) and os.path.exists(f) and \
        name in open(f).read().split()


def ref_eval(pb, x, c, cp):
    """The reference's own evaluators (dev-eval-indxing-<p>.cuh, compiled by oracle/ref/build_ref.py)
    at track x [N] with coefficients c_k(t), c'_k(t) [M+1] (PH: p(t), p1 - p0 [P+1]):
    returns (Hx [N, N], -H_t [N], H [N])."""
    global _REF_EVAL
    if _REF_EVAL is None:
        _REF_EVAL = ctypes.CDLL(os.path.join(HERE, "_ref", "libeval_ref.so"))
    fn = getattr(_REF_EVAL, "ref_eval_%s" % pb.name)
    p = ctypes.c_void_p
    fn.argtypes = [p] * 8
    N = pb.N
    xs = _cx(np.append(np.asarray(x, dtype=np.complex128), 1.0), np.float64)
    cc, ccp = _cx(c, np.float64), _cx(cp, np.float64)
    hx_idx = np.ascontiguousarray(pb.hx_idx, dtype=np.int32)
    ht_idx = np.ascontiguousarray(pb.ht_idx, dtype=np.int32)
    Hx = np.zeros((N, N, 2))
    Ht = np.zeros((N, 2))
    H = np.zeros((N, 2))
    fn(xs.ctypes.data, cc.ctypes.data, ccp.ctypes.data, hx_idx.ctypes.data, ht_idx.ctypes.data, Hx.ctypes.data,
       Ht.ctypes.data, H.ctypes.data)
    cx = lambda a: a[..., 0] + 1j * a[..., 1]  # noqa: E731
    return cx(Hx), cx(Ht), cx(H)


# ----------------------------------------------------------------------------
# tracker (ctypes)
# ----------------------------------------------------------------------------

class _Prob(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("N", ctypes.c_int32), ("P", ctypes.c_int32),
                ("M", ctypes.c_int32), ("K", ctypes.c_int32), ("Tx", ctypes.c_int32),
                ("Px", ctypes.c_int32), ("Tt", ctypes.c_int32), ("Pt", ctypes.c_int32),
                ("max_steps", ctypes.c_int32), ("max_corr", ctypes.c_int32),
                ("incr_steps", ctypes.c_int32), ("polish_iters", ctypes.c_int32),
                ("hx_idx", ctypes.c_void_p), ("ht_idx", ctypes.c_void_p), ("corr_tol2", ctypes.c_double),
                ("first_tol2", ctypes.c_double), ("dt_max", ctypes.c_double),
                ("t_handover", ctypes.c_double), ("fail_limit", ctypes.c_int32), ("resume", ctypes.c_int32),
                ("cond_limit", ctypes.c_double), ("dt_floor", ctypes.c_double)]

# step control of the reference (kernel_HC_Solver_P3P.cu:214, no contraction test, no dt cap)
REFERENCE_STEP = dict(corr_tol2=1e-6, first_tol2=float("inf"), dt_max=float("inf"))
ROBUST_STEP = dict(corr_tol2=1e-12, first_tol2=1e-2, dt_max=0.05)


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        import importlib.util
        spec = importlib.util.spec_from_file_location("oracle_build", os.path.join(HERE, "build.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        _LIB = ctypes.CDLL(mod.build())
    return _LIB


def _cx(a, rt):
    a = np.asarray(a, dtype=np.complex128)
    out = np.empty(a.shape + (2,), dtype=rt)
    out[..., 0] = a.real
    out[..., 1] = a.imag
    return np.ascontiguousarray(out)


def _prob_struct(pb, polish_iters, max_steps=None, max_corr=None, incr=None, step=None):
    s = _Prob()
    s.kind, s.N, s.P, s.M, s.K = pb.kind, pb.N, pb.P, pb.M, pb.K
    s.Tx, s.Px, s.Tt, s.Pt = pb.Tx, pb.Px, pb.Tt, pb.Pt
    s.max_steps = pb.max_steps if max_steps is None else max_steps
    s.max_corr = pb.max_corr if max_corr is None else max_corr
    s.incr_steps = pb.incr if incr is None else incr
    s.polish_iters = polish_iters
    s.hx_idx = pb.hx_idx.ctypes.data
    s.ht_idx = pb.ht_idx.ctypes.data
    st = dict(REFERENCE_STEP)
    st.update(step or {})
    s.corr_tol2, s.first_tol2, s.dt_max = st["corr_tol2"], st["first_tol2"], st["dt_max"]
    return s


# the tracker library's two-phase mixed precision (csrc/tracker.cu): the mixed tracker (double state,
# residual and step control, float H_x, H_t and LU) to t = 1 or t_switch < 1, a path handed over after
# a step whose float solve had pivot magnitudes spanning more than cond_limit, once its step falls below
# dt_floor, after 4 failed steps in a row, or on divergence; then the double tracker resumes every path
MIXED_FAIL_LIMIT = 4
MIXED_COND_LIMIT = 1e5
MIXED_DT_FLOOR = 1e-4


def track(pb, start_sols, hx=None, ht=None, p_start=None, p_target=None, precision="d",
          polish_iters=0, nthreads=0, max_steps=None, max_corr=None, incr=None, step=None, t_switch=1.0,
          cond_limit=MIXED_COND_LIMIT, dt_floor=MIXED_DT_FLOOR):
    """Track all start paths for H hypotheses.

    P2C: hx [H, (M+1)(K+1)], ht [H, (M+1)K] complex.
    PH:  p_start [P+1], p_target [H, P+1] complex.
    precision "d", "f", or "mixed": the mixed tracker (double state and residual, float linear
    algebra) to t_switch (>= 1: to t = 1), then double resumed from each path's stopping point,
    as the tracker library does.
    Returns a dict of numpy arrays (endpoints [H*paths, N], flags, counters).
    """
    kw = dict(hx=hx, ht=ht, p_start=p_start, p_target=p_target, nthreads=nthreads, max_steps=max_steps,
              max_corr=max_corr, incr=incr, step=step)
    if precision != "mixed":
        return _track(pb, start_sols, precision=precision, polish_iters=polish_iters, **kw)
    if not t_switch > 0:
        return _track(pb, start_sols, precision="d", polish_iters=polish_iters, **kw)
    first = _track(pb, start_sols, precision="m", polish_iters=0,
                   handover=(t_switch if t_switch < 1 else 0.0, MIXED_FAIL_LIMIT, cond_limit, dt_floor), **kw)
    return _track(pb, start_sols, precision="d", polish_iters=polish_iters, resume=first, **kw)


def _track(pb, start_sols, hx=None, ht=None, p_start=None, p_target=None, precision="d",
           polish_iters=0, nthreads=0, max_steps=None, max_corr=None, incr=None, step=None, handover=None,
           resume=None):
    rt = np.float32 if precision == "f" else np.float64
    fn = {"d": lib().orc_track_d, "f": lib().orc_track_f, "m": lib().orc_track_m}[precision]
    start_sols = np.asarray(start_sols)
    paths = start_sols.shape[0]
    ss = _cx(start_sols, rt)
    null = None
    if pb.kind == P2C:
        hx = np.atleast_2d(hx)
        ht = np.atleast_2d(ht)
        H = hx.shape[0]
        chx, cht = _cx(hx, rt), _cx(ht, rt)
        shx, sht = hx.shape[1], ht.shape[1]
        ps = pt = pd = null
        sp_ = 0
    else:
        p_target = np.atleast_2d(p_target)
        H = p_target.shape[0]
        diff = p_target - np.asarray(p_start)[None, :]
        ps, pt, pd = _cx(p_start, rt), _cx(p_target, rt), _cx(diff, rt)
        chx = cht = null
        shx = sht = 0
        sp_ = pb.P + 1
    n = H * paths
    ep = np.zeros((n, pb.N, 2), dtype=rt)
    out = dict(conv=np.zeros(n, np.uint8), inf=np.zeros(n, np.uint8), status=np.zeros(n, np.uint8),
               steps=np.zeros(n, np.int32), corr=np.zeros(n, np.int32), t_end=np.zeros(n),
               dt_end=np.zeros(n), resid=np.zeros(n))
    s = _prob_struct(pb, polish_iters, max_steps, max_corr, incr, step)
    if handover is not None:
        s.t_handover, s.fail_limit = handover[:2]
        if len(handover) > 2:
            s.cond_limit = handover[2]
        if len(handover) > 3:
            s.dt_floor = handover[3]
    if resume is not None:
        s.resume = 1
        ep[...] = resume["endpoints_raw"].astype(rt)
        for k in ("steps", "corr", "t_end", "dt_end"):
            out[k][:] = resume[k]
    P = ctypes.c_void_p

    def ptr(a):
        return None if a is None else a.ctypes.data

    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.POINTER(_Prob), ctypes.c_int64, ctypes.c_int32, P, P, P, ctypes.c_int64,
                   ctypes.c_int64, P, P, P, ctypes.c_int64, P, P, P, P, P, P, P, P, P, ctypes.c_int32]
    rc = fn(ctypes.byref(s), n, paths, ptr(ss), ptr(chx), ptr(cht), shx, sht, ptr(ps), ptr(pt), ptr(pd),
            sp_, ptr(ep), ptr(out["conv"]), ptr(out["inf"]), ptr(out["status"]), ptr(out["steps"]),
            ptr(out["corr"]), ptr(out["t_end"]), ptr(out["dt_end"]), ptr(out["resid"]), nthreads)
    if rc != 0:
        raise RuntimeError("orc_track failed: %d" % rc)
    out["endpoints"] = ep[..., 0].astype(np.float64) + 1j * ep[..., 1].astype(np.float64)
    out["endpoints_raw"] = ep
    return out


def eval_system(pb, x, t, hx=None, ht=None, p_start=None, p_target=None, precision="d"):
    """H, -H_t... (as tracked: returns H, Ht_sum, Hx) at (x, t)."""
    rt = np.float64 if precision == "d" else np.float32
    fn = lib().orc_eval_d if precision == "d" else lib().orc_eval_f
    s = _prob_struct(pb, 0)
    N = pb.N
    H = np.zeros((N, 2), rt)
    Ht = np.zeros((N, 2), rt)
    Hx = np.zeros((N, N, 2), rt)
    xs = _cx(x, rt)
    args = [None] * 5
    keep = []
    if pb.kind == P2C:
        a, b = _cx(hx, rt), _cx(ht, rt)
        keep += [a, b]
        args[0], args[1] = a.ctypes.data, b.ctypes.data
    else:
        a, b, c = _cx(p_start, rt), _cx(p_target, rt), _cx(np.asarray(p_target) - np.asarray(p_start), rt)
        keep += [a, b, c]
        args[2], args[3], args[4] = a.ctypes.data, b.ctypes.data, c.ctypes.data
    P = ctypes.c_void_p
    fn.argtypes = [ctypes.POINTER(_Prob), P, P, P, P, P, P, (ctypes.c_double if precision == "d" else ctypes.c_float),
                   P, P, P]
    rc = fn(ctypes.byref(s), *args, xs.ctypes.data, t, H.ctypes.data, Ht.ctypes.data, Hx.ctypes.data)
    assert rc == 0
    c = lambda a: a[..., 0].astype(np.float64) + 1j * a[..., 1].astype(np.float64)  # noqa: E731
    return c(H), c(Ht), c(Hx)


def lu_solve(A, b, precision="d"):
    rt = np.float64 if precision == "d" else np.float32
    fn = lib().orc_lu_solve_d if precision == "d" else lib().orc_lu_solve_f
    N = A.shape[0]
    a, bb = _cx(A, rt), _cx(b, rt)
    z = np.zeros((N, 2), rt)
    P = ctypes.c_void_p
    fn.argtypes = [ctypes.c_int32, P, P, P]
    assert fn(N, a.ctypes.data, bb.ctypes.data, z.ctypes.data) == 0
    return z[:, 0].astype(np.float64) + 1j * z[:, 1].astype(np.float64)


def lu_pivots(A, b, precision="d"):
    """One linear solve with its pivot trace: (z [N], piv [N] = the pivot position of each column,
    mags [N, N] = |Re|+|Im| of the row at position j when column i was searched, j >= i)."""
    rt = np.float64 if precision == "d" else np.float32
    fn = lib().orc_lu_pivots_d if precision == "d" else lib().orc_lu_pivots_f
    N = A.shape[0]
    a, bb = _cx(A, rt), _cx(b, rt)
    z = np.zeros((N, 2), rt)
    piv = np.zeros(N, np.int32)
    mags = np.full((N, N), np.nan, rt)
    P = ctypes.c_void_p
    fn.argtypes = [ctypes.c_int32, P, P, P, P, P]
    assert fn(N, a.ctypes.data, bb.ctypes.data, z.ctypes.data, piv.ctypes.data, mags.ctypes.data) == 0
    return z[:, 0].astype(np.float64) + 1j * z[:, 1].astype(np.float64), piv, mags


# ----------------------------------------------------------------------------
# result counts (Evaluations.cpp:88-176 restated)
# ----------------------------------------------------------------------------

def count_results(endpoints, conv, inf, imag_tol=ZERO_IMAG_PART_TOL_FOR_SP, dup_tol=DUPLICATE_SOL_DIFF_TOL):
    """(converged, real, infinity, unique) for ONE hypothesis, reference rules.

    real: converged and every |Im x_v| <= imag_tol.
    unique: the reference's Find_Unique_Sols walk -- for each converged bs not
    in the current skip set, collect later ds (any convergence state) that
    agree in every Re and Im within dup_tol; none -> bs is unique, else the
    skip set is replaced by them (and bs is not counted).
    """
    z = np.asarray(endpoints)
    conv = np.asarray(conv).astype(bool)
    inf = np.asarray(inf).astype(bool)
    n = z.shape[0]
    n_conv = int(conv.sum())
    n_inf = int(inf.sum())
    n_real = int((conv & np.all(np.abs(z.imag) <= imag_tol, axis=1)).sum())
    zr, zi = z.real, z.imag
    skip = set()
    uniq = 0
    for bs in range(n):
        if not conv[bs]:
            continue
        if skip and bs in skip:
            continue
        if bs + 1 < n:
            close = np.all((np.abs(zr[bs + 1:] - zr[bs]) < dup_tol) & (np.abs(zi[bs + 1:] - zi[bs]) < dup_tol), axis=1)
            dups = set((np.nonzero(close)[0] + bs + 1).tolist())
        else:
            dups = set()
        if not dups:
            uniq += 1
        else:
            skip = dups
    return dict(converged=n_conv, real=n_real, infinity=n_inf, unique=uniq)
