"""Python binding of the tracker's C ABI (include/ghc.h) via ctypes.

PyTorch is used only for device memory and streams.  There is no CPU
fallback: importing this module loads libghc_b200.so and raises if it is
missing, and every call goes through the CUDA library.

Complex arrays are float tensors with a trailing (re, im) dimension of 2.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libghc_b200.so")
PROBLEMS = os.path.join(HERE, "problems")

PREC_FP64, PREC_FP32, PREC_MIXED = 0, 1, 2

# Step control without path jumping: tight corrector, contraction test on the
# first Newton update, bounded step.  Used with a corrector limit of 3.
ROBUST_STEP = dict(corr_tol2=1e-12, first_tol2=1e-2, dt_max=0.05)
KIND_P2C, KIND_PH = 0, 1
STATUS_CONVERGED, STATUS_DIVERGED, STATUS_STEP_CAP, STATUS_NONFINITE, STATUS_SINGULAR = 0, 1, 2, 3, 4

if not os.path.exists(LIB_PATH):
    raise ImportError("libghc_b200.so is not built (run homotopy-continuation-tracker-on-gpu_b200/build.py)")
_lib = ctypes.CDLL(LIB_PATH)

_P = ctypes.c_void_p
_I32 = ctypes.c_int32
_I64 = ctypes.c_int64


class ProblemInfo(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 96), ("kind", _I32), ("N", _I32), ("P", _I32), ("M", _I32), ("K", _I32),
                ("paths", _I32), ("Tx", _I32), ("Px", _I32), ("Tt", _I32), ("Pt", _I32), ("max_steps", _I32),
                ("max_corr", _I32), ("incr_steps", _I32), ("n_hx_terms", _I32), ("n_ht_terms", _I32),
                ("has_p2c_terms", _I32), ("subwarp", _I32), ("device", _I32)]


class Counts(ctypes.Structure):
    _fields_ = [("converged", _I32), ("real", _I32), ("infinity", _I32), ("unique", _I32)]


class TuneChoice(ctypes.Structure):
    _fields_ = [("variant", _I32), ("flat", _I32), ("ms", ctypes.c_double), ("candidates", _I32),
                ("variant_f32", _I32)]


class TrackArgs(ctypes.Structure):
    _fields_ = [("n_hyp", _I64), ("precision", _I32), ("max_steps", _I32), ("max_corr", _I32),
                ("incr_steps", _I32), ("t_switch", ctypes.c_double), ("polish_iters", _I32),
                ("corr_tol2", ctypes.c_double), ("first_tol2", ctypes.c_double), ("dt_max", ctypes.c_double),
                ("d_start_sols", _P), ("d_coef_hx", _P), ("d_coef_ht", _P), ("d_p_start", _P),
                ("d_p_target", _P), ("d_p_diff", _P), ("d_endpoints", _P), ("d_status", _P), ("d_conv", _P),
                ("d_inf", _P), ("d_steps", _P), ("d_corr", _P), ("d_t_end", _P), ("d_dt_end", _P),
                ("d_resid", _P), ("d_counter", _P), ("paths", _I32), ("cond_limit", ctypes.c_double),
                ("dt_floor", ctypes.c_double)]


def _sig(name, res, args):
    f = getattr(_lib, name)
    f.restype = res
    f.argtypes = args
    return f


ghc_last_error = _sig("ghc_last_error", ctypes.c_char_p, [])
ghc_version = _sig("ghc_version", ctypes.c_int, [])
ghc_problem_load = _sig("ghc_problem_load", ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(_P)])
ghc_problem_free = _sig("ghc_problem_free", None, [_P])
ghc_problem_get_info = _sig("ghc_problem_get_info", ctypes.c_int, [_P, ctypes.POINTER(ProblemInfo)])
ghc_problem_start_sols = _sig("ghc_problem_start_sols", ctypes.c_int, [_P, _P])
ghc_problem_params = _sig("ghc_problem_params", ctypes.c_int, [_P, _P, _P])
ghc_problem_raw_tables = _sig("ghc_problem_raw_tables", ctypes.c_int, [_P, _P, _P])
ghc_problem_compiled_tables = _sig("ghc_problem_compiled_tables", ctypes.c_int, [_P, _P, _I32, _P, _I32, _P, _P])
ghc_p2c = _sig("ghc_p2c", ctypes.c_int, [_P, _P, _P, _P, _P, ctypes.c_int])
ghc_p2c_device = _sig("ghc_p2c_device", ctypes.c_int, [_P, _I64, _P, _P, _P, _P, ctypes.c_int, _P])
ghc_track = _sig("ghc_track", ctypes.c_int, [_P, ctypes.POINTER(TrackArgs), _P])
ghc_track_noalloc = _sig("ghc_track_noalloc", ctypes.c_int, [_P, ctypes.POINTER(TrackArgs), _P])
ghc_autotune = _sig("ghc_autotune", ctypes.c_int, [_P, ctypes.POINTER(TrackArgs), _P, ctypes.POINTER(TuneChoice)])
ghc_set_tuning = _sig("ghc_set_tuning", ctypes.c_int, [_P, _I32, _I32, _I32])
ghc_get_tuning = _sig("ghc_get_tuning", ctypes.c_int, [_P, _I32, ctypes.POINTER(_I32), ctypes.POINTER(_I32)])
ghc_count_results = _sig("ghc_count_results", ctypes.c_int,
                         [_I32, _I32, _P, _P, _P, ctypes.c_double, ctypes.c_double, ctypes.POINTER(Counts)])
ghc_count_results_device = _sig("ghc_count_results_device", ctypes.c_int,
                                [_I32, _I32, _I64, _P, _P, _P, ctypes.c_double, ctypes.c_double, _P, _P, _P])
ghc_solve_host = _sig("ghc_solve_host", ctypes.c_int,
                      [_P, _I32, _I64, _P, ctypes.c_double, _I32, _P, _P, _P, _P, _P, _P])
_DROPIN_P2C = [_P, _P, ctypes.c_int, ctypes.c_int, ctypes.c_int, _P, _P, _P, _P, _P, _P, _P, _P, _P]
_DROPIN_PH = [_P, _P, ctypes.c_int, ctypes.c_int, ctypes.c_int, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]
ghc_kernel_HC_Solver_P2C = _sig("ghc_kernel_HC_Solver_P2C", ctypes.c_double, _DROPIN_P2C)
ghc_kernel_HC_Solver_P2C_z = _sig("ghc_kernel_HC_Solver_P2C_z", ctypes.c_double, _DROPIN_P2C)
ghc_kernel_HC_Solver_PH = _sig("ghc_kernel_HC_Solver_PH", ctypes.c_double, _DROPIN_PH)
ghc_kernel_HC_Solver_PH_z = _sig("ghc_kernel_HC_Solver_PH_z", ctypes.c_double, _DROPIN_PH)
ghc_measure_fma_peak = _sig("ghc_measure_fma_peak", ctypes.c_int, [ctypes.c_int, _P, _P])
ghc_lu_solve_device = _sig("ghc_lu_solve_device", ctypes.c_int, [_I32, _I32, _I64, _P, _P, _P, _P])
ghc_track_mix = _sig("ghc_track_mix", ctypes.c_int, [_P, _P, _I32, _P])


class GhcError(RuntimeError):
    pass


def _check(rc, what):
    if rc != 0:
        raise GhcError("%s failed (%d): %s" % (what, rc, ghc_last_error().decode()))


def _cx_np(a):
    a = np.asarray(a, dtype=np.complex128)
    out = np.empty(a.shape + (2,), dtype=np.float64)
    out[..., 0] = a.real
    out[..., 1] = a.imag
    return np.ascontiguousarray(out)


def _np_cx(a):
    a = np.asarray(a)
    return a[..., 0].astype(np.float64) + 1j * a[..., 1].astype(np.float64)


def _ptr(t):
    return None if t is None else t.data_ptr()


def _stream():
    import torch
    return torch.cuda.current_stream().cuda_stream


class Problem:
    """A problem folder (reference layout) loaded through ghc_problem_load."""

    def __init__(self, name, root=PROBLEMS):
        h = _P()
        _check(ghc_problem_load(root.encode(), name.encode(), ctypes.byref(h)), "ghc_problem_load(%s)" % name)
        self.h = h
        info = ProblemInfo()
        _check(ghc_problem_get_info(h, ctypes.byref(info)), "ghc_problem_get_info")
        self.info = info
        for f, _ in ProblemInfo._fields_:
            if f != "name":
                setattr(self, f, getattr(info, f))
        self.name = info.name.decode()

    def bound_device(self):
        """Device holding the handle's compiled tables (uploaded by its first tracking call), -1: none."""
        info = ProblemInfo()
        _check(ghc_problem_get_info(self.h, ctypes.byref(info)), "ghc_problem_get_info")
        return info.device

    def __del__(self):
        h = getattr(self, "h", None)
        if h and ghc_problem_free is not None:
            ghc_problem_free(h)
            self.h = None

    def start_sols(self):
        out = np.zeros((self.paths, self.N, 2))
        _check(ghc_problem_start_sols(self.h, out.ctypes.data), "ghc_problem_start_sols")
        return _np_cx(out)

    def params(self):
        s = np.zeros((self.P + 1, 2))
        t = np.zeros((self.P + 1, 2))
        _check(ghc_problem_params(self.h, s.ctypes.data, t.ctypes.data), "ghc_problem_params")
        return _np_cx(s), _np_cx(t)

    def raw_tables(self):
        hx = np.zeros(self.N * self.N * self.Tx * self.Px, dtype=np.int32)
        ht = np.zeros(self.N * self.Tt * self.Pt, dtype=np.int32)
        _check(ghc_problem_raw_tables(self.h, hx.ctypes.data, ht.ctypes.data), "ghc_problem_raw_tables")
        return hx, ht

    def compiled_hx(self):
        """The compiled H_x tables the tracker walks: (uint64 term words, uint16 offsets)."""
        nw, no = _I32(), _I32()
        _check(ghc_problem_compiled_tables(self.h, None, 0, None, 0, ctypes.byref(nw), ctypes.byref(no)),
               "ghc_problem_compiled_tables")
        w = np.zeros(nw.value, dtype=np.uint64)
        o = np.zeros(no.value, dtype=np.uint16)
        _check(ghc_problem_compiled_tables(self.h, w.ctypes.data, nw.value, o.ctypes.data, no.value,
                                           ctypes.byref(nw), ctypes.byref(no)), "ghc_problem_compiled_tables")
        return w, o

    def p2c(self, start, target, exact_ht=False):
        """Host coefficient tables for one hypothesis -> (hx [(M+1)(K+1)], ht [(M+1)K]) complex."""
        s, t = _cx_np(start), _cx_np(target)
        hx = np.zeros(((self.M + 1) * (self.K + 1), 2))
        ht = np.zeros((max(1, (self.M + 1) * self.K), 2))
        _check(ghc_p2c(self.h, s.ctypes.data, t.ctypes.data, hx.ctypes.data, ht.ctypes.data, int(exact_ht)),
               "ghc_p2c")
        return _np_cx(hx), _np_cx(ht)[: (self.M + 1) * self.K]

    def p2c_device(self, d_start, d_targets, exact_ht=False):
        """Device tables for n_hyp hypotheses (torch float64 [.., 2] tensors on cuda)."""
        import torch
        n = d_targets.shape[0]
        hx = torch.empty((n, (self.M + 1) * (self.K + 1), 2), dtype=torch.float64, device=d_targets.device)
        ht = torch.empty((n, max(1, (self.M + 1) * self.K), 2), dtype=torch.float64, device=d_targets.device)
        _check(ghc_p2c_device(self.h, n, d_start.data_ptr(), d_targets.data_ptr(), hx.data_ptr(), ht.data_ptr(),
                              int(exact_ht), _stream()), "ghc_p2c_device")
        return hx, ht


class Workspace:
    """Device output buffers for ``track`` (reused across calls)."""

    def __init__(self, pb, n_hyp, precision, device="cuda", paths=None):
        import torch
        self.paths = pb.paths if paths is None else paths
        n = n_hyp * self.paths
        rt = torch.float32 if precision == PREC_FP32 else torch.float64
        self.n_hyp = n_hyp
        self.precision = precision
        self.endpoints = torch.zeros((n, pb.N, 2), dtype=rt, device=device)
        self.status = torch.zeros(n, dtype=torch.uint8, device=device)
        self.conv = torch.zeros(n, dtype=torch.uint8, device=device)
        self.inf = torch.zeros(n, dtype=torch.uint8, device=device)
        self.steps = torch.zeros(n, dtype=torch.int32, device=device)
        self.corr = torch.zeros(n, dtype=torch.int32, device=device)
        self.t_end = torch.zeros(n, dtype=torch.float64, device=device)
        self.dt_end = torch.zeros(n, dtype=torch.float64, device=device)
        self.resid = torch.zeros(n, dtype=torch.float64, device=device)
        self.counter = torch.zeros(4, dtype=torch.int32, device=device)


def track(pb, ws, d_start_sols, d_coef_hx=None, d_coef_ht=None, d_p_start=None, d_p_target=None, d_p_diff=None,
          t_switch=1.0, polish_iters=0, max_steps=0, max_corr=0, incr_steps=0, want_resid=False, step=None,
          no_alloc=False, cond_limit=0.0, dt_floor=0.0):
    """Launch the batched tracker (asynchronous on torch's current stream).

    step: optional dict(corr_tol2=, first_tol2=, dt_max=) step control; the
    default is the reference's (see ROBUST_STEP for the path-jump-free one).
    PREC_MIXED: the mixed tracker (FP64 state and residual, FP32 H_x, H_t and LU) for
    t < t_switch (>= 1: the whole path), then FP64 for the paths it hands over
    (cond_limit: pivot-magnitude span of an FP32 solve that hands a path over, 0: 1e5;
    dt_floor: step size below which a path is handed over, 0: 1e-4).
    """
    a = _track_args(ws, d_start_sols, d_coef_hx, d_coef_ht, d_p_start, d_p_target, d_p_diff, t_switch,
                    polish_iters, max_steps, max_corr, incr_steps, want_resid, step, cond_limit, dt_floor)
    if no_alloc:
        # ghc_track_noalloc: counter and tables in the library's fixed device array
        a.d_counter = None
        _check(ghc_track_noalloc(pb.h, ctypes.byref(a), _stream()), "ghc_track_noalloc")
    else:
        _check(ghc_track(pb.h, ctypes.byref(a), _stream()), "ghc_track")


def track_mix(buckets):
    """Batches of different problems in one persistent launch (ghc_track_mix), asynchronous on
    torch's current stream.  buckets: list of (pb, ws, d_start_sols, kw), kw as for track
    (plain FP64, no polish).  Bit-identical to calling track for each bucket."""
    n = len(buckets)
    pbs = (_P * n)(*[b[0].h for b in buckets])
    args = (TrackArgs * n)()
    for i, (pb, ws, ss, kw) in enumerate(buckets):
        args[i] = _track_args(ws, ss, **kw)
    _check(ghc_track_mix(ctypes.cast(pbs, _P), ctypes.cast(args, _P), n, _stream()), "ghc_track_mix")


def autotune(pb, ws, d_start_sols, **kw):
    """Time the launch choices on this sample batch (track's arguments; outputs overwritten),
    keep the fastest in the problem handle for the workspace's precision and return it
    as dict(variant, flat, ms, candidates).  Synchronises torch's current stream."""
    a = _track_args(ws, d_start_sols, **kw)
    out = TuneChoice()
    _check(ghc_autotune(pb.h, ctypes.byref(a), _stream(), ctypes.byref(out)), "ghc_autotune")
    return dict(variant=out.variant, flat=out.flat, ms=out.ms, candidates=out.candidates,
                variant_f32=out.variant_f32)


def set_tuning(pb, precision, variant, flat=-1):
    """Launch choice for ``precision``: register-budget ``variant`` (0, 1) and H_x walk ``flat``
    (0 entry-wise, 1 row-wise, 2 balanced over all lanes, -1 from the table structure)."""
    _check(ghc_set_tuning(pb.h, precision, variant, flat), "ghc_set_tuning")


def get_tuning(pb, precision):
    v, f = _I32(), _I32()
    _check(ghc_get_tuning(pb.h, precision, ctypes.byref(v), ctypes.byref(f)), "ghc_get_tuning")
    return v.value, f.value


def _track_args(ws, d_start_sols, d_coef_hx=None, d_coef_ht=None, d_p_start=None, d_p_target=None, d_p_diff=None,
                t_switch=1.0, polish_iters=0, max_steps=0, max_corr=0, incr_steps=0, want_resid=False, step=None,
                cond_limit=0.0, dt_floor=0.0):
    a = TrackArgs()
    a.n_hyp = ws.n_hyp
    a.precision = ws.precision
    a.max_steps, a.max_corr, a.incr_steps = max_steps, max_corr, incr_steps
    a.t_switch = t_switch
    a.polish_iters = polish_iters
    st = step or {}
    a.corr_tol2 = st.get("corr_tol2", 0.0)
    a.first_tol2 = st.get("first_tol2", 0.0)
    a.dt_max = st.get("dt_max", 0.0)
    a.d_start_sols = _ptr(d_start_sols)
    a.d_coef_hx, a.d_coef_ht = _ptr(d_coef_hx), _ptr(d_coef_ht)
    a.d_p_start, a.d_p_target, a.d_p_diff = _ptr(d_p_start), _ptr(d_p_target), _ptr(d_p_diff)
    a.d_endpoints = ws.endpoints.data_ptr()
    a.d_status, a.d_conv, a.d_inf = ws.status.data_ptr(), ws.conv.data_ptr(), ws.inf.data_ptr()
    a.d_steps, a.d_corr = ws.steps.data_ptr(), ws.corr.data_ptr()
    a.d_t_end, a.d_dt_end = ws.t_end.data_ptr(), ws.dt_end.data_ptr()
    a.d_resid = ws.resid.data_ptr() if (want_resid or polish_iters > 0) and ws.precision != PREC_FP32 else None
    a.d_counter = ws.counter.data_ptr()
    a.paths = ws.paths
    a.cond_limit = cond_limit
    a.dt_floor = dt_floor
    return a


def measure_fma_peak(precision=PREC_FP64):
    """Measured FMA throughput of the current device in FLOP/s."""
    f = ctypes.c_double()
    ms = ctypes.c_double()
    _check(ghc_measure_fma_peak(precision, ctypes.byref(f), ctypes.byref(ms)), "ghc_measure_fma_peak")
    return f.value


def lu_solve_device(d_A, d_b, precision=PREC_FP64):
    """The tracker's linear solve on the device: d_A [n, N, N, 2], d_b [n, N, 2] float64 (FP64) or
    float32 (FP32) tensors -> d_z [n, N, 2] (torch's current stream)."""
    import torch
    n, N = d_A.shape[0], d_A.shape[1]
    z = torch.empty_like(d_b)
    _check(ghc_lu_solve_device(N, precision, n, d_A.data_ptr(), d_b.data_ptr(), z.data_ptr(), _stream()),
           "ghc_lu_solve_device")
    return z


def count_results(endpoints, conv, inf, imag_tol=1e-4, dup_tol=1e-4):
    """Reference counts for one hypothesis (host): endpoints complex [paths, N]."""
    z = _cx_np(endpoints)
    c = np.ascontiguousarray(np.asarray(conv, dtype=np.uint8))
    i = np.ascontiguousarray(np.asarray(inf, dtype=np.uint8))
    out = Counts()
    _check(ghc_count_results(z.shape[1], z.shape[0], z.ctypes.data, c.ctypes.data, i.ctypes.data, imag_tol, dup_tol,
                             ctypes.byref(out)), "ghc_count_results")
    return dict(converged=out.converged, real=out.real, infinity=out.infinity, unique=out.unique)


def count_results_device(ws, N, imag_tol=1e-4, dup_tol=1e-4, want_class=False, out=None, class_out=None):
    """Counts of every hypothesis of a workspace, on the device (torch's current stream).

    Returns (counts int32 tensor [n_hyp, 4] = converged, real, infinity, unique;
    class uint8 tensor [n_hyp * paths] or None): bit 0 converged, bit 1 real,
    bit 2 counted as unique.  Needs FP64 endpoints (FP64 or mixed workspace).
    out / class_out: preallocated int32 [>= n_hyp, 4] / uint8 [>= n_hyp * paths] device tensors.
    """
    import torch
    if ws.endpoints.dtype != torch.float64:
        raise GhcError("count_results_device needs FP64 endpoints")
    counts = out if out is not None else torch.zeros((ws.n_hyp, 4), dtype=torch.int32, device=ws.endpoints.device)
    cls = class_out
    if cls is None and want_class:
        cls = torch.zeros(ws.n_hyp * ws.paths, dtype=torch.uint8, device=ws.endpoints.device)
    _check(ghc_count_results_device(N, ws.paths, ws.n_hyp, ws.endpoints.data_ptr(), ws.conv.data_ptr(),
                                    ws.inf.data_ptr(), imag_tol, dup_tol, counts.data_ptr(),
                                    None if cls is None else cls.data_ptr(), _stream()), "ghc_count_results_device")
    return counts, cls


def solve_outputs(pb, n_hyp):
    """Host output arrays for solve_host (reusable across calls of the same size)."""
    n = n_hyp * pb.paths
    return dict(endpoints=np.zeros((n, pb.N), np.complex128), status=np.zeros(n, np.uint8),
                conv=np.zeros(n, np.uint8), inf=np.zeros(n, np.uint8), steps=np.zeros(n, np.int32),
                ms=np.zeros(3))


def solve_host(pb, precision=PREC_FP64, targets=None, t_switch=1.0, polish_iters=0, out=None):
    """One-call host solve (host buffers in and out, copies included).

    targets: [n_hyp, P+1] complex (None: the problem's target, n_hyp = 1).  out: arrays from
    solve_outputs() to fill in place (fresh ones otherwise).  Returns the dict of arrays;
    endpoints [n_hyp * paths, N] complex128 is written directly by the library."""
    n_hyp = 1 if targets is None else np.asarray(targets).shape[0]
    o = out if out is not None else solve_outputs(pb, n_hyp)
    if o["endpoints"].shape != (n_hyp * pb.paths, pb.N) or o["endpoints"].dtype != np.complex128:
        raise GhcError("solve_host: output arrays of the wrong size")
    tg = None
    if targets is not None:
        tg = np.asarray(targets)
        if tg.dtype != np.complex128 or not tg.flags.c_contiguous:
            tg = np.ascontiguousarray(tg, dtype=np.complex128)
    _check(ghc_solve_host(pb.h, precision, n_hyp, None if tg is None else tg.ctypes.data, t_switch, polish_iters,
                          o["endpoints"].ctypes.data, o["status"].ctypes.data, o["conv"].ctypes.data,
                          o["inf"].ctypes.data, o["steps"].ctypes.data, o["ms"].ctypes.data), "ghc_solve_host")
    return o
