"""ghc_track_noalloc against ghc_track (needs a B200).

ghc_track_noalloc serves callers that cannot allocate device memory (their
application owns every byte through its own pool or budget, or their loop
cannot afford cudaMalloc's synchronisation or failure mid-run).  It must
return exactly what ghc_track returns for the same inputs -- the tests here
use the same bit-for-bit bar as the other parity tests, in FP64, FP32 and mixed
precision -- on two calls in a row, since every call reuses the same fixed
device array, and it must leave the problem handle without device memory.
(Its rejection of problems whose tables exceed the array is a CPU test in
test_host_lib.py: it happens before any device work.)

This file sorts last so that a run stopping at its first failure has already
run every other test.
"""
import ctypes

import numpy as np
import pytest

import ghc

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def cx_t(a):
    a = np.asarray(a, dtype=np.complex128)
    return torch.from_numpy(np.ascontiguousarray(np.stack([a.real, a.imag], -1))).cuda()


def outputs(ws):
    return {k: getattr(ws, k).cpu().numpy().copy() for k in ("endpoints", "conv", "inf", "status", "steps", "corr",
                                                             "t_end", "resid")}


def compare(ref, got, tag):
    for k in ref:
        a, b = ref[k], got[k]
        if a.dtype.kind == "f":
            fin = np.isfinite(a)
            assert np.array_equal(np.isfinite(b), fin), (tag, k)
            assert np.array_equal(a[fin], b[fin]), (tag, k)
        else:
            assert np.array_equal(a, b), (tag, k)


@pytest.mark.parametrize("name,n_hyp,prec", [("generalized_3views_4pts", 3, ghc.PREC_FP64),
                                             ("trifocal_2op1p_30x30", 2, ghc.PREC_FP64),
                                             ("uncalibrated_trifocal_rel_pos_CY", 2, ghc.PREC_FP32),
                                             ("generalized_3views_4pts", 3, ghc.PREC_MIXED)])
def test_no_alloc_matches_track_on_two_calls(name, n_hyp, prec):
    """The first call comes on a fresh problem handle, which must stay unbound to any device
    afterwards (nothing was uploaded into it); both calls must equal ghc_track's results,
    computed afterwards on a second handle of the same problem."""
    fresh, other = ghc.Problem(name), ghc.Problem(name)
    s, t = fresh.params()
    rng = np.random.default_rng(17)
    tg = np.array([np.append(t[:-1] + 0.05 * (rng.normal(size=fresh.P) + 1j * rng.normal(size=fresh.P)), 1.0)
                   for _ in range(n_hyp)])
    rt = torch.float32 if prec == ghc.PREC_FP32 else torch.float64
    sols = cx_t(fresh.start_sols()).to(rt)
    if fresh.kind == ghc.KIND_P2C:
        # the coefficient tables come from the other handle (device P2C uploads into its handle)
        hx, ht = other.p2c_device(cx_t(s), cx_t(tg))
        kw = dict(d_coef_hx=hx, d_coef_ht=ht)
    else:
        kw = dict(d_p_start=cx_t(s), d_p_target=cx_t(tg), d_p_diff=cx_t(tg - s[None, :]))
    polish = 0 if prec == ghc.PREC_FP32 else 2
    got = []
    for call in range(2):
        ws = ghc.Workspace(fresh, n_hyp, prec)
        ghc.track(fresh, ws, sols, polish_iters=polish, no_alloc=True, **kw)
        torch.cuda.synchronize()
        got.append(outputs(ws))
    assert fresh.bound_device() == -1
    ref_ws = ghc.Workspace(other, n_hyp, prec)
    ghc.track(other, ref_ws, sols, polish_iters=polish, **kw)
    torch.cuda.synchronize()
    ref = outputs(ref_ws)
    for call in range(2):
        compare(ref, got[call], call)


def test_no_alloc_alternating_problems():
    """Calls for two different problems in turn on one stream: each copies its own tables into the
    shared array (the array held the other problem's), and each result equals ghc_track's."""
    out = {}
    for name in ("P3P", "generalized_3views_4pts", "P3P"):
        pb = ghc.Problem(name)
        s, t = pb.params()
        hx, ht = pb.p2c_device(cx_t(s), cx_t(t[None, :]))
        ws = ghc.Workspace(pb, 1, ghc.PREC_FP64)
        ghc.track(pb, ws, cx_t(pb.start_sols()), d_coef_hx=hx, d_coef_ht=ht, no_alloc=True)
        ref = ghc.Workspace(pb, 1, ghc.PREC_FP64)
        ghc.track(pb, ref, cx_t(pb.start_sols()), d_coef_hx=hx, d_coef_ht=ht)
        torch.cuda.synchronize()
        compare(outputs(ref), outputs(ws), name)
        out.setdefault(name, []).append(outputs(ws))
    compare(out["P3P"][0], out["P3P"][1], "P3P again")


def test_no_alloc_ignores_the_counter_argument():
    pb = ghc.Problem("P3P")
    s, t = pb.params()
    hx, ht = pb.p2c_device(cx_t(s), cx_t(t[None, :]))
    ws = ghc.Workspace(pb, 1, ghc.PREC_FP64)
    a = ghc.TrackArgs()
    a.n_hyp, a.precision = 1, ghc.PREC_FP64
    a.d_start_sols = cx_t(pb.start_sols()).data_ptr()
    keep = [hx, ht]
    a.d_coef_hx, a.d_coef_ht = keep[0].data_ptr(), keep[1].data_ptr()
    a.d_endpoints, a.d_conv, a.d_inf = ws.endpoints.data_ptr(), ws.conv.data_ptr(), ws.inf.data_ptr()
    a.d_counter = None
    st = torch.cuda.current_stream().cuda_stream
    assert ghc.ghc_track_noalloc(pb.h, ctypes.byref(a), st) == 0, ghc.ghc_last_error()
    torch.cuda.synchronize()
    assert ws.conv.cpu().numpy().all()
