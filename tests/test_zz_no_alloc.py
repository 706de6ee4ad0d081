"""ghc_track_noalloc against ghc_track (needs a B200).

ghc_track_noalloc serves callers that cannot allocate device memory (their
application owns every byte through its own pool or budget, or their loop
cannot afford cudaMalloc's synchronisation or failure mid-run).  It must
return exactly what ghc_track returns for the same inputs -- the tests here
use the same bit-for-bit bar as the other FP64 parity tests -- on two calls in
a row, since every call reuses the same fixed device array.

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


@pytest.mark.parametrize("name,n_hyp", [("generalized_3views_4pts", 3), ("trifocal_2op1p_30x30", 2)])
def test_no_alloc_matches_track_on_two_calls(name, n_hyp):
    pb = ghc.Problem(name)
    s, t = pb.params()
    rng = np.random.default_rng(17)
    tg = np.array([np.append(t[:-1] + 0.05 * (rng.normal(size=pb.P) + 1j * rng.normal(size=pb.P)), 1.0)
                   for _ in range(n_hyp)])
    sols = cx_t(pb.start_sols())
    if pb.kind == ghc.KIND_P2C:
        hx, ht = pb.p2c_device(cx_t(s), cx_t(tg))
        kw = dict(d_coef_hx=hx, d_coef_ht=ht)
    else:
        kw = dict(d_p_start=cx_t(s), d_p_target=cx_t(tg), d_p_diff=cx_t(tg - s[None, :]))
    ref_ws = ghc.Workspace(pb, n_hyp, ghc.PREC_FP64)
    ghc.track(pb, ref_ws, sols, polish_iters=2, **kw)
    torch.cuda.synchronize()
    ref = outputs(ref_ws)
    for call in range(2):
        ws = ghc.Workspace(pb, n_hyp, ghc.PREC_FP64)
        ghc.track(pb, ws, sols, polish_iters=2, no_alloc=True, **kw)
        torch.cuda.synchronize()
        got = outputs(ws)
        for k in ref:
            a, b = ref[k], got[k]
            if a.dtype.kind == "f":
                fin = np.isfinite(a)
                assert np.array_equal(np.isfinite(b), fin), (call, k)
                assert np.array_equal(a[fin], b[fin]), (call, k)
            else:
                assert np.array_equal(a, b), (call, k)


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
