"""The device LU (ghc_lu_solve_device, the solve inside every tracker step) vs the oracle's LU,
bit for bit, on random matrices, exact ties, near ties one unit in the last place apart, zero
pivots and NaN, at every compiled size in FP64 and FP32 (needs a B200).  The oracle's pivot rule
is pinned to the reference's scan in test_oracle_pins.py, so equal solutions here mean the
device takes the reference's pivots."""
import numpy as np
import pytest

import ghc
import oracle as O
from lu_cases import SIZES, cases

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def cx_t(a, dtype):
    a = np.asarray(a, dtype=np.complex128)
    return torch.from_numpy(np.ascontiguousarray(np.stack([a.real, a.imag], -1))).to(dtype).cuda()


@pytest.mark.parametrize("prec", [ghc.PREC_FP64, ghc.PREC_FP32])
@pytest.mark.parametrize("N", SIZES)
def test_device_lu_equals_oracle(N, prec):
    rt = np.float64 if prec == ghc.PREC_FP64 else np.float32
    tt = torch.float64 if prec == ghc.PREC_FP64 else torch.float32
    cs = cases(N, rt, seed=3)
    A = np.array([a for _, a, _ in cs])
    b = np.array([v for _, _, v in cs])
    z = ghc.lu_solve_device(cx_t(A, tt), cx_t(b, tt), prec)
    torch.cuda.synchronize()
    z = z.double().cpu().numpy()
    z = z[..., 0] + 1j * z[..., 1]
    for s, (kind, a, v) in enumerate(cs):
        ref = O.lu_solve(a, v, "d" if prec == ghc.PREC_FP64 else "f")
        assert np.array_equal(z[s], ref, equal_nan=True), (kind, N, s)
