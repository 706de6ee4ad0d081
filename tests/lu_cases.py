"""Seeded linear systems for the LU tests: random, exact ties, near ties, zero pivots, NaN.

Test helper (imported by test_oracle_pins.py and test_gpu_lu.py); every case is an
(A [N, N], b [N]) complex pair.  The pivot rule under test is the reference's
(GPU-HC/magmaHC/dev-cgesv-batched-small.cuh:54-65): largest |Re|+|Im| among the
unpivoted positions, strict '>' in position order, so the lowest position wins ties.
"""
import numpy as np

SIZES = [3, 4, 5, 6, 8, 10, 11, 12, 16, 18, 30]


def _cn(rng, shape):
    return rng.normal(size=shape) + 1j * rng.normal(size=shape)


def cases(N, rt=np.float64, seed=0, n_each=6):
    """A list of (kind, A, b) for size N in real type rt (values representable in rt)."""
    rng = np.random.default_rng(seed + 1000 * N + (0 if rt == np.float64 else 7))
    out = []
    for _ in range(n_each):
        out.append(("random", _cn(rng, (N, N)), _cn(rng, N)))
    for _ in range(n_each):
        # small Gaussian integers: exact ties in |Re|+|Im| in every early column
        A = rng.integers(-2, 3, size=(N, N)) + 1j * rng.integers(-2, 3, size=(N, N))
        A += np.eye(N) * 0.125  # keep most of them non-singular
        out.append(("integer ties", A, _cn(rng, N)))
    for _ in range(n_each):
        # exact ties: column 0 holds a + bi in forms of equal |Re|+|Im| (swapped, negated)
        A = _cn(rng, (N, N))
        a, b = rng.normal(), rng.normal()
        forms = [a + 1j * b, b + 1j * a, -a + 1j * b, a - 1j * b, -b - 1j * a]
        for r in range(N):
            A[r, 0] = forms[rng.integers(len(forms))]
        out.append(("exact ties", A, _cn(rng, N)))
    for _ in range(n_each):
        # near ties: column 0 magnitudes one unit in the last place apart, the larger one below
        A = _cn(rng, (N, N))
        m = abs(rng.normal()) + 1.0
        base = np.array(m, dtype=rt)
        up = np.nextafter(base, np.array(np.inf, dtype=rt))
        for r in range(N):
            A[r, 0] = complex(float(base), 0.0) if r < N - 1 else complex(float(up), 0.0)
        A[0, 0] = complex(float(np.nextafter(base, np.array(0, dtype=rt))), 0.0)
        out.append(("near ties", A, _cn(rng, N)))
    # zero column (zero pivot), NaN at the first position, NaN below, a zero row
    A = _cn(rng, (N, N))
    A[:, N // 2] = 0
    out.append(("zero pivot", A, _cn(rng, N)))
    A = _cn(rng, (N, N))
    A[0, 0] = complex(np.nan, 0.0)
    out.append(("nan first", A, _cn(rng, N)))
    A = _cn(rng, (N, N))
    A[N - 1, 0] = complex(np.nan, 1.0)
    A[N // 2, 1] = complex(0.0, np.nan)
    out.append(("nan below", A, _cn(rng, N)))
    A = _cn(rng, (N, N))
    A[N - 1, :] = 0
    out.append(("zero row", A, _cn(rng, N)))
    # round every entry to rt so both sides start from the same values
    return [(k, A.astype(np.complex64).astype(np.complex128) if rt == np.float32 else A,
             b.astype(np.complex64).astype(np.complex128) if rt == np.float32 else b) for k, A, b in out]


def strict_argmax(mags, i):
    """The reference's scan of column i: start at position i, move to a strictly larger magnitude
    in position order (NaN comparisons are false)."""
    best, best_pos = mags[i], i
    for j in range(i + 1, len(mags)):
        if mags[j] > best:
            best, best_pos = mags[j], j
    return best_pos
