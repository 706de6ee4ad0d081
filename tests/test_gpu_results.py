"""On-device result counts (ghc_count_results_device) vs the host rule and the oracle (needs a B200).

The device kernel must reproduce the reference's counting rules exactly:
converged / infinity flags, real = converged with every |Im| <= tol, and the
sequential unique walk whose skip set is replaced by each duplicate set.
"""
import numpy as np
import pytest

import ghc
import oracle as O
import scenes

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _cx_t(a):
    a = np.asarray(a, dtype=np.complex128)
    return torch.from_numpy(np.ascontiguousarray(np.stack([a.real, a.imag], -1))).cuda()


class _WS:
    """Workspace-like holder for synthetic endpoints and flags."""

    def __init__(self, z, conv, inf):
        self.n_hyp, self.paths = z.shape[0], z.shape[1]
        self.endpoints = _cx_t(z.reshape(-1, z.shape[2]))
        self.conv = torch.from_numpy(conv.reshape(-1).astype(np.uint8)).cuda()
        self.inf = torch.from_numpy(inf.reshape(-1).astype(np.uint8)).cuda()


def _check_against_host(z, conv, inf, imag_tol=1e-4, dup_tol=1e-4):
    ws = _WS(z, conv, inf)
    counts, cls = ghc.count_results_device(ws, z.shape[2], imag_tol, dup_tol, want_class=True)
    torch.cuda.synchronize()
    counts = counts.cpu().numpy()
    cls = cls.cpu().numpy().reshape(z.shape[0], z.shape[1])
    for h in range(z.shape[0]):
        host = ghc.count_results(z[h], conv[h], inf[h], imag_tol, dup_tol)
        orc = O.count_results(z[h], conv[h], inf[h], imag_tol, dup_tol)
        dev = dict(converged=counts[h, 0], real=counts[h, 1], infinity=counts[h, 2], unique=counts[h, 3])
        assert dev == host == orc, (h, dev, host, orc)
        assert (cls[h] & 1).sum() == host["converged"]
        assert ((cls[h] >> 1) & 1).sum() == host["real"]
        assert ((cls[h] >> 2) & 1).sum() == host["unique"]
        assert np.array_equal((cls[h] & 1).astype(bool), conv[h].astype(bool))
    return counts


@pytest.mark.parametrize("paths", [1, 31, 33, 64, 700])
def test_synthetic_clusters_nans_and_sizes(paths):
    rng = np.random.default_rng(paths)
    H, N = 5, 4
    z = rng.normal(size=(H, paths, N)) + 1j * rng.normal(size=(H, paths, N))
    # plant duplicate clusters (within tolerance) and real points
    for h in range(H):
        for _ in range(paths // 4):
            a, b = rng.integers(0, paths, 2)
            z[h, b] = z[h, a] + 1e-6 * rng.normal(size=N)
        real = rng.random(paths) < 0.3
        z[h, real] = z[h, real].real + 1e-6j
    z[0, 0, 1] = np.nan + 0j
    z[1, -1, 0] = complex(0.0, np.nan)
    conv = rng.random((H, paths)) < 0.8
    inf = ~conv & (rng.random((H, paths)) < 0.5)
    _check_against_host(z, conv, inf)


def test_everything_duplicates():
    """dup_tol larger than the spread: the first converged path's duplicate set is every later path."""
    rng = np.random.default_rng(1)
    z = (rng.normal(size=(3, 70, 3)) + 1j * rng.normal(size=(3, 70, 3))) * 1e-3
    conv = rng.random((3, 70)) < 0.7
    inf = np.zeros_like(conv)
    counts = _check_against_host(z, conv, inf, dup_tol=1.0)
    assert (counts[:, 3] <= 1).all()


def test_tracker_output_with_path_jumps():
    """generalized_3views_4pts under the reference step control: many paths end on the same point."""
    pb = ghc.Problem("generalized_3views_4pts")
    s, _ = pb.params()
    tg, _ = scenes.generalized_3views_4pts(4, seed=11)
    ws = ghc.Workspace(pb, 4, ghc.PREC_FP64)
    hx, ht = pb.p2c_device(_cx_t(s), _cx_t(tg))
    ghc.track(pb, ws, _cx_t(pb.start_sols()), d_coef_hx=hx, d_coef_ht=ht, polish_iters=2)
    counts, _ = ghc.count_results_device(ws, pb.N)
    torch.cuda.synchronize()
    counts = counts.cpu().numpy()
    e = ws.endpoints.cpu().numpy()
    e = (e[..., 0] + 1j * e[..., 1]).reshape(4, pb.paths, pb.N)
    conv = ws.conv.cpu().numpy().reshape(4, -1)
    inf = ws.inf.cpu().numpy().reshape(4, -1)
    for h in range(4):
        host = ghc.count_results(e[h], conv[h], inf[h])
        assert [host["converged"], host["real"], host["infinity"], host["unique"]] == counts[h].tolist()
    assert (counts[:, 3] < counts[:, 0]).all()  # the reference control leaves duplicates


def test_real_scenes_have_real_solutions():
    pb = ghc.Problem("P3P_TD")
    (st, tg), _ = scenes.p3p_td(16, seed=2)
    ws = ghc.Workspace(pb, 16, ghc.PREC_FP64)
    hx, ht = pb.p2c_device(_cx_t(st), _cx_t(tg))
    ghc.track(pb, ws, _cx_t(pb.start_sols()), d_coef_hx=hx, d_coef_ht=ht, polish_iters=2)
    counts, cls = ghc.count_results_device(ws, pb.N, want_class=True)
    torch.cuda.synchronize()
    counts = counts.cpu().numpy()
    assert (counts[:, 1] >= 1).all()  # every real scene has its real pose among the solutions
    assert cls.numel() == 16 * pb.paths


def test_empty_batch():
    ws = _WS(np.zeros((1, 4, 3), complex), np.zeros((1, 4), bool), np.zeros((1, 4), bool))
    ws.n_hyp = 0
    counts, _ = ghc.count_results_device(ws, 3)
    assert counts.shape == (0, 4)
