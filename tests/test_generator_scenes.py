"""Native table generator and seeded scenes (no GPU).

* gen/p2c_gen.py derive mode reproduces the committed coefficient expressions
  from the reference's polynomial systems (needs the reference tree);
* the generated P3P_TD tables evaluate to the polynomial system they encode;
* known-answer tests: noise-free scenes have their ground truth as a root, and
  the oracle tracker recovers it.
"""
import os
import sys

import numpy as np
import pytest

import oracle as O
import scenes

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GEN = os.path.join(REPO, "homotopy-continuation-tracker-on-gpu_b200", "gen")
sys.path.insert(0, GEN)
import make_p3p_td  # noqa: E402
import p2c_gen  # noqa: E402

REF = os.environ.get("GHC_REFERENCE_ROOT") or os.path.join(os.path.dirname(os.path.dirname(os.path.dirname(
    os.path.abspath(__file__)))), "reference")


@pytest.mark.skipif(not os.path.isdir(REF), reason="reference tree not present")
@pytest.mark.parametrize("name", ["P3P", "generalized_3views_4pts", "uncalibrated_trifocal_rel_pos_CY"])
def test_derive_reproduces_committed_terms(name):
    d = os.path.join(O.PKG_PROBLEMS, name)
    info = p2c_gen.derive(d, os.path.join(REF, "auto-data-gen-tools", "p2c-problems", "sys_%s.m" % name))
    committed = O.read_p2c_terms(os.path.join(d, "p2c_terms.txt"))
    assert info["M"] == committed["M"] and info["K"] == committed["K"]
    for k in range(info["M"]):
        a = sorted((float(c), tuple(f)) for c, f in info["coefs"][k])
        b = sorted((float(c), tuple(f)) for c, f in committed["terms"][k])
        assert a == b, k


def test_p3p_td_tables_encode_the_system():
    pb = O.Problem("P3P_TD")
    rng = np.random.default_rng(0)
    p = rng.normal(size=12) + 1j * rng.normal(size=12)
    q = rng.normal(size=12) + 1j * rng.normal(size=12)
    hx, ht = O.p2c_tables(pb.terms, np.append(q, 1), np.append(p, 1), exact_ht=True)
    x = rng.normal(size=3) + 1j * rng.normal(size=3)
    t = 0.3
    pt = (1 - t) * q + t * p
    H, Ht, Hx = O.eval_system(pb, x, t, hx=hx, ht=ht)
    for e, (i, j) in enumerate(make_p3p_td.PAIRS):
        a = pt[4 * e:4 * e + 4]
        da = (p - q)[4 * e:4 * e + 4]
        f = a[0] * x[i] ** 2 + a[1] * x[j] ** 2 + a[2] * x[i] * x[j] + a[3]
        ft = da[0] * x[i] ** 2 + da[1] * x[j] ** 2 + da[2] * x[i] * x[j] + da[3]
        assert abs(H[e] - f) < 1e-12 and abs(Ht[e] - ft) < 1e-12
        assert abs(Hx[e, i] - (2 * a[0] * x[i] + a[2] * x[j])) < 1e-12
        assert abs(Hx[e, j] - (2 * a[1] * x[j] + a[2] * x[i])) < 1e-12


def test_p3p_td_known_answer():
    pb = O.Problem("P3P_TD")
    (st, tg), gt = scenes.p3p_td(10, seed=11)
    for h in range(10):
        hx, ht = O.p2c_tables(pb.terms, st, tg[h])
        H, _, _ = O.eval_system(pb, gt[h].astype(complex), 1.0, hx=hx, ht=ht)
        assert np.abs(H).max() < 1e-10
        r = O.track(pb, pb.start_sols, hx=hx, ht=ht, polish_iters=3)
        assert r["conv"].all()
        E = r["endpoints"]
        assert np.abs(E - gt[h]).max(axis=1).min() < 1e-9


def test_generalized_3views_4pts_scene_known_answer():
    pb = O.Problem("generalized_3views_4pts")
    tg, gt = scenes.generalized_3views_4pts(1, seed=1, noise_px=0.0)
    hx, ht = O.p2c_tables(pb.terms, pb.start_params, tg[0])
    H, _, _ = O.eval_system(pb, gt[0].astype(complex), 1.0, hx=hx, ht=ht)
    assert np.abs(H).max() < 1e-10
    r = O.track(pb, pb.start_sols, hx=hx, ht=ht, polish_iters=3, nthreads=os.cpu_count(), step=O.ROBUST_STEP,
                max_corr=3, max_steps=2000)
    E = r["endpoints"][r["conv"] == 1]
    assert np.abs(E - gt[0]).max(axis=1).min() < 1e-9


def test_trifocal_30x30_scene_known_answer():
    """Scenes -> the 33 parameters of the Chicago-style trifocal system: the scene's unknowns
    solve F(x; c) = 0, and tracking the shipped 312-path start system recovers them."""
    pb = O.Problem("trifocal_2op1p_30x30")
    tg, gt = scenes.trifocal_2op1p_30x30(3, seed=5)
    for h in range(3):
        H, _, _ = O.eval_system(pb, gt[h].astype(complex), 1.0, p_start=pb.start_params, p_target=tg[h])
        assert np.abs(H).max() < 1e-12 * max(1.0, np.abs(gt[h]).max() ** 3)
    r = O.track(pb, pb.start_sols, p_start=pb.start_params, p_target=tg[:1], polish_iters=3,
                nthreads=os.cpu_count())
    E = r["endpoints"][r["conv"] == 1]
    assert np.abs(E - gt[0]).max(axis=1).min() < 1e-9 * np.abs(gt[0]).max()


def test_cayley_is_a_scaled_rotation():
    rng = np.random.default_rng(0)
    for _ in range(5):
        r = rng.normal(size=3)
        R = scenes.cayley(r) / (1 + r @ r)
        assert np.allclose(R @ R.T, np.eye(3), atol=1e-12) and abs(np.linalg.det(R) - 1) < 1e-12


def test_quadratic_total_degree_generator(tmp_path):
    """gen/make_quadratic_td.py writes a folder both readers accept, whose start solutions solve the
    start system, and whose paths the oracle tracks to solutions of the target system."""
    import make_quadratic_td
    make_quadratic_td.write(str(tmp_path), 5, paths=12, seed=1)
    ob = O.Problem("QTD_5", root=str(tmp_path))
    assert ob.paths == 12 and ob.N == 5
    hx, ht = O.p2c_tables(ob.terms, ob.start_params, ob.target_params)
    hx0, ht0 = O.p2c_tables(ob.terms, ob.start_params, ob.start_params)
    for x in ob.start_sols:
        H, _, _ = O.eval_system(ob, x, 0.0, hx=hx0, ht=ht0)
        assert np.abs(H).max() < 1e-12
    r = O.track(ob, ob.start_sols, hx=hx, ht=ht, polish_iters=2)
    assert (r["resid"][r["conv"] == 1] < 1e-10).all() and r["conv"].mean() > 0.9
