"""GPU tracker vs the CPU oracle on identical inputs (needs a B200).

FP64 and FP32 modes follow the oracle's operation order, so endpoints, flags
and step/iteration counters must be identical (compared as values).  Mixed
precision (the mixed tracker with FP32 linear algebra and an FP64 residual, then FP64 for the
paths it hands over) is compared the same way
with the oracle's two-phase run, and by recall of the FP64 real endpoints.
"""
import os

import numpy as np
import pytest

import ghc
import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

SUPPORTED = ["P3P", "5pt_rel_pos_alg_form_quat", "generalized_3views_4pts", "uncalibrated_trifocal_rel_pos_CY",
             "3view_triangulation", "6pt_RS_abs_pos", "dual_reciever_TDOA_5pt", "distorted_2view_triangulation",
             "P3P_10x10", "trifocal_2op1p_30x30", "P3P_TD", "3pt_rel_pos_homog", "4view_triangulation",
             "5pt_rel_pos_full_form_quat", "5pt_rel_pos_geo_form_quat", "6pt_RS_abs_pos_1lin",
             "PnP_unkn_principal_pt", "generalized_3views_6lines", "optimal_P4P_abs_pos", "optimal_PnP_quat",
             "rel_pos_quiver", "uncalibrated_trifocal_rel_pos_CH"]
NCPU = os.cpu_count() or 1


def cx_t(a, dtype=torch.float64):
    a = np.asarray(a, dtype=np.complex128)
    return torch.from_numpy(np.ascontiguousarray(np.stack([a.real, a.imag], -1))).to(dtype).cuda()


def to_cx(t):
    a = t.double().cpu().numpy()
    return a[..., 0] + 1j * a[..., 1]


def inputs(name, n_hyp=1, seed=0):
    """problem handles + per-hypothesis targets (hypothesis 0 = shipped target)."""
    pb, ob = ghc.Problem(name), O.Problem(name)
    rng = np.random.default_rng(seed)
    tg = [ob.target_params]
    for _ in range(n_hyp - 1):
        # small seeded perturbations of the shipped target keep the problems well posed
        d = 0.05 * (rng.normal(size=ob.P) + 1j * rng.normal(size=ob.P))
        tg.append(np.append(ob.target_params[:-1] + d, 1.0))
    return pb, ob, np.array(tg)


def run_gpu(pb, ob, targets, precision, polish=0, p2c="oracle", start=None, **kw):
    n_hyp = len(targets)
    start = ob.start_params if start is None else start
    rt = torch.float32 if precision == ghc.PREC_FP32 else torch.float64
    ws = ghc.Workspace(pb, n_hyp, precision)
    ss = cx_t(ob.start_sols, rt)
    if pb.kind == ghc.KIND_P2C:
        if p2c == "device":
            dhx, dht = pb.p2c_device(cx_t(start), cx_t(targets))
            hx, ht = to_cx(dhx), to_cx(dht)[:, : (pb.M + 1) * pb.K]
        else:
            hx = np.array([O.p2c_tables(ob.terms, start, t)[0] for t in targets])
            ht = np.array([O.p2c_tables(ob.terms, start, t)[1] for t in targets])
            dhx, dht = cx_t(hx), cx_t(ht)
        ghc.track(pb, ws, ss, d_coef_hx=dhx, d_coef_ht=dht, polish_iters=polish, **kw)
        oargs = dict(hx=hx, ht=ht)
    else:
        ps = cx_t(start)
        pt = cx_t(targets)
        if precision == ghc.PREC_FP32:
            # the FP32 oracle subtracts in float: hand the kernel the same rounded difference
            pd = cx_t(targets.astype(np.complex64) - start.astype(np.complex64)[None, :])
        else:
            pd = cx_t(targets - start[None, :])
        ghc.track(pb, ws, ss, d_p_start=ps, d_p_target=pt, d_p_diff=pd, polish_iters=polish, **kw)
        oargs = dict(p_start=start, p_target=targets)
    torch.cuda.synchronize()
    return ws, oargs


def compare(ws, r, exact=True):
    ep = to_cx(ws.endpoints)
    assert np.array_equal(ws.conv.cpu().numpy(), r["conv"])
    assert np.array_equal(ws.inf.cpu().numpy(), r["inf"])
    assert np.array_equal(ws.status.cpu().numpy(), r["status"])
    assert np.array_equal(ws.steps.cpu().numpy(), r["steps"])
    assert np.array_equal(ws.corr.cpu().numpy(), r["corr"])
    assert np.array_equal(ws.t_end.cpu().numpy(), r["t_end"])
    fin = np.isfinite(r["endpoints"])
    assert np.array_equal(np.isfinite(ep), fin)
    assert np.array_equal(ep[fin], r["endpoints"][fin])


@pytest.mark.parametrize("name", SUPPORTED)
def test_fp64_bit_exact_vs_oracle(name):
    pb, ob, tg = inputs(name)
    ws, oargs = run_gpu(pb, ob, tg, ghc.PREC_FP64, polish=2)
    r = O.track(ob, ob.start_sols, polish_iters=2, nthreads=NCPU, **oargs)
    compare(ws, r)
    res = ws.resid.cpu().numpy()
    conv = r["conv"] == 1
    assert np.array_equal(res[conv], r["resid"][conv])
    assert ghc.count_results(to_cx(ws.endpoints), ws.conv.cpu().numpy(), ws.inf.cpu().numpy()) == \
        O.count_results(r["endpoints"], r["conv"], r["inf"])


@pytest.mark.parametrize("name", ["P3P", "generalized_3views_4pts", "uncalibrated_trifocal_rel_pos_CY",
                                  "trifocal_2op1p_30x30", "5pt_rel_pos_alg_form_quat", "generalized_3views_6lines",
                                  "uncalibrated_trifocal_rel_pos_CH", "optimal_PnP_quat"])
def test_fp32_bit_exact_vs_oracle(name):
    pb, ob, tg = inputs(name)
    ws, oargs = run_gpu(pb, ob, tg, ghc.PREC_FP32)
    oargs = {k: (v.astype(np.complex64) if isinstance(v, np.ndarray) else v) for k, v in oargs.items()}
    r = O.track(ob, ob.start_sols.astype(np.complex64), precision="f", nthreads=NCPU, **oargs)
    compare(ws, r)


SYNTH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "problems")


@pytest.mark.parametrize("N", [4, 11, 16, 18])
@pytest.mark.parametrize("prec", [ghc.PREC_FP64, ghc.PREC_FP32, ghc.PREC_MIXED])
def test_synthetic_sizes_bit_exact(N, prec):
    """The sizes no shipped problem has (coupled quadratics generated by gen/make_quadratic_td.py):
    every compiled P2C size runs and matches the oracle bit for bit, with both H_x walks."""
    name = "QTD_%d" % N
    pb, ob = ghc.Problem(name, root=SYNTH), O.Problem(name, root=SYNTH)
    rng = np.random.default_rng(N)
    tg = np.array([ob.target_params, np.append(ob.target_params[:-1] + 0.1 * rng.normal(size=ob.P), 1.0)])
    hx = np.array([O.p2c_tables(ob.terms, ob.start_params, t)[0] for t in tg])
    ht = np.array([O.p2c_tables(ob.terms, ob.start_params, t)[1] for t in tg])
    rt = torch.float32 if prec == ghc.PREC_FP32 else torch.float64
    if prec == ghc.PREC_FP32:
        r = O.track(ob, ob.start_sols.astype(np.complex64), hx=hx.astype(np.complex64), ht=ht.astype(np.complex64),
                    precision="f", nthreads=NCPU)
    else:
        r = O.track(ob, ob.start_sols, hx=hx, ht=ht, precision="mixed" if prec == ghc.PREC_MIXED else "d",
                    t_switch=0.9, nthreads=NCPU)
    for flat in ([1] if N > 16 else [0, 1]):
        ghc.set_tuning(pb, prec, 0, flat)
        ws = ghc.Workspace(pb, 2, prec)
        ghc.track(pb, ws, cx_t(ob.start_sols, rt), d_coef_hx=cx_t(hx), d_coef_ht=cx_t(ht), t_switch=0.9)
        torch.cuda.synchronize()
        compare(ws, r)
    assert r["conv"].mean() > 0.9


@pytest.mark.parametrize("name,robust,t_switch", [("P3P", False, 0.9), ("generalized_3views_4pts", False, 0.9),
                                                  ("generalized_3views_4pts", True, 0.5),
                                                  ("uncalibrated_trifocal_rel_pos_CY", False, 0.9),
                                                  ("5pt_rel_pos_alg_form_quat", False, 0.7),
                                                  ("trifocal_2op1p_30x30", False, 0.9)])
def test_mixed_bit_exact_vs_oracle(name, robust, t_switch):
    """Both phases, the handover state and the FP64 resume match the oracle bit for bit."""
    pb, ob, tg = inputs(name, n_hyp=2, seed=3)
    kw = ROBUST if robust else {}
    ws, oargs = run_gpu(pb, ob, tg, ghc.PREC_MIXED, polish=2, t_switch=t_switch, **kw)
    r = O.track(ob, ob.start_sols, precision="mixed", t_switch=t_switch, polish_iters=2, nthreads=NCPU,
                **oargs, **kw)
    compare(ws, r)
    conv = r["conv"] == 1
    assert np.array_equal(ws.resid.cpu().numpy()[conv], r["resid"][conv])


def test_mixed_handover_happens():
    """The mixed phase stops every path by t_switch, and the FP64 phase carries its step
    counts on (a path's steps are those of both phases, under one step cap)."""
    pb, ob, tg = inputs("generalized_3views_4pts")
    ws, oargs = run_gpu(pb, ob, tg, ghc.PREC_MIXED, t_switch=0.5, max_steps=6)
    r_mixed = O.track(ob, ob.start_sols, precision="mixed", t_switch=0.5, max_steps=6, nthreads=NCPU, **oargs)
    compare(ws, r_mixed)
    first = O._track(ob, ob.start_sols, precision="m", max_steps=6,
                     handover=(0.5, O.MIXED_FAIL_LIMIT, O.MIXED_COND_LIMIT, O.MIXED_DT_FLOOR), **oargs)
    assert (first["t_end"] <= 0.5 + 1e-6).all()
    assert (ws.steps.cpu().numpy() >= first["steps"]).all()


@pytest.mark.parametrize("name,cond_limit,dt_floor", [("generalized_3views_4pts", 1e3, 1e-4),
                                                      ("generalized_3views_4pts", 1e5, 1e-4),
                                                      ("generalized_3views_4pts", 1e7, 1e-3),
                                                      ("uncalibrated_trifocal_rel_pos_CY", 1e5, 1e-4),
                                                      ("trifocal_2op1p_30x30", 1e5, 1e-4)])
def test_mixed_conditioning_handover_bit_exact(name, cond_limit, dt_floor):
    """The mixed tracker to t = 1 under the path-jump-free control, handing a path to FP64 after a
    step whose FP32 solve had a pivot-magnitude span above cond_limit or once its step falls below
    dt_floor: both phases equal the oracle's bit for bit, and some paths do take the FP64 phase."""
    pb, ob, tg = inputs(name, n_hyp=2, seed=7)
    ws, oargs = run_gpu(pb, ob, tg, ghc.PREC_MIXED, polish=2, cond_limit=cond_limit, dt_floor=dt_floor, **ROBUST)
    r = O.track(ob, ob.start_sols, precision="mixed", polish_iters=2, nthreads=NCPU, cond_limit=cond_limit,
                dt_floor=dt_floor, step=O.ROBUST_STEP, max_corr=3, max_steps=2000, **oargs)
    compare(ws, r)
    first = O._track(ob, ob.start_sols, precision="m", handover=(0.0, O.MIXED_FAIL_LIMIT, cond_limit, dt_floor),
                     step=O.ROBUST_STEP, max_corr=3, max_steps=2000, nthreads=NCPU, **oargs)
    assert 0 < (first["conv"] == 0).sum() < first["conv"].size


@pytest.mark.parametrize("name", ["P3P", "generalized_3views_4pts", "uncalibrated_trifocal_rel_pos_CY"])
def test_batched_hypotheses_equal_single_runs(name):
    pb, ob, tg = inputs(name, n_hyp=3, seed=5)
    ws, oargs = run_gpu(pb, ob, tg, ghc.PREC_FP64)
    r = O.track(ob, ob.start_sols, nthreads=NCPU, **oargs)
    compare(ws, r)
    # hypothesis 2 alone gives the same results as inside the batch
    ws1, _ = run_gpu(pb, ob, tg[2:3], ghc.PREC_FP64)
    n = pb.paths
    assert np.array_equal(to_cx(ws1.endpoints), to_cx(ws.endpoints)[2 * n:3 * n])
    assert np.array_equal(ws1.steps.cpu().numpy(), ws.steps.cpu().numpy()[2 * n:3 * n])


ROBUST = dict(step=ghc.ROBUST_STEP, max_corr=3, max_steps=2000)


@pytest.mark.parametrize("name", ["generalized_3views_4pts", "uncalibrated_trifocal_rel_pos_CY", "trifocal_2op1p_30x30"])
def test_fp64_robust_step_bit_exact_vs_oracle(name):
    pb, ob, tg = inputs(name)
    ws, oargs = run_gpu(pb, ob, tg, ghc.PREC_FP64, polish=2, **ROBUST)
    r = O.track(ob, ob.start_sols, polish_iters=2, nthreads=NCPU, step=O.ROBUST_STEP, max_corr=3, max_steps=2000,
                **oargs)
    compare(ws, r)


def real_targets(ob, n_hyp, seed):
    """real perturbations of the shipped target: real instances have real solutions"""
    rng = np.random.default_rng(seed)
    base = ob.target_params[:-1].real
    return np.array([np.append(base + 0.05 * rng.normal(size=ob.P), 1.0) for _ in range(n_hyp)])


@pytest.mark.parametrize("name", ["generalized_3views_4pts", "5pt_rel_pos_alg_form_quat",
                                  "uncalibrated_trifocal_rel_pos_CY"])
def test_mixed_precision_recall(name):
    """The mixed tracker (FP32 linear algebra, FP64 residual) to t = 1, FP64 for the paths it hands
    over, both runs with path-jump-free step control:
    >= 99.5% of the FP64 run's real endpoints are found by the mixed run within 1e-8
    (8 hypotheses: several hundred real endpoints, so that the bar admits a miss)."""
    pb, ob = ghc.Problem(name), O.Problem(name)
    tg = real_targets(ob, 8, 9)
    w64, _ = run_gpu(pb, ob, tg, ghc.PREC_FP64, polish=3, **ROBUST)
    wmx, _ = run_gpu(pb, ob, tg, ghc.PREC_MIXED, polish=3, **ROBUST)
    e64, emx = to_cx(w64.endpoints), to_cx(wmx.endpoints)
    c64, cmx = w64.conv.cpu().numpy() == 1, wmx.conv.cpu().numpy() == 1
    r64 = w64.resid.cpu().numpy()
    real64 = c64 & (np.abs(e64.imag).max(axis=1) <= 1e-8) & (r64 < 1e-10)
    found = 0
    n = pb.paths
    for i in np.nonzero(real64)[0]:
        h = i // n
        cand = emx[h * n:(h + 1) * n][cmx[h * n:(h + 1) * n]]
        err = np.abs(cand - e64[i]).max(axis=1) / max(1.0, np.abs(e64[i]).max())
        found += bool(err.size and err.min() <= 1e-8)
    assert real64.sum() > 0
    assert found >= 0.995 * real64.sum(), (found, real64.sum())
    rmx = wmx.resid.cpu().numpy()[cmx]
    assert np.median(rmx) < 1e-10


@pytest.mark.parametrize("name,step", [("generalized_3views_4pts", "reference"), ("generalized_3views_4pts", "robust"),
                                       ("uncalibrated_trifocal_rel_pos_CY", "reference"),
                                       ("uncalibrated_trifocal_rel_pos_CY", "robust"), ("P3P_TD", "reference"),
                                       ("trifocal_2op1p_30x30", "reference")])
def test_scene_targets_bit_exact_vs_oracle(name, step):
    """The seeded scene generators the benchmarks draw from (scenes.py: generalized 3-view 4-point
    scenes with 0.5 px noise, uncalibrated trifocal scenes with 30 % outliers, P3P by total degree,
    trifocal 30x30 from points and tangents): the FP64 tracker equals the oracle bit for bit on
    those targets, polished endpoints and residuals included, under both step controls."""
    import scenes
    pb, ob = ghc.Problem(name), O.Problem(name)
    st, tg, _ = scenes.targets_for(name, 3, 17, ob.start_params, ob.target_params)
    kw = ROBUST if step == "robust" else {}
    okw = dict(step=O.ROBUST_STEP, max_corr=3, max_steps=2000) if step == "robust" else {}
    ws, oargs = run_gpu(pb, ob, tg, ghc.PREC_FP64, polish=3, start=st, **kw)
    r = O.track(ob, ob.start_sols, polish_iters=3, nthreads=NCPU, **oargs, **okw)
    compare(ws, r)
    conv = r["conv"] == 1
    assert conv.mean() > 0.5
    assert np.array_equal(ws.resid.cpu().numpy()[conv], r["resid"][conv])


def test_path_status_singular_and_nonfinite():
    """Per-path status beyond converged / diverged / step cap: a path started where H_x is singular
    (x = 0 of the total-degree start system x_i^2 - 1, so every solve has a zero pivot) ends at the
    step cap with its last solve singular, a path started at NaN ends non-finite; the others
    converge.  Equal to the oracle's statuses."""
    pb, ob, tg = inputs("P3P_TD")
    starts = np.array(ob.start_sols)
    starts[0] = 0.0
    starts[1] = np.nan
    hx = np.array([O.p2c_tables(ob.terms, ob.start_params, t)[0] for t in tg])
    ht = np.array([O.p2c_tables(ob.terms, ob.start_params, t)[1] for t in tg])
    ws = ghc.Workspace(pb, 1, ghc.PREC_FP64)
    ghc.track(pb, ws, cx_t(starts), d_coef_hx=cx_t(hx), d_coef_ht=cx_t(ht), max_steps=40)
    torch.cuda.synchronize()
    r = O.track(ob, starts, hx=hx, ht=ht, nthreads=NCPU, max_steps=40)
    st = ws.status.cpu().numpy()
    assert np.array_equal(st, r["status"])
    assert st[0] == ghc.STATUS_SINGULAR and st[1] == ghc.STATUS_NONFINITE
    assert (st[2:] == ghc.STATUS_CONVERGED).all()


def test_step_cap_and_short_corrector():
    pb, ob, tg = inputs("generalized_3views_4pts")
    ws, oargs = run_gpu(pb, ob, tg, ghc.PREC_FP64, max_steps=5, max_corr=2)
    r = O.track(ob, ob.start_sols, nthreads=NCPU, max_steps=5, max_corr=2, **oargs)
    compare(ws, r)
    assert (ws.status.cpu().numpy() == ghc.STATUS_STEP_CAP).any()


def test_device_p2c_matches_host():
    pb, ob, tg = inputs("generalized_3views_4pts", n_hyp=4, seed=3)
    hx, ht = pb.p2c_device(cx_t(ob.start_params), cx_t(tg))
    torch.cuda.synchronize()
    for h in range(4):
        rhx, rht = pb.p2c(ob.start_params, tg[h])
        assert np.allclose(to_cx(hx[h]), rhx, rtol=1e-14, atol=1e-13 * np.abs(rhx).max())
        assert np.allclose(to_cx(ht[h])[: len(rht)], rht, rtol=1e-14, atol=1e-13 * np.abs(rht).max())


def test_empty_batch_is_a_noop():
    pb, ob, tg = inputs("P3P")
    ws = ghc.Workspace(pb, 0, ghc.PREC_FP64)
    hx = torch.zeros((0, (pb.M + 1) * (pb.K + 1), 2), dtype=torch.float64, device="cuda")
    ghc.track(pb, ws, cx_t(ob.start_sols), d_coef_hx=hx, d_coef_ht=hx)
    torch.cuda.synchronize()


@pytest.mark.parametrize("name,prec", [("generalized_3views_4pts", ghc.PREC_FP64), ("P3P", ghc.PREC_FP32),
                                       ("trifocal_2op1p_30x30", ghc.PREC_FP64)])
def test_solve_host_end_to_end(name, prec):
    pb, ob, tg = inputs(name)
    out = ghc.solve_host(pb, prec)
    ws, oargs = run_gpu(pb, ob, tg, prec, p2c="device")
    assert np.array_equal(out["conv"], ws.conv.cpu().numpy())
    assert np.array_equal(out["endpoints"], to_cx(ws.endpoints))


def test_solve_host_arena_and_reused_outputs():
    """Calls of different sizes on one handle (the device arena grows, then is reused) give the
    same results as fresh calls, also when the output arrays are reused."""
    pb, ob, tg = inputs("generalized_3views_4pts", n_hyp=5, seed=21)
    small1 = ghc.solve_host(pb, ghc.PREC_FP64, targets=tg[:2])
    large = ghc.solve_host(pb, ghc.PREC_FP64, targets=tg)
    out = ghc.solve_outputs(pb, 2)
    small2 = ghc.solve_host(pb, ghc.PREC_FP64, targets=tg[:2], out=out)
    small3 = ghc.solve_host(pb, ghc.PREC_FP64, targets=tg[:2], out=out)
    assert small3 is out
    n = 2 * pb.paths
    for k in ("endpoints", "conv", "status", "steps"):
        assert np.array_equal(small1[k], small3[k]) and np.array_equal(large[k][:n], small1[k])
    with pytest.raises(ghc.GhcError):
        ghc.solve_host(pb, ghc.PREC_FP64, targets=tg, out=out)


@pytest.mark.parametrize("name,prec", [("P3P", "f"), ("uncalibrated_trifocal_rel_pos_CY", "f"),
                                       ("generalized_3views_4pts", "d"), ("trifocal_2op1p_30x30", "f"),
                                       ("trifocal_2op1p_30x30", "d")])
def test_dropin_reference_abi(name, prec):
    """kernel_HC_Solver_<p>-style call: pointer arrays, reference layout [N+1], bool flags, debug (t, dt)."""
    import ctypes
    pb, ob, tg = inputs(name)
    rt = torch.float32 if prec == "f" else torch.float64
    N, n = pb.N, pb.paths
    sols = np.concatenate([ob.start_sols, np.ones((n, 1))], axis=1)
    d_start = cx_t(sols, rt)
    d_track = cx_t(sols, rt)
    esz = 2 * (4 if prec == "f" else 8)
    p_start = torch.tensor([d_start.data_ptr() + i * (N + 1) * esz for i in range(n)], dtype=torch.int64).cuda()
    p_track = torch.tensor([d_track.data_ptr() + i * (N + 1) * esz for i in range(n)], dtype=torch.int64).cuda()
    hxr, htr = ob.hx_idx, ob.ht_idx
    d_hxi = torch.from_numpy(hxr).cuda()
    d_hti = torch.from_numpy(htr).cuda()
    conv = torch.zeros(n, dtype=torch.uint8, device="cuda")
    inf = torch.zeros(n, dtype=torch.uint8, device="cuda")
    dbg = torch.zeros((n, 2), dtype=rt, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    if pb.kind == ghc.KIND_P2C:
        hx, ht = O.p2c_tables(ob.terms, ob.start_params, ob.target_params)
        fn = ghc.ghc_kernel_HC_Solver_P2C if prec == "f" else ghc.ghc_kernel_HC_Solver_P2C_z
        keep = [cx_t(hx, rt), cx_t(ht, rt)]  # hold the tables alive across the call
        sec = fn(pb.h, st, pb.max_steps, pb.max_corr, pb.incr_steps, p_start.data_ptr(), p_track.data_ptr(),
                 d_hxi.data_ptr(), d_hti.data_ptr(), keep[0].data_ptr(), keep[1].data_ptr(),
                 conv.data_ptr(), inf.data_ptr(), dbg.data_ptr())
        oargs = dict(hx=hx, ht=ht)
    else:
        fn = ghc.ghc_kernel_HC_Solver_PH if prec == "f" else ghc.ghc_kernel_HC_Solver_PH_z
        ps, pt = ob.start_params, ob.target_params
        if prec == "f":  # the FP32 oracle subtracts in float
            pd = pt.astype(np.complex64) - ps.astype(np.complex64)
        else:
            pd = pt - ps
        keep = [cx_t(ps, rt), cx_t(pt, rt), cx_t(pd, rt)]
        sec = fn(pb.h, st, pb.max_steps, pb.max_corr, pb.incr_steps, p_start.data_ptr(), p_track.data_ptr(),
                 keep[0].data_ptr(), keep[1].data_ptr(), keep[2].data_ptr(), d_hxi.data_ptr(), d_hti.data_ptr(),
                 conv.data_ptr(), inf.data_ptr(), dbg.data_ptr())
        oargs = dict(p_start=ps, p_target=pt[None, :])
    assert sec >= 0, ghc.ghc_last_error()
    if prec == "f":
        oargs = {k: (v.astype(np.complex64) if isinstance(v, np.ndarray) else v) for k, v in oargs.items()}
    r = O.track(ob, ob.start_sols.astype(np.complex64 if prec == "f" else np.complex128), precision=prec,
                nthreads=NCPU, **oargs)
    ep = to_cx(d_track)[:, :N]
    assert np.array_equal(conv.cpu().numpy(), r["conv"])
    assert np.array_equal(inf.cpu().numpy(), r["inf"])
    fin = np.isfinite(r["endpoints"])
    assert np.array_equal(ep[fin], r["endpoints"][fin])
    d = to_cx(dbg)
    c = r["conv"] == 1
    assert np.all(d[c] == 1)
    assert np.allclose(d[~c].real, r["t_end"][~c]) and np.allclose(d[~c].imag, r["dt_end"][~c])


@pytest.mark.parametrize("name,precision", [("P3P", ghc.PREC_FP64), ("P3P", ghc.PREC_FP32),
                                            ("5pt_rel_pos_alg_form_quat", ghc.PREC_MIXED)])
def test_single_instance_spread_equals_batch(name, precision):
    """A launch with fewer paths than one warp per scheduler gives each path its own warp (spread);
    the same instance inside a large batch runs sub-warps side by side: both are bit-identical
    with each other, and the single one with the oracle."""
    pb, ob = ghc.Problem(name), O.Problem(name)
    tg = ob.target_params[None, :]
    one, oargs = run_gpu(pb, ob, tg, precision)
    assert pb.paths <= 148 * 4  # spread
    many, _ = run_gpu(pb, ob, np.repeat(tg, 100, axis=0), precision)
    assert 100 * pb.paths > 148 * 4  # packed sub-warps
    n = pb.paths
    assert np.array_equal(to_cx(one.endpoints), to_cx(many.endpoints)[:n], equal_nan=True)
    for f in ("conv", "inf", "status", "steps", "corr"):
        assert np.array_equal(getattr(one, f).cpu().numpy(), getattr(many, f).cpu().numpy()[:n])
    if precision == ghc.PREC_FP32:
        oargs = {k: (v.astype(np.complex64) if isinstance(v, np.ndarray) else v) for k, v in oargs.items()}
        r = O.track(ob, ob.start_sols.astype(np.complex64), precision="f", nthreads=NCPU, **oargs)
    elif precision == ghc.PREC_MIXED:
        r = O.track(ob, ob.start_sols, precision="mixed", nthreads=NCPU, **oargs)
    else:
        r = O.track(ob, ob.start_sols, nthreads=NCPU, **oargs)
    compare(one, r)


def test_dropin_caller_tables_differ_from_loaded():
    """A drop-in call handed index tables that differ from the problem folder's (here the terms of
    every H_x entry in reverse order: the same system, another summation order) tracks with those
    tables -- compiled once and kept in the handle, so a second call reuses them -- and equals the
    oracle reading the same tables; the handle's own tables serve a later call with the loaded ones."""
    pb, ob, tg = inputs("P3P")
    N, n = pb.N, pb.paths
    rev = np.ascontiguousarray(ob.hx_idx.reshape(N, N, ob.Tx, ob.Px)[:, :, ::-1, :].reshape(-1))
    hx, ht = O.p2c_tables(ob.terms, ob.start_params, ob.target_params)
    keep = [cx_t(hx), cx_t(ht)]
    st = torch.cuda.current_stream().cuda_stream
    sols = np.concatenate([ob.start_sols, np.ones((n, 1))], axis=1)

    def call(hx_idx):
        d_start, d_track = cx_t(sols), cx_t(sols)
        ps = torch.tensor([d_start.data_ptr() + i * (N + 1) * 16 for i in range(n)], dtype=torch.int64).cuda()
        pt = torch.tensor([d_track.data_ptr() + i * (N + 1) * 16 for i in range(n)], dtype=torch.int64).cuda()
        d_hxi, d_hti = torch.from_numpy(hx_idx).cuda(), torch.from_numpy(ob.ht_idx).cuda()
        conv = torch.zeros(n, dtype=torch.uint8, device="cuda")
        inf = torch.zeros(n, dtype=torch.uint8, device="cuda")
        sec = ghc.ghc_kernel_HC_Solver_P2C_z(pb.h, st, pb.max_steps, pb.max_corr, pb.incr_steps, ps.data_ptr(),
                                             pt.data_ptr(), d_hxi.data_ptr(), d_hti.data_ptr(), keep[0].data_ptr(),
                                             keep[1].data_ptr(), conv.data_ptr(), inf.data_ptr(), None)
        assert sec >= 0, ghc.ghc_last_error()
        return to_cx(d_track)[:, :N], conv.cpu().numpy()

    loaded = ob.hx_idx
    ob.hx_idx = rev
    r = O.track(ob, ob.start_sols, hx=hx, ht=ht, nthreads=NCPU)
    ob.hx_idx = loaded
    r0 = O.track(ob, ob.start_sols, hx=hx, ht=ht, nthreads=NCPU)
    for _ in range(2):
        ep, conv = call(rev)
        assert np.array_equal(conv, r["conv"]) and np.array_equal(ep, r["endpoints"])
    ep, conv = call(np.ascontiguousarray(loaded))
    assert np.array_equal(conv, r0["conv"]) and np.array_equal(ep, r0["endpoints"])
