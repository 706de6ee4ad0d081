"""Launch tuning (needs a B200): every compiled variant and H_x walk gives bit-identical
results, and ghc_autotune keeps one of them in the problem handle."""
import numpy as np
import pytest

import ghc
import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _cx_t(a, dtype=torch.float64):
    a = np.asarray(a, dtype=np.complex128)
    return torch.from_numpy(np.ascontiguousarray(np.stack([a.real, a.imag], -1))).to(dtype).cuda()


def _inputs(name, H=3):
    pb, ob = ghc.Problem(name), O.Problem(name)
    rng = np.random.default_rng(4)
    tg = np.array([np.append(ob.target_params[:-1] + 0.05 * (rng.normal(size=ob.P) + 1j * rng.normal(size=ob.P)), 1.0)
                   for _ in range(H)])
    return pb, ob, tg


def _run(pb, ob, tg, prec, tune=None):
    rt = torch.float32 if prec == ghc.PREC_FP32 else torch.float64
    ws = ghc.Workspace(pb, len(tg), prec)
    ss = _cx_t(ob.start_sols, rt)
    if pb.kind == ghc.KIND_P2C:
        hx, ht = pb.p2c_device(_cx_t(ob.start_params), _cx_t(tg))
        kw = dict(d_coef_hx=hx, d_coef_ht=ht)
    else:
        kw = dict(d_p_start=_cx_t(ob.start_params), d_p_target=_cx_t(tg), d_p_diff=_cx_t(tg - ob.start_params[None]))
    if tune == "auto":
        choice = ghc.autotune(pb, ws, ss, **kw)
    else:
        choice = None
        if tune is not None:
            ghc.set_tuning(pb, prec, *tune)
        ghc.track(pb, ws, ss, **kw)
    torch.cuda.synchronize()
    return ws, choice


@pytest.mark.parametrize("name", ["P3P", "generalized_3views_4pts", "5pt_rel_pos_alg_form_quat",
                                  "trifocal_2op1p_30x30"])
@pytest.mark.parametrize("prec", [ghc.PREC_FP64, ghc.PREC_FP32, ghc.PREC_MIXED])
def test_every_choice_is_bit_identical(name, prec):
    pb, ob, tg = _inputs(name)
    base, _ = _run(pb, ob, tg, prec, (0, -1))
    for tune in [(0, 0), (0, 1), (0, 2), (1, 0), (1, 1), (1, 2)]:
        ws, _ = _run(pb, ob, tg, prec, tune)
        for f in ("endpoints", "conv", "inf", "status", "steps", "corr", "t_end"):
            assert torch.equal(getattr(ws, f), getattr(base, f)), (tune, f)


def test_autotune_keeps_a_candidate():
    pb, ob, tg = _inputs("generalized_3views_4pts", H=8)
    ref, _ = _run(pb, ob, tg, ghc.PREC_FP64, (0, -1))
    ws, choice = _run(pb, ob, tg, ghc.PREC_FP64, "auto")
    assert choice["candidates"] == 6 and choice["ms"] > 0  # 2 register budgets x 3 H_x walks
    assert ghc.get_tuning(pb, ghc.PREC_FP64) == (choice["variant"], choice["flat"])
    assert torch.equal(ws.endpoints, ref.endpoints)  # the sample's outputs are a regular run's
    again, _ = _run(pb, ob, tg, ghc.PREC_FP64)
    assert torch.equal(again.endpoints, ref.endpoints)


def test_mixed_autotune_chooses_each_phase():
    """Mixed precision tunes the FP64 and FP32 phases' variants independently (2 x 2 x 3 walks at N = 12)."""
    pb, ob, tg = _inputs("generalized_3views_4pts", H=8)
    ref, _ = _run(pb, ob, tg, ghc.PREC_MIXED, (0, -1))
    ws, choice = _run(pb, ob, tg, ghc.PREC_MIXED, "auto")
    assert choice["candidates"] == 12
    assert ghc.get_tuning(pb, ghc.PREC_FP64) == (choice["variant"], choice["flat"])
    assert ghc.get_tuning(pb, ghc.PREC_FP32) == (choice["variant_f32"], choice["flat"])
    assert torch.equal(ws.endpoints, ref.endpoints)
