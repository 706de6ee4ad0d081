"""ghc_track_mix (needs a B200): batches of the four size buckets of the uneven-mix workload in one
persistent launch must give, path for path, the results of ghc_track launches of the buckets one
by one (every path is tracked with the same arithmetic; only the CTA that takes it differs)."""
import numpy as np
import pytest

import ghc
import scenes

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

MIX = [("P3P_TD", 64), ("5pt_rel_pos_alg_form_quat", 32), ("generalized_3views_4pts", 8), ("trifocal_2op1p_30x30", 4)]


def cx_t(a):
    a = np.asarray(a, dtype=np.complex128)
    return torch.from_numpy(np.ascontiguousarray(np.stack([a.real, a.imag], -1))).cuda()


def bucket(name, H, seed):
    pb = ghc.Problem(name)
    s, t = pb.params()
    st, tg, _ = scenes.targets_for(name, H, seed, s, t)
    if pb.kind == ghc.KIND_P2C:
        hx, ht = pb.p2c_device(cx_t(st), cx_t(tg))
        kw = dict(d_coef_hx=hx, d_coef_ht=ht)
    else:
        kw = dict(d_p_start=cx_t(st), d_p_target=cx_t(tg), d_p_diff=cx_t(tg - st[None, :]))
    return pb, cx_t(pb.start_sols()), kw


def outputs(ws):
    return {k: getattr(ws, k).cpu().numpy().copy() for k in ("endpoints", "conv", "inf", "status", "steps", "corr",
                                                             "t_end")}


@pytest.mark.parametrize("which", [[0, 1, 2, 3], [2, 3], [0]])
def test_mix_equals_separate_launches(which):
    bs = [bucket(*MIX[i], seed=60 + i) for i in which]
    alone = []
    for pb, ss, kw in bs:
        ws = ghc.Workspace(pb, MIX[which[len(alone)]][1], ghc.PREC_FP64)
        ghc.track(pb, ws, ss, **kw)
        alone.append(ws)
    torch.cuda.synchronize()
    for rep in range(2):
        mixed = [ghc.Workspace(pb, MIX[i][1], ghc.PREC_FP64) for i, (pb, _, _) in zip(which, bs)]
        ghc.track_mix([(pb, ws, ss, kw) for (pb, ss, kw), ws in zip(bs, mixed)])
        torch.cuda.synchronize()
        for a, m in zip(alone, mixed):
            oa, om = outputs(a), outputs(m)
            for k in oa:
                assert np.array_equal(oa[k], om[k], equal_nan=oa[k].dtype.kind == "f"), (rep, k)


def test_mix_rejects_uncompiled_buckets():
    """A problem whose size and term shape have no compiled slot (N = 12 with (2,3) terms), or two
    problems for one slot, is refused before any launch."""
    pb, ss, kw = bucket("uncalibrated_trifocal_rel_pos_CY", 2, 1)
    ws = ghc.Workspace(pb, 2, ghc.PREC_FP64)
    with pytest.raises(ghc.GhcError):
        ghc.track_mix([(pb, ws, ss, kw)])
    a, sa, ka = bucket("P3P", 2, 1)
    b, sb, kb = bucket("P3P_TD", 2, 1)
    with pytest.raises(ghc.GhcError):
        ghc.track_mix([(a, ghc.Workspace(a, 2, ghc.PREC_FP64), sa, ka), (b, ghc.Workspace(b, 2, ghc.PREC_FP64), sb, kb)])
