"""Serving loop (needs a B200): every request's result is the same alone and in the mix.

Requests of two problems arrive as a Poisson stream and are packed into
shared launches by serve.Server; each request is then tracked alone with
ghc.track on the same targets.  Per-hypothesis arithmetic does not depend on
the batch, so endpoints and flags must be identical (the same bit-for-bit bar
as the other FP64 parity tests).  The monodromy solver is checked here too.
"""
import numpy as np
import pytest

import ghc
import serve

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def cx_t(a):
    a = np.asarray(a, dtype=np.complex128)
    return torch.from_numpy(np.ascontiguousarray(np.stack([a.real, a.imag], -1))).cuda()


def test_requests_same_alone_and_in_the_mix():
    server = serve.Server(torch, problems=["P3P_TD", "generalized_3views_4pts"], max_batch=512)
    lat, hyp, wall, reqs = serve.run_stream(server, lam=2000, n_req=12, seed=4)
    assert all(r.done is not None for r in reqs)
    assert server.launches < len(reqs)  # requests did share launches
    for r in reqs:
        prob = server.problems[r.problem]
        n = r.targets.shape[0]
        ws = ghc.Workspace(prob.pb, n, ghc.PREC_FP64)
        hx, ht = prob.pb.p2c_device(prob.d_start, cx_t(r.targets))
        ghc.track(prob.pb, ws, prob.d_sols, d_coef_hx=hx, d_coef_ht=ht)
        torch.cuda.synchronize()
        e = ws.endpoints.cpu().numpy()
        e = e[..., 0] + 1j * e[..., 1]
        assert np.array_equal(ws.conv.cpu().numpy(), r.conv)
        fin = np.isfinite(e)
        assert np.array_equal(e[fin], r.endpoints[fin])
        # per-hypothesis counts from the device equal the host rule on the returned endpoints
        P = prob.paths
        for h in range(n):
            c = ghc.count_results(r.endpoints[h * P:(h + 1) * P], r.conv[h * P:(h + 1) * P], r.inf[h * P:(h + 1) * P])
            assert [c["converged"], c["real"], c["infinity"], c["unique"]] == r.counts[h].tolist()


def test_mixed_server_and_tuning_keep_results():
    """A mixed-precision server gives each request what a mixed run alone gives; an
    autotuned server gives bit-identical results to an untuned one."""
    names = ["P3P_TD", "trifocal_2op1p_30x30"]
    mixed = serve.Server(torch, problems=names, max_batch=512, precision=ghc.PREC_MIXED, tune=True)
    _, _, _, reqs = serve.run_stream(mixed, lam=3000, n_req=6, seed=12)
    for r in reqs:
        prob = mixed.problems[r.problem]
        n = r.targets.shape[0]
        ws = ghc.Workspace(prob.pb, n, ghc.PREC_MIXED)
        if prob.pb.kind == ghc.KIND_P2C:
            hx, ht = prob.pb.p2c_device(prob.d_start, cx_t(r.targets))
            ghc.track(prob.pb, ws, prob.d_sols, d_coef_hx=hx, d_coef_ht=ht)
        else:
            tg = cx_t(r.targets)
            ghc.track(prob.pb, ws, prob.d_sols, d_p_start=prob.d_start, d_p_target=tg,
                      d_p_diff=tg - prob.d_start[None])
        torch.cuda.synchronize()
        e = ws.endpoints.cpu().numpy()
        e = e[..., 0] + 1j * e[..., 1]
        fin = np.isfinite(e)
        assert np.array_equal(ws.conv.cpu().numpy(), r.conv)
        assert np.array_equal(e[fin], r.endpoints[fin])
    tuned = serve.Server(torch, problems=["P3P_TD"], max_batch=512, tune=True)
    plain = serve.Server(torch, problems=["P3P_TD"], max_batch=512)
    assert tuned.problems["P3P_TD"].tuning["candidates"] == 6  # 2 register budgets x 3 H_x walks
    _, _, _, rt = serve.run_stream(tuned, lam=5000, n_req=5, seed=9)
    _, _, _, rp = serve.run_stream(plain, lam=5000, n_req=5, seed=9)
    for x, y in zip(rt, rp):
        assert np.array_equal(x.endpoints, y.endpoints) and np.array_equal(x.counts, y.counts)


def test_sequential_baseline_matches_batched():
    b = serve.Server(torch, problems=["P3P_TD"], max_batch=512)
    s = serve.Server(torch, problems=["P3P_TD"], sequential=True, max_batch=512)
    _, _, _, rb = serve.run_stream(b, lam=5000, n_req=6, seed=8)
    _, _, _, rs = serve.run_stream(s, lam=5000, n_req=6, seed=8)
    for x, y in zip(rb, rs):
        assert np.array_equal(x.endpoints, y.endpoints)


def test_monodromy_finds_all_p3p_solutions():
    import monodromy
    pb = ghc.Problem("P3P")
    q, Sq, S = monodromy.start_system(pb, seed=3)
    assert len(S) == 8 and len(Sq) == 8


def test_admission_waits_for_free_memory():
    """With the device reporting too little free memory, batches wait in the queue (in order) and
    start once memory frees up; results are those of an unconstrained server."""
    calls = {"n": 0}

    def scarce():
        calls["n"] += 1
        free, total = torch.cuda.mem_get_info()
        return (0 if 2 <= calls["n"] <= 40 else free), total  # the first call sizes the slots

    tight = serve.Server(torch, problems=["P3P_TD"], max_batch=512, mem_info=scarce)
    free = serve.Server(torch, problems=["P3P_TD"], max_batch=512)
    _, _, _, rt = serve.run_stream(tight, lam=5000, n_req=6, seed=21)
    _, _, _, rf = serve.run_stream(free, lam=5000, n_req=6, seed=21)
    assert tight.deferred > 0 and free.deferred == 0
    for x, y in zip(rt, rf):
        assert x.done is not None
        assert np.array_equal(x.endpoints, y.endpoints) and np.array_equal(x.counts, y.counts)
