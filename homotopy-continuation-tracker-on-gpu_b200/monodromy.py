"""Monodromy solver: all solutions of a parametric system at generic parameters.

Replaces, for this build's problems, HomotopyContinuation.jl's
monodromy_solve used by the reference to make its start systems
(start-sys-gen/*_monodromySolve.jl).  Starting from one solution x0 of
F(x; p0) = 0, the known solutions are tracked around triangles
p0 -> p1 -> p2 -> p0 of random complex parameter points; endpoints that are
new solutions of F(x; p0) are added, until the count reaches the expected
root count or stops growing.  Every leg is one batched launch of the GPU
tracker (P2C tables built on the device for the leg's parameter pair), with
the path-jump-free step control and FP64 polish.
"""
import numpy as np

import ghc

STEP = dict(corr_tol2=1e-12, first_tol2=1e-2, dt_max=0.05)
RESID_TOL = 1e-9    # |F(x; p)| after polish, relative to max(1, |x|)^2
MERGE_TOL = 1e-8    # two endpoints are the same solution within this relative max-norm distance


def _cx(a, torch):
    a = np.asarray(a, dtype=np.complex128)
    return torch.from_numpy(np.ascontiguousarray(np.stack([a.real, a.imag], -1))).cuda()


def track_leg(pb, starts, p_from, p_to, polish_iters=2, max_steps=4000):
    """Track solutions of F(.; p_from) to F(.; p_to); returns the converged, finite endpoints."""
    import torch
    starts = np.asarray(starts, dtype=np.complex128)
    if starts.shape[0] == 0:
        return starts
    ws = ghc.Workspace(pb, 1, ghc.PREC_FP64, paths=starts.shape[0])
    hx, ht = pb.p2c_device(_cx(p_from, torch), _cx(np.asarray(p_to)[None], torch))
    ghc.track(pb, ws, _cx(starts, torch), d_coef_hx=hx, d_coef_ht=ht, step=STEP, max_corr=3,
              max_steps=max_steps, polish_iters=polish_iters, want_resid=True)
    torch.cuda.synchronize()
    e = ws.endpoints.cpu().numpy()
    e = e[..., 0] + 1j * e[..., 1]
    res = ws.resid.cpu().numpy()
    scale = np.maximum(1.0, np.abs(e).max(axis=1)) ** 2
    ok = (ws.conv.cpu().numpy() == 1) & np.all(np.isfinite(e), axis=1) & (res >= 0) & (res <= RESID_TOL * scale)
    return e[ok]


def _merge(S, cand, tol=MERGE_TOL):
    """Append to S the candidates that are new (relative max-norm distance > tol)."""
    out = list(S)
    arr = np.array(out) if out else np.zeros((0, cand.shape[1] if cand.size else 0), dtype=complex)
    for x in cand:
        if arr.shape[0]:
            d = np.abs(arr - x).max(axis=1) / np.maximum(1.0, np.abs(x).max())
            if d.min() <= tol:
                continue
        out.append(x)
        arr = np.vstack([arr, x[None]]) if arr.shape[0] else x[None].copy()
    return np.array(out)


def monodromy_solve(pb, x0, p0, target=None, max_loops=200, stall_loops=8, seed=0, log=None):
    """All (discoverable) solutions of F(x; p0) from a seed solution x0 [N] (or a known set [n, N])."""
    if pb.kind != ghc.KIND_P2C:
        raise ValueError("monodromy needs a P2C problem (device coefficient tables)")
    rng = np.random.default_rng(seed)
    S = np.atleast_2d(np.asarray(x0, dtype=np.complex128))
    stall = 0
    for loop in range(max_loops):
        if target is not None and len(S) >= target:
            break
        if stall >= stall_loops:
            break
        p1 = np.append(rng.normal(size=pb.P) + 1j * rng.normal(size=pb.P), 1.0)
        p2 = np.append(rng.normal(size=pb.P) + 1j * rng.normal(size=pb.P), 1.0)
        X = track_leg(pb, S, p0, p1)
        X = track_leg(pb, X, p1, p2)
        X = track_leg(pb, X, p2, p0, polish_iters=3)
        n_before = len(S)
        S = _merge(S, X)
        stall = 0 if len(S) > n_before else stall + 1
        if log:
            log("loop %d: %d solutions" % (loop, len(S)))
    return S


def start_system(pb, seed=0, target=None, log=None):
    """Start parameters q ~ complex N(0,1) (seeded) and all solutions there.

    A complexified seed pair is solved by monodromy and the solution set is
    then moved to q by one parameter-homotopy leg; solutions lost on that leg
    are recovered by monodromy loops at q from the moved set.
    """
    import scenes
    x0, p_seed = scenes.seed_pair(pb.name, seed=seed)
    S = monodromy_solve(pb, x0, p_seed, target=target, seed=seed, log=log)
    rng = np.random.default_rng(10_000 + seed)
    q = np.append(rng.normal(size=pb.P) + 1j * rng.normal(size=pb.P), 1.0)
    Sq = _merge(np.zeros((0, pb.N), dtype=complex), track_leg(pb, S, p_seed, q, polish_iters=3))
    if 0 < len(Sq) < len(S):
        Sq = monodromy_solve(pb, Sq, q, target=len(S), stall_loops=4, seed=seed + 1, log=log)
    return q, Sq, S
