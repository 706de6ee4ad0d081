"""Workloads of the scope beyond bench.py's headline (``bench.py --config ...``).

cy       batched: 4096 RANSAC hypotheses of the uncalibrated trifocal problem
         (12 unknowns, 668 paths; seeded 3-camera scenes, minimal samples with
         30 % outlier correspondences) -- device P2C + tracker + FP64 polish
         captured in one CUDA graph and replayed per step: plain FP64 with the
         reference's step control, then plain FP64 and the mixed tracker (FP32
         linear algebra, FP64 end game) under the path-jump-free control with
         the mixed run's recall of the FP64 run's real solutions.
p3p_td   P3P by a total-degree homotopy: one instance (latency, p50/p99) and
         a batch of 65536 instances (throughput), plain FP64.
mix      uneven mix in one persistent launch (ghc_track_mix): P3P_TD 8192,
         5-point 4096, generalized 3-view 2048, trifocal 30x30 1024 hypotheses,
         beside the same four launches forked on four streams of one graph and
         each bucket alone.
served   Poisson request stream through serve.Server (continuous batching).
g3v4_mono  generalized 3-view with start parameters ~ complex N(0,1) and
         start solutions from the monodromy solver, plain FP64 vs mixed.
problem  any problem folder (--problem), --hyp hypotheses per launch, one
         precision (--precision) and step control (--step): the tracker alone.
latency  one instance per launch on each problem's shipped parameters (P3P,
         5-point, generalized 3-view, CY, 30x30), FP32 / FP64 / mixed, p50/p99
         ms beside the reference's published single-instance times.

Each prints one JSON line with the bench contract's keys.
"""
import json
import os
import statistics
import time

import numpy as np

import ghc
import scenes

UNIT = "hypotheses/s"


def _cx(a, torch, dt=None):
    a = np.asarray(a, dtype=np.complex128)
    t = torch.from_numpy(np.ascontiguousarray(np.stack([a.real, a.imag], -1)))
    return t.to(dt or torch.float64).cuda()


def _to_cx(t):
    a = t.double().cpu().numpy()
    return a[..., 0] + 1j * a[..., 1]


def _line(metric, value, args, config, **extra):
    d = {"metric": metric, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
         "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "complex128",
         "data": "synthetic (seeded scenes)", "config": config}
    d.update(extra)
    return d


class Batch:
    """One problem's batch: inputs on the device, a workspace, and the launch."""

    def __init__(self, torch, name, H, seed, precision=ghc.PREC_FP64, polish=0, step=None, start=None, sols=None,
                 scene=None, shipped=False):
        self.pb = ghc.Problem(name)
        s, t = self.pb.params()
        if shipped:  # the problem folder's own instance: its start and target parameters
            st, tg, truth = s, np.repeat(np.asarray(t)[None, :], H, axis=0), None
        else:
            st, tg, truth = scenes.targets_for(name, H, seed, s, t, **(scene or {}))
        if start is not None:
            st = start
        self.name, self.H, self.truth, self.targets = name, H, truth, tg
        self.d_start = _cx(st, torch)
        self.d_tg = _cx(tg, torch)
        self.d_diff = _cx(tg - np.asarray(st)[None, :], torch)
        s0 = self.pb.start_sols() if sols is None else sols
        self.paths = s0.shape[0]
        self.d_sols = _cx(s0, torch, torch.float32 if precision == ghc.PREC_FP32 else None)
        self.ws = ghc.Workspace(self.pb, H, precision, paths=self.paths)
        self.kw = dict(polish_iters=polish, want_resid=polish > 0)
        if step:
            self.kw.update(step)

    def _inputs(self):
        if self.pb.kind == ghc.KIND_P2C:
            hx, ht = self.pb.p2c_device(self.d_start, self.d_tg)
            return dict(d_coef_hx=hx, d_coef_ht=ht)
        return dict(d_p_start=self.d_start, d_p_target=self.d_tg, d_p_diff=self.d_diff)

    def launch(self):
        ghc.track(self.pb, self.ws, self.d_sols, **self._inputs(), **self.kw)

    def tune(self):
        """Autotune the launch on this batch (before any capture); returns the choice."""
        self.tuning = ghc.autotune(self.pb, self.ws, self.d_sols, **self._inputs(), **self.kw)
        return self.tuning


def _time_graph(torch, g, steps, flush):
    ms = []
    for _ in range(steps):
        flush.fill_(1.0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        g.replay()
        e1.record()
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    return ms


def _capture(torch, fn):
    fn()  # warm-up outside capture: uploads problem tables, sets kernel attributes
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        fn()
    torch.cuda.synchronize()
    return g


def config_cy(args, torch, robust_hyp=None):
    H = args.hyp if args.hyp != 1024 else 4096
    HR = min(H, robust_hyp or H)
    # Inlier correspondences are exact (no pixel noise), so an all-inlier hypothesis has the
    # scene's unknowns as an exact solution and the known answer can be checked at 1e-6.  With
    # 0.5 px noise this minimal problem is so ill-conditioned (focal length from 4 points) that
    # the nearest solution moves 10-40 % away from the noise-free scene.
    b = Batch(torch, "uncalibrated_trifocal_rel_pos_CY", H, 1000 + args.seed, polish=2, scene={"noise_px": 0.0})
    _, _, inlier = scenes.uncalibrated_trifocal_rel_pos_CY(H, seed=1000 + args.seed, noise_px=0.0)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    tuning = b.tune() if args.tune else None
    g = _capture(torch, b.launch)
    for _ in range(args.warmup):
        g.replay()
    torch.cuda.synchronize()
    ms = _time_graph(torch, g, args.steps, flush)
    ep = _to_cx(b.ws.endpoints).reshape(H, b.paths, -1)
    conv = b.ws.conv.cpu().numpy().reshape(H, b.paths) == 1
    found = 0
    for h in np.nonzero(inlier)[0]:
        E = ep[h][conv[h]]
        best = 9.0
        for s2 in (1, -1):
            for s3 in (1, -1):
                gt = b.truth[h].copy()
                gt[4:8] *= s2
                gt[8:12] *= s3
                if E.size:
                    best = min(best, (np.abs(E - gt).max(axis=1) / np.abs(gt).max()).min())
        found += best < 1e-6
    steps = b.ws.steps.cpu().numpy()
    total = sum(ms)
    # the same hypotheses under the path-jump-free control: plain FP64 and the mixed tracker
    robust = dict(step=ghc.ROBUST_STEP, max_corr=3, max_steps=2000)
    runs = {}
    for name, prec in (("fp64", ghc.PREC_FP64), ("mixed", ghc.PREC_MIXED)):
        r = Batch(torch, "uncalibrated_trifocal_rel_pos_CY", HR, 1000 + args.seed, precision=prec, polish=3,
                  step=robust, scene={"noise_px": 0.0})
        r_tuning = r.tune() if args.tune else None
        gr = _capture(torch, r.launch)
        for _ in range(args.warmup):
            gr.replay()
        rms = _time_graph(torch, gr, args.steps, flush)
        runs[name] = dict(value=HR * len(rms) / (sum(rms) * 1e-3), ms=sum(rms) / len(rms), e=_to_cx(r.ws.endpoints),
                          c=r.ws.conv.cpu().numpy(), r=r.ws.resid.cpu().numpy(), tuning=r_tuning,
                          steps=float(r.ws.steps.float().mean()))
    rec, n_real, err = recall_and_error(runs["fp64"], runs["mixed"], b.paths)
    robust_line = {k: {"value": v["value"], "ms_per_step": v["ms"], "mean_steps": v["steps"], "tuning": v["tuning"]}
                   for k, v in runs.items()}
    robust_line["mixed"].update(speedup_vs_fp64=runs["mixed"]["value"] / runs["fp64"]["value"], recall_vs_fp64=rec,
                                fp64_real_solutions=n_real, endpoint_error_vs_fp64=err)
    return _line("hypothesis-solves/s (batched, one graph replay per step)", H * len(ms) / (total * 1e-3), args,
          {"workload": "uncalibrated_trifocal_rel_pos_CY: %d RANSAC hypotheses x 668 paths (%d paths) per step, "
                       "30%% outlier correspondences (inliers exact), FP64, reference step control, FP64 polish, one CUDA graph"
                       % (H, H * b.paths), "hypotheses_per_step": H, "l2": "flushed before each step"},
          ms_per_step=total / len(ms), p50_ms=float(np.percentile(ms, 50)), p99_ms=float(np.percentile(ms, 99)),
          paths={"per_step": H * b.paths, "converged_frac": float(conv.mean()), "mean_steps": float(steps.mean()),
                 "max_steps": int(steps.max())},
          inlier_hypotheses=int(inlier.sum()), inlier_ground_truth_found=found / max(1, int(inlier.sum())),
          tuning=tuning, gpu_launches=3 * args.steps,
          path_jump_free_control={"hypotheses": HR, "note": "hypotheses from the same seeded scene generator, corrector |dx|^2 < 1e-12 |x|^2, first-update test "
                                          "1e-2, dt <= 0.05, 3 iterations, FP64 polish 3; recall = share of the FP64 "
                                          "run's real solutions (|Im| <= 1e-8, |H(x,1)| < 1e-10) the mixed run "
                                          "finds within 1e-8", **robust_line})


def recall_and_error(ref, cand, paths):
    """Share of ref's real solutions (converged, |Im| <= 1e-8, |H(x,1)| < 1e-10) that cand finds within
    1e-8 (max-norm, relative to max(1, |x|)), hypothesis by hypothesis, with the max and 99th
    percentile error of the matched endpoints."""
    e_r, c_r, r_r = ref["e"], ref["c"], ref["r"]
    real = (c_r == 1) & (np.abs(e_r.imag).max(axis=1) <= 1e-8) & (r_r >= 0) & (r_r < 1e-10)
    found, errs = 0, []
    for i in np.nonzero(real)[0]:
        h = i // paths
        blk = cand["e"][h * paths:(h + 1) * paths][cand["c"][h * paths:(h + 1) * paths] == 1]
        d = (np.abs(blk - e_r[i]).max(axis=1) / max(1.0, np.abs(e_r[i]).max())).min() if blk.size else np.inf
        found += bool(d <= 1e-8)
        if d <= 1e-8:
            errs.append(float(d))
    errs = np.array(errs) if errs else np.zeros(1)
    return found / max(1, int(real.sum())), int(real.sum()), {"max": float(errs.max()),
                                                               "p99": float(np.percentile(errs, 99))}


def config_p3p_td(args, torch):
    single = Batch(torch, "P3P_TD", 1, 7 + args.seed, polish=2)
    lat = []
    for i in range(args.warmup + max(args.steps, 50)):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        single.launch()
        e1.record()
        e1.synchronize()
        if i >= args.warmup:
            lat.append(e0.elapsed_time(e1))
    E = _to_cx(single.ws.endpoints)
    gt_ok = bool(np.abs(E - single.truth[0]).max(axis=1).min() < 1e-9)
    H = 65536
    batch = Batch(torch, "P3P_TD", H, 8 + args.seed, polish=2)
    tuning = batch.tune() if args.tune else None
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    g = _capture(torch, batch.launch)
    for _ in range(args.warmup):
        g.replay()
    ms = _time_graph(torch, g, args.steps, flush)
    E = _to_cx(batch.ws.endpoints).reshape(H, 8, 3)
    hit = np.mean([np.abs(E[h] - batch.truth[h]).max(axis=1).min() < 1e-9 for h in range(0, H, 64)])
    return _line("hypothesis-solves/s (P3P total degree)", H * len(ms) / (sum(ms) * 1e-3), args,
          {"workload": "P3P_TD: 3 depths, 8 total-degree paths, seeded unit-modulus gamma; 1 instance (latency) "
                       "and %d instances per step (throughput); FP64 with polish" % H},
          ms_per_step=sum(ms) / len(ms), single_instance={"p50_ms": float(np.percentile(lat, 50)),
                                                          "p99_ms": float(np.percentile(lat, 99)),
                                                          "ground_truth_found": gt_ok},
          ground_truth_found_frac=float(hit), tuning=tuning, gpu_launches=3 * args.steps)


MIX = [("P3P_TD", 8192), ("5pt_rel_pos_alg_form_quat", 4096), ("generalized_3views_4pts", 2048),
       ("trifocal_2op1p_30x30", 1024)]


def config_mix(args, torch):
    batches = [Batch(torch, n, h, 50 + i + args.seed) for i, (n, h) in enumerate(MIX)]
    tuning = {b.name: b.tune() for b in batches} if args.tune else None
    streams = [torch.cuda.Stream() for _ in batches]

    def fork_join():
        main = torch.cuda.current_stream()
        ev = torch.cuda.Event()
        ev.record(main)
        for b, st in zip(batches, streams):
            with torch.cuda.stream(st):
                st.wait_event(ev)
                b.launch()
        for st in streams:
            main.wait_stream(st)

    def one_launch():
        ghc.track_mix([(b.pb, b.ws, b.d_sols, dict(b._inputs(), **b.kw)) for b in batches])

    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    g = _capture(torch, one_launch)
    for _ in range(args.warmup):
        g.replay()
    ms = _time_graph(torch, g, args.steps, flush)
    gf = _capture(torch, fork_join)
    for _ in range(args.warmup):
        gf.replay()
    fork_ms = _time_graph(torch, gf, args.steps, flush)
    # each problem alone, for the overlap benefit
    alone = {}
    for b in batches:
        gb = _capture(torch, b.launch)
        alone[b.name] = statistics.median(_time_graph(torch, gb, 2, flush))
    total_h = sum(h for _, h in MIX)
    return _line("hypothesis-solves/s (uneven mix, one persistent launch)", total_h * len(ms) / (sum(ms) * 1e-3), args,
          {"workload": "uneven mix in one persistent launch (ghc_track_mix, captured in a CUDA graph): " +
                       ", ".join("%s %d hyp" % m for m in MIX) + "; FP64, reference step control"},
          ms_per_step=sum(ms) / len(ms), alone_ms=alone, sum_alone_ms=sum(alone.values()),
          four_streams_in_one_graph_ms=statistics.median(fork_ms),
          tuning=tuning,
          per_problem={b.name: {"hypotheses": b.H, "paths": b.H * b.paths,
                                "converged_frac": float(b.ws.conv.float().mean())} for b in batches},
          gpu_launches=4 * args.steps)


def config_g3v4_mono(args, torch):
    import monodromy
    pb = ghc.Problem("generalized_3views_4pts")
    t0 = time.time()
    q, Sq, S = monodromy.start_system(pb, seed=args.seed)
    mono_s = time.time() - t0
    H = min(args.hyp, 512)
    out = {}
    runs = {}
    step = dict(step=dict(corr_tol2=1e-12, first_tol2=1e-2, dt_max=0.05), max_corr=3, max_steps=2000)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    for name, prec in (("fp64", ghc.PREC_FP64), ("mixed", ghc.PREC_MIXED)):
        # exact scenes, so the scene's unknowns are a solution (known-answer check at 1e-6); with
        # 0.5 px noise this minimal problem moves its solutions by ~5 % (ill-conditioned)
        b = Batch(torch, "generalized_3views_4pts", H, 77 + args.seed, precision=prec, polish=3, step=step,
                  start=q, sols=Sq, scene={"noise_px": 0.0})
        if args.tune:
            b.tune()
        g = _capture(torch, b.launch)
        ms = _time_graph(torch, g, max(1, args.steps // 2), flush)
        runs[name] = (_to_cx(b.ws.endpoints).reshape(H, b.paths, -1), b.ws.conv.cpu().numpy().reshape(H, -1) == 1,
                      b.truth)
        out[name] = {"value": H / (statistics.median(ms) * 1e-3), "unit": UNIT, "ms": statistics.median(ms)}
    e64, c64, truth = runs["fp64"]
    emx, cmx, _ = runs["mixed"]
    real = 0
    found = 0
    gt_hits = 0
    for h in range(H):
        r = e64[h][c64[h] & (np.abs(e64[h].imag).max(axis=1) <= 1e-8)]
        m = emx[h][cmx[h]]
        for e in r:
            real += 1
            d = np.abs(m - e).max(axis=1) / max(1.0, np.abs(e).max())
            found += bool(d.size and d.min() <= 1e-8)
        E = e64[h][c64[h]]
        gt_hits += bool(E.size and (np.abs(E - truth[h]).max(axis=1) / np.abs(truth[h]).max()).min() < 1e-6)
    return _line("hypothesis-solves/s at real-sol recall, mixed vs plain FP64 (own start system)", out["mixed"]["value"],
          args, {"workload": "generalized_3views_4pts: start params ~ complex N(0,1) (seed %d), %d start solutions "
                             "from the monodromy solver, %d seeded exact scenes per step, path-jump-free "
                             "step control, FP64 polish" % (args.seed, len(Sq), H)},
          modes=out, recall_mixed_vs_fp64=found / max(1, real), real_solutions_fp64=real,
          ground_truth_found_frac=gt_hits / H, monodromy={"solutions": len(S), "seconds": mono_s})


def config_problem(args, torch):
    prec = {"fp64": ghc.PREC_FP64, "fp32": ghc.PREC_FP32, "mixed": ghc.PREC_MIXED}[args.precision]
    step = None
    if args.step == "robust":
        step = dict(step=dict(corr_tol2=1e-12, first_tol2=1e-2, dt_max=0.05), max_corr=3, max_steps=2000)
    H = args.hyp
    b = Batch(torch, args.problem, H, 500 + args.seed, precision=prec, step=step)
    tuning = b.tune() if args.tune else None
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    g = _capture(torch, b.launch)
    for _ in range(args.warmup):
        g.replay()
    ms = _time_graph(torch, g, args.steps, flush)
    steps = b.ws.steps.cpu().numpy().astype(np.int64)
    solves = 4 * steps + b.ws.corr.cpu().numpy()
    total = sum(ms)
    return _line("hypothesis-solves/s (one problem, batched)", H * len(ms) / (total * 1e-3), args,
          {"workload": "%s: %d hypotheses x %d paths per launch, %s, %s step control, one CUDA graph"
                       % (args.problem, H, b.paths, args.precision, args.step), "l2": "flushed before each step"},
          ms_per_step=total / len(ms), p50_ms=float(np.percentile(ms, 50)),
          paths={"per_step": H * b.paths, "converged_frac": float(b.ws.conv.float().mean()),
                 "mean_solves": float(solves.mean()), "p99_solves": float(np.percentile(solves, 99)),
                 "max_solves": int(solves.max())},
          tuning=tuning,
          solves_per_s=float(solves.sum()) / (statistics.median(ms) * 1e-3), gpu_launches=len(ms) * (2 if
          b.pb.kind == ghc.KIND_P2C else 1))


# The reference's published single-instance times (ms per problem instance, complex FP32 kernels, GPU
# model not stated): GPU-HC README.md:41-63.
PUBLISHED_MS = [("P3P", 0.15), ("5pt_rel_pos_alg_form_quat", 1.77), ("generalized_3views_4pts", 4.77),
                ("uncalibrated_trifocal_rel_pos_CY", 16.67), ("trifocal_2op1p_30x30", 54.44)]


def config_latency(args, torch):
    """One instance per launch: each problem's shipped start and target parameters, the reference's
    step control, the tracker timed by CUDA events with the coefficients resident (the reference
    builds them on the host before its kernel) as replays of a captured launch, and beside it eager
    launches and eager device P2C + tracker, in FP32 (the reference's precision), FP64 and mixed;
    p50 / p99 beside the reference's published time."""
    n = max(args.steps, 30)
    out, ratios, launches = {}, [], 0
    for name, pub in PUBLISHED_MS:
        row = {"published_ms": pub}
        for pname, prec in (("fp32", ghc.PREC_FP32), ("fp64", ghc.PREC_FP64), ("mixed", ghc.PREC_MIXED)):
            b = Batch(torch, name, 1, 0, precision=prec, shipped=True)
            inp = b._inputs()  # coefficients resident: the tracker alone, as the reference times it
            track = lambda: ghc.track(b.pb, b.ws, b.d_sols, **inp, **b.kw)  # noqa: E731
            # replays of a captured launch (device time, as a C++ caller that captures its solve sees
            # it), beside eager launches from Python (host launch overhead inside the events) and
            # eager device P2C + tracker
            g = _capture(torch, track)
            lat, lat_eager, lat_p2c = [], [], []
            for i in range(args.warmup + n):
                for fn, acc in ((g.replay, lat), (track, lat_eager), (b.launch, lat_p2c)):
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record()
                    fn()
                    e1.record()
                    e1.synchronize()
                    if i >= args.warmup:
                        acc.append(e0.elapsed_time(e1))
            row[pname] = {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                          "eager_p50_ms": float(np.percentile(lat_eager, 50)),
                          "p2c_and_track_p50_ms": float(np.percentile(lat_p2c, 50)),
                          "converged": int(b.ws.conv.sum()), "paths": b.paths}
            launches += n * ((2 if prec == ghc.PREC_MIXED else 1) * 3 + (1 if b.pb.kind == ghc.KIND_P2C else 0))
        row["fp32_speedup_vs_published"] = pub / row["fp32"]["p50_ms"]
        ratios.append(row["fp32_speedup_vs_published"])
        out[name] = row
    gm = float(np.exp(np.mean(np.log(ratios))))
    return _line("single-instance latency vs the reference's published times (geometric mean of ratios, FP32)", gm, args,
          {"workload": "one instance per launch: the shipped start/target parameters of P3P, 5-point, "
                       "generalized 3-view, uncalibrated trifocal CY and trifocal 30x30; reference step control; "
                       "p50 over %d launches each" % n},
          unit="x (published ms / p50 ms)", data="the problem folders' own instances", problems=out,
          gpu_launches=launches)


def config_served(args, torch, lams=None, n_req=None):
    import serve
    return serve.bench(args, torch, lams=lams, n_req=n_req)


def run(args):
    import torch
    torch.cuda.set_device(0)
    line = {"cy": config_cy, "p3p_td": config_p3p_td, "mix": config_mix, "served": config_served,
            "g3v4_mono": config_g3v4_mono, "problem": config_problem,
            "latency": config_latency}[args.config](args, torch)
    print(json.dumps(line), flush=True)


def summary(args, torch):
    """Short runs of the other configured workloads, for the headline bench line: P3P by total
    degree (config 1), CY RANSAC batch (config 3; the path-jump-free comparison on its first 512
    hypotheses), the uneven mix (config 4) and the served stream (config 5: one load point of 200
    requests).  Each entry is that workload's own line."""
    import argparse
    short = argparse.Namespace(**vars(args))
    short.steps, short.warmup, short.hyp = 2, 1, 1024
    out = {}
    for name, fn, kw in (("p3p_td", config_p3p_td, {}), ("cy", config_cy, {"robust_hyp": 512}),
                         ("mix", config_mix, {}), ("served", config_served, {"lams": [20], "n_req": 200})):
        t0 = time.time()
        line = fn(short, torch, **kw)
        line["wall_s"] = time.time() - t0
        out[name] = line
    return out
