"""Serving loop: continuous batching of tracking requests of mixed problems.

A request is (problem, target parameters of n hypotheses).  The server keeps
per problem a CUDA stream and two buffer slots (targets, coefficient tables,
endpoints and flags for up to ``capacity`` hypotheses), sized at start-up from
the free device memory (the budget is split evenly over the problems and slots,
capped at ``max_batch`` hypotheses per launch).  Admission is by live free
memory too: before every launch the server asks the device for its free bytes
and starts the batch only if the tables the launch allocates leave
``reserve_bytes`` free; otherwise the requests stay queued, in order, until
memory frees up (``deferred`` counts the waits).

The loop admits every request that has arrived into its problem's queue;
whenever a slot of that problem is free it packs the queued requests (FIFO,
whole requests, up to the slot's capacity) into one batch, copies the targets
from pinned host memory, builds the coefficient tables on the device and
launches the tracker on the problem's stream -- while batches of the other
problems (and the other slot of the same problem) are still running.  When a
batch's event has completed, each request's slice of the endpoints and flags
is copied back and the request is complete, with its per-hypothesis result
counts (converged, real, infinity, unique) computed on the device.  Results do
not depend on which other requests shared a launch: every hypothesis is tracked
with the same arithmetic alone or in a batch (tests/test_gpu_serve.py checks this).

``precision`` selects the tracker (plain FP64 or the two-phase mixed one);
``tune=True`` autotunes each problem's launch on a sample batch at start-up.
``sequential=True`` gives the baseline of the same GPU without batching: one
request per launch, one stream, FIFO; ``dropin_rate`` measures the drop-in's
one hypothesis per launch.
"""
import collections
import json
import os
import time

import numpy as np

import ghc
import scenes

MIX = ["P3P_TD", "5pt_rel_pos_alg_form_quat", "generalized_3views_4pts", "trifocal_2op1p_30x30"]


class Request:
    __slots__ = ("rid", "problem", "targets", "arrival", "done", "endpoints", "conv", "inf", "status", "counts")

    def __init__(self, rid, problem, targets, arrival):
        self.rid, self.problem, self.targets, self.arrival = rid, problem, targets, arrival
        self.done = None
        # endpoints [n * paths, N], conv / inf / status [n * paths]; counts [n, 4] per hypothesis
        # (converged, real, infinity, unique; computed on the device)
        self.endpoints = self.conv = self.inf = self.status = self.counts = None


class _Slot:
    def __init__(self, torch, pb, cap, paths, N, P1, precision):
        self.cap = cap
        self.h_tg = torch.zeros((cap, P1, 2), dtype=torch.float64).pin_memory()
        self.d_tg = torch.zeros((cap, P1, 2), dtype=torch.float64, device="cuda")
        self.d_diff = torch.zeros((cap, P1, 2), dtype=torch.float64, device="cuda")
        self.ws = ghc.Workspace(pb, cap, precision, paths=paths)
        self.d_counts = torch.zeros((cap, 4), dtype=torch.int32, device="cuda")
        self.h_counts = torch.zeros((cap, 4), dtype=torch.int32).pin_memory()
        self.h_ep = torch.zeros((cap * paths, N, 2), dtype=torch.float64).pin_memory()
        self.h_conv = torch.zeros(cap * paths, dtype=torch.uint8).pin_memory()
        self.h_inf = torch.zeros(cap * paths, dtype=torch.uint8).pin_memory()
        self.h_status = torch.zeros(cap * paths, dtype=torch.uint8).pin_memory()
        self.event = None
        self.requests = []


class _Problem:
    def __init__(self, torch, name, cap, slots, precision):
        self.name = name
        self.pb = ghc.Problem(name)
        s, t = self.pb.params()
        if name == "P3P_TD":
            (s, _), _ = scenes.p3p_td(1, seed=0)
        self.start = s
        self.target = t
        self.paths = self.pb.paths
        self.d_start = torch.from_numpy(np.stack([s.real, s.imag], -1).copy()).cuda()
        sols = self.pb.start_sols()
        self.d_sols = torch.from_numpy(np.stack([sols.real, sols.imag], -1).copy()).cuda()
        self.stream = torch.cuda.Stream()
        self.slots = [_Slot(torch, self.pb, cap, self.paths, self.pb.N, self.pb.P + 1, precision)
                      for _ in range(slots)]
        self.queue = collections.deque()
        self.tuning = None

    def sample_targets(self, n, seed):
        if self.name == "P3P_TD":
            return scenes.p3p_td(n, seed=seed)[0][1]
        if self.name in scenes.GENERATORS:
            return scenes.GENERATORS[self.name](n, seed=seed)[0]
        return scenes.perturbed_targets(self.target, n, seed=seed)

    def inputs(self, torch, slot, n):
        if self.pb.kind == ghc.KIND_P2C:
            hx, ht = self.pb.p2c_device(self.d_start, slot.d_tg[:n])
            return dict(d_coef_hx=hx, d_coef_ht=ht)
        torch.sub(slot.d_tg[:n], self.d_start[None], out=slot.d_diff[:n])
        return dict(d_p_start=self.d_start, d_p_target=slot.d_tg[:n], d_p_diff=slot.d_diff[:n])

    def tune(self, torch, n=128):
        """Autotune this problem's launch on a sample batch of n hypotheses (at start-up)."""
        slot = self.slots[0]
        n = min(n, slot.cap)
        tg = self.sample_targets(n, seed=4711)
        slot.d_tg[:n].copy_(torch.from_numpy(np.stack([tg.real, tg.imag], -1)))
        slot.ws.n_hyp = n
        self.tuning = ghc.autotune(self.pb, slot.ws, self.d_sols, **self.inputs(torch, slot, n))


def transient_bytes(pb, n):
    """Device bytes a launch of n hypotheses takes beyond its slot's buffers: the per-hypothesis
    coefficient tables the device P2C builder writes (P2C problems; PH launches use the slot's
    parameter buffers only)."""
    if pb.kind != ghc.KIND_P2C:
        return 0
    return 16 * n * (pb.M + 1) * (2 * pb.K + 1)


def admit(free_bytes, need_bytes, reserve_bytes):
    """Admission by live free device memory: a batch starts only if it leaves the reserve free."""
    return free_bytes - need_bytes >= reserve_bytes


def bytes_per_hypothesis(pb):
    P1 = pb.P + 1
    tables = 16 * (pb.M + 1) * (2 * pb.K + 1) if pb.kind == ghc.KIND_P2C else 0
    per_path = 16 * pb.N + 3 + 4 * 2 + 8 * 3
    return 2 * 16 * P1 + tables + 2 * 16 + pb.paths * (per_path + 16 * pb.N + 3)


class Server:
    def __init__(self, torch, problems=MIX, max_batch=2048, hbm_fraction=0.25, sequential=False, max_request=512,
                 tune=False, precision=ghc.PREC_FP64, reserve_bytes=1 << 30, mem_info=None):
        self.torch = torch
        self.sequential = sequential
        # live free device memory (cudaMemGetInfo), asked again before every launch: a batch is
        # admitted only while its transient tables leave reserve_bytes free, else it waits queued
        self.mem_info = mem_info or torch.cuda.mem_get_info
        self.reserve = reserve_bytes
        self.deferred = 0
        free, _ = self.mem_info()
        slots = 1 if sequential else 2
        self.problems = {}
        for name in problems:
            pb = ghc.Problem(name)
            budget = hbm_fraction * free / (len(problems) * slots)
            cap = int(min(max(max_batch, max_request), budget // bytes_per_hypothesis(pb)))
            if cap < max_request:
                raise MemoryError("%s: %d hypotheses per slot fit in the memory budget, requests may have %d"
                                  % (name, cap, max_request))
            self.problems[name] = _Problem(torch, name, cap, slots, precision)
        self.fifo = collections.deque()  # sequential mode: global order
        self.launches = 0
        if tune:
            for prob in self.problems.values():
                prob.tune(torch)

    def submit(self, req):
        cap = self.problems[req.problem].slots[0].cap
        if req.targets.shape[0] > cap:
            raise ValueError("request of %d hypotheses exceeds the %d of a launch slot" % (req.targets.shape[0], cap))
        if self.sequential:
            self.fifo.append(req)
        else:
            self.problems[req.problem].queue.append(req)

    def _admit(self, prob, n):
        free, _ = self.mem_info()
        if admit(free, transient_bytes(prob.pb, n), self.reserve):
            return True
        self.deferred += 1
        return False

    def _launch(self, prob, slot, reqs):
        torch = self.torch
        n = sum(r.targets.shape[0] for r in reqs)
        tg = np.concatenate([r.targets for r in reqs])
        slot.h_tg[:n, :, 0] = torch.from_numpy(tg.real)
        slot.h_tg[:n, :, 1] = torch.from_numpy(tg.imag)
        slot.requests = reqs
        with torch.cuda.stream(prob.stream):
            slot.d_tg[:n].copy_(slot.h_tg[:n], non_blocking=True)
            ws = slot.ws
            ws.n_hyp = n
            ghc.track(prob.pb, ws, prob.d_sols, **prob.inputs(torch, slot, n))
            ghc.count_results_device(ws, prob.pb.N, out=slot.d_counts[:n])
            slot.h_counts[:n].copy_(slot.d_counts[:n], non_blocking=True)
            m = n * prob.paths
            slot.h_ep[:m].copy_(ws.endpoints[:m], non_blocking=True)
            slot.h_conv[:m].copy_(ws.conv[:m], non_blocking=True)
            slot.h_inf[:m].copy_(ws.inf[:m], non_blocking=True)
            slot.h_status[:m].copy_(ws.status[:m], non_blocking=True)
            slot.event = torch.cuda.Event()
            slot.event.record(prob.stream)
        self.launches += 1

    def _complete(self, prob, slot, now):
        off = 0
        hoff = 0
        for r in slot.requests:
            nh = r.targets.shape[0]
            r.counts = slot.h_counts[hoff:hoff + nh].numpy().copy()
            hoff += nh
            m = nh * prob.paths
            e = slot.h_ep[off:off + m].numpy()
            r.endpoints = e[..., 0] + 1j * e[..., 1]
            r.conv = slot.h_conv[off:off + m].numpy().copy()
            r.inf = slot.h_inf[off:off + m].numpy().copy()
            r.status = slot.h_status[off:off + m].numpy().copy()
            r.done = now
            off += m
        slot.requests = []
        slot.event = None

    def step(self, now):
        """Complete finished batches, then admit queued requests into free slots."""
        busy = False
        for prob in self.problems.values():
            for slot in prob.slots:
                if slot.event is not None:
                    if slot.event.query():
                        self._complete(prob, slot, now)
                    else:
                        busy = True
        if self.sequential:
            prob = None
            if self.fifo and not busy:
                r = self.fifo.popleft()
                prob = self.problems[r.problem]
                if self._admit(prob, r.targets.shape[0]):
                    self._launch(prob, prob.slots[0], [r])
                    busy = True
                else:
                    self.fifo.appendleft(r)
            return busy or bool(self.fifo)
        for prob in self.problems.values():
            for slot in prob.slots:
                if slot.event is None and prob.queue:
                    reqs, n = [], 0
                    while prob.queue and n + prob.queue[0].targets.shape[0] <= slot.cap:
                        reqs.append(prob.queue[0])
                        n += prob.queue.popleft().targets.shape[0]
                    if not self._admit(prob, n):
                        prob.queue.extendleft(reversed(reqs))  # back to the head, in order
                        continue
                    self._launch(prob, slot, reqs)
                    busy = True
        return busy or any(p.queue for p in self.problems.values())


def poisson_requests(lam, n_req, seed=0, problems=MIX, max_hyp=512):
    """Arrival offsets (s), problem and log-uniform size in [1, max_hyp] of n_req requests."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / lam, size=n_req)
    t = np.cumsum(gaps) - gaps[0]
    sizes = np.floor(np.exp(rng.uniform(0, np.log(max_hyp + 1), size=n_req))).astype(int)
    sizes = np.clip(sizes, 1, max_hyp)
    which = rng.integers(0, len(problems), size=n_req)
    return t, [problems[i] for i in which], sizes


def run_stream(server, lam, n_req, seed=0):
    """Feed a Poisson stream in real time; returns (latencies s, hypotheses, wall s)."""
    t_arr, probs, sizes = poisson_requests(lam, n_req, seed=seed, problems=list(server.problems))
    reqs = []
    for i in range(n_req):
        prob = server.problems[probs[i]]
        reqs.append(Request(i, probs[i], prob.sample_targets(int(sizes[i]), seed=seed * 100003 + i), None))
    server.torch.cuda.synchronize()
    t0 = time.perf_counter()
    nxt = 0
    while True:
        now = time.perf_counter() - t0
        while nxt < n_req and t_arr[nxt] <= now:
            reqs[nxt].arrival = t_arr[nxt]
            server.submit(reqs[nxt])
            nxt += 1
        active = server.step(now)
        if nxt >= n_req and not active:
            break
        if not active and nxt < n_req:
            time.sleep(min(1e-3, max(0.0, t_arr[nxt] - now)))
    wall = time.perf_counter() - t0
    lat = np.array([r.done - r.arrival for r in reqs])
    return lat, int(sizes.sum()), wall, reqs


def dropin_rate(server, n, seed=0):
    """One hypothesis per launch, FIFO on one stream: the drop-in tracker's service rate
    on the stream's problem mix (hypotheses/s over n single-hypothesis requests)."""
    rng = np.random.default_rng(seed)
    names = list(server.problems)
    # one untimed single-hypothesis request per problem first (the one-instance launch shape)
    warm = [Request(-1 - j, name, server.problems[name].sample_targets(1, seed=seed + j), 0.0)
            for j, name in enumerate(names)]
    for r in warm:
        server.submit(r)
    while server.step(0.0):
        pass
    reqs = [Request(i, names[k], server.problems[names[k]].sample_targets(1, seed=seed * 7919 + i), 0.0)
            for i, k in enumerate(rng.integers(0, len(names), size=n))]
    server.torch.cuda.synchronize()
    t0 = time.perf_counter()
    for r in reqs:
        server.submit(r)
    while server.step(time.perf_counter() - t0):
        pass
    return n / (time.perf_counter() - t0)


def _stats(lat, hyp, wall):
    return {"throughput": hyp / wall, "p50_ms": 1e3 * float(np.percentile(lat, 50)),
            "p99_ms": 1e3 * float(np.percentile(lat, 99)), "wall_s": wall}


def bench(args, torch, lams=None, n_req=None):
    """The served sweep; returns its JSON line (load points from GHC_SERVE_LAMBDAS or lams, requests
    per point from GHC_SERVE_REQUESTS or n_req)."""
    torch.cuda.set_device(0)
    if lams is None:
        lams = [int(v) for v in os.environ.get("GHC_SERVE_LAMBDAS", "10,20,40").split(",")]
    if n_req is None:
        n_req = int(os.environ.get("GHC_SERVE_REQUESTS", "1000"))
    tune = bool(getattr(args, "tune", 1))
    modes = {"batched_fp64": Server(torch, tune=tune),
             "batched_mixed": Server(torch, tune=tune, precision=ghc.PREC_MIXED),
             "sequential_fp64": Server(torch, sequential=True, tune=tune)}
    for i, srv in enumerate(modes.values()):  # warm-up (kernel attributes, tables)
        run_stream(srv, 1000, 8, seed=990 + i)
    rows = []
    for lam in lams:
        row = {"lambda_req_s": lam, "requests": n_req}
        for name, srv in modes.items():
            lat, hyp, wall, _ = run_stream(srv, lam, n_req, seed=lam)
            row["hypotheses"] = hyp
            # offered load: the stream's hypotheses over its arrival window (n_req / lambda)
            row["offered_hyp_s"] = hyp * lam / n_req
            row[name] = _stats(lat, hyp, wall)
        rows.append(row)
    # capacity: the same kind of stream with every request arriving at once (the server saturated)
    n_cap = max(50, n_req // 5)
    capacity = {}
    for name, srv in modes.items():
        lat, hyp, wall, _ = run_stream(srv, 1e9, n_cap, seed=4321)
        capacity[name] = dict(_stats(lat, hyp, wall), requests=n_cap, hypotheses=hyp)
    dropin = dropin_rate(modes["sequential_fp64"], 128, seed=5)
    best = max(capacity["batched_fp64"]["throughput"], capacity["batched_mixed"]["throughput"])
    line = {"metric": "served hypothesis-solves/s at capacity, and p50/p99 request latency vs offered load",
            "value": best,
            "unit": "hypotheses/s", "n_gpus": 1, "steps": len(lams), "warmup": 1, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "complex128", "data": "synthetic (seeded)",
            "config": {"workload": "Poisson request stream, %d requests per load point, 1-512 hypotheses "
                                   "(log-uniform) of a problem drawn uniformly from %s; continuous batching "
                                   "on per-problem streams (FP64 and mixed) vs one request per launch (FP64) vs "
                                   "one hypothesis per launch (the drop-in, FP64)" % (n_req, MIX)},
            "capacity_hypotheses_per_launch": {n: p.slots[0].cap for n, p in modes["batched_fp64"].problems.items()},
            "dropin_one_hypothesis_per_launch": {"throughput": dropin, "hypotheses": 128},
            "capacity": capacity,
            "capacity_vs_dropin": {k: v["throughput"] / dropin for k, v in capacity.items()},
            "note": "batched FP64 is bit-identical per hypothesis to the drop-in (recall 1.0 of its real solutions); "
                    "the mixed tracker runs the reference's step control here, under which a change of arithmetic "
                    "lands jumping paths on other roots",
            "tuning": {n: p.tuning for n, p in modes["batched_fp64"].problems.items()},
            "sweep": rows}
    return line
