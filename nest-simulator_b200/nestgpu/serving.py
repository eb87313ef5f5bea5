"""Serving: a request loop that runs many independent network simulations on
one GPU with continuous batching.

Requests are Brunel-type iaf_psc_exp networks (sizes, coupling and drive
drawn per request).  The batched server keeps one serving engine
(``ng_config.serving``): a request is admitted as soon as its neurons and
edges fit the engine's free pool (admission by device-memory footprint), its
graph is drawn on the device, it advances together with every other live
network in the same slice kernels, and it is retired -- its spikes drained,
its pool space freed -- at the first slice boundary after its duration.  The
plain server runs the same requests one at a time in the FP64 form.

A network's result does not depend on the mix it runs in: its Philox streams
(graph and drive) are keyed by its own seed and counted in its own neuron
numbering and local time, and the FP32 form's int64 ring sums are order
independent.
"""

import math
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import _abi

H = 0.1                      # ms
DELAY_STEPS = 15             # 1.5 ms
J_EXC = 87.8                 # pA
TAU_SYN = 0.5                # ms
# external rate that brings the mean membrane potential of an iaf_psc_exp
# neuron (C_m 250 pF, tau_m 10 ms, threshold 15 mV above rest) to threshold:
# nu_th = 15 mV * C_m / (J * tau_syn * tau_m) [1/ms]
NU_TH_HZ = 15.0 * 250.0 * 1000.0 / (J_EXC * TAU_SYN * 10.0)


@dataclass
class Request:
    rid: int
    arrival: float           # s after the start of the run
    n: int
    n_exc: int
    k_exc: int
    k_inh: int
    g: float
    eta: float
    steps: int
    seed: int
    enqueued: float = math.nan   # s: the arrival (real-time runs) or 0 (all queued at the start)
    admitted: float = math.nan
    finished: float = math.nan
    spikes: tuple = field(default=None, repr=False)
    syn_events: int = 0

    @property
    def latency(self):
        return self.finished - self.enqueued

    def syn_events_from_spikes(self):
        """Recurrent synaptic events: spikes times the source's out-degree (the
        graph's expected out-degree equals its in-degree per population)."""
        src = self.spikes[0]
        exc = np.count_nonzero(src < self.n_exc)
        inh = len(src) - exc
        return exc * (self.n * self.k_exc / max(1, self.n_exc)) + inh * (self.n * self.k_inh / max(1, self.n - self.n_exc))


def make_requests(count=256, rate_hz=20.0, seed=2026, n_min=1000, n_max=50000, t_min_ms=500.0, t_max_ms=2000.0):
    """Request stream of the serving benchmark: Poisson arrivals at `rate_hz`,
    N ~ log-uniform[n_min, n_max] (80 % excitatory), K_E = min(0.1 N, 1000),
    K_I = K_E / 4, g ~ U[3, 7], eta ~ U[0.9, 2.0], T ~ U[t_min, t_max] ms."""
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate_hz, count)) if rate_hz > 0 else np.zeros(count)
    out = []
    for i in range(count):
        n = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
        n_exc = int(round(0.8 * n))
        k_exc = int(min(round(0.1 * n), 1000))
        k_inh = max(1, k_exc // 4)
        t_ms = rng.uniform(t_min_ms, t_max_ms)
        out.append(Request(rid=i, arrival=float(arrivals[i]), n=n, n_exc=n_exc, k_exc=k_exc, k_inh=k_inh,
                           g=float(rng.uniform(3.0, 7.0)), eta=float(rng.uniform(0.9, 2.0)),
                           steps=int(round(t_ms / H)), seed=int(rng.integers(1, 2**62))))
    return out


def _admit(eng, r, record=True):
    rng = np.random.default_rng(r.seed)
    V0 = rng.normal(-58.0, 10.0, r.n)
    V0 += 70.0                                   # V_m relative to E_L = -70 mV
    build = dict(n_exc=r.n_exc, k_exc=r.k_exc, k_inh=r.k_inh, w_exc=J_EXC, w_inh=-r.g * J_EXC,
                 delay_steps=DELAY_STEPS, allow_autapses=0, seed=r.seed ^ 0x5A5A5A5A)
    rate = r.eta * NU_TH_HZ
    return eng.net_add(r.n, r.steps, r.seed, {"tau_syn_ex": TAU_SYN, "tau_syn_in": TAU_SYN, "V_m_rel": V0},
                       build=build, poisson=(rate, J_EXC, DELAY_STEPS), record=record)


def footprint(r):
    """Neurons and edge slots a request needs in the pool."""
    return r.n, r.n * (r.k_exc + r.k_inh) + 3 * r.n


def new_engine(precision="fp32", capacity_neurons=2_000_000, capacity_edges=1_200_000_000, max_networks=512,
               device=0, graph_slices=64):
    prec = _abi.NG_FP32 if precision == "fp32" else _abi.NG_FP64
    eng = _abi.Engine([(_abi.NG_IAF_PSC_EXP, capacity_neurons)], H, DELAY_STEPS, DELAY_STEPS, precision=prec,
                      device=device, serving=True, max_networks=max_networks, edge_capacity=capacity_edges,
                      max_abs_weight=8.0 * J_EXC)
    eng.set_graph_slices(graph_slices)
    return eng


def run_batched(requests, eng, chunk_slices=32, clock=time.perf_counter, realtime=True, tune_slices=0):
    """Continuous batching.  Returns (requests, stats).

    Every live network advances in chunks of `chunk_slices` min_delay slices;
    between chunks, the networks whose duration has passed are retired (their
    spikes drained, their pool space freed) and the waiting requests that fit
    the free pool are admitted, oldest first.  A request is only built (its
    initial state drawn, its graph requested) when its footprint fits the
    largest free runs of the pool.

    The chunks are enqueued with ng_simulate_async: the host reads the spikes
    of the networks that ended by the start of the running chunk while the
    device runs it, so a network is retired one chunk after its end (or at
    once when no live network is left to advance).

    With `tune_slices` > 0 and the engine's autotuner not measured yet, the
    first chunk is `tune_slices` long: the tuner needs one call with room for
    its trial groups (which run the live networks' own slices), and chunks of
    `chunk_slices` are too short for it (on the serving sweep the tuned and
    the default launch configurations measured the same, so it is off by
    default)."""
    pending = sorted(requests, key=lambda r: r.arrival)
    waiting = []
    active = {}                       # network id -> (request, engine step at which it ends)
    t0 = clock()
    st0 = eng.stats()
    ev0 = st0["syn_events"]
    now_steps = st0["clock_steps"]
    steps_run = 0
    while pending or waiting or active:
        now = clock() - t0
        while pending and (pending[0].arrival <= now or not realtime):
            r = pending.pop(0)
            r.enqueued = r.arrival if realtime else 0.0
            waiting.append(r)
        if waiting:
            free_n, free_e = eng.net_capacity()
            still = []
            for r in waiting:
                fn, fe = footprint(r)
                nid = None
                if fn <= free_n and fe <= free_e and len(active) < eng.max_networks:
                    nid = _admit(eng, r)
                if nid is None:
                    still.append(r)
                    continue
                r.admitted = clock() - t0
                active[nid] = (r, now_steps + r.steps)
                free_n, free_e = eng.net_capacity()
            waiting = still
        if not active:
            if waiting:
                raise RuntimeError("a request does not fit the empty pool")
            if pending:
                time.sleep(max(0.0, pending[0].arrival - (clock() - t0)))
            continue
        # one chunk, or less when every live network ends before its end
        left = max(end for _, end in active.values()) - now_steps
        if left <= 0:
            eng.sync()
            ended = now_steps
        else:
            want = chunk_slices
            if tune_slices and eng.tuned()["state"] == "pending":
                want = max(chunk_slices, tune_slices)
            slices = max(1, min(want, -(-left // DELAY_STEPS)))
            ended = now_steps
            eng.simulate_async(slices * DELAY_STEPS)
            now_steps += slices * DELAY_STEPS
            steps_run += slices * DELAY_STEPS
        # networks that ended by the start of the running chunk: their spikes are
        # all drained; read them all before the first removal (which waits for
        # the device)
        done = [k for k, (_, end) in active.items() if end <= ended]
        for nid in done:
            r, _ = active[nid]
            r.spikes = eng.net_spikes(nid)
            r.finished = clock() - t0
        for nid in done:
            active.pop(nid)
            eng.net_remove(nid)
    eng.sync()
    makespan = clock() - t0
    ev = eng.stats()["syn_events"] - ev0
    return requests, {"makespan_s": makespan, "syn_events": ev, "syn_events_per_s": ev / makespan,
                      "engine_steps": steps_run}


def run_plain(requests, eng, clock=time.perf_counter, realtime=True):
    """One network at a time (FIFO), each run to completion."""
    order = sorted(requests, key=lambda r: r.arrival)
    t0 = clock()
    ev0 = eng.stats()["syn_events"]
    for r in order:
        now = clock() - t0
        if realtime and r.arrival > now:
            time.sleep(r.arrival - now)
        r.enqueued = r.arrival if realtime else 0.0
        nid = _admit(eng, r)
        if nid is None:
            raise RuntimeError("a request does not fit the empty pool")
        r.admitted = clock() - t0
        eng.simulate(-(-r.steps // DELAY_STEPS) * DELAY_STEPS)
        r.spikes = eng.net_spikes(nid)
        eng.net_remove(nid)
        r.finished = clock() - t0
    makespan = clock() - t0
    ev = eng.stats()["syn_events"] - ev0
    return order, {"makespan_s": makespan, "syn_events": ev, "syn_events_per_s": ev / makespan}


def spike_stats(r):
    """Mean rate [Hz] and mean CV of the inter-spike intervals (neurons with
    at least 3 spikes) of a finished request."""
    src, stamp = r.spikes
    t_s = r.steps * H * 1e-3
    rate = len(src) / (r.n * t_s)
    if len(src) < 3:
        return rate, float("nan")
    o = np.lexsort((stamp, src))
    s, t = src[o], stamp[o].astype(np.float64)
    same = s[1:] == s[:-1]
    isi = np.diff(t)[same]
    who = s[1:][same]
    cnt = np.bincount(who, minlength=r.n)
    sm = np.bincount(who, weights=isi, minlength=r.n)
    sq = np.bincount(who, weights=isi * isi, minlength=r.n)
    ok = cnt >= 2
    if not ok.any():
        return rate, float("nan")
    mu = sm[ok] / cnt[ok]
    var = np.maximum(sq[ok] / cnt[ok] - mu * mu, 0.0)
    return rate, float(np.mean(np.sqrt(var) / mu))


def accuracy(test, ref):
    """Rate and CV-ISI error of `test` (e.g. batched FP32) against `ref` (the
    FP64 form) over the same requests: aggregate rate error (total spikes),
    the median per-request rate error, and the mean and max absolute CV-ISI
    difference."""
    by_id = {r.rid: r for r in ref}
    rel, dcv = [], []
    tot_t = tot_r = 0
    for r in test:
        q = by_id[r.rid]
        rt, ct = spike_stats(r)
        rr, cr = spike_stats(q)
        tot_t += len(r.spikes[0])
        tot_r += len(q.spikes[0])
        if rr > 0:
            rel.append(abs(rt - rr) / rr)
        if np.isfinite(ct) and np.isfinite(cr):
            dcv.append(abs(ct - cr))
    return {"rate_err_total": abs(tot_t - tot_r) / max(1, tot_r),
            "rate_err_median": float(np.median(rel)) if rel else None,
            "cv_isi_err_mean": float(np.mean(dcv)) if dcv else None,
            "cv_isi_err_max": float(np.max(dcv)) if dcv else None,
            "requests": len(test)}


def latency_summary(requests):
    lat = np.array([r.latency for r in requests])
    return {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "max_s": float(lat.max())}


class OnlineBatcher:
    """Continuous batching of requests that arrive while the engine runs (the
    serving routes of nestgpu.server): one worker thread owns the FP32
    serving engine; ``submit`` queues a Brunel-type network and returns its
    id at once; the worker admits queued networks as pool space frees up,
    advances every live network in chunks of ``chunk_slices`` slices, and
    retires a network (spikes read, pool space freed) after its duration,
    as run_batched does for a stream known in advance."""

    def __init__(self, precision="fp32", capacity_neurons=2_000_000, capacity_edges=1_200_000_000, max_networks=512,
                 device=0, chunk_slices=32, clock=time.perf_counter):
        self.clock = clock
        self.t0 = clock()
        self.cv = threading.Condition()
        self.waiting = []
        self.requests = {}
        self.active = {}
        self.next_id = 0
        self.closed = False
        self.error = None
        self.cached_stats = {}
        self.chunk = chunk_slices
        self._args = (precision, capacity_neurons, capacity_edges, max_networks, device)
        self.ready = threading.Event()
        self.thread = threading.Thread(target=self._loop, daemon=True)
        self.thread.start()
        self.ready.wait(timeout=120)
        if self.error:
            raise RuntimeError(self.error)

    def submit(self, n, g=5.0, eta=2.0, t_ms=1000.0, seed=1):
        n = int(n)
        if n < 2:
            raise ValueError("a network needs at least 2 neurons")
        k_exc = int(min(round(0.1 * n), 1000))
        with self.cv:
            rid = self.next_id
            self.next_id += 1
            r = Request(rid=rid, arrival=self.clock() - self.t0, n=n, n_exc=int(round(0.8 * n)), k_exc=max(1, k_exc),
                        k_inh=max(1, k_exc // 4), g=float(g), eta=float(eta), steps=int(round(t_ms / H)),
                        seed=int(seed))
            r.enqueued = r.arrival
            self.requests[rid] = r
            self.waiting.append(r)
            self.cv.notify_all()
        return rid

    def result(self, rid, spikes=False):
        with self.cv:
            r = self.requests.get(rid)
            if r is None:
                return None
            if r.spikes is None:
                return {"request": rid, "status": "running" if not math.isnan(r.admitted) else "queued"}
        rate, cv = spike_stats(r)
        out = {"request": rid, "status": "done", "n": r.n, "steps": r.steps, "spikes": int(len(r.spikes[0])),
               "rate_hz": rate, "cv_isi": cv, "latency_s": r.latency, "admitted_after_s": r.admitted - r.enqueued}
        if spikes:
            out["senders"] = r.spikes[0]
            out["times_ms"] = r.spikes[1] * H
        return out

    def stats(self):
        with self.cv:
            return dict(self.cached_stats, queued=len(self.waiting), live=len(self.active),
                        done=sum(1 for r in self.requests.values() if r.spikes is not None))

    def close(self):
        with self.cv:
            self.closed = True
            self.cv.notify_all()
        self.thread.join(timeout=60)

    def _loop(self):
        try:
            eng = new_engine(self._args[0], capacity_neurons=self._args[1], capacity_edges=self._args[2],
                             max_networks=self._args[3], device=self._args[4])
        except Exception as err:  # surfaced by the constructor
            self.error = f"serving engine: {err}"
            self.ready.set()
            return
        self.ready.set()
        now_steps = eng.stats()["clock_steps"]
        try:
            while True:
                with self.cv:
                    if self.closed:
                        break
                    if not self.waiting and not self.active:
                        self.cv.wait(timeout=0.5)
                        continue
                    waiting = list(self.waiting)
                # admissions (engine calls outside the lock: submit never waits for the device)
                if waiting:
                    free_n, free_e = eng.net_capacity()
                    admitted = []
                    for r in waiting:
                        fn, fe = footprint(r)
                        if fn <= free_n and fe <= free_e and len(self.active) < eng.max_networks:
                            nid = _admit(eng, r)
                            if nid is not None:
                                r.admitted = self.clock() - self.t0
                                self.active[nid] = (r, now_steps + r.steps)
                                admitted.append(r)
                                free_n, free_e = eng.net_capacity()
                    with self.cv:
                        self.waiting = [r for r in self.waiting if r not in admitted]
                if not self.active:
                    time.sleep(0.01)
                    continue
                left = max(end for _, end in self.active.values()) - now_steps
                ended = now_steps
                if left <= 0:
                    eng.sync()
                else:
                    slices = max(1, min(self.chunk, -(-left // DELAY_STEPS)))
                    eng.simulate_async(slices * DELAY_STEPS)
                    now_steps += slices * DELAY_STEPS
                done = [k for k, (_, end) in self.active.items() if end <= ended]
                results = {nid: eng.net_spikes(nid) for nid in done}
                for nid in done:
                    r, _ = self.active.pop(nid)
                    eng.net_remove(nid)
                    with self.cv:
                        r.spikes = results[nid]
                        r.finished = self.clock() - self.t0
                st = eng.stats()
                with self.cv:
                    self.cached_stats = {k: st[k] for k in ("clock_steps", "spikes", "syn_events", "gather_slices")}
        finally:
            eng.close()
