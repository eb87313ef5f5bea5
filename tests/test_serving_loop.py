"""Host logic of the batched serving loop (no GPU: the serving engine is a
stand-in with a neuron pool, network slots and a device that runs one chunk
behind the host).  Every request is admitted once, advanced for its whole
duration, retired only after the chunk that ends it has been drained, and its
spikes are read exactly once; the pool is never oversubscribed."""

import copy

import numpy as np

from nestgpu import serving


class _StandInEngine:
    def __init__(self, capacity_neurons, max_networks):
        self.cap = capacity_neurons
        self.max_networks = max_networks
        self.free = capacity_neurons
        self.nets = {}                  # id -> dict(n, step0, until)
        self.clock = 0                  # steps enqueued
        self.drained = 0                # steps whose spikes the host can read
        self.events = 0
        self.reads = {}
        self.log = []
        self.tune_state = "cached"       # "pending": the autotuner waits for a long enough call
        self.calls = []                  # steps of each simulate_async call

    # -- the subset of _abi.Engine the loop uses
    def stats(self):
        return {"syn_events": self.events, "clock_steps": self.clock}

    def net_capacity(self):
        return self.free, 10**12

    def net_add(self, n, steps, seed, var_values, build=None, poisson=None, record=True):
        if n > self.free or len(self.nets) >= self.max_networks:
            return None
        nid = next(i for i in range(self.max_networks) if i not in self.nets)
        self.nets[nid] = {"n": n, "step0": self.clock, "until": self.clock + steps}
        self.free -= n
        self.log.append(("add", nid, self.clock))
        return nid

    def tuned(self):
        return {"state": self.tune_state}

    def simulate_async(self, k):
        assert k > 0 and k % serving.DELAY_STEPS == 0
        self.calls.append(k)
        if self.tune_state == "pending" and k >= 112 * serving.DELAY_STEPS:
            self.tune_state = "tuned"   # the call had room for the trial groups
        self.drained = self.clock      # the previous call's last group is drained now
        for nw in self.nets.values():
            live = max(0, min(nw["until"], self.clock + k) - max(nw["step0"], self.clock))
            self.events += live * nw["n"]
        self.clock += k

    def sync(self):
        self.drained = self.clock

    def net_spikes(self, nid):
        nw = self.nets[nid]
        assert nw["until"] <= self.drained, "spikes read before the chunk that ends the network was drained"
        assert nid not in self.reads
        self.reads[nid] = nw["until"] - nw["step0"]
        return np.zeros(0, np.int32), np.zeros(0, np.int64)

    def net_remove(self, nid):
        assert nid in self.reads
        self.free += self.nets.pop(nid)["n"]
        self.reads.pop(nid)
        self.log.append(("remove", nid, self.clock))


def test_batched_loop_lifecycle():
    reqs = serving.make_requests(count=60, rate_hz=0.0, seed=7)
    eng = _StandInEngine(capacity_neurons=150_000, max_networks=8)
    done, st = serving.run_batched([copy.copy(r) for r in reqs], eng, realtime=False)
    assert not eng.nets and eng.free == eng.cap
    assert all(np.isfinite(r.finished) and r.finished >= r.admitted >= 0 for r in done)
    assert all(r.spikes is not None for r in done)
    # each network ran exactly its duration: the events add up to sum(n * steps)
    assert st["syn_events"] == sum(r.n * r.steps for r in reqs)
    adds = sum(1 for e in eng.log if e[0] == "add")
    removes = sum(1 for e in eng.log if e[0] == "remove")
    assert adds == removes == len(reqs)


def test_batched_loop_single_slot():
    """One network slot: strictly one request at a time, each retired before
    the next is admitted."""
    reqs = serving.make_requests(count=5, rate_hz=0.0, seed=9)
    eng = _StandInEngine(capacity_neurons=100_000, max_networks=1)
    done, st = serving.run_batched([copy.copy(r) for r in reqs], eng, realtime=False)
    kinds = [e[0] for e in eng.log]
    assert kinds == ["add", "remove"] * 5
    assert st["syn_events"] == sum(r.n * r.steps for r in reqs)


def test_first_chunk_long_enough_for_the_autotuner():
    """While the engine's autotuner waits for a long enough call, the loop's
    first chunk is tune_slices long; after it the chunks are chunk_slices;
    durations and events stay exact."""
    reqs = serving.make_requests(count=20, rate_hz=0.0, seed=3)
    eng = _StandInEngine(capacity_neurons=150_000, max_networks=8)
    eng.tune_state = "pending"
    done, st = serving.run_batched([copy.copy(r) for r in reqs], eng, realtime=False, chunk_slices=32,
                                   tune_slices=112)
    assert eng.calls[0] == 112 * serving.DELAY_STEPS
    assert eng.tune_state == "tuned"
    assert max(eng.calls[1:]) <= 32 * serving.DELAY_STEPS
    assert st["syn_events"] == sum(r.n * r.steps for r in reqs)
