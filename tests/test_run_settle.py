"""Host logic of the asynchronous Run of the PyNEST mirror (no GPU: the
engine is a stand-in that logs its calls).  A Run is enqueued in up to four
calls of whole slice graphs; after each call the spikes drained so far (those
of the earlier calls) reach the recorders, the last call's are held until the
next read or change of the network (settle), and nothing is lost or counted
twice across Runs."""

import numpy as np

from nestgpu.kernel import Device, Kernel
from nestgpu.models import DEVICE_MODELS


class _StandIn:
    """simulate_async(k): the spikes of a call become readable when the next
    call is made or on sync, as with the engine's last undrained group."""

    def __init__(self, n_src, rate):
        self.n_src, self.rate = n_src, rate
        self.rng = np.random.default_rng(0)
        self.calls, self.syncs = [], 0
        self.clock = 0
        self.pending = (np.zeros(0, np.int32), np.zeros(0, np.int64))
        self.ready = [self.pending]
        self.total = 0

    def simulate_async(self, k):
        self.calls.append(k)
        self.ready.append(self.pending)
        n = int(self.rate * k)
        src = self.rng.integers(0, self.n_src, n).astype(np.int32)
        stamp = np.sort(self.rng.integers(self.clock + 1, self.clock + k + 1, n)).astype(np.int64)
        self.clock += k
        self.total += n
        self.pending = (src, stamp)

    def sync(self):
        self.syncs += 1
        self.ready.append(self.pending)
        self.pending = (np.zeros(0, np.int32), np.zeros(0, np.int64))

    def spikes(self):
        src = np.concatenate([r[0] for r in self.ready])
        stamp = np.concatenate([r[1] for r in self.ready])
        self.ready = []
        return src, stamp

    def stats(self):
        return {"spikes": self.total}


def _kernel(n_src=400):
    k = Kernel()
    d = dict(DEVICE_MODELS["spike_recorder"])
    k.devices = [Device("spike_recorder", d)]
    k.node_local = np.zeros(1, dtype=np.int64)
    mask = np.ones(n_src, dtype=bool)
    k.compiled = {"N": n_src, "eng_to_node": np.arange(n_src, dtype=np.int64) + 1, "recorders": {1: mask},
                  "rec_part": None, "samplers": {}, "blocks": [], "min_delay": 15}
    k.engine = _StandIn(n_src, rate=2.0)
    k.trace_neurons = None
    k.structure_changed = False
    k.prepared = True
    return k


def _recorded(k):
    return sum(len(x) for x in k.devices[0].events["senders"])


def test_run_in_calls_and_settle():
    k = _kernel()
    eng = k.engine
    k.run(100.0)                       # 1,000 steps: calls of 64 slices x 15 steps
    assert eng.calls == [960, 40]
    assert eng.syncs == 0
    assert k._unsettled
    # the first call's spikes are routed, the second call's still held
    assert _recorded(k) == int(2.0 * 960)
    k.settle()
    assert not k._unsettled and eng.syncs == 1
    assert _recorded(k) == eng.total == k.stats["spikes"]
    assert k.clock == 1000


def test_runs_back_to_back_lose_nothing():
    k = _kernel()
    eng = k.engine
    for _ in range(5):
        k.run(1000.0)                  # 10,000 steps: 4 calls of 2,880, the last 1,360
    assert eng.calls[:4] == [2880, 2880, 2880, 1360]
    assert len(eng.calls) == 20 and eng.syncs == 0
    k.settle()
    ev = k.devices[0].events
    times = np.concatenate(ev["times"])
    assert len(times) == eng.total
    assert np.all(np.diff(times) >= 0)  # emission order kept across calls and Runs
    k.settle()                           # idempotent
    assert eng.syncs == 1
