"""Host side of a run: the spikes a run logged reach the spike recorders the
same way whether the recorders cover disjoint sources (one counting sort of
the run's spikes by recorder) or overlapping ones (one source mask per
recorder), with each recorder's start/stop window and time_in_steps
(spike_recorder semantics of the reference: recording_device.cpp,
spike_recorder.cpp).  No GPU: the engine is replaced by a fixed spike list.
"""

import numpy as np

from nestgpu.kernel import Device, Kernel
from nestgpu.models import DEVICE_MODELS


class _FixedSpikes:
    def __init__(self, src, stamp):
        self.src, self.stamp = src, stamp

    def spikes(self):
        return self.src, self.stamp


def _kernel(masks, params, src, stamp, partition):
    k = Kernel()
    k.devices = []
    for p in params:
        d = dict(DEVICE_MODELS["spike_recorder"])
        d.update(p)
        k.devices.append(Device("spike_recorder", d))
    k.node_local = np.arange(len(masks), dtype=np.int64)
    n_src = len(masks[0])
    rec = {rid: m for rid, m in zip(range(1, len(masks) + 1), masks)}
    part = None
    if partition:
        of = np.full(n_src, -1, dtype=np.int16)
        for j, m in enumerate(masks):
            of[m] = j
        part = (list(rec), of)
    k.compiled = {"N": n_src, "eng_to_node": np.arange(n_src, dtype=np.int64) + 1000, "recorders": rec,
                  "rec_part": part, "samplers": {}}
    k.engine = _FixedSpikes(src, stamp)
    k.trace_neurons = None
    k._collect()
    return [{key: np.concatenate(v) if v else np.zeros(0) for key, v in d.events.items()} for d in k.devices], \
        [d.n_events for d in k.devices]


def test_partitioned_routing_equals_masks():
    rng = np.random.default_rng(3)
    n_src, n = 5000, 200_000
    src = rng.integers(0, n_src, n).astype(np.int32)
    stamp = np.sort(rng.integers(1, 20_000, n)).astype(np.int64)
    owner = rng.integers(-1, 4, n_src)                 # 4 recorders over disjoint sources, some unrecorded
    masks = [owner == j for j in range(4)]
    params = [{}, {"start": 300.0}, {"stop": 1200.0}, {"start": 100.0, "stop": 900.0, "time_in_steps": True}]
    ev_p, n_p = _kernel(masks, params, src, stamp, partition=True)
    ev_m, n_m = _kernel(masks, params, src, stamp, partition=False)
    assert n_p == n_m
    for a, b in zip(ev_p, ev_m):
        for key in ("senders", "times"):
            np.testing.assert_array_equal(a[key], b[key])
    # against a direct restatement of the window rule (stamp in (t_min, t_max], steps of 0.1 ms)
    for j, (m, p) in enumerate(zip(masks, params)):
        t_min = round(p.get("start", 0.0) * 10)
        t_max = np.inf if "stop" not in p else round(p["stop"] * 10)
        sel = m[src] & (stamp > t_min) & (stamp <= t_max)
        np.testing.assert_array_equal(ev_p[j]["senders"], src[sel] + 1000)
        want_t = stamp[sel] if p.get("time_in_steps") else stamp[sel] * 0.1
        np.testing.assert_allclose(ev_p[j]["times"], want_t, rtol=0, atol=1e-9)
        assert n_p[j] == sel.sum()


def test_overlapping_recorders_use_masks():
    rng = np.random.default_rng(4)
    n_src, n = 300, 10_000
    src = rng.integers(0, n_src, n).astype(np.int32)
    stamp = np.sort(rng.integers(1, 5000, n)).astype(np.int64)
    masks = [np.arange(n_src) < 200, np.arange(n_src) >= 100]   # sources 100..199 in both
    ev, cnt = _kernel(masks, [{}, {}], src, stamp, partition=False)
    for j, m in enumerate(masks):
        np.testing.assert_array_equal(ev[j]["senders"], src[m[src]] + 1000)
        assert cnt[j] == m[src].sum()
