"""The allocation-free entry point, ng_simulate_noalloc, against the engine's
regular path (ng_create + ng_simulate) through the C ABI.

ng_simulate_noalloc serves callers that may not allocate device memory while
they step a network (a host that owns all device memory through its own
allocator, a controller stepping a small network every tick).  Inputs and
outputs are device buffers the caller owns -- here the test allocates them
with torch, outside the entry point -- and its scratch is a static device
array.  The network is the deterministic balanced iaf_psc_delta network of
the golden fixture, whose dyadic weights make the FP64 ring sums order
independent, so both paths must agree bit for bit.  Two calls in a row
check that the second call starts from a cleared scratch array; further
cases cover delays spread over [min_delay, max_delay], a start step other
than 0, a partial last slice, a chain of continued calls, an output buffer
that is too small, and edges whose target or delay is out of range.
"""

import ctypes
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


class NoAllocNet(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int64), ("min_delay", ctypes.c_int32), ("max_delay", ctypes.c_int32),
        ("start_step", ctypes.c_int64),
        ("P33", ctypes.c_void_p), ("P30", ctypes.c_void_p), ("V_th_rel", ctypes.c_void_p),
        ("V_reset_rel", ctypes.c_void_p), ("V_min_rel", ctypes.c_void_p), ("I_e", ctypes.c_void_p),
        ("refr_counts", ctypes.c_void_p), ("V_m_rel", ctypes.c_void_p), ("r", ctypes.c_void_p),
        ("row_ptr", ctypes.c_void_p), ("target", ctypes.c_void_p), ("weight", ctypes.c_void_p),
        ("delay", ctypes.c_void_p), ("out_src", ctypes.c_void_p), ("out_stamp", ctypes.c_void_p),
        ("out_cap", ctypes.c_int64), ("out_count", ctypes.c_void_p),
        ("continue_run", ctypes.c_int32), ("reserved", ctypes.c_int32), ("out_skipped", ctypes.c_void_p),
    ]


def _network(fx, ie_scale, delays=None):
    """The golden balanced network as noalloc inputs (host arrays); `delays`
    (per edge of the fixture's edge order, in steps) default to 15."""
    C_m, tau_m, t_ref, E_L, V_th, V_reset = (float(x) for x in fx["params"])
    n = len(fx["I_e"])
    h = (1.0 / 1000.0) * 100  # Time::get_resolution().get_ms() at 0.1 ms
    P33 = math.exp(-h / tau_m)
    P30 = 1 / C_m * (1 - P33) * tau_m
    refr = int((int(t_ref * 1000.0 + 0.5) + 99) * (1.0 / 100))
    src = fx["src"].astype(np.int64)
    order = np.argsort(src, kind="stable")
    row_ptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(src, minlength=n), out=row_ptr[1:])
    d = np.full(len(src), 15, dtype=np.int32) if delays is None else np.asarray(delays, dtype=np.int32)
    return {
        "n": n, "P33": np.full(n, P33), "P30": np.full(n, P30), "V_th_rel": np.full(n, V_th - E_L),
        "V_reset_rel": np.full(n, V_reset - E_L), "V_min_rel": np.full(n, -np.finfo(np.float64).max),
        "I_e": fx["I_e"] * ie_scale, "refr": np.full(n, refr, dtype=np.int32), "V0": fx["V0"] - E_L,
        "row_ptr": row_ptr, "target": fx["tgt"].astype(np.int32)[order],
        "weight": np.where(fx["exc"], 0.125, -0.625)[order], "delay": d[order],
        "params": (C_m, tau_m, t_ref, E_L, V_th, V_reset),
        "min_delay": int(d.min()), "max_delay": int(d.max()),
    }


def _run_engine(net, steps, start_step=0, keep=None):
    """The regular entry points: ng_create, ng_set_*, ng_simulate.  `keep`
    (a boolean mask over the CSR edges) drops the other edges."""
    from nestgpu import _abi

    n = net["n"]
    C_m, tau_m, t_ref, E_L, V_th, V_reset = net["params"]
    eng = _abi.Engine([(_abi.NG_IAF_PSC_DELTA, n)], 0.1, net["min_delay"], net["max_delay"], start_step=start_step)
    for name, val in (("C_m", C_m), ("tau_m", tau_m), ("t_ref", t_ref), ("V_th_rel", V_th - E_L),
                      ("V_reset_rel", V_reset - E_L)):
        eng.set_var(0, name, np.full(n, val))
    eng.set_var(0, "I_e", net["I_e"])
    eng.set_var(0, "V_m_rel", net["V0"])
    row_ptr, tgt, w, d = net["row_ptr"], net["target"], net["weight"], net["delay"]
    if keep is not None:
        src = np.repeat(np.arange(n), np.diff(row_ptr))[keep]
        row_ptr = np.zeros(n + 1, dtype=np.int64)
        np.cumsum(np.bincount(src, minlength=n), out=row_ptr[1:])
        tgt, w, d = tgt[keep], w[keep], d[keep]
    eng.set_connections(row_ptr, tgt, w, d)
    eng.set_recording(np.ones(n, dtype=np.uint8))
    eng.simulate(steps)
    src, stamp = eng.spikes()
    V = eng.get_var(0, "V_m_rel")
    eng.close()
    return src, stamp, V


class _NoAlloc:
    """Caller-owned device buffers of one network (allocated by the test,
    outside the entry point) and calls of ng_simulate_noalloc on them."""

    def __init__(self, net, cap=200000):
        import torch

        from nestgpu import _abi

        self.L = _abi.load()
        self.fn = self.L.ng_simulate_noalloc
        self.fn.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p]
        self.fn.restype = ctypes.c_int
        dev = torch.device("cuda", 0)
        self.dev = dev
        self.net = net
        self.t = {k: torch.as_tensor(np.ascontiguousarray(v)).to(dev)
                  for k, v in net.items() if isinstance(v, np.ndarray)}
        self.V = self.t["V0"].clone()
        self.r = torch.zeros(net["n"], dtype=torch.int32, device=dev)
        self.cap = cap
        self.out_src = torch.empty(max(cap, 1), dtype=torch.int32, device=dev)
        self.out_stamp = torch.empty(max(cap, 1), dtype=torch.int64, device=dev)
        self.out_count = torch.zeros(1, dtype=torch.int64, device=dev)
        self.out_skipped = torch.zeros(1, dtype=torch.int64, device=dev)

    def struct(self, start_step, continue_run):
        t = self.t
        return NoAllocNet(
            n=self.net["n"], min_delay=self.net["min_delay"], max_delay=self.net["max_delay"], start_step=start_step,
            P33=t["P33"].data_ptr(), P30=t["P30"].data_ptr(), V_th_rel=t["V_th_rel"].data_ptr(),
            V_reset_rel=t["V_reset_rel"].data_ptr(), V_min_rel=t["V_min_rel"].data_ptr(), I_e=t["I_e"].data_ptr(),
            refr_counts=t["refr"].data_ptr(), V_m_rel=self.V.data_ptr(), r=self.r.data_ptr(),
            row_ptr=t["row_ptr"].data_ptr(), target=t["target"].data_ptr(), weight=t["weight"].data_ptr(),
            delay=t["delay"].data_ptr(), out_src=self.out_src.data_ptr(), out_stamp=self.out_stamp.data_ptr(),
            out_cap=self.cap, out_count=self.out_count.data_ptr(), continue_run=continue_run, reserved=0,
            out_skipped=self.out_skipped.data_ptr())

    def call(self, steps, start_step=0, continue_run=0):
        """One call; returns (sources, stamps, spike count, skipped edges)."""
        import torch

        s = self.struct(start_step, continue_run)
        stream = torch.cuda.current_stream(self.dev)
        rc = self.fn(ctypes.byref(s), int(steps), ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, self.L.ng_last_error().decode()
        torch.cuda.synchronize(self.dev)
        k = int(self.out_count.item())
        w = min(k, self.cap)
        return (self.out_src[:w].cpu().numpy(), self.out_stamp[:w].cpu().numpy(), k, int(self.out_skipped.item()))


def _run_noalloc(net, steps, start_step=0):
    na = _NoAlloc(net)
    src, stamp, k, skipped = na.call(steps, start_step)
    assert k <= na.cap and skipped == 0
    return src, stamp, na.V.cpu().numpy()


def _sorted(src, stamp):
    o = np.lexsort((src, stamp))
    return np.asarray(src)[o].astype(np.int64), np.asarray(stamp)[o].astype(np.int64)


def _assert_same(a, b):
    as_, at = _sorted(a[0], a[1])
    bs, bt = _sorted(b[0], b[1])
    np.testing.assert_array_equal(as_, bs)
    np.testing.assert_array_equal(at, bt)
    np.testing.assert_array_equal(a[2], b[2])


def test_noalloc_matches_engine_two_calls(golden):
    fx = golden("c0_delta_balanced.npz")
    for call, ie_scale in enumerate((1.0, 1.05)):
        net = _network(fx, ie_scale)
        eng = _run_engine(net, 3000)
        na = _run_noalloc(net, 3000)
        assert len(eng[0]) > 1000, call
        _assert_same(na, eng)


def test_noalloc_mixed_delays_offset_start_partial_slice(golden):
    """Delays spread over [5, 20] steps (the allocation-free ring holds
    min_delay + max_delay slots, the engine's max_delay), a first slice at
    step 3 * min_delay, and a run that ends 3 steps into a slice."""
    fx = golden("c0_delta_balanced.npz")
    rng = np.random.default_rng(11)
    delays = rng.integers(5, 21, size=len(fx["src"]))
    delays[0], delays[1] = 5, 20
    net = _network(fx, 1.0, delays)
    assert (net["min_delay"], net["max_delay"]) == (5, 20)
    steps = 5 * 400 + 3
    eng = _run_engine(net, steps, start_step=15)
    na = _run_noalloc(net, steps, start_step=15)
    assert len(eng[0]) > 1000
    assert eng[1].min() >= 16
    _assert_same(na, eng)


def test_noalloc_continued_calls_equal_one_call(golden):
    """A controller's chain of short calls (continue_run = 1), stopping and
    resuming inside slices, gives the raster and V_m of one long call."""
    fx = golden("c0_delta_balanced.npz")
    rng = np.random.default_rng(5)
    net = _network(fx, 1.0, rng.integers(5, 21, size=len(fx["src"])))
    total = 1200
    one = _NoAlloc(net)
    s1, t1, k1, _ = one.call(total, start_step=0)
    chain = _NoAlloc(net)
    srcs, stamps = [], []
    pos = 0
    for i, n in enumerate([7, 13, 1, 4, 5, 370, 2, 798]):
        s, t, k, sk = chain.call(n, start_step=pos, continue_run=1 if i else 0)
        assert k == len(s) and sk == 0
        srcs.append(s)
        stamps.append(t)
        pos += n
    assert pos == total and k1 > 500
    _assert_same((np.concatenate(srcs), np.concatenate(stamps), chain.V.cpu().numpy()),
                 (s1, t1, one.V.cpu().numpy()))
    eng = _run_engine(net, total)
    _assert_same((s1, t1, one.V.cpu().numpy()), eng)
    # a continuation that does not start where the previous call stopped
    from nestgpu import _abi

    s = chain.struct(pos + 1, 1)
    assert chain.fn(ctypes.byref(s), 10, None) == _abi.NG_ERR_STATE
    assert "continue_run" in chain.L.ng_last_error().decode()


def test_noalloc_output_capacity(golden):
    """Spikes beyond out_cap are counted, not written; those written are
    spikes of the full run."""
    fx = golden("c0_delta_balanced.npz")
    net = _network(fx, 1.0)
    full = _NoAlloc(net)
    fs, ft, fk, _ = full.call(600)
    small = _NoAlloc(net, cap=100)
    ss, st, sk, _ = small.call(600)
    assert sk == fk > 100 and len(ss) == 100
    have = set(zip(fs.tolist(), ft.tolist()))
    assert all(p in have for p in zip(ss.tolist(), st.tolist()))


def test_noalloc_skips_out_of_range_edges(golden):
    """Edges with a target >= n, a negative target, or a delay above
    max_delay or below min_delay are skipped on the device and counted: the
    run equals the engine's on the network without them."""
    fx = golden("c0_delta_balanced.npz")
    net = _network(fx, 1.0)
    n = net["n"]
    nnz = len(net["target"])
    bad = np.zeros(nnz, dtype=bool)
    rng = np.random.default_rng(3)
    idx = rng.choice(nnz, size=400, replace=False)
    bad[idx] = True
    tg = net["target"].copy()
    d = net["delay"].copy()
    tg[idx[:100]] = n
    tg[idx[100:200]] = -7
    d[idx[200:300]] = net["max_delay"] + 1
    d[idx[300:]] = 0
    net_bad = dict(net, target=tg, delay=d)
    na = _NoAlloc(net_bad)
    s, t, k, skipped = na.call(1500)
    assert skipped > 0
    eng = _run_engine(net, 1500, keep=~bad)
    _assert_same((s, t, na.V.cpu().numpy()), eng)


def test_noalloc_rejects_oversized_network():
    import torch

    from nestgpu import _abi

    L = _abi.load()
    fn = L.ng_simulate_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = dummy.data_ptr()
    s = NoAllocNet(n=10_000_000, min_delay=15, max_delay=15, start_step=0, P33=p, P30=p, V_th_rel=p,
                   V_reset_rel=p, V_min_rel=p, I_e=p, refr_counts=p, V_m_rel=p, r=p, row_ptr=p, target=p,
                   weight=p, delay=p, out_src=p, out_stamp=p, out_cap=0, out_count=p)
    assert fn(ctypes.byref(s), 10, None) == _abi.NG_ERR_CAPACITY
    assert "16 MiB" in L.ng_last_error().decode()
    s2 = NoAllocNet(n=100, min_delay=15, max_delay=15, start_step=0, P33=p, P30=p, V_th_rel=p,
                    V_reset_rel=p, V_min_rel=p, I_e=p, refr_counts=p, V_m_rel=p, r=p, row_ptr=p, target=None,
                    weight=p, delay=p, out_src=p, out_stamp=p, out_cap=0, out_count=p)
    assert fn(ctypes.byref(s2), 10, None) == _abi.NG_ERR_ARG
