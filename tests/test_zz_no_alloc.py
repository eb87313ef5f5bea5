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
check that the second call starts from a cleared scratch array.
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
    ]


def _network(fx, ie_scale):
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
    return {
        "n": n, "P33": np.full(n, P33), "P30": np.full(n, P30), "V_th_rel": np.full(n, V_th - E_L),
        "V_reset_rel": np.full(n, V_reset - E_L), "V_min_rel": np.full(n, -np.finfo(np.float64).max),
        "I_e": fx["I_e"] * ie_scale, "refr": np.full(n, refr, dtype=np.int32), "V0": fx["V0"] - E_L,
        "row_ptr": row_ptr, "target": fx["tgt"].astype(np.int32)[order],
        "weight": np.where(fx["exc"], 0.125, -0.625)[order], "delay": np.full(len(src), 15, dtype=np.int32),
        "params": (C_m, tau_m, t_ref, E_L, V_th, V_reset),
    }


def _run_engine(net, steps):
    """The regular entry points: ng_create, ng_set_*, ng_simulate."""
    from nestgpu import _abi

    n = net["n"]
    C_m, tau_m, t_ref, E_L, V_th, V_reset = net["params"]
    eng = _abi.Engine([(_abi.NG_IAF_PSC_DELTA, n)], 0.1, 15, 15)
    for name, val in (("C_m", C_m), ("tau_m", tau_m), ("t_ref", t_ref), ("V_th_rel", V_th - E_L),
                      ("V_reset_rel", V_reset - E_L)):
        eng.set_var(0, name, np.full(n, val))
    eng.set_var(0, "I_e", net["I_e"])
    eng.set_var(0, "V_m_rel", net["V0"])
    eng.set_connections(net["row_ptr"], net["target"], net["weight"], net["delay"])
    eng.set_recording(np.ones(n, dtype=np.uint8))
    eng.simulate(steps)
    src, stamp = eng.spikes()
    V = eng.get_var(0, "V_m_rel")
    eng.close()
    return src, stamp, V


def _run_noalloc(net, steps):
    import torch

    from nestgpu import _abi

    L = _abi.load()
    fn = L.ng_simulate_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    dev = torch.device("cuda", 0)
    t = {k: torch.as_tensor(np.ascontiguousarray(v)).to(dev)
         for k, v in net.items() if isinstance(v, np.ndarray)}
    V = t["V0"].clone()
    r = torch.zeros(net["n"], dtype=torch.int32, device=dev)
    cap = 200000
    out_src = torch.empty(cap, dtype=torch.int32, device=dev)
    out_stamp = torch.empty(cap, dtype=torch.int64, device=dev)
    out_count = torch.zeros(1, dtype=torch.int64, device=dev)
    s = NoAllocNet(n=net["n"], min_delay=15, max_delay=15, start_step=0,
                   P33=t["P33"].data_ptr(), P30=t["P30"].data_ptr(), V_th_rel=t["V_th_rel"].data_ptr(),
                   V_reset_rel=t["V_reset_rel"].data_ptr(), V_min_rel=t["V_min_rel"].data_ptr(),
                   I_e=t["I_e"].data_ptr(), refr_counts=t["refr"].data_ptr(), V_m_rel=V.data_ptr(),
                   r=r.data_ptr(), row_ptr=t["row_ptr"].data_ptr(), target=t["target"].data_ptr(),
                   weight=t["weight"].data_ptr(), delay=t["delay"].data_ptr(), out_src=out_src.data_ptr(),
                   out_stamp=out_stamp.data_ptr(), out_cap=cap, out_count=out_count.data_ptr())
    stream = torch.cuda.current_stream(dev)
    rc = fn(ctypes.byref(s), int(steps), ctypes.c_void_p(stream.cuda_stream))
    assert rc == 0, L.ng_last_error().decode()
    torch.cuda.synchronize(dev)
    k = int(out_count.item())
    assert k <= cap
    return out_src[:k].cpu().numpy(), out_stamp[:k].cpu().numpy(), V.cpu().numpy()


def _sorted(src, stamp):
    o = np.lexsort((src, stamp))
    return np.asarray(src)[o].astype(np.int64), np.asarray(stamp)[o].astype(np.int64)


def test_noalloc_matches_engine_two_calls(golden):
    fx = golden("c0_delta_balanced.npz")
    for call, ie_scale in enumerate((1.0, 1.05)):
        net = _network(fx, ie_scale)
        es, et, eV = _run_engine(net, 3000)
        ns, nt, nV = _run_noalloc(net, 3000)
        es, et = _sorted(es, et)
        ns, nt = _sorted(ns, nt)
        assert len(es) > 1000, call
        np.testing.assert_array_equal(ns, es)
        np.testing.assert_array_equal(nt, et)
        np.testing.assert_array_equal(nV, eV)


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
