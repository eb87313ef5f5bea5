"""ng_update: the slice-aligned entry point a NEST node's update(origin,
from, to) maps onto (nestkernel/node.h:297).  Driving the network slice by
slice -- in partial slices too, mixed with ng_simulate -- gives the raster and
state of one ng_simulate call bit for bit (the golden balanced network's
dyadic weights make the FP64 ring sums order independent), and a call that
does not start where the engine stands is refused."""

import numpy as np
import pytest

from nestgpu import _abi

pytestmark = pytest.mark.gpu


def _engine(fx):
    C_m, tau_m, t_ref, E_L, V_th, V_reset = (float(x) for x in fx["params"])
    n = len(fx["I_e"])
    src = fx["src"].astype(np.int64)
    order = np.argsort(src, kind="stable")
    row = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(src, minlength=n), out=row[1:])
    eng = _abi.Engine([(_abi.NG_IAF_PSC_DELTA, n)], 0.1, 15, 15)
    for name, val in (("C_m", C_m), ("tau_m", tau_m), ("t_ref", t_ref), ("V_th_rel", V_th - E_L),
                      ("V_reset_rel", V_reset - E_L)):
        eng.set_var(0, name, np.full(n, val))
    eng.set_var(0, "I_e", fx["I_e"])
    eng.set_var(0, "V_m_rel", fx["V0"] - E_L)
    eng.set_connections(row, fx["tgt"].astype(np.int32)[order], np.where(fx["exc"], 0.125, -0.625)[order],
                        np.full(len(src), 15, dtype=np.int32))
    eng.set_recording(np.ones(n, dtype=np.uint8))
    return eng


def _result(eng):
    eng.sync()
    s, t = eng.spikes()
    V = eng.get_var(0, "V_m_rel")
    st = eng.stats()
    eng.close()
    o = np.lexsort((s, t))
    return s[o], t[o], V, st


def test_update_slice_by_slice_equals_simulate(golden):
    fx = golden("c0_delta_balanced.npz")
    ref = _engine(fx)
    ref.simulate(6000)
    a = _result(ref)
    eng = _engine(fx)
    origin = 0
    k = 0
    while origin < 3000:
        if k % 7 == 3:                     # a slice in three calls
            for frm, to in ((0, 4), (4, 5), (5, 15)):
                eng.update(origin, frm, to)
        else:
            eng.update(origin, 0, 15)
        origin += 15
        k += 1
    eng.simulate(1500)                     # then the bulk path, then slices again
    origin += 1500
    while origin < 6000:
        eng.update(origin, 0, 15)
        origin += 15
    b = _result(eng)
    assert len(a[0]) > 5000
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])
    np.testing.assert_array_equal(a[2], b[2])
    assert a[3]["syn_events"] == b[3]["syn_events"]
    assert b[3]["clock_steps"] == 6000


def test_update_refuses_misaligned_calls(golden):
    fx = golden("c0_delta_balanced.npz")
    eng = _engine(fx)
    eng.update(0, 0, 7)
    for bad in ((0, 0, 15), (15, 7, 15), (0, 8, 15)):
        with pytest.raises(_abi.EngineError) as ei:
            eng.update(*bad)
        assert ei.value.code == _abi.NG_ERR_STATE
    with pytest.raises(_abi.EngineError) as ei:
        eng.update(0, 7, 16)               # beyond the slice
    assert ei.value.code == _abi.NG_ERR_ARG
    eng.update(0, 7, 15)
    eng.close()
