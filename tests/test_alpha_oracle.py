"""iaf_psc_alpha on the CPU oracle, pinned to the reference: its propagator
equals the reference's own IAFPropagatorAlpha compiled from its sources
(bit for bit, singular branches included); the DC traces and spike time
equal the expected values of the reference test suite
(testsuite/pytests/neurons/test_iaf_psc_alpha.py, stored in
tests/golden/iaf_psc_alpha_kat.npz, rtol 1e-6 as there); and the
postsynaptic potential of a spike follows the analytic alpha-PSP solution
to 1e-12 relative (testsuite/pytests/neurons/test_iaf_psc_alpha_1to2.py)."""

import ctypes
import os

import numpy as np
import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libnestprop.so")


def _single(I_e, h, t_ms):
    steps = int(round(t_ms / h))
    net = O.OracleNet("iaf_psc_alpha", 1, h, 1, 1)
    net.set("I_e", I_e)
    net.set_record(np.ones(1, dtype=np.uint8))
    net.set_trace([0], "V_m_rel")
    net.run(steps)
    V = net.trace()[:, 0] - 70.0
    times = (np.arange(steps) + 1) * h
    s, st = net.spikes()
    return times, V, st * h


def _join(h, times, V, expected):
    """Rows of `expected` (time, value) at the recorded times (the reference
    test's get_comparable_timesamples: an inner join on steps)."""
    steps = np.rint(times / h).astype(np.int64)
    e_steps = np.rint(expected[:, 0] / h).astype(np.int64)
    e_ok = np.isclose(expected[:, 0] / h, e_steps)
    common, ia, ib = np.intersect1d(steps, e_steps[e_ok], return_indices=True)
    return V[ia], expected[e_ok][ib, 1]


def test_alpha_propagator_equals_reference():
    if not os.path.exists(REF_LIB):
        pytest.skip("oracle/_ref not built (the reference's sources are not on this machine)")
    ref = ctypes.CDLL(REF_LIB)
    ref.ref_iaf_propagator_alpha.argtypes = [ctypes.c_double] * 4 + [ctypes.c_void_p]
    ref.ref_iaf_propagator_alpha.restype = None
    L = O.lib()
    a = np.zeros(2)
    b = np.zeros(2)
    n_singular = 0
    for h in (0.001, 0.01, 0.1, 1.0):
        for tau_m in (1.0, 10.0, 100.0):
            for eps in (0.0, 1e-15, 1e-12, 1e-10, 1e-7, 1e-4, 1e-1, -1e-12, -1e-7, -0.5):
                tau_s = tau_m * (1 + eps)
                ref.ref_iaf_propagator_alpha(tau_s, tau_m, 250.0, h, a.ctypes.data)
                L.orc_iaf_propagator_alpha(tau_s, tau_m, 250.0, h, b.ctypes.data)
                assert a.tobytes() == b.tobytes(), (h, tau_m, eps, a, b)
                n_singular += abs(eps) < 1e-9
    assert n_singular > 0


def test_alpha_dc_trace_and_spike(golden):
    fx = golden("iaf_psc_alpha_kat.npz")
    times, V, spikes = _single(1000.0, 0.1, 8.0)
    got, exp = _join(0.1, times, V, fx["i0_vm"])
    assert len(got) == len(fx["i0_vm"])
    np.testing.assert_allclose(got, exp, rtol=1e-6)
    np.testing.assert_allclose(spikes, fx["i0_spikes"][:, 1])


@pytest.mark.parametrize("h", [0.1, 0.2, 0.5, 1.0])
def test_alpha_refractory_alignment(golden, h):
    fx = golden("iaf_psc_alpha_kat.npz")
    times, V, spikes = _single(1450.0, h, 8.0)
    got, exp = _join(h, times, V, fx["i0_refractory_vm"])
    assert len(got) >= 6
    np.testing.assert_allclose(got, exp, rtol=1e-6)


def vm_theory(t, C_m, tau_m, tau_syn, E_L, w):
    """V_m of an iaf_psc_alpha neuron at rest after one alpha-shaped
    current of weight w at t = 0 (solution of the linear membrane equation
    driven by w e t / tau_syn exp(-t / tau_syn))."""
    a = 1 / tau_syn - 1 / tau_m
    pref = w * np.e / (tau_syn * C_m)
    return E_L + pref * ((np.exp(-t / tau_m) - np.exp(-t / tau_syn)) / a ** 2 - t * np.exp(-t / tau_syn) / a)


@pytest.mark.parametrize("h,min_delay", [(0.1, 1.0), (0.2, 1.0), (0.5, 1.0), (1.0, 1.0), (0.1, 0.1), (0.1, 0.5)])
def test_alpha_psp_matches_analytic_solution(h, min_delay):
    md = int(round(min_delay / h))
    d = int(round(1.0 / h))
    net = O.OracleNet("iaf_psc_alpha", 2, h, md, d)
    net.set("I_e", np.array([1450.0, 0.0]))
    net.set_edges(np.array([0]), np.array([1]), np.array([100.0]), np.array([d]))
    net.set_record(np.ones(2, dtype=np.uint8))
    net.set_trace([1], "V_m_rel")
    steps = int(round(8.0 / h))
    net.run(steps)
    s, st = net.spikes()
    assert list(st[s == 0]) == [round(3.0 / h), round(8.0 / h)]
    V = net.trace()[:, 0] - 70.0
    stamps = np.arange(steps) + 1
    arrive = round(4.0 / h)
    np.testing.assert_array_equal(V[stamps <= arrive], -70.0)
    post = stamps >= arrive
    t = stamps[post] * h - 4.0
    np.testing.assert_allclose(V[post], vm_theory(t, 250.0, 10.0, 2.0, -70.0, 100.0), rtol=1e-12)
