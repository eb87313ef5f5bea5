"""iaf_psc_alpha on the engine (FP64): the reference test suite's expected
DC traces and spike times (tests/golden/iaf_psc_alpha_kat.npz, rtol 1e-6),
the analytic alpha PSP of a transmitted spike (rtol 1e-12, as
testsuite/pytests/neurons/test_iaf_psc_alpha_1to2.py), and a Poisson-driven
network with dyadic weights bit-identical to the CPU oracle."""

import numpy as np
import pytest

import oracle as O
from test_alpha_oracle import _join, vm_theory

pytestmark = pytest.mark.gpu


def _trace(mm, n_rec=1):
    ev = mm.events
    o = np.lexsort((ev["senders"], ev["times"]))
    return np.asarray(ev["times"])[o], np.asarray(ev["V_m"])[o]


def test_alpha_dc_trace_and_spike_on_gpu(nest, golden):
    fx = golden("iaf_psc_alpha_kat.npz")
    nest.set(resolution=0.1)
    n = nest.Create("iaf_psc_alpha", params={"I_e": 1000.0})
    vm = nest.Create("voltmeter", params={"interval": 0.1})
    sr = nest.Create("spike_recorder")
    nest.Connect(vm, n)
    nest.Connect(n, sr)
    nest.Simulate(8.0)
    t, V = _trace(vm)
    got, exp = _join(0.1, t, V, fx["i0_vm"])
    assert len(got) == len(fx["i0_vm"])
    np.testing.assert_allclose(got, exp, rtol=1e-6)
    np.testing.assert_allclose(np.asarray(sr.events["times"]), fx["i0_spikes"][:, 1])


@pytest.mark.parametrize("h", [0.1, 0.2, 0.5, 1.0])
def test_alpha_refractory_alignment_on_gpu(nest, golden, h):
    fx = golden("iaf_psc_alpha_kat.npz")
    nest.set(resolution=h)
    n = nest.Create("iaf_psc_alpha", params={"I_e": 1450.0})
    vm = nest.Create("voltmeter", params={"interval": h})
    nest.Connect(vm, n)
    nest.Simulate(8.0)
    t, V = _trace(vm)
    got, exp = _join(h, t, V, fx["i0_refractory_vm"])
    assert len(got) >= 6
    np.testing.assert_allclose(got, exp, rtol=1e-6)


@pytest.mark.parametrize("h", [0.1, 0.2, 0.5, 1.0])
def test_alpha_psp_matches_analytic_solution_on_gpu(nest, h):
    nest.set(resolution=h)
    n1, n2 = nest.Create("iaf_psc_alpha", 2)
    n1.I_e = 1450.0
    sr = nest.Create("spike_recorder")
    vm = nest.Create("voltmeter", params={"interval": h})
    nest.Connect(n1, sr)
    nest.Connect(vm, n2)
    nest.Connect(n1, n2, syn_spec={"weight": 100.0, "delay": 1.0})
    nest.Simulate(8.0)
    assert list(np.rint(np.asarray(sr.events["times"]) / h).astype(int)) == [round(3.0 / h), round(8.0 / h)]
    t, V = _trace(vm)
    pre = t <= 4.0 + 1e-9
    np.testing.assert_array_equal(V[pre], -70.0)
    post = ~pre | np.isclose(t, 4.0)
    np.testing.assert_allclose(V[post], vm_theory(t[post] - 4.0, 250.0, 10.0, 2.0, -70.0, 100.0), rtol=1e-12)


def test_alpha_network_bit_exact_vs_oracle(nest):
    """1,500 Poisson-driven iaf_psc_alpha neurons, random graph with delays
    of 1.5-3.5 ms and dyadic weights: the engine's raster and final V_m
    equal the oracle's (ring sums are order independent)."""
    from nestgpu.kernel import KERNEL

    nest.set(resolution=0.1, rng_seed=91)
    N = 1500
    pop = nest.Create("iaf_psc_alpha", N, params={"tau_syn_ex": 0.5, "tau_syn_in": 1.0})
    pop.set(V_m=np.random.default_rng(5).uniform(-70.0, -56.0, N))
    rng = np.random.default_rng(6)
    src = rng.integers(0, N, 120_000)
    tgt = rng.integers(0, N, 120_000)
    w = rng.choice([32.0, 16.5, -64.0, -128.25], 120_000, p=[0.4, 0.4, 0.1, 0.1])
    d = rng.integers(15, 36, 120_000) * 0.1
    nest.Connect(src + 1, tgt + 1, "one_to_one", {"weight": w, "delay": d})
    pg = nest.Create("poisson_generator", params={"rate": 9000.0})
    nest.Connect(pg, pop, syn_spec={"weight": 40.0, "delay": 1.5})
    sr = nest.Create("spike_recorder")
    nest.Connect(pop, sr)
    net, c = O.net_from_kernel(KERNEL)
    nest.Simulate(500.0)
    net.run(5000)
    ev = sr.events
    s = np.asarray(ev["senders"], dtype=np.int64) - 1
    st = np.rint(np.asarray(ev["times"]) / 0.1).astype(np.int64)
    os_, ost = net.spikes()
    assert len(s) > 2000
    o1, o2 = np.lexsort((s, st)), np.lexsort((os_, ost))
    np.testing.assert_array_equal(s[o1], os_[o2])
    np.testing.assert_array_equal(st[o1], ost[o2])
    np.testing.assert_array_equal(np.asarray(pop.get("V_m")), net.get("V_m_rel") - 70.0)
