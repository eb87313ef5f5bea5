"""Parity of the CUDA engine with the reference (golden fixtures produced by
running the reference) and with the CPU oracle, through the C ABI.

Bars:
- plain FP64 form, deterministic inputs with order-independent ring sums:
  bit-exact spike raster and state (config 0; dyadic iaf_psc_exp net);
- plain FP64 form with real-valued weights: membrane traces within 1e-12
  relative of the reference (order of FP64 atomic ring adds may differ);
- generator timing cases of the reference's own tests.
"""

import numpy as np
import pytest

from netbuild import build_c0, build_exp_net, raster

pytestmark = pytest.mark.gpu


def test_c0_raster_bit_exact(nest, golden):
    fx = golden("c0_delta_balanced.npz")
    pop, sr = build_c0(nest, fx)
    nest.Simulate(1000.0)
    s, t = raster(sr)
    assert len(s) == len(fx["spike_senders"])
    np.testing.assert_array_equal(s - 1, fx["spike_senders"].astype(np.int64))
    np.testing.assert_array_equal(t, fx["spike_steps"].astype(np.int64))
    V = np.asarray(pop.get("V_m"))
    np.testing.assert_array_equal(V, fx["V_end"])
    assert nest.GetKernelStatus("local_spike_counter") == len(fx["spike_senders"])


def test_c0_stepped_equals_single_run(nest, golden):
    """Simulate(1000) == 4 x Simulate(250) incl. partial slices (test_stepped_simulation)."""
    fx = golden("c0_delta_balanced.npz")
    pop, sr = build_c0(nest, fx)
    for _ in range(4):
        nest.Simulate(250.0)
    s, t = raster(sr)
    np.testing.assert_array_equal(s - 1, fx["spike_senders"].astype(np.int64))
    np.testing.assert_array_equal(t, fx["spike_steps"].astype(np.int64))
    # partial slices (0.7 ms is not a multiple of min_delay 1.5 ms)
    pop, sr = build_c0(nest, fx)
    for _ in range(100):
        nest.Simulate(0.7)
    nest.Simulate(1000.0 - 70.0)
    s, t = raster(sr)
    np.testing.assert_array_equal(t, fx["spike_steps"].astype(np.int64))
    np.testing.assert_array_equal(s - 1, fx["spike_senders"].astype(np.int64))


def test_c0_without_graphs(nest, golden):
    fx = golden("c0_delta_balanced.npz")
    pop, sr = build_c0(nest, fx)
    nest.set(graph_slices=0)
    nest.Simulate(1000.0)
    s, t = raster(sr)
    np.testing.assert_array_equal(t, fx["spike_steps"].astype(np.int64))
    np.testing.assert_array_equal(s - 1, fx["spike_senders"].astype(np.int64))


@pytest.mark.parametrize("name", ["exp_dyadic_net.npz", "exp_real_net.npz"])
def test_exp_net_against_reference(nest, golden, name):
    fx = golden(name)
    pop, sr, mm = build_exp_net(nest, fx)
    nest.Simulate(200.0)
    s, t = raster(sr)
    np.testing.assert_array_equal(s - 1, fx["spike_senders"].astype(np.int64))
    np.testing.assert_array_equal(t, fx["spike_steps"].astype(np.int64))
    ev = mm.events
    ms = np.asarray(ev["senders"]) - 1
    mt = np.asarray(ev["times"])
    o = np.lexsort((ms, mt))
    np.testing.assert_array_equal(ms[o], fx["mm_senders"])
    np.testing.assert_array_equal(mt[o], fx["mm_times"])
    for key, ref in (("V_m", fx["mm_V"]), ("I_syn_ex", fx["mm_Iex"]), ("I_syn_in", fx["mm_Iin"])):
        got = np.asarray(ev[key])[o]
        if "dyadic" in name:
            np.testing.assert_array_equal(got, ref)
        else:
            # FP64 atomics may sum a slot in another order: 1e-12 relative
            np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
    V = np.asarray(pop.get("V_m"))
    if "dyadic" in name:
        np.testing.assert_array_equal(V, fx["V_end"])
    else:
        np.testing.assert_allclose(V, fx["V_end"], rtol=1e-12)


def test_compare_delta_spike_time(nest, golden):
    """recording/test_compare_delta.py: spike at exactly 4.1 ms (h = 0.01)."""
    fx = golden("single_neuron_cases.npz")
    nest.ResetKernel()
    nest.resolution = 0.01
    n = nest.Create("iaf_psc_delta", params={"E_L": -49.0, "V_m": -60.0, "V_th": -50.0, "V_reset": -60.0,
                                             "C_m": 200.0, "tau_m": 20.0, "t_ref": 5.0})
    sg = nest.Create("spike_generator", params={"spike_times": [1.0, 2.0, 3.0, 4.0, 5.0, 10.5, 12.0]})
    sr = nest.Create("spike_recorder")
    vm = nest.Create("voltmeter", params={"interval": 0.01})
    nest.SetDefaults("static_synapse", {"delay": 0.1, "weight": 2.5})
    nest.Connect(sg, n)
    nest.Connect(n, sr)
    nest.Connect(vm, n)
    nest.Simulate(200.0)
    np.testing.assert_array_equal(np.asarray(sr.events["times"]), fx["cmpdelta_spike_times"])
    assert np.asarray(sr.events["times"])[0] == pytest.approx(4.1)
    v = np.asarray(vm.events["V_m"])[:3000]
    np.testing.assert_array_equal(np.asarray(vm.events["times"])[:3000], fx["cmpdelta_vm_times"])
    np.testing.assert_array_equal(v, fx["cmpdelta_vm_V"])


@pytest.mark.parametrize("h", [0.001, 0.1])
@pytest.mark.parametrize("tau_m", [1.0, 10.0, 100.0])
def test_iaf_psc_exp_singularity(nest, golden, h, tau_m):
    """neurons/test_iaf_singularity.py: tau_syn = tau_m +- eps, smooth V_m,
    and the reference's own trace at its sample points."""
    fx = golden("single_neuron_cases.npz")
    key = f"sing_h{h}_tau{tau_m}"
    tau_syn = fx[key + "_tau_syn"]
    nest.ResetKernel()
    nest.resolution = h
    neurons = nest.Create("iaf_psc_exp", n=len(tau_syn),
                          params={"tau_m": tau_m, "tau_syn_ex": tau_syn, "tau_syn_in": tau_syn, "V_th": np.inf})
    sg = nest.Create("spike_generator", params={"spike_times": [1.0]})
    vm = nest.Create("voltmeter", params={"interval": h})
    nest.Connect(sg, neurons, syn_spec={"weight": 1000.0, "delay": 1.0})
    nest.Connect(sg, neurons, syn_spec={"weight": -1000.0, "delay": 2.0})
    nest.Connect(vm, neurons)
    nest.Simulate(10 * tau_m)
    ev = vm.events
    s = np.asarray(ev["senders"])
    t = np.asarray(ev["times"])
    v = np.asarray(ev["V_m"])
    o = np.lexsort((s, t))
    V = v[o].reshape(-1, len(tau_syn))
    assert not np.any(np.isnan(V))
    V_range = V.max() - V.min()
    assert V_range > 1
    dV = np.abs(np.diff(V, axis=0)).max(axis=0)
    assert np.all(dV < 3 * V_range * h)
    stride = int(fx[key + "_stride"])
    ref = fx[key + "_V"]
    np.testing.assert_allclose(V[::stride][:len(ref)], ref, rtol=1e-12, atol=1e-12)


def test_iaf_psc_exp_dc_trace(nest, golden):
    """neurons/test_iaf_psc_exp.py-style DC drive incl. refractoriness."""
    fx = golden("single_neuron_cases.npz")
    nest.ResetKernel()
    nest.resolution = 0.1
    n = nest.Create("iaf_psc_exp", params={"I_e": 1000.0, "tau_syn_ex": 0.5, "tau_syn_in": 0.5})
    vm = nest.Create("voltmeter", params={"interval": 0.1})
    sr = nest.Create("spike_recorder")
    nest.Connect(vm, n)
    nest.Connect(n, sr)
    nest.Simulate(100.0)
    np.testing.assert_array_equal(np.asarray(vm.events["times"]), fx["dcexp_vm_times"])
    np.testing.assert_array_equal(np.asarray(vm.events["V_m"]), fx["dcexp_vm_V"])
    np.testing.assert_array_equal(np.asarray(sr.events["times"]), fx["dcexp_spike_times"])
