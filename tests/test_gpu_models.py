"""GPU tests of the Poisson drive, the precision form, aeif_cond_alpha and
the statistical oracle (the engine against the reference's statistics and
against the CPU oracle on the same network)."""

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _cv_isi(senders, stamps, n, h):
    o = np.lexsort((stamps, senders))
    s, t = senders[o], stamps[o] * h
    cv = np.full(n, np.nan)
    starts = np.searchsorted(s, np.arange(n))
    ends = np.searchsorted(s, np.arange(n), side="right")
    for i in range(n):
        ts = t[starts[i]:ends[i]]
        if len(ts) >= 3:
            isi = np.diff(ts)
            cv[i] = isi.std() / isi.mean()
    return cv


def _engine_raster(nest, sr):
    ev = sr.events
    s = np.asarray(ev["senders"], dtype=np.int64) - 1
    st = np.rint(np.asarray(ev["times"]) / 0.1).astype(np.int64)
    return s, st


def test_poisson_drive_bit_exact_vs_oracle(nest):
    """Feed-forward Poisson-driven iaf_psc_exp neurons: the engine's Philox
    drive and sampler give the oracle's values exactly (FP64 form)."""
    from nestgpu.kernel import KERNEL

    nest.set(resolution=0.1, rng_seed=2024)
    pop = nest.Create("iaf_psc_exp", 3000, params={"tau_syn_ex": 0.5, "tau_syn_in": 0.5})
    pop.set(V_m=np.random.default_rng(3).uniform(-70, -56, 3000))
    pg = nest.Create("poisson_generator", params={"rate": 15000.0})
    nest.Connect(pg, pop, syn_spec={"weight": 87.8, "delay": 1.0})
    sr = nest.Create("spike_recorder")
    nest.Connect(pop, sr)
    net, c = O.net_from_kernel(KERNEL)
    nest.Simulate(300.0)
    net.run(3000)
    s, st = _engine_raster(nest, sr)
    os_, ost = net.spikes()
    assert len(s) > 1000
    o1 = np.lexsort((s, st))
    o2 = np.lexsort((os_, ost))
    np.testing.assert_array_equal(s[o1], os_[o2])
    np.testing.assert_array_equal(st[o1], ost[o2])
    np.testing.assert_array_equal(np.asarray(pop.get("V_m")), net.get("V_m_rel") - 70.0)


def test_c1_fp64_statistics_vs_reference(nest, golden):
    """Config-1 network, plain FP64 form: mean rate inside the reference's
    spread over realizations, CV-ISI distribution matching (KS)."""
    from scipy import stats

    from nestgpu import workloads

    fx = golden("c1_exp_poisson_stats.npz")
    pop, sr = workloads.c1(nest, precision="fp64")
    nest.Simulate(1000.0)
    s, st = _engine_raster(nest, sr)
    rate = len(s) / 12500
    ref_rates = np.concatenate([fx["seed_rates"], [fx["counts"].mean()]])
    lo, hi = ref_rates.min(), ref_rates.max()
    spread = hi - lo
    assert lo - spread / 2 <= rate <= hi + spread / 2, (rate, ref_rates)
    cv = _cv_isi(s, st, 12500, 0.1)
    ref_cv = fx["cv"][~np.isnan(fx["cv"])]
    assert abs(np.nanmean(cv) - np.mean(fx["seed_mean_cv"])) < 0.03
    assert stats.ks_2samp(cv[~np.isnan(cv)], ref_cv).statistic < 0.05


def test_c1_engine_vs_oracle_same_network(nest):
    """The same graph and drive on the engine (FP64) and the CPU oracle:
    rates within 2 %, mean CV-ISI within 0.02 (trajectories decorrelate
    because FP64 atomics sum a ring slot in varying order)."""
    from nestgpu import workloads
    from nestgpu.kernel import KERNEL

    pop, sr = workloads.c1(nest, precision="fp64")
    net, c = O.net_from_kernel(KERNEL)
    nest.Simulate(1000.0)
    net.run(10000)
    s, st = _engine_raster(nest, sr)
    os_, ost = net.spikes()
    assert abs(len(s) / len(os_) - 1) < 0.02
    cv_e = np.nanmean(_cv_isi(s, st, 12500, 0.1))
    cv_o = np.nanmean(_cv_isi(os_.astype(np.int64), ost, 12500, 0.1))
    assert abs(cv_e - cv_o) < 0.02
    # syn events = sum of out-degrees of the spikes
    ev = nest.engine_stats()["syn_events"]
    assert ev == net.syn_events or abs(ev / net.syn_events - 1) < 0.02


def test_aeif_against_lsodar_on_gpu(nest, golden):
    """neurons/test_aeif_lsodar.py on the engine: mean relative difference
    to the LSODAR reference < 5e-4 (V_m) and < 1e-4 (w)."""
    from scipy.interpolate import interp1d

    fx = golden("aeif_lsodar.npz")
    p = {"V_reset": -58.0, "V_peak": 0.0, "V_th": -50.0, "I_e": 420.0, "g_L": 11.0, "tau_w": 300.0, "E_L": -70.0,
         "Delta_T": 2.0, "a": 3.0, "b": 0.0, "C_m": 200.0, "V_m": -70.0, "w": 5.0}
    nest.resolution = 0.01
    n = nest.Create("aeif_cond_alpha", params=p)
    mm = nest.Create("multimeter", params={"interval": 0.01, "record_from": ["V_m", "w"]})
    nest.Connect(mm, n)
    nest.Simulate(100.0)
    ev = mm.events
    t = np.asarray(ev["times"])
    V = np.asarray(ev["V_m"])
    W = np.asarray(ev["w"])
    ref_V = interp1d(fx["t"], fx["V_m"])(t)
    ref_w = interp1d(fx["t"], fx["w"])(t)
    V_lim = (p["V_th"] + p["V_peak"]) / 2.0

    def rel(ref, x, isV):
        nz = ~np.isclose(ref, 0.0)
        r = np.abs(ref - x)[nz] / np.abs(ref[nz])
        if isV:
            r = r[~(x[nz] > V_lim)]
        return r.mean()

    assert rel(ref_V, V, True) < 5e-4
    assert rel(ref_w, W, False) < 1e-4


def test_aeif_network_vs_oracle(nest):
    """A small Poisson-driven aeif_cond_alpha network on the engine and the
    oracle: same graph and drive, spike counts within 8 % (a small chaotic
    network: the two trajectories decorrelate)."""
    from nestgpu.kernel import KERNEL

    nest.set(resolution=0.1, rng_seed=77)
    N, NE = 1000, 800
    pop = nest.Create("aeif_cond_alpha", N, params={"a": 4.0, "b": 80.5, "tau_w": 144.0, "Delta_T": 2.0,
                                                    "I_e": 700.0})
    nest.Connect(pop[:NE], pop, {"rule": "fixed_indegree", "indegree": 80}, {"weight": 1.0, "delay": 1.5})
    nest.Connect(pop[NE:], pop, {"rule": "fixed_indegree", "indegree": 20}, {"weight": -5.0, "delay": 1.5})
    pg = nest.Create("poisson_generator", params={"rate": 10000.0})
    nest.Connect(pg, pop, syn_spec={"weight": 0.5, "delay": 1.5})
    sr = nest.Create("spike_recorder")
    nest.Connect(pop, sr, syn_spec={"delay": 1.5})
    net, c = O.net_from_kernel(KERNEL)
    nest.Simulate(300.0)
    net.run(3000)
    s, st = _engine_raster(nest, sr)
    os_, ost = net.spikes()
    assert len(os_) > 100
    assert abs(len(s) / len(os_) - 1) < 0.08


def test_numerical_instability_reported(nest):
    """A diverging aeif neuron raises the reference's NumericalInstability
    (aeif_cond_alpha.cpp:481-490) through the C ABI's error status."""
    from nestgpu import _abi

    n = nest.Create("aeif_cond_alpha", params={"I_e": -1e7})
    with pytest.raises(_abi.EngineError) as ei:
        nest.Simulate(50.0)
    assert ei.value.code == _abi.NG_ERR_NUMERIC
    assert "NumericalInstability" in str(ei.value)
