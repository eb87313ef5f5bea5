"""The CPU oracle pinned to the reference: golden rasters and traces produced
by running the reference, the reference test suite's own LSODAR data and
Random123 known-answer vectors, and the reference's propagator code compiled
from its sources (oracle/_ref, when built)."""

import ctypes
import os

import numpy as np
import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("nthreads", [1, 3])
def test_c0_raster_bit_exact(golden, nthreads):
    fx = golden("c0_delta_balanced.npz")
    net = O.c0_network(fx, nthreads=nthreads)
    net.run(10000, nthreads=nthreads)
    s, t = net.spikes()
    o = np.lexsort((s, t))
    np.testing.assert_array_equal(s[o], fx["spike_senders"].astype(np.int32))
    np.testing.assert_array_equal(t[o], fx["spike_steps"].astype(np.int64))
    np.testing.assert_array_equal(net.get("V_m_rel") + fx["params"][3], fx["V_end"])


@pytest.mark.parametrize("name", ["exp_dyadic_net.npz", "exp_real_net.npz"])
def test_exp_nets_bit_exact(golden, name):
    fx = golden(name)
    n = len(fx["I_e"])
    net = O.OracleNet("iaf_psc_exp", n, 0.1, int(round(fx["min_delay"] / 0.1)), int(round(fx["max_delay"] / 0.1)))
    net.set("tau_syn_ex", 0.5)
    net.set("tau_syn_in", 0.5)
    net.set("I_e", fx["I_e"])
    net.set("V_m_rel", fx["V0"] + 70.0)
    net.set_edges(fx["src"], fx["tgt"], fx["w"], np.rint(fx["d"] / 0.1).astype(np.int32), nthreads=1)
    net.set_trace(fx["rec_idx"], "V_m_rel")
    net.run(2000, nthreads=1)
    s, t = net.spikes()
    o = np.lexsort((s, t))
    np.testing.assert_array_equal(s[o], fx["spike_senders"])
    np.testing.assert_array_equal(t[o], fx["spike_steps"])
    tr = net.trace() - 70.0
    steps = np.rint(fx["mm_times"] / 0.1).astype(int) - 1
    col = {r: i for i, r in enumerate(fx["rec_idx"])}
    mine = tr[steps, [col[x] for x in fx["mm_senders"]]]
    np.testing.assert_array_equal(mine, fx["mm_V"])


def test_aeif_against_lsodar(golden):
    """neurons/test_aeif_lsodar.py: mean relative difference to the LSODAR
    reference below 5e-4 (V_m, away from spikes) and 1e-4 (w)."""
    from scipy.interpolate import interp1d

    fx = golden("aeif_lsodar.npz")
    p = {"V_reset": -58.0, "V_peak": 0.0, "V_th": -50.0, "I_e": 420.0, "g_L": 11.0, "tau_w": 300.0, "E_L": -70.0,
         "Delta_T": 2.0, "a": 3.0, "b": 0.0, "C_m": 200.0, "V_m": -70.0, "w": 5.0}
    out = {}
    for var in ("V_m", "w"):
        net = O.OracleNet("aeif_cond_alpha", 1, 0.01, 100, 100)
        for k, v in p.items():
            net.set(k, v)
        net.set("integration_step", 0.01)
        net.set_trace([0], var)
        net.run(10000)
        out[var] = net.trace()[:, 0]
    times = (np.arange(10000) + 1) * 0.01
    m = times <= 99.0 + 1e-9
    ref_V = interp1d(fx["t"], fx["V_m"])(times[m])
    ref_w = interp1d(fx["t"], fx["w"])(times[m])
    V, W = out["V_m"][m], out["w"][m]
    V_lim = (p["V_th"] + p["V_peak"]) / 2.0

    def rel(ref, x, isV):
        nz = ~np.isclose(ref, 0.0)
        r = np.abs(ref - x)[nz] / np.abs(ref[nz])
        if isV:
            r = r[~(x[nz] > V_lim)]
        return r.mean()

    assert rel(ref_V, V, True) < 5e-4
    assert rel(ref_w, W, False) < 1e-4


def test_philox_known_answers(golden):
    fx = golden("philox_kat.npz")
    assert len(fx["rounds"]) >= 6
    for r, c, k, o in zip(fx["rounds"], fx["ctr"], fx["key"], fx["out"]):
        np.testing.assert_array_equal(O.philox4x32(c, k, int(r)), o)


def test_poisson_sampler_distribution():
    from scipy import stats

    rng = np.random.default_rng(1)
    for lam in (0.05, 0.8, 2.0, 9.7, 35.0):
        u = rng.random(20000)
        k = np.array([O.poisson_draw(lam, x) for x in u])
        assert abs(k.mean() - lam) < 5 * np.sqrt(lam / len(k))
        # inversion is exact: k is the smallest integer with F(k) >= u
        F = stats.poisson.cdf(k, lam)
        Fm = stats.poisson.cdf(k - 1, lam)
        assert np.all(u <= F + 1e-12) and np.all(u > Fm - 1e-12)


def _ref_lib():
    path = os.path.join(ROOT, "oracle", "_ref", "libnestprop.so")
    if not os.path.exists(path):
        pytest.skip("oracle/_ref not built (needs the reference sources)")
    L = ctypes.CDLL(path)
    f = L.ref_iaf_propagator_exp
    f.restype = ctypes.c_double
    f.argtypes = [ctypes.c_double] * 4
    return f


def test_propagator_matches_reference_code():
    """libnestutil/iaf_propagator.cpp, incl. the singular tau_m ~ tau_syn branch."""
    f = _ref_lib()
    for tm in (1.0, 10.0, 100.0):
        for h in (0.001, 0.01, 0.1, 1.0):
            for dt in np.concatenate([-np.logspace(-12, -1, 12), [0.0], np.logspace(-12, -1, 12)]):
                assert O.iaf_propagator_exp(tm + dt, tm, 250.0, h) == f(tm + dt, tm, 250.0, h)


def test_propagator_singular_branch_is_finite():
    for tm in (1.0, 10.0, 100.0):
        for h in (0.001, 0.1):
            p0 = O.iaf_propagator_exp(tm, tm, 250.0, h)
            assert np.isfinite(p0) and p0 > 0
            assert abs(O.iaf_propagator_exp(tm * (1 + 1e-9), tm, 250.0, h) - p0) < 1e-6 * p0


def test_refractory_clamp_length():
    """other/test_refractory.py: V_m stays at V_reset for exactly t_ref."""
    for t_ref in (0.1, 2.0, 2.05, 3.3):
        net = O.OracleNet("iaf_psc_delta", 1, 0.1, 1, 1)
        net.set("I_e", 1000.0)
        net.set("t_ref", t_ref)
        net.set_trace([0], "V_m_rel")
        net.run(400)
        v = net.trace()[:, 0]
        s, t = net.spikes()
        first = int(t[0])  # stamp of the first spike: V_reset is recorded at that stamp
        clamped = 0
        while first - 1 + clamped < len(v) and v[first - 1 + clamped] == 0.0:
            clamped += 1
        tics = int(t_ref * 1000 + 0.5)
        steps = int((tics + 99) * (1 / 100.0))
        assert clamped == steps + 1


def test_poisson_drive_mean():
    """Feed-forward check of the fused drive: with a non-leaky membrane V_m
    sums the drive, whose mean is rate * h * 1e-3 per step from step 2 on
    (generator steps t_g > start = 0, delay 1 step)."""
    n = 4000
    net = O.OracleNet("iaf_psc_delta", n, 0.1, 1, 1)
    net.set("V_th_rel", 1e9)
    net.set("tau_m", 1e12)
    w = 1e-3
    net.set_poisson(np.full(n, 5000.0), np.full(n, w), np.full(n, 1, dtype=np.int32), seed=7)
    net.run(1000)
    V = net.get("V_m_rel")
    lam = 0.1 * 5000.0 * 1e-3
    draws = 1000 - 2
    expect = w * lam * draws
    sd = w * np.sqrt(lam * draws) / np.sqrt(n)
    assert abs(V.mean() - expect) < 5 * sd
    # the per-neuron counts are Poisson(lam * draws): variance equals mean
    counts = V / w
    assert abs(counts.var() / counts.mean() - 1.0) < 0.1
