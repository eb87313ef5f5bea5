"""Statistical parity on Poisson-driven networks: firing rate, CV of the
inter-spike intervals and pairwise spike-count correlations (KS tests), for
the engine against the reference, against the CPU oracle on the same
network, and for the FP32 precision form against the plain FP64 form.

The networks are chaotic: two runs that differ in the last bit of one sum
decorrelate within a few hundred ms, so single trajectories are compared only
where they cannot have diverged (V_m over the first 100 ms) and otherwise
through distributions.  The tolerances are stated against the spread that
the plain FP64 form itself shows across realizations (seeds) of the same
network: on the 12,500-neuron network, 1.5 s windows, rates differ by up
to 1.6 % between seeds, and the KS statistic of two seeds' correlation
samples (3,000 pairs, 5 ms bins) is 0.03-0.05; on the 50,000-neuron aeif
network, 0.4 s windows, rates differ by up to 7 %.
"""

import numpy as np
import pytest

import oracle as O
import spikestats as S

pytestmark = pytest.mark.gpu

H = 0.1


def _raster(sr):
    ev = sr.events
    s = np.asarray(ev["senders"], dtype=np.int64) - 1
    st = np.rint(np.asarray(ev["times"]) / H).astype(np.int64)
    return s, st


def test_c1_population_fluctuations_vs_reference(nest, golden):
    """Config-1 network, FP64, three realizations against the reference's
    1 ms population spike counts (tests/golden/c1_exp_poisson_stats.npz):
    the Fano factor of the population count -- which the pairwise
    correlations set (Var = sum of the variances + sum of the covariances)
    -- of the reference lies inside the engine's spread across
    realizations, widened by a quarter, and the mean count per bin inside
    the reference's own spread of rates."""
    from nestgpu import workloads

    fx = golden("c1_exp_poisson_stats.npz")
    ref = fx["pop_counts_1ms"][100:1000].astype(np.float64)
    ref_ff = ref.var() / ref.mean()
    ffs, means = [], []
    for seed in (4242, 11, 23):
        pop, sr = workloads.c1(nest, precision="fp64", seed=seed)
        nest.Simulate(1000.0)
        s, st = _raster(sr)
        c = S.pop_counts(st, 10, 1000, 10000).astype(np.float64)
        ffs.append(c.var() / c.mean())
        means.append(c.mean())
        nest.ResetKernel()
    print(f"population Fano factor (1 ms bins): reference {ref_ff:.1f}, engine {np.round(ffs, 1)}")
    assert 0.75 * min(ffs) <= ref_ff <= 1.25 * max(ffs)
    ref_rates = np.concatenate([fx["seed_rates"], [fx["counts"].mean()]])
    lo, hi = ref_rates.min() * 12.5, ref_rates.max() * 12.5   # spikes per 1 ms bin
    spread = hi - lo
    assert lo - spread <= np.mean(means) <= hi + spread


def test_c1_engine_vs_oracle_correlations(nest):
    """The same graph and drive on the engine (FP64) and the oracle, 1.5 s:
    rates within 2 %, CV-ISI and pairwise-correlation distributions equal
    within KS statistics of 0.03 (below the seed-to-seed spread)."""
    from nestgpu import workloads
    from nestgpu.kernel import KERNEL

    pop, sr = workloads.c1(nest, precision="fp64", seed=4242)
    net, c = O.net_from_kernel(KERNEL)
    nest.Simulate(1500.0)
    net.run(15000)
    e = S.summary(*_raster(sr), 12500, H, 500.0, 1500.0, n_pairs=3000, seed=1)
    os_, ost = net.spikes()
    o = S.summary(os_.astype(np.int64), ost.astype(np.int64), 12500, H, 500.0, 1500.0, n_pairs=3000, seed=1)
    cmp = S.compare(e, o)
    print("engine vs oracle:", cmp)
    assert abs(cmp["rate_err"]) <= 0.02
    assert cmp["ks_cv"] <= 0.03
    assert cmp["ks_corr"] <= 0.03


def test_c1_fp32_form_vs_fp64(nest):
    """The precision form (FP32 state, int64 fixed-point rings) against the
    plain FP64 form on the same networks and drive, four realizations of
    2 s: pooled rate error <= 2 %, CV-ISI error <= 0.05, correlation KS
    statistic <= 0.06 per realization (the FP64 seed-to-seed spread reaches
    0.05), and V_m over the first 100 ms (200 neurons, every step) within
    1e-4 mV RMS -- the trajectories have not diverged there, the difference
    is FP32 rounding (measured: 6e-6 mV)."""
    from nestgpu import workloads

    spikes = {"fp64": 0, "fp32": 0}
    cvs = {"fp64": [], "fp32": []}
    ks = []
    V = {}
    for seed in (4242, 11, 23, 37):
        summ = {}
        for prec in ("fp64", "fp32"):
            pop, sr = workloads.c1(nest, precision=prec, seed=seed)
            mm = None
            if seed == 4242:
                mm = nest.Create("multimeter", params={"interval": H, "record_from": ["V_m"]})
                nest.Connect(mm, pop[:200])
            nest.Simulate(2000.0)
            s, st = _raster(sr)
            spikes[prec] += len(s)
            summ[prec] = S.summary(s, st, 12500, H, 500.0, 2000.0, n_pairs=3000, seed=seed)
            cvs[prec].append(summ[prec]["cv_isi_mean"])
            if mm is not None:
                ev = mm.events
                o = np.lexsort((ev["senders"], ev["times"]))
                V[prec] = np.asarray(ev["V_m"])[o].reshape(-1, 200)[:1000]
            nest.ResetKernel()
        ks.append(S.compare(summ["fp32"], summ["fp64"])["ks_corr"])
    rate_err = spikes["fp32"] / spikes["fp64"] - 1
    cv_err = np.mean(cvs["fp32"]) - np.mean(cvs["fp64"])
    rms = float(np.sqrt(np.mean((V["fp32"] - V["fp64"]) ** 2)))
    print(f"fp32 vs fp64: rate {rate_err:+.4f}, CV-ISI {cv_err:+.4f}, correlation KS {np.round(ks, 3)}, "
          f"V_m RMS (first 100 ms) {rms:.2e} mV")
    assert abs(rate_err) <= 0.02
    assert abs(cv_err) <= 0.05
    assert max(ks) <= 0.06
    assert rms <= 1e-4


def _layered_pair(scale, ms):
    """The layered 8-population network drawn on the device (FP64) and its
    oracle copy: same graph (exported with ng_net_get_connections), initial
    state and drive stream."""
    from nestgpu import workloads

    spec = workloads.layered_spec(scale=scale)
    n = sum(spec["sizes"])
    eng = workloads.layered_engine(spec, "fp64")
    nid = workloads.layered_add(eng, spec, 10 ** 7)
    src, tgt, w, d = eng.net_get_connections(nid)
    steps = int(round(ms / H))
    eng.simulate(steps)
    es, et = eng.net_spikes(nid)
    eng.close()
    net = O.OracleNet("iaf_psc_exp", n, H, 1, max(int(d.max()), 15))
    E_L = spec["E_L"]
    V0 = np.random.default_rng(spec["seed"]).normal(-58.0, 10.0, n) - E_L
    for k, v in {"tau_syn_ex": spec["tau_syn"], "tau_syn_in": spec["tau_syn"], "tau_m": spec["tau_m"],
                 "C_m": spec["C_m"], "t_ref": spec["t_ref"], "V_th_rel": spec["V_th"] - E_L,
                 "V_reset_rel": spec["V_reset"] - E_L, "V_m_rel": V0}.items():
        net.set(k, v)
    net.set_edges(src, tgt, w, d)
    rate = np.repeat(np.asarray(spec["k_ext"], dtype=np.float64) * spec["nu_ext_hz"], spec["sizes"])
    net.set_poisson(rate, spec["J"], int(round(spec["d_ext_ms"] / H)), spec["seed"])
    net.set_record(np.ones(n, dtype=np.uint8))
    net.run(steps)
    os_, ost = net.spikes()
    return spec, (es.astype(np.int64), et.astype(np.int64)), (os_.astype(np.int64), ost.astype(np.int64))


def test_layered_scaled_engine_vs_oracle():
    """The layered network (config 2's populations and connection
    probabilities, min_delay one step, delays spread to 8 ms) at a quarter of
    its size, 300 ms, engine against oracle on the same graph and drive:
    every population's rate within 2 %, and the CV-ISI and correlation
    distributions equal within KS statistics of 0.03."""
    spec, (es, et), (os_, ost) = _layered_pair(0.25, 300.0)
    n = sum(spec["sizes"])
    bounds = np.concatenate([[0], np.cumsum(spec["sizes"])])
    assert len(es) > 100000
    for p in range(8):
        a = np.count_nonzero((es >= bounds[p]) & (es < bounds[p + 1]))
        b = np.count_nonzero((os_ >= bounds[p]) & (os_ < bounds[p + 1]))
        assert abs(a - b) <= max(0.02 * b, 10), (p, a, b)
    e = S.summary(es, et, n, H, 50.0, 300.0, n_pairs=3000, seed=1)
    o = S.summary(os_, ost, n, H, 50.0, 300.0, n_pairs=3000, seed=1)
    cmp = S.compare(e, o)
    print("layered (scale 0.25) engine vs oracle:", cmp)
    assert cmp["ks_cv"] <= 0.03
    assert cmp["ks_corr"] <= 0.03


def test_aeif_fp32_form_vs_fp64():
    """The 50,000-neuron aeif_cond_alpha network (config 3) in the FP32-state
    form (FP64 RKF45 error control) against the FP64 form, three
    realizations of 500 ms: pooled rate error <= 2 % (a single realization's
    rate varies by up to 7 % across seeds in the FP64 form itself), CV-ISI
    error <= 0.05 and correlation KS statistic <= 0.06 per realization."""
    from nestgpu import workloads

    spec0 = workloads.aeif_spec()
    n = spec0["n_exc"] + spec0["n_inh"]
    spikes = {"fp64": 0, "fp32": 0}
    cv = {"fp64": [], "fp32": []}
    ks = []
    for seed in (77, 78, 79):
        summ = {}
        for prec in ("fp64", "fp32"):
            spec = dict(spec0, seed=seed)
            eng = workloads.aeif_engine(spec, prec)
            nid = workloads.aeif_add(eng, spec, 10 ** 6)
            eng.simulate(5000)
            s, st = eng.net_spikes(nid)
            eng.close()
            spikes[prec] += len(s)
            summ[prec] = S.summary(s.astype(np.int64), st.astype(np.int64), n, H, 100.0, 500.0, n_pairs=3000, seed=1)
            cv[prec].append(summ[prec]["cv_isi_mean"])
        ks.append(S.compare(summ["fp32"], summ["fp64"])["ks_corr"])
    rate_err = spikes["fp32"] / spikes["fp64"] - 1
    cv_err = np.mean(cv["fp32"]) - np.mean(cv["fp64"])
    print(f"aeif fp32 vs fp64: rate {rate_err:+.4f}, CV-ISI {cv_err:+.4f}, correlation KS {np.round(ks, 3)}")
    assert abs(rate_err) <= 0.02
    assert abs(cv_err) <= 0.05
    assert max(ks) <= 0.06
