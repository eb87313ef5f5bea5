"""Serving engine: networks admitted into and retired from a running engine.

- a network's spikes are the same alone and in a mix (FP32 form with int64
  rings, Philox streams keyed and counted per network): bit-identical;
- the FP64 serving path matches the static engine on the same explicit graph;
- admission by footprint, capacity errors, and slot reuse;
- device-drawn fixed_indegree graphs have the requested in-degrees;
- device-drawn pairwise_bernoulli graphs have the requested statistics and
  are read back through ng_net_get_connections;
- the per-target gather of the precision form equals the scatter.
"""

import numpy as np
import pytest

from nestgpu import _abi, serving

pytestmark = pytest.mark.gpu


def _req(rid, n, steps, seed, k=None, g=5.0, eta=1.5):
    k_exc = k if k is not None else min(int(0.1 * n), 1000)
    return serving.Request(rid=rid, arrival=0.0, n=n, n_exc=int(0.8 * n), k_exc=k_exc, k_inh=max(1, k_exc // 4), g=g,
                           eta=eta, steps=steps, seed=seed)


def _run_alone(r, precision="fp32"):
    eng = serving.new_engine(precision, capacity_neurons=200_000, capacity_edges=60_000_000, max_networks=16)
    nid = serving._admit(eng, r)
    eng.simulate(-(-r.steps // 15) * 15)
    s, t = eng.net_spikes(nid)
    V = eng.net_get_var(nid, "V_m_rel", r.n)
    eng.close()
    return s, t, V


def test_same_result_alone_and_in_a_mix():
    target = _req(0, 6000, 3000, seed=1234)
    s_alone, t_alone, V_alone = _run_alone(target)
    assert len(s_alone) > 500
    eng = serving.new_engine("fp32", capacity_neurons=200_000, capacity_edges=60_000_000, max_networks=16)
    others = [_req(i, n, 4000, seed=99 + i) for i, n in enumerate((3000, 20000, 1500), start=1)]
    ids = [serving._admit(eng, o) for o in others[:2]]
    eng.simulate(45 * 15)            # the others run for a while first
    tid = serving._admit(eng, target)  # admitted later, at another place in the pool
    ids.append(serving._admit(eng, others[2]))
    eng.simulate(-(-target.steps // 15) * 15)
    done, fin = eng.net_poll(tid)
    assert fin and done == target.steps
    s_mix, t_mix = eng.net_spikes(tid)
    V_mix = eng.net_get_var(tid, "V_m_rel", target.n)
    o1 = np.lexsort((s_alone, t_alone))
    o2 = np.lexsort((s_mix, t_mix))
    np.testing.assert_array_equal(s_mix[o2], s_alone[o1])
    np.testing.assert_array_equal(t_mix[o2], t_alone[o1])
    np.testing.assert_array_equal(V_mix, V_alone)
    eng.close()


def test_fixed_indegree_drawn_on_device():
    """Every target gets exactly k_exc + k_inh inputs (through the delivered
    drive-free response: one spike per source fired by a huge I_e pulse would
    be indirect; instead read the realized graph statistics via syn events)."""
    eng = serving.new_engine("fp64", capacity_neurons=50_000, capacity_edges=20_000_000, max_networks=4)
    r = _req(0, 5000, 150, seed=7, k=200)
    nid = serving._admit(eng, r)
    eng.simulate(150)
    s, t = eng.net_spikes(nid)
    st = eng.stats()
    # each spike of an excitatory source delivers its out-degree; totals agree
    # with n * k per population on average (multapses allowed)
    exp_deg = {True: r.n * r.k_exc / r.n_exc, False: r.n * r.k_inh / (r.n - r.n_exc)}
    approx = sum(exp_deg[bool(x < r.n_exc)] for x in s)
    assert len(s) > 100
    assert abs(st["syn_events"] / approx - 1) < 0.1
    eng.close()


def test_admission_by_footprint_and_slot_reuse():
    eng = serving.new_engine("fp32", capacity_neurons=30_000, capacity_edges=10_000_000, max_networks=2)
    a = serving._admit(eng, _req(0, 20_000, 300, seed=1, k=100))
    assert a is not None
    assert serving._admit(eng, _req(1, 20_000, 300, seed=2, k=100)) is None   # neurons do not fit
    b = serving._admit(eng, _req(2, 5_000, 300, seed=3, k=100))
    assert b is not None
    assert serving._admit(eng, _req(3, 1_000, 300, seed=4, k=100)) is None    # no free slot
    eng.simulate(300)
    assert eng.net_poll(a)[1] and eng.net_poll(b)[1]
    eng.net_remove(a)
    with pytest.raises(_abi.EngineError):
        eng.net_remove(a)
    c = serving._admit(eng, _req(1, 20_000, 300, seed=2, k=100))
    assert c is not None
    eng.close()


def test_fp64_serving_matches_static_engine():
    """An explicit graph through ng_net_add (FP64) equals ng_set_connections."""
    rng = np.random.default_rng(5)
    n, nnz = 800, 40_000
    src = rng.integers(0, n, nnz).astype(np.int32)
    tgt = rng.integers(0, n, nnz).astype(np.int32)
    w = np.where(src < 640, 64.0, -256.0)
    d = np.full(nnz, 15, dtype=np.int32)
    Ie = rng.uniform(350, 450, n)
    V0 = rng.uniform(0, 14, n)
    eng = serving.new_engine("fp64", capacity_neurons=10_000, capacity_edges=1_000_000, max_networks=4)
    nid = eng.net_add(n, 3000, 11, {"tau_syn_ex": 0.5, "tau_syn_in": 0.5, "I_e": Ie, "V_m_rel": V0},
                      edges=(src, tgt, w, d))
    eng.simulate(3000)
    s1, t1 = eng.net_spikes(nid)
    eng.close()
    st = _abi.Engine([(_abi.NG_IAF_PSC_EXP, n)], 0.1, 15, 15)
    st.set_var(0, "tau_syn_ex", np.full(n, 0.5))
    st.set_var(0, "tau_syn_in", np.full(n, 0.5))
    st.set_var(0, "I_e", Ie)
    st.set_var(0, "V_m_rel", V0)
    order = np.argsort(src, kind="stable")
    row = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(src, minlength=n), out=row[1:])
    st.set_connections(row, tgt[order], w[order], d[order])
    st.set_recording(np.ones(n, dtype=np.uint8))
    st.simulate(3000)
    s2, t2 = st.spikes()
    st.close()
    assert len(s1) > 100
    o1, o2 = np.lexsort((s1, t1)), np.lexsort((s2, t2))
    np.testing.assert_array_equal(s1[o1], s2[o2])
    np.testing.assert_array_equal(t1[o1], t2[o2])


def test_small_serving_run_latency_accounting():
    reqs = serving.make_requests(count=12, rate_hz=200.0, seed=3, n_min=1000, n_max=8000, t_min_ms=100, t_max_ms=300)
    eng = serving.new_engine("fp32", capacity_neurons=100_000, capacity_edges=40_000_000, max_networks=32)
    done, stats = serving.run_batched(reqs, eng)
    eng.close()
    assert all(np.isfinite(r.finished) for r in done)
    assert all(r.finished >= r.admitted >= r.enqueued >= r.arrival - 1e-9 for r in done)
    lat = serving.latency_summary(done)
    assert lat["p99_s"] >= lat["p50_s"] > 0
    assert stats["syn_events"] > 0


def _pb_engine(precision, cap_edges=30_000_000):
    prec = _abi.NG_FP32 if precision == "fp32" else _abi.NG_FP64
    return _abi.Engine([(_abi.NG_IAF_PSC_EXP, 20_000)], 0.1, 1, 40, precision=prec, serving=True, max_networks=4,
                       edge_capacity=cap_edges, max_abs_weight=1000.0)


PB_SIZES = (3000, 700, 2300, 1)
PB_EXC = (1, 0, 1, 0)
PB_P = np.array([[0.05, 0.10, 0.00, 0.3],
                 [0.20, 0.02, 0.15, 1.0],
                 [0.01, 1.00, 0.08, 0.0],
                 [0.50, 0.50, 0.50, 1.0]])


def _pb(seed=77, allow_autapses=0):
    return _abi.NGPairwiseBernoulli.make(PB_SIZES, PB_EXC, PB_P, w_mean=(-351.2, 87.8), w_sd=(35.12, 8.78),
                                         d_mean_ms=(0.75, 1.5), d_sd_ms=(0.375, 0.75), d_max_ms=3.95,
                                         allow_autapses=allow_autapses, seed=seed)


def test_pairwise_bernoulli_drawn_on_device():
    """Per population pair the connection count is binomial(n_i n_j, p_ij)
    (p = 0 and p = 1 exactly), no autapses, normal weights per source type,
    delays = round(clip(N(mu, sd), h, d_max) / h); the same seed gives the same
    graph, and the FP32 engine draws the same graph up to weight rounding."""
    n = sum(PB_SIZES)
    lo = np.concatenate([[0], np.cumsum(PB_SIZES)])
    pop = np.repeat(np.arange(len(PB_SIZES)), PB_SIZES)
    eng = _pb_engine("fp64")
    a = eng.net_add(n, 0, 1, {}, build=_pb())
    b = eng.net_add(n, 0, 1, {}, build=_pb())
    s, t, w, d = eng.net_get_connections(a)
    s2, t2, w2, d2 = eng.net_get_connections(b)
    eng.close()
    np.testing.assert_array_equal(s, s2)
    np.testing.assert_array_equal(t, t2)
    np.testing.assert_array_equal(w, w2)
    np.testing.assert_array_equal(d, d2)
    assert np.all(s != t)
    assert np.all(np.diff(s) >= 0)
    k = len(PB_SIZES)
    cnt = np.zeros((k, k), dtype=np.int64)
    np.add.at(cnt, (pop[s], pop[t]), 1)
    for i in range(k):
        for j in range(k):
            pairs = PB_SIZES[i] * PB_SIZES[j] - (PB_SIZES[i] if i == j else 0)
            mu = pairs * PB_P[i, j]
            sd = np.sqrt(pairs * PB_P[i, j] * (1 - PB_P[i, j]))
            if PB_P[i, j] in (0.0, 1.0):
                assert cnt[i, j] == mu, (i, j)
            else:
                assert abs(cnt[i, j] - mu) < 5 * sd + 1, (i, j, cnt[i, j], mu)
    # no duplicate (source, target) pairs: Bernoulli trials, not multapses
    key = s.astype(np.int64) * n + t
    assert len(np.unique(key)) == len(key)
    ex = np.asarray(PB_EXC)[pop[s]].astype(bool)
    for sel, m, sdv, dm, dsd in ((ex, 87.8, 8.78, 1.5, 0.75), (~ex, -351.2, 35.12, 0.75, 0.375)):
        ws = w[sel]
        assert abs(ws.mean() - m) < 5 * sdv / np.sqrt(len(ws))
        assert abs(ws.std() / sdv - 1) < 0.02
        rng = np.random.default_rng(1)
        ref = np.floor(np.clip(rng.normal(dm, dsd, 2_000_000), 0.1, 3.95) / 0.1 + 0.5).astype(int)
        h_dev = np.bincount(d[sel], minlength=41)[:41] / sel.sum()
        h_ref = np.bincount(ref, minlength=41)[:41] / len(ref)
        assert np.abs(h_dev - h_ref).max() < 0.01
    assert d.min() >= 1 and d.max() <= 40
    # the FP32 engine: the same draws, weights on the fixed-point grid
    e32 = _pb_engine("fp32")
    c = e32.net_add(n, 0, 1, {}, build=_pb())
    s3, t3, w3, d3 = e32.net_get_connections(c)
    e32.close()
    np.testing.assert_array_equal(s3, s)
    np.testing.assert_array_equal(t3, t)
    np.testing.assert_array_equal(d3, d)
    np.testing.assert_allclose(w3, w, rtol=0, atol=1e-4)


def test_pairwise_bernoulli_seed_and_autapses():
    n = sum(PB_SIZES)
    eng = _pb_engine("fp64")
    a = eng.net_add(n, 0, 1, {}, build=_pb(seed=5))
    b = eng.net_add(n, 0, 1, {}, build=_pb(seed=6, allow_autapses=1))
    s, t, _, _ = eng.net_get_connections(a)
    s2, t2, _, _ = eng.net_get_connections(b)
    eng.close()
    assert len(s) != len(s2) or not np.array_equal(t, t2)
    # with autapses allowed the p = 1 block of the single-neuron population has its self-connection
    last = n - 1
    assert np.any((s2 == last) & (t2 == last))
    assert not np.any((s == last) & (t == last))


def test_get_connections_of_explicit_graph():
    rng = np.random.default_rng(3)
    n, nnz = 300, 5000
    src = rng.integers(0, n, nnz).astype(np.int32)
    tgt = rng.integers(0, n, nnz).astype(np.int32)
    w = rng.choice([64.0, -256.0, 12.5], nnz)
    d = rng.integers(1, 30, nnz).astype(np.int32)
    eng = _pb_engine("fp64")
    nid = eng.net_add(n, 0, 1, {}, edges=(src, tgt, w, d))
    s, t, ww, dd = eng.net_get_connections(nid)
    eng.close()
    a = np.lexsort((d, w, tgt, src))
    b = np.lexsort((dd, ww, t, s))
    np.testing.assert_array_equal(s[b], src[a])
    np.testing.assert_array_equal(t[b], tgt[a])
    np.testing.assert_array_equal(ww[b], w[a])
    np.testing.assert_array_equal(dd[b], d[a])


@pytest.mark.parametrize("frac", [0.0, 0.03])
def test_gather_equals_scatter(frac):
    """The per-target gather (always on with fraction 0; switching per slice
    with 0.03) gives the scatter's spikes and state bit for bit: both add the
    same integers into the int64 rings."""
    def run(opts):
        eng = serving.new_engine("fp32", capacity_neurons=100_000, capacity_edges=40_000_000, max_networks=8)
        for k, v in opts.items():
            eng.set_option(k, v)
        ids = [serving._admit(eng, _req(i, n, 1500, seed=500 + i, g=g, eta=eta))
               for i, (n, g, eta) in enumerate(((4000, 3.5, 1.8), (7000, 5.0, 1.2), (2500, 6.0, 2.0)))]
        eng.simulate(1500)
        out = [(eng.net_spikes(i), eng.net_get_var(i, "V_m_rel", n)) for i, n in zip(ids, (4000, 7000, 2500))]
        st = eng.stats()
        eng.close()
        return out, st

    ref, st0 = run({"gather": 0})
    got, st1 = run({"gather_frac": frac})
    assert st0["syn_events"] == st1["syn_events"]
    assert st0["gather_slices"] == 0
    assert st1["gather_slices"] > (250 if frac == 0.0 else 10)
    for ((s0, t0), v0), ((s1, t1), v1) in zip(ref, got):
        assert len(s0) > 100
        o0, o1 = np.lexsort((s0, t0)), np.lexsort((s1, t1))
        np.testing.assert_array_equal(s0[o0], s1[o1])
        np.testing.assert_array_equal(t0[o0], t1[o1])
        np.testing.assert_array_equal(v0, v1)


@pytest.mark.parametrize("variant", [0, 1])
def test_serving_update_variants_agree(variant):
    """A serving engine updates with variant 6 unless told otherwise (one
    thread per neuron, 2 lags of inputs at a time); the 4- and 8-lag forms
    give its spikes and state bit for bit, in gather and scatter slices."""
    def run(v):
        eng = serving.new_engine("fp32", capacity_neurons=100_000, capacity_edges=40_000_000, max_networks=8)
        if v is not None:
            eng.set_tuning(0, v)
        ids = [serving._admit(eng, _req(i, n, 1200, seed=700 + i, g=g, eta=eta))
               for i, (n, g, eta) in enumerate(((5000, 4.0, 1.6), (1800, 6.0, 2.0)))]
        eng.simulate(1200)
        out = [(eng.net_spikes(i), eng.net_get_var(i, "V_m_rel", n)) for i, n in zip(ids, (5000, 1800))]
        st, t = eng.stats(), eng.tuned()
        eng.close()
        return out, st, t

    ref, st0, t0 = run(None)
    got, st1, t1 = run(variant)
    assert t0["update_variant"] == 6 and t1["update_variant"] == variant
    assert st0["syn_events"] == st1["syn_events"] and st0["gather_slices"] > 0
    for ((s0, u0), v0), ((s1, u1), v1) in zip(ref, got):
        assert len(s0) > 100
        o0, o1 = np.lexsort((s0, u0)), np.lexsort((s1, u1))
        np.testing.assert_array_equal(s0[o0], s1[o1])
        np.testing.assert_array_equal(u0[o0], u1[o1])
        np.testing.assert_array_equal(v0, v1)


def test_ring32_equals_ring64_on_representable_weights():
    """32-bit ring cells hold the same sums as 64-bit ones when the weights
    are exact at both scales (multiples of 2^-10): identical spikes and
    state.  A network whose in-edge weight sums exceed ring_bound is
    refused at admission."""
    def run(ring32):
        eng = _abi.Engine([(_abi.NG_IAF_PSC_EXP, 20_000)], 0.1, 15, 15, precision=_abi.NG_FP32, serving=True,
                          max_networks=4, edge_capacity=20_000_000, max_abs_weight=1000.0, ring32=ring32,
                          ring_bound=400_000.0 if ring32 else 0.0)
        r = _req(0, 5000, 2000, seed=31, k=400, g=4.0)
        build = dict(n_exc=r.n_exc, k_exc=r.k_exc, k_inh=r.k_inh, w_exc=87.75, w_inh=-351.0, delay_steps=15,
                     allow_autapses=0, seed=77)
        V0 = np.random.default_rng(3).normal(-58.0, 10.0, r.n) + 70.0
        nid = eng.net_add(r.n, r.steps, 5, {"tau_syn_ex": 0.5, "tau_syn_in": 0.5, "V_m_rel": V0}, build=build,
                          poisson=(1.5 * serving.NU_TH_HZ, 87.75, 15))
        eng.simulate(r.steps)
        s, t = eng.net_spikes(nid)
        V = eng.net_get_var(nid, "V_m_rel", r.n)
        if ring32:
            with pytest.raises(_abi.EngineError):
                eng.net_add(r.n, 100, 6, {}, build=dict(build, k_exc=4000, k_inh=1000))
        eng.close()
        return s, t, V

    s1, t1, V1 = run(False)
    s2, t2, V2 = run(True)
    assert len(s1) > 1000
    o1, o2 = np.lexsort((s1, t1)), np.lexsort((s2, t2))
    np.testing.assert_array_equal(s1[o1], s2[o2])
    np.testing.assert_array_equal(t1[o1], t2[o2])
    np.testing.assert_array_equal(V1, V2)


@pytest.mark.parametrize("ring32", [False, True])
def test_tiled_delivery_equals_scatter(ring32):
    """Target-tiled delivery (shared-memory accumulation per target tile) of a
    pairwise_bernoulli network equals the scatter bit for bit in the FP32
    form (the same integers are added), with 64- and 32-bit ring cells."""
    n = sum(PB_SIZES)

    def run(tiled):
        eng = _abi.Engine([(_abi.NG_IAF_PSC_EXP, 20_000)], 0.1, 1, 40, precision=_abi.NG_FP32, serving=True,
                          max_networks=4, edge_capacity=30_000_000, max_abs_weight=1000.0, ring32=ring32,
                          ring_bound=2.0e6 if ring32 else 0.0,
                          tile_capacity=_abi.tile_table_entries(n, 40, ring32) if tiled else 0)
        V0 = np.random.default_rng(8).uniform(0.0, 14.0, n)
        rate = np.full(n, 9000.0)
        nid = eng.net_add(n, 3000, 17, {"tau_syn_ex": 0.5, "tau_syn_in": 0.5, "V_m_rel": V0}, build=_pb(seed=21),
                          poisson=(rate, 87.8, 15))
        eng.simulate(3000)
        s, t = eng.net_spikes(nid)
        V = eng.net_get_var(nid, "V_m_rel", n)
        st = eng.stats()
        eng.close()
        return s, t, V, st

    s0, t0, V0, st0 = run(False)
    s1, t1, V1, st1 = run(True)
    assert len(s0) > 1000
    assert st0["syn_events"] == st1["syn_events"]
    o0, o1 = np.lexsort((s0, t0)), np.lexsort((s1, t1))
    np.testing.assert_array_equal(s0[o0], s1[o1])
    np.testing.assert_array_equal(t0[o0], t1[o1])
    np.testing.assert_array_equal(V0, V1)


def test_async_simulate_equals_sync():
    """ng_simulate_async leaves the last group running: the spikes of a network
    that ended before it are complete without a sync, a network still
    running is drained on read, and the results equal ng_simulate's."""
    def run(asynchronous):
        eng = serving.new_engine("fp32", capacity_neurons=50_000, capacity_edges=20_000_000, max_networks=4)
        a = serving._admit(eng, _req(0, 4000, 15 * 40, seed=71))
        b = serving._admit(eng, _req(1, 6000, 15 * 200, seed=72))
        step = eng.simulate_async if asynchronous else eng.simulate
        for _ in range(4):
            step(15 * 32)
        sa = eng.net_spikes(a)          # ended long before the running group
        eng.net_remove(a)
        step(15 * 32)
        sb = eng.net_spikes(b)          # b ran in the last group: drained on read
        Vb = eng.net_get_var(b, "V_m_rel", 6000)
        eng.close()
        return sa, sb, Vb

    (sa0, sb0, V0), (sa1, sb1, V1) = run(False), run(True)
    assert len(sa0[0]) > 100 and len(sb0[0]) > 1000
    for (s0, t0), (s1, t1) in ((sa0, sa1), (sb0, sb1)):
        o0, o1 = np.lexsort((s0, t0)), np.lexsort((s1, t1))
        np.testing.assert_array_equal(s0[o0], s1[o1])
        np.testing.assert_array_equal(t0[o0], t1[o1])
    np.testing.assert_array_equal(V0, V1)
