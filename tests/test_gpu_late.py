"""Late delivery: the edges of delay >= 2 min_delay of a slice's spikes are
delivered on a second stream while the next slice updates.  Each row holds
its shorter-delay edges first.  With ring sums that do not depend on the
order of the adds (dyadic FP64 weights, or the FP32 form's integer rings) the
result equals the delivery of every edge at the slice's close bit for bit:

- static engine, FP64 and FP32, the three update kernels (one thread per
  neuron, two-phase, aeif RKF45) and both iaf models, explicit CSR with delays
  over [min_delay, max_delay], run in partial slices, slice graphs and a
  profiled stretch (where the late delivery runs after the slice-close one);
- serving engine, a pairwise_bernoulli network drawn on the device (rows
  split after the draw) and an explicit one (rows split on the host).
"""

import numpy as np
import pytest

from nestgpu import _abi

pytestmark = pytest.mark.gpu


def _static_run(late, precision, model=_abi.NG_IAF_PSC_EXP, md=2):
    n, maxd = 3000, 30
    rng = np.random.default_rng(11)
    deg = rng.integers(40, 160, n)
    row = np.concatenate([[0], np.cumsum(deg)]).astype(np.int64)
    nnz = int(row[-1])
    tgt = rng.integers(0, n, nnz)
    d = rng.integers(md, maxd + 1, nnz)
    eng = _abi.Engine([(model, n)], 0.1, md, maxd, precision=precision)
    eng.set_option("late_delivery", 1 if late else 0)
    if model == _abi.NG_AEIF_COND_ALPHA:
        w = rng.choice([1.0, 0.5, -2.0, -4.0], nnz)                # nS
        eng.set_var(0, "tau_syn_ex", np.full(n, 1.0))
        drive = (np.full(n, 15000.0), np.full(n, 1.0))
        eng.set_var(0, "V_m", rng.uniform(-70.6, -52.0, n))
    else:
        w = rng.choice([24.0, 12.5, -48.0, -100.0], nnz)            # pA (iaf_psc_exp) or mV (iaf_psc_delta)
        if model == _abi.NG_IAF_PSC_DELTA:
            w = w / 64.0
        drive = (np.full(n, 12000.0), np.full(n, 16.0 if model == _abi.NG_IAF_PSC_EXP else 0.25))
        eng.set_var(0, "V_m_rel", rng.uniform(0.0, 15.0, n))
    eng.set_connections(row, tgt, w, d)
    eng.set_recording(np.ones(n, dtype=np.uint8))
    eng.set_poisson(drive[0], drive[1], np.full(n, md), 0, 10**9, 5)
    for k in (7, 13, 3):              # partial slices
        eng.simulate(k)
    eng.simulate(977)                 # slice graphs
    eng.set_profiling(True)           # late delivery after the slice-close one, timed with it
    eng.simulate(200)
    eng.set_profiling(False)
    eng.set_graph_slices(0)           # slice by slice without graphs
    eng.simulate(301)
    s, t = eng.spikes()
    V = eng.get_var(0, "V_m" if model == _abi.NG_AEIF_COND_ALPHA else "V_m_rel")
    st = eng.stats()
    eng.close()
    return s, t, V, st


@pytest.mark.parametrize("precision,model,md", [
    (_abi.NG_FP64, _abi.NG_IAF_PSC_EXP, 2),      # one thread per neuron, 4 lags of inputs gathered
    (_abi.NG_FP32, _abi.NG_IAF_PSC_EXP, 2),
    (_abi.NG_FP64, _abi.NG_IAF_PSC_EXP, 3),      # two-phase update kernel (slices of 3 steps)
    (_abi.NG_FP64, _abi.NG_IAF_PSC_DELTA, 3),
    (_abi.NG_FP64, _abi.NG_AEIF_COND_ALPHA, 2),  # RKF45 kernel, per-spike appends
])
def test_late_delivery_static_engine(precision, model, md):
    s0, t0, V0, st0 = _static_run(False, precision, model, md)
    s1, t1, V1, st1 = _static_run(True, precision, model, md)
    assert len(s0) > 500
    assert st0["syn_events"] == st1["syn_events"]
    o0, o1 = np.lexsort((s0, t0)), np.lexsort((s1, t1))
    np.testing.assert_array_equal(s0[o0], s1[o1])
    np.testing.assert_array_equal(t0[o0], t1[o1])
    np.testing.assert_array_equal(V0, V1)


PB_SIZES = (3000, 700, 2300)
PB_P = np.array([[0.05, 0.10, 0.02],
                 [0.20, 0.02, 0.15],
                 [0.01, 0.30, 0.08]])


def _serving_run(late):
    n = sum(PB_SIZES)
    eng = _abi.Engine([(_abi.NG_IAF_PSC_EXP, 20_000)], 0.1, 1, 40, precision=_abi.NG_FP32, serving=True,
                      max_networks=4, edge_capacity=30_000_000, max_abs_weight=1000.0)
    eng.set_option("late_delivery", 1 if late else 0)
    pb = _abi.NGPairwiseBernoulli.make(PB_SIZES, (1, 0, 1), PB_P, w_mean=(-351.2, 87.8), w_sd=(35.12, 8.78),
                                       d_mean_ms=(0.75, 1.5), d_sd_ms=(0.375, 0.75), d_max_ms=3.95, seed=21)
    V0 = np.random.default_rng(8).uniform(0.0, 14.0, n)
    a = eng.net_add(n, 2500, 17, {"tau_syn_ex": 0.5, "tau_syn_in": 0.5, "V_m_rel": V0}, build=pb,
                    poisson=(np.full(n, 9000.0), 87.8, 15))
    rng = np.random.default_rng(4)
    m, nnz = 1500, 60_000
    edges = (rng.integers(0, m, nnz), rng.integers(0, m, nnz), rng.choice([87.75, -351.0], nnz, p=[0.8, 0.2]),
             rng.integers(1, 41, nnz))
    b = eng.net_add(m, 2500, 3, {"tau_syn_ex": 0.5, "tau_syn_in": 0.5,
                                 "V_m_rel": rng.uniform(0.0, 14.0, m)}, edges=edges,
                    poisson=(np.full(m, 9000.0), 87.8, 15))
    eng.simulate(1200)
    eng.simulate(1300)
    out = [(eng.net_spikes(i), eng.net_get_var(i, "V_m_rel", k)) for i, k in ((a, n), (b, m))]
    conn = eng.net_get_connections(a)
    st = eng.stats()
    eng.close()
    return out, conn, st


def test_late_delivery_serving_engine():
    ref, c0, st0 = _serving_run(False)
    got, c1, st1 = _serving_run(True)
    assert st0["syn_events"] == st1["syn_events"]
    for ((s0, t0), v0), ((s1, t1), v1) in zip(ref, got):
        assert len(s0) > 500
        o0, o1 = np.lexsort((s0, t0)), np.lexsort((s1, t1))
        np.testing.assert_array_equal(s0[o0], s1[o1])
        np.testing.assert_array_equal(t0[o0], t1[o1])
        np.testing.assert_array_equal(v0, v1)
    # the split only reorders each row: the same connections
    k0 = np.lexsort((c0[3], c0[1], c0[0]))
    k1 = np.lexsort((c1[3], c1[1], c1[0]))
    for x0, x1 in zip(c0, c1):
        np.testing.assert_array_equal(x0[k0], x1[k1])
    # rows hold their delay-1 edges first
    s, d = c1[0], c1[3]
    for src in np.unique(s)[:200]:
        dd = d[s == src]
        assert np.all(np.diff((dd >= 2).astype(int)) >= 0)
