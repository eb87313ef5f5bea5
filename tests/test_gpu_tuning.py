"""The launch configurations the autotuner chooses between, and the
autotuner itself.

Every configuration -- update kernel (one thread per neuron with 4 or 8
lags of inputs gathered, two-phase with 256- or 128-thread CTAs, or the
persistent kernel that runs update and delivery of many slices in one
cooperative launch), resident
delivery CTAs per SM, edge chunks per delivery warp -- must compute the same
result: on networks whose ring sums do not depend on the order of the adds
(the FP32 form's integer rings; dyadic FP64 weights) the rasters and final
states are identical bit for bit.  The autotuner runs its trials on the
network's own next slices, so a tuned run equals a run with a fixed
configuration, and a second engine of the same shape and activity takes the
choice from the process cache.
"""

import numpy as np
import pytest

from nestgpu import _abi

pytestmark = pytest.mark.gpu

# (update variant, delivery CTAs per SM, chunks per warp); variant 5 is the
# persistent slice kernel (update and delivery of many slices in one launch),
# 6 the one-thread kernel with 2 lags of inputs at a time
CONFIGS = [(0, -1, -1), (1, -1, -1), (2, -1, -1), (3, -1, -1), (0, 1, 1), (3, 2, 8), (2, 8, 2), (5, -1, -1),
           (5, 2, 1), (6, -1, -1), (6, 2, 4)]


def _exp_engine(precision, n=6000, md=15, seed=3):
    """A Poisson-driven iaf_psc_exp network with delays in [md, 2 md + 5]
    and weights exact in the FP32 form's fixed point (multiples of 1/64 pA)
    and dyadic in FP64."""
    rng = np.random.default_rng(seed)
    deg = rng.integers(100, 400, n)
    row = np.concatenate([[0], np.cumsum(deg)]).astype(np.int64)
    nnz = int(row[-1])
    tgt = rng.integers(0, n, nnz).astype(np.int32)
    w = rng.choice([40.0, 20.5, -80.0, -161.25], nnz, p=[0.4, 0.4, 0.1, 0.1])
    d = rng.integers(md, 2 * md + 6, nnz).astype(np.int32)
    eng = _abi.Engine([(_abi.NG_IAF_PSC_EXP, n)], 0.1, md, 2 * md + 5, precision=precision)
    eng.set_var(0, "V_m_rel", rng.uniform(0.0, 14.0, n))
    eng.set_connections(row, tgt, w, d)
    eng.set_recording(np.ones(n, dtype=np.uint8))
    eng.set_poisson(np.full(n, 9000.0), np.full(n, 40.0), np.full(n, md, dtype=np.int32), 0, 10**9, 11)
    return eng


def _delta_engine(fx):
    """The golden balanced iaf_psc_delta network (dyadic weights, FP64)."""
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


def _finish(eng, var="V_m_rel"):
    s, t = eng.spikes()
    V = eng.get_var(0, var)
    st = eng.stats()
    tn = eng.tuned()
    eng.close()
    o = np.lexsort((s, t))
    return s[o], t[o], V, st, tn


def _same(a, b):
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])
    np.testing.assert_array_equal(a[2], b[2])
    assert a[3]["syn_events"] == b[3]["syn_events"]


@pytest.mark.parametrize("precision", [_abi.NG_FP32, _abi.NG_FP64])
def test_every_configuration_gives_the_same_result(precision):
    ref = None
    for cfg in CONFIGS:
        eng = _exp_engine(precision)
        eng.set_tuning(0, *cfg)
        for k in (7, 23, 970):          # partial slices, then graphs of slices
            eng.simulate(k)
        r = _finish(eng)
        assert r[4]["state"] == "fixed"
        assert r[4]["update_variant"] == cfg[0]
        if ref is None:
            ref = r
            assert len(r[0]) > 1000
        else:
            _same(r, ref)


def test_autotuner_measures_then_caches(golden):
    fx = golden("c0_delta_balanced.npz")
    fixed = _delta_engine(fx)
    fixed.set_tuning(0, 2, -1, -1)
    fixed.simulate(9000)
    ref = _finish(fixed)
    tuned = _delta_engine(fx)
    tuned.set_tuning(2)                 # measure even if the process cache knows this shape
    tuned.simulate(9000)                # long enough for the probe and every trial group
    a = _finish(tuned)
    _same(a, ref)
    t = a[4]
    assert t["state"] == "tuned"
    # every update kernel; then the delivery launch shapes unless the
    # persistent kernel (which delivers inside itself) won
    assert len(t["candidates"]) >= (5 if t["update_variant"] == 5 else 8)
    assert all(c["us_per_slice"] > 0 for c in t["candidates"])
    best = min(t["candidates"], key=lambda c: c["us_per_slice"])
    assert (t["update_variant"], t["deliver_ctas_per_sm"], t["deliver_chunks_per_warp"]) in \
        {(c["update_variant"], c["deliver_ctas_per_sm"], c["deliver_chunks_per_warp"]) for c in t["candidates"]}
    assert (best["update_variant"], best["deliver_ctas_per_sm"], best["deliver_chunks_per_warp"]) == \
        (t["update_variant"], t["deliver_ctas_per_sm"], t["deliver_chunks_per_warp"])
    again = _delta_engine(fx)
    again.simulate(9000)                # default mode: the process cache first
    b = _finish(again)
    _same(b, ref)
    assert b[4]["state"] == "cached"
    assert (b[4]["update_variant"], b[4]["deliver_ctas_per_sm"], b[4]["deliver_chunks_per_warp"]) == \
        (t["update_variant"], t["deliver_ctas_per_sm"], t["deliver_chunks_per_warp"])


def test_short_calls_leave_tuning_pending(golden):
    fx = golden("c0_delta_balanced.npz")
    eng = _delta_engine(fx)
    eng.set_tuning(2)
    for _ in range(10):
        eng.simulate(45)
    t = eng.tuned()
    eng.close()
    assert t["state"] == "pending"


def test_tuning_arguments_checked():
    eng = _exp_engine(_abi.NG_FP32, n=500)
    with pytest.raises(_abi.EngineError):
        eng.set_tuning(0, 7, -1, -1)
    with pytest.raises(_abi.EngineError):
        eng.set_option("no_such_option", 1)
    with pytest.raises(_abi.EngineError):
        eng.set_option("gather", 1)      # a static engine has no per-target gather
    eng.close()


@pytest.mark.parametrize("precision", [_abi.NG_FP64, _abi.NG_FP32])
def test_aeif_binning_changes_no_result(precision):
    """aeif_cond_alpha neurons ordered by their RKF45 step size before each
    slice (so a warp's neurons need similar numbers of sub-steps) give the
    raster and state of the identity order: only which thread computes a
    neuron changes."""
    def run(binning):
        n = 3000
        rng = np.random.default_rng(21)
        deg = rng.integers(40, 160, n)
        row = np.concatenate([[0], np.cumsum(deg)]).astype(np.int64)
        nnz = int(row[-1])
        eng = _abi.Engine([(_abi.NG_AEIF_COND_ALPHA, n)], 0.1, 15, 30, precision=precision)
        eng.set_option("aeif_binning", binning)
        eng.set_var(0, "tau_syn_ex", np.full(n, 1.0))
        eng.set_var(0, "V_m", rng.uniform(-70.6, -52.0, n))
        eng.set_connections(row, rng.integers(0, n, nnz).astype(np.int32),
                            rng.choice([1.0, 0.5, -2.0, -4.0], nnz), rng.integers(15, 31, nnz).astype(np.int32))
        eng.set_recording(np.ones(n, dtype=np.uint8))
        eng.set_poisson(np.full(n, 15000.0), np.full(n, 1.0), np.full(n, 15, dtype=np.int32), 0, 10**9, 5)
        for k in (7, 1493, 1500):
            eng.simulate(k)
        return _finish(eng, "V_m")

    a, b = run(0), run(1)
    assert len(a[0]) > 500
    _same(a, b)


@pytest.mark.parametrize("precision,model", [
    (_abi.NG_FP64, _abi.NG_IAF_PSC_EXP), (_abi.NG_FP32, _abi.NG_IAF_PSC_EXP),
    (_abi.NG_FP64, _abi.NG_IAF_PSC_DELTA), (_abi.NG_FP64, _abi.NG_IAF_PSC_ALPHA),
])
def test_persistent_multi_group_equals_graph_form(precision, model):
    """A network larger than one resident wave of the persistent kernel
    (30,000 neurons: each CTA walks several 32-neuron groups per slice, their
    state reloaded from memory) gives the graph form's raster, state and
    event count bit for bit (dyadic weights: order-independent ring sums)."""
    def run(variant):
        n, md = 30000, 15
        rng = np.random.default_rng(8)
        deg = rng.integers(100, 300, n)
        row = np.concatenate([[0], np.cumsum(deg)]).astype(np.int64)
        nnz = int(row[-1])
        tgt = rng.integers(0, n, nnz).astype(np.int32)
        w = rng.choice([40.0, 20.5, -80.0, -161.25], nnz, p=[0.4, 0.4, 0.1, 0.1])
        if model == _abi.NG_IAF_PSC_DELTA:
            w = w / 128.0
        d = rng.integers(md, 2 * md + 6, nnz).astype(np.int32)
        eng = _abi.Engine([(model, n)], 0.1, md, 2 * md + 5, precision=precision)
        eng.set_tuning(0, variant, -1, -1)
        eng.set_var(0, "V_m_rel", rng.uniform(0.0, 14.0, n))
        eng.set_connections(row, tgt, w, d)
        eng.set_recording(np.ones(n, dtype=np.uint8))
        drive_w = 0.3 if model == _abi.NG_IAF_PSC_DELTA else 40.0
        eng.set_poisson(np.full(n, 9000.0), np.full(n, drive_w), np.full(n, md, dtype=np.int32), 0, 10**9, 11)
        for k in (7, 23, 970, 1500):
            eng.simulate(k)
        return _finish(eng)
    a, b = run(0), run(5)
    assert len(a[0]) > 5000
    assert b[4]["update_variant"] == 5
    _same(a, b)
