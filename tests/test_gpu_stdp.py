"""stdp_pl_synapse_hom on the engine: a Poisson-driven network whose
excitatory connections of 500 sources are plastic (models/stdp_pl_synapse_hom.h
with nestkernel/archiving_node.cpp's postsynaptic history) runs in partial
slices, slice graphs and slice by slice.  The raster equals the CPU oracle's
and every plastic weight equals the oracle's to rtol 1e-10 (the engine's and
the host's exp/pow may differ in the last bit; the static weights are dyadic).
The FP32 form (FP32 state, fixed-point rings, FP64 weights) follows FP64 in
rate and mean weight change; a target history that cannot reach back to a
presynaptic neuron's previous spike is an error."""

import numpy as np
import pytest

import oracle as O
from nestgpu import _abi

pytestmark = pytest.mark.gpu

H = 0.1
MODELS = {_abi.NG_IAF_PSC_DELTA: "iaf_psc_delta", _abi.NG_IAF_PSC_EXP: "iaf_psc_exp",
          _abi.NG_IAF_PSC_ALPHA: "iaf_psc_alpha"}
RULE = dict(lam=0.05, alpha=1.2, mu=0.4, tau_plus=15.0)


def _spec(model, md, maxd, n=2000, seed=3):
    rng = np.random.default_rng(seed)
    deg = rng.integers(40, 120, n)
    src = np.repeat(np.arange(n), deg)
    tgt = rng.integers(0, n, len(src))
    d = rng.integers(md, maxd + 1, len(src))
    scale = 1.0 / 64.0 if model == _abi.NG_IAF_PSC_DELTA else 1.0
    w = rng.choice([24.0, 12.5, -48.0, -100.0], len(src)) * scale
    n_pl = 500
    pdeg = rng.integers(20, 60, n_pl)
    psrc = np.repeat(np.arange(n_pl), pdeg)
    ptgt = rng.integers(0, n, len(psrc))
    pd = rng.integers(md, maxd + 1, len(psrc))
    pw = rng.uniform(5.0, 40.0, len(psrc)) * scale
    V0 = rng.uniform(0.0, 15.0, n)
    tau_minus = rng.uniform(15.0, 40.0, n)
    drive = (12000.0, 16.0 * scale if model != _abi.NG_IAF_PSC_DELTA else 0.25)
    return dict(n=n, md=md, maxd=maxd, src=src, tgt=tgt, w=w, d=d, psrc=psrc, ptgt=ptgt, pd=pd, pw=pw, V0=V0,
                tau_minus=tau_minus, drive=drive, n_pl=n_pl)


def _csr(src, n_src, *cols):
    o = np.argsort(src, kind="stable")
    row = np.zeros(n_src + 1, dtype=np.int64)
    np.cumsum(np.bincount(src, minlength=n_src), out=row[1:])
    return row, [np.asarray(c)[o] for c in cols], o


def _engine_run(model, sp, precision, calls):
    n = sp["n"]
    eng = _abi.Engine([(model, n)], H, sp["md"], sp["maxd"], precision=precision)
    eng.set_var(0, "V_m_rel", sp["V0"])
    eng.set_var(0, "tau_minus", sp["tau_minus"])
    row, (tg, w, d), _ = _csr(sp["src"], n, sp["tgt"], sp["w"], sp["d"])
    eng.set_connections(row, tg, w, d)
    prow, (ptg, pw, pd), po = _csr(sp["psrc"], sp["n_pl"], sp["ptgt"], sp["pw"], sp["pd"])
    eng.set_plastic(prow, ptg, pw, pd, **RULE)
    eng.set_recording(np.ones(n, dtype=np.uint8))
    eng.set_poisson(np.full(n, sp["drive"][0]), np.full(n, sp["drive"][1]), np.full(n, sp["md"]), 0, 10**9, 5)
    for k in calls:
        if k == "graphs_off":
            eng.set_graph_slices(0)
        else:
            eng.simulate(k)
    s, t = eng.spikes()
    V = eng.get_var(0, "V_m_rel")
    wout = np.empty(len(po))
    wout[po] = eng.plastic_weights()
    assert np.array_equal(eng.get_var(0, "tau_minus"), sp["tau_minus"])
    eng.close()
    o = np.lexsort((s, t))
    return s[o].astype(np.int64), t[o].astype(np.int64), V, wout


def _oracle_run(model, sp, steps):
    n = sp["n"]
    net = O.OracleNet(MODELS[model], n, H, sp["md"], sp["maxd"])
    net.set("V_m_rel", sp["V0"])
    net.set("tau_minus", sp["tau_minus"])
    net.set_edges(sp["src"], sp["tgt"], sp["w"], sp["d"])
    net.set_plastic(sp["psrc"], sp["ptgt"], sp["pw"], sp["pd"], n_src=sp["n_pl"], **RULE)
    net.set_poisson(np.full(n, sp["drive"][0]), np.full(n, sp["drive"][1]), sp["md"], 5)
    net.set_record(np.ones(n, dtype=np.uint8))
    net.run(steps)
    s, t = net.spikes()
    o = np.lexsort((s, t))
    return s[o].astype(np.int64), t[o].astype(np.int64), net.get("V_m_rel"), net.plastic_weights()


@pytest.mark.parametrize("model,md,maxd", [
    (_abi.NG_IAF_PSC_DELTA, 10, 20),
    (_abi.NG_IAF_PSC_EXP, 2, 30),
    (_abi.NG_IAF_PSC_ALPHA, 15, 15),
])
def test_stdp_engine_equals_oracle(model, md, maxd):
    sp = _spec(model, md, maxd)
    calls = [7, 13, 3, 977, "graphs_off", 1000]
    es, et, eV, ew = _engine_run(model, sp, _abi.NG_FP64, calls)
    os_, ot, oV, ow = _oracle_run(model, sp, 2000)
    n_pl_spk = int(np.sum(es < sp["n_pl"]))
    print(f"{MODELS[model]}: {len(es)} spikes ({n_pl_spk} of plastic sources), mean weight "
          f"{sp['pw'].mean():.3f} -> {ew.mean():.3f}, {np.sum(ew != sp['pw'])} of {len(ew)} changed")
    assert len(es) > 2000 and n_pl_spk > 300
    np.testing.assert_array_equal(es, os_)
    np.testing.assert_array_equal(et, ot)
    np.testing.assert_allclose(eV, oV, rtol=1e-10, atol=1e-10)
    assert np.sum(ew != sp["pw"]) > 0.5 * len(ew)
    np.testing.assert_allclose(ew, ow, rtol=1e-10)


def test_stdp_fp32_form_follows_fp64():
    sp = _spec(_abi.NG_IAF_PSC_EXP, 10, 20, n=4000, seed=9)
    calls = [5000]
    s64, _, _, w64 = _engine_run(_abi.NG_IAF_PSC_EXP, sp, _abi.NG_FP64, calls)
    s32, _, _, w32 = _engine_run(_abi.NG_IAF_PSC_EXP, sp, _abi.NG_FP32, calls)
    dw64, dw32 = np.mean(w64 - sp["pw"]), np.mean(w32 - sp["pw"])
    print(f"spikes fp64 {len(s64)} fp32 {len(s32)}; mean weight change fp64 {dw64:+.4f} fp32 {dw32:+.4f}")
    assert abs(len(s32) / len(s64) - 1) <= 0.02
    assert abs(dw32 - dw64) <= 0.05 * abs(dw64) + 1e-3


def test_stdp_long_silent_source_equals_oracle():
    """A source firing every ~77 ms onto targets firing every ~0.9 ms: each
    target's 64-entry history is flushed many times between two presynaptic
    spikes (its oldest entries' facilitation applied early, then dropped),
    and the weights still equal the oracle's, which keeps every entry."""
    n = 4
    I_e = np.array([375.2, 5000.0, 3000.0, 1000.0])     # V_inf 15.008 mV: a spike every ~77 ms; then fast ones
    t_ref = np.array([2.0, 0.1, 0.3, 0.5])
    row = np.array([0, 3, 3, 3, 3], dtype=np.int64)
    tgt = np.array([1, 2, 3], np.int32)
    w0 = np.array([1.0, 2.0, 3.0])
    dl = np.array([1, 3, 5], np.int32)
    eng = _abi.Engine([(_abi.NG_IAF_PSC_DELTA, n)], H, 1, 5)
    eng.set_var(0, "I_e", I_e)
    eng.set_var(0, "t_ref", t_ref)
    eng.set_connections(np.array([0, 1, 1, 1, 1], dtype=np.int64), np.array([0], np.int32), np.array([0.0]),
                        np.array([1], np.int32))
    rule = dict(RULE, alpha=0.0513)
    eng.set_plastic(row, tgt, w0, dl, **rule)
    eng.set_recording(np.ones(n, dtype=np.uint8))
    for k in (1234, 5000, 13766):
        eng.simulate(k)
    s, t = eng.spikes()
    w = eng.plastic_weights()
    eng.close()
    net = O.OracleNet("iaf_psc_delta", n, H, 1, 5)
    net.set("I_e", I_e)
    net.set("t_ref", t_ref)
    net.set_plastic(np.zeros(3, np.int64), tgt, w0, dl, n_src=n, **rule)
    net.set_record(np.ones(n, dtype=np.uint8))
    net.run(20000)
    os_, ot = net.spikes()
    assert np.sum(s == 0) >= 20 and np.sum(s == 1) > 1500
    o1, o2 = np.lexsort((s, t)), np.lexsort((os_, ot))
    np.testing.assert_array_equal(s[o1], os_[o2])
    np.testing.assert_array_equal(t[o1], ot[o2])
    assert np.all(w != w0)
    np.testing.assert_allclose(w, net.plastic_weights(), rtol=1e-10)


def test_stdp_history_ring_full_is_an_error():
    """More than 32 postsynaptic spikes of one neuron within max_delay (a
    target spiking every 0.2 ms, plastic delays of 10 ms): the entries the
    next slice needs no longer fit the 64-entry ring, and the engine says so
    at its next synchronisation."""
    eng = _abi.Engine([(_abi.NG_IAF_PSC_DELTA, 2)], H, 1, 100)
    eng.set_var(0, "I_e", np.array([375.2, 50000.0]))
    eng.set_var(0, "t_ref", np.array([2.0, 0.1]))
    eng.set_connections(np.array([0, 1, 1], dtype=np.int64), np.array([0], np.int32), np.array([0.0]),
                        np.array([1], np.int32))
    eng.set_plastic(np.array([0, 1], dtype=np.int64), np.array([1], np.int32), np.array([1.0]),
                    np.array([100], np.int32))
    with pytest.raises(_abi.EngineError) as err:
        eng.simulate(2000)
        eng.sync()
    assert err.value.code == _abi.NG_ERR_CAPACITY and "history" in str(err.value)
    eng.close()


def test_stdp_arguments_checked():
    eng = _abi.Engine([(_abi.NG_IAF_PSC_EXP, 10)], H, 2, 5)
    row = np.array([0, 1], dtype=np.int64)
    with pytest.raises(_abi.EngineError):
        eng.set_plastic(row, np.array([10], np.int32), np.array([1.0]), np.array([2], np.int32))   # target
    with pytest.raises(_abi.EngineError):
        eng.set_plastic(row, np.array([3], np.int32), np.array([-1.0]), np.array([2], np.int32))   # weight < 0
    with pytest.raises(_abi.EngineError):
        eng.set_plastic(row, np.array([3], np.int32), np.array([1.0]), np.array([1], np.int32))    # delay < min
    with pytest.raises(_abi.EngineError):
        eng.set_var(0, "tau_minus", np.zeros(10))
    eng.close()


def test_hpc_benchmark_style_network_vs_oracle(nest):
    """The reference's hpc_benchmark network at scale 0.1 with in-degrees
    thinned to a tenth, through the front-end: iaf_psc_alpha, E->E
    stdp_pl_synapse_hom_hpc (alpha 0.0513, lambda 0.1, mu 0.4, tau_plus
    15 ms, tau_minus 30 ms), static E->I, I->E, I->I, Poisson drive, delays
    1.5 ms.  Raster and plastic weights equal the oracle's copy of the same
    network (weights to rtol 1e-10)."""
    from nestgpu import workloads
    from nestgpu.kernel import KERNEL

    E, I, sr = workloads.hpc_benchmark(nest, scale=0.1, indegree_scale=0.1, seed=7)
    JE = nest.GetDefaults("syn_ex", "weight")
    net, c = O.net_from_kernel(KERNEL)
    nest.Simulate(300.0)
    net.run(3000)
    ev = sr.events
    s = np.asarray(ev["senders"], dtype=np.int64) - 1
    st = np.rint(np.asarray(ev["times"]) / 0.1).astype(np.int64)
    os_, ost = net.spikes()
    print(f"hpc_benchmark scale 0.1: {len(s)} spikes in 300 ms, JE {JE:.3f} pA")
    assert len(s) > 1000
    o1, o2 = np.lexsort((s, st)), np.lexsort((os_, ost))
    np.testing.assert_array_equal(s[o1], os_[o2])
    np.testing.assert_array_equal(st[o1], ost[o2])
    conns = nest.GetConnections(synapse_model="stdp_pl_synapse_hom_hpc")
    w = np.asarray(conns.get("weight"))
    src = np.asarray(conns.get("source")) - 1
    tgt = np.asarray(conns.get("target")) - 1
    ow = net.plastic_weights()           # engine CSR order
    p = c["pl"]
    osrc = np.repeat(np.arange(c["N"]), np.diff(p["row"]))
    # both lists sorted by (source, target); multapses keep their stable order
    k1 = np.lexsort((tgt, src))
    k2 = np.lexsort((p["tgt"], osrc))
    assert np.sum(w != JE) > 0.5 * len(w)
    np.testing.assert_allclose(w[k1], ow[k2], rtol=1e-10)
