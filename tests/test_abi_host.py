"""CPU-side checks of the C ABI library and of the front-end's host logic.

No kernel runs here: the library must load and export every symbol the
header declares, refuse to create an engine without a GPU (no CPU
fallback), and the front-end's network compilation -- fed to the CPU oracle
-- must reproduce the reference's raster."""

import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "nestgpu.h")


def declared_symbols():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(ng_\w+)\s*\(", src, re.M)))


def test_header_and_binding_agree():
    from nestgpu import _abi

    assert declared_symbols() == sorted(_abi.EXPORTED)


def test_library_exports_every_declared_symbol():
    from nestgpu import _abi

    L = _abi.load()
    for name in declared_symbols():
        assert hasattr(L, name), name
    assert L.ng_abi_version() == 1


def test_no_cpu_fallback_without_gpu():
    from nestgpu import _abi

    if _abi.device_count() > 0:
        pytest.skip("a GPU is visible")
    with pytest.raises(_abi.EngineError) as ei:
        _abi.Engine([(_abi.NG_IAF_PSC_DELTA, 10)], 0.1, 1, 1)
    assert ei.value.code == _abi.NG_ERR_CUDA
    assert "CUDA" in str(ei.value)


def test_create_rejects_bad_config():
    from nestgpu import _abi

    with pytest.raises(_abi.EngineError) as ei:
        _abi.Engine([(_abi.NG_IAF_PSC_DELTA, 10)], 0.1, 3, 2)
    assert ei.value.code == _abi.NG_ERR_ARG


def test_frontend_compile_reproduces_reference_raster(nest, golden):
    """The front-end's graph, parameters and recorder lowering, run on the oracle."""
    import oracle as O
    from netbuild import build_c0

    from nestgpu.kernel import KERNEL

    fx = golden("c0_delta_balanced.npz")
    build_c0(nest, fx)
    net, c = O.net_from_kernel(KERNEL)
    assert c["min_delay"] == 15 and c["max_delay"] == 15
    net.run(10000)
    s, t = net.spikes()
    o = np.lexsort((s, t))
    np.testing.assert_array_equal(s[o], fx["spike_senders"].astype(np.int32))
    np.testing.assert_array_equal(t[o], fx["spike_steps"].astype(np.int64))


def test_E_L_relative_bookkeeping(nest):
    """models/iaf_psc_delta.cpp Parameters_::set: V_th, V_reset and V_m are
    stored relative to E_L and shifted when E_L changes, so their absolute
    values stay put (values checked against the reference)."""
    n = nest.Create("iaf_psc_delta")
    assert n.get("V_th") == -55.0 and n.get("V_m") == -70.0
    n.set(E_L=-65.0)
    assert n.get(["V_th", "V_reset", "V_m"]) == {"V_th": -55.0, "V_reset": -70.0, "V_m": -70.0}
    n.set(E_L=-60.0, V_th=-40.0)
    assert n.get(["V_th", "V_reset", "V_m"]) == {"V_th": -40.0, "V_reset": -70.0, "V_m": -70.0}
    with pytest.raises(nest.BadProperty):
        n.set(V_reset=-30.0)


def test_aeif_parameter_checks(nest):
    n = nest.Create("aeif_cond_alpha")
    with pytest.raises(nest.BadProperty):
        n.set(V_reset=10.0)
    with pytest.raises(nest.BadProperty):
        n.set(g_ex=-1.0)
    assert n.get("V_m") == -70.6


def test_delay_rounding_and_extrema(nest):
    """Time::delay_ms_to_steps rounds half up; min/max delay include device
    connections (connection_manager.cpp:485-530)."""
    a = nest.Create("iaf_psc_exp", 3)
    nest.Connect(a[0], a[1], syn_spec={"delay": 1.04})
    nest.Connect(a[1], a[2], syn_spec={"delay": 1.05})
    c = nest.GetConnections(a[:2]).get("delay")
    assert c == [1.0, 1.1]
    assert nest.GetKernelStatus("min_delay") == 1.0
    sr = nest.Create("spike_recorder")
    nest.Connect(a, sr, syn_spec={"delay": 0.5})
    assert nest.GetKernelStatus("min_delay") == 0.5
    assert nest.GetKernelStatus("max_delay") == pytest.approx(1.1)
    with pytest.raises(nest.BadProperty):
        nest.Connect(a[0], a[2], syn_spec={"delay": 0.01})


def test_connection_rules(nest):
    nest.set(rng_seed=11)
    pre = nest.Create("iaf_psc_exp", 200)
    post = nest.Create("iaf_psc_exp", 100)
    nest.Connect(pre, post, {"rule": "fixed_indegree", "indegree": 20, "allow_multapses": False})
    c = nest.GetConnections(pre, post)
    tgt = np.asarray(c.get("target"))
    src = np.asarray(c.get("source"))
    assert len(tgt) == 2000
    assert np.all(np.bincount(tgt - post.tolist()[0], minlength=100) == 20)
    pairs = set(zip(src.tolist(), tgt.tolist()))
    assert len(pairs) == 2000
    nest.ResetKernel()
    pop = nest.Create("iaf_psc_exp", 300)
    nest.Connect(pop, pop, {"rule": "pairwise_bernoulli", "p": 0.1, "allow_autapses": False})
    c = nest.GetConnections(pop, pop)
    s, t = np.asarray(c.get("source")), np.asarray(c.get("target"))
    assert np.all(s != t)
    assert abs(len(s) / (300 * 299) - 0.1) < 0.01
    nest.ResetKernel()
    pop = nest.Create("iaf_psc_delta", 50)
    nest.Connect(pop, pop, {"rule": "fixed_outdegree", "outdegree": 5, "allow_autapses": False})
    s = np.asarray(nest.GetConnections(pop).get("source"))
    assert np.all(np.bincount(s - 1, minlength=50) == 5)
    nest.ResetKernel()
    pop = nest.Create("iaf_psc_delta", 10)
    nest.Connect(pop, pop, "all_to_all", {"weight": nest.random.uniform(1.0, 2.0)})
    w = np.asarray(nest.GetConnections(pop).get("weight"))
    assert len(w) == 100 and np.all((w >= 1.0) & (w < 2.0))


def test_kernel_status_and_errors(nest):
    nest.resolution = 0.05
    assert nest.resolution == 0.05
    nest.Create("iaf_psc_delta")
    with pytest.raises(nest.KernelException):
        nest.resolution = 0.1
    with pytest.raises(nest.KernelException):
        nest.Create("no_such_model")
    with pytest.raises(nest.KernelException):
        nest.Simulate(0.123)
    assert "iaf_psc_exp" in nest.Models("nodes")
    assert nest.GetDefaults("static_synapse")["delay"] == 1.0


def test_unsupported_paths_fail_loudly(nest):
    n = nest.Create("iaf_psc_exp")
    with pytest.raises(NotImplementedError):
        n.set(delta=1.0)
    with pytest.raises(nest.BadProperty):
        nest.Connect(n, n, syn_spec={"synapse_model": "stdp_synapse"})
