"""Host side of stdp_pl_synapse_hom in the PyNEST-compatible front-end (no
GPU): the synapse model table with the reference's defaults
(models/stdp_pl_synapse_hom.cpp STDPPLHomCommonProperties), CopyModel /
SetDefaults / GetDefaults, Connect into the plastic connection table,
GetConnections by synapse model, the common-property rules, the neurons'
tau_minus (nestkernel/archiving_node.cpp), and the lowering to the engine's
plastic CSR (stable order by source, one set of common properties)."""

import numpy as np
import pytest


def test_models_and_defaults(nest):
    syn = nest.Models("synapses")
    for m in ("static_synapse", "stdp_pl_synapse_hom", "stdp_pl_synapse_hom_hpc", "static_synapse_hpc"):
        assert m in syn
    d = nest.GetDefaults("stdp_pl_synapse_hom")
    assert (d["lambda"], d["alpha"], d["mu"], d["tau_plus"], d["weight"], d["delay"]) == (0.1, 1.0, 0.4, 20.0, 1.0,
                                                                                         1.0)
    nest.CopyModel("stdp_pl_synapse_hom", "stdp_x", {"alpha": 0.0513, "tau_plus": 15.0, "weight": 2.5})
    d = nest.GetDefaults("stdp_x")
    assert (d["alpha"], d["tau_plus"], d["weight"], d["lambda"]) == (0.0513, 15.0, 2.5, 0.1)
    assert nest.GetDefaults("stdp_pl_synapse_hom", "alpha") == 1.0
    with pytest.raises(nest.KernelException):
        nest.CopyModel("stdp_pl_synapse_hom", "stdp_x")
    with pytest.raises(nest.BadProperty):
        nest.CopyModel("stdp_pl_synapse_hom", "stdp_bad", {"tau_plus": 0.0})
    assert "stdp_bad" not in nest.Models("synapses")
    with pytest.raises(nest.BadProperty):
        nest.SetDefaults("stdp_pl_synapse_hom", {"no_such_key": 1.0})
    nest.CopyModel("static_synapse", "syn_ex", {"weight": 87.8})
    assert nest.GetDefaults("syn_ex", "weight") == 87.8


def test_connect_plastic_and_get_connections(nest):
    nest.set(resolution=0.1)
    pop = nest.Create("iaf_psc_alpha", 20)
    pg = nest.Create("poisson_generator", params={"rate": 1000.0})
    nest.SetDefaults("stdp_pl_synapse_hom", {"delay": 1.5, "weight": 3.0})
    nest.Connect(pop[:10], pop, {"rule": "fixed_indegree", "indegree": 4, "allow_autapses": False},
                 {"synapse_model": "stdp_pl_synapse_hom"})
    nest.Connect(pop[10:], pop, {"rule": "fixed_indegree", "indegree": 2}, {"weight": -5.0, "delay": 1.0})
    nest.Connect(pg, pop, syn_spec={"weight": 20.0})
    assert nest.GetKernelStatus("num_connections") == 80 + 40 + 20
    pl = nest.GetConnections(synapse_model="stdp_pl_synapse_hom")
    assert len(pl) == 80
    assert set(pl.get("synapse_model")) == {"stdp_pl_synapse_hom"}
    assert np.all(np.asarray(pl.get("weight")) == 3.0) and np.allclose(pl.get("delay"), 1.5)
    assert np.all(np.asarray(pl.get("source")) <= 10)
    assert np.all(np.asarray(pl.get("alpha")) == 1.0)
    st = nest.GetConnections(synapse_model="static_synapse")
    assert len(st) == 60
    assert len(nest.GetConnections()) == 140
    assert len(nest.GetConnections(source=pop[:1])) == 4
    # weights of plastic connections set through the collection
    sub = nest.GetConnections(source=pop[:2], synapse_model="stdp_pl_synapse_hom")
    sub.set(weight=7.0)
    assert np.all(np.asarray(nest.GetConnections(source=pop[:2], synapse_model="stdp_pl_synapse_hom")
                             .get("weight")) == 7.0)
    with pytest.raises(nest.BadProperty):
        sub.set(weight=-1.0)
    with pytest.raises(nest.BadProperty):
        sub.set(alpha=0.5)
    # lowering: a CSR over neuron sources with the model's common properties
    from nestgpu.kernel import KERNEL

    c = KERNEL.compile()
    p = c["pl"]
    assert p["row"][-1] == 80 and len(p["row"]) == c["N"] + 1
    assert p["common"] == {"lambda": 0.1, "alpha": 1.0, "mu": 0.4, "tau_plus": 20.0}
    assert c["min_delay"] == 10 and c["max_delay"] == 15
    src, tgt, w, d, _ = KERNEL.plastic_edges()
    eng_src = c["node_to_eng"][src][p["order"]]
    assert np.all(np.diff(eng_src) >= 0)
    assert np.array_equal(p["tgt"], c["node_to_eng"][tgt][p["order"]])
    assert np.array_equal(p["w"], w[p["order"]])


def test_common_properties_and_checks(nest):
    pop = nest.Create("iaf_psc_exp", 5)
    pg = nest.Create("poisson_generator")
    with pytest.raises(nest.BadProperty):
        nest.Connect(pop, pop, syn_spec={"synapse_model": "stdp_pl_synapse_hom", "alpha": 0.5})
    with pytest.raises(nest.BadProperty):
        nest.Connect(pop, pop, syn_spec={"synapse_model": "stdp_pl_synapse_hom", "weight": -1.0})
    with pytest.raises(nest.KernelException):
        nest.Connect(pg, pop, syn_spec={"synapse_model": "stdp_pl_synapse_hom"})
    with pytest.raises(nest.BadProperty):
        nest.Connect(pop, pop, syn_spec={"synapse_model": "tsodyks_synapse"})
    nest.CopyModel("stdp_pl_synapse_hom", "stdp_a", {"mu": 0.5})
    nest.Connect(pop, pop, syn_spec={"synapse_model": "stdp_pl_synapse_hom"})
    nest.Connect(pop, pop, syn_spec={"synapse_model": "stdp_a"})
    from nestgpu.kernel import KERNEL

    with pytest.raises(NotImplementedError):
        KERNEL.compile()
    nest.SetDefaults("stdp_a", {"mu": 0.4})
    assert KERNEL.compile()["pl"]["common"]["mu"] == 0.4
    assert len(nest.GetConnections(synapse_model="stdp_a")) == 25


def test_tau_minus_on_iaf_neurons(nest):
    for m in ("iaf_psc_delta", "iaf_psc_exp", "iaf_psc_alpha"):
        n = nest.Create(m, 3, params={"tau_minus": 30.0})
        assert list(n.get("tau_minus")) == [30.0] * 3
        assert nest.GetDefaults(m, "tau_minus") == 20.0
        n.set(tau_minus=[10.0, 20.0, 40.0])
        assert list(n.get("tau_minus")) == [10.0, 20.0, 40.0]
        with pytest.raises(nest.BadProperty):
            n.set(tau_minus=0.0)
        assert list(n.get("tau_minus")) == [10.0, 20.0, 40.0]
