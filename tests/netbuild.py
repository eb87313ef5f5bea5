"""Builders shared by the parity tests: the golden fixtures' networks,
written with the PyNEST API so they run on the engine (nestgpu) unchanged."""

import numpy as np


def build_c0(nest, fx, precision="fp64"):
    """Config 0 with the reference's exported graph (connect-arrays path)."""
    nest.ResetKernel()
    nest.set(resolution=0.1, precision=precision)
    C_m, tau_m, t_ref, E_L, V_th, V_reset = fx["params"]
    pop = nest.Create("iaf_psc_delta", len(fx["I_e"]),
                      params=dict(C_m=C_m, tau_m=tau_m, t_ref=t_ref, E_L=E_L, V_th=V_th, V_reset=V_reset))
    pop.set(I_e=fx["I_e"], V_m=fx["V0"])
    src = fx["src"].astype(np.int64) + 1
    tgt = fx["tgt"].astype(np.int64) + 1
    w = np.where(fx["exc"], 0.125, -0.625)
    nest.Connect(src, tgt, "one_to_one", {"weight": w, "delay": 1.5})
    sr = nest.Create("spike_recorder")
    nest.Connect(pop, sr, syn_spec={"delay": 1.5})
    return pop, sr


def build_exp_net(nest, fx, precision="fp64"):
    nest.ResetKernel()
    nest.set(resolution=0.1, precision=precision)
    n = len(fx["I_e"])
    pop = nest.Create("iaf_psc_exp", n, params=dict(tau_syn_ex=0.5, tau_syn_in=0.5, t_ref=2.0))
    pop.set(I_e=fx["I_e"], V_m=fx["V0"])
    nest.Connect(fx["src"].astype(np.int64) + 1, fx["tgt"].astype(np.int64) + 1, "one_to_one",
                 {"weight": fx["w"], "delay": fx["d"]})
    sr = nest.Create("spike_recorder")
    nest.Connect(pop, sr)
    mm = nest.Create("multimeter", params={"interval": 0.1, "record_from": ["V_m", "I_syn_ex", "I_syn_in"]})
    nest.Connect(mm, pop[fx["rec_idx"].tolist()])
    return pop, sr, mm


def raster(sr):
    ev = sr.events
    s = np.asarray(ev["senders"], dtype=np.int64)
    t = np.rint(np.asarray(ev["times"]) / 0.1).astype(np.int64)
    o = np.lexsort((s, t))
    return s[o], t[o]
