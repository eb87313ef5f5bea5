"""Network builders for the benchmark configurations, written with the
PyNEST API (they run unchanged on the reference).  Sizes and parameters
follow the benchmark definitions; the reference's published microcircuit
data is not used (synthetic stand-ins with the stated shapes).

c1: Poisson-driven iaf_psc_exp network, 12,500 neurons (10,000 exc, 2,500
    inh), tau_syn 0.5 ms, fixed_indegree K_E=1,000, K_I=250, J=87.8 pA, g=5,
    delay 1.5 ms, 8 kHz Poisson drive per neuron, V_m ~ N(-58, 10) mV.
"""

import numpy as np


def brunel_exp(nest, n_exc=10000, n_inh=2500, k_exc=1000, k_inh=250, J=87.8, g=5.0, rate=8000.0, delay=1.5,
               tau_syn=0.5, seed=4242, record=True, precision="fp64", resolution=0.1, extra_kernel=None):
    """Build a Brunel-type iaf_psc_exp network; returns (pop, recorder)."""
    nest.ResetKernel()
    kw = dict(resolution=resolution, rng_seed=seed, precision=precision)
    if extra_kernel:
        kw.update(extra_kernel)
    nest.set(**kw)
    N = n_exc + n_inh
    pop = nest.Create("iaf_psc_exp", N, params={"tau_syn_ex": tau_syn, "tau_syn_in": tau_syn})
    rng = np.random.default_rng(seed)
    pop.set(V_m=rng.normal(-58.0, 10.0, N))
    nest.Connect(pop[:n_exc], pop, {"rule": "fixed_indegree", "indegree": k_exc, "allow_autapses": False},
                 {"weight": J, "delay": delay})
    nest.Connect(pop[n_exc:], pop, {"rule": "fixed_indegree", "indegree": k_inh, "allow_autapses": False},
                 {"weight": -g * J, "delay": delay})
    pg = nest.Create("poisson_generator", params={"rate": rate})
    nest.Connect(pg, pop, syn_spec={"weight": J, "delay": delay})
    sr = None
    if record:
        sr = nest.Create("spike_recorder")
        nest.Connect(pop, sr, syn_spec={"delay": delay})
    return pop, sr


def c1(nest, precision="fp64", seed=4242):
    return brunel_exp(nest, precision=precision, seed=seed)


def brunel_exp_batch(nest, copies, n_exc=10000, n_inh=2500, k_exc=1000, k_inh=250, J=87.8, g=5.0, rate=8000.0,
                     delay=1.5, tau_syn=0.5, seed=4242, precision="fp32", record=True):
    """`copies` independent realizations of the Brunel-type iaf_psc_exp network
    in one kernel: the engine advances them together (one node-update and one
    delivery launch per slice for all of them, concatenated CSRs)."""
    nest.ResetKernel()
    nest.set(resolution=0.1, rng_seed=seed, precision=precision)
    N = n_exc + n_inh
    rng = np.random.default_rng(seed)
    pops, recs = [], []
    for _ in range(copies):
        pop = nest.Create("iaf_psc_exp", N, params={"tau_syn_ex": tau_syn, "tau_syn_in": tau_syn})
        pop.set(V_m=rng.normal(-58.0, 10.0, N))
        nest.Connect(pop[:n_exc], pop, {"rule": "fixed_indegree", "indegree": k_exc, "allow_autapses": False},
                     {"weight": J, "delay": delay})
        nest.Connect(pop[n_exc:], pop, {"rule": "fixed_indegree", "indegree": k_inh, "allow_autapses": False},
                     {"weight": -g * J, "delay": delay})
        pg = nest.Create("poisson_generator", params={"rate": rate})
        nest.Connect(pg, pop, syn_spec={"weight": J, "delay": delay})
        if record:
            sr = nest.Create("spike_recorder")
            nest.Connect(pop, sr, syn_spec={"delay": delay})
            recs.append(sr)
        pops.append(pop)
    return pops, recs
