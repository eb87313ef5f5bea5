"""Network builders for the benchmark configurations, written with the
PyNEST API (they run unchanged on the reference).  Sizes and parameters
follow the benchmark definitions; the reference's published microcircuit
data is not used (synthetic stand-ins with the stated shapes).

c1: Poisson-driven iaf_psc_exp network, 12,500 neurons (10,000 exc, 2,500
    inh), tau_syn 0.5 ms, fixed_indegree K_E=1,000, K_I=250, J=87.8 pA, g=5,
    delay 1.5 ms, 8 kHz Poisson drive per neuron, V_m ~ N(-58, 10) mV.
hpc_benchmark: the reference's HPC benchmark (iaf_psc_alpha, STDP E->E).
"""

import math

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


# ---------------------------------------------------------------------------
# hpc_benchmark: the reference's HPC benchmark network (pynest/examples/
# hpc_benchmark.py): iaf_psc_alpha, NE = 9000 scale, NI = 2250 scale,
# fixed in-degrees CE = 9000, CI = 2250 (independent of scale), E->E
# connections stdp_pl_synapse_hom, the rest static, delays 1.5 ms, one
# Poisson drive at 1.685 times the threshold rate.
# ---------------------------------------------------------------------------
HPC_TAU_SYN = 0.32582722403722841


def alpha_pa_per_mv(tau_m, tau_syn, C_m):
    """Current amplitude (pA) of an alpha-shaped PSC whose PSP peaks at 1 mV
    in a leaky membrane: the PSP's maximum lies where its derivative
    vanishes, t* = (W_-1(-exp(-1/a)/a) stretched) with a = tau_m / tau_syn,
    from the Lambert W function's -1 branch."""
    from scipy.special import lambertw

    a = tau_m / tau_syn
    b = 1.0 / tau_syn - 1.0 / tau_m
    t_peak = (1.0 / b) * (-lambertw(-math.exp(-1.0 / a) / a, k=-1).real - 1.0 / a)
    v_max = (math.e / (tau_syn * C_m * b)) * ((math.exp(-t_peak / tau_m) - math.exp(-t_peak / tau_syn)) / b
                                              - t_peak * math.exp(-t_peak / tau_syn))
    return 1.0 / v_max


def hpc_benchmark(nest, scale=1.0, indegree_scale=1.0, precision="fp64", seed=4242, record=True, plastic=True):
    """Build the HPC benchmark network; returns (E, I, recorder).
    indegree_scale < 1 thins every in-degree (for CPU-sized checks)."""
    nest.ResetKernel()
    nest.set(resolution=0.1, rng_seed=seed, precision=precision)
    NE, NI = int(9000 * scale), int(2250 * scale)
    tau_m, C_m, V_th = 10.0, 250.0, 20.0
    params = {"E_L": 0.0, "C_m": C_m, "tau_m": tau_m, "t_ref": 0.5, "V_th": V_th, "V_reset": 0.0,
              "tau_syn_ex": HPC_TAU_SYN, "tau_syn_in": HPC_TAU_SYN, "tau_minus": 30.0, "V_m": 5.7}
    E = nest.Create("iaf_psc_alpha", NE, params=params)
    I = nest.Create("iaf_psc_alpha", NI, params=params)
    rng = np.random.default_rng(seed)
    E.set(V_m=rng.normal(5.7, 7.2, NE))
    I.set(V_m=rng.normal(5.7, 7.2, NI))
    CE, CI = int(9000 * indegree_scale), int(2250 * indegree_scale)
    JE = alpha_pa_per_mv(tau_m, HPC_TAU_SYN, C_m) * 0.14          # 0.14 mV peak EPSP
    nu_th = V_th / (9000 * tau_m / C_m * JE * math.e * HPC_TAU_SYN)
    pg = nest.Create("poisson_generator", params={"rate": 1.685 * nu_th * 9000 * 1000.0})
    nest.SetDefaults("static_synapse_hpc", {"delay": 1.5})
    nest.CopyModel("static_synapse_hpc", "syn_ex", {"weight": JE})
    nest.CopyModel("static_synapse_hpc", "syn_in", {"weight": -5.0 * JE})
    ee = "stdp_pl_synapse_hom_hpc" if plastic else "syn_ex"
    nest.SetDefaults("stdp_pl_synapse_hom_hpc", {"delay": 1.5, "alpha": 0.0513, "lambda": 0.1, "mu": 0.4,
                                                 "tau_plus": 15.0, "weight": JE})
    nest.Connect(pg, E, {"rule": "all_to_all"}, {"synapse_model": "syn_ex"})
    nest.Connect(pg, I, {"rule": "all_to_all"}, {"synapse_model": "syn_ex"})
    kin = {"allow_autapses": False, "allow_multapses": True}
    nest.Connect(E, E, dict(rule="fixed_indegree", indegree=CE, **kin), {"synapse_model": ee})
    nest.Connect(I, E, dict(rule="fixed_indegree", indegree=CI, **kin), {"synapse_model": "syn_in"})
    nest.Connect(E, I, dict(rule="fixed_indegree", indegree=CE, **kin), {"synapse_model": "syn_ex"})
    nest.Connect(I, I, dict(rule="fixed_indegree", indegree=CI, **kin), {"synapse_model": "syn_in"})
    sr = None
    if record:
        sr = nest.Create("spike_recorder")
        nest.Connect(E + I, sr, syn_spec={"delay": 1.5})
    return E, I, sr


# ---------------------------------------------------------------------------
# c2: layered 8-population iaf_psc_exp network (microcircuit-shaped, synthetic
# connection probabilities), 77,169 neurons, pairwise_bernoulli.
# ---------------------------------------------------------------------------
LAYERED_SIZES = (20683, 5834, 21915, 5479, 4850, 1065, 14395, 2948)
LAYERED_EXC = (1, 0, 1, 0, 1, 0, 1, 0)


def layered_spec(seed=2024, scale=1.0):
    """Populations [E, I] x 4 layers; p[i][j] (source population i -> target
    population j) ~ U[0.01, 0.15]; weights N(87.8, 8.78) pA, inhibitory
    sources x -4; delays N(1.5, 0.75) ms (exc) / N(0.75, 0.375) ms (inh)
    clipped to >= dt; per-population Poisson drive 8 Hz x K_ext with
    K_ext ~ U[1500, 2500]; neurons: C_m 250 pF, tau_m 10 ms, t_ref 2 ms,
    E_L -65 mV, V_th -50 mV, V_reset -65 mV, tau_syn 0.5 ms, V_m(0) ~
    N(-58, 10) mV.  `scale` shrinks the populations (connection
    probabilities kept) for cases the oracle can run."""
    rng = np.random.default_rng(seed)
    p = rng.uniform(0.01, 0.15, (8, 8))
    k_ext = rng.integers(1500, 2501, 8)
    sizes = [max(1, int(round(s * scale))) for s in LAYERED_SIZES]
    return {"sizes": sizes, "exc": list(LAYERED_EXC), "p": p, "k_ext": k_ext, "J": 87.8, "J_sd": 8.78, "g": -4.0,
            "d_exc": (1.5, 0.75), "d_inh": (0.75, 0.375), "nu_ext_hz": 8.0, "tau_syn": 0.5, "E_L": -65.0,
            "V_th": -50.0, "V_reset": -65.0, "C_m": 250.0, "tau_m": 10.0, "t_ref": 2.0, "d_ext_ms": 1.5,
            "d_max_ms": 8.0, "seed": seed}


def layered_expected_edges(spec):
    n = np.asarray(spec["sizes"], dtype=np.float64)
    return float(np.sum(np.outer(n, n) * spec["p"]))


def layered_ring_bound(spec):
    """A bound on the sum of |weight| over one neuron's in-edges: per target
    population, mean + 8 standard deviations of that sum (binomial
    in-degrees, normal weights), 5 % margin.  The engine checks the drawn
    graph against it."""
    n = np.asarray(spec["sizes"], dtype=np.float64)
    exc = np.asarray(spec["exc"], dtype=bool)
    mu_w = np.where(exc, spec["J"], abs(spec["g"]) * spec["J"])
    sd_w = np.where(exc, spec["J_sd"], abs(spec["g"]) * spec["J_sd"])
    p = spec["p"]
    mean = (n[:, None] * p * mu_w[:, None]).sum(axis=0)
    var = (n[:, None] * p * (1 - p) * (mu_w ** 2)[:, None] + n[:, None] * p * (sd_w ** 2)[:, None]).sum(axis=0)
    return float(np.max(mean + 8 * np.sqrt(var)) * 1.05)


def layered_engine(spec, precision="fp64", device=0, graph_slices=64, ring32=False, tiled=False):
    """A serving engine sized for one layered network (the graph is drawn on
    the device by the pairwise_bernoulli builder).  ring32: the FP32 form
    with 32-bit ring cells, scaled by layered_ring_bound; tiled: target-tiled
    delivery (segment tables sized here)."""
    from . import _abi

    n = sum(spec["sizes"])
    h = 0.1
    max_steps = int(math.floor(spec["d_max_ms"] / h + 0.5))
    e_need = layered_expected_edges(spec)
    cap = int(e_need + 6.0 * math.sqrt(e_need) + 4 * n + 1024)
    prec = _abi.NG_FP32 if precision == "fp32" else _abi.NG_FP64
    J = spec["J"]
    eng = _abi.Engine([(_abi.NG_IAF_PSC_EXP, n)], h, 1, max(max_steps, int(round(spec["d_ext_ms"] / h))),
                      precision=prec, device=device, serving=True, max_networks=1, edge_capacity=cap,
                      max_abs_weight=abs(spec["g"]) * (J + 12 * spec["J_sd"]) * 2, ring32=ring32,
                      ring_bound=layered_ring_bound(spec) if ring32 else 0.0,
                      tile_capacity=_abi.tile_table_entries(n, max(max_steps, 15), ring32) if tiled else 0)
    eng.set_graph_slices(graph_slices)
    return eng


def layered_add(eng, spec, steps, record=True):
    """Admit the layered network into `eng`; returns its network id."""
    from . import _abi

    sizes, exc = spec["sizes"], spec["exc"]
    n = sum(sizes)
    J, sd, g = spec["J"], spec["J_sd"], spec["g"]
    pb = _abi.NGPairwiseBernoulli.make(sizes, exc, spec["p"], w_mean=(g * J, J), w_sd=(abs(g) * sd, sd),
                                       d_mean_ms=(spec["d_inh"][0], spec["d_exc"][0]),
                                       d_sd_ms=(spec["d_inh"][1], spec["d_exc"][1]), d_max_ms=spec["d_max_ms"],
                                       allow_autapses=0, seed=spec["seed"] * 7919 + 1)
    rng = np.random.default_rng(spec["seed"])
    E_L = spec["E_L"]
    V0 = rng.normal(-58.0, 10.0, n) - E_L
    rate = np.repeat(np.asarray(spec["k_ext"], dtype=np.float64) * spec["nu_ext_hz"], sizes)
    d_ext = int(round(spec["d_ext_ms"] / 0.1))
    var = {"tau_syn_ex": spec["tau_syn"], "tau_syn_in": spec["tau_syn"], "tau_m": spec["tau_m"], "C_m": spec["C_m"],
           "t_ref": spec["t_ref"], "V_th_rel": spec["V_th"] - E_L, "V_reset_rel": spec["V_reset"] - E_L, "V_m_rel": V0}
    nid = eng.net_add(n, steps, spec["seed"], var, build=pb, poisson=(rate, J, d_ext), record=record)
    if nid is None:
        raise RuntimeError("the layered network does not fit the engine")
    return nid


# ---------------------------------------------------------------------------
# c3: adaptive-integrator network, 50,000 aeif_cond_alpha neurons
# ---------------------------------------------------------------------------
def aeif_spec(seed=77, n_exc=40000, n_inh=10000):
    """aeif_cond_alpha network: fixed_indegree K = 1,000 (800 exc, 200 inh),
    conductance weights g_E = 1 nS, g_I = -5 nS (inhibitory conductance
    5 nS), a = 4 nS, b = 80.5 pA, Delta_T = 2 mV, tau_w = 144 ms, delay
    1.5 ms; Poisson drive 10 kHz x 0.5 nS per neuron; V_m(0) ~ U[E_L, V_th)
    from seed.  tau_syn_ex = 1 ms (with the model's default 0.2 ms this
    drive keeps every neuron below threshold: mean conductance 2.7 nS, 6 mV
    of depolarisation); the other parameters are the model's defaults."""
    return {"n_exc": n_exc, "n_inh": n_inh, "k_exc": 800, "k_inh": 200, "g_E": 1.0, "g_I": -5.0, "a": 4.0,
            "b": 80.5, "Delta_T": 2.0, "tau_w": 144.0, "tau_syn_ex": 1.0, "delay_ms": 1.5, "nu_ext_hz": 10000.0,
            "w_ext": 0.5, "E_L": -70.6, "V_th": -50.4, "seed": seed}


def aeif_engine(spec, precision="fp64", device=0, graph_slices=64):
    """A serving engine sized for one aeif network (fixed_indegree graph
    drawn on the device)."""
    from . import _abi

    n = spec["n_exc"] + spec["n_inh"]
    d = int(round(spec["delay_ms"] / 0.1))
    K = spec["k_exc"] + spec["k_inh"]
    prec = _abi.NG_FP32 if precision == "fp32" else _abi.NG_FP64
    eng = _abi.Engine([(_abi.NG_AEIF_COND_ALPHA, n)], 0.1, d, d, precision=prec, device=device, serving=True,
                      max_networks=1, edge_capacity=n * (K + 3) + 1024,
                      max_abs_weight=4 * max(abs(spec["g_E"]), abs(spec["g_I"]), spec["w_ext"]))
    eng.set_graph_slices(graph_slices)
    return eng


def aeif_add(eng, spec, steps, record=True):
    """Admit the aeif network into `eng`; returns its network id."""
    n = spec["n_exc"] + spec["n_inh"]
    rng = np.random.default_rng(spec["seed"])
    V0 = rng.uniform(spec["E_L"], spec["V_th"], n)
    d = int(round(spec["delay_ms"] / 0.1))
    build = dict(n_exc=spec["n_exc"], k_exc=spec["k_exc"], k_inh=spec["k_inh"], w_exc=spec["g_E"], w_inh=spec["g_I"],
                 delay_steps=d, allow_autapses=0, seed=spec["seed"] * 104729 + 3)
    var = {"a": spec["a"], "b": spec["b"], "Delta_T": spec["Delta_T"], "tau_w": spec["tau_w"],
           "tau_syn_ex": spec["tau_syn_ex"], "V_m": V0}
    nid = eng.net_add(n, steps, spec["seed"], var, build=build, poisson=(spec["nu_ext_hz"], spec["w_ext"], d),
                      record=record)
    if nid is None:
        raise RuntimeError("the aeif network does not fit the engine")
    return nid
