"""Generate the golden fixtures under tests/golden/ from the reference itself.

This script is run once, in a container where the reference NEST
(nest-simulator 3.10.0-post0.dev0) is importable as PyNEST, e.g.

    NEST_REFERENCE_ROOT=<reference source tree> \
    PYTHONPATH=<install prefix>/lib/python3.12/site-packages python tests/golden/make_golden.py [fixture ...]

(the PyNEST install was built from the reference's sources with CMake, GSL off,
OpenMP on).  It writes small ``.npz`` files that the test
suite reads on any machine; the reference is never needed at test time.

Fixtures written
----------------
c0_delta_balanced.npz
    The deterministic balanced iaf_psc_delta network (1,000 neurons,
    fixed_indegree 80/20, dyadic weights +0.125/-0.625 mV, delay 1.5 ms,
    I_e ~ U[300,500] pA, V_m ~ U[0,20) mV, 1,000 ms).  Holds the graph as
    exported by ``nest.GetConnections``, the per-neuron drive and initial
    state, the full spike raster and the final V_m of every neuron.
exp_dyadic_net.npz / exp_real_net.npz
    Small iaf_psc_exp networks (tau_syn 0.5 ms, DC drive) with dyadic
    (order-independent) and real-valued weights: raster, multimeter V_m
    traces of 8 neurons, final state.
single_neuron_cases.npz
    test_compare_delta-style (spike_generator -> iaf_psc_delta, h=0.01) and
    test_iaf_singularity-style (tau_syn = tau_m +- eps) voltmeter traces,
    and a DC-driven iaf_psc_exp trace (test_iaf_psc_exp-style).
c1_exp_poisson_stats.npz
    Config-1-shaped Poisson-driven iaf_psc_exp network (12,500 neurons,
    K_E=1,000, K_I=250, J=87.8 pA, g=5, 8 kHz drive): per-neuron spike
    counts and CV-ISI and binned population counts, for the statistical
    (KS) oracle.
iaf_psc_alpha_kat.npz
    The expected V_m traces and spike times that the reference test suite
    holds for iaf_psc_alpha with an internal DC current
    (testsuite/pytests/neurons/test_iaf_psc_alpha.py: test_iaf_psc_alpha_i0,
    and test_iaf_psc_alpha_i0_refractory at resolutions 0.1, 0.2, 0.5, 1.0
    ms), read from the test file's array literals with the ast module.
aeif_lsodar.npz
    The LSODAR reference solution the reference test suite pins
    aeif_cond_alpha to (testsuite/pytests/neurons/test_aeif_data_lsodar.dat,
    read with numpy.loadtxt and stored verbatim as float64).
philox_kat.npz
    The Philox4x32 known-answer vectors of the vendored Random123
    (thirdparty/Random123/tests/kat_vectors, philox4x32 lines).
"""

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference's source tree (its test-suite data files are read from it)
REF = os.environ.get("NEST_REFERENCE_ROOT", "")


def _nest():
    import nest  # noqa: the reference PyNEST

    try:
        nest.verbosity = nest.VerbosityLevel.ERROR
    except Exception:
        nest.set_verbosity("M_ERROR")
    return nest


def make_c0(nest):
    """Config 0: plain deterministic balanced network, FP64, bit-exact oracle."""
    nest.ResetKernel()
    nest.set(resolution=0.1, local_num_threads=4, rng_seed=12345)
    p = dict(C_m=250.0, tau_m=20.0, t_ref=2.0, E_L=0.0, V_th=20.0, V_reset=10.0)
    NE, NI = 800, 200
    N = NE + NI
    pop = nest.Create("iaf_psc_delta", N, params=p)
    rng = np.random.default_rng(20260101)
    I_e = rng.uniform(300.0, 500.0, N)
    V0 = rng.uniform(0.0, 20.0, N)
    pop.set(I_e=list(I_e), V_m=list(V0))
    E, I = pop[:NE], pop[NE:]
    nest.Connect(E, pop, {"rule": "fixed_indegree", "indegree": 80, "allow_autapses": False},
                 {"weight": 0.125, "delay": 1.5})
    nest.Connect(I, pop, {"rule": "fixed_indegree", "indegree": 20, "allow_autapses": False},
                 {"weight": -0.625, "delay": 1.5})
    sr = nest.Create("spike_recorder")
    nest.Connect(pop, sr, syn_spec={"delay": 1.5})
    conns = nest.GetConnections(source=pop, target=pop).get(["source", "target", "weight", "delay"])
    t0 = time.perf_counter()
    nest.Simulate(1000.0)
    wall = time.perf_counter() - t0
    ev = sr.events
    snd = np.asarray(ev["senders"], dtype=np.int64)
    tms = np.asarray(ev["times"], dtype=np.float64)
    steps = np.rint(tms / 0.1).astype(np.int64)
    order = np.lexsort((snd, steps))
    src = np.asarray(conns["source"], dtype=np.int64)
    tgt = np.asarray(conns["target"], dtype=np.int64)
    w = np.asarray(conns["weight"], dtype=np.float64)
    d = np.asarray(conns["delay"], dtype=np.float64)
    assert set(np.unique(w)) == {0.125, -0.625}
    assert np.all(d == 1.5)
    Vend = np.asarray(pop.get("V_m"), dtype=np.float64)
    np.savez_compressed(
        os.path.join(HERE, "c0_delta_balanced.npz"),
        params=np.array([p["C_m"], p["tau_m"], p["t_ref"], p["E_L"], p["V_th"], p["V_reset"]]),
        first_id=np.int64(pop[0].global_id),
        I_e=I_e, V0=V0,
        src=(src - 1).astype(np.uint16), tgt=(tgt - 1).astype(np.uint16), exc=(w > 0),
        spike_senders=(snd[order] - 1).astype(np.uint16), spike_steps=steps[order].astype(np.int32),
        V_end=Vend,
        min_delay=np.float64(nest.min_delay), max_delay=np.float64(nest.max_delay),
        sim_ms=np.float64(1000.0), h=np.float64(0.1), ref_wall_s=np.float64(wall),
    )
    print("c0: spikes", len(snd), "rate", len(snd) / N, "Hz; wall", wall, "s; min/max delay",
          nest.min_delay, nest.max_delay)


def make_exp_net(nest, dyadic):
    """Small DC-driven iaf_psc_exp network with multimeter traces."""
    nest.ResetKernel()
    nest.set(resolution=0.1, local_num_threads=2)
    N, NE = 200, 160
    params = dict(tau_syn_ex=0.5, tau_syn_in=0.5, t_ref=2.0)
    pop = nest.Create("iaf_psc_exp", N, params=params)
    rng = np.random.default_rng(7 if dyadic else 11)
    I_e = rng.uniform(350.0, 450.0, N)
    V0 = rng.uniform(-70.0, -56.0, N)
    pop.set(I_e=list(I_e), V_m=list(V0))
    if dyadic:
        we, wi = 64.0, -256.0
    else:
        we, wi = 87.8, -439.0
    nest.Connect(pop[:NE], pop, {"rule": "fixed_indegree", "indegree": 16, "allow_autapses": False},
                 {"weight": we, "delay": 1.5})
    nest.Connect(pop[NE:], pop, {"rule": "fixed_indegree", "indegree": 4, "allow_autapses": False},
                 {"weight": wi, "delay": 1.0})
    sr = nest.Create("spike_recorder")
    nest.Connect(pop, sr)
    rec = pop[::25]
    mm = nest.Create("multimeter", params={"interval": 0.1, "record_from": ["V_m", "I_syn_ex", "I_syn_in"]})
    nest.Connect(mm, rec)
    conns = nest.GetConnections(source=pop, target=pop).get(["source", "target", "weight", "delay"])
    nest.Simulate(200.0)
    ev = sr.events
    snd = np.asarray(ev["senders"], dtype=np.int64)
    steps = np.rint(np.asarray(ev["times"]) / 0.1).astype(np.int64)
    order = np.lexsort((snd, steps))
    mev = mm.events
    msnd = np.asarray(mev["senders"], dtype=np.int64)
    mt = np.asarray(mev["times"], dtype=np.float64)
    mv = np.asarray(mev["V_m"], dtype=np.float64)
    mex = np.asarray(mev["I_syn_ex"], dtype=np.float64)
    min_ = np.asarray(mev["I_syn_in"], dtype=np.float64)
    morder = np.lexsort((msnd, mt))
    V_end = np.asarray(pop.get("V_m"), dtype=np.float64)
    name = "exp_dyadic_net.npz" if dyadic else "exp_real_net.npz"
    np.savez_compressed(
        os.path.join(HERE, name),
        I_e=I_e, V0=V0,
        src=np.asarray(conns["source"], dtype=np.int32) - 1,
        tgt=np.asarray(conns["target"], dtype=np.int32) - 1,
        w=np.asarray(conns["weight"], dtype=np.float64),
        d=np.asarray(conns["delay"], dtype=np.float64),
        spike_senders=(snd[order] - 1).astype(np.int32), spike_steps=steps[order].astype(np.int32),
        rec_idx=np.asarray(rec.tolist(), dtype=np.int32) - 1,
        mm_senders=(msnd[morder] - 1).astype(np.int32), mm_times=mt[morder], mm_V=mv[morder],
        mm_Iex=mex[morder], mm_Iin=min_[morder], V_end=V_end,
        min_delay=np.float64(nest.min_delay), max_delay=np.float64(nest.max_delay),
        n_exc=np.int64(NE), sim_ms=np.float64(200.0),
    )
    print(name, "spikes", len(snd), "min/max", nest.min_delay, nest.max_delay, "mm samples", len(mt))


def make_single_neuron_cases(nest):
    out = {}
    # test_compare_delta-style: spike_generator -> iaf_psc_delta at h = 0.01
    nest.ResetKernel()
    nest.resolution = 0.01
    npar = {"E_L": -49.0, "V_m": -60.0, "V_th": -50.0, "V_reset": -60.0, "C_m": 200.0, "tau_m": 20.0,
            "t_ref": 5.0}
    n = nest.Create("iaf_psc_delta", params=npar)
    sg = nest.Create("spike_generator", params={"spike_times": [1.0, 2.0, 3.0, 4.0, 5.0, 10.5, 12.0]})
    sr = nest.Create("spike_recorder")
    vm = nest.Create("voltmeter", params={"interval": 0.01})
    nest.Connect(sg, n, syn_spec={"delay": 0.1, "weight": 2.5})
    nest.Connect(n, sr)
    nest.Connect(vm, n)
    nest.Simulate(200.0)
    out["cmpdelta_spike_times"] = np.asarray(sr.events["times"], dtype=np.float64)
    out["cmpdelta_vm_times"] = np.asarray(vm.events["times"], dtype=np.float64)[:3000]
    out["cmpdelta_vm_V"] = np.asarray(vm.events["V_m"], dtype=np.float64)[:3000]

    # test_iaf_singularity-style grid for iaf_psc_exp
    for h in (0.001, 0.1):
        for tau_m in (1.0, 10.0, 100.0):
            delta_tau = np.hstack((-np.logspace(-10, -1, 5), [0], np.logspace(-10, -1, 5)))
            tau_syn = tau_m + delta_tau
            nest.ResetKernel()
            nest.resolution = h
            neurons = nest.Create("iaf_psc_exp", n=len(tau_syn),
                                  params={"tau_m": tau_m, "tau_syn_ex": tau_syn, "tau_syn_in": tau_syn,
                                          "V_th": np.inf})
            sgen = nest.Create("spike_generator", params={"spike_times": [1.0]})
            vmt = nest.Create("voltmeter", params={"interval": h})
            nest.Connect(sgen, neurons, syn_spec={"weight": 1000.0, "delay": 1.0})
            nest.Connect(sgen, neurons, syn_spec={"weight": -1000.0, "delay": 2.0})
            nest.Connect(vmt, neurons)
            nest.Simulate(10 * tau_m)
            ev = vmt.events
            s = np.asarray(ev["senders"], dtype=np.int64)
            t = np.asarray(ev["times"], dtype=np.float64)
            v = np.asarray(ev["V_m"], dtype=np.float64)
            o = np.lexsort((s, t))
            s, t, v = s[o], t[o], v[o]
            nsend = len(tau_syn)
            V = v.reshape(-1, nsend)  # rows: times, columns: senders in id order
            times = t.reshape(-1, nsend)[:, 0]
            # smoothness figures over the full trace, samples on a coarse grid
            dV = np.abs(np.diff(V, axis=0)).max(axis=0)
            stride = max(1, len(times) // 400)
            key = f"sing_h{h}_tau{tau_m}"
            out[key + "_tau_syn"] = tau_syn
            out[key + "_times"] = times[::stride]
            out[key + "_V"] = V[::stride]
            out[key + "_max_dV"] = dV
            out[key + "_V_range"] = np.float64(V.max() - V.min())
            out[key + "_stride"] = np.int64(stride)

    # test_iaf_psc_exp-style: DC drive through I_e, V_m trace incl. refractoriness
    nest.ResetKernel()
    nest.resolution = 0.1
    n = nest.Create("iaf_psc_exp", params={"I_e": 1000.0, "tau_syn_ex": 0.5, "tau_syn_in": 0.5})
    vm = nest.Create("voltmeter", params={"interval": 0.1})
    sr = nest.Create("spike_recorder")
    nest.Connect(vm, n)
    nest.Connect(n, sr)
    nest.Simulate(100.0)
    out["dcexp_vm_times"] = np.asarray(vm.events["times"], dtype=np.float64)
    out["dcexp_vm_V"] = np.asarray(vm.events["V_m"], dtype=np.float64)
    out["dcexp_spike_times"] = np.asarray(sr.events["times"], dtype=np.float64)
    np.savez_compressed(os.path.join(HERE, "single_neuron_cases.npz"), **out)
    print("single-neuron cases:", sorted(k for k in out if k.endswith("spike_times")),
          out["cmpdelta_spike_times"][:3])


def make_c1_stats(nest):
    """Config-1-shaped Poisson-driven iaf_psc_exp network, statistics only."""
    nest.ResetKernel()
    nest.set(resolution=0.1, local_num_threads=8, rng_seed=4242)
    NE, NI = 10000, 2500
    N = NE + NI
    pop = nest.Create("iaf_psc_exp", N, params={"tau_syn_ex": 0.5, "tau_syn_in": 0.5})
    rng = np.random.default_rng(99)
    pop.set(V_m=list(rng.normal(-58.0, 10.0, N)))
    J, g = 87.8, 5.0
    nest.Connect(pop[:NE], pop, {"rule": "fixed_indegree", "indegree": 1000, "allow_autapses": False},
                 {"weight": J, "delay": 1.5})
    nest.Connect(pop[NE:], pop, {"rule": "fixed_indegree", "indegree": 250, "allow_autapses": False},
                 {"weight": -g * J, "delay": 1.5})
    pg = nest.Create("poisson_generator", params={"rate": 8000.0})
    nest.Connect(pg, pop, syn_spec={"weight": J, "delay": 1.5})
    sr = nest.Create("spike_recorder")
    nest.Connect(pop, sr, syn_spec={"delay": 1.5})
    t0 = time.perf_counter()
    nest.Simulate(1000.0)
    wall = time.perf_counter() - t0
    ev = sr.events
    snd = np.asarray(ev["senders"], dtype=np.int64) - 1
    t = np.asarray(ev["times"], dtype=np.float64)
    counts = np.bincount(snd, minlength=N)
    o = np.lexsort((t, snd))
    snd, t = snd[o], t[o]
    cv = np.full(N, np.nan)
    starts = np.searchsorted(snd, np.arange(N))
    ends = np.searchsorted(snd, np.arange(N), side="right")
    for i in range(N):
        ts = t[starts[i]:ends[i]]
        if len(ts) >= 3:
            isi = np.diff(ts)
            cv[i] = isi.std() / isi.mean()
    pop_counts = np.bincount(np.rint(t / 1.0).astype(np.int64), minlength=1001)
    ks = nest.GetKernelStatus()
    # spread of the population statistics across network realizations
    seed_rates, seed_cvs = [], []
    for seed in (1, 2, 3, 5, 6):
        r, c = _c1_once(nest, seed)
        seed_rates.append(r)
        seed_cvs.append(c)
    np.savez_compressed(os.path.join(HERE, "c1_exp_poisson_stats.npz"),
                        counts=counts.astype(np.int32), cv=cv, pop_counts_1ms=pop_counts.astype(np.int32),
                        ref_wall_s=np.float64(wall), ref_threads=np.int64(8),
                        time_simulate=np.float64(ks.get("time_simulate", np.nan)),
                        seed_rates=np.array(seed_rates), seed_mean_cv=np.array(seed_cvs))
    print("c1: rate", counts.mean(), "Hz; mean CV", np.nanmean(cv), "; wall", wall)


def _c1_once(nest, seed):
    """Mean rate and mean CV-ISI of one realization of the config-1 network."""
    nest.ResetKernel()
    nest.set(resolution=0.1, local_num_threads=8, rng_seed=seed)
    NE, NI = 10000, 2500
    N = NE + NI
    pop = nest.Create("iaf_psc_exp", N, params={"tau_syn_ex": 0.5, "tau_syn_in": 0.5})
    pop.set(V_m=list(np.random.default_rng(seed).normal(-58.0, 10.0, N)))
    nest.Connect(pop[:NE], pop, {"rule": "fixed_indegree", "indegree": 1000, "allow_autapses": False},
                 {"weight": 87.8, "delay": 1.5})
    nest.Connect(pop[NE:], pop, {"rule": "fixed_indegree", "indegree": 250, "allow_autapses": False},
                 {"weight": -5.0 * 87.8, "delay": 1.5})
    pg = nest.Create("poisson_generator", params={"rate": 8000.0})
    nest.Connect(pg, pop, syn_spec={"weight": 87.8, "delay": 1.5})
    sr = nest.Create("spike_recorder")
    nest.Connect(pop, sr, syn_spec={"delay": 1.5})
    nest.Simulate(1000.0)
    snd = np.asarray(sr.events["senders"], dtype=np.int64) - 1
    t = np.asarray(sr.events["times"])
    o = np.lexsort((t, snd))
    snd, t = snd[o], t[o]
    cvs = []
    starts = np.searchsorted(snd, np.arange(N))
    ends = np.searchsorted(snd, np.arange(N), side="right")
    for i in range(N):
        ts = t[starts[i]:ends[i]]
        if len(ts) >= 3:
            isi = np.diff(ts)
            cvs.append(isi.std() / isi.mean())
    return len(t) / N, float(np.mean(cvs))


def make_aeif_lsodar():
    path = os.path.join(REF, "testsuite/pytests/neurons/test_aeif_data_lsodar.dat")
    data = np.loadtxt(path)
    np.savez_compressed(os.path.join(HERE, "aeif_lsodar.npz"), t=data[:, 0], V_m=data[:, 1], w=data[:, 2])
    print("aeif lsodar rows", data.shape)


def _array_literals(path, func):
    """The np.array([...]) literals inside function `func` of a test file,
    in source order (evaluated as plain Python lists)."""
    import ast

    tree = ast.parse(open(path).read())
    out = []
    for node in ast.walk(tree):
        if isinstance(node, ast.FunctionDef) and node.name == func:
            for sub in ast.walk(node):
                if (isinstance(sub, ast.Call) and isinstance(sub.func, ast.Attribute) and sub.func.attr == "array"
                        and sub.args and isinstance(sub.args[0], ast.List)):
                    out.append((sub.lineno, np.array(ast.literal_eval(sub.args[0]), dtype=np.float64)))
    return [a for _, a in sorted(out, key=lambda x: x[0])]


def make_alpha_kat():
    path = os.path.join(REF, "testsuite/pytests/neurons/test_iaf_psc_alpha.py")
    i0 = _array_literals(path, "test_iaf_psc_alpha_i0")
    refr = _array_literals(path, "test_iaf_psc_alpha_i0_refractory")
    np.savez_compressed(os.path.join(HERE, "iaf_psc_alpha_kat.npz"), i0_vm=i0[0], i0_spikes=i0[1],
                        i0_refractory_vm=refr[0])
    print("iaf_psc_alpha KAT rows", i0[0].shape, i0[1].shape, refr[0].shape)


def make_philox_kat():
    path = os.path.join(REF, "thirdparty/Random123/tests/kat_vectors")
    rounds, ctr, key, out = [], [], [], []
    with open(path) as f:
        for line in f:
            parts = line.split()
            if len(parts) == 12 and parts[0] == "philox4x32":
                vals = [int(x, 16) for x in parts[2:]]
                rounds.append(int(parts[1]))
                ctr.append(vals[0:4])
                key.append(vals[4:6])
                out.append(vals[6:10])
    np.savez_compressed(os.path.join(HERE, "philox_kat.npz"), rounds=np.array(rounds, dtype=np.int32),
                        ctr=np.array(ctr, dtype=np.uint32), key=np.array(key, dtype=np.uint32),
                        out=np.array(out, dtype=np.uint32))
    print("philox KAT vectors", len(rounds))


if __name__ == "__main__":
    which = set(sys.argv[1:]) or {"c0", "exp", "single", "c1", "aeif", "philox", "alpha"}
    if "aeif" in which:
        make_aeif_lsodar()
    if "alpha" in which:
        make_alpha_kat()
    if "philox" in which:
        make_philox_kat()
    if which & {"c0", "exp", "single", "c1"}:
        nest = _nest()
        if "c0" in which:
            make_c0(nest)
        if "exp" in which:
            make_exp_net(nest, dyadic=True)
            make_exp_net(nest, dyadic=False)
        if "single" in which:
            make_single_neuron_cases(nest)
        if "c1" in which:
            make_c1_stats(nest)
