"""ctypes wrapper of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: the checker the CUDA engine is compared with.
Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg
import this module.  See nest_oracle.h for what it restates.
"""

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

IAF_PSC_DELTA, IAF_PSC_EXP, AEIF_COND_ALPHA, IAF_PSC_ALPHA = 0, 1, 2, 3
MODEL_IDS = {"iaf_psc_delta": 0, "iaf_psc_exp": 1, "aeif_cond_alpha": 2, "iaf_psc_alpha": 3}

_lib = None


def build():
    """Compile liboracle.so with the committed Makefile."""
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
    subprocess.run(["make", "-s", "-C", HERE, f"CC={cc}"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(os.path.join(HERE, "nest_oracle.c")):
            build()
        L = ctypes.CDLL(LIB)
        P = ctypes.c_void_p
        i64, i32, dbl = ctypes.c_int64, ctypes.c_int32, ctypes.c_double
        L.orc_create.restype = P
        L.orc_create.argtypes = [ctypes.c_int, i64, dbl, i32, i32]
        L.orc_destroy.argtypes = [P]
        L.orc_error.restype = ctypes.c_char_p
        L.orc_set.argtypes = [P, ctypes.c_char_p, P]
        L.orc_get.argtypes = [P, ctypes.c_char_p, P]
        L.orc_set_csr.argtypes = [P, i64, P, P, P, P, ctypes.c_int]
        L.orc_set_sched.argtypes = [P, i64, P, P]
        L.orc_set_poisson.argtypes = [P, P, P, P, i64, i64, ctypes.c_uint64]
        L.orc_set_record.argtypes = [P, P]
        L.orc_set_trace.argtypes = [P, i64, P, ctypes.c_char_p]
        L.orc_run.argtypes = [P, i64, ctypes.c_int]
        for f in ("orc_n_spikes", "orc_n_trace", "orc_clock", "orc_syn_events"):
            getattr(L, f).restype = i64
            getattr(L, f).argtypes = [P]
        L.orc_get_spikes.restype = i64
        L.orc_get_spikes.argtypes = [P, P, P, i64]
        L.orc_get_trace.restype = i64
        L.orc_get_trace.argtypes = [P, P, i64]
        L.orc_iaf_propagator_exp.restype = dbl
        L.orc_iaf_propagator_exp.argtypes = [dbl, dbl, dbl, dbl]
        L.orc_set_plastic.argtypes = [P, i64, P, P, P, P, dbl, dbl, dbl, dbl]
        L.orc_get_plastic.argtypes = [P, P]
        L.orc_iaf_propagator_alpha.restype = None
        L.orc_iaf_propagator_alpha.argtypes = [dbl, dbl, dbl, dbl, P]
        L.orc_philox4x32.argtypes = [P, P, ctypes.c_int, P]
        L.orc_poisson_draw.restype = i64
        L.orc_poisson_draw.argtypes = [dbl, dbl]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class OracleNet:
    """One network of a single neuron model, simulated on the CPU."""

    def __init__(self, model, n, h, min_delay, max_delay):
        self.L = lib()
        self.model = MODEL_IDS.get(model, model)
        self.n = int(n)
        self.h = float(h)
        self.ptr = self.L.orc_create(self.model, self.n, self.h, int(min_delay), int(max_delay))
        if not self.ptr:
            raise RuntimeError(self.L.orc_error().decode())
        self._keep = []

    def __del__(self):
        if getattr(self, "ptr", None):
            self.L.orc_destroy(self.ptr)
            self.ptr = None

    def _chk(self, rc):
        if rc != 0:
            raise RuntimeError(self.L.orc_error().decode())

    def set(self, name, values):
        v = np.ascontiguousarray(np.broadcast_to(np.asarray(values, dtype=np.float64), (self.n,)))
        self._chk(self.L.orc_set(self.ptr, name.encode(), _p(v)))

    def get(self, name):
        out = np.empty(self.n, dtype=np.float64)
        self._chk(self.L.orc_get(self.ptr, name.encode(), _p(out)))
        return out

    def set_csr(self, row_ptr, tgt, w, d, nthreads=0):
        row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int64)
        tgt = np.ascontiguousarray(tgt, dtype=np.int32)
        w = np.ascontiguousarray(w, dtype=np.float64)
        d = np.ascontiguousarray(d, dtype=np.int32)
        self._chk(self.L.orc_set_csr(self.ptr, len(row_ptr) - 1, _p(row_ptr), _p(tgt), _p(w), _p(d), int(nthreads)))

    def set_edges(self, src, tgt, w, d, n_src=None, nthreads=0):
        """Edges in any order; grouped by source keeping their relative order."""
        src = np.asarray(src, dtype=np.int64)
        n_src = self.n if n_src is None else int(n_src)
        order = np.argsort(src, kind="stable")
        counts = np.bincount(src, minlength=n_src)
        row_ptr = np.zeros(n_src + 1, dtype=np.int64)
        np.cumsum(counts, out=row_ptr[1:])
        self.set_csr(row_ptr, np.asarray(tgt)[order], np.asarray(w)[order], np.asarray(d)[order], nthreads)

    def set_plastic(self, src, tgt, w, d, lam=0.1, alpha=1.0, mu=0.4, tau_plus=20.0, n_src=None):
        """stdp_pl_synapse_hom connections (sources are neurons), any order;
        grouped by source keeping their order."""
        src = np.asarray(src, dtype=np.int64)
        n_src = self.n if n_src is None else int(n_src)
        order = np.argsort(src, kind="stable")
        row_ptr = np.zeros(n_src + 1, dtype=np.int64)
        np.cumsum(np.bincount(src, minlength=n_src), out=row_ptr[1:])
        self._pl_order = order
        tg = np.ascontiguousarray(np.asarray(tgt)[order], dtype=np.int32)
        ww = np.ascontiguousarray(np.asarray(w, dtype=np.float64)[order])
        dd = np.ascontiguousarray(np.asarray(d)[order], dtype=np.int32)
        self._chk(self.L.orc_set_plastic(self.ptr, n_src, _p(row_ptr), _p(tg), _p(ww), _p(dd), float(lam), float(alpha),
                                         float(mu), float(tau_plus)))

    def plastic_weights(self):
        """Weights of the plastic connections, in the order they were given."""
        k = len(self._pl_order)
        out = np.empty(k, dtype=np.float64)
        self._chk(self.L.orc_get_plastic(self.ptr, _p(out)))
        res = np.empty(k, dtype=np.float64)
        res[self._pl_order] = out
        return res

    def set_sched(self, steps, srcs):
        steps = np.ascontiguousarray(steps, dtype=np.int64)
        srcs = np.ascontiguousarray(srcs, dtype=np.int32)
        self._chk(self.L.orc_set_sched(self.ptr, len(steps), _p(steps), _p(srcs)))

    def set_poisson(self, rate_hz, w, d, seed, start_step=0, stop_step=2**62):
        n = self.n
        r = np.ascontiguousarray(np.broadcast_to(np.asarray(rate_hz, dtype=np.float64), (n,)))
        ww = np.ascontiguousarray(np.broadcast_to(np.asarray(w, dtype=np.float64), (n,)))
        dd = np.ascontiguousarray(np.broadcast_to(np.asarray(d, dtype=np.int32), (n,)))
        self._chk(self.L.orc_set_poisson(self.ptr, _p(r), _p(ww), _p(dd), int(start_step), int(stop_step),
                                         int(seed) & (2**64 - 1)))

    def set_record(self, flags):
        f = np.ascontiguousarray(flags, dtype=np.uint8)
        self._keep.append(f)
        self._chk(self.L.orc_set_record(self.ptr, _p(f)))

    def set_trace(self, idx, var):
        idx = np.ascontiguousarray(idx, dtype=np.int32)
        self._chk(self.L.orc_set_trace(self.ptr, len(idx), _p(idx), var.encode()))
        self._n_trace_idx = len(idx)

    def run(self, n_steps, nthreads=0):
        rc = self.L.orc_run(self.ptr, int(n_steps), int(nthreads))
        if rc != 0:
            raise RuntimeError(self.L.orc_error().decode())

    def spikes(self):
        k = self.L.orc_n_spikes(self.ptr)
        src = np.empty(k, dtype=np.int32)
        st = np.empty(k, dtype=np.int64)
        self.L.orc_get_spikes(self.ptr, _p(src), _p(st), k)
        return src, st

    def trace(self):
        k = self.L.orc_n_trace(self.ptr)
        out = np.empty(k, dtype=np.float64)
        self.L.orc_get_trace(self.ptr, _p(out), k)
        return out.reshape(-1, self._n_trace_idx)

    @property
    def clock(self):
        return self.L.orc_clock(self.ptr)

    @property
    def syn_events(self):
        return self.L.orc_syn_events(self.ptr)


def iaf_propagator_exp(tau_syn, tau_m, c_m, h):
    return lib().orc_iaf_propagator_exp(tau_syn, tau_m, c_m, h)


def philox4x32(ctr, key, rounds=10):
    c = np.ascontiguousarray(ctr, dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    o = np.empty(4, dtype=np.uint32)
    lib().orc_philox4x32(_p(c), _p(k), int(rounds), _p(o))
    return o


def poisson_draw(lam, u):
    return lib().orc_poisson_draw(float(lam), float(u))


def c0_network(fx, nthreads=0):
    """Build the config-0 network of the golden fixture on the oracle."""
    C_m, tau_m, t_ref, E_L, V_th, V_reset = fx["params"]
    n = len(fx["I_e"])
    md = int(round(float(fx["min_delay"]) / 0.1))
    Md = int(round(float(fx["max_delay"]) / 0.1))
    net = OracleNet("iaf_psc_delta", n, 0.1, md, Md)
    net.set("tau_m", tau_m)
    net.set("C_m", C_m)
    net.set("t_ref", t_ref)
    net.set("V_th_rel", V_th - E_L)
    net.set("V_reset_rel", V_reset - E_L)
    net.set("I_e", fx["I_e"])
    net.set("V_m_rel", fx["V0"] - E_L)
    w = np.where(fx["exc"], 0.125, -0.625)
    d = np.full(len(w), 15, dtype=np.int32)
    net.set_edges(fx["src"].astype(np.int64), fx["tgt"].astype(np.int32), w, d, nthreads=nthreads)
    return net


def net_from_kernel(K, nthreads=0):
    """Oracle copy of a network built with the engine's front-end (one model).

    Uses the front-end's compiled arrays (graph, drive, generators) and its
    model storage (internal representation), so the oracle and the engine run
    the same network."""
    c = K.compile()
    if len(c["blocks"]) != 1:
        raise ValueError("the oracle runs one neuron model per network")
    b = c["blocks"][0]
    st = K.models[b["model"]]
    net = OracleNet(b["model"], c["N"], K.h, c["min_delay"], c["max_delay"])
    for k, ev in st.engine_vars.items():
        net.set(ev, st.data[k][:b["n"]])
    net.set_edges(c["src"], c["tgt"], c["w"], c["d"], n_src=c["n_src"], nthreads=nthreads)
    if len(c["sched_step"]):
        net.set_sched(c["sched_step"], c["sched_src"])
    if np.any(c["pois_rate"] > 0):
        start, stop = c["pois_window"]
        net.set_poisson(c["pois_rate"], c["pois_w"], c["pois_d"], K.rng_seed, start, stop)
    net.set_record(c["rec_flags"])
    if c.get("pl") is not None:
        p, cm = c["pl"], c["pl"]["common"]
        psrc = np.repeat(np.arange(c["N"]), np.diff(p["row"]))
        # weights come back in the engine's CSR order (c["pl"]["order"] maps it to the front-end's)
        net.set_plastic(psrc, p["tgt"], p["w"], p["d"], lam=cm["lambda"], alpha=cm["alpha"], mu=cm["mu"],
                        tau_plus=cm["tau_plus"], n_src=c["N"])
    return net, c
