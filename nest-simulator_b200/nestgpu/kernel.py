"""Kernel state of the front-end: nodes, connections, time grid, and the
engine that runs the min_delay-slice cycle on the GPU.

Mirrors the parts of the reference kernel the cycle needs:
- time grid and rounding: nestkernel/nest_time.{h,cpp}
- delay extrema over all connections (devices included):
  nestkernel/connection_manager.cpp:485-530
- Simulate/Run/Prepare/Cleanup: nestkernel/nest.cpp:499-534,
  nestkernel/simulation_manager.cpp:507-671
- recorder windows t_min < stamp <= t_max: nestkernel/recording_device.cpp:206-211
- multimeter data of slice s becomes visible in slice s+1:
  nestkernel/universal_data_logger_impl.h:89-180
"""

import math
import time

import numpy as np

from . import _abi
from .models import (DEVICE_MODELS, GENERATORS, NEURON_MODELS, RECORDERS, SAMPLERS, BadProperty)
from .random import Parameter

INF_STEPS = 2**62


STATIC_SYNAPSES = ("static_synapse", "static_synapse_hom_w", "static_synapse_hpc")
STDP_SYNAPSES = ("stdp_pl_synapse_hom", "stdp_pl_synapse_hom_hpc")
STDP_COMMON = ("lambda", "alpha", "mu", "tau_plus")


class KernelException(RuntimeError):
    """Invalid kernel operation (the reference's KernelException)."""


class Device:
    def __init__(self, model, params):
        self.model = model
        self.params = {k: (list(v) if isinstance(v, list) else v) for k, v in params.items()}
        self.events = {}
        self.n_events = 0
        self.reset_events()

    def reset_events(self):
        if self.model in RECORDERS:
            self.events = {"senders": [], "times": []}
        elif self.model in SAMPLERS:
            self.events = {"senders": [], "times": []}
        self.n_events = 0


class Kernel:
    def __init__(self):
        self.reset()

    # ------------------------------------------------------------------
    # kernel status
    # ------------------------------------------------------------------
    def reset(self):
        old = getattr(self, "engine", None)
        if old is not None:
            old.close()
        self.tics_per_ms = 1000.0
        self.tics_per_step = 100
        self.rng_seed = 143202461
        self.local_num_threads = 1
        self.precision = "fp64"
        self.graph_slices = 64
        self.device = 0
        self.print_time = False
        self.user_min_delay = None
        self.user_max_delay = None
        self.models = {name: cls() for name, cls in NEURON_MODELS.items()}
        self.model_defaults = {m: dict(p) for m, p in DEVICE_MODELS.items()}
        # synapse models: defaults and kind ("static" or "stdp_pl"); the _hpc
        # variants are the reference's thread-indexed copies of the same rules
        stdp = {"weight": 1.0, "delay": 1.0, "lambda": 0.1, "alpha": 1.0, "mu": 0.4, "tau_plus": 20.0}
        self.syn_defaults = {m: {"weight": 1.0, "delay": 1.0} for m in STATIC_SYNAPSES}
        self.syn_defaults.update({m: dict(stdp) for m in STDP_SYNAPSES})
        self.syn_kind = {m: "static" for m in STATIC_SYNAPSES}
        self.syn_kind.update({m: "stdp_pl" for m in STDP_SYNAPSES})
        self.pl_src, self.pl_tgt, self.pl_w, self.pl_d, self.pl_model = [], [], [], [], []
        self.pl_models = []     # synapse model names of the plastic connections (index in pl_model)
        self._pl_fresh = True   # the host copy of the plastic weights is the engine's
        self.node_kind = np.zeros(0, dtype=np.int8)     # 0 neuron, 1 device
        self.node_model = []                             # model name per node
        self.node_local = np.zeros(0, dtype=np.int64)    # index in model storage / device list
        self.devices = []
        self.conn_src, self.conn_tgt, self.conn_w, self.conn_d = [], [], [], []
        self.n_conns = 0
        self.engine = None
        self.compiled = None
        self.structure_changed = True
        self.clock = 0          # steps simulated
        self.prepared = False
        self.time_simulate = 0.0
        self.spike_count = 0
        self.stats = {}
        self._rng = None
        self._unsettled = False  # a Run's last group still runs on the device

    @property
    def h(self):
        return (1.0 / self.tics_per_ms) * self.tics_per_step

    @property
    def ms_per_step(self):
        return self.tics_per_step / self.tics_per_ms

    @property
    def steps_per_ms(self):
        return 1 / self.ms_per_step

    def rng(self):
        if self._rng is None:
            self._rng = np.random.Generator(np.random.Philox(int(self.rng_seed)))
        return self._rng

    def set_resolution(self, h):
        self.settle()
        if len(self.node_kind) > 0:
            raise KernelException("Cannot change time representation after nodes have been created. "
                                  "Please call ResetKernel first.")
        tps = int(math.floor(self.tics_per_ms * float(h) + 0.5))
        if tps < 1:
            raise KernelException("Resolution must be at least one tic.")
        self.tics_per_step = tps

    def ms_to_steps_exact(self, t, what="Simulation time"):
        """Time(ms(t)) that must lie on the step grid (Simulate, spike times)."""
        tics = int(math.floor(float(t) * self.tics_per_ms + 0.5))
        if tics % self.tics_per_step != 0:
            raise KernelException(f"{what} must be a multiple of the simulation resolution.")
        return tics // self.tics_per_step

    def ms_to_steps_roundup(self, t):
        """Time(Time::ms(t)).get_steps(): round tics, then steps up."""
        if np.isinf(t):
            return INF_STEPS if t > 0 else -INF_STEPS
        tics = int(float(t) * self.tics_per_ms + 0.5)
        return int((tics + self.tics_per_step - 1) * (1.0 / self.tics_per_step))

    def delay_ms_to_steps(self, d):
        """Time::delay_ms_to_steps: ld_round(ms * STEPS_PER_MS) (nest_time.h:539-542)."""
        return np.floor(np.asarray(d, dtype=np.float64) * self.steps_per_ms + 0.5).astype(np.int64)

    def stamp_to_ms(self, stamps):
        """Time::step(s).get_ms() = MS_PER_TIC * (s * TICS_PER_STEP)."""
        return (1.0 / self.tics_per_ms) * (np.asarray(stamps, dtype=np.int64) * self.tics_per_step).astype(np.float64)

    # ------------------------------------------------------------------
    # nodes
    # ------------------------------------------------------------------
    def create(self, model, n, params):
        self.settle()
        if n < 1:
            raise BadProperty("Create: n must be >= 1")
        first_id = len(self.node_kind) + 1
        if model in self.models:
            st = self.models[model]
            first = st.grow(n)
            self.node_kind = np.concatenate([self.node_kind, np.zeros(n, dtype=np.int8)])
            self.node_local = np.concatenate([self.node_local, np.arange(first, first + n, dtype=np.int64)])
            self.node_model.extend([model] * n)
        elif model in DEVICE_MODELS:
            first = len(self.devices)
            for _ in range(n):
                self.devices.append(Device(model, self.model_defaults[model]))
            self.node_kind = np.concatenate([self.node_kind, np.ones(n, dtype=np.int8)])
            self.node_local = np.concatenate([self.node_local, np.arange(first, first + n, dtype=np.int64)])
            self.node_model.extend([model] * n)
        else:
            raise KernelException(f"Unknown model '{model}' (the engine provides "
                                  f"{sorted(list(NEURON_MODELS) + list(DEVICE_MODELS))})")
        self.structure_changed = True
        ids = np.arange(first_id, first_id + n, dtype=np.int64)
        if params:
            self.set_status(ids, params)
        return ids

    def _group(self, ids):
        """Split node ids into (model, positions-in-ids, local indices)."""
        ids = np.asarray(ids, dtype=np.int64)
        if len(ids) and (ids.min() < 1 or ids.max() > len(self.node_kind)):
            raise KernelException("Unknown node id")
        models = np.array(self.node_model, dtype=object)[ids - 1] if len(ids) else np.zeros(0, dtype=object)
        out = []
        for m in dict.fromkeys(models.tolist()):
            pos = np.nonzero(models == m)[0]
            out.append((m, pos, self.node_local[ids[pos] - 1]))
        return out

    def set_status(self, ids, params):
        self.settle()
        ids = np.asarray(ids, dtype=np.int64)
        if isinstance(params, (list, tuple)):
            if len(params) != len(ids):
                raise BadProperty("SetStatus: list of dictionaries must have one entry per node")
            for i, p in zip(ids, params):
                self.set_status(np.array([i]), p)
            return
        params = dict(params)
        for m, pos, loc in self._group(ids):
            sub = {}
            for k, v in params.items():
                if isinstance(v, Parameter):
                    v = v.sample(self.rng(), len(ids))
                if isinstance(v, (list, tuple, np.ndarray)) and not (m in DEVICE_MODELS and k in (
                        "spike_times", "record_from", "spike_weights", "spike_multiplicities")):
                    a = np.asarray(v)
                    if a.ndim >= 1 and len(a) == len(ids):
                        v = a[pos]
                    elif a.ndim >= 1 and len(ids) == 1:
                        pass
                    else:
                        raise BadProperty(f"SetStatus: '{k}' needs one value per node")
                sub[k] = v
            if m in self.models:
                st = self.models[m]
                unknown = [k for k in sub if k not in st.public and k not in ("frozen",)]
                if unknown:
                    raise BadProperty(f"Unaccessed dictionary entries for {m}: {unknown}")
                st.set(loc, sub)
            else:
                for j, li in enumerate(loc):
                    dev = self.devices[li]
                    for k, v in sub.items():
                        vv = v[j] if isinstance(v, np.ndarray) and v.ndim >= 1 and len(v) == len(loc) \
                            and k not in ("spike_times", "record_from") else v
                        self._set_device(dev, k, vv)

    def _set_device(self, dev, k, v):
        if k == "n_events":
            if int(v) != 0:
                raise BadProperty("n_events can only be set to 0.")
            dev.reset_events()
            return
        if k not in dev.params:
            raise BadProperty(f"Unaccessed dictionary entries for {dev.model}: ['{k}']")
        if dev.model in SAMPLERS and k in ("interval", "offset", "record_from") and self.prepared:
            raise BadProperty("The recording interval, the interval offset and the list of properties to record "
                              "cannot be changed after the multimeter has been connected and nodes have been "
                              "updated.")
        if k == "spike_times":
            v = [float(x) for x in np.asarray(v, dtype=np.float64).ravel()]
            for x in v:
                self.ms_to_steps_exact(x, "spike_generator: spike time")
            if any(b < a for a, b in zip(v, v[1:])):
                raise BadProperty("spike_generator: spike times must be sorted in non-descending order")
        elif k == "record_from":
            v = [str(x) for x in v]
        elif k in ("interval",):
            v = float(v)
            if self.ms_to_steps_roundup(v) < 1:
                raise BadProperty("The sampling interval must be at least as long as the simulation resolution.")
            self.ms_to_steps_exact(v, "The sampling interval")
        elif k == "offset":
            if float(v) != 0.0:
                raise NotImplementedError("multimeter offset != 0 is not supported by the engine")
            v = 0.0
        elif k in ("rate",):
            v = float(v)
            if v < 0:
                raise BadProperty("The rate cannot be negative.")
        elif k in ("start", "stop", "origin"):
            v = float(v)
        dev.params[k] = v
        self.structure_changed = True

    def get_status(self, ids, key=None):
        """List of per-node dicts (key None) or list of values."""
        self.settle()
        ids = np.asarray(ids, dtype=np.int64)
        out = [None] * len(ids)
        for m, pos, loc in self._group(ids):
            if m in self.models:
                st = self.models[m]
                if self.engine is not None and not self.structure_changed:
                    self._pull_state()
                keys = [key] if key is not None else list(st.public)
                vals = {}
                for k in keys:
                    if k in st.public:
                        vals[k] = st.get(loc, k)
                for j, p in enumerate(pos):
                    i = int(ids[p])
                    if key is not None:
                        if key in vals:
                            out[p] = vals[key][j].item()
                        else:
                            out[p] = self._common(i, m, key, True)
                    else:
                        d = {k: vals[k][j].item() for k in vals}
                        d.update(self._common(i, m, None, True))
                        d["recordables"] = list(st.recordables)
                        out[p] = d
            else:
                for j, p in enumerate(pos):
                    i = int(ids[p])
                    dev = self.devices[loc[j]]
                    d = dict(dev.params)
                    d.update(self._common(i, m, None, False))
                    if m in RECORDERS or m in SAMPLERS:
                        d["events"] = {k: (np.concatenate(v) if len(v) else
                                           np.zeros(0, dtype=np.int64 if k == "senders" else np.float64))
                                           for k, v in dev.events.items()}
                        d["n_events"] = dev.n_events
                    if key is not None:
                        if key not in d:
                            raise KeyError(key)
                        out[p] = d[key]
                    else:
                        out[p] = d
        return out

    def _common(self, i, m, key, neuron):
        d = {"global_id": i, "model": m, "element_type": "neuron" if neuron else (
            "recorder" if m in RECORDERS or m in SAMPLERS else "stimulator"),
            "local": True, "frozen": False, "thread": 0, "vp": 0}
        if key is not None:
            if key not in d:
                raise KeyError(key)
            return d[key]
        return d

    # ------------------------------------------------------------------
    # connections
    # ------------------------------------------------------------------
    def add_edges(self, src, tgt, w, d_ms):
        self.settle()
        src = np.asarray(src, dtype=np.int64).ravel()
        tgt = np.asarray(tgt, dtype=np.int64).ravel()
        n = len(src)
        if n == 0:
            return
        w = np.broadcast_to(np.asarray(w, dtype=np.float64), (n,)).copy()
        d_ms = np.broadcast_to(np.asarray(d_ms, dtype=np.float64), (n,))
        steps = self.delay_ms_to_steps(d_ms)
        if np.any(steps < 1):
            raise BadProperty("Delay must be greater than or equal to resolution")
        if src.max() > len(self.node_kind) or tgt.max() > len(self.node_kind) or src.min() < 1 or tgt.min() < 1:
            raise KernelException("Connect: unknown node id")
        self.conn_src.append(src.astype(np.int32))
        self.conn_tgt.append(tgt.astype(np.int32))
        self.conn_w.append(w)
        self.conn_d.append(steps.astype(np.int32))
        self.n_conns += n
        self.structure_changed = True

    def add_plastic_edges(self, src, tgt, w, d_ms, model):
        """stdp_pl_synapse_hom connections (neuron -> neuron)."""
        self.settle()
        self._pull_plastic()
        src = np.asarray(src, dtype=np.int64).ravel()
        tgt = np.asarray(tgt, dtype=np.int64).ravel()
        n = len(src)
        if n == 0:
            return
        w = np.broadcast_to(np.asarray(w, dtype=np.float64), (n,)).copy()
        steps = self.delay_ms_to_steps(np.broadcast_to(np.asarray(d_ms, dtype=np.float64), (n,)))
        if np.any(steps < 1):
            raise BadProperty("Delay must be greater than or equal to resolution")
        if src.max() > len(self.node_kind) or tgt.max() > len(self.node_kind) or src.min() < 1 or tgt.min() < 1:
            raise KernelException("Connect: unknown node id")
        if np.any(self.node_kind[src - 1] != 0) or np.any(self.node_kind[tgt - 1] != 0):
            raise KernelException(f"{model} connects neurons to neurons")
        if np.any(w < 0):
            raise BadProperty("Weight of stdp_pl_synapse_hom must be non-negative (power-law facilitation)")
        if model not in self.pl_models:
            self.pl_models.append(model)
        self.pl_src.append(src.astype(np.int32))
        self.pl_tgt.append(tgt.astype(np.int32))
        self.pl_w.append(w)
        self.pl_d.append(steps.astype(np.int32))
        self.pl_model.append(np.full(n, self.pl_models.index(model), dtype=np.int16))
        self.structure_changed = True

    def plastic_edges(self):
        """(src, tgt, weight, delay steps, model index) of the plastic
        connections; weights as the engine has them after the last run."""
        self._pull_plastic()
        if not self.pl_src:
            z = np.zeros(0, dtype=np.int32)
            return z, z, np.zeros(0), z, np.zeros(0, dtype=np.int16)
        if len(self.pl_src) > 1:
            for a in ("pl_src", "pl_tgt", "pl_w", "pl_d", "pl_model"):
                setattr(self, a, [np.concatenate(getattr(self, a))])
        return self.pl_src[0], self.pl_tgt[0], self.pl_w[0], self.pl_d[0], self.pl_model[0]

    def _pull_plastic(self):
        c = self.compiled
        if self.engine is None or c is None or c.get("pl") is None or self._pl_fresh:
            return
        self.settle()
        self._pl_fresh = True
        w = self.engine.plastic_weights()
        self.pl_w[0][c["pl"]["order"]] = w

    def stdp_common(self):
        """The common properties of the network's plastic connections (one
        set per network on the engine)."""
        if not self.pl_models:
            return None
        sets = {tuple(float(self.syn_defaults[m][k]) for k in STDP_COMMON) for m in self.pl_models}
        if len(sets) > 1:
            raise NotImplementedError("stdp_pl_synapse_hom models with different common properties in one network "
                                      "are not supported by the engine")
        return dict(zip(STDP_COMMON, sets.pop()))

    def edges(self):
        if not self.conn_src:
            z = np.zeros(0, dtype=np.int32)
            return z, z, np.zeros(0), z
        if len(self.conn_src) > 1:
            self.conn_src = [np.concatenate(self.conn_src)]
            self.conn_tgt = [np.concatenate(self.conn_tgt)]
            self.conn_w = [np.concatenate(self.conn_w)]
            self.conn_d = [np.concatenate(self.conn_d)]
        return self.conn_src[0], self.conn_tgt[0], self.conn_w[0], self.conn_d[0]

    # ------------------------------------------------------------------
    # compile the network into engine arrays
    # ------------------------------------------------------------------
    def compile(self):
        """Lower the node/connection tables to the engine's inputs (numpy)."""
        kinds = self.node_kind
        n_nodes = len(kinds)
        model_arr = np.array(self.node_model, dtype=object)
        blocks = []
        node_to_eng = np.full(n_nodes + 1, -1, dtype=np.int64)
        off = 0
        for name, st in self.models.items():
            if st.n == 0:
                continue
            ids = np.nonzero(model_arr == name)[0] + 1
            node_to_eng[ids] = off + self.node_local[ids - 1]
            blocks.append({"model": name, "engine_model": st.engine_model, "n": st.n, "off": off})
            off += st.n
        N = off
        gen_ids = [i + 1 for i in range(n_nodes) if self.node_model[i] == "spike_generator"]
        for k, i in enumerate(gen_ids):
            node_to_eng[i] = N + k
        n_src = N + len(gen_ids)
        eng_to_node = np.zeros(n_src, dtype=np.int64)
        valid = node_to_eng >= 0
        eng_to_node[node_to_eng[valid]] = np.nonzero(valid)[0]

        src, tgt, w, dsteps = self.edges()
        is_neuron = np.concatenate([[False], kinds == 0])
        smodel = np.concatenate([[""], model_arr]) if n_nodes else np.array([""], dtype=object)
        s_neu = is_neuron[src]
        t_neu = is_neuron[tgt]
        s_mod = smodel[src]
        t_mod = smodel[tgt]
        s_gen = s_mod == "spike_generator"
        m_syn = (s_neu | s_gen) & t_neu
        m_pg = (s_mod == "poisson_generator") & t_neu
        m_rec = (s_neu | s_gen) & (t_mod == "spike_recorder")
        m_mm = ((s_mod == "multimeter") | (s_mod == "voltmeter")) & t_neu
        bad = ~(m_syn | m_pg | m_rec | m_mm)
        if np.any(bad):
            k = int(np.nonzero(bad)[0][0])
            raise KernelException(f"Connection {s_mod[k]} -> {t_mod[k]} is not supported by the engine")
        psrc, ptgt, pw, pdl, _ = self.plastic_edges()
        alld = np.concatenate([dsteps, pdl]) if len(pdl) else dsteps
        # delay extrema over all connections, devices included
        if self.user_min_delay is not None:
            min_d, max_d = self.user_min_delay, self.user_max_delay
            if len(alld) and (alld.min() < min_d or alld.max() > max_d):
                raise BadProperty("Connection delays lie outside the user-set min_delay/max_delay")
        elif len(alld):
            min_d, max_d = int(alld.min()), int(alld.max())
        else:
            min_d = max_d = 1
        c = {"blocks": blocks, "N": N, "n_src": n_src, "min_delay": min_d, "max_delay": max_d,
             "node_to_eng": node_to_eng, "eng_to_node": eng_to_node, "gen_ids": gen_ids}
        # recurrent + generator edges (COO over engine indices)
        c["src"] = node_to_eng[src[m_syn]].astype(np.int32)
        c["tgt"] = node_to_eng[tgt[m_syn]].astype(np.int32)
        c["w"] = w[m_syn]
        c["d"] = dsteps[m_syn].astype(np.int32)
        # plastic connections: a CSR over neuron sources (stable order by source)
        c["pl"] = None
        if len(psrc):
            es, et = node_to_eng[psrc], node_to_eng[ptgt]
            order = np.argsort(es, kind="stable")
            row = np.zeros(N + 1, dtype=np.int64)
            np.cumsum(np.bincount(es, minlength=N), out=row[1:])
            c["pl"] = {"row": row, "tgt": et[order].astype(np.int32), "w": pw[order], "d": pdl[order],
                       "order": order, "common": self.stdp_common()}
        # Poisson drive, fused per target neuron
        rate = np.zeros(N)
        pw = np.zeros(N)
        pd = np.full(N, min_d, dtype=np.int32)
        windows = set()
        if np.any(m_pg):
            ps, pt, pwv, pdv = src[m_pg], node_to_eng[tgt[m_pg]], w[m_pg], dsteps[m_pg]
            seen_w = np.full(N, np.nan)
            seen_d = np.full(N, -1, dtype=np.int64)
            for k in range(len(ps)):
                dev = self.devices[self.node_local[ps[k] - 1]]
                r = float(dev.params["rate"])
                t = pt[k]
                if not np.isnan(seen_w[t]) and (seen_w[t] != pwv[k] or seen_d[t] != pdv[k]):
                    raise NotImplementedError("a neuron with Poisson inputs of different weights or delays is not "
                                              "supported by the engine's fused drive")
                seen_w[t], seen_d[t] = pwv[k], pdv[k]
                rate[t] += r
                pw[t] = pwv[k]
                pd[t] = pdv[k]
                o = float(dev.params["origin"])
                start = self.ms_to_steps_roundup(o + float(dev.params["start"]))
                stop = INF_STEPS if np.isinf(dev.params["stop"]) else \
                    self.ms_to_steps_roundup(o + float(dev.params["stop"]))
                windows.add((start, stop))
        if len(windows) > 1:
            raise NotImplementedError("Poisson generators with different start/stop windows are not supported")
        c["pois_rate"], c["pois_w"], c["pois_d"] = rate, pw, pd
        c["pois_window"] = windows.pop() if windows else (0, INF_STEPS)
        # spike generator schedule: emission step = stamp - 1
        sched_s, sched_src = [], []
        for k, gid in enumerate(gen_ids):
            dev = self.devices[self.node_local[gid - 1]]
            p = dev.params
            o = self.ms_to_steps_roundup(float(p["origin"]))
            t_min = self.ms_to_steps_roundup(float(p["origin"]) + float(p["start"]))
            t_max = INF_STEPS if np.isinf(p["stop"]) else self.ms_to_steps_roundup(float(p["origin"]) +
                                                                                    float(p["stop"]))
            for ts in p["spike_times"]:
                stamp = o + self.ms_to_steps_exact(ts, "spike_generator: spike time")
                if t_min < stamp <= t_max:
                    sched_s.append(stamp - 1)
                    sched_src.append(N + k)
        order = np.argsort(np.asarray(sched_s, dtype=np.int64), kind="stable")
        c["sched_step"] = np.asarray(sched_s, dtype=np.int64)[order]
        c["sched_src"] = np.asarray(sched_src, dtype=np.int32)[order]
        # recorders
        rec_ids = [i + 1 for i in range(n_nodes) if self.node_model[i] in RECORDERS]
        flags = np.zeros(n_src, dtype=np.uint8)
        c["recorders"] = {}
        if np.any(m_rec):
            rs, rt = node_to_eng[src[m_rec]], tgt[m_rec]
            for rid in rec_ids:
                mask = np.zeros(n_src, dtype=bool)
                mask[rs[rt == rid]] = True
                c["recorders"][rid] = mask
                flags |= mask.astype(np.uint8)
        c["rec_flags"] = flags
        # recorders over disjoint sources (one population each, the usual case):
        # a source's recorder index, so a run's spikes are split in one pass
        c["rec_part"] = None
        if c["recorders"] and len(c["recorders"]) < 32767:
            rids = list(c["recorders"])
            cover = np.zeros(n_src, dtype=np.int32)
            for rid in rids:
                cover += c["recorders"][rid]
            if cover.max() <= 1:
                of = np.full(n_src, -1, dtype=np.int16)
                for j, rid in enumerate(rids):
                    of[c["recorders"][rid]] = j
                c["rec_part"] = (rids, of)
        # samplers (multimeter / voltmeter)
        c["samplers"] = {}
        if np.any(m_mm):
            ms_, mt_ = src[m_mm], node_to_eng[tgt[m_mm]]
            for mid in dict.fromkeys(ms_.tolist()):
                dev = self.devices[self.node_local[mid - 1]]
                c["samplers"][mid] = np.unique(mt_[ms_ == mid])
        return c

    # ------------------------------------------------------------------
    # engine lifecycle
    # ------------------------------------------------------------------
    def _engine_var_names(self, model):
        return self.models[model].engine_vars

    def _pull_state(self):
        """Copy engine state back into the front-end storage."""
        if self.engine is None or self.compiled is None:
            return
        self._pull_plastic()
        for bi, b in enumerate(self.compiled["blocks"]):
            st = self.models[b["model"]]
            for k in st.state_vars:
                if k in st.dirty:  # a value set by the user and not pushed yet wins
                    continue
                st.data[k][:b["n"]] = self.engine.get_var(bi, st.engine_vars[k])
            st.engine_r = self.engine.get_var(bi, "r")
            if b["model"] == "aeif_cond_alpha":
                st.engine_istep = self.engine.get_var(bi, "integration_step")

    def _push_dirty(self):
        for bi, b in enumerate(self.compiled["blocks"]):
            st = self.models[b["model"]]
            for k in sorted(st.dirty):
                if k in st.engine_vars:
                    self.engine.set_var(bi, st.engine_vars[k], st.data[k][:b["n"]])
            st.dirty = set()

    def _build_engine(self):
        keep_r = {}
        if self.engine is not None:
            self._pull_state()
            for b in self.compiled["blocks"]:
                st = self.models[b["model"]]
                keep_r[b["model"]] = (getattr(st, "engine_r", None), getattr(st, "engine_istep", None))
            self.engine.close()
            self.engine = None
        c = self.compile()
        if c["N"] == 0:
            self.compiled = c
            return
        prec = _abi.NG_FP32 if self.precision == "fp32" else _abi.NG_FP64
        eng = _abi.Engine([(b["engine_model"], b["n"]) for b in c["blocks"]], self.h, c["min_delay"],
                          c["max_delay"], n_generators=len(c["gen_ids"]), precision=prec, device=self.device,
                          tics_per_ms=self.tics_per_ms, start_step=self.clock)
        self.engine = eng
        self.engine_start = self.clock
        self.compiled = c
        for bi, b in enumerate(c["blocks"]):
            st = self.models[b["model"]]
            for k, ev in st.engine_vars.items():
                eng.set_var(bi, ev, st.data[k][:b["n"]])
            st.dirty = set()
            r, istep = keep_r.get(b["model"], (None, None))
            if r is not None and len(r) <= b["n"]:
                eng.set_var(bi, "r", r)
                if istep is not None:
                    eng.set_var(bi, "integration_step", istep)
        eng.set_connections_coo(c["src"], c["tgt"], c["w"], c["d"], c["n_src"])
        if c["pl"] is not None:
            p = c["pl"]
            cm = p["common"]
            eng.set_plastic(p["row"], p["tgt"], p["w"], p["d"], lam=cm["lambda"], alpha=cm["alpha"], mu=cm["mu"],
                            tau_plus=cm["tau_plus"])
        self._pl_fresh = True
        if len(c["sched_step"]):
            eng.set_spike_schedule(c["sched_step"], c["sched_src"])
        if np.any(c["pois_rate"] > 0):
            start, stop = c["pois_window"]
            eng.set_poisson(c["pois_rate"], c["pois_w"], c["pois_d"], start, stop, self.rng_seed)
        eng.set_recording(c["rec_flags"])
        self._setup_samplers(c)
        eng.set_graph_slices(self.graph_slices)
        self.structure_changed = False

    def _setup_samplers(self, c):
        self.trace_neurons = None
        self._trace_buf = []
        if not c["samplers"]:
            return
        intervals = set()
        vars_ = []
        models = set()
        for mid, neurons in c["samplers"].items():
            dev = self.devices[self.node_local[mid - 1]]
            intervals.add(self.ms_to_steps_exact(dev.params["interval"], "The sampling interval"))
            for v in dev.params["record_from"]:
                if v not in vars_:
                    vars_.append(v)
            for bi, b in enumerate(c["blocks"]):
                sel = (neurons >= b["off"]) & (neurons < b["off"] + b["n"])
                if np.any(sel):
                    models.add(b["model"])
        if len(intervals) > 1:
            raise NotImplementedError("multimeters with different intervals are not supported together")
        if len(models) > 1:
            raise NotImplementedError("multimeters recording from several neuron models are not supported together")
        model = models.pop()
        st = self.models[model]
        for v in vars_:
            if v not in st.recordables:
                raise BadProperty(f"{model} has no recordable '{v}'")
        neurons = np.unique(np.concatenate(list(c["samplers"].values())))
        evars = [("V_m_rel" if "V_m_rel" in st.engine_vars else "V_m") if v == "V_m" else v for v in vars_]
        self.engine.set_trace(neurons, evars, intervals.pop())
        self.trace_neurons = neurons
        self.trace_vars = vars_
        self.trace_model = model
        self.trace_interval = self.ms_to_steps_exact(
            self.devices[self.node_local[next(iter(c["samplers"])) - 1]].params["interval"], "The sampling interval")

    def settle(self):
        """Wait for the steps a Run left running on the device and hand their
        spikes to the recorders (every read or change of the network does
        this first; Run itself returns while its last group still runs)."""
        if self._unsettled and self.engine is not None:
            self._unsettled = False
            self.engine.sync()
            self._collect()
            self.stats = self.engine.stats()
        self._unsettled = False

    def prepare(self):
        self.settle()
        if self.structure_changed or self.engine is None:
            self._build_engine()
        elif self.engine is not None:
            self._push_dirty()
        self.prepared = True

    def run(self, t_ms):
        if not self.prepared:
            raise KernelException("Run: call Prepare first")
        steps = self.ms_to_steps_exact(t_ms)
        if steps < 0:
            raise KernelException("Simulation time must be >= 0")
        if self.structure_changed:
            self.prepare()
        t0 = time.perf_counter()
        if self.engine is not None and steps > 0:
            self._push_dirty()
            # the Run in up to four calls of whole slice graphs, each leaving its
            # last group running: the spikes drained before it (the previous
            # call's) reach the recorders while it runs
            unit = max(1, self.graph_slices) * int(self.compiled["min_delay"])
            part = max(unit, -(-steps // (4 * unit)) * unit)
            left = steps
            while left > 0:
                k = min(part, left)
                self.engine.simulate_async(k)
                self._pl_fresh = False
                self.clock += k
                left -= k
                self._unsettled = True
                self._collect()
        else:
            self.clock += steps
        self.time_simulate = time.perf_counter() - t0

    def simulate(self, t_ms):
        if self.ms_to_steps_exact(t_ms) < 0:
            raise KernelException("Simulation time must be >= 0")
        self.prepare()
        self.run(t_ms)
        self.cleanup()

    def cleanup(self):
        self.settle()
        self.prepared = False

    def _collect(self):
        c = self.compiled
        src, stamp = self.engine.spikes()
        self.spike_count += int(np.sum(src < c["N"]))
        if len(src) and c["recorders"]:
            senders = c["eng_to_node"][src]
            times = self.stamp_to_ms(stamp)
            part = c.get("rec_part")
            if part is not None:
                # one stable counting sort by recorder, then each recorder's
                # spikes are a contiguous run (in emission order)
                rids, of = part
                k = of[src]
                order = np.argsort(k, kind="stable")
                bounds = np.concatenate([[0], np.cumsum(np.bincount(k.astype(np.int64) + 1,
                                                                    minlength=len(rids) + 1))])
                for j, rid in enumerate(rids):
                    o = order[bounds[j + 1]:bounds[j + 2]]
                    if len(o):
                        self._record(rid, senders[o], stamp[o], times[o])
            else:
                for rid, mask in c["recorders"].items():
                    sel = mask[src]
                    if np.any(sel):
                        self._record(rid, senders[sel], stamp[sel], times[sel])
        if c["samplers"] and self.trace_neurons is not None:
            first, rows = self.engine.trace()
            if len(rows):
                self._trace_buf.append((first, rows))
            self._flush_samplers()

    def _record(self, rid, senders, stamp, times):
        """Spikes of a recorder's sources into its events (start/stop window)."""
        dev = self.devices[self.node_local[rid - 1]]
        p = dev.params
        t_min = self.ms_to_steps_roundup(float(p["origin"]) + float(p["start"]))
        t_max = INF_STEPS if np.isinf(p["stop"]) else self.ms_to_steps_roundup(float(p["origin"]) +
                                                                                float(p["stop"]))
        sel = (stamp > t_min) & (stamp <= t_max)
        if not np.any(sel):
            return
        if not np.all(sel):
            senders, stamp, times = senders[sel], stamp[sel], times[sel]
        dev.events["senders"].append(senders)
        dev.events["times"].append(stamp if p.get("time_in_steps") else times)
        dev.n_events += len(senders)

    def _flush_samplers(self):
        """Hand trace rows to the multimeters when the reference would: data
        recorded in slice s reaches the multimeter during slice s + 1, so after
        a run that ends on a slice boundary the last slice is still pending."""
        c = self.compiled
        md = c["min_delay"]
        pos = (self.clock - self.engine_start) % md
        slice_origin = self.clock - pos
        limit = slice_origin - md if pos == 0 else slice_origin
        keep = []
        st = self.models[self.trace_model]
        neurons = self.trace_neurons
        node_ids = c["eng_to_node"][neurons]
        block = [b for b in c["blocks"] if b["model"] == self.trace_model][0]
        loc = neurons - block["off"]
        interval = self.trace_interval
        for first, rows in self._trace_buf:
            stamps = first + interval * np.arange(len(rows))
            vis = stamps <= limit
            if np.any(vis):
                for mid, sel_neurons in c["samplers"].items():
                    dev = self.devices[self.node_local[mid - 1]]
                    p = dev.params
                    t_min = self.ms_to_steps_roundup(float(p["origin"]) + float(p["start"]))
                    t_max = INF_STEPS if np.isinf(p["stop"]) else self.ms_to_steps_roundup(
                        float(p["origin"]) + float(p["stop"]))
                    cols = np.searchsorted(neurons, sel_neurons)
                    srow = vis & (stamps > t_min) & (stamps <= t_max)
                    if not np.any(srow):
                        continue
                    nr = int(srow.sum())
                    dev.events["senders"].append(np.tile(node_ids[cols], nr))
                    dev.events["times"].append(np.repeat(self.stamp_to_ms(stamps[srow]), len(cols)))
                    for vi, v in enumerate(self.trace_vars):
                        if v not in p["record_from"]:
                            continue
                        vals = rows[srow][:, vi, :][:, cols]
                        vals = st.recordable_value(v, vals, loc[cols][None, :])
                        dev.events.setdefault(v, []).append(np.asarray(vals).ravel())
                    dev.n_events += nr * len(cols)
            if not np.all(vis):
                keep.append((first + interval * int(np.sum(vis)), rows[~vis]))
        self._trace_buf = keep

    def num_connections(self):
        src, tgt, _, _ = self.edges()
        return len(src) + sum(len(a) for a in self.pl_src)

    def get_connections(self, source=None, target=None, plastic=False):
        self.settle()
        if plastic:
            src, tgt = self.plastic_edges()[:2]
        else:
            src, tgt, w, d = self.edges()
        m = np.ones(len(src), dtype=bool)
        if source is not None:
            m &= np.isin(src, np.asarray(source))
        if target is not None:
            m &= np.isin(tgt, np.asarray(target))
        idx = np.nonzero(m)[0]
        order = np.lexsort((tgt[idx], src[idx]))
        return idx[order]


KERNEL = Kernel()
