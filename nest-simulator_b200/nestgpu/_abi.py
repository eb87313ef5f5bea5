"""ctypes binding of the engine's C ABI (include/nestgpu.h).

The product path is this library and nothing else: if ``libnestgpu.so`` is
missing or no CUDA device is present, the calls raise -- there is no CPU
fallback.
"""

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnestgpu.so")

NG_OK = 0
NG_ERR_ARG = -1
NG_ERR_CUDA = -2
NG_ERR_STATE = -3
NG_ERR_NUMERIC = -4
NG_ERR_MEMORY = -5
NG_ERR_CAPACITY = -6
NG_ERR_UNKNOWN_NAME = -7

NG_IAF_PSC_DELTA, NG_IAF_PSC_EXP, NG_AEIF_COND_ALPHA, NG_IAF_PSC_ALPHA = 0, 1, 2, 3
NG_FP64, NG_FP32 = 0, 1
NG_MAX_BLOCKS = 8

#: every symbol include/nestgpu.h declares
EXPORTED = [
    "ng_abi_version", "ng_last_error", "ng_device_count", "ng_create", "ng_destroy", "ng_set_var", "ng_get_var",
    "ng_set_connections", "ng_set_connections_coo", "ng_set_spike_schedule", "ng_set_poisson", "ng_set_recording", "ng_set_trace",
    "ng_simulate", "ng_simulate_async", "ng_sync", "ng_spike_count", "ng_get_spikes", "ng_trace_count", "ng_get_trace", "ng_get_stats",
    "ng_set_profiling", "ng_set_stream", "ng_set_graph_slices", "ng_debug_coefficients", "ng_net_add", "ng_net_poll",
    "ng_net_spikes", "ng_net_get_var", "ng_net_get_connections", "ng_net_remove", "ng_net_capacity",
    "ng_simulate_noalloc", "ng_set_tuning", "ng_get_tuning", "ng_set_option", "ng_update",
    "ng_set_plastic_connections", "ng_get_plastic_weights",
]


class NGConfig(ctypes.Structure):
    _fields_ = [
        ("device", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("h", ctypes.c_double),
        ("tics_per_ms", ctypes.c_double),
        ("min_delay", ctypes.c_int32),
        ("max_delay", ctypes.c_int32),
        ("n_blocks", ctypes.c_int32),
        ("block_model", ctypes.c_int32 * NG_MAX_BLOCKS),
        ("block_size", ctypes.c_int64 * NG_MAX_BLOCKS),
        ("n_generators", ctypes.c_int64),
        ("spike_log_capacity", ctypes.c_int64),
        ("start_step", ctypes.c_int64),
        ("serving", ctypes.c_int32),
        ("max_networks", ctypes.c_int32),
        ("edge_capacity", ctypes.c_int64),
        ("max_abs_weight", ctypes.c_double),
        ("ring32", ctypes.c_int32),
        ("ring_bound", ctypes.c_double),
        ("tile_capacity", ctypes.c_int64),
    ]


class NGFixedIndegree(ctypes.Structure):
    _fields_ = [
        ("n_exc", ctypes.c_int64),
        ("k_exc", ctypes.c_int32),
        ("k_inh", ctypes.c_int32),
        ("w_exc", ctypes.c_double),
        ("w_inh", ctypes.c_double),
        ("delay_steps", ctypes.c_int32),
        ("allow_autapses", ctypes.c_int32),
        ("seed", ctypes.c_uint64),
    ]


NG_MAX_POPS = 16


def tile_targets(max_delay, ring32=False):
    """Largest number of targets per tile of the target-tiled delivery (as
    the engine computes it)."""
    esz = 4 if ring32 else 8
    return min(1024, (163840 // (min(max_delay, 32) * 2 * esz)) // 32 * 32)


def tile_table_entries(n, max_delay, ring32=False, sms=None):
    """Segment-table entries a tiled network of n neurons takes (the
    engine's rule: about a multiple of the SM count of tiles)."""
    if sms is None:
        try:
            import torch

            sms = torch.cuda.get_device_properties(0).multi_processor_count
        except Exception:
            sms = 148
    T = tile_targets(max_delay, ring32)
    rounds = -(-n // (T * sms))
    tt = min(T, (-(-n // (rounds * sms)) + 31) // 32 * 32)
    return n * (-(-n // tt) + 1)


class NGPairwiseBernoulli(ctypes.Structure):
    _fields_ = [
        ("n_pops", ctypes.c_int32),
        ("pop_size", ctypes.c_int64 * NG_MAX_POPS),
        ("pop_exc", ctypes.c_int32 * NG_MAX_POPS),
        ("p", ctypes.c_double * (NG_MAX_POPS * NG_MAX_POPS)),
        ("w_mean", ctypes.c_double * 2),
        ("w_sd", ctypes.c_double * 2),
        ("d_mean_ms", ctypes.c_double * 2),
        ("d_sd_ms", ctypes.c_double * 2),
        ("d_max_ms", ctypes.c_double),
        ("allow_autapses", ctypes.c_int32),
        ("seed", ctypes.c_uint64),
    ]

    @classmethod
    def make(cls, pop_size, pop_exc, p, w_mean, w_sd, d_mean_ms, d_sd_ms, d_max_ms, allow_autapses=0, seed=0):
        """p[i][j]: probability that a neuron of population i projects to one
        of population j; w_*/d_*: (inhibitory source, excitatory source)."""
        k = len(pop_size)
        if not 1 <= k <= NG_MAX_POPS:
            raise ValueError("1 to 16 populations")
        s = cls(n_pops=k, d_max_ms=float(d_max_ms), allow_autapses=int(allow_autapses), seed=int(seed) & (2**64 - 1))
        pp = np.asarray(p, dtype=np.float64).reshape(k, k)
        for i in range(k):
            s.pop_size[i] = int(pop_size[i])
            s.pop_exc[i] = 1 if pop_exc[i] else 0
            for j in range(k):
                s.p[i * NG_MAX_POPS + j] = float(pp[i, j])
        for a in range(2):
            s.w_mean[a], s.w_sd[a] = float(w_mean[a]), float(w_sd[a])
            s.d_mean_ms[a], s.d_sd_ms[a] = float(d_mean_ms[a]), float(d_sd_ms[a])
        return s


class NGNetDesc(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int64),
        ("steps", ctypes.c_int64),
        ("seed", ctypes.c_uint64),
        ("record", ctypes.c_int32),
        ("n_vars", ctypes.c_int32),
        ("var_names", ctypes.c_void_p),
        ("var_values", ctypes.c_void_p),
        ("nnz", ctypes.c_int64),
        ("source", ctypes.c_void_p),
        ("target", ctypes.c_void_p),
        ("weight", ctypes.c_void_p),
        ("delay_steps", ctypes.c_void_p),
        ("build", ctypes.c_void_p),
        ("poisson_rate", ctypes.c_void_p),
        ("poisson_weight", ctypes.c_void_p),
        ("poisson_delay", ctypes.c_void_p),
        ("build_pb", ctypes.c_void_p),
    ]


class NGStats(ctypes.Structure):
    _fields_ = [
        ("clock_steps", ctypes.c_int64),
        ("slices", ctypes.c_int64),
        ("spikes", ctypes.c_int64),
        ("syn_events", ctypes.c_int64),
        ("drive_events", ctypes.c_int64),
        ("update_ms", ctypes.c_double),
        ("deliver_ms", ctypes.c_double),
        ("update_launches", ctypes.c_int64),
        ("deliver_launches", ctypes.c_int64),
        ("simulate_ms", ctypes.c_double),
        ("gather_slices", ctypes.c_int64),
        ("wait_ms", ctypes.c_double),
        ("drain_ms", ctypes.c_double),
    ]


class EngineError(RuntimeError):
    """Error status returned by the engine's C ABI."""

    def __init__(self, code, msg):
        super().__init__(f"nestgpu error {code}: {msg}")
        self.code = code


_lib = None


def load():
    """Load libnestgpu.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with __graft_entry__.build() "
                          "or `make -C nest-simulator_b200/csrc`; the engine has no CPU fallback")
    L = ctypes.CDLL(LIB_PATH)
    P = ctypes.c_void_p
    i32, i64, dbl = ctypes.c_int32, ctypes.c_int64, ctypes.c_double
    sig = {
        "ng_abi_version": ([], ctypes.c_int),
        "ng_last_error": ([], ctypes.c_char_p),
        "ng_device_count": ([P], ctypes.c_int),
        "ng_create": ([P, P], ctypes.c_int),
        "ng_destroy": ([P], ctypes.c_int),
        "ng_set_var": ([P, i32, ctypes.c_char_p, P, i64, i64], ctypes.c_int),
        "ng_get_var": ([P, i32, ctypes.c_char_p, P, i64, i64], ctypes.c_int),
        "ng_set_connections": ([P, i64, P, P, P, P], ctypes.c_int),
        "ng_set_connections_coo": ([P, i64, i64, P, P, P, P], ctypes.c_int),
        "ng_set_spike_schedule": ([P, i64, P, P], ctypes.c_int),
        "ng_set_poisson": ([P, P, P, P, i64, i64, ctypes.c_uint64], ctypes.c_int),
        "ng_set_recording": ([P, P], ctypes.c_int),
        "ng_set_trace": ([P, i64, P, i32, P, i32], ctypes.c_int),
        "ng_simulate": ([P, i64], ctypes.c_int),
        "ng_simulate_async": ([P, i64], ctypes.c_int),
        "ng_sync": ([P], ctypes.c_int),
        "ng_spike_count": ([P, P], ctypes.c_int),
        "ng_get_spikes": ([P, P, P, i64, P], ctypes.c_int),
        "ng_trace_count": ([P, P, P], ctypes.c_int),
        "ng_get_trace": ([P, P, i64, P], ctypes.c_int),
        "ng_get_stats": ([P, P], ctypes.c_int),
        "ng_set_profiling": ([P, i32], ctypes.c_int),
        "ng_set_stream": ([P, P], ctypes.c_int),
        "ng_set_graph_slices": ([P, i32], ctypes.c_int),
        "ng_debug_coefficients": ([P, i32, i64, P, i32, P], ctypes.c_int),
        "ng_net_add": ([P, P, P], ctypes.c_int),
        "ng_net_poll": ([P, i32, P, P], ctypes.c_int),
        "ng_net_spikes": ([P, i32, P, P, i64, P], ctypes.c_int),
        "ng_net_get_var": ([P, i32, ctypes.c_char_p, P], ctypes.c_int),
        "ng_net_get_connections": ([P, i32, P, P, P, P, i64, P], ctypes.c_int),
        "ng_net_remove": ([P, i32], ctypes.c_int),
        "ng_net_capacity": ([P, P, P], ctypes.c_int),
        "ng_set_tuning": ([P, i32, i32, i32, i32], ctypes.c_int),
        "ng_get_tuning": ([P, P], ctypes.c_int),
        "ng_set_option": ([P, ctypes.c_char_p, dbl], ctypes.c_int),
        "ng_update": ([P, i64, i32, i32], ctypes.c_int),
        "ng_set_plastic_connections": ([P, i64, P, P, P, P, dbl, dbl, dbl, dbl], ctypes.c_int),
        "ng_get_plastic_weights": ([P, P, i64], ctypes.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def _p(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None and a.size else ctypes.c_void_p(0)


def check(rc):
    if rc != NG_OK:
        raise EngineError(rc, load().ng_last_error().decode(errors="replace"))


def device_count():
    n = ctypes.c_int32(0)
    rc = load().ng_device_count(ctypes.byref(n))
    return n.value if rc == NG_OK else 0


class NGTuning(ctypes.Structure):
    _fields_ = [
        ("mode", ctypes.c_int32),
        ("state", ctypes.c_int32),
        ("update_variant", ctypes.c_int32),
        ("deliver_per_sm", ctypes.c_int32),
        ("deliver_group", ctypes.c_int32),
        ("cache_hit", ctypes.c_int32),
        ("rate_bucket", ctypes.c_int32),
        ("n_candidates", ctypes.c_int32),
        ("cand_variant", ctypes.c_int32 * 32),
        ("cand_per_sm", ctypes.c_int32 * 32),
        ("cand_group", ctypes.c_int32 * 32),
        ("cand_us_per_slice", ctypes.c_double * 32),
        ("trial_steps", ctypes.c_int64),
    ]


UPDATE_VARIANTS = {0: "k_update_iaf (one thread per neuron, 4 lags of inputs at a time)",
                   1: "k_update_iaf (one thread per neuron, 8 lags of inputs at a time)",
                   2: "k_update_iaf2 (two-phase, 32 neurons per 256-thread CTA)",
                   3: "k_update_iaf2 (two-phase, 32 neurons per 128-thread CTA)",
                   4: "k_update_aeif",
                   5: "k_run_slices (persistent: node update and delivery of many slices in one cooperative launch; "
                      "k_run_slices_mg for networks larger than one resident wave)",
                   6: "k_update_iaf (one thread per neuron, 2 lags of inputs at a time)"}
UPDATE_KERNELS = {0: "k_update_iaf", 1: "k_update_iaf", 2: "k_update_iaf2", 3: "k_update_iaf2", 4: "k_update_aeif",
                  5: "k_run_slices", 6: "k_update_iaf"}


def tuning_dict(t):
    n = t.n_candidates
    return {"mode": ["fixed", "auto"][t.mode] if t.mode in (0, 1) else t.mode,
            "state": ["pending", "tuned", "cached", "fixed"][t.state] if 0 <= t.state < 4 else t.state,
            "update_variant": t.update_variant, "update_kernel": UPDATE_KERNELS.get(t.update_variant, "?"),
            "update_variant_name": UPDATE_VARIANTS.get(t.update_variant, "?"),
            "deliver_ctas_per_sm": t.deliver_per_sm, "deliver_chunks_per_warp": t.deliver_group,
            "rate_bucket": t.rate_bucket, "trial_steps": t.trial_steps,
            "candidates": [{"update_variant": t.cand_variant[k], "deliver_ctas_per_sm": t.cand_per_sm[k],
                            "deliver_chunks_per_warp": t.cand_group[k], "us_per_slice": t.cand_us_per_slice[k]}
                           for k in range(n)]}


class Engine:
    """Thin owner of one ng_engine handle."""

    def __init__(self, blocks, h, min_delay, max_delay, n_generators=0, precision=NG_FP64, device=0,
                 tics_per_ms=1000.0, spike_log_capacity=0, start_step=0, serving=False, max_networks=0,
                 edge_capacity=0, max_abs_weight=0.0, ring32=False, ring_bound=0.0, tile_capacity=0):
        L = load()
        cfg = NGConfig()
        cfg.device = int(device)
        cfg.precision = int(precision)
        cfg.h = float(h)
        cfg.tics_per_ms = float(tics_per_ms)
        cfg.min_delay = int(min_delay)
        cfg.max_delay = int(max_delay)
        if len(blocks) > NG_MAX_BLOCKS:
            raise ValueError("too many model blocks")
        cfg.n_blocks = len(blocks)
        for k, (model, n) in enumerate(blocks):
            cfg.block_model[k] = int(model)
            cfg.block_size[k] = int(n)
        cfg.n_generators = int(n_generators)
        cfg.spike_log_capacity = int(spike_log_capacity)
        cfg.start_step = int(start_step)
        cfg.serving = 1 if serving else 0
        cfg.max_networks = int(max_networks)
        cfg.edge_capacity = int(edge_capacity)
        cfg.max_abs_weight = float(max_abs_weight)
        cfg.ring32 = 1 if ring32 else 0
        cfg.ring_bound = float(ring_bound)
        cfg.tile_capacity = int(tile_capacity)
        self.handle = ctypes.c_void_p()
        self.L = L
        check(L.ng_create(ctypes.byref(cfg), ctypes.byref(self.handle)))
        self.blocks = list(blocks)
        self.max_networks = int(max_networks)
        self.n_trace = 0
        self.n_trace_vars = 0

    def close(self):
        if getattr(self, "handle", None) and self.handle.value:
            self.L.ng_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_var(self, block, name, values, first=0):
        v = np.ascontiguousarray(values, dtype=np.float64).ravel()
        check(self.L.ng_set_var(self.handle, int(block), name.encode(), _p(v), int(first), len(v)))

    def get_var(self, block, name, first=0, count=None):
        if count is None:
            count = self.blocks[block][1] - first
        out = np.empty(int(count), dtype=np.float64)
        check(self.L.ng_get_var(self.handle, int(block), name.encode(), _p(out), int(first), int(count)))
        return out

    def set_connections(self, row_ptr, target, weight, delay_steps):
        row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int64)
        target = np.ascontiguousarray(target, dtype=np.int32)
        weight = np.ascontiguousarray(weight, dtype=np.float64)
        delay_steps = np.ascontiguousarray(delay_steps, dtype=np.int32)
        check(self.L.ng_set_connections(self.handle, len(row_ptr) - 1, _p(row_ptr), _p(target), _p(weight),
                                        _p(delay_steps)))

    def set_connections_coo(self, source, target, weight, delay_steps, n_src):
        source = np.ascontiguousarray(source, dtype=np.int32)
        target = np.ascontiguousarray(target, dtype=np.int32)
        weight = np.ascontiguousarray(weight, dtype=np.float64)
        delay_steps = np.ascontiguousarray(delay_steps, dtype=np.int32)
        check(self.L.ng_set_connections_coo(self.handle, int(n_src), len(source), _p(source), _p(target),
                                            _p(weight), _p(delay_steps)))

    def set_plastic(self, row_ptr, target, weight, delay_steps, lam=0.1, alpha=1.0, mu=0.4, tau_plus=20.0):
        """stdp_pl_synapse_hom connections as a CSR over neuron sources."""
        row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int64)
        target = np.ascontiguousarray(target, dtype=np.int32)
        weight = np.ascontiguousarray(weight, dtype=np.float64)
        delay_steps = np.ascontiguousarray(delay_steps, dtype=np.int32)
        check(self.L.ng_set_plastic_connections(self.handle, len(row_ptr) - 1, _p(row_ptr), _p(target), _p(weight),
                                                _p(delay_steps), float(lam), float(alpha), float(mu),
                                                float(tau_plus)))
        self._n_plastic = len(target)

    def plastic_weights(self):
        out = np.empty(getattr(self, "_n_plastic", 0), dtype=np.float64)
        check(self.L.ng_get_plastic_weights(self.handle, _p(out), len(out)))
        return out

    def set_spike_schedule(self, emit_step, source):
        emit_step = np.ascontiguousarray(emit_step, dtype=np.int64)
        source = np.ascontiguousarray(source, dtype=np.int32)
        check(self.L.ng_set_spike_schedule(self.handle, len(emit_step), _p(emit_step), _p(source)))

    def set_poisson(self, rate_hz, weight, delay_steps, start_step, stop_step, seed):
        r = np.ascontiguousarray(rate_hz, dtype=np.float64)
        w = np.ascontiguousarray(weight, dtype=np.float64)
        d = np.ascontiguousarray(delay_steps, dtype=np.int32)
        check(self.L.ng_set_poisson(self.handle, _p(r), _p(w), _p(d), int(start_step), int(stop_step),
                                    int(seed) & (2**64 - 1)))

    def set_recording(self, flags):
        f = np.ascontiguousarray(flags, dtype=np.uint8)
        check(self.L.ng_set_recording(self.handle, _p(f)))

    def set_trace(self, neurons, var_names, interval_steps):
        idx = np.ascontiguousarray(neurons, dtype=np.int32)
        names = [ctypes.c_char_p(v.encode()) for v in var_names]
        arr = (ctypes.c_char_p * max(1, len(names)))(*names)
        check(self.L.ng_set_trace(self.handle, len(idx), _p(idx), len(names), ctypes.cast(arr, ctypes.c_void_p),
                                  int(interval_steps)))
        self.n_trace = len(idx)
        self.n_trace_vars = len(names)

    def simulate(self, n_steps):
        check(self.L.ng_simulate(self.handle, int(n_steps)))

    def simulate_async(self, n_steps):
        """Enqueue n_steps; the last group still runs when this returns."""
        check(self.L.ng_simulate_async(self.handle, int(n_steps)))

    def update(self, origin, frm, to):
        """Steps [frm, to) of the slice at `origin` (Node::update), enqueued."""
        check(self.L.ng_update(self.handle, int(origin), int(frm), int(to)))

    def sync(self):
        check(self.L.ng_sync(self.handle))

    def spikes(self):
        n = ctypes.c_int64(0)
        check(self.L.ng_spike_count(self.handle, ctypes.byref(n)))
        src = np.empty(n.value, dtype=np.int32)
        st = np.empty(n.value, dtype=np.int64)
        got = ctypes.c_int64(0)
        check(self.L.ng_get_spikes(self.handle, _p(src), _p(st), n.value, ctypes.byref(got)))
        return src[:got.value], st[:got.value]

    def trace(self):
        """Drain trace rows: (first_stamp, array [rows, n_vars, n_neurons])."""
        rows = ctypes.c_int64(0)
        first = ctypes.c_int64(0)
        check(self.L.ng_trace_count(self.handle, ctypes.byref(rows), ctypes.byref(first)))
        width = max(1, self.n_trace * self.n_trace_vars)
        out = np.empty(rows.value * width, dtype=np.float64)
        got = ctypes.c_int64(0)
        check(self.L.ng_get_trace(self.handle, _p(out), rows.value, ctypes.byref(got)))
        return first.value, out[:got.value * width].reshape(got.value, max(1, self.n_trace_vars),
                                                            max(1, self.n_trace))

    def stats(self):
        s = NGStats()
        check(self.L.ng_get_stats(self.handle, ctypes.byref(s)))
        return {f: getattr(s, f) for f, _ in NGStats._fields_}

    def tuned(self):
        """The launch configuration the engine runs with (and, once the
        autotuner has run, what it measured)."""
        t = NGTuning()
        check(self.L.ng_get_tuning(self.handle, ctypes.byref(t)))
        return tuning_dict(t)

    def set_tuning(self, mode=1, update_variant=-1, deliver_ctas_per_sm=-1, deliver_chunks_per_warp=-1):
        """mode 1: autotune (process cache first), 2: autotune ignoring the
        cache, 0: fixed configuration (-1: the defaults)."""
        check(self.L.ng_set_tuning(self.handle, int(mode), int(update_variant), int(deliver_ctas_per_sm),
                                   int(deliver_chunks_per_warp)))

    def set_option(self, name, value):
        check(self.L.ng_set_option(self.handle, name.encode(), float(value)))

    def set_profiling(self, on):
        check(self.L.ng_set_profiling(self.handle, 1 if on else 0))

    def set_stream(self, stream_ptr):
        check(self.L.ng_set_stream(self.handle, ctypes.c_void_p(int(stream_ptr) if stream_ptr else 0)))

    def set_graph_slices(self, k):
        check(self.L.ng_set_graph_slices(self.handle, int(k)))

    def coefficients(self, block, index):
        out = np.empty(32, dtype=np.float64)
        n = ctypes.c_int32(0)
        check(self.L.ng_debug_coefficients(self.handle, int(block), int(index), _p(out), 32, ctypes.byref(n)))
        return out[:n.value]

    # ---- serving
    def _per_neuron(self, slot, value, n, dtype):
        """`value` as a contiguous array of n entries.  A scalar is written
        into a buffer kept per slot and reused by later admissions (the
        library copies the values before ng_net_add returns): a server
        admitting networks back to back then allocates, and first-touches,
        no host memory per admission."""
        v = np.asarray(value, dtype=dtype)
        if v.ndim > 0:
            return np.ascontiguousarray(np.broadcast_to(v, (n,)))
        bufs = self.__dict__.setdefault("_fill", {})
        buf = bufs.get(slot)
        if buf is None or buf.dtype != v.dtype or len(buf) < n:
            buf = np.empty(max(n, 2 * (0 if buf is None else len(buf))), dtype=dtype)
            bufs[slot] = buf
        out = buf[:n]
        out.fill(v)
        return out

    def net_add(self, n, steps, seed, var_values, build=None, edges=None, poisson=None, record=True):
        """Admit a network; returns its id, or None if it does not fit now.

        build: a dict of NGFixedIndegree fields, or an NGPairwiseBernoulli;
        edges: (source, target, weight, delay_steps) in network-local ids."""
        names = list(var_values)
        arrays = [self._per_neuron(("var", j), var_values[k], n, np.float64) for j, k in enumerate(names)]
        cnames = (ctypes.c_char_p * max(1, len(names)))(*[k.encode() for k in names])
        cvals = (ctypes.c_void_p * max(1, len(arrays)))(*[a.ctypes.data for a in arrays])
        desc = NGNetDesc(n=int(n), steps=int(steps), seed=int(seed) & (2**64 - 1), record=1 if record else 0,
                         n_vars=len(names), var_names=ctypes.cast(cnames, ctypes.c_void_p),
                         var_values=ctypes.cast(cvals, ctypes.c_void_p))
        keep = [arrays, cnames, cvals]
        if isinstance(build, NGPairwiseBernoulli):
            keep.append(build)
            desc.build_pb = ctypes.cast(ctypes.pointer(build), ctypes.c_void_p)
        elif build is not None:
            fb = NGFixedIndegree(**build)
            keep.append(fb)
            desc.build = ctypes.cast(ctypes.pointer(fb), ctypes.c_void_p)
        elif edges is not None:
            src, tgt, w, d = (np.ascontiguousarray(edges[0], dtype=np.int32), np.ascontiguousarray(edges[1], dtype=np.int32),
                              np.ascontiguousarray(edges[2], dtype=np.float64), np.ascontiguousarray(edges[3], dtype=np.int32))
            keep += [src, tgt, w, d]
            desc.nnz = len(src)
            desc.source, desc.target, desc.weight, desc.delay_steps = (src.ctypes.data, tgt.ctypes.data, w.ctypes.data,
                                                                      d.ctypes.data)
        if poisson is not None:
            r = self._per_neuron("rate", poisson[0], n, np.float64)
            pw = self._per_neuron("weight", poisson[1], n, np.float64)
            pd = self._per_neuron("delay", poisson[2], n, np.int32)
            keep += [r, pw, pd]
            desc.poisson_rate, desc.poisson_weight, desc.poisson_delay = r.ctypes.data, pw.ctypes.data, pd.ctypes.data
        nid = ctypes.c_int32(-1)
        rc = self.L.ng_net_add(self.handle, ctypes.byref(desc), ctypes.byref(nid))
        del keep
        if rc == NG_ERR_CAPACITY:
            return None
        check(rc)
        return nid.value

    def net_poll(self, nid):
        done = ctypes.c_int64(0)
        fin = ctypes.c_int32(0)
        check(self.L.ng_net_poll(self.handle, int(nid), ctypes.byref(done), ctypes.byref(fin)))
        return done.value, bool(fin.value)

    def net_spikes(self, nid):
        """Drain the network's spikes: (local source, local stamp)."""
        got = ctypes.c_int64(0)
        check(self.L.ng_net_spikes(self.handle, int(nid), None, None, 0, ctypes.byref(got)))
        k = got.value
        src = np.empty(k, dtype=np.int32)
        st = np.empty(k, dtype=np.int64)
        if k:
            check(self.L.ng_net_spikes(self.handle, int(nid), _p(src), _p(st), k, ctypes.byref(got)))
        return src[:got.value], st[:got.value]

    def net_get_var(self, nid, name, n):
        out = np.empty(int(n), dtype=np.float64)
        check(self.L.ng_net_get_var(self.handle, int(nid), name.encode(), _p(out)))
        return out

    def net_connection_count(self, nid):
        n = ctypes.c_int64(0)
        check(self.L.ng_net_get_connections(self.handle, int(nid), None, None, None, None, 0, ctypes.byref(n)))
        return n.value

    def net_get_connections(self, nid):
        """(source, target, weight, delay_steps) of the network, local ids."""
        n = ctypes.c_int64(0)
        check(self.L.ng_net_get_connections(self.handle, int(nid), None, None, None, None, 0, ctypes.byref(n)))
        k = n.value
        s = np.empty(k, dtype=np.int32)
        t = np.empty(k, dtype=np.int32)
        w = np.empty(k, dtype=np.float64)
        d = np.empty(k, dtype=np.int32)
        if k:
            check(self.L.ng_net_get_connections(self.handle, int(nid), _p(s), _p(t), _p(w), _p(d), k, ctypes.byref(n)))
        return s, t, w, d

    def net_remove(self, nid):
        check(self.L.ng_net_remove(self.handle, int(nid)))

    def net_capacity(self):
        a = ctypes.c_int64(0)
        b = ctypes.c_int64(0)
        check(self.L.ng_net_capacity(self.handle, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value
