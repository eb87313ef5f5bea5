"""nestgpu -- PyNEST-compatible front-end of the B200 slice engine.

A script written for the reference's PyNEST runs unchanged on the engine
for the models on its path (iaf_psc_delta, iaf_psc_exp, iaf_psc_alpha,
aeif_cond_alpha, static_synapse, stdp_pl_synapse_hom, poisson_generator,
spike_generator, spike_recorder, multimeter, voltmeter):

    import nestgpu as nest
    nest.ResetKernel()
    nest.resolution = 0.1
    pop = nest.Create("iaf_psc_delta", 1000, params={"I_e": 376.0})
    nest.Connect(pop, pop, {"rule": "fixed_indegree", "indegree": 100}, {"weight": 0.1, "delay": 1.5})
    sr = nest.Create("spike_recorder")
    nest.Connect(pop, sr)
    nest.Simulate(1000.0)
    sr.events["senders"], sr.events["times"]

The API mirrors pynest/nest/lib/hl_api_{nodes,connections,simulation,info,
types}.py.  Every Simulate runs on the GPU through libnestgpu.so (C ABI in
include/nestgpu.h); there is no CPU fallback.
"""

import sys
import types
from contextlib import contextmanager

import numpy as np

from . import _abi
from . import random  # noqa: F401  (nest.random)
from .connect import SynapseCollection, connect as _connect, get_connections as _get_connections
from .kernel import KERNEL, KernelException
from .models import DEVICE_MODELS, NEURON_MODELS, BadProperty
from .nodes import NodeCollection
from .random import math  # noqa: F401  (nest.math)

__version__ = "3.10.0-b200"

__all__ = ["ResetKernel", "Create", "Connect", "Simulate", "Run", "Prepare", "Cleanup", "RunManager", "GetStatus",
           "SetStatus", "GetConnections", "GetKernelStatus", "SetKernelStatus", "SetDefaults", "GetDefaults",
           "NodeCollection", "SynapseCollection", "Models", "CopyModel", "BadProperty", "KernelException", "set",
           "get",
           "random", "math", "engine_stats"]


def ResetKernel():
    """Reset the kernel: delete all nodes and connections, free the engine."""
    KERNEL.reset()


def Create(model, n=1, params=None, positions=None):
    if positions is not None:
        raise NotImplementedError("spatial networks are not on the engine's path")
    if isinstance(params, (list, tuple)) and len(params) != n:
        raise BadProperty("Create: list of parameter dictionaries must have n entries")
    ids = KERNEL.create(model, int(n), None)
    if params is not None:
        KERNEL.set_status(ids, params)
    return NodeCollection(ids)


def Connect(pre, post, conn_spec=None, syn_spec=None, return_synapsecollection=False):
    return _connect(pre, post, conn_spec, syn_spec, return_synapsecollection)


def Prepare():
    KERNEL.prepare()


def Run(t):
    KERNEL.run(float(t))


def Cleanup():
    KERNEL.cleanup()


def Simulate(t):
    """Simulate the network for t ms (Prepare; Run(t); Cleanup)."""
    KERNEL.simulate(float(t))


@contextmanager
def RunManager():
    Prepare()
    try:
        yield
    finally:
        Cleanup()


def GetConnections(source=None, target=None, synapse_model=None, synapse_label=None):
    return _get_connections(source, target, synapse_model, synapse_label)


def GetStatus(nodes, keys=None, output=""):
    if isinstance(nodes, SynapseCollection):
        r = nodes.get(keys, output=output)
        return r
    per = KERNEL.get_status(nodes.ids)
    if keys is None:
        return tuple(per)
    if isinstance(keys, str):
        return tuple(d[keys] for d in per)
    return tuple(tuple(d[k] for k in keys) for d in per)


def SetStatus(nodes, params, val=None):
    if isinstance(params, str):
        params = {params: val}
    if isinstance(nodes, SynapseCollection):
        nodes.set(params)
        return
    KERNEL.set_status(nodes.ids, params)


def _set_syn_defaults(model, params):
    d = KERNEL.syn_defaults[model]
    for k, v in params.items():
        if k not in d:
            raise BadProperty(f"Unaccessed dictionary entries for {model}: ['{k}']")
        if k == "tau_plus" and not float(v) > 0:
            raise BadProperty("tau_plus must be > 0.")
        if k == "weight" and KERNEL.syn_kind[model] == "stdp_pl" and float(v) < 0:
            raise BadProperty("Weight of stdp_pl_synapse_hom must be non-negative")
    for k, v in params.items():
        d[k] = float(v)
    if KERNEL.syn_kind[model] == "stdp_pl" and model in KERNEL.pl_models:
        KERNEL.structure_changed = True    # common properties of existing connections changed


def SetDefaults(model, params, val=None):
    if isinstance(params, str):
        params = {params: val}
    if model in KERNEL.syn_defaults:
        KERNEL.settle()
        _set_syn_defaults(model, params)
        return
    if model in KERNEL.models:
        KERNEL.models[model].set_defaults(params)
        return
    if model in KERNEL.model_defaults:
        KERNEL.model_defaults[model].update(params)
        return
    raise KernelException(f"Unknown model '{model}'")


def GetDefaults(model, keys=None):
    if model in KERNEL.syn_defaults:
        d = dict(KERNEL.syn_defaults[model])
        d["synapse_model"] = model
    elif model in KERNEL.models:
        d = KERNEL.models[model].get_defaults()
        d["model"] = model
    elif model in KERNEL.model_defaults:
        d = dict(KERNEL.model_defaults[model])
        d["model"] = model
    else:
        raise KernelException(f"Unknown model '{model}'")
    if keys is None:
        return d
    if isinstance(keys, str):
        return d[keys]
    return tuple(d[k] for k in keys)


def CopyModel(existing, new, params=None):
    """Copy a synapse model under a new name with changed defaults
    (hl_api_models.py CopyModel); copies of neuron and device models are not
    on the engine's path."""
    if new in KERNEL.syn_defaults or new in KERNEL.models or new in KERNEL.model_defaults:
        raise KernelException(f"NewModelNameExists: {new}")
    if existing not in KERNEL.syn_defaults:
        if existing in KERNEL.models or existing in KERNEL.model_defaults:
            raise NotImplementedError("CopyModel of neuron and device models is not on the engine's path")
        raise KernelException(f"UnknownSynapseType: {existing}")
    KERNEL.syn_defaults[new] = dict(KERNEL.syn_defaults[existing])
    KERNEL.syn_kind[new] = KERNEL.syn_kind[existing]
    if params:
        try:
            _set_syn_defaults(new, dict(params))
        except Exception:
            del KERNEL.syn_defaults[new], KERNEL.syn_kind[new]
            raise


def Models(mtype="all", sel=None):
    nodes = sorted(list(NEURON_MODELS) + list(DEVICE_MODELS))
    syn = sorted(KERNEL.syn_defaults)
    out = nodes if mtype == "nodes" else syn if mtype == "synapses" else nodes + syn
    return tuple(m for m in out if sel is None or sel in m)


_KERNEL_KEYS = ("resolution", "biological_time", "min_delay", "max_delay", "rng_seed", "local_num_threads",
                "num_connections", "network_size", "time_simulate", "local_spike_counter", "tics_per_ms",
                "tics_per_step", "ms_per_tic", "precision", "graph_slices", "device", "print_time",
                "total_num_virtual_procs", "rng_type", "engine")


def GetKernelStatus(keys=None):
    K = KERNEL
    K.settle()
    c = K.compiled if not K.structure_changed else None
    if c is None and len(K.node_kind):
        try:
            c = K.compile()
        except Exception:
            c = None
    md = c["min_delay"] if c else 1
    Md = c["max_delay"] if c else 1
    st = {
        "resolution": K.h,
        "biological_time": float(K.stamp_to_ms(K.clock)),
        "min_delay": md * K.ms_per_step,
        "max_delay": Md * K.ms_per_step,
        "rng_seed": K.rng_seed,
        "rng_type": "philox4x32",
        "local_num_threads": K.local_num_threads,
        "total_num_virtual_procs": K.local_num_threads,
        "num_connections": K.num_connections(),
        "network_size": len(K.node_kind),
        "time_simulate": K.time_simulate,
        "local_spike_counter": K.spike_count,
        "tics_per_ms": K.tics_per_ms,
        "tics_per_step": K.tics_per_step,
        "ms_per_tic": 1.0 / K.tics_per_ms,
        "precision": K.precision,
        "graph_slices": K.graph_slices,
        "device": K.device,
        "print_time": K.print_time,
        "engine": dict(K.stats),
    }
    if keys is None:
        return st
    if isinstance(keys, str):
        return st[keys]
    return tuple(st[k] for k in keys)


def SetKernelStatus(params):
    K = KERNEL
    K.settle()
    params = dict(params)
    if "tics_per_ms" in params:
        if len(K.node_kind):
            raise KernelException("Cannot change time representation after nodes have been created.")
        K.tics_per_ms = float(params.pop("tics_per_ms"))
    if "resolution" in params:
        K.set_resolution(float(params.pop("resolution")))
    if "min_delay" in params or "max_delay" in params:
        mn = params.pop("min_delay", None)
        mx = params.pop("max_delay", None)
        if mn is None or mx is None:
            raise BadProperty("min_delay and max_delay must be set together")
        K.user_min_delay = int(K.delay_ms_to_steps(mn))
        K.user_max_delay = int(K.delay_ms_to_steps(mx))
        if K.user_min_delay < 1 or K.user_max_delay < K.user_min_delay:
            raise BadProperty("need resolution <= min_delay <= max_delay")
        K.structure_changed = True
    if "rng_seed" in params:
        K.rng_seed = int(params.pop("rng_seed"))
        K._rng = None
        K.structure_changed = True
    if "precision" in params:
        p = str(params.pop("precision"))
        if p not in ("fp64", "fp32"):
            raise BadProperty("precision must be 'fp64' or 'fp32'")
        K.precision = p
        K.structure_changed = True
    for k in ("local_num_threads", "total_num_virtual_procs"):
        if k in params:
            K.local_num_threads = int(params.pop(k))
    if "graph_slices" in params:
        K.graph_slices = int(params.pop("graph_slices"))
        K.structure_changed = True
    if "device" in params:
        K.device = int(params.pop("device"))
        K.structure_changed = True
    if "print_time" in params:
        K.print_time = bool(params.pop("print_time"))
    for k in ("rng_type", "overwrite_files", "data_path", "data_prefix", "dict_miss_is_error"):
        params.pop(k, None)
    if params:
        raise BadProperty(f"Unaccessed kernel status entries: {sorted(params)}")


def set(**kwargs):  # noqa: A001  (nest.set)
    SetKernelStatus(kwargs)


def get(*keys):
    if len(keys) == 0:
        return GetKernelStatus()
    if len(keys) == 1:
        return GetKernelStatus(keys[0])
    return GetKernelStatus(list(keys))


def set_verbosity(level):
    pass


def engine_stats():
    """Counters of the last run: spikes, synaptic events, drive events, timings."""
    KERNEL.settle()
    return dict(KERNEL.stats)


def engine_available():
    """True if libnestgpu.so loads and a CUDA device is visible."""
    try:
        return _abi.device_count() > 0
    except Exception:
        return False


class _KernelModule(types.ModuleType):
    """Module attributes as kernel properties: ``nest.resolution = 0.1``."""

    def __getattr__(self, name):
        if name in _KERNEL_KEYS:
            return GetKernelStatus(name)
        raise AttributeError(name)

    def __setattr__(self, name, value):
        if name in _KERNEL_KEYS:
            SetKernelStatus({name: value})
        else:
            super().__setattr__(name, value)


sys.modules[__name__].__class__ = _KernelModule
