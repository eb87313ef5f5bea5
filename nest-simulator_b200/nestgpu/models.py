"""Neuron and device models of the min_delay-slice path.

Each neuron model keeps its parameters and state in the reference's internal
representation, as numpy FP64 arrays over all nodes of the model, and applies
``set`` exactly as the reference's ``Parameters_::set`` / ``State_::set``
do (the iaf models hold V_m, V_th, V_reset and V_min relative to E_L and
shift them when E_L changes):

- iaf_psc_delta: models/iaf_psc_delta.cpp:94-200
- iaf_psc_exp:   models/iaf_psc_exp.cpp:100-195
- iaf_psc_alpha: models/iaf_psc_alpha.cpp (Parameters_::set, State_::set)
- aeif_cond_alpha: models/aeif_cond_alpha.cpp:130-300
"""

import numpy as np

from . import _abi

DBL_MAX = np.finfo(np.float64).max


class BadProperty(ValueError):
    """A parameter value the model rejects (the reference's BadProperty)."""


def _as(v, n):
    a = np.asarray(v, dtype=np.float64)
    if a.ndim == 0:
        return np.full(n, float(a))
    if len(a) != n:
        raise BadProperty(f"expected {n} values, got {len(a)}")
    return a.astype(np.float64)


class NeuronModel:
    """Storage and NEST set/get semantics of one neuron model."""

    name = ""
    engine_model = 0
    # internal storage variables and their defaults
    storage = {}
    # internal -> engine variable name
    engine_vars = {}
    # internal vars that are engine state (pushed as state) -- others are parameters
    state_vars = ()
    recordables = ()
    public = ()

    def __init__(self):
        self.data = {k: np.zeros(0) for k in self.storage}
        self.defaults = dict(self.storage)
        self.n = 0
        self.dirty = set(self.storage)

    def grow(self, n):
        for k in self.storage:
            self.data[k] = np.concatenate([self.data[k], np.full(n, self.defaults[k], dtype=np.float64)])
        first = self.n
        self.n += n
        self.dirty |= set(self.storage)
        return first

    def set_defaults(self, d):
        tmp = type(self)()
        tmp.grow(1)
        for k in self.storage:
            tmp.data[k][0] = self.defaults[k]
        tmp.set(np.array([0]), d)
        for k in self.storage:
            self.defaults[k] = float(tmp.data[k][0])

    def get_defaults(self):
        tmp = type(self)()
        tmp.grow(1)
        for k in self.storage:
            tmp.data[k][0] = self.defaults[k]
        return {k: tmp.get(np.array([0]), k)[0] for k in self.public}

    def set(self, idx, d):  # pragma: no cover - overridden
        raise NotImplementedError

    def get(self, idx, key):  # pragma: no cover - overridden
        raise NotImplementedError

    def recordable_value(self, key, engine_values, idx):
        """Public value of a recordable from the engine's internal value."""
        return engine_values

    def _touch(self, *keys):
        self.dirty |= set(keys)


class IafPscDelta(NeuronModel):
    name = "iaf_psc_delta"
    engine_model = _abi.NG_IAF_PSC_DELTA
    storage = {"tau_m": 10.0, "C_m": 250.0, "t_ref": 2.0, "E_L": -70.0, "I_e": 0.0,
               "V_th_rel": -55.0 - (-70.0), "V_reset_rel": -70.0 - (-70.0), "V_min_rel": -DBL_MAX,
               "V_m_rel": 0.0, "refractory_input": 0.0}
    engine_vars = {"tau_m": "tau_m", "C_m": "C_m", "t_ref": "t_ref", "V_th_rel": "V_th_rel",
                   "V_reset_rel": "V_reset_rel", "V_min_rel": "V_min_rel", "V_m_rel": "V_m_rel", "I_e": "I_e"}
    state_vars = ("V_m_rel",)
    recordables = ("V_m",)
    public = ("C_m", "E_L", "I_e", "V_m", "V_min", "V_reset", "V_th", "t_ref", "tau_m", "refractory_input")

    def set(self, idx, d):
        D = self.data
        n = len(idx)
        d = dict(d)
        if "refractory_input" in d and bool(np.any(np.asarray(d["refractory_input"]))):
            raise NotImplementedError("refractory_input=True is not on the engine's path")
        EL_old = D["E_L"][idx].copy()
        EL = _as(d["E_L"], n) if "E_L" in d else EL_old
        dEL = EL - EL_old
        Vreset = _as(d["V_reset"], n) - EL if "V_reset" in d else D["V_reset_rel"][idx] - dEL
        Vth = _as(d["V_th"], n) - EL if "V_th" in d else D["V_th_rel"][idx] - dEL
        Vmin = _as(d["V_min"], n) - EL if "V_min" in d else D["V_min_rel"][idx] - dEL
        I_e = _as(d["I_e"], n) if "I_e" in d else D["I_e"][idx]
        C_m = _as(d["C_m"], n) if "C_m" in d else D["C_m"][idx]
        tau_m = _as(d["tau_m"], n) if "tau_m" in d else D["tau_m"][idx]
        t_ref = _as(d["t_ref"], n) if "t_ref" in d else D["t_ref"][idx]
        if np.any(Vreset >= Vth):
            raise BadProperty("Reset potential must be smaller than threshold.")
        if np.any(C_m <= 0):
            raise BadProperty("Capacitance must be >0.")
        if np.any(t_ref < 0):
            raise BadProperty("Refractory time must not be negative.")
        if np.any(tau_m <= 0):
            raise BadProperty("Membrane time constant must be > 0.")
        V = _as(d["V_m"], n) - EL if "V_m" in d else D["V_m_rel"][idx] - dEL
        D["E_L"][idx] = EL
        D["V_reset_rel"][idx] = Vreset
        D["V_th_rel"][idx] = Vth
        D["V_min_rel"][idx] = Vmin
        D["I_e"][idx] = I_e
        D["C_m"][idx] = C_m
        D["tau_m"][idx] = tau_m
        D["t_ref"][idx] = t_ref
        D["V_m_rel"][idx] = V
        self._touch("E_L", "V_reset_rel", "V_th_rel", "V_min_rel", "I_e", "C_m", "tau_m", "t_ref", "V_m_rel")

    def get(self, idx, key):
        D = self.data
        if key in ("V_m", "V_th", "V_reset", "V_min"):
            return D[key + "_rel"][idx] + D["E_L"][idx]
        if key == "refractory_input":
            return D[key][idx].astype(bool)
        return D[key][idx]

    def recordable_value(self, key, v, idx):
        return v + self.data["E_L"][idx]


class IafPscExp(NeuronModel):
    name = "iaf_psc_exp"
    engine_model = _abi.NG_IAF_PSC_EXP
    storage = {"tau_m": 10.0, "C_m": 250.0, "t_ref": 2.0, "E_L": -70.0, "I_e": 0.0,
               "V_th_rel": -55.0 - (-70.0), "V_reset_rel": -70.0 - (-70.0), "tau_syn_ex": 2.0,
               "tau_syn_in": 2.0, "rho": 0.01, "delta": 0.0, "V_m_rel": 0.0}
    engine_vars = {"tau_m": "tau_m", "C_m": "C_m", "t_ref": "t_ref", "V_th_rel": "V_th_rel",
                   "V_reset_rel": "V_reset_rel", "tau_syn_ex": "tau_syn_ex", "tau_syn_in": "tau_syn_in",
                   "V_m_rel": "V_m_rel", "I_e": "I_e"}
    state_vars = ("V_m_rel",)
    recordables = ("I_syn_ex", "I_syn_in", "V_m")
    public = ("C_m", "E_L", "I_e", "V_m", "V_reset", "V_th", "delta", "rho", "t_ref", "tau_m", "tau_syn_ex",
              "tau_syn_in")

    def set(self, idx, d):
        D = self.data
        n = len(idx)
        EL_old = D["E_L"][idx].copy()
        EL = _as(d["E_L"], n) if "E_L" in d else EL_old
        dEL = EL - EL_old
        Vreset = _as(d["V_reset"], n) - EL if "V_reset" in d else D["V_reset_rel"][idx] - dEL
        Vth = _as(d["V_th"], n) - EL if "V_th" in d else D["V_th_rel"][idx] - dEL
        vals = {}
        for k in ("I_e", "C_m", "tau_m", "tau_syn_ex", "tau_syn_in", "t_ref", "rho", "delta"):
            vals[k] = _as(d[k], n) if k in d else D[k][idx]
        if np.any(Vreset >= Vth):
            raise BadProperty("Reset potential must be smaller than threshold.")
        if np.any(vals["C_m"] <= 0):
            raise BadProperty("Capacitance must be strictly positive.")
        if np.any(vals["tau_m"] <= 0) or np.any(vals["tau_syn_ex"] <= 0) or np.any(vals["tau_syn_in"] <= 0):
            raise BadProperty("Membrane and synapse time constant(s) must be strictly positive.")
        if np.any(vals["t_ref"] < 0):
            raise BadProperty("Refractory time must not be negative.")
        if np.any(vals["rho"] < 0):
            raise BadProperty("Stochastic firing intensity must not be negative.")
        if np.any(vals["delta"] < 0):
            raise BadProperty("Width of threshold region must not be negative.")
        if np.any(vals["delta"] > 1e-10):
            raise NotImplementedError("the stochastic threshold (delta > 0) is not on the engine's path")
        V = _as(d["V_m"], n) - EL if "V_m" in d else D["V_m_rel"][idx] - dEL
        D["E_L"][idx] = EL
        D["V_reset_rel"][idx] = Vreset
        D["V_th_rel"][idx] = Vth
        for k, v in vals.items():
            D[k][idx] = v
        D["V_m_rel"][idx] = V
        self._touch(*self.storage)

    def get(self, idx, key):
        D = self.data
        if key in ("V_m", "V_th", "V_reset"):
            return D[key + "_rel"][idx] + D["E_L"][idx]
        return D[key][idx]

    def recordable_value(self, key, v, idx):
        return v + self.data["E_L"][idx] if key == "V_m" else v


class IafPscAlpha(NeuronModel):
    """iaf_psc_alpha: alpha-shaped synaptic currents (I_syn and its
    derivative per channel); V_m, V_th, V_reset, V_min relative to E_L."""
    name = "iaf_psc_alpha"
    engine_model = _abi.NG_IAF_PSC_ALPHA
    storage = {"tau_m": 10.0, "C_m": 250.0, "t_ref": 2.0, "E_L": -70.0, "I_e": 0.0,
               "V_th_rel": -55.0 - (-70.0), "V_reset_rel": -70.0 - (-70.0), "tau_syn_ex": 2.0,
               "tau_syn_in": 2.0, "V_min_rel": -np.inf, "V_m_rel": 0.0, "I_syn_ex": 0.0, "I_syn_in": 0.0,
               "dI_syn_ex": 0.0, "dI_syn_in": 0.0}
    engine_vars = {"tau_m": "tau_m", "C_m": "C_m", "t_ref": "t_ref", "V_th_rel": "V_th_rel",
                   "V_reset_rel": "V_reset_rel", "tau_syn_ex": "tau_syn_ex", "tau_syn_in": "tau_syn_in",
                   "V_min_rel": "V_min_rel", "V_m_rel": "V_m_rel", "I_syn_ex": "I_syn_ex", "I_syn_in": "I_syn_in",
                   "dI_syn_ex": "dI_syn_ex", "dI_syn_in": "dI_syn_in", "I_e": "I_e"}
    state_vars = ("V_m_rel", "I_syn_ex", "I_syn_in", "dI_syn_ex", "dI_syn_in")
    recordables = ("I_syn_ex", "I_syn_in", "V_m")
    public = ("C_m", "E_L", "I_e", "V_m", "V_min", "V_reset", "V_th", "t_ref", "tau_m", "tau_syn_ex", "tau_syn_in",
              "I_syn_ex", "I_syn_in", "dI_syn_ex", "dI_syn_in")

    def set(self, idx, d):
        D = self.data
        n = len(idx)
        EL_old = D["E_L"][idx].copy()
        EL = _as(d["E_L"], n) if "E_L" in d else EL_old
        dEL = EL - EL_old
        Vreset = _as(d["V_reset"], n) - EL if "V_reset" in d else D["V_reset_rel"][idx] - dEL
        Vth = _as(d["V_th"], n) - EL if "V_th" in d else D["V_th_rel"][idx] - dEL
        Vmin = _as(d["V_min"], n) - EL if "V_min" in d else D["V_min_rel"][idx] - dEL
        vals = {}
        for k in ("I_e", "C_m", "tau_m", "tau_syn_ex", "tau_syn_in", "t_ref", "I_syn_ex", "I_syn_in", "dI_syn_ex",
                  "dI_syn_in"):
            vals[k] = _as(d[k], n) if k in d else D[k][idx]
        if np.any(Vreset >= Vth):
            raise BadProperty("Reset potential must be smaller than threshold.")
        if np.any(vals["C_m"] <= 0):
            raise BadProperty("Capacitance must be > 0.")
        if np.any(vals["tau_m"] <= 0):
            raise BadProperty("Membrane time constant must be > 0.")
        if np.any(vals["tau_syn_ex"] <= 0) or np.any(vals["tau_syn_in"] <= 0):
            raise BadProperty("All synaptic time constants must be > 0.")
        if np.any(vals["t_ref"] < 0):
            raise BadProperty("Refractory time must not be negative.")
        V = _as(d["V_m"], n) - EL if "V_m" in d else D["V_m_rel"][idx] - dEL
        D["E_L"][idx] = EL
        D["V_reset_rel"][idx] = Vreset
        D["V_th_rel"][idx] = Vth
        D["V_min_rel"][idx] = Vmin
        for k, v in vals.items():
            D[k][idx] = v
        D["V_m_rel"][idx] = V
        self._touch(*self.storage)

    def get(self, idx, key):
        D = self.data
        if key in ("V_m", "V_th", "V_reset", "V_min"):
            return D[key + "_rel"][idx] + D["E_L"][idx]
        return D[key][idx]

    def recordable_value(self, key, v, idx):
        return v + self.data["E_L"][idx] if key == "V_m" else v


class AeifCondAlpha(NeuronModel):
    name = "aeif_cond_alpha"
    engine_model = _abi.NG_AEIF_COND_ALPHA
    storage = {"V_peak": 0.0, "V_reset": -60.0, "t_ref": 0.0, "g_L": 30.0, "C_m": 281.0, "E_ex": 0.0,
               "E_in": -85.0, "E_L": -70.6, "Delta_T": 2.0, "tau_w": 144.0, "a": 4.0, "b": 80.5, "V_th": -50.4,
               "tau_syn_ex": 0.2, "tau_syn_in": 2.0, "I_e": 0.0, "gsl_error_tol": 1e-6,
               "V_m": -70.6, "g_ex": 0.0, "dg_ex": 0.0, "g_in": 0.0, "dg_in": 0.0, "w": 0.0}
    engine_vars = {k: k for k in storage}
    state_vars = ("V_m", "g_ex", "dg_ex", "g_in", "dg_in", "w")
    recordables = ("V_m", "g_ex", "g_in", "w")
    public = tuple(storage)

    def set(self, idx, d):
        D = self.data
        n = len(idx)
        new = {k: (_as(d[k], n) if k in d else D[k][idx]) for k in self.storage}
        if np.any(new["V_reset"] >= new["V_peak"]):
            raise BadProperty("Ensure that: V_reset < V_peak .")
        if np.any(new["Delta_T"] < 0.0):
            raise BadProperty("Delta_T must be positive.")
        pos = new["Delta_T"] > 0.0
        if np.any(pos):
            max_exp_arg = np.log(DBL_MAX / 1e20)
            if np.any((new["V_peak"][pos] - new["V_th"][pos]) / new["Delta_T"][pos] >= max_exp_arg):
                raise BadProperty("The current combination of V_peak, V_th and Delta_T will lead to numerical "
                                  "overflow at spike time.")
        if np.any(new["V_peak"] < new["V_th"]):
            raise BadProperty("V_peak >= V_th required.")
        if np.any(new["C_m"] <= 0):
            raise BadProperty("Capacitance must be strictly positive.")
        if np.any(new["t_ref"] < 0):
            raise BadProperty("Refractory time cannot be negative.")
        if np.any(new["tau_syn_ex"] <= 0) or np.any(new["tau_syn_in"] <= 0) or np.any(new["tau_w"] <= 0):
            raise BadProperty("All time constants must be strictly positive.")
        if np.any(new["gsl_error_tol"] <= 0.0):
            raise BadProperty("The gsl_error_tol must be strictly positive.")
        if np.any(new["g_ex"] < 0) or np.any(new["g_in"] < 0):
            raise BadProperty("Conductances must not be negative.")
        for k, v in new.items():
            D[k][idx] = v
        self._touch(*[k for k in self.storage if k in d])

    def get(self, idx, key):
        return self.data[key][idx]


def _archiving(cls):
    """Give an iaf model ArchivingNode's tau_minus (nestkernel/archiving_node.cpp:232-245):
    the time constant of the postsynaptic trace that STDP connections onto the
    neuron read (default 20 ms; every value must be > 0)."""
    model_set = cls.set

    def set(self, idx, d):
        tm = None
        if "tau_minus" in d:
            d = dict(d)
            tm = _as(d.pop("tau_minus"), len(idx))
            if np.any(tm <= 0):
                raise BadProperty("All time constants must be strictly positive.")
        model_set(self, idx, d)
        if tm is not None:
            self.data["tau_minus"][idx] = tm
            self._touch("tau_minus")

    cls.set = set
    cls.storage = dict(cls.storage, tau_minus=20.0)
    cls.engine_vars = dict(cls.engine_vars, tau_minus="tau_minus")
    cls.public = tuple(sorted(cls.public + ("tau_minus",)))


for _m in (IafPscDelta, IafPscExp, IafPscAlpha):
    _archiving(_m)

NEURON_MODELS = {"iaf_psc_delta": IafPscDelta, "iaf_psc_exp": IafPscExp, "iaf_psc_alpha": IafPscAlpha,
                 "aeif_cond_alpha": AeifCondAlpha}

#: device models and their parameter defaults
DEVICE_MODELS = {
    "spike_recorder": {"start": 0.0, "stop": np.inf, "origin": 0.0, "record_to": "memory", "time_in_steps": False,
                       "label": ""},
    "poisson_generator": {"rate": 0.0, "start": 0.0, "stop": np.inf, "origin": 0.0},
    "spike_generator": {"spike_times": [], "start": 0.0, "stop": np.inf, "origin": 0.0, "precise_times": False,
                        "allow_offgrid_times": False, "shift_now_spikes": False, "spike_weights": [],
                        "spike_multiplicities": []},
    "multimeter": {"interval": 1.0, "offset": 0.0, "record_from": [], "start": 0.0, "stop": np.inf, "origin": 0.0,
                   "record_to": "memory", "label": ""},
    "voltmeter": {"interval": 1.0, "offset": 0.0, "record_from": ["V_m"], "start": 0.0, "stop": np.inf,
                  "origin": 0.0, "record_to": "memory", "label": ""},
}

RECORDERS = ("spike_recorder",)
SAMPLERS = ("multimeter", "voltmeter")
GENERATORS = ("poisson_generator", "spike_generator")
