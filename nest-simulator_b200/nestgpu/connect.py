"""Connect and GetConnections (mirrors pynest/nest/lib/hl_api_connections.py
and the connection rules of nestkernel/conn_builder.cpp).

The rules draw from a numpy Philox stream seeded by rng_seed, so a network
built here has the reference's connection statistics but not its exact
edges.  To run the reference's exact graph, export it with the reference's
``GetConnections`` and connect the arrays with ``one_to_one`` (the
connect-arrays path of ``nest.Connect``).
"""

import numpy as np

from .kernel import KERNEL, STDP_COMMON, KernelException
from .models import BadProperty
from .nodes import NodeCollection
from .random import Parameter

RULES = ("one_to_one", "all_to_all", "fixed_indegree", "fixed_outdegree", "fixed_total_number",
         "pairwise_bernoulli")


def _ids(x):
    if isinstance(x, NodeCollection):
        return x.ids
    return np.asarray(x, dtype=np.int64).ravel()


def _values(v, n, rng, shape_ok=None):
    if isinstance(v, Parameter):
        return v.sample(rng, n)
    a = np.asarray(v, dtype=np.float64)
    if a.ndim == 0:
        return np.full(n, float(a))
    a = a.ravel()
    if len(a) != n:
        raise BadProperty(f"syn_spec array has {len(a)} entries, the rule makes {n} connections")
    return a


def _unique_rows(rows, n_choices, exclude, rng, allow_multapses, allow_autapses):
    """Redraw entries of `rows` (int array [m, k], indices into choices) that
    are autapses (== exclude[row]) or repeated within their row."""
    m, k = rows.shape
    for _ in range(10000):
        bad = np.zeros(rows.shape, dtype=bool)
        if not allow_autapses and exclude is not None:
            bad |= rows == exclude[:, None]
        if not allow_multapses and k > 1:
            order = np.argsort(rows, axis=1, kind="stable")
            srt = np.take_along_axis(rows, order, axis=1)
            dup = np.zeros_like(bad)
            dup[:, 1:] = srt[:, 1:] == srt[:, :-1]
            bad_sorted = np.zeros_like(bad)
            np.put_along_axis(bad_sorted, order, dup, axis=1)
            bad |= bad_sorted
        nb = int(bad.sum())
        if nb == 0:
            return rows
        rows[bad] = rng.integers(0, n_choices, nb)
    raise KernelException("could not draw connections without autapses/multapses")


def connect(pre, post, conn_spec=None, syn_spec=None, return_synapsecollection=False):
    K = KERNEL
    rng = K.rng()
    arrays = not isinstance(pre, NodeCollection) or not isinstance(post, NodeCollection)
    spre, spost = _ids(pre), _ids(post)
    if conn_spec is None:
        conn_spec = {"rule": "all_to_all"}
    if isinstance(conn_spec, str):
        conn_spec = {"rule": conn_spec}
    conn_spec = dict(conn_spec)
    rule = conn_spec.pop("rule", "all_to_all")
    if rule not in RULES:
        raise BadProperty(f"Unknown connection rule '{rule}'")
    if arrays and rule != "one_to_one":
        raise BadProperty("When connecting two arrays of node IDs, the rule must be one_to_one")
    if syn_spec is None:
        syn_spec = {}
    if isinstance(syn_spec, str):
        syn_spec = {"synapse_model": syn_spec}
    syn_spec = dict(syn_spec)
    model = syn_spec.pop("synapse_model", "static_synapse")
    if model not in K.syn_defaults:
        raise BadProperty(f"synapse model '{model}' is not on the engine's path (static_synapse and "
                          "stdp_pl_synapse_hom and their copies)")
    defaults = K.syn_defaults[model]
    plastic = K.syn_kind[model] == "stdp_pl"
    common = [k for k in STDP_COMMON if k in syn_spec]
    if plastic and common:
        # stdp_pl_synapse_hom's STDPPLHomCommonProperties are per model
        raise BadProperty(f"{common} are common properties of {model}: set them with SetDefaults or CopyModel")
    allow_autapses = bool(conn_spec.pop("allow_autapses", True))
    allow_multapses = bool(conn_spec.pop("allow_multapses", True))
    npre, npost = len(spre), len(spost)

    if rule == "one_to_one":
        if npre != npost:
            raise BadProperty("one_to_one connect requires sources and targets of equal size")
        s, t = spre, spost
        if not allow_autapses:
            keep = s != t
            s, t = s[keep], t[keep]
    elif rule == "all_to_all":
        # target-major, like the reference's AllToAllBuilder
        t = np.repeat(spost, npre)
        s = np.tile(spre, npost)
        if not allow_autapses:
            keep = s != t
            s, t = s[keep], t[keep]
    elif rule == "fixed_indegree":
        k = int(conn_spec.pop("indegree"))
        if not allow_multapses and k > npre:
            raise BadProperty("indegree cannot be larger than the number of sources without multapses")
        pos = {int(v): i for i, v in enumerate(spre)}
        exclude = np.array([pos.get(int(v), -1) for v in spost], dtype=np.int64)
        rows = rng.integers(0, npre, (npost, k))
        rows = _unique_rows(rows, npre, exclude, rng, allow_multapses, allow_autapses)
        s = spre[rows].ravel()
        t = np.repeat(spost, k)
    elif rule == "fixed_outdegree":
        k = int(conn_spec.pop("outdegree"))
        if not allow_multapses and k > npost:
            raise BadProperty("outdegree cannot be larger than the number of targets without multapses")
        pos = {int(v): i for i, v in enumerate(spost)}
        exclude = np.array([pos.get(int(v), -1) for v in spre], dtype=np.int64)
        rows = rng.integers(0, npost, (npre, k))
        rows = _unique_rows(rows, npost, exclude, rng, allow_multapses, allow_autapses)
        t = spost[rows].ravel()
        s = np.repeat(spre, k)
    elif rule == "fixed_total_number":
        n = int(conn_spec.pop("N"))
        s = spre[rng.integers(0, npre, n)]
        t = spost[rng.integers(0, npost, n)]
        if not allow_autapses:
            bad = s == t
            while np.any(bad):
                s[bad] = spre[rng.integers(0, npre, int(bad.sum()))]
                bad = s == t
    else:  # pairwise_bernoulli: geometric skipping over the source x target grid
        p = float(conn_spec.pop("p"))
        if not (0.0 <= p <= 1.0):
            raise BadProperty("Connection probability 0 <= p <= 1 required.")
        total = npre * npost
        if p == 0.0 or total == 0:
            flat = np.zeros(0, dtype=np.int64)
        elif p == 1.0:
            flat = np.arange(total, dtype=np.int64)
        else:
            parts, pos_ = [], -1
            chunk = max(1024, int(p * total * 1.05) + 1024)
            while True:
                gaps = rng.geometric(p, chunk).astype(np.int64)
                idx = pos_ + np.cumsum(gaps)
                inside = idx < total
                parts.append(idx[inside])
                if not np.all(inside):
                    break
                pos_ = int(idx[-1])
            flat = np.concatenate(parts)
        s = spre[flat // npost]
        t = spost[flat % npost]
        if not allow_autapses:
            keep = s != t
            s, t = s[keep], t[keep]
    if conn_spec:
        raise BadProperty(f"Unaccessed conn_spec entries: {sorted(conn_spec)}")
    n = len(s)
    w = syn_spec.pop("weight", defaults["weight"])
    d = syn_spec.pop("delay", defaults["delay"])
    if syn_spec:
        raise BadProperty(f"Unaccessed syn_spec entries: {sorted(syn_spec)}")
    if rule == "all_to_all" and not isinstance(w, Parameter) and np.ndim(w) == 2:
        w = np.asarray(w, dtype=np.float64).ravel()
    if rule == "all_to_all" and not isinstance(d, Parameter) and np.ndim(d) == 2:
        d = np.asarray(d, dtype=np.float64).ravel()
    wv = _values(w, n, rng)
    dv = _values(d, n, rng)
    if plastic:
        K.add_plastic_edges(s, t, wv, dv, model)
    else:
        K.add_edges(s, t, wv, dv)
    if return_synapsecollection:
        return get_connections(NodeCollection(np.unique(s)), NodeCollection(np.unique(t)), model)
    return None


class SynapseCollection:
    """Connections selected by GetConnections: indices into the kernel's
    static edge table and into its plastic (stdp_pl_synapse_hom) table, each
    sorted by source then target."""

    def __init__(self, idx, pidx=None):
        self._idx = np.asarray(idx, dtype=np.int64)
        self._pidx = np.zeros(0, dtype=np.int64) if pidx is None else np.asarray(pidx, dtype=np.int64)

    def __len__(self):
        return len(self._idx) + len(self._pidx)

    def _col(self, key):
        i, j = self._idx, self._pidx
        src, tgt, w, d = KERNEL.edges()
        if len(j):
            ps, pt, pw, pd, pm = KERNEL.plastic_edges()
        else:
            ps = pt = pd = np.zeros(0, dtype=np.int32)
            pw, pm = np.zeros(0), np.zeros(0, dtype=np.int16)
        if key == "source":
            return np.concatenate([src[i], ps[j]]).astype(np.int64)
        if key == "target":
            return np.concatenate([tgt[i], pt[j]]).astype(np.int64)
        if key == "weight":
            return np.concatenate([w[i], pw[j]])
        if key == "delay":
            return np.concatenate([d[i], pd[j]]).astype(np.int64) * KERNEL.ms_per_step
        if key == "synapse_model":
            names = np.array(KERNEL.pl_models or [""], dtype=object)
            return np.concatenate([np.array(["static_synapse"] * len(i), dtype=object), names[pm[j]]])
        if key in ("receptor", "port", "target_thread", "synapse_id"):
            return np.zeros(len(self), dtype=np.int64)
        if key in STDP_COMMON and len(i) == 0:
            names = [KERNEL.pl_models[k] for k in pm[j]]
            return np.array([KERNEL.syn_defaults[m][key] for m in names], dtype=np.float64)
        raise KeyError(key)

    def get(self, keys=None, output=""):
        if keys is None:
            keys = ["delay", "port", "receptor", "source", "synapse_id", "synapse_model", "target",
                    "target_thread", "weight"]
        single = isinstance(keys, str)
        ks = [keys] if single else list(keys)
        cols = {k: self._col(k) for k in ks}
        if output == "pandas":
            import pandas as pd

            return pd.DataFrame(cols)
        if single:
            c = cols[keys]
            return c.tolist()[0] if len(c) == 1 else c.tolist()
        return {k: (v.tolist()[0] if len(v) == 1 else v.tolist()) for k, v in cols.items()}

    def set(self, params=None, **kw):
        params = dict(params or {}, **kw)
        ni = len(self._idx)
        src, tgt, w, d = KERNEL.edges()
        if len(self._pidx):
            _, _, pw, pd, _ = KERNEL.plastic_edges()
        for k, v in params.items():
            vals = np.broadcast_to(np.asarray(v, dtype=np.float64), (len(self),))
            if k == "weight":
                if len(self._pidx) and np.any(vals[ni:] < 0):
                    raise BadProperty("Weight of stdp_pl_synapse_hom must be non-negative")
                w[self._idx] = vals[:ni]
                if len(self._pidx):
                    pw[self._pidx] = vals[ni:]
            elif k == "delay":
                steps = KERNEL.delay_ms_to_steps(vals)
                if np.any(steps < 1):
                    raise BadProperty("Delay must be greater than or equal to resolution")
                d[self._idx] = steps[:ni]
                if len(self._pidx):
                    pd[self._pidx] = steps[ni:]
            elif k in STDP_COMMON:
                raise BadProperty(f"'{k}' is a common property of stdp_pl_synapse_hom: set it with SetDefaults")
            else:
                raise BadProperty(f"cannot set '{k}' on these connections")
        # the engine is rebuilt at the next run (the plastic traces start over)
        KERNEL.structure_changed = True

    def __getattr__(self, name):
        if name.startswith("_"):
            raise AttributeError(name)
        return self.get(name)

    @property
    def source(self):
        return self.get("source")

    @property
    def target(self):
        return self.get("target")


def get_connections(source=None, target=None, synapse_model=None, synapse_label=None):
    """Static connections are reported as static_synapse; the plastic ones
    under the synapse model they were made with."""
    kind = None if synapse_model is None else KERNEL.syn_kind.get(synapse_model)
    s = None if source is None else _ids(source)
    t = None if target is None else _ids(target)
    idx = KERNEL.get_connections(s, t) if kind in (None, "static") else []
    pidx = KERNEL.get_connections(s, t, plastic=True) if kind in (None, "stdp_pl") else []
    if synapse_model is not None and kind == "stdp_pl" and len(pidx):
        _, _, _, _, pm = KERNEL.plastic_edges()
        names = np.array(KERNEL.pl_models, dtype=object)
        pidx = pidx[names[pm[pidx]] == synapse_model]
    if synapse_model is not None and kind is None:
        idx, pidx = [], []
    return SynapseCollection(idx, pidx)
