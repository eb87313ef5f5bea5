"""Connect and GetConnections (mirrors pynest/nest/lib/hl_api_connections.py
and the connection rules of nestkernel/conn_builder.cpp).

The rules draw from a numpy Philox stream seeded by rng_seed, so a network
built here has the reference's connection statistics but not its exact
edges.  To run the reference's exact graph, export it with the reference's
``GetConnections`` and connect the arrays with ``one_to_one`` (the
connect-arrays path of ``nest.Connect``).
"""

import numpy as np

from .kernel import KERNEL, KernelException
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
    if model not in ("static_synapse", "static_synapse_hom_w"):
        raise BadProperty(f"synapse model '{model}' is not on the engine's path (static_synapse only)")
    defaults = K.syn_defaults["static_synapse"]
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
    K.add_edges(s, t, wv, dv)
    if return_synapsecollection:
        return get_connections(NodeCollection(np.unique(s)), NodeCollection(np.unique(t)))
    return None


class SynapseCollection:
    """Connections selected by GetConnections (indices into the kernel's
    edge table, sorted by source then target)."""

    def __init__(self, idx):
        self._idx = np.asarray(idx, dtype=np.int64)

    def __len__(self):
        return len(self._idx)

    def _col(self, key):
        src, tgt, w, d = KERNEL.edges()
        i = self._idx
        if key == "source":
            return src[i].astype(np.int64)
        if key == "target":
            return tgt[i].astype(np.int64)
        if key == "weight":
            return w[i]
        if key == "delay":
            return d[i].astype(np.int64) * KERNEL.ms_per_step
        if key == "synapse_model":
            return np.array(["static_synapse"] * len(i), dtype=object)
        if key in ("receptor", "port", "target_thread", "synapse_id"):
            return np.zeros(len(i), dtype=np.int64)
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
        src, tgt, w, d = KERNEL.edges()
        for k, v in params.items():
            vals = np.broadcast_to(np.asarray(v, dtype=np.float64), (len(self._idx),))
            if k == "weight":
                w[self._idx] = vals
            elif k == "delay":
                steps = KERNEL.delay_ms_to_steps(vals)
                if np.any(steps < 1):
                    raise BadProperty("Delay must be greater than or equal to resolution")
                d[self._idx] = steps
            else:
                raise BadProperty(f"cannot set '{k}' on static_synapse connections")
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
    if synapse_model not in (None, "static_synapse"):
        return SynapseCollection([])
    return SynapseCollection(KERNEL.get_connections(None if source is None else _ids(source),
                                                    None if target is None else _ids(target)))
