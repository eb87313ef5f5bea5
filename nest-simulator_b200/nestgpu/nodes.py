"""NodeCollection (mirrors pynest/nest/lib/hl_api_types.py NodeCollection)."""

import numpy as np

from .kernel import KERNEL


class NodeCollection:
    """An ordered set of node ids with PyNEST-style get/set."""

    def __init__(self, ids=()):
        object.__setattr__(self, "_ids", np.asarray(ids, dtype=np.int64).ravel())

    # --- container protocol -------------------------------------------------
    def __len__(self):
        return len(self._ids)

    def __iter__(self):
        for i in self._ids:
            yield NodeCollection([i])

    def __getitem__(self, key):
        if isinstance(key, (int, np.integer)):
            if key >= len(self._ids) or key < -len(self._ids):
                raise IndexError("NodeCollection index out of range")
            return NodeCollection([self._ids[key]])
        if isinstance(key, slice):
            return NodeCollection(self._ids[key])
        key = np.asarray(key)
        if key.dtype == bool:
            return NodeCollection(self._ids[key])
        return NodeCollection(self._ids[key.astype(np.int64)])

    def __add__(self, other):
        ids = np.concatenate([self._ids, np.asarray(other.tolist() if isinstance(other, NodeCollection) else other)])
        if len(np.unique(ids)) != len(ids):
            raise ValueError("Cannot add NodeCollections with overlapping node ids")
        return NodeCollection(np.sort(ids))

    def __eq__(self, other):
        return isinstance(other, NodeCollection) and np.array_equal(self._ids, other._ids)

    def __hash__(self):
        return hash(self._ids.tobytes())

    def __contains__(self, node_id):
        return int(node_id) in set(self._ids.tolist())

    def __repr__(self):
        if len(self._ids) == 0:
            return "NodeCollection()"
        return f"NodeCollection(metadata=None, model={KERNEL.node_model[self._ids[0] - 1]}, " \
               f"size={len(self._ids)}, first={self._ids[0]}, last={self._ids[-1]})"

    def tolist(self):
        return [int(i) for i in self._ids]

    def index(self, node_id):
        w = np.nonzero(self._ids == int(node_id))[0]
        if len(w) == 0:
            raise ValueError(f"{node_id} is not in NodeCollection")
        return int(w[0])

    @property
    def global_id(self):
        return self.get("global_id")

    @property
    def ids(self):
        return self._ids

    # --- status ---------------------------------------------------------------
    def get(self, *keys, output=""):
        if len(keys) == 1 and isinstance(keys[0], (list, tuple)):
            keys = tuple(keys[0])
        if len(keys) == 0:
            per = KERNEL.get_status(self._ids)
            allk = list(dict.fromkeys(k for d in per for k in d))
            res = {k: tuple(d.get(k) for d in per) if len(per) != 1 else per[0].get(k) for k in allk}
        elif len(keys) == 1:
            vals = KERNEL.get_status(self._ids, keys[0])
            res = _unwrap(vals)
        else:
            res = {k: _unwrap(KERNEL.get_status(self._ids, k)) for k in keys}
        if output == "pandas":
            import pandas as pd

            if isinstance(res, dict):
                return pd.DataFrame({k: (v if isinstance(v, tuple) else [v]) for k, v in res.items()},
                                    index=self.tolist())
            return pd.DataFrame({keys[0]: res if isinstance(res, tuple) else [res]}, index=self.tolist())
        return res

    def set(self, params=None, **kwargs):
        if params is None:
            params = kwargs
        elif kwargs:
            raise TypeError("set: give a dictionary or keyword arguments, not both")
        KERNEL.set_status(self._ids, params)

    def __getattr__(self, name):
        if name.startswith("_"):
            raise AttributeError(name)
        return self.get(name)

    def __setattr__(self, name, value):
        if name.startswith("_"):
            object.__setattr__(self, name, value)
        else:
            self.set({name: value})


def _unwrap(vals):
    vals = [_events(v) for v in vals]
    if len(vals) == 1:
        return vals[0]
    return tuple(vals)


def _events(v):
    if isinstance(v, dict):
        out = {}
        for k, x in v.items():
            if isinstance(x, list):
                out[k] = np.concatenate(x) if x else np.zeros(0)
            else:
                out[k] = np.asarray(x)
        return out
    return v
