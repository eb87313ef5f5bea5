"""Random parameters for Create/Connect (mirrors PyNEST's nest.random and
nest.math, pynest/nest/random/hl_api_random.py, pynest/nest/math).

Values are drawn from a numpy Philox generator seeded by the kernel's
rng_seed; the streams differ from the reference's mt19937_64 draws, so a
network built here is statistically, not bitwise, the reference's network.
Connectivity that must be identical is passed as explicit arrays.
"""

import numpy as np


class Parameter:
    """A lazily drawn per-connection / per-node value."""

    def sample(self, rng, n):  # pragma: no cover - overridden
        raise NotImplementedError

    def _bin(self, other, op):
        return _BinOp(self, other, op)

    def __add__(self, o):
        return self._bin(o, np.add)

    def __radd__(self, o):
        return _BinOp(o, self, np.add)

    def __sub__(self, o):
        return self._bin(o, np.subtract)

    def __rsub__(self, o):
        return _BinOp(o, self, np.subtract)

    def __mul__(self, o):
        return self._bin(o, np.multiply)

    def __rmul__(self, o):
        return _BinOp(o, self, np.multiply)

    def __truediv__(self, o):
        return self._bin(o, np.divide)

    def __neg__(self):
        return _BinOp(-1.0, self, np.multiply)


def _draw(x, rng, n):
    if isinstance(x, Parameter):
        return x.sample(rng, n)
    return np.full(n, float(x))


class _BinOp(Parameter):
    def __init__(self, a, b, op):
        self.a, self.b, self.op = a, b, op

    def sample(self, rng, n):
        return self.op(_draw(self.a, rng, n), _draw(self.b, rng, n))


class _Normal(Parameter):
    def __init__(self, mean=0.0, std=1.0):
        self.mean, self.std = float(mean), float(std)

    def sample(self, rng, n):
        return rng.normal(self.mean, self.std, n)


class _Uniform(Parameter):
    def __init__(self, min=0.0, max=1.0):
        self.lo, self.hi = float(min), float(max)

    def sample(self, rng, n):
        return rng.uniform(self.lo, self.hi, n)


class _Lognormal(Parameter):
    def __init__(self, mean=0.0, std=1.0):
        self.mean, self.std = float(mean), float(std)

    def sample(self, rng, n):
        return rng.lognormal(self.mean, self.std, n)


class _Exponential(Parameter):
    def __init__(self, beta=1.0):
        self.beta = float(beta)

    def sample(self, rng, n):
        return rng.exponential(self.beta, n)


class _UniformInt(Parameter):
    def __init__(self, max=1):
        self.hi = int(max)

    def sample(self, rng, n):
        return rng.integers(0, self.hi, n).astype(np.float64)


def normal(mean=0.0, std=1.0):
    return _Normal(mean, std)


def uniform(min=0.0, max=1.0):
    return _Uniform(min, max)


def lognormal(mean=0.0, std=1.0):
    return _Lognormal(mean, std)


def exponential(beta=1.0):
    return _Exponential(beta)


def uniform_int(max):
    return _UniformInt(max)


class _Clip(Parameter):
    def __init__(self, p, lo, hi):
        self.p, self.lo, self.hi = p, lo, hi

    def sample(self, rng, n):
        v = _draw(self.p, rng, n)
        if self.lo is not None:
            v = np.maximum(v, self.lo)
        if self.hi is not None:
            v = np.minimum(v, self.hi)
        return v


class _Redraw(Parameter):
    def __init__(self, p, lo, hi):
        self.p, self.lo, self.hi = p, float(lo), float(hi)

    def sample(self, rng, n):
        v = _draw(self.p, rng, n)
        bad = (v < self.lo) | (v > self.hi)
        tries = 0
        while np.any(bad):
            tries += 1
            if tries > 1000:
                raise ValueError("redraw: parameter could not be drawn inside [min, max]")
            v[bad] = _draw(self.p, rng, int(bad.sum()))
            bad = (v < self.lo) | (v > self.hi)
        return v


class _MathNS:
    """nest.math: max/min/redraw/exp on parameters."""

    @staticmethod
    def max(p, value):
        return _Clip(p, float(value), None)

    @staticmethod
    def min(p, value):
        return _Clip(p, None, float(value))

    @staticmethod
    def redraw(p, min=-np.inf, max=np.inf):
        return _Redraw(p, min, max)

    @staticmethod
    def exp(p):
        class _E(Parameter):
            def sample(self, rng, n):
                return np.exp(_draw(p, rng, n))

        return _E()


math = _MathNS()
