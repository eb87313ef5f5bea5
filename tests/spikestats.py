"""Spike-train statistics for the statistical comparisons (engine vs
reference, engine vs oracle, FP32 form vs FP64 form): per-neuron rates,
CV of the inter-spike intervals, and pairwise spike-count correlations.

Inputs are rasters as (sender index 0..n-1, stamp in steps) arrays.  The
pairwise correlation is the Pearson coefficient of two neurons' spike
counts in bins of `bin_ms`, over random pairs of neurons that spiked at
least `min_spikes` times -- the statistic the population-activity
analyses of the reference's examples use for asynchronous-irregular
states.
"""

import numpy as np


def rates_hz(senders, n, t_ms):
    return np.bincount(np.asarray(senders, dtype=np.int64), minlength=n)[:n] / (t_ms * 1e-3)


def cv_isi(senders, stamps, n, h, min_spikes=3):
    """CV of the ISIs per neuron (NaN for neurons with fewer than
    min_spikes spikes)."""
    s = np.asarray(senders, dtype=np.int64)
    t = np.asarray(stamps, dtype=np.int64)
    o = np.lexsort((t, s))
    s, t = s[o], t[o] * h
    same = s[1:] == s[:-1]
    isi = np.diff(t)[same]
    who = s[1:][same]
    cnt = np.bincount(who, minlength=n)[:n].astype(np.float64)
    sm = np.bincount(who, weights=isi, minlength=n)[:n]
    sq = np.bincount(who, weights=isi * isi, minlength=n)[:n]
    cv = np.full(n, np.nan)
    ok = cnt >= max(1, min_spikes - 1)
    mean = sm[ok] / cnt[ok]
    var = np.maximum(sq[ok] / cnt[ok] - mean * mean, 0.0)
    cv[ok] = np.sqrt(var) / mean
    return cv


def binned_counts(senders, stamps, neurons, h, bin_ms, t0_ms, t1_ms):
    """Spike counts [len(neurons), bins] in bins of bin_ms over [t0, t1)."""
    neurons = np.asarray(neurons, dtype=np.int64)
    idx = np.full(int(np.max(neurons)) + 1 if len(neurons) else 1, -1, dtype=np.int64)
    idx[neurons] = np.arange(len(neurons))
    s = np.asarray(senders, dtype=np.int64)
    t = np.asarray(stamps, dtype=np.int64) * h
    keep = (s < len(idx)) & (t >= t0_ms) & (t < t1_ms)
    s, t = s[keep], t[keep]
    row = idx[s]
    ok = row >= 0
    nb = int(round((t1_ms - t0_ms) / bin_ms))
    col = np.minimum(((t[ok] - t0_ms) / bin_ms).astype(np.int64), nb - 1)
    out = np.zeros((len(neurons), nb), dtype=np.float64)
    np.add.at(out, (row[ok], col), 1.0)
    return out


def pair_correlations(senders, stamps, n, h, t0_ms, t1_ms, bin_ms=5.0, n_pairs=2000, seed=0, min_spikes=4,
                      pool=None):
    """Spike-count correlation coefficients of n_pairs random pairs of
    distinct neurons (drawn from `pool`, default all n) that spiked at
    least min_spikes times in [t0, t1)."""
    rng = np.random.default_rng(seed)
    s = np.asarray(senders, dtype=np.int64)
    t = np.asarray(stamps, dtype=np.int64) * h
    win = (t >= t0_ms) & (t < t1_ms)
    cnt = np.bincount(s[win], minlength=n)[:n]
    cand = np.arange(n) if pool is None else np.asarray(pool, dtype=np.int64)
    cand = cand[cnt[cand] >= min_spikes]
    if len(cand) < 2:
        return np.zeros(0)
    a = rng.choice(cand, size=n_pairs)
    b = rng.choice(cand, size=n_pairs)
    keep = a != b
    a, b = a[keep], b[keep]
    uniq = np.unique(np.concatenate([a, b]))
    X = binned_counts(senders, stamps, uniq, h, bin_ms, t0_ms, t1_ms)
    X = X - X.mean(axis=1, keepdims=True)
    sd = np.sqrt((X * X).mean(axis=1))
    pos = np.searchsorted(uniq, a), np.searchsorted(uniq, b)
    num = (X[pos[0]] * X[pos[1]]).mean(axis=1)
    den = sd[pos[0]] * sd[pos[1]]
    ok = den > 0
    return num[ok] / den[ok]


def pop_counts(stamps, bin_steps, t0_step, t1_step):
    """Population spike counts in bins of bin_steps over [t0, t1)."""
    t = np.asarray(stamps, dtype=np.int64)
    t = t[(t >= t0_step) & (t < t1_step)]
    nb = (t1_step - t0_step) // bin_steps
    return np.bincount((t - t0_step) // bin_steps, minlength=nb)[:nb]


def summary(senders, stamps, n, h, t0_ms, t1_ms, bin_ms=5.0, n_pairs=2000, seed=0):
    """Mean rate [Hz], mean CV-ISI and the correlation sample of a raster
    over [t0, t1)."""
    s = np.asarray(senders, dtype=np.int64)
    st = np.asarray(stamps, dtype=np.int64)
    win = (st * h >= t0_ms) & (st * h < t1_ms)
    cv = cv_isi(s[win], st[win], n, h)
    return {
        "rate_hz": float(win.sum() / n / ((t1_ms - t0_ms) * 1e-3)),
        "cv_isi_mean": float(np.nanmean(cv)),
        "cv": cv[~np.isnan(cv)],
        "corr": pair_correlations(s, st, n, h, t0_ms, t1_ms, bin_ms=bin_ms, n_pairs=n_pairs, seed=seed),
    }


def compare(a, b):
    """Errors of summary `a` against summary `b`: relative rate error,
    CV-ISI error, KS statistics of the CV-ISI and correlation
    distributions, and the mean correlations."""
    from scipy import stats

    return {
        "rate_err": a["rate_hz"] / b["rate_hz"] - 1.0,
        "cv_isi_err": a["cv_isi_mean"] - b["cv_isi_mean"],
        "ks_cv": float(stats.ks_2samp(a["cv"], b["cv"]).statistic),
        "ks_corr": float(stats.ks_2samp(a["corr"], b["corr"]).statistic),
        "ks_corr_p": float(stats.ks_2samp(a["corr"], b["corr"]).pvalue),
        "corr_mean": (float(np.mean(a["corr"])), float(np.mean(b["corr"]))),
    }
