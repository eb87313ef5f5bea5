"""stdp_pl_synapse_hom on the CPU oracle, pinned to the published rule:
a self-contained restatement of the power-law STDP update (facilitation by
the postsynaptic spikes since the last presynaptic one, depression by the
postsynaptic trace at the arrival; models/stdp_pl_synapse_hom.h:255-298 with
nestkernel/archiving_node.cpp's history and trace) applied to the oracle's own
pre- and postsynaptic spike times gives the oracle's weights bit for bit --
the check the reference's test_stdp_pl_synapse_hom.py makes of NEST."""

import math

import numpy as np
import pytest

import oracle as O

EPS = 1e-6
H = 0.1


def stdp_pl(pre_ms, post_ms, d_ms, w0, lam, alpha, mu, tau_plus, tau_minus):
    """Weight after each presynaptic spike (the rule restated in Python)."""
    # the postsynaptic trace at each postsynaptic spike
    Km, last, post = 0.0, 0.0, []
    for t in post_ms:
        Km = Km * math.exp((last - t) * (1.0 / tau_minus)) + 1.0
        last = t
        post.append((t, Km))
    w, Kplus, t_last = w0, 0.0, 0.0
    out = []
    for t_pre in pre_ms:
        t1, t2 = t_last - d_ms + EPS, t_pre - d_ms + EPS
        for tp, _ in post:
            if t1 <= tp < t2:
                minus_dt = t_last - (tp + d_ms)
                w = w + (lam * w ** mu * (Kplus * math.exp(minus_dt * (1.0 / tau_plus))))
        kminus = 0.0
        for tp, kp in reversed(post):
            if (t_pre - d_ms) - tp > EPS:
                kminus = kp * math.exp((tp - (t_pre - d_ms)) * (1.0 / tau_minus))
                break
        new_w = w - (lam * alpha * w * kminus)
        w = new_w if new_w > 0.0 else 0.0
        Kplus = Kplus * math.exp((t_last - t_pre) * (1.0 / tau_plus)) + 1.0
        t_last = t_pre
        out.append(w)
    return out


def _pair(pre_gen_steps, post_gen_steps, d_steps, w0, steps, **rule):
    """Two iaf_psc_delta neurons each made to spike by its own generator
    (one step after each generator spike), a plastic edge pre -> post."""
    net = O.OracleNet("iaf_psc_delta", 2, H, 1, max(d_steps, 1))
    net.set("t_ref", 0.1)
    net.set("tau_minus", rule.get("tau_minus", 20.0))
    gsteps = np.concatenate([pre_gen_steps, post_gen_steps]).astype(np.int64)
    gsrc = np.concatenate([np.full(len(pre_gen_steps), 2), np.full(len(post_gen_steps), 3)]).astype(np.int32)
    o = np.argsort(gsteps, kind="stable")
    net.set_edges(np.array([2, 3]), np.array([0, 1]), np.array([100.0, 100.0]), np.array([1, 1]), n_src=4)
    net.set_sched(gsteps[o], gsrc[o])
    net.set_plastic([0], [1], [w0], [d_steps], lam=rule["lam"], alpha=rule["alpha"], mu=rule["mu"],
                    tau_plus=rule["tau_plus"], n_src=2)
    net.set_record(np.ones(2, dtype=np.uint8))
    return net


@pytest.mark.parametrize("d_steps", [1, 10, 17])
def test_oracle_stdp_pl_equals_the_rule(d_steps):
    rng = np.random.default_rng(d_steps)
    T = 6000
    pre_g = np.unique(rng.integers(0, T - 50, 80))
    post_g = np.unique(np.concatenate([rng.integers(0, T - 50, 90), pre_g[::7] + 3, pre_g[::5]]))
    rule = dict(lam=0.1, alpha=1.0, mu=0.4, tau_plus=20.0, tau_minus=33.7)
    net = _pair(pre_g, post_g, d_steps, 0.5, T, **rule)
    checkpoints = []
    done = 0
    for chunk in (777, 1500, 2223, T - 4500):
        net.run(chunk)
        done += chunk
        checkpoints.append((done, net.plastic_weights()[0]))
    s, st = net.spikes()
    # spike times from their stamps, in Python floats throughout (libm's exp
    # and pow, as the oracle calls them)
    pre_ms = [int(t) * 100 * (1.0 / 1000.0) for t in st[s == 0]]
    post_ms = [int(t) * 100 * (1.0 / 1000.0) for t in st[s == 1]]
    assert len(pre_ms) > 60 and len(post_ms) > 80
    ws = stdp_pl(pre_ms, post_ms, d_steps * (100 * (1.0 / 1000.0)), 0.5, rule["lam"], rule["alpha"], rule["mu"],
                 rule["tau_plus"], rule["tau_minus"])
    # the weight after the last presynaptic spike delivered by each checkpoint
    # (a spike of stamp t is delivered at the close of the one-step slice
    # that ends at step t)
    for done, w in checkpoints:
        k = sum(1 for t in st[s == 0] if t <= done)
        assert w == (ws[k - 1] if k else 0.5), (done, k)
    assert ws[-1] != 0.5
