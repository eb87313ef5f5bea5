"""Runnable cases of the benchmark workloads at chosen sizes, for profiling
a kernel on a small instance:

  python -m nestgpu.cases layered --scale 0.5 --ms 300 --precision fp32
  python -m nestgpu.cases aeif --neurons 10000 --ms 60
  python -m nestgpu.cases serving --requests 40 --capacity-neurons 300000 --capacity-edges 200000000 --slices 40

(run from the package directory's parent with it on sys.path, as bench.py
does).  Each case builds its network on the device, simulates, prints one
summary line and exits 0.
"""

import argparse
import copy
import sys


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["layered", "aeif", "serving"])
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--scale", type=float, default=1.0, help="layered: population size factor")
    ap.add_argument("--neurons", type=int, default=50000, help="aeif: network size (80 % excitatory)")
    ap.add_argument("--ms", type=float, default=100.0, help="simulated time")
    ap.add_argument("--requests", type=int, default=40, help="serving: requests admitted at once")
    ap.add_argument("--capacity-neurons", type=int, default=300_000)
    ap.add_argument("--capacity-edges", type=int, default=200_000_000)
    ap.add_argument("--slices", type=int, default=40, help="serving: min_delay slices simulated")
    ap.add_argument("--ring32", action="store_true", help="layered: 32-bit ring cells")
    ap.add_argument("--no-tiled", action="store_true", help="layered: scatter delivery only")
    a = ap.parse_args(argv)
    from . import serving, workloads

    if a.case == "layered":
        spec = workloads.layered_spec(scale=a.scale)
        eng = workloads.layered_engine(spec, a.precision, ring32=a.ring32, tiled=not a.no_tiled)
        steps = int(round(a.ms / 0.1))
        workloads.layered_add(eng, spec, steps + 10)
        eng.simulate(steps)
    elif a.case == "aeif":
        n_exc = int(round(0.8 * a.neurons))
        spec = workloads.aeif_spec(n_exc=n_exc, n_inh=a.neurons - n_exc)
        eng = workloads.aeif_engine(spec, a.precision)
        steps = int(round(a.ms / 0.1))
        workloads.aeif_add(eng, spec, steps + 10)
        eng.simulate(steps)
    else:
        reqs = serving.make_requests(count=a.requests, rate_hz=20.0, seed=2026)
        eng = serving.new_engine(a.precision, capacity_neurons=a.capacity_neurons, capacity_edges=a.capacity_edges,
                                 max_networks=max(64, a.requests))
        for r in reqs:
            serving._admit(eng, copy.copy(r))
        eng.simulate(a.slices * serving.DELAY_STEPS)
    st = eng.stats()
    print(f"{a.case}: steps {st['clock_steps']} spikes {st['spikes']} syn_events {st['syn_events']} "
          f"gathered {st['gather_slices']}", flush=True)
    eng.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
