"""Runnable cases of the benchmark workloads at chosen sizes, for profiling
a kernel on a small instance (run from the repository root):

  python bench_cases.py c1 --precision fp64 --ms 1000 --runs 4
  python bench_cases.py layered --scale 0.5 --ms 300 --precision fp32
  python bench_cases.py aeif --neurons 10000 --ms 60
  python bench_cases.py serving --requests 40 --capacity-neurons 300000 --capacity-edges 200000000 --slices 40
  python bench_cases.py hpc --scale 0.5 --ms 200 --precision fp64
  python bench_cases.py atomics --precision fp64

The atomics case measures the device's rate of FP64 (or int64) atomic adds to
random cells of a ring the size of the layered network's (77,169 neurons x
80 slots x 2 channels), 9.2e6 adds per launch -- one step's deliveries at its
mean rate -- through torch.index_add_ (atomics into global memory): the wall
a scatter delivery of that network meets.

Each case builds its network, simulates, prints one summary line and exits 0.
The c1 case is bench.py's headline network (12,500 iaf_psc_exp neurons,
K_E = 1,000, K_I = 250, 8 kHz drive) built with the PyNEST-compatible
front-end and run as `runs` calls of Simulate(ms) -- the first one long
enough for the autotuner, as in the bench's warm-up.
"""

import os
import sys

ROOT = os.path.dirname(os.path.abspath(__file__))
if os.path.join(ROOT, "nest-simulator_b200") not in sys.path:
    sys.path.insert(0, os.path.join(ROOT, "nest-simulator_b200"))

import argparse
import copy
import sys


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["c1", "layered", "aeif", "serving", "hpc", "atomics"])
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--scale", type=float, default=1.0, help="layered, hpc: population size factor")
    ap.add_argument("--neurons", type=int, default=50000, help="aeif: network size (80 % excitatory)")
    ap.add_argument("--ms", type=float, default=100.0, help="simulated time")
    ap.add_argument("--requests", type=int, default=40, help="serving: requests admitted at once")
    ap.add_argument("--capacity-neurons", type=int, default=300_000)
    ap.add_argument("--capacity-edges", type=int, default=200_000_000)
    ap.add_argument("--slices", type=int, default=40, help="serving: min_delay slices simulated")
    ap.add_argument("--runs", type=int, default=4, help="c1, hpc: Simulate(ms) calls")
    ap.add_argument("--fixed", default="", help="c1: fixed launch configuration 'variant,ctas_per_sm,chunks_per_warp' "
                                                  "instead of the autotuner (which measures differently under a profiler)")
    ap.add_argument("--ring32", action="store_true", help="layered: 32-bit ring cells")
    ap.add_argument("--no-tiled", action="store_true", help="layered: scatter delivery only")
    a = ap.parse_args(argv)
    import nestgpu as nest
    from nestgpu import serving, workloads
    from nestgpu.kernel import KERNEL

    if a.case == "atomics":
        import torch

        dev = torch.device("cuda", 0)
        dt = torch.float64 if a.precision == "fp64" else torch.int64
        cells, n_ev = 77169 * 80 * 2, 9_200_000
        g = torch.Generator(device=dev).manual_seed(1)
        ring = torch.zeros(cells, dtype=dt, device=dev)
        idx = torch.randint(0, cells, (n_ev,), device=dev, generator=g)
        val = torch.ones(n_ev, dtype=dt, device=dev)
        for _ in range(3):
            ring.index_add_(0, idx, val)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(20):
            ring.index_add_(0, idx, val)
        e1.record()
        torch.cuda.synchronize()
        us = e0.elapsed_time(e1) * 1e3 / 20
        print(f"atomics ({dt}): {n_ev} random adds into {cells} cells in {us:.1f} us: {n_ev / us * 1e6:.3e} adds/s",
              flush=True)
        return 0
    if a.case == "hpc":
        # the hpc_benchmark network (iaf_psc_alpha, E->E stdp_pl_synapse_hom_hpc)
        workloads.hpc_benchmark(nest, scale=a.scale, precision=a.precision, record=False)
        for _ in range(a.runs):
            nest.Simulate(a.ms)
        st = nest.engine_stats()
        print(f"hpc: steps {st['clock_steps']} spikes {st['spikes']} syn_events {st['syn_events']}", flush=True)
        nest.ResetKernel()
        return 0
    if a.case == "c1":
        workloads.c1(nest, precision=a.precision, seed=4242)
        if a.fixed:
            nest.Prepare()
            KERNEL.engine.set_tuning(0, *[int(x) for x in a.fixed.split(",")])
        for _ in range(a.runs):
            nest.Simulate(a.ms)
        st = nest.engine_stats()
        print(f"c1: steps {st['clock_steps']} spikes {st['spikes']} syn_events {st['syn_events']} "
              f"tuned {KERNEL.engine.tuned()['update_kernel']}", flush=True)
        nest.ResetKernel()
        return 0
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
