"""The N>1 bench path on CPU: world_size-2 gloo ranks.

The path has no cross-GPU exchange (independent network replicas, one per
GPU), so the only collectives are the timing/aggregation reductions in
bench.py: time = max over ranks, events = sum over ranks.  Each rank here
runs its own oracle replica of a small network with its own seed, as the
engine replicas do on GPUs."""

import os
import socket

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_dir):
    import sys

    for p in (os.path.join(ROOT, "nest-simulator_b200"), os.path.join(ROOT, "oracle"), ROOT):
        sys.path.insert(0, p)
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    import oracle as O

    import nestgpu as nest
    from nestgpu import workloads
    from nestgpu.kernel import KERNEL

    workloads.brunel_exp(nest, n_exc=400, n_inh=100, k_exc=40, k_inh=10, seed=100 + rank)
    net, c = O.net_from_kernel(KERNEL, nthreads=1)
    net.run(500, nthreads=1)
    ev = net.syn_events
    t_local = float(10 + rank)
    t_max = bench.max_over_ranks(t_local, dist)
    ev_sum = bench.sum_over_ranks(ev, dist)
    np.save(os.path.join(out_dir, f"r{rank}.npy"), np.array([ev, t_max, ev_sum], dtype=np.float64))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_replica_aggregation(tmp_path):
    import torch.multiprocessing as mp

    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    r0 = np.load(tmp_path / "r0.npy")
    r1 = np.load(tmp_path / "r1.npy")
    assert r0[1] == r1[1] == 11.0                       # max over ranks
    assert r0[2] == r1[2] == r0[0] + r1[0]              # whole-job events
    assert r0[0] != r1[0]                               # independent replicas (different seeds)
    assert r0[0] > 0 and r1[0] > 0


def test_reference_arm_other_ranks_exit_clean(tmp_path):
    """`bench.py --impl reference` under torchrun: rank 0 alone works."""
    import subprocess
    import sys

    port = _free_port()
    env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2", RANK="1",
               LOCAL_RANK="1")
    p1 = subprocess.Popen([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                           "--warmup", "0", "--gpus", "2"], env=env, stdout=subprocess.PIPE,
                          stderr=subprocess.PIPE, text=True)
    env0 = dict(env, RANK="0", LOCAL_RANK="0")
    p0 = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                         "--warmup", "0", "--gpus", "2"], env=env0, capture_output=True, text=True, timeout=600)
    out1, err1 = p1.communicate(timeout=600)
    assert p0.returncode == 0, p0.stderr[-2000:]
    assert p1.returncode == 0, err1[-2000:]
    assert '"impl": "reference"' in p0.stdout
    assert out1.strip() == ""
