"""Multi-rank (replica) plumbing of bench.py on CPU: two gloo ranks.

Pairs are independent, so N ranks run N replicas with no exchange on the data
path.  This checks the host side of that design without a GPU: each rank
works on its own seeded pair (here through the CPU oracle as the stand-in
for the device pipeline), the timed region's maximum is taken over ranks, and
the whole-job rate counts the units of every rank.  The reference arm's rule
(rank 0 alone works, the others exit without work) is checked through
bench.py under torchrun.
"""
import os
import socket
import subprocess
import sys
import time
import types

import numpy as np
import pytest

from conftest import REPO


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out_dir):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, REPO)
    import torch
    import torch.distributed as dist

    import bench
    import elas_b200 as eb
    import oracle

    w, r, _ = bench.dist_setup(types.SimpleNamespace(impl="ours"), backend="gloo")
    assert (w, r) == (world, rank)
    L, R, _, _ = eb.synth_pair(3, bench.replica_seed(rank), width=96, height=64, disp_max=16, gt=False)
    p = eb.params_config(16)
    bench.barrier(world)
    t0 = time.perf_counter()
    D1 = oracle.process(L, R, p, threads=1)[0]
    el = time.perf_counter() - t0
    bench.barrier(world)
    tmax = bench.max_over_ranks(el, world)
    sums = [torch.zeros(1, dtype=torch.float64) for _ in range(world)]
    dist.all_gather(sums, torch.tensor([float(np.abs(D1).sum())], dtype=torch.float64))
    rate = bench.aggregate_rate(1, tmax, world)
    np.save(os.path.join(out_dir, f"r{rank}.npy"),
            np.array([el, tmax, rate] + [float(x.item()) for x in sums], np.float64))
    dist.destroy_process_group()


def test_two_gloo_replicas(tmp_path):
    import torch.multiprocessing as mp

    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    r = [np.load(tmp_path / f"r{k}.npy") for k in range(world)]
    # every rank saw the same maximum, which is the slower rank's own time
    assert r[0][1] == r[1][1] == max(r[0][0], r[1][0])
    # whole-job rate = pairs of all ranks / slowest rank
    assert r[0][2] == pytest.approx(world / r[0][1])
    # the replicas processed different pairs (distinct seeds), and agree on what each did
    assert np.array_equal(r[0][3:], r[1][3:])
    assert r[0][3] != r[0][4]


def test_reference_arm_rank0_only(tmp_path):
    """`bench.py --impl reference` under torchrun with two ranks: one JSON line."""
    env = dict(os.environ, OMP_NUM_THREADS="1")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(_free_port()), os.path.join(REPO, "bench.py"), "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "3"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=300, env=env, cwd=str(tmp_path))
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    lines = [x for x in out.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    import json

    rec = json.loads(lines[0])
    assert rec["impl"] == "reference" and rec["n_gpus"] == 2 and rec["value"] > 0
    assert rec["e2e"]["h2d_bytes_per_step"] == 0
