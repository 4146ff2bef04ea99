"""The multi-GPU pair-parallel runner's plan, on the host (no GPU).

elas_b200_group_plan deals pairs to device entries largest estimated cost
first, each to the least-loaded entry.  The plan is a pure function of the
sizes, so every process that computes it agrees; two gloo ranks here each
take their share of a batch by the plan (the CPU oracle standing in for the
device pipeline) and together reproduce the single-process result.
"""
import os
import socket
import sys

import numpy as np
import pytest

import elas_b200 as eb
from conftest import REPO


def _costs(dims, dmax):
    d = np.asarray(dims).reshape(-1, 2)
    return d[:, 0].astype(float) * d[:, 1] * (1.0 + np.asarray(dmax, float) / 128.0)


@pytest.mark.parametrize("ndev", [1, 2, 3, 8])
def test_plan_is_a_balanced_deterministic_lpt(ndev):
    sys.path.insert(0, REPO)
    from bench import batch_workload

    shapes = batch_workload()
    dims = [(w, h) for (w, h, _) in shapes]
    dmax = [d for (_, _, d) in shapes]
    a = eb.group_plan(dims, ndev, dmax)
    b = eb.group_plan(dims, ndev, dmax)
    assert np.array_equal(a, b)
    assert a.min() >= 0 and a.max() < ndev
    cost = _costs(dims, dmax)
    # the host restatement of the rule gives the same plan
    load = np.zeros(ndev)
    ref = np.zeros(len(dims), np.int32)
    for i in sorted(range(len(dims)), key=lambda i: -cost[i]):     # stable: ties keep pair order
        k = int(np.argmin(load))
        ref[i] = k
        load[k] += cost[i]
    assert np.array_equal(a, ref)
    loads = np.bincount(a, weights=cost, minlength=ndev)
    # LPT bound: no entry exceeds the mean by more than the largest single pair
    assert loads.max() <= loads.mean() + cost.max() + 1e-6


def test_plan_edge_cases():
    assert eb.group_plan([], 4).size == 0
    assert eb.group_plan([(320, 240)], 4).tolist() == [0]
    assert eb.group_plan([(320, 240)] * 4, 4).tolist() == [0, 1, 2, 3]    # equal costs, pair order
    with pytest.raises(eb.ElasError):
        eb.group_plan([(320, 240)], 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


SHAPES = [(96, 64, 16), (128, 80, 24), (64, 64, 16), (112, 96, 32), (80, 48, 16)]


def _pairs():
    return [eb.synth_pair(3, 300 + i, width=w, height=h, disp_max=d, gt=False) for i, (w, h, d) in enumerate(SHAPES)]


def _rank_main(rank, world, port, out_dir):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch
    import torch.distributed as dist

    import oracle

    dist.init_process_group("gloo")
    plan = eb.group_plan([(w, h) for (w, h, _) in SHAPES], world, [d for (_, _, d) in SHAPES])
    mine = {}
    for i, (L, R, _, _) in enumerate(_pairs()):
        if plan[i] == rank:
            mine[i] = oracle.process(L, R, eb.params_config(SHAPES[i][2]), threads=1)[0]
    got = [None] * world
    dist.all_gather_object(got, {i: d.tobytes() for i, d in mine.items()})
    if rank == 0:
        merged = {}
        for part in got:
            assert not (set(part) & set(merged)), "a pair ran on two ranks"
            merged.update(part)
        np.save(os.path.join(out_dir, "keys.npy"), np.array(sorted(merged)))
        for i, buf in merged.items():
            np.save(os.path.join(out_dir, f"d{i}.npy"), np.frombuffer(buf, np.float32))
    dist.destroy_process_group()


def test_two_gloo_ranks_split_a_batch_by_the_plan(tmp_path):
    import torch.multiprocessing as mp

    import oracle

    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    keys = np.load(tmp_path / "keys.npy")
    assert keys.tolist() == list(range(len(SHAPES)))
    for i, (L, R, _, _) in enumerate(_pairs()):
        ref = oracle.process(L, R, eb.params_config(SHAPES[i][2]), threads=1)[0]
        assert np.array_equal(np.load(tmp_path / f"d{i}.npy"), ref.reshape(-1))
