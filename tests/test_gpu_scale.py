"""Parity at the large configuration, the 64-pair batch, and the fallback paths.

* 2880x1988 with disparities 0-511: stage by stage against the oracle
  (descriptors, candidate lattice, support list, 16-word grid bitsets, the
  cluster flip kernel's triangulation checked exactly and against the
  reference's Triangle, priors, dense disparities, L/R, post-filters).
* The 64-pair heterogeneous batch the benchmark times, replayed as a CUDA
  graph, bit-equal to 64 single-pair runs; first batches on fresh handles
  (whose workers allocate and zero their workspaces) bit-equal as well.
* Fallbacks the usual inputs never reach, forced through
  elas_b200_set_test_mode: the global-memory flip kernel, the dense bitset
  walk, each size's other prior paint path, and the flip round limit
  returning ELAS_ERR_TIMEOUT.
"""
import numpy as np
import pytest

import elas_b200 as eb
from test_gpu_parity import run_and_compare

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def elas():
    e = eb.Elas(eb.params_reference())
    yield e
    e.close()


@pytest.mark.parametrize("seed", [1, 2])
def test_stagewise_parity_config2(elas, seed):
    """2880x1988, D 0-511: every stage bit-exact, post-filtered maps within
    1e-4, both triangulations exact and equal to Triangle's wherever no four
    points are co-circular."""
    L, R, gt, _ = eb.synth_pair(2, seed)
    p = eb.params_config(511)
    D1, D2, g = run_and_compare(elas, L, R, p)
    assert g["grid_left"].shape[2] == 513
    ctr = elas.stage("del_counters").view(np.int32).reshape(2, 16)
    assert (ctr[:, 0] > 4096).all(), "the large case must exceed the one-SM flip kernel"
    valid = D1 >= 0
    assert valid.mean() > 0.5


def test_stagewise_parity_config2_star_construction(elas):
    """2880x1988, D 0-511, with the triangulations found star by star (the
    size takes the strips and flips by default): every stage against the
    oracle, the same triangle sets as the flip construction."""
    L, R, gt, _ = eb.synth_pair(2, 3)
    p = eb.params_config(511)
    elas.set_params(p)
    elas.process(L, R)
    flips = [elas.stage(k).view(np.int32).reshape(-1, 3).copy() for k in ("tri_left", "tri_right")]
    elas.set_test_mode(eb.Elas.TEST_DELAUNAY_STARS)
    try:
        D1, D2, g = run_and_compare(elas, L, R, p, check_triangle=False)
    finally:
        elas.set_test_mode(0)
    for key, ref in zip(("tri_left", "tri_right"), flips):
        assert {tuple(t) for t in ref.tolist()} == {tuple(t) for t in g[key].tolist()}, key


def _batch_pairs(shapes, seed0):
    return [eb.synth_pair(3, seed0 + i, width=w, height=h, disp_max=d, gt=False)
            for i, (w, h, d) in enumerate(shapes)]


def _singles(e, pairs, dmax):
    out = []
    for (L, R, _, _), d in zip(pairs, dmax):
        e.set_params(eb.params_config(d))
        out.append(e.process(L, R))
    return out


def test_batch64_graph_equals_singles(elas):
    """The benchmark's 64-pair batch (widths 320-1920, heights 240-1080,
    disparity ranges 64/128/256) through the device batch call: the eager
    first call and two graph replays with new image contents each equal
    64 single-pair runs bit for bit."""
    import torch

    from bench import batch_workload

    shapes = batch_workload()
    assert len(shapes) == 64
    dims = [(w, h) for (w, h, _) in shapes]
    dmax = [d for (_, _, d) in shapes]
    bufs = [[torch.empty((h, w), dtype=torch.uint8, device="cuda"),
             torch.empty((h, w), dtype=torch.uint8, device="cuda"),
             torch.empty((h, w), dtype=torch.float32, device="cuda"),
             torch.empty((h, w), dtype=torch.float32, device="cuda")] for (w, h, _) in shapes]
    ptrs = [[b[k].data_ptr() for b in bufs] for k in range(4)]
    batch = eb.Elas(eb.params_config(64))
    try:
        batch.set_graphs(True)
        for rep, seed0 in enumerate((5000, 6000, 7000)):
            pairs = _batch_pairs(shapes, seed0)
            for b, (L, R, _, _) in zip(bufs, pairs):
                b[0].copy_(torch.from_numpy(L))
                b[1].copy_(torch.from_numpy(R))
            torch.cuda.synchronize()
            batch.process_batch_device(*ptrs, dims, dmax)
            torch.cuda.synchronize()
            got = [(b[2].cpu().numpy(), b[3].cpu().numpy()) for b in bufs]
            ref = _singles(elas, pairs, dmax)
            bad = [i for i, ((x1, x2), (s1, s2)) in enumerate(zip(got, ref))
                   if not (np.array_equal(x1, s1) and np.array_equal(x2, s2))]
            assert not bad, f"replay {rep}: pairs {bad} differ from single runs"
        lat = batch.batch_latency(64)
        assert lat.shape == (64,) and (lat > 0).all()
    finally:
        batch.close()


def test_fresh_handle_batches_equal_singles(elas):
    """A batch's first call on a new handle creates its workers, whose
    workspaces are allocated and zeroed during the call; the zero fill must
    be complete before the workers' kernels run.  Several fresh handles,
    each compared bit for bit with single runs."""
    shapes = [(320, 240, 64), (480, 272, 128), (400, 304, 64), (1024, 512, 256), (640, 480, 128)]
    dmax = [d for (_, _, d) in shapes]
    pairs = _batch_pairs(shapes, 900)
    ref = _singles(elas, pairs, dmax)
    for trial in range(4):
        e = eb.Elas(eb.params_config(64))
        try:
            b1, b2 = e.process_batch([x[0] for x in pairs], [x[1] for x in pairs], disp_max=dmax)
        finally:
            e.close()
        for i, ((s1, s2), x1, x2) in enumerate(zip(ref, b1, b2)):
            assert np.array_equal(s1, x1) and np.array_equal(s2, x2), f"trial {trial}, pair {i}"


def test_repeated_batches_are_identical(elas):
    """The same batch, run many times on one handle (eager, then as a graph),
    gives identical bytes every time."""
    shapes = [(320, 240, 64), (480, 272, 128), (400, 304, 64), (336, 256, 64)]
    dmax = [d for (_, _, d) in shapes]
    pairs = _batch_pairs(shapes, 77)
    e = eb.Elas(eb.params_config(64))
    try:
        first = e.process_batch([x[0] for x in pairs], [x[1] for x in pairs], disp_max=dmax)
        for rep in range(10):
            again = e.process_batch([x[0] for x in pairs], [x[1] for x in pairs], disp_max=dmax)
            for i in range(len(shapes)):
                assert np.array_equal(first[0][i], again[0][i]) and np.array_equal(first[1][i], again[1][i]), \
                    f"repeat {rep}, pair {i}"
    finally:
        e.close()


@pytest.mark.parametrize("preset,seed", [(1, 21), (2, 22)])
def test_forced_global_flip_kernel(elas, preset, seed):
    """Every triangulation through the global-memory flip kernel: the same
    stages as the oracle, and the same triangles as the default kernels."""
    W, H, D = eb.synth_dims(preset)
    L, R, _, _ = eb.synth_pair(preset, seed)
    p = eb.params_config(D)
    elas.set_params(p)
    elas.process(L, R)
    default_tris = [elas.stage(k).view(np.int32).reshape(-1, 3) for k in ("tri_left", "tri_right")]
    elas.set_test_mode(eb.Elas.TEST_FLIP_GLOBAL)
    try:
        D1, D2, g = run_and_compare(elas, L, R, p, check_triangle=(preset == 1))
        ctr = elas.stage("del_counters").view(np.int32).reshape(2, 16)
        assert (ctr[:, 4] > 1).all(), "the global kernel ran no flip rounds"
    finally:
        elas.set_test_mode(0)
    for key, ref in zip(("tri_left", "tri_right"), default_tris):
        assert {tuple(t) for t in ref.tolist()} == {tuple(t) for t in g[key].tolist()}, key


@pytest.mark.parametrize("preset,seed", [(1, 31), (2, 32)])
def test_forced_dense_bitset_walk(elas, preset, seed):
    """Every grid cell's candidates walked as a bitset (the branch of cells
    with more candidates than the per-row list holds): dense disparities
    bit-exact against the oracle and equal to the default path."""
    W, H, D = eb.synth_dims(preset)
    L, R, _, _ = eb.synth_pair(preset, seed)
    p = eb.params_config(D)
    elas.set_params(p)
    elas.process(L, R)
    ref = [elas.stage(k).view(np.float32).copy() for k in ("disp_left", "disp_right")]
    elas.set_test_mode(eb.Elas.TEST_DENSE_BITSET)
    try:
        D1, D2, g = run_and_compare(elas, L, R, p, check_triangle=False)
    finally:
        elas.set_test_mode(0)
    assert np.array_equal(g["disp_left"].reshape(-1), ref[0])
    assert np.array_equal(g["disp_right"].reshape(-1), ref[1])


@pytest.mark.parametrize("preset,seed,flag", [(1, 61, "TEST_PRIOR_TILED"), (2, 62, "TEST_PRIOR_DIRECT"),
                                               (1, 63, "TEST_PRIOR_TILED TEST_PRIOR_SMALL_BINS"),
                                               (2, 64, "TEST_PRIOR_SMALL_BINS")])
def test_forced_prior_paint(elas, preset, seed, flag):
    """The plane prior through the paint path the image size does not pick
    (tile by tile at 1242x375, global atomics at 2880x1988), and the tiled
    paint with 2-entry tile bins (most triangles through the overflow
    list): every stage bit-exact against the oracle, and the prior equal to
    the default path's."""
    W, H, D = eb.synth_dims(preset)
    L, R, _, _ = eb.synth_pair(preset, seed)
    p = eb.params_config(D)
    elas.set_params(p)
    elas.process(L, R)
    ref = [elas.stage(k).copy() for k in ("prior_left", "prior_right")]
    elas.set_test_mode(sum(getattr(eb.Elas, f) for f in flag.split()))
    try:
        run_and_compare(elas, L, R, p, check_triangle=False)
        got = [elas.stage(k) for k in ("prior_left", "prior_right")]
    finally:
        elas.set_test_mode(0)
    assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1])


def test_flip_round_limit_returns_timeout(elas):
    """A one-round cap on edge flipping: the call reports ELAS_ERR_TIMEOUT
    (the bounded device loop gave up), and the same handle then runs the
    pair normally."""
    L, R, _, _ = eb.synth_pair(1, 41)
    p = eb.params_config(255)
    elas.set_params(p)
    good1, good2 = elas.process(L, R)
    for flags in (0, eb.Elas.TEST_FLIP_GLOBAL):
        elas.set_test_mode(flags, flip_round_limit=1)
        try:
            with pytest.raises(eb.ElasError) as ei:
                elas.process(L, R)
            assert ei.value.status == 7
        finally:
            elas.set_test_mode(0)
    again1, again2 = elas.process(L, R)
    assert np.array_equal(good1, again1) and np.array_equal(good2, again2)


def test_group_batch_equals_singles(elas):
    """The pair-parallel runner with two entries on device 0 (two handles,
    each on its own host thread, no wait between them): every pair equals
    its single-pair run, and the plan it reports is the host plan."""
    shapes = [(320, 240, 64), (640, 480, 128), (480, 272, 256), (336, 256, 64), (1024, 512, 128)]
    dmax = [d for (_, _, d) in shapes]
    pairs = _batch_pairs(shapes, 4200)
    ref = _singles(elas, pairs, dmax)
    g = eb.ElasGroup(eb.params_config(64), [0, 0])
    try:
        d1, d2, plan = g.process_batch([x[0] for x in pairs], [x[1] for x in pairs], disp_max=dmax)
    finally:
        g.close()
    assert plan.tolist() == eb.group_plan([(w, h) for (w, h, _) in shapes], 2, dmax).tolist()
    assert set(plan.tolist()) == {0, 1}
    for i, ((s1, s2), x1, x2) in enumerate(zip(ref, d1, d2)):
        assert np.array_equal(s1, x1) and np.array_equal(s2, x2), i


@pytest.mark.parametrize("mode", ["config", "reference", "only_left", "subsampling"])
def test_pinned_outputs_equal_pageable(elas, mode):
    """Host-buffer calls whose output buffers are pinned (device-mapped)
    receive the maps from the last post-filter pass directly; the maps equal
    those of the same call with pageable buffers, bit for bit, on the first
    (eager) and the later (graph) calls."""
    import ctypes

    import torch

    L, R, _, _ = eb.synth_pair(1, 51)
    H, W = L.shape
    p = eb.params_reference() if mode == "reference" else eb.params_config(255)
    if mode == "only_left":
        p.postprocess_only_left = True
    if mode == "subsampling":
        p.subsampling = True
    elas.set_params(p)
    ref1, ref2 = elas.process(L, R)
    shape = ref1.shape
    d1 = torch.full(shape, 7.0, dtype=torch.float32).pin_memory()
    d2 = torch.full(shape, 7.0, dtype=torch.float32).pin_memory()
    dims = np.array([W, H, W], np.int32)
    lib = eb.library()
    for call in range(3):
        d1.fill_(7.0)
        d2.fill_(7.0)
        rc = lib.elas_b200_process(elas._h, L.ctypes.data_as(ctypes.c_void_p), R.ctypes.data_as(ctypes.c_void_p),
                                   ctypes.c_void_p(d1.data_ptr()), ctypes.c_void_p(d2.data_ptr()),
                                   dims.ctypes.data_as(ctypes.c_void_p), None)
        elas._check(rc)
        assert np.array_equal(d1.numpy(), ref1), (mode, call)
        assert np.array_equal(d2.numpy(), ref2), (mode, call)
