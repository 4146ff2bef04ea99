"""Parity of the CUDA pipeline with the CPU oracle, stage by stage.

Every stage is bit-exact except the post-filtered output (float, 1e-4).
The oracle consumes the GPU's triangle list, so the dense stages are
compared on identical triangulations; the triangulation itself is checked
exactly (valid, empty-circumcircle under the symbolic perturbation) and
against the reference's Triangle (equal wherever no four points are
co-circular).
"""
import numpy as np
import pytest

import elas_b200 as eb
import oracle

pytestmark = pytest.mark.gpu

POST_TOL = 1e-4


@pytest.fixture(scope="module")
def elas():
    e = eb.Elas(eb.params_reference())
    yield e
    e.close()


def gpu_stages(e, W, H, p):
    cw, ch, gw, gh = oracle.geom(W, H, p)
    st = {}
    st["desc_left"] = e.stage("desc_left").reshape(H, W, 16)
    st["desc_right"] = e.stage("desc_right").reshape(H, W, 16)
    st["can_lr"] = e.stage("can_lr").view(np.int32).reshape(ch, cw)
    st["can"] = e.stage("can").view(np.int32).reshape(ch, cw)
    st["support"] = e.stage("support").view(np.int32).reshape(-1, 3)
    st["grid_left"] = e.stage("grid_left").view(np.int32).reshape(gh, gw, p.disp_max + 2)
    st["grid_right"] = e.stage("grid_right").view(np.int32).reshape(gh, gw, p.disp_max + 2)
    st["tri_left"] = e.stage("tri_left").view(np.int32).reshape(-1, 3)
    st["tri_right"] = e.stage("tri_right").view(np.int32).reshape(-1, 3)
    for k in ("prior_left", "prior_right"):
        st[k] = e.stage(k).view(np.int32).reshape(H, W)
    Ho, Wo = (H // 2, W // 2) if p.subsampling else (H, W)
    for k in ("disp_left", "disp_right", "lr_left", "lr_right"):
        st[k] = e.stage(k).view(np.float32).reshape(Ho, Wo)
    return st


def run_and_compare(e, L, R, p, check_triangle=True):
    e.set_params(p)
    H, W = L.shape
    D1, D2 = e.process(L, R)
    g = gpu_stages(e, W, H, p)
    o1, o2, o = oracle.process(L, R, p, tri_left=g["tri_left"], tri_right=g["tri_right"], dumps=True)
    # the library stores the plane prior clamped (every d_plane <= 0 and every
    # d_plane > disp_max + radius act alike in the dense step)
    dcap = p.disp_max + max(int(np.ceil(np.float32(p.sigma) * np.float32(p.sradius))), 2) + 1
    for k in ("prior_left", "prior_right"):
        o[k] = np.where(o[k] <= 0, -1, np.minimum(o[k], dcap)).astype(np.int32)
    for k in ("desc_left", "desc_right", "can_lr", "can", "support", "grid_left", "grid_right", "prior_left",
              "prior_right"):
        assert g[k].shape == o[k].shape, k
        mism = np.count_nonzero(g[k] != o[k])
        assert mism == 0, f"{k}: {mism} mismatches"
    for k in ("disp_left", "disp_right", "lr_left", "lr_right"):
        assert np.array_equal(g[k], o[k]), f"{k}: {np.count_nonzero(g[k] != o[k])} mismatches"
    np.testing.assert_allclose(D1, o1, atol=POST_TOL, rtol=0)
    np.testing.assert_allclose(D2, o2, atol=POST_TOL, rtol=0)
    uvd = g["support"]
    for right, key in ((0, "tri_left"), (1, "tri_right")):
        xy = oracle.support_points(uvd, right)
        ok, stats = oracle.delaunay_check(xy, g[key])
        assert ok, (key, stats)
        if check_triangle and oracle.have_triangle() and len(uvd) >= 3:
            ref = oracle.triangulate_ref(xy.astype(np.float32))
            assert ref.shape[0] == g[key].shape[0], key
            cmp = oracle.tri_compare(xy, g[key], ref)
            assert cmp[4] == 0, (key, cmp)
    return D1, D2, g


def test_stagewise_parity_config0(elas):
    L, R, gt, _ = eb.synth_pair(0, 1)
    D1, D2, g = run_and_compare(elas, L, R, eb.params_config(63))
    valid = D1 >= 0
    assert valid.mean() > 0.5
    assert (np.abs(D1 - gt) > 2)[valid].mean() < 0.2


def test_reference_parameters_config0(elas):
    L, R, _, _ = eb.synth_pair(0, 2)
    run_and_compare(elas, L, R, eb.params_reference())


def test_stagewise_parity_config1(elas):
    L, R, _, _ = eb.synth_pair(1, 1)
    run_and_compare(elas, L, R, eb.params_config(255))


@pytest.mark.parametrize("W,H,D", [(97, 61, 31), (160, 120, 47), (333, 211, 95), (16, 16, 8)])
def test_odd_sizes(elas, W, H, D):
    L, R, _, _ = eb.synth_pair(3, 7, width=W, height=H, disp_max=D)
    run_and_compare(elas, L, R, eb.params_config(D))


def test_non_default_parameters(elas):
    L, R, _, _ = eb.synth_pair(3, 9, width=400, height=300, disp_max=80)
    p = eb.params_config(80)
    p.candidate_stepsize = 4
    p.grid_size = 16
    p.disp_min = 3
    p.support_threshold = 0.95
    p.incon_window_size = 3
    p.lr_threshold = 1
    p.match_texture = 6
    p.sradius = 3
    p.gamma = 5
    p.postprocess_only_left = True
    run_and_compare(elas, L, R, p)


@pytest.mark.parametrize("width,height,ws", [(2000, 300, 0), (2000, 300, 10), (2000, 300, 40), (1200, 600, 60),
                                             (2800, 300, 40)])
def test_inconsistency_window_sizes(elas, width, height, ws):
    """The inconsistency filter shares a candidate among 4, 2 or 1 lanes by
    the lattice width (240, 400 and 560 candidates per row here) and stages
    its window rows in shared memory when they fit; the half windows of 60
    at 1200x600 and of 40 at 2000x300 and 2800x300 do not fit and read the
    lattice in place."""
    L, R, _, _ = eb.synth_pair(3, 21, width=width, height=height, disp_max=96)
    p = eb.params_config(96)
    p.incon_window_size = ws
    run_and_compare(elas, L, R, p, check_triangle=False)


@pytest.mark.parametrize("filt", ["speckle", "gap", "gap_wide", "mean", "median"])
def test_post_filters_individually(elas, filt):
    L, R, _, _ = eb.synth_pair(1, 3)
    p = eb.params_reference()
    if filt == "speckle":
        p.speckle_size = 200
    elif filt == "gap":
        p.ipol_gap_width = 3
    elif filt == "gap_wide":
        p.ipol_gap_width = 5000
    elif filt == "mean":
        p.filter_adaptive_mean = True
    else:
        p.filter_median = True
    run_and_compare(elas, L, R, p, check_triangle=False)


def test_constructor_default_parameters(elas):
    """Elas::parameters() defaults (support_threshold 0.95, gamma 5, sradius 3,
    ipol_gap_width 5000, median on)."""
    L, R, _, _ = eb.synth_pair(1, 6)
    run_and_compare(elas, L, R, eb.params_default(), check_triangle=False)


def test_textureless_and_tiny_inputs(elas):
    flat = np.full((64, 80), 128, np.uint8)
    elas.set_params(eb.params_config(31))
    D1, D2 = elas.process(flat, flat)
    assert (D1 == -1).all() and (D2 == -1).all()
    assert elas.stage("support").size == 0
    noise = np.random.default_rng(0).integers(0, 256, (16, 16), dtype=np.uint8)
    run_and_compare(elas, noise, noise, eb.params_config(8))


def test_end_to_end_against_triangle(elas):
    """Same pair through the oracle with the reference's Triangle: only pixels
    whose plane prior comes from a co-circular or duplicate-point choice may
    differ."""
    if not oracle.have_triangle():
        pytest.skip("reference Triangle not built")
    L, R, _, _ = eb.synth_pair(1, 4)
    p = eb.params_reference()
    elas.set_params(p)
    D1, D2 = elas.process(L, R)
    o1, o2, _ = oracle.process(L, R, p)
    diff = (np.count_nonzero(D1 != o1) + np.count_nonzero(D2 != o2)) / (2.0 * D1.size)
    print(f"pixels differing from the Triangle pipeline: {diff:.5f}")
    assert diff < 0.02


def test_deterministic_repeat(elas):
    L, R, _, _ = eb.synth_pair(1, 8)
    p = eb.params_config(255)
    elas.set_params(p)
    a1, a2 = elas.process(L, R)
    sa = gpu_stages(elas, L.shape[1], L.shape[0], p)
    b1, b2 = elas.process(L, R)
    sb = gpu_stages(elas, L.shape[1], L.shape[0], p)
    assert np.array_equal(a1, b1) and np.array_equal(a2, b2)
    for k in sa:
        assert np.array_equal(sa[k], sb[k]), k


def test_batch_equals_singles(elas):
    pairs = [eb.synth_pair(3, s, width=w, height=h, disp_max=d)
             for s, (w, h, d) in enumerate([(320, 240, 64), (480, 272, 128), (400, 304, 64)])]
    dmax = [64, 128, 64]
    elas.set_params(eb.params_config(64))
    b1, b2 = elas.process_batch([x[0] for x in pairs], [x[1] for x in pairs], disp_max=dmax)
    for (L, R, _, _), d, x1, x2 in zip(pairs, dmax, b1, b2):
        elas.set_params(eb.params_config(d))
        s1, s2 = elas.process(L, R)
        assert np.array_equal(s1, x1) and np.array_equal(s2, x2)


def test_device_api_matches_host_api(elas):
    import torch

    L, R, _, _ = eb.synth_pair(0, 5)
    p = eb.params_config(63)
    elas.set_params(p)
    h1, h2 = elas.process(L, R)
    H, W = L.shape
    dl = torch.from_numpy(L).cuda()
    dr = torch.from_numpy(R).cuda()
    o1 = torch.empty((H, W), dtype=torch.float32, device="cuda")
    o2 = torch.empty_like(o1)
    torch.cuda.synchronize()
    elas.process_device(dl.data_ptr(), dr.data_ptr(), o1.data_ptr(), o2.data_ptr(), W, H,
                        stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert np.array_equal(o1.cpu().numpy(), h1) and np.array_equal(o2.cpu().numpy(), h2)


@pytest.mark.parametrize("shift", [1, 3])
def test_device_api_unaligned_images(elas, shift):
    """Device images that do not start on a 16-byte boundary take the
    descriptor's byte-wise staging; the result equals the host-buffer call
    (whose workspace copies are aligned)."""
    import torch

    L, R, _, _ = eb.synth_pair(3, 11, width=333, height=211, disp_max=95)
    p = eb.params_config(95)
    elas.set_params(p)
    h1, h2 = elas.process(L, R)
    H, W = L.shape
    bl = torch.zeros(H * W + 16, dtype=torch.uint8, device="cuda")
    br = torch.zeros_like(bl)
    bl[shift:shift + H * W] = torch.from_numpy(L.reshape(-1)).cuda()
    br[shift:shift + H * W] = torch.from_numpy(R.reshape(-1)).cuda()
    o1 = torch.empty((H, W), dtype=torch.float32, device="cuda")
    o2 = torch.empty_like(o1)
    torch.cuda.synchronize()
    elas.process_device(bl.data_ptr() + shift, br.data_ptr() + shift, o1.data_ptr(), o2.data_ptr(), W, H,
                        stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert np.array_equal(o1.cpu().numpy(), h1) and np.array_equal(o2.cpu().numpy(), h2)


def test_cpp_drop_in_class_runs(tmp_path):
    import os
    import subprocess

    from conftest import REPO
    exe = tmp_path / "demo"
    subprocess.run(["g++", "-std=c++17", "-I", os.path.join(REPO, "include"),
                    os.path.join(REPO, "tests", "native", "elas_class_demo.cpp"), "-o", str(exe),
                    "-L", os.path.dirname(eb.LIB_PATH), "-lelas_b200",
                    "-Wl,-rpath," + os.path.dirname(eb.LIB_PATH)], check=True)
    out = subprocess.run([str(exe), "run"], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "density" in out.stdout


def test_batch_device_graph_replay_equals_singles(elas):
    """Batched device call: the first call runs eagerly and captures a CUDA
    graph, the second (same buffers, new image contents) replays it; both
    must equal single-pair runs with each pair's own disparity range."""
    import torch

    shapes = [(320, 240, 64), (640, 480, 128), (480, 272, 256), (336, 256, 64)]
    p = eb.params_config(64)
    elas.set_params(p)
    bufs = []
    for (w, h, _) in shapes:
        bufs.append([torch.empty((h, w), dtype=torch.uint8, device="cuda"),
                     torch.empty((h, w), dtype=torch.uint8, device="cuda"),
                     torch.empty((h, w), dtype=torch.float32, device="cuda"),
                     torch.empty((h, w), dtype=torch.float32, device="cuda")])
    dims = [(w, h) for (w, h, _) in shapes]
    dmax = [d for (_, _, d) in shapes]
    elas.set_graphs(True)
    for seed in (11, 12, 13):
        pairs = [eb.synth_pair(3, seed * 10 + i, width=w, height=h, disp_max=d, gt=False)
                 for i, (w, h, d) in enumerate(shapes)]
        for b, (L, R, _, _) in zip(bufs, pairs):
            b[0].copy_(torch.from_numpy(L))
            b[1].copy_(torch.from_numpy(R))
        torch.cuda.synchronize()
        elas.process_batch_device([b[0].data_ptr() for b in bufs], [b[1].data_ptr() for b in bufs],
                                  [b[2].data_ptr() for b in bufs], [b[3].data_ptr() for b in bufs], dims, dmax)
        lat = elas.batch_latency(len(shapes))
        assert lat.shape == (len(shapes),) and (lat > 0).all()
        got = [(b[2].cpu().numpy(), b[3].cpu().numpy()) for b in bufs]
        for (L, R, _, _), d, (x1, x2) in zip(pairs, dmax, got):
            elas.set_params(eb.params_config(d))
            s1, s2 = elas.process(L, R)
            assert np.array_equal(s1, x1) and np.array_equal(s2, x2)
        elas.set_params(p)
    for (w, _, d) in shapes:
        assert elas.dense_shape(w, d) in (128, 256, 512, 1024)


def _read_pfm(path):
    with open(path, "rb") as f:
        assert f.readline().strip() == b"Pf"
        w, h = (int(x) for x in f.readline().split())
        assert float(f.readline()) < 0
        return np.frombuffer(f.read(), "<f4").reshape(h, w)[::-1]


def test_cli_matches_library(tmp_path):
    """The command-line front end on PGM files: its PFM output equals the
    library's maps for the same pair and parameters, bit for bit; the demo
    mode runs a synthetic pair and reports bad-2px."""
    import os
    import subprocess

    cli = os.path.join(os.path.dirname(eb.LIB_PATH), "elas_b200_cli")
    L, R, _, _ = eb.synth_pair(0, 7)
    for path, img in ((tmp_path / "l.pgm", L), (tmp_path / "r.pgm", R)):
        with open(path, "wb") as f:
            f.write(b"P5\n%d %d\n255\n" % (img.shape[1], img.shape[0]))
            f.write(img.tobytes())
    out = subprocess.run([cli, str(tmp_path / "l.pgm"), str(tmp_path / "r.pgm"), "--out", str(tmp_path / "o"),
                          "--disp-max", "63"], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    p = eb.params_default()
    p.disp_max = 63
    e = eb.Elas(p)
    try:
        D1, D2 = e.process(L, R)
    finally:
        e.close()
    assert np.array_equal(_read_pfm(tmp_path / "o_left.pfm"), D1)
    assert np.array_equal(_read_pfm(tmp_path / "o_right.pfm"), D2)
    assert (tmp_path / "o_left.pgm").stat().st_size == L.size + len(b"P5\n450 375\n255\n")
    out = subprocess.run([cli, "demo", "0", "--out", str(tmp_path / "demo")], capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "bad-2px" in out.stdout


@pytest.mark.parametrize("preset,seed,D,size", [(0, 3, 63, None), (1, 4, 255, None), (3, 9, 31, (97, 61))])
def test_subsampling_parity(elas, preset, seed, D, size):
    """Subsampling (every second row and column, the project's mode for the
    reference's declared-only parameter): stage-wise parity with the oracle,
    and the half-size dense maps equal the full-resolution ones at even
    pixels."""
    kw = dict(width=size[0], height=size[1], disp_max=D) if size else {}
    L, R, _, _ = eb.synth_pair(preset, seed, **kw)
    H, W = L.shape
    p = eb.params_config(D)
    p.subsampling = True
    D1, D2, g = run_and_compare(elas, L, R, p)
    assert D1.shape == (H // 2, W // 2) and D2.shape == (H // 2, W // 2)
    p.subsampling = False
    elas.set_params(p)
    elas.process(L, R)
    for k in ("disp_left", "disp_right"):
        full = elas.stage(k).view(np.float32).reshape(H, W)
        assert np.array_equal(g[k], full[0:2 * (H // 2):2, 0:2 * (W // 2):2]), k


@pytest.mark.parametrize("preset,seed,D", [(0, 11, 63), (1, 12, 255)])
def test_add_corners_parity(elas, preset, seed, D):
    """add_corners (the project's mode for the reference's declared-only
    parameter): the framed support list, both triangulations (exact check
    and Triangle), the priors and every later stage against the oracle."""
    L, R, _, _ = eb.synth_pair(preset, seed)
    H, W = L.shape
    p = eb.params_config(D)
    p.add_corners = True
    D1, D2, g = run_and_compare(elas, L, R, p)
    uvd = g["support"]
    assert uvd[:3, :2].tolist() == [[0, 0], [W - 1, 0], [W - 1 + int(uvd[2, 2]), 0]]
    assert uvd[-3:, 1].tolist() == [H - 1, H - 1, H - 1]


@pytest.mark.parametrize("preset", [1, 2])
def test_stars_match_host_emulation(elas, emu_lib, preset):
    """The star kernels (forced at 2880x1988, which takes the flips by
    default) give, list order included, the triangles of the sequential
    host emulation of the star construction: each search is a
    minimum under a strict total order, so how the lanes split the
    candidates cannot change it, and the list is in point order."""
    from test_delaunay_cpu import emu_star

    W, H, D = eb.synth_dims(preset)
    L, R, _, _ = eb.synth_pair(preset, 1)
    elas.set_params(eb.params_config(D))
    elas.set_test_mode(eb.Elas.TEST_DELAUNAY_STARS)
    try:
        elas.process(L, R)
    finally:
        elas.set_test_mode(0)
    uvd = elas.stage("support").view(np.int32).reshape(-1, 3)
    ctr = elas.stage("del_counters").view(np.int32).reshape(2, 16)
    for right, key in ((0, "tri_left"), (1, "tri_right")):
        xy = oracle.support_points(uvd, right)
        tris, st = emu_star(emu_lib, xy, uvd[:, 1] // 5)
        got = elas.stage(key).view(np.int32).reshape(-1, 3)
        assert ctr[right, 0] == tris.shape[0]
        assert np.array_equal(got, tris), key
        assert (ctr[right, 12], ctr[right, 13]) == (st[0], st[1]), (right, ctr[right], st)


@pytest.mark.parametrize("preset", [1, 2])
def test_flip_rounds_match_host_emulation(elas, emu_lib, preset):
    """The flip construction (forced): the flip kernels (one SM at 1242x375,
    a cluster at 2880x1988) take the same rounds and flips as the sequential
    host emulation of the algorithm: each round's outcome is fixed by the
    edge priorities, whatever the order in which threads reach the lists."""
    from test_delaunay_cpu import emu_triangulate

    W, H, D = eb.synth_dims(preset)
    L, R, _, _ = eb.synth_pair(preset, 1)
    elas.set_params(eb.params_config(D))
    elas.set_test_mode(eb.Elas.TEST_DELAUNAY_FLIPS)
    try:
        elas.process(L, R)
    finally:
        elas.set_test_mode(0)
    uvd = elas.stage("support").view(np.int32).reshape(-1, 3)
    ctr = elas.stage("del_counters").view(np.int32).reshape(2, 16)
    for right, key in ((0, "tri_left"), (1, "tri_right")):
        xy = oracle.support_points(uvd, right)
        tris, st = emu_triangulate(emu_lib, xy, uvd[:, 1] // 5)
        assert ctr[right, 0] == tris.shape[0]
        assert (ctr[right, 4], ctr[right, 5]) == (st[0], st[1]), (right, ctr[right], st)
        ok, stats = oracle.delaunay_check(xy, elas.stage(key).view(np.int32).reshape(-1, 3))
        assert ok, (key, stats)
