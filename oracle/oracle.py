"""ORACLE -- test infrastructure only.

ctypes binding of oracle/liboracle.so (the CPU restatement of the reference
pipeline, elas_oracle.cpp) and of the reference's own Triangle
(oracle/_ref/libreftriangle.so).  Only tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg use it, always as the checker.
"""
import ctypes
import os
import sys
from ctypes import POINTER, c_int, c_int32, c_longlong, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(REPO, "cuda-stereo-matching_b200"))
from elas_b200 import ElasParams  # noqa: E402  (pure ctypes struct, does not load the product library)

LIB = os.path.join(HERE, "liboracle.so")
REF_TRI = os.path.join(HERE, "_ref", "libreftriangle.so")
REF_ELAS = os.path.join(HERE, "_ref", "libelasref.so")


class Dumps(ctypes.Structure):
    _fields_ = [("desc_left", c_void_p), ("desc_right", c_void_p), ("can_lr", c_void_p), ("can", c_void_p),
                ("support", c_void_p), ("n_support", c_void_p), ("grid_left", c_void_p), ("grid_right", c_void_p),
                ("tri_left", c_void_p), ("n_tri_left", c_void_p), ("tri_right", c_void_p),
                ("n_tri_right", c_void_p), ("tri_cap", c_int32), ("prior_left", c_void_p),
                ("prior_right", c_void_p), ("disp_left", c_void_p), ("disp_right", c_void_p),
                ("lr_left", c_void_p), ("lr_right", c_void_p)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            sys.path.insert(0, HERE)
            import build_oracle
            build_oracle.build_oracle()
        l = ctypes.CDLL(LIB)
        l.orc_incircle.restype = c_longlong
        if os.path.exists(REF_TRI):
            l.orc_load_triangle(REF_TRI.encode())
        _lib = l
    return _lib


def have_triangle():
    return os.path.exists(REF_TRI)


_ref_elas = None


def have_ref_elas():
    return os.path.exists(REF_ELAS)


def ref_elas_process(left, right):
    """The reference's own GPU pipeline (Elas::process built from the
    reference tree; needs a GPU).  Its kernels use the compile-time
    constants of src/Kernels/KernelsCommon.h and it stops after the L/R
    check.  Returns (D1, D2) float32."""
    global _ref_elas
    if _ref_elas is None:
        _ref_elas = ctypes.CDLL(REF_ELAS)
    left = np.ascontiguousarray(left, np.uint8)
    right = np.ascontiguousarray(right, np.uint8)
    H, W = left.shape
    D1 = np.empty((H, W), np.float32)
    D2 = np.empty((H, W), np.float32)
    rc = _ref_elas.ref_elas_process(P(left), P(right), P(D1), P(D2), W, H)
    if rc != 0:
        raise RuntimeError(f"reference pipeline failed with status {rc}")
    return D1, D2


def P(a):
    return a.ctypes.data_as(c_void_p)


# ---- parameter presets and benchmark inputs without the product library ----
# (the benchmark's CPU baseline and reference arm use these, so they load
# only oracle libraries)

def params_reference():
    """The constants the reference kernels are compiled with
    (src/Kernels/KernelsCommon.h:8-27) on the Elas::parameters layout, every
    post-filter off (the reference's process() stops after the left/right
    check, src/Elas.cu:107-119).  Equal to the library's
    elas_params_reference(); the tests compare the two."""
    p = ElasParams()
    p.disp_min, p.disp_max = 0, 255
    p.support_threshold, p.support_texture, p.candidate_stepsize = 0.85, 10, 5
    p.incon_window_size, p.incon_threshold, p.incon_min_support = 5, 5, 5
    p.add_corners, p.grid_size = False, 20
    p.beta, p.gamma, p.sigma, p.sradius = 0.02, 3.0, 1.0, 2.0
    p.match_texture, p.lr_threshold, p.speckle_sim_threshold = 0, 2, 1.0
    p.speckle_size, p.ipol_gap_width = 0, 0
    p.filter_median = p.filter_adaptive_mean = p.postprocess_only_left = p.subsampling = False
    return p


def params_config(disp_max, post=True):
    """The benchmark configurations' parameters: the reference constants with
    the configured disparity range, post-filters (speckle 200, gap width 3,
    median and adaptive mean) on unless post is False."""
    p = params_reference()
    p.disp_max = int(disp_max)
    if post:
        p.speckle_size, p.ipol_gap_width = 200, 3
        p.filter_median = p.filter_adaptive_mean = True
    return p


def synth_dims(preset):
    w, h, d = c_int32(), c_int32(), c_int32()
    if lib().elas_b200_synth_dims(preset, ctypes.byref(w), ctypes.byref(h), ctypes.byref(d)) != 0:
        raise RuntimeError(f"unknown scene preset {preset}")
    return w.value, h.value, d.value


def synth_pair(preset, seed, width=0, height=0, disp_max=0, gt=True):
    """The seeded synthetic pair of the benchmark (the same generator source
    as the product's, compiled into the oracle library):
    (left, right, gt_left, gt_right), the ground truths None unless gt."""
    W, H, _ = synth_dims(preset)
    W, H = width or W, height or H
    left = np.empty((H, W), np.uint8)
    right = np.empty((H, W), np.uint8)
    gl = np.empty((H, W), np.float32) if gt else None
    gr = np.empty((H, W), np.float32) if gt else None
    rc = lib().elas_b200_synth_pair(preset, ctypes.c_uint64(seed), W, H, disp_max, P(left), P(right),
                                    P(gl) if gt else None, P(gr) if gt else None)
    if rc != 0:
        raise RuntimeError(f"synthetic pair failed with status {rc}")
    return left, right, gl, gr


def geom(W, H, p):
    cw, ch = W // p.candidate_stepsize, H // p.candidate_stepsize
    gw = int(np.ceil(np.float32(W) / np.float32(p.grid_size)))
    gh = int(np.ceil(np.float32(H) / np.float32(p.grid_size)))
    return cw, ch, gw, gh


def descriptor(img):
    img = np.ascontiguousarray(img, np.uint8)
    H, W = img.shape
    out = np.empty((H, W, 16), np.uint8)
    assert lib().orc_descriptor(P(img), W, H, P(out)) == 0
    return out


def support_sweep(d0, d1, p):
    H, W = d0.shape[:2]
    cw, ch, _, _ = geom(W, H, p)
    can = np.empty((ch, cw), np.int32)
    assert lib().orc_support_sweep(P(d0), P(d1), W, H, ctypes.byref(p), P(can)) == 0
    return can


def filter_inconsistent(can, p):
    c = np.ascontiguousarray(can, np.int32).copy()
    assert lib().orc_filter_inconsistent(P(c), c.shape[1], c.shape[0], ctypes.byref(p)) == 0
    return c


def filter_redundant(can):
    c = np.ascontiguousarray(can, np.int32).copy()
    assert lib().orc_filter_redundant(P(c), c.shape[1], c.shape[0]) == 0
    return c


def support_list(can, step):
    can = np.ascontiguousarray(can, np.int32)
    n = lib().orc_support_list(P(can), can.shape[1], can.shape[0], step, None)
    out = np.empty((max(n, 0), 3), np.int32)
    lib().orc_support_list(P(can), can.shape[1], can.shape[0], step, P(out))
    return out


def grid(can, W, H, p):
    _, _, gw, gh = geom(W, H, p)
    g0 = np.empty((gh, gw, p.disp_max + 2), np.int32)
    g1 = np.empty_like(g0)
    assert lib().orc_grid(P(np.ascontiguousarray(can, np.int32)), W, H, ctypes.byref(p), P(g0), P(g1)) == 0
    return g0, g1


def triangulate_ref(xy):
    """The reference's Triangle ("zQB") on float points (n, 2)."""
    xy = np.ascontiguousarray(xy, np.float32)
    n = xy.shape[0]
    cap = 2 * n + 16
    out = np.empty((cap, 3), np.int32)
    t = lib().orc_triangulate_ref(P(xy), n, P(out), cap)
    if t < 0:
        raise RuntimeError("Triangle unavailable")
    return out[:t].copy()


def prior(can, uvd, tris, right, W, H, step):
    can = np.ascontiguousarray(can, np.int32)
    uvd = np.ascontiguousarray(uvd, np.int32)
    tris = np.ascontiguousarray(tris, np.int32).reshape(-1, 3)
    out = np.empty((H, W), np.int32)
    assert lib().orc_prior(P(can), can.shape[1], step, P(uvd), P(tris), tris.shape[0], int(right), W, H,
                           P(out)) == 0
    return out


def dense(grid_arr, d0, d1, prior_arr, right, p):
    H, W = d0.shape[:2]
    out = np.empty((H, W), np.float32)
    assert lib().orc_dense(P(np.ascontiguousarray(grid_arr, np.int32)), P(d0), P(d1),
                           P(np.ascontiguousarray(prior_arr, np.int32)), int(right), W, H, ctypes.byref(p),
                           P(out)) == 0
    return out


def lr(D1, D2, p):
    a = np.ascontiguousarray(D1, np.float32).copy()
    b = np.ascontiguousarray(D2, np.float32).copy()
    assert lib().orc_lr(P(a), P(b), a.shape[1], a.shape[0], ctypes.byref(p)) == 0
    return a, b


def postprocess(D, p):
    a = np.ascontiguousarray(D, np.float32).copy()
    assert lib().orc_postprocess(P(a), a.shape[1], a.shape[0], ctypes.byref(p)) == 0
    return a


def penalty(dd, p):
    return lib().orc_penalty(dd, ctypes.byref(p))


def process(left, right, p, tri_left=None, tri_right=None, dumps=False, threads=0):
    """Full CPU pipeline.  Returns (D1, D2, stages dict or None)."""
    left = np.ascontiguousarray(left, np.uint8)
    right = np.ascontiguousarray(right, np.uint8)
    H, W = left.shape
    cw, ch, gw, gh = geom(W, H, p)
    D1 = np.empty((H, W), np.float32)
    D2 = np.empty((H, W), np.float32)
    tl = np.ascontiguousarray(tri_left, np.int32).reshape(-1, 3) if tri_left is not None else None
    tr = np.ascontiguousarray(tri_right, np.int32).reshape(-1, 3) if tri_right is not None else None
    st = None
    dp = None
    if dumps:
        cap = 2 * (cw * ch + 6) + 16
        st = {"desc_left": np.empty((H, W, 16), np.uint8), "desc_right": np.empty((H, W, 16), np.uint8),
              "can_lr": np.empty((ch, cw), np.int32), "can": np.empty((ch, cw), np.int32),
              "support": np.empty((cw * ch + 6, 3), np.int32), "n_support": np.zeros(1, np.int32),
              "grid_left": np.empty((gh, gw, p.disp_max + 2), np.int32),
              "grid_right": np.empty((gh, gw, p.disp_max + 2), np.int32),
              "tri_left": np.empty((cap, 3), np.int32), "n_tri_left": np.zeros(1, np.int32),
              "tri_right": np.empty((cap, 3), np.int32), "n_tri_right": np.zeros(1, np.int32),
              "prior_left": np.empty((H, W), np.int32), "prior_right": np.empty((H, W), np.int32),
              "disp_left": np.empty((H, W), np.float32), "disp_right": np.empty((H, W), np.float32),
              "lr_left": np.empty((H, W), np.float32), "lr_right": np.empty((H, W), np.float32)}
        dp = Dumps(*[P(st[k]) for k in ["desc_left", "desc_right", "can_lr", "can", "support", "n_support",
                                         "grid_left", "grid_right", "tri_left", "n_tri_left", "tri_right",
                                         "n_tri_right"]], cap,
                   *[P(st[k]) for k in ["prior_left", "prior_right", "disp_left", "disp_right", "lr_left",
                                        "lr_right"]])
    rc = lib().orc_process(P(left), P(right), W, H, ctypes.byref(p), P(tl) if tl is not None else None,
                           tl.shape[0] if tl is not None else 0, P(tr) if tr is not None else None,
                           tr.shape[0] if tr is not None else 0, P(D1), P(D2),
                           ctypes.byref(dp) if dp is not None else None, threads)
    if rc != 0:
        raise RuntimeError(f"oracle failed with status {rc}")
    if st is not None:
        st["support"] = st["support"][:st["n_support"][0]]
        st["tri_left"] = st["tri_left"][:st["n_tri_left"][0]]
        st["tri_right"] = st["tri_right"][:st["n_tri_right"][0]]
    if p.subsampling:   # (H / 2) x (W / 2) maps in the leading values
        Ho, Wo = H // 2, W // 2
        D1 = D1.reshape(-1)[:Ho * Wo].reshape(Ho, Wo).copy()
        D2 = D2.reshape(-1)[:Ho * Wo].reshape(Ho, Wo).copy()
        if st is not None:
            for k in ("disp_left", "disp_right", "lr_left", "lr_right"):
                st[k] = st[k].reshape(-1)[:Ho * Wo].reshape(Ho, Wo).copy()
    return D1, D2, st


def delaunay_check(xy, tris):
    """Exact checks (int64, symbolic perturbation); returns (ok, stats[8])."""
    xy = np.ascontiguousarray(xy, np.int32)
    tris = np.ascontiguousarray(tris, np.int32).reshape(-1, 3)
    stats = np.zeros(8, np.int64)
    rc = lib().orc_delaunay_check(P(xy), xy.shape[0], P(tris), tris.shape[0], P(stats))
    return rc == 0, stats


def tri_compare(xy, a, b):
    """stats: [common, only_a, only_b, differing explained by co-circularity, unexplained]."""
    xy = np.ascontiguousarray(xy, np.int32)
    a = np.ascontiguousarray(a, np.int32).reshape(-1, 3)
    b = np.ascontiguousarray(b, np.int32).reshape(-1, 3)
    stats = np.zeros(5, np.int64)
    lib().orc_tri_compare(P(xy), xy.shape[0], P(a), a.shape[0], P(b), b.shape[0], P(stats))
    return stats


def support_points(uvd, right):
    """(n, 2) int32 point coordinates of one view from the support list."""
    xy = np.stack([uvd[:, 0] - (uvd[:, 2] if right else 0), uvd[:, 1]], 1)
    return np.ascontiguousarray(xy, np.int32)
