"""CPU checks of the oracle: arithmetic equivalences the CUDA kernels rely
on, the literal lane merge of the support sweep against the closed form the
kernels compute, and determinism of the full CPU pipeline."""
import numpy as np
import pytest

import oracle
import elas_b200 as eb


def test_sobel_integer_form_equals_reference_float_form():
    # reference: (uint8_t)(min(max(-128.f, s/4), 127.f) + 128)  (KerDescriptor.cu:40-41)
    s = np.arange(-1020, 1021, dtype=np.int32)
    f = (np.minimum(np.maximum(np.float32(-128), s.astype(np.float32) / np.float32(4)), np.float32(127))
         + np.float32(128)).astype(np.uint8)
    q = np.clip((s >> 2) + 128, 0, 255).astype(np.uint8)
    assert np.array_equal(f, q)


def test_support_threshold_float_equals_double_macro():
    # reference compares (float)E1 < SUPPORT_THRESHOLD*(float)E2 with the double
    # macro 0.85; the runtime parameter is the float 0.85f.  Same for all E.
    e2 = np.arange(0, 64 * 255 + 1, dtype=np.int64)
    t_f = np.float32(0.85) * e2.astype(np.float32)
    t_d = 0.85 * e2.astype(np.float64)
    first_fail_f = np.ceil(t_f.astype(np.float64))
    first_fail_d = np.ceil(t_d)
    assert np.array_equal(first_fail_f, first_fail_d)


def test_penalty_table_reference_values():
    p = eb.params_reference()
    assert [oracle.penalty(d, p) for d in range(3)] == [-14, -9, -2]


def _literal_merge(E, dmin, thr):
    """kerComputeSupportMatches' lane sweep + lane-0 merge, literally."""
    n = len(E)
    lanes = []
    for l in range(32):
        a1, b1, a2, b2 = 32767, -1, 32767, -1
        for k in range(l, n, 32):
            e, d = int(E[k]), dmin + k
            if e < a1:
                a2, b2, a1, b1 = a1, b1, e, d
            elif e < a2:
                a2, b2 = e, d
        lanes.append((a1, b1, a2, b2))
    M1E, M1d, M2E, M2d = lanes[0]
    for i in range(64):
        l = lanes[i >> 1]
        tE, td = (l[2], l[3]) if i & 1 else (l[0], l[1])
        if tE < M1E:
            M2E, M2d, M1E, M1d = M1E, M1d, tE, td
        elif tE < M2E:
            M2E, M2d = tE, td
    if M1d >= 0 and M2d >= 0 and np.float32(M1E) < np.float32(thr) * np.float32(M2E):
        return M1d
    return -1


def _closed_form(E, dmin, thr):
    """The commutative state the warp reduction computes."""
    e1, key, c, e2 = 1 << 31, 1 << 31, 0, 1 << 31
    for k, e in enumerate(E):
        e = int(e)
        d = dmin + k
        kk = ((k & 31) << 16) | d
        if e < e1:
            e2, e1, key, c = e1, e, kk, 1
        elif e == e1:
            c, e2, key = 2, e, min(key, kk)
        elif e < e2:
            e2 = e
    second = e1 if (c >= 2 or (key >> 16) == 0) else e2
    if c >= 1 and np.float32(e1) < np.float32(thr) * np.float32(second):
        return key & 0xFFFF
    return -1


@pytest.mark.parametrize("thr", [0.85, 0.95, 1.3])
def test_support_merge_closed_form(thr):
    rng = np.random.default_rng(7)
    for it in range(600):
        n = int(rng.integers(11, 140))
        dmin = int(rng.integers(0, 3))
        E = rng.integers(0, 60, size=n)
        if it % 3 == 0:          # force a unique clear minimum
            E[rng.integers(0, n)] = 0
        if it % 5 == 0:          # force a tie
            i, j = rng.integers(0, n, 2)
            E[j] = E[i]
        if it % 7 == 0:          # unique minimum in lane 0
            E[32 * int(rng.integers(0, (n + 31) // 32)) % n] = -1
            E = E + 1
        assert _literal_merge(E, dmin, thr) == _closed_form(E, dmin, thr), (it, list(E))


def _numpy_descriptor(img):
    I = img.astype(np.int32)
    H, W = I.shape
    du = np.zeros((H, W), np.int32)
    dv = np.zeros((H, W), np.int32)
    c = I[1:-1, :-2] * 0
    sdu = (I[:-2, :-2] + 2 * I[1:-1, :-2] + I[2:, :-2] - I[:-2, 2:] - 2 * I[1:-1, 2:] - I[2:, 2:])
    sdv = (I[:-2, :-2] + 2 * I[:-2, 1:-1] + I[:-2, 2:] - I[2:, :-2] - 2 * I[2:, 1:-1] - I[2:, 2:])
    du[1:-1, 1:-1] = np.clip((sdu >> 2) + 128, 0, 255)
    dv[1:-1, 1:-1] = np.clip((sdv >> 2) + 128, 0, 255)
    del c
    taps = [(du, 0, -2), (du, -2, -1), (du, 0, -1), (du, 2, -1), (du, -1, 0), (du, 0, 0), (du, 0, 0), (du, 1, 0),
            (du, -2, 1), (du, 0, 1), (du, 2, 1), (du, 0, 2), (dv, 0, -1), (dv, -1, 0), (dv, 1, 0), (dv, 0, 1)]
    out = np.zeros((H, W, 16), np.uint8)
    for k, (a, dx, dy) in enumerate(taps):
        out[3:H - 3, 3:W - 3, k] = a[3 + dy:H - 3 + dy, 3 + dx:W - 3 + dx]
    return out


def test_descriptor_against_numpy_restatement():
    rng = np.random.default_rng(3)
    img = rng.integers(0, 256, size=(37, 53), dtype=np.uint8)
    assert np.array_equal(oracle.descriptor(img), _numpy_descriptor(img))


def test_oracle_pipeline_deterministic_and_thread_independent():
    L, R, gt, _ = eb.synth_pair(0, 11)
    p = eb.params_config(63)
    a1, a2, _ = oracle.process(L, R, p, threads=1)
    b1, b2, _ = oracle.process(L, R, p, threads=4)
    assert np.array_equal(a1, b1) and np.array_equal(a2, b2)
    valid = a1 >= 0
    assert valid.mean() > 0.5
    bad = np.abs(a1 - gt) > 2
    assert (bad & valid).sum() / valid.sum() < 0.2


@pytest.mark.skipif(not oracle.have_triangle(), reason="reference Triangle not built")
def test_triangle_known_answers():
    sq = np.array([[0, 0], [10, 0], [10, 10], [0, 10], [5, 5]], np.float32)
    t = oracle.triangulate_ref(sq)
    assert t.shape == (4, 3)
    ok, st = oracle.delaunay_check(sq.astype(np.int32), t)
    assert ok, st
    line = np.array([[0, 0], [5, 0], [10, 0], [15, 0]], np.float32)
    assert oracle.triangulate_ref(line).shape[0] == 0
    dup = np.array([[0, 0], [10, 0], [0, 10], [10, 0]], np.float32)
    t = oracle.triangulate_ref(dup)
    assert t.shape[0] == 1


def test_subsampling_keeps_every_second_pixel():
    """Subsampling in the oracle: the maps before the L/R check are the
    full-resolution dense maps at even rows and columns; the L/R check and
    the post-filters then run on the half-size maps."""
    L, R, _, _ = eb.synth_pair(0, 5)
    H, W = L.shape
    p = eb.params_config(63)
    _, _, full = oracle.process(L, R, p, dumps=True)
    p.subsampling = True
    D1, D2, sub = oracle.process(L, R, p, tri_left=full["tri_left"], tri_right=full["tri_right"], dumps=True)
    assert D1.shape == (H // 2, W // 2) and D2.shape == (H // 2, W // 2)
    assert np.array_equal(sub["disp_left"], full["disp_left"][0:2 * (H // 2):2, 0:2 * (W // 2):2])
    assert np.array_equal(sub["disp_right"], full["disp_right"][0:2 * (H // 2):2, 0:2 * (W // 2):2])
    # L/R on the half-size maps warps by d / 2
    a, b = sub["disp_left"], sub["disp_right"]
    exp = a.copy()
    for v in range(a.shape[0]):
        for u in range(a.shape[1]):
            d = a[v, u]
            uw = np.float32(u) - d * np.float32(0.5)
            if not (d >= 0 and 0 <= uw < a.shape[1]) or abs(b[v, int(uw)] - d) > p.lr_threshold:
                exp[v, u] = -1
    assert np.array_equal(sub["lr_left"], exp)


def test_add_corners_support_list():
    """add_corners in the oracle: the regular list is framed by the corner
    points (row 0's three first, row H-1's three last) with the disparity of
    the nearest support point, the right corners also moved by it.  (The
    triangulation of the framed list is checked on the GPU algorithm's
    emulation in test_delaunay_cpu.py.)"""
    L, R, _, _ = eb.synth_pair(0, 6)
    H, W = L.shape
    p = eb.params_config(63)
    _, _, a = oracle.process(L, R, p, dumps=True)
    p.add_corners = True
    _, _, b = oracle.process(L, R, p, dumps=True)
    reg, sb = a["support"], b["support"]
    assert len(sb) == len(reg) + 6
    assert np.array_equal(sb[3:-3], reg)

    def nearest(u, v):
        dist = (reg[:, 0].astype(np.int64) - u) ** 2 + (reg[:, 1].astype(np.int64) - v) ** 2
        return int(reg[np.argmin(dist), 2])          # argmin: the first minimum in list order

    d = [nearest(0, 0), nearest(W - 1, 0), nearest(0, H - 1), nearest(W - 1, H - 1)]
    assert sb[:3].tolist() == [[0, 0, d[0]], [W - 1, 0, d[1]], [W - 1 + d[1], 0, d[1]]]
    assert sb[-3:].tolist() == [[0, H - 1, d[2]], [W - 1, H - 1, d[3]], [W - 1 + d[3], H - 1, d[3]]]
