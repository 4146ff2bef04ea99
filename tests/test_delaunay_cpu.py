"""The GPU Delaunay algorithm (delaunay_core.h), run by its sequential host
emulation, against the exact checker and the reference's Triangle."""
import ctypes

import numpy as np
import pytest

import oracle
import elas_b200 as eb


def emu_triangulate(lib, xy, row_of, phased=False):
    """xy: (n,2) int32 in lattice-row order; row_of: lattice row per point.
    phased: run the flips in the three-phase round formulation of the
    one-SM and cluster kernels instead of the worklist formulation."""
    n = xy.shape[0]
    nrows = int(row_of.max()) + 1 if n else 1
    row_off = np.zeros(nrows + 1, np.int32)
    np.add.at(row_off, row_of + 1, 1)
    row_off = np.cumsum(row_off).astype(np.int32)
    x = np.ascontiguousarray(xy[:, 0], np.int32)
    y = np.ascontiguousarray(xy[:, 1], np.int32)
    cap = 2 * n + 16
    out = np.zeros((cap, 3), np.int32)
    st = np.zeros(2, np.int64)
    fn = lib.emu_delaunay_phased if phased else lib.emu_delaunay
    T = fn(x.ctypes.data_as(ctypes.c_void_p), y.ctypes.data_as(ctypes.c_void_p), n,
           row_off.ctypes.data_as(ctypes.c_void_p), nrows, out.ctypes.data_as(ctypes.c_void_p), cap,
           st.ctypes.data_as(ctypes.c_void_p))
    assert T >= 0
    return out[:T], st


def emu_star(lib, xy, row_of):
    """The star construction (the hull in k_plan, k_star and its scan and
    emit kernels), run point by point on the host: (triangles in point
    order, [phase-2 searches, squares grown, candidates examined outside the
    staged windows])."""
    n = xy.shape[0]
    nrows = int(row_of.max()) + 1 if n else 1
    row_off = np.zeros(nrows + 1, np.int32)
    np.add.at(row_off, row_of + 1, 1)
    row_off = np.cumsum(row_off).astype(np.int32)
    x = np.ascontiguousarray(xy[:, 0], np.int32)
    y = np.ascontiguousarray(xy[:, 1], np.int32)
    cap = 2 * n + 16
    out = np.zeros((cap, 3), np.int32)
    st = np.zeros(3, np.int64)
    T = lib.emu_delaunay_star(x.ctypes.data_as(ctypes.c_void_p), y.ctypes.data_as(ctypes.c_void_p), n,
                              row_off.ctypes.data_as(ctypes.c_void_p), nrows, out.ctypes.data_as(ctypes.c_void_p),
                              cap, st.ctypes.data_as(ctypes.c_void_p))
    assert T >= 0
    return out[:T], st


def check_case(lib, xy, row_of, compare=True):
    """Both constructions (strips and flips; stars): each passes the exact
    check (and matches Triangle up to co-circular ties), and they give the
    same triangle set; the stars' list is in point order with every
    triangle starting at its smallest vertex."""
    tris, st = emu_triangulate(lib, xy, row_of)
    stars, _ = emu_star(lib, xy, row_of)
    for t in (tris, stars):
        ok, stats = oracle.delaunay_check(xy, t)
        assert ok, stats
        if compare and oracle.have_triangle() and xy.shape[0] >= 3:
            ref = oracle.triangulate_ref(xy.astype(np.float32))
            assert ref.shape[0] == t.shape[0]
            cmp = oracle.tri_compare(xy, t, ref)
            assert cmp[4] == 0, cmp      # every difference is a co-circular tie
    assert {tuple(t) for t in tris.tolist()} == {tuple(t) for t in stars.tolist()}
    if stars.shape[0]:
        assert (stars[:, 0] < stars[:, 1]).all() and (stars[:, 0] < stars[:, 2]).all()
        assert (np.diff(stars[:, 0]) >= 0).all()
    return tris


def lattice_points(rng, rows, cols, step, keep, jitter_d=0):
    pts, row_of = [], []
    for r in range(rows):
        for c in range(cols):
            if rng.random() < keep:
                d = int(rng.integers(0, jitter_d + 1)) if jitter_d else 0
                pts.append((c * step - d, r * step))
                row_of.append(r)
    return np.array(pts, np.int32).reshape(-1, 2), np.array(row_of, np.int64)


@pytest.mark.parametrize("preset", [0, 1])
def test_support_points_of_synthetic_pairs(emu_lib, preset):
    L, R, _, _ = eb.synth_pair(preset, 5)
    p = eb.params_config(eb.synth_dims(preset)[2])
    _, _, st = oracle.process(L, R, p, dumps=True)
    uvd = st["support"]
    for right in (0, 1):
        check_case(emu_lib, oracle.support_points(uvd, right), uvd[:, 1] // 5)


@pytest.mark.parametrize("keep", [1.0, 0.6, 0.2, 0.05])
def test_lattice_subsets_cocircular_heavy(emu_lib, keep):
    rng = np.random.default_rng(int(keep * 100))
    xy, row_of = lattice_points(rng, 30, 40, 5, keep)
    if xy.shape[0] >= 3:
        check_case(emu_lib, xy, row_of)


def test_shifted_rows_with_duplicates(emu_lib):
    rng = np.random.default_rng(1)
    xy, row_of = lattice_points(rng, 25, 30, 5, 0.7, jitter_d=12)
    assert len(np.unique(xy, axis=0)) < len(xy)          # duplicates present
    check_case(emu_lib, xy, row_of)


def test_degenerate_inputs(emu_lib):
    for build in (emu_triangulate, emu_star):
        # one row: collinear -> no triangles
        xy = np.array([[0, 0], [5, 0], [10, 0]], np.int32)
        tris, _ = build(emu_lib, xy, np.zeros(3, np.int64))
        assert tris.shape[0] == 0
        # two points, one point, nothing
        for n in (0, 1, 2):
            xy = np.array([[5 * i, 5 * i] for i in range(n)], np.int32).reshape(-1, 2)
            tris, _ = build(emu_lib, xy, np.arange(n))
            assert tris.shape[0] == 0
        # single-point rows on a vertical line -> collinear
        xy = np.array([[10, 5 * i] for i in range(6)], np.int32)
        tris, _ = build(emu_lib, xy, np.arange(6))
        assert tris.shape[0] == 0
    # a column of single points with wide rows above and below
    xy = np.array([[0, 0], [100, 0], [50, 5], [50, 10], [0, 15], [100, 15]], np.int32)
    check_case(emu_lib, xy, np.array([0, 0, 1, 2, 3, 3]))


def test_random_large(emu_lib):
    rng = np.random.default_rng(9)
    xy, row_of = lattice_points(rng, 120, 150, 5, 0.3, jitter_d=40)
    check_case(emu_lib, xy, row_of)


def test_stars_across_empty_regions_and_rings(emu_lib):
    """Cases for the star windows: clusters far apart (nearest neighbours
    and circles beyond the first windows, hull edges proven over every
    point), a ring of co-circular lattice points around an empty disc with
    one point at its centre (a high degree and ties broken by the
    perturbation), and a long thin hull (huge circumcircles)."""
    rng = np.random.default_rng(21)
    pts = []
    for cx, cy in ((20, 20), (400, 30), (60, 300), (500, 280)):
        for _ in range(40):
            pts.append((cx + 5 * int(rng.integers(-4, 5)), cy + 5 * int(rng.integers(-4, 5))))
    ring = [(300 + x, 200 + y) for x in range(-50, 51, 5) for y in range(-50, 51, 5)
            if 48 ** 2 <= x * x + y * y <= 50 ** 2]
    pts += ring + [(300, 200)]
    pts += [(x, 600) for x in range(0, 900, 5)] + [(450, 605)]
    xy = np.array(sorted(set(pts), key=lambda q: (q[1], q[0])), np.int32)
    row_of = xy[:, 1] // 5
    _, st = emu_star(emu_lib, xy, row_of)
    assert st[1] > 0 and st[2] > 0      # windows grew and searched beyond the first square
    check_case(emu_lib, xy, row_of)


def test_parallel_hull_test_equals_stack_walk(emu_lib):
    """The device decides the hull chains point by point (hull_on_chain);
    the stack walk (hull_chain) must keep the same points, collinear runs
    included, on random chains, lattice chains with many collinear points
    and chains with repeated x."""
    rng = np.random.default_rng(5)
    for it in range(300):
        R = int(rng.integers(1, 60))
        ys = np.sort(rng.choice(np.arange(0, 5 * 200, 5), size=R, replace=False)).astype(np.int32)
        if it % 3 == 0:
            xs = (5 * rng.integers(0, 6, size=R)).astype(np.int32)       # few columns: collinear runs
        elif it % 3 == 1:
            xs = rng.integers(-300, 300, size=R).astype(np.int32)
        else:
            xs = (np.abs(np.arange(R) - R // 2) * 5 + rng.integers(0, 2, size=R)).astype(np.int32)
        for side in (0, 1):
            assert emu_lib.emu_hull_agree(xs.ctypes.data_as(ctypes.c_void_p), ys.ctypes.data_as(ctypes.c_void_p),
                                          R, side) == 1, (it, side, xs.tolist(), ys.tolist())


@pytest.mark.parametrize("preset", [0, 1])
def test_support_points_with_corners(emu_lib, preset):
    """The GPU algorithm with add_corners: the corner points of row 0 join
    lattice row 0, those of row H-1 form one more row after the lattice."""
    W, H, D = eb.synth_dims(preset)
    L, R, _, _ = eb.synth_pair(preset, 2)
    p = eb.params_config(D)
    p.add_corners = True
    _, _, st = oracle.process(L, R, p, dumps=True)
    uvd = st["support"]
    ch = H // p.candidate_stepsize
    row_of = np.where(uvd[:, 1] == H - 1, ch, uvd[:, 1] // p.candidate_stepsize)
    for right in (0, 1):
        check_case(emu_lib, oracle.support_points(uvd, right), row_of)


def test_packed_predicates_exact_at_the_size_limits(emu_lib):
    """orient_p / incircle_p against Python integers over the coordinate
    range the size limits allow: x in [-4095, 13999] (right view: u - d with
    disp_max <= 4095, width <= 14000), y in [0, 16383] (height <= 16384)."""
    import ctypes

    emu_lib.emu_orient_p.restype = ctypes.c_longlong
    emu_lib.emu_incircle_p.restype = ctypes.c_longlong
    rng = np.random.default_rng(7)
    lo, hi = np.array([-4095, 0]), np.array([13999, 16383])
    for it in range(4000):
        if it % 4 == 0:      # corners of the range: the largest terms
            pts = np.stack([np.where(rng.random(2) < 0.5, lo, hi) for _ in range(4)])
        else:
            pts = rng.integers(lo, hi + 1, size=(4, 2))
        pts = pts.astype(np.int32)
        (ax, ay), (bx, by), (cx, cy), (dx, dy) = [tuple(int(v) for v in p) for p in pts]
        o = (bx - ax) * (cy - ay) - (by - ay) * (cx - ax)
        adx, ady, bdx, bdy, cdx, cdy = ax - dx, ay - dy, bx - dx, by - dy, cx - dx, cy - dy
        det = (adx * (bdy * (cdx * cdx + cdy * cdy) - (bdx * bdx + bdy * bdy) * cdy)
               - ady * (bdx * (cdx * cdx + cdy * cdy) - (bdx * bdx + bdy * bdy) * cdx)
               + (adx * adx + ady * ady) * (bdx * cdy - bdy * cdx))
        buf = np.ascontiguousarray(pts.reshape(-1))
        assert emu_lib.emu_orient_p(buf.ctypes.data_as(ctypes.c_void_p)) == o
        assert emu_lib.emu_incircle_p(buf.ctypes.data_as(ctypes.c_void_p)) == det


def test_three_phase_rounds_equal_worklist_rounds(emu_lib):
    """The flip kernels run each round as flip / resolve-and-propose /
    relink-and-repropose, testing the next round's edges while resolving.
    That formulation must make the same flips in every round as the
    propose / flip / resolve / relink worklist one: same triangles in the
    same slots, same rounds, same flips."""
    sets = []
    for preset in (0, 1):
        L, R, _, _ = eb.synth_pair(preset, 3)
        p = eb.params_config(eb.synth_dims(preset)[2])
        _, _, st = oracle.process(L, R, p, dumps=True)
        uvd = st["support"]
        for right in (0, 1):
            sets.append((oracle.support_points(uvd, right), uvd[:, 1] // 5))
    rng = np.random.default_rng(11)
    for keep in (1.0, 0.5, 0.1):
        sets.append(lattice_points(rng, 30, 40, 5, keep, jitter_d=8))
    for xy, row_of in sets:
        if xy.shape[0] < 3:
            continue
        t0, s0 = emu_triangulate(emu_lib, xy, row_of)
        t1, s1 = emu_triangulate(emu_lib, xy, row_of, phased=True)
        assert np.array_equal(t0, t1)
        assert tuple(s0) == tuple(s1)
