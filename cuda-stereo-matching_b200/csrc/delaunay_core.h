// Delaunay triangulation of the support points with exact int64 predicates.
//
// Replaces the reference's CPU round trip through Shewchuk's Triangle
// (Elas::computeDelaunyTrianguation, src/Elas.cu:282-328).
//
// Algorithm (all steps data-parallel except two short serial chains):
//  1. Per candidate row, sort the row's points by x and drop duplicated
//     coordinates (the lowest support index of a group is kept; Triangle
//     keeps the first of its randomised sort, src/triangle.cpp divconqdelaunay).
//  2. Insert the points row by row: the strip between two consecutive
//     non-empty rows is triangulated by merging the two rows by x; every
//     point finds its own triangle by a binary search in the other row
//     (merge path), so the strips are built fully in parallel.
//  3. Fill the pockets between the rows' first (last) points and the convex
//     hull with the monotone-chain stack walk.
//  4. Build edge adjacency with an open-addressing hash of undirected edges.
//  5. Lawson edge flipping in rounds driven by a worklist: round 0 tests
//     every interior edge; later rounds test only the four outer edges of
//     each quad flipped in the previous round and the proposals that lost
//     their lock.  An edge flips when it holds the minimum priority on both
//     of its triangles; neighbour links are repaired through a forwarding
//     table in two phases (resolve, then write).  Converges to the unique
//     Delaunay triangulation under the symbolic perturbation below.
//
// Predicates: orientation and incircle on integer coordinates, exact in
// int32 / int64 arithmetic for the library's image limits (pack_xy below).
// Ties (four
// co-circular points) are broken by simulation of simplicity: point i is
// lifted to x^2+y^2 - eps^(i+1); then d is inside circle(a,b,c) iff the
// lowest index m of {a,b,c,d} is d, or d's barycentric coordinate for m is
// negative.  That makes the triangulation unique, and equal to Triangle's
// wherever no four points are co-circular.
//
// Everything here is __host__ __device__ so the same code runs in a
// sequential host emulation used by the CPU tests.
#pragma once

#include <cstdint>
#include "common.cuh"

namespace elas {
namespace del {

struct Pts {
    const int32_t* x;
    const int32_t* y;
};

// Strip between an upper row A[0..m) and a lower row B[0..n), both sorted
// by strictly increasing x: walking the merge of A[1..m) and B[1..n) by x
// (A first on equal x), each element advances its row by one point and
// creates one counter-clockwise triangle.  These two functions give the
// triangle of one element and its position in the strip, so every point
// can emit its triangles independently.
//
// Number of elements of the sorted X[0..n) with x < v (strict) or x <= v.
HD int count_below(Pts P, const int32_t* X, int n, int32_t v, bool inclusive) {
    int lo = 0, hi = n;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        int32_t x = P.x[X[mid]];
        if (inclusive ? (x <= v) : (x < v)) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Element A[k], 1 <= k < m: triangle (A[k-1], A[k], B[j]); returns its position.
HD int strip_tri_upper(Pts P, const int32_t* A, const int32_t* B, int n, int k, int32_t* tri) {
    int cl = count_below(P, B, n, P.x[A[k]], false);
    int j = cl > 0 ? cl - 1 : 0;
    tri[0] = A[k - 1]; tri[1] = A[k]; tri[2] = B[j];
    return (k - 1) + j;
}

// Element B[k], 1 <= k < n: triangle (A[i], B[k], B[k-1]); returns its position.
HD int strip_tri_lower(Pts P, const int32_t* A, int m, const int32_t* B, int k, int32_t* tri) {
    int cl = count_below(P, A, m, P.x[B[k]], true);
    int i = cl > 0 ? cl - 1 : 0;
    tri[0] = A[i]; tri[1] = B[k]; tri[2] = B[k - 1];
    return i + (k - 1);
}

// Fill the pocket between a boundary chain (one point per non-empty row,
// top to bottom: point index ci[k] at (cx[k], cy[k])) and its convex hull.
// side = +1 for the left chain (first points), -1 for the right chain
// (last points).  `stack` has room for 4 * len ints: an entry is the
// record (point index, x, y, -) of a chain point, so a pop reads one
// 16-byte record.  The next chain point is loaded one step ahead.  Returns
// the number of counter-clockwise triangles written.
HD int fill_pockets(const int32_t* ci, const int32_t* cx, const int32_t* cy, int len, int side, int32_t* stack,
                    int32_t* tri) {
    // the two top stack entries are kept in registers: (a, b) = stack[sp-2], stack[sp-1]
    int sp = 0, k = 0;
    // orientations are exact in int32 within the library's coordinate range
    // (|dx| <= 18094, |dy| <= 16383, see orient_p)
    int32_t ia = 0, ib = 0;
    int32_t ax = 0, ay = 0, bx = 0, by = 0;
    int32_t nx = len > 0 ? cx[0] : 0, ny = len > 0 ? cy[0] : 0, ni = len > 0 ? ci[0] : 0;
    for (int i = 0; i < len; ++i) {
        const int32_t x = nx, y = ny;
        const int32_t ii = ni;
        if (i + 1 < len) { nx = cx[i + 1]; ny = cy[i + 1]; ni = ci[i + 1]; }
        while (sp >= 2) {
            const int32_t o = (bx - ax) * (y - ay) - (by - ay) * (x - ax);
            if (side > 0 ? (o > 0) : (o < 0)) {
                tri[3 * k] = ia;
                tri[3 * k + 1] = side > 0 ? ib : ii;
                tri[3 * k + 2] = side > 0 ? ii : ib;
                ++k;
                --sp;
                ib = ia; bx = ax; by = ay;
                if (sp >= 2) {
                    const int32_t* q = stack + 4 * (sp - 2);
                    ia = q[0]; ax = q[1]; ay = q[2];
                }
            } else {
                break;
            }
        }
        int32_t* e = stack + 4 * sp;
        e[0] = ii; e[1] = x; e[2] = y; e[3] = 0;
        ++sp;
        ia = ib; ax = bx; ay = by;
        ib = ii; bx = x; by = y;
    }
    return k;
}

HD uint32_t hash64(uint64_t k) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ull;
    k ^= k >> 33;
    return uint32_t(k);
}

HD uint64_t edge_key(int a, int b) {
    return a < b ? (uint64_t(uint32_t(a)) << 32 | uint32_t(b)) : (uint64_t(uint32_t(b)) << 32 | uint32_t(a));
}

// Bijective 32-bit mix: unique flip priorities per edge within a round.
HD uint32_t prio(uint32_t e, uint32_t round) {
    uint32_t x = e + round * 0x9E3779B9u;
    x ^= x >> 16; x *= 0x7feb352du;
    x ^= x >> 15; x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

constexpr int32_t FINAL = 1 << 30;          // opp entry already refers to the new slot
constexpr uint32_t LOCK_FREE = 0xFFFFFFFFu;
constexpr unsigned long long HASH_EMPTY = ~0ull;

// Packed point coordinates, 16 bits each with a bias of 2^15 (coordinates
// in [-32768, 32767]; the predicates are translation invariant): every
// triangle record carries its vertices' coordinates, so the predicates
// never chase the point arrays.
HD uint32_t pack_xy(int32_t x, int32_t y) {
    return (uint32_t(x + 32768) & 0xffffu) | ((uint32_t(y + 32768) & 0xffffu) << 16);
}
HD int32_t px_of(uint32_t p) { return int32_t(p & 0xffffu) - 32768; }
HD int32_t py_of(uint32_t p) { return int32_t(p >> 16) - 32768; }

// Coordinate differences of packed points (the bias cancels).
HD int32_t dx_p(uint32_t a, uint32_t b) { return int32_t(a & 0xffffu) - int32_t(b & 0xffffu); }
HD int32_t dy_p(uint32_t a, uint32_t b) { return int32_t(a >> 16) - int32_t(b >> 16); }

// Narrow exact predicates.  The library accepts width <= 14000,
// height <= 16384 and disp_max <= 4095, so point x lies in [-4095, 13999]
// (right view: u - d) and y in [0, 16383]: |dx| <= 18094, |dy| <= 16383.
// Then every square sum and every 2x2 orientation term is below 2^30 in
// magnitude (int32), and the lifted determinant is a sum of three 32x32-bit
// products below 2^59 each (int64).  Both are exact.
HD int64_t orient_p(uint32_t a, uint32_t b, uint32_t c) {
    return int64_t(dx_p(b, a) * dy_p(c, a) - dy_p(b, a) * dx_p(c, a));
}

// > 0 iff d lies inside the circumcircle of the counter-clockwise (a,b,c):
// the 3x3 lifted determinant expanded along its lifted column,
// |a-d|^2 * orient(b,c) + |b-d|^2 * orient(c,a) + |c-d|^2 * orient(a,b)
// with every orientation taken relative to d.
HD int64_t incircle_p(uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
    const int32_t adx = dx_p(a, d), ady = dy_p(a, d);
    const int32_t bdx = dx_p(b, d), bdy = dy_p(b, d);
    const int32_t cdx = dx_p(c, d), cdy = dy_p(c, d);
    const int32_t al = adx * adx + ady * ady, bl = bdx * bdx + bdy * bdy, cl = cdx * cdx + cdy * cdy;
    const int32_t obc = bdx * cdy - bdy * cdx, oca = cdx * ady - cdy * adx, oab = adx * bdy - ady * bdx;
    return int64_t(al) * obc + int64_t(bl) * oca + int64_t(cl) * oab;
}

// inside_sos on packed coordinates; ia..id are the point indices that order
// the symbolic perturbation.
HD bool inside_sos_p(int ia, uint32_t a, int ib, uint32_t b, int ic, uint32_t c, int id, uint32_t d) {
    int64_t det = incircle_p(a, b, c, d);
    if (det != 0) return det > 0;
    int m = imin(imin(ia, ib), imin(ic, id));
    if (m == id) return true;
    if (m == ia) return orient_p(d, b, c) < 0;
    if (m == ib) return orient_p(a, d, c) < 0;
    return orient_p(a, b, d) < 0;
}

// Flip rounds are written against an accessor M that stores, per triangle t:
// v(t,k) vertex indices, xy(t,k) packed coordinates, opp(3t+k) neighbour
// half-edges, a lock word and the last round t was flipped in.  The flat
// accessor (global memory, host emulation) and the cluster accessor
// (distributed shared memory) share this code.
//
// Is the edge of half-edge h (twin tw) not locally Delaunay?  Tested from
// h's side: h's triangle (a, b, c) against the vertex of tw's triangle
// opposite the edge.
template <class M>
HD bool edge_flippable(const M& m, int h, int tw) {
    const int t = h / 3, s = h % 3, n = tw / 3, sn = tw % 3;
    const int s1 = s == 2 ? 0 : s + 1, s2 = s1 == 2 ? 0 : s1 + 1, sd = sn == 0 ? 2 : sn - 1;
    return inside_sos_p(m.v(t, s), m.xy(t, s), m.v(t, s1), m.xy(t, s1), m.v(t, s2), m.xy(t, s2), m.v(n, sd),
                        m.xy(n, sd));
}

// Phase A: test half-edge h; propose it if its edge is not locally Delaunay.
// `owner`: only the triangle with the smaller index tests a shared edge.
template <class M, class Append>
HD bool flip_propose(M& m, int h, int T, uint32_t round, bool owner, Append append_cand) {
    int t = h / 3;
    int o = m.opp(h);
    if (o < 0) return true;
    int n = o / 3;
    if (n >= T || t >= T) return false;
    if (owner && n <= t) return true;
    if (edge_flippable(m, h, o)) {
        uint32_t p = prio(uint32_t(h), round);
        m.lock_min(t, p);
        m.lock_min(n, p);
        append_cand(h, n);
    }
    return true;
}

// Phase B: flip the proposal (h, n) if it won both locks.
template <class M>
HD bool flip_apply(M& m, int h, int n, uint32_t round) {
    int t = h / 3, s = h % 3;
    uint32_t p = prio(uint32_t(h), round);
    if (m.lock(t) != p || m.lock(n) != p) return false;
    int sn = m.opp(h) % 3;
    int s1 = s == 2 ? 0 : s + 1, s2 = s1 == 2 ? 0 : s1 + 1;
    int sn1 = sn == 2 ? 0 : sn + 1, sn2 = sn1 == 2 ? 0 : sn1 + 1;
    int a = m.v(t, s), b = m.v(t, s1), c = m.v(t, s2), d = m.v(n, sn2);
    uint32_t pa = m.xy(t, s), pb = m.xy(t, s1), pc = m.xy(t, s2), pd = m.xy(n, sn2);
    int O_bc = m.opp(3 * t + s1), O_ca = m.opp(3 * t + s2);
    int O_ad = m.opp(3 * n + sn1), O_db = m.opp(3 * n + sn2);
    // t' = (c, a, d), n' = (d, b, c); the new diagonal is slot 2 of both
    m.set_v(t, c, a, d, pc, pa, pd);
    m.set_v(n, d, b, c, pd, pb, pc);
    m.set_opp(3 * t, O_ca); m.set_opp(3 * t + 1, O_ad); m.set_opp(3 * t + 2, FINAL | (3 * n + 2));
    m.set_opp(3 * n, O_db); m.set_opp(3 * n + 1, O_bc); m.set_opp(3 * n + 2, FINAL | (3 * t + 2));
    m.set_fround(t, int32_t(round));
    m.set_fround(n, int32_t(round));
    return true;
}

// The four outer half-edges of a flipped pair (t, n): t' slots 0,1 and n' slots 0,1.
HD int outer_slot(int t, int n, int k) { return k < 2 ? 3 * t + k : 3 * n + (k - 2); }

// Phase C1 (read only): where does the neighbour across outer slot x of a
// flipped pair live now?  Its old reference o still holds if o's triangle
// did not flip this round; otherwise the edge is one of the outer slots of
// that triangle's new pair, found by matching the reversed edge.  Returns
// the half-edge, -1 for the hull, or -2 if nothing matched or an index left
// [0, T) (corrupt state).
template <class M>
HD int flip_resolve_slot(M& m, int x, uint32_t round, int T) {
    int o = m.opp(x);
    if (o < 0) return -1;
    int mt = o / 3;
    if (mt >= T) return -2;
    if (m.fround(mt) != int32_t(round)) return o;
    int xt = x / 3, xk = x % 3;
    int a = m.v(xt, xk), b = m.v(xt, xk == 2 ? 0 : xk + 1);
    const int o2 = m.opp(3 * mt + 2);
    if (o2 < 0) return -2;
    int mt2 = (o2 & ~FINAL) / 3;
    if (mt2 >= T) return -2;
    const int cand_t[2] = {mt, mt2};
    for (int i = 0; i < 2; ++i)
        for (int k = 0; k < 2; ++k) {
            int tt = cand_t[i];
            if (m.v(tt, k) == b && m.v(tt, k + 1) == a) return 3 * tt + k;
        }
    return -2;
}

// Phase C2: write the links both ways and clear the FINAL marks.
template <class M>
HD void flip_relink(M& m, int t, int n, const int32_t* res) {
    for (int k = 0; k < 4; ++k) {
        int x = outer_slot(t, n, k);
        int r = res[k];
        m.set_opp(x, r);
        if (r >= 0) m.set_opp(r, x);
    }
    m.set_opp(3 * t + 2, m.opp(3 * t + 2) & ~FINAL);
    m.set_opp(3 * n + 2, m.opp(3 * n + 2) & ~FINAL);
}

// Flat storage: plain arrays (global memory on the device, host memory in
// the emulation).  AMin performs the lock's atomic minimum.
template <class AMin>
struct FlatTri {
    int32_t* tv;      // [3T] vertex indices
    uint32_t* txy;    // [3T] packed coordinates
    int32_t* topp;    // [3T]
    uint32_t* tlock;  // [T]
    int32_t* tround;  // [T]
    AMin amin;
    HD int v(int t, int k) const { return tv[3 * t + k]; }
    HD uint32_t xy(int t, int k) const { return txy[3 * t + k]; }
    HD int opp(int h) const { return topp[h]; }
    HD uint32_t lock(int t) const { return tlock[t]; }
    HD int32_t fround(int t) const { return tround[t]; }
    HD void lock_min(int t, uint32_t p) { amin(&tlock[t], p); }
    HD void set_v(int t, int a, int b, int c, uint32_t pa, uint32_t pb, uint32_t pc) {
        tv[3 * t] = a; tv[3 * t + 1] = b; tv[3 * t + 2] = c;
        txy[3 * t] = pa; txy[3 * t + 1] = pb; txy[3 * t + 2] = pc;
    }
    HD void set_opp(int h, int o) { topp[h] = o; }
    HD void set_fround(int t, int32_t r) { tround[t] = r; }
};

// Rotate a triangle so its smallest vertex index comes first.
HD void normalise(int32_t* v) {
    int a = v[0], b = v[1], c = v[2];
    while (a > b || a > c) { int x = a; a = b; b = c; c = x; }
    v[0] = a; v[1] = b; v[2] = c;
}

}  // namespace del
}  // namespace elas
