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

#include <cmath>
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

// ---------------------------------------------------------------------------
// Stars: the Delaunay neighbours of one point, found directly.
//
// Under the perturbation the triangulation is unique, so each point's star
// (its neighbours in counter-clockwise order) can be computed on its own and
// the stars of all points agree.  The walk around p starts at p's nearest
// neighbour q0 (the disc with diameter p q0 holds no other point, so p q0 is
// an edge of every Delaunay triangulation).  From an edge p->q the next
// neighbour on a side is, among the points strictly on that side, the one
// whose circle through p and q holds no other of them: the circles through
// p and q form a pencil, and "b lies inside the circle through p, q, a" is a
// strict total order on the points of one side (the perturbed incircle
// determinant is antisymmetric in a and b).  The minimum of that order is the
// next neighbour; a side with no point marks a hull edge.  The walk goes
// counter-clockwise until it returns to q0 (an interior point) or meets the
// hull, and then clockwise from q0 to the hull on the other side.

constexpr uint32_t PXY_NONE = 0xFFFFFFFFu;   // a dropped duplicate point

// For the edge p->q and two points a, b on the walk's side, is b the better
// next neighbour (inside the circle through p, q and a)?  side > 0: left of
// p->q, triangle (p, q, a) counter-clockwise; side < 0: right, triangle
// (p, a, q).
HD bool star_better(int ip, uint32_t pp, int iq, uint32_t pq, int ia, uint32_t pa, int ib, uint32_t pb, int side) {
    return side > 0 ? inside_sos_p(ip, pp, iq, pq, ia, pa, ib, pb) : inside_sos_p(ip, pp, ia, pa, iq, pq, ib, pb);
}

// Is b strictly on the walk's side of p->q?
HD bool star_side(uint32_t pp, uint32_t pq, uint32_t pb, int side) {
    const int64_t o = orient_p(pp, pq, pb);
    return side > 0 ? o > 0 : o < 0;
}

// Does every point inside the circle through p, q and r lie in the square
// |x - px|, |y - py| <= R?  Points exist only in the box [bx0, bx1] x
// [by0, by1] (all points of the problem), so only the part of the circle
// inside the box counts: its extent is bounded through the circle's chords
// at the box edges nearest the centre.  Every point outside the square is
// at least R + 1 away from p in x or in y, which leaves a pixel of margin
// for the rounding of the centre and the chords (the centre's numerators
// and denominator are exact integers in double).  *need: the square that
// would pass.
HD bool circle_within(uint32_t pp, uint32_t pq, uint32_t pr, int R, const int32_t* box, int* need) {
    const double qx = dx_p(pq, pp), qy = dy_p(pq, pp), rx = dx_p(pr, pp), ry = dy_p(pr, pp);
    const double d = 2.0 * (qx * ry - qy * rx);
    const double q2 = qx * qx + qy * qy, r2 = rx * rx + ry * ry;
    const double cx = (ry * q2 - qy * r2) / d, cy = (qx * r2 - rx * q2) / d;
    const double rho2 = cx * cx + cy * cy;
    // the box relative to p
    const double bx0 = box[0] - px_of(pp), by0 = box[1] - py_of(pp), bx1 = box[2] - px_of(pp), by1 = box[3] - py_of(pp);
    const double ey = fmin(fmax(cy, by0), by1) - cy, ex = fmin(fmax(cx, bx0), bx1) - cx;
    double ext = 0.0;
    if (ey * ey < rho2 && ex * ex < rho2) {
        const double h = sqrt(rho2 - ey * ey), v = sqrt(rho2 - ex * ex);
        const double x0 = fmax(cx - h, bx0), x1 = fmin(cx + h, bx1);
        const double y0 = fmax(cy - v, by0), y1 = fmin(cy + v, by1);
        ext = fmax(fmax(-x0, x1), fmax(-y0, y1));
    }
    if (need) *need = ext < 1e9 ? int(ext) + 2 : (1 << 30);
    return ext <= double(R);
}

// circle_within's answer without its extent, by comparisons only: every
// quantity scaled by D = |2 cross(q - p, r - p)| (the centre's numerators,
// the box, R), so no division and no square root.  The centre numerators
// and the scaled box are exact integers in double; the squared terms
// (below 2^93) carry a relative rounding of 2^-53, which moves a decision
// by far less than the pixel of margin circle_within relies on.
HD bool circle_inside(uint32_t pp, uint32_t pq, uint32_t pr, int R, const int32_t* box) {
    const double qx = dx_p(pq, pp), qy = dy_p(pq, pp), rx = dx_p(pr, pp), ry = dy_p(pr, pp);
    const double d2x = 2.0 * (qx * ry - qy * rx);
    const double q2 = qx * qx + qy * qy, r2 = rx * rx + ry * ry;
    const double sg = d2x < 0.0 ? -1.0 : 1.0, D = fabs(d2x);
    const double CX = sg * (ry * q2 - qy * r2), CY = sg * (qx * r2 - rx * q2);   // centre * D
    const double RHO2 = CX * CX + CY * CY;                                       // radius^2 * D^2
    const double BX0 = (box[0] - px_of(pp)) * D, BY0 = (box[1] - py_of(pp)) * D;
    const double BX1 = (box[2] - px_of(pp)) * D, BY1 = (box[3] - py_of(pp)) * D;
    const double EY = fmin(fmax(CY, BY0), BY1) - CY, EX = fmin(fmax(CX, BX0), BX1) - CX;
    if (EY * EY >= RHO2 || EX * EX >= RHO2) return true;     // the circle misses the box
    const double RD = double(R) * D, H2 = RHO2 - EY * EY, V2 = RHO2 - EX * EX;
    // each side of the clipped extent: the box edge itself, or the chord end
    auto side_ok = [](double edge, double c, double rd, double h2) {
        // max(c - h, edge) >= -rd  (edge, c scaled), i.e. edge >= -rd or h <= c + rd
        return edge >= -rd || (c + rd >= 0.0 && h2 <= (c + rd) * (c + rd));
    };
    return side_ok(BX0, CX, RD, H2) && side_ok(-BX1, -CX, RD, H2) && side_ok(BY0, CY, RD, V2) &&
           side_ok(-BY1, -CY, RD, V2);
}

// Search policy of the star walk.  A search first takes a point's window,
// the points with |x - px|, |y - py| <= R0, staged once per point (up to
// STAR_CAP of them), and then squares of doubling half-size Rs
// (star_square) around p until its answer is proven:
//  * nearest neighbour at distance d: proven once d <= Rs; if the first
//    square with a candidate does not prove it, the square of half-size d
//    holds the answer and is searched last;
//  * next neighbour r: proven once its circle passes circle_within(Rs).
//    When the circle reaches no further than 2 Rs, the part of the circle
//    through p, q, r inside the box is searched instead of the next square
//    (the answer's circle on that side of p->q nests inside it, so the
//    answer lies there).  A near-collinear r has a huge circle although the
//    answer is often just outside the window: growing the square finds it
//    at a small cost where the circle would cover much of the box.
// A square covering the box holds every point, so its answer is final (and
// "none" proves a hull edge).
constexpr int STAR_CAP = 512;

// The window's half-size R0 of a problem: 3.5 mean point spacings (the
// square root of the box area per point), within [16, 128] pixels.  Most
// stars then need no second search (a smaller window makes most steps
// search again, a larger one makes every step scan more points).  Exact
// double operations: the same value on the host and the device.
HD int star_r0(const int32_t* box, int n) {
    const double area = double(box[2] - box[0] + 1) * double(box[3] - box[1] + 1);
    const double r = 3.5 * sqrt(area / double(n > 0 ? n : 1));
    return r < 16.0 ? 16 : (r > 128.0 ? 128 : int(r));
}
constexpr int STAR_NB = 256;      // neighbours of one point on each side of its start

// Half-size of the next square after one of half-size R held no candidate.
HD int star_square(int R) { return R < (1 << 20) ? 2 * R : R; }

// The rows [y0, y1] and, per row y, the columns [x0, x1] of a region:
// a square of half-size R around (px, py), or the circle (centre (cx, cy),
// squared radius rho2, absolute coordinates) with a pixel of margin; both
// clipped to the box.  An empty range has y0 > y1 or x0 > x1.
struct StarRegion {
    bool circle;
    double cx, cy, rho2;
    int32_t sx0, sx1;     // square columns
    int32_t y0, y1;
    // optional half-plane (a square searched for a next neighbour): only
    // the points strictly on side `side` of the line through (hx, hy) with
    // direction (ux, uy) count, kept with a pixel of margin
    int32_t hx, hy, ux, uy, side;
    // optional hole (a ring, the square minus a smaller one): rows
    // [ky0, ky1] lose the columns [kx0, kx1]
    int32_t kx0, kx1, ky0, ky1;
    bool hole;
    // The columns of row y as up to two ranges [x0, x1], [x2, x3] (empty
    // when the first bound exceeds the second).
    HD void cols2(int32_t y, const int32_t* box, int32_t* x0, int32_t* x1, int32_t* x2, int32_t* x3) const {
        cols(y, box, x0, x1);
        *x2 = 1;
        *x3 = 0;
        if (hole && y >= ky0 && y <= ky1) {
            *x2 = imax(*x0, kx1 + 1);
            *x3 = *x1;
            *x1 = imin(*x1, kx0 - 1);
        }
    }
    HD void cols(int32_t y, const int32_t* box, int32_t* x0, int32_t* x1) const {
        if (!circle) {
            *x0 = sx0;
            *x1 = sx1;
            if (side != 0) {
                if (uy == 0) {
                    if (int64_t(ux) * (y - hy) * side <= 0) *x0 = *x1 + 1;
                } else {
                    const double xl = double(hx) + double(ux) * double(y - hy) / double(uy);
                    if ((uy > 0) == (side > 0))
                        *x1 = int32_t(fmax(fmin(double(*x1), ceil(xl) + 1.0), double(*x0) - 1.0));
                    else
                        *x0 = int32_t(fmin(fmax(double(*x0), floor(xl) - 1.0), double(*x1) + 1.0));
                }
            }
            return;
        }
        // half-chord at row y, plus a pixel for the rounding of the centre
        // and radius (both far below a pixel at these coordinates)
        const double dy = double(y) - cy;
        const double h = sqrt(fmax(rho2 - dy * dy, 0.0)) + 1.0;
        // clamped into the box (an empty range stays empty) before the
        // conversion: a near-degenerate circle's centre can lie far outside
        *x0 = int32_t(fmin(fmax(floor(cx - h) - 1.0, double(box[0])), double(box[2]) + 1.0));
        *x1 = int32_t(fmax(fmin(ceil(cx + h) + 1.0, double(box[2])), double(box[0]) - 1.0));
    }
};

HD StarRegion star_square_region(uint32_t pp, int R, const int32_t* box) {
    StarRegion g;
    g.circle = false;
    g.cx = g.cy = g.rho2 = 0.0;
    g.hx = g.hy = g.ux = g.uy = g.side = 0;
    g.kx0 = g.kx1 = g.ky0 = g.ky1 = 0;
    g.hole = false;
    const int32_t px = px_of(pp), py = py_of(pp);
    g.sx0 = imax(px - R, box[0]);
    g.sx1 = imin(px + R, box[2]);
    g.y0 = imax(py - R, box[1]);
    g.y1 = imin(py + R, box[3]);
    return g;
}

// The ring between the squares of half-sizes R and 2R around p.
HD StarRegion star_ring_region(uint32_t pp, int R, const int32_t* box) {
    StarRegion g = star_square_region(pp, 2 * R, box);
    const int32_t px = px_of(pp), py = py_of(pp);
    g.hole = true;
    g.kx0 = px - R;
    g.kx1 = px + R;
    g.ky0 = py - R;
    g.ky1 = py + R;
    return g;
}

// The square of half-size R around p restricted to side `side` of p->q.
HD StarRegion star_half_region(uint32_t pp, uint32_t pq, int side, int R, const int32_t* box) {
    StarRegion g = star_square_region(pp, R, box);
    g.hx = px_of(pp);
    g.hy = py_of(pp);
    g.ux = dx_p(pq, pp);
    g.uy = dy_p(pq, pp);
    g.side = side;
    return g;
}

// The circle through p, q and r (any order), clipped to the box.
HD StarRegion star_circle_region(uint32_t pp, uint32_t pq, uint32_t pr, const int32_t* box) {
    const double qx = dx_p(pq, pp), qy = dy_p(pq, pp), rx = dx_p(pr, pp), ry = dy_p(pr, pp);
    const double d = 2.0 * (qx * ry - qy * rx);
    const double q2 = qx * qx + qy * qy, r2 = rx * rx + ry * ry;
    const double cx = (ry * q2 - qy * r2) / d, cy = (qx * r2 - rx * q2) / d;
    StarRegion g;
    g.circle = true;
    g.hx = g.hy = g.ux = g.uy = g.side = 0;
    g.kx0 = g.kx1 = g.ky0 = g.ky1 = 0;
    g.hole = false;
    g.cx = cx + px_of(pp);
    g.cy = cy + py_of(pp);
    g.rho2 = cx * cx + cy * cy;
    g.sx0 = g.sx1 = 0;
    const double rho = sqrt(g.rho2);
    g.y0 = int32_t(fmax(floor(g.cy - rho) - 1.0, double(box[1])));
    g.y1 = int32_t(fmin(ceil(g.cy + rho) + 1.0, double(box[3])));
    return g;
}

// Walk the star.  An interior point (hn < 0) starts at nearest(), p's
// nearest neighbour, and walks counter-clockwise until it is back there.  A
// point of the hull boundary starts at hn, its successor on the boundary
// (counter-clockwise, the interior on the left), and walks until it reaches
// hp, its predecessor.  next(q, side) returns the next neighbour after q on
// that side (-1: none, so p->q is a hull edge; -2: the search failed).
// The neighbours are appended to ccw (counter-clockwise) and, should an
// interior point meet the hull (all points collinear), to cw (clockwise from
// the start); star_at gives them in counter-clockwise order.  Returns false
// if a search failed or a list would pass cap.
template <class Nearest, class Next>
HD bool star_walk(int hn, int hp, Nearest nearest, Next next, int32_t* ccw, int32_t* cw, int cap, int* m, int* k,
                  bool* closed) {
    *m = 0;
    *k = 0;
    *closed = false;
    const int q0 = hn >= 0 ? hn : nearest();
    if (q0 < 0) return q0 == -1;
    ccw[(*m)++] = q0;
    int q = q0;
    for (;;) {
        const int r = next(q, +1);
        if (r == -2) return false;
        if (r < 0) break;
        if (r == q0) {
            *closed = hn < 0;
            return hn < 0;
        }
        if (*m >= cap) return false;
        ccw[(*m)++] = r;
        if (r == hp) return true;
        q = r;
    }
    if (hn >= 0) return true;
    q = q0;
    for (;;) {
        const int r = next(q, -1);
        if (r == -2) return false;
        if (r < 0) break;
        if (*k >= cap) return false;
        cw[(*k)++] = r;
        q = r;
    }
    return true;
}

// The hull boundary, counter-clockwise (the interior on the left of each
// step), from the rows' extreme points: the top row left to right, the
// right chain down, the bottom row right to left, the left chain up.  The
// chains are the rows' last (first) points with the concave ones removed by
// the monotone stack walk; collinear points stay, as every point on the
// boundary is a vertex of the triangulation.  xy[s] holds the packed
// coordinates of the leftmost (side 0) or rightmost (side 1) point of
// non-empty row s (of R, top to bottom).  Writes the chain as row positions
// (top to bottom; room for R) and its length.
HD void hull_chain(int side, int R, const uint32_t* xy, int32_t* st, int* len) {
    int sp = 0;
    uint32_t a = 0, b = 0;     // the stack's top two points
    for (int s = 0; s < R; ++s) {
        const uint32_t x = xy[s];
        while (sp >= 2) {
            const int64_t o = orient_p(a, b, x);
            if (side ? o < 0 : o > 0) {
                --sp;
                b = a;
                if (sp >= 2) a = xy[st[sp - 2]];
            } else {
                break;
            }
        }
        st[sp++] = s;
        a = b;
        b = x;
    }
    *len = sp;
}

// The same chain, decided point by point (for a parallel build): row i's
// point is dropped by the stack walk exactly when it lies strictly inside
// the segment of two other chain points j < i < k (strictly right of L_j ->
// L_k for the left chain, left of it for the right chain).  With
// coordinates relative to point i and x mirrored for the right chain, that
// holds iff min_{j<i} x_j / -y_j + min_{k>i} x_k / y_k < 0 (the rows above
// have y < 0, those below y > 0); both minima and their sum are compared
// as exact fractions.  |x| <= 18094 and 0 < y <= 16383 (the coordinate
// limits of orient_p), so every cross product is below 2^29 and the final
// sum below 2^30: exact in int32.
HD bool hull_on_chain(int side, int R, const uint32_t* xy, int i) {
    if (i == 0 || i == R - 1) return true;
    const uint32_t c = xy[i];
    const int sg = side ? -1 : 1;
    // each minimum over four interleaved partial minima (independent chains)
    int32_t n[2][4], d[2][4];
    for (int h = 0; h < 2; ++h)
        for (int u = 0; u < 4; ++u) {
            n[h][u] = 1;
            d[h][u] = 0;     // +infinity: 1/0 compares above every fraction below
        }
    auto fold = [&](int h, int u, uint32_t v, int dsign) {
        const int32_t x = sg * dx_p(v, c), dd = dsign * dy_p(v, c);
        if (d[h][u] == 0 || x * d[h][u] < n[h][u] * dd) {
            n[h][u] = x;
            d[h][u] = dd;
        }
    };
    int j = 0;
    for (; j + 4 <= i; j += 4)
        for (int u = 0; u < 4; ++u) fold(0, u, xy[j + u], -1);
    for (; j < i; ++j) fold(0, 0, xy[j], -1);
    int k = i + 1;
    for (; k + 4 <= R; k += 4)
        for (int u = 0; u < 4; ++u) fold(1, u, xy[k + u], 1);
    for (; k < R; ++k) fold(1, 0, xy[k], 1);
    int32_t sn = n[0][0], sd = d[0][0], tn = n[1][0], td = d[1][0];
    for (int u = 1; u < 4; ++u) {
        if (d[0][u] != 0 && n[0][u] * sd < sn * d[0][u]) { sn = n[0][u]; sd = d[0][u]; }
        if (d[1][u] != 0 && n[1][u] * td < tn * d[1][u]) { tn = n[1][u]; td = d[1][u]; }
    }
    return sn * td + tn * sd >= 0;
}

// Position j of the boundary cycle (hull_chain's layout): top row (tl
// points) left to right, right chain rows 1..nr-1, bottom row (bl points)
// right to left from its second last, left chain rows nl-2..1.  Returns
// (row position, index within that row); the cycle has
// tl + (nr - 1) + (bl - 1) + (nl - 2) points when the top and bottom rows
// differ.
HD int hull_cycle_len(int tl, int bl, int nl, int nr) { return tl + (nr - 1) + (bl - 1) + (nl - 2); }
HD void hull_cycle_at(int j, int R, int tl, int bl, const int32_t* lstk, int nl, const int32_t* rstk, int nr,
                      int* row, int* pos, bool* last) {
    *last = false;
    if (j < tl) { *row = 0; *pos = j; return; }
    j -= tl;
    if (j < nr - 1) { *row = rstk[j + 1]; *pos = 0; *last = true; return; }
    j -= nr - 1;
    if (j < bl - 1) { *row = R - 1; *pos = bl - 2 - j; return; }
    j -= bl - 1;
    *row = lstk[nl - 2 - j];
    *pos = 0;
}

// Neighbour i in counter-clockwise order: the clockwise part reversed, then
// the counter-clockwise part.
HD int32_t star_at(const int32_t* ccw, int m, const int32_t* cw, int k, int i) {
    (void)m;
    return i < k ? cw[k - 1 - i] : ccw[i - k];
}

// Triangles of a star of deg neighbours: (p, nb(i), nb(i+1)), wrapping when
// closed.  Triangle i is emitted by p when p is its smallest vertex, which
// makes it come out normalised (see normalise below).
HD int star_tris(int deg, bool closed) { return closed ? deg : (deg > 0 ? deg - 1 : 0); }

// Rotate a triangle so its smallest vertex index comes first.
HD void normalise(int32_t* v) {
    int a = v[0], b = v[1], c = v[2];
    while (a > b || a > c) { int x = a; a = b; b = c; c = x; }
    v[0] = a; v[1] = b; v[2] = c;
}

}  // namespace del
}  // namespace elas
