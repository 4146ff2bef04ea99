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
// Predicates: orientation and incircle on integer coordinates in int64 --
// exact for |coordinates| < 2^15 (terms stay below 2^62).  Ties (four
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

HD int64_t orient(Pts P, int a, int b, int c) {
    int64_t ax = P.x[a], ay = P.y[a];
    return (int64_t(P.x[b]) - ax) * (int64_t(P.y[c]) - ay) -
           (int64_t(P.y[b]) - ay) * (int64_t(P.x[c]) - ax);
}

// > 0 iff d lies inside the circumcircle of the counter-clockwise (a,b,c).
HD int64_t incircle(Pts P, int a, int b, int c, int d) {
    int64_t dx = P.x[d], dy = P.y[d];
    int64_t adx = P.x[a] - dx, ady = P.y[a] - dy;
    int64_t bdx = P.x[b] - dx, bdy = P.y[b] - dy;
    int64_t cdx = P.x[c] - dx, cdy = P.y[c] - dy;
    int64_t al = adx * adx + ady * ady;
    int64_t bl = bdx * bdx + bdy * bdy;
    int64_t cl = cdx * cdx + cdy * cdy;
    return adx * (bdy * cl - bl * cdy) - ady * (bdx * cl - bl * cdx) + al * (bdx * cdy - bdy * cdx);
}

HD bool inside_sos(Pts P, int a, int b, int c, int d) {
    int64_t det = incircle(P, a, b, c, d);
    if (det != 0) return det > 0;
    int m = imin(imin(a, b), imin(c, d));
    if (m == d) return true;
    if (m == a) return orient(P, d, b, c) < 0;
    if (m == b) return orient(P, a, d, c) < 0;
    return orient(P, a, b, d) < 0;
}

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
// (last points).  `stack` (chain positions) has room for `len` entries.
// Returns the number of counter-clockwise triangles written.
HD int fill_pockets(const int32_t* ci, const int32_t* cx, const int32_t* cy, int len, int side, int32_t* stack,
                    int32_t* tri) {
    int sp = 0, k = 0;
    for (int i = 0; i < len; ++i) {
        while (sp >= 2) {
            int a = stack[sp - 2], b = stack[sp - 1];
            int64_t o = (int64_t(cx[b]) - cx[a]) * (int64_t(cy[i]) - cy[a]) -
                        (int64_t(cy[b]) - cy[a]) * (int64_t(cx[i]) - cx[a]);
            if (side > 0 ? (o > 0) : (o < 0)) {
                tri[3 * k] = ci[a];
                tri[3 * k + 1] = side > 0 ? ci[b] : ci[i];
                tri[3 * k + 2] = side > 0 ? ci[i] : ci[b];
                ++k;
                --sp;
            } else {
                break;
            }
        }
        stack[sp++] = i;
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

// Per-problem state of one triangulation during flipping.
struct Flip {
    Pts P;
    int32_t* tri;       // [3*Tmax] vertex triples, counter-clockwise
    int32_t* opp;       // [3*Tmax] neighbour half-edge (3*t+s) across edge (v_s, v_s+1), -1 = hull
    uint32_t* lock;     // [Tmax]   minimum proposal priority on the triangle this round
    int32_t* fround;    // [Tmax]   last round the triangle was flipped (-1 = never)
    int32_t* fwd;       // [3*Tmax] old half-edge -> new half-edge, valid for one round
    int32_t* cand;      // [2*3*Tmax] proposals of the round: (half-edge, neighbour triangle)
    int32_t* flips;     // [Tmax]   flipped pairs of the round: (t, n)
    int32_t* res;       // [2*Tmax] resolved outer neighbours of the flipped pairs (4 per pair)
    int32_t* fwdl;      // [2*Tmax] forwarding entries written this round (to clear next round)
    int32_t* wl[2];     // [6*Tmax] worklists of half-edges
    int Tmax;
};

// Phase A: test half-edge h; propose it if its edge is not locally Delaunay.
// `owner`: only the triangle with the smaller index tests a shared edge
// (round 0 walks every half-edge).
template <class AtomicMin, class Append>
HD bool flip_propose(Flip& S, int h, int T, uint32_t round, bool owner, AtomicMin amin, Append append_cand) {
    int t = h / 3, s = h % 3;
    int o = S.opp[h];
    if (o < 0) return true;
    int n = o / 3;
    if (n >= T || t >= T) return false;
    if (owner && n <= t) return true;
    int sn = o % 3;
    int a = S.tri[3 * t + s], b = S.tri[3 * t + (s + 1) % 3], c = S.tri[3 * t + (s + 2) % 3];
    int d = S.tri[3 * n + (sn + 2) % 3];
    if (inside_sos(S.P, a, b, c, d)) {
        uint32_t p = prio(uint32_t(h), round);
        amin(&S.lock[t], p);
        amin(&S.lock[n], p);
        append_cand(h, n);
    }
    return true;
}

// Phase B: flip the proposal (h, n) if it won both locks.  Returns true if
// flipped; the caller records the pair and the four forwarding slots.
HD bool flip_apply(Flip& S, int h, int n, uint32_t round, int32_t* fwd_slots) {
    int t = h / 3, s = h % 3;
    uint32_t p = prio(uint32_t(h), round);
    if (S.lock[t] != p || S.lock[n] != p) return false;
    int o = S.opp[h];
    int sn = o % 3;
    int a = S.tri[3 * t + s], b = S.tri[3 * t + (s + 1) % 3], c = S.tri[3 * t + (s + 2) % 3];
    int d = S.tri[3 * n + (sn + 2) % 3];
    int O_bc = S.opp[3 * t + (s + 1) % 3], O_ca = S.opp[3 * t + (s + 2) % 3];
    int O_ad = S.opp[3 * n + (sn + 1) % 3], O_db = S.opp[3 * n + (sn + 2) % 3];
    // t' = (c, a, d), n' = (d, b, c); the new diagonal (d,c)/(c,d) is slot 2 of both
    S.tri[3 * t] = c; S.tri[3 * t + 1] = a; S.tri[3 * t + 2] = d;
    S.tri[3 * n] = d; S.tri[3 * n + 1] = b; S.tri[3 * n + 2] = c;
    S.opp[3 * t] = O_ca; S.opp[3 * t + 1] = O_ad; S.opp[3 * t + 2] = FINAL | (3 * n + 2);
    S.opp[3 * n] = O_db; S.opp[3 * n + 1] = O_bc; S.opp[3 * n + 2] = FINAL | (3 * t + 2);
    fwd_slots[0] = 3 * t + (s + 2) % 3; S.fwd[fwd_slots[0]] = 3 * t;        // edge c-a -> t' slot 0
    fwd_slots[1] = 3 * t + (s + 1) % 3; S.fwd[fwd_slots[1]] = 3 * n + 1;    // edge b-c -> n' slot 1
    fwd_slots[2] = 3 * n + (sn + 1) % 3; S.fwd[fwd_slots[2]] = 3 * t + 1;   // edge a-d -> t' slot 1
    fwd_slots[3] = 3 * n + (sn + 2) % 3; S.fwd[fwd_slots[3]] = 3 * n;       // edge d-b -> n' slot 0
    S.fround[t] = int32_t(round);
    S.fround[n] = int32_t(round);
    return true;
}

// The four outer half-edges of a flipped pair (t, n): t' slots 0,1 and n' slots 0,1.
HD int outer_slot(int t, int n, int k) { return k < 2 ? 3 * t + k : 3 * n + (k - 2); }

// Phase C1 (read only): resolve where the outer neighbours of pair f now live.
HD void flip_resolve(Flip& S, int f) {
    int t = S.flips[2 * f], n = S.flips[2 * f + 1];
    for (int k = 0; k < 4; ++k) {
        int o = S.opp[outer_slot(t, n, k)];
        int r = o;
        if (o >= 0) {
            int fw = S.fwd[o];
            if (fw >= 0) r = fw;
        }
        S.res[4 * f + k] = r;
    }
}

// Phase C2: write the links in both directions, clear the FINAL marks and
// queue the outer edges for the next round.
template <class Append>
HD void flip_relink(Flip& S, int f, Append append_next) {
    int t = S.flips[2 * f], n = S.flips[2 * f + 1];
    for (int k = 0; k < 4; ++k) {
        int x = outer_slot(t, n, k);
        int r = S.res[4 * f + k];
        S.opp[x] = r;
        if (r >= 0) S.opp[r] = x;
        append_next(x);
    }
    S.opp[3 * t + 2] &= ~FINAL;
    S.opp[3 * n + 2] &= ~FINAL;
}

// Rotate a triangle so its smallest vertex index comes first.
HD void normalise(int32_t* v) {
    int a = v[0], b = v[1], c = v[2];
    while (a > b || a > c) { int x = a; a = b; b = c; c = x; }
    v[0] = a; v[1] = b; v[2] = c;
}

}  // namespace del
}  // namespace elas
