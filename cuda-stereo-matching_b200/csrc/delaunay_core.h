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
//     non-empty rows is triangulated by one merge ("zipper") pass, choosing
//     at each step the diagonal that the incircle test prefers.
//  3. Fill the pockets between the rows' first (last) points and the convex
//     hull with the monotone-chain stack walk.
//  4. Build edge adjacency with an open-addressing hash of undirected edges.
//  5. Lawson edge flipping in parallel rounds: every non-locally-Delaunay
//     interior edge proposes itself, an edge flips when it holds the minimum
//     priority on both of its triangles, neighbour links are repaired through
//     a forwarding table.  Converges to the unique Delaunay triangulation
//     under the symbolic perturbation below.
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

// Triangulate the strip between an upper row A[0..m) and a lower row
// B[0..n), both sorted by strictly increasing x.  Writes (m-1)+(n-1)
// counter-clockwise triangles.
HD void zipper(Pts P, const int32_t* A, int m, const int32_t* B, int n, int32_t* tri) {
    int i = 0, j = 0, k = 0;
    while (i < m - 1 || j < n - 1) {
        bool adv_a;
        if (i == m - 1) adv_a = false;
        else if (j == n - 1) adv_a = true;
        else adv_a = incircle(P, A[i], A[i + 1], B[j], B[j + 1]) <= 0;
        if (adv_a) {
            tri[3 * k] = A[i]; tri[3 * k + 1] = A[i + 1]; tri[3 * k + 2] = B[j];
            ++i;
        } else {
            tri[3 * k] = A[i]; tri[3 * k + 1] = B[j + 1]; tri[3 * k + 2] = B[j];
            ++j;
        }
        ++k;
    }
}

// Fill the pocket between a boundary chain (one point per non-empty row,
// top to bottom) and its convex hull.  side = +1 for the left chain (first
// points), -1 for the right chain (last points).  `stack` has room for
// `len` entries.  Returns the number of triangles written.
HD int fill_pockets(Pts P, const int32_t* chain, int len, int side, int32_t* stack, int32_t* tri) {
    int sp = 0, k = 0;
    for (int i = 0; i < len; ++i) {
        int p = chain[i];
        while (sp >= 2) {
            int64_t o = orient(P, stack[sp - 2], stack[sp - 1], p);
            if (side > 0 ? (o > 0) : (o < 0)) {
                if (side > 0) {
                    tri[3 * k] = stack[sp - 2]; tri[3 * k + 1] = stack[sp - 1]; tri[3 * k + 2] = p;
                } else {
                    tri[3 * k] = stack[sp - 2]; tri[3 * k + 1] = p; tri[3 * k + 2] = stack[sp - 1];
                }
                ++k;
                --sp;
            } else {
                break;
            }
        }
        stack[sp++] = p;
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

// Per-problem state of one triangulation.
struct Tri {
    Pts P;
    int32_t* tri;       // [3*Tmax] vertex triples, counter-clockwise
    int32_t* opp;       // [3*Tmax] neighbour half-edge (3*t+s) across edge (v_s, v_s+1), -1 = hull
    uint32_t* lock;     // [Tmax]
    int32_t* fwd;       // [3*Tmax] old half-edge -> new half-edge within a flip round
    int32_t* cand;      // [2*Tmax] candidate half-edges of the current round
    int32_t* ctr;       // counters: [0] triangles, [1] strip triangles, [2],[3] candidates (round parity),
                        //           [4] rounds used, [5] flips done, [6] non-empty rows
    int Tmax;
};

// Phase A of a flip round for triangle t: clear forwarding, test the edges
// this triangle owns (neighbour index larger), propose the illegal ones.
// Returns false if an index is out of range.
template <class AtomicMin, class AtomicAdd>
HD bool flip_propose(Tri& S, int t, int T, uint32_t round, AtomicMin amin, AtomicAdd aadd) {
    for (int s = 0; s < 3; ++s) S.fwd[3 * t + s] = -1;
    bool ok = true;
    for (int s = 0; s < 3; ++s) {
        int o = S.opp[3 * t + s];
        if (o < 0) continue;
        int n = o / 3;
        if (n <= t) continue;
        if (n >= T) { ok = false; continue; }
        int sn = o % 3;
        int a = S.tri[3 * t + s], b = S.tri[3 * t + (s + 1) % 3], c = S.tri[3 * t + (s + 2) % 3];
        int d = S.tri[3 * n + (sn + 2) % 3];
        if (inside_sos(S.P, a, b, c, d)) {
            uint32_t p = prio(uint32_t(3 * t + s), round);
            amin(&S.lock[t], p);
            amin(&S.lock[n], p);
            int idx = aadd(&S.ctr[2 + (round & 1)], 1);
            if (idx < 2 * S.Tmax) S.cand[idx] = 3 * t + s;
            else ok = false;
        }
    }
    return ok;
}

// Phase B for one candidate half-edge e: flip if it won both locks.
HD bool flip_apply(Tri& S, int e, uint32_t round) {
    int t = e / 3, s = e % 3;
    int o = S.opp[e];
    if (o < 0) return false;
    int n = o / 3, sn = o % 3;
    uint32_t p = prio(uint32_t(e), round);
    if (S.lock[t] != p || S.lock[n] != p) return false;
    int a = S.tri[3 * t + s], b = S.tri[3 * t + (s + 1) % 3], c = S.tri[3 * t + (s + 2) % 3];
    int d = S.tri[3 * n + (sn + 2) % 3];
    int O_bc = S.opp[3 * t + (s + 1) % 3], O_ca = S.opp[3 * t + (s + 2) % 3];
    int O_ad = S.opp[3 * n + (sn + 1) % 3], O_db = S.opp[3 * n + (sn + 2) % 3];
    // t' = (c, a, d), n' = (d, b, c); the new diagonal (d,c)/(c,d) is slot 2 of both
    S.tri[3 * t] = c; S.tri[3 * t + 1] = a; S.tri[3 * t + 2] = d;
    S.tri[3 * n] = d; S.tri[3 * n + 1] = b; S.tri[3 * n + 2] = c;
    S.opp[3 * t] = O_ca; S.opp[3 * t + 1] = O_ad; S.opp[3 * t + 2] = FINAL | (3 * n + 2);
    S.opp[3 * n] = O_db; S.opp[3 * n + 1] = O_bc; S.opp[3 * n + 2] = FINAL | (3 * t + 2);
    S.fwd[3 * t + (s + 2) % 3] = 3 * t;        // edge c-a  -> t' slot 0
    S.fwd[3 * t + (s + 1) % 3] = 3 * n + 1;    // edge b-c  -> n' slot 1
    S.fwd[3 * n + (sn + 1) % 3] = 3 * t + 1;   // edge a-d  -> t' slot 1
    S.fwd[3 * n + (sn + 2) % 3] = 3 * n;       // edge d-b  -> n' slot 0
    return true;
}

// Phase C for triangle t: resolve neighbour links through the forwarding
// table and release the lock.
HD void flip_repair(Tri& S, int t) {
    for (int s = 0; s < 3; ++s) {
        int o = S.opp[3 * t + s];
        if (o < 0) continue;
        if (o & FINAL) {
            S.opp[3 * t + s] = o & ~FINAL;
        } else {
            int f = S.fwd[o];
            if (f >= 0) S.opp[3 * t + s] = f;
        }
    }
    S.lock[t] = LOCK_FREE;
}

// Rotate a triangle so its smallest vertex index comes first.
HD void normalise(int32_t* v) {
    int a = v[0], b = v[1], c = v[2];
    while (a > b || a > c) { int x = a; a = b; b = c; c = x; }
    v[0] = a; v[1] = b; v[2] = c;
}

}  // namespace del
}  // namespace elas
