// Support-point matching and the filters on the candidate lattice.
//
// Replaces kerComputeSupportMatches (src/Kernels/KerSupportMatches.cu:12-193,
// launched L->R then R->L from src/Elas.cu:200-225), the inconsistency and
// redundancy filters (:195-357), the compaction (kerFlag + cub scan +
// kerCompact, :360-421 and src/Elas.cu:338-394) and the disparity grid
// (kerLoadGridValues + kerCreateGird, src/Kernels/KerGrid.cu:8-126).
//
// Sweep design.  A CTA owns a segment of one candidate row and stages the
// four descriptor rows every candidate of that row reads (rows v-2 and v+2
// of both images) in shared memory, so the d-sweep reads shared memory only.
// A warp sweeps one candidate: lane l takes d = dmin + l + 32k, as the
// reference's 32-thread block does, and per-lane states are merged with
// shuffles.  The SAD of a 16-byte descriptor pair is four chained
// vabsdiff4.add; the four rows arrive in shared memory by bulk copy (TMA).
//
// Reduction.  The reference keeps (best, second best) per lane with strict
// '<' and lets lane 0 merge its own registers and then all 32 lanes' pairs
// from shared memory -- lane 0's pair a second time.  Its outcome is a
// function of a commutative state (E1 = min energy, key = (lane, d) of the
// first minimum in merge order, c = number of minima capped at 2,
// E2 = smallest energy among the other disparities):
//   second = (c >= 2 or lane(d*) == 0) ? E1 : E2
//   accept iff c >= 1 and (float)E1 < support_threshold * (float)second
// which is what the warp computes; the oracle restates the reference's
// lane-by-lane merge literally and the tests compare the two.
#include <cuda_runtime.h>
#include "common.cuh"
#include "launch.cuh"
#include "kernels.h"
#include "proposal.h"

namespace elas {

namespace {

constexpr int INF_E = 0x7fffffff;

struct Top2 {
    int e1, key, c, e2;
};

__device__ __forceinline__ void top2_add(Top2& s, int e, int key) {
    if (e < s.e1) { s.e2 = s.e1; s.e1 = e; s.key = key; s.c = 1; }
    else if (e == s.e1) { s.c = s.c >= 1 ? 2 : 1; s.e2 = e; s.key = min(s.key, key); }
    else if (e < s.e2) { s.e2 = e; }
}

__device__ __forceinline__ void top2_merge(Top2& a, const Top2& b) {
    if (b.e1 < a.e1) {
        a.e2 = min(a.e1, b.e2);
        a.e1 = b.e1; a.key = b.key; a.c = b.c;
    } else if (b.e1 == a.e1) {
        if (a.e1 != INF_E) {
            a.c = min(a.c + b.c, 2);
            a.e2 = a.e1;
            a.key = min(a.key, b.key);
        }
    } else {
        a.e2 = min(a.e2, b.e1);
    }
}

// One candidate sweep by a full warp.  self_m2/self_p2: rows v-2/v+2 of the
// image the candidate lives in; oth_m2/oth_p2: the same rows of the other
// image.  dir = -1 (left view: u_warp = u - d) or +1 (right view).
// Returns the accepted disparity or -1 (lane 0's value is authoritative,
// all lanes return the same value).
__device__ __forceinline__ int sweep_candidate(const uint4* self_m2, const uint4* self_p2,
                                               const uint4* oth_m2, const uint4* oth_p2, int u, int dmin,
                                               int dmax, int dir, float thr) {
    const int lane = threadIdx.x & 31;
    const uint4 c0 = self_m2[u - 2], c1 = self_m2[u + 2], c2 = self_p2[u - 2], c3 = self_p2[u + 2];
    Top2 s{INF_E, 0x7fffffff, 0, INF_E};
    for (int d = dmin + lane; d <= dmax; d += 32) {
        int uw = u + dir * d;
        int e = sad16(c0, oth_m2[uw - 2]);
        e = sad16(c1, oth_m2[uw + 2], e);
        e = sad16(c2, oth_p2[uw - 2], e);
        e = sad16(c3, oth_p2[uw + 2], e);
        top2_add(s, e, (((d - dmin) & 31) << 16) | d);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        Top2 t;
        t.e1 = __shfl_xor_sync(0xffffffffu, s.e1, o);
        t.key = __shfl_xor_sync(0xffffffffu, s.key, o);
        t.c = __shfl_xor_sync(0xffffffffu, s.c, o);
        t.e2 = __shfl_xor_sync(0xffffffffu, s.e2, o);
        top2_merge(s, t);
    }
    if (s.c < 1) return -1;
    int second = (s.c >= 2 || (s.key >> 16) == 0) ? s.e1 : s.e2;
    if (float(s.e1) < thr * float(second)) return s.key & 0xffff;
    return -1;
}

// Learned-proposal sweep of one candidate by a full warp: only the
// disparities of the packed bin set `bins` (up to four bins of width w, each
// widened by pn::MARGIN pixels on both sides, clipped to [dmin, dmax]) are
// matched.  Accepted iff the minimum energy is attained once and
// (float)E1 < thr * (float)E2, E2 the smallest energy of the other
// disparities of the set; returns the disparity or -1.
__device__ __forceinline__ int sweep_restricted(const uint4* self_m2, const uint4* self_p2, const uint4* oth_m2,
                                                const uint4* oth_p2, int u, int dmin, int dmax, int dir, float thr,
                                                uint32_t bins, int w) {
    const int lane = threadIdx.x & 31;
    const int L = w + 2 * pn::MARGIN;
    int lo[pn::TOPK];
#pragma unroll
    for (int r = 0; r < pn::TOPK; ++r) {
        const uint32_t b = (bins >> (8 * r)) & 0xffu;
        lo[r] = b == pn::NO_BIN ? INT32_MIN / 2 : int(b) * w - pn::MARGIN;
    }
    const uint4 c0 = self_m2[u - 2], c1 = self_m2[u + 2], c2 = self_p2[u - 2], c3 = self_p2[u + 2];
    int e1 = INF_E, d1 = 0x7fffffff, c = 0, e2 = INF_E;
    for (int e = lane; e < pn::TOPK * L; e += 32) {
        static_assert(pn::TOPK == 4, "e / L below assumes four bins");
        const int r = int(e >= L) + int(e >= 2 * L) + int(e >= 3 * L);   // e / L, as e < 4 L
        const int lor = r == 0 ? lo[0] : r == 1 ? lo[1] : r == 2 ? lo[2] : lo[3];
        if (lor == INT32_MIN / 2) continue;
        const int d = lor + (e - r * L);
        if (d < dmin || d > dmax) continue;
        bool dup = false;
#pragma unroll
        for (int q = 0; q < pn::TOPK - 1; ++q)
            if (q < r && d >= lo[q] && d < lo[q] + L) dup = true;
        if (dup) continue;
        const int uw = u + dir * d;
        int en = sad16(c0, oth_m2[uw - 2]);
        en = sad16(c1, oth_m2[uw + 2], en);
        en = sad16(c2, oth_p2[uw - 2], en);
        en = sad16(c3, oth_p2[uw + 2], en);
        if (en < e1) { e2 = e1; e1 = en; d1 = d; c = 1; }
        else if (en == e1) { e2 = en; c = 2; d1 = min(d1, d); }
        else if (en < e2) { e2 = en; }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const int oe1 = __shfl_xor_sync(0xffffffffu, e1, o), od1 = __shfl_xor_sync(0xffffffffu, d1, o);
        const int oc = __shfl_xor_sync(0xffffffffu, c, o), oe2 = __shfl_xor_sync(0xffffffffu, e2, o);
        if (oe1 < e1) { e2 = min(e1, oe2); e1 = oe1; d1 = od1; c = oc; }
        else if (oe1 == e1) { if (e1 != INF_E) { c = min(c + oc, 2); e2 = e1; d1 = min(d1, od1); } }
        else { e2 = min(e2, oe1); }
    }
    if (c != 1) return -1;
    return float(e1) < thr * float(e2) ? d1 : -1;
}

// Block: SWEEP_THREADS threads (one candidate per warp at a time).  grid.x =
// segments per candidate row, grid.y = candidate rows.  SMEM: stage the four
// rows when they fit.
constexpr int SWEEP_THREADS = 1024;
constexpr int PROP_FINAL = 1 << 20;     // res[] flag: accepted by the learned proposal, no R->L pass
template <bool SMEM, bool PROP>
__global__ void __launch_bounds__(SWEEP_THREADS) k_support_sweep(const uint4* __restrict__ desc0,
                                                       const uint4* __restrict__ desc1,
                                                       int32_t* __restrict__ can_out, Geom g, DevParams p,
                                                       int seg, unsigned* err, const uint32_t* __restrict__ bins,
                                                       int32_t* __restrict__ stats) {
    grid_dep_wait();
    extern __shared__ __align__(128) uint4 rows[];
    __shared__ int res[256];
    __shared__ uint64_t bar;
    const int W = g.W, H = g.H;
    const int vc = blockIdx.y;
    const int v = vc * g.step;
    const int c_begin = blockIdx.x * seg, c_end = min(g.cw, c_begin + seg);
    if (c_begin >= c_end) return;
    const bool row_ok = v >= 5 && v <= H - 6;
    const uint4 *L_m2, *L_p2, *R_m2, *R_p2;
    if (row_ok) {
        if (SMEM) {
            if (threadIdx.x == 0) {
                const uint4* src[4] = {desc0 + size_t(v - 2) * W, desc0 + size_t(v + 2) * W,
                                       desc1 + size_t(v - 2) * W, desc1 + size_t(v + 2) * W};
                mbar_init(&bar, 1);
                mbar_expect_tx(&bar, 4u * unsigned(W) * 16u);
                for (int r = 0; r < 4; ++r) bulk_g2s_chunked(rows + r * W, src[r], unsigned(W) * 16u, &bar);
            }
            L_m2 = rows; L_p2 = rows + W; R_m2 = rows + 2 * W; R_p2 = rows + 3 * W;
        } else {
            L_m2 = desc0 + size_t(v - 2) * W; L_p2 = desc0 + size_t(v + 2) * W;
            R_m2 = desc1 + size_t(v - 2) * W; R_p2 = desc1 + size_t(v + 2) * W;
        }
    }
    __syncthreads();
    if (SMEM && row_ok && !mbar_wait_bounded(&bar, 0, MBAR_WAIT_LIMIT)) {
        if (threadIdx.x == 0) atomicOr(err, ERRF_TMA_TIMEOUT);
        mbar_wait_bounded(&bar, 0, MBAR_WAIT_LIMIT);   // let the copies in flight land before exiting
        return;
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    // left view: candidates of the segment
    for (int ci = c_begin + warp; ci < c_end; ci += nw) {
        int u = ci * g.step;
        int r = -1;
        if (row_ok && u >= 5 && u <= W - 6) {
            uint4 ctr = desc0[size_t(v) * W + u];
            if (texture16(ctr) >= p.support_texture) {
                int dmax = min(g.D, u - 5);
                if (dmax - g.dmin >= 10) {
                    bool done = false;
                    if (PROP) {
                        // learned search set first: accepted only if the same
                        // uniqueness and left/right tests pass on it
                        const uint32_t bset = bins[size_t(vc) * g.cw + ci];
                        const int w = pn::bin_width(g.D);
                        const int rl = bset == 0xffffffffu ? -1
                                           : sweep_restricted(L_m2, L_p2, R_m2, R_p2, u, g.dmin, dmax, -1,
                                                              p.support_threshold, bset, w);
                        if (rl >= 0) {
                            const int ur = u - rl;
                            const uint4 cr = desc1[size_t(v) * W + ur];
                            const int dmaxr = min(g.D, W - ur - 5);
                            if (texture16(cr) >= p.support_texture && dmaxr - g.dmin >= 10) {
                                const int rr = sweep_restricted(R_m2, R_p2, L_m2, L_p2, ur, g.dmin, dmaxr, +1,
                                                                p.support_threshold, bset, w);
                                if (rr >= 0 && abs(rl - rr) <= p.lr_threshold) {
                                    r = rl | PROP_FINAL;
                                    done = true;
                                }
                            }
                        }
                        if (lane == 0) atomicAdd(&stats[done ? 0 : 1], 1);
                    }
                    if (!done)   // the full sweep
                        r = sweep_candidate(L_m2, L_p2, R_m2, R_p2, u, g.dmin, dmax, -1, p.support_threshold);
                }
            }
        }
        if (lane == 0) res[ci - c_begin] = r;
    }
    __syncthreads();
    // right view: re-match accepted candidates from u - d
    for (int ci = c_begin + warp; ci < c_end; ci += nw) {
        int dl = res[ci - c_begin];
        if (dl < 0) continue;
        if (PROP && (dl & PROP_FINAL)) {
            if (lane == 0) res[ci - c_begin] = dl & ~PROP_FINAL;
            continue;
        }
        int u = ci * g.step - dl;
        int r = -1;
        uint4 ctr = desc1[size_t(v) * W + u];
        if (texture16(ctr) >= p.support_texture) {
            int dmax = min(g.D, W - u - 5);
            if (dmax - g.dmin >= 10) {
                int dr = sweep_candidate(R_m2, R_p2, L_m2, L_p2, u, g.dmin, dmax, +1, p.support_threshold);
                if (dr >= 0 && abs(dl - dr) <= p.lr_threshold) r = dl;
            }
        }
        __syncwarp();
        if (lane == 0) res[ci - c_begin] = r;
    }
    __syncthreads();
    for (int ci = c_begin + threadIdx.x; ci < c_end; ci += blockDim.x)
        can_out[size_t(vc) * g.cw + ci] = res[ci - c_begin];
}

// ---------------------------------------------------------------------------
// Plain sweep with Q threads per candidate.  Thread j of a candidate's group
// takes a contiguous slice of its disparity range and keeps a commutative
// state of its slice (Best2 below, equivalent to Top2); the Q states merge
// by shuffles and the closed form above decides, so the result equals the
// reference's lane-by-lane merge whatever the slicing.  Inside a slice the
// other view's descriptors slide: the column read fresh at disparity d
// (u + dir (d + 2)) is the one the four-rows energy needs again at d + 4
// (u + dir (d - 2) then), so each disparity loads one descriptor per row
// instead of two; the last loads live in two register banks.
//
// Packed state of the plain sweep: the two smallest values of
// energy << 17 | lane << 12 | d over the disparities seen (energy < 2^14,
// d < 2^12, lane = (d - dmin) & 31).  The smallest value is the Top2
// state's (E1, first minimum in merge order); the second smallest carries
// the smallest energy among the other disparities, and it equals E1
// exactly when the minimum is attained more than once.  Updates are three
// min/max operations and the state merges by the same rule.
constexpr uint32_t PK_INF = 0xffffffffu;
struct Best2 {
    uint32_t v1, v2;
};
__device__ __forceinline__ uint32_t pack_ek(int e, int d, int dmin) {
    return (uint32_t(e) << 17) | (uint32_t((d - dmin) & 31) << 12) | uint32_t(d);
}
__device__ __forceinline__ void best2_add(Best2& b, uint32_t v) {
    const uint32_t hi = max(b.v1, v);
    b.v1 = min(b.v1, v);
    b.v2 = min(b.v2, hi);
}
__device__ __forceinline__ void best2_merge(Best2& a, const Best2& b) {
    const uint32_t lo = min(a.v1, b.v1), hi = max(a.v1, b.v1);
    a.v2 = min(hi, min(a.v2, b.v2));
    a.v1 = lo;
}
// The reference's decision on a merged state: the disparity, or -1.
__device__ __forceinline__ int best2_decide(const Best2& b, float thr) {
    if (b.v1 == PK_INF) return -1;
    const int e1 = int(b.v1 >> 17);
    const int e2 = b.v2 == PK_INF ? INF_E : int(b.v2 >> 17);
    const int second = ((b.v1 >> 12) & 31u) == 0 ? e1 : e2;
    return float(e1) < thr * float(second) ? int(b.v1 & 0xfffu) : -1;
}

// Energy of disparity d from the fresh and the lagging columns of both rows.
template <int DIR>
__device__ __forceinline__ int slice_energy(const uint4& c0, const uint4& c1, const uint4& c2, const uint4& c3,
                                            const uint4& fm, const uint4& fp, const uint4& lm, const uint4& lp) {
    // c0 / c2 pair with column u + dir d - 2, c1 / c3 with u + dir d + 2
    const int em = DIR < 0 ? sad16(c1, lm, sad16(c0, fm)) : sad16(c1, fm, sad16(c0, lm));
    const int ep = DIR < 0 ? sad16(c3, lp, sad16(c2, fp)) : sad16(c3, fp, sad16(c2, lp));
    return em + ep;
}

template <int DIR>
__device__ __forceinline__ Best2 sweep_slice(const uint4* self_m2, const uint4* self_p2, const uint4* oth_m2,
                                             const uint4* oth_p2, int u, int dmin, int da, int db) {
    Best2 s{PK_INF, PK_INF};
    if (da > db) return s;
    const uint4 c0 = self_m2[u - 2], c1 = self_m2[u + 2], c2 = self_p2[u - 2], c3 = self_p2[u + 2];
    // two register banks of lagging columns: bank A serves d = d0 .. d0+3
    // and receives the fresh columns of d0+4 .. d0+7, which serve the next
    // block; no register is copied
    uint4 Am[4], Ap[4], Bm[4], Bp[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int d = da + k;
        if (d <= db) {
            const int x = u + DIR * (d - 2);
            Am[k] = oth_m2[x];
            Ap[k] = oth_p2[x];
        }
    }
    int d0 = da;
    for (; d0 + 7 <= db; d0 += 8) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int d = d0 + k;
            const int x = u + DIR * (d + 2);
            Bm[k] = oth_m2[x];
            Bp[k] = oth_p2[x];
            best2_add(s, pack_ek(slice_energy<DIR>(c0, c1, c2, c3, Bm[k], Bp[k], Am[k], Ap[k]), d, dmin));
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int d = d0 + 4 + k;
            const int x = u + DIR * (d + 2);
            Am[k] = oth_m2[x];
            Ap[k] = oth_p2[x];
            best2_add(s, pack_ek(slice_energy<DIR>(c0, c1, c2, c3, Am[k], Ap[k], Bm[k], Bp[k]), d, dmin));
        }
    }
    // tail: fewer than 8 disparities left (bank A lags d0 .. d0+3)
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int d = d0 + k;
        if (d <= db) {
            const int x = u + DIR * (d + 2);
            Bm[k] = oth_m2[x];
            Bp[k] = oth_p2[x];
            best2_add(s, pack_ek(slice_energy<DIR>(c0, c1, c2, c3, Bm[k], Bp[k], Am[k], Ap[k]), d, dmin));
        }
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int d = d0 + 4 + k;
        if (d <= db) {
            const int x = u + DIR * (d + 2);
            const uint4 fm = oth_m2[x], fp = oth_p2[x];
            best2_add(s, pack_ek(slice_energy<DIR>(c0, c1, c2, c3, fm, fp, Bm[k], Bp[k]), d, dmin));
        }
    }
    return s;
}

// Merge the states of a group of Q consecutive lanes and decide; every
// lane of the group returns the same value.
template <int Q>
__device__ __forceinline__ int group_decide(Best2 s, float thr) {
#pragma unroll
    for (int o = Q / 2; o > 0; o >>= 1) {
        Best2 t;
        t.v1 = __shfl_xor_sync(0xffffffffu, s.v1, o);
        t.v2 = __shfl_xor_sync(0xffffffffu, s.v2, o);
        best2_merge(s, t);
    }
    return best2_decide(s, thr);
}

// Slice [da, db] of thread j of Q over the range [lo, hi].  The slice
// length is odd, so the eight slices of a candidate start in eight
// different 16-byte bank groups and one shared-memory phase (8 lanes of a
// 16-byte load) is free of conflicts.
__device__ __forceinline__ void slice_of(int lo, int hi, int j, int Q, int& da, int& db) {
    const int n = hi - lo + 1;
    int per = (n + Q - 1) / Q;
    per |= 1;
    da = lo + j * per;
    db = imin(hi, da + per - 1);
}

// Restricted sweep (learned proposal) by the Q threads of a group: thread j
// matches elements j, j + Q, ... of the packed bin set (up to four bins of
// width w, each widened by pn::MARGIN on both sides; overlaps counted once,
// clipped to [dmin, dmax]) into a packed state of energy << 17 | d.
template <int DIR>
__device__ __forceinline__ Best2 restricted_slice(const uint4* self_m2, const uint4* self_p2, const uint4* oth_m2,
                                                  const uint4* oth_p2, int u, int dmin, int dmax, uint32_t bins,
                                                  int w, int j, int Q) {
    Best2 s{PK_INF, PK_INF};
    const int L = w + 2 * pn::MARGIN;
    int lo[pn::TOPK];
#pragma unroll
    for (int r = 0; r < pn::TOPK; ++r) {
        const uint32_t b = (bins >> (8 * r)) & 0xffu;
        lo[r] = b == pn::NO_BIN ? INT32_MIN / 2 : int(b) * w - pn::MARGIN;
    }
    const uint4 c0 = self_m2[u - 2], c1 = self_m2[u + 2], c2 = self_p2[u - 2], c3 = self_p2[u + 2];
    for (int e = j; e < pn::TOPK * L; e += Q) {
        static_assert(pn::TOPK == 4, "e / L below assumes four bins");
        const int r = int(e >= L) + int(e >= 2 * L) + int(e >= 3 * L);   // e / L, as e < 4 L
        const int lor = r == 0 ? lo[0] : r == 1 ? lo[1] : r == 2 ? lo[2] : lo[3];
        if (lor == INT32_MIN / 2) continue;
        const int d = lor + (e - r * L);
        if (d < dmin || d > dmax) continue;
        bool dup = false;
#pragma unroll
        for (int q = 0; q < pn::TOPK - 1; ++q)
            if (q < r && d >= lo[q] && d < lo[q] + L) dup = true;
        if (dup) continue;
        const int uw = u + DIR * d;
        int en = sad16(c0, oth_m2[uw - 2]);
        en = sad16(c1, oth_m2[uw + 2], en);
        en = sad16(c2, oth_p2[uw - 2], en);
        en = sad16(c3, oth_p2[uw + 2], en);
        best2_add(s, (uint32_t(en) << 17) | uint32_t(d));
    }
    return s;
}

// The restricted sweep's decision: accepted iff the minimum energy of the
// set is attained once and (float)E1 < thr * (float)E2, E2 the smallest
// energy of the other disparities of the set.
template <int Q>
__device__ __forceinline__ int group_decide_unique(Best2 s, float thr) {
#pragma unroll
    for (int o = Q / 2; o > 0; o >>= 1) {
        Best2 t;
        t.v1 = __shfl_xor_sync(0xffffffffu, s.v1, o);
        t.v2 = __shfl_xor_sync(0xffffffffu, s.v2, o);
        best2_merge(s, t);
    }
    if (s.v1 == PK_INF) return -1;
    const int e1 = int(s.v1 >> 17);
    const int e2 = s.v2 == PK_INF ? INF_E : int(s.v2 >> 17);
    if (e2 == e1) return -1;
    return float(e1) < thr * float(e2) ? int(s.v1 & 0xfffu) : -1;
}

// grid.x = segments of a candidate row, grid.y = candidate rows; blockDim =
// Q x candidates per pass.  SMEM: the four descriptor rows arrive by bulk
// copy (TMA); otherwise they are read through L1 from global memory.
//
// The candidates that need a sweep are compacted into shared-memory lists
// before each sweep pass, so the groups of a warp all have work:
//   PROP  every candidate first tries its learned search set (left view,
//         then the right view from u - d, both with the restricted rule,
//         then the left/right test); the ones it settles are final, the
//         rest join the list of full sweeps;
//   left  full L->R sweeps of the listed candidates;
//   right full R->L sweeps from u - d of the candidates the left pass
//         accepted, and the left/right test.
constexpr int SWEEP_Q_THREADS = 512;   // at most 64 candidates x 8 threads per pass (128 registers)
constexpr int SETTLED = 1 << 20;       // res[] flag: accepted by the learned proposal, no full right pass
template <int Q, bool SMEM, bool PROP>
__global__ void __launch_bounds__(SWEEP_Q_THREADS) k_support_sweep_q(const uint4* __restrict__ desc0,
                                                          const uint4* __restrict__ desc1,
                                                          int32_t* __restrict__ can_out, Geom g, DevParams p,
                                                          int seg, unsigned* err, const uint32_t* __restrict__ bins,
                                                          int32_t* __restrict__ stats) {
    grid_dep_wait();
    extern __shared__ __align__(128) uint4 rows[];
    __shared__ int res[256];
    __shared__ int16_t lst[256];
    __shared__ int nlst;
    __shared__ uint64_t bar;
    const int W = g.W, H = g.H;
    const int vc = blockIdx.y;
    const int v = vc * g.step;
    const int c_begin = blockIdx.x * seg, c_end = min(g.cw, c_begin + seg);
    if (c_begin >= c_end) return;
    const bool row_ok = v >= 5 && v <= H - 6;
    if (!row_ok) {                       // CTA-uniform: no copy is issued for these rows
        for (int ci = c_begin + threadIdx.x; ci < c_end; ci += blockDim.x) can_out[size_t(vc) * g.cw + ci] = -1;
        return;
    }
    const uint4 *L_m2, *L_p2, *R_m2, *R_p2;
    if (SMEM) {
        if (threadIdx.x == 0) {
            const uint4* src[4] = {desc0 + size_t(v - 2) * W, desc0 + size_t(v + 2) * W,
                                   desc1 + size_t(v - 2) * W, desc1 + size_t(v + 2) * W};
            mbar_init(&bar, 1);
            mbar_expect_tx(&bar, 4u * unsigned(W) * 16u);
            for (int r = 0; r < 4; ++r) bulk_g2s_chunked(rows + r * W, src[r], unsigned(W) * 16u, &bar);
        }
        L_m2 = rows; L_p2 = rows + W; R_m2 = rows + 2 * W; R_p2 = rows + 3 * W;
    } else {
        L_m2 = desc0 + size_t(v - 2) * W; L_p2 = desc0 + size_t(v + 2) * W;
        R_m2 = desc1 + size_t(v - 2) * W; R_p2 = desc1 + size_t(v + 2) * W;
    }
    const int n_seg = c_end - c_begin;
    for (int i = threadIdx.x; i < n_seg; i += blockDim.x) res[i] = -1;
    if (threadIdx.x == 0) nlst = 0;
    __syncthreads();
    if (SMEM && !mbar_wait_bounded(&bar, 0, MBAR_WAIT_LIMIT)) {
        if (threadIdx.x == 0) atomicOr(err, ERRF_TMA_TIMEOUT);
        mbar_wait_bounded(&bar, 0, MBAR_WAIT_LIMIT);   // let the copies in flight land before exiting
        return;
    }
    const int j = threadIdx.x % Q, grp = threadIdx.x / Q, per_pass = blockDim.x / Q;
    // candidates that pass the texture and range tests (the learned search set first, with PROP)
    const int passes = (n_seg + per_pass - 1) / per_pass;   // uniform: every lane joins the shuffles
    for (int pass = 0; pass < passes; ++pass) {
        const int k = pass * per_pass + grp, ci = c_begin + k;
        const int u = ci * g.step;
        bool active = false;
        int dmax = 0;
        if (k < n_seg && u >= 5 && u <= W - 6 && texture16(desc0[size_t(v) * W + u]) >= p.support_texture) {
            dmax = min(g.D, u - 5);
            active = dmax - g.dmin >= 10;
        }
        bool settled = false;
        if (PROP) {
            const uint32_t bset = active ? bins[size_t(vc) * g.cw + ci] : 0xffffffffu;
            const int w = pn::bin_width(g.D);
            Best2 sl{PK_INF, PK_INF};
            if (bset != 0xffffffffu)
                sl = restricted_slice<-1>(L_m2, L_p2, R_m2, R_p2, u, g.dmin, dmax, bset, w, j, Q);
            const int rl = group_decide_unique<Q>(sl, p.support_threshold);
            bool tryr = false;
            int ur = 0, dmaxr = 0;
            if (rl >= 0) {
                ur = u - rl;
                dmaxr = min(g.D, W - ur - 5);
                tryr = texture16(desc1[size_t(v) * W + ur]) >= p.support_texture && dmaxr - g.dmin >= 10;
            }
            Best2 sr{PK_INF, PK_INF};
            if (tryr) sr = restricted_slice<1>(R_m2, R_p2, L_m2, L_p2, ur, g.dmin, dmaxr, bset, w, j, Q);
            const int rr = group_decide_unique<Q>(sr, p.support_threshold);
            settled = tryr && rr >= 0 && abs(rl - rr) <= p.lr_threshold;
            if (j == 0 && active) {
                atomicAdd(&stats[settled ? 0 : 1], 1);
                if (settled) res[k] = rl | SETTLED;
            }
        }
        if (j == 0 && active && !settled) lst[atomicAdd(&nlst, 1)] = int16_t(k);
    }
    __syncthreads();
    // left view: full L->R sweeps of the listed candidates
    {
        const int nl = nlst;
        const int lp = (nl + per_pass - 1) / per_pass;
        for (int pass = 0; pass < lp; ++pass) {
            const int q = pass * per_pass + grp;
            const bool active = q < nl;
            const int k = active ? lst[q] : 0;
            const int u = (c_begin + k) * g.step;
            Best2 st{PK_INF, PK_INF};
            if (active) {
                int da, db;
                slice_of(g.dmin, min(g.D, u - 5), j, Q, da, db);
                st = sweep_slice<-1>(L_m2, L_p2, R_m2, R_p2, u, g.dmin, da, db);
            }
            const int r = group_decide<Q>(st, p.support_threshold);
            if (active && j == 0) res[k] = r;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) nlst = 0;
    __syncthreads();
    for (int k = threadIdx.x; k < n_seg; k += blockDim.x) {
        const int r = res[k];
        if (r >= 0 && !(r & SETTLED)) lst[atomicAdd(&nlst, 1)] = int16_t(k);
    }
    __syncthreads();
    // right view: re-match the candidates the full left sweep accepted, from u - d
    {
        const int nl = nlst;
        const int rp = (nl + per_pass - 1) / per_pass;
        for (int pass = 0; pass < rp; ++pass) {
            const int q = pass * per_pass + grp;
            const int k = q < nl ? lst[q] : 0;
            const int dl = q < nl ? res[k] : -1;
            bool active = false;
            int ur = 0, dmax = 0;
            if (dl >= 0) {
                ur = (c_begin + k) * g.step - dl;
                if (texture16(desc1[size_t(v) * W + ur]) >= p.support_texture) {
                    dmax = min(g.D, W - ur - 5);
                    active = dmax - g.dmin >= 10;
                }
            }
            Best2 st{PK_INF, PK_INF};
            if (active) {
                int da, db;
                slice_of(g.dmin, dmax, j, Q, da, db);
                st = sweep_slice<1>(R_m2, R_p2, L_m2, L_p2, ur, g.dmin, da, db);
            }
            const int dr = group_decide<Q>(st, p.support_threshold);
            __syncwarp();
            if (q < nl && j == 0) res[k] = (active && dr >= 0 && abs(dl - dr) <= p.lr_threshold) ? dl : -1;
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < n_seg; k += blockDim.x) {
        const int r = res[k];
        can_out[size_t(vc) * g.cw + c_begin + k] = r >= 0 ? (r & ~SETTLED) : -1;
    }
}

// removeInconsistentSupportPoints with snapshot semantics (k_incon_rows
// below reads the unfiltered lattice and writes a separate one).  The
// reference's bound `y < can_width` (KerSupportMatches.cu:208) is kept: rows
// y >= cw pass through.

// Redundancy filter along one line (removeRedundantSupportPoints*,
// KerSupportMatches.cu:241-357): point k is removed when it has a similar
// (|d - d2| <= 1) valid point within 5 cells on BOTH sides, the left side
// seen after the removals already made on this line, the right side as it
// was.  The lanes precompute, per point, "valid", "right support" and the
// 5-bit mask of similar valid points on the left; what remains serial is a
// 32-state automaton over the 5-bit history of removals
// (hist' = (hist << 1 | rem) & 31, rem = valid & right & (left & ~hist)).
// Each lane runs the automaton over its chunk of the line for all 32
// entry states at once (bit s of H[b] = history bit b when the chunk was
// entered in state s), the lanes then chain their entry states in order,
// and each lane replays its chunk from its actual entry state.
__device__ void redundant_line(int* a, uint8_t* code, int len, int lane) {
    for (int k = lane; k < len; k += 32) {
        // the ten neighbours are loaded independently (no early exit), so
        // their loads overlap
        const int d = a[k];
        int c = 0;
        if (d >= 0) {
            c = 1;
            bool right = false;
#pragma unroll
            for (int j = 1; j <= 5; ++j) {
                const int d2 = k + j < len ? a[k + j] : -1;
                right = right || (d2 >= 0 && abs(d - d2) <= 1);
            }
            c |= right ? 2 : 0;
#pragma unroll
            for (int b = 0; b < 5; ++b) {
                const int d2 = k - 1 - b >= 0 ? a[k - 1 - b] : -1;
                if (d2 >= 0 && abs(d - d2) <= 1) c |= 4 << b;
            }
        }
        code[k] = uint8_t(c);
    }
    __syncwarp();
    const int chunk = (len + 31) / 32;
    const int k0 = imin(len, lane * chunk), k1 = imin(len, k0 + chunk);
    uint32_t H0 = 0xAAAAAAAAu, H1 = 0xCCCCCCCCu, H2 = 0xF0F0F0F0u, H3 = 0xFF00FF00u, H4 = 0xFFFF0000u;
#pragma unroll 4
    for (int k = k0; k < k1; ++k) {
        const unsigned c = code[k];
        uint32_t R = 0;
        if ((c & 3u) == 3u) {
            if (c & 4u) R |= ~H0;
            if (c & 8u) R |= ~H1;
            if (c & 16u) R |= ~H2;
            if (c & 32u) R |= ~H3;
            if (c & 64u) R |= ~H4;
        }
        H4 = H3; H3 = H2; H2 = H1; H1 = H0; H0 = R;
    }
    // entry state of every lane: chain the lanes' maps from state 0
    unsigned s = 0, mine = 0;
    for (int i = 0; i < 32; ++i) {
        const uint32_t h0 = __shfl_sync(0xffffffffu, H0, i), h1 = __shfl_sync(0xffffffffu, H1, i),
                       h2 = __shfl_sync(0xffffffffu, H2, i), h3 = __shfl_sync(0xffffffffu, H3, i),
                       h4 = __shfl_sync(0xffffffffu, H4, i);
        if (lane == i) mine = s;
        s = ((h0 >> s) & 1u) | (((h1 >> s) & 1u) << 1) | (((h2 >> s) & 1u) << 2) | (((h3 >> s) & 1u) << 3) |
            (((h4 >> s) & 1u) << 4);
    }
    unsigned hist = mine;   // bit b: point k-1-b was removed
#pragma unroll 4
    for (int k = k0; k < k1; ++k) {
        const unsigned c = code[k];
        const unsigned rem = (c & 1u) && (c & 2u) && ((c >> 2) & ~hist & 31u) ? 1u : 0u;
        hist = ((hist << 1) | rem) & 31u;
        if (rem) a[k] = -1;
    }
    __syncwarp();
}

// One warp per line; horizontal = 1: rows, 0: columns.  row_cnt (vertical
// pass, zeroed by k_incon_rows): every point kept adds 1 to its row's count,
// which k_compact turns into the row's first list position.
__global__ void k_redundant(int32_t* __restrict__ can, Geom g, int horizontal, int32_t* __restrict__ row_cnt) {
    grid_dep_wait();
    extern __shared__ int lines[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nlines = horizontal ? g.ch : g.cw;
    const int len = horizontal ? g.cw : g.ch;
    int l = blockIdx.x * (blockDim.x >> 5) + warp;
    if (l >= nlines) return;
    int* a = lines + warp * len;
    uint8_t* code = reinterpret_cast<uint8_t*>(lines + (blockDim.x >> 5) * len) + warp * len;
    for (int k = lane; k < len; k += 32)
        a[k] = horizontal ? can[size_t(l) * g.cw + k] : can[size_t(k) * g.cw + l];
    __syncwarp();
    redundant_line(a, code, len, lane);
    for (int k = lane; k < len; k += 32) {
        if (horizontal) can[size_t(l) * g.cw + k] = a[k];
        else can[size_t(k) * g.cw + l] = a[k];
        if (row_cnt && !horizontal && a[k] >= 0) atomicAdd(&row_cnt[k], 1);
    }
}

// k_incon and the horizontal k_redundant pass in one kernel: one CTA per
// candidate row computes the row's inconsistency filter (as k_incon, reading
// the unfiltered lattice) into shared memory, warp 0 runs the row's
// redundancy recurrence there, and the row is written once.  The window's
// lattice rows are staged in shared memory first (STAGED; windows too tall
// for it read the lattice in place), and PARTS neighbouring lanes share a
// candidate, each counting every PARTS-th window row; the counts are summed
// across the lanes.  Narrow lattices (few candidates per row, too few CTAs
// to fill the GPU) take 4 lanes per candidate, wide ones 1.
constexpr size_t INCON_STAGE_MAX = 96 * 1024;   // shared-memory bytes up to which the window is staged
template <bool STAGED, int PARTS>
__global__ void k_incon_rows(const int32_t* __restrict__ cin, int32_t* __restrict__ cout, Geom g, DevParams p,
                             int32_t* __restrict__ row_cnt) {
    grid_dep_wait();
    if (threadIdx.x == 0) row_cnt[blockIdx.x] = 0;     // counted by the vertical redundancy pass
    extern __shared__ int sm[];                  // [window rows x cw ints when STAGED], cw ints, cw code bytes
    const int ws = p.incon_window, y = blockIdx.x;
    const int ylo = max(0, y - ws), yhi = min(g.ch - 1, y + ws), nr = yhi - ylo + 1;
    int* row = sm + (STAGED ? nr * g.cw : 0);
    uint8_t* code = reinterpret_cast<uint8_t*>(row + g.cw);
    const int* win = STAGED ? sm : cin + size_t(ylo) * g.cw;    // the window's rows, from ylo
    if (STAGED) {
        for (int i = threadIdx.x; i < nr * g.cw; i += blockDim.x) sm[i] = cin[size_t(ylo) * g.cw + i];
        __syncthreads();
    }
    const int part = threadIdx.x % PARTS, per = blockDim.x / PARTS;
    for (int x0 = 0; x0 < g.cw; x0 += per) {   // every lane of a warp takes the same trips (the shuffles)
        const int x = x0 + int(threadIdx.x) / PARTS;
        const int d = x < g.cw ? win[(y - ylo) * g.cw + x] : -1;
        const bool check = d >= 0 && y < g.cw;
        int support = 0;
        if (check) {
            const int xa = max(0, x - ws), xb = min(g.cw - 1, x + ws);
            for (int r = part; r < nr; r += PARTS)
                for (int x2 = xa; x2 <= xb; ++x2) {
                    const int d2 = win[r * g.cw + x2];
                    support += d2 >= 0 && abs(d - d2) <= p.incon_threshold;
                }
        }
#pragma unroll
        for (int o = 1; o < PARTS; o <<= 1) support += __shfl_xor_sync(0xffffffffu, support, o);
        if (x < g.cw && part == 0) row[x] = check && support < p.incon_min_support ? -1 : d;
    }
    __syncthreads();
    if (threadIdx.x < 32) redundant_line(row, code, g.cw, threadIdx.x);
    __syncthreads();
    for (int x = threadIdx.x; x < g.cw; x += blockDim.x) cout[size_t(y) * g.cw + x] = row[x];
}

// Write the support list in raster order: uvd (u, v, d), and the point
// coordinates of both views (x0 = u, x1 = u - d, y = v).  One CTA per
// lattice row; the row's first list position is the sum of the counts of
// the rows before it (row_cnt, counted by the vertical redundancy pass),
// summed here, so no scan pass runs.  row_off gets every row's first
// position, row_off[ch] the total.  front = 3 with add_corners: three
// corner points lead row 0 (row_off[0] stays 0, row 0 spans them) and three
// more form the extra row ch (row_off[ch + 1] = total + 6).
__global__ void k_compact(const int32_t* __restrict__ can, const int32_t* __restrict__ row_cnt,
                          int32_t* __restrict__ row_off, int32_t* __restrict__ uvd, int32_t* __restrict__ x0,
                          int32_t* __restrict__ x1, int32_t* __restrict__ y, Geom g, int front) {
    grid_dep_wait();
    __shared__ int warp_tot[32];
    __shared__ int base;
    const int r = blockIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int pre = 0;
    for (int i = threadIdx.x; i < r; i += blockDim.x) pre += row_cnt[i];
    pre = __reduce_add_sync(0xffffffffu, pre);
    if (lane == 0) warp_tot[warp] = pre;
    __syncthreads();
    if (threadIdx.x == 0) {
        int sum = 0;
        for (int w = 0; w < nw; ++w) sum += warp_tot[w];
        base = sum + front;
        row_off[r] = sum + (r > 0 ? front : 0);
        if (r == g.ch - 1) {
            const int total = sum + row_cnt[r];
            row_off[g.ch] = total + front;
            if (front) row_off[g.ch + 1] = total + 6;
        }
    }
    __syncthreads();
    for (int x0c = 0; x0c < g.cw; x0c += blockDim.x) {
        int x = x0c + threadIdx.x;
        int d = x < g.cw ? can[size_t(r) * g.cw + x] : -1;
        unsigned m = __ballot_sync(0xffffffffu, d >= 0);
        if (lane == 0) warp_tot[warp] = __popc(m);
        __syncthreads();
        int off = 0, tot = 0;
        for (int w = 0; w < nw; ++w) { if (w < warp) off += warp_tot[w]; tot += warp_tot[w]; }
        if (d >= 0) {
            int i = base + off + __popc(m & ((1u << lane) - 1));
            int u = x * g.step, vv = r * g.step;
            uvd[3 * i] = u; uvd[3 * i + 1] = vv; uvd[3 * i + 2] = d;
            x0[i] = u; x1[i] = u - d; y[i] = vv;
        }
        __syncthreads();
        if (threadIdx.x == 0) base += tot;
        __syncthreads();
    }
}

// add_corners (the reference declares the parameter only, src/Elas.h:23):
// support points at the image corners with the disparity of the nearest
// support point (squared distance, the first one in list order on ties; 0
// when there is none), and, for the right view, the two right corners moved
// by their disparity (u = W - 1 + d, so that u - d = W - 1).  Layout: the
// three points of row 0 -- (0, 0), (W-1, 0), (W-1+d, 0) -- lead the list,
// the three of row H-1 -- (0, H-1), (W-1, H-1), (W-1+d, H-1) -- end it as
// the extra row ch.  Every corner lies in a border cell of the grid, which
// the grid leaves empty, so only the triangulations change.
__global__ void __launch_bounds__(1024) k_corners(const int32_t* __restrict__ row_off, int32_t* __restrict__ uvd,
                                                  int32_t* __restrict__ x0, int32_t* __restrict__ x1,
                                                  int32_t* __restrict__ y, Geom g) {
    grid_dep_wait();
    __shared__ unsigned long long best[4][32];
    const int n0 = 3, n1 = row_off[g.ch];          // regular points are [3, n1)
    const int cu[4] = {0, g.W - 1, 0, g.W - 1}, cv[4] = {0, 0, g.H - 1, g.H - 1};
    unsigned long long b[4] = {~0ull, ~0ull, ~0ull, ~0ull};
    for (int i = n0 + threadIdx.x; i < n1; i += blockDim.x) {
        const int u = uvd[3 * i], v = uvd[3 * i + 1];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const long long du = u - cu[k], dv = v - cv[k];
            const unsigned long long key = (unsigned long long)(du * du + dv * dv) << 32 | unsigned(i);
            b[k] = b[k] < key ? b[k] : key;
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long x = __shfl_xor_sync(0xffffffffu, b[k], o);
            b[k] = b[k] < x ? b[k] : x;
        }
        if (lane == 0) best[k][warp] = b[k];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int d[4];
        for (int k = 0; k < 4; ++k) {
            unsigned long long m = ~0ull;
            for (int w = 0; w < int(blockDim.x >> 5); ++w) m = best[k][w] < m ? best[k][w] : m;
            d[k] = m == ~0ull ? 0 : uvd[3 * int(m & 0xffffffffu) + 2];
        }
        const int top[3][3] = {{0, 0, d[0]}, {g.W - 1, 0, d[1]}, {g.W - 1 + d[1], 0, d[1]}};
        const int bot[3][3] = {{0, g.H - 1, d[2]}, {g.W - 1, g.H - 1, d[3]}, {g.W - 1 + d[3], g.H - 1, d[3]}};
        for (int k = 0; k < 6; ++k) {
            const int* q = k < 3 ? top[k] : bot[k - 3];
            const int i = k < 3 ? k : n1 + (k - 3);
            uvd[3 * i] = q[0]; uvd[3 * i + 1] = q[1]; uvd[3 * i + 2] = q[2];
            x0[i] = q[0]; x1[i] = q[0] - q[2]; y[i] = q[1];
        }
    }
}

// kerLoadGridValues as bitsets: for every support point set bits d-1..d+1
// (clamped to [0, D]) in its left cell floor(u/gs) and right cell
// floor((u-d)/gs) of row floor(v/gs).
__global__ void k_grid_load(const int32_t* __restrict__ can, uint32_t* __restrict__ t0,
                            uint32_t* __restrict__ t1, Geom g) {
    grid_dep_wait();
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= g.cw || y >= g.ch) return;
    int dc = can[size_t(y) * g.cw + x];
    if (dc < 0) return;
    int u = x * g.step, v = y * g.step;
    int ug0 = floordiv(u, g.gs), ug1 = floordiv(u - dc, g.gs), vg = floordiv(v, g.gs);
    if (vg < 0 || vg >= g.gh) return;
    for (int d = max(dc - 1, 0); d <= min(dc + 1, g.D); ++d) {
        uint32_t bit = 1u << (d & 31);
        if (ug0 >= 0 && ug0 < g.gw) atomicOr(&t0[(size_t(vg) * g.gw + ug0) * g.words + (d >> 5)], bit);
        if (ug1 >= 0 && ug1 < g.gw) atomicOr(&t1[(size_t(vg) * g.gw + ug1) * g.words + (d >> 5)], bit);
    }
}

// kerCreateGird: 3x3 OR-diffusion for interior cells; border cells empty.
// One thread per (cell, word); blockIdx.z selects the view.
__global__ void k_grid_diffuse(const uint32_t* __restrict__ t0, const uint32_t* __restrict__ t1,
                               uint32_t* __restrict__ g0, uint32_t* __restrict__ g1, Geom g) {
    grid_dep_wait();
    const uint32_t* t = blockIdx.z ? t1 : t0;
    uint32_t* out = blockIdx.z ? g1 : g0;
    size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    size_t n = size_t(g.gw) * g.gh * g.words;
    if (i >= n) return;
    int w = int(i % g.words);
    int cell = int(i / g.words);
    int ug = cell % g.gw, vg = cell / g.gw;
    uint32_t o = 0;
    if (ug > 0 && ug < g.gw - 1 && vg > 0 && vg < g.gh - 1)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) o |= t[(size_t(vg + dy) * g.gw + ug + dx) * g.words + w];
    out[i] = o;
}

}  // namespace

cudaError_t launch_support(const uint4* desc0, const uint4* desc1, int32_t* can_lr, int32_t* can_tmp,
                           int32_t* can, int32_t* row_cnt, const Geom& g, const DevParams& p, int num_sms,
                           unsigned* err, cudaStream_t st, const uint32_t* bins, int32_t* stats) {
    // segments: about 4 CTAs per SM in flight
    int rows = g.ch;
    int segs = imax(1, (4 * num_sms + rows - 1) / imax(rows, 1));
    int seg = imin(256, imax(8, (g.cw + segs - 1) / segs));
    segs = (g.cw + seg - 1) / seg;
    size_t smem = size_t(4) * g.W * sizeof(uint4);
    dim3 grid(segs, rows);
    if (!bins && smem <= 200 * 1024) {
        // plain sweep: 8 threads per candidate, segments of 32..128
        // candidates sized for about two CTAs per SM
        // plain sweep: 8 threads per candidate; segments of at most 256
        // candidates (each CTA stages the four rows once), sized for about
        // two CTAs per SM over the whole lattice
        constexpr int Q = 8;
        const long long cands = (long long)g.cw * imax(rows, 1);
        const int want = int(imin(256, imax(32, int((cands + 2 * num_sms - 1) / (2 * num_sms)))));
        const int qsegs = imax(1, (g.cw + want - 1) / want);
        int qseg = imax(1, (g.cw + qsegs - 1) / qsegs);
        qseg = (qseg + 3) & ~3;
        const int threads = imin(qseg, SWEEP_Q_THREADS / Q) * Q;
        allow_smem(k_support_sweep_q<Q, true, false>);
        launch_k(k_support_sweep_q<Q, true, false>, dim3(qsegs, rows), threads, smem, st, desc0, desc1, can_lr, g, p,
                 qseg, err, nullptr, nullptr);
    } else if (bins && smem <= 200 * 1024) {
        // learned proposal: the same kernel, search sets first, fallbacks compacted
        constexpr int Q = 8;
        const long long cands = (long long)g.cw * imax(rows, 1);
        const int want = int(imin(256, imax(32, int((cands + 2 * num_sms - 1) / (2 * num_sms)))));
        const int qsegs = imax(1, (g.cw + want - 1) / want);
        int qseg = imax(1, (g.cw + qsegs - 1) / qsegs);
        qseg = (qseg + 3) & ~3;
        const int threads = imin(qseg, SWEEP_Q_THREADS / Q) * Q;
        allow_smem(k_support_sweep_q<Q, true, true>);
        launch_k(k_support_sweep_q<Q, true, true>, dim3(qsegs, rows), threads, smem, st, desc0, desc1, can_lr, g, p,
                 qseg, err, bins, stats);
    } else if (smem <= 200 * 1024) {
        if (bins) {
            allow_smem(k_support_sweep<true, true>);
            launch_k(k_support_sweep<true, true>, grid, SWEEP_THREADS, smem, st, desc0, desc1, can_lr, g, p, seg, err, bins,
                                                                           stats);
        } else {
            allow_smem(k_support_sweep<true, false>);
            launch_k(k_support_sweep<true, false>, grid, SWEEP_THREADS, smem, st, desc0, desc1, can_lr, g, p, seg, err,
                                                                            nullptr, nullptr);
        }
    } else {
        if (bins)
            launch_k(k_support_sweep<false, true>, grid, SWEEP_THREADS, 0, st, desc0, desc1, can_lr, g, p, seg, err, bins,
                                                                         stats);
        else
            launch_k(k_support_sweep<false, false>, grid, SWEEP_THREADS, 0, st, desc0, desc1, can_lr, g, p, seg, err,
                                                                          nullptr, nullptr);
    }
    {
        const size_t sm = size_t(g.cw) * (sizeof(int) + 1);
        const size_t wsm = size_t(imin(2 * p.incon_window + 1, g.ch)) * g.cw * sizeof(int);
        const int parts = g.cw <= 256 ? 4 : (g.cw <= 512 ? 2 : 1);
        const int threads = imin(1024, imax(32, ((parts * g.cw + 31) / 32) * 32));
        const bool staged = sm + wsm <= INCON_STAGE_MAX;
        auto go = [&](auto kern, size_t bytes) {
            allow_smem(kern);
            launch_k(kern, g.ch, threads, bytes, st, can_lr, can, g, p, row_cnt);
        };
        if (staged) {
            if (parts == 4) go(k_incon_rows<true, 4>, sm + wsm);
            else if (parts == 2) go(k_incon_rows<true, 2>, sm + wsm);
            else go(k_incon_rows<true, 1>, sm + wsm);
        } else {
            if (parts == 4) go(k_incon_rows<false, 4>, sm);
            else if (parts == 2) go(k_incon_rows<false, 2>, sm);
            else go(k_incon_rows<false, 1>, sm);
        }
        const int wpb = 4;
        const size_t smv = size_t(wpb) * g.ch * (sizeof(int) + 1);
        launch_k(k_redundant, (g.cw + wpb - 1) / wpb, 32 * wpb, smv, st, can, g, 0, row_cnt);
    }
    (void)can_tmp;
    return cudaGetLastError();
}

cudaError_t launch_compact(const int32_t* can, const int32_t* row_cnt, int32_t* row_off, int32_t* uvd, int32_t* x0,
                           int32_t* x1, int32_t* y, const Geom& g, cudaStream_t st, int corners, int* nlaunch) {
    const int launched = 1 + (corners ? 1 : 0);
    launch_k(k_compact, g.ch, 256, 0, st, can, row_cnt, row_off, uvd, x0, x1, y, g, corners ? 3 : 0);
    if (corners) launch_k(k_corners, 1, 1024, 0, st, row_off, uvd, x0, x1, y, g);
    if (nlaunch) *nlaunch += launched;
    return cudaGetLastError();
}

cudaError_t launch_grid(const int32_t* can, uint32_t* tmp0, uint32_t* tmp1, uint32_t* grid0, uint32_t* grid1,
                        const Geom& g, cudaStream_t st, int* nlaunch) {
    if (nlaunch) *nlaunch += 2;
    size_t n = size_t(g.gw) * g.gh * g.words;
    cudaMemsetAsync(tmp0, 0, n * sizeof(uint32_t), st);
    cudaMemsetAsync(tmp1, 0, n * sizeof(uint32_t), st);
    launch_k(k_grid_load, dim3((g.cw + 127) / 128, g.ch), 128, 0, st, can, tmp0, tmp1, g);
    launch_k(k_grid_diffuse, dim3(unsigned((n + 255) / 256), 1, 2), 256, 0, st, tmp0, tmp1, grid0, grid1, g);
    return cudaGetLastError();
}

}  // namespace elas
