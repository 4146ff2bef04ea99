// GPU Delaunay triangulation of the support points of both views
// (algorithm and predicates: delaunay_core.h).  Replaces the reference's
// device->host copy, Triangle call and host->device copy
// (src/Elas.cu:282-328, called twice from :89-90).
//
// Both views run as two independent problems inside the same launches:
// problem 0 triangulates (u, v), problem 1 triangulates (u - d, v).
#include <climits>
#include <cooperative_groups.h>
#include <type_traits>
#include <cuda_runtime.h>
#include "common.cuh"
#include "launch.cuh"
#include "delaunay_core.h"
#include "kernels.h"

namespace elas {

using namespace del;
namespace cg = cooperative_groups;

namespace {

constexpr int SORT_CAP = 2048;   // max candidates per lattice row
constexpr int FLIP_THREADS = 1024;

__device__ __forceinline__ void set_err(unsigned* err, unsigned f) { atomicOr(err, f); }

// Exclusive scan of one int per thread over a 1024-thread block; *total
// receives the sum.  `warp_sums` has 32 entries.
__device__ int block_scan(int v, int* warp_sums, int* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int w = lane < (blockDim.x >> 5) ? warp_sums[lane] : 0;
        int ws = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, ws, o);
            if (lane >= o) ws += y;
        }
        warp_sums[lane] = ws - w;
        if (lane == 31) warp_sums[32] = ws;
    }
    __syncthreads();
    int r = x - v + warp_sums[warp];
    *total = warp_sums[32];
    __syncthreads();
    return r;
}

// Reserve one slot per calling lane in a list whose length counter `ctr`
// is shared by many threads: one atomic per converged group of lanes
// instead of one per lane (shared-memory atomics on one address serialise).
// The order of entries within a list carries no meaning.
__device__ __forceinline__ int agg_inc(int* ctr) {
    const unsigned mask = __activemask();
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(mask) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(ctr, __popc(mask));
    base = __shfl_sync(mask, base, leader);
    return base + __popc(mask & ((1u << lane) - 1u));
}

// As agg_inc, for lanes whose counters may differ (grouped by address).
__device__ __forceinline__ int agg_inc_keyed(int* ctr) {
    const unsigned mask = __activemask();
    const unsigned peers = __match_any_sync(mask, reinterpret_cast<unsigned long long>(ctr));
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(ctr, __popc(peers));
    base = __shfl_sync(mask, base, leader);
    return base + __popc(peers & ((1u << lane) - 1u));
}

// Worklists hold every interior edge at most once per round, as its lower
// half-edge c = min(x, r) (x a half-edge, r its twin; hull edges, r < 0,
// never flip).  `mark` is the round's bitset over half-edges, cleared before
// the round's pushes; the lane that sets c's bit queues it.  With one entry
// per edge, no edge is proposed twice in a round.
__device__ __forceinline__ bool claim_edge(uint32_t* mark, int x, int r, int& c) {
    if (r < 0) return false;
    c = min(x, r);
    const uint32_t bit = 1u << (c & 31);
    return (atomicOr(mark + (c >> 5), bit) & bit) == 0u;
}

// Round 0 of a flip kernel: propose every interior edge of the half-edges
// [h0, h1) once (the owner rule: the half-edge whose triangle has the
// smaller index).  Each warp compacts its owned half-edges through a
// 64-entry ring in shared memory (`ring`, per warp) and proposes them 32 at
// a time, so no lane idles on a twin.  `opp_of(h)` reads a link, `prop(h)`
// proposes; all 32 lanes of every warp of the block must call this.
template <class Opp, class Prop>
__device__ __forceinline__ void propose_owned(int h0, int h1, int32_t* ring, Opp opp_of, Prop prop) {
    const int lane = threadIdx.x & 31;
    int head = 0, cnt = 0;
    for (int base = h0 + int(threadIdx.x & ~31u); base < h1; base += int(blockDim.x)) {
        const int h = base + lane;
        bool own = false;
        if (h < h1) {
            const int o = opp_of(h);
            own = o >= 0 && o / 3 > h / 3;
        }
        const unsigned bal = __ballot_sync(0xffffffffu, own);
        if (own) ring[(head + cnt + __popc(bal & ((1u << lane) - 1u))) & 63] = h;
        cnt += __popc(bal);
        __syncwarp();
        if (cnt >= 32) {
            const int hh = ring[(head + lane) & 63];
            __syncwarp();
            prop(hh);
            head = (head + 32) & 63;
            cnt -= 32;
        }
    }
    __syncwarp();
    if (lane < cnt) prop(ring[(head + lane) & 63]);
}

// Per lattice row: sort the row's points by (x, index), drop repeated x
// (keeps the lowest index), write the unique list to srt[row_off[r] ..]
// (with the packed coordinates beside it in sxy) and its length to rcnt[r];
// pxy[i] gets point i's packed coordinates, or PXY_NONE if it was dropped.
__global__ void __launch_bounds__(512) k_rowsort(DelDev d0, DelDev d1, const int32_t* __restrict__ row_off,
                                                 int nrows, unsigned* err) {
    grid_dep_wait();
    __shared__ unsigned long long key[SORT_CAP];
    __shared__ int keep[SORT_CAP];
    const DelDev& D = blockIdx.y ? d1 : d0;
    const int r = blockIdx.x;
    if (r >= nrows) return;
    const int b = row_off[r], n = row_off[r + 1] - b;
    if (n > SORT_CAP) {
        if (threadIdx.x == 0) { set_err(err, ERRF_BOUNDS); D.rcnt[r] = 0; }
        return;
    }
    int np = 1;
    while (np < n) np <<= 1;
    for (int i = threadIdx.x; i < np; i += blockDim.x)
        // x with its sign bit flipped orders signed coordinates as unsigned keys
        // (the right view's corner points of add_corners lie left of x = 0)
        key[i] = i < n ? (uint64_t(uint32_t(D.x[b + i]) ^ 0x80000000u) << 32 | uint32_t(b + i)) : ~0ull;
    __syncthreads();
    for (int k = 2; k <= np; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < np; i += blockDim.x) {
                int ixj = i ^ j;
                if (ixj > i) {
                    bool up = (i & k) == 0;
                    unsigned long long a = key[i], c = key[ixj];
                    if ((a > c) == up) { key[i] = c; key[ixj] = a; }
                }
            }
            __syncthreads();
        }
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        keep[i] = (i == 0 || (key[i] >> 32) != (key[i - 1] >> 32)) ? 1 : 0;
    __syncthreads();
    // compaction: each warp counts its span, warp 0 turns the counts into offsets
    __shared__ int wcnt[17];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int span = (n + nw - 1) / nw;
    int c = 0;
    for (int i = warp * span + lane; i < min(n, (warp + 1) * span); i += 32) c += keep[i];
    c = __reduce_add_sync(0xffffffffu, c);
    if (lane == 0) wcnt[warp] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int run = 0;
        for (int w = 0; w < nw; ++w) { int t = wcnt[w]; wcnt[w] = run; run += t; }
        wcnt[16] = run;
        D.rcnt[r] = run;
    }
    __syncthreads();
    int base = wcnt[warp];
    const int32_t yr = n > 0 ? D.y[b] : 0;      // the row's y
    for (int i0 = warp * span; i0 < min(n, (warp + 1) * span); i0 += 32) {
        int i = i0 + lane;
        const bool in = i < min(n, (warp + 1) * span);
        bool k = in && keep[i];
        unsigned m = __ballot_sync(0xffffffffu, k);
        if (in) {
            const int32_t idx = int32_t(key[i] & 0xffffffffu);
            const uint32_t xy = pack_xy(int32_t(uint32_t(key[i] >> 32) ^ 0x80000000u), yr);
            // packed coordinates by point (the star searches), PXY_NONE for a dropped duplicate
            D.pxy[idx] = k ? xy : PXY_NONE;
            D.hnext[idx] = -1;
            D.hprev[idx] = -1;
            if (k) {
                const int pos = b + base + __popc(m & ((1u << lane) - 1));
                D.srt[pos] = idx;
                D.sxy[pos] = xy;
            }
        }
        base += __popc(m);
    }
}

// For the star construction, in the block of k_plan once the non-empty
// rows (ne, with their y in ney, both in shared memory) are known: the
// table ylut (y -> first non-empty row at or below y, for y in [0, H]),
// the box of all points (box[0..3]) and the window half-size (box[4],
// star_r0), and the hull boundary (hnext / hprev of every boundary point;
// the rows' extreme points are staged in shared memory and each decided by
// hull_on_chain).  roff and cnt: the rows' offsets and unique counts, also
// in shared memory.
__device__ void star_setup(const DelDev& D, const int32_t* roff, const int32_t* cnt, const int32_t* ne,
                           const int32_t* ney, int R, int H, int npts, uint32_t* xyf, uint32_t* xyl, int32_t* lstk,
                           int32_t* rstk, int* ws) {
    __shared__ int box_s[4];
    const int tid = threadIdx.x, nt = blockDim.x;
    if (tid == 0) {
        box_s[0] = INT_MAX;
        box_s[2] = INT_MIN;
    }
    __syncthreads();
    for (int s = tid; s <= R; s += nt) {
        const int lo = s ? ney[s - 1] + 1 : 0, hi = s < R ? ney[s] : H;
        for (int v = lo; v <= hi && v <= H; ++v) D.ylut[v] = s;
    }
    for (int s = tid; s < R; s += nt) {
        const int r = ne[s], b = roff[r];
        const uint32_t f = D.sxy[b], l = D.sxy[b + cnt[r] - 1];
        xyf[s] = f;
        xyl[s] = l;
        atomicMin(&box_s[0], px_of(f));
        atomicMax(&box_s[2], px_of(l));
    }
    __syncthreads();
    if (tid == 0) {
        const int32_t b[4] = {R ? box_s[0] : 0, R ? ney[0] : 0, R ? box_s[2] : 0, R ? ney[R - 1] : 0};
        for (int k = 0; k < 4; ++k) D.box[k] = b[k];
        D.box[4] = star_r0(b, npts);
    }
    if (R < 2) return;
    // the chains, decided point by point and compacted in row order
    int nl = 0, nr = 0;
    for (int b = 0; b < R; b += nt) {
        const int i = b + tid;
        const int fl = i < R && hull_on_chain(0, R, xyf, i) ? 1 : 0;
        const int fr = i < R && hull_on_chain(1, R, xyl, i) ? 1 : 0;
        int tl_ = 0, tr_ = 0;
        const int pl = block_scan(fl, ws, &tl_);
        const int pr = block_scan(fr, ws, &tr_);
        if (fl) lstk[nl + pl] = i;
        if (fr) rstk[nr + pr] = i;
        nl += tl_;
        nr += tr_;
    }
    __syncthreads();
    const int tl = cnt[ne[0]], bl = cnt[ne[R - 1]];
    const int C = hull_cycle_len(tl, bl, nl, nr);
    auto at = [&](int j) {
        int row, pos;
        bool last;
        hull_cycle_at(j, R, tl, bl, lstk, nl, rstk, nr, &row, &pos, &last);
        const int r = ne[row];
        return D.srt[roff[r] + (last ? cnt[r] - 1 : pos)];
    };
    for (int j = tid; j < C; j += nt) {
        const int v = at(j);
        D.hnext[v] = at(j + 1 == C ? 0 : j + 1);
        D.hprev[v] = at(j == 0 ? C - 1 : j - 1);
    }
}

// Non-empty rows (list, and their y for the star searches), then either the
// star set-up (stars) or the strip offsets (flips).  One 1024-thread block
// per problem; the per-row arrays are staged in shared memory (8 arrays of
// nrows entries).  ctr[7] = 1 when the strip plan holds (two non-empty rows
// at least, strips and pockets within Tmax); the strips and pockets are then
// built by k_strips, which also sets the triangle count ctr[0].
__global__ void __launch_bounds__(1024) k_plan(DelDev d0, DelDev d1, const int32_t* __restrict__ row_off,
                                               int nrows, int H, int flips, unsigned* err) {
    grid_dep_wait();
    __shared__ int ws[33];
    extern __shared__ int32_t psm[];
    int32_t* roff = psm;
    int32_t* cnt = psm + nrows;
    int32_t* ne = psm + 2 * nrows;
    int32_t* ney = psm + 3 * nrows;
    DelDev D = blockIdx.x ? d1 : d0;
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int r = tid; r < nrows; r += nt) {
        roff[r] = row_off[r];
        cnt[r] = D.rcnt[r];
    }
    __syncthreads();
    int R = 0, total = 0;
    // non-empty rows in order
    for (int r0 = 0; r0 < nrows; r0 += nt) {
        const int r = r0 + tid;
        const int f = (r < nrows && cnt[r] > 0) ? 1 : 0;
        const int pos = block_scan(f, ws, &total);
        if (f) ne[R + pos] = r;
        R += total;
    }
    __syncthreads();
    for (int s = tid; s < R; s += nt) {
        const int r = ne[s];
        const int y = D.y[roff[r]];
        ney[s] = y;
        D.ne[s] = r;
        D.ne_y[s] = y;
        D.rinfo[s] = make_int4(y, roff[r], cnt[r], 0);
    }
    __syncthreads();
    const int npts = row_off[nrows];
    int off = 0;
    if (!flips) {
        star_setup(D, roff, cnt, ne, ney, R, H, npts, reinterpret_cast<uint32_t*>(psm + 4 * nrows),
                   reinterpret_cast<uint32_t*>(psm + 5 * nrows), psm + 6 * nrows, psm + 7 * nrows, ws);
    } else {
        // strip s between ne[s] and ne[s+1] holds cnt[ne[s]] + cnt[ne[s+1]] - 2 triangles
        for (int s0 = 0; s0 < R - 1; s0 += nt) {
            const int s2 = s0 + tid;
            const int c = s2 < R - 1 ? cnt[ne[s2]] + cnt[ne[s2 + 1]] - 2 : 0;
            const int pos = block_scan(c, ws, &total);
            if (s2 < R - 1) D.soff[s2] = off + pos;
            off += total;
        }
    }
    if (tid == 0) {
        const bool fits = off + 2 * R <= D.Tmax;
        if (flips && R >= 2 && !fits) set_err(err, ERRF_TRI_COUNT);
        D.ctr[0] = 0;
        D.ctr[1] = off;
        D.ctr[6] = R;
        D.ctr[7] = (flips && R >= 2 && fits) ? 1 : 0;
        D.ctr[8] = 0;    // set to 1 by the flip kernel that handles the problem
        D.ctr[9] = npts;  // support points (vertex ids) of the problem
        D.ctr[4] = 0;    // flip rounds and flips (the flip kernels set them)
        D.ctr[5] = 0;
        D.ctr[11] = 0;   // star construction: overflow pool cursor, searches beyond the window, windows grown
        D.ctr[12] = 0;
        D.ctr[13] = 0;
    }
}

// ---------------------------------------------------------------------------
// Star construction (delaunay_core.h, star_walk): one warp per point finds
// the point's Delaunay neighbours directly, with no initial triangulation
// and no flips.  Candidates come from the rows (ne_y gives each non-empty
// row's y; a row's points are sorted by x with their packed coordinates in
// sxy), gathered into shared memory per window; every search is a warp-wide
// minimum under the star order, so its answer does not depend on how the
// lanes split the candidates.

constexpr int STAR_WARPS = 8;      // points in flight per CTA
constexpr int STAR_SLOT = 12;      // owned triangles kept in a point's own slot; more go to the pool

// The star order as a float key: for the edge p->q (u = q - p) and a
// candidate s (relative to p) strictly on the walk's side, the centre of
// the circle through p, q, s lies at q/2 + t (-uy, ux) with
// t = (|s|^2 - u.s) / (2 cross(u, s)); the next neighbour has the smallest
// t on the left and the largest on the right, i.e. the smallest
// (|s|^2 - u.s) / |cross(u, s)| on either side.  Numerator and denominator
// are exact in int32 (below 2^31 at the coordinate limits of orient_p);
// the key carries at most three roundings (two conversions, one division of
// at most 2 ulp), a relative error below 4e-7, so keys further apart than
// 4e-6 of the larger order their points correctly and closer ones are
// compared exactly.
__device__ __forceinline__ bool star_key(int32_t ux, int32_t uy, int32_t sx, int32_t sy, int side, float* key) {
    const int32_t cr = ux * sy - uy * sx;           // orient(p, q, s)
    if (side > 0 ? cr <= 0 : cr >= 0) return false;
    const int32_t num = sx * sx + sy * sy - (ux * sx + uy * sy);
    *key = __fdividef(__int2float_rn(num), __int2float_rn(cr > 0 ? cr : -cr));
    return true;
}

struct StarSmem {
    int32_t cid[STAR_CAP];         // the point's window: point index
    uint32_t cxy[STAR_CAP];        // and packed coordinates
    int32_t ccw[STAR_NB];          // the walk's two neighbour lists
    int32_t cw[STAR_NB];
};

__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w < v ? w : v;
    }
    return v;
}

// Every point of a region, spread evenly over the warp's lanes: each lane
// takes a row (ylut gives the rows of the region's y range, rinfo each
// row's y, first position and count in one 16-byte load), finds the
// row's column ranges (one, or two beside a ring's hole) by binary search
// in the row's sorted coordinates, and the ranges of 32 rows are then dealt
// out one point per lane (a lane finds the row of its point by a binary
// search over the lanes' offsets).
// take(index, packed xy, k) receives each point with its running number k.
template <class Take>
__device__ void star_stream(const DelDev& D, const int32_t* __restrict__ row_off, const StarRegion& g,
                            const int32_t* box, int lane, Take&& take) {
    if (g.y0 > g.y1) return;
    const int s0 = D.ylut[g.y0], s1 = D.ylut[g.y1 + 1];
    int done = 0;
    // positions [lo, hi) of the row's sorted points with x in [x0, x1]
    auto range = [&](const uint32_t* xs, int cnt, int32_t x0, int32_t x1, int* b, int* n) {
        int l = 0, h = cnt;
        while (l < h) {
            const int mid = (l + h) >> 1;
            if (px_of(xs[mid]) < x0) l = mid + 1;
            else h = mid;
        }
        const int lb = l;
        h = cnt;
        while (l < h) {
            const int mid = (l + h) >> 1;
            if (px_of(xs[mid]) <= x1) l = mid + 1;
            else h = mid;
        }
        *b = lb;
        *n = l - lb;
    };
    for (int sb = s0; sb < s1; sb += 32) {
        const int srow = sb + lane;
        int b = 0, n0 = 0, b1 = 0, n1 = 0;
        if (srow < s1) {
            const int4 ri = D.rinfo[srow];      // y, first position, unique points
            int32_t x0, x1, x2, x3;
            g.cols2(ri.x, box, &x0, &x1, &x2, &x3);
            if (x0 <= x1 || x2 <= x3) {
                const int base = ri.y, cnt = ri.z;
                const uint32_t* xs = D.sxy + base;
                if (x0 <= x1) {
                    range(xs, cnt, x0, x1, &b, &n0);
                    b += base;
                }
                if (x2 <= x3) {
                    range(xs, cnt, x2, x3, &b1, &n1);
                    b1 += base;
                }
            }
        }
        const int n = n0 + n1;
        int incl = n;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const int tot = __shfl_sync(0xffffffffu, incl, 31), excl = incl - n;
        for (int kb = 0; kb < tot; kb += 32) {
            const int k = kb + lane;
            int j = 0;
#pragma unroll
            for (int st = 16; st > 0; st >>= 1) {
                const int c = j + st;
                const int e = __shfl_sync(0xffffffffu, excl, c & 31);
                if (c < 32 && e <= k) j = c;
            }
            const int jb = __shfl_sync(0xffffffffu, b, j), je = __shfl_sync(0xffffffffu, excl, j);
            const int jn0 = __shfl_sync(0xffffffffu, n0, j), jb1 = __shfl_sync(0xffffffffu, b1, j);
            if (k < tot) {
                const int o = k - je;
                const int pos = o < jn0 ? jb + o : jb1 + (o - jn0);
                take(D.srt[pos], D.sxy[pos], done + k);
            }
        }
        done += tot;
    }
}

// Grid-stride over (point, view) with one warp per point: the star
// (star_walk with the two-phase searches of the search policy), its owned
// triangles (p the smallest vertex) counted into tcnt[p] and stored as
// vertex pairs in p's slot (or in the pool when more than STAR_SLOT).
// Three CTAs per SM (80 registers a thread): measured faster at 1242x375
// than four (64 registers, more spills) and than two (no spills, but the
// points no longer fit one wave).
__global__ void __launch_bounds__(STAR_WARPS * 32, 3) k_star(DelDev d0, DelDev d1,
                                                           const int32_t* __restrict__ row_off, unsigned* err) {
    grid_dep_wait();
    __shared__ StarSmem smem[STAR_WARPS];
    // blockIdx.x is the view, so that the two views' first blocks (the ones
    // with points) are dispatched side by side
    const DelDev& D = blockIdx.x ? d1 : d0;
    const int N = D.ctr[9];
    const int32_t box[4] = {D.box[0], D.box[1], D.box[2], D.box[3]};
    const int R0 = D.box[4];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    StarSmem& sm = smem[warp];
    for (int p = blockIdx.y * STAR_WARPS + warp; p < N; p += gridDim.y * STAR_WARPS) {
        const uint32_t pp = D.pxy[p];
        if (pp == PXY_NONE) {
            if (lane == 0) D.tcnt[p] = 0;
            continue;
        }
        const int px = px_of(pp), py = py_of(pp);
        const int hn = D.hnext[p], hp = D.hprev[p];
        int circles = 0, squares = 0;
        // phase 1: the window, staged once (streamed again by each search if it holds more than STAR_CAP)
        const StarRegion win = star_square_region(pp, R0, box);
        int K = 0;
        star_stream(D, row_off, win, box, lane, [&](int32_t s, uint32_t sxy, int k) {
            if (k < STAR_CAP) {
                sm.cid[k] = s;
                sm.cxy[k] = sxy;
            }
            K = k + 1;
        });
        K = __reduce_max_sync(0xffffffffu, K);
        __syncwarp();
        const bool staged = K <= STAR_CAP;
        // the window grows (and stays grown for the point's later searches)
        // while its rings fit behind the staged points
        int Rw = R0;
        bool ring_full = !staged;
        auto grow = [&](auto&& take) {
            ++squares;
            int T = 0;
            star_stream(D, row_off, star_ring_region(pp, Rw, box), box, lane, [&](int32_t s, uint32_t sxy, int k) {
                take(s, sxy);
                if (K + k < STAR_CAP) {
                    sm.cid[K + k] = s;
                    sm.cxy[K + k] = sxy;
                }
                T = k + 1;
            });
            T = __reduce_max_sync(0xffffffffu, T);
            __syncwarp();
            if (K + T > STAR_CAP) {
                ring_full = true;
                return false;
            }
            K += T;
            Rw *= 2;
            return true;
        };
        auto window = [&](auto&& take) {
            if (staged) {
                for (int k = lane; k < K; k += 32) take(sm.cid[k], sm.cxy[k]);
            } else {
                star_stream(D, row_off, win, box, lane, [&](int32_t s, uint32_t sxy, int) { take(s, sxy); });
            }
        };
        auto covers = [&](int Rs) {
            return px - Rs <= box[0] && px + Rs >= box[2] && py - Rs <= box[1] && py + Rs >= box[3];
        };
        // coordinates of the walk's start (q0) and of the last neighbour
        // found, so a step need not load its edge's far end again
        int c0 = hn, c1 = -1;
        uint32_t x0c = hn >= 0 ? D.pxy[hn] : 0u, x1c = 0u;
        auto nearest = [&]() -> int {
            unsigned long long best = ~0ull;
            uint32_t nxy = 0;
            auto take = [&](int32_t s, uint32_t sxy) {
                if (s == p) return;
                const int32_t dx = dx_p(sxy, pp), dy = dy_p(sxy, pp);
                const unsigned long long key = uint64_t(uint32_t(dx * dx + dy * dy)) << 32 | uint32_t(s);
                if (key < best) {
                    best = key;
                    nxy = sxy;
                }
            };
            auto take3 = [&](int32_t s, uint32_t sxy, int) { take(s, sxy); };
            auto finish = [&]() {
                const unsigned long long g = warp_min_u64(best);
                const int wl = __ffs(__ballot_sync(0xffffffffu, best == g)) - 1;
                nxy = __shfl_sync(0xffffffffu, nxy, wl < 0 ? 0 : wl);
                best = g;
            };
            window(take);
            finish();
            for (int Rs = Rw;;) {
                const uint64_t d2 = best >> 32;
                if (best != ~0ull && d2 <= uint64_t(Rs) * uint64_t(Rs)) break;
                if (covers(Rs)) break;
                if (Rs == Rw && !ring_full) {
                    Rs = grow(take) ? Rw : 2 * Rs;
                    finish();
                    continue;
                }
                if (best != ~0ull) {
                    // the nearest lies within distance sqrt(d2): the square of that half-size
                    int d = int(sqrt(double(d2)));
                    while (uint64_t(d) * uint64_t(d) < d2) ++d;
                    ++circles;
                    best = ~0ull;
                    star_stream(D, row_off, star_square_region(pp, d, box), box, lane, take3);
                    finish();
                    break;
                }
                Rs = star_square(Rs);
                ++squares;
                star_stream(D, row_off, star_square_region(pp, Rs, box), box, lane, take3);
                finish();
            }
            if (best == ~0ull) return -1;
            c0 = int(uint32_t(best));
            x0c = nxy;
            return c0;
        };
        auto next = [&](int q, int side) -> int {
            const uint32_t pq = q == c1 ? x1c : (q == c0 ? x0c : D.pxy[q]);
            const int32_t ux = dx_p(pq, pp), uy = dy_p(pq, pp);
            int bi = -1;
            uint32_t bxy = 0;
            float bk = 0.0f;
            // b replaces a (keys ka, kb) under the star order: decided by the
            // keys when they differ by more than their rounding can explain,
            // else exactly (star_better)
            auto wins = [&](float ka, int a, uint32_t axy, float kb, int b, uint32_t bxy2) {
                const float m = 4e-6f * fmaxf(fabsf(ka), fabsf(kb));
                if (kb < ka - m) return true;
                if (kb > ka + m) return false;
                return star_better(p, pp, q, pq, a, axy, b, bxy2, side);
            };
            auto take = [&](int32_t s, uint32_t sxy) {
                float k;
                if (!star_key(ux, uy, dx_p(sxy, pp), dy_p(sxy, pp), side, &k)) return;
                if (bi < 0 || wins(bk, bi, bxy, k, s, sxy)) {
                    bi = s;
                    bxy = sxy;
                    bk = k;
                }
            };
            auto take3 = [&](int32_t s, uint32_t sxy, int) { take(s, sxy); };
            // Minimum under the star order over the lanes' bests.  Fast path:
            // the smallest key (one reduction over order-preserving key
            // bits), final unless another lane's best lies within the keys'
            // rounding of it; then a butterfly decides exactly (the order is
            // strict and total, so every lane ends with the same point).  A
            // lane's other candidates need no look: each is worse than its
            // lane's best, which the winner beats.
            auto reduce = [&]() {
                const uint32_t kb = __float_as_uint(bk);
                const uint32_t u = bi < 0 ? 0xffffffffu : ((kb & 0x80000000u) ? ~kb : (kb | 0x80000000u));
                const uint32_t umin = __reduce_min_sync(0xffffffffu, u);
                if (umin == 0xffffffffu) return;            // no lane holds a candidate
                const int wl = __ffs(__ballot_sync(0xffffffffu, u == umin)) - 1;
                const int wi = __shfl_sync(0xffffffffu, bi, wl);
                const uint32_t wxy = __shfl_sync(0xffffffffu, bxy, wl);
                const float wk = __shfl_sync(0xffffffffu, bk, wl);
                const bool tie = bi >= 0 && bi != wi && fabsf(bk - wk) <= 4e-6f * fmaxf(fabsf(bk), fabsf(wk));
                if (__ballot_sync(0xffffffffu, tie) == 0u) {
                    bi = wi;
                    bxy = wxy;
                    bk = wk;
                    return;
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                    const uint32_t oxy = __shfl_xor_sync(0xffffffffu, bxy, o);
                    const float ok = __shfl_xor_sync(0xffffffffu, bk, o);
                    if (oi >= 0 && oi != bi && (bi < 0 || wins(bk, bi, bxy, ok, oi, oxy))) {
                        bi = oi;
                        bxy = oxy;
                        bk = ok;
                    }
                }
            };
            window(take);
            reduce();
            for (int Rs = Rw;;) {
                if (bi >= 0 && circle_inside(pp, pq, bxy, Rs, box)) break;
                if (covers(Rs)) break;
                if (Rs == Rw && !ring_full) {
                    Rs = grow(take) ? Rw : 2 * Rs;
                    reduce();
                    continue;
                }
                int need = 0;
                if (bi >= 0) circle_within(pp, pq, bxy, Rs, box, &need);
                if (bi >= 0 && need <= 2 * Rs) {
                    ++circles;
                    star_stream(D, row_off, star_circle_region(pp, pq, bxy, box), box, lane, take3);
                    reduce();
                    break;
                }
                Rs = star_square(Rs);
                ++squares;
                star_stream(D, row_off, star_half_region(pp, pq, side, Rs, box), box, lane, take3);
                reduce();
            }
            if (bi >= 0) {
                c1 = bi;
                x1c = bxy;
            }
            return bi;
        };
        int m = 0, k = 0;
        bool closed = false;
        const bool ok = star_walk(hn, hp, nearest, next, sm.ccw, sm.cw, STAR_NB, &m, &k, &closed);
        __syncwarp();
        int own = 0;
        const int deg = m + k, nt = ok ? star_tris(deg, closed) : 0;
        for (int b = 0; b < nt; b += 32) {
            const int i = b + lane;
            bool o = false;
            if (i < nt) {
                const int a = star_at(sm.ccw, m, sm.cw, k, i), c = star_at(sm.ccw, m, sm.cw, k, i + 1 == deg ? 0 : i + 1);
                o = p < a && p < c;
            }
            own += __popc(__ballot_sync(0xffffffffu, o));
        }
        int32_t* dst = D.sown + size_t(p) * 2 * STAR_SLOT;
        if (own > STAR_SLOT) {
            int base = 0;
            if (lane == 0) base = atomicAdd(&D.ctr[11], own);
            base = __shfl_sync(0xffffffffu, base, 0);
            if (base + own > D.Tmax) {
                if (lane == 0) set_err(err, ERRF_BOUNDS);
                own = 0;
            } else {
                if (lane == 0) dst[0] = base;
                dst = D.spool + 2 * size_t(base);
            }
        }
        if (!ok && lane == 0) set_err(err, ERRF_BOUNDS);
        int pos = 0;
        for (int b = 0; b < nt && own > 0; b += 32) {
            const int i = b + lane;
            bool o = false;
            int a = 0, c = 0;
            if (i < nt) {
                a = star_at(sm.ccw, m, sm.cw, k, i);
                c = star_at(sm.ccw, m, sm.cw, k, i + 1 == deg ? 0 : i + 1);
                o = p < a && p < c;
            }
            const unsigned bal = __ballot_sync(0xffffffffu, o);
            if (o) {
                const int j = pos + __popc(bal & ((1u << lane) - 1u));
                dst[2 * j] = a;
                dst[2 * j + 1] = c;
            }
            pos += __popc(bal);
        }
        if (lane == 0) {
            D.tcnt[p] = own;
            if (circles) atomicAdd(&D.ctr[12], circles);
            if (squares) atomicAdd(&D.ctr[13], squares);
        }
        __syncwarp();
    }
}

// 256 points per CTA, both problems: each point's owned triangles (p, a,
// b) at its offset, the exclusive prefix sum of the owned counts in point
// order, so the list is in point order and the same on every run.  A CTA
// finds the sum of all points before its range itself (the star
// construction runs up to 2^21 pixels, some 10^4 points a view, so the
// repeated sums are cheap and save a separate scan launch); CTA 0 also
// sums every point and writes the triangle count ctr[0].
constexpr int EMIT_THREADS = 256;
__global__ void __launch_bounds__(EMIT_THREADS) k_star_emit(DelDev d0, DelDev d1, unsigned* err) {
    grid_dep_wait();
    __shared__ int ws[33];
    const DelDev& D = blockIdx.y ? d1 : d0;
    const int N = D.ctr[9];
    const int start = blockIdx.x * EMIT_THREADS, tid = threadIdx.x;
    if (start >= N && blockIdx.x != 0) return;
    const int lim = blockIdx.x == 0 ? N : start;     // CTA 0 sums everything (the total), the others their prefix
    int pre = 0, total = 0, tmp = 0;
    for (int i = tid; i < lim; i += EMIT_THREADS) {
        if (i < start) pre += D.tcnt[i];
        total += D.tcnt[i];
    }
    block_scan(pre, ws, &tmp);
    pre = tmp;
    block_scan(total, ws, &tmp);
    total = tmp;
    const int p = start + tid;
    const int c = p < N ? D.tcnt[p] : 0;
    int mine = 0;
    const int off = pre + block_scan(c, ws, &mine);
    if (blockIdx.x == 0 && tid == 0) {
        const bool fits = total <= D.Tmax;
        if (!fits) set_err(err, ERRF_TRI_COUNT);
        D.ctr[0] = fits ? total : 0;
    }
    if (c == 0) return;
    if (off + c > D.Tmax) {
        set_err(err, ERRF_TRI_COUNT);
        return;
    }
    const int32_t* slot = D.sown + size_t(p) * 2 * STAR_SLOT;
    const int32_t* src = c <= STAR_SLOT ? slot : D.spool + 2 * size_t(slot[0]);
    int32_t* t = D.tri + 3 * size_t(off);
    for (int j = 0; j < c; ++j) {
        t[3 * j] = p;
        t[3 * j + 1] = src[2 * j];
        t[3 * j + 2] = src[2 * j + 1];
    }
}

// The two hull pockets of one problem, walked at once by lanes 0 of warps 0
// and 1, each on its own copy of the chain (in `sh` when R <= smem_rows,
// else in D.chain); the right side writes behind the left one's room (at
// most R-2 triangles) and is moved down when both are done.  Sets ctr[0].
__device__ void pocket_block(const DelDev& D, const int32_t* __restrict__ row_off, int nrows, int smem_rows,
                             int32_t* sh) {
    __shared__ int npk[2];
    const int R = D.ctr[6], off = D.ctr[1];
    const bool in_smem = R <= smem_rows;
    const int cap = in_smem ? smem_rows : nrows;
    for (int e = threadIdx.x; e < 2 * R; e += blockDim.x) {
        const int side = e >= R, s = e - side * R;
        int32_t* ci = (in_smem ? sh : D.chain) + side * 7 * cap;
        const int r = D.ne[s];
        const int i = D.srt[row_off[r] + (side ? D.rcnt[r] - 1 : 0)];
        ci[s] = i; ci[cap + s] = D.x[i]; ci[2 * cap + s] = D.y[i];
    }
    __syncthreads();
    if ((threadIdx.x & 31) == 0 && threadIdx.x < 64) {
        const int side = threadIdx.x >> 5;
        int32_t* ci = (in_smem ? sh : D.chain) + side * 7 * cap;
        npk[side] = fill_pockets(ci, ci + cap, ci + 2 * cap, R, side ? -1 : +1, ci + 3 * cap,
                                 D.tri + 3 * size_t(off + side * R));
    }
    __syncthreads();
    const int k0 = npk[0], k1 = npk[1];
    // move the right side's triangles from off+R to off+k0 (k0 <= R-2, so
    // a forward copy in rounds of one block never overwrites unread data)
    for (int b0 = 0; b0 < 3 * k1; b0 += blockDim.x) {
        const int j = b0 + threadIdx.x;
        int32_t v = 0;
        if (j < 3 * k1) v = D.tri[3 * size_t(off + R) + j];
        __syncthreads();
        if (j < 3 * k1) D.tri[3 * size_t(off + k0) + j] = v;
        __syncthreads();
    }
    if (threadIdx.x == 0) D.ctr[0] = off + k0 + k1;
}

// Blocks [0, gridDim.x - 1): one thread per sorted point of a non-empty
// row: the point's triangle in the strip below its row (as the upper row)
// and in the strip above (as the lower row), placed by merge path.  The last
// block walks the problem's two hull pockets meanwhile.
__global__ void k_strips(DelDev d0, DelDev d1, const int32_t* __restrict__ row_off, int nrows, int nmax,
                         int smem_rows) {
    grid_dep_wait();
    extern __shared__ int32_t sh[];
    const DelDev& D = blockIdx.y ? d1 : d0;
    if (D.ctr[7] == 0) return;
    if (blockIdx.x == gridDim.x - 1) {
        pocket_block(D, row_off, nrows, smem_rows, sh);
        return;
    }
    const int R = D.ctr[6];
    Pts P{D.x, D.y};
    const int nb = gridDim.x - 1;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < nmax; g += nb * blockDim.x) {
        // g walks the support index space; map it to (row, position) through the row offsets
        int lo = 0, hi = R;    // find the non-empty row whose range holds g
        // rows are in support-index order, so binary search ne by row_off
        while (lo < hi) {
            int mid = (lo + hi) >> 1;
            if (row_off[D.ne[mid] + 1] <= g) lo = mid + 1;
            else hi = mid;
        }
        if (lo >= R) continue;
        int r = D.ne[lo];
        int k = g - row_off[r];
        if (k < 1 || k >= D.rcnt[r]) continue;
        const int32_t* A_row = D.srt + row_off[r];
        int32_t tri[3];
        if (lo + 1 < R) {       // as the upper row of strip lo
            int rb = D.ne[lo + 1];
            int pos = strip_tri_upper(P, A_row, D.srt + row_off[rb], D.rcnt[rb], k, tri);
            int32_t* o = D.tri + 3 * size_t(D.soff[lo] + pos);
            o[0] = tri[0]; o[1] = tri[1]; o[2] = tri[2];
        }
        if (lo >= 1) {          // as the lower row of strip lo-1
            int ra = D.ne[lo - 1];
            int pos = strip_tri_lower(P, D.srt + row_off[ra], D.rcnt[ra], A_row, k, tri);
            int32_t* o = D.tri + 3 * size_t(D.soff[lo - 1] + pos);
            o[0] = tri[0]; o[1] = tri[1]; o[2] = tri[2];
        }
    }
}

__device__ __forceinline__ uint32_t hash_cap(int T) {
    uint32_t need = uint32_t(imax(64, 6 * T));
    uint32_t c = 64;
    while (c < need) c <<= 1;
    return c;
}

__global__ void k_hash_clear(DelDev d0, DelDev d1) {
    grid_dep_wait();
    const DelDev& D = blockIdx.y ? d1 : d0;
    uint32_t cap = hash_cap(D.ctr[0]);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cap && i < D.Hmax; i += gridDim.x * blockDim.x) {
        D.hkey[i] = HASH_EMPTY;
        D.hcnt[i] = 0;
    }
}

__global__ void k_hash_insert(DelDev d0, DelDev d1, unsigned* err) {
    grid_dep_wait();
    const DelDev& D = blockIdx.y ? d1 : d0;
    const int T = D.ctr[0];
    const uint32_t cap = hash_cap(T), mask = cap - 1;
    if (cap > D.Hmax) { if (blockIdx.x == 0 && threadIdx.x == 0) set_err(err, ERRF_HASH); return; }
    for (int h = blockIdx.x * blockDim.x + threadIdx.x; h < 3 * T; h += gridDim.x * blockDim.x) {
        int t = h / 3, s = h % 3;
        uint64_t key = edge_key(D.tri[3 * t + s], D.tri[3 * t + (s + 1) % 3]);
        uint32_t slot = hash64(key) & mask;
        bool done = false;
        for (uint32_t probe = 0; probe < cap; ++probe) {
            unsigned long long prev = atomicCAS(&D.hkey[slot], HASH_EMPTY, (unsigned long long)key);
            if (prev == HASH_EMPTY || prev == key) {
                int pos = atomicAdd(&D.hcnt[slot], 1);
                if (pos < 2) D.hval[2 * slot + pos] = h;
                else set_err(err, ERRF_HASH);
                D.hslot[h] = int(slot);
                done = true;
                break;
            }
            slot = (slot + 1) & mask;
        }
        if (!done) set_err(err, ERRF_HASH);
    }
}

// Neighbour links from the hash, and the per-triangle flip state.
__global__ void k_link(DelDev d0, DelDev d1, unsigned* err) {
    grid_dep_wait();
    const DelDev& D = blockIdx.y ? d1 : d0;
    const int T = D.ctr[0];
    for (int h = blockIdx.x * blockDim.x + threadIdx.x; h < 3 * T; h += gridDim.x * blockDim.x) {
        int slot = D.hslot[h];
        if (slot < 0 || uint32_t(slot) >= D.Hmax) { set_err(err, ERRF_BOUNDS); D.opp[h] = -1; continue; }
        int c = D.hcnt[slot];
        int o = -1;
        if (c == 2) o = D.hval[2 * slot] == h ? D.hval[2 * slot + 1] : D.hval[2 * slot];
        else if (c != 1) set_err(err, ERRF_HASH);
        if (o >= 3 * T) { set_err(err, ERRF_BOUNDS); o = -1; }
        D.opp[h] = o;
    }
}

struct GAMin {
    __device__ void operator()(uint32_t* p, uint32_t v) const { atomicMin(p, v); }
};

// Shared round driver: one "group" (a CTA, or a cluster of CTAs) runs the
// rounds; `Sync` is its barrier.  Lists live in global memory; their
// counters in shared memory of the owning CTA.
//
// Fallback: one 1024-thread CTA per problem on global memory, for
// triangulations larger than the cluster kernel holds.  Every loop is
// bounded: `max_rounds` rounds at most (ERRF_FLIP_LIMIT).
__global__ void __launch_bounds__(FLIP_THREADS) k_flip_global(DelDev d0, DelDev d1, int max_rounds, unsigned* err) {
    grid_dep_wait();
    __shared__ int n_cand, n_flip, n_next, n_cur, stop;
    const DelDev& D = blockIdx.x ? d1 : d0;
    if (D.ctr[8] != 0) return;            // the cluster kernel handled this problem
    const int T = D.ctr[0];
    FlatTri<GAMin> m{D.tri, D.txy, D.opp, D.lock, D.fround, GAMin()};
    const int cand_cap = 3 * D.Tmax, wl_cap = 6 * D.Tmax;
    const int tid = threadIdx.x;
    // the two per-round push bitsets live in hslot, which k_link was the last to read
    const int mark_words = (3 * D.Tmax + 31) / 32, used_words = (3 * T + 31) / 32;
    uint32_t* const mark0 = reinterpret_cast<uint32_t*>(D.hslot);
    uint32_t* const mark1 = mark0 + mark_words;
    for (int t = tid; t < T; t += FLIP_THREADS) { D.lock[t] = LOCK_FREE; D.fround[t] = -1; }
    for (int i = tid; i < 3 * T; i += FLIP_THREADS) {     // packed corner coordinates of the flat storage
        const int v = D.tri[i];
        D.txy[i] = pack_xy(D.x[v], D.y[v]);
    }
    if (tid == 0) { n_cur = 3 * T; stop = 0; }
    __syncthreads();
    int round = 0, flips_total = 0;
    for (; round < max_rounds; ++round) {
        const int32_t* cur = (round & 1) ? D.wl1 : D.wl0;
        int32_t* nxt = (round & 1) ? D.wl0 : D.wl1;
        if (tid == 0) { n_cand = 0; n_next = 0; n_flip = 0; }
        __syncthreads();
        const int items = n_cur;
        for (int k = tid; k < items; k += FLIP_THREADS) {
            int h = round == 0 ? k : cur[k];
            if (!flip_propose(m, h, T, uint32_t(round), round == 0, [&](int hh, int nn) {
                    int idx = agg_inc(&n_cand);
                    if (idx < cand_cap) { D.cand[2 * idx] = hh; D.cand[2 * idx + 1] = nn; }
                }))
                set_err(err, ERRF_BOUNDS);
        }
        // this round's push bitset was last used two rounds ago
        uint32_t* const mark_nxt = (round & 1) ? mark0 : mark1;
        for (int i = tid; i < used_words; i += FLIP_THREADS) mark_nxt[i] = 0u;
        __syncthreads();
        const int nc = n_cand;
        if (tid == 0 && nc > cand_cap) { set_err(err, ERRF_BOUNDS); stop = 1; }
        __syncthreads();
        if (nc == 0 || stop) break;
        for (int c = tid; c < nc; c += FLIP_THREADS) {
            int h = D.cand[2 * c], n = D.cand[2 * c + 1];
            if (flip_apply(m, h, n, uint32_t(round))) {
                int f = agg_inc(&n_flip);
                D.flips[6 * f] = h / 3;
                D.flips[6 * f + 1] = n;
            }
        }
        __syncthreads();
        const int nf = n_flip;
        for (int f = tid; f < nf; f += FLIP_THREADS) {
            int t = D.flips[6 * f], n = D.flips[6 * f + 1];
            for (int k = 0; k < 4; ++k) {
                int r = flip_resolve_slot(m, outer_slot(t, n, k), uint32_t(round), T);
                if (r == -2) { set_err(err, ERRF_BOUNDS); r = -1; }
                D.flips[6 * f + 2 + k] = r;
            }
        }
        __syncthreads();
        auto push = [&](int x, int r) {
            int c;
            if (!claim_edge(mark_nxt, x, r, c)) return;
            int idx = agg_inc(&n_next);
            if (idx < wl_cap) nxt[idx] = c;
        };
        for (int f = tid; f < nf; f += FLIP_THREADS) {
            int t = D.flips[6 * f], n = D.flips[6 * f + 1];
            flip_relink(m, t, n, D.flips + 6 * f + 2);
            for (int k = 0; k < 4; ++k) push(outer_slot(t, n, k), D.flips[6 * f + 2 + k]);
        }
        for (int c = tid; c < nc; c += FLIP_THREADS) {
            int h = D.cand[2 * c], n = D.cand[2 * c + 1], t = h / 3;
            D.lock[t] = LOCK_FREE;
            D.lock[n] = LOCK_FREE;
            if (D.fround[t] != round && D.fround[n] != round) push(h, D.opp[h]);
        }
        flips_total += nf;
        __syncthreads();
        if (tid == 0) {
            if (n_next > wl_cap) { set_err(err, ERRF_BOUNDS); stop = 1; }
            n_cur = min(n_next, wl_cap);
        }
        __syncthreads();
        if (stop) break;
    }
    __syncthreads();
    for (int t = tid; t < T; t += FLIP_THREADS) normalise(D.tri + 3 * size_t(t));
    if (tid == 0) {
        D.ctr[4] = round + 1;
        D.ctr[5] = flips_total;
        if (round >= max_rounds) set_err(err, ERRF_FLIP_LIMIT);
    }
}

// ---------------------------------------------------------------------------
// Cluster kernel: the triangulation of one problem lives in the distributed
// shared memory of a cluster of CL_MAX CTAs.  Triangle t sits in CTA
// t >> shift at slot t & mask (a power-of-two slice); a record is 48 bytes
// (3 vertex indices, 3 packed coordinates, 3 links, two locks, flip round), so a
// cluster of 16 CTAs holds up to 65536 triangles.  Every access to another
// CTA's triangle is a distributed-shared-memory load, store or atomic; the
// phases are separated by cluster barriers.
constexpr int CL_THREADS = 1024;
constexpr int SLICE_MAX_LOG2 = 12;                 // 4096 triangles per CTA
constexpr int SLICE_MAX = 1 << SLICE_MAX_LOG2;
constexpr int WL_PER_CTA = 6 * SLICE_MAX;           // worklist entries per CTA and round
constexpr int CAND_PER_CTA = 6 * SLICE_MAX;         // proposals per CTA and round
constexpr int FLIP_PER_CTA = SLICE_MAX;             // flipped pairs per CTA and round
constexpr int CL_MARK = 3 * SLICE_MAX / 32;         // words of a per-round half-edge bitset
// shared memory: the triangle slice (48 bytes a triangle), two push bitsets
// and the round-0 staging rings (64 entries per warp)
constexpr size_t CL_SMEM = size_t(SLICE_MAX) * 48 + size_t(8) * CL_MARK + size_t(4) * 64 * (CL_THREADS / 32);

struct ClusterTri {
    int32_t* lv;      // [3*SLICE_MAX] in this CTA's shared memory
    uint32_t* lxy;    // [3*SLICE_MAX]
    int32_t* lopp;    // [3*SLICE_MAX]
    uint32_t* llock;  // [SLICE_MAX]
    int32_t* lround;  // [SLICE_MAX]
    int shift, mask;
    template <class X>
    __device__ __forceinline__ X* at(X* base, int t) const {
        return cg::this_cluster().map_shared_rank(base, unsigned(t >> shift));
    }
    __device__ int v(int t, int k) const { return at(lv, t)[3 * (t & mask) + k]; }
    __device__ uint32_t xy(int t, int k) const { return at(lxy, t)[3 * (t & mask) + k]; }
    __device__ int opp(int h) const { int t = h / 3; return at(lopp, t)[3 * (t & mask) + h - 3 * t]; }
    __device__ uint32_t lock(int t) const { return *((volatile uint32_t*)at(llock, t) + (t & mask)); }
    __device__ int32_t fround(int t) const { return at(lround, t)[t & mask]; }
    __device__ void lock_min(int t, uint32_t p) { atomicMin(at(llock, t) + (t & mask), p); }
    __device__ void set_v(int t, int a, int b, int c, uint32_t pa, uint32_t pb, uint32_t pc) {
        int32_t* V = at(lv, t) + 3 * (t & mask);
        uint32_t* X = at(lxy, t) + 3 * (t & mask);
        V[0] = a; V[1] = b; V[2] = c;
        X[0] = pa; X[1] = pb; X[2] = pc;
    }
    __device__ void set_opp(int h, int o) { int t = h / 3; at(lopp, t)[3 * (t & mask) + h - 3 * t] = o; }
    __device__ void set_fround(int t, int32_t r) { at(lround, t)[t & mask] = r; }
};

// Point-table accessor for a problem that fits one SM: corner coordinates
// are looked up per vertex (4 bytes per support point instead of 12 per
// triangle), which leaves shared memory for the round lists.
struct PtTri {
    int32_t* lv;
    const uint32_t* pxy;
    int32_t* lopp;
    uint32_t* llock;
    int32_t* lround;
    __device__ int v(int t, int k) const { return lv[3 * t + k]; }
    __device__ uint32_t xy(int t, int k) const { return pxy[lv[3 * t + k]]; }
    __device__ int opp(int h) const { return lopp[h]; }
    __device__ uint32_t lock(int t) const { return *((volatile uint32_t*)llock + t); }
    __device__ int32_t fround(int t) const { return lround[t]; }
    __device__ void lock_min(int t, uint32_t p) { atomicMin(llock + t, p); }
    __device__ void set_v(int t, int a, int b, int c, uint32_t, uint32_t, uint32_t) {
        lv[3 * t] = a; lv[3 * t + 1] = b; lv[3 * t + 2] = c;
    }
    __device__ void set_opp(int h, int o) { lopp[h] = o; }
    __device__ void set_fround(int t, int32_t r) { lround[t] = r; }
};

// A round list whose first entries live in shared memory and the rest in
// global memory (records of `width` ints).
struct List2 {
    int32_t* s;
    int32_t* g;
    int scap, gcap, width;
    __device__ int32_t* slot(int i) const { return i < scap ? s + width * i : g + width * (i - scap); }
    __device__ int cap() const { return scap + gcap; }
};

constexpr int LOC_T = 4096;        // triangles of a one-SM problem
constexpr int LOC_PTS = 4096;      // support points (vertex ids) of a one-SM problem
constexpr int LOC_CAND = 1536;     // proposals of a round in shared memory (two round lists)
constexpr int LOC_FLIP = 1280;     // flipped pairs in shared memory
constexpr int LOC_MARK = (3 * LOC_T + 31) / 32;   // words of a per-round half-edge bitset
constexpr int FLIP_TAIL = 64;      // rounds with at most this many proposals run on one warp
constexpr size_t LOC_SMEM = size_t(36) * LOC_T + size_t(4) * LOC_PTS + size_t(16) * LOC_CAND +
                            size_t(24) * LOC_FLIP + size_t(8) * LOC_MARK;
// round 0 stages each warp's owned half-edges (64 entries) in the flip list's
// shared part, which is unused until the first flips
static_assert(6 * LOC_FLIP >= 64 * (1024 / 32), "round-0 staging does not fit");

// Flip rounds of one problem in one CTA: triangles, points and the round
// lists in shared memory.  Problems with more triangles or points are left
// (ctr[8] stays 0) to the cluster kernel.
//
// A round is three phases between barriers:
//   B   flip the proposals that won both locks; release the locks of the
//       round before; clear the next round's edge bitset;
//   C1  resolve the outer neighbours of every flipped pair (read only) and
//       propose, for the next round, each outer edge that is not locally
//       Delaunay (vertices are final once B is over, so the test needs no
//       links);
//   C2  write the links; re-propose the proposals that lost a lock while
//       neither of their triangles flipped (their test result is unchanged).
// Proposals of consecutive rounds use two lock arrays, so the next round's
// locks fill while this round's are still held.  The rounds, proposals and
// flips are those of the propose / flip / resolve / relink formulation with
// a worklist (the host emulation): only the tests move forward a phase.
__global__ void __launch_bounds__(1024) k_flip_local(DelDev d0, DelDev d1, int max_rounds, unsigned* err) {
    grid_dep_wait();
    extern __shared__ __align__(16) uint8_t lsm[];
    __shared__ int n_cand[2], n_flip;
    const DelDev& D = blockIdx.x ? d1 : d0;
    const int T = D.ctr[0], NP = D.ctr[9];
    if (D.ctr[8] != 0 || T > LOC_T || NP > LOC_PTS) return;
    const int tid = threadIdx.x, NT = blockDim.x;
    PtTri m;
    m.lv = reinterpret_cast<int32_t*>(lsm);
    m.lopp = m.lv + 3 * LOC_T;
    uint32_t* const lock0 = reinterpret_cast<uint32_t*>(m.lopp + 3 * LOC_T);
    uint32_t* const lock1 = lock0 + LOC_T;
    m.lround = reinterpret_cast<int32_t*>(lock1 + LOC_T);
    uint32_t* pxy = reinterpret_cast<uint32_t*>(m.lround + LOC_T);
    m.pxy = pxy;
    int32_t* sw = reinterpret_cast<int32_t*>(pxy + LOC_PTS);
    const List2 cand0{sw, D.ccand, LOC_CAND, CAND_PER_CTA, 2};
    const List2 cand1{sw + 2 * LOC_CAND, D.ccand + 2 * CAND_PER_CTA, LOC_CAND, CAND_PER_CTA, 2};
    const List2 flips{sw + 4 * LOC_CAND, D.cflips, LOC_FLIP, FLIP_PER_CTA, 6};
    uint32_t* const mark0 = reinterpret_cast<uint32_t*>(sw + 4 * LOC_CAND + 6 * LOC_FLIP);
    uint32_t* const mark1 = mark0 + LOC_MARK;
    for (int i = tid; i < NP; i += NT) pxy[i] = pack_xy(D.x[i], D.y[i]);
    for (int t = tid; t < T; t += NT) {
        for (int k = 0; k < 3; ++k) {
            m.lv[3 * t + k] = D.tri[3 * t + k];
            m.lopp[3 * t + k] = D.opp[3 * t + k];
        }
        lock0[t] = LOCK_FREE;
        lock1[t] = LOCK_FREE;
        m.lround[t] = -1;
    }
    if (tid == 0) { n_cand[0] = 0; n_cand[1] = 0; n_flip = 0; }
    __syncthreads();
    // round 0's proposals: every interior edge once
    m.llock = lock0;
    {
        auto add0 = [&](int hh, int nn) {
            int idx = agg_inc(&n_cand[0]);
            if (idx < cand0.cap()) { int32_t* c = cand0.slot(idx); c[0] = hh; c[1] = nn; }
        };
        propose_owned(0, 3 * T, flips.s + 64 * (tid >> 5), [&](int h) { return m.lopp[h]; }, [&](int h) {
            if (!flip_propose(m, h, T, 0u, false, add0)) set_err(err, ERRF_BOUNDS);
        });
    }
    __syncthreads();
    int round = 0, flips_total = 0, nc_prev = 0;
    bool converged = false;
    // One round with threads [0, nt) of the CTA (index `me`), `sync` the
    // barrier among them.  Returns 0 to continue, 1 when converged, 2 on
    // an overflow.
    auto flip_round = [&](const int me, const int nt, auto&& sync) -> int {
        const int cur = round & 1, nxt = cur ^ 1;
        // selected by value: a dynamically indexed pair would live in local memory
        const List2 cand_cur = cur ? cand1 : cand0, cand_nxt = cur ? cand0 : cand1;
        uint32_t* const lock_cur = cur ? lock1 : lock0;
        uint32_t* const lock_nxt = cur ? lock0 : lock1;
        uint32_t* const mark_nxt = cur ? mark0 : mark1;
        const int nc = n_cand[cur];             // final since the last barrier; equal in every thread
        if (nc == 0) { converged = true; return 1; }
        if (nc > cand_cur.cap()) {
            if (me == 0) set_err(err, ERRF_BOUNDS);
            return 2;
        }
        // B: flip the winners; release the previous round's locks; clear the next round's bitset
        m.llock = lock_cur;
        for (int c = me; c < nc; c += nt) {
            const int32_t* cc = cand_cur.slot(c);
            int h = cc[0], n = cc[1];
            if (flip_apply(m, h, n, uint32_t(round))) {
                int f = agg_inc(&n_flip);     // at most T/2 <= flips.cap()
                int32_t* q = flips.slot(f);
                q[0] = h / 3; q[1] = n;
            }
        }
        for (int c = me; c < nc_prev; c += nt) {
            const int32_t* cc = cand_nxt.slot(c);
            lock_nxt[cc[0] / 3] = LOCK_FREE;
            lock_nxt[cc[1]] = LOCK_FREE;
        }
        for (int i = me; i < LOC_MARK; i += nt) mark_nxt[i] = 0u;
        sync();
        const int nf = n_flip;
        auto add_next = [&](int hh, int nn, uint32_t p) {
            atomicMin(lock_nxt + hh / 3, p);
            atomicMin(lock_nxt + nn, p);
            int idx = agg_inc(&n_cand[nxt]);
            if (idx < cand_nxt.cap()) { int32_t* c = cand_nxt.slot(idx); c[0] = hh; c[1] = nn; }
        };
        // C1: resolve the outer neighbours (read only); propose the outer edges.
        // The four edges of a pair go through each step together (claims,
        // tests, one list reservation per warp), so their latencies overlap.
        for (int f = me; f < nf; f += nt) {
            int32_t* q = flips.slot(f);
            const int t = q[0], n = q[1];
            int r[4], c[4], tw[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                r[k] = flip_resolve_slot(m, outer_slot(t, n, k), uint32_t(round), T);
                if (r[k] == -2) { set_err(err, ERRF_BOUNDS); r[k] = -1; }
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) q[2 + k] = r[k];
            uint32_t old[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int x = outer_slot(t, n, k);
                // a hull edge (r < 0) tests against its own triangle, is never claimed, and is masked out
                c[k] = r[k] >= 0 ? min(x, r[k]) : x;
                tw[k] = r[k] >= 0 ? (c[k] == x ? r[k] : x) : x;
                old[k] = r[k] >= 0 ? atomicOr(mark_nxt + (c[k] >> 5), 1u << (c[k] & 31)) : ~0u;
            }
            // the four tests are independent (no branch between them), so their loads overlap
            bool flippable[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) flippable[k] = edge_flippable(m, c[k], tw[k]);
            unsigned want = 0;
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (!(old[k] & (1u << (c[k] & 31))) && flippable[k]) want |= 1u << k;
            // reserve popc(want) entries per lane with one atomic per warp
            const unsigned act = __activemask();
            const int lane = tid & 31, cnt = __popc(want);
            const unsigned b0 = __ballot_sync(act, cnt & 1), b1 = __ballot_sync(act, cnt & 2),
                           b2 = __ballot_sync(act, cnt & 4);
            const unsigned lt = (1u << lane) - 1u;
            const int before = __popc(b0 & lt) + 2 * __popc(b1 & lt) + 4 * __popc(b2 & lt);
            const int total = __popc(b0) + 2 * __popc(b1) + 4 * __popc(b2);
            const int leader = __ffs(act) - 1;
            int base = 0;
            if (lane == leader && total > 0) base = atomicAdd(&n_cand[nxt], total);
            base = __shfl_sync(act, base, leader) + before;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                if (!(want & (1u << k))) continue;
                const uint32_t p = prio(uint32_t(c[k]), uint32_t(round + 1));
                atomicMin(lock_nxt + c[k] / 3, p);
                atomicMin(lock_nxt + tw[k] / 3, p);
                if (base < cand_nxt.cap()) { int32_t* e = cand_nxt.slot(base); e[0] = c[k]; e[1] = tw[k] / 3; }
                ++base;
            }
        }
        sync();
        // C2: relink; re-propose the lost proposals (their edges are no outer
        // edge of a flipped pair, so the bitset need not see them)
        if (me == 0) { n_flip = 0; n_cand[cur] = 0; }   // both were read before the last barrier
        for (int f = me; f < nf; f += nt) {
            int32_t* q = flips.slot(f);
            flip_relink(m, q[0], q[1], q + 2);
        }
        for (int c = me; c < nc; c += nt) {
            const int32_t* cc = cand_cur.slot(c);
            const int h = cc[0], n = cc[1], t = h / 3;
            if (m.fround(t) != round && m.fround(n) != round) add_next(h, n, prio(uint32_t(h), uint32_t(round + 1)));
        }
        flips_total += nf;
        nc_prev = nc;
        sync();
        return 0;
    };
    // The whole CTA runs the rounds while they are large; once a round
    // starts with at most FLIP_TAIL proposals, warp 0 runs every remaining
    // round alone with warp barriers (the same rounds: the phases only lose
    // the cost of block-wide barriers), and the other warps wait at the end.
    int state = 0;
    for (; round < max_rounds; ++round) {
        const int nc_top = n_cand[round & 1];   // uniform: read after a block barrier
        if (nc_top > 0 && nc_top <= FLIP_TAIL) break;
        state = flip_round(tid, NT, [] { __syncthreads(); });
        if (state) break;
    }
    if (state == 0 && round < max_rounds && tid < 32) {
        for (; round < max_rounds; ++round) {
            state = flip_round(tid, 32, [] { __syncwarp(); });
            if (state) break;
        }
    }
    __syncthreads();
    for (int t = tid; t < T; t += NT) {
        int32_t v[3] = {m.lv[3 * t], m.lv[3 * t + 1], m.lv[3 * t + 2]};
        normalise(v);
        for (int k = 0; k < 3; ++k) D.tri[3 * t + k] = v[k];
    }
    if (tid == 0) {
        D.ctr[8] = 1;
        D.ctr[4] = round + 1;
        D.ctr[5] = flips_total;
        if (!converged) set_err(err, ERRF_FLIP_LIMIT);
    }
}

struct ClusterSync {
    __device__ void operator()() const { cg::this_cluster().sync(); }
    template <class X>
    __device__ X* remote(X* p, int r) const { return cg::this_cluster().map_shared_rank(p, unsigned(r)); }
    __device__ int rank() const { return int(cg::this_cluster().block_rank()); }
};

// Flip rounds in distributed shared memory: a cluster of csize CTAs, each
// holding a slice of at most SLICE_MAX triangles.  A problem already handled
// (ctr[8] set by the one-SM kernel) or larger than csize * SLICE_MAX is
// skipped; the kernel that handles a problem sets ctr[8].
//
// The rounds are those of k_flip_local (three phases between cluster
// barriers: B flip, C1 resolve + propose the outer edges, C2 relink +
// re-propose the lost proposals; two lock arrays by round parity).  A
// proposal is queued at the CTA that owns its lower half-edge, so a CTA
// flips at most its own triangles in a round (f < FLIP_PER_CTA), and that
// CTA releases the proposal's locks in the next round.
__global__ void __launch_bounds__(CL_THREADS) k_flip_smem(DelDev d0, DelDev d1, int csize, int max_rounds,
                                                          unsigned* err) {
    grid_dep_wait();
    using Sync = ClusterSync;
    extern __shared__ __align__(16) uint8_t csm[];
    __shared__ int n_cand[2], n_flip, s_flips;
    Sync sync;
    const int rank = sync.rank();
    const int prob = blockIdx.x / csize;
    const DelDev& D = prob ? d1 : d0;
    const int T = D.ctr[0];
    // uniform over the CTAs of a problem: no barrier has been passed yet
    if (D.ctr[8] != 0 || T > csize * SLICE_MAX) return;
    int shift = 6;
    while ((csize << shift) < T) ++shift;
    ClusterTri m;
    m.lv = reinterpret_cast<int32_t*>(csm);
    m.lxy = reinterpret_cast<uint32_t*>(m.lv + 3 * SLICE_MAX);
    m.lopp = reinterpret_cast<int32_t*>(m.lxy + 3 * SLICE_MAX);
    uint32_t* const lock0 = reinterpret_cast<uint32_t*>(m.lopp + 3 * SLICE_MAX);
    uint32_t* const lock1 = lock0 + SLICE_MAX;
    m.lround = reinterpret_cast<int32_t*>(lock1 + SLICE_MAX);
    uint32_t* const mark0 = reinterpret_cast<uint32_t*>(m.lround + SLICE_MAX);
    uint32_t* const mark1 = mark0 + CL_MARK;
    int32_t* const ring = reinterpret_cast<int32_t*>(mark1 + CL_MARK);
    m.shift = shift;
    m.mask = (1 << shift) - 1;
    const int t0 = rank << shift, t1 = min(T, (rank + 1) << shift);
    const int tid = threadIdx.x;
    for (int t = t0 + tid; t < t1; t += CL_THREADS) {
        int l = t - t0;
        for (int k = 0; k < 3; ++k) {
            int v = D.tri[3 * t + k];
            m.lv[3 * l + k] = v;
            m.lxy[3 * l + k] = pack_xy(D.x[v], D.y[v]);
            m.lopp[3 * l + k] = D.opp[3 * t + k];
        }
        lock0[l] = LOCK_FREE;
        lock1[l] = LOCK_FREE;
        m.lround[l] = -1;
    }
    if (tid == 0) { n_cand[0] = 0; n_cand[1] = 0; n_flip = 0; }
    // the proposal lists of CTA r, by round parity, in global memory
    auto cand_list = [&](int parity, int r) -> int32_t* {
        return parity ? D.cwl + size_t(r) * 2 * WL_PER_CTA : D.ccand + size_t(r) * 2 * CAND_PER_CTA;
    };
    int32_t* const flips = D.cflips + size_t(rank) * 6 * FLIP_PER_CTA;
    sync();
    // round 0's proposals: every interior edge of the own slice once
    m.llock = lock0;
    {
        int32_t* const c0 = cand_list(0, rank);
        auto add0 = [&](int hh, int nn) {
            int idx = agg_inc(&n_cand[0]);
            if (idx < CAND_PER_CTA) { c0[2 * idx] = hh; c0[2 * idx + 1] = nn; }
        };
        propose_owned(3 * t0, 3 * t1, ring + 64 * (tid >> 5), [&](int h) { return m.opp(h); }, [&](int h) {
            if (!flip_propose(m, h, T, 0u, false, add0)) set_err(err, ERRF_BOUNDS);
        });
    }
    sync();
    int round = 0, flips_total = 0, nc_prev = 0;
    bool converged = false;
    for (; round < max_rounds; ++round) {
        const int cur = round & 1, nxt = cur ^ 1;
        int32_t* const cand_cur = cand_list(cur, rank);
        int32_t* const cand_old = cand_list(nxt, rank);   // the previous round's list, until C1 refills it
        uint32_t* const lock_cur = cur ? lock1 : lock0;
        uint32_t* const lock_nxt = cur ? lock0 : lock1;
        uint32_t* const mark_nxt = cur ? mark0 : mark1;
        // every CTA's count is final since the last barrier, so all CTAs take the same decision
        int total = 0;
        bool over = false;
        for (int r = 0; r < csize; ++r) {
            const int c = *sync.remote(&n_cand[cur], r);
            total += c;
            over |= c > CAND_PER_CTA;
        }
        if (over) {
            if (tid == 0) set_err(err, ERRF_BOUNDS);
            break;
        }
        if (total == 0) { converged = true; break; }
        const int nc = n_cand[cur];
        // B: flip the winners (own triangles); release the previous round's locks; clear the next bitset
        m.llock = lock_cur;
        for (int c = tid; c < nc; c += CL_THREADS) {
            int h = cand_cur[2 * c], n = cand_cur[2 * c + 1];
            if (flip_apply(m, h, n, uint32_t(round))) {
                int f = agg_inc(&n_flip);
                if (f < FLIP_PER_CTA) { flips[6 * f] = h / 3; flips[6 * f + 1] = n; }
            }
        }
        for (int c = tid; c < nc_prev; c += CL_THREADS) {
            const int t = cand_old[2 * c] / 3, n = cand_old[2 * c + 1];
            *(m.at(lock_nxt, t) + (t & m.mask)) = LOCK_FREE;
            *(m.at(lock_nxt, n) + (n & m.mask)) = LOCK_FREE;
        }
        for (int i = tid; i < CL_MARK; i += CL_THREADS) mark_nxt[i] = 0u;
        sync();
        const int nf = min(n_flip, FLIP_PER_CTA);
        // a proposal for the next round, queued at the CTA owning its lower half-edge h
        auto add_next = [&](int h, int n, uint32_t p) {
            atomicMin(m.at(lock_nxt, h / 3) + ((h / 3) & m.mask), p);
            atomicMin(m.at(lock_nxt, n) + (n & m.mask), p);
            const int owner = (h / 3) >> shift;
            int idx = agg_inc_keyed(sync.remote(&n_cand[nxt], owner));
            if (idx < CAND_PER_CTA) {
                int32_t* e = cand_list(nxt, owner) + 2 * idx;
                e[0] = h;
                e[1] = n;
            }
        };
        // C1: resolve the outer neighbours (read only); propose the outer edges
        for (int f = tid; f < nf; f += CL_THREADS) {
            int32_t* q = flips + 6 * f;
            const int t = q[0], n = q[1];
            int r[4], c[4], tw[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                r[k] = flip_resolve_slot(m, outer_slot(t, n, k), uint32_t(round), T);
                if (r[k] == -2) { set_err(err, ERRF_BOUNDS); r[k] = -1; }
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) q[2 + k] = r[k];
            unsigned claimed = 0;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int x = outer_slot(t, n, k);
                // a hull edge (r < 0) tests against its own triangle, is never claimed, and is masked out
                c[k] = r[k] >= 0 ? min(x, r[k]) : x;
                tw[k] = r[k] >= 0 ? (c[k] == x ? r[k] : x) : x;
                // the edge's bit lives at the CTA that owns its lower half-edge
                const int owner = (c[k] / 3) >> shift;
                const int lb = c[k] - 3 * (owner << shift);
                const uint32_t bit = 1u << (lb & 31);
                if (r[k] >= 0 && !(atomicOr(sync.remote(mark_nxt, owner) + (lb >> 5), bit) & bit)) claimed |= 1u << k;
            }
            unsigned flippable = 0;
#pragma unroll
            for (int k = 0; k < 4; ++k) flippable |= edge_flippable(m, c[k], tw[k]) ? 1u << k : 0u;
            const unsigned want = claimed & flippable;
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (want & (1u << k)) add_next(c[k], tw[k] / 3, prio(uint32_t(c[k]), uint32_t(round + 1)));
        }
        sync();
        // C2: relink; re-propose the own proposals that lost (no outer edge of a flipped pair)
        if (tid == 0) { n_flip = 0; n_cand[cur] = 0; }   // both were read before the last barrier
        for (int f = tid; f < nf; f += CL_THREADS) flip_relink(m, flips[6 * f], flips[6 * f + 1], flips + 6 * f + 2);
        for (int c = tid; c < nc; c += CL_THREADS) {
            const int h = cand_cur[2 * c], n = cand_cur[2 * c + 1], t = h / 3;
            if (m.fround(t) != round && m.fround(n) != round) add_next(h, n, prio(uint32_t(h), uint32_t(round + 1)));
        }
        flips_total += nf;
        nc_prev = nc;
        sync();
    }
    // write back this CTA's slice
    for (int t = t0 + tid; t < t1; t += CL_THREADS) {
        const int l = t - t0;
        int32_t v[3] = {m.lv[3 * l], m.lv[3 * l + 1], m.lv[3 * l + 2]};
        normalise(v);
        for (int k = 0; k < 3; ++k) D.tri[3 * t + k] = v[k];
    }
    if (tid == 0) s_flips = flips_total;
    sync();
    if (rank == 0 && tid == 0) {
        int total = 0;
        for (int r = 0; r < csize; ++r) total += *sync.remote(&s_flips, r);
        D.ctr[8] = 1;
        D.ctr[4] = round + 1;
        D.ctr[5] = total;
        if (!converged) set_err(err, ERRF_FLIP_LIMIT);
    }
    sync();   // keep every CTA's shared memory alive until remote readers are done
}

}  // namespace

int cluster_size_for_flip() {
    int sizes[2] = {16, 8};
    size_t smem = CL_SMEM;
    allow_smem(k_flip_smem);
    cudaFuncSetAttribute(k_flip_smem, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    for (int cs : sizes) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(2 * cs);
        cfg.blockDim = dim3(CL_THREADS);
        cfg.dynamicSmemBytes = smem;
        cudaLaunchAttribute attr;
        attr.id = cudaLaunchAttributeClusterDimension;
        attr.val.clusterDim.x = cs;
        attr.val.clusterDim.y = 1;
        attr.val.clusterDim.z = 1;
        cfg.attrs = &attr;
        cfg.numAttrs = 1;
        int n = 0;
        if (cudaOccupancyMaxActiveClusters(&n, k_flip_smem, &cfg) == cudaSuccess && n >= 2) return cs;
        cudaGetLastError();
    }
    return 0;
}

cudaError_t launch_delaunay(DelDev& d0, DelDev& d1, const int32_t* row_off, int nrows, int nmax, int H, int num_sms,
                            int csize, unsigned* err, cudaStream_t st, int* nlaunch, bool flips,
                            bool force_global, int round_limit) {
    launch_k(k_rowsort, dim3(nrows, 2), 512, 0, st, d0, d1, row_off, nrows, err);
    const size_t plan_smem = size_t(32) * nrows;
    allow_smem(k_plan);
    launch_k(k_plan, 2, 1024, plan_smem, st, d0, d1, row_off, nrows, H, flips ? 1 : 0, err);
    if (!flips) {
        launch_k(k_star, dim3(2, imax(1, imin((nmax + STAR_WARPS - 1) / STAR_WARPS, 6 * num_sms))), STAR_WARPS * 32,
                 0, st, d0, d1, row_off, err);
        launch_k(k_star_emit, dim3(imax(1, (nmax + EMIT_THREADS - 1) / EMIT_THREADS), 2), EMIT_THREADS, 0, st, d0, d1,
                 err);
        if (nlaunch) *nlaunch += 4;
        return cudaGetLastError();
    }
    // the pocket walk's chain and stack (2 sides x (index, x, y, 4-int stack
    // records) = 56 bytes a row) in shared memory up to 32 KiB; every block
    // of k_strips carries it
    const int smem_rows = imin(nrows, (32 * 1024) / 56);
    const size_t smem = size_t(smem_rows) * 56;
    int blocks = 4 * num_sms;
    launch_k(k_strips, dim3(imax(1, imin(blocks, (nmax + 255) / 256)) + 1, 2), 256, smem, st, d0, d1, row_off,
             nrows, nmax, smem_rows);
    launch_k(k_hash_clear, dim3(blocks, 2), 256, 0, st, d0, d1);
    launch_k(k_hash_insert, dim3(blocks, 2), 256, 0, st, d0, d1, err);
    launch_k(k_link, dim3(blocks, 2), 256, 0, st, d0, d1, err);
    int launched = 6;
    const int max_rounds = round_limit > 0 ? round_limit : 100000;
    if (!force_global) {
        allow_smem(k_flip_local);
        launch_k(k_flip_local, 2, 1024, LOC_SMEM, st, d0, d1, max_rounds, err);
        ++launched;
    }
    if (csize > 0 && !force_global) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(2 * csize);
        cfg.blockDim = dim3(CL_THREADS);
        cfg.dynamicSmemBytes = CL_SMEM;
        cfg.stream = st;
        cudaLaunchAttribute attr;
        attr.id = cudaLaunchAttributeClusterDimension;
        attr.val.clusterDim.x = csize;
        attr.val.clusterDim.y = 1;
        attr.val.clusterDim.z = 1;
        cfg.attrs = &attr;
        cfg.numAttrs = 1;
        cudaError_t e = cudaLaunchKernelEx(&cfg, k_flip_smem, d0, d1, csize, max_rounds, err);
        if (e != cudaSuccess) return e;
        ++launched;
    }
    // The fallback, for triangulations larger than a cluster holds; not
    // launched when none can be (at most 2 * nmax + 16 triangles).  It packs
    // the corner coordinates itself; every flip kernel writes its triangles
    // rotated to start at their smallest vertex index.
    if (force_global || csize == 0 || 2LL * nmax + 16 > (long long)csize * SLICE_MAX) {
        launch_k(k_flip_global, 2, FLIP_THREADS, 0, st, d0, d1, max_rounds, err);
        ++launched;
    }
    if (nlaunch) *nlaunch += launched;
    return cudaGetLastError();
}

}  // namespace elas
