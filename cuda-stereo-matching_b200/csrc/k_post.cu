// Post-filters: speckle removal, gap interpolation, adaptive mean, median.
//
// The reference declares these only as parameters (src/Elas.h:31-36,
// KernelsCommon.h:19-21) and its process() stops after the left/right check
// (src/Elas.cu:107-119).  The semantics are the project's own and are
// written out in the CPU oracle (oracle/elas_oracle.cpp, orc_postprocess):
//   speckle   4-connected segments (|d_p - d_q| <= speckle_sim_threshold);
//             segments smaller than speckle_size become invalid.  Union-find
//             with atomic hooking of the larger root under the smaller.
//   gap       rows, then columns: a run of <= ipol_gap_width invalid pixels
//             between valid a and b becomes (a+b)/2 if |a-b| <= 3 else
//             min(a,b).  Widths up to 8 run inside the fused tile kernel,
//             wider gaps as one thread per line.
//   mean      5x5 weighted mean of valid pixels, w = 1/(1+(d_q-d_p)^2).
//   median    lower median of the valid pixels of the 3x3 window.
#include <cuda_runtime.h>
#include <mutex>
#include "../../include/elas_b200.h"
#include "common.cuh"
#include "launch.cuh"
#include "kernels.h"

namespace elas {

namespace {

constexpr int UF_LIMIT = 1 << 22;   // bound on any union-find walk / retry loop

// Root of x with path halving (labels only ever move to a smaller index, so
// concurrent halving keeps every node in its tree).
__device__ __forceinline__ int uf_find(int32_t* lab, int x, unsigned* err) {
    for (int it = 0; it < UF_LIMIT; ++it) {
        int p = lab[x];
        if (p == x) return x;
        int gp = lab[p];
        if (gp != p) lab[x] = gp;
        x = p;
    }
    atomicOr(err, ERRF_BOUNDS);
    return x;
}

// Labels start at the left neighbour when it is connected (the most common
// union), else at the pixel itself.  One thread per pixel on a 1-D grid (a
// map of any height fits).
__global__ void k_uf_init(const float* __restrict__ D, int32_t* __restrict__ lab, int32_t* __restrict__ sz, int W,
                          int H, float thr) {
    grid_dep_wait();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= W * H) return;
    const int u = i % W;
    float d = D[i];
    int l = -1;
    if (d >= 0) {
        l = i;
        if (u > 0) {
            float q = D[i - 1];
            if (q >= 0 && fabsf(q - d) <= thr) l = i - 1;
        }
    }
    lab[i] = l;
    sz[i] = 0;
}

__device__ void uf_union(int32_t* lab, int a, int b, unsigned* err) {
    for (int it = 0; it < UF_LIMIT; ++it) {
        int ra = uf_find(lab, a, err), rb = uf_find(lab, b, err);
        if (ra == rb) return;
        if (ra < rb) {   // keep (a, ra) and (b, rb) paired: hook the larger root
            int t = ra; ra = rb; rb = t;
            t = a; a = b; b = t;
        }
        int old = atomicCAS(&lab[ra], ra, rb);
        if (old == ra) return;
        a = old;         // ra gained a parent meanwhile: continue from it
    }
    atomicOr(err, ERRF_BOUNDS);
}

__global__ void k_uf_union(const float* __restrict__ D, int32_t* lab, int W, int H, float thr, unsigned* err) {
    grid_dep_wait();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= W * H) return;
    const int u = i % W, v = i / W;
    float d = D[i];
    if (d < 0) return;
    if (u + 1 < W) {
        float q = D[i + 1];
        if (q >= 0 && fabsf(q - d) <= thr) uf_union(lab, i, i + 1, err);
    }
    if (v + 1 < H) {
        float q = D[i + W];
        if (q >= 0 && fabsf(q - d) <= thr) uf_union(lab, i, i + W, err);
    }
}

// Root of every pixel into `root` (written only by its own thread: `lab`
// itself may still receive path-halving writes from other threads) and
// segment sizes; lanes of a warp that share a root add once (segments are
// large, so this removes most of the contention on the root counters).
__global__ void k_uf_count(int32_t* lab, int32_t* __restrict__ root, int32_t* sz, int n, unsigned* err) {
    grid_dep_wait();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int r = -1;
    if (i < n && lab[i] >= 0) r = uf_find(lab, i, err);
    if (i < n) root[i] = r;
    unsigned peers = __match_any_sync(0xffffffffu, r);
    int leader = __ffs(peers) - 1;
    if (r >= 0 && (threadIdx.x & 31) == leader) atomicAdd(&sz[r], __popc(peers));
}

// ---------------------------------------------------------------------------
// Speckle segmentation in tiles.  The segments (4-connected valid pixels,
// |d_p - d_q| <= thr) are labelled first inside every 32x32 tile with a
// union-find in shared memory; only links across tile borders then go
// through the global union-find, and sizes are counted once per tile-local
// component.  The segments, hence the result, are those of a whole-image
// union-find.
//   lab[i]  the global index of i's tile-local root (-1 invalid); the local
//           roots are the nodes of the global forest (a local root's entry is
//           its parent there, itself until the border pass hooks it)
//   sz[r]   at a local root r only: the pixel count of its tile component;
//           after the count, -(global root + 1)
//   acc[g]  the segment size at global root g (zeroed at every local root by
//           the tile kernel; global roots are local roots)
//   roots   [0] the number of local roots, then their global indices
// Only lab is written per pixel.  A pixel j's segment size is then
// acc[-sz[lab[j]] - 1]: lab[j] is j's local root or, for a local root that
// was hooked, another local root of the same segment.
constexpr int SPK_T = 32;

__device__ __forceinline__ int lfind(int* L, int x) {
    for (int it = 0; it < SPK_T * SPK_T; ++it) {
        const int p = L[x];
        if (p == x) return x;
        const int gp = L[p];
        if (gp != p) L[x] = gp;
        x = p;
    }
    return x;
}
__device__ __forceinline__ void lunion(int* L, int a, int b) {
    for (int it = 0; it < SPK_T * SPK_T; ++it) {
        int ra = lfind(L, a), rb = lfind(L, b);
        if (ra == rb) return;
        if (ra < rb) { int t = ra; ra = rb; rb = t; t = a; a = b; b = t; }
        const int old = atomicCAS(&L[ra], ra, rb);
        if (old == ra) return;
        a = old;
    }
}

// A CTA of 32 x 8 threads per 32x32 tile, each thread taking the tile rows
// ty, ty + 8, ty + 16, ty + 24 (a warp holds one tile row at a time, for
// the run ballots): eight such CTAs fit on an SM where a tile per
// 1024-thread CTA fitted two, so the waits at the tile's barriers overlap
// with other tiles' work.
constexpr int SPK_ROWS = 8;
constexpr int SPK_RPT = SPK_T / SPK_ROWS;
__global__ void __launch_bounds__(SPK_T * SPK_ROWS) k_spk_tile(PostViews pv, int W, int H, float thr) {
    grid_dep_wait();
    __shared__ float S[SPK_T][SPK_T];
    __shared__ int L[SPK_T * SPK_T];
    __shared__ int C[SPK_T * SPK_T];
    __shared__ int n_roots, base;
    const int view = blockIdx.z;
    const float* __restrict__ D = pv.cur[view];
    const int tx = threadIdx.x, tid = threadIdx.y * SPK_T + tx;
    const int x = blockIdx.x * SPK_T + tx;
    float d[SPK_RPT], dl[SPK_RPT];
    bool conn_l[SPK_RPT];
#pragma unroll
    for (int j = 0; j < SPK_RPT; ++j) {
        const int ty = threadIdx.y + SPK_ROWS * j, t = ty * SPK_T + tx, y = blockIdx.y * SPK_T + ty;
        const bool in = x < W && y < H;
        d[j] = in ? D[size_t(y) * W + x] : -1.0f;
        const bool valid = d[j] >= 0;
        S[ty][tx] = d[j];
        C[t] = 0;
        // runs of the row: every pixel points at the first pixel of its run
        dl[j] = __shfl_up_sync(0xffffffffu, d[j], 1);
        conn_l[j] = valid && tx > 0 && dl[j] >= 0 && fabsf(d[j] - dl[j]) <= thr;
        const unsigned starts = __ballot_sync(0xffffffffu, valid && !conn_l[j]);
        const unsigned mine = starts & (0xffffffffu >> (31 - tx));
        L[t] = valid ? ty * SPK_T + (31 - __clz(mine)) : t;
    }
    if (tid == 0) n_roots = 0;
    __syncthreads();
    // vertical links; a link is implied when the left neighbours make the same one
#pragma unroll
    for (int j = 0; j < SPK_RPT; ++j) {
        const int ty = threadIdx.y + SPK_ROWS * j, t = ty * SPK_T + tx;
        if (d[j] >= 0 && ty + 1 < SPK_T) {
            const float q = S[ty + 1][tx];
            if (q >= 0 && fabsf(q - d[j]) <= thr) {
                bool implied = false;
                if (tx > 0) {
                    const float ql = S[ty + 1][tx - 1];
                    implied = conn_l[j] && ql >= 0 && fabsf(ql - q) <= thr && fabsf(ql - dl[j]) <= thr;
                }
                if (!implied) lunion(L, t, t + SPK_T);
            }
        }
    }
    __syncthreads();
    // roots: the run heads (the only nodes of the forest) walk to their
    // root and keep it; every pixel then reads its head's entry
    int r[SPK_RPT];
#pragma unroll
    for (int j = 0; j < SPK_RPT; ++j) {
        const int t = (threadIdx.y + SPK_ROWS * j) * SPK_T + tx;
        r[j] = d[j] >= 0 && !conn_l[j] ? lfind(L, t) : -1;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < SPK_RPT; ++j)
        if (d[j] >= 0 && !conn_l[j]) L[(threadIdx.y + SPK_ROWS * j) * SPK_T + tx] = r[j];
    __syncthreads();
#pragma unroll
    for (int j = 0; j < SPK_RPT; ++j) {
        const int t = (threadIdx.y + SPK_ROWS * j) * SPK_T + tx;
        if (d[j] >= 0 && conn_l[j]) r[j] = L[L[t]];
        // component sizes, one shared atomic per group of lanes with the same root
        const unsigned peers = __match_any_sync(0xffffffffu, r[j]);
        if (r[j] >= 0 && tx == __ffs(peers) - 1) atomicAdd(&C[r[j]], __popc(peers));
    }
    // the tile's local roots take consecutive list slots: one reservation per tile
    int slot[SPK_RPT];
#pragma unroll
    for (int j = 0; j < SPK_RPT; ++j) {
        const int ty = threadIdx.y + SPK_ROWS * j, t = ty * SPK_T + tx;
        const bool is_root = x < W && blockIdx.y * SPK_T + ty < H && r[j] == t;
        slot[j] = is_root ? atomicAdd(&n_roots, 1) : -1;
    }
    __syncthreads();
    if (tid == 0) base = n_roots > 0 ? atomicAdd(pv.roots[view], n_roots) : 0;
    __syncthreads();
#pragma unroll
    for (int j = 0; j < SPK_RPT; ++j) {
        const int ty = threadIdx.y + SPK_ROWS * j, t = ty * SPK_T + tx, y = blockIdx.y * SPK_T + ty;
        if (x < W && y < H) {
            const size_t i = size_t(y) * W + x;
            const int rx = blockIdx.x * SPK_T + (r[j] & (SPK_T - 1)), ry = blockIdx.y * SPK_T + (r[j] / SPK_T);
            pv.lab[view][i] = r[j] >= 0 ? int(size_t(ry) * W + rx) : -1;
            if (slot[j] >= 0) {         // a local root: its count, its segment-size slot, its list entry
                pv.sz[view][i] = C[t];
                pv.root[view][i] = 0;
                pv.roots[view][1 + base + slot[j]] = int(i);
            }
        }
    }
}

// Links across tile borders: item k < H * (tx_n - 1) is row k % H of the
// right border of tile column k / H; the rest are bottom borders, x
// fastest.  Neighbouring lanes thus hold neighbouring pixel pairs of one
// border, and a segment crossing it over many pixels makes the same union
// (the same two tile-local roots) many times: a lane skips its union when
// the lane before it holds the same connected pair (unions are idempotent,
// so the segments are the same).
__global__ void k_spk_border(PostViews pv, int W, int H, float thr, unsigned* err) {
    grid_dep_wait();
    const int view = blockIdx.z;
    const float* __restrict__ D = pv.cur[view];
    int32_t* lab = pv.lab[view];
    const int txn = (W + SPK_T - 1) / SPK_T, tyn = (H + SPK_T - 1) / SPK_T;
    const long long nr = (long long)H * (txn - 1), nb = (long long)W * (tyn - 1);
    const int lane = threadIdx.x & 31;
    // every lane of a warp runs the same trip count (the shuffle below)
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long k0 = blockIdx.x * (long long)blockDim.x + (threadIdx.x & ~31); k0 < nr + nb; k0 += stride) {
        const long long k = k0 + lane;
        int a = -1, b = -1;
        if (k < nr + nb) {
            int x, y, x2, y2;
            if (k < nr) {
                y = int(k % H);
                x = int(k / H) * SPK_T + SPK_T - 1;
                x2 = x + 1; y2 = y;
            } else {
                const long long kb = k - nr;
                x = int(kb % W);
                y = int(kb / W) * SPK_T + SPK_T - 1;
                x2 = x; y2 = y + 1;
            }
            const size_t i = size_t(y) * W + x, j = size_t(y2) * W + x2;
            const float d = D[i], q = D[j];
            if (d >= 0 && q >= 0 && fabsf(q - d) <= thr) {
                a = lab[i];
                b = lab[j];
            }
        }
        const int pa = __shfl_up_sync(0xffffffffu, a, 1), pb = __shfl_up_sync(0xffffffffu, b, 1);
        const bool same = lane > 0 && pa == a && pb == b;
        if (a >= 0 && !same) uf_union(lab, a, b, err);
    }
}

// Sizes: every tile-local root (from the roots list) adds its count at its
// global root g and keeps -(g + 1) in its size slot (only this thread reads
// that slot).
__global__ void k_spk_count(PostViews pv, int n, unsigned* err) {
    grid_dep_wait();
    const int view = blockIdx.z;
    int32_t* lab = pv.lab[view];
    int32_t* sz = pv.sz[view];
    int32_t* acc = pv.root[view];
    const int32_t* roots = pv.roots[view];
    const int nr = min(roots[0], n);
    const int lane = threadIdx.x & 31;
    // warp-uniform trips; lanes with the same global root add their counts
    // with one atomic (neighbouring list entries often share a segment)
    for (int k0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31); k0 < nr; k0 += gridDim.x * blockDim.x) {
        const int k = k0 + lane;
        int i = -1, c = 0, g = -1;
        if (k < nr) {
            i = roots[1 + k];
            c = sz[i];
            g = uf_find(lab, i, err);
        }
        const unsigned peers = __match_any_sync(0xffffffffu, g);
        const int total = __reduce_add_sync(peers, c);
        if (g >= 0 && lane == __ffs(peers) - 1) atomicAdd(&acc[g], total);
        if (i >= 0) sz[i] = -(g + 1);
    }
}

// out = in with the pixels of segments smaller than min_size set invalid:
// a pixel's tile-local root (itself, or lab[i]) holds -(global root + 1).
__global__ void k_spk_apply(PostViews pv, int n, int min_size) {
    grid_dep_wait();
    const int view = blockIdx.z;
    const float* __restrict__ D = pv.cur[view];
    float* __restrict__ O = pv.nxt[view];
    const int32_t* __restrict__ lab = pv.lab[view];
    const int32_t* __restrict__ sz = pv.sz[view];
    const int32_t* __restrict__ acc = pv.root[view];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float d = D[i];
        float o = d;
        if (d >= 0 && acc[-sz[lab[i]] - 1] < min_size) o = -1.0f;
        O[i] = o;
    }
}

__global__ void k_uf_apply(float* D, const int32_t* __restrict__ root, const int32_t* sz, int n, int min_size) {
    grid_dep_wait();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int r = root[i];
    if (r >= 0 && sz[r] < min_size) D[i] = -1.0f;
}

// horizontal = 1: one thread per row; 0: one thread per column (used for
// gap widths too large for the per-pixel search).
__global__ void k_gap(PostViews pv, int W, int H, int gap, int horizontal) {
    grid_dep_wait();
    float* D = pv.cur[blockIdx.z];
    int l = blockIdx.x * blockDim.x + threadIdx.x;
    int lines = horizontal ? H : W, len = horizontal ? W : H;
    if (l >= lines) return;
    size_t base = horizontal ? size_t(l) * W : size_t(l);
    size_t stride = horizontal ? 1 : size_t(W);
    int k = 0;
    while (k < len) {
        if (D[base + k * stride] >= 0) { ++k; continue; }
        int k0 = k;
        while (k < len && D[base + k * stride] < 0) ++k;
        if (k0 > 0 && k < len && k - k0 <= gap) {
            float a = D[base + (k0 - 1) * stride], b = D[base + k * stride];
            float f = fabsf(a - b) <= 3.0f ? __fmul_rn(0.5f, __fadd_rn(a, b)) : fminf(a, b);
            for (int q = k0; q < k; ++q) D[base + q * stride] = f;
        }
    }
}

// Gap interpolation (rows, then columns), adaptive mean and median in one
// pass over a 32x32 output tile, every intermediate in shared memory.  The
// input region carries a halo of G + 3 for gaps up to G (the column pass
// needs the row pass G rows away, the mean 2 more, the median 1 more).
// Each stage is computed exactly as its separate kernel (k_gap_px,
// k_mean_median) does.
constexpr int PT = 32, PGMAX = 8;
__device__ __forceinline__ float gap_fill(const float* line, int stride, int k, int len, int gap, float c) {
    // line[k*stride] is the pixel; positions < 0 or >= len are outside the image
    if (c >= 0) return c;
    int lo = -1, hi = -1;
    for (int j = 1; j <= gap && k - j >= 0; ++j)
        if (line[-j * stride] >= 0) { lo = k - j; break; }
    if (lo >= 0)
        for (int j = 1; j <= gap && k + j < len; ++j)
            if (line[j * stride] >= 0) { hi = k + j; break; }
    if (lo >= 0 && hi >= 0 && hi - lo - 1 <= gap) {
        float a = line[-(k - lo) * stride], b = line[(hi - k) * stride];
        return fabsf(a - b) <= 3.0f ? __fmul_rn(0.5f, __fadd_rn(a, b)) : fminf(a, b);
    }
    return c;
}

// 9-input sorting network (25 compare-exchanges, depth 7; checked by the
// 0-1 principle on all 512 binary inputs).
template <int I, int J>
__device__ __forceinline__ void cex(float (&a)[9]) {
    const float x = a[I], y = a[J];
    a[I] = fminf(x, y);
    a[J] = fmaxf(x, y);
}
__device__ __forceinline__ void sort9(float (&a)[9]) {
    cex<0, 3>(a); cex<1, 7>(a); cex<2, 5>(a); cex<4, 8>(a); cex<0, 7>(a); cex<2, 4>(a); cex<3, 8>(a);
    cex<5, 6>(a); cex<0, 2>(a); cex<1, 3>(a); cex<4, 5>(a); cex<7, 8>(a); cex<1, 4>(a); cex<3, 6>(a);
    cex<5, 7>(a); cex<0, 1>(a); cex<2, 4>(a); cex<3, 5>(a); cex<6, 8>(a); cex<2, 3>(a); cex<4, 5>(a);
    cex<6, 7>(a); cex<1, 2>(a); cex<3, 4>(a); cex<5, 6>(a);
}

// Adaptive-mean weights.  Every value the mean reads is a multiple of 1/4
// (integer disparities, halves from the row gap pass, quarters from the
// column pass) in [0, disp_max], so with the key K = 4 * d the weight of a
// valid pair is WT[|K_q - K_p|], WT[j] = 1 / (1 + (j/4)^2) made by the same
// correctly rounded operations as the direct formula, for j <= 4 disp_max.
// Invalid pixels get a key far away from every valid one, which lands on
// the table's last entry, weight 0: an invalid neighbour adds 0 to both
// sums (bit for bit the same as skipping it).  The table has
// 4 disp_max + 2 entries.  The neighbour's value is read back from its key
// (K / 4 is exact for these quarters), so the 5x5 window loads one array.
constexpr int K_INVALID = 1 << 20;

// spk_min > 0: the input is the L/R result before speckle removal, and
// every loaded pixel goes through the speckle decision of k_spk_apply
// (segments smaller than spk_min become invalid) on the way in.
// Persistent: each CTA builds the weight table once and walks 32x32 tiles
// of both views with a stride of the grid size.
constexpr int POST_THREADS = 512;    // threads of a tile-filter CTA (measured against 256 and 1024)
template <int G, bool GAP, bool MEAN, bool MEDIAN, int NT>
__global__ void __launch_bounds__(NT, 2048 / NT) k_post_tile(PostViews pv, int W, int H, int gap, int spk_min,
                                                             int wt_n, int nviews) {
    grid_dep_wait();
    constexpr int PHALO = G + 3, PS = PT + 2 * PHALO;   // S tile side
    extern __shared__ float WT[];               // wt_n weights when MEAN
    __shared__ float S[PS][PS];                 // input, halo PHALO
    __shared__ float G2[PS][PT + 6];            // after the row pass: columns [-3, 35)
    __shared__ float V[PT + 6][PT + 6];         // after the column pass: [-3, 35)^2
    __shared__ int K[MEAN ? PT + 6 : 1][PT + 6];   // mean keys of V
    __shared__ float M[PT + 2][PT + 2];         // after the mean: [-1, 33)^2
    const int tid = threadIdx.x;
    const float OUT = -2.0f;                    // outside the image (never valid, never filled)
    if (MEAN)
        for (int j = tid; j < wt_n; j += NT) {
            const float q = float(j) * 0.25f;
            WT[j] = j < wt_n - 1 ? __frcp_rn(__fmaf_rn(q, q, 1.0f)) : 0.0f;
        }
    const int tiles_x = (W + PT - 1) / PT, tiles_y = (H + PT - 1) / PT, per_view = tiles_x * tiles_y;
    for (int tile = blockIdx.x; tile < nviews * per_view; tile += gridDim.x) {
        const int view = tile / per_view, tv = tile - view * per_view;
        const float* __restrict__ src = pv.cur[view];
        float* __restrict__ dst = pv.nxt[view];
        const int u0 = (tv % tiles_x) * PT, v0 = (tv / tiles_x) * PT;
        const int32_t* __restrict__ lab = pv.lab[view];
        const int32_t* __restrict__ sz = pv.sz[view];
        const int32_t* __restrict__ acc = pv.root[view];
        __syncthreads();                        // the previous tile (and the table) is done with
        // The speckle decision of k_spk_apply: the local root lab[j] holds
        // -(global root + 1) in its size slot, whose segment size is
        // acc[global root].  The value and lab[j] are loaded together, so each
        // pixel waits on three dependent loads, and the loop is unrolled so that
        // two pixels' chains overlap.
#pragma unroll 2
        for (int i = tid; i < PS * PS; i += NT) {
            int r = i / PS, c = i % PS;
            int x = u0 - PHALO + c, y = v0 - PHALO + r;
            float d = OUT;
            if (x >= 0 && x < W && y >= 0 && y < H) {
                const size_t j = size_t(y) * W + x;
                d = src[j];
                if (spk_min > 0) {
                    const int l = lab[j];
                    if (d >= 0 && acc[-sz[l] - 1] < spk_min) d = -1.0f;   // a valid pixel has l >= 0
                }
            }
            S[r][c] = d;
        }
        __syncthreads();
        // row pass on rows [-PHALO, 32+PHALO), columns [-3, 35)
        for (int i = tid; i < PS * (PT + 6); i += NT) {
            int r = i / (PT + 6), c = i % (PT + 6);
            int x = u0 - 3 + c;
            float val = S[r][c + PHALO - 3];
            if (GAP && val != OUT && val < 0) val = gap_fill(&S[r][c + PHALO - 3], 1, x, W, gap, val);
            G2[r][c] = val;
        }
        __syncthreads();
        // column pass on [-3, 35)^2
        for (int i = tid; i < (PT + 6) * (PT + 6); i += NT) {
            int r = i / (PT + 6), c = i % (PT + 6);
            int y = v0 - 3 + r;
            float val = G2[r + PHALO - 3][c];
            if (GAP && val != OUT && val < 0) val = gap_fill(&G2[r + PHALO - 3][c], PT + 6, y, H, gap, val);
            V[r][c] = val;
            if (MEAN) K[r][c] = val >= 0 ? __float2int_rn(val * 4.0f) : K_INVALID;
        }
        __syncthreads();
        // mean on [-1, 33)^2, in the oracle's (dy, dx) order: num by fma, den by add
        for (int i = tid; i < (PT + 2) * (PT + 2); i += NT) {
            int r = i / (PT + 2), c = i % (PT + 2);
            float dp = V[r + 2][c + 2];
            float out = dp;
            if (MEAN && dp >= 0) {
                const int kp = K[r + 2][c + 2];
                float num = 0.0f, den = 0.0f;
#pragma unroll
                for (int dy = -2; dy <= 2; ++dy)
#pragma unroll
                    for (int dx = -2; dx <= 2; ++dx) {
                        const int kq = K[r + 2 + dy][c + 2 + dx];
                        const float dq = __int2float_rn(kq) * 0.25f;
                        const int j = min(abs(kq - kp), wt_n - 1);
                        const float w = WT[j];
                        num = __fmaf_rn(w, dq, num);
                        den = __fadd_rn(den, w);
                    }
                out = __fdiv_rn(num, den);
            }
            M[r][c] = out;
        }
        __syncthreads();
        for (int o = tid; o < PT * PT; o += NT) {
            int ty = o / PT, tx = o % PT;
            int u = u0 + tx, v = v0 + ty;
            if (u < W && v < H) {
                float c = M[ty + 1][tx + 1];
                float out = c;
                if (MEDIAN && c >= 0) {
                    // invalid neighbours sort last as +inf; the lower median of the
                    // n valid values is then element (n-1)/2 (all in registers)
                    float a[9];
                    int n = 0;
#pragma unroll
                    for (int k = 0; k < 9; ++k) {
                        float q = M[ty + k / 3][tx + k % 3];
                        n += q >= 0 ? 1 : 0;
                        a[k] = q >= 0 ? q : INFINITY;
                    }
                    sort9(a);
                    const int m = (n - 1) >> 1;     // n >= 1 (the centre), so m in [0, 4]
                    out = a[0];
#pragma unroll
                    for (int k = 1; k < 5; ++k) out = m == k ? a[k] : out;
                }
                dst[size_t(v) * W + u] = out;
            }
        }
    }
}

}  // namespace

bool post_fuses_speckle(const DevParams& p, bool median, bool adaptive_mean) {
    const int gap = p.ipol_gap_width;
    return p.speckle_size > 0 && gap <= PGMAX && (gap > 0 || adaptive_mean || median);
}

cudaError_t launch_post(PostViews pv, int nviews, const Geom& g, const DevParams& p, bool median,
                        bool adaptive_mean, unsigned* err, cudaStream_t st, int* nlaunch, int num_sms) {
    const int W = g.W, H = g.H, n = W * H;
    int launched = 0;
    auto flip = [&]() {
        for (int k = 0; k < 2; ++k) { float* t = pv.cur[k]; pv.cur[k] = pv.nxt[k]; pv.nxt[k] = t; }
    };
    // with the tile filter following, speckle removal is applied as it loads
    const bool fuse = post_fuses_speckle(p, median, adaptive_mean);
    if (p.speckle_size > 0) {
        for (int k = 0; k < nviews; ++k) cudaMemsetAsync(pv.roots[k], 0, sizeof(int32_t), st);
        const dim3 tiles((W + SPK_T - 1) / SPK_T, (H + SPK_T - 1) / SPK_T, nviews);
        launch_k(k_spk_tile, tiles, dim3(SPK_T, SPK_ROWS), 0, st, pv, W, H, p.speckle_sim_threshold);
        const long long border = (long long)H * (tiles.x - 1) + (long long)W * (tiles.y - 1);
        const int gb = int(border / 256 + 1 < 4096 ? border / 256 + 1 : 4096);
        launch_k(k_spk_border, dim3(gb, 1, nviews), 256, 0, st, pv, W, H, p.speckle_sim_threshold, err);
        const int gn = imax(1, imin(8 * 1024, (n + 255) / 256));
        // the roots list is far shorter than the image: a grid of one CTA per
        // SM walks it (idle CTAs cost their launch; measured against four)
        launch_k(k_spk_count, dim3(imin(gn, num_sms), 1, nviews), 256, 0, st, pv, n, err);
        launched += 3;
        if (!fuse) {
            launch_k(k_spk_apply, dim3(gn, 1, nviews), 256, 0, st, pv, n, p.speckle_size);
            flip();
            launched += 1;
        }
    }
    const int gap = p.ipol_gap_width;
    const int spk = fuse ? p.speckle_size : 0;
    const bool tile_gap = gap > 0 && gap <= PGMAX;
    if (gap > PGMAX) {   // wide gaps: serial scans per line, in place
        launch_k(k_gap, dim3((H + 127) / 128, 1, nviews), 128, 0, st, pv, W, H, gap, 1);
        launch_k(k_gap, dim3((W + 127) / 128, 1, nviews), 128, 0, st, pv, W, H, gap, 0);
        launched += 2;
    }
    if (tile_gap || adaptive_mean || median) {
        // the tile pass is the chain's last: it writes the final buffers
        // directly unless one of them is its own input
        bool direct = true;
        for (int k = 0; k < nviews; ++k) direct = direct && pv.out[k] != pv.cur[k];
        if (direct)
            for (int k = 0; k < nviews; ++k) pv.nxt[k] = pv.out[k];
        const int tiles = ((W + PT - 1) / PT) * ((H + PT - 1) / PT) * nviews;
        const int grid = imax(1, imin(tiles, (2048 / POST_THREADS) * num_sms));
        const int wt_n = 4 * g.D + 2;
        const size_t smem = adaptive_mean ? size_t(wt_n) * sizeof(float) : 0;
        const int key = (tile_gap ? 4 : 0) | (adaptive_mean ? 2 : 0) | (median ? 1 : 0);
        auto go = [&](auto kern) {
            if (smem) allow_smem(kern);
            launch_k(kern, grid, POST_THREADS, smem, st, pv, W, H, gap, spk, wt_n, nviews);
        };
        if (!tile_gap || gap <= 3) {   // halo 6
            switch (key) {
            case 1: go(k_post_tile<3, false, false, true, POST_THREADS>); break;
            case 2: go(k_post_tile<3, false, true, false, POST_THREADS>); break;
            case 3: go(k_post_tile<3, false, true, true, POST_THREADS>); break;
            case 4: go(k_post_tile<3, true, false, false, POST_THREADS>); break;
            case 5: go(k_post_tile<3, true, false, true, POST_THREADS>); break;
            case 6: go(k_post_tile<3, true, true, false, POST_THREADS>); break;
            default: go(k_post_tile<3, true, true, true, POST_THREADS>); break;
            }
        } else {                       // gaps 4..8: halo 11
            switch (key) {
            case 4: go(k_post_tile<PGMAX, true, false, false, POST_THREADS>); break;
            case 5: go(k_post_tile<PGMAX, true, false, true, POST_THREADS>); break;
            case 6: go(k_post_tile<PGMAX, true, true, false, POST_THREADS>); break;
            default: go(k_post_tile<PGMAX, true, true, true, POST_THREADS>); break;
            }
        }
        flip();
        launched += 1;
    }
    for (int k = 0; k < nviews; ++k)   // cudaMemcpyDefault: the final buffer may be mapped host memory
        if (pv.cur[k] != pv.out[k])
            cudaMemcpyAsync(pv.out[k], pv.cur[k], size_t(n) * sizeof(float), cudaMemcpyDefault, st);
    if (nlaunch) *nlaunch += launched;
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Allocation-free speckle removal (elas_b200_speckle_noalloc).
//
// For callers that must not allocate device memory -- code inside a CUDA
// stream capture (cudaMalloc cannot be captured), plugin hosts and real-time
// loops that forbid allocation after start-up.  Its scratch (labels, roots,
// segment sizes and an error word) is this one file-scope array, resident on
// every GPU that loads the library until the process exits.  In host code
// the array's name is only a host-side stand-in, so its device address is
// looked up with cudaGetSymbolAddress once per device and CUDA context (the
// first call on a device, and the first after a cudaDeviceReset, which
// should therefore happen outside any stream capture) and cached.  Every
// call reuses the array; the kernels initialise all of it that must start
// at zero, and calls that overlap on the GPU race.
//
// The error word receives the bounds flag of the union-find walks, which
// valid inputs cannot raise: labels only ever decrease, so a find walks at
// most width*height <= 2^19 nodes, and a union retries only after another
// thread's hook succeeded, at most 2^19 times -- both below UF_LIMIT.  The
// call does not read it back (that would synchronise the caller's stream).
static __device__ __align__(256) int32_t g_noalloc_scratch[3 * ELAS_NOALLOC_MAX_PIXELS + 64];

namespace {
constexpr int kNoallocMaxDevices = 64;
struct NoallocSlot {
    void* ctx = nullptr;        // CUcontext the address was looked up in
    int32_t* base = nullptr;
};
NoallocSlot g_noalloc_slot[kNoallocMaxDevices];
std::mutex g_noalloc_mutex;

// The current CUDA context through the runtime's driver entry point (no
// link against libcuda); null if the entry point is unavailable.
void* current_context() {
    using GetCtx = int (*)(void**);
    static GetCtx fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<GetCtx>(p);
    }();
    void* ctx = nullptr;
    if (!fn || fn(&ctx) != 0) return nullptr;
    return ctx;
}
}  // namespace

}  // namespace elas

extern "C" int elas_b200_speckle_noalloc(const float* d_in, float* d_out, int32_t width, int32_t height,
                                         float sim_threshold, int32_t min_size, void* stream) {
    using namespace elas;
    if (!d_in || !d_out || width <= 0 || height <= 0 || min_size < 0) return ELAS_ERR_INVALID_ARG;
    if (int64_t(width) * height > ELAS_NOALLOC_MAX_PIXELS) return ELAS_ERR_TOO_LARGE;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoallocMaxDevices) return ELAS_ERR_NO_DEVICE;
    int32_t* base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mutex);
        NoallocSlot& slot = g_noalloc_slot[dev];
        void* ctx = current_context();
        if (!slot.base || ctx != slot.ctx) {
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return ELAS_ERR_CUDA;
            slot.base = static_cast<int32_t*>(p);
            slot.ctx = ctx;
        }
        base = slot.base;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int W = width, H = height, n = W * H, tb = 256;
    int32_t* lab = base;
    int32_t* root = base + ELAS_NOALLOC_MAX_PIXELS;
    int32_t* sz = base + 2 * ELAS_NOALLOC_MAX_PIXELS;
    unsigned* err = reinterpret_cast<unsigned*>(base + 3 * ELAS_NOALLOC_MAX_PIXELS);
    // each call's own status: an earlier, unrelated launch error is not this call's
    if (d_out != d_in &&
        cudaMemcpyAsync(d_out, d_in, size_t(n) * sizeof(float), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        return ELAS_ERR_CUDA;
    if (cudaMemsetAsync(err, 0, sizeof(unsigned), st) != cudaSuccess) return ELAS_ERR_CUDA;
    if (min_size > 0) {
        const int blocks = (n + tb - 1) / tb;
        if (launch_k(k_uf_init, blocks, tb, 0, st, d_out, lab, sz, W, H, sim_threshold) != cudaSuccess ||
            launch_k(k_uf_union, blocks, tb, 0, st, d_out, lab, W, H, sim_threshold, err) != cudaSuccess ||
            launch_k(k_uf_count, blocks, tb, 0, st, lab, root, sz, n, err) != cudaSuccess ||
            launch_k(k_uf_apply, blocks, tb, 0, st, d_out, root, sz, n, min_size) != cudaSuccess)
            return ELAS_ERR_CUDA;
    }
    return ELAS_OK;
}
