// GPU Delaunay triangulation of the support points of both views
// (algorithm and predicates: delaunay_core.h).  Replaces the reference's
// device->host copy, Triangle call and host->device copy
// (src/Elas.cu:282-328, called twice from :89-90).
//
// Both views run as two independent problems inside the same launches:
// problem 0 triangulates (u, v), problem 1 triangulates (u - d, v).
#include <cuda_runtime.h>
#include "common.cuh"
#include "delaunay_core.h"
#include "kernels.h"

namespace elas {

using namespace del;

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

// Per lattice row: sort the row's points by (x, index), drop repeated x
// (keeps the lowest index), write the unique list to srt[row_off[r] ..] and
// its length to rcnt[r].
__global__ void __launch_bounds__(512) k_rowsort(DelDev d0, DelDev d1, const int32_t* __restrict__ row_off,
                                                 int nrows, unsigned* err) {
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
        key[i] = i < n ? (uint64_t(uint32_t(D.x[b + i])) << 32 | uint32_t(b + i)) : ~0ull;
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
    for (int i0 = warp * span; i0 < min(n, (warp + 1) * span); i0 += 32) {
        int i = i0 + lane;
        bool k = i < min(n, (warp + 1) * span) && keep[i];
        unsigned m = __ballot_sync(0xffffffffu, k);
        if (k) D.srt[b + base + __popc(m & ((1u << lane) - 1))] = int32_t(key[i] & 0xffffffffu);
        base += __popc(m);
    }
}

// Non-empty rows (list + rank), strip offsets and the two hull pockets.
// One 1024-thread block per problem; dynamic shared memory holds the chain
// (index, x, y) and the stack of the pocket walk when it fits.
__global__ void __launch_bounds__(1024) k_plan(DelDev d0, DelDev d1, const int32_t* __restrict__ row_off,
                                               int nrows, int smem_rows, unsigned* err) {
    extern __shared__ int32_t sh[];
    __shared__ int ws[33];
    DelDev D = blockIdx.x ? d1 : d0;
    int R = 0, total = 0;
    // non-empty rows in order, and each row's rank
    for (int r0 = 0; r0 < nrows; r0 += blockDim.x) {
        int r = r0 + threadIdx.x;
        int f = (r < nrows && D.rcnt[r] > 0) ? 1 : 0;
        int pos = block_scan(f, ws, &total);
        if (f) D.ne[R + pos] = r;
        R += total;
    }
    __syncthreads();
    // strip s between ne[s] and ne[s+1] holds rcnt[ne[s]] + rcnt[ne[s+1]] - 2 triangles
    int off = 0;
    for (int s0 = 0; s0 < R - 1; s0 += blockDim.x) {
        int s = s0 + threadIdx.x;
        int c = s < R - 1 ? D.rcnt[D.ne[s]] + D.rcnt[D.ne[s + 1]] - 2 : 0;
        int pos = block_scan(c, ws, &total);
        if (s < R - 1) D.soff[s] = off + pos;
        off += total;
    }
    const bool in_smem = R <= smem_rows;
    int32_t* ci = in_smem ? sh : D.chain;
    int32_t* cx = ci + (in_smem ? smem_rows : nrows);
    int32_t* cy = cx + (in_smem ? smem_rows : nrows);
    int32_t* stk = cy + (in_smem ? smem_rows : nrows);
    int pockets = 0;
    if (R >= 2 && off + 2 * R > D.Tmax) {
        if (threadIdx.x == 0) set_err(err, ERRF_TRI_COUNT);
    } else if (R >= 2) {
        for (int side = 0; side < 2; ++side) {
            for (int s = threadIdx.x; s < R; s += blockDim.x) {
                int r = D.ne[s];
                int i = D.srt[row_off[r] + (side ? D.rcnt[r] - 1 : 0)];
                ci[s] = i; cx[s] = D.x[i]; cy[s] = D.y[i];
            }
            __syncthreads();
            if (threadIdx.x == 0)
                pockets += fill_pockets(ci, cx, cy, R, side ? -1 : +1, stk, D.tri + 3 * size_t(off + pockets));
            __syncthreads();
        }
    }
    if (threadIdx.x == 0) {
        D.ctr[0] = (R >= 2 && off + 2 * R <= D.Tmax) ? off + pockets : 0;
        D.ctr[1] = off;
        D.ctr[6] = R;
    }
}

// One thread per sorted point of a non-empty row: the point's triangle in
// the strip below its row (as the upper row) and in the strip above (as the
// lower row), placed by merge path.
__global__ void k_strips(DelDev d0, DelDev d1, const int32_t* __restrict__ row_off, int nmax) {
    const DelDev& D = blockIdx.y ? d1 : d0;
    const int R = D.ctr[6];
    if (D.ctr[0] == 0) return;
    Pts P{D.x, D.y};
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < nmax; g += gridDim.x * blockDim.x) {
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
    const DelDev& D = blockIdx.y ? d1 : d0;
    uint32_t cap = hash_cap(D.ctr[0]);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cap && i < D.Hmax; i += gridDim.x * blockDim.x) {
        D.hkey[i] = HASH_EMPTY;
        D.hcnt[i] = 0;
    }
}

__global__ void k_hash_insert(DelDev d0, DelDev d1, unsigned* err) {
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
        D.fwd[h] = -1;
    }
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < T; t += gridDim.x * blockDim.x) {
        D.lock[t] = LOCK_FREE;
        D.fround[t] = -1;
    }
}

struct SAMin {
    __device__ void operator()(uint32_t* p, uint32_t v) const { atomicMin(p, v); }
};

// Worklist-driven Lawson flipping, one 1024-thread CTA per problem, every
// phase separated by __syncthreads.  At most `max_rounds` rounds; hitting the
// limit raises ERRF_FLIP_LIMIT.
__global__ void __launch_bounds__(FLIP_THREADS) k_flip(DelDev d0, DelDev d1, int max_rounds, unsigned* err) {
    __shared__ int n_cand, n_flip, n_fwd, n_next, n_cur, stop, prev_fwd;
    const DelDev& D = blockIdx.x ? d1 : d0;
    const int T = D.ctr[0];
    Flip S{Pts{D.x, D.y}, D.tri, D.opp, D.lock, D.fround, D.fwd, D.cand, D.flips, D.res, D.fwdl,
           {D.wl0, D.wl1}, D.Tmax};
    const int cand_cap = 3 * D.Tmax, wl_cap = 6 * D.Tmax;
    const int tid = threadIdx.x;
    if (tid == 0) { n_cur = 3 * T; n_fwd = 0; prev_fwd = 0; stop = 0; }
    __syncthreads();
    int round = 0;
    int flips_total = 0;
    for (; round < max_rounds; ++round) {
        int32_t* cur = S.wl[round & 1];
        int32_t* nxt = S.wl[(round + 1) & 1];
        if (tid == 0) { n_cand = 0; n_next = 0; }
        // clear the forwarding entries of the previous round
        for (int k = tid; k < prev_fwd; k += FLIP_THREADS) S.fwd[S.fwdl[k]] = -1;
        __syncthreads();
        // A: propose
        const int items = n_cur;
        for (int k = tid; k < items; k += FLIP_THREADS) {
            int h = round == 0 ? k : cur[k];
            bool ok = flip_propose(S, h, T, uint32_t(round), round == 0, SAMin(), [&](int hh, int nn) {
                int idx = atomicAdd(&n_cand, 1);
                if (idx < cand_cap) { S.cand[2 * idx] = hh; S.cand[2 * idx + 1] = nn; }
            });
            if (!ok) set_err(err, ERRF_BOUNDS);
        }
        __syncthreads();
        const int nc = n_cand;
        if (nc > cand_cap) { if (tid == 0) { set_err(err, ERRF_BOUNDS); stop = 1; } }
        if (tid == 0) { n_flip = 0; n_fwd = 0; }
        __syncthreads();
        if (nc == 0 || stop) break;
        // B: flip the winners
        for (int c = tid; c < nc; c += FLIP_THREADS) {
            int slots[4];
            if (flip_apply(S, S.cand[2 * c], S.cand[2 * c + 1], uint32_t(round), slots)) {
                int f = atomicAdd(&n_flip, 1);
                int h = S.cand[2 * c];
                S.flips[2 * f] = h / 3;
                S.flips[2 * f + 1] = S.cand[2 * c + 1];
                int q = atomicAdd(&n_fwd, 4);
                for (int k = 0; k < 4; ++k) S.fwdl[q + k] = slots[k];
            }
        }
        __syncthreads();
        const int nf = n_flip;
        // C1: resolve the outer neighbours (read only)
        for (int f = tid; f < nf; f += FLIP_THREADS) flip_resolve(S, f);
        __syncthreads();
        // C2: relink, queue the outer edges, release locks, requeue lost proposals
        for (int f = tid; f < nf; f += FLIP_THREADS)
            flip_relink(S, f, [&](int x) {
                int idx = atomicAdd(&n_next, 1);
                if (idx < wl_cap) nxt[idx] = x;
            });
        for (int c = tid; c < nc; c += FLIP_THREADS) {
            int h = S.cand[2 * c], n = S.cand[2 * c + 1], t = h / 3;
            S.lock[t] = LOCK_FREE;
            S.lock[n] = LOCK_FREE;
            if (S.fround[t] != round && S.fround[n] != round) {
                int idx = atomicAdd(&n_next, 1);
                if (idx < wl_cap) nxt[idx] = h;
            }
        }
        flips_total += nf;
        __syncthreads();
        if (tid == 0) {
            if (n_next > wl_cap) { set_err(err, ERRF_BOUNDS); stop = 1; }
            n_cur = min(n_next, wl_cap);
            prev_fwd = n_fwd;
        }
        __syncthreads();
        if (stop) break;
    }
    if (tid == 0) {
        D.ctr[4] = round + 1;
        D.ctr[5] = flips_total;
        if (round >= max_rounds) set_err(err, ERRF_FLIP_LIMIT);
    }
}

__global__ void k_normalise(DelDev d0, DelDev d1) {
    const DelDev& D = blockIdx.y ? d1 : d0;
    const int T = D.ctr[0];
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < T; t += gridDim.x * blockDim.x)
        normalise(D.tri + 3 * size_t(t));
}

}  // namespace

cudaError_t launch_delaunay(DelDev& d0, DelDev& d1, const int32_t* row_off, int nrows, int nmax, int num_sms,
                            unsigned* err, cudaStream_t st, int* nlaunch) {
    k_rowsort<<<dim3(nrows, 2), 512, 0, st>>>(d0, d1, row_off, nrows, err);
    int smem_rows = imin(nrows, (96 * 1024) / 16);
    size_t smem = size_t(smem_rows) * 16;
    cudaFuncSetAttribute(k_plan, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    k_plan<<<2, 1024, smem, st>>>(d0, d1, row_off, nrows, smem_rows, err);
    int blocks = 4 * num_sms;
    k_strips<<<dim3(imax(1, imin(blocks, (nmax + 255) / 256)), 2), 256, 0, st>>>(d0, d1, row_off, nmax);
    k_hash_clear<<<dim3(blocks, 2), 256, 0, st>>>(d0, d1);
    k_hash_insert<<<dim3(blocks, 2), 256, 0, st>>>(d0, d1, err);
    k_link<<<dim3(blocks, 2), 256, 0, st>>>(d0, d1, err);
    k_flip<<<2, FLIP_THREADS, 0, st>>>(d0, d1, 100000, err);
    k_normalise<<<dim3(blocks, 2), 256, 0, st>>>(d0, d1);
    if (nlaunch) *nlaunch += 8;
    return cudaGetLastError();
}

}  // namespace elas
