// GPU Delaunay triangulation of the support points of both views
// (algorithm and predicates: delaunay_core.h).  Replaces the reference's
// device->host copy, Triangle call and host->device copy
// (src/Elas.cu:282-328, called twice from :89-90).
//
// Both views run as two independent problems inside the same launches:
// problem 0 triangulates (u, v), problem 1 triangulates (u - d, v).
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include "common.cuh"
#include "delaunay_core.h"
#include "kernels.h"

namespace cg = cooperative_groups;

namespace elas {

using namespace del;

namespace {

constexpr int SORT_CAP = 2048;   // max candidates per lattice row

__device__ __forceinline__ void set_err(unsigned* err, unsigned f) { atomicOr(err, f); }

// Per lattice row: sort the row's points by (x, index), drop repeated x
// (keeps the lowest index), write the unique list to srt[row_off[r] ..] and
// its length to rcnt[r].
__global__ void __launch_bounds__(512) k_rowsort(DelDev d0, DelDev d1, const int32_t* __restrict__ row_off,
                                                 int nrows, unsigned* err) {
    __shared__ unsigned long long key[SORT_CAP];
    __shared__ int keep_scan[SORT_CAP];
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
        keep_scan[i] = (i == 0 || (key[i] >> 32) != (key[i - 1] >> 32)) ? 1 : 0;
    __syncthreads();
    if (threadIdx.x == 0) {   // n <= 2048: serial compaction is short
        int m = 0;
        for (int i = 0; i < n; ++i)
            if (keep_scan[i]) D.srt[b + m++] = int32_t(key[i] & 0xffffffffu);
        D.rcnt[r] = m;
    }
}

// Non-empty rows, strip offsets and the two hull pockets (one thread per
// problem; the chains are one point per lattice row).
__global__ void k_plan(DelDev d0, DelDev d1, const int32_t* __restrict__ row_off, int nrows, unsigned* err) {
    if (threadIdx.x != 0) return;
    DelDev D = blockIdx.x ? d1 : d0;
    int R = 0;
    for (int r = 0; r < nrows; ++r)
        if (D.rcnt[r] > 0) D.ne[R++] = r;
    int off = 0;
    for (int s = 0; s + 1 < R; ++s) {
        D.soff[s] = off;
        off += D.rcnt[D.ne[s]] + D.rcnt[D.ne[s + 1]] - 2;
    }
    D.ctr[1] = off;
    D.ctr[6] = R;
    if (R >= 2 && off + 2 * R <= D.Tmax) {
        Pts P{D.x, D.y};
        for (int s = 0; s < R; ++s) D.chain[s] = D.srt[row_off[D.ne[s]]];
        off += fill_pockets(P, D.chain, R, +1, D.stack, D.tri + 3 * size_t(off));
        for (int s = 0; s < R; ++s) D.chain[s] = D.srt[row_off[D.ne[s]] + D.rcnt[D.ne[s]] - 1];
        off += fill_pockets(P, D.chain, R, -1, D.stack, D.tri + 3 * size_t(off));
    } else if (R >= 2) {
        set_err(err, ERRF_TRI_COUNT);
        off = 0;
    }
    D.ctr[0] = off;
    D.ctr[2] = 0;
    D.ctr[3] = 0;
}

// One thread per strip: zipper between consecutive non-empty rows.
__global__ void k_strips(DelDev d0, DelDev d1, const int32_t* __restrict__ row_off, int max_strips) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    const DelDev& D = blockIdx.y ? d1 : d0;
    int R = D.ctr[6];
    if (i >= max_strips || i + 1 >= R) return;
    int ra = D.ne[i], rb = D.ne[i + 1];
    Pts P{D.x, D.y};
    zipper(P, D.srt + row_off[ra], D.rcnt[ra], D.srt + row_off[rb], D.rcnt[rb], D.tri + 3 * size_t(D.soff[i]));
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
    }
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < T; t += gridDim.x * blockDim.x)
        D.lock[t] = LOCK_FREE;
}

struct AMin {
    __device__ void operator()(uint32_t* p, uint32_t v) const { atomicMin(p, v); }
};
struct AAdd {
    __device__ int operator()(int32_t* p, int v) const { return atomicAdd(p, v); }
};

// Parallel Lawson flipping, all rounds in one cooperative launch.  Every
// loop is bounded: `max_rounds` rounds at most, after which ERRF_FLIP_LIMIT
// is raised and the kernel returns.
__global__ void k_flip(DelDev d0, DelDev d1, int max_rounds, unsigned* err) {
    cg::grid_group grid = cg::this_grid();
    const int T0 = d0.ctr[0], T1 = d1.ctr[0];
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int gstride = gridDim.x * blockDim.x;
    Tri S0{Pts{d0.x, d0.y}, d0.tri, d0.opp, d0.lock, d0.fwd, d0.cand, d0.ctr, d0.Tmax};
    Tri S1{Pts{d1.x, d1.y}, d1.tri, d1.opp, d1.lock, d1.fwd, d1.cand, d1.ctr, d1.Tmax};
    bool converged = false;
    int round = 0;
    for (; round < max_rounds; ++round) {
        for (int i = gtid; i < T0 + T1; i += gstride) {
            bool ok = i < T0 ? flip_propose(S0, i, T0, round, AMin(), AAdd())
                             : flip_propose(S1, i - T0, T1, round, AMin(), AAdd());
            if (!ok) set_err(err, ERRF_BOUNDS);
        }
        grid.sync();
        const int n0 = imin(((volatile int32_t*)d0.ctr)[2 + (round & 1)], 2 * d0.Tmax);
        const int n1 = imin(((volatile int32_t*)d1.ctr)[2 + (round & 1)], 2 * d1.Tmax);
        if (n0 + n1 == 0) { converged = true; break; }
        for (int i = gtid; i < n0 + n1; i += gstride) {
            if (i < n0) flip_apply(S0, d0.cand[i], round);
            else flip_apply(S1, d1.cand[i - n0], round);
        }
        grid.sync();
        for (int i = gtid; i < T0 + T1; i += gstride) {
            Tri& S = i < T0 ? S0 : S1;
            int t = i < T0 ? i : i - T0;
            int T = i < T0 ? T0 : T1;
            // validate links before the forwarding lookup
            for (int s = 0; s < 3; ++s) {
                int o = S.opp[3 * t + s];
                if (o >= 0 && (o & ~FINAL) >= 3 * T) { set_err(err, ERRF_BOUNDS); S.opp[3 * t + s] = -1; }
            }
            flip_repair(S, t);
        }
        if (gtid == 0) {
            d0.ctr[2 + ((round + 1) & 1)] = 0;
            d1.ctr[2 + ((round + 1) & 1)] = 0;
        }
        grid.sync();
    }
    if (gtid == 0) {
        d0.ctr[4] = round + 1;
        d1.ctr[4] = round + 1;
        if (!converged) set_err(err, ERRF_FLIP_LIMIT);
    }
}

__global__ void k_normalise(DelDev d0, DelDev d1) {
    const DelDev& D = blockIdx.y ? d1 : d0;
    const int T = D.ctr[0];
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < T; t += gridDim.x * blockDim.x)
        normalise(D.tri + 3 * size_t(t));
}

}  // namespace

cudaError_t launch_delaunay(DelDev& d0, DelDev& d1, const int32_t* row_off, int nrows, int num_sms,
                            int flip_blocks, unsigned* err, cudaStream_t st, int* nlaunch) {
    k_rowsort<<<dim3(nrows, 2), 512, 0, st>>>(d0, d1, row_off, nrows, err);
    k_plan<<<2, 32, 0, st>>>(d0, d1, row_off, nrows, err);
    k_strips<<<dim3((nrows + 127) / 128, 2), 128, 0, st>>>(d0, d1, row_off, nrows);
    int blocks = 4 * num_sms;
    k_hash_clear<<<dim3(blocks, 2), 256, 0, st>>>(d0, d1);
    k_hash_insert<<<dim3(blocks, 2), 256, 0, st>>>(d0, d1, err);
    k_link<<<dim3(blocks, 2), 256, 0, st>>>(d0, d1, err);
    int max_rounds = 4096;
    void* args[] = {&d0, &d1, &max_rounds, &err};
    cudaError_t e = cudaLaunchCooperativeKernel((const void*)k_flip, dim3(flip_blocks), dim3(256), args, 0, st);
    if (e != cudaSuccess) return e;
    k_normalise<<<dim3(blocks, 2), 256, 0, st>>>(d0, d1);
    if (nlaunch) *nlaunch += 8;
    return cudaGetLastError();
}

int flip_blocks_for(int num_sms) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_flip, 256, 0);
    if (per_sm < 1) per_sm = 1;
    return per_sm * num_sms;
}

}  // namespace elas
