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
//             min(a,b).  One thread per line.
//   mean      5x5 weighted mean of valid pixels, w = 1/(1+(d_q-d_p)^2).
//   median    lower median of the valid pixels of the 3x3 window.
#include <cuda_runtime.h>
#include <mutex>
#include "../../include/elas_b200.h"
#include "common.cuh"
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

// Labels start as stars over the runs of each row: every pixel points at the
// first pixel of its connected run (one warp per row, ballot scan over
// 32-pixel chunks).  Only vertical unions remain for k_uf_union_v.
__global__ void k_uf_init_rows(PostViews pv, int W, int H, float thr) {
    const int view = blockIdx.z;
    const float* D = pv.cur[view];
    int32_t* lab = pv.lab[view];
    int32_t* sz = pv.sz[view];
    const int lane = threadIdx.x & 31;
    const int v = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (v >= H) return;
    int carry = -1;
    float prev = -1.0f;
    for (int u0 = 0; u0 < W; u0 += 32) {
        const int u = u0 + lane;
        const size_t i = size_t(v) * W + u;
        float d = u < W ? D[i] : -1.0f;
        float dl = __shfl_up_sync(0xffffffffu, d, 1);
        if (lane == 0) dl = prev;
        const bool valid = d >= 0;
        const bool conn = valid && u > 0 && dl >= 0 && fabsf(d - dl) <= thr;
        const unsigned starts = __ballot_sync(0xffffffffu, valid && !conn);
        const unsigned mine = starts & (0xffffffffu >> (31 - lane));
        const int rs = mine ? int(size_t(v) * W + u0 + 31 - __clz(mine)) : carry;
        if (u < W) {
            lab[i] = valid ? rs : -1;
            sz[i] = 0;
        }
        carry = __shfl_sync(0xffffffffu, rs, 31);
        prev = __shfl_sync(0xffffffffu, d, 31);
    }
}

// Labels start at the left neighbour when it is connected (the most common
// union), else at the pixel itself.
__global__ void k_uf_init(const float* __restrict__ D, int32_t* __restrict__ lab, int32_t* __restrict__ sz, int W,
                          int H, float thr) {
    int u = blockIdx.x * blockDim.x + threadIdx.x, v = blockIdx.y;
    if (u >= W || v >= H) return;
    int i = v * W + u;
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

__global__ void k_uf_union_v(PostViews pv, int W, int H, float thr, unsigned* err) {
    const int view = blockIdx.z;
    const float* D = pv.cur[view];
    int32_t* lab = pv.lab[view];
    int u = blockIdx.x * blockDim.x + threadIdx.x, v = blockIdx.y;
    if (u >= W || v + 1 >= H) return;
    int i = v * W + u;
    float d = D[i];
    if (d < 0) return;
    float q = D[i + W];
    if (q >= 0 && fabsf(q - d) <= thr) uf_union(lab, i, i + W, err);
}

__global__ void k_uf_union(const float* __restrict__ D, int32_t* lab, int W, int H, float thr, unsigned* err) {
    int u = blockIdx.x * blockDim.x + threadIdx.x, v = blockIdx.y;
    if (u >= W || v >= H) return;
    int i = v * W + u;
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
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int r = -1;
    if (i < n && lab[i] >= 0) r = uf_find(lab, i, err);
    if (i < n) root[i] = r;
    unsigned peers = __match_any_sync(0xffffffffu, r);
    int leader = __ffs(peers) - 1;
    if (r >= 0 && (threadIdx.x & 31) == leader) atomicAdd(&sz[r], __popc(peers));
}

__global__ void k_uf_count_v(PostViews pv, int n, unsigned* err) {
    const int view = blockIdx.z;
    int32_t* lab = pv.lab[view];
    int32_t* root = pv.root[view];
    int32_t* sz = pv.sz[view];
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int r = -1;
    if (i < n && lab[i] >= 0) r = uf_find(lab, i, err);
    if (i < n) root[i] = r;
    unsigned peers = __match_any_sync(0xffffffffu, r);
    int leader = __ffs(peers) - 1;
    if (r >= 0 && (threadIdx.x & 31) == leader) atomicAdd(&sz[r], __popc(peers));
}

__global__ void k_uf_apply_v(PostViews pv, int n, int min_size) {
    const int view = blockIdx.z;
    float* D = pv.cur[view];
    const int32_t* root = pv.root[view];
    const int32_t* sz = pv.sz[view];
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int r = root[i];
    if (r >= 0 && sz[r] < min_size) D[i] = -1.0f;
}

__global__ void k_uf_apply(float* D, const int32_t* __restrict__ root, const int32_t* sz, int n, int min_size) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int r = root[i];
    if (r >= 0 && sz[r] < min_size) D[i] = -1.0f;
}

// Gap interpolation, one pixel per thread: an invalid pixel looks for the
// nearest valid pixel on each side within `gap`; both found and the run
// between them no longer than `gap` -> fill.  Equivalent to the serial
// per-line scan because filled runs never touch the pixels that bound
// other runs.  S = pass input, O = pass output.
__global__ void k_gap_px(PostViews pv, int W, int H, int gap, int horizontal) {
    const float* __restrict__ S = pv.cur[blockIdx.z];
    float* __restrict__ O = pv.nxt[blockIdx.z];
    int u = blockIdx.x * blockDim.x + threadIdx.x, v = blockIdx.y;
    if (u >= W || v >= H) return;
    size_t i = size_t(v) * W + u;
    float c = S[i];
    if (c < 0) {
        const int len = horizontal ? W : H, k = horizontal ? u : v;
        const long stride = horizontal ? 1 : W;
        int lo = -1, hi = -1;
        for (int j = 1; j <= gap && k - j >= 0; ++j)
            if (S[i - j * stride] >= 0) { lo = k - j; break; }
        if (lo >= 0)
            for (int j = 1; j <= gap && k + j < len; ++j)
                if (S[i + j * stride] >= 0) { hi = k + j; break; }
        if (lo >= 0 && hi >= 0 && hi - lo - 1 <= gap) {
            float a = S[i - (k - lo) * stride], b = S[i + (hi - k) * stride];
            c = fabsf(a - b) <= 3.0f ? __fmul_rn(0.5f, __fadd_rn(a, b)) : fminf(a, b);
        }
    }
    O[i] = c;
}

// horizontal = 1: one thread per row; 0: one thread per column (used for
// gap widths too large for the per-pixel search).
__global__ void k_gap(PostViews pv, int W, int H, int gap, int horizontal) {
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

// Adaptive mean and/or median in one pass over a 32x8 output tile: the
// input tile (halo 3) and the mean of the tile plus halo 1 live in shared
// memory; the median reads the mean.  Same arithmetic as k_mean/k_median.
template <bool MEAN, bool MEDIAN>
__global__ void __launch_bounds__(256) k_mean_median(PostViews pv, int W, int H) {
    constexpr int TXo = 32, TYo = 8, HX = TXo + 6, HY = TYo + 6, MX = TXo + 2, MY = TYo + 2;
    __shared__ float in[HY][HX];
    __shared__ float mn[MY][MX];
    const float* __restrict__ S = pv.cur[blockIdx.z];
    float* __restrict__ O = pv.nxt[blockIdx.z];
    const int u0 = blockIdx.x * TXo, v0 = blockIdx.y * TYo, tid = threadIdx.x;
    for (int i = tid; i < HY * HX; i += 256) {
        int r = i / HX, c = i % HX;
        int x = u0 - 3 + c, y = v0 - 3 + r;
        in[r][c] = (x >= 0 && x < W && y >= 0 && y < H) ? S[size_t(y) * W + x] : -2.0f;   // -2: outside
    }
    __syncthreads();
    for (int i = tid; i < MY * MX; i += 256) {
        int r = i / MX, c = i % MX;       // mean at (u0-1+c, v0-1+r) = in[r+2][c+2]
        float dp = in[r + 2][c + 2];
        float out = dp;
        if (MEAN && dp >= 0) {
            float num = 0.0f, den = 0.0f;
            for (int dy = -2; dy <= 2; ++dy)
                for (int dx = -2; dx <= 2; ++dx) {
                    float dq = in[r + 2 + dy][c + 2 + dx];
                    if (dq < 0) continue;      // invalid (-1) or outside (-2)
                    float diff = __fsub_rn(dq, dp);
                    float w = __fdiv_rn(1.0f, __fmaf_rn(diff, diff, 1.0f));
                    num = __fmaf_rn(w, dq, num);
                    den = __fadd_rn(den, w);
                }
            out = __fdiv_rn(num, den);
        }
        mn[r][c] = out;
    }
    __syncthreads();
    {
        int ty = tid / TXo, tx = tid % TXo;
        int u = u0 + tx, v = v0 + ty;
        if (u < W && v < H) {
            float c = mn[ty + 1][tx + 1];
            float out = c;
            if (MEDIAN && c >= 0) {
                float a[9];
                int n = 0;
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx) {
                        float q = mn[ty + 1 + dy][tx + 1 + dx];
                        if (q >= 0) a[n++] = q;
                    }
                for (int i = 1; i < n; ++i) {
                    float x = a[i];
                    int j = i - 1;
                    while (j >= 0 && a[j] > x) { a[j + 1] = a[j]; --j; }
                    a[j + 1] = x;
                }
                out = a[(n - 1) / 2];
            }
            O[size_t(v) * W + u] = out;
        }
    }
}

}  // namespace

cudaError_t launch_post(PostViews pv, int nviews, const Geom& g, const DevParams& p, bool median,
                        bool adaptive_mean, unsigned* err, cudaStream_t st, int* nlaunch) {
    const int W = g.W, H = g.H, n = W * H;
    const int tb = 256;
    int launched = 0;
    const dim3 grid2((W + tb - 1) / tb, H, nviews);
    auto flip = [&]() {
        for (int k = 0; k < 2; ++k) { float* t = pv.cur[k]; pv.cur[k] = pv.nxt[k]; pv.nxt[k] = t; }
    };
    if (p.speckle_size > 0) {
        const int wpb = 8;
        k_uf_init_rows<<<dim3((H + wpb - 1) / wpb, 1, nviews), 32 * wpb, 0, st>>>(pv, W, H, p.speckle_sim_threshold);
        k_uf_union_v<<<grid2, tb, 0, st>>>(pv, W, H, p.speckle_sim_threshold, err);
        k_uf_count_v<<<dim3((n + tb - 1) / tb, 1, nviews), tb, 0, st>>>(pv, n, err);
        k_uf_apply_v<<<dim3((n + tb - 1) / tb, 1, nviews), tb, 0, st>>>(pv, n, p.speckle_size);
        launched += 4;
    }
    if (p.ipol_gap_width > 0) {
        if (p.ipol_gap_width <= 64) {
            k_gap_px<<<grid2, tb, 0, st>>>(pv, W, H, p.ipol_gap_width, 1);
            flip();
            k_gap_px<<<grid2, tb, 0, st>>>(pv, W, H, p.ipol_gap_width, 0);
            flip();
        } else {
            k_gap<<<dim3((H + 127) / 128, 1, nviews), 128, 0, st>>>(pv, W, H, p.ipol_gap_width, 1);
            k_gap<<<dim3((W + 127) / 128, 1, nviews), 128, 0, st>>>(pv, W, H, p.ipol_gap_width, 0);
        }
        launched += 2;
    }
    if (adaptive_mean || median) {
        dim3 grid((W + 31) / 32, (H + 7) / 8, nviews);
        if (adaptive_mean && median) k_mean_median<true, true><<<grid, 256, 0, st>>>(pv, W, H);
        else if (adaptive_mean) k_mean_median<true, false><<<grid, 256, 0, st>>>(pv, W, H);
        else k_mean_median<false, true><<<grid, 256, 0, st>>>(pv, W, H);
        flip();
        launched += 1;
    }
    for (int k = 0; k < nviews; ++k)
        if (pv.cur[k] != pv.out[k])
            cudaMemcpyAsync(pv.out[k], pv.cur[k], size_t(n) * sizeof(float), cudaMemcpyDeviceToDevice, st);
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
// looked up once per device with cudaGetSymbolAddress (the first call on a
// device, which should therefore happen outside any stream capture) and
// cached.  Every call reuses the array; the kernels initialise all of it
// that must start at zero, and calls that overlap on the GPU race.
static __device__ __align__(256) int32_t g_noalloc_scratch[3 * ELAS_NOALLOC_MAX_PIXELS + 64];

namespace {
constexpr int kNoallocMaxDevices = 64;
int32_t* g_noalloc_base[kNoallocMaxDevices] = {};
std::mutex g_noalloc_mutex;
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
        if (!g_noalloc_base[dev]) {
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return ELAS_ERR_CUDA;
            g_noalloc_base[dev] = static_cast<int32_t*>(p);
        }
        base = g_noalloc_base[dev];
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int W = width, H = height, n = W * H, tb = 256;
    int32_t* lab = base;
    int32_t* root = base + ELAS_NOALLOC_MAX_PIXELS;
    int32_t* sz = base + 2 * ELAS_NOALLOC_MAX_PIXELS;
    unsigned* err = reinterpret_cast<unsigned*>(base + 3 * ELAS_NOALLOC_MAX_PIXELS);
    if (d_out != d_in &&
        cudaMemcpyAsync(d_out, d_in, size_t(n) * sizeof(float), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        return ELAS_ERR_CUDA;
    if (cudaMemsetAsync(err, 0, sizeof(unsigned), st) != cudaSuccess) return ELAS_ERR_CUDA;
    if (min_size > 0) {
        const dim3 grid2((W + tb - 1) / tb, H);
        k_uf_init<<<grid2, tb, 0, st>>>(d_out, lab, sz, W, H, sim_threshold);
        k_uf_union<<<grid2, tb, 0, st>>>(d_out, lab, W, H, sim_threshold, err);
        k_uf_count<<<(n + tb - 1) / tb, tb, 0, st>>>(lab, root, sz, n, err);
        k_uf_apply<<<(n + tb - 1) / tb, tb, 0, st>>>(d_out, root, sz, n, min_size);
    }
    return cudaGetLastError() == cudaSuccess ? ELAS_OK : ELAS_ERR_CUDA;
}

