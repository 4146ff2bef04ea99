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
__global__ void k_gap_px(const float* __restrict__ S, float* __restrict__ O, int W, int H, int gap, int horizontal) {
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
__global__ void k_gap(float* D, int W, int H, int gap, int horizontal) {
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

__global__ void k_mean(const float* __restrict__ S, float* __restrict__ D, int W, int H) {
    int u = blockIdx.x * blockDim.x + threadIdx.x, v = blockIdx.y;
    if (u >= W || v >= H) return;
    float dp = S[size_t(v) * W + u];
    float out = dp;
    if (dp >= 0) {
        float num = 0.0f, den = 0.0f;
        for (int dy = -2; dy <= 2; ++dy)
            for (int dx = -2; dx <= 2; ++dx) {
                int x = u + dx, y = v + dy;
                if (x < 0 || x >= W || y < 0 || y >= H) continue;
                float dq = S[size_t(y) * W + x];
                if (dq < 0) continue;
                float diff = __fsub_rn(dq, dp);
                float w = __fdiv_rn(1.0f, __fmaf_rn(diff, diff, 1.0f));
                num = __fmaf_rn(w, dq, num);
                den = __fadd_rn(den, w);
            }
        out = __fdiv_rn(num, den);
    }
    D[size_t(v) * W + u] = out;
}

__global__ void k_median(const float* __restrict__ S, float* __restrict__ D, int W, int H) {
    int u = blockIdx.x * blockDim.x + threadIdx.x, v = blockIdx.y;
    if (u >= W || v >= H) return;
    float c = S[size_t(v) * W + u];
    float out = c;
    if (c >= 0) {
        float a[9];
        int n = 0;
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
                int x = u + dx, y = v + dy;
                if (x < 0 || x >= W || y < 0 || y >= H) continue;
                float q = S[size_t(y) * W + x];
                if (q >= 0) a[n++] = q;
            }
        for (int i = 1; i < n; ++i) {   // insertion sort, n <= 9
            float x = a[i];
            int j = i - 1;
            while (j >= 0 && a[j] > x) { a[j + 1] = a[j]; --j; }
            a[j + 1] = x;
        }
        out = a[(n - 1) / 2];
    }
    D[size_t(v) * W + u] = out;
}

}  // namespace

cudaError_t launch_post(float* disp, float* tmp, int32_t* lab, int32_t* size, const Geom& g, const DevParams& p,
                        bool median, bool adaptive_mean, unsigned* err, cudaStream_t st, int* nlaunch) {
    const int W = g.W, H = g.H, n = W * H;
    const int tb = 256;
    int launched = 0;
    const dim3 grid2((W + tb - 1) / tb, H);
    if (p.speckle_size > 0) {
        k_uf_init<<<grid2, tb, 0, st>>>(disp, lab, size, W, H, p.speckle_sim_threshold);
        k_uf_union<<<grid2, tb, 0, st>>>(disp, lab, W, H, p.speckle_sim_threshold, err);
        int32_t* root = reinterpret_cast<int32_t*>(tmp);   // tmp is free during speckle removal
        k_uf_count<<<(n + tb - 1) / tb, tb, 0, st>>>(lab, root, size, n, err);
        k_uf_apply<<<(n + tb - 1) / tb, tb, 0, st>>>(disp, root, size, n, p.speckle_size);
        launched += 4;
    }
    if (p.ipol_gap_width > 0) {
        if (p.ipol_gap_width <= 64) {
            k_gap_px<<<grid2, tb, 0, st>>>(disp, tmp, W, H, p.ipol_gap_width, 1);
            k_gap_px<<<grid2, tb, 0, st>>>(tmp, disp, W, H, p.ipol_gap_width, 0);
        } else {
            k_gap<<<(H + 127) / 128, 128, 0, st>>>(disp, W, H, p.ipol_gap_width, 1);
            k_gap<<<(W + 127) / 128, 128, 0, st>>>(disp, W, H, p.ipol_gap_width, 0);
        }
        launched += 2;
    }
    if (adaptive_mean) {
        k_mean<<<dim3((W + tb - 1) / tb, H), tb, 0, st>>>(disp, tmp, W, H);
        cudaMemcpyAsync(disp, tmp, size_t(n) * sizeof(float), cudaMemcpyDeviceToDevice, st);
        launched += 1;
    }
    if (median) {
        k_median<<<dim3((W + tb - 1) / tb, H), tb, 0, st>>>(disp, tmp, W, H);
        cudaMemcpyAsync(disp, tmp, size_t(n) * sizeof(float), cudaMemcpyDeviceToDevice, st);
        launched += 1;
    }
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

