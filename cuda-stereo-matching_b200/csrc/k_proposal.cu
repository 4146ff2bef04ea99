// Learned support-point proposal: feature pooling, the training kernels
// (fp32 forward / backward of the 4-layer 3x3 CNN, correlation loss, Adam)
// and the bf16 inference path (tcgen05 implicit-GEMM convolutions, top-4
// bins per candidate).  The reference has no learned component; the
// network, its parameter layout and the proposal rule are defined once, in
// the CPU oracle's module docstring, and restated here.
//
// Layouts.  Feature maps are NHWC: [image][Hd][Wd][32], image = 2*pair +
// view (0 left, 1 right).  Training parameters, per layer: W[tap][ci][co]
// (tap = 3*(dy+1) + (dx+1)) then b[co], fp32.  Inference weights: bf16
// B operands [layer][tap][co][ci] (K-major, 64-byte rows) plus fp32 bias.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cstdint>

#include "common.cuh"
#include "launch.cuh"
#include "proposal.h"

namespace elas {
namespace pn {

namespace {

// ---------------------------------------------------------------------------
// Pooled descriptor features: cell (x, y) of image v covers pixels
// [4x, 4x+4) x [4y, 4y+4).  Channel c < 16: (mean_c - 128) / 64; channel
// 16 + c: mean |byte_c - 128| / 64.  Both are exact in fp32 before the bf16
// rounding.
__global__ void k_features(const uint4* __restrict__ desc0, const uint4* __restrict__ desc1,
                           __nv_bfloat16* __restrict__ out, int W, int Hd, int Wd) {
    grid_dep_wait();
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y, v = blockIdx.z;
    if (x >= Wd) return;
    const uint4* D = v ? desc1 : desc0;
    int sum[16], dev[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) sum[c] = dev[c] = 0;
    for (int r = 0; r < 4; ++r)
        for (int q = 0; q < 4; ++q) {
            uint4 d = D[size_t(4 * y + r) * W + 4 * x + q];
            const uint32_t w4[4] = {d.x, d.y, d.z, d.w};
#pragma unroll
            for (int k = 0; k < 4; ++k)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    int b = int((w4[k] >> (8 * j)) & 0xffu);
                    sum[4 * k + j] += b;
                    dev[4 * k + j] += abs(b - 128);
                }
        }
    __align__(16) __nv_bfloat16 o[CH];
#pragma unroll
    for (int c = 0; c < 16; ++c) {
        o[c] = __float2bfloat16_rn((float(sum[c]) * 0.0625f - 128.0f) * 0.015625f);
        o[16 + c] = __float2bfloat16_rn(float(dev[c]) * (1.0f / 1024.0f));
    }
    uint4* dst = reinterpret_cast<uint4*>(out + ((size_t(v) * Hd + y) * Wd + x) * CH);
    const uint4* src = reinterpret_cast<const uint4*>(o);
#pragma unroll
    for (int k = 0; k < 4; ++k) dst[k] = src[k];
}

__global__ void k_bf16_to_f32(const __nv_bfloat16* __restrict__ in, float* __restrict__ out, size_t n) {
    grid_dep_wait();
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        out[i] = __bfloat162float(in[i]);
}

// ---------------------------------------------------------------------------
// Training convolution (fp32): one block = one image row segment of SEG
// cells x 32 output channels (lane = output channel, warp = cell).  The
// three input rows of the segment (with a one-cell halo) and all nine taps
// of weights sit in shared memory.  `mask` (nullable) multiplies each input
// value by (mask > 0): the ReLU derivative when this kernel computes the
// gradient of the layer input.
constexpr int SEG = 32;

constexpr size_t CONV_F32_SMEM = sizeof(float) * (TAPS * CH * CH + 3 * (SEG + 2) * CH);

__global__ void __launch_bounds__(SEG * CH) k_conv_f32(const float* __restrict__ x, const float* __restrict__ mask,
                                                   const float* __restrict__ w, const float* __restrict__ b,
                                                   float* __restrict__ y, int Hd, int Wd, int relu) {
    grid_dep_wait();
    extern __shared__ float conv_sm[];
    float* sw = conv_sm;                                                  // [TAPS*CH*CH]
    float(*sx)[SEG + 2][CH] = reinterpret_cast<float(*)[SEG + 2][CH]>(conv_sm + TAPS * CH * CH);
    const int n = blockIdx.z, row = blockIdx.y, x0 = blockIdx.x * SEG;
    const int co = threadIdx.x & 31, cell = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < TAPS * CH * CH; i += blockDim.x) sw[i] = w[i];
    for (int i = threadIdx.x; i < 3 * (SEG + 2) * CH; i += blockDim.x) {
        const int c = i % CH, j = (i / CH) % (SEG + 2), r = i / (CH * (SEG + 2));
        const int yy = row + r - 1, xx = x0 + j - 1;
        float v = 0.0f;
        if (yy >= 0 && yy < Hd && xx >= 0 && xx < Wd) {
            const size_t idx = ((size_t(n) * Hd + yy) * Wd + xx) * CH + c;
            v = x[idx];
            if (mask && !(mask[idx] > 0.0f)) v = 0.0f;
        }
        sx[r][j][c] = v;
    }
    __syncthreads();
    const int xo = x0 + cell;
    if (xo >= Wd) return;
    float acc = b ? b[co] : 0.0f;
#pragma unroll
    for (int t = 0; t < TAPS; ++t) {
        const int r = t / 3, j = cell + t % 3;
        const float* xs = sx[r][j];
        const float* ws = sw + t * CH * CH + co;
#pragma unroll 8
        for (int ci = 0; ci < CH; ++ci) acc = fmaf(xs[ci], ws[ci * CH], acc);
    }
    if (relu) acc = fmaxf(acc, 0.0f);
    y[((size_t(n) * Hd + row) * Wd + xo) * CH + co] = acc;
}

// Wt[8 - t][co][ci] = W[t][ci][co]: the gradient of a layer input is the
// same convolution of the output gradient with these weights.
__global__ void k_flip_weights(const float* __restrict__ w, float* __restrict__ wt) {
    grid_dep_wait();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= TAPS * CH * CH) return;
    const int t = i / (CH * CH), ci = (i / CH) % CH, co = i % CH;
    wt[((TAPS - 1 - t) * CH + co) * CH + ci] = w[i];
}

// Weight and bias gradients: dW[t][ci][co] += sum_cells x[cell + off_t][ci] * g[cell][co],
// db[co] += sum g[cell][co], with g = dy * (y > 0) when `y` is given.  One
// block accumulates a band of ROWS rows of one SEG-cell segment (thread =
// (ci, co)) and adds its partial sums atomically.
constexpr int WG_ROWS = 8;

__global__ void __launch_bounds__(CH * CH) k_conv_wgrad(const float* __restrict__ x, const float* __restrict__ dy,
                                                      const float* __restrict__ y, float* __restrict__ dw,
                                                      float* __restrict__ db, int Hd, int Wd) {
    grid_dep_wait();
    __shared__ float sx[3][SEG + 2][CH];
    __shared__ float sg[SEG][CH];
    const int n = blockIdx.z, x0 = blockIdx.x * SEG, r0 = blockIdx.y * WG_ROWS;
    const int co = threadIdx.x & 31, ci = threadIdx.x >> 5;
    float acc[TAPS];
#pragma unroll
    for (int t = 0; t < TAPS; ++t) acc[t] = 0.0f;
    float bacc = 0.0f;
    for (int row = r0; row < min(Hd, r0 + WG_ROWS); ++row) {
        __syncthreads();
        for (int i = threadIdx.x; i < 3 * (SEG + 2) * CH; i += blockDim.x) {
            const int c = i % CH, j = (i / CH) % (SEG + 2), r = i / (CH * (SEG + 2));
            const int yy = row + r - 1, xx = x0 + j - 1;
            sx[r][j][c] = (yy >= 0 && yy < Hd && xx >= 0 && xx < Wd) ? x[((size_t(n) * Hd + yy) * Wd + xx) * CH + c]
                                                                     : 0.0f;
        }
        for (int i = threadIdx.x; i < SEG * CH; i += blockDim.x) {
            const int c = i % CH, j = i / CH, xx = x0 + j;
            float g = 0.0f;
            if (xx < Wd) {
                const size_t idx = ((size_t(n) * Hd + row) * Wd + xx) * CH + c;
                g = dy[idx];
                if (y && !(y[idx] > 0.0f)) g = 0.0f;
            }
            sg[j][c] = g;
        }
        __syncthreads();
        for (int j = 0; j < SEG; ++j) {
            const float g = sg[j][co];
#pragma unroll
            for (int t = 0; t < TAPS; ++t) acc[t] = fmaf(sx[t / 3][j + t % 3][ci], g, acc[t]);
            if (ci == 0) bacc += g;
        }
    }
#pragma unroll
    for (int t = 0; t < TAPS; ++t) atomicAdd(&dw[(t * CH + ci) * CH + co], acc[t]);
    if (ci == 0) atomicAdd(&db[co], bacc);
}

// Correlation scores, softmax cross-entropy and the feature gradients, one
// warp per label (pair, cx, cy, bin).  Lane l owns bins l and l + 32.
__global__ void k_corr_loss(const float* __restrict__ F, const int32_t* __restrict__ labels, int nlab, int Hd,
                            int Wd, int D, float inv_n, float* __restrict__ dF, float* __restrict__ loss_sum,
                            int32_t* __restrict__ correct) {
    grid_dep_wait();
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= nlab) return;
    const int pair = labels[4 * warp], cx = labels[4 * warp + 1], cy = labels[4 * warp + 2],
              tb = labels[4 * warp + 3];
    const int w = bin_width(D);
    const size_t Lrow = ((size_t(2 * pair) * Hd + cy) * Wd) * CH;
    const size_t Rrow = ((size_t(2 * pair + 1) * Hd + cy) * Wd) * CH;
    const float fl = F[Lrow + size_t(cx) * CH + lane];     // lane = channel
    float s[2];
    bool valid[2];
    int xr[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const int b = lane + 32 * k;
        xr[k] = cx - bin_shift(b, w);
        valid[k] = xr[k] >= 0;
        s[k] = 0.0f;
    }
    // dot products: for every bin, a warp reduction over channels
    for (int b = 0; b < NBINS; ++b) {
        const int x2 = cx - bin_shift(b, w);
        float p = x2 >= 0 ? fl * F[Rrow + size_t(x2) * CH + lane] : 0.0f;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) p += __shfl_xor_sync(0xffffffffu, p, o);
        if ((b & 31) == lane) {
            if (b >= 32) s[1] = SCALE * p;
            else s[0] = SCALE * p;
        }
    }
    float m = -INFINITY;
#pragma unroll
    for (int k = 0; k < 2; ++k) if (valid[k]) m = fmaxf(m, s[k]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    const bool tvalid = cx - bin_shift(tb, w) >= 0;
    if (!tvalid) return;                                   // the oracle skips these labels
    float e[2], z = 0.0f;
#pragma unroll
    for (int k = 0; k < 2; ++k) { e[k] = valid[k] ? expf(s[k] - m) : 0.0f; z += e[k]; }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) z += __shfl_xor_sync(0xffffffffu, z, o);
    // argmax (lowest bin on ties) for the accuracy count
    float best = -INFINITY;
    int bi = NBINS;
#pragma unroll
    for (int k = 0; k < 2; ++k)
        if (valid[k] && (s[k] > best)) { best = s[k]; bi = lane + 32 * k; }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        float ob = __shfl_xor_sync(0xffffffffu, best, o);
        int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
    }
    float st = __shfl_sync(0xffffffffu, tb >= 32 ? s[1] : s[0], tb & 31);
    if (lane == 0) {
        atomicAdd(loss_sum, -(st - m - logf(z)));
        if (bi == tb) atomicAdd(correct, 1);
    }
    float g[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const int b = lane + 32 * k;
        g[k] = valid[k] ? (e[k] / z - (b == tb ? 1.0f : 0.0f)) * inv_n * SCALE : 0.0f;
    }
    // dF_L[c] = sum_b g_b F_R(x - s_b)[c];  dF_R(x - s_b)[c] += g_b F_L[c]
    float dl = 0.0f;
    for (int b = 0; b < NBINS; ++b) {
        const float gb = __shfl_sync(0xffffffffu, b >= 32 ? g[1] : g[0], b & 31);
        const int x2 = cx - bin_shift(b, w);
        if (x2 < 0 || gb == 0.0f) continue;
        dl = fmaf(gb, F[Rrow + size_t(x2) * CH + lane], dl);
        atomicAdd(&dF[Rrow + size_t(x2) * CH + lane], gb * fl);
    }
    atomicAdd(&dF[Lrow + size_t(cx) * CH + lane], dl);
}

__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, int n, float lr, float b1, float b2, float eps, float c1, float c2) {
    grid_dep_wait();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

}  // namespace

cudaError_t launch_features(const uint4* desc0, const uint4* desc1, __nv_bfloat16* out, int W, int H,
                            cudaStream_t st) {
    const int Hd = H / 4, Wd = W / 4;
    if (Hd <= 0 || Wd <= 0) return cudaSuccess;
    launch_k(k_features, dim3((Wd + 63) / 64, Hd, 2), 64, 0, st, desc0, desc1, out, W, Hd, Wd);
    return cudaGetLastError();
}

cudaError_t launch_bf16_to_f32(const __nv_bfloat16* in, float* out, size_t n, cudaStream_t st) {
    k_bf16_to_f32<<<1024, 256, 0, st>>>(in, out, n);
    return cudaGetLastError();
}

cudaError_t launch_conv_f32(const float* x, const float* mask, const float* w, const float* b, float* y, int nimg,
                            int Hd, int Wd, int relu, cudaStream_t st) {
    allow_smem(k_conv_f32);
    k_conv_f32<<<dim3((Wd + SEG - 1) / SEG, Hd, nimg), SEG * CH, CONV_F32_SMEM, st>>>(x, mask, w, b, y, Hd, Wd,
                                                                                       relu);
    return cudaGetLastError();
}

cudaError_t launch_flip_weights(const float* w, float* wt, cudaStream_t st) {
    k_flip_weights<<<(TAPS * CH * CH + 255) / 256, 256, 0, st>>>(w, wt);
    return cudaGetLastError();
}

cudaError_t launch_conv_wgrad(const float* x, const float* dy, const float* y, float* dw, float* db, int nimg,
                              int Hd, int Wd, cudaStream_t st) {
    k_conv_wgrad<<<dim3((Wd + SEG - 1) / SEG, (Hd + WG_ROWS - 1) / WG_ROWS, nimg), CH * CH, 0, st>>>(x, dy, y, dw, db,
                                                                                                   Hd, Wd);
    return cudaGetLastError();
}

cudaError_t launch_corr_loss(const float* F, const int32_t* labels, int nlab, int Hd, int Wd, int D, float* dF,
                             float* loss_sum, int32_t* correct, cudaStream_t st) {
    if (nlab <= 0) return cudaSuccess;
    k_corr_loss<<<(nlab * 32 + 255) / 256, 256, 0, st>>>(F, labels, nlab, Hd, Wd, D, 1.0f / float(nlab), dF,
                                                         loss_sum, correct);
    return cudaGetLastError();
}

cudaError_t launch_adam(float* p, const float* g, float* m, float* v, int n, float lr, float b1, float b2, float eps,
                        int t, cudaStream_t st) {
    const float c1 = 1.0f - powf(b1, float(t)), c2 = 1.0f - powf(b2, float(t));
    k_adam<<<(n + 255) / 256, 256, 0, st>>>(p, g, m, v, n, lr, b1, b2, eps, c1, c2);
    return cudaGetLastError();
}

}  // namespace pn
}  // namespace elas
