// Inference path of the learned proposal on the 5th-generation tensor cores.
//
// Convolution as implicit GEMM: a tile is M = 128 consecutive cells of one
// row of one image, N = 32 output channels, K = 9 taps x 32 input channels,
// issued as 18 tcgen05.mma (kind::f16, bf16 x bf16 -> fp32, K = 16 each) by
// one thread into a 128 x 32 fp32 accumulator in tensor memory.
//
// Operands in shared memory use the no-swizzle K-major layout: 8-row x
// 16-byte core matrices, rows 16 B apart, 8-row groups 128 B apart (SBO),
// K chunks of 8 channels one "plane" apart (LBO).  A tile's input is the
// 3 x 130-cell halo block, loaded by 12 TMA copies (3 rows x 4 channel
// chunks, box = 8 channels x 130 cells, out-of-range cells read as zero =
// the convolution's zero padding).  The operand of tap (dy, dx) is the same
// block seen from row dy+1, one 16-byte step per dx, so each activation
// crosses L2 -> shared memory once per tile instead of nine times.  The
// weights (B operand, [tap][chunk][co] 16-byte rows) are one bulk copy.
//
// Pipeline: a persistent CTA of 4 warps walks its tiles with STAGES halo
// buffers in flight; thread 0 issues the copies and the MMAs, all four
// warps read the accumulator back (tcgen05.ld, warp w owns TMEM lanes
// 32w..32w+31 = cells), add the bias, apply ReLU and store bf16 NHWC.
// Every wait is bounded; on a timeout the kernel records ERRF_TMA_TIMEOUT,
// drains what it issued (bounded), frees its tensor memory and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "launch.cuh"
#include "proposal.h"

namespace elas {
namespace pn {

namespace {

constexpr int TILE_M = 128;
constexpr int HALO = TILE_M + 2;                       // cells per halo row
constexpr int PLANE = 2176;                            // bytes per (row, chunk) plane: 130 x 16 B padded to 128
constexpr int STAGE_BYTES = 3 * 4 * PLANE;             // 26112
constexpr int STAGES = 3;
constexpr int W_TAP_BYTES = 4 * CH * 16;               // 2048: 4 chunk planes of 32 rows x 16 B
constexpr int W_BYTES = TAPS * W_TAP_BYTES;            // 18432
constexpr int TC_THREADS = 128;
constexpr size_t TC_SMEM = 1024 + size_t(W_BYTES) + size_t(STAGES) * STAGE_BYTES;
constexpr uint32_t TMEM_COLS = 32;

// Instruction descriptor, kind::f16: D fp32, A and B bf16, both K-major,
// N = 32, M = 128.
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(CH >> 3) << 17) | (uint32_t(TILE_M >> 4) << 24);

// Shared-memory matrix descriptor, no swizzle: start, LBO (K-chunk stride),
// SBO (8-row group stride), version 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return uint64_t((addr >> 4) & 0x3FFFu) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) |
           (uint64_t((sbo >> 4) & 0x3FFFu) << 32) | (uint64_t(1) << 46);
}

__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(IDESC), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Halo block of tile (img, y, x0) into stage buffer `buf`: rows y-1..y+1,
// cells x0-1 .. x0+128, channel chunks 0..3.
__device__ __forceinline__ void load_halo(uint8_t* buf, const CUtensorMap* map, int img, int y, int x0,
                                          uint64_t* bar) {
    mbar_expect_tx(bar, uint32_t(12 * HALO * 16));
    for (int r = 0; r < 3; ++r)
        for (int k = 0; k < 4; ++k) tma_load_4d(buf + (r * 4 + k) * PLANE, map, 8 * k, x0 - 1, y + r - 1, img, bar);
}

__global__ void __launch_bounds__(TC_THREADS, 1)
    k_conv_tc(const __grid_constant__ CUtensorMap in_map, const __nv_bfloat16* __restrict__ wts,
              const float* __restrict__ bias, __nv_bfloat16* __restrict__ out, int Hd, int Wd, int relu,
              unsigned* err) {
    // Launched with programmatic dependent launch: everything up to
    // grid_dep_wait() below (barriers, tensor memory, the weights and
    // biases, which no earlier kernel writes) overlaps the previous layer's
    // tail; the activations are read only after the wait.
    extern __shared__ uint8_t tc_raw[];
    __shared__ __align__(8) uint64_t full[STAGES];
    __shared__ __align__(8) uint64_t wbar, mbar;
    __shared__ uint32_t tmem_base;
    __shared__ float sbias[CH];
    uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(tc_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* wsm = sm;                         // W_BYTES
    uint8_t* stage0 = sm + W_BYTES;            // STAGES x STAGE_BYTES
    const int tid = threadIdx.x, warp = tid >> 5;
    const int xt = (Wd + TILE_M - 1) / TILE_M;
    const int tiles = 2 * Hd * xt;
    const int ntile = tiles > int(blockIdx.x) ? (tiles - int(blockIdx.x) + int(gridDim.x) - 1) / int(gridDim.x) : 0;
    if (tid < CH) sbias[tid] = bias[tid];
    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s) mbar_init(&full[s], 1);
        mbar_init(&wbar, 1);
        mbar_init(&mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = tmem_base;
    auto tile_coords = [&](int i, int& img, int& y, int& x0) {
        const int t = int(blockIdx.x) + i * int(gridDim.x);
        img = t / (Hd * xt);
        const int rem = t - img * Hd * xt;
        y = rem / xt;
        x0 = (rem - y * xt) * TILE_M;
    };
    if (tid == 0 && ntile > 0) {
        mbar_expect_tx(&wbar, uint32_t(W_BYTES));
        bulk_g2s_chunked(wsm, wts, uint32_t(W_BYTES), &wbar);
    }
    grid_dep_wait();
    if (tid == 0 && ntile > 0) {
        for (int i = 0; i < STAGES - 1 && i < ntile; ++i) {
            int img, y, x0;
            tile_coords(i, img, y, x0);
            load_halo(stage0 + i * STAGE_BYTES, &in_map, img, y, x0, &full[i]);
        }
    }
    int issued = ntile < STAGES - 1 ? ntile : STAGES - 1;   // tiles whose halo copy was issued
    bool ok = true;
    int mma_pending = 0, i_stop = 0;
    if (ntile > 0) ok = __syncthreads_and(mbar_wait_bounded(&wbar, 0, MBAR_WAIT_LIMIT));
    for (int i = 0; ok && i < ntile; ++i) {
        i_stop = i;
        const int s = i % STAGES;
        if (tid == 0 && issued < ntile) {      // its stage was freed by tile i-1's completed MMAs
            int img, y, x0;
            tile_coords(issued, img, y, x0);
            load_halo(stage0 + (issued % STAGES) * STAGE_BYTES, &in_map, img, y, x0, &full[issued % STAGES]);
        }
        if (issued < ntile) ++issued;
        ok = __syncthreads_and(mbar_wait_bounded(&full[s], uint32_t((i / STAGES) & 1), MBAR_WAIT_LIMIT));
        if (!ok) break;
        fence_after();
        if (tid == 0) {
            const uint32_t a0 = smem_u32(stage0 + s * STAGE_BYTES), b0 = smem_u32(wsm);
            for (int t = 0; t < TAPS; ++t) {
                const int dy = t / 3, dx = t % 3;
                for (int kk = 0; kk < 2; ++kk) {
                    const uint64_t ad = smem_desc(a0 + uint32_t((dy * 4 + 2 * kk) * PLANE + dx * 16), PLANE, 128);
                    const uint64_t bd = smem_desc(b0 + uint32_t(t * W_TAP_BYTES + 2 * kk * CH * 16), CH * 16, 128);
                    mma_bf16(tmem, ad, bd, (t | kk) != 0);
                }
            }
            mma_commit(&mbar);
        }
        mma_pending = 1;
        ok = __syncthreads_and(mbar_wait_bounded(&mbar, uint32_t(i & 1), MBAR_WAIT_LIMIT));
        if (!ok) break;
        mma_pending = 0;
        fence_after();
        {
            int img, y, x0;
            tile_coords(i, img, y, x0);
            uint32_t r[32];
            tmem_ld32(tmem + (uint32_t(warp * 32) << 16), r);
            const int x = x0 + tid;
            if (x < Wd) {
                __align__(16) __nv_bfloat16 o[CH];
#pragma unroll
                for (int c = 0; c < CH; ++c) {
                    float v = __uint_as_float(r[c]) + sbias[c];
                    o[c] = __float2bfloat16_rn(relu ? fmaxf(v, 0.0f) : v);
                }
                uint4* dst = reinterpret_cast<uint4*>(out + ((size_t(img) * Hd + y) * Wd + x) * CH);
                const uint4* src = reinterpret_cast<const uint4*>(o);
#pragma unroll
                for (int k = 0; k < 4; ++k) dst[k] = src[k];
            }
        }
        fence_before();
        __syncthreads();
    }
    if (!ok) {
        // record, then let what was issued land before the shared memory goes
        // away: the MMAs of tile i (if committed) and the halo copies of
        // tiles i .. issued-1
        if (tid == 0) atomicOr(err, ERRF_TMA_TIMEOUT);
        if (ntile > 0) mbar_wait_bounded(&wbar, 0, MBAR_WAIT_LIMIT);
        if (mma_pending) mbar_wait_bounded(&mbar, uint32_t(i_stop & 1), MBAR_WAIT_LIMIT);
        for (int j = i_stop; j < issued; ++j)
            mbar_wait_bounded(&full[j % STAGES], uint32_t((j / STAGES) & 1), MBAR_WAIT_LIMIT);
        fence_before();
        __syncthreads();
    }
    fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
}

// Top-4 bins per candidate: one warp per candidate, lane l scores bins l and
// l + 32 from the bf16 features (fp32 dot products).
__global__ void k_topk(const __nv_bfloat16* __restrict__ F, uint32_t* __restrict__ bins, int Hd, int Wd, int cw,
                       int ch, int step, int D) {
    grid_dep_wait();
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= cw * ch) return;
    const int u = (warp % cw) * step, v = (warp / cw) * step;
    const int cx = min(u / 4, Wd - 1), cy = min(v / 4, Hd - 1);
    const int w = bin_width(D);
    const __nv_bfloat16* fl = F + ((size_t(0) * Hd + cy) * Wd + cx) * CH;
    const __nv_bfloat16* frow = F + ((size_t(1) * Hd + cy) * Wd) * CH;
    float s[2];
    bool valid[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const int b = lane + 32 * k;
        const int x2 = cx - bin_shift(b, w);
        valid[k] = x2 >= 0;
        float acc = 0.0f;
        if (valid[k]) {
            const uint4* pl = reinterpret_cast<const uint4*>(fl);
            const uint4* pr = reinterpret_cast<const uint4*>(frow + size_t(x2) * CH);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                uint4 a = pl[q], c = pr[q];
                const __nv_bfloat162* a2 = reinterpret_cast<const __nv_bfloat162*>(&a);
                const __nv_bfloat162* c2 = reinterpret_cast<const __nv_bfloat162*>(&c);
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    float2 fa = __bfloat1622float2(a2[j]), fc = __bfloat1622float2(c2[j]);
                    acc = fmaf(fa.x, fc.x, acc);
                    acc = fmaf(fa.y, fc.y, acc);
                }
            }
        }
        s[k] = SCALE * acc;
    }
    uint32_t packed = 0xffffffffu;
    for (int r = 0; r < TOPK; ++r) {
        float best = -INFINITY;
        int bi = NBINS;
#pragma unroll
        for (int k = 0; k < 2; ++k)
            if (valid[k] && (s[k] > best || (s[k] == best && lane + 32 * k < bi))) { best = s[k]; bi = lane + 32 * k; }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const float ob = __shfl_xor_sync(0xffffffffu, best, o);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
        }
        if (bi >= NBINS) break;
        packed = (packed & ~(0xffu << (8 * r))) | (uint32_t(bi) << (8 * r));
        if ((bi & 31) == lane) {
            if (bi >= 32) valid[1] = false;
            else valid[0] = false;
        }
    }
    if (lane == 0) bins[warp] = packed;
}

// Top-4 bins with the right view's feature row in shared memory: one CTA
// per candidate row, one thread per candidate.  A thread keeps its left
// cell's 32 features in registers, walks the 64 bins in ascending order and
// keeps the four best (score descending, lower bin first on ties) -- the
// same order k_topk's repeated warp maximum yields.  Scores are the same
// fp32 FMA chain over channels 0..31.  The row is stored with the four
// 16-byte chunks of cell x rotated by (x >> 1) & 3, which spreads the
// chunks that neighbouring candidates read over distinct banks.
__device__ __forceinline__ int topk_slot(int x, int q) { return 4 * x + (q ^ ((x >> 1) & 3)); }

__global__ void __launch_bounds__(256) k_topk_rows(const __nv_bfloat16* __restrict__ F, uint32_t* __restrict__ bins,
                                                   int Hd, int Wd, int cw, int step, int D) {
    grid_dep_wait();
    extern __shared__ __align__(16) uint4 frow[];
    const int vc = blockIdx.x;
    const int v = vc * step;
    const int cy = min(v / 4, Hd - 1);
    const uint4* src = reinterpret_cast<const uint4*>(F + ((size_t(1) * Hd + cy) * Wd) * CH);
    for (int i = threadIdx.x; i < 4 * Wd; i += blockDim.x) frow[topk_slot(i >> 2, i & 3)] = src[i];
    __syncthreads();
    const int w = bin_width(D);
    const uint4* lrow = reinterpret_cast<const uint4*>(F + ((size_t(0) * Hd + cy) * Wd) * CH);
    for (int ci = threadIdx.x; ci < cw; ci += blockDim.x) {
        const int cx = min((ci * step) / 4, Wd - 1);
        float fl[CH];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            uint4 a = lrow[size_t(cx) * 4 + q];
            const __nv_bfloat162* a2 = reinterpret_cast<const __nv_bfloat162*>(&a);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                float2 f = __bfloat1622float2(a2[j]);
                fl[8 * q + 2 * j] = f.x;
                fl[8 * q + 2 * j + 1] = f.y;
            }
        }
        float ts[TOPK];
        int tb[TOPK];
#pragma unroll
        for (int r = 0; r < TOPK; ++r) { ts[r] = -INFINITY; tb[r] = int(NO_BIN); }
        for (int b = 0; b < NBINS; ++b) {
            const int x2 = cx - bin_shift(b, w);
            if (x2 < 0) break;            // the shift grows with b
            float acc = 0.0f;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                uint4 c = frow[topk_slot(x2, q)];
                const __nv_bfloat162* c2 = reinterpret_cast<const __nv_bfloat162*>(&c);
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    float2 fc = __bfloat1622float2(c2[j]);
                    acc = fmaf(fl[8 * q + 2 * j], fc.x, acc);
                    acc = fmaf(fl[8 * q + 2 * j + 1], fc.y, acc);
                }
            }
            const float sc = SCALE * acc;
            if (tb[TOPK - 1] != int(NO_BIN) && !(sc > ts[TOPK - 1])) continue;
            // insert (sc, b) behind every kept entry with a score >= sc
#pragma unroll
            for (int r = TOPK - 1; r >= 0; --r) {
                const bool above = r > 0 && (tb[r - 1] == int(NO_BIN) || sc > ts[r - 1]);
                const bool here = tb[r] == int(NO_BIN) || sc > ts[r];
                if (here) {
                    if (above) { ts[r] = ts[r - 1]; tb[r] = tb[r - 1]; }
                    else { ts[r] = sc; tb[r] = b; }
                }
            }
        }
        uint32_t packed = 0;
#pragma unroll
        for (int r = 0; r < TOPK; ++r) packed |= uint32_t(tb[r] & 0xff) << (8 * r);
        bins[size_t(vc) * cw + ci] = packed;
    }
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against libcuda).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    return fn;
}

// Map over an [2][Hd][Wd][32] bf16 activation: dims (channel, x, y, image),
// box 8 channels x 130 cells x 1 x 1, no swizzle, zero fill out of range.
bool make_act_map(CUtensorMap* map, const __nv_bfloat16* base, int Hd, int Wd) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    const cuuint64_t dims[4] = {cuuint64_t(CH), cuuint64_t(Wd), cuuint64_t(Hd), 2};
    const cuuint64_t strides[3] = {cuuint64_t(CH) * 2, cuuint64_t(Wd) * CH * 2, cuuint64_t(Hd) * Wd * CH * 2};
    const cuuint32_t box[4] = {8, cuuint32_t(HALO), 1, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<__nv_bfloat16*>(base), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

// Training parameters (per layer W[tap][ci][co], b[co]) -> inference layout
// (per layer and tap, 4 chunk planes of [co][8 ci] bf16 rows, then biases).
cudaError_t upload_weights(const float* host_params, InferWeights& iw, cudaStream_t st) {
    std::vector<__nv_bfloat16> w(size_t(LAYERS) * TAPS * CH * CH);
    std::vector<float> b(size_t(LAYERS) * CH);
    for (int l = 0; l < LAYERS; ++l) {
        const float* p = host_params + size_t(l) * LAYER_PARAMS;
        for (int t = 0; t < TAPS; ++t)
            for (int ci = 0; ci < CH; ++ci)
                for (int co = 0; co < CH; ++co) {
                    const size_t dst = ((size_t(l) * TAPS + t) * 4 + ci / 8) * CH * 8 + size_t(co) * 8 + ci % 8;
                    w[dst] = __float2bfloat16_rn(p[(t * CH + ci) * CH + co]);
                }
        for (int co = 0; co < CH; ++co) b[size_t(l) * CH + co] = p[TAPS * CH * CH + co];
    }
    cudaError_t e = cudaMemcpyAsync(iw.w, w.data(), w.size() * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(iw.b, b.data(), b.size() * sizeof(float), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(st);   // the host staging vectors go out of scope
}

cudaError_t launch_infer(const InferWeights& iw, const __nv_bfloat16* in, __nv_bfloat16* act0, __nv_bfloat16* act1,
                         __nv_bfloat16* out, int Hd, int Wd, int num_sms, unsigned* err, cudaStream_t st) {
    if (Hd <= 0 || Wd <= 0) return cudaSuccess;
    const __nv_bfloat16* src[LAYERS] = {in, act0, act1, act0};
    __nv_bfloat16* dst[LAYERS] = {act0, act1, act0, out};
    const int tiles = 2 * Hd * ((Wd + TILE_M - 1) / TILE_M);
    cudaError_t e = allow_smem(k_conv_tc);
    if (e != cudaSuccess) return e;
    // persistent CTAs: as many per SM as shared memory allows (each holds its
    // own 32-column accumulator), so one CTA's epilogue overlaps another's MMAs
    int per_sm = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_conv_tc, TC_THREADS, TC_SMEM) != cudaSuccess ||
        per_sm < 1)
        per_sm = 1;
    const int grid = imax(1, imin(tiles, per_sm * num_sms));
    for (int l = 0; l < LAYERS; ++l) {
        CUtensorMap map;
        if (!make_act_map(&map, src[l], Hd, Wd)) return cudaErrorInvalidValue;
        e = launch_k(k_conv_tc, grid, TC_THREADS, TC_SMEM, st, map,
                     static_cast<const __nv_bfloat16*>(iw.w + size_t(l) * TAPS * CH * CH),
                     static_cast<const float*>(iw.b + size_t(l) * CH), dst[l], Hd, Wd, int(l < LAYERS - 1), err);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_topk(const __nv_bfloat16* F, uint32_t* bins, int Hd, int Wd, int cw, int ch, int step, int D,
                        cudaStream_t st) {
    const int n = cw * ch;
    if (n <= 0) return cudaSuccess;
    const size_t smem = size_t(Wd) * CH * sizeof(__nv_bfloat16);
    if (smem <= 200 * 1024) {
        cudaError_t e = allow_smem(k_topk_rows);
        if (e != cudaSuccess) return e;
        launch_k(k_topk_rows, ch, 256, smem, st, F, bins, Hd, Wd, cw, step, D);
    } else {
        launch_k(k_topk, (n * 32 + 255) / 256, 256, 0, st, F, bins, Hd, Wd, cw, ch, step, D);
    }
    return cudaGetLastError();
}

}  // namespace pn
}  // namespace elas
