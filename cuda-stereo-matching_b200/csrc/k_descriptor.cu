// Fused Sobel + 16-byte descriptor.
//
// Replaces kerComputeSobel (src/Kernels/KerDescriptor.cu:8-50) and
// kerComputeDescriptor (src/Kernels/KerDescriptor.cu:52-101), which write
// the du/dv images to global memory and read them back with 16 scalar byte
// loads per pixel.  Here one CTA stages a 70x22 image tile in shared memory
// with 16-byte vector loads (each tile row is covered by the aligned 16-byte
// words around it; an aligned 16-byte word never crosses a page, so the
// bytes it carries beyond the row are harmless and ignored), computes du/dv
// for the 68x20 halo region there, four columns per thread, and writes the
// 64x16 descriptors, four per thread assembled by byte permutes and stored
// as 32-byte pixel pairs: global traffic is 1 byte read + 16 bytes written
// per pixel and both images run in one launch.  (128x16 tiles of 512
// threads measured slower.)
//
// Arithmetic: du = clamp((s >> 2) + 128, 0, 255) with s the integer Sobel
// sum; this equals the reference's float form
// (uint8_t)(min(max(-128.f, s/4), 127.f) + 128) for every reachable s
// (|s| <= 1020; checked exhaustively by the tests).  Border descriptors
// (u or v outside [3, size-4]) are written as zero; the reference leaves
// them uninitialised.
#include <cuda_runtime.h>
#include <cstdlib>
#include "common.cuh"
#include "launch.cuh"
#include "kernels.h"

namespace elas {

namespace {

constexpr int TX = 64, TY = 16;                // output tile
constexpr int IW = TX + 6, IH = TY + 6;        // image tile (halo 3)
constexpr int GW = TX + 4, GH = TY + 4;        // du/dv tile (halo 2)
constexpr int RW = 7;                          // 16-byte words staged per image tile row (70 + 15 bytes at most)
constexpr int IWP = 72;                        // image tile row in shared memory: IW rounded up to whole words
static_assert(TX * TY / 4 == 256 && GW % 4 == 0 && IWP % 4 == 0 && IWP >= IW, "descriptor tile layout");

// One 32-byte store (the address must be 32-byte aligned).
__device__ __forceinline__ void st_global_32b(uint4* p, const uint4& a, const uint4& b) {
    asm volatile("st.global.v8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(p), "r"(a.x), "r"(a.y), "r"(a.z),
                 "r"(a.w), "r"(b.x), "r"(b.y), "r"(b.z), "r"(b.w)
                 : "memory");
}

__device__ __forceinline__ int sobel_u8(int s) {
    int q = (s >> 2) + 128;
    return q < 0 ? 0 : (q > 255 ? 255 : q);
}

// VEC: both image bases are 16-byte aligned and rows are staged by 16-byte
// loads; otherwise by byte loads (caller buffers of any alignment).  Either
// way the staged bytes are then laid out as a zero-padded tile, so the
// Sobel pass reads shared memory with no bounds tests.
template <bool VEC>
__global__ void __launch_bounds__(256) k_descriptor(const uint8_t* __restrict__ img0,
                                                    const uint8_t* __restrict__ img1,
                                                    uint4* __restrict__ desc0,
                                                    uint4* __restrict__ desc1, int W, int H) {
    grid_dep_wait();
    __shared__ __align__(16) uint8_t raw[VEC ? IH : 1][RW * 16];   // staged words of each tile row
    __shared__ int roff[IH];                              // byte of image column u0 - 3 within raw[r]
    __shared__ __align__(4) uint8_t im[IH][IWP];          // the tile, 0 outside the image
    __shared__ __align__(4) uint8_t du[GH][GW];
    __shared__ __align__(4) uint8_t dv[GH][GW];
    const uint8_t* img = blockIdx.z ? img1 : img0;
    uint4* desc = blockIdx.z ? desc1 : desc0;
    const int u0 = blockIdx.x * TX, v0 = blockIdx.y * TY;
    const int tid = threadIdx.x;
    if (VEC) {
        const int ulo = imax(u0 - 3, 0), uhi = imin(u0 + TX + 3, W);   // image columns of the tile, [ulo, uhi)
        for (int i = tid; i < IH * RW; i += 256) {
            const int r = i / RW, k = i % RW;
            const int v = v0 - 3 + r;
            if (v < 0 || v >= H) continue;
            const size_t s = size_t(v) * W + ulo;
            const size_t a = s & ~size_t(15);                      // first aligned word of the row's bytes
            const size_t e = size_t(v) * W + uhi;
            if (k == 0) roff[r] = int(s - a) - (ulo - (u0 - 3));
            if (a + size_t(k) * 16 < e)
                reinterpret_cast<uint4*>(raw[r])[k] = *reinterpret_cast<const uint4*>(img + a + size_t(k) * 16);
        }
        __syncthreads();
    }
    // the zero-padded image tile, one 32-bit word (4 columns) per step: a
    // word inside the image is two aligned words of its staged row funnel-
    // shifted, a word across the image border is assembled byte by byte
    for (int i = tid; i < IH * (IWP / 4); i += 256) {
        const int r = i / (IWP / 4), c = (i - r * (IWP / 4)) * 4;
        const int u = u0 - 3 + c, v = v0 - 3 + r;
        uint32_t w = 0;
        if (v >= 0 && v < H) {
            if (VEC && u >= 0 && u + 3 < W) {
                const uint32_t* rw = reinterpret_cast<const uint32_t*>(raw[r]);
                const int o = c + roff[r];
                w = __funnelshift_r(rw[o >> 2], rw[(o + 3) >> 2], 8 * (o & 3));
            } else {
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    if (u + j >= 0 && u + j < W)
                        w |= uint32_t(VEC ? raw[r][c + j + roff[r]] : img[size_t(v) * W + u + j]) << (8 * j);
            }
        }
        *reinterpret_cast<uint32_t*>(&im[r][c]) = w;
    }
    __syncthreads();
    // du/dv of four neighbouring columns per step, from six image words:
    // du = column sums (1 2 1) differenced two columns apart, dv = row sums
    // (1 2 1) of the rows above and below differenced
    for (int i = tid; i < GH * (GW / 4); i += 256) {
        const int r = i / (GW / 4), c = (i - r * (GW / 4)) * 4;
        int a[3][6];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const uint32_t w0 = *reinterpret_cast<const uint32_t*>(&im[r + k][c]);
            const uint32_t w1 = *reinterpret_cast<const uint32_t*>(&im[r + k][c + 4]);
#pragma unroll
            for (int x = 0; x < 4; ++x) a[k][x] = int((w0 >> (8 * x)) & 0xffu);
            a[k][4] = int(w1 & 0xffu);
            a[k][5] = int((w1 >> 8) & 0xffu);
        }
        int cs[6];
#pragma unroll
        for (int x = 0; x < 6; ++x) cs[x] = a[0][x] + 2 * a[1][x] + a[2][x];
        uint32_t wu = 0, wv = 0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int sdu = cs[j] - cs[j + 2];
            const int sdv = (a[0][j] + 2 * a[0][j + 1] + a[0][j + 2]) - (a[2][j] + 2 * a[2][j + 1] + a[2][j + 2]);
            wu |= uint32_t(sobel_u8(sdu)) << (8 * j);
            wv |= uint32_t(sobel_u8(sdv)) << (8 * j);
        }
        *reinterpret_cast<uint32_t*>(&du[r][c]) = wu;
        *reinterpret_cast<uint32_t*>(&dv[r][c]) = wv;
    }
    __syncthreads();
    // four neighbouring descriptors per thread: the du/dv bytes at the
    // reference's offsets picked out of two words per tile row by byte
    // permutes (byte 2 + j + dx of the pair holds column dx of pixel j)
    {
        const int ty = tid / (TX / 4), q = tid - ty * (TX / 4);
        const int r = ty + 2, c = 4 * q;
        const int v = v0 + ty;
        uint32_t U0[5], U1[5], V0[3], V1[3];
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            U0[k] = *reinterpret_cast<const uint32_t*>(&du[r - 2 + k][c]);
            U1[k] = *reinterpret_cast<const uint32_t*>(&du[r - 2 + k][c + 4]);
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            V0[k] = *reinterpret_cast<const uint32_t*>(&dv[r - 1 + k][c]);
            V1[k] = *reinterpret_cast<const uint32_t*>(&dv[r - 1 + k][c + 4]);
        }
        uint4 o[4];
        bool ok[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int u = u0 + 4 * q + j;
            ok[j] = u < W && v < H;
            o[j] = make_uint4(0, 0, 0, 0);
            if (u > 2 && u < W - 3 && v > 2 && v < H - 3) {
                // selector nibbles index the 8 bytes (hi:lo) = (w1:w0) of a row
                auto sel = [](int b0, int b1, int b2, int b3) { return unsigned(b0 | b1 << 4 | b2 << 8 | b3 << 12); };
                // the word of a row holding pair byte b
                auto wd = [&](const uint32_t* X0, const uint32_t* X1, int k, int b) { return b < 4 ? X0[k] : X1[k]; };
                // x: DU(0,-2) | DU(-2,-1) << 8 | DU(0,-1) << 16 | DU(2,-1) << 24
                const uint32_t x1 = __byte_perm(U0[1], U1[1], sel(0, j, j + 2, j + 4));
                o[j].x = __byte_perm(x1, wd(U0, U1, 0, j + 2), sel(4 + ((j + 2) & 3), 1, 2, 3));
                // y: DU(-1,0) | DU(0,0) << 8 | DU(0,0) << 16 | DU(1,0) << 24
                o[j].y = __byte_perm(U0[2], U1[2], sel(j + 1, j + 2, j + 2, j + 3));
                // z: DU(-2,1) | DU(0,1) << 8 | DU(2,1) << 16 | DU(0,2) << 24
                const uint32_t z1 = __byte_perm(U0[3], U1[3], sel(j, j + 2, j + 4, 0));
                o[j].z = __byte_perm(z1, wd(U0, U1, 4, j + 2), sel(0, 1, 2, 4 + ((j + 2) & 3)));
                // w: DV(0,-1) | DV(-1,0) << 8 | DV(1,0) << 16 | DV(0,1) << 24
                const uint32_t w1 = __byte_perm(V0[1], V1[1], sel(0, j + 1, j + 3, 0));
                const uint32_t w2 = __byte_perm(wd(V0, V1, 0, j + 2), wd(V0, V1, 2, j + 2),
                                                sel((j + 2) & 3, 0, 0, 4 + ((j + 2) & 3)));
                o[j].w = __byte_perm(w1, w2, sel(4, 1, 2, 7));
            }
        }
        // 32-byte stores of pixel pairs that start on a 32-byte boundary (a
        // lane's 16-byte stores alone would fill each sector in two halves)
        if (v < H) {
            uint4* out = desc + size_t(v) * W + (u0 + 4 * q);
            auto pair = [&](int j) {
                if (ok[j] && ok[j + 1]) {
                    st_global_32b(out + j, o[j], o[j + 1]);
                } else if (ok[j]) {
                    out[j] = o[j];
                }
            };
            if ((reinterpret_cast<uintptr_t>(out) & 31) == 0) {
                pair(0);
                pair(2);
            } else {
                if (ok[0]) out[0] = o[0];
                pair(1);
                if (ok[3]) out[3] = o[3];
            }
        }
    }
}

}  // namespace

cudaError_t launch_descriptor(const uint8_t* img0, const uint8_t* img1, uint4* desc0, uint4* desc1,
                              int W, int H, cudaStream_t st) {
    dim3 grid((W + TX - 1) / TX, (H + TY - 1) / TY, 2);
    static const bool vec_on = [] {
        const char* e = std::getenv("ELAS_B200_DESC_VEC");
        return !(e && e[0] == '0');
    }();
    const bool vec = vec_on && ((reinterpret_cast<uintptr_t>(img0) | reinterpret_cast<uintptr_t>(img1)) & 15) == 0;
    if (vec) launch_k(k_descriptor<true>, grid, 256, 0, st, img0, img1, desc0, desc1, W, H);
    else launch_k(k_descriptor<false>, grid, 256, 0, st, img0, img1, desc0, desc1, W, H);
    return cudaGetLastError();
}

}  // namespace elas
