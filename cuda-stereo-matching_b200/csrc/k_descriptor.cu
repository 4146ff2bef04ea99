// Fused Sobel + 16-byte descriptor.
//
// Replaces kerComputeSobel (src/Kernels/KerDescriptor.cu:8-50) and
// kerComputeDescriptor (src/Kernels/KerDescriptor.cu:52-101), which write
// the du/dv images to global memory and read them back with 16 scalar byte
// loads per pixel.  Here one CTA stages a 70x22 image tile in shared memory
// with 16-byte vector loads (each tile row is covered by the aligned 16-byte
// words around it; an aligned 16-byte word never crosses a page, so the
// bytes it carries beyond the row are harmless and ignored), computes du/dv
// for the 68x20 halo region there and writes the 64x16 descriptors as
// coalesced 16-byte stores: global traffic is 1 byte read + 16 bytes
// written per pixel and both images run in one launch.
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
    __shared__ uint8_t im[IH][IW + 2];                    // the tile, 0 outside the image
    __shared__ uint8_t du[GH][GW];
    __shared__ uint8_t dv[GH][GW];
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
    for (int i = tid; i < IH * IW; i += 256) {
        const int r = i / IW, c = i % IW;
        const int u = u0 - 3 + c, v = v0 - 3 + r;
        uint8_t b = 0;
        if (u >= 0 && u < W && v >= 0 && v < H) b = VEC ? raw[r][c + roff[r]] : img[size_t(v) * W + u];
        im[r][c] = b;
    }
    __syncthreads();
    for (int i = tid; i < GH * GW; i += 256) {
        int r = i / GW, c = i % GW;
        // image tile coordinates of (u, v) = (c + 1, r + 1)
        int a00 = im[r][c], a01 = im[r][c + 1], a02 = im[r][c + 2];
        int a10 = im[r + 1][c], a12 = im[r + 1][c + 2];
        int a20 = im[r + 2][c], a21 = im[r + 2][c + 1], a22 = im[r + 2][c + 2];
        int sdu = a00 + 2 * a10 + a20 - a02 - 2 * a12 - a22;
        int sdv = a00 + 2 * a01 + a02 - a20 - 2 * a21 - a22;
        du[r][c] = uint8_t(sobel_u8(sdu));
        dv[r][c] = uint8_t(sobel_u8(sdv));
    }
    __syncthreads();
    for (int i = tid; i < TX * TY; i += 256) {
        int ty = i / TX, tx = i % TX;
        int u = u0 + tx, v = v0 + ty;
        if (u >= W || v >= H) continue;
        uint4 o = make_uint4(0, 0, 0, 0);
        if (u > 2 && u < W - 3 && v > 2 && v < H - 3) {
            int r = ty + 2, c = tx + 2;   // du/dv tile coordinates of (u, v)
            auto DU = [&](int dx, int dy) { return uint32_t(du[r + dy][c + dx]); };
            auto DV = [&](int dx, int dy) { return uint32_t(dv[r + dy][c + dx]); };
            o.x = DU(0, -2) | DU(-2, -1) << 8 | DU(0, -1) << 16 | DU(2, -1) << 24;
            o.y = DU(-1, 0) | DU(0, 0) << 8 | DU(0, 0) << 16 | DU(1, 0) << 24;
            o.z = DU(-2, 1) | DU(0, 1) << 8 | DU(2, 1) << 16 | DU(0, 2) << 24;
            o.w = DV(0, -1) | DV(-1, 0) << 8 | DV(1, 0) << 16 | DV(0, 1) << 24;
        }
        desc[size_t(v) * W + u] = o;
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
