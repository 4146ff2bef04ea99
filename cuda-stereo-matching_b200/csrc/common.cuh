// Shared definitions of the ELAS B200 kernels.
#pragma once

#include <cstdint>
#include <cstddef>

#if defined(__CUDACC__)
#define HD __host__ __device__ __forceinline__
#else
#define HD inline
#endif

namespace elas {

// Geometry of one stereo pair, derived from the image size and the runtime
// parameters exactly as the reference host code does
// (src/Elas.cu:29-30 for the candidate lattice, :411-412 for the grid).
struct Geom {
    int W, H;          // image size
    int cw, ch;        // candidate lattice = W / step, H / step
    int gw, gh;        // grid cells = ceil(W / grid_size), ceil(H / grid_size)
    int D;             // disp_max
    int dmin;          // max(disp_min, 0): first disparity of the support sweep
    int step;          // candidate_stepsize
    int gs;            // grid_size
    int words;         // 32-bit words of one grid cell's disparity bitset
};

// Runtime parameters needed on the device, pre-digested on the host.
struct DevParams {
    float support_threshold;
    int support_texture;
    int lr_threshold;
    int incon_window;
    int incon_threshold;
    int incon_min_support;
    int match_texture;
    int plane_radius;       // (int)max(ceil(sigma*sradius), 2)   (KerComputeDisparity.cu:194)
    int penalty[16];        // P(|d - d_plane|) for |d - d_plane| <= plane_radius
    int window_negative;    // every penalty[0..plane_radius] is < 0
    float speckle_sim_threshold;
    int speckle_size;
    int ipol_gap_width;
};

// Device error flags (bit mask written with atomicOr).
enum : unsigned {
    ERRF_BOUNDS = 1u,       // an index read from memory was out of range
    ERRF_HASH = 2u,         // adjacency hash table overflow / non-manifold edge
    ERRF_FLIP_LIMIT = 4u,   // edge flipping did not converge within its round limit
    ERRF_TRI_COUNT = 8u,    // triangle count mismatch (Euler)
    ERRF_TMA_TIMEOUT = 16u, // a bulk copy did not complete within its bounded wait
};

#if defined(__CUDACC__)
// First statement of every kernel: wait until the preceding work of the
// stream has completed and its writes are visible (programmatic dependent
// launch; a no-op for a kernel launched without the attribute).  No kernel
// triggers its dependents early: measured on the B200, an explicit
// launch_dependents after the wait made the 1242x375 pipeline slower.
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Sum of absolute differences of two 16-byte descriptors: four
// vabsdiff4.u32.u32.u32.add (byte-wise |a-b| summed into the accumulator),
// the fastest of the packed-byte forms on sm_100a.
__device__ __forceinline__ int sad16(const uint4& a, const uint4& b, int acc = 0) {
    unsigned r = unsigned(acc);
    asm("vabsdiff4.u32.u32.u32.add %0, %1, %2, %0;" : "+r"(r) : "r"(a.x), "r"(b.x));
    asm("vabsdiff4.u32.u32.u32.add %0, %1, %2, %0;" : "+r"(r) : "r"(a.y), "r"(b.y));
    asm("vabsdiff4.u32.u32.u32.add %0, %1, %2, %0;" : "+r"(r) : "r"(a.z), "r"(b.z));
    asm("vabsdiff4.u32.u32.u32.add %0, %1, %2, %0;" : "+r"(r) : "r"(a.w), "r"(b.w));
    return int(r);
}

// sum over the 16 bytes of |b - 128| (the texture measure of the reference)
__device__ __forceinline__ int texture16(const uint4& a) {
    return sad16(a, make_uint4(0x80808080u, 0x80808080u, 0x80808080u, 0x80808080u));
}

// ---- bulk (TMA) copies global -> shared, completed on an mbarrier ----
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return uint32_t(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// One bulk copy of `bytes` (multiple of 16, both addresses 16-byte aligned).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
// Copy `bytes` in chunks of at most 32 KiB; call from one thread after
// mbar_expect_tx(bar, bytes).
__device__ __forceinline__ void bulk_g2s_chunked(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    const unsigned chunk = 32768;
    for (unsigned off = 0; off < bytes; off += chunk) {
        unsigned n = bytes - off < chunk ? bytes - off : chunk;
        bulk_g2s(static_cast<char*>(dst) + off, static_cast<const char*>(src) + off, n, bar);
    }
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait for phase `parity` of the barrier: false after `limit` polls.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity, int limit) {
    for (int i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
constexpr int MBAR_WAIT_LIMIT = 1 << 22;
#endif

HD int imin(int a, int b) { return a < b ? a : b; }
HD int imax(int a, int b) { return a > b ? a : b; }
HD int iabs_(int a) { return a < 0 ? -a : a; }

// floor(a / b) for b > 0, as floor((float)a / (float)b) in the reference
// (exact for |a| < 2^24).
HD int floordiv(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }

}  // namespace elas
