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
};

HD int imin(int a, int b) { return a < b ? a : b; }
HD int imax(int a, int b) { return a > b ? a : b; }
HD int iabs_(int a) { return a < 0 ? -a : a; }

// floor(a / b) for b > 0, as floor((float)a / (float)b) in the reference
// (exact for |a| < 2^24).
HD int floordiv(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }

}  // namespace elas
