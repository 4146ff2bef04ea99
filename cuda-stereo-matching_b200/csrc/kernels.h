// Launchers of the ELAS B200 kernels (internal interface of the library).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include "common.cuh"

namespace elas {

// Device view of one triangulation problem (see delaunay_core.h).
struct DelDev {
    const int32_t* x;      // [Nmax] point x (u for the left view, u-d for the right)
    const int32_t* y;      // [Nmax] point y (v)
    int32_t* srt;          // [Nmax] per-row sorted unique point indices (at row_off offsets)
    int32_t* rcnt;         // [rows] unique points per row
    int32_t* ne;           // [rows] non-empty rows
    int32_t* soff;         // [rows] strip triangle offsets
    int32_t* chain;        // [14*rows] pocket walk scratch (2 sides) when it does not fit in shared memory
    int32_t* tri;          // [3*Tmax]
    int32_t* opp;          // [3*Tmax]
    uint32_t* txy;         // [3*Tmax] packed corner coordinates (global flip kernel)
    uint32_t* lock;        // [Tmax]
    int32_t* fround;       // [Tmax]
    int32_t* cand;         // [6*Tmax]
    int32_t* flips;        // [3*Tmax]
    int32_t* wl0;          // [6*Tmax]
    int32_t* wl1;          // [6*Tmax]
    int32_t* cwl;          // cluster kernel: per-CTA worklists  [16 * 2 * 6 * 4096]
    int32_t* ccand;        // cluster kernel: per-CTA proposals  [16 * 2 * 6 * 4096]
    int32_t* cflips;       // cluster kernel: per-CTA flips      [16 * 6 * 4096]
    int32_t* ctr;          // [16]: 0 triangles, 1 strip triangles, 4 flip rounds, 5 flips,
                           //       6 non-empty rows, 8 handled by the cluster kernel, 9 points,
                           //       11 star pool cursor, 12 star windows grown,
                           //       13 star searches over every point
    uint32_t* pxy;         // [Nmax] packed coordinates by point (PXY_NONE: dropped duplicate)
    uint32_t* sxy;         // [Nmax] packed coordinates beside srt
    int32_t* ne_y;         // [rows] y of each non-empty row
    int4* rinfo;           // [rows] non-empty row: y, first position in srt, unique points
    int32_t* tcnt;         // [Nmax] triangles owned by each point (star construction)
    int32_t* toff;         // [Nmax] their offsets in tri
    int32_t* sown;         // [24*Nmax] owned triangles' vertex pairs, per point
    int32_t* spool;        // [2*Tmax] pairs of points owning more than the slot holds
    int32_t* hnext;        // [Nmax] successor on the hull boundary (-1: interior point)
    int32_t* hprev;        // [Nmax] predecessor on the hull boundary
    int32_t* box;          // [8] x0, y0, x1, y1 of all points, [4] star window half-size
    int32_t* ylut;         // [H+2] y -> first non-empty row at or below y
    unsigned long long* hkey;  // [Hmax]
    int32_t* hcnt;         // [Hmax]
    int32_t* hval;         // [2*Hmax]
    int32_t* hslot;        // [3*Tmax]
    int Tmax;
    uint32_t Hmax;         // power of two
};

cudaError_t launch_descriptor(const uint8_t* img0, const uint8_t* img1, uint4* desc0, uint4* desc1,
                              int W, int H, cudaStream_t st);

// bins (nullable): packed learned search sets per candidate; then stats[0]
// counts candidates the proposal settled and stats[1] those that fell back
// to the full sweep.
// row_cnt (ch entries) receives the number of support points per lattice
// row, which launch_compact consumes.
cudaError_t launch_support(const uint4* desc0, const uint4* desc1, int32_t* can_lr, int32_t* can_tmp,
                           int32_t* can, int32_t* row_cnt, const Geom& g, const DevParams& p, int num_sms,
                           unsigned* err, cudaStream_t st, const uint32_t* bins = nullptr, int32_t* stats = nullptr);

cudaError_t launch_compact(const int32_t* can, const int32_t* row_cnt, int32_t* row_off, int32_t* uvd, int32_t* x0,
                           int32_t* x1, int32_t* y, const Geom& g, cudaStream_t st, int corners, int* nlaunch);

cudaError_t launch_grid(const int32_t* can, uint32_t* tmp0, uint32_t* tmp1, uint32_t* grid0, uint32_t* grid1,
                        const Geom& g, cudaStream_t st, int* nlaunch);

// Default: every point's star found directly (k_star).  flips: row strips
// and Lawson edge flips instead; then force_global flips every problem with
// the global-memory kernel (tests) and round_limit > 0 caps the flip rounds
// (ERRF_FLIP_LIMIT when hit).  Both give the same triangles (the unique
// triangulation under the perturbation), in different list orders.
cudaError_t launch_delaunay(DelDev& d0, DelDev& d1, const int32_t* row_off, int nrows, int nmax, int H, int num_sms,
                            int cluster_size, unsigned* err, cudaStream_t st, int* nlaunch, bool flips = false,
                            bool force_global = false, int round_limit = 0);
// Largest cluster (16 or 8 CTAs) with two co-resident copies for the flip
// kernel, or 0 if none fits.
int cluster_size_for_flip();

// Triangles binned by 64x32 prior tile, both views: a bin of PT_BIN
// entries per tile, the rest of a full bin's triangles in an overflow list.
constexpr int PT_BIN = 128;
struct PriorTiles {
    int32_t* cnt;      // [2][tiles + 1] triangles per tile; [tiles]: overflow pairs
    int32_t* bins;     // [2][tiles][PT_BIN] triangle indices
    int32_t* ovf;      // [2][ovf_cap][2] (tile, triangle) beyond full bins
    int ovf_cap;       // pairs per view (more raise ERRF_BOUNDS)
};
size_t prior_tile_count(const Geom& g);
size_t prior_overflow_capacity(const Geom& g, int Tmax);

// Plane prior of both views: prior[v*W+u] = (triangle+1) << pshift | d,
// d = d_plane clamped to [0, dcap] (dcap = disp_max + plane_radius + 1),
// 0 where no triangle covers the pixel.  Every pixel is written.
// rast: scratch of 2 * Tmax * raster_bytes() for the per-triangle set-up.
// tiled: paint tile by tile in shared memory (tl used) instead of with
// global atomics into the zeroed prior; the same bytes either way.
// zeroed: (direct paint) the caller has zeroed both priors already.
// bin_cap: (tiled paint) entries used of each tile's bin (tests lower it so
// that the overflow list is used).
cudaError_t launch_prior(const int32_t* tri0, const int32_t* tri1, const int32_t* ctr0, const int32_t* ctr1,
                         int Tmax, const int32_t* can, const int32_t* uvd, void* rast, const PriorTiles& tl,
                         uint32_t* prior0, uint32_t* prior1, const Geom& g, int pshift, int dcap, int num_sms,
                         unsigned* err, cudaStream_t st, int* nlaunch, bool tiled, bool zeroed = false,
                         int bin_cap = PT_BIN);
// Images from this many pixels up take the tiled prior paint (measured:
// the direct paint is faster at 1242x375, the tiled one at 2880x1988).
constexpr long long PRIOR_TILED_MIN_PIXELS = 1LL << 20;
// Images up to this many pixels take the star construction of the
// Delaunay triangulations, larger ones the strips and flips (measured: the
// stars are faster at 1242x375, the flips at 2880x1988).
constexpr long long DELAUNAY_STARS_MAX_PIXELS = 1LL << 21;
size_t raster_bytes();

size_t dense_smem_bytes(const Geom& g);
cudaError_t launch_dense(const uint4* desc0, const uint4* desc1, const uint32_t* prior0, const uint32_t* prior1,
                         const uint32_t* grid0, const uint32_t* grid1, float* disp0, float* disp1, const Geom& g,
                         const DevParams& p, int pshift, unsigned* err, cudaStream_t st, int threads, int sub = 0,
                         bool force_bitset = false);

// L/R check into o0/o1 and, where c0 is not null, also into c0/c1
cudaError_t launch_lr(const float* d0, const float* d1, float* o0, float* o1, float* c0, float* c1, const Geom& g,
                      int lr_threshold, cudaStream_t st, int sub);

// Buffers of the post-filter chain, per view: the filters ping-pong between
// cur and nxt (the chain starts in cur; the result is copied to out if it
// does not end there); lab/root/sz are union-find scratch (W*H int32 each),
// roots the list of tile-local roots (W*H + 1 int32).
struct PostViews {
    float* cur[2];
    float* nxt[2];
    float* out[2];
    int32_t* lab[2];
    int32_t* root[2];
    int32_t* sz[2];
    int32_t* roots[2];
};

// True when launch_post applies the speckle result while loading the fused
// tile filter instead of in a pass of its own; the filter chain then must
// not start in the output buffer (it never writes in place), so the caller
// starts it in pv.nxt.
bool post_fuses_speckle(const DevParams& p, bool median, bool adaptive_mean);

// Post-filters on nviews (1 or 2) disparity images.
cudaError_t launch_post(PostViews pv, int nviews, const Geom& g, const DevParams& p, bool median, bool adaptive_mean,
                        unsigned* err, cudaStream_t st, int* nlaunch, int num_sms);

}  // namespace elas
