// Plane prior, dense matching and the left/right check.
//
// Prior: replaces kerComputeDepthApproximation
// (src/Kernels/KerComputeDisparity.cu:9-152), one thread per triangle with
// long serial scanline loops.  Here one thread per triangle solves the plane
// (same double Gauss-Jordan as kerSolve, :321-375) and sets up the edges.
// Two ways to paint, chosen by image size (both give the same bytes):
//   * direct: a warp per triangle, lanes over its pixels, atomics straight
//     into the zeroed prior (one launch after the memset, each warp setting
//     its triangle up itself; the faster one for small images);
//   * tiled: the set-up also finds the 64x32 prior tiles a triangle's pixels
//     can fall in and drops the triangle into each tile's fixed bin (the
//     slot its count's atomic returns; no scan), and one CTA per tile paints
//     it in shared memory and writes it once (no memset, no global atomics
//     on the prior; the faster one from about a megapixel up).
// A pixel covered by more than one triangle (rounding at shared vertices)
// must keep the last triangle in list order, as a sequential rasteriser
// would; both paint with a 32-bit atomicMax of (triangle+1) << pshift |
// d_plane, which makes the result independent of scheduling.  d_plane is stored clamped to
// [0, disp_max + plane_radius + 1] (0 standing for every d_plane <= 0): the
// dense step treats all values beyond either end alike.
//
// Floating point follows the reference expressions with the contraction
// nvcc applies to them made explicit (fma where a*b+c occurs); the CPU
// oracle evaluates the identical operation sequence.
//
// Dense: replaces kerComputeDisparity (KerComputeDisparity.cu:155-316).
// One CTA per image row and view; the other view's descriptor row is
// staged in shared memory; the candidate list of the pixel's grid cell is a
// bitset walked in ascending order (the reference's sorted int list),
// skipping the plane window, then the plane window with the penalty added.
// Strict '<' keeps the first minimum in that order, as the reference does.
#include <cuda_runtime.h>
#include "common.cuh"
#include "launch.cuh"
#include "kernels.h"

namespace elas {

namespace {

// kerSolve with the row update written as fma(-y, dum, x).  The pivot row
// and column are data-dependent; every access to A and B goes through
// compile-time indices and selects, so the system stays in registers (an
// indexed 3x3 array would live in local memory).  The arithmetic and its
// order are kerSolve's: the pivot row is scaled after its pivot is set to
// 1, and the other rows are updated column by column with the pivot
// column's entry zeroed first.
template <int N, typename T>
__device__ __forceinline__ T pick(const T (&v)[N], int i) {
    T r = v[0];
#pragma unroll
    for (int k = 1; k < N; ++k) r = i == k ? v[k] : r;
    return r;
}
__device__ __forceinline__ bool solve3(double (&A)[3][3], double (&B)[3]) {
    const double eps = 1e-20;
    int ipiv[3] = {0, 0, 0};
    int irow = 0, icol = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        double big = 0.0;
#pragma unroll
        for (int j = 0; j < 3; ++j)
            if (ipiv[j] != 1)
#pragma unroll
                for (int k = 0; k < 3; ++k)
                    if (ipiv[k] == 0)
                        if (fabs(A[j][k]) >= big) { big = fabs(A[j][k]); irow = j; icol = k; }
#pragma unroll
        for (int k = 0; k < 3; ++k) ipiv[k] += k == icol;
        // swap rows irow and icol (a no-op when they are equal)
#pragma unroll
        for (int l = 0; l < 3; ++l) {
            const double col[3] = {A[0][l], A[1][l], A[2][l]};
            const double ar = pick(col, irow), ac = pick(col, icol);
#pragma unroll
            for (int r = 0; r < 3; ++r) A[r][l] = r == irow ? ac : (r == icol ? ar : A[r][l]);
        }
        {
            const double br = pick(B, irow), bc = pick(B, icol);
#pragma unroll
            for (int r = 0; r < 3; ++r) B[r] = r == irow ? bc : (r == icol ? br : B[r]);
        }
        double prow[3];
#pragma unroll
        for (int l = 0; l < 3; ++l) {
            const double col[3] = {A[0][l], A[1][l], A[2][l]};
            prow[l] = pick(col, icol);
        }
        const double piv = pick(prow, icol);
        if (fabs(piv) < eps) return false;
        const double pivinv = __ddiv_rn(1.0, piv);
#pragma unroll
        for (int l = 0; l < 3; ++l) prow[l] = __dmul_rn(l == icol ? 1.0 : prow[l], pivinv);
        const double bp = __dmul_rn(pick(B, icol), pivinv);
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            if (r == icol) {
#pragma unroll
                for (int l = 0; l < 3; ++l) A[r][l] = prow[l];
                B[r] = bp;
            } else {
                const double dum = pick(A[r], icol);
#pragma unroll
                for (int l = 0; l < 3; ++l) A[r][l] = __fma_rn(-prow[l], dum, l == icol ? 0.0 : A[r][l]);
                B[r] = __fma_rn(-bp, dum, B[r]);
            }
        }
    }
    return true;
}

struct Raster {
    float pa, pb, pc;
    float A_u, B_u, C_u;
    float AB_a, AC_a, BC_a, AB_b, AC_b, BC_b;
    int tx0, tx1, ty0, ty1;     // prior tiles its pixels can fall in (tx0 > tx1: none)
};

// Prior tiles: each is painted by one CTA in shared memory and written once.
constexpr int PT_W = 64, PT_H = 32;

// Rows of one part of the scan-line raster: columns u in [ua, ub) write the
// rows [va, vb) with va = max(min(v1, v2), 0), vb = min(max(v1, v2), H),
// v1 from the long edge AC and v2 from the part's edge.  Each of v1, v2 is
// a truncated fma of u, monotone in u, so the extremes over the part are at
// its first and last column.
__device__ __forceinline__ int raster_row(float a, float b, int u) {
    return int(__float2uint_rz(__fmaf_rn(a, float(u), b)));
}
__device__ void part_rows(const Raster& R, int part, int W, int H, int& r0, int& r1) {
    const int ua = part ? int(R.B_u) : int(R.A_u), ub = part ? int(R.C_u) : int(R.B_u);
    const int u0 = imax(ua, 0), u1 = imin(ub, W) - 1;
    if (ua == ub || u0 > u1) return;
    const float ea = part ? R.BC_a : R.AB_a, eb = part ? R.BC_b : R.AB_b;
    const int a0 = raster_row(R.AC_a, R.AC_b, u0), a1 = raster_row(R.AC_a, R.AC_b, u1);
    const int b0 = raster_row(ea, eb, u0), b1 = raster_row(ea, eb, u1);
    const int lo = imax(imin(imin(a0, a1), imin(b0, b1)), 0);
    const int hi = imin(imax(imax(a0, a1), imax(b0, b1)), H) - 1;
    if (lo > hi) return;
    r0 = imin(r0, lo);
    r1 = imax(r1, hi);
}

__device__ void setup_triangle(const int32_t* tri, const int32_t* can, const int32_t* uvd, int cw, int step,
                               bool right, Raster& R) {
    int tu[3], tv[3], td[3];
    for (int k = 0; k < 3; ++k) {
        int c = tri[k];
        tu[k] = uvd[3 * c];
        tv[k] = uvd[3 * c + 1];
        // the point's own disparity: for a lattice point the value the
        // reference reads at can[(v * cw + u) / step]; corner points
        // (add_corners) have no lattice cell
        td[k] = uvd[3 * c + 2];
    }
    double A[3][3], B[3];
    for (int k = 0; k < 3; ++k) {
        A[k][0] = right ? double(tu[k] - td[k]) : double(tu[k]);
        A[k][1] = double(tv[k]);
        A[k][2] = 1.0;
        B[k] = double(td[k]);
    }
    R.pa = R.pb = R.pc = 0.0f;
    if (solve3(A, B)) {
        R.pa = __double2float_rn(B[0]);
        R.pb = __double2float_rn(B[1]);
        R.pc = __double2float_rn(B[2]);
    }
    if (right)
        for (int k = 0; k < 3; ++k) tu[k] -= td[k];
    for (int j = 0; j < 3; ++j)
        for (int k = 0; k < j; ++k)
            if (tu[k] > tu[j]) {
                int t = tu[j]; tu[j] = tu[k]; tu[k] = t;
                t = tv[j]; tv[j] = tv[k]; tv[k] = t;
            }
    float A_u = float(tu[0]), A_v = float(tv[0]);
    float B_u = float(tu[1]), B_v = float(tv[1]);
    float C_u = float(tu[2]), C_v = float(tv[2]);
    R.A_u = A_u; R.B_u = B_u; R.C_u = C_u;
    R.AB_a = 0.0f; R.AC_a = 0.0f; R.BC_a = 0.0f;
    if (int(A_u) != int(B_u)) R.AB_a = __fdiv_rn(__fsub_rn(A_v, B_v), __fsub_rn(A_u, B_u));
    if (int(A_u) != int(C_u)) R.AC_a = __fdiv_rn(__fsub_rn(A_v, C_v), __fsub_rn(A_u, C_u));
    if (int(B_u) != int(C_u)) R.BC_a = __fdiv_rn(__fsub_rn(B_v, C_v), __fsub_rn(B_u, C_u));
    R.AB_b = __fmaf_rn(-R.AB_a, A_u, A_v);
    R.AC_b = __fmaf_rn(-R.AC_a, A_u, A_v);
    R.BC_b = __fmaf_rn(-R.BC_a, B_u, B_v);
}

// One thread per (view, triangle): plane and edge set-up and, for the tiled
// paint (tcnt non-null), the prior tiles its pixels can fall in (from the
// exact row range of the raster and its column range).  The triangle goes
// into each such tile's bin of PT_BIN entries at the slot its count's
// atomic returns, or, once a bin is full, into the view's overflow list of
// (tile, triangle) pairs (tcnt[ntiles] counts those).  A triangle whose box
// spans more than four tiles (the long hull triangles) has its tiles shared
// out over the warp's lanes: one lane would wait for each returning atomic
// in turn.
__global__ void __launch_bounds__(256) k_prior_setup(const int32_t* __restrict__ tri0,
                                                     const int32_t* __restrict__ tri1,
                                                     const int32_t* __restrict__ ctr0,
                                                     const int32_t* __restrict__ ctr1,
                                                     const int32_t* __restrict__ can, const int32_t* __restrict__ uvd,
                                                     Raster* __restrict__ rast, int Tmax, Geom g, int32_t* tcnt,
                                                     int ntx, int ntiles, int32_t* bins, int32_t* ovf, int ovf_cap,
                                                     int bin_cap, unsigned* err) {
    grid_dep_wait();
    const int T0 = ctr0[0], T1 = ctr1[0], lane = threadIdx.x & 31;
    // whole warps step through the list, so that a warp can share the
    // tile loop of a triangle whose bounding box spans many tiles
    for (int base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31; base < T0 + T1; base += gridDim.x * blockDim.x) {
        const int i = base + lane;
        const bool valid = i < T0 + T1, right = i >= T0;
        const int t = right ? i - T0 : i;
        Raster R;
        int tx0 = 0, tx1 = -1, ty0 = 0, ty1 = -1;
        if (valid) {
            setup_triangle((right ? tri1 : tri0) + 3 * size_t(t), can, uvd, g.cw, g.step, right, R);
            if (tcnt) {
                int r0 = g.H, r1 = -1;
                part_rows(R, 0, g.W, g.H, r0, r1);
                part_rows(R, 1, g.W, g.H, r0, r1);
                const int u0 = imax(int(R.A_u), 0), u1 = imin(int(R.C_u), g.W) - 1;
                R.tx0 = 1; R.tx1 = 0; R.ty0 = 1; R.ty1 = 0;
                if (r0 <= r1 && u0 <= u1) {
                    R.tx0 = tx0 = u0 / PT_W; R.tx1 = tx1 = u1 / PT_W;
                    R.ty0 = ty0 = r0 / PT_H; R.ty1 = ty1 = r1 / PT_H;
                }
            }
            rast[(right ? Tmax : 0) + t] = R;
        }
        if (!tcnt) continue;
        // one (tile, triangle) entry: the triangle goes into the tile's bin
        // at the slot its count's atomic returns, or into the overflow list
        auto drop = [&](int tile, int tt, bool rt) {
            int32_t* c = tcnt + (rt ? ntiles + 1 : 0);
            const int pos = atomicAdd(c + tile, 1);
            if (pos < bin_cap) {
                bins[(rt ? size_t(ntiles) * PT_BIN : 0) + size_t(tile) * PT_BIN + pos] = tt;
            } else {
                const int k = atomicAdd(c + ntiles, 1);
                int32_t* o = ovf + (rt ? 2 * size_t(ovf_cap) : 0);
                if (k < ovf_cap) {
                    o[2 * k] = tile;
                    o[2 * k + 1] = tt;
                } else {
                    atomicOr(err, ERRF_BOUNDS);
                }
            }
        };
        const int nx = tx1 - tx0 + 1, ntl = nx * (ty1 - ty0 + 1);   // 0 when empty
        const bool wide = ntl > 4;
        if (!wide)
            for (int ty = ty0; ty <= ty1; ++ty)
                for (int tx = tx0; tx <= tx1; ++tx) drop(ty * ntx + tx, t, right);
        for (unsigned m = __ballot_sync(0xffffffffu, wide); m; m &= m - 1) {
            const int src = __ffs(m) - 1;
            const int wt = __shfl_sync(0xffffffffu, t, src), wr = __shfl_sync(0xffffffffu, int(right), src);
            const int wx0 = __shfl_sync(0xffffffffu, tx0, src), wy0 = __shfl_sync(0xffffffffu, ty0, src);
            const int wnx = __shfl_sync(0xffffffffu, nx, src), wn = __shfl_sync(0xffffffffu, ntl, src);
            for (int k = lane; k < wn; k += 32) {
                const int ty = wy0 + k / wnx, tx = wx0 + k % wnx;
                drop(ty * ntx + tx, wt, wr != 0);
            }
        }
    }
}

// A warp paints one triangle's pixels inside the window [wu0, wu1) x
// [wv0, wv1): column u of [A_u, C_u) writes the rows between the long edge
// AC and the edge AB (u < B_u) or BC (u >= B_u), the reference's two
// scan-line parts (KerComputeDisparity.cu:57-150) run as one column range,
// with its contraction made explicit; the window clips exactly as the
// image bounds do.  The lanes are laid out as cw columns x 32/cw rows, cw
// the smallest of 4, 8, 16, 32 that covers the range, so that a narrow
// triangle keeps most lanes busy.
template <typename Put>
__device__ __forceinline__ void paint_warp(const Raster& R, int wu0, int wu1, int wv0, int wv1, int lane, int dcap,
                                           Put put) {
    const int ub = int(R.B_u);
    const int cu0 = imax(int(R.A_u), wu0), cu1 = imin(int(R.C_u), wu1), nc = cu1 - cu0;
    if (nc <= 0) return;
    const int lg = nc <= 4 ? 2 : (nc <= 8 ? 3 : (nc <= 16 ? 4 : 5));
    const int cw = 1 << lg, cl = lane & (cw - 1), rl = lane >> lg, rh = 32 >> lg;
    for (int c0 = cu0; c0 < cu1; c0 += cw) {
        const int u = c0 + cl;
        if (u >= cu1) continue;
        const bool second = u >= ub;
        const float ea = second ? R.BC_a : R.AB_a, eb = second ? R.BC_b : R.AB_b;
        const float fu = float(u);
        const int v1 = raster_row(R.AC_a, R.AC_b, u), v2 = raster_row(ea, eb, u);
        const int va = imax(imin(v1, v2), wv0), vb = imin(imax(v1, v2), wv1);
        for (int v = va + rl; v < vb; v += rh) {
            const float dp = __fadd_rn(__fmaf_rn(R.pa, fu, __fmul_rn(R.pb, float(v))), R.pc);
            int d = __float2int_rz(dp);
            d = d <= 0 ? 0 : (d > dcap ? dcap : d);
            put(u, v, uint32_t(d));
        }
    }
}

// Direct paint: one warp per (view, triangle), which first sets the
// triangle up itself (every lane the same operations on the same loads, so
// no per-triangle record goes through memory and no set-up launch runs);
// every pixel keeps the last covering triangle through atomicMax on the
// packed value in the zeroed prior.
__global__ void __launch_bounds__(256) k_prior_raster(const int32_t* __restrict__ tri0,
                                                      const int32_t* __restrict__ tri1,
                                                      const int32_t* __restrict__ ctr0,
                                                      const int32_t* __restrict__ ctr1,
                                                      const int32_t* __restrict__ can, const int32_t* __restrict__ uvd,
                                                      uint32_t* prior0, uint32_t* prior1, Geom g, int pshift,
                                                      int dcap) {
    grid_dep_wait();
    const int lane = threadIdx.x & 31;
    const int T0 = ctr0[0], T1 = ctr1[0];
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < T0 + T1; i += nw) {
        const bool right = i >= T0;
        const int t = right ? i - T0 : i;
        Raster R;
        setup_triangle((right ? tri1 : tri0) + 3 * size_t(t), can, uvd, g.cw, g.step, right, R);
        const uint32_t tag = uint32_t(t + 1) << pshift;
        uint32_t* prior = right ? prior1 : prior0;
        paint_warp(R, 0, g.W, 0, g.H, lane, dcap,
                   [&](int u, int v, uint32_t d) { atomicMax(&prior[size_t(v) * g.W + u], tag | d); });
    }
}

// One CTA per (prior tile, view): every triangle of the tile's list paints
// the pixels it covers in the tile into shared memory with atomicMax of
// (triangle+1) << pshift | d_plane -- the last triangle in list order wins,
// as a sequential rasteriser writing the triangles in order would leave it
// -- and the tile is then written out whole (0 where nothing covers a
// pixel), so no memset is needed.  A warp per triangle.
__global__ void __launch_bounds__(256) k_prior_tiles(const Raster* __restrict__ rast, int Tmax,
                                                     const int32_t* __restrict__ tcnt,
                                                     const int32_t* __restrict__ bins,
                                                     const int32_t* __restrict__ ovf, int ovf_cap, int bin_cap,
                                                     uint32_t* prior0, uint32_t* prior1, Geom g, int pshift, int dcap,
                                                     int ntx, int ntiles) {
    grid_dep_wait();
    __shared__ uint32_t pt[PT_H][PT_W];
    const int view = blockIdx.z, tu0 = blockIdx.x * PT_W, tv0 = blockIdx.y * PT_H;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    for (int i = tid; i < PT_W * PT_H; i += blockDim.x) (&pt[0][0])[i] = 0u;
    __syncthreads();
    const int32_t* c = tcnt + view * (ntiles + 1);
    const int tile = blockIdx.y * ntx + blockIdx.x;
    const int n = c[tile];
    const int32_t* b = bins + (view ? size_t(ntiles) * PT_BIN : 0) + size_t(tile) * PT_BIN;
    const Raster* rs = rast + (view ? Tmax : 0);
    const int wu1 = imin(tu0 + PT_W, g.W), wv1 = imin(tv0 + PT_H, g.H);
    auto paint = [&](int t) {
        const Raster R = rs[t];
        const uint32_t tag = uint32_t(t + 1) << pshift;
        paint_warp(R, tu0, wu1, tv0, wv1, lane, dcap,
                   [&](int u, int v, uint32_t d) { atomicMax(&pt[v - tv0][u - tu0], tag | d); });
    };
    for (int k = warp; k < imin(n, bin_cap); k += nw) paint(b[k]);
    if (n > bin_cap) {      // a full bin: the rest of its triangles are in the overflow list
        const int no = imin(c[ntiles], ovf_cap);
        const int32_t* o = ovf + (view ? 2 * size_t(ovf_cap) : 0);
        for (int k = warp; k < no; k += nw)
            if (o[2 * k] == tile) paint(o[2 * k + 1]);
    }
    __syncthreads();
    uint32_t* prior = view ? prior1 : prior0;
    for (int i = tid; i < PT_W * PT_H; i += blockDim.x) {
        const int r = i / PT_W, cc = i - r * PT_W, u = tu0 + cc, v = tv0 + r;
        if (u < g.W && v < g.H) prior[size_t(v) * g.W + u] = pt[r][cc];
    }
}

// Candidate-list entries per grid cell kept in shared memory; cells with
// more candidates walk their bitset instead.
constexpr int LMAX = 48;

// Energy update with the reference's strict '<' (the first minimum in
// evaluation order wins).
// Both passes (the cell list, then the plane window) walk their
// disparities in ascending order, so the reference's strict '<' keeps, per
// pass, the smallest energy and among equal energies the smallest d: the
// minimum of e * 4096 + d (d < 4096, energies above -2^18).  The window
// result replaces the list result only with a strictly smaller energy.
constexpr int PK_NONE = 10000 * 4096;   // the reference's start value: energy 10000, no disparity
__device__ __forceinline__ int pk_ed(int e, int d) { return e * 4096 + d; }
__device__ __forceinline__ void take_min(int e, int d, int& best) { best = min(best, pk_ed(e, d)); }

// blockIdx.x = row, blockIdx.y = view (0 left, 1 right).  The other view's
// descriptor row arrives by bulk copy (TMA) while the CTA expands the
// candidate lists of the row's grid cells into shared memory.
//
// Per pixel u the reference evaluates the cell's sorted list, skipping the
// plane window [d_plane - r, d_plane + r] and every d whose warped column
// leaves [3, W - 3), then the window with the penalty added.  Here:
//   * the warped-column test is one bound on d (dlim below): the left view
//     needs d <= u - 3, the right view d <= W - 4 - u, every other bound
//     holds for 3 < u < W - 3; the list is ascending, so the walk stops at
//     the first d > dlim;
//   * when every window penalty is negative (the usual parameters), the
//     window entries need no skipping in the list walk: the window pass
//     re-evaluates each of them with a strictly lower energy, so it ends
//     at the same (value, first index) as the reference's walk;
//   * RFIX > 0 unrolls the window for plane_radius == RFIX;
//   * the own descriptor and the prior of the thread's next pixel are
//     loaded before the current pixel is matched.
template <int RFIX>
__global__ void __launch_bounds__(1024) k_dense(const uint4* __restrict__ desc0, const uint4* __restrict__ desc1,
                                               const uint32_t* __restrict__ prior0, const uint32_t* __restrict__ prior1,
                                               const uint32_t* __restrict__ grid0, const uint32_t* __restrict__ grid1,
                                               float* __restrict__ disp0, float* __restrict__ disp1, Geom g,
                                               DevParams p, int pshift, int sub, int lcap, unsigned* err) {
    grid_dep_wait();
    extern __shared__ __align__(128) uint8_t sm[];
    __shared__ uint64_t bar;
    // sub = 1: every second row and column (output (W/2) x (H/2))
    const int v = int(blockIdx.x) << sub;
    const bool right = blockIdx.y != 0;
    const int W = g.W, H = g.H;
    const int tid = threadIdx.x, NT = blockDim.x;
    const int Wo = W >> sub;
    float* disp = (right ? disp1 : disp0) + size_t(blockIdx.x) * Wo;
    if (!(v > 3 && v < H - 3)) {           // CTA-uniform: no copy is issued for these rows
        for (int o = tid; o < Wo; o += NT) disp[o] = -1.0f;
        return;
    }
    uint4* row = reinterpret_cast<uint4*>(sm);
    int16_t* lst = reinterpret_cast<int16_t*>(sm + size_t(W) * 16);
    uint8_t* lcnt = reinterpret_cast<uint8_t*>(lst + size_t(g.gw) * LMAX);
    const uint4* self = (right ? desc1 : desc0) + size_t(v) * W;
    const uint4* other = (right ? desc0 : desc1) + size_t(v) * W;
    const uint32_t* prior = (right ? prior1 : prior0) + size_t(v) * W;
    const uint32_t* grid = right ? grid1 : grid0;
    if (tid == 0) {
        mbar_init(&bar, 1);
        mbar_expect_tx(&bar, unsigned(W) * 16u);
        bulk_g2s_chunked(row, other, unsigned(W) * 16u, &bar);
    }
    const int gy = floordiv(v, g.gs);
    for (int c = tid; c < g.gw; c += NT) {
        const uint32_t* cell = grid + (size_t(gy) * g.gw + c) * g.words;
        int n = 0;
        for (int w = 0; w < g.words; ++w) {
            uint32_t bits = cell[w];
            while (bits) {
                int d = 32 * w + __ffs(bits) - 1;
                bits &= bits - 1;
                if (n < lcap) lst[c * LMAX + n] = int16_t(d);
                ++n;
            }
        }
        lcnt[c] = uint8_t(n > lcap ? 255 : n);
    }
    // first pixel of this thread and its prefetch
    int o = tid, u = o << sub;
    uint32_t pk_next = o < Wo ? prior[u] : 0u;
    uint4 I_next = o < Wo ? self[u] : make_uint4(0, 0, 0, 0);
    __syncthreads();
    if (!mbar_wait_bounded(&bar, 0, MBAR_WAIT_LIMIT)) {
        if (tid == 0) atomicOr(err, ERRF_TMA_TIMEOUT);
        mbar_wait_bounded(&bar, 0, MBAR_WAIT_LIMIT);   // let the copy in flight land before exiting
        return;
    }
    const int dir = right ? 1 : -1;
    const int r = RFIX > 0 ? RFIX : p.plane_radius;
    const uint32_t dmask = (1u << pshift) - 1u;
    const int gs = g.gs;
    // cell of u, advanced incrementally (u grows by NT per iteration)
    int cell = u / gs, rem = u - cell * gs;
    const int ustep = NT << sub;
    const int cstep = ustep / gs, rstep = ustep - cstep * gs;
    for (; o < Wo; o += NT, u += ustep) {
        const uint32_t pk = pk_next;
        const uint4 I1 = I_next;
        const int c = cell;
        {
            if (o + NT < Wo) { pk_next = prior[u + ustep]; I_next = self[u + ustep]; }
            cell += cstep;
            rem += rstep;
            if (rem >= gs) { rem -= gs; ++cell; }
        }
        float out = -1.0f;
        const int dp = int(pk & dmask);
        if (u > 3 && u < W - 3 && (pk >> pshift) != 0 && dp > 0 &&
            (p.match_texture <= 0 || texture16(I1) >= p.match_texture)) {
            const int dlim = right ? W - 4 - u : u - 3;
            const int dpmin = imax(dp - r, 0);
            const int dpmax = imin(dp + r, g.D);
            int best_l = PK_NONE, best_w = PK_NONE;
            const int n = lcnt[c];
            if (n != 255) {
                const int16_t* Ls = lst + c * LMAX;
                int i = 0;
                if (p.window_negative) {
                    const uint32_t* L2 = reinterpret_cast<const uint32_t*>(Ls);
                    for (; i + 1 < n; i += 2) {
                        const uint32_t pr = L2[i >> 1];
                        const int da = int(pr & 0xffffu), db = int(pr >> 16);
                        if (db > dlim) break;
                        const int ea = sad16(I1, row[u + dir * da]);
                        const int eb = sad16(I1, row[u + dir * db]);
                        take_min(ea, da, best_l);
                        take_min(eb, db, best_l);
                    }
                    for (; i < n; ++i) {
                        const int d = Ls[i];
                        if (d > dlim) break;
                        take_min(sad16(I1, row[u + dir * d]), d, best_l);
                    }
                } else {
                    for (; i < n; ++i) {
                        const int d = Ls[i];
                        if (d > dlim) break;
                        if (d >= dpmin && d <= dpmax) continue;
                        take_min(sad16(I1, row[u + dir * d]), d, best_l);
                    }
                }
            } else {
                const uint32_t* cw = grid + (size_t(gy) * g.gw + c) * g.words;
                bool done = false;
                for (int w = 0; w < g.words && !done; ++w) {
                    uint32_t bits = cw[w];
                    while (bits) {
                        const int d = 32 * w + __ffs(bits) - 1;
                        bits &= bits - 1;
                        if (d > dlim) { done = true; break; }
                        if (d >= dpmin && d <= dpmax) continue;
                        take_min(sad16(I1, row[u + dir * d]), d, best_l);
                    }
                }
            }
            if (RFIX > 0) {
#pragma unroll
                for (int k = -RFIX; k <= RFIX; ++k) {
                    const int d = dp + k;
                    if (d >= 0 && d <= g.D && d <= dlim)
                        take_min(sad16(I1, row[u + dir * d], p.penalty[k < 0 ? -k : k]), d, best_w);
                }
            } else {
                const int dhi = imin(dpmax, dlim);
                for (int d = dpmin; d <= dhi; ++d)
                    take_min(sad16(I1, row[u + dir * d], p.penalty[d > dp ? d - dp : dp - d]), d, best_w);
            }
            const int best = (best_w >> 12) < (best_l >> 12) ? best_w : best_l;
            out = best < PK_NONE ? float(best & 4095) : -1.0f;
        }
        disp[o] = out;
    }
}

// kerLeftRightConsistencyCheck (src/Kernels/KerLeftRightConsistencyCheck.cu:7-64)
// reading the dense results and writing separate outputs (the reference's
// snapshot copies, src/Elas.cu:542-546).
// scale = 0.5 on subsampled maps: a disparity (in full-resolution pixels)
// moves d / 2 columns there.
// The checked maps go to O1/O2 and, where given, also to C1/C2 (the
// buffers the post-filters then work on in place).
__global__ void k_lr(const float* __restrict__ D1, const float* __restrict__ D2, float* __restrict__ O1,
                     float* __restrict__ O2, float* __restrict__ C1, float* __restrict__ C2, int W, int H, float thr,
                     float scale) {
    grid_dep_wait();
    int u = blockIdx.x * blockDim.x + threadIdx.x, v = blockIdx.y;
    if (u >= W || v >= H) return;
    size_t a = size_t(v) * W + u;
    float d1 = D1[a], d2 = D2[a];
    float uw1 = float(u) - d1 * scale, uw2 = float(u) + d2 * scale;
    float o1 = d1, o2 = d2;
    if (d1 >= 0 && uw1 >= 0 && uw1 < W) {
        if (fabsf(D2[size_t(v) * W + int(uw1)] - d1) > thr) o1 = -1;
    } else {
        o1 = -1;
    }
    if (d2 >= 0 && uw2 >= 0 && uw2 < W) {
        if (fabsf(D1[size_t(v) * W + int(uw2)] - d2) > thr) o2 = -1;
    } else {
        o2 = -1;
    }
    O1[a] = o1;
    O2[a] = o2;
    if (C1) {
        C1[a] = o1;
        C2[a] = o2;
    }
}

}  // namespace

size_t prior_tile_count(const Geom& g) { return size_t((g.W + PT_W - 1) / PT_W) * ((g.H + PT_H - 1) / PT_H); }

size_t prior_overflow_capacity(const Geom& g, int Tmax) {
    // bins overflow only where a 64x32 tile meets more than PT_BIN triangles
    return size_t(2) * Tmax + size_t(16) * prior_tile_count(g);
}

cudaError_t launch_prior(const int32_t* tri0, const int32_t* tri1, const int32_t* ctr0, const int32_t* ctr1,
                         int Tmax, const int32_t* can, const int32_t* uvd, void* rast, const PriorTiles& tl,
                         uint32_t* prior0, uint32_t* prior1, const Geom& g, int pshift, int dcap, int num_sms,
                         unsigned* err, cudaStream_t st, int* nlaunch, bool tiled, bool zeroed, int bin_cap) {
    Raster* R = static_cast<Raster*>(rast);
    const int tblocks = imax(1, imin(8 * num_sms, (2 * Tmax + 255) / 256));
    if (!tiled) {
        const size_t n = size_t(g.W) * g.H * sizeof(uint32_t);
        if (!zeroed) {
            cudaMemsetAsync(prior0, 0, n, st);
            cudaMemsetAsync(prior1, 0, n, st);
        }
        launch_k(k_prior_raster, imax(1, imin(16 * num_sms, (2 * Tmax + 7) / 8)), 256, 0, st, tri0, tri1, ctr0, ctr1,
                 can, uvd, prior0, prior1, g, pshift, dcap);
        if (nlaunch) *nlaunch += 1;
        return cudaGetLastError();
    }
    const int ntx = (g.W + PT_W - 1) / PT_W, nty = (g.H + PT_H - 1) / PT_H, ntiles = ntx * nty;
    cudaMemsetAsync(tl.cnt, 0, size_t(2) * (ntiles + 1) * sizeof(int32_t), st);
    launch_k(k_prior_setup, tblocks, 256, 0, st, tri0, tri1, ctr0, ctr1, can, uvd, R, Tmax, g, tl.cnt, ntx, ntiles,
             tl.bins, tl.ovf, tl.ovf_cap, bin_cap, err);
    launch_k(k_prior_tiles, dim3(ntx, nty, 2), 256, 0, st, R, Tmax, tl.cnt, tl.bins, tl.ovf, tl.ovf_cap, bin_cap,
             prior0, prior1, g, pshift, dcap, ntx, ntiles);
    if (nlaunch) *nlaunch += 2;
    return cudaGetLastError();
}

size_t raster_bytes() { return sizeof(Raster); }

size_t dense_smem_bytes(const Geom& g) { return size_t(g.W) * 16 + size_t(g.gw) * (LMAX * 2 + 1); }

cudaError_t launch_dense(const uint4* desc0, const uint4* desc1, const uint32_t* prior0, const uint32_t* prior1,
                         const uint32_t* grid0, const uint32_t* grid1, float* disp0, float* disp1, const Geom& g,
                         const DevParams& p, int pshift, unsigned* err, cudaStream_t st, int threads, int sub,
                         bool force_bitset) {
    // list capacity per cell (0 sends every non-empty cell to the bitset walk)
    const int lcap = force_bitset ? 0 : LMAX;
    size_t smem = dense_smem_bytes(g);
    if (threads <= 0) threads = 512;
    threads = imin(threads, (((g.W >> sub) + 31) / 32) * 32);
    const dim3 grid(g.H >> sub, 2);
    if (p.plane_radius == 2) {
        allow_smem(k_dense<2>);
        launch_k(k_dense<2>, grid, threads, smem, st, desc0, desc1, prior0, prior1, grid0, grid1, disp0, disp1, g, p,
                                                pshift, sub, lcap, err);
    } else {
        allow_smem(k_dense<0>);
        launch_k(k_dense<0>, grid, threads, smem, st, desc0, desc1, prior0, prior1, grid0, grid1, disp0, disp1, g, p,
                                                pshift, sub, lcap, err);
    }
    return cudaGetLastError();
}

cudaError_t launch_lr(const float* d0, const float* d1, float* o0, float* o1, float* c0, float* c1, const Geom& g,
                      int lr_threshold, cudaStream_t st, int sub) {
    const int W = g.W >> sub, H = g.H >> sub;
    launch_k(k_lr, dim3((W + 255) / 256, H), 256, 0, st, d0, d1, o0, o1, c0, c1, W, H, float(lr_threshold),
             sub ? 0.5f : 1.0f);
    return cudaGetLastError();
}

}  // namespace elas
