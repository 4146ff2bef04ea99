// ORACLE -- test infrastructure only.
//
// A CPU restatement of the reference ELAS pipeline (beautifulv0id/
// CUDA-Stereo-Matching), stage by stage, used to check the CUDA library.
// Only the tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg
// may load it; the product never does.
//
// Each function cites the reference kernel it restates.  Where the
// reference is nondeterministic or reads uninitialised memory, the decision
// taken here is stated at the function (quirks Q1-Q10 of the project notes):
//   Q3  removeInconsistentSupportPoints races in place -> snapshot semantics
//   Q5  descriptor border bytes are uninitialised      -> zero
//   Q7  nvcc contracts a*b+c into FMA                  -> explicit fma below
//   Q10 overlapping triangle rasterisation             -> list order, last wins
//   dense match_texture: the reference returns from the whole thread (and so
//       skips that thread's later pixels); here only the pixel is skipped.
//       Identical at match_texture = 0, the value of every configuration.
// Delaunay: the reference calls Shewchuk's Triangle ("zQB", src/Elas.cu:316);
// that exact code is compiled from the reference sources into
// oracle/_ref/libreftriangle.so and loaded at run time.
//
// Parity pins: the Triangle stage is the reference's own code.  The ELAS
// kernels have no golden vectors in the reference tree; tests/golden holds
// fixtures made by running the reference's kernels (compiled from its
// sources) on a B200, with the generating script beside them.
#include <algorithm>
#include <array>
#include <iterator>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <dlfcn.h>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/elas_b200.h"

namespace {

inline int iabs(int x) { return x < 0 ? -x : x; }

// Float -> int32 with the GPU's conversion semantics (cvt.rzi.s32.f32:
// truncate, saturate, NaN -> 0).
inline int32_t f2i_sat(float x) {
    if (std::isnan(x)) return 0;
    if (x >= 2147483648.0f) return INT32_MAX;
    if (x <= -2147483648.0f) return INT32_MIN;
    return int32_t(x);
}
// Float -> uint32 with the GPU's conversion semantics (negative -> 0).
inline uint32_t f2u_sat(float x) {
    if (std::isnan(x)) return 0u;
    if (x <= 0.0f) return 0u;
    if (x >= 4294967296.0f) return UINT32_MAX;
    return uint32_t(x);
}

struct Dims {
    int W, H, cw, ch, gw, gh, D, step, gs;
};

Dims dims_of(int W, int H, const elas_params& p) {
    Dims d;
    d.W = W; d.H = H; d.D = p.disp_max; d.step = p.candidate_stepsize; d.gs = p.grid_size;
    d.cw = W / p.candidate_stepsize;                           // src/Elas.cu:29
    d.ch = H / p.candidate_stepsize;                           // src/Elas.cu:30
    d.gw = int(std::ceil(float(W) / float(p.grid_size)));      // src/Elas.cu:411
    d.gh = int(std::ceil(float(H) / float(p.grid_size)));      // src/Elas.cu:412
    return d;
}

}  // namespace

extern "C" {

// ---------------------------------------------------------------------------
// Descriptor: kerComputeSobel (src/Kernels/KerDescriptor.cu:8-50) and
// kerComputeDescriptor (src/Kernels/KerDescriptor.cu:52-101).
// Q5: the reference leaves the border descriptors uninitialised
// (src/Elas.cu:142 allocates without a fill); here they are zero.
int orc_descriptor(const uint8_t* img, int W, int H, uint8_t* desc) {
    if (!img || !desc || W < 7 || H < 7) return ELAS_ERR_INVALID_ARG;
    std::vector<uint8_t> du(size_t(W) * H, 0), dv(size_t(W) * H, 0);
#pragma omp parallel for schedule(static)
    for (int v = 1; v < H - 1; ++v) {
        for (int u = 1; u < W - 1; ++u) {
            auto I = [&](int x, int y) { return float(img[size_t(y) * W + x]); };
            float sdu = I(u - 1, v - 1) + 2 * I(u - 1, v) + I(u - 1, v + 1)
                      - I(u + 1, v - 1) - 2 * I(u + 1, v) - I(u + 1, v + 1);
            float sdv = I(u - 1, v - 1) + 2 * I(u, v - 1) + I(u + 1, v - 1)
                      - I(u - 1, v + 1) - 2 * I(u, v + 1) - I(u + 1, v + 1);
            du[size_t(v) * W + u] = uint8_t(std::min(std::max(-128.f, sdu / 4), 127.f) + 128);
            dv[size_t(v) * W + u] = uint8_t(std::min(std::max(-128.f, sdv / 4), 127.f) + 128);
        }
    }
    std::memset(desc, 0, size_t(W) * H * 16);
#pragma omp parallel for schedule(static)
    for (int v = 3; v < H - 3; ++v) {
        for (int u = 3; u < W - 3; ++u) {
            auto DU = [&](int x, int y) { return du[size_t(y) * W + x]; };
            auto DV = [&](int x, int y) { return dv[size_t(y) * W + x]; };
            uint8_t* o = desc + (size_t(v) * W + u) * 16;
            o[0] = DU(u, v - 2);
            o[1] = DU(u - 2, v - 1); o[2] = DU(u, v - 1); o[3] = DU(u + 2, v - 1);
            o[4] = DU(u - 1, v); o[5] = DU(u, v); o[6] = DU(u, v); o[7] = DU(u + 1, v);
            o[8] = DU(u - 2, v + 1); o[9] = DU(u, v + 1); o[10] = DU(u + 2, v + 1);
            o[11] = DU(u, v + 2);
            o[12] = DV(u, v - 1); o[13] = DV(u - 1, v); o[14] = DV(u + 1, v); o[15] = DV(u, v + 1);
        }
    }
    return ELAS_OK;
}

// ---------------------------------------------------------------------------
// Support matching: kerComputeSupportMatches
// (src/Kernels/KerSupportMatches.cu:12-193), launched L->R then R->L
// (src/Elas.cu:200-225).  The 32-thread block is simulated literally: lane l
// sweeps d = dmin + l + 32k keeping (best, second best) with strict '<', then
// lane 0 merges its own registers followed by every lane's (best, second)
// pair from shared memory, lane 0's included (Q1/Q2).
static void support_pass(const uint8_t* desc0, const uint8_t* desc1, const Dims& g,
                         const elas_params& p, int32_t* can, bool right_image) {
    const int W = g.W, H = g.H;
    const int x_step = 2, y_step = 2, desc_window = 3;
    const long off[4] = {-16L * x_step - 16L * W * y_step, +16L * x_step - 16L * W * y_step,
                         -16L * x_step + 16L * W * y_step, +16L * x_step + 16L * W * y_step};
#pragma omp parallel for schedule(dynamic, 4)
    for (int v_can = 0; v_can < g.ch; ++v_can) {
        for (int u_can = 0; u_can < g.cw; ++u_can) {
            int u = u_can * g.step, v = v_can * g.step;
            int32_t& c = can[size_t(v_can) * g.cw + u_can];
            if (!(u >= x_step + desc_window && u <= W - x_step - desc_window - 1 &&
                  v >= y_step + desc_window && v <= H - y_step - desc_window - 1))
                continue;
            int d_left = 0;
            if (right_image) {
                d_left = c;
                if (d_left < 0) continue;
                u = u - d_left;
            }
            const long line = 16L * W * v;
            const uint8_t* self = (right_image ? desc1 : desc0) + line;
            const uint8_t* other = (right_image ? desc0 : desc1) + line;
            const uint8_t* blk = self + 16L * u;
            int sum = 0;
            for (int i = 0; i < 16; ++i) sum += iabs(int(blk[i]) - 128);
            if (sum < p.support_texture) { c = -1; continue; }
            uint8_t corner[4][16];
            for (int i = 0; i < 4; ++i) std::memcpy(corner[i], blk + off[i], 16);
            int disp_min_valid = std::max(p.disp_min, 0);
            int disp_max_valid = right_image ? std::min(p.disp_max, W - u - desc_window - x_step)
                                             : std::min(p.disp_max, u - desc_window - x_step);
            if (disp_max_valid - disp_min_valid < 10) { c = -1; continue; }
            int16_t m1E[32], m1d[32], m2E[32], m2d[32];
            for (int l = 0; l < 32; ++l) {
                int16_t a1 = 32767, b1 = -1, a2 = 32767, b2 = -1;
                for (int d = disp_min_valid + l; d <= disp_max_valid; d += 32) {
                    int uw = right_image ? u + d : u - d;
                    const uint8_t* ob = other + 16L * uw;
                    int e = 0;
                    for (int i = 0; i < 4; ++i)
                        for (int j = 0; j < 16; ++j) e += iabs(int(corner[i][j]) - int(ob[off[i] + j]));
                    if (e < a1) { a2 = a1; b2 = b1; a1 = int16_t(e); b1 = int16_t(d); }
                    else if (e < a2) { a2 = int16_t(e); b2 = int16_t(d); }
                }
                m1E[l] = a1; m1d[l] = b1; m2E[l] = a2; m2d[l] = b2;
            }
            int16_t M1E = m1E[0], M1d = m1d[0], M2E = m2E[0], M2d = m2d[0];
            for (int i = 0; i < 64; ++i) {
                int l = i >> 1;
                int tE = (i & 1) ? m2E[l] : m1E[l];
                int td = (i & 1) ? m2d[l] : m1d[l];
                if (tE < M1E) { M2E = M1E; M2d = M1d; M1E = int16_t(tE); M1d = int16_t(td); }
                else if (tE < M2E) { M2E = int16_t(tE); M2d = int16_t(td); }
            }
            if (M1d >= 0 && M2d >= 0 && float(M1E) < p.support_threshold * float(M2E)) {
                if (!right_image) c = M1d;
                else if (iabs(d_left - M1d) > p.lr_threshold) c = -1;
            } else {
                c = -1;
            }
        }
    }
}

int orc_support_sweep(const uint8_t* desc0, const uint8_t* desc1, int W, int H,
                      const elas_params* p, int32_t* can) {
    if (!desc0 || !desc1 || !p || !can) return ELAS_ERR_INVALID_ARG;
    Dims g = dims_of(W, H, *p);
    std::fill(can, can + size_t(g.cw) * g.ch, -1);              // src/Elas.cu:190
    support_pass(desc0, desc1, g, *p, can, false);
    support_pass(desc0, desc1, g, *p, can, true);
    return ELAS_OK;
}

// removeInconsistentSupportPoints (src/Kernels/KerSupportMatches.cu:195-239).
// Q3: the kernel reads and writes `can` in place from concurrent threads;
// here every read sees the array as it was before the pass.  The reference's
// bound `y_can < can_width` (:208) is kept.
int orc_filter_inconsistent(int32_t* can, int cw, int ch, const elas_params* p) {
    if (!can || !p) return ELAS_ERR_INVALID_ARG;
    std::vector<int32_t> snap(can, can + size_t(cw) * ch);
    const int ws = p->incon_window_size;
#pragma omp parallel for schedule(static)
    for (int y = 0; y < ch; ++y) {
        for (int x = 0; x < cw; ++x) {
            if (!(x < cw && y < cw)) continue;
            int d = snap[size_t(y) * cw + x];
            if (d < 0) continue;
            int support = 0;
            for (int x2 = x - ws; x2 <= x + ws; ++x2)
                for (int y2 = y - ws; y2 <= y + ws; ++y2)
                    if (x2 >= 0 && x2 < cw && y2 >= 0 && y2 < ch) {
                        int d2 = snap[size_t(y2) * cw + x2];
                        if (d2 >= 0 && iabs(d - d2) <= p->incon_threshold) ++support;
                    }
            if (support < p->incon_min_support) can[size_t(y) * cw + x] = -1;
        }
    }
    return ELAS_OK;
}

// removeRedundantSupportPointsHorizontal then ...Vertical
// (src/Kernels/KerSupportMatches.cu:241-357, order src/Elas.cu:254-272).
// Each line is processed serially in place; REDUN_MAX_DIST 5 and
// REDUN_THRESHOLD 1 are fixed constants (KernelsCommon.h:16-17).
int orc_filter_redundant(int32_t* can, int cw, int ch) {
    if (!can) return ELAS_ERR_INVALID_ARG;
    const int max_dist = 5, thr = 1;
    for (int pass = 0; pass < 2; ++pass) {
        const int lines = pass == 0 ? ch : cw, len = pass == 0 ? cw : ch;
        for (int l = 0; l < lines; ++l) {
            auto at = [&](int k) -> int32_t& {
                return pass == 0 ? can[size_t(l) * cw + k] : can[size_t(k) * cw + l];
            };
            for (int k = 0; k < len; ++k) {
                int d = at(k);
                if (d < 0) continue;
                bool redundant = true;
                for (int dir = -1; dir <= 1; dir += 2) {
                    int k2 = k;
                    bool support = false;
                    for (int j = 0; j < max_dist; ++j) {
                        k2 += dir;
                        if (k2 < 0 || k2 >= len) break;
                        int d2 = at(k2);
                        if (d2 >= 0 && iabs(d - d2) <= thr) { support = true; break; }
                    }
                    if (!support) { redundant = false; break; }
                }
                if (redundant) at(k) = -1;
            }
        }
    }
    return ELAS_OK;
}

// Compaction (kerFlag + scan + kerCompact, src/Kernels/KerSupportMatches.cu:
// 360-421, src/Elas.cu:338-394): valid candidates in raster order of the
// candidate lattice; out[3i..3i+2] = (u, v, d).  sp0 = (u, v), sp1 = (u-d, v).
int orc_support_list(const int32_t* can, int cw, int ch, int step, int32_t* out) {
    if (!can) return -ELAS_ERR_INVALID_ARG;
    int n = 0;
    for (int v = 0; v < ch; ++v)
        for (int u = 0; u < cw; ++u) {
            int d = can[size_t(v) * cw + u];
            if (d >= 0) {
                if (out) { out[3 * n] = u * step; out[3 * n + 1] = v * step; out[3 * n + 2] = d; }
                ++n;
            }
        }
    return n;
}

// Disparity grid: kerLoadGridValues + kerCreateGird
// (src/Kernels/KerGrid.cu:8-126, src/Elas.cu:403-464).  Output layout as the
// reference: int32 [gh][gw][D+2] = {count, d_0 < d_1 < ...}; border cells
// keep count 0 (KerGrid.cu:70).
int orc_grid(const int32_t* can, int W, int H, const elas_params* p,
             int32_t* grid_left, int32_t* grid_right) {
    if (!can || !p) return ELAS_ERR_INVALID_ARG;
    Dims g = dims_of(W, H, *p);
    const int D = g.D;
    std::vector<uint8_t> t0(size_t(g.gw) * g.gh * (D + 1), 0), t1(t0.size(), 0);
    for (int v_can = 0; v_can < g.ch; ++v_can)
        for (int u_can = 0; u_can < g.cw; ++u_can) {
            int dc = can[size_t(v_can) * g.cw + u_can];
            if (dc < 0) continue;
            int dmin = std::max(dc - 1, 0), dmax = std::min(dc + 1, D);
            int u_img = u_can * g.step, v_img = v_can * g.step;
            for (int d = dmin; d <= dmax; ++d) {
                int ug0 = int(std::floor(float(u_img) / float(g.gs)));
                int ug1 = int(std::floor(float(u_img - dc) / float(g.gs)));
                int vg = int(std::floor(float(v_img) / float(g.gs)));
                if (vg >= 0 && vg < g.gh) {
                    if (ug0 >= 0 && ug0 < g.gw) t0[(size_t(vg) * g.gw + ug0) * (D + 1) + d] = 1;
                    if (ug1 >= 0 && ug1 < g.gw) t1[(size_t(vg) * g.gw + ug1) * (D + 1) + d] = 1;
                }
            }
        }
    for (int side = 0; side < 2; ++side) {
        int32_t* grid = side == 0 ? grid_left : grid_right;
        if (!grid) continue;
        const std::vector<uint8_t>& t = side == 0 ? t0 : t1;
        std::memset(grid, 0, sizeof(int32_t) * size_t(g.gw) * g.gh * (D + 2));
        for (int vg = 1; vg < g.gh - 1; ++vg)
            for (int ug = 1; ug < g.gw - 1; ++ug) {
                int32_t* cell = grid + (size_t(vg) * g.gw + ug) * (D + 2);
                int k = 1;
                for (int d = 0; d <= D; ++d) {
                    uint8_t o = 0;
                    for (int dy = -1; dy <= 1; ++dy)
                        for (int dx = -1; dx <= 1; ++dx)
                            o |= t[(size_t(vg + dy) * g.gw + ug + dx) * (D + 1) + d];
                    if (o) cell[k++] = d;
                }
                cell[0] = k - 1;
            }
    }
    return ELAS_OK;
}

// kerSolve (src/Kernels/KerComputeDisparity.cu:321-375): Gauss-Jordan with
// full pivoting in double, eps 1e-20 (KerComputeDisparity.h:36).
// Q7: the row updates `x -= y*dum` are evaluated as fma(-y, dum, x).
static bool solve3(double A[3][3], double B[3], double eps = 1e-20) {
    int ipiv[3] = {0, 0, 0};
    int irow = 0, icol = 0;
    for (int i = 0; i < 3; ++i) {
        double big = 0.0;
        for (int j = 0; j < 3; ++j)
            if (ipiv[j] != 1)
                for (int k = 0; k < 3; ++k)
                    if (ipiv[k] == 0)
                        if (std::fabs(A[j][k]) >= big) { big = std::fabs(A[j][k]); irow = j; icol = k; }
        ++ipiv[icol];
        if (irow != icol) {
            for (int l = 0; l < 3; ++l) std::swap(A[irow][l], A[icol][l]);
            std::swap(B[irow], B[icol]);
        }
        if (std::fabs(A[icol][icol]) < eps) return false;
        double pivinv = 1.0 / A[icol][icol];
        A[icol][icol] = 1.0;
        for (int l = 0; l < 3; ++l) A[icol][l] *= pivinv;
        B[icol] *= pivinv;
        for (int ll = 0; ll < 3; ++ll)
            if (ll != icol) {
                double dum = A[ll][icol];
                A[ll][icol] = 0.0;
                for (int l = 0; l < 3; ++l) A[ll][l] = std::fma(-A[icol][l], dum, A[ll][l]);
                B[ll] = std::fma(-B[icol], dum, B[ll]);
            }
    }
    return true;
}

// Plane prior: kerComputeDepthApproximation
// (src/Kernels/KerComputeDisparity.cu:9-152).  Triangles are rasterised in
// list order; a pixel written by several triangles keeps the last (Q10).
// `prior` receives the integer d_plane (the reference stores it in a float
// image and converts back; identical for |d_plane| < 2^24, and every larger
// value behaves alike in the dense step).  Q7 contractions:
//   AB_b = fma(-AB_a, A_u, A_v);  v_edge = fma(AC_a, u, AC_b);
//   d_plane = fma(a, u, b*v) + c.
int orc_prior(const int32_t* can, int cw, int step, const int32_t* uvd, const int32_t* tris,
              int ntri, int right_image, int W, int H, int32_t* prior) {
    if (!can || !uvd || (!tris && ntri > 0) || !prior) return ELAS_ERR_INVALID_ARG;
    std::fill(prior, prior + size_t(W) * H, -1);
    for (int t = 0; t < ntri; ++t) {
        int c[3] = {tris[3 * t], tris[3 * t + 1], tris[3 * t + 2]};
        int tu[3], tv[3], td[3];
        for (int k = 0; k < 3; ++k) {
            tu[k] = uvd[3 * c[k]];
            tv[k] = uvd[3 * c[k] + 1];
            // KerComputeDisparity.cu:53-55 reads can[(v * cw + u) / step], the
            // lattice point's disparity, which the list holds as well; corner
            // points (add_corners) exist only in the list
            td[k] = uvd[3 * c[k] + 2];
        }
        double A[3][3], B[3];
        for (int k = 0; k < 3; ++k) {
            A[k][0] = right_image ? double(tu[k] - td[k]) : double(tu[k]);
            A[k][1] = tv[k];
            A[k][2] = 1;
            B[k] = td[k];
        }
        float pa = 0, pb = 0, pc = 0;
        if (solve3(A, B)) { pa = float(B[0]); pb = float(B[1]); pc = float(B[2]); }
        if (right_image)
            for (int k = 0; k < 3; ++k) tu[k] -= td[k];
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < j; ++k)
                if (tu[k] > tu[j]) { std::swap(tu[j], tu[k]); std::swap(tv[j], tv[k]); }
        float A_u = float(tu[0]), A_v = float(tv[0]);
        float B_u = float(tu[1]), B_v = float(tv[1]);
        float C_u = float(tu[2]), C_v = float(tv[2]);
        float AB_a = 0, AC_a = 0, BC_a = 0;
        if (int(A_u) != int(B_u)) AB_a = (A_v - B_v) / (A_u - B_u);
        if (int(A_u) != int(C_u)) AC_a = (A_v - C_v) / (A_u - C_u);
        if (int(B_u) != int(C_u)) BC_a = (B_v - C_v) / (B_u - C_u);
        float AB_b = std::fma(-AB_a, A_u, A_v);
        float AC_b = std::fma(-AC_a, A_u, A_v);
        float BC_b = std::fma(-BC_a, B_u, B_v);
        auto span = [&](int u0, int u1, float ea, float eb) {
            for (int u = std::max(u0, 0); u < std::min(u1, W); ++u) {
                int v1 = int32_t(f2u_sat(std::fma(AC_a, float(u), AC_b)));
                int v2 = int32_t(f2u_sat(std::fma(ea, float(u), eb)));
                for (int v = std::min(v1, v2); v < std::max(v1, v2); ++v) {
                    if (v < 0 || v >= H) continue;   // never taken for triangles inside the image
                    float dp = std::fma(pa, float(u), pb * float(v)) + pc;
                    prior[size_t(v) * W + u] = f2i_sat(dp);
                }
            }
        };
        if (int(A_u) != int(B_u)) span(int(A_u), int(B_u), AB_a, AB_b);
        if (int(B_u) != int(C_u)) span(int(B_u), int(C_u), BC_a, BC_b);
    }
    return ELAS_OK;
}

// Posterior penalty of kerComputeDisparity (KerComputeDisparity.cu:270-271):
//   P(dd) = (int)((-log(gamma + exp(-dd^2 / (2 sigma^2))) + log(gamma)) / beta)
// in float except the final division, which the double literal BETA makes
// double.
static int penalty(int dd, const elas_params& p) {
    float two_sigma_squared = 2 * p.sigma * p.sigma;
    float e = std::exp(float(-dd * dd) / two_sigma_squared);
    float num = -std::log(p.gamma + e) + std::log(p.gamma);
    return int32_t(double(num) / double(p.beta));
}

int orc_penalty(int dd, const elas_params* p) { return p ? penalty(dd, *p) : 0; }

// Dense matching: kerComputeDisparity + kerUpdatePosteriorMinimum
// (src/Kernels/KerComputeDisparity.cu:155-316, :377-402).  `disp` is filled
// with -1 first (d_disp0/1 are created with -1, src/Elas.cu:94-95).
int orc_dense(const int32_t* grid, const uint8_t* desc0, const uint8_t* desc1, const int32_t* prior,
              int right_image, int W, int H, const elas_params* pp, float* disp) {
    if (!grid || !desc0 || !desc1 || !prior || !pp || !disp) return ELAS_ERR_INVALID_ARG;
    const elas_params& p = *pp;
    Dims g = dims_of(W, H, p);
    const int desc_window = 3;
    const int disp_num = p.disp_max + 1;
    const int plane_radius = int32_t(std::max(float(std::ceil(p.sigma * p.sradius)), 2.0f));
    std::fill(disp, disp + size_t(W) * H, -1.0f);
#pragma omp parallel for schedule(dynamic, 2)
    for (int v = desc_window + 1; v < H - desc_window; ++v) {
        const long line = 16L * W * v;
        const uint8_t* I1 = (right_image ? desc1 : desc0) + line;
        const uint8_t* I2 = (right_image ? desc0 : desc1) + line;
        for (int u = desc_window + 1; u < W - desc_window; ++u) {
            int dp = prior[size_t(v) * W + u];
            if (dp <= 0) continue;
            const uint8_t* b1 = I1 + 16L * u;
            int sum = 0;
            for (int i = 0; i < 16; ++i) sum += iabs(int(b1[i]) - 128);
            if (sum < p.match_texture) continue;
            long dpmin = std::max<long>(long(dp) - plane_radius, 0);
            long dpmax = std::min<long>(long(dp) + plane_radius, disp_num - 1);
            int gx = int(std::floor(float(u) / float(g.gs)));
            int gy = int(std::floor(float(v) / float(g.gs)));
            const int32_t* cell = grid + (size_t(gy) * g.gw + gx) * (p.disp_max + 2);
            int num_grid = cell[0];
            int min_val = 10000, min_d = -1;
            auto sad = [&](int uw) {
                const uint8_t* b2 = I2 + 16L * uw;
                int s = 0;
                for (int j = 0; j < 16; ++j) s += iabs(int(b2[j]) - int(b1[j]));
                return s;
            };
            for (int i = 0; i < num_grid; ++i) {
                int d = cell[1 + i];
                if (d < dpmin || d > dpmax) {
                    int uw = right_image ? u + d : u - d;
                    if (uw < desc_window || uw >= W - desc_window) continue;
                    int val = sad(uw);
                    if (val < min_val) { min_val = val; min_d = d; }
                }
            }
            for (long d = dpmin; d <= dpmax; ++d) {
                int uw = right_image ? u + int(d) : u - int(d);
                if (uw < desc_window || uw >= W - desc_window) continue;
                int val = penalty(iabs(int(d - dp)), p) + sad(uw);
                if (val < min_val) { min_val = val; min_d = int(d); }
            }
            disp[size_t(v) * W + u] = min_d >= 0 ? float(min_d) : -1.0f;
        }
    }
    return ELAS_OK;
}

// Left/right consistency: kerLeftRightConsistencyCheck
// (src/Kernels/KerLeftRightConsistencyCheck.cu:7-64) against snapshot copies
// (src/Elas.cu:542-546).
// scale 0.5 on subsampled maps (the project's subsampling mode: a
// disparity in full-resolution pixels moves d / 2 columns of the half-size
// map).
int orc_lr_scaled(float* D1, float* D2, int W, int H, const elas_params* p, float scale) {
    if (!D1 || !D2 || !p) return ELAS_ERR_INVALID_ARG;
    std::vector<float> c1(D1, D1 + size_t(W) * H), c2(D2, D2 + size_t(W) * H);
    const float thr = float(p->lr_threshold);
    for (int v = 0; v < H; ++v)
        for (int u = 0; u < W; ++u) {
            size_t a = size_t(v) * W + u;
            float d1 = c1[a], d2 = c2[a];
            float uw1 = float(u) - d1 * scale, uw2 = float(u) + d2 * scale;
            if (d1 >= 0 && uw1 >= 0 && uw1 < W) {
                if (std::fabs(c2[size_t(v) * W + int32_t(uw1)] - d1) > thr) D1[a] = -1;
            } else {
                D1[a] = -1;
            }
            if (d2 >= 0 && uw2 >= 0 && uw2 < W) {
                if (std::fabs(c1[size_t(v) * W + int32_t(uw2)] - d2) > thr) D2[a] = -1;
            } else {
                D2[a] = -1;
            }
        }
    return ELAS_OK;
}

int orc_lr(float* D1, float* D2, int W, int H, const elas_params* p) { return orc_lr_scaled(D1, D2, W, H, p, 1.0f); }

// ---------------------------------------------------------------------------
// Post-filters.  The reference has none (its process() ends after the L/R
// check, src/Elas.cu:107-119; only the parameter fields exist,
// src/Elas.h:31-36), so these are the project's own definitions, written
// from the ELAS parameter semantics.  Parity against the reference is
// therefore unpinned; the CUDA filters are checked against these.
//
// speckle: 4-connected segments of valid pixels whose neighbours differ by
//   <= speckle_sim_threshold; segments with fewer than speckle_size pixels
//   become invalid.
// gap interpolation: along rows, then along columns, a run of invalid pixels
//   of length <= ipol_gap_width with valid pixels a and b on both ends is
//   filled with (a+b)/2 when |a-b| <= 3 and with min(a,b) otherwise.
// adaptive mean: each valid pixel becomes the weighted mean of the valid
//   pixels of its 5x5 window, weight 1/(1+(d_q-d_p)^2) (edge preserving).
// median: each valid pixel becomes the lower median of the valid pixels of
//   its 3x3 window.
// Order: speckle, gap interpolation, adaptive mean, median.
static void speckle(float* D, int W, int H, const elas_params& p) {
    const size_t N = size_t(W) * H;
    std::vector<int32_t> lab(N, -1);
    std::vector<int32_t> stack;
    std::vector<int32_t> members;
    for (size_t s = 0; s < N; ++s) {
        if (D[s] < 0 || lab[s] >= 0) continue;
        members.clear();
        stack.clear();
        stack.push_back(int32_t(s));
        lab[s] = int32_t(s);
        while (!stack.empty()) {
            int32_t q = stack.back();
            stack.pop_back();
            members.push_back(q);
            int x = q % W, y = q / W;
            const int nx[4] = {x - 1, x + 1, x, x};
            const int ny[4] = {y, y, y - 1, y + 1};
            for (int k = 0; k < 4; ++k) {
                if (nx[k] < 0 || nx[k] >= W || ny[k] < 0 || ny[k] >= H) continue;
                size_t r = size_t(ny[k]) * W + nx[k];
                if (D[r] < 0 || lab[r] >= 0) continue;
                if (std::fabs(D[r] - D[q]) <= p.speckle_sim_threshold) {
                    lab[r] = int32_t(s);
                    stack.push_back(int32_t(r));
                }
            }
        }
        if (int(members.size()) < p.speckle_size)
            for (int32_t q : members) D[q] = -1;
    }
}

static void gap_interpolate(float* D, int W, int H, const elas_params& p) {
    const int gw = p.ipol_gap_width;
    for (int pass = 0; pass < 2; ++pass) {
        const int lines = pass == 0 ? H : W, len = pass == 0 ? W : H;
        for (int l = 0; l < lines; ++l) {
            auto at = [&](int k) -> float& {
                return pass == 0 ? D[size_t(l) * W + k] : D[size_t(k) * W + l];
            };
            int k = 0;
            while (k < len) {
                if (at(k) >= 0) { ++k; continue; }
                int k0 = k;
                while (k < len && at(k) < 0) ++k;
                int k1 = k;  // run [k0, k1)
                if (k0 > 0 && k1 < len && k1 - k0 <= gw) {
                    float a = at(k0 - 1), b = at(k1);
                    float f = std::fabs(a - b) <= 3.0f ? 0.5f * (a + b) : std::min(a, b);
                    for (int q = k0; q < k1; ++q) at(q) = f;
                }
            }
        }
    }
}

static void adaptive_mean(float* D, int W, int H) {
    std::vector<float> S(D, D + size_t(W) * H);
#pragma omp parallel for schedule(static)
    for (int v = 0; v < H; ++v)
        for (int u = 0; u < W; ++u) {
            float dp = S[size_t(v) * W + u];
            if (dp < 0) continue;
            float num = 0.0f, den = 0.0f;
            for (int dy = -2; dy <= 2; ++dy)
                for (int dx = -2; dx <= 2; ++dx) {
                    int x = u + dx, y = v + dy;
                    if (x < 0 || x >= W || y < 0 || y >= H) continue;
                    float dq = S[size_t(y) * W + x];
                    if (dq < 0) continue;
                    float diff = dq - dp;
                    float w = 1.0f / std::fma(diff, diff, 1.0f);
                    num = std::fma(w, dq, num);
                    den += w;
                }
            D[size_t(v) * W + u] = num / den;
        }
}

static void median3(float* D, int W, int H) {
    std::vector<float> S(D, D + size_t(W) * H);
#pragma omp parallel for schedule(static)
    for (int v = 0; v < H; ++v)
        for (int u = 0; u < W; ++u) {
            if (S[size_t(v) * W + u] < 0) continue;
            float vals[9];
            int n = 0;
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    int x = u + dx, y = v + dy;
                    if (x < 0 || x >= W || y < 0 || y >= H) continue;
                    float q = S[size_t(y) * W + x];
                    if (q >= 0) vals[n++] = q;
                }
            std::sort(vals, vals + n);
            D[size_t(v) * W + u] = vals[(n - 1) / 2];
        }
}

int orc_postprocess(float* D, int W, int H, const elas_params* p) {
    if (!D || !p) return ELAS_ERR_INVALID_ARG;
    if (p->speckle_size > 0) speckle(D, W, H, *p);
    if (p->ipol_gap_width > 0) gap_interpolate(D, W, H, *p);
    if (p->filter_adaptive_mean) adaptive_mean(D, W, H);
    if (p->filter_median) median3(D, W, H);
    return ELAS_OK;
}

// ---------------------------------------------------------------------------
// Triangle (the reference's own CPU Delaunay, src/triangle.cpp) through the
// shim compiled into oracle/_ref/libreftriangle.so.
typedef int (*ref_tri_fn)(const float*, int, int32_t*, int);
static ref_tri_fn g_ref_tri = nullptr;

int orc_load_triangle(const char* path) {
    void* h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
    if (!h) return ELAS_ERR_INVALID_ARG;
    g_ref_tri = (ref_tri_fn)dlsym(h, "ref_triangulate");
    return g_ref_tri ? ELAS_OK : ELAS_ERR_INVALID_ARG;
}

// Returns the triangle count (>= 0) or -status.
int orc_triangulate_ref(const float* xy, int n, int32_t* tris, int cap) {
    if (!g_ref_tri) return -ELAS_ERR_UNSUPPORTED;
    return g_ref_tri(xy, n, tris, cap);
}

// ---------------------------------------------------------------------------
// Full pipeline, host sequencing of Elas::process (src/Elas.cu:19-120).
// tri_left/tri_right: if non-null, these triangle lists are used (e.g. the
// CUDA library's) instead of Triangle's.  `dumps` (nullable) receives
// intermediate stages; `post` selects whether post-filters run.
struct orc_dumps {
    uint8_t* desc_left; uint8_t* desc_right;
    int32_t* can_lr; int32_t* can;
    int32_t* support; int32_t* n_support;
    int32_t* grid_left; int32_t* grid_right;
    int32_t* tri_left; int32_t* n_tri_left; int32_t* tri_right; int32_t* n_tri_right; int32_t tri_cap;
    int32_t* prior_left; int32_t* prior_right;
    float* disp_left; float* disp_right;
    float* lr_left; float* lr_right;
};

int orc_process(const uint8_t* L, const uint8_t* R, int W, int H, const elas_params* pp,
                const int32_t* tri_left, int n_tri_left, const int32_t* tri_right, int n_tri_right,
                float* D1, float* D2, orc_dumps* dumps, int threads) {
    if (!L || !R || !pp || !D1 || !D2) return ELAS_ERR_INVALID_ARG;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#endif
    const elas_params& p = *pp;
    Dims g = dims_of(W, H, p);
    const size_t N = size_t(W) * H;
    std::vector<uint8_t> d0(N * 16), d1(N * 16);
    orc_descriptor(L, W, H, d0.data());
    orc_descriptor(R, W, H, d1.data());
    std::vector<int32_t> can(size_t(g.cw) * g.ch);
    orc_support_sweep(d0.data(), d1.data(), W, H, &p, can.data());
    if (dumps && dumps->can_lr) std::copy(can.begin(), can.end(), dumps->can_lr);
    orc_filter_inconsistent(can.data(), g.cw, g.ch, &p);
    orc_filter_redundant(can.data(), g.cw, g.ch);
    int n = orc_support_list(can.data(), g.cw, g.ch, g.step, nullptr);
    std::vector<int32_t> uvd(size_t(3) * std::max(n, 1));
    orc_support_list(can.data(), g.cw, g.ch, g.step, uvd.data());
    if (p.add_corners) {
        // add_corners (declared only in the reference, src/Elas.h:23): the
        // image corners with the disparity of the nearest support point
        // (squared distance, first in list order on ties, 0 without any),
        // plus the two right corners moved by their disparity for the right
        // view.  Row 0's three points lead the list, row H-1's three end it.
        const int cu[4] = {0, W - 1, 0, W - 1}, cv[4] = {0, 0, H - 1, H - 1};
        int d[4] = {0, 0, 0, 0};
        for (int k = 0; k < 4; ++k) {
            long long best = -1;
            for (int i = 0; i < n; ++i) {
                const long long du = uvd[3 * i] - cu[k], dv = uvd[3 * i + 1] - cv[k];
                const long long dist = du * du + dv * dv;
                if (best < 0 || dist < best) { best = dist; d[k] = uvd[3 * i + 2]; }
            }
        }
        std::vector<int32_t> full(size_t(3) * (n + 6));
        const int top[3][3] = {{0, 0, d[0]}, {W - 1, 0, d[1]}, {W - 1 + d[1], 0, d[1]}};
        const int bot[3][3] = {{0, H - 1, d[2]}, {W - 1, H - 1, d[3]}, {W - 1 + d[3], H - 1, d[3]}};
        for (int k = 0; k < 3; ++k)
            for (int j = 0; j < 3; ++j) {
                full[3 * k + j] = top[k][j];
                full[3 * (n + 3 + k) + j] = bot[k][j];
            }
        std::copy(uvd.begin(), uvd.begin() + size_t(3) * n, full.begin() + 9);
        uvd.swap(full);
        n += 6;
    }
    std::vector<int32_t> grid0(size_t(g.gw) * g.gh * (g.D + 2)), grid1(grid0.size());
    orc_grid(can.data(), W, H, &p, grid0.data(), grid1.data());

    std::vector<int32_t> t0, t1;
    const int32_t* tl = tri_left;
    const int32_t* tr = tri_right;
    int ntl = n_tri_left, ntr = n_tri_right;
    if (!tl || !tr) {
        std::vector<float> xy0(size_t(2) * std::max(n, 1)), xy1(xy0.size());
        for (int i = 0; i < n; ++i) {
            xy0[2 * i] = float(uvd[3 * i]);
            xy0[2 * i + 1] = float(uvd[3 * i + 1]);
            xy1[2 * i] = float(uvd[3 * i] - uvd[3 * i + 2]);
            xy1[2 * i + 1] = float(uvd[3 * i + 1]);
        }
        int cap = 2 * n + 16;
        if (!tl) {
            t0.resize(size_t(3) * cap);
            ntl = orc_triangulate_ref(xy0.data(), n, t0.data(), cap);
            if (ntl < 0) return -ntl;
            tl = t0.data();
        }
        if (!tr) {
            t1.resize(size_t(3) * cap);
            ntr = orc_triangulate_ref(xy1.data(), n, t1.data(), cap);
            if (ntr < 0) return -ntr;
            tr = t1.data();
        }
    }
    std::vector<int32_t> pr0(N), pr1(N);
    orc_prior(can.data(), g.cw, g.step, uvd.data(), tl, ntl, 0, W, H, pr0.data());
    orc_prior(can.data(), g.cw, g.step, uvd.data(), tr, ntr, 1, W, H, pr1.data());
    orc_dense(grid0.data(), d0.data(), d1.data(), pr0.data(), 0, W, H, &p, D1);
    orc_dense(grid1.data(), d0.data(), d1.data(), pr1.data(), 1, W, H, &p, D2);
    // Subsampling (the project's own definition; the reference declares only
    // the parameter, src/Elas.h:37-39): the maps keep every second row and
    // column, (W / 2) x (H / 2), each value the full-resolution MAP
    // disparity of pixel (2u, 2v); L/R check and post-filters then run on
    // the half-size maps.  D1 / D2 then hold (W / 2) * (H / 2) values.
    const int Wo = p.subsampling ? W / 2 : W, Ho = p.subsampling ? H / 2 : H;
    const size_t No = size_t(Wo) * Ho;
    if (p.subsampling) {
        for (int v = 0; v < Ho; ++v)
            for (int u = 0; u < Wo; ++u) {
                D1[size_t(v) * Wo + u] = D1[size_t(2 * v) * W + 2 * u];
                D2[size_t(v) * Wo + u] = D2[size_t(2 * v) * W + 2 * u];
            }
    }
    if (dumps) {
        if (dumps->desc_left) std::copy(d0.begin(), d0.end(), dumps->desc_left);
        if (dumps->desc_right) std::copy(d1.begin(), d1.end(), dumps->desc_right);
        if (dumps->can) std::copy(can.begin(), can.end(), dumps->can);
        if (dumps->n_support) *dumps->n_support = n;
        if (dumps->support) std::copy(uvd.begin(), uvd.begin() + size_t(3) * n, dumps->support);
        if (dumps->grid_left) std::copy(grid0.begin(), grid0.end(), dumps->grid_left);
        if (dumps->grid_right) std::copy(grid1.begin(), grid1.end(), dumps->grid_right);
        if (dumps->n_tri_left) *dumps->n_tri_left = ntl;
        if (dumps->n_tri_right) *dumps->n_tri_right = ntr;
        if (dumps->tri_left && ntl <= dumps->tri_cap) std::copy(tl, tl + size_t(3) * ntl, dumps->tri_left);
        if (dumps->tri_right && ntr <= dumps->tri_cap) std::copy(tr, tr + size_t(3) * ntr, dumps->tri_right);
        if (dumps->prior_left) std::copy(pr0.begin(), pr0.end(), dumps->prior_left);
        if (dumps->prior_right) std::copy(pr1.begin(), pr1.end(), dumps->prior_right);
        if (dumps->disp_left) std::copy(D1, D1 + No, dumps->disp_left);
        if (dumps->disp_right) std::copy(D2, D2 + No, dumps->disp_right);
    }
    orc_lr_scaled(D1, D2, Wo, Ho, &p, p.subsampling ? 0.5f : 1.0f);
    if (dumps) {
        if (dumps->lr_left) std::copy(D1, D1 + No, dumps->lr_left);
        if (dumps->lr_right) std::copy(D2, D2 + No, dumps->lr_right);
    }
    orc_postprocess(D1, Wo, Ho, &p);
    if (!p.postprocess_only_left) orc_postprocess(D2, Wo, Ho, &p);
    return ELAS_OK;
}

// ---------------------------------------------------------------------------
// Exact Delaunay checks on integer coordinates (int64 predicates).
//
// The canonical triangulation is the Delaunay triangulation under symbolic
// perturbation: point i is lifted to x^2+y^2 - eps^(i+1) (a smaller index
// gets the larger infinitesimal weight).  When incircle(a,b,c,d) == 0 the
// point of {a,b,c,d} with the smallest index m decides: d is inside iff
// m == d, or the barycentric coordinate of d for vertex m is negative.
// That triangulation is unique, so a valid triangulation of the convex hull
// whose every interior edge passes this test is it.
static inline int64_t orient(const int32_t* P, int a, int b, int c) {
    int64_t ax = P[2 * a], ay = P[2 * a + 1];
    int64_t bx = P[2 * b], by = P[2 * b + 1];
    int64_t cx = P[2 * c], cy = P[2 * c + 1];
    return (bx - ax) * (cy - ay) - (by - ay) * (cx - ax);
}
static inline int64_t incircle(const int32_t* P, int a, int b, int c, int d) {
    int64_t dx = P[2 * d], dy = P[2 * d + 1];
    int64_t adx = P[2 * a] - dx, ady = P[2 * a + 1] - dy;
    int64_t bdx = P[2 * b] - dx, bdy = P[2 * b + 1] - dy;
    int64_t cdx = P[2 * c] - dx, cdy = P[2 * c + 1] - dy;
    int64_t al = adx * adx + ady * ady, bl = bdx * bdx + bdy * bdy, cl = cdx * cdx + cdy * cdy;
    return adx * (bdy * cl - bl * cdy) - ady * (bdx * cl - bl * cdx) + al * (bdx * cdy - bdy * cdx);
}
static bool inside_sos(const int32_t* P, int a, int b, int c, int d) {
    int64_t det = incircle(P, a, b, c, d);
    if (det != 0) return det > 0;
    int m = std::min(std::min(a, b), std::min(c, d));
    if (m == d) return true;
    if (m == a) return orient(P, d, b, c) < 0;
    if (m == b) return orient(P, a, d, c) < 0;
    return orient(P, a, b, d) < 0;
}

int orc_inside_sos(const int32_t* P, int a, int b, int c, int d) { return inside_sos(P, a, b, c, d); }
long long orc_incircle(const int32_t* P, int a, int b, int c, int d) { return incircle(P, a, b, c, d); }

// stats[0] triangles, [1] non-positive orientation, [2] edges used by more
// than two triangles or twice in one direction, [3] interior edges failing
// the (SoS) Delaunay test, [4] hull edges with a point strictly outside,
// [5] distinct points not used by any triangle, [6] Euler mismatch
// (t != 2n - 2 - h), [7] hull edge count.  Duplicated coordinates: only the
// lowest index of a group may be used.  Returns 0 if every check passes.
int orc_delaunay_check(const int32_t* P, int n, const int32_t* tris, int nt, long long* stats) {
    long long st[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    st[0] = nt;
    // canonical representative of duplicated points
    std::vector<int> order(n), rep(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](int a, int b) {
        if (P[2 * a] != P[2 * b]) return P[2 * a] < P[2 * b];
        if (P[2 * a + 1] != P[2 * b + 1]) return P[2 * a + 1] < P[2 * b + 1];
        return a < b;
    });
    int n_distinct = 0;
    for (int i = 0; i < n; ++i) {
        int k = order[i];
        if (i > 0 && P[2 * k] == P[2 * order[i - 1]] && P[2 * k + 1] == P[2 * order[i - 1] + 1])
            rep[k] = rep[order[i - 1]];
        else { rep[k] = k; ++n_distinct; }
    }
    if (nt == 0) {
        // no triangles is right only when every point is collinear (or n < 3)
        bool collinear = true;
        for (int i = 2; i < n && collinear; ++i)
            if (orient(P, order[0], order[n - 1], i) != 0) collinear = false;
        st[5] = collinear ? 0 : n_distinct;
        if (stats) std::memcpy(stats, st, sizeof(st));
        return collinear ? 0 : 1;
    }
    std::vector<char> used(n, 0);
    struct E { uint64_t key; int t, s; };
    std::vector<E> edges;
    edges.reserve(size_t(3) * nt);
    for (int t = 0; t < nt; ++t) {
        const int* v = tris + 3 * t;
        for (int k = 0; k < 3; ++k) {
            if (v[k] < 0 || v[k] >= n || rep[v[k]] != v[k]) { st[1]++; continue; }
            used[v[k]] = 1;
        }
        if (orient(P, v[0], v[1], v[2]) <= 0) st[1]++;
        for (int k = 0; k < 3; ++k) {
            uint32_t a = uint32_t(v[k]), b = uint32_t(v[(k + 1) % 3]);
            uint64_t key = a < b ? (uint64_t(a) << 32 | b) : (uint64_t(b) << 32 | a);
            edges.push_back({key, t, k});
        }
    }
    std::sort(edges.begin(), edges.end(), [](const E& x, const E& y) {
        return x.key != y.key ? x.key < y.key : (x.t != y.t ? x.t < y.t : x.s < y.s);
    });
    std::vector<std::pair<int, int>> hull;
    for (size_t i = 0; i < edges.size();) {
        size_t j = i;
        while (j < edges.size() && edges[j].key == edges[i].key) ++j;
        if (j - i == 1) {
            const int* v = tris + 3 * edges[i].t;
            hull.push_back({v[edges[i].s], v[(edges[i].s + 1) % 3]});
        } else if (j - i == 2) {
            const int* v1 = tris + 3 * edges[i].t;
            const int* v2 = tris + 3 * edges[i + 1].t;
            int a = v1[edges[i].s], b = v1[(edges[i].s + 1) % 3];
            int a2 = v2[edges[i + 1].s], b2 = v2[(edges[i + 1].s + 1) % 3];
            if (!(a == b2 && b == a2)) st[2]++;
            int c = v1[(edges[i].s + 2) % 3];
            int d = v2[(edges[i + 1].s + 2) % 3];
            if (inside_sos(P, a, b, c, d)) st[3]++;
            if (inside_sos(P, a2, b2, d, c)) st[3]++;
        } else {
            st[2]++;
        }
        i = j;
    }
    st[7] = (long long)hull.size();
    // every hull edge a->b must have no point strictly to its right
    for (auto& e : hull) {
        for (int i = 0; i < n; ++i)
            if (orient(P, e.first, e.second, i) < 0) { st[4]++; break; }
    }
    for (int i = 0; i < n; ++i)
        if (rep[i] == i && !used[i]) st[5]++;
    if (nt > 0) {
        long long expect = 2LL * n_distinct - 2 - (long long)hull.size();
        if (expect != nt) st[6] = 1;
    }
    if (stats) std::memcpy(stats, st, sizeof(st));
    return (st[1] || st[2] || st[3] || st[4] || st[5] || st[6]) ? 1 : 0;
}

// Compare two triangle sets on the same points.  Triangles are normalised
// (rotation with the smallest index first, duplicate points mapped to the
// lowest index).  stats[0] common, [1] only in A, [2] only in B, [3] of the
// differing triangles, those with a fourth point exactly on their
// circumcircle (co-circular, so not unique), [4] differing triangles that
// are not explained that way.
int orc_tri_compare(const int32_t* P, int n, const int32_t* A, int na, const int32_t* B, int nb,
                    long long* stats) {
    std::vector<int> order(n), rep(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](int a, int b) {
        if (P[2 * a] != P[2 * b]) return P[2 * a] < P[2 * b];
        if (P[2 * a + 1] != P[2 * b + 1]) return P[2 * a + 1] < P[2 * b + 1];
        return a < b;
    });
    for (int i = 0; i < n; ++i) {
        int k = order[i];
        if (i > 0 && P[2 * k] == P[2 * order[i - 1]] && P[2 * k + 1] == P[2 * order[i - 1] + 1])
            rep[k] = rep[order[i - 1]];
        else rep[k] = k;
    }
    auto norm = [&](const int32_t* t) {
        int a = rep[t[0]], b = rep[t[1]], c = rep[t[2]];
        while (a > b || a > c) { int x = a; a = b; b = c; c = x; }
        return std::array<int, 3>{a, b, c};
    };
    std::vector<std::array<int, 3>> sa, sb;
    for (int i = 0; i < na; ++i) sa.push_back(norm(A + 3 * i));
    for (int i = 0; i < nb; ++i) sb.push_back(norm(B + 3 * i));
    std::sort(sa.begin(), sa.end());
    std::sort(sb.begin(), sb.end());
    std::vector<std::array<int, 3>> oa, ob, common;
    std::set_difference(sa.begin(), sa.end(), sb.begin(), sb.end(), std::back_inserter(oa));
    std::set_difference(sb.begin(), sb.end(), sa.begin(), sa.end(), std::back_inserter(ob));
    std::set_intersection(sa.begin(), sa.end(), sb.begin(), sb.end(), std::back_inserter(common));
    long long explained = 0, unexplained = 0;
    auto cocircular = [&](const std::array<int, 3>& t) {
        for (int i = 0; i < n; ++i) {
            if (rep[i] != i || i == t[0] || i == t[1] || i == t[2]) continue;
            if (incircle(P, t[0], t[1], t[2], i) == 0) return true;
        }
        return false;
    };
    for (auto& t : oa) (cocircular(t) ? explained : unexplained)++;
    for (auto& t : ob) (cocircular(t) ? explained : unexplained)++;
    if (stats) {
        stats[0] = (long long)common.size();
        stats[1] = (long long)oa.size();
        stats[2] = (long long)ob.size();
        stats[3] = explained;
        stats[4] = unexplained;
    }
    return unexplained ? 1 : 0;
}

}  // extern "C"
