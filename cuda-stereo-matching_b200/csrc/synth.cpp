// Seeded synthetic stereo scenes: slanted textured planes, z-buffered
// right view, float ground truth.  The reference ships no generator (its only
// inputs are the img/*.pgm demo pairs, src/Main.cu:108-113); these scenes
// stand in for the KITTI / Middlebury shapes the benchmark configurations
// name.
//
// Scene model
//   * plane k:  d_k(u,v) = a_k*u + b_k*v + c_k (+ ripple), u,v in LEFT-view
//     pixel coordinates; plane 0 is the background and covers everything,
//     the others cover an ellipse or a rectangle (a ground plane covers the
//     lower half of the image).
//   * the visible plane at a left pixel is the covering plane with the
//     largest disparity (z-buffer: nearer wins).
//   * texture: one toroidal field of Gaussian-blurred (sigma 1.5) uniform
//     noise, normalised to mean 128 / std 40; plane k samples it at its own
//     offset, so textures move with the surface between the two views.
//     Textureless patches are rectangles (left-view coordinates) of one
//     constant intensity.
//   * right view: pixel x of row v shows the surface point whose left
//     coordinate u solves u = x + d_k(u,v) (fixed-point iteration), again
//     z-buffered over planes; intensity is bilinear in u plus N(0, 2) noise.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>

#include "../../include/elas_b200.h"

namespace {

struct Rng {  // xoshiro256** seeded by splitmix64
    uint64_t s[4];
    explicit Rng(uint64_t seed) {
        uint64_t x = seed;
        for (int i = 0; i < 4; ++i) {
            x += 0x9E3779B97F4A7C15ull;
            uint64_t z = x;
            z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
            z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
            s[i] = z ^ (z >> 31);
        }
    }
    static uint64_t rotl(uint64_t v, int k) { return (v << k) | (v >> (64 - k)); }
    uint64_t next() {
        uint64_t r = rotl(s[1] * 5, 7) * 9;
        uint64_t t = s[1] << 17;
        s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
        s[2] ^= t; s[3] = rotl(s[3], 45);
        return r;
    }
    double uni() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
    double uni(double a, double b) { return a + (b - a) * uni(); }
    double gauss() {
        double u1 = uni(), u2 = uni();
        if (u1 < 1e-300) u1 = 1e-300;
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
};

struct Preset {
    int w, h, dmax;
    int n_planes;          // including the background
    double max_slope;      // |a|,|b| bound of the non-ground planes
    double near_max;       // largest plane disparity
    bool ground;           // ground plane over the lower half
    double ground_b;
    double textureless_frac;  // fraction of the image covered by flat patches
    int textureless_patch;    // patch side (0 = derive from the fraction)
    double ripple;         // sinusoidal ripple amplitude in px
};

Preset preset_of(int id) {
    switch (id) {
    case 0: return {450, 375, 63, 6, 0.05, 60.0, false, 0.0, 0.0, 40, 0.0};
    case 1: return {1242, 375, 255, 12, 0.05, 200.0, true, 0.3, 0.08, 0, 0.0};
    case 2: return {2880, 1988, 511, 40, 0.05, 480.0, false, 0.0, 0.02, 0, 2.0};
    default: return {640, 480, 128, 8, 0.05, 0.0, false, 0.0, 0.03, 0, 0.0};
    }
}

struct Plane {
    double a, b, c;
    int shape;                 // 0 = everywhere, 1 = ellipse, 2 = rectangle, 3 = lower half
    double cx, cy, rx, ry;     // ellipse / rectangle extent (left view)
    double ox, oy;             // texture offset
    double ripple, lu, lv, pu, pv;
};

struct Patch { int u0, v0, u1, v1; float value; };

inline bool covers(const Plane& p, double u, double v, int H) {
    switch (p.shape) {
    case 0: return true;
    case 1: { double x = (u - p.cx) / p.rx, y = (v - p.cy) / p.ry; return x * x + y * y <= 1.0; }
    case 2: return std::fabs(u - p.cx) <= p.rx && std::fabs(v - p.cy) <= p.ry;
    default: return v >= 0.5 * H;
    }
}

inline double disp_of(const Plane& p, double u, double v) {
    double d = p.a * u + p.b * v + p.c;
    if (p.ripple != 0.0)
        d += p.ripple * std::sin(6.283185307179586 * u / p.lu + p.pu) *
             std::sin(6.283185307179586 * v / p.lv + p.pv);
    return d;
}

struct Scene {
    int W, H, D;
    std::vector<Plane> planes;
    std::vector<Patch> patches;
    int FW, FH;                 // texture field size (toroidal)
    std::vector<float> field;
};

// Range of a plane's disparity over the image box, used to keep every
// plane inside [lo, hi].
void plane_range(const Plane& p, int W, int H, double& mn, double& mx) {
    double xs[2] = {0.0, double(W - 1)}, ys[2] = {0.0, double(H - 1)};
    if (p.shape == 1 || p.shape == 2) {
        xs[0] = std::max(0.0, p.cx - p.rx); xs[1] = std::min(double(W - 1), p.cx + p.rx);
        ys[0] = std::max(0.0, p.cy - p.ry); ys[1] = std::min(double(H - 1), p.cy + p.ry);
    } else if (p.shape == 3) {
        ys[0] = 0.5 * H;
    }
    mn = 1e300; mx = -1e300;
    for (double x : xs) for (double y : ys) {
        double d = p.a * x + p.b * y + p.c;
        mn = std::min(mn, d); mx = std::max(mx, d);
    }
    mn -= std::fabs(p.ripple); mx += std::fabs(p.ripple);
}

void fit_plane(Plane& p, int W, int H, double lo, double hi) {
    double mn, mx;
    plane_range(p, W, H, mn, mx);
    if (mx - mn > hi - lo) {  // too steep for the range: flatten
        p.a *= 0.5; p.b *= 0.5;
        plane_range(p, W, H, mn, mx);
        if (mx - mn > hi - lo) { p.a = 0; p.b = 0; plane_range(p, W, H, mn, mx); }
    }
    if (mn < lo) p.c += lo - mn;
    plane_range(p, W, H, mn, mx);
    if (mx > hi) p.c -= mx - hi;
}

void build_field(Scene& s, Rng& rng) {
    s.FW = s.W + 64;
    s.FH = s.H + 64;
    const int FW = s.FW, FH = s.FH;
    std::vector<float> a(size_t(FW) * FH), b(size_t(FW) * FH);
    for (auto& x : a) x = float(rng.uni());
    // separable Gaussian, sigma 1.5, radius 5, toroidal
    const double sig = 1.5;
    const int R = 5;
    double k[2 * R + 1], ks = 0;
    for (int i = -R; i <= R; ++i) { k[i + R] = std::exp(-0.5 * i * i / (sig * sig)); ks += k[i + R]; }
    for (auto& x : k) x /= ks;
    for (int y = 0; y < FH; ++y)
        for (int x = 0; x < FW; ++x) {
            double acc = 0;
            for (int i = -R; i <= R; ++i) acc += k[i + R] * a[size_t(y) * FW + (x + i + FW) % FW];
            b[size_t(y) * FW + x] = float(acc);
        }
    for (int y = 0; y < FH; ++y)
        for (int x = 0; x < FW; ++x) {
            double acc = 0;
            for (int i = -R; i <= R; ++i) acc += k[i + R] * b[size_t((y + i + FH) % FH) * FW + x];
            a[size_t(y) * FW + x] = float(acc);
        }
    double m = 0, m2 = 0;
    for (float x : a) { m += x; m2 += double(x) * x; }
    m /= a.size();
    double sd = std::sqrt(std::max(1e-12, m2 / a.size() - m * m));
    s.field.resize(a.size());
    for (size_t i = 0; i < a.size(); ++i) s.field[i] = float(128.0 + 40.0 * (a[i] - m) / sd);
}

inline double field_at(const Scene& s, double x, int y) {
    // bilinear in x, nearest row; toroidal
    double fx = std::floor(x);
    double t = x - fx;
    long xi = long(fx) % s.FW;
    if (xi < 0) xi += s.FW;
    long xj = (xi + 1) % s.FW;
    long yi = y % s.FH;
    if (yi < 0) yi += s.FH;
    const float* row = &s.field[size_t(yi) * s.FW];
    return (1.0 - t) * row[xi] + t * row[xj];
}

inline double intensity(const Scene& s, int k, double u, int v) {
    for (const Patch& p : s.patches)
        if (u >= p.u0 && u < p.u1 && v >= p.v0 && v < p.v1) return p.value;
    const Plane& p = s.planes[k];
    return field_at(s, u + p.ox, int(v + p.oy));
}

inline uint8_t quant(double x) {
    long r = std::lround(x);
    return uint8_t(r < 0 ? 0 : (r > 255 ? 255 : r));
}

Scene make_scene(int preset, uint64_t seed, int W, int H, int D) {
    Preset pr = preset_of(preset);
    Scene s;
    s.W = W; s.H = H; s.D = D;
    Rng rng(seed * 0x2545F4914F6CDD1Dull + uint64_t(preset) + 1);
    const double lo = std::max(2.0, 0.04 * D), hi_all = 0.92 * D;
    const double near_max = pr.near_max > 0 ? std::min(pr.near_max, hi_all) : hi_all;

    // background
    Plane bg{};
    bg.shape = 0;
    bg.a = rng.uni(-pr.max_slope, pr.max_slope) * 0.5;
    bg.b = rng.uni(-pr.max_slope, pr.max_slope) * 0.5;
    bg.c = rng.uni(lo, lo + 0.25 * (near_max - lo));
    fit_plane(bg, W, H, lo, lo + 0.35 * (near_max - lo));
    s.planes.push_back(bg);

    int remaining = pr.n_planes - 1;
    if (pr.ground && remaining > 0) {
        Plane g{};
        g.shape = 3;
        g.a = 0.0;
        g.b = pr.ground_b;
        g.c = lo + 2.0 - pr.ground_b * 0.5 * H;   // d = lo+2 at mid height, grows downward
        fit_plane(g, W, H, lo, near_max);
        s.planes.push_back(g);
        --remaining;
    }
    for (int i = 0; i < remaining; ++i) {
        Plane p{};
        p.shape = (rng.uni() < 0.6) ? 1 : 2;
        p.cx = rng.uni(0.0, W);
        p.cy = rng.uni(0.0, H);
        double scale = std::min(W, H);
        p.rx = rng.uni(0.06, 0.22) * scale * (W > 2 * H ? 1.6 : 1.0);
        p.ry = rng.uni(0.06, 0.22) * scale;
        p.a = rng.uni(-pr.max_slope, pr.max_slope);
        p.b = rng.uni(-pr.max_slope, pr.max_slope);
        // nearer planes for later indices so the z-buffer has work to do
        double target = lo + (near_max - lo) * (0.25 + 0.75 * rng.uni());
        p.c = target - p.a * p.cx - p.b * p.cy;
        fit_plane(p, W, H, lo, near_max);
        s.planes.push_back(p);
    }
    for (size_t k = 0; k < s.planes.size(); ++k) {
        Plane& p = s.planes[k];
        p.ox = rng.uni(0.0, 4096.0);
        p.oy = std::floor(rng.uni(0.0, 4096.0));
        if (pr.ripple > 0) {
            p.ripple = pr.ripple;
            p.lu = rng.uni(40.0, 120.0);
            p.lv = rng.uni(40.0, 120.0);
            p.pu = rng.uni(0.0, 6.283185307179586);
            p.pv = rng.uni(0.0, 6.283185307179586);
            fit_plane(p, W, H, lo, k == 0 ? lo + 0.35 * (near_max - lo) : near_max);
        }
    }
    // textureless patches
    int n_patch = 0, side = pr.textureless_patch;
    if (pr.textureless_frac > 0.0) {
        if (side <= 0) side = std::max(16, int(std::sqrt(pr.textureless_frac * W * H / 6.0)));
        n_patch = std::max(1, int(std::lround(pr.textureless_frac * W * H / double(side * side))));
    } else if (side > 0) {
        n_patch = 2;
    }
    for (int i = 0; i < n_patch; ++i) {
        Patch p;
        p.u0 = int(rng.uni(0.0, std::max(1, W - side)));
        p.v0 = int(rng.uni(0.0, std::max(1, H - side)));
        p.u1 = p.u0 + side;
        p.v1 = p.v0 + side;
        p.value = float(std::floor(rng.uni(60.0, 200.0)));
        s.patches.push_back(p);
    }
    build_field(s, rng);
    return s;
}

}  // namespace

extern "C" int elas_b200_synth_dims(int preset, int32_t* w, int32_t* h, int32_t* disp_max) {
    if (preset < 0 || preset > 3) return ELAS_ERR_INVALID_ARG;
    Preset p = preset_of(preset);
    if (w) *w = p.w;
    if (h) *h = p.h;
    if (disp_max) *disp_max = p.dmax;
    return ELAS_OK;
}

extern "C" int elas_b200_synth_pair(int preset, uint64_t seed, int32_t w, int32_t h, int32_t disp_max,
                                    uint8_t* left, uint8_t* right, float* gt_left, float* gt_right) {
    if (preset < 0 || preset > 3 || !left || !right) return ELAS_ERR_INVALID_ARG;
    Preset pr = preset_of(preset);
    const int W = w > 0 ? w : pr.w;
    const int H = h > 0 ? h : pr.h;
    const int D = disp_max > 0 ? disp_max : pr.dmax;
    if (W < 16 || H < 16 || D < 8) return ELAS_ERR_INVALID_ARG;
    Scene s = make_scene(preset, seed, W, H, D);
    const int NP = int(s.planes.size());

    // left view
#pragma omp parallel for schedule(static)
    for (int v = 0; v < H; ++v) {
        for (int u = 0; u < W; ++u) {
            int best = 0;
            double bd = -1e300;
            for (int k = 0; k < NP; ++k) {
                if (!covers(s.planes[k], u, v, H)) continue;
                double d = disp_of(s.planes[k], u, v);
                if (d > bd) { bd = d; best = k; }
            }
            left[size_t(v) * W + u] = quant(intensity(s, best, u, v));
            if (gt_left) gt_left[size_t(v) * W + u] = float(bd);
        }
    }
    // right view: inverse warp with z-buffer, noise sigma 2 (per-row streams)
#pragma omp parallel for schedule(static)
    for (int v = 0; v < H; ++v) {
        Rng nrng(seed ^ (0xA5A5A5A5ull + uint64_t(v) * 0x9E3779B97F4A7C15ull));
        for (int x = 0; x < W; ++x) {
            int best = -1;
            double bd = -1e300, bu = 0;
            for (int k = 0; k < NP; ++k) {
                const Plane& p = s.planes[k];
                // closed-form solution of u = x + a*u + b*v + c, refined for the ripple
                double u = (x + p.b * v + p.c) / (1.0 - p.a);
                if (p.shape == 1 || p.shape == 2) {
                    double m = 2.0 * std::fabs(p.ripple) + 1.0;
                    if (u < p.cx - p.rx - m || u > p.cx + p.rx + m || v < p.cy - p.ry || v > p.cy + p.ry) continue;
                }
                if (p.ripple != 0.0)
                    for (int it = 0; it < 6; ++it) u = x + disp_of(p, u, v);
                if (!covers(p, u, v, H)) continue;
                double d = u - x;
                if (d > bd) { bd = d; best = k; bu = u; }
            }
            double val = intensity(s, best, bu, v) + 2.0 * nrng.gauss();
            right[size_t(v) * W + x] = quant(val);
            if (gt_right) gt_right[size_t(v) * W + x] = float(bd);
        }
    }
    return ELAS_OK;
}
