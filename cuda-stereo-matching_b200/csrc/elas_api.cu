// C ABI and host orchestration of the B200 ELAS pipeline.
//
// Replaces Elas::process and its helpers (src/Elas.cu:19-565).  Differences
// in how the work is organised, not in what is computed:
//  * one device workspace arena per handle, grown on demand; the reference
//    allocates (and partly leaks, src/Elas.cu:349-371) every buffer per call;
//  * no host round trips inside the pipeline: the support-point count and the
//    triangle counts stay on the device (the reference reads num_sp back,
//    src/Elas.cu:374, and triangulates on the CPU, :282-328);
//  * errors are returned as status codes instead of exit() (src/Utils.h:11-38).
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "../../include/elas_b200.h"
#include "common.cuh"
#include "kernels.h"
#include "proposal.h"

using namespace elas;

struct elas_handle {
    elas_params params;
    int device = 0;
    int num_sms = 0;
    int cluster_size = 0;   // CTAs per cluster of the Delaunay flip kernel (0 = global fallback only)
    std::string last_error;
    int64_t launches = 0;

    // fallback switches for tests (elas_b200_set_test_mode)
    int test_flags = 0;
    int flip_round_limit = 0;     // 0 = the library's own bound

    // workspace arena
    void* arena = nullptr;
    size_t arena_bytes = 0;
    Geom g{};          // geometry of the last call
    bool have_last = false;

    uint8_t *img0 = nullptr, *img1 = nullptr;
    uint4 *desc0 = nullptr, *desc1 = nullptr;
    int32_t *can_lr = nullptr, *can = nullptr, *row_cnt = nullptr, *row_off = nullptr;
    int32_t *uvd = nullptr, *x0 = nullptr, *x1 = nullptr, *y = nullptr;
    uint32_t *gtmp0 = nullptr, *gtmp1 = nullptr, *grid0 = nullptr, *grid1 = nullptr;
    DelDev del[2]{};
    uint32_t *prior0 = nullptr, *prior1 = nullptr;
    void* rast = nullptr;   // per-triangle plane/edge set-up of both views
    PriorTiles ptiles{};    // triangles binned by prior tile, both views
    float *raw0 = nullptr, *raw1 = nullptr, *lr0 = nullptr, *lr1 = nullptr;
    float *out0 = nullptr, *out1 = nullptr;
    float* tmp[2] = {nullptr, nullptr};          // post-filter ping-pong buffer per view
    int32_t* lab[2] = {nullptr, nullptr};        // union-find labels per view
    int32_t* root[2] = {nullptr, nullptr};       // union-find roots per view
    int32_t* usize[2] = {nullptr, nullptr};      // segment sizes per view
    int32_t* roots[2] = {nullptr, nullptr};      // tile-local roots of the speckle labelling per view
    unsigned* err = nullptr;
    unsigned* err_host = nullptr;   // pinned copy of the error word (read back after each host-buffer call)

    // side stream for the disparity grid, which runs beside the Delaunay
    // and prior stages (it needs only the support list)
    cudaStream_t side = nullptr;
    cudaEvent_t side_fork = nullptr, side_join = nullptr;

    // per-stage timing
    bool timing = false;
    cudaEvent_t ev[ELAS_TIME_COUNT + 1] = {};

    // dense-matching autotuner: (width class, disp_max) -> threads per CTA
    std::map<std::pair<int, int>, int> dense_threads;

    // batch execution: one worker (own workspace and stream) per pair
    std::vector<elas_handle*> slots;
    std::vector<cudaStream_t> slot_streams;
    std::vector<cudaEvent_t> slot_done;
    cudaEvent_t batch_start = nullptr;
    cudaEvent_t lat_start = nullptr;          // per-pair latency marks (graph nodes when captured)
    std::vector<cudaEvent_t> lat_done;
    cudaStream_t own_stream = nullptr;
    bool use_graphs = true;
    cudaGraphExec_t graph_exec = nullptr;
    std::vector<int64_t> graph_sig;   // what the cached graph was captured for
    int last_batch = 0;
    elas_handle* owner = nullptr;     // the user's handle, for a batch worker

    // single-pair CUDA graph: captured on the second call with the same
    // signature (buffers, size, parameters, workspace), replayed after that
    cudaGraphExec_t single_exec = nullptr;
    std::vector<int64_t> single_sig, single_seen;
    long long single_launches = 0;

    // learned support-point proposal (off until weights are set)
    bool prop = false;
    int prop_version = 0;             // bumped by every elas_b200_set_proposal
    std::vector<float> prop_params;   // host copy (batch workers upload it)
    pn::InferWeights pw{};
    __nv_bfloat16 *pn_in = nullptr, *pn_a0 = nullptr, *pn_a1 = nullptr, *pn_out = nullptr;
    uint32_t* pn_bins = nullptr;
    int32_t* pn_stats = nullptr;      // [4]: settled by the proposal, fell back, -, -
    size_t pn_map_elems = 0, pn_cands = 0;
    bool pn_used = false;             // the last call ran the proposal
};

namespace {

int fail(elas_handle* h, int code, const std::string& msg) {
    if (h) h->last_error = msg;
    return code;
}

int cuda_fail(elas_handle* h, cudaError_t e, const char* where) {
    return fail(h, ELAS_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                                      \
    do {                                                              \
        cudaError_t e_ = (call);                                      \
        if (e_ != cudaSuccess) return cuda_fail(h, e_, #call);        \
    } while (0)

size_t align_up(size_t x) { return (x + 255) & ~size_t(255); }

uint32_t next_pow2(size_t x) {
    uint32_t c = 64;
    while (c < x) c <<= 1;
    return c;
}

int penalty(int dd, const elas_params& p);

int check_params(const elas_params& p, std::string& why) {
    if (p.candidate_stepsize < 1) { why = "candidate_stepsize must be >= 1"; return ELAS_ERR_INVALID_ARG; }
    if (p.grid_size < 1) { why = "grid_size must be >= 1"; return ELAS_ERR_INVALID_ARG; }
    if (p.disp_max < 1 || p.disp_max > 4095) { why = "disp_max must be in [1, 4095]"; return ELAS_ERR_INVALID_ARG; }
    if (p.disp_min > p.disp_max) { why = "disp_min > disp_max"; return ELAS_ERR_INVALID_ARG; }
    if (!(p.beta > 0.0f) || !(p.gamma > 0.0f) || !(p.sigma > 0.0f) || !(p.sradius >= 0.0f)) {
        why = "beta, gamma, sigma must be > 0 and sradius >= 0";
        return ELAS_ERR_INVALID_ARG;
    }
    float r = std::max(std::ceil(p.sigma * p.sradius), 2.0f);
    if (r > 15.0f) { why = "sigma*sradius must be <= 15"; return ELAS_ERR_UNSUPPORTED; }
    // dense matching packs energy * 4096 + d into an int: the prior penalty
    // (negative, growing as 1/beta) must stay above -2^18
    for (int dd = 0; dd <= int(r); ++dd)
        if (penalty(dd, p) < -(1 << 18)) { why = "beta is too small (prior penalty below -2^18)"; return ELAS_ERR_UNSUPPORTED; }
    if (p.incon_window_size < 0) { why = "incon_window_size must be >= 0"; return ELAS_ERR_INVALID_ARG; }
    return ELAS_OK;
}

// P(|d - d_plane|) of kerComputeDisparity (src/Kernels/KerComputeDisparity.cu:
// 270-271) evaluated once on the host: float exp/log, double division by beta.
int penalty(int dd, const elas_params& p) {
    float two_sigma_squared = 2 * p.sigma * p.sigma;
    float e = std::exp(float(-dd * dd) / two_sigma_squared);
    float num = -std::log(p.gamma + e) + std::log(p.gamma);
    return int32_t(double(num) / double(p.beta));
}

DevParams dev_params(const elas_params& p) {
    DevParams d{};
    d.support_threshold = p.support_threshold;
    d.support_texture = p.support_texture;
    d.lr_threshold = p.lr_threshold;
    d.incon_window = p.incon_window_size;
    d.incon_threshold = p.incon_threshold;
    d.incon_min_support = p.incon_min_support;
    d.match_texture = p.match_texture;
    d.plane_radius = int32_t(std::max(float(std::ceil(p.sigma * p.sradius)), 2.0f));
    for (int i = 0; i < 16; ++i) d.penalty[i] = i <= d.plane_radius ? penalty(i, p) : 0;
    d.window_negative = 1;
    for (int i = 0; i <= d.plane_radius; ++i)
        if (d.penalty[i] >= 0) d.window_negative = 0;
    d.speckle_sim_threshold = p.speckle_sim_threshold;
    d.speckle_size = p.speckle_size;
    d.ipol_gap_width = p.ipol_gap_width;
    return d;
}

Geom geom_of(int W, int H, const elas_params& p) {
    Geom g;
    g.W = W; g.H = H;
    g.step = p.candidate_stepsize;
    g.gs = p.grid_size;
    g.cw = W / g.step;
    g.ch = H / g.step;
    g.gw = int(std::ceil(float(W) / float(g.gs)));
    g.gh = int(std::ceil(float(H) / float(g.gs)));
    g.D = p.disp_max;
    g.dmin = std::max(p.disp_min, 0);
    g.words = (g.D + 1 + 31) / 32;
    return g;
}

// Bits of the packed prior word that hold d_plane: enough for
// [0, disp_max + plane_radius + 1]; the rest numbers the triangle.
int prior_shift(const Geom& g, const DevParams& dp) {
    int need = g.D + dp.plane_radius + 2, b = 1;
    while ((1 << b) < need) ++b;
    return b;
}

// Pixels of one output map: W x H, or (W / 2) x (H / 2) when subsampling.
size_t out_pixels(int W, int H, const elas_params& p) {
    return p.subsampling ? size_t(W / 2) * (H / 2) : size_t(W) * H;
}

// Lay out (and, if `base` is non-null, assign) every workspace buffer.
size_t layout(elas_handle* h, const Geom& g, char* base) {
    size_t off = 0;
    auto take = [&](size_t bytes) -> char* {
        char* p = base ? base + off : nullptr;
        off += align_up(bytes);
        return p;
    };
    const size_t px = size_t(g.W) * g.H;
    // support points: the lattice plus six corner points (add_corners),
    // rows: the lattice rows plus the corners' extra row
    const size_t nmax = size_t(std::max(g.cw, 1)) * std::max(g.ch, 1) + 6;
    const size_t rows = size_t(std::max(g.ch, 1)) + 1;
    const size_t tmax = 2 * nmax + 16;
    const size_t hmax = next_pow2(6 * tmax);
    const size_t cells = size_t(g.gw) * g.gh * g.words;
    h->img0 = (uint8_t*)take(px);
    h->img1 = (uint8_t*)take(px);
    h->desc0 = (uint4*)take(px * 16);
    h->desc1 = (uint4*)take(px * 16);
    h->can_lr = (int32_t*)take(nmax * 4);
    h->can = (int32_t*)take(nmax * 4);
    h->row_cnt = (int32_t*)take(rows * 4);
    h->row_off = (int32_t*)take((rows + 1) * 4);
    h->uvd = (int32_t*)take(3 * nmax * 4);
    h->x0 = (int32_t*)take(nmax * 4);
    h->x1 = (int32_t*)take(nmax * 4);
    h->y = (int32_t*)take(nmax * 4);
    h->gtmp0 = (uint32_t*)take(cells * 4);
    h->gtmp1 = (uint32_t*)take(cells * 4);
    h->grid0 = (uint32_t*)take(cells * 4);
    h->grid1 = (uint32_t*)take(cells * 4);
    for (int k = 0; k < 2; ++k) {
        DelDev& D = h->del[k];
        D.srt = (int32_t*)take(nmax * 4);
        D.rcnt = (int32_t*)take(rows * 4);
        D.ne = (int32_t*)take(rows * 4);
        D.soff = (int32_t*)take(rows * 4);
        D.chain = (int32_t*)take(14 * rows * 4);   // 2 sides x (index, x, y, 4-int stack records)
        D.tri = (int32_t*)take(3 * tmax * 4);
        D.opp = (int32_t*)take(3 * tmax * 4);
        D.txy = (uint32_t*)take(3 * tmax * 4);
        D.lock = (uint32_t*)take(tmax * 4);
        D.fround = (int32_t*)take(tmax * 4);
        D.cand = (int32_t*)take(6 * tmax * 4);
        D.flips = (int32_t*)take(3 * tmax * 4);
        D.wl0 = (int32_t*)take(6 * tmax * 4);
        D.wl1 = (int32_t*)take(6 * tmax * 4);
        const size_t per_cta = 6 * 4096;
        D.cwl = (int32_t*)take(16 * 2 * per_cta * 4);
        D.ccand = (int32_t*)take(16 * 2 * per_cta * 4);
        D.cflips = (int32_t*)take(16 * per_cta * 4);
        D.ctr = (int32_t*)take(16 * 4);
        D.pxy = (uint32_t*)take(nmax * 4);
        D.sxy = (uint32_t*)take(nmax * 4);
        D.ne_y = (int32_t*)take(rows * 4);
        D.rinfo = (int4*)take(rows * 16);
        D.tcnt = (int32_t*)take(nmax * 4);
        D.toff = (int32_t*)take(nmax * 4);
        D.sown = (int32_t*)take(24 * nmax * 4);
        D.spool = (int32_t*)take(2 * tmax * 4);
        D.hnext = (int32_t*)take(nmax * 4);
        D.hprev = (int32_t*)take(nmax * 4);
        D.box = (int32_t*)take(32);
        D.ylut = (int32_t*)take((size_t(g.H) + 2) * 4);
        D.hkey = (unsigned long long*)take(hmax * 8);
        D.hcnt = (int32_t*)take(hmax * 4);
        D.hval = (int32_t*)take(2 * hmax * 4);
        D.hslot = (int32_t*)take(3 * tmax * 4);
        D.Tmax = int(tmax);
        D.Hmax = uint32_t(hmax);
    }
    h->rast = take(2 * tmax * raster_bytes());
    {
        const size_t nt = prior_tile_count(g), cap = prior_overflow_capacity(g, int(tmax));
        h->ptiles.cnt = (int32_t*)take(2 * (nt + 1) * 4);
        h->ptiles.bins = (int32_t*)take(2 * nt * PT_BIN * 4);
        h->ptiles.ovf = (int32_t*)take(2 * cap * 2 * 4);
        h->ptiles.ovf_cap = int(cap);
    }
    h->prior0 = (uint32_t*)take(px * 4);
    h->prior1 = (uint32_t*)take(px * 4);
    h->raw0 = (float*)take(px * 4);
    h->raw1 = (float*)take(px * 4);
    h->lr0 = (float*)take(px * 4);
    h->lr1 = (float*)take(px * 4);
    h->out0 = (float*)take(px * 4);
    h->out1 = (float*)take(px * 4);
    for (int k = 0; k < 2; ++k) {
        h->tmp[k] = (float*)take(px * 4);
        h->lab[k] = (int32_t*)take(px * 4);
        h->root[k] = (int32_t*)take(px * 4);
        h->usize[k] = (int32_t*)take(px * 4);
        h->roots[k] = (int32_t*)take(px * 4 + 4);
    }
    h->err = (unsigned*)take(64);
    return off;
}

int ensure_workspace(elas_handle* h, const Geom& g) {
    size_t need = layout(h, g, nullptr);
    if (need > h->arena_bytes) {
        if (h->arena) {
            CK(cudaDeviceSynchronize());
            CK(cudaFree(h->arena));
            h->arena = nullptr;
            h->arena_bytes = 0;
        }
        cudaError_t e = cudaMalloc(&h->arena, need);
        if (e != cudaSuccess) {
            h->arena = nullptr;
            return fail(h, ELAS_ERR_OOM, std::string("workspace allocation of ") + std::to_string(need) +
                                             " bytes failed: " + cudaGetErrorString(e));
        }
        h->arena_bytes = need;
        // cudaMemset runs on the legacy default stream, which the caller's
        // stream and the batch workers' non-blocking streams are not ordered
        // after: without the wait, the zero fill can land after the first
        // kernels of this call have written the workspace.
        CK(cudaMemset(h->arena, 0, need));
        CK(cudaDeviceSynchronize());
    }
    layout(h, g, (char*)h->arena);
    for (int k = 0; k < 2; ++k) {
        h->del[k].x = k == 0 ? h->x0 : h->x1;
        h->del[k].y = h->y;
    }
    return ELAS_OK;
}

int check_dims(elas_handle* h, const int32_t* dims, int& W, int& H) {
    if (!dims) return fail(h, ELAS_ERR_INVALID_ARG, "dims is null");
    W = dims[0];
    H = dims[1];
    if (W < 16 || H < 16) return fail(h, ELAS_ERR_INVALID_ARG, "images must be at least 16x16");
    if (W > 14000 || H > 16384) return fail(h, ELAS_ERR_UNSUPPORTED, "images wider than 14000 or taller than 16384");
    if (W / h->params.candidate_stepsize > 2048)
        return fail(h, ELAS_ERR_UNSUPPORTED, "more than 2048 candidates per lattice row");
    {
        Geom g = geom_of(W, H, h->params);
        DevParams dp = dev_params(h->params);
        int64_t tmax = 2LL * g.cw * g.ch + 16;
        if ((tmax + 1) >> (32 - prior_shift(g, dp)) != 0)
            return fail(h, ELAS_ERR_UNSUPPORTED, "too many candidate points for the packed plane prior");
        if (dense_smem_bytes(g) > 220 * 1024)
            return fail(h, ELAS_ERR_UNSUPPORTED, "image too wide for the dense row in shared memory");
    }
    return ELAS_OK;
}

// Dense-matching autotuner.  The CTA shape (threads per row CTA) changes
// only how the row's pixels are spread over threads, never the result; the
// first call with a new (width class, disp_max) times each shape on its own
// data (CUDA events on the stream) and keeps the fastest.  Inside a stream
// capture an untuned class uses 512 threads.
constexpr int DENSE_SHAPES[4] = {128, 256, 512, 1024};

int dense_threads_for(elas_handle* h, const Geom& g, const DevParams& dp, cudaStream_t st, int* nlaunch, int* out) {
    elas_handle* t = h->owner ? h->owner : h;
    const int sub = h->params.subsampling ? 1 : 0;
    const std::pair<int, int> key(((g.W >> sub) + 127) / 128, g.D);
    auto it = t->dense_threads.find(key);
    if (it != t->dense_threads.end()) { *out = it->second; return ELAS_OK; }
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(st, &cs));
    if (cs != cudaStreamCaptureStatusNone) { *out = 512; return ELAS_OK; }
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    int best = 512;
    float best_ms = 1e30f;
    for (int shape : DENSE_SHAPES) {
        float shape_ms = 1e30f;
        for (int rep = 0; rep < 3; ++rep) {
            CK(cudaEventRecord(e0, st));
            CK(launch_dense(h->desc0, h->desc1, h->prior0, h->prior1, h->grid0, h->grid1, h->raw0, h->raw1, g, dp,
                            prior_shift(g, dp), h->err, st, shape, sub));
            CK(cudaEventRecord(e1, st));
            CK(cudaEventSynchronize(e1));
            float ms = 0;
            CK(cudaEventElapsedTime(&ms, e0, e1));
            shape_ms = std::min(shape_ms, ms);
            *nlaunch += 1;
        }
        if (shape_ms < best_ms) { best_ms = shape_ms; best = shape; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    t->dense_threads[key] = best;
    *out = best;
    return ELAS_OK;
}

// The whole pipeline on device buffers (inputs img0/img1 already on the device).
// Proposal buffers: four [2][H/4][W/4][32] bf16 maps and the packed bins of
// every candidate; grown on demand (outside any stream capture: the first
// call of a batch runs eagerly).
int ensure_pn(elas_handle* h, const Geom& g) {
    const size_t elems = size_t(2) * (g.H / 4) * (g.W / 4) * pn::CH;
    const size_t cands = size_t(g.cw) * g.ch;
    if (elems > h->pn_map_elems) {
        CK(cudaDeviceSynchronize());
        __nv_bfloat16** bufs[4] = {&h->pn_in, &h->pn_a0, &h->pn_a1, &h->pn_out};
        for (auto b : bufs) {
            if (*b) cudaFree(*b);
            *b = nullptr;
            if (cudaMalloc(reinterpret_cast<void**>(b), elems * sizeof(__nv_bfloat16)) != cudaSuccess)
                return fail(h, ELAS_ERR_OOM, "proposal feature maps");
        }
        h->pn_map_elems = elems;
    }
    if (cands > h->pn_cands) {
        CK(cudaDeviceSynchronize());
        if (h->pn_bins) cudaFree(h->pn_bins);
        h->pn_bins = nullptr;
        if (cudaMalloc(&h->pn_bins, cands * sizeof(uint32_t)) != cudaSuccess)
            return fail(h, ELAS_ERR_OOM, "proposal bins");
        h->pn_cands = cands;
    }
    return ELAS_OK;
}

int set_proposal_weights(elas_handle* h, const float* params, int n) {
    if (n == 0) { h->prop = false; ++h->prop_version; return ELAS_OK; }
    if (!params || n != pn::NPARAMS) return fail(h, ELAS_ERR_INVALID_ARG, "proposal parameter count");
    for (int i = 0; i < n; ++i)
        if (!std::isfinite(params[i])) return fail(h, ELAS_ERR_INVALID_ARG, "non-finite proposal parameter");
    if (!h->pw.w) {
        if (cudaMalloc(&h->pw.w, size_t(pn::LAYERS) * pn::TAPS * pn::CH * pn::CH * sizeof(__nv_bfloat16)) !=
                cudaSuccess ||
            cudaMalloc(&h->pw.b, size_t(pn::LAYERS) * pn::CH * sizeof(float)) != cudaSuccess ||
            cudaMalloc(&h->pn_stats, 4 * sizeof(int32_t)) != cudaSuccess)
            return fail(h, ELAS_ERR_OOM, "proposal weights");
        CK(cudaMemset(h->pn_stats, 0, 4 * sizeof(int32_t)));
    }
    CK(pn::upload_weights(params, h->pw, nullptr));
    h->prop_params.assign(params, params + n);
    h->prop = true;
    ++h->prop_version;
    return ELAS_OK;
}

void free_pn(elas_handle* h) {
    __nv_bfloat16* bufs[4] = {h->pn_in, h->pn_a0, h->pn_a1, h->pn_out};
    for (auto b : bufs)
        if (b) cudaFree(b);
    if (h->pn_bins) cudaFree(h->pn_bins);
    if (h->pn_stats) cudaFree(h->pn_stats);
    if (h->pw.w) cudaFree(h->pw.w);
    if (h->pw.b) cudaFree(h->pw.b);
}

// host_out: out0/out1 are device-mapped pinned host memory.  Every
// intermediate then stays in device memory and only the last pass of each
// view writes there, so the results cross PCIe while that pass computes.
int run_pipeline(elas_handle* h, const uint8_t* img0, const uint8_t* img1, float* out0, float* out1, int W, int H,
                 cudaStream_t st, bool host_out = false) {
    const elas_params& p = h->params;
    Geom g = geom_of(W, H, p);
    DevParams dp = dev_params(p);
    int rc = ensure_workspace(h, g);
    if (rc != ELAS_OK) return rc;
    h->g = g;
    int n = 0;
    // stage marks; inside a capture they become event-record nodes of the graph
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(st, &cs));
    const unsigned ev_flags = cs != cudaStreamCaptureStatusNone ? cudaEventRecordExternal : cudaEventRecordDefault;
    auto mark = [&](int i) -> cudaError_t {
        return h->timing ? cudaEventRecordWithFlags(h->ev[i], st, ev_flags) : cudaSuccess;
    };
    CK(cudaMemsetAsync(h->err, 0, sizeof(unsigned), st));
    CK(mark(ELAS_TIME_DESCRIPTOR));
    CK(launch_descriptor(img0, img1, h->desc0, h->desc1, W, H, st));
    n += 1;
    CK(mark(ELAS_TIME_SUPPORT));
    const uint32_t* bins = nullptr;
    h->pn_used = h->prop && H >= 4 && W >= 4 && g.cw > 0 && g.ch > 0;
    if (h->pn_used) {
        rc = ensure_pn(h, g);
        if (rc != ELAS_OK) return rc;
        CK(cudaMemsetAsync(h->pn_stats, 0, 4 * sizeof(int32_t), st));
        CK(pn::launch_features(h->desc0, h->desc1, h->pn_in, W, H, st));
        CK(pn::launch_infer(h->pw, h->pn_in, h->pn_a0, h->pn_a1, h->pn_out, H / 4, W / 4, h->num_sms, h->err, st));
        CK(pn::launch_topk(h->pn_out, h->pn_bins, H / 4, W / 4, g.cw, g.ch, g.step, g.D, st));
        bins = h->pn_bins;
        n += 6;
    }
    CK(launch_support(h->desc0, h->desc1, h->can_lr, nullptr, h->can, h->row_cnt, g, dp, h->num_sms, h->err, st,
                      bins, h->pn_used ? h->pn_stats : nullptr));
    n += 3;
    CK(mark(ELAS_TIME_COMPACT));
    const int corners = p.add_corners ? 1 : 0;
    CK(launch_compact(h->can, h->row_cnt, h->row_off, h->uvd, h->x0, h->x1, h->y, g, st, corners, &n));
    CK(mark(ELAS_TIME_GRID));
    // The grid needs only the support list: it runs on the side stream
    // beside the Delaunay and prior stages and joins before dense matching
    // (recorded as graph edges inside a capture).  With stage timing on it
    // runs in line, so that the stage marks keep their meaning.
    // The direct prior paint also needs zeroed prior maps, which the side
    // stream clears meanwhile; the join then comes before the prior stage.
    const bool fork = !h->timing;
    const bool tiled = (h->test_flags & ELAS_TEST_PRIOR_TILED) != 0 ||
                       ((h->test_flags & ELAS_TEST_PRIOR_DIRECT) == 0 && (long long)W * H >= PRIOR_TILED_MIN_PIXELS);
    if (fork) {
        if (!h->side) CK(cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking));
        if (!h->side_fork) CK(cudaEventCreateWithFlags(&h->side_fork, cudaEventDisableTiming));
        if (!h->side_join) CK(cudaEventCreateWithFlags(&h->side_join, cudaEventDisableTiming));
        CK(cudaEventRecordWithFlags(h->side_fork, st, 0));
        CK(cudaStreamWaitEvent(h->side, h->side_fork, 0));
        CK(launch_grid(h->can, h->gtmp0, h->gtmp1, h->grid0, h->grid1, g, h->side, &n));
        if (!tiled) {
            CK(cudaMemsetAsync(h->prior0, 0, size_t(W) * H * sizeof(uint32_t), h->side));
            CK(cudaMemsetAsync(h->prior1, 0, size_t(W) * H * sizeof(uint32_t), h->side));
        }
        CK(cudaEventRecordWithFlags(h->side_join, h->side, 0));
    } else {
        CK(launch_grid(h->can, h->gtmp0, h->gtmp1, h->grid0, h->grid1, g, st, &n));
    }
    CK(mark(ELAS_TIME_DELAUNAY));
    const bool flips = (h->test_flags & (ELAS_TEST_DELAUNAY_FLIPS | ELAS_TEST_FLIP_GLOBAL)) != 0 ||
                       h->flip_round_limit > 0 ||
                       ((h->test_flags & ELAS_TEST_DELAUNAY_STARS) == 0 &&
                        (long long)W * H > DELAUNAY_STARS_MAX_PIXELS);
    CK(launch_delaunay(h->del[0], h->del[1], h->row_off, g.ch + corners, g.cw * g.ch + 6 * corners, H, h->num_sms,
                       h->cluster_size, h->err, st, &n, flips, (h->test_flags & ELAS_TEST_FLIP_GLOBAL) != 0,
                       h->flip_round_limit));
    CK(mark(ELAS_TIME_PRIOR));
    if (fork) CK(cudaStreamWaitEvent(st, h->side_join, 0));
    CK(launch_prior(h->del[0].tri, h->del[1].tri, h->del[0].ctr, h->del[1].ctr, h->del[0].Tmax, h->can, h->uvd,
                    h->rast, h->ptiles, h->prior0, h->prior1, g, prior_shift(g, dp), g.D + dp.plane_radius + 1,
                    h->num_sms, h->err, st, &n, tiled, fork && !tiled,
                    (h->test_flags & ELAS_TEST_PRIOR_SMALL_BINS) ? 2 : PT_BIN));
    int shape = 512;
    rc = dense_threads_for(h, g, dp, st, &n, &shape);
    if (rc != ELAS_OK) return rc;
    CK(mark(ELAS_TIME_DENSE));
    // subsampling: dense, L/R and post-filters on every second row and column
    const int sub = p.subsampling ? 1 : 0;
    Geom go = g;
    go.W = W >> sub;
    go.H = H >> sub;
    CK(launch_dense(h->desc0, h->desc1, h->prior0, h->prior1, h->grid0, h->grid1, h->raw0, h->raw1, g, dp,
                    prior_shift(g, dp), h->err, st, shape, sub, (h->test_flags & ELAS_TEST_DENSE_BITSET) != 0));
    n += 1;
    CK(mark(ELAS_TIME_LR));
    // The checked maps also land where the post-filter chain starts: in the
    // outputs, or, when the chain's first pass cannot work in place (speckle
    // removal applied inside the tile filter), in the scratch maps, so that
    // the last pass writes the outputs.
    const int nviews = p.postprocess_only_left ? 1 : 2;
    const bool from_tmp = host_out || post_fuses_speckle(dp, p.filter_median, p.filter_adaptive_mean);
    float* outs[2] = {out0, out1};
    float* dev_outs[2] = {host_out ? h->out0 : out0, host_out ? h->out1 : out1};   // device partners of tmp
    float* start[2];
    for (int k = 0; k < 2; ++k) start[k] = from_tmp && k < nviews ? h->tmp[k] : outs[k];
    CK(launch_lr(h->raw0, h->raw1, h->lr0, h->lr1, start[0], start[1], g, p.lr_threshold, st, sub));
    n += 1;
    CK(mark(ELAS_TIME_POST));
    PostViews pv;
    for (int k = 0; k < 2; ++k) {
        pv.cur[k] = start[k];
        pv.nxt[k] = start[k] == dev_outs[k] ? h->tmp[k] : dev_outs[k];
        pv.out[k] = outs[k];
        pv.lab[k] = h->lab[k];
        pv.root[k] = h->root[k];
        pv.sz[k] = h->usize[k];
        pv.roots[k] = h->roots[k];
    }
    CK(launch_post(pv, nviews, go, dp, p.filter_median, p.filter_adaptive_mean, h->err, st, &n, h->num_sms));
    CK(mark(ELAS_TIME_COUNT));
    h->launches += n;
    h->have_last = true;
    return ELAS_OK;
}

// run_pipeline through a cached CUDA graph.  A call whose signature was
// not seen before runs eagerly (it sizes the workspaces and tunes the dense
// shape); the next call with the same signature is captured on the handle's
// own stream (the caller's stream may be the legacy default stream, which
// cannot be captured) and launched into the caller's stream; later calls
// only launch the graph.  A caller that is itself capturing gets the plain
// launches, which join its capture.
int run_pipeline_graphed(elas_handle* h, const uint8_t* img0, const uint8_t* img1, float* out0, float* out1, int W,
                         int H, cudaStream_t st, bool host_out = false) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(st, &cs));
    if (!h->use_graphs || cs != cudaStreamCaptureStatusNone)
        return run_pipeline(h, img0, img1, out0, out1, W, H, st, host_out);
    const Geom g = geom_of(W, H, h->params);
    int rc = ensure_workspace(h, g);
    if (rc != ELAS_OK) return rc;
    if (h->prop && H >= 4 && W >= 4 && g.cw > 0 && g.ch > 0) {
        rc = ensure_pn(h, g);
        if (rc != ELAS_OK) return rc;
    }
    std::vector<int64_t> sig = {int64_t(img0), int64_t(img1), int64_t(out0), int64_t(out1), W, H,
                                int64_t(h->arena), int64_t(h->arena_bytes), int64_t(h->pn_in), int64_t(h->pn_bins),
                                int64_t(h->pn_stats), h->timing ? 1 : 0, h->prop ? 1 : 0, h->prop_version,
                                h->test_flags, h->flip_round_limit, host_out ? 1 : 0};
    int64_t pw[sizeof(elas_params) / 8 + 1] = {};
    std::memcpy(pw, &h->params, sizeof(elas_params));
    for (int64_t x : pw) sig.push_back(x);
    if (h->single_exec && sig == h->single_sig) {
        CK(cudaGraphLaunch(h->single_exec, st));
        h->g = g;   // what run_pipeline leaves behind for the stage dumps
        h->pn_used = h->prop && H >= 4 && W >= 4 && g.cw > 0 && g.ch > 0;
        h->launches += h->single_launches;
        h->have_last = true;
        return ELAS_OK;
    }
    if (sig != h->single_seen) {
        h->single_seen = sig;
        return run_pipeline(h, img0, img1, out0, out1, W, H, st, host_out);
    }
    if (!h->own_stream) CK(cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking));
    if (h->single_exec) { cudaGraphExecDestroy(h->single_exec); h->single_exec = nullptr; }
    const long long before = h->launches;
    CK(cudaStreamBeginCapture(h->own_stream, cudaStreamCaptureModeThreadLocal));
    rc = run_pipeline(h, img0, img1, out0, out1, W, H, h->own_stream, host_out);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(h->own_stream, &graph);
    if (rc != ELAS_OK) { if (graph) cudaGraphDestroy(graph); return rc; }
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(&h->single_exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) { h->single_exec = nullptr; return cuda_fail(h, e, "cudaGraphInstantiate"); }
    h->single_sig = sig;
    h->single_launches = h->launches - before;
    CK(cudaGraphLaunch(h->single_exec, st));
    return ELAS_OK;
}

// Batch workers: one handle (own workspace) and one stream per pair.
int ensure_slots(elas_handle* h, int n) {
    while (int(h->slots.size()) < n) {
        elas_handle* w = new elas_handle();
        w->params = h->params;
        w->device = h->device;
        w->num_sms = h->num_sms;
        w->cluster_size = h->cluster_size;
        w->owner = h;
        cudaStream_t st;
        cudaEvent_t ev;
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) { delete w; return ELAS_ERR_CUDA; }
        if (cudaEventCreate(&ev) != cudaSuccess) { cudaStreamDestroy(st); delete w; return ELAS_ERR_CUDA; }
        cudaEvent_t lev;
        if (cudaEventCreate(&lev) != cudaSuccess) {
            cudaEventDestroy(ev);
            cudaStreamDestroy(st);
            delete w;
            return ELAS_ERR_CUDA;
        }
        h->lat_done.push_back(lev);
        h->slots.push_back(w);
        h->slot_streams.push_back(st);
        h->slot_done.push_back(ev);
    }
    if (!h->batch_start) CK(cudaEventCreate(&h->batch_start));
    if (!h->lat_start) CK(cudaEventCreate(&h->lat_start));
    if (!h->own_stream) CK(cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking));
    return ELAS_OK;
}

// Fork from `st`, run pair i on worker stream i, join back into `st`.  With
// host buffers (hl/hr/hd1/hd2 non-null) the copies in both directions go on
// the worker streams as well.  Works inside a stream capture (the workers
// join it through the fork event) as long as every workspace is sized.
// lat_start / lat_done are recorded as event nodes of a captured graph, so
// per-pair latencies stay readable after a replay.
int issue_batch(elas_handle* h, int n, const uint8_t* const* l, const uint8_t* const* r, float* const* d1,
                float* const* d2, const int32_t* dims, const int32_t* dmax, bool host, cudaStream_t st,
                bool capturing = false) {
    const unsigned lat_flags = capturing ? cudaEventRecordExternal : cudaEventRecordDefault;
    CK(cudaEventRecordWithFlags(h->lat_start, st, lat_flags));
    CK(cudaEventRecord(h->batch_start, st));
    for (int i = 0; i < n; ++i) {
        elas_handle* w = h->slots[i];
        cudaStream_t ws = h->slot_streams[i];
        w->params = h->params;
        w->test_flags = h->test_flags;
        w->flip_round_limit = h->flip_round_limit;
        if (dmax) w->params.disp_max = dmax[i];
        if (w->prop_version != h->prop_version) {
            int rc = set_proposal_weights(w, h->prop ? h->prop_params.data() : nullptr,
                                          h->prop ? int(h->prop_params.size()) : 0);
            if (rc != ELAS_OK) return fail(h, rc, w->last_error);
            w->prop_version = h->prop_version;
        }
        const int W = dims[2 * i], H = dims[2 * i + 1];
        const size_t px = size_t(W) * H;
        CK(cudaStreamWaitEvent(ws, h->batch_start, 0));
        int rc = ensure_workspace(w, geom_of(W, H, w->params));
        if (rc != ELAS_OK) return fail(h, rc, w->last_error);
        const uint8_t* il = l[i];
        const uint8_t* ir = r[i];
        float* o1 = d1[i];
        float* o2 = d2[i];
        if (host) {
            CK(cudaMemcpyAsync(w->img0, l[i], px, cudaMemcpyHostToDevice, ws));
            CK(cudaMemcpyAsync(w->img1, r[i], px, cudaMemcpyHostToDevice, ws));
            il = w->img0;
            ir = w->img1;
            o1 = w->out0;
            o2 = w->out1;
        }
        rc = run_pipeline(w, il, ir, o1, o2, W, H, ws);
        if (rc != ELAS_OK) return fail(h, rc, w->last_error);
        if (host) {
            const size_t po = out_pixels(W, H, w->params);
            CK(cudaMemcpyAsync(d1[i], w->out0, po * 4, cudaMemcpyDeviceToHost, ws));
            CK(cudaMemcpyAsync(d2[i], w->out1, po * 4, cudaMemcpyDeviceToHost, ws));
        }
        CK(cudaEventRecordWithFlags(h->lat_done[i], ws, lat_flags));
        CK(cudaEventRecord(h->slot_done[i], ws));
        CK(cudaStreamWaitEvent(st, h->slot_done[i], 0));
    }
    h->last_batch = n;
    return ELAS_OK;
}

int check_batch(elas_handle* h, int n, const int32_t* dims, const int32_t* dmax) {
    for (int i = 0; i < n; ++i) {
        elas_params q = h->params;
        if (dmax) q.disp_max = dmax[i];
        std::string why;
        int rc = check_params(q, why);
        if (rc != ELAS_OK) return fail(h, rc, "pair " + std::to_string(i) + ": " + why);
        elas_params saved = h->params;
        h->params = q;
        int W, H;
        rc = check_dims(h, dims + 2 * i, W, H);
        h->params = saved;
        if (rc != ELAS_OK) return rc;
    }
    return ELAS_OK;
}

// The device address of a pinned, device-mapped host buffer; null for any
// other pointer (pageable memory, device memory) or when
// ELAS_B200_ZERO_COPY=0 is set in the environment.
float* mapped_host(float* p) {
    static const bool on = [] {
        const char* e = std::getenv("ELAS_B200_ZERO_COPY");
        return !(e && e[0] == '0');
    }();
    if (!on) return nullptr;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return a.type == cudaMemoryTypeHost && a.devicePointer ? static_cast<float*>(a.devicePointer) : nullptr;
}

int check_device_errors(elas_handle* h, cudaStream_t st) {
    if (!h->err_host) CK(cudaHostAlloc(reinterpret_cast<void**>(&h->err_host), sizeof(unsigned), cudaHostAllocDefault));
    CK(cudaMemcpyAsync(h->err_host, h->err, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    const unsigned e = *h->err_host;
    if (e & ERRF_FLIP_LIMIT) return fail(h, ELAS_ERR_TIMEOUT, "edge flipping hit its round limit");
    if (e) return fail(h, ELAS_ERR_INTERNAL, "device consistency check failed, flags " + std::to_string(e));
    return ELAS_OK;
}

}  // namespace

extern "C" {

void elas_params_default(elas_params* p) {
    if (!p) return;
    // src/Elas.h:42-66
    p->disp_min = 0;
    p->disp_max = 255;
    p->support_threshold = 0.95f;
    p->support_texture = 10;
    p->candidate_stepsize = 5;
    p->incon_window_size = 5;
    p->incon_threshold = 5;
    p->incon_min_support = 5;
    p->add_corners = true;
    p->grid_size = 20;
    p->beta = 0.02f;
    p->gamma = 5;
    p->sigma = 1;
    p->sradius = 3;
    p->match_texture = 0;
    p->lr_threshold = 2;
    p->speckle_sim_threshold = 1;
    p->speckle_size = 200;
    p->ipol_gap_width = 5000;
    p->filter_median = true;
    p->filter_adaptive_mean = false;
    p->postprocess_only_left = false;
    p->subsampling = false;
}

void elas_params_reference(elas_params* p) {
    if (!p) return;
    elas_params_default(p);
    // src/Kernels/KernelsCommon.h:8-27
    p->disp_min = 0;
    p->disp_max = 255;
    p->support_threshold = 0.85f;
    p->support_texture = 10;
    p->candidate_stepsize = 5;
    p->incon_window_size = 5;
    p->incon_threshold = 5;
    p->incon_min_support = 5;
    p->add_corners = false;
    p->grid_size = 20;
    p->beta = 0.02f;
    p->gamma = 3;
    p->sigma = 1;
    p->sradius = 2;
    p->match_texture = 0;
    p->lr_threshold = 2;
    p->speckle_sim_threshold = 1;
    // the reference runs no post-filter (src/Elas.cu:107-119)
    p->speckle_size = 0;
    p->ipol_gap_width = 0;
    p->filter_median = false;
    p->filter_adaptive_mean = false;
    p->postprocess_only_left = false;
    p->subsampling = false;
}

const char* elas_b200_status_string(int s) {
    switch (s) {
    case ELAS_OK: return "ok";
    case ELAS_ERR_INVALID_ARG: return "invalid argument";
    case ELAS_ERR_UNSUPPORTED: return "unsupported";
    case ELAS_ERR_CUDA: return "CUDA error";
    case ELAS_ERR_OOM: return "out of memory";
    case ELAS_ERR_INTERNAL: return "internal consistency check failed";
    case ELAS_ERR_NO_DEVICE: return "no usable sm_100 device";
    case ELAS_ERR_TIMEOUT: return "bounded device loop hit its limit";
    case ELAS_ERR_TOO_LARGE: return "input exceeds the fixed scratch capacity of the allocation-free entry point";
    default: return "unknown status";
    }
}

int elas_b200_create(const elas_params* params, int device, elas_handle** out) {
    if (!out) return ELAS_ERR_INVALID_ARG;
    *out = nullptr;
    elas_params p;
    if (params) p = *params;
    else elas_params_default(&p);
    std::string why;
    int rc = check_params(p, why);
    if (rc != ELAS_OK) return rc;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
        cudaGetLastError();
        return ELAS_ERR_NO_DEVICE;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return ELAS_ERR_NO_DEVICE;
    if (prop.major != 10 || prop.minor != 0) return ELAS_ERR_NO_DEVICE;
    if (cudaSetDevice(device) != cudaSuccess) return ELAS_ERR_NO_DEVICE;
    elas_handle* h = new elas_handle();
    h->params = p;
    h->device = device;
    h->num_sms = prop.multiProcessorCount;
    h->cluster_size = cluster_size_for_flip();
    *out = h;
    return ELAS_OK;
}

int elas_b200_set_timing(elas_handle* h, int enable) {
    if (!h) return ELAS_ERR_INVALID_ARG;
    CK(cudaSetDevice(h->device));
    if (enable && !h->ev[0])
        for (int i = 0; i <= ELAS_TIME_COUNT; ++i) CK(cudaEventCreate(&h->ev[i]));
    h->timing = enable != 0;
    return ELAS_OK;
}

int elas_b200_get_timing(elas_handle* h, float* ms_out, int n) {
    if (!h || !ms_out || n < ELAS_TIME_COUNT) return ELAS_ERR_INVALID_ARG;
    if (!h->timing || !h->have_last) return fail(h, ELAS_ERR_INVALID_ARG, "timing not enabled or no call yet");
    CK(cudaEventSynchronize(h->ev[ELAS_TIME_COUNT]));
    for (int i = 0; i < ELAS_TIME_COUNT; ++i) CK(cudaEventElapsedTime(&ms_out[i], h->ev[i], h->ev[i + 1]));
    return ELAS_OK;
}

int elas_b200_destroy(elas_handle* h) {
    if (!h) return ELAS_ERR_INVALID_ARG;
    cudaSetDevice(h->device);
    if (h->graph_exec) cudaGraphExecDestroy(h->graph_exec);
    for (size_t i = 0; i < h->slots.size(); ++i) {
        cudaStreamSynchronize(h->slot_streams[i]);
        elas_b200_destroy(h->slots[i]);
        cudaStreamDestroy(h->slot_streams[i]);
        cudaEventDestroy(h->slot_done[i]);
        cudaEventDestroy(h->lat_done[i]);
    }
    if (h->batch_start) cudaEventDestroy(h->batch_start);
    if (h->lat_start) cudaEventDestroy(h->lat_start);
    free_pn(h);
    if (h->single_exec) cudaGraphExecDestroy(h->single_exec);
    if (h->own_stream) cudaStreamDestroy(h->own_stream);
    if (h->side) cudaStreamDestroy(h->side);
    if (h->side_fork) cudaEventDestroy(h->side_fork);
    if (h->side_join) cudaEventDestroy(h->side_join);
    for (int i = 0; i <= ELAS_TIME_COUNT; ++i)
        if (h->ev[i]) cudaEventDestroy(h->ev[i]);
    if (h->arena) {
        cudaSetDevice(h->device);
        cudaDeviceSynchronize();
        cudaFree(h->arena);
    }
    if (h->err_host) cudaFreeHost(h->err_host);
    delete h;
    return ELAS_OK;
}

int elas_b200_set_params(elas_handle* h, const elas_params* params) {
    if (!h || !params) return ELAS_ERR_INVALID_ARG;
    std::string why;
    int rc = check_params(*params, why);
    if (rc != ELAS_OK) return fail(h, rc, why);
    h->params = *params;
    return ELAS_OK;
}

int elas_b200_get_params(const elas_handle* h, elas_params* out) {
    if (!h || !out) return ELAS_ERR_INVALID_ARG;
    *out = h->params;
    return ELAS_OK;
}

const char* elas_b200_last_error(const elas_handle* h) { return h ? h->last_error.c_str() : ""; }

int64_t elas_b200_launch_count(const elas_handle* h) { return h ? h->launches : 0; }

int elas_b200_process_device(elas_handle* h, const uint8_t* d_left, const uint8_t* d_right, float* d_disp_left,
                             float* d_disp_right, const int32_t* dims, void* stream) {
    if (!h) return ELAS_ERR_INVALID_ARG;
    if (!d_left || !d_right || !d_disp_left || !d_disp_right) return fail(h, ELAS_ERR_INVALID_ARG, "null buffer");
    int W, H;
    int rc = check_dims(h, dims, W, H);
    if (rc != ELAS_OK) return rc;
    CK(cudaSetDevice(h->device));
    return run_pipeline_graphed(h, d_left, d_right, d_disp_left, d_disp_right, W, H, (cudaStream_t)stream);
}

int elas_b200_process(elas_handle* h, const uint8_t* left, const uint8_t* right, float* disp_left,
                      float* disp_right, const int32_t* dims, void* stream) {
    if (!h) return ELAS_ERR_INVALID_ARG;
    if (!left || !right || !disp_left || !disp_right) return fail(h, ELAS_ERR_INVALID_ARG, "null buffer");
    int W, H;
    int rc = check_dims(h, dims, W, H);
    if (rc != ELAS_OK) return rc;
    CK(cudaSetDevice(h->device));
    cudaStream_t st = (cudaStream_t)stream;
    rc = ensure_workspace(h, geom_of(W, H, h->params));
    if (rc != ELAS_OK) return rc;
    const size_t px = size_t(W) * H;
    CK(cudaMemcpyAsync(h->img0, left, px, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(h->img1, right, px, cudaMemcpyHostToDevice, st));
    // Pinned, device-mapped output buffers receive the results from the
    // last post-filter pass itself (no separate device-to-host copy).
    float* m1 = mapped_host(disp_left);
    float* m2 = mapped_host(disp_right);
    if (m1 && m2) {
        rc = run_pipeline_graphed(h, h->img0, h->img1, m1, m2, W, H, st, true);
        if (rc != ELAS_OK) return rc;
        return check_device_errors(h, st);
    }
    rc = run_pipeline_graphed(h, h->img0, h->img1, h->out0, h->out1, W, H, st);
    if (rc != ELAS_OK) return rc;
    const size_t po = out_pixels(W, H, h->params);
    CK(cudaMemcpyAsync(disp_left, h->out0, po * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(disp_right, h->out1, po * 4, cudaMemcpyDeviceToHost, st));
    return check_device_errors(h, st);
}

int elas_b200_process_batch(elas_handle* h, int n, const uint8_t* const* lefts, const uint8_t* const* rights,
                            float* const* disp_lefts, float* const* disp_rights, const int32_t* dims,
                            const int32_t* disp_max_per_pair, void* stream) {
    if (!h || n < 0 || (n > 0 && (!lefts || !rights || !disp_lefts || !disp_rights || !dims)))
        return ELAS_ERR_INVALID_ARG;
    if (n == 0) return ELAS_OK;
    CK(cudaSetDevice(h->device));
    int rc = check_batch(h, n, dims, disp_max_per_pair);
    if (rc != ELAS_OK) return rc;
    rc = ensure_slots(h, n);
    if (rc != ELAS_OK) return fail(h, rc, "creating batch workers failed");
    cudaStream_t st = stream ? (cudaStream_t)stream : h->own_stream;
    rc = issue_batch(h, n, lefts, rights, disp_lefts, disp_rights, dims, disp_max_per_pair, true, st);
    if (rc != ELAS_OK) return rc;
    CK(cudaStreamSynchronize(st));
    for (int i = 0; i < n; ++i) {
        rc = check_device_errors(h->slots[i], h->slot_streams[i]);
        if (rc != ELAS_OK) return fail(h, rc, h->slots[i]->last_error);
    }
    return ELAS_OK;
}

int elas_b200_process_batch_device(elas_handle* h, int n, const uint8_t* const* d_lefts,
                                   const uint8_t* const* d_rights, float* const* d_disp_lefts,
                                   float* const* d_disp_rights, const int32_t* dims,
                                   const int32_t* disp_max_per_pair, void* stream) {
    if (!h || n < 0 || (n > 0 && (!d_lefts || !d_rights || !d_disp_lefts || !d_disp_rights || !dims)))
        return ELAS_ERR_INVALID_ARG;
    if (n == 0) return ELAS_OK;
    CK(cudaSetDevice(h->device));
    int rc = check_batch(h, n, dims, disp_max_per_pair);
    if (rc != ELAS_OK) return rc;
    rc = ensure_slots(h, n);
    if (rc != ELAS_OK) return fail(h, rc, "creating batch workers failed");
    cudaStream_t st = stream ? (cudaStream_t)stream : h->own_stream;
    // what a captured graph depends on: sizes, disparity ranges, buffers, parameters
    std::vector<int64_t> sig;
    sig.push_back(n);
    for (int i = 0; i < n; ++i) {
        sig.push_back(dims[2 * i]);
        sig.push_back(dims[2 * i + 1]);
        sig.push_back(disp_max_per_pair ? disp_max_per_pair[i] : h->params.disp_max);
        sig.push_back(int64_t(d_lefts[i]));
        sig.push_back(int64_t(d_rights[i]));
        sig.push_back(int64_t(d_disp_lefts[i]));
        sig.push_back(int64_t(d_disp_rights[i]));
    }
    int64_t pw[sizeof(elas_params) / 8 + 1] = {};
    std::memcpy(pw, &h->params, sizeof(elas_params));
    for (int64_t x : pw) sig.push_back(x);
    sig.push_back(int64_t(st));
    sig.push_back(h->test_flags);
    sig.push_back(h->flip_round_limit);
    if (h->use_graphs && h->graph_exec && sig == h->graph_sig) {
        CK(cudaGraphLaunch(h->graph_exec, st));
    } else {
        // eager run: sizes every workspace, tunes the dense shape, produces the result
        rc = issue_batch(h, n, d_lefts, d_rights, d_disp_lefts, d_disp_rights, dims, disp_max_per_pair, false, st);
        if (rc != ELAS_OK) return rc;
        if (h->use_graphs) {
            CK(cudaStreamSynchronize(st));
            if (h->graph_exec) { cudaGraphExecDestroy(h->graph_exec); h->graph_exec = nullptr; }
            CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            rc = issue_batch(h, n, d_lefts, d_rights, d_disp_lefts, d_disp_rights, dims, disp_max_per_pair, false,
                             st, true);
            cudaGraph_t graph = nullptr;
            cudaError_t e = cudaStreamEndCapture(st, &graph);
            if (rc != ELAS_OK) { if (graph) cudaGraphDestroy(graph); return rc; }
            if (e != cudaSuccess) return cuda_fail(h, e, "cudaStreamEndCapture");
            e = cudaGraphInstantiate(&h->graph_exec, graph, 0);
            cudaGraphDestroy(graph);
            if (e != cudaSuccess) { h->graph_exec = nullptr; return cuda_fail(h, e, "cudaGraphInstantiate"); }
            h->graph_sig = sig;
        }
    }
    if (!stream) CK(cudaStreamSynchronize(st));
    return ELAS_OK;
}

int elas_b200_set_test_mode(elas_handle* h, int32_t flags, int32_t flip_round_limit) {
    if (!h) return ELAS_ERR_INVALID_ARG;
    const int32_t known = ELAS_TEST_FLIP_GLOBAL | ELAS_TEST_DENSE_BITSET | ELAS_TEST_PRIOR_TILED |
                          ELAS_TEST_PRIOR_DIRECT | ELAS_TEST_DELAUNAY_FLIPS | ELAS_TEST_DELAUNAY_STARS |
                          ELAS_TEST_PRIOR_SMALL_BINS;
    if ((flags & ~known) != 0 || flip_round_limit < 0)
        return fail(h, ELAS_ERR_INVALID_ARG, "unknown test flag or negative round limit");
    if ((flags & ELAS_TEST_DELAUNAY_STARS) &&
        ((flags & (ELAS_TEST_DELAUNAY_FLIPS | ELAS_TEST_FLIP_GLOBAL)) || flip_round_limit > 0))
        return fail(h, ELAS_ERR_INVALID_ARG, "both Delaunay constructions forced");
    if ((flags & ELAS_TEST_PRIOR_TILED) && (flags & ELAS_TEST_PRIOR_DIRECT))
        return fail(h, ELAS_ERR_INVALID_ARG, "both prior paint paths forced");
    h->test_flags = flags;
    h->flip_round_limit = flip_round_limit;
    return ELAS_OK;
}

int elas_b200_set_graphs(elas_handle* h, int enable) {
    if (!h) return ELAS_ERR_INVALID_ARG;
    h->use_graphs = enable != 0;
    return ELAS_OK;
}

int elas_b200_batch_latency(elas_handle* h, float* ms_out, int n) {
    if (!h || !ms_out || n < h->last_batch) return -ELAS_ERR_INVALID_ARG;
    for (int i = 0; i < h->last_batch; ++i) {
        if (cudaEventSynchronize(h->lat_done[i]) != cudaSuccess ||
            cudaEventElapsedTime(&ms_out[i], h->lat_start, h->lat_done[i]) != cudaSuccess)
            return -ELAS_ERR_CUDA;
    }
    return h->last_batch;
}

int elas_b200_dense_shape(const elas_handle* h, int32_t width, int32_t disp_max) {
    if (!h) return 0;
    auto it = h->dense_threads.find(std::make_pair((width + 127) / 128, int(disp_max)));
    return it == h->dense_threads.end() ? 0 : it->second;
}

int elas_b200_get_stage(elas_handle* h, int stage, void* dst, size_t bytes, size_t* needed) {
    if (!h) return ELAS_ERR_INVALID_ARG;
    if (!h->have_last) return fail(h, ELAS_ERR_INVALID_ARG, "no previous call");
    if (stage < 0 || stage >= ELAS_STAGE_COUNT) return fail(h, ELAS_ERR_INVALID_ARG, "bad stage");
    CK(cudaSetDevice(h->device));
    CK(cudaDeviceSynchronize());
    const Geom& g = h->g;
    const size_t px = size_t(g.W) * g.H;
    const size_t can_n = size_t(g.cw) * g.ch;
    const size_t cells = size_t(g.gw) * g.gh;
    size_t need = 0;
    int32_t nsup = 0, ntri = 0;
    switch (stage) {
    case ELAS_STAGE_DESC_LEFT: case ELAS_STAGE_DESC_RIGHT: need = px * 16; break;
    case ELAS_STAGE_CAN_LR: case ELAS_STAGE_CAN: need = can_n * 4; break;
    case ELAS_STAGE_SUPPORT:
        CK(cudaMemcpy(&nsup, h->row_off + g.ch + (h->params.add_corners ? 1 : 0), 4, cudaMemcpyDeviceToHost));
        need = size_t(nsup) * 12;
        break;
    case ELAS_STAGE_GRID_LEFT: case ELAS_STAGE_GRID_RIGHT: need = cells * (g.D + 2) * 4; break;
    case ELAS_STAGE_TRI_LEFT: case ELAS_STAGE_TRI_RIGHT:
        CK(cudaMemcpy(&ntri, h->del[stage - ELAS_STAGE_TRI_LEFT].ctr, 4, cudaMemcpyDeviceToHost));
        need = size_t(ntri) * 12;
        break;
    case ELAS_STAGE_PRIOR_LEFT: case ELAS_STAGE_PRIOR_RIGHT: need = px * 4; break;
    case ELAS_STAGE_PN_FEATURES: case ELAS_STAGE_PN_OUTPUT:
        if (!h->pn_used) return fail(h, ELAS_ERR_INVALID_ARG, "the last call did not run the proposal");
        need = size_t(2) * (g.H / 4) * (g.W / 4) * pn::CH * 2;
        break;
    case ELAS_STAGE_PN_BINS:
        if (!h->pn_used) return fail(h, ELAS_ERR_INVALID_ARG, "the last call did not run the proposal");
        need = can_n * 4;
        break;
    case ELAS_STAGE_DEL_COUNTERS: need = 2 * 16 * 4; break;
    case ELAS_STAGE_DISP_LEFT: case ELAS_STAGE_DISP_RIGHT: case ELAS_STAGE_LR_LEFT: case ELAS_STAGE_LR_RIGHT:
        need = out_pixels(g.W, g.H, h->params) * 4;
        break;
    default: need = px * 4; break;
    }
    if (needed) *needed = need;
    if (!dst) return ELAS_OK;
    if (bytes < need) return fail(h, ELAS_ERR_INVALID_ARG, "destination too small");
    switch (stage) {
    case ELAS_STAGE_DESC_LEFT: CK(cudaMemcpy(dst, h->desc0, need, cudaMemcpyDeviceToHost)); break;
    case ELAS_STAGE_DESC_RIGHT: CK(cudaMemcpy(dst, h->desc1, need, cudaMemcpyDeviceToHost)); break;
    case ELAS_STAGE_CAN_LR: CK(cudaMemcpy(dst, h->can_lr, need, cudaMemcpyDeviceToHost)); break;
    case ELAS_STAGE_CAN: CK(cudaMemcpy(dst, h->can, need, cudaMemcpyDeviceToHost)); break;
    case ELAS_STAGE_SUPPORT: CK(cudaMemcpy(dst, h->uvd, need, cudaMemcpyDeviceToHost)); break;
    case ELAS_STAGE_GRID_LEFT: case ELAS_STAGE_GRID_RIGHT: {
        std::vector<uint32_t> bits(cells * g.words);
        CK(cudaMemcpy(bits.data(), stage == ELAS_STAGE_GRID_LEFT ? h->grid0 : h->grid1, bits.size() * 4,
                      cudaMemcpyDeviceToHost));
        int32_t* o = (int32_t*)dst;
        std::memset(o, 0, need);
        for (size_t c = 0; c < cells; ++c) {
            int32_t* cell = o + c * (g.D + 2);
            int k = 1;
            for (int d = 0; d <= g.D; ++d)
                if (bits[c * g.words + d / 32] >> (d % 32) & 1u) cell[k++] = d;
            cell[0] = k - 1;
        }
        break;
    }
    case ELAS_STAGE_TRI_LEFT: CK(cudaMemcpy(dst, h->del[0].tri, need, cudaMemcpyDeviceToHost)); break;
    case ELAS_STAGE_TRI_RIGHT: CK(cudaMemcpy(dst, h->del[1].tri, need, cudaMemcpyDeviceToHost)); break;
    case ELAS_STAGE_PRIOR_LEFT: case ELAS_STAGE_PRIOR_RIGHT: {
        std::vector<uint32_t> pk(px);
        CK(cudaMemcpy(pk.data(), stage == ELAS_STAGE_PRIOR_LEFT ? h->prior0 : h->prior1, px * 4,
                      cudaMemcpyDeviceToHost));
        const int sh = prior_shift(g, dev_params(h->params));
        int32_t* o = (int32_t*)dst;
        for (size_t i = 0; i < px; ++i) {
            int32_t d = int32_t(pk[i] & ((1u << sh) - 1u));
            o[i] = ((pk[i] >> sh) != 0 && d > 0) ? d : -1;
        }
        break;
    }
    case ELAS_STAGE_DISP_LEFT: CK(cudaMemcpy(dst, h->raw0, need, cudaMemcpyDeviceToHost)); break;
    case ELAS_STAGE_DISP_RIGHT: CK(cudaMemcpy(dst, h->raw1, need, cudaMemcpyDeviceToHost)); break;
    case ELAS_STAGE_LR_LEFT: CK(cudaMemcpy(dst, h->lr0, need, cudaMemcpyDeviceToHost)); break;
    case ELAS_STAGE_LR_RIGHT: CK(cudaMemcpy(dst, h->lr1, need, cudaMemcpyDeviceToHost)); break;
    case ELAS_STAGE_PN_FEATURES: CK(cudaMemcpy(dst, h->pn_in, need, cudaMemcpyDeviceToHost)); break;
    case ELAS_STAGE_PN_OUTPUT: CK(cudaMemcpy(dst, h->pn_out, need, cudaMemcpyDeviceToHost)); break;
    case ELAS_STAGE_PN_BINS: CK(cudaMemcpy(dst, h->pn_bins, need, cudaMemcpyDeviceToHost)); break;
    case ELAS_STAGE_DEL_COUNTERS:
        CK(cudaMemcpy(dst, h->del[0].ctr, 16 * 4, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(static_cast<char*>(dst) + 64, h->del[1].ctr, 16 * 4, cudaMemcpyDeviceToHost));
        break;
    default: return fail(h, ELAS_ERR_INVALID_ARG, "bad stage");
    }
    return ELAS_OK;
}

int elas_b200_set_proposal(elas_handle* h, const float* params, int32_t n) {
    if (!h) return ELAS_ERR_INVALID_ARG;
    CK(cudaSetDevice(h->device));
    return set_proposal_weights(h, params, n);
}

int elas_b200_proposal_stats(elas_handle* h, int32_t* out, int32_t n) {
    if (!h || !out || n < 2) return ELAS_ERR_INVALID_ARG;
    if (!h->pn_used) { out[0] = out[1] = 0; return ELAS_OK; }
    CK(cudaSetDevice(h->device));
    CK(cudaDeviceSynchronize());
    int32_t st[4];
    CK(cudaMemcpy(st, h->pn_stats, sizeof(st), cudaMemcpyDeviceToHost));
    out[0] = st[0];
    out[1] = st[1];
    return ELAS_OK;
}

int elas_b200_pn_infer(elas_handle* h, const void* d_in, void* d_out, int32_t hd, int32_t wd, void* stream) {
    if (!h || !d_in || !d_out || hd <= 0 || wd <= 0) return ELAS_ERR_INVALID_ARG;
    if (!h->prop) return fail(h, ELAS_ERR_INVALID_ARG, "no proposal weights set");
    CK(cudaSetDevice(h->device));
    Geom g{};
    g.W = 4 * wd;
    g.H = 4 * hd;
    g.cw = g.ch = 0;
    int rc = ensure_pn(h, g);
    if (rc != ELAS_OK) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned* err = reinterpret_cast<unsigned*>(h->pn_stats + 2);
    CK(cudaMemsetAsync(err, 0, sizeof(unsigned), st));
    CK(pn::launch_infer(h->pw, static_cast<const __nv_bfloat16*>(d_in), h->pn_a0, h->pn_a1,
                        static_cast<__nv_bfloat16*>(d_out), hd, wd, h->num_sms, err, st));
    h->launches += pn::LAYERS;
    unsigned e = 0;
    CK(cudaMemcpyAsync(&e, err, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (e) return fail(h, ELAS_ERR_TIMEOUT, "proposal inference: a bounded wait ran out");
    return ELAS_OK;
}

int elas_b200_pn_features(elas_handle* h, void* d_out, void* stream) {
    if (!h || !d_out) return ELAS_ERR_INVALID_ARG;
    if (!h->have_last) return fail(h, ELAS_ERR_INVALID_ARG, "no previous call");
    CK(cudaSetDevice(h->device));
    CK(pn::launch_features(h->desc0, h->desc1, static_cast<__nv_bfloat16*>(d_out), h->g.W, h->g.H,
                           static_cast<cudaStream_t>(stream)));
    h->launches += 1;
    return ELAS_OK;
}

int elas_b200_pn_bf16_to_f32(const void* d_in, float* d_out, size_t n, void* stream) {
    if (!d_in || !d_out) return ELAS_ERR_INVALID_ARG;
    cudaError_t e = pn::launch_bf16_to_f32(static_cast<const __nv_bfloat16*>(d_in), d_out, n,
                                           static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? ELAS_OK : ELAS_ERR_CUDA;
}

int elas_b200_pn_conv_forward(const float* x, const float* w, const float* b, float* y, int32_t nimg, int32_t hd,
                              int32_t wd, int32_t relu, void* stream) {
    if (!x || !w || !y || nimg <= 0 || hd <= 0 || wd <= 0) return ELAS_ERR_INVALID_ARG;
    cudaError_t e = pn::launch_conv_f32(x, nullptr, w, b, y, nimg, hd, wd, relu, static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? ELAS_OK : ELAS_ERR_CUDA;
}

int elas_b200_pn_conv_backward(const float* x, const float* y, const float* w, const float* dy, float* dx,
                               float* dw, float* db, float* w_scratch, int32_t nimg, int32_t hd, int32_t wd,
                               int32_t relu, void* stream) {
    if (!x || !y || !w || !dy || !dw || !db || !w_scratch || nimg <= 0 || hd <= 0 || wd <= 0)
        return ELAS_ERR_INVALID_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const float* mask = relu ? y : nullptr;
    cudaError_t e = pn::launch_conv_wgrad(x, dy, mask, dw, db, nimg, hd, wd, st);
    if (e == cudaSuccess && dx) {
        e = pn::launch_flip_weights(w, w_scratch, st);
        if (e == cudaSuccess) e = pn::launch_conv_f32(dy, mask, w_scratch, nullptr, dx, nimg, hd, wd, 0, st);
    }
    return e == cudaSuccess ? ELAS_OK : ELAS_ERR_CUDA;
}

int elas_b200_pn_corr_loss(const float* f, const int32_t* labels, int32_t nlab, int32_t hd, int32_t wd,
                           int32_t disp_max, float* df, float* loss_sum, int32_t* correct, void* stream) {
    if (!f || !df || !loss_sum || !correct || nlab < 0 || (nlab > 0 && !labels) || hd <= 0 || wd <= 0 ||
        disp_max < 1)
        return ELAS_ERR_INVALID_ARG;
    cudaError_t e = pn::launch_corr_loss(f, labels, nlab, hd, wd, disp_max, df, loss_sum, correct,
                                         static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? ELAS_OK : ELAS_ERR_CUDA;
}

int elas_b200_pn_adam(float* p, const float* g, float* m, float* v, int32_t n, float lr, float beta1, float beta2,
                      float eps, int32_t step, void* stream) {
    if (!p || !g || !m || !v || n <= 0 || step < 1) return ELAS_ERR_INVALID_ARG;
    cudaError_t e = pn::launch_adam(p, g, m, v, n, lr, beta1, beta2, eps, step, static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? ELAS_OK : ELAS_ERR_CUDA;
}

}  // extern "C"
