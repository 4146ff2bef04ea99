/*
 * elas_b200.h -- C ABI of the B200-native ELAS stereo matcher.
 *
 * The library replaces the GPU pipeline behind the reference's
 *   void Elas::process(uint8_t* h_img0, uint8_t* h_img1,
 *                      float* h_disp0, float* h_disp1, const int32_t* dims)
 * (reference src/Elas.h:76-83, body src/Elas.cu:19-120).  Every entry point
 * takes plain pointers and sizes, returns an int status (ELAS_OK == 0) and
 * never exits the process (the reference calls exit() on any CUDA error,
 * src/Utils.h:11-38).
 *
 * Threading: a handle owns its device workspaces and is used by one host
 * thread at a time.  Work is enqueued on the stream passed to each call
 * (NULL = the legacy default stream); host-buffer calls return after the
 * results are in host memory.
 */
#ifndef ELAS_B200_H
#define ELAS_B200_H

#include <stddef.h>
#include <stdint.h>
#ifndef __cplusplus
#include <stdbool.h>
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define ELAS_B200_VERSION 1

/* status codes */
#define ELAS_OK                 0
#define ELAS_ERR_INVALID_ARG    1  /* null pointer, bad size, bad parameter */
#define ELAS_ERR_UNSUPPORTED    2  /* parameter combination not implemented */
#define ELAS_ERR_CUDA           3  /* a CUDA runtime call failed */
#define ELAS_ERR_OOM            4  /* device or host allocation failed */
#define ELAS_ERR_INTERNAL       5  /* a device-side consistency check failed */
#define ELAS_ERR_NO_DEVICE      6  /* no usable sm_100 device */
#define ELAS_ERR_TIMEOUT        7  /* a bounded device loop hit its limit */
#define ELAS_ERR_TOO_LARGE      8  /* input exceeds the fixed scratch of elas_b200_speckle_noalloc */

/*
 * Parameter block.  Field order, types and meaning are those of
 * Elas::parameters (reference src/Elas.h:14-40) so the struct is
 * byte-compatible with it.  Unlike the reference, whose kernels read
 * compile-time macros (src/Kernels/KernelsCommon.h:8-27), every field that
 * has a macro counterpart is honoured at run time.
 */
typedef struct elas_params {
    int32_t disp_min;               /* min disparity (support sweep starts at max(disp_min,0)) */
    int32_t disp_max;               /* max disparity */
    float   support_threshold;      /* max uniqueness ratio best / second best */
    int32_t support_texture;        /* min texture for support points */
    int32_t candidate_stepsize;     /* step of the support candidate lattice */
    int32_t incon_window_size;      /* half window of the inconsistency filter */
    int32_t incon_threshold;        /* disparity similarity of the inconsistency filter */
    int32_t incon_min_support;      /* min number of consistent support points */
    bool    add_corners;            /* frame the support points with the four image corners (declared
                                       but unimplemented in the reference; implemented here, and on
                                       in the Elas::parameters() defaults, src/Elas.h:51) */
    int32_t grid_size;              /* cell size of the disparity candidate grid */
    float   beta;                   /* image likelihood parameter */
    float   gamma;                  /* prior constant */
    float   sigma;                  /* prior sigma */
    float   sradius;                /* prior sigma radius */
    int32_t match_texture;          /* min texture for dense matching */
    int32_t lr_threshold;           /* left/right consistency threshold */
    float   speckle_sim_threshold;  /* similarity threshold for speckle segmentation */
    int32_t speckle_size;           /* speckles smaller than this are removed (0 = off) */
    int32_t ipol_gap_width;         /* gaps up to this width are interpolated (0 = off) */
    bool    filter_median;          /* 3x3 median filter */
    bool    filter_adaptive_mean;   /* edge-preserving adaptive mean filter */
    bool    postprocess_only_left;  /* post-filters on D1 only */
    bool    subsampling;            /* outputs at every second row and column: (W/2) x (H/2) maps
                                     * (disparities in full-resolution pixels); L/R check and
                                     * post-filters on the half-size maps.  The reference declares
                                     * the field only (src/Elas.h:37-39); this is the project's mode */
} elas_params;

/* Defaults of the Elas::parameters constructor (reference src/Elas.h:42-66). */
void elas_params_default(elas_params* p);

/* The values the reference kernels are compiled with
 * (src/Kernels/KernelsCommon.h:8-27: DISP_MAX 255, SUPPORT_THRESHOLD 0.85,
 * GAMMA 3, SRADIUS 2, ...) with every post-filter off, because the
 * reference's process() stops after the left/right check
 * (src/Elas.cu:107-119).  With these parameters the output equals the
 * reference's. */
void elas_params_reference(elas_params* p);

/* Human-readable text for a status code. */
const char* elas_b200_status_string(int status);

typedef struct elas_handle elas_handle;

/* Create a matcher bound to CUDA device `device` (reference: the Elas()
 * constructor, src/Elas.h:70-72, which reads device 0's properties).
 * `params` may be NULL for elas_params_default(). */
int elas_b200_create(const elas_params* params, int device, elas_handle** out);

/* Release the handle and its device workspaces. */
int elas_b200_destroy(elas_handle* h);

/* Replace the parameter block used by subsequent calls. */
int elas_b200_set_params(elas_handle* h, const elas_params* params);
int elas_b200_get_params(const elas_handle* h, elas_params* out);

/* Text of the last error on this handle ("" when none). */
const char* elas_b200_last_error(const elas_handle* h);

/*
 * Drop-in for Elas::process (src/Elas.h:76-83, src/Elas.cu:19-120).
 *   left, right : host uint8 images, dims[0] x dims[1], row-major, stride dims[0]
 *   disp_left, disp_right : host float outputs of dims[0]*dims[1] values
 *                 ((dims[0]/2)*(dims[1]/2) with subsampling, row stride dims[0]/2);
 *                 -1 marks an invalid pixel, as in the reference.
 *   dims        : only dims[0] (width) and dims[1] (height) are read
 *                 (the reference ignores a libelas-style dims[2]).
 *   stream      : cudaStream_t (NULL = legacy default stream).
 * Blocks until the outputs are in host memory.
 */
int elas_b200_process(elas_handle* h, const uint8_t* left, const uint8_t* right,
                      float* disp_left, float* disp_right, const int32_t* dims,
                      void* stream);

/* Same computation on caller-owned device buffers; asynchronous on `stream`
 * (no host synchronisation except the one-off workspace growth). */
int elas_b200_process_device(elas_handle* h, const uint8_t* d_left, const uint8_t* d_right,
                             float* d_disp_left, float* d_disp_right, const int32_t* dims,
                             void* stream);

/*
 * Batched form: n independent pairs of possibly different sizes.  lefts[i],
 * rights[i], disp_lefts[i], disp_rights[i] are host pointers; dims holds
 * 2*n int32 (w_i, h_i); disp_max_per_pair (nullable) overrides the handle's
 * disp_max per pair.  Outputs equal n single elas_b200_process calls.
 */
int elas_b200_process_batch(elas_handle* h, int n,
                            const uint8_t* const* lefts, const uint8_t* const* rights,
                            float* const* disp_lefts, float* const* disp_rights,
                            const int32_t* dims, const int32_t* disp_max_per_pair,
                            void* stream);

/*
 * Batched form on device buffers (pointer arrays in host memory).  Pair i
 * runs on its own worker (workspace + stream); the whole batch -- fork, n
 * pipelines, join -- is captured once into a CUDA graph and later calls with
 * the same sizes, disparity ranges, buffers, parameters and stream replay it
 * with a single graph launch.  The first call of a new signature runs
 * eagerly (sizing workspaces, tuning the dense kernel) and then captures.
 * stream NULL: an internal stream, and the call returns when done.
 * No counterpart in the reference (one pair per call, src/Elas.cu:19).
 */
int elas_b200_process_batch_device(elas_handle* h, int n,
                                   const uint8_t* const* d_lefts, const uint8_t* const* d_rights,
                                   float* const* d_disp_lefts, float* const* d_disp_rights,
                                   const int32_t* dims, const int32_t* disp_max_per_pair,
                                   void* stream);

/* Capture and replay as CUDA graphs (1, default) or run eagerly (0): batches,
 * and single pairs through elas_b200_process / _process_device, whose second
 * call with the same buffers, size, parameters and settings is captured (on
 * the handle's own stream) and whose later calls replay the graph.  A caller
 * that is itself capturing a stream gets plain launches. */
int elas_b200_set_graphs(elas_handle* h, int enable);

/* Fallback switches, for tests of paths that the usual inputs never reach.
 * No counterpart in the reference (its Delaunay runs on the CPU and its
 * dense kernel has one path, src/Kernels/KerComputeDisparity.cu:155-316).
 *   ELAS_TEST_DELAUNAY_FLIPS the triangulations are built from row strips
 *                           and repaired by edge flips (otherwise above
 *                           2^21 pixels) instead of being found star by
 *                           star (the same triangles, listed in another
 *                           order);
 *   ELAS_TEST_DELAUNAY_STARS the triangulations are found star by star
 *                           (otherwise up to 2^21 pixels); not together
 *                           with the flip switches or a round limit;
 *   ELAS_TEST_FLIP_GLOBAL   (implies the flip construction) every
 *                           triangulation is flipped by the global-
 *                           memory kernel, which otherwise runs only for
 *                           triangulations larger than a cluster holds;
 *   ELAS_TEST_DENSE_BITSET  every grid cell's candidates are walked as a
 *                           bitset, the path otherwise taken only by cells
 *                           with more candidates than the per-row list holds;
 *   ELAS_TEST_PRIOR_TILED   the plane prior is painted tile by tile in shared
 *                           memory (otherwise from 2^20 pixels up);
 *   ELAS_TEST_PRIOR_DIRECT  the plane prior is painted with global atomics
 *                           (otherwise below 2^20 pixels); not together with
 *                           ELAS_TEST_PRIOR_TILED;
 *   ELAS_TEST_PRIOR_SMALL_BINS the tiled paint keeps 2 triangles per tile in
 *                           each tile's bin (otherwise 128), so that most go
 *                           through the overflow list.
 * The results are the same as without the flags.  flip_round_limit > 0
 * (which implies the flip construction) caps the edge-flipping rounds
 * (0 = the library's own bound); a
 * triangulation that needs more rounds makes the call return
 * ELAS_ERR_TIMEOUT with the device still usable.  Batches pass the settings
 * on to their workers. */
#define ELAS_TEST_FLIP_GLOBAL   1
#define ELAS_TEST_DENSE_BITSET  2
#define ELAS_TEST_PRIOR_TILED   4
#define ELAS_TEST_PRIOR_DIRECT  8
#define ELAS_TEST_DELAUNAY_FLIPS 16
#define ELAS_TEST_DELAUNAY_STARS 32
#define ELAS_TEST_PRIOR_SMALL_BINS 256
int elas_b200_set_test_mode(elas_handle* h, int32_t flags, int32_t flip_round_limit);

/* Per-pair latency (ms from the batch's start to the pair's completion) of
 * the last batch.  Returns the number of pairs (>= 0), or minus a status
 * code (too small an output, a failed event query). */
int elas_b200_batch_latency(elas_handle* h, float* ms_out, int n);

/* Threads per CTA the dense-matching autotuner chose for this width class
 * and disparity range (0 = not tuned yet). */
int elas_b200_dense_shape(const elas_handle* h, int32_t width, int32_t disp_max);

/* ---- learned support-point proposal (no counterpart in the reference) ----
 *
 * A 4-layer 3x3 CNN (32 channels, bf16 with fp32 accumulation, tcgen05
 * implicit-GEMM kernels) over the descriptors pooled to 4x4-pixel cells
 * scores 64 disparity bins per support candidate; the candidate is first
 * matched only on its 4 best bins (each widened by 2 pixels) and must pass
 * the same uniqueness and left/right tests there, else it falls back to the
 * full sweep of the reference (src/Kernels/KerSupportMatches.cu:12-193).
 * Parameters: ELAS_PN_PARAMS floats, per layer W[tap][ci][co] then b[co]. */
#define ELAS_PN_PARAMS 36992

/* Enable the proposal with these parameters (n == ELAS_PN_PARAMS) or
 * disable it (n == 0). */
int elas_b200_set_proposal(elas_handle* h, const float* params, int32_t n);

/* Candidates of the last call settled by the proposal (out[0]) and sent to
 * the full sweep (out[1]); zeros when the proposal did not run. */
int elas_b200_proposal_stats(elas_handle* h, int32_t* out, int32_t n);

/* The network alone on caller features (bf16 [2][hd][wd][32] in and out,
 * device memory), with the handle's weights; blocks until done. */
int elas_b200_pn_infer(elas_handle* h, const void* d_in, void* d_out, int32_t hd, int32_t wd, void* stream);

/* Training kernels (fp32, device pointers, asynchronous on `stream`).
 * Feature maps are [nimg][hd][wd][32]; a pair's left image is 2*pair and
 * its right image 2*pair+1. */
int elas_b200_pn_features(elas_handle* h, void* d_out, void* stream);  /* bf16 input features of the last call */
int elas_b200_pn_bf16_to_f32(const void* d_in, float* d_out, size_t n, void* stream);
int elas_b200_pn_conv_forward(const float* x, const float* w, const float* b, float* y, int32_t nimg, int32_t hd,
                              int32_t wd, int32_t relu, void* stream);
/* dw, db accumulate (+=); dx (nullable) is overwritten; w_scratch holds
 * 9*32*32 floats. */
int elas_b200_pn_conv_backward(const float* x, const float* y, const float* w, const float* dy, float* dx,
                               float* dw, float* db, float* w_scratch, int32_t nimg, int32_t hd, int32_t wd,
                               int32_t relu, void* stream);
/* Mean softmax cross-entropy over labels (nlab x {pair, cx, cy, bin}):
 * adds the summed loss to *loss_sum, the count of top-1 hits to *correct
 * and the gradient to df (accumulated). */
int elas_b200_pn_corr_loss(const float* f, const int32_t* labels, int32_t nlab, int32_t hd, int32_t wd,
                           int32_t disp_max, float* df, float* loss_sum, int32_t* correct, void* stream);
int elas_b200_pn_adam(float* p, const float* g, float* m, float* v, int32_t n, float lr, float beta1, float beta2,
                      float eps, int32_t step, void* stream);

/* ---- introspection of the last call (for stage-wise parity checks) ---- */

/* Stages that can be copied out after a process call. */
#define ELAS_STAGE_DESC_LEFT     0   /* uint8  [h][w][16] */
#define ELAS_STAGE_DESC_RIGHT    1   /* uint8  [h][w][16] */
#define ELAS_STAGE_CAN_LR        2   /* int32  [ch][cw] after the L->R and R->L sweeps */
#define ELAS_STAGE_CAN           3   /* int32  [ch][cw] after inconsistency + redundancy filters */
#define ELAS_STAGE_SUPPORT       4   /* int32  [n][3] (u, v, d) in candidate raster order */
#define ELAS_STAGE_GRID_LEFT     5   /* int32  [gh][gw][disp_max+2] {count, d0 < d1 < ...} */
#define ELAS_STAGE_GRID_RIGHT    6   /* int32  [gh][gw][disp_max+2] */
#define ELAS_STAGE_TRI_LEFT      7   /* int32  [t][3] support indices, CCW, smallest index first */
#define ELAS_STAGE_TRI_RIGHT     8   /* int32  [t][3] */
#define ELAS_STAGE_PRIOR_LEFT    9   /* int32  [h][w] plane prior d_plane clamped to at most
                                        disp_max + plane_radius + 1; -1 where no triangle covers
                                        the pixel or d_plane <= 0 (the dense step skips both) */
#define ELAS_STAGE_PRIOR_RIGHT  10   /* int32  [h][w] */
#define ELAS_STAGE_DISP_LEFT    11   /* float  [h][w] dense result before the L/R check */
#define ELAS_STAGE_DISP_RIGHT   12   /* float  [h][w] */
#define ELAS_STAGE_LR_LEFT      13   /* float  [h][w] after the L/R check, before post-filters */
#define ELAS_STAGE_LR_RIGHT     14   /* float  [h][w] */
#define ELAS_STAGE_PN_FEATURES  15   /* bf16   [2][h/4][w/4][32] proposal input (left, right) */
#define ELAS_STAGE_PN_OUTPUT    16   /* bf16   [2][h/4][w/4][32] proposal network output */
#define ELAS_STAGE_PN_BINS      17   /* uint32 [ch][cw] top-4 bins per candidate, one byte each
                                      * (best first, 0xff = none) */
#define ELAS_STAGE_DEL_COUNTERS 18   /* int32  [2][16] Delaunay counters per view: [0] triangles,
                                      * [4] flip rounds, [5] flips, [6] non-empty lattice rows,
                                      * [8] set by the flip kernel that ran, [9] support points */
#define ELAS_STAGE_COUNT        19

/* Copy stage `stage` of the last single-pair call into host memory `dst`
 * of `bytes` bytes.  *needed receives the size in bytes (call with
 * dst == NULL to query).  Returns ELAS_ERR_INVALID_ARG if bytes is too small. */
int elas_b200_get_stage(elas_handle* h, int stage, void* dst, size_t bytes, size_t* needed);

/* Number of kernels this handle has launched since creation. */
int64_t elas_b200_launch_count(const elas_handle* h);

/* ---- per-stage device timing (CUDA events on the launch stream) ---- */

#define ELAS_TIME_DESCRIPTOR  0   /* fused Sobel + descriptor, both views */
#define ELAS_TIME_SUPPORT     1   /* support sweep L->R and R->L + filters */
#define ELAS_TIME_COMPACT     2   /* support list compaction */
#define ELAS_TIME_GRID        3   /* disparity grid, both views */
#define ELAS_TIME_DELAUNAY    4   /* triangulation, both views */
#define ELAS_TIME_PRIOR       5   /* plane prior, both views */
#define ELAS_TIME_DENSE       6   /* dense matching, both views */
#define ELAS_TIME_LR          7   /* left/right check */
#define ELAS_TIME_POST        8   /* post-filters */
#define ELAS_TIME_COUNT       9

/* Enable (1) or disable (0) recording of per-stage events. */
int elas_b200_set_timing(elas_handle* h, int enable);

/* Wait for the last call and write its per-stage device times in ms
 * (ELAS_TIME_COUNT values) to ms_out. */
int elas_b200_get_timing(elas_handle* h, float* ms_out, int n);

/* ---- pair-parallel batches over several GPUs ---- */

/*
 * A group of matchers, one handle per entry of `devices` (a device may
 * appear more than once).  No counterpart in the reference, which runs one
 * pair on device 0 (src/Elas.h:70-83).  Stereo pairs are independent, so a
 * batch is dealt to the devices with no exchange between them: no peer
 * memory access and no collective.
 */
typedef struct elas_group elas_group;
int elas_b200_group_create(const elas_params* params, const int32_t* devices, int ndev, elas_group** out);
int elas_b200_group_destroy(elas_group* g);
int elas_b200_group_set_params(elas_group* g, const elas_params* params);
const char* elas_b200_group_last_error(const elas_group* g);

/* The plan a group batch uses: pair i goes to device entry assign[i].
 * Pairs are taken largest estimated cost first (width * height *
 * (1 + disp_max / 128)), each to the least-loaded entry; equal costs keep
 * pair order, so the plan is a pure function of its inputs (host only, no
 * device needed).  disp_max_per_pair (nullable) overrides disp_max. */
int elas_b200_group_plan(int n, const int32_t* dims, const int32_t* disp_max_per_pair, int32_t disp_max, int ndev,
                         int32_t* assign);

/* elas_b200_process_batch over the group: every device entry runs its share
 * of the plan as one batch on its own host thread; blocks until all outputs
 * are in host memory.  assign_out (nullable) receives the plan.  Outputs
 * equal single-pair elas_b200_process calls with each pair's disp_max. */
int elas_b200_group_process_batch(elas_group* g, int n,
                                  const uint8_t* const* lefts, const uint8_t* const* rights,
                                  float* const* disp_lefts, float* const* disp_rights,
                                  const int32_t* dims, const int32_t* disp_max_per_pair,
                                  int32_t* assign_out);

/* ---- allocation-free speckle removal ---- */

/* Largest image (width * height) elas_b200_speckle_noalloc accepts. */
#define ELAS_NOALLOC_MAX_PIXELS (1 << 19)

/*
 * Speckle removal on one disparity map without any memory allocation, for
 * callers that may not call cudaMalloc: code running while a stream is
 * being captured into a CUDA graph (cudaMalloc is not capturable), plugin
 * hosts and real-time loops that forbid allocation after start-up, and
 * tools that must not touch the device allocator.  No counterpart in the
 * reference, which has no post-filters.
 *
 *   d_in, d_out   : device float maps of width*height values (-1 = invalid);
 *                   they may be the same buffer.
 *   sim_threshold : neighbours with |d_p - d_q| <= sim_threshold connect.
 *   min_size      : 4-connected segments smaller than this become -1.
 *   stream        : cudaStream_t (NULL = legacy default stream); asynchronous.
 * The result equals the speckle stage of elas_b200_process run with
 * speckle_size = min_size and speckle_sim_threshold = sim_threshold.
 *
 * Scratch lives in one fixed array of 3 * ELAS_NOALLOC_MAX_PIXELS int32
 * (6 MiB) in the library's device image; every GPU that loads the library
 * holds it until the process exits.  width * height above
 * ELAS_NOALLOC_MAX_PIXELS returns ELAS_ERR_TOO_LARGE; any aspect ratio
 * within it is accepted.  The first call on a device, and the first after a
 * cudaDeviceReset, looks up the array's device address
 * (cudaGetSymbolAddress), so make that call outside any stream capture.
 * All calls share the array: calls that overlap on the GPU (other streams,
 * other threads) race and give wrong results; serialise them.
 *
 * The call is asynchronous and returns only host-side and launch errors.
 * The kernels' own bounds check is not reported: valid inputs cannot
 * trigger it (every union-find walk and retry loop is bounded well above
 * the 2^19 steps a map of this size can need).
 */
int elas_b200_speckle_noalloc(const float* d_in, float* d_out, int32_t width, int32_t height,
                              float sim_threshold, int32_t min_size, void* stream);

/* ---- seeded synthetic stereo pairs (the benchmark inputs) ---- */

/* Scene presets: 0 = 450x375 D 0-63 (6 planes, two 40x40 textureless
 * patches); 1 = 1242x375 D 0-255 (12 planes incl. a ground plane, 8%
 * textureless); 2 = 2880x1988 D 0-511 (40 planes + 2 px sinusoidal ripple);
 * 3 = batch member (size and disp_max from the arguments).  w/h/disp_max
 * <= 0 take the preset's values.  gt_left / gt_right (nullable) receive the
 * float ground-truth disparity of each view. */
int elas_b200_synth_pair(int preset, uint64_t seed, int32_t w, int32_t h, int32_t disp_max,
                         uint8_t* left, uint8_t* right, float* gt_left, float* gt_right);

/* Preset geometry (width, height, disp_max) for a scene preset. */
int elas_b200_synth_dims(int preset, int32_t* w, int32_t* h, int32_t* disp_max);

#ifdef __cplusplus
}
#endif

#endif /* ELAS_B200_H */
