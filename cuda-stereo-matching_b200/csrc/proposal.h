// Learned support-point proposal: shared constants and launchers (internal
// interface of the library).  The network and the proposal rule are defined
// in csrc/k_proposal.cu.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cstdint>

#include "common.cuh"

namespace elas {
namespace pn {

constexpr int CH = 32;                       // channels of every layer
constexpr int TAPS = 9;                      // 3x3
constexpr int LAYERS = 4;
constexpr int NBINS = 64;                    // disparity bins of the scores
constexpr int TOPK = 4;                      // bins in the search set
constexpr int MARGIN = 2;                    // pixels added on both sides of a bin
constexpr float SCALE = 0.125f;              // score = SCALE * <F_L, F_R>
constexpr int LAYER_PARAMS = TAPS * CH * CH + CH;
constexpr int NPARAMS = LAYERS * LAYER_PARAMS;
constexpr uint32_t NO_BIN = 0xffu;           // unused byte of a packed bin set

// Bin width in pixels for disparities 0..D, and the cell shift of bin b.
HD int bin_width(int D) { return (D + 1 + NBINS - 1) / NBINS; }
HD int bin_shift(int b, int w) { return (b * w + w / 2) / 4; }

// Training (fp32) --------------------------------------------------------
cudaError_t launch_features(const uint4* desc0, const uint4* desc1, __nv_bfloat16* out, int W, int H,
                            cudaStream_t st);
cudaError_t launch_bf16_to_f32(const __nv_bfloat16* in, float* out, size_t n, cudaStream_t st);
// y = act(conv(x * (mask > 0)) + b) over nimg images; mask and b nullable.
cudaError_t launch_conv_f32(const float* x, const float* mask, const float* w, const float* b, float* y, int nimg,
                            int Hd, int Wd, int relu, cudaStream_t st);
cudaError_t launch_flip_weights(const float* w, float* wt, cudaStream_t st);
// dw += sum x (x) g, db += sum g with g = dy * (y > 0) (y nullable: no mask).
cudaError_t launch_conv_wgrad(const float* x, const float* dy, const float* y, float* dw, float* db, int nimg,
                              int Hd, int Wd, cudaStream_t st);
// labels: nlab x (pair, cx, cy, bin); F holds images 2*pair (left) and 2*pair+1 (right).
cudaError_t launch_corr_loss(const float* F, const int32_t* labels, int nlab, int Hd, int Wd, int D, float* dF,
                             float* loss_sum, int32_t* correct, cudaStream_t st);
cudaError_t launch_adam(float* p, const float* g, float* m, float* v, int n, float lr, float b1, float b2, float eps,
                        int t, cudaStream_t st);

// Inference (bf16, tcgen05) ----------------------------------------------
// Device weights of the inference path: per layer 9 taps of a [32 co][32 ci]
// bf16 B operand, then fp32 biases.
struct InferWeights {
    __nv_bfloat16* w;   // [LAYERS][TAPS][CH][CH]
    float* b;           // [LAYERS][CH]
};
cudaError_t upload_weights(const float* host_params, InferWeights& iw, cudaStream_t st);
// Four layers over the two feature maps of a pair: in -> act0 -> act1 -> act0 -> out.
cudaError_t launch_infer(const InferWeights& iw, const __nv_bfloat16* in, __nv_bfloat16* act0, __nv_bfloat16* act1,
                         __nv_bfloat16* out, int Hd, int Wd, int num_sms, unsigned* err, cudaStream_t st);
// Top-4 bins of every candidate of the lattice (cw x ch, step), packed one
// byte per bin (best first, NO_BIN when fewer are valid).
cudaError_t launch_topk(const __nv_bfloat16* F, uint32_t* bins, int Hd, int Wd, int cw, int ch, int step, int D,
                        cudaStream_t st);

}  // namespace pn
}  // namespace elas
