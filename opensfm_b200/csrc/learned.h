// Host-side entry points of the learned-initialisation kernels (learned.cu).
#pragma once

#include <cuda_bf16.h>

#include "kernels.h"

namespace dn {

constexpr int kFeatC = 32;  // network input channels (1 + 2 x planes used, zero padded)
// Sweep planes: channel 0 is the intensity, 1 + 2 p + k the NCC of plane p
// against matching view k (k < 2).
constexpr int kMaxSweepPlanes = (kFeatC - 1) / 2;

struct ConvArgs {
  const __nv_bfloat16* x;       // input activations [n_pix][cin]
  const __nv_bfloat16* w;       // weights [cout][9 cin]
  const float* bias;            // [cout]
  long long n_pix;              // pixels over the whole batch (images of H x W)
  int H, W, cin, cout, relu;
  __nv_bfloat16* y;             // forward output [n_pix][cout] (BF16) or null
  float* y32;                   // forward output in FP32 or null
  // backward
  const __nv_bfloat16* dy;      // gradient of the (post-activation) output
  const __nv_bfloat16* x_mask;  // input activations for the ReLU mask of dx, or null
  __nv_bfloat16* dx;            // gradient of the input (null: not needed)
  float* dw;                    // [cout][9 cin] accumulated (atomic adds)
  float* db;                    // [cout] accumulated
};

// Forward on the tcgen05 tensor cores (TMEM accumulators); the mma.sync
// variant is kept as the comparison the tests and the bench time it against.
cudaError_t conv3x3_forward(const ConvArgs& c, cudaStream_t s);
cudaError_t conv3x3_forward_mma_sync(const ConvArgs& c, cudaStream_t s);
// 1 if a bounded wait of the tcgen05 forward expired since the last call
// (and clears it), 0 if not, -1 if the flag could not be read.
int take_tc_error();
cudaError_t conv3x3_backward(const ConvArgs& c, __nv_bfloat16* wt_scratch, cudaStream_t s);
// The same backward on the tcgen05 tensor cores: weight and bias gradients
// as a split-K GEMM with TMEM accumulators, the input gradient as the
// forward kernel on the gradient with flipped weights and the ReLU mask.
// wt_scratch: 32 x 288 BF16; dy_pad: n_pix x 32 BF16 when cout != 32.
cudaError_t conv3x3_backward_tc(const ConvArgs& c, __nv_bfloat16* wt_scratch,
                                __nv_bfloat16* dy_pad, cudaStream_t s);
// Sweep features on the grid of every `stride`-th pixel (1 or 2); map k's
// grid at feat + k map_stride, or at its MapDev::prop_off when map_stride < 0.
cudaError_t launch_sweep(const LaunchArgs& a, __nv_bfloat16* feat, long long map_stride,
                         int n_planes, int stride, cudaStream_t s);
cudaError_t launch_l1_loss(const float* pred, const float* target, long long n_pix,
                           float normal_weight, __nv_bfloat16* dpred, float* loss_sum, float* count,
                           cudaStream_t s);
cudaError_t launch_adam(float* w, float* m, float* v, const float* grad, int n, const float* count,
                        float lr, float b1, float b2, float eps, float bc1, float bc2,
                        __nv_bfloat16* w16, cudaStream_t s);
cudaError_t launch_output_to_planes(const float* out, int W, int H, const MapDev* maps, int map,
                                    float* planes, cudaStream_t s);
cudaError_t launch_planes_to_target(const float4* state, const float* score, int W, int H,
                                    int stride, const MapDev* maps, int map, float min_score,
                                    float* target, cudaStream_t s);
// Network outputs on every map's proposal grid (out + 4 prop_off) -> the
// maps' MapDev::prop_init planes, upsampled by each map's MapDev::prop_S.
cudaError_t launch_proposal_to_planes(const float* out, const MapDev* maps, int n_maps,
                                      int max_pixels, cudaStream_t s);

}  // namespace dn
