// net_kernels.cuh — device kernels of the learned initial-guess network.
//
// Tensors are NHWC bf16 (channels innermost), one image per batch entry.  The
// 3x3 convolutions ("same" size, zero padding) are implicit GEMMs on the tensor
// cores (tcgen05.mma for widths that are multiples of 128, mma.sync m16n8k16
// otherwise and for the weight gradients; bf16 inputs, FP32 accumulation):
//   forward        out[p][co] = Σ_tap Σ_ci x[p + tap][ci] · Wf[tap][co][ci]
//   backward data  the same kernel with Wb[tap][ci][co] = W[8 - tap][ci][co]
//   weight grads   dW[tap][ci][co] = Σ_p x[p + tap][ci] · g[p][co]
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cstdint>

namespace cdm {
namespace net {

enum Epilogue : int {
  EPI_NONE = 0,   // out = acc (+ bias)
  EPI_RELU = 1,   // out = max(acc + bias, 0)
  EPI_MASK = 2,   // out = acc · (mask > 0)       (ReLU derivative of the layer below)
};

struct ConvArgs {
  const __nv_bfloat16* x;   // [B][H][W][CIN]
  const __nv_bfloat16* w;   // [9][COUT][CIN]
  const float* bias;        // [COUT] or NULL
  const __nv_bfloat16* mask;  // [B][H][W][COUT] for EPI_MASK
  __nv_bfloat16* out;       // [B][H][W][COUT] (bf16 output) or NULL
  float* out_f32;           // [B][H][W][COUT] (fp32 output) or NULL
  int B, H, W;
  int epi;
};

struct WgradArgs {
  const __nv_bfloat16* x;   // [B][H][W][CIN]
  const __nv_bfloat16* g;   // [B][H][W][COUT]
  float* dw;                // [9][CIN][COUT], accumulated
  float* db;                // [COUT], accumulated
  int B, H, W;
};

// Dispatch: the tcgen05 kernel (net_conv_tc.cu) for images whose width is a
// multiple of 128, the mma.sync kernel otherwise or when the environment
// variable CDM_NET_CONV is "mma" (kept for comparisons).
cudaError_t conv3x3(int cin, int cout, const ConvArgs& a, cudaStream_t s);
// tcgen05 / TMA convolution (forward and backward-data), M = 128 pixels per tile
bool conv3x3_tc_supported(int cin, int cout, int W);
cudaError_t conv3x3_tc(int cin, int cout, const ConvArgs& a, cudaStream_t s);
// *flag = 1 when a bounded wait of the tcgen05 convolution ran out since the last
// call (the flag is cleared); call after the stream has been synchronised
cudaError_t conv3x3_tc_error(int* flag);
cudaError_t conv3x3_wgrad(int cin, int cout, const WgradArgs& a, cudaStream_t s);

// elementwise helpers (C = 32 channels)
cudaError_t pool2(const __nv_bfloat16* in, __nv_bfloat16* out, int B, int H, int W, cudaStream_t s);
cudaError_t up_add(const __nv_bfloat16* coarse, const __nv_bfloat16* skip, __nv_bfloat16* out, int B, int H, int W,
                   cudaStream_t s);
cudaError_t up_bwd_mask(const __nv_bfloat16* gfine, const __nv_bfloat16* mask, __nv_bfloat16* gcoarse, int B, int H,
                        int W, cudaStream_t s);
cudaError_t pool_bwd_add_mask(const __nv_bfloat16* ga, const __nv_bfloat16* gp, const __nv_bfloat16* mask,
                              __nv_bfloat16* out, int B, int H, int W, cudaStream_t s);

// features / targets / loss / guess (see net_kernels.cu for their definitions)
struct FeatArgs {
  const double* const* tprev;  // per sample: full arrays (nx x ny, i fastest)
  const double* const* tcur;
  const double* const* tnext;  // NULL for inference
  const double* J;             // full array, shared by all samples
  const int* ox;               // per sample crop origin (domain cell index)
  const int* oy;
  const double* scale;         // per sample ΔT scale
  int nx, nh;                  // full row length, halo width
  int B, H, W;                 // crop size
  double k0, kn, log_jmean;
  double dt, rho_cp;           // loss weights when dt > 0 (see features_kernel)
  __nv_bfloat16* x;            // [B][H][W][16]
  float* target;               // [B][H][W] or NULL
  float* weight;               // [B][H][W] or NULL
};
cudaError_t features(const FeatArgs& a, cudaStream_t s);
cudaError_t delta_scale(const double* const* tprev, const double* const* tcur, int nsamp, int ni, int nj, int nx,
                        int nh, double* acc, cudaStream_t s);
cudaError_t finish_scale(double* acc, int nsamp, int64_t ncells, cudaStream_t s);
cudaError_t loss_grad(const float* y, const float* target, const float* weight, __nv_bfloat16* gy, int64_t npix,
                      float* loss_acc, cudaStream_t s);
cudaError_t smooth3x3(const float* in, int in_stride, float* out, int H, int W, cudaStream_t s);
cudaError_t apply_guess(const double* tprev, const double* tcur, const float* y, int y_stride, const double* scale,
                        double* u0, int ni, int nj, int nx, int nh, cudaStream_t s);

// parameters: master fp32 W[9][cin][cout] → Wf bf16 [9][cout][cin], Wb bf16 [9][cin][cout] (flipped taps)
cudaError_t prep_weights(const float* w, __nv_bfloat16* wf, __nv_bfloat16* wb, int cin, int cout, cudaStream_t s);
cudaError_t adam(float* p, const float* g, float* m, float* v, int64_t n, float lr, float b1, float b2, float eps,
                 float c1, float c2, cudaStream_t s);

}  // namespace net
}  // namespace cdm
