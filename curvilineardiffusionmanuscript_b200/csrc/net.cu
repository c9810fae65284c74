// net.cu — the learned initial-guess network: parameters, activations,
// forward / backward schedule, Adam, and the C ABI of cdm_net.h.
//
// Schedule (U-Net with additive skips; level l has (H >> l) x (W >> l) pixels):
//   forward   X →L0a→ A0 →L0b→ S0 →pool→ P1 →L1→ S1 →pool→ P2 →L2→ S2 →pool→ P3 →L3→ B3
//             U2 = up(B3) + S2 →L4→ D2;  U1 = up(D2) + S1 →L5→ D1;  U0 = up(D1) + S0 →L6→ D0 →L7→ Y
//   backward  gY → (W7, gD0 = convᵀ·[D0>0]) → (W6, gU0) → gD1 = up⁻¹(gU0)·[D1>0] → (W5, gU1)
//             → gD2 → (W4, gU2) → gB3 → (W3, gP3) → gS2 = (gU2 + pool⁻¹(gP3))·[S2>0] → (W2, gP2)
//             → gS1 = (gU1 + pool⁻¹(gP2))·[S1>0] → (W1, gP1) → gS0 = (gU0 + pool⁻¹(gP1))·[S0>0]
//             → (W0b, gA0 = convᵀ·[A0>0]) → W0a
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "cdm_apt.h"
#include "cdm_net.h"
#include "engine.h"
#include "net_kernels.cuh"

namespace cdm {
namespace net {

struct Layer {
  int cin, cout;
  int64_t w_off, b_off;  // into the FP32 parameter vector
  __nv_bfloat16* wf = nullptr;
  __nv_bfloat16* wb = nullptr;
};

class Net {
 public:
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  Layer L[9];
  int64_t nparams = 0;
  float *params = nullptr, *grads = nullptr, *m = nullptr, *v = nullptr;
  __nv_bfloat16* wbuf = nullptr;
  int adam_t = 0;
  bool weights_dirty = true;
  // activations for the current shape
  int B = 0, H = 0, W = 0;
  std::vector<void*> allocs;
  __nv_bfloat16 *X = nullptr, *A0, *S0, *U0, *D0, *P1, *S1, *U1, *D1, *P2, *S2, *U2, *D2, *P3, *B3;
  __nv_bfloat16 *gY = nullptr, *ga[4], *gb[4];
  float *Y = nullptr, *target = nullptr, *weight = nullptr, *d_loss = nullptr;
  float *sm0 = nullptr, *sm1 = nullptr;  // smoothing of the predicted correction
  int smooth_passes = 8;
  bool use_weight = false;
  // training batch scratch
  double* d_scale = nullptr;
  const double** d_ptrs = nullptr;  // tprev, tcur, tnext arrays (3 x cap)
  int* d_orig = nullptr;            // ox, oy (2 x cap)
  int cap = 0;

  ~Net() {
    free_acts();
    cudaFree(params);
    cudaFree(grads);
    cudaFree(m);
    cudaFree(v);
    cudaFree(wbuf);
    cudaFree(d_scale);
    cudaFree(d_ptrs);
    cudaFree(d_orig);
    cudaFree(d_loss);
    if (own_stream && stream) cudaStreamDestroy(stream);
  }

  void free_acts() {
    for (void* p : allocs) cudaFree(p);
    allocs.clear();
    B = H = W = 0;
  }

  template <typename T>
  cudaError_t alloc(T** p, size_t n) {
    cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
    if (e == cudaSuccess) allocs.push_back(*p);
    return e;
  }

  int init(int dev, uint64_t seed, void* s) {
    device = dev;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= dev) {
      set_error("no CUDA device available for the guess network");
      return CDM_NO_DEVICE;
    }
    CDM_CK(cudaSetDevice(dev));
    if (s) {
      stream = (cudaStream_t)s;
    } else {
      CDM_CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
      own_stream = true;
    }
    const int cins[9] = {16, 32, 32, 32, 32, 32, 32, 32, 32};
    const int couts[9] = {32, 32, 32, 32, 32, 32, 32, 32, 16};
    int64_t off = 0, woff = 0;
    for (int l = 0; l < 9; ++l) {
      L[l].cin = cins[l];
      L[l].cout = couts[l];
      L[l].w_off = off;
      off += 9 * cins[l] * couts[l];
      L[l].b_off = off;
      off += couts[l];
      woff += 2 * 9 * cins[l] * couts[l];
    }
    nparams = off;
    CDM_CK(cudaMalloc((void**)&params, nparams * sizeof(float)));
    CDM_CK(cudaMalloc((void**)&grads, nparams * sizeof(float)));
    CDM_CK(cudaMalloc((void**)&m, nparams * sizeof(float)));
    CDM_CK(cudaMalloc((void**)&v, nparams * sizeof(float)));
    CDM_CK(cudaMalloc((void**)&wbuf, woff * sizeof(__nv_bfloat16)));
    CDM_CK(cudaMalloc((void**)&d_loss, sizeof(float)));
    int64_t wo = 0;
    for (int l = 0; l < 9; ++l) {
      L[l].wf = wbuf + wo;
      wo += 9 * L[l].cin * L[l].cout;
      L[l].wb = wbuf + wo;
      wo += 9 * L[l].cin * L[l].cout;
    }
    // He initialisation (normal, std √(2 / fan_in)); the input layer's fan-in
    // counts its 4 used channels, the output layer starts near zero so that the
    // initial guess is the linear extrapolation 2Tⁿ − Tⁿ⁻¹
    std::vector<float> h(nparams, 0.0f);
    uint64_t st = seed ^ 0x9e3779b97f4a7c15ull;
    auto next = [&]() {
      st += 0x9e3779b97f4a7c15ull;
      uint64_t z = st;
      z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
      z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
      return (double)((z ^ (z >> 31)) >> 11) * (1.0 / 9007199254740992.0);
    };
    for (int l = 0; l < 9; ++l) {
      const int fan_in = 9 * (l == 0 ? 4 : L[l].cin);
      double sd = std::sqrt(2.0 / fan_in);
      if (l == 8) sd *= 0.01;
      for (int t = 0; t < 9; ++t)
        for (int ci = 0; ci < L[l].cin; ++ci)
          for (int co = 0; co < L[l].cout; ++co) {
            const double u1 = std::max(next(), 1e-300), u2 = next();
            const double z = std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
            const bool live = (l != 0 || ci < 4) && (l != 8 || co < 1);
            h[L[l].w_off + ((int64_t)t * L[l].cin + ci) * L[l].cout + co] = live ? (float)(sd * z) : 0.0f;
          }
    }
    CDM_CK(cudaMemcpyAsync(params, h.data(), nparams * sizeof(float), cudaMemcpyHostToDevice, stream));
    CDM_CK(cudaMemsetAsync(m, 0, nparams * sizeof(float), stream));
    CDM_CK(cudaMemsetAsync(v, 0, nparams * sizeof(float), stream));
    CDM_CK(cudaMemsetAsync(grads, 0, nparams * sizeof(float), stream));
    CDM_CK(cudaStreamSynchronize(stream));
    weights_dirty = true;
    return CDM_OK;
  }

  int ensure_shape(int b, int hh, int ww) {
    if (hh % 8 || ww % 8 || hh < 8 || ww < 8 || b < 1) {
      set_error("network input sizes must be positive multiples of 8");
      return CDM_BAD_INPUT;
    }
    if (b == B && hh == H && ww == W) return CDM_OK;
    free_acts();
    const size_t n0 = (size_t)b * hh * ww, c = 32;
    const size_t n[4] = {n0, n0 / 4, n0 / 16, n0 / 64};
    CDM_CK(alloc(&X, n0 * 16));
    CDM_CK(alloc(&gY, n0 * 16));
    CDM_CK(alloc(&Y, n0 * 16));
    CDM_CK(alloc(&target, n0));
    CDM_CK(alloc(&weight, n0));
    CDM_CK(alloc(&sm0, n0));
    CDM_CK(alloc(&sm1, n0));
    CDM_CK(alloc(&A0, n[0] * c));
    CDM_CK(alloc(&S0, n[0] * c));
    CDM_CK(alloc(&U0, n[0] * c));
    CDM_CK(alloc(&D0, n[0] * c));
    CDM_CK(alloc(&P1, n[1] * c));
    CDM_CK(alloc(&S1, n[1] * c));
    CDM_CK(alloc(&U1, n[1] * c));
    CDM_CK(alloc(&D1, n[1] * c));
    CDM_CK(alloc(&P2, n[2] * c));
    CDM_CK(alloc(&S2, n[2] * c));
    CDM_CK(alloc(&U2, n[2] * c));
    CDM_CK(alloc(&D2, n[2] * c));
    CDM_CK(alloc(&P3, n[3] * c));
    CDM_CK(alloc(&B3, n[3] * c));
    for (int l = 0; l < 4; ++l) {
      CDM_CK(alloc(&ga[l], n[l] * c));
      CDM_CK(alloc(&gb[l], n[l] * c));
    }
    B = b;
    H = hh;
    W = ww;
    return CDM_OK;
  }

  cudaError_t refresh_weights() {
    if (!weights_dirty) return cudaSuccess;
    for (int l = 0; l < 9; ++l) {
      cudaError_t e = prep_weights(params + L[l].w_off, L[l].wf, L[l].wb, L[l].cin, L[l].cout, stream);
      if (e != cudaSuccess) return e;
    }
    weights_dirty = false;
    return cudaSuccess;
  }

  cudaError_t conv(int l, const __nv_bfloat16* x, __nv_bfloat16* out, int lev, bool relu, float* out_f32 = nullptr) {
    ConvArgs a{};
    a.x = x;
    a.w = L[l].wf;
    a.bias = params + L[l].b_off;
    a.out = out;
    a.out_f32 = out_f32;
    a.B = B;
    a.H = H >> lev;
    a.W = W >> lev;
    a.epi = relu ? EPI_RELU : EPI_NONE;
    return conv3x3(L[l].cin, L[l].cout, a, stream);
  }

  // gradient w.r.t. the layer input: convᵀ(g) (· [mask > 0])
  cudaError_t conv_bwd(int l, const __nv_bfloat16* g, __nv_bfloat16* out, int lev, const __nv_bfloat16* mask) {
    ConvArgs a{};
    a.x = g;
    a.w = L[l].wb;
    a.out = out;
    a.mask = mask;
    a.B = B;
    a.H = H >> lev;
    a.W = W >> lev;
    a.epi = mask ? EPI_MASK : EPI_NONE;
    return conv3x3(L[l].cout, L[l].cin, a, stream);
  }

  cudaError_t wgrad(int l, const __nv_bfloat16* x, const __nv_bfloat16* g, int lev) {
    WgradArgs a{};
    a.x = x;
    a.g = g;
    a.dw = grads + L[l].w_off;
    a.db = grads + L[l].b_off;
    a.B = B;
    a.H = H >> lev;
    a.W = W >> lev;
    return conv3x3_wgrad(L[l].cin, L[l].cout, a, stream);
  }

  // forward of the features in X; output in Y
  int forward() {
    CDM_CK(refresh_weights());
    CDM_CK(conv(0, X, A0, 0, true));
    CDM_CK(conv(1, A0, S0, 0, true));
    CDM_CK(pool2(S0, P1, B, H, W, stream));
    CDM_CK(conv(2, P1, S1, 1, true));
    CDM_CK(pool2(S1, P2, B, H >> 1, W >> 1, stream));
    CDM_CK(conv(3, P2, S2, 2, true));
    CDM_CK(pool2(S2, P3, B, H >> 2, W >> 2, stream));
    CDM_CK(conv(4, P3, B3, 3, true));
    CDM_CK(up_add(B3, S2, U2, B, H >> 2, W >> 2, stream));
    CDM_CK(conv(5, U2, D2, 2, true));
    CDM_CK(up_add(D2, S1, U1, B, H >> 1, W >> 1, stream));
    CDM_CK(conv(6, U1, D1, 1, true));
    CDM_CK(up_add(D1, S0, U0, B, H, W, stream));
    CDM_CK(conv(7, U0, D0, 0, true));
    CDM_CK(conv(8, D0, nullptr, 0, false, Y));
    return CDM_OK;
  }

  // loss of Y against target and the parameter gradient (zeroed first)
  int backward() {
    const int64_t npix = (int64_t)B * H * W;
    CDM_CK(cudaMemsetAsync(grads, 0, nparams * sizeof(float), stream));
    CDM_CK(cudaMemsetAsync(d_loss, 0, sizeof(float), stream));
    CDM_CK(loss_grad(Y, target, use_weight ? weight : nullptr, gY, npix, d_loss, stream));
    CDM_CK(wgrad(8, D0, gY, 0));
    CDM_CK(conv_bwd(8, gY, ga[0], 0, D0));                              // gD0
    CDM_CK(wgrad(7, U0, ga[0], 0));
    CDM_CK(conv_bwd(7, ga[0], gb[0], 0, nullptr));                      // gU0
    CDM_CK(up_bwd_mask(gb[0], D1, ga[1], B, H, W, stream));             // gD1
    CDM_CK(wgrad(6, U1, ga[1], 1));
    CDM_CK(conv_bwd(6, ga[1], gb[1], 1, nullptr));                      // gU1
    CDM_CK(up_bwd_mask(gb[1], D2, ga[2], B, H >> 1, W >> 1, stream));   // gD2
    CDM_CK(wgrad(5, U2, ga[2], 2));
    CDM_CK(conv_bwd(5, ga[2], gb[2], 2, nullptr));                      // gU2
    CDM_CK(up_bwd_mask(gb[2], B3, ga[3], B, H >> 2, W >> 2, stream));   // gB3
    CDM_CK(wgrad(4, P3, ga[3], 3));
    CDM_CK(conv_bwd(4, ga[3], gb[3], 3, nullptr));                      // gP3
    CDM_CK(pool_bwd_add_mask(gb[2], gb[3], S2, ga[2], B, H >> 2, W >> 2, stream));  // gS2
    CDM_CK(wgrad(3, P2, ga[2], 2));
    CDM_CK(conv_bwd(3, ga[2], gb[2], 2, nullptr));                      // gP2
    CDM_CK(pool_bwd_add_mask(gb[1], gb[2], S1, ga[1], B, H >> 1, W >> 1, stream));  // gS1
    CDM_CK(wgrad(2, P1, ga[1], 1));
    CDM_CK(conv_bwd(2, ga[1], gb[1], 1, nullptr));                      // gP1
    CDM_CK(pool_bwd_add_mask(gb[0], gb[1], S0, ga[0], B, H, W, stream));  // gS0
    CDM_CK(wgrad(1, A0, ga[0], 0));
    CDM_CK(conv_bwd(1, ga[0], gb[0], 0, A0));                           // gA0
    CDM_CK(wgrad(0, X, gb[0], 0));
    return CDM_OK;
  }

  int adam_step(float lr) {
    ++adam_t;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = (float)(1.0 / (1.0 - std::pow((double)b1, adam_t)));
    const float c2 = (float)(1.0 / (1.0 - std::pow((double)b2, adam_t)));
    CDM_CK(adam(params, grads, m, v, nparams, lr, b1, b2, 1e-8f, c1, c2, stream));
    weights_dirty = true;
    return CDM_OK;
  }

  int ensure_batch_scratch(int n) {
    if (n <= cap) return CDM_OK;
    cudaFree(d_scale);
    cudaFree(d_ptrs);
    cudaFree(d_orig);
    CDM_CK(cudaMalloc((void**)&d_scale, n * sizeof(double)));
    CDM_CK(cudaMalloc((void**)&d_ptrs, 3 * n * sizeof(double*)));
    CDM_CK(cudaMalloc((void**)&d_orig, 2 * n * sizeof(int)));
    cap = n;
    return CDM_OK;
  }

  // CDM_TIMEOUT when a bounded wait of the tensor-core convolution ran out
  int conv_status() {
    int flag = 0;
    CDM_CK(conv3x3_tc_error(&flag));
    if (flag) {
      set_error("guess network: a tensor-core convolution's wait ran out");
      return CDM_TIMEOUT;
    }
    return CDM_OK;
  }

  float read_loss() {
    float l = 0.f;
    if (cudaMemcpyAsync(&l, d_loss, sizeof(float), cudaMemcpyDeviceToHost, stream) != cudaSuccess) return NAN;
    if (cudaStreamSynchronize(stream) != cudaSuccess) return NAN;
    return l / (float)((int64_t)B * H * W);
  }
};

}  // namespace net
}  // namespace cdm

using cdm::net::Net;
struct cdm_net {
  Net n;
};

extern "C" {

int cdm_net_create(int device, uint64_t seed, void* stream, cdm_net** out) {
  if (!out) return CDM_BAD_INPUT;
  *out = nullptr;
  cdm_net* h = new cdm_net();
  int rc = h->n.init(device, seed, stream);
  if (rc != CDM_OK) {
    delete h;
    return rc;
  }
  *out = h;
  return CDM_OK;
}

int cdm_net_destroy(cdm_net* net) {
  if (!net) return CDM_BAD_INPUT;
  cudaSetDevice(net->n.device);
  cudaStreamSynchronize(net->n.stream);
  delete net;
  return CDM_OK;
}

int cdm_net_set_guess_smoothing(cdm_net* net, int passes) {
  if (!net || passes < 0 || passes > 1024) return CDM_BAD_INPUT;
  net->n.smooth_passes = passes;
  return CDM_OK;
}

int cdm_net_num_params(const cdm_net* net, int64_t* n) {
  if (!net || !n) return CDM_BAD_INPUT;
  *n = net->n.nparams;
  return CDM_OK;
}

int cdm_net_get_params(cdm_net* net, float* params) {
  if (!net || !params) return CDM_BAD_INPUT;
  Net& n = net->n;
  CDM_CK(cudaSetDevice(n.device));
  CDM_CK(cudaMemcpyAsync(params, n.params, n.nparams * sizeof(float), cudaMemcpyDeviceToHost, n.stream));
  CDM_CK(cudaStreamSynchronize(n.stream));
  return CDM_OK;
}

int cdm_net_set_params(cdm_net* net, const float* params) {
  if (!net || !params) return CDM_BAD_INPUT;
  Net& n = net->n;
  CDM_CK(cudaSetDevice(n.device));
  CDM_CK(cudaMemcpyAsync(n.params, params, n.nparams * sizeof(float), cudaMemcpyHostToDevice, n.stream));
  CDM_CK(cudaStreamSynchronize(n.stream));
  n.weights_dirty = true;
  return CDM_OK;
}

int cdm_net_get_grads(cdm_net* net, float* grads) {
  if (!net || !grads) return CDM_BAD_INPUT;
  Net& n = net->n;
  CDM_CK(cudaSetDevice(n.device));
  CDM_CK(cudaMemcpyAsync(grads, n.grads, n.nparams * sizeof(float), cudaMemcpyDeviceToHost, n.stream));
  CDM_CK(cudaStreamSynchronize(n.stream));
  return CDM_OK;
}

int cdm_net_forward(cdm_net* net, const uint16_t* x, int B, int H, int W, float* y) {
  if (!net || !x || !y) return CDM_BAD_INPUT;
  Net& n = net->n;
  CDM_CK(cudaSetDevice(n.device));
  int rc = n.ensure_shape(B, H, W);
  if (rc != CDM_OK) return rc;
  const size_t np = (size_t)B * H * W;
  CDM_CK(cudaMemcpyAsync(n.X, x, np * 16 * sizeof(uint16_t), cudaMemcpyDeviceToDevice, n.stream));
  rc = n.forward();
  if (rc != CDM_OK) return rc;
  CDM_CK(cudaMemcpyAsync(y, n.Y, np * 16 * sizeof(float), cudaMemcpyDeviceToDevice, n.stream));
  CDM_CK(cudaStreamSynchronize(n.stream));
  return n.conv_status();
}

int cdm_net_backward(cdm_net* net, const float* target, float* loss) {
  if (!net || !target || !loss) return CDM_BAD_INPUT;
  Net& n = net->n;
  if (n.B == 0) {
    cdm::set_error("cdm_net_backward needs a forward pass first");
    return CDM_BAD_INPUT;
  }
  CDM_CK(cudaSetDevice(n.device));
  const size_t np = (size_t)n.B * n.H * n.W;
  CDM_CK(cudaMemcpyAsync(n.target, target, np * sizeof(float), cudaMemcpyDeviceToDevice, n.stream));
  n.use_weight = false;
  int rc = n.backward();
  if (rc != CDM_OK) return rc;
  *loss = n.read_loss();
  return n.conv_status();
}

int cdm_net_train_step(cdm_net* net, const cdm_net_batch* bt, float lr, float* loss) {
  if (!net || !bt || !loss || bt->nsamp < 1 || !bt->tprev || !bt->tcur || !bt->tnext || !bt->J || !bt->ox ||
      !bt->oy)
    return CDM_BAD_INPUT;
  Net& n = net->n;
  const int ns = bt->nsamp;
  if (ns > 1024) {
    cdm::set_error("at most 1024 samples per training batch");
    return CDM_BAD_INPUT;
  }
  if (bt->crop > bt->ni || bt->crop > bt->nj) {
    cdm::set_error("crop larger than the domain");
    return CDM_BAD_INPUT;
  }
  for (int b = 0; b < ns; ++b)
    if (bt->ox[b] < 0 || bt->oy[b] < 0 || bt->ox[b] + bt->crop > bt->ni || bt->oy[b] + bt->crop > bt->nj) {
      cdm::set_error("crop origin outside the domain");
      return CDM_BAD_INPUT;
    }
  CDM_CK(cudaSetDevice(n.device));
  int rc = n.ensure_shape(ns, bt->crop, bt->crop);
  if (rc != CDM_OK) return rc;
  rc = n.ensure_batch_scratch(ns);
  if (rc != CDM_OK) return rc;
  std::vector<const double*> ptrs(3 * ns);
  std::vector<int> orig(2 * ns);
  for (int b = 0; b < ns; ++b) {
    ptrs[b] = bt->tprev[b];
    ptrs[ns + b] = bt->tcur[b];
    ptrs[2 * ns + b] = bt->tnext[b];
    orig[b] = bt->ox[b];
    orig[ns + b] = bt->oy[b];
  }
  CDM_CK(cudaMemcpyAsync(n.d_ptrs, ptrs.data(), 3 * ns * sizeof(double*), cudaMemcpyHostToDevice, n.stream));
  CDM_CK(cudaMemcpyAsync(n.d_orig, orig.data(), 2 * ns * sizeof(int), cudaMemcpyHostToDevice, n.stream));
  const int nx = bt->ni + 2 * bt->nhalo;
  CDM_CK(cdm::net::delta_scale(n.d_ptrs, n.d_ptrs + ns, ns, bt->ni, bt->nj, nx, bt->nhalo, n.d_scale, n.stream));
  CDM_CK(cdm::net::finish_scale(n.d_scale, ns, (int64_t)bt->ni * bt->nj, n.stream));
  cdm::net::FeatArgs fa{};
  fa.tprev = n.d_ptrs;
  fa.tcur = n.d_ptrs + ns;
  fa.tnext = n.d_ptrs + 2 * ns;
  fa.J = bt->J;
  fa.ox = n.d_orig;
  fa.oy = n.d_orig + ns;
  fa.scale = n.d_scale;
  fa.nx = nx;
  fa.nh = bt->nhalo;
  fa.B = ns;
  fa.H = bt->crop;
  fa.W = bt->crop;
  fa.k0 = bt->k0;
  fa.kn = bt->kn;
  fa.log_jmean = bt->log_jmean;
  fa.dt = bt->dt;
  fa.rho_cp = bt->rho_cp > 0.0 ? bt->rho_cp : 1.0;
  fa.x = n.X;
  fa.target = n.target;
  fa.weight = n.weight;
  CDM_CK(cdm::net::features(fa, n.stream));
  rc = n.forward();
  if (rc != CDM_OK) return rc;
  n.use_weight = bt->dt > 0.0;
  rc = n.backward();
  if (rc != CDM_OK) return rc;
  rc = n.adam_step(lr);
  if (rc != CDM_OK) return rc;
  *loss = n.read_loss();
  return n.conv_status();
}

int cdm_net_predict(cdm_net* net, const double* tprev, const double* tcur, const double* J, int ni, int nj,
                    int nhalo, double k0, double kn, double log_jmean, double* u0) {
  if (!net || !tprev || !tcur || !J || !u0 || nhalo < 1) return CDM_BAD_INPUT;
  Net& n = net->n;
  CDM_CK(cudaSetDevice(n.device));
  int rc = n.ensure_shape(1, nj, ni);
  if (rc != CDM_OK) return rc;
  rc = n.ensure_batch_scratch(1);
  if (rc != CDM_OK) return rc;
  const int nx = ni + 2 * nhalo, ny = nj + 2 * nhalo;
  const double* ptrs[3] = {tprev, tcur, tcur};
  const int orig[2] = {0, 0};
  CDM_CK(cudaMemcpyAsync(n.d_ptrs, ptrs, 3 * sizeof(double*), cudaMemcpyHostToDevice, n.stream));
  CDM_CK(cudaMemcpyAsync(n.d_orig, orig, 2 * sizeof(int), cudaMemcpyHostToDevice, n.stream));
  CDM_CK(cdm::net::delta_scale(n.d_ptrs, n.d_ptrs + 1, 1, ni, nj, nx, nhalo, n.d_scale, n.stream));
  CDM_CK(cdm::net::finish_scale(n.d_scale, 1, (int64_t)ni * nj, n.stream));
  cdm::net::FeatArgs fa{};
  fa.tprev = n.d_ptrs;
  fa.tcur = n.d_ptrs + 1;
  fa.tnext = nullptr;
  fa.J = J;
  fa.ox = n.d_orig;
  fa.oy = n.d_orig + 1;
  fa.scale = n.d_scale;
  fa.nx = nx;
  fa.nh = nhalo;
  fa.B = 1;
  fa.H = nj;
  fa.W = ni;
  fa.k0 = k0;
  fa.kn = kn;
  fa.log_jmean = log_jmean;
  fa.x = n.X;
  fa.target = nullptr;
  CDM_CK(cdm::net::features(fa, n.stream));
  rc = n.forward();
  if (rc != CDM_OK) return rc;
  // the correction over linear extrapolation, smoothed: grid-scale noise of the
  // bf16 activations would enter the step's residual amplified by the local
  // diffusion number
  const float* y = n.Y;
  int ystride = 16;
  for (int k = 0; k < n.smooth_passes; ++k) {
    float* dst = (k & 1) ? n.sm1 : n.sm0;
    CDM_CK(cdm::net::smooth3x3(y, ystride, dst, nj, ni, n.stream));
    y = dst;
    ystride = 1;
  }
  CDM_CK(cudaMemcpyAsync(u0, tcur, (size_t)nx * ny * sizeof(double), cudaMemcpyDeviceToDevice, n.stream));
  CDM_CK(cdm::net::apply_guess(tprev, tcur, y, ystride, n.d_scale, u0, ni, nj, nx, nhalo, n.stream));
  CDM_CK(cudaStreamSynchronize(n.stream));
  return n.conv_status();
}

}  // extern "C"
