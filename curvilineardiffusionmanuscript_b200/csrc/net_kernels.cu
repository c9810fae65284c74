// net_kernels.cu — tensor-core convolutions and helpers of the learned
// initial-guess network (bf16 storage, FP32 accumulation).
//
// Convolution tiling: a block computes a 32 x 8 tile of output pixels of one
// image.  The input tile with its one-pixel halo (34 x 10 pixels) and the
// layer's weights are staged in shared memory with rows padded by 8 bf16, so
// that the eight 16-byte rows one ldmatrix phase reads fall in distinct banks.
// Forward: warp w computes output row w (two m16 tiles of pixels) against all
// output channels; K runs over the 9 taps x CIN input channels in steps of 16.
// Weight gradients: warp w owns tap w (9 warps); K runs over the tile's 256
// pixels, and the block accumulates in registers over the tiles it visits
// before one atomic reduction into the FP32 gradient.
#include "net_kernels.cuh"

#include <cmath>
#include <cstdlib>
#include <cstring>

namespace cdm {
namespace net {

namespace {

constexpr int TXP = 32, TYP = 8;            // output tile (pixels)
constexpr int HX = TXP + 2, HY = TYP + 2;   // with halo

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void ldsm_x4(uint32_t* r, const void* p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(smem_u32(p)));
}

__device__ __forceinline__ void ldsm_x4_t(uint32_t* r, const void* p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(smem_u32(p)));
}

__device__ __forceinline__ void mma_bf16(float* d, const uint32_t* a, uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// stage the 34 x 10 input halo tile of image b at output origin (x0, y0)
template <int CIN, int NTHR>
__device__ __forceinline__ void load_halo(__nv_bfloat16* xs, const __nv_bfloat16* __restrict__ x, int b, int H, int W,
                                          int x0, int y0) {
  constexpr int XS = CIN + 8, VPP = CIN / 8;
  for (int v = threadIdx.x; v < HX * HY * VPP; v += NTHR) {
    const int pix = v / VPP, part = v - pix * VPP;
    const int hy = pix / HX, hx = pix - hy * HX;
    const int gy = y0 - 1 + hy, gx = x0 - 1 + hx;
    uint4 val = make_uint4(0u, 0u, 0u, 0u);
    if (gy >= 0 && gy < H && gx >= 0 && gx < W)
      val = *reinterpret_cast<const uint4*>(x + (((size_t)b * H + gy) * W + gx) * CIN + part * 8);
    *reinterpret_cast<uint4*>(xs + pix * XS + part * 8) = val;
  }
}

template <int CIN, int COUT>
__global__ void __launch_bounds__(256) conv3x3_kernel(ConvArgs a) {
  constexpr int XS = CIN + 8, NT = COUT / 8, KC = CIN / 16;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __nv_bfloat16* xs = reinterpret_cast<__nv_bfloat16*>(smem_raw);
  __nv_bfloat16* ws = xs + HX * HY * XS;
  const int tiles_x = (a.W + TXP - 1) / TXP;
  const int x0 = (blockIdx.x % tiles_x) * TXP, y0 = (blockIdx.x / tiles_x) * TYP, b = blockIdx.y;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  load_halo<CIN, 256>(xs, a.x, b, a.H, a.W, x0, y0);
  for (int v = tid; v < 9 * COUT * (CIN / 8); v += 256) {
    const int row = v / (CIN / 8), part = v - row * (CIN / 8);
    *reinterpret_cast<uint4*>(ws + row * XS + part * 8) =
        *reinterpret_cast<const uint4*>(a.w + (size_t)row * CIN + part * 8);
  }
  __syncthreads();
  float acc[2][NT][4];
#pragma unroll
  for (int m = 0; m < 2; ++m)
#pragma unroll
    for (int n = 0; n < NT; ++n)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[m][n][e] = 0.f;
  const int q = lane >> 3, r = lane & 7;
#pragma unroll
  for (int tap = 0; tap < 9; ++tap) {
    const int dy = tap / 3, dx = tap - 3 * (tap / 3);
#pragma unroll
    for (int kc = 0; kc < KC; ++kc) {
      uint32_t af[2][4];
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) {
        const int i = r + ((q & 1) ? 8 : 0);
        const int cio = 16 * kc + ((q & 2) ? 8 : 0);
        ldsm_x4(af[mt], xs + ((warp + dy) * HX + 16 * mt + i + dx) * XS + cio);
      }
#pragma unroll
      for (int np = 0; np < NT / 2; ++np) {
        uint32_t bf[4];
        const int co = 8 * (2 * np + (q >> 1)) + r;
        const int cio = 16 * kc + ((q & 1) ? 8 : 0);
        ldsm_x4(bf, ws + (tap * COUT + co) * XS + cio);
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
          mma_bf16(acc[mt][2 * np], af[mt], bf[0], bf[1]);
          mma_bf16(acc[mt][2 * np + 1], af[mt], bf[2], bf[3]);
        }
      }
    }
  }
  // epilogue: rows g and g+8 of each m16 tile, channel pair (2c, 2c+1) of each n8 tile
  const int g = lane >> 2, c = lane & 3, y = y0 + warp;
  if (y >= a.H) return;
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int xx = x0 + 16 * mt + g + 8 * h;
      if (xx >= a.W) continue;
      const size_t pix = ((size_t)b * a.H + y) * a.W + xx;
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) {
        const int co = 8 * nt + 2 * c;
        float v0 = acc[mt][nt][2 * h], v1 = acc[mt][nt][2 * h + 1];
        if (a.bias) {
          v0 += a.bias[co];
          v1 += a.bias[co + 1];
        }
        if (a.epi == EPI_RELU) {
          v0 = fmaxf(v0, 0.f);
          v1 = fmaxf(v1, 0.f);
        } else if (a.epi == EPI_MASK) {
          const __nv_bfloat162 mk = *reinterpret_cast<const __nv_bfloat162*>(a.mask + pix * COUT + co);
          if (!(__bfloat162float(mk.x) > 0.f)) v0 = 0.f;
          if (!(__bfloat162float(mk.y) > 0.f)) v1 = 0.f;
        }
        if (a.out) *reinterpret_cast<__nv_bfloat162*>(a.out + pix * COUT + co) = __floats2bfloat162_rn(v0, v1);
        if (a.out_f32) *reinterpret_cast<float2*>(a.out_f32 + pix * COUT + co) = make_float2(v0, v1);
      }
    }
}

template <int CIN, int COUT>
__global__ void __launch_bounds__(288) wgrad_kernel(WgradArgs a, int ntiles) {
  constexpr int XS = CIN + 8, GS = COUT + 8, NT = COUT / 8, MT = CIN / 16;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __nv_bfloat16* xs = reinterpret_cast<__nv_bfloat16*>(smem_raw);
  __nv_bfloat16* gs = xs + HX * HY * XS;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int dy = warp / 3, dx = warp - 3 * (warp / 3);  // this warp's tap
  const int q = lane >> 3, r = lane & 7;
  const int tiles_x = (a.W + TXP - 1) / TXP, tiles_y = (a.H + TYP - 1) / TYP;
  float acc[MT][NT][4];
#pragma unroll
  for (int m = 0; m < MT; ++m)
#pragma unroll
    for (int n = 0; n < NT; ++n)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[m][n][e] = 0.f;
  float dbacc = 0.f;
  const int dbco = tid % COUT, dbpart = tid / COUT;  // bias-gradient share (threads < 8·COUT)
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int b = t / (tiles_x * tiles_y), tt = t - b * tiles_x * tiles_y;
    const int x0 = (tt % tiles_x) * TXP, y0 = (tt / tiles_x) * TYP;
    __syncthreads();  // previous tile's readers are done
    load_halo<CIN, 288>(xs, a.x, b, a.H, a.W, x0, y0);
    for (int v = tid; v < TXP * TYP * (COUT / 8); v += 288) {
      const int pix = v / (COUT / 8), part = v - pix * (COUT / 8);
      const int yy = pix / TXP, xx = pix - yy * TXP;
      const int gy = y0 + yy, gx = x0 + xx;
      uint4 val = make_uint4(0u, 0u, 0u, 0u);
      if (gy < a.H && gx < a.W)
        val = *reinterpret_cast<const uint4*>(a.g + (((size_t)b * a.H + gy) * a.W + gx) * COUT + part * 8);
      *reinterpret_cast<uint4*>(gs + pix * GS + part * 8) = val;
    }
    __syncthreads();
    if (dbpart < 8)
      for (int p = dbpart; p < TXP * TYP; p += 8) dbacc += __bfloat162float(gs[p * GS + dbco]);
#pragma unroll 2
    for (int ks = 0; ks < TYP * 2; ++ks) {
      const int yy = ks >> 1, h = ks & 1;
      uint32_t af[MT][4];
#pragma unroll
      for (int mt = 0; mt < MT; ++mt) {
        const int i = r + ((q & 2) ? 8 : 0);
        const int cio = 16 * mt + ((q & 1) ? 8 : 0);
        ldsm_x4_t(af[mt], xs + ((yy + dy) * HX + 16 * h + i + dx) * XS + cio);
      }
#pragma unroll
      for (int np = 0; np < NT / 2; ++np) {
        uint32_t bf[4];
        const int i = r + ((q & 1) ? 8 : 0);
        const int co = 16 * np + ((q & 2) ? 8 : 0);
        ldsm_x4_t(bf, gs + (yy * TXP + 16 * h + i) * GS + co);
#pragma unroll
        for (int mt = 0; mt < MT; ++mt) {
          mma_bf16(acc[mt][2 * np], af[mt], bf[0], bf[1]);
          mma_bf16(acc[mt][2 * np + 1], af[mt], bf[2], bf[3]);
        }
      }
    }
  }
  const int g = lane >> 2, c = lane & 3;
#pragma unroll
  for (int mt = 0; mt < MT; ++mt)
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
      const int m0 = warp * CIN + 16 * mt + g, n0 = 8 * nt + 2 * c;
      atomicAdd(a.dw + (size_t)m0 * COUT + n0, acc[mt][nt][0]);
      atomicAdd(a.dw + (size_t)m0 * COUT + n0 + 1, acc[mt][nt][1]);
      atomicAdd(a.dw + (size_t)(m0 + 8) * COUT + n0, acc[mt][nt][2]);
      atomicAdd(a.dw + (size_t)(m0 + 8) * COUT + n0 + 1, acc[mt][nt][3]);
    }
  if (dbpart < 8 && a.db) atomicAdd(a.db + dbco, dbacc);
}

__device__ __forceinline__ void unpack8(const uint4& v, float* f) {
  const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&v);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const float2 t = __bfloat1622float2(h[k]);
    f[2 * k] = t.x;
    f[2 * k + 1] = t.y;
  }
}

__device__ __forceinline__ uint4 pack8(const float* f) {
  uint4 v;
  __nv_bfloat162* h = reinterpret_cast<__nv_bfloat162*>(&v);
#pragma unroll
  for (int k = 0; k < 4; ++k) h[k] = __floats2bfloat162_rn(f[2 * k], f[2 * k + 1]);
  return v;
}

constexpr int C = 32, V = C / 8;  // channels of the inner layers, 16-byte vectors per pixel

// out (H/2 x W/2) = mean of 2x2 blocks of in (H x W)
__global__ void pool2_kernel(const uint4* __restrict__ in, uint4* __restrict__ out, int B, int H, int W) {
  const int Ho = H / 2, Wo = W / 2;
  const int64_t n = (int64_t)B * Ho * Wo * V;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int v = (int)(e % V);
    const int64_t p = e / V;
    const int x = (int)(p % Wo);
    const int64_t r = p / Wo;
    const int y = (int)(r % Ho), b = (int)(r / Ho);
    float s[8] = {0, 0, 0, 0, 0, 0, 0, 0}, f[8];
#pragma unroll
    for (int dy = 0; dy < 2; ++dy)
#pragma unroll
      for (int dx = 0; dx < 2; ++dx) {
        unpack8(in[(((int64_t)b * H + 2 * y + dy) * W + 2 * x + dx) * V + v], f);
#pragma unroll
        for (int k = 0; k < 8; ++k) s[k] += f[k];
      }
#pragma unroll
    for (int k = 0; k < 8; ++k) s[k] *= 0.25f;
    out[e] = pack8(s);
  }
}

// out (H x W) = coarse[p/2] + skip[p]
__global__ void up_add_kernel(const uint4* __restrict__ coarse, const uint4* __restrict__ skip, uint4* __restrict__ out,
                              int B, int H, int W) {
  const int64_t n = (int64_t)B * H * W * V;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int v = (int)(e % V);
    const int64_t p = e / V;
    const int x = (int)(p % W);
    const int64_t r = p / W;
    const int y = (int)(r % H), b = (int)(r / H);
    float a[8], s[8];
    unpack8(coarse[(((int64_t)b * (H / 2) + y / 2) * (W / 2) + x / 2) * V + v], a);
    unpack8(skip[e], s);
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] += s[k];
    out[e] = pack8(a);
  }
}

// gcoarse (H/2 x W/2) = (Σ over the 2x2 block of gfine) · (mask > 0)
__global__ void up_bwd_mask_kernel(const uint4* __restrict__ gfine, const uint4* __restrict__ mask,
                                   uint4* __restrict__ gcoarse, int B, int H, int W) {
  const int Ho = H / 2, Wo = W / 2;
  const int64_t n = (int64_t)B * Ho * Wo * V;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int v = (int)(e % V);
    const int64_t p = e / V;
    const int x = (int)(p % Wo);
    const int64_t r = p / Wo;
    const int y = (int)(r % Ho), b = (int)(r / Ho);
    float s[8] = {0, 0, 0, 0, 0, 0, 0, 0}, f[8], m[8];
#pragma unroll
    for (int dy = 0; dy < 2; ++dy)
#pragma unroll
      for (int dx = 0; dx < 2; ++dx) {
        unpack8(gfine[(((int64_t)b * H + 2 * y + dy) * W + 2 * x + dx) * V + v], f);
#pragma unroll
        for (int k = 0; k < 8; ++k) s[k] += f[k];
      }
    unpack8(mask[e], m);
#pragma unroll
    for (int k = 0; k < 8; ++k) s[k] = m[k] > 0.f ? s[k] : 0.f;
    gcoarse[e] = pack8(s);
  }
}

// out (H x W) = (ga[p] + gp[p/2] / 4) · (mask[p] > 0); ga may be NULL
__global__ void pool_bwd_add_mask_kernel(const uint4* __restrict__ ga, const uint4* __restrict__ gp,
                                         const uint4* __restrict__ mask, uint4* __restrict__ out, int B, int H,
                                         int W) {
  const int64_t n = (int64_t)B * H * W * V;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int v = (int)(e % V);
    const int64_t p = e / V;
    const int x = (int)(p % W);
    const int64_t r = p / W;
    const int y = (int)(r % H), b = (int)(r / H);
    float s[8], f[8], m[8];
    unpack8(gp[(((int64_t)b * (H / 2) + y / 2) * (W / 2) + x / 2) * V + v], s);
#pragma unroll
    for (int k = 0; k < 8; ++k) s[k] *= 0.25f;
    if (ga) {
      unpack8(ga[e], f);
#pragma unroll
      for (int k = 0; k < 8; ++k) s[k] += f[k];
    }
    unpack8(mask[e], m);
#pragma unroll
    for (int k = 0; k < 8; ++k) s[k] = m[k] > 0.f ? s[k] : 0.f;
    out[e] = pack8(s);
  }
}

__device__ __forceinline__ double kappa_of(double T, double k0, double kn) {
  if (!isfinite(T)) return 0.0;
  return kn == 0.0 ? k0 : k0 * pow(fabs(T), kn);
}

// input features of crop pixel (x, y) of sample b: log|Tⁿ|, (Tⁿ − Tⁿ⁻¹)/s,
// log κ(Tⁿ)/4, log J − log J̄; channels 4..15 are zero.  Target: the departure
// from linear extrapolation, (Tⁿ⁺¹ − 2Tⁿ + Tⁿ⁻¹)/s, formed in FP64.
__global__ void features_kernel(FeatArgs a) {
  const int64_t n = (int64_t)a.B * a.H * a.W;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(e % a.W);
    const int64_t r = e / a.W;
    const int y = (int)(r % a.H), b = (int)(r / a.H);
    const int64_t o = (int64_t)(a.ox[b] + x + a.nh) + (int64_t)a.nx * (a.oy[b] + y + a.nh);
    const double tc = a.tcur[b][o], tp = a.tprev[b][o], s = a.scale[b];
    const double is = 1.0 / s;
    float f[16];
#pragma unroll
    for (int k = 4; k < 16; ++k) f[k] = 0.f;
    f[0] = (float)log(fmax(fabs(tc), 1e-30));
    f[1] = (float)((tc - tp) * is);
    f[2] = (float)(0.25 * log(fmax(kappa_of(tc, a.k0, a.kn), 1e-30)));
    f[3] = (float)(log(fmax(a.J[o], 1e-300)) - a.log_jmean);
    uint4* dst = reinterpret_cast<uint4*>(a.x + e * 16);
    dst[0] = pack8(f);
    dst[1] = pack8(f + 8);
    if (a.target) a.target[e] = (float)(((a.tnext[b][o] - tc) - (tc - tp)) * is);
    // A smooth error of the guess enters the step's residual amplified by about
    // 1 + D(h/ℓ)² with D = κΔt/(ρcₚJ) the local diffusion number and ℓ its
    // length scale; the loss weights each pixel by that factor at ℓ = 4 cells.
    if (a.weight)
      a.weight[e] = a.dt > 0.0 ? (float)(1.0 + kappa_of(tc, a.k0, a.kn) * a.dt / (a.rho_cp * a.J[o]) / 16.0)
                               : 1.0f;
  }
}

// Σ (Tⁿ − Tⁿ⁻¹)² over the domain of each sample (blockIdx.y)
__global__ void delta_scale_kernel(const double* const* tprev, const double* const* tcur, int ni, int nj, int nx,
                                   int nh, double* acc) {
  const int b = blockIdx.y;
  const int64_t n = (int64_t)ni * nj;
  double s = 0.0;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % ni), j = (int)(e / ni);
    const int64_t o = (int64_t)(i + nh) + (int64_t)nx * (j + nh);
    const double d = tcur[b][o] - tprev[b][o];
    s += d * d;
  }
#pragma unroll
  for (int k = 16; k > 0; k >>= 1) s += __shfl_xor_sync(0xffffffffu, s, k);
  __shared__ double red[8];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    atomicAdd(acc + b, t);
  }
}

__global__ void finish_scale_kernel(double* acc, int nsamp, int64_t ncells) {
  const int b = threadIdx.x;
  if (b < nsamp) {
    const double s = sqrt(acc[b] / (double)ncells);
    acc[b] = (s > 0.0 && isfinite(s)) ? s : 1.0;
  }
}

// (weighted) squared error of channel 0, w²(y − t)², and its gradient
// 2w²(y − t)/N (channels 1..15 zero); w = 1 without weights
__global__ void loss_grad_kernel(const float* __restrict__ y, const float* __restrict__ t,
                                 const float* __restrict__ w, __nv_bfloat16* __restrict__ gy, int64_t npix,
                                 float* loss_acc) {
  float l = 0.f;
  const float sc = 2.f / (float)npix;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < npix; p += (int64_t)gridDim.x * blockDim.x) {
    const float ww = w ? w[p] * w[p] : 1.f;
    const float d = y[p * 16] - t[p];
    l += ww * d * d;
    float f[16];
#pragma unroll
    for (int k = 1; k < 16; ++k) f[k] = 0.f;
    f[0] = sc * ww * d;
    uint4* dst = reinterpret_cast<uint4*>(gy + p * 16);
    dst[0] = pack8(f);
    dst[1] = pack8(f + 8);
  }
#pragma unroll
  for (int k = 16; k > 0; k >>= 1) l += __shfl_xor_sync(0xffffffffu, l, k);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss_acc, l);
}

// out = ((1 2 1)ᵀ(1 2 1) / 16) * in on an H x W image, edge pixels replicated
__global__ void smooth3x3_kernel(const float* __restrict__ in, int in_stride, float* __restrict__ out, int H,
                                 int W) {
  const int64_t n = (int64_t)H * W;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(e % W), y = (int)(e / W);
    float s = 0.f;
#pragma unroll
    for (int dy = -1; dy <= 1; ++dy) {
      const int yy = min(max(y + dy, 0), H - 1);
#pragma unroll
      for (int dx = -1; dx <= 1; ++dx) {
        const int xx = min(max(x + dx, 0), W - 1);
        s += (float)((2 - (dx < 0 ? -dx : dx)) * (2 - (dy < 0 ? -dy : dy))) * in[((int64_t)yy * W + xx) * in_stride];
      }
    }
    out[e] = s * (1.f / 16.f);
  }
}

// u0 = 2Tⁿ − Tⁿ⁻¹ + s·y on the domain (y: one image of ni x nj pixels, y_stride floats apart)
__global__ void apply_guess_kernel(const double* __restrict__ tprev, const double* __restrict__ tcur,
                                   const float* __restrict__ y, int y_stride, const double* __restrict__ scale,
                                   double* __restrict__ u0, int ni, int nj, int nx, int nh) {
  const int64_t n = (int64_t)ni * nj;
  const double s = scale[0];
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % ni), j = (int)(e / ni);
    const int64_t o = (int64_t)(i + nh) + (int64_t)nx * (j + nh);
    u0[o] = (2.0 * tcur[o] - tprev[o]) + s * (double)y[e * y_stride];
  }
}

__global__ void prep_weights_kernel(const float* __restrict__ w, __nv_bfloat16* __restrict__ wf,
                                    __nv_bfloat16* __restrict__ wb, int cin, int cout) {
  const int n = 9 * cin * cout;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const int co = e % cout, ci = (e / cout) % cin, t = e / (cout * cin);
    const __nv_bfloat16 v = __float2bfloat16_rn(w[e]);
    wf[((size_t)t * cout + co) * cin + ci] = v;
    wb[((size_t)(8 - t) * cin + ci) * cout + co] = v;
  }
}

__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, int64_t n, float lr, float b1, float b2, float eps, float c1,
                            float c2) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const float gg = g[e];
    const float mm = b1 * m[e] + (1.f - b1) * gg;
    const float vv = b2 * v[e] + (1.f - b2) * gg * gg;
    m[e] = mm;
    v[e] = vv;
    p[e] -= lr * (mm * c1) / (sqrtf(vv * c2) + eps);
  }
}

int grid_for(int64_t n, int per = 256) {
  const int64_t g = (n + per - 1) / per;
  return (int)(g < 148 * 16 ? (g > 0 ? g : 1) : 148 * 16);
}

template <int CIN, int COUT>
cudaError_t launch_conv(const ConvArgs& a, cudaStream_t s) {
  constexpr int smem = (HX * HY * (CIN + 8) + 9 * COUT * (CIN + 8)) * 2;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(conv3x3_kernel<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  const int tiles = ((a.W + TXP - 1) / TXP) * ((a.H + TYP - 1) / TYP);
  conv3x3_kernel<CIN, COUT><<<dim3(tiles, a.B), 256, smem, s>>>(a);
  return cudaGetLastError();
}

template <int CIN, int COUT>
cudaError_t launch_wgrad(const WgradArgs& a, cudaStream_t s) {
  constexpr int smem = (HX * HY * (CIN + 8) + TXP * TYP * (COUT + 8)) * 2;
  static bool attr = false;
  static int grid_max = 0;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(wgrad_kernel<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    int per_sm = 1, dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, wgrad_kernel<CIN, COUT>, 288, smem);
    grid_max = nsm * (per_sm > 0 ? per_sm : 1);
    attr = true;
  }
  const int ntiles = a.B * ((a.W + TXP - 1) / TXP) * ((a.H + TYP - 1) / TYP);
  const int grid = ntiles < grid_max ? ntiles : grid_max;
  wgrad_kernel<CIN, COUT><<<grid, 288, smem, s>>>(a, ntiles);
  return cudaGetLastError();
}

}  // namespace

cudaError_t conv3x3(int cin, int cout, const ConvArgs& a, cudaStream_t s) {
  const char* path = std::getenv("CDM_NET_CONV");
  const bool mma_only = path && std::strcmp(path, "mma") == 0;
  if (!mma_only && conv3x3_tc_supported(cin, cout, a.W)) return conv3x3_tc(cin, cout, a, s);
  if (cin == 16 && cout == 32) return launch_conv<16, 32>(a, s);
  if (cin == 32 && cout == 32) return launch_conv<32, 32>(a, s);
  if (cin == 32 && cout == 16) return launch_conv<32, 16>(a, s);
  return cudaErrorInvalidValue;
}

cudaError_t conv3x3_wgrad(int cin, int cout, const WgradArgs& a, cudaStream_t s) {
  if (cin == 16 && cout == 32) return launch_wgrad<16, 32>(a, s);
  if (cin == 32 && cout == 32) return launch_wgrad<32, 32>(a, s);
  if (cin == 32 && cout == 16) return launch_wgrad<32, 16>(a, s);
  return cudaErrorInvalidValue;
}

cudaError_t pool2(const __nv_bfloat16* in, __nv_bfloat16* out, int B, int H, int W, cudaStream_t s) {
  pool2_kernel<<<grid_for((int64_t)B * (H / 2) * (W / 2) * V), 256, 0, s>>>(
      reinterpret_cast<const uint4*>(in), reinterpret_cast<uint4*>(out), B, H, W);
  return cudaGetLastError();
}

cudaError_t up_add(const __nv_bfloat16* coarse, const __nv_bfloat16* skip, __nv_bfloat16* out, int B, int H, int W,
                   cudaStream_t s) {
  up_add_kernel<<<grid_for((int64_t)B * H * W * V), 256, 0, s>>>(reinterpret_cast<const uint4*>(coarse),
                                                                 reinterpret_cast<const uint4*>(skip),
                                                                 reinterpret_cast<uint4*>(out), B, H, W);
  return cudaGetLastError();
}

cudaError_t up_bwd_mask(const __nv_bfloat16* gfine, const __nv_bfloat16* mask, __nv_bfloat16* gcoarse, int B, int H,
                        int W, cudaStream_t s) {
  up_bwd_mask_kernel<<<grid_for((int64_t)B * (H / 2) * (W / 2) * V), 256, 0, s>>>(
      reinterpret_cast<const uint4*>(gfine), reinterpret_cast<const uint4*>(mask),
      reinterpret_cast<uint4*>(gcoarse), B, H, W);
  return cudaGetLastError();
}

cudaError_t pool_bwd_add_mask(const __nv_bfloat16* ga, const __nv_bfloat16* gp, const __nv_bfloat16* mask,
                              __nv_bfloat16* out, int B, int H, int W, cudaStream_t s) {
  pool_bwd_add_mask_kernel<<<grid_for((int64_t)B * H * W * V), 256, 0, s>>>(
      reinterpret_cast<const uint4*>(ga), reinterpret_cast<const uint4*>(gp), reinterpret_cast<const uint4*>(mask),
      reinterpret_cast<uint4*>(out), B, H, W);
  return cudaGetLastError();
}

cudaError_t features(const FeatArgs& a, cudaStream_t s) {
  features_kernel<<<grid_for((int64_t)a.B * a.H * a.W), 256, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t delta_scale(const double* const* tprev, const double* const* tcur, int nsamp, int ni, int nj, int nx,
                        int nh, double* acc, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(acc, 0, sizeof(double) * nsamp, s);
  if (e != cudaSuccess) return e;
  const int gx = grid_for((int64_t)ni * nj) / 4 + 1;
  delta_scale_kernel<<<dim3(gx, nsamp), 256, 0, s>>>(tprev, tcur, ni, nj, nx, nh, acc);
  return cudaGetLastError();
}

cudaError_t finish_scale(double* acc, int nsamp, int64_t ncells, cudaStream_t s) {
  finish_scale_kernel<<<1, 1024, 0, s>>>(acc, nsamp, ncells);
  return cudaGetLastError();
}

cudaError_t loss_grad(const float* y, const float* target, const float* weight, __nv_bfloat16* gy, int64_t npix,
                      float* loss_acc, cudaStream_t s) {
  loss_grad_kernel<<<grid_for(npix), 256, 0, s>>>(y, target, weight, gy, npix, loss_acc);
  return cudaGetLastError();
}

cudaError_t smooth3x3(const float* in, int in_stride, float* out, int H, int W, cudaStream_t s) {
  smooth3x3_kernel<<<grid_for((int64_t)H * W), 256, 0, s>>>(in, in_stride, out, H, W);
  return cudaGetLastError();
}

cudaError_t apply_guess(const double* tprev, const double* tcur, const float* y, int y_stride, const double* scale,
                        double* u0, int ni, int nj, int nx, int nh, cudaStream_t s) {
  apply_guess_kernel<<<grid_for((int64_t)ni * nj), 256, 0, s>>>(tprev, tcur, y, y_stride, scale, u0, ni, nj, nx,
                                                                 nh);
  return cudaGetLastError();
}

cudaError_t prep_weights(const float* w, __nv_bfloat16* wf, __nv_bfloat16* wb, int cin, int cout, cudaStream_t s) {
  prep_weights_kernel<<<grid_for(9 * cin * cout), 256, 0, s>>>(w, wf, wb, cin, cout);
  return cudaGetLastError();
}

cudaError_t adam(float* p, const float* g, float* m, float* v, int64_t n, float lr, float b1, float b2, float eps,
                 float c1, float c2, cudaStream_t s) {
  adam_kernel<<<grid_for(n), 256, 0, s>>>(p, g, m, v, n, lr, b1, b2, eps, c1, c2);
  return cudaGetLastError();
}

}  // namespace net
}  // namespace cdm
