// apt_aux.cu — once-per-step and once-per-mesh kernels of the APT path.
#include <algorithm>

#include "cdm_device.cuh"
#include "cdm_fast.cuh"
#include "cdm_kernels.h"
#include "cdm_tz.cuh"

namespace cdm {

namespace {

__device__ __forceinline__ void domain_coords(const Problem& P, int64_t e, int& a, int& b, int& c) {
  a = (int)(e % P.ni);
  const int64_t r = e / P.ni;
  b = (int)(r % P.nj);
  c = (int)(r / P.nj);
}

// mesh_metric_cache.jl:39-250: for each cache entry b (xi, eta, zeta), sum
// over face family f and component comp, in the reference's order, of
// metric[f][comp] * (hat_b.comp / J |_{f+1/2} - hat_b.comp / J |_{f-1/2})
__global__ void metric_cache_kernel(Problem P, MeshPtrs m, double* c0, double* c1, double* c2) {
  const int64_t n = (int64_t)P.ni * P.nj * (P.ndim == 3 ? P.nk : 1);
  const int nd = P.ndim;
  double* out[3] = {c0, c1, c2};
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    int a, b, c;
    domain_coords(P, e, a, b, c);
    const int64_t id = fidx(P, a, b, c);
    const int64_t im[3] = {fidx(P, a - 1, b, c), fidx(P, a, b - 1, c), nd == 3 ? fidx(P, a, b, c - 1) : 0};
    for (int bb = 0; bb < nd; ++bb) {
      double acc = 0.0;
      bool first = true;
      for (int f = 0; f < nd; ++f) {
        const double Jp = m.edgeJ[f][id];
        const double Jm = m.edgeJ[f][im[f]];
        for (int comp = 0; comp < nd; ++comp) {
          const double metric = m.inv[3 * f + comp][id];
          const double plus = m.edgehat[f][3 * bb + comp][id] / Jp;
          const double minus = m.edgehat[f][3 * bb + comp][im[f]] / Jm;
          const double term = metric * (plus - minus);
          acc = first ? term : acc + term;
          first = false;
        }
      }
      out[bb][id] = acc;
    }
  }
}

// Packed coefficients of flux_divergence.jl, each the exact subexpression the
// reference evaluates (so the FP64 result is unchanged):
//   2D: (ξx²+ξy²), (ηx²+ηy²), 0.25(ηxξx+ηyξy), α, β            (:21-37)
//   3D: |∇ξ|², |∇η|², |∇ζ|², 0.5(∇η·∇ξ), 0.5(∇ζ·∇η), 0.5(∇ζ·∇ξ), α, β, γ (:145-219)
__global__ void coefficient_kernel(Problem P, MeshPtrs m, double* ca0, double* ca1, double* ca2, double* k0,
                                   double* k1, double* k2, double* k3, double* k4, double* k5, double* k6,
                                   double* k7, double* k8) {
  const int64_t n = (int64_t)P.ni * P.nj * (P.ndim == 3 ? P.nk : 1);
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    int a, b, c;
    domain_coords(P, e, a, b, c);
    const int64_t id = fidx(P, a, b, c);
    if (P.ndim == 2) {
      const double xx = m.inv[0][id], xy = m.inv[1][id], ex = m.inv[3][id], ey = m.inv[4][id];
      k0[id] = xx * xx + xy * xy;
      k1[id] = ex * ex + ey * ey;
      k2[id] = 0.25 * (ex * xx + ey * xy);
      k3[id] = ca0[id];
      k4[id] = ca1[id];
    } else {
      const double xx = m.inv[0][id], xy = m.inv[1][id], xz = m.inv[2][id];
      const double ex = m.inv[3][id], ey = m.inv[4][id], ez = m.inv[5][id];
      const double zx = m.inv[6][id], zy = m.inv[7][id], zz = m.inv[8][id];
      k0[id] = xx * xx + xy * xy + xz * xz;
      k1[id] = ex * ex + ey * ey + ez * ez;
      k2[id] = zx * zx + zy * zy + zz * zz;
      k3[id] = 0.5 * (ex * xx + ey * xy + ez * xz);
      k4[id] = 0.5 * (zx * ex + zy * ey + zz * ez);
      k5[id] = 0.5 * (zx * xx + zy * xy + zz * xz);
      k6[id] = ca0[id];
      k7[id] = ca1[id];
      k8[id] = ca2[id];
    }
  }
}

// twilight_zone.jl:69-183: the α-independent forcing terms of every domain
// cell for this step (tz::terms), written as kNumTerms full-size arrays
__global__ void tz_terms_kernel(Problem P, TzMesh m, const double* __restrict__ rho, double cp, double t, int no_t,
                                double* __restrict__ out) {
  const int64_t n = (int64_t)P.ni * P.nj;
  const int64_t st = (int64_t)P.nx * P.ny;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t I = e % P.ni + P.nh, J = e / P.ni + P.nh;
    const int64_t id = I + (int64_t)P.nx * J;
    const tz::Terms T = tz::terms(m.x[id], m.y[id], m.xxi[id], m.xeta[id], m.yxi[id], m.yeta[id], rho[id], cp, t,
                                  no_t, I, J, m.nnx, m.nny);
    out[id] = T.ut;
    out[id + st] = T.p1;
    out[id + 2 * st] = T.uxx;
    out[id + 3 * st] = T.p2;
    out[id + 4 * st] = T.uee;
    out[id + 5 * st] = T.uxe;
    out[id + 6 * st] = T.p3;
    out[id + 7 * st] = T.p4;
    out[id + 8 * st] = T.ux;
    out[id + 9 * st] = T.ue;
  }
}

// validity_checks.jl:1-43 over the domain and the first halo layer (corners excluded)
__global__ void validate_kernel(Problem P, const double* __restrict__ f, int* flag) {
  const int nd = P.ndim;
  const int64_t ex = P.ni + 2, ey = P.nj + 2, ez = nd == 3 ? P.nk + 2 : 1;
  const int64_t n = ex * ey * ez;
  int bits = 0;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int a = (int)(e % ex) - 1;
    const int64_t r = e / ex;
    const int b = (int)(r % ey) - 1;
    const int c = nd == 3 ? (int)(r / ey) - 1 : 0;
    const int out = (a < 0 || a >= P.ni) + (b < 0 || b >= P.nj) + (nd == 3 ? (c < 0 || c >= P.nk) : 0);
    if (out > 1) continue;
    const double v = f[fidx(P, a, b, c)];
    if (!isfinite(v)) bits |= 1;
    if (v < 0.0) bits |= 2;
  }
  if (bits) atomicOr(flag, bits);
}

// 2D Dirichlet: u[begin:(ilo-1), jlo:jhi] .= val (boundary_operators.jl:143-150),
// layers beyond the first (the sweep writes the first one every iteration)
__global__ void dirichlet_fill_kernel(Problem P, double* u) {
  const int nh = P.nh;
  for (int side = 0; side < 4; ++side) {
    if (P.rule[side] != GR_DIRICHLET) continue;
    const double v = P.val[side];
    const int len = side < 2 ? P.nj : P.ni;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < len * (nh - 1); t += gridDim.x * blockDim.x) {
      const int s = t % len, layer = 2 + t / len;  // layer 2..nh
      int a, b;
      if (side == 0) { a = -layer; b = s; }
      else if (side == 1) { a = P.ni - 1 + layer; b = s; }
      else if (side == 2) { a = s; b = -layer; }
      else { a = s; b = P.nj - 1 + layer; }
      u[fidx(P, a, b)] = v;
    }
  }
}

// PseudoTransientSolver.jl:323-331 and cutoff! (:366-368)
__global__ void clamp_kernel(double* u, int64_t n, int positivity, int cutoff) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    double a = u[e];
    if (positivity) a = fabs(a);
    if (cutoff) a = isfinite(a) ? 0.5 * (fabs(a) + a) : 0.0;
    u[e] = a;
  }
}

constexpr int kRedBlocks = 592;  // 4 x 148 SMs
constexpr int kRedThreads = 256;

// pass 1: max(u_prev) with NaN propagation, energy sums and source integral;
// block `blk` of `nblk` writes its 4 partials to dst
__device__ __forceinline__ void pass1_body(const Problem& P, const double* __restrict__ u,
                                           const double* __restrict__ J, int blk, int nblk, double* dst) {
  const int64_t nfull = (int64_t)P.nx * P.ny * P.nz;
  double mx = -INFINITY;
  bool nan = false;
  for (int64_t e = blk * (int64_t)blockDim.x + threadIdx.x; e < nfull; e += (int64_t)nblk * blockDim.x) {
    const double v = P.u_prev[e];
    if (v != v) nan = true;
    else mx = fmax(mx, v);
  }
  const int64_t n = (int64_t)P.ni * P.nj * (P.ndim == 3 ? P.nk : 1);
  double e0 = 0.0, e1 = 0.0, sj = 0.0;
  for (int64_t e = blk * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)nblk * blockDim.x) {
    int a, b, c;
    domain_coords(P, e, a, b, c);
    const int64_t id = fidx(P, a, b, c);
    const double w = P.rho[id] * P.cp;
    e0 += w * P.u_prev[id] * J[id];
    e1 += w * u[id] * J[id];
    sj += P.S[id] * J[id];
  }
  __shared__ double sm[4][kRedThreads / 32];
  const int anynan = __syncthreads_or(nan);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    e0 += __shfl_xor_sync(0xffffffffu, e0, o);
    e1 += __shfl_xor_sync(0xffffffffu, e1, o);
    sj += __shfl_xor_sync(0xffffffffu, sj, o);
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) { sm[0][w] = mx; sm[1][w] = e0; sm[2][w] = e1; sm[3][w] = sj; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < kRedThreads / 32; ++k) {
      mx = fmax(mx, sm[0][k]);
    }
    double a0 = sm[1][0], a1 = sm[2][0], a2 = sm[3][0];
    for (int k = 1; k < kRedThreads / 32; ++k) { a0 += sm[1][k]; a1 += sm[2][k]; a2 += sm[3][k]; }
    if (anynan) mx = __longlong_as_double(0x7ff8000000000000ll);
    dst[0] = mx;
    dst[1] = a0;
    dst[2] = a1;
    dst[3] = a2;
  }
}

__global__ void reduce_pass1(Problem P, const double* __restrict__ u, const double* __restrict__ J,
                             double* scratch) {
  pass1_body(P, u, J, blockIdx.x, gridDim.x, scratch + 4 * blockIdx.x);
}

// finish pass 1 in one thread (fixed order), then pass 2 needs umax
__device__ __forceinline__ void finish1_body(const double* scratch, int nb, double* out) {
  double mx = -INFINITY, a0 = 0, a1 = 0, a2 = 0;
  bool nan = false;
  for (int k = 0; k < nb; ++k) {
    const double v = scratch[4 * k];
    if (v != v) nan = true;
    else mx = fmax(mx, v);
    a0 += scratch[4 * k + 1];
    a1 += scratch[4 * k + 2];
    a2 += scratch[4 * k + 3];
  }
  out[0] = nan ? __longlong_as_double(0x7ff8000000000000ll) : mx;
  out[2] = a0;
  out[3] = a1;
  out[4] = a2;
}

__global__ void reduce_finish1(const double* scratch, int nb, double* out) {
  if (threadIdx.x != 0) return;
  finish1_body(scratch, nb, out);
}

// pass 2: max over the full arrays of |a-b|/(a+u0) masked by isfinite
// (timestep_control.jl:67-73)
__device__ __forceinline__ void pass2_body(const Problem& P, const double* __restrict__ u, double tol,
                                           const double* out, int blk, int nblk, double* dst) {
  const int64_t nfull = (int64_t)P.nx * P.ny * P.nz;
  const double u0 = out[0] * tol;
  double mx = -INFINITY;
  for (int64_t e = blk * (int64_t)blockDim.x + threadIdx.x; e < nfull; e += (int64_t)nblk * blockDim.x) {
    const double a = u[e], b = P.u_prev[e];
    double d = fabs(a - b) / (a + u0);
    d = isfinite(d) ? d : 0.0;
    mx = fmax(mx, d);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  __shared__ double sm[kRedThreads / 32];
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < kRedThreads / 32; ++k) mx = fmax(mx, sm[k]);
    *dst = mx;
  }
}

__global__ void reduce_pass2(Problem P, const double* __restrict__ u, double tol, const double* out,
                             double* scratch) {
  pass2_body(P, u, tol, out, blockIdx.x, gridDim.x, scratch + blockIdx.x);
}

__global__ void reduce_finish2(const double* scratch, int nb, double* out) {
  if (threadIdx.x != 0) return;
  double mx = -INFINITY;
  for (int k = 0; k < nb; ++k) mx = fmax(mx, scratch[k]);
  out[1] = mx;
}

// Batched form: one launch per pass for every problem of a batch.  Job j owns
// blocks [b0, b0 + nb) of the grid (found by binary search over b0) and its
// partials at scratch[4·b0 ...]; its results go to out[8·p ...].
template <class Job>
__device__ __forceinline__ int job_of_block(const Job* jobs, int njobs) {
  int lo = 0, hi = njobs - 1;
  const int b = blockIdx.x;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (jobs[mid].b0 <= b) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__global__ void breduce_pass1(const Problem* __restrict__ probs, const RedJob* __restrict__ jobs, int njobs,
                              double* scratch) {
  const RedJob jb = jobs[job_of_block(jobs, njobs)];
  const int blk = blockIdx.x - jb.b0;
  pass1_body(probs[jb.p], jb.u, jb.J, blk, jb.nb, scratch + 4 * (jb.b0 + blk));
}

__global__ void breduce_finish1(const RedJob* __restrict__ jobs, const double* scratch, double* out) {
  if (threadIdx.x != 0) return;
  const RedJob jb = jobs[blockIdx.x];
  finish1_body(scratch + 4 * jb.b0, jb.nb, out + 8 * jb.p);
}

__global__ void breduce_pass2(const Problem* __restrict__ probs, const RedJob* __restrict__ jobs, int njobs,
                              double tol, const double* out, double* scratch) {
  const RedJob jb = jobs[job_of_block(jobs, njobs)];
  const int blk = blockIdx.x - jb.b0;
  pass2_body(probs[jb.p], jb.u, tol, out + 8 * jb.p, blk, jb.nb, scratch + jb.b0 + blk);
}

__global__ void breduce_finish2(const RedJob* __restrict__ jobs, const double* scratch, double* out) {
  if (threadIdx.x != 0) return;
  const RedJob jb = jobs[blockIdx.x];
  double mx = -INFINITY;
  for (int k = 0; k < jb.nb; ++k) mx = fmax(mx, scratch[jb.b0 + k]);
  out[8 * jb.p + 1] = mx;
}

int grid_for(int64_t n, int threads) {
  int64_t b = (n + threads - 1) / threads;
  if (b > 148 * 16) b = 148 * 16;
  if (b < 1) b = 1;
  return (int)b;
}

}  // namespace

cudaError_t launch_metric_cache(const Problem& P, const MeshPtrs& m, double* cache[3], cudaStream_t s) {
  const int64_t n = (int64_t)P.ni * P.nj * (P.ndim == 3 ? P.nk : 1);
  metric_cache_kernel<<<grid_for(n, 256), 256, 0, s>>>(P, m, cache[0], cache[1], cache[2]);
  return cudaGetLastError();
}

cudaError_t launch_coefficients(const Problem& P, const MeshPtrs& m, double* const cache[3], double* coef[9],
                                cudaStream_t s) {
  const int64_t n = (int64_t)P.ni * P.nj * (P.ndim == 3 ? P.nk : 1);
  coefficient_kernel<<<grid_for(n, 256), 256, 0, s>>>(P, m, cache[0], cache[1], cache[2], coef[0], coef[1],
                                                       coef[2], coef[3], coef[4], coef[5], coef[6], coef[7],
                                                       coef[8]);
  return cudaGetLastError();
}

cudaError_t launch_tz_terms(const Problem& P, const TzMesh& m, const double* rho, double cp, double t, int no_t,
                            double* out, cudaStream_t s) {
  if (P.ndim != 2) return cudaErrorInvalidValue;
  const int64_t n = (int64_t)P.ni * P.nj;
  tz_terms_kernel<<<grid_for(n, 256), 256, 0, s>>>(P, m, rho, cp, t, no_t, out);
  return cudaGetLastError();
}

cudaError_t launch_validate(const Problem& P, const double* f, int* flag, cudaStream_t s) {
  const int64_t n = (int64_t)(P.ni + 2) * (P.nj + 2) * (P.ndim == 3 ? P.nk + 2 : 1);
  validate_kernel<<<grid_for(n, 256), 256, 0, s>>>(P, f, flag);
  return cudaGetLastError();
}

cudaError_t launch_dirichlet_fill(const Problem& P, double* u, cudaStream_t s) {
  if (P.ndim != 2 || P.nh < 2) return cudaSuccess;
  dirichlet_fill_kernel<<<64, 256, 0, s>>>(P, u);
  return cudaGetLastError();
}

cudaError_t launch_clamp(double* u, int64_t n, int positivity, int cutoff, cudaStream_t s) {
  if (!positivity && !cutoff) return cudaSuccess;
  clamp_kernel<<<grid_for(n, 256), 256, 0, s>>>(u, n, positivity, cutoff);
  return cudaGetLastError();
}

// extrapolated start: out = 2a - b (a = Tⁿ, b = Tⁿ⁻¹) over the full array
__global__ void extrapolate_kernel(double* __restrict__ out, const double* __restrict__ a,
                                   const double* __restrict__ b, int64_t n) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
    out[e] = 2.0 * a[e] - b[e];
}

cudaError_t launch_extrapolate(double* out, const double* a, const double* b, int64_t n, cudaStream_t s) {
  extrapolate_kernel<<<grid_for(n, 256), 256, 0, s>>>(out, a, b, n);
  return cudaGetLastError();
}

int step_reduction_blocks(int64_t nfull) {
  int64_t nb = (nfull + kRedThreads - 1) / kRedThreads;
  if (nb > kRedBlocks) nb = kRedBlocks;
  if (nb < 1) nb = 1;
  return (int)nb;
}

int plan_step_reductions(RedJob* jobs, int njobs, const int64_t* nfull) {
  int64_t total = 0;
  for (int j = 0; j < njobs; ++j) total += nfull[j];
  int b0 = 0;
  for (int j = 0; j < njobs; ++j) {
    // a share of kRedBlocks in proportion to the array size (all of it for a lone problem)
    int64_t nb = total > 0 ? (kRedBlocks * nfull[j] + total - 1) / total : 1;
    nb = std::min<int64_t>(std::max<int64_t>(nb, 1), step_reduction_blocks(nfull[j]));
    jobs[j].b0 = b0;
    jobs[j].nb = (int)nb;
    b0 += (int)nb;
  }
  return b0;
}

// one read of each job's source array, written to up to three destinations
__global__ void batch_copy_kernel(const CopyJob* __restrict__ jobs, int njobs) {
  const CopyJob jb = jobs[job_of_block(jobs, njobs)];
  const int blk = blockIdx.x - jb.b0;
  for (int64_t e = blk * (int64_t)blockDim.x + threadIdx.x; e < jb.n; e += (int64_t)jb.nb * blockDim.x) {
    const double v = jb.src[e];
    jb.dst[0][e] = v;
    if (jb.dst[1]) jb.dst[1][e] = v;
    if (jb.dst[2]) jb.dst[2][e] = v;
  }
}

int plan_batch_copy(CopyJob* jobs, int njobs) {
  constexpr int kCopyBlocks = 148 * 8, kCopyThreads = 256;
  int64_t total = 0;
  for (int j = 0; j < njobs; ++j) total += jobs[j].n;
  int b0 = 0;
  for (int j = 0; j < njobs; ++j) {
    int64_t nb = total > 0 ? (kCopyBlocks * jobs[j].n + total - 1) / total : 1;
    nb = std::min<int64_t>(std::max<int64_t>(nb, 1), (jobs[j].n + kCopyThreads - 1) / kCopyThreads);
    jobs[j].b0 = b0;
    jobs[j].nb = (int)std::max<int64_t>(nb, 1);
    b0 += jobs[j].nb;
  }
  return b0;
}

cudaError_t launch_batch_copy(const CopyJob* jobs, int njobs, int nblocks, cudaStream_t s) {
  if (njobs <= 0) return cudaSuccess;
  batch_copy_kernel<<<nblocks, 256, 0, s>>>(jobs, njobs);
  return cudaGetLastError();
}

cudaError_t launch_step_reductions_batch(const Problem* probs, const RedJob* jobs, int njobs, int nblocks,
                                         double tol, double* scratch, double* out, cudaStream_t s) {
  if (njobs <= 0) return cudaSuccess;
  breduce_pass1<<<nblocks, kRedThreads, 0, s>>>(probs, jobs, njobs, scratch);
  breduce_finish1<<<njobs, 32, 0, s>>>(jobs, scratch, out);
  breduce_pass2<<<nblocks, kRedThreads, 0, s>>>(probs, jobs, njobs, tol, out, scratch);
  breduce_finish2<<<njobs, 32, 0, s>>>(jobs, scratch, out);
  return cudaGetLastError();
}

cudaError_t launch_step_reductions(const Problem& P, const double* u, const double* cellJ, double tol,
                                   double* scratch, double* out, cudaStream_t s) {
  const int64_t nfull = (int64_t)P.nx * P.ny * P.nz;
  const int nb = step_reduction_blocks(nfull);
  reduce_pass1<<<nb, kRedThreads, 0, s>>>(P, u, cellJ, scratch);
  reduce_finish1<<<1, 32, 0, s>>>(scratch, nb, out);
  reduce_pass2<<<nb, kRedThreads, 0, s>>>(P, u, tol, out, scratch);
  reduce_finish2<<<1, 32, 0, s>>>(scratch, nb, out);
  return cudaGetLastError();
}

// the reciprocal form's Newton-refined reciprocals next to CUDA's correctly
// rounded division: out[3i .. 3i+2] = rcp_nr(x), rcp_pos(x), 1/x
__global__ void fastmath_probe(const double* __restrict__ x, int n, double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double v = x[i];
  out[3 * i] = fastmath::rcp_nr(v);
  out[3 * i + 1] = fastmath::rcp_pos(v);
  out[3 * i + 2] = 1.0 / v;
}

cudaError_t launch_fastmath_probe(const double* x, int n, double* out, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  fastmath_probe<<<(n + 255) / 256, 256, 0, s>>>(x, n, out);
  return cudaGetLastError();
}

}  // namespace cdm
