// cdm_finish.cuh — end of a pseudo-iteration: residual partial of the block,
// arrival count and, in the last block of a problem, the stopping rule of
// step! (PseudoTransientSolver.jl:284-318) evaluated on the device.
#pragma once
#include "cdm_device.cuh"

namespace cdm {

// block-wide reduction of the residual partial and the last-block finish.
// `wave_count` (wavefront schedule only): the problem's count of iterations
// finished in the current launch, raised by kWaveDone once it is done.
template <int NT>
__device__ __forceinline__ void finish_iteration(const Problem& P, Ctrl* C, int tile, int iter,
                                                 bool check, double local, bool local_nan, int bad,
                                                 double* s_red, int* s_flag, int* wave_count = nullptr) {
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const bool rms = C->norm_kind == 1;
  // validity bits of the diffusivity of this iteration (validate_scalar, next step)
  const int anybad = __syncthreads_or(bad);
  if (tid == 0 && anybad) atomicOr(&C->abad[iter & 1], anybad);
  if (check) {
    const int anynan = __syncthreads_or(local_nan ? 1 : 0);
    double v = local;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double w = __shfl_xor_sync(0xffffffffu, v, o);
      v = rms ? v + w : fmax(v, w);
    }
    if (lane == 0) s_red[warp] = v;
    __syncthreads();
    if (tid == 0) {
      double r = s_red[0];
      for (int w = 1; w < NT / 32; ++w) r = rms ? r + s_red[w] : fmax(r, s_red[w]);
      if (anynan && !rms) r = __longlong_as_double(0x7ff8000000000000ll);
      P.partial[tile] = r;
    }
  }
  // arrival; the last block of this problem finishes the iteration
  if (tid == 0) {
    __threadfence();
    const unsigned prev = atomicAdd(&C->arrive, 1u);
    *s_flag = (prev == (unsigned)P.ntiles - 1u);
  }
  __syncthreads();
  if (!*s_flag) return;
  __threadfence();
  double L2 = 0.0;
  if (check) {
    // deterministic: fixed partition of partials over threads, fixed tree
    double v = rms ? 0.0 : 0.0;
    bool nan = false;
    for (int t = tid; t < P.ntiles; t += NT) {
      const double w = ld_cg_double(&P.partial[t]);
      if (w != w) nan = true;
      v = rms ? v + w : fmax(v, w);
    }
    const int anynan = __syncthreads_or(nan ? 1 : 0);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double w = __shfl_xor_sync(0xffffffffu, v, o);
      v = rms ? v + w : fmax(v, w);
    }
    if (lane == 0) s_red[warp] = v;
    __syncthreads();
    if (tid == 0) {
      double r = s_red[0];
      for (int w = 1; w < NT / 32; ++w) r = rms ? r + s_red[w] : fmax(r, s_red[w]);
      if (anynan) r = __longlong_as_double(0x7ff8000000000000ll);
      L2 = rms ? sqrt(r / C->nfull) : r / C->sqrtN;
    }
  }
  if (tid == 0) {
    // PseudoTransientSolver.jl:284-318
    if (check) {
      C->n_checks += 1;
      if (iter == 1 && !C->init_fixed) C->init_L2 = L2;
      C->rel = L2 / C->init_L2;
      C->abs = L2;
    }
    const double rel = C->rel, ab = C->abs;
    if (!isfinite(rel) || !isfinite(ab)) {
      C->status = ST_NONFINITE;
      C->done = 1;
    } else if (iter > C->max_iter) {
      C->status = ST_MAX_ITER;
      C->done = 1;
    } else if (rel <= C->rtol || ab <= C->atol) {
      C->done = 1;
    }
    C->abad[(iter + 1) & 1] = 0;
    C->arrive = 0u;
    __threadfence();
    C->iter = iter;
    if (wave_count) {
      __threadfence();
      atomicAdd(wave_count, C->done ? kWaveDone : 1);
    }
  }
}

}  // namespace cdm
