// apt_noalloc.cu — end-of-step reductions that allocate no device memory.
//
// Some callers cannot call cudaMalloc once they are running: a Julia host whose
// CUDA.jl memory pool already holds the device memory the process may use, a
// service that forbids allocation on its latency path, or a process whose
// device memory is capped by the application that embeds it.  For them,
// cdm_step_reductions_noalloc computes what cdm_apt_step computes after the
// pseudo-time loop — next_dt (timestep_control.jl:33-73) and the energy
// balance — from arrays the caller already owns.  Its scratch (per-block
// partials and the results) is the file-scope device array g_scratch below,
// which every GPU that loads this library holds until the process exits.
//
// Sizes: one block reduces kChunk cells of the full array, so at most
// kMaxBlocks * kChunk = 134,217,728 cells fit the scratch; larger meshes are
// rejected with CDM_BAD_INPUT.
//
// The scratch is shared by every call on a device and keeps the last call's
// contents; each call overwrites every partial it reads, so nothing needs
// clearing.  Calls that overlap on the GPU (different streams or threads at
// once) race on the scratch and must not be issued.
//
// Set-up: the first call on a device looks up the device address of the
// scratch with cudaGetSymbolAddress while that device is current.
//
// The call is synchronous: it copies the results into host memory and returns
// once they are there, so it cannot be issued inside a stream capture at any
// time.  Its wait for the device is bounded (CDM_STEP_TIMEOUT_S seconds,
// default 3600) and ends with CDM_TIMEOUT, like every other entry point.
//
// Arguments are checked before anything is launched: every array must be
// device (or managed) memory of the current device, reaching at least the full
// array's size within its allocation, and the stream must belong to the
// current device.  A host pointer or a short array is CDM_BAD_INPUT, not a
// fault on the GPU.
#include <cuda.h>

#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <mutex>
#include <string>
#include <thread>

#include "cdm_apt.h"
#include "engine.h"

namespace cdm {

namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 8192;
constexpr int64_t kChunk = 16384;
constexpr int64_t kMaxCells = (int64_t)kMaxBlocks * kChunk;
constexpr int kResults = 4 * kMaxBlocks;  // results start here: umax, max change, E0, E1, ∫SJ

__device__ __align__(256) double g_scratch[4 * kMaxBlocks + 8];

constexpr int kMaxDevices = 64;
double* g_scratch_ptr[kMaxDevices] = {nullptr};
std::mutex g_setup_mutex;

struct Grid {
  int ndim, ni, nj, nk, nh;
  int64_t nx, ny, nfull;
};

__device__ __forceinline__ bool in_domain(const Grid& g, int64_t e) {
  const int64_t i = e % g.nx, r = e / g.nx, j = r % g.ny, k = r / g.ny;
  const bool ok = i >= g.nh && i < g.nh + g.ni && j >= g.nh && j < g.nh + g.nj;
  return g.ndim == 2 ? ok : (ok && k >= g.nh && k < g.nh + g.nk);
}

// pass 1: max(uⁿ) over the full array (NaN propagates) and, over the domain,
// Σρcₚuⁿ J, Σρcₚuⁿ⁺¹ J and ΣS J; one partial quadruple per block
__global__ void __launch_bounds__(kThreads) noalloc_pass1(Grid g, const double* __restrict__ u_new,
                                                          const double* __restrict__ u_prev,
                                                          const double* __restrict__ rho, const double* __restrict__ S,
                                                          const double* __restrict__ J, double cp, double* scratch) {
  const int64_t e0 = blockIdx.x * kChunk, e1 = min(e0 + kChunk, g.nfull);
  double mx = -INFINITY, a0 = 0.0, a1 = 0.0, a2 = 0.0;
  bool nan = false;
  for (int64_t e = e0 + threadIdx.x; e < e1; e += kThreads) {
    const double up = u_prev[e];
    if (up != up) nan = true;
    else mx = fmax(mx, up);
    if (in_domain(g, e)) {
      const double w = rho[e] * cp;
      a0 += w * up * J[e];
      a1 += w * u_new[e] * J[e];
      if (S) a2 += S[e] * J[e];
    }
  }
  __shared__ double sm[4][kThreads / 32];
  const int anynan = __syncthreads_or(nan);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    a0 += __shfl_xor_sync(0xffffffffu, a0, o);
    a1 += __shfl_xor_sync(0xffffffffu, a1, o);
    a2 += __shfl_xor_sync(0xffffffffu, a2, o);
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) {
    sm[0][w] = mx;
    sm[1][w] = a0;
    sm[2][w] = a1;
    sm[3][w] = a2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = sm[0][0], s0 = sm[1][0], s1 = sm[2][0], s2 = sm[3][0];
    for (int k = 1; k < kThreads / 32; ++k) {
      m = fmax(m, sm[0][k]);
      s0 += sm[1][k];
      s1 += sm[2][k];
      s2 += sm[3][k];
    }
    if (anynan) m = __longlong_as_double(0x7ff8000000000000ll);
    scratch[4 * blockIdx.x + 0] = m;
    scratch[4 * blockIdx.x + 1] = s0;
    scratch[4 * blockIdx.x + 2] = s1;
    scratch[4 * blockIdx.x + 3] = s2;
  }
}

// fold the pass-1 partials in block order (deterministic)
__global__ void noalloc_finish1(int nb, double* scratch) {
  if (threadIdx.x != 0) return;
  double m = -INFINITY, s0 = 0.0, s1 = 0.0, s2 = 0.0;
  bool nan = false;
  for (int b = 0; b < nb; ++b) {
    const double v = scratch[4 * b];
    if (v != v) nan = true;
    else m = fmax(m, v);
    s0 += scratch[4 * b + 1];
    s1 += scratch[4 * b + 2];
    s2 += scratch[4 * b + 3];
  }
  scratch[kResults + 0] = nan ? __longlong_as_double(0x7ff8000000000000ll) : m;
  scratch[kResults + 2] = s0;
  scratch[kResults + 3] = s1;
  scratch[kResults + 4] = s2;
}

// pass 2: max over the full array of |uⁿ⁺¹ − uⁿ| / (uⁿ⁺¹ + u0), masked where not
// finite, u0 = tol·max(uⁿ) (timestep_control.jl:43-47, :67-73)
__global__ void __launch_bounds__(kThreads) noalloc_pass2(Grid g, const double* __restrict__ u_new,
                                                          const double* __restrict__ u_prev, double tol,
                                                          double* scratch) {
  const double u0 = scratch[kResults] * tol;
  const int64_t e0 = blockIdx.x * kChunk, e1 = min(e0 + kChunk, g.nfull);
  double mx = -INFINITY;
  for (int64_t e = e0 + threadIdx.x; e < e1; e += kThreads) {
    const double a = u_new[e], b = u_prev[e];
    double d = fabs(a - b) / (a + u0);
    d = isfinite(d) ? d : 0.0;
    mx = fmax(mx, d);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  __shared__ double sm[kThreads / 32];
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < kThreads / 32; ++k) mx = fmax(mx, sm[k]);
    scratch[blockIdx.x] = mx;
  }
}

__global__ void noalloc_finish2(int nb, double* scratch) {
  if (threadIdx.x != 0) return;
  double m = -INFINITY;
  for (int b = 0; b < nb; ++b) m = fmax(m, scratch[b]);
  scratch[kResults + 1] = m;
}

// device address of the scratch on the current device (looked up once per device)
int scratch_on_current_device(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    return CDM_CUDA_ERROR;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("device ordinal out of range for the allocation-free reductions");
    return CDM_NO_DEVICE;
  }
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess) {
      set_error(std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
      return CDM_CUDA_ERROR;
    }
    g_scratch_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_ptr[dev];
  return CDM_OK;
}

// cuMemGetAddressRange through the runtime's driver entry point (no link
// against the driver library); NULL when the driver does not provide it
using AddressRangeFn = CUresult (*)(CUdeviceptr*, size_t*, CUdeviceptr);
AddressRangeFn address_range_fn() {
  static AddressRangeFn fn = nullptr;
  static bool looked = false;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!looked) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuMemGetAddressRange", &p, 12000, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<AddressRangeFn>(p);
    looked = true;
  }
  return fn;
}

// `name` must be device or managed memory that the current device `dev` can
// read for `bytes` bytes from `ptr` within one allocation
int check_device_array(const char* name, const void* ptr, int64_t bytes, int dev) {
  cudaPointerAttributes at;
  cudaError_t e = cudaPointerGetAttributes(&at, ptr);
  if (e != cudaSuccess) {
    cudaGetLastError();  // the query's error is not sticky; clear it
    set_error(std::string("cdm_step_reductions_noalloc: ") + name + " is not a CUDA pointer (" +
              cudaGetErrorString(e) + ")");
    return CDM_BAD_INPUT;
  }
  if (at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged) {
    set_error(std::string("cdm_step_reductions_noalloc: ") + name + " must be device memory (got " +
              (at.type == cudaMemoryTypeHost ? "page-locked host memory" : "host memory") + ")");
    return CDM_BAD_INPUT;
  }
  if (at.type == cudaMemoryTypeDevice && at.device != dev) {
    set_error(std::string("cdm_step_reductions_noalloc: ") + name + " lives on device " +
              std::to_string(at.device) + ", the current device is " + std::to_string(dev));
    return CDM_BAD_INPUT;
  }
  // the extent check is what keeps a short array from being read past its end
  const AddressRangeFn fn = address_range_fn();
  if (!fn) {
    set_error("cdm_step_reductions_noalloc: the driver does not provide cuMemGetAddressRange");
    return CDM_CUDA_ERROR;
  }
  CUdeviceptr base = 0;
  size_t size = 0;
  if (fn(&base, &size, (CUdeviceptr)ptr) != CUDA_SUCCESS) {
    set_error(std::string("cdm_step_reductions_noalloc: ") + name + " is not inside a device allocation");
    return CDM_BAD_INPUT;
  }
  const uint64_t left = (uint64_t)base + size - (uint64_t)(uintptr_t)ptr;
  if ((uint64_t)bytes > left) {
    set_error(std::string("cdm_step_reductions_noalloc: ") + name + " holds " + std::to_string(left / 8) +
              " doubles within its allocation; the full array needs " + std::to_string(bytes / 8));
    return CDM_BAD_INPUT;
  }
  return CDM_OK;
}

// wait for `s` with a bound, polling (no event: nothing is created here)
int wait_bounded(cudaStream_t s) {
  double limit = 3600.0;
  if (const char* v = std::getenv("CDM_STEP_TIMEOUT_S")) limit = std::atof(v);
  const auto t0 = std::chrono::steady_clock::now();
  for (int spins = 0;; ++spins) {
    const cudaError_t e = cudaStreamQuery(s);
    if (e == cudaSuccess) return CDM_OK;
    if (e != cudaErrorNotReady) {
      set_error(std::string("cdm_step_reductions_noalloc: device error: ") + cudaGetErrorString(e));
      return CDM_CUDA_ERROR;
    }
    if (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > limit) {
      set_error("cdm_step_reductions_noalloc: timed out waiting for the device");
      return CDM_TIMEOUT;
    }
    if (spins > 64) std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
}

}  // namespace

}  // namespace cdm

extern "C" int cdm_step_reductions_noalloc(int ndim, int ni, int nj, int nk, int nhalo, const double* u_new,
                                           const double* u_prev, const double* rho, const double* S,
                                           const double* cell_J, double cp, double dt, double ndt_tol,
                                           double maximum_u_change, double timestep_growth_factor,
                                           double* out, void* stream) {
  using namespace cdm;
  if ((ndim != 2 && ndim != 3) || ni < 1 || nj < 1 || (ndim == 3 && nk < 1) || nhalo < 1 || !u_new || !u_prev ||
      !rho || !cell_J || !out || !(dt > 0)) {
    set_error("cdm_step_reductions_noalloc: invalid arguments");
    return CDM_BAD_INPUT;
  }
  Grid g;
  g.ndim = ndim;
  g.ni = ni;
  g.nj = nj;
  g.nk = ndim == 3 ? nk : 1;
  g.nh = nhalo;
  g.nx = ni + 2 * (int64_t)nhalo;
  g.ny = nj + 2 * (int64_t)nhalo;
  const int64_t nz = ndim == 3 ? nk + 2 * (int64_t)nhalo : 1;
  g.nfull = g.nx * g.ny * nz;
  if (g.nfull > kMaxCells) {
    set_error("cdm_step_reductions_noalloc: the full array has " + std::to_string(g.nfull) +
              " cells; the allocation-free scratch holds at most " + std::to_string(kMaxCells));
    return CDM_BAD_INPUT;
  }
  int dev = 0;
  CDM_CK(cudaGetDevice(&dev));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (s) {
    int sdev = -1;
    CDM_CK(cudaStreamGetDevice(s, &sdev));
    if (sdev != dev) {
      set_error("cdm_step_reductions_noalloc: the stream belongs to device " + std::to_string(sdev) +
                ", the current device is " + std::to_string(dev));
      return CDM_BAD_INPUT;
    }
  }
  const int64_t bytes = g.nfull * (int64_t)sizeof(double);
  int rc = CDM_OK;
  const struct {
    const char* name;
    const double* p;
  } arrays[] = {{"u_new", u_new}, {"u_prev", u_prev}, {"rho", rho}, {"S", S}, {"cell_J", cell_J}};
  for (const auto& a : arrays)
    if (a.p && (rc = check_device_array(a.name, a.p, bytes, dev)) != CDM_OK) return rc;
  double* scratch = nullptr;
  rc = scratch_on_current_device(&scratch);
  if (rc != CDM_OK) return rc;
  const int nb = (int)((g.nfull + kChunk - 1) / kChunk);
  noalloc_pass1<<<nb, kThreads, 0, s>>>(g, u_new, u_prev, rho, S, cell_J, cp, scratch);
  noalloc_finish1<<<1, 32, 0, s>>>(nb, scratch);
  noalloc_pass2<<<nb, kThreads, 0, s>>>(g, u_new, u_prev, ndt_tol, scratch);
  noalloc_finish2<<<1, 32, 0, s>>>(nb, scratch);
  double r[5];
  CDM_CK(cudaGetLastError());
  // a bounded wait for the reductions; the copy into pageable host memory that
  // follows then completes at once
  rc = wait_bounded(s);
  if (rc != CDM_OK) return rc;
  CDM_CK(cudaMemcpyAsync(r, scratch + kResults, sizeof(r), cudaMemcpyDeviceToHost, s));
  rc = wait_bounded(s);
  if (rc != CDM_OK) return rc;
  // next_dt (timestep_control.jl:49-51), the same formula cdm_apt_step applies
  const double cand = dt * std::sqrt(std::fabs(maximum_u_change / r[1]));
  const double cap = timestep_growth_factor * dt;
  out[0] = cand < cap ? cand : cap;
  out[1] = r[2];
  out[2] = r[3];
  out[3] = dt * r[4];
  return CDM_OK;
}
