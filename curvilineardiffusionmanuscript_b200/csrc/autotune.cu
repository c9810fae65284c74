// autotune.cu — picks the row-marching strip height and the iteration-block
// length of a batch by timing complete steps.
//
// Strip height trades the two ring rows a strip stages (2/h of extra row work)
// against the latency of one strip: a block marches its h rows one after the
// other, and once most problems of a batch have converged the remaining few
// strips set the time of an iteration.  The iteration-block length trades the
// host polls between graph launches against the no-op sweeps launched after a
// problem converged inside a block.  Both depend on the batch's size mix, so
// they are measured: one full step per candidate, from the same inputs and the
// same solver state, fastest kept.
#include <chrono>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "engine.h"

struct cdm_batch {
  cdm::Engine e;
};

namespace cdm {

namespace {

constexpr int kStripH[] = {8, 16, 32, 64};
constexpr int kBlock[] = {4, 8, 16};
constexpr int kNumBlock = 3;
constexpr int kWaveH[] = {16, 32, 64};
constexpr int kWaveBlock[] = {16, 32, 64};
// candidates 0..11: marching kernel, strip height kStripH[c / 3], block kBlock[c % 3];
// 12..17 (2D FP64): tile kernels (variants 2, 3: 32x16 and 32x8 tiles, every row of a
// tile at once, for grids too small to hide a strip's serial march), block kBlock[c % 3];
// 18..26 (2D FP64, reciprocal form): the marching kernel on the wavefront schedule
// (variant 4), strip height kWaveH[t / 3], iterations per launch kWaveBlock[t % 3];
// 27..35: the same with 64-thread blocks (variant 5), which leave fewer columns of
// a narrow problem's last block idle.  3D FP64 (reciprocal form): 0..11 the plane
// march on 32 x 8 column tiles, 12..23 on 16 x 16 tiles (variant 3), strip height
// kStripH[c / 3] and block kBlock[c % 3] in both
constexpr int kNumMarch = 4 * kNumBlock;
constexpr int kNumTile = kNumMarch + 2 * kNumBlock;
constexpr int kNumCand = kNumTile + 18;

struct Cand {
  int variant, strip_h, block;
};

Cand candidate(int c, int ndim) {
  if (c < kNumMarch) return {0, kStripH[c / kNumBlock], kBlock[c % kNumBlock]};
  if (ndim == 3) {
    const int t = c - kNumMarch;
    return {3, kStripH[t / kNumBlock], kBlock[t % kNumBlock]};
  }
  if (c < kNumTile) {
    const int t = c - kNumMarch;
    return {2 + t / kNumBlock, 0, kBlock[t % kNumBlock]};
  }
  const int t = c - kNumTile;
  return {4 + t / 9, kWaveH[(t % 9) / 3], kWaveBlock[t % 3]};
}

double seconds() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// batch fingerprint: dimension, precision, mean and every problem's size
std::string fingerprint(const Engine& e) {
  uint64_t h = 1469598103934665603ull;
  auto mix = [&](uint64_t v) {
    for (int b = 0; b < 8; ++b) {
      h ^= (v >> (8 * b)) & 0xffu;
      h *= 1099511628211ull;
    }
  };
  for (const ProbState& s : e.ps) {
    mix((uint64_t)s.ni);
    mix((uint64_t)s.nj);
    mix((uint64_t)s.nk);
  }
  char buf[96];
  std::snprintf(buf, sizeof(buf), "d%d_p%d_m%d_n%zu_%016llx", e.ndim, e.precision, e.mean, e.ps.size(),
                (unsigned long long)h);
  return buf;
}

// the cache file is a flat JSON object {"fingerprint": index, ...}
int cache_lookup(const char* path, const std::string& key) {
  std::ifstream f(path);
  if (!f) return -1;
  std::stringstream ss;
  ss << f.rdbuf();
  const std::string text = ss.str();
  const std::string pat = "\"" + key + "\":";
  const size_t at = text.find(pat);
  if (at == std::string::npos) return -1;
  const int v = std::atoi(text.c_str() + at + pat.size());
  return (v >= 0 && v < kNumCand) ? v : -1;
}

void cache_store(const char* path, const std::string& key, int value) {
  std::string body;
  {
    std::ifstream f(path);
    if (f) {
      std::stringstream ss;
      ss << f.rdbuf();
      body = ss.str();
    }
  }
  const size_t open = body.find('{'), close = body.rfind('}');
  std::string inner = (open != std::string::npos && close != std::string::npos && close > open)
                          ? body.substr(open + 1, close - open - 1)
                          : std::string();
  while (!inner.empty() && (inner.back() == ' ' || inner.back() == '\n')) inner.pop_back();
  std::ofstream o(path, std::ios::trunc);
  o << "{" << inner << (inner.empty() ? "" : ",") << "\n  \"" << key << "\": " << value << "\n}\n";
}

}  // namespace

int Engine::autotune(double* const* T, const double* const* rho, const double* cp, const cdm_kappa* kappa,
                     const double* dt, const cdm_step_opts* opts, const char* cache_path, int* chosen) {
  *chosen = -1;
  if (!tile_shape(ndim, variant).march) return CDM_OK;  // the 3D tile kernels have no strip height
  // the tile kernels are candidates for 2D FP64 (the mixed sweeps use the marching layout),
  // the wavefront schedule for the reciprocal form
  const int ncand = ndim == 3 ? (precision == CDM_PREC_FP64 ? 2 * kNumMarch : kNumMarch)
                    : precision == CDM_PREC_MIXED ? kNumMarch
                    : (precision == CDM_PREC_FP64_EXACT ? kNumTile : kNumCand);
  const std::string key = fingerprint(*this);
  auto apply = [&](int c) -> int {
    const Cand k = candidate(c, ndim);
    variant = k.variant;
    strip_h_override = k.strip_h;
    tuned_iter_block = k.block;
    return build_items();
  };
  if (cache_path) {
    const int c = cache_lookup(cache_path, key);
    if (c >= 0 && c < ncand) {
      *chosen = c;
      return apply(c);
    }
  }
  cdm_step_opts o;
  cdm_step_opts_default(&o);
  if (opts) o = *opts;
  const int nprob = (int)ps.size();
  CDM_CK(cudaSetDevice(device));
  // scratch inputs on the device: T is copied before every trial, rho once
  std::vector<double*> tin(nprob, nullptr), twork(nprob, nullptr), rdev(nprob, nullptr), qsave;
  std::vector<const double*> rptr(nprob, nullptr);
  std::vector<int> qpar0(nprob), last0(nprob), hist0(nprob);
  int rc = CDM_OK;
  auto cleanup = [&]() {
    for (double* p : tin) cudaFree(p);
    for (double* p : twork) cudaFree(p);
    for (double* p : rdev) cudaFree(p);
    for (double* p : qsave) cudaFree(p);
  };
  const cudaMemcpyKind kind = o.mem == CDM_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  CDM_CK(fence_caller());
  for (int p = 0; p < nprob && rc == CDM_OK; ++p) {
    const size_t bytes = (size_t)ps[p].nfull * sizeof(double);
    if (cudaMalloc((void**)&tin[p], bytes) != cudaSuccess || cudaMalloc((void**)&twork[p], bytes) != cudaSuccess ||
        cudaMemcpyAsync(tin[p], T[p], bytes, kind, stream) != cudaSuccess)
      rc = CDM_CUDA_ERROR;
    if (rc == CDM_OK && o.mem != CDM_MEM_DEVICE) {
      if (cudaMalloc((void**)&rdev[p], bytes) != cudaSuccess ||
          cudaMemcpyAsync(rdev[p], rho[p], bytes, kind, stream) != cudaSuccess)
        rc = CDM_CUDA_ERROR;
      rptr[p] = rdev[p];
    } else {
      rptr[p] = rho[p];
    }
    // the state that carries across steps
    ProbState& s = ps[p];
    qpar0[p] = s.qpar;
    last0[p] = s.last_err_check;
    hist0[p] = s.has_hist;
    for (int d = 0; d < ndim && rc == CDM_OK; ++d) {
      double* q = nullptr;
      if (cudaMalloc((void**)&q, bytes) != cudaSuccess ||
          cudaMemcpyAsync(q, s.q[s.qpar][d], bytes, cudaMemcpyDeviceToDevice, stream) != cudaSuccess)
        rc = CDM_CUDA_ERROR;
      qsave.push_back(q);
    }
  }
  auto restore = [&]() -> int {
    for (int p = 0; p < nprob; ++p) {
      ProbState& s = ps[p];
      const size_t bytes = (size_t)s.nfull * sizeof(double);
      s.qpar = qpar0[p];
      s.last_err_check = last0[p];
      s.has_hist = hist0[p];
      for (int d = 0; d < ndim; ++d)
        CDM_CK(cudaMemcpyAsync(s.q[s.qpar][d], qsave[(size_t)p * ndim + d], bytes, cudaMemcpyDeviceToDevice,
                               stream));
      CDM_CK(cudaMemcpyAsync(twork[p], tin[p], bytes, cudaMemcpyDeviceToDevice, stream));
    }
    CDM_CK(cudaStreamSynchronize(stream));
    return CDM_OK;
  };
  if (rc != CDM_OK) {
    cleanup();
    set_error("autotune: scratch allocation failed");
    return rc;
  }
  o.mem = CDM_MEM_DEVICE;
  o.iter_block = 0;
  std::vector<cdm_stats> st(nprob);
  std::vector<double> ndt(nprob);
  int best = -1;
  double best_t = 1e300;
  for (int c = 0; c < ncand && rc == CDM_OK; ++c) {
    rc = apply(c);
    // twice from the same state: the first also captures the graph
    for (int rep = 0; rep < 2 && rc == CDM_OK; ++rep) {
      rc = restore();
      if (rc != CDM_OK) break;
      const double t0 = seconds();
      rc = step(twork.data(), rptr.data(), cp, kappa, dt, &o, st.data(), ndt.data());
      const double t = seconds() - t0;
      if (rc == CDM_OK && rep == 1 && t < best_t) {
        best_t = t;
        best = c;
      }
    }
  }
  const int rr = restore();
  cleanup();
  if (rc != CDM_OK) return rc;
  if (rr != CDM_OK) return rr;
  *chosen = best;
  rc = apply(best);
  if (rc == CDM_OK && cache_path) cache_store(cache_path, key, best);
  return rc;
}

}  // namespace cdm

extern "C" int cdm_batch_autotune(cdm_batch* b, double* const* T, const double* const* rho, const double* cp,
                                  const cdm_kappa* kappa, const double* dt, const cdm_step_opts* opts,
                                  const char* cache_path, int* chosen) {
  if (!b || !T || !rho || !cp || !kappa || !dt || !chosen) {
    cdm::set_error("NULL argument");
    return CDM_BAD_INPUT;
  }
  return b->e.autotune(T, rho, cp, kappa, dt, opts, cache_path, chosen);
}

extern "C" int cdm_batch_tuning(const cdm_batch* b, int* variant, int* strip_h, int* iter_block) {
  if (!b || !variant || !strip_h || !iter_block) return CDM_BAD_INPUT;
  *variant = b->e.variant;
  *strip_h = b->e.strip_h_override;
  *iter_block = b->e.tuned_iter_block;
  return CDM_OK;
}

extern "C" int cdm_batch_set_tuning(cdm_batch* b, int variant, int strip_h, int iter_block) {
  if (!b) return CDM_BAD_INPUT;
  cdm::Engine& e = b->e;
  const int nv = cdm::num_tile_shapes(e.ndim);
  const bool exact3d = e.ndim == 3 && e.precision == CDM_PREC_FP64_EXACT;
  bool ok = variant >= 0 && variant < nv && strip_h >= 0 && iter_block >= 1 && iter_block <= 64;
  if (e.precision == CDM_PREC_MIXED) ok = ok && variant == 0;           // FP32 sweeps march
  // 3D: the form fixes the kernel (tile kernels for the exact form, the plane march otherwise)
  if (e.ndim == 3) ok = ok && (exact3d ? (variant == 1 || variant == 2) : (variant == 0 || variant == 3));
  if (variant >= 4) ok = ok && e.precision == CDM_PREC_FP64;              // wavefront: reciprocal form
  if (!ok) {
    cdm::set_error("cdm_batch_set_tuning: variant, strip height or block length not valid for this batch");
    return CDM_BAD_INPUT;
  }
  CDM_CK(cudaSetDevice(e.device));
  e.variant = variant;
  e.strip_h_override = strip_h;
  e.tuned_iter_block = iter_block;
  return e.build_items();
}
