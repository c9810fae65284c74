// engine.cu — host orchestration of the APT solver and the C ABI (cdm_apt.h).
//
// The reference's step! (PseudoTransientSolver.jl:180-351) issues ~11-13
// launches per pseudo-iteration and reads the residual norm back to the host
// at every check.  Here one fused kernel performs a whole iteration, the
// stopping rule runs on the device, blocks of iterations are replayed from a
// captured CUDA graph, and the host polls the control blocks only between
// blocks.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>

#include "engine.h"
#include "cdm_tz.cuh"

namespace cdm {

static thread_local std::string g_error;

void set_error(const std::string& msg) { g_error = msg; }

double now_seconds() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

// applybcs! applies the BCs in tuple order (boundary_operators.jl:26-30);
// every rule writes only its own ghost slab except Periodic at a LO location,
// which writes both slabs of its axis (:229-237) and Periodic at a HI
// location, which writes nothing.  Folding that order gives one rule per side.
int resolve_ghost_rules(int ndim, const cdm_bc* bcs, int* rule, double* val) {
  for (int axis = 0; axis < ndim; ++axis) {
    const cdm_bc lo = bcs[2 * axis], hi = bcs[2 * axis + 1];
    for (const cdm_bc* b : {&lo, &hi})
      if (b->kind < CDM_BC_NEUMANN || b->kind > CDM_BC_NEG_SYMMETRY) return CDM_BAD_INPUT;
    rule[2 * axis] = lo.kind;  // LO: own rule; Periodic LO reads the HI interior
    val[2 * axis] = lo.value;
    if (hi.kind != CDM_BC_PERIODIC) {
      rule[2 * axis + 1] = hi.kind;
      val[2 * axis + 1] = hi.value;
    } else {
      rule[2 * axis + 1] = (lo.kind == CDM_BC_PERIODIC) ? GR_PERIODIC : GR_NONE;
      val[2 * axis + 1] = 0.0;
    }
  }
  return CDM_OK;
}

static void kappa_decompose(double n, int& mode, int& m, int& half) {
  mode = 2;
  m = 0;
  half = 0;
  if (n == 0.0) {
    mode = 0;
    return;
  }
  const double twice = 2.0 * n;
  if (n > 0.0 && n <= 16.0 && twice == std::floor(twice)) {
    mode = 1;
    m = (int)std::floor(n);
    half = (twice != 2.0 * m) ? 1 : 0;
  }
}

template <typename T>
static cudaError_t dalloc(T** p, size_t count) {
  *p = nullptr;
  if (count == 0) return cudaSuccess;
  cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
  if (e != cudaSuccess) return e;
  return cudaMemsetAsync(*p, 0, count * sizeof(T));
}

template <typename T>
static void dfree(T*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

Engine::~Engine() {
  free_graphs();
  for (auto& s : ps) {
    for (int b = 0; b < 2; ++b) {
      dfree(s.u[b]);
      dfree(s.d32[b]);
      dfree(s.ub64[b]);
      for (int d = 0; d < 3; ++d) {
        dfree(s.q[b][d]);
        dfree(s.e32[b][d]);
      }
    }
    dfree(s.u_prev);
    dfree(s.S);
    dfree(s.rho_buf);
    for (int k = 0; k < 9; ++k) {
      dfree(s.coef[k]);
      dfree(s.coef32[k]);
    }
    for (int d = 0; d < 3; ++d) dfree(s.cache[d]);
    dfree(s.cellJ);
    dfree(s.partial);
    dfree(s.guess);
    dfree(s.t_hist);
    dfree(s.tz_mesh);
    dfree(s.tz_terms);
    dfree(s.ub32);
    dfree(s.ab32);
    dfree(s.R32);
    dfree(s.rho32);
  }
  dfree(d_probs);
  dfree(d_ctrl);
  dfree(d_items);
  dfree(d_flags);
  dfree(d_counters);
  dfree(d_wave);
  dfree(wave_plan.head);
  dfree(wave_plan.tb);
  dfree(wave_plan.pj);
  dfree(wave_plan.mask);
  dfree(d_red);
  dfree(d_redout);
  dfree(d_jobs);
  dfree(d_bred);
  dfree(d_cjobs);
  if (h_ctrl) cudaFreeHost(h_ctrl);
  if (h_redout) cudaFreeHost(h_redout);
  if (h_jobs) cudaFreeHost(h_jobs);
  if (h_cjobs) cudaFreeHost(h_cjobs);
  if (h_wave_err) cudaFreeHost(h_wave_err);
  if (ev) cudaEventDestroy(ev);
  for (cudaEvent_t e : ev_pool) cudaEventDestroy(e);
  if (ev_caller) cudaEventDestroy(ev_caller);
  if (ev_fork) cudaEventDestroy(ev_fork);
  if (ev_join) cudaEventDestroy(ev_join);
  if (side_stream) cudaStreamDestroy(side_stream);
  if (own_stream && stream) cudaStreamDestroy(stream);
}

int Engine::free_graphs() {
  if (mixed_graph) cudaGraphExecDestroy(mixed_graph);
  mixed_graph = nullptr;
  for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
  for (auto& kv : graph_defs) cudaGraphDestroy(kv.second);
  graphs.clear();
  graph_defs.clear();
  return CDM_OK;
}

// copy a full-size array given in `mem` space into device buffer dst
static cudaError_t stage_in(double* dst, const double* src, int64_t n, int mem, cudaStream_t s) {
  return cudaMemcpyAsync(dst, src, (size_t)n * sizeof(double),
                         mem == CDM_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s);
}

int Engine::init(int nprob, const cdm_mesh_desc* meshes, const cdm_bc* bcs, const cdm_apt_config* cfg) {
  cdm_apt_config c;
  cdm_apt_config_default(&c);
  if (cfg) c = *cfg;
  device = c.device;
  mean = c.mean;
  precision = c.precision;
  if (nprob < 1) {
    set_error("nprob must be >= 1");
    return CDM_BAD_INPUT;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= device) {
    set_error("no CUDA device available for the APT library");
    return CDM_NO_DEVICE;
  }
  CDM_CK(cudaSetDevice(device));
  cudaDeviceProp prop;
  CDM_CK(cudaGetDeviceProperties(&prop, device));
  if (prop.major != 10) {
    set_error("the APT library is built for sm_100a (B200); device is sm_" + std::to_string(prop.major) +
              std::to_string(prop.minor));
    return CDM_NO_DEVICE;
  }
  if (c.stream) {
    stream = (cudaStream_t)c.stream;
    own_stream = false;
  } else {
    CDM_CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    own_stream = true;
  }
  CDM_CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  CDM_CK(cudaEventCreateWithFlags(&ev_caller, cudaEventDisableTiming));
  CDM_CK(fence_caller());
  CDM_CK(cudaStreamCreateWithFlags(&side_stream, cudaStreamNonBlocking));
  CDM_CK(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
  CDM_CK(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
  ndim = meshes[0].ndim;
  if (ndim != 2 && ndim != 3) {
    set_error("ndim must be 2 or 3");
    return CDM_BAD_INPUT;
  }
  // 3D: the plane-marching kernel computes the reciprocal form; the exact form
  // runs the operation-for-operation tile kernel
  variant = (ndim == 3 && precision == CDM_PREC_FP64_EXACT) ? 1 : 0;
  if (mean != CDM_MEAN_HARMONIC && mean != CDM_MEAN_ARITHMETIC) {
    set_error("mean must be CDM_MEAN_HARMONIC or CDM_MEAN_ARITHMETIC");
    return CDM_BAD_INPUT;
  }
  ps.resize(nprob);
  hp.resize(nprob);
  for (int p = 0; p < nprob; ++p) {
    const cdm_mesh_desc& m = meshes[p];
    ProbState& s = ps[p];
    if (m.ndim != ndim) {
      set_error("all problems of a batch must have the same ndim");
      return CDM_BAD_INPUT;
    }
    if (m.ni < 1 || m.nj < 1 || (ndim == 3 && m.nk < 1) || m.nhalo < 1) {
      set_error("mesh sizes must be >= 1 and nhalo >= 1");
      return CDM_BAD_INPUT;
    }
    s.ndim = ndim;
    s.ni = m.ni;
    s.nj = m.nj;
    s.nk = ndim == 3 ? m.nk : 1;
    s.nh = m.nhalo;
    const int64_t nx = s.ni + 2 * s.nh, ny = s.nj + 2 * s.nh, nz = ndim == 3 ? s.nk + 2 * s.nh : 1;
    s.nfull = nx * ny * nz;
    s.ndomain = (int64_t)s.ni * s.nj * s.nk;
    if (nx * ny > (int64_t)2147483647 || s.nfull > ((int64_t)1 << 40)) {
      set_error("mesh too large");
      return CDM_BAD_INPUT;
    }
    const cdm_bc* pb = bcs + (size_t)p * 2 * ndim;
    for (int l = 0; l < 2 * ndim; ++l) s.bc_kind[l] = pb[l].kind;
    if (resolve_ghost_rules(ndim, pb, s.rule, s.val) != CDM_OK) {
      set_error("invalid boundary-condition kind");
      return CDM_BAD_INPUT;
    }
    // phys_dims (PseudoTransientSolver.jl:122-153)
    s.L = m.L;
    for (int d = 0; d < 3; ++d) s.spacing[d] = m.spacing[d];
    bool need_L = !(m.L > 0), need_sp = !(m.spacing[0] > 0);
    const int64_t nnx = s.ni + 1, nny = s.nj + 1, nnz = ndim == 3 ? s.nk + 1 : 1;
    if (need_L) {
      double Lmin = INFINITY;
      for (int d = 0; d < ndim; ++d) {
        if (!m.node_x[d]) {
          set_error("L not given and node coordinates missing");
          return CDM_BAD_INPUT;
        }
        double lo = INFINITY, hi = -INFINITY;
        for (int64_t e = 0; e < nnx * nny * nnz; ++e) {
          lo = std::min(lo, m.node_x[d][e]);
          hi = std::max(hi, m.node_x[d][e]);
        }
        Lmin = std::min(Lmin, std::fabs(hi - lo));
      }
      s.L = Lmin;
    }
    if (need_sp) {
      if (ndim == 2) {
        if (m.mem != CDM_MEM_HOST || !m.cell_J) {
          set_error("spacing not given: cell_J must be a host array to derive it");
          return CDM_BAD_INPUT;
        }
        double jmin = INFINITY;
        for (int64_t b = 0; b < s.nj; ++b)
          for (int64_t a = 0; a < s.ni; ++a) jmin = std::min(jmin, m.cell_J[(a + s.nh) + nx * (b + s.nh)]);
        s.spacing[0] = s.spacing[1] = std::sqrt(jmin);
      } else {
        for (int d = 0; d < 3; ++d) {
          if (!m.node_x[d]) {
            set_error("spacing not given and node coordinates missing");
            return CDM_BAD_INPUT;
          }
          const int64_t st = d == 0 ? 1 : (d == 1 ? nnx : nnx * nny);
          double mn = INFINITY;
          for (int64_t kk = 0; kk < nnz; ++kk)
            for (int64_t jj = 0; jj < nny; ++jj)
              for (int64_t ii = 0; ii < nnx; ++ii) {
                const int64_t e = ii + nnx * (jj + nny * kk);
                const bool has = d == 0 ? ii + 1 < nnx : (d == 1 ? jj + 1 < nny : kk + 1 < nnz);
                if (has) mn = std::min(mn, m.node_x[d][e + st] - m.node_x[d][e]);
              }
          s.spacing[d] = mn;
        }
      }
    }
    if (!(s.L > 0)) {
      set_error("physical length L must be > 0");
      return CDM_BAD_INPUT;
    }
    // allocations
    const size_t N = (size_t)s.nfull;
    for (int b = 0; b < 2; ++b) {
      CDM_CK(dalloc(&s.u[b], N));
      for (int d = 0; d < ndim; ++d) CDM_CK(dalloc(&s.q[b][d], N));
    }
    CDM_CK(dalloc(&s.u_prev, N));
    CDM_CK(dalloc(&s.S, N));
    for (int k = 0; k < (ndim == 2 ? 5 : 9); ++k) CDM_CK(dalloc(&s.coef[k], N));
    for (int d = 0; d < ndim; ++d) CDM_CK(dalloc(&s.cache[d], N));
    CDM_CK(dalloc(&s.cellJ, N));
    // partials are sized for the smallest tile of any shape
    CDM_CK(dalloc(&s.partial, (size_t)s.ndomain + 64));
    // mesh inputs on the device
    MeshPtrs mp;
    std::memset(&mp, 0, sizeof(mp));
    std::vector<double*> tmp;
    auto dev_in = [&](const double* src, const double** dst) -> int {
      *dst = nullptr;
      if (!src) return CDM_OK;
      if (m.mem == CDM_MEM_DEVICE) {
        *dst = src;
        return CDM_OK;
      }
      double* d = nullptr;
      CDM_CK(cudaMalloc((void**)&d, N * sizeof(double)));
      tmp.push_back(d);
      CDM_CK(cudaMemcpyAsync(d, src, N * sizeof(double), cudaMemcpyHostToDevice, stream));
      *dst = d;
      return CDM_OK;
    };
    int rc = CDM_OK;
    for (int a = 0; a < ndim && rc == CDM_OK; ++a)
      for (int cc = 0; cc < ndim && rc == CDM_OK; ++cc) {
        if (!m.cell_inv[3 * a + cc]) {
          set_error("missing cell_inv metric");
          rc = CDM_BAD_INPUT;
          break;
        }
        rc = dev_in(m.cell_inv[3 * a + cc], &mp.inv[3 * a + cc]);
      }
    for (int f = 0; f < ndim && rc == CDM_OK; ++f) {
      if (!m.edge_J[f]) {
        set_error("missing edge_J metric");
        rc = CDM_BAD_INPUT;
        break;
      }
      rc = dev_in(m.edge_J[f], &mp.edgeJ[f]);
      for (int k = 0; k < 9 && rc == CDM_OK; ++k) {
        const int a = k / 3, cc = k % 3;
        if (a >= ndim || cc >= ndim) continue;
        if (!m.edge_hat[f][k]) {
          set_error("missing edge_hat metric");
          rc = CDM_BAD_INPUT;
          break;
        }
        rc = dev_in(m.edge_hat[f][k], &mp.edgehat[f][k]);
      }
    }
    if (rc == CDM_OK && m.cell_J) {
      CDM_CK(stage_in(s.cellJ, m.cell_J, s.nfull, m.mem, stream));
    }
    if (rc == CDM_OK) {
      Problem P;
      std::memset(&P, 0, sizeof(P));
      P.ndim = ndim;
      P.ni = s.ni;
      P.nj = s.nj;
      P.nk = s.nk;
      P.nh = s.nh;
      P.nx = (int)nx;
      P.ny = (int)ny;
      P.nz = (int)nz;
      cudaError_t e1 = launch_metric_cache(P, mp, s.cache, stream);
      cudaError_t e2 = launch_coefficients(P, mp, s.cache, s.coef, stream);
      if (e1 != cudaSuccess || e2 != cudaSuccess) {
        set_error(std::string("metric kernels: ") + cudaGetErrorString(e1 != cudaSuccess ? e1 : e2));
        rc = CDM_CUDA_ERROR;
      }
    }
    cudaError_t es = cudaStreamSynchronize(stream);
    for (double* d : tmp) cudaFree(d);
    if (rc != CDM_OK) return rc;
    if (es != cudaSuccess) {
      set_error(std::string("mesh setup: ") + cudaGetErrorString(es));
      return CDM_CUDA_ERROR;
    }
  }
  CDM_CK(dalloc(&d_probs, (size_t)nprob));
  CDM_CK(dalloc(&d_ctrl, (size_t)nprob));
  CDM_CK(cudaMallocHost((void**)&h_ctrl, sizeof(Ctrl) * nprob));
  std::memset(h_ctrl, 0, sizeof(Ctrl) * nprob);
  CDM_CK(dalloc(&d_flags, (size_t)nprob));
  CDM_CK(dalloc(&d_counters, (size_t)4));
  CDM_CK(dalloc(&d_wave, (size_t)nprob));
  wave_plan.cap = (long long)kWaveMaxRounds * nprob;
  CDM_CK(dalloc(&wave_plan.head, (size_t)2));
  CDM_CK(dalloc(&wave_plan.tb, (size_t)wave_plan.cap + 1));
  CDM_CK(dalloc(&wave_plan.pj, (size_t)wave_plan.cap));
  CDM_CK(dalloc(&wave_plan.mask, (size_t)nprob));
  if (const char* e = std::getenv("CDM_WAVE_PACE")) wave_pace = std::atoi(e) != 0 ? 1 : 0;
  CDM_CK(cudaMallocHost((void**)&h_wave_err, sizeof(unsigned int)));
  *h_wave_err = 0u;
  CDM_CK(dalloc(&d_red, (size_t)4 * 1024));
  CDM_CK(dalloc(&d_redout, (size_t)8 * nprob));
  CDM_CK(cudaMallocHost((void**)&h_redout, sizeof(double) * 8 * nprob));
  CDM_CK(dalloc(&d_jobs, (size_t)nprob));
  CDM_CK(cudaMallocHost((void**)&h_jobs, sizeof(RedJob) * nprob));
  CDM_CK(dalloc(&d_bred, (size_t)4 * (1024 + nprob)));
  CDM_CK(dalloc(&d_cjobs, (size_t)2 * nprob));
  CDM_CK(cudaMallocHost((void**)&h_cjobs, sizeof(CopyJob) * 2 * nprob));
  if (precision == CDM_PREC_MIXED) {
    int rc = mixed_alloc();
    if (rc != CDM_OK) return rc;
  }
  int rc = build_items();
  if (rc != CDM_OK) return rc;
  CDM_CK(cudaStreamSynchronize(stream));
  return CDM_OK;
}

int Engine::build_items() {
  const TileShape ts = tile_shape(ndim, variant);
  std::vector<int2> items;
  const int nprob = (int)ps.size();
  for (int p = 0; p < nprob; ++p) {
    ProbState& s = ps[p];
    if (ts.march == 2) {
      // 3D: (i, j) column tiles of tx x ty cells marching strips of k-planes;
      // a single problem gets about 12 strips per SM, none shorter than 8 planes
      s.tiles_i = (s.ni + ts.tx - 1) / ts.tx;
      s.tiles_j = (s.nj + ts.ty - 1) / ts.ty;
      int h = 32;
      if (strip_h_override > 0) {
        h = strip_h_override;
      } else if (nprob == 1) {
        const int cols = s.tiles_i * s.tiles_j;
        int nstrips = (148 * 12 + cols - 1) / cols;
        nstrips = std::max(1, std::min(nstrips, (s.nk + 7) / 8));
        h = (s.nk + nstrips - 1) / nstrips;
      }
      s.strip_h = std::max(1, std::min(h, s.nk));
      s.tiles_k = (s.nk + s.strip_h - 1) / s.strip_h;
    } else if (ts.march) {
      // column blocks of tx-2 owned columns; strips of rows sized so that a
      // single problem fills several waves of 148 SMs
      const int ow = ts.tx - 2;
      s.tiles_i = (s.ni + ow - 1) / ow;
      // a single problem: about 24 strips per SM (several waves), no shorter
      // than 8 rows (the two staged ring rows cost 2/h); a batch: 64-row strips
      int h = 64;
      if (strip_h_override > 0) {
        h = strip_h_override;
      } else if (nprob == 1) {
        const int target = 148 * 24;
        int nstrips = (target + s.tiles_i - 1) / s.tiles_i;
        nstrips = std::max(1, std::min(nstrips, (s.nj + 7) / 8));
        h = (s.nj + nstrips - 1) / nstrips;
      }
      s.strip_h = std::max(1, std::min(h, s.nj));
      s.tiles_j = (s.nj + s.strip_h - 1) / s.strip_h;
      s.tiles_k = 1;
    } else {
      s.tiles_i = (s.ni + ts.tx - 1) / ts.tx;
      s.tiles_j = (s.nj + ts.ty - 1) / ts.ty;
      s.tiles_k = ndim == 3 ? (s.nk + ts.tz - 1) / ts.tz : 1;
      s.strip_h = 0;
    }
    s.ntiles = s.tiles_i * s.tiles_j * s.tiles_k;
    for (int t = 0; t < s.ntiles; ++t) items.push_back(make_int2((int)p, t));
  }
  // interleave tiles of different problems so that a launch spreads every
  // problem over the whole GPU (uneven batches).  The wavefront schedule keeps
  // each problem's strips together instead: a problem's strips of the next
  // iteration then come a whole batch of tickets after its strips of this one,
  // which have finished by the time they are reached, and boundary strips are
  // tagged in bit 30 of the tile index.
  if (ts.march == 3) {
    int first = 0;
    for (ProbState& s : ps) {
      s.item0 = first;
      first += s.ntiles;
    }
    for (int2& it : items) {
      const ProbState& s = ps[it.x];
      if (!march_tile_no_ghost_rows(s.nj, s.tiles_i, s.strip_h, it.y)) it.y |= 1 << 30;
    }
  } else if (ps.size() > 1) {
    std::vector<int2> mixed;
    mixed.reserve(items.size());
    std::vector<int> next(ps.size(), 0);
    bool more = true;
    while (more) {
      more = false;
      for (size_t p = 0; p < ps.size(); ++p)
        if (next[p] < ps[p].ntiles) {
          mixed.push_back(make_int2((int)p, next[p]++));
          more = true;
        }
    }
    items.swap(mixed);
  }
  // the fast 2D and 3D kernels run boundary strips and interior strips as two launches
  n_edge = (int)items.size();
  if (ts.march == 2) {
    std::vector<int2> edge, inner;
    for (const int2& it : items) {
      const ProbState& s = ps[it.x];
      (march3d_tile_interior(s.ni, s.nj, s.tiles_i, s.tiles_j, ts.tx, ts.ty, it.y) ? inner : edge).push_back(it);
    }
    n_edge = (int)edge.size();
    items.assign(edge.begin(), edge.end());
    items.insert(items.end(), inner.begin(), inner.end());
  } else if (ts.march == 1 && precision != CDM_PREC_FP64_EXACT) {
    std::vector<int2> edge, inner;
    for (const int2& it : items) {
      const ProbState& s = ps[it.x];
      const bool in = precision == CDM_PREC_MIXED ? march_tile_interior(s.ni, s.nj, s.tiles_i, s.strip_h, ts.tx, it.y)
                                                  : march_tile_no_ghost_rows(s.nj, s.tiles_i, s.strip_h, it.y);
      (in ? inner : edge).push_back(it);
    }
    n_edge = (int)edge.size();
    items.assign(edge.begin(), edge.end());
    items.insert(items.end(), inner.begin(), inner.end());
  }
  dfree(d_items);
  nitems = (int)items.size();
  items_cap = nitems;
  retiled = false;
  CDM_CK(cudaMalloc((void**)&d_items, sizeof(int2) * items.size()));
  CDM_CK(cudaMemcpyAsync(d_items, items.data(), sizeof(int2) * items.size(), cudaMemcpyHostToDevice, stream));
  CDM_CK(cudaStreamSynchronize(stream));
  free_graphs();
  return CDM_OK;
}

int Engine::set_source(int p, const double* S, int mem) {
  ProbState& s = ps[p];
  CDM_CK(cudaSetDevice(device));
  CDM_CK(fence_caller());
  CDM_CK(stage_in(s.S, S, s.nfull, mem, stream));
  Problem P;
  std::memset(&P, 0, sizeof(P));
  P.ndim = ndim;
  P.ni = s.ni;
  P.nj = s.nj;
  P.nk = s.nk;
  P.nh = s.nh;
  P.nx = s.ni + 2 * s.nh;
  P.ny = s.nj + 2 * s.nh;
  P.nz = ndim == 3 ? s.nk + 2 * s.nh : 1;
  CDM_CK(cudaMemsetAsync(d_flags + p, 0, sizeof(int), stream));
  CDM_CK(launch_validate(P, s.S, d_flags + p, stream));
  int flag = 0;
  CDM_CK(cudaMemcpyAsync(&flag, d_flags + p, sizeof(int), cudaMemcpyDeviceToHost, stream));
  CDM_CK(cudaStreamSynchronize(stream));
  s.s_bad = flag;
  return CDM_OK;
}

int Engine::set_guess(int p, const double* u0, int mem) {
  ProbState& s = ps[p];
  CDM_CK(cudaSetDevice(device));
  if (!s.guess) CDM_CK(dalloc(&s.guess, (size_t)s.nfull));
  CDM_CK(fence_caller());
  CDM_CK(stage_in(s.guess, u0, s.nfull, mem, stream));
  CDM_CK(cudaStreamSynchronize(stream));
  s.has_guess = 1;
  return CDM_OK;
}

// define_forcing_wavy's mesh inputs beyond the mesh description: centroids,
// forward metrics and mesh.nnodes (twilight_zone.jl:72-75, :115-118)
int Engine::set_twilight_zone(int p, const cdm_tz_desc* d) {
  ProbState& s = ps[p];
  if (ndim != 2) {
    set_error("the twilight-zone forcing is two-dimensional (twilight_zone.jl:70)");
    return CDM_BAD_INPUT;
  }
  const double* src[6] = {d->x, d->y, d->x_xi, d->x_eta, d->y_xi, d->y_eta};
  for (const double* a : src)
    if (!a) {
      set_error("cdm_tz_desc: every array must be given");
      return CDM_BAD_INPUT;
    }
  if (d->nnodes[0] < 2 || d->nnodes[1] < 2 || (d->mem != CDM_MEM_HOST && d->mem != CDM_MEM_DEVICE)) {
    set_error("cdm_tz_desc: nnodes must be >= 2 and mem a cdm_mem value");
    return CDM_BAD_INPUT;
  }
  CDM_CK(cudaSetDevice(device));
  if (!s.tz_mesh) CDM_CK(dalloc(&s.tz_mesh, (size_t)6 * s.nfull));
  if (!s.tz_terms) CDM_CK(dalloc(&s.tz_terms, (size_t)tz::kNumTerms * s.nfull));
  CDM_CK(fence_caller());
  for (int k = 0; k < 6; ++k) CDM_CK(stage_in(s.tz_mesh + k * s.nfull, src[k], s.nfull, d->mem, stream));
  CDM_CK(cudaStreamSynchronize(stream));
  s.tz_nn[0] = d->nnodes[0];
  s.tz_nn[1] = d->nnodes[1];
  return CDM_OK;
}

// A twilight-zone step runs the operation-for-operation row-marching kernel
// (the only one that adds the forcing): other tuned variants are set aside
// for the step and restored after it.
int Engine::begin_tz_step() {
  tz_active = true;
  if (variant != 0 && variant != 1) {
    tz_saved_variant = variant;
    variant = 0;
    return build_items();
  }
  return CDM_OK;
}

int Engine::end_tz_step() {
  tz_active = false;
  if (tz_saved_variant >= 0) {
    variant = tz_saved_variant;
    tz_saved_variant = -1;
    return build_items();
  }
  return CDM_OK;
}

cudaError_t Engine::fence_caller() {
  if (!own_stream) return cudaSuccess;
  cudaError_t e = cudaEventRecord(ev_caller, cudaStreamLegacy);
  if (e != cudaSuccess) return e;
  return cudaStreamWaitEvent(stream, ev_caller, 0);
}

int Engine::wait_stream(double timeout_s) {
  CDM_CK(cudaEventRecord(ev, stream));
  const double t0 = now_seconds();
  int spins = 0;
  while (true) {
    cudaError_t e = cudaEventQuery(ev);
    if (e == cudaSuccess) return CDM_OK;
    if (e != cudaErrorNotReady) {
      set_error(std::string("device error: ") + cudaGetErrorString(e));
      return CDM_CUDA_ERROR;
    }
    if (now_seconds() - t0 > timeout_s) {
      set_error("timed out waiting for the device");
      return CDM_TIMEOUT;
    }
    if (++spins > 64) std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
}

SweepStreams Engine::sweep_streams() const {
  SweepStreams ss;
  ss.main = stream;
  ss.side = side_stream;
  ss.ev_fork = ev_fork;
  ss.ev_join = ev_join;
  return ss;
}

int Engine::record_pair() {
  if (ev_used + 2 > (int)ev_pool.size()) {
    for (int k = 0; k < 64; ++k) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) != cudaSuccess) return -1;
      ev_pool.push_back(e);
    }
  }
  const int i = ev_used;
  ev_used += 2;
  return i;
}

double Engine::collect_profile_ms() {
  double ms = 0.0;
  for (int i = 0; i + 1 < ev_used; i += 2) {
    float t = 0.f;
    if (cudaEventElapsedTime(&t, ev_pool[i], ev_pool[i + 1]) == cudaSuccess) ms += t;
  }
  ev_used = 0;
  return ms;
}

// K pseudo-iterations: K sweep launches, or one wavefront launch (and its prologue)
cudaError_t Engine::launch_iters(int K) {
  if (tile_shape(ndim, variant).march == 3)
    return launch_march2d_wave(tile_shape(ndim, variant).tx, mean == CDM_MEAN_HARMONIC, d_probs, (int)ps.size(),
                               d_items, nitems, K, wave_pace, d_counters, d_wave, wave_plan, stream);
  cudaError_t le = cudaSuccess;
  for (int k = 0; k < K && le == cudaSuccess; ++k)
    le = launch_sweep_fp64(ndim, variant, precision == CDM_PREC_FP64_EXACT || tz_active, mean == CDM_MEAN_HARMONIC,
                           d_probs, d_items, nitems, n_edge, d_counters, sweep_streams(), tz_active ? 1 : 0);
  return le;
}

int Engine::launch_block(int K, bool use_graph) {
  const int pe = record_pair();
  if (pe >= 0) CDM_CK(cudaEventRecord(ev_pool[pe], stream));
  // kernels launched: the wavefront kernel (its prologue counts as another
  // kernel), or per iteration the fast 2D pair (boundary and interior strips) or
  // one sweep kernel
  const TileShape ts = tile_shape(ndim, variant);
  if (ts.march == 3) {
    prof.sweep_launches += 1;
    prof.other_launches += 1;
  } else if ((ts.march == 1 && precision != CDM_PREC_FP64_EXACT && !tz_active) || ts.march == 2) {
    prof.sweep_launches += (int64_t)K * ((n_edge > 0 ? 1 : 0) + (nitems - n_edge > 0 ? 1 : 0));
  } else {
    prof.sweep_launches += K;
  }
  if (!use_graph) {
    CDM_CK(launch_iters(K));
    if (pe >= 0) CDM_CK(cudaEventRecord(ev_pool[pe + 1], stream));
    return CDM_OK;
  }
  if (graph_variant != variant || graph_tz != tz_active) {
    free_graphs();
    graph_variant = variant;
    graph_tz = tz_active;
  }
  auto it = graphs.find(K);
  if (it == graphs.end()) {
    cudaGraph_t g;
    CDM_CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    const cudaError_t le = launch_iters(K);
    cudaError_t ce = cudaStreamEndCapture(stream, &g);
    if (le != cudaSuccess) {
      set_error(std::string("sweep launch during capture: ") + cudaGetErrorString(le));
      return CDM_CUDA_ERROR;
    }
    CDM_CK(ce);
    cudaGraphExec_t ge;
    CDM_CK(cudaGraphInstantiate(&ge, g, 0));
    graphs[K] = ge;
    graph_defs[K] = g;
    it = graphs.find(K);
  }
  CDM_CK(cudaGraphLaunch(it->second, stream));
  if (pe >= 0) CDM_CK(cudaEventRecord(ev_pool[pe + 1], stream));
  return CDM_OK;
}

// Launch iteration blocks until every problem's control block says done.
int Engine::run_iterations(const cdm_step_opts* o, int predicted, double t_start, double timeout_s) {
  const int K = o->iter_block > 0 ? o->iter_block : tuned_iter_block;
  const bool use_graph = o->use_graph != 0;
  const int nprob = (int)ps.size();
  int launched = 0;
  // launch up to the predicted iteration count without polling
  while (launched + K <= predicted) {
    int rc = launch_block(K, use_graph);
    if (rc != CDM_OK) return rc;
    launched += K;
  }
  while (true) {
    int rc = launch_block(K, use_graph);
    if (rc != CDM_OK) return rc;
    launched += K;
    CDM_CK(cudaMemcpyAsync(h_ctrl, d_ctrl, sizeof(Ctrl) * nprob, cudaMemcpyDeviceToHost, stream));
    CDM_CK(cudaMemcpyAsync(h_wave_err, d_counters + 3, sizeof(unsigned int), cudaMemcpyDeviceToHost, stream));
    rc = wait_stream(timeout_s - (now_seconds() - t_start));
    if (rc != CDM_OK) return rc;
    if (*h_wave_err) {
      set_error("wavefront sweep: a dependency wait exceeded its limit");
      return CDM_TIMEOUT;
    }
    bool all = true;
    for (int p = 0; p < nprob; ++p) all = all && h_ctrl[p].done;
    if (all) return CDM_OK;
    if (now_seconds() - t_start > timeout_s) {
      set_error("step exceeded its wall-clock limit");
      return CDM_TIMEOUT;
    }
    if (tile_shape(ndim, variant).march == 3 && h_ctrl[0].norm_kind == CDM_NORM_MAX) {
      rc = retile_tail();
      if (rc != CDM_OK) return rc;
    }
  }
}

// the shortest strip of the tail re-tiling: a strip's iteration costs the march
// of its rows plus two staged ring rows, one after the other, so with the GPU
// underfilled shorter strips finish an iteration sooner despite the ring rows
constexpr int kTailMinRows = 4;

// Wavefront schedule, once most problems of a batch have converged: the
// strips of the problems still iterating no longer fill the GPU, and an
// iteration of each costs the march of one whole strip.  Halve the strip
// height of those problems (down to kTailMinRows rows) until their strips
// number at least twice the blocks the launch keeps resident, and drop
// converged problems from the ticket list.  Tiling changes no result under the
// max norm (the partials of a problem reduce by max), so this applies between
// launches only.  The step after restores the tuned tiling.
int Engine::retile_tail() {
  const int nprob = (int)ps.size();
  const TileShape ts = tile_shape(ndim, variant);
  const long long target = 2ll * march2d_wave_slots(ts.tx, mean == CDM_MEAN_HARMONIC);
  long long strips = 0;
  int h = 0;
  for (int p = 0; p < nprob; ++p)
    if (!h_ctrl[p].done) {
      strips += ps[p].ntiles;
      h = std::max(h, ps[p].strip_h);
    }
  if (strips >= target || h <= kTailMinRows) return CDM_OK;
  auto count = [&](int hh) {
    long long n = 0;
    for (int p = 0; p < nprob; ++p)
      if (!h_ctrl[p].done) n += (long long)ps[p].tiles_i * ((ps[p].nj + hh - 1) / hh);
    return n;
  };
  int hn = h;
  while (hn > kTailMinRows && count(hn) < target) hn = std::max(kTailMinRows, hn / 2);
  std::vector<int2> items;
  for (int p = 0; p < nprob; ++p) {
    if (h_ctrl[p].done) {
      ps[p].item0 = hp[p].item0 = -1;
      continue;
    }
    ProbState& s = ps[p];
    s.strip_h = std::min(hn, s.nj);
    s.tiles_j = (s.nj + s.strip_h - 1) / s.strip_h;
    s.ntiles = s.tiles_i * s.tiles_j;
    s.item0 = (int)items.size();
    hp[p].strip_h = s.strip_h;
    hp[p].tiles_j = s.tiles_j;
    hp[p].ntiles = s.ntiles;
    hp[p].item0 = s.item0;
    for (int t = 0; t < s.ntiles; ++t) {
      int2 it = make_int2(p, t);
      if (!march_tile_no_ghost_rows(s.nj, s.tiles_i, s.strip_h, t)) it.y |= 1 << 30;
      items.push_back(it);
    }
  }
  if (items.empty()) return CDM_OK;
  if ((int)items.size() > items_cap) {
    dfree(d_items);
    CDM_CK(cudaMalloc((void**)&d_items, sizeof(int2) * items.size()));
    items_cap = (int)items.size();
  }
  CDM_CK(cudaMemcpyAsync(d_items, items.data(), sizeof(int2) * items.size(), cudaMemcpyHostToDevice, stream));
  CDM_CK(cudaMemcpyAsync(d_probs, hp.data(), sizeof(Problem) * nprob, cudaMemcpyHostToDevice, stream));
  CDM_CK(cudaStreamSynchronize(stream));
  nitems = (int)items.size();
  n_edge = nitems;
  retiled = true;
  free_graphs();
  return CDM_OK;
}

// Network prediction of this step's solution from (Tⁿ⁻¹, Tⁿ, κ, J): 1 when
// s.guess holds it, 0 when the step starts from Tⁿ (no network, no previous
// step, 3D, or sizes the network does not take), negative on error
// (-1 CUDA error, otherwise minus the network's status).
int Engine::learned_guess(int p, const cdm_kappa& kappa) {
  ProbState& s = ps[p];
  if (!guess_net || !s.has_hist || ndim != 2 || s.ni % 8 || s.nj % 8 || !s.cellJ) return 0;
  if (!s.guess && dalloc(&s.guess, (size_t)s.nfull) != cudaSuccess) return -1;
  if (cudaStreamSynchronize(stream) != cudaSuccess) return -1;  // Tⁿ staged
  const int rc = cdm_net_predict(guess_net, s.t_hist, s.u_prev, s.cellJ, s.ni, s.nj, s.nh, kappa.k0, kappa.n,
                                 log_jmean, s.guess);
  if (rc != CDM_OK) return -rc;
  prof.other_launches += 22;
  return 1;
}

// Linear extrapolation of this step's solution from the last two steps,
// 2Tⁿ − Tⁿ⁻¹ (the part of the learned guess the network corrects): 1 when
// s.guess holds it, 0 when the step starts from Tⁿ (no previous step), -1 on
// a CUDA error.  No reference counterpart (the reference starts from Tⁿ).
int Engine::extrapolated_guess(int p) {
  ProbState& s = ps[p];
  if (!s.has_hist) return 0;
  if (!s.guess && dalloc(&s.guess, (size_t)s.nfull) != cudaSuccess) return -1;
  if (launch_extrapolate(s.guess, s.u_prev, s.t_hist, s.nfull, stream) != cudaSuccess) return -1;
  prof.other_launches += 1;
  return 1;
}

// A guessed start is stopped where the plain start would stop: the relative
// criterion (:297) divides by the residual norm that the plain start (u = Tⁿ)
// reaches at its first check.  One FP64 iteration from Tⁿ gives that norm;
// then the control block is reset, the iterates are set to the guess and, in
// 2D, the damped flux to the plain flux of the guess.
int Engine::probe_plain_norm(const std::vector<int>& guessed, const std::vector<const double*>& init,
                             double t_start, double timeout_s) {
  const int nprob = (int)ps.size();
  std::vector<Ctrl> c0(h_ctrl, h_ctrl + nprob);
  int rc = launch_block(1, false);
  if (rc != CDM_OK) return rc;
  CDM_CK(cudaMemcpyAsync(h_ctrl, d_ctrl, sizeof(Ctrl) * nprob, cudaMemcpyDeviceToHost, stream));
  rc = wait_stream(timeout_s - (now_seconds() - t_start));
  if (rc != CDM_OK) return rc;
  for (int p = 0; p < nprob; ++p) {
    ProbState& s = ps[p];
    const double ref = h_ctrl[p].init_L2;
    h_ctrl[p] = c0[p];
    if (guessed[p]) {
      h_ctrl[p].init_L2 = ref;
      h_ctrl[p].init_fixed = 1;
    }
    prof.cell_iters += s.ndomain;
    const size_t bytes = (size_t)s.nfull * sizeof(double);
    CDM_CK(cudaMemcpyAsync(s.u[0], init[p], bytes, cudaMemcpyDeviceToDevice, stream));
    CDM_CK(cudaMemcpyAsync(s.u[1], init[p], bytes, cudaMemcpyDeviceToDevice, stream));
    if (ndim == 2 && s.nh > 1) {
      CDM_CK(launch_dirichlet_fill(hp[p], s.u[0], stream));
      CDM_CK(launch_dirichlet_fill(hp[p], s.u[1], stream));
      prof.other_launches += 2;
    }
    if (guessed[p] && ndim == 2) {
      CDM_CK(launch_flux_init2d(hp[p], s.u[0], s.q[s.qpar][0], s.q[s.qpar][1], stream));
      prof.other_launches += 1;
    }
  }
  CDM_CK(cudaMemsetAsync(d_counters, 0, 4 * sizeof(unsigned int), stream));
  CDM_CK(cudaMemcpyAsync(d_ctrl, h_ctrl, sizeof(Ctrl) * nprob, cudaMemcpyHostToDevice, stream));
  return CDM_OK;
}

int Engine::step(double* const* T, const double* const* rho, const double* cp, const cdm_kappa* kappa,
                 const double* dt, const cdm_step_opts* opts, cdm_stats* stats, double* next_dt) {
  const double t0 = now_seconds();
  cdm_step_opts o;
  cdm_step_opts_default(&o);
  if (opts) o = *opts;
  const int nprob = (int)ps.size();
  CDM_CK(cudaSetDevice(device));
  std::memset(&prof, 0, sizeof(prof));
  ev_used = 0;
  if (retiled) {  // the last step's tail shortened strips: back to the tuned tiling
    const int rb = build_items();
    if (rb != CDM_OK) return rb;
  }
  double timeout_s = 3600.0;
  if (const char* e = std::getenv("CDM_STEP_TIMEOUT_S")) timeout_s = std::atof(e);
  for (int p = 0; p < nprob; ++p) {
    std::memset(&stats[p], 0, sizeof(cdm_stats));
    stats[p].status = CDM_OK;
  }
  // argument checks (:225-227) and validate_scalar (:238-250)
  int predicted = 1 << 30;
  int bad = CDM_OK;
  for (int p = 0; p < nprob; ++p) {
    ProbState& s = ps[p];
    double msp = s.spacing[0];
    for (int d = 1; d < ndim; ++d) msp = std::min(msp, s.spacing[d]);
    const double Vp = o.CFL * msp;
    const Ctrl& prev = h_ctrl[p];
    const int abad = prev.abad[prev.iter & 1];
    std::string why;
    if (!(dt[p] > 0)) why = "dt must be > 0";
    else if (!(Vp > 0)) why = "CFL * spacing must be > 0";
    else if (!T[p] || !rho[p]) why = "T and rho must not be NULL";
    else if ((abad & 1) || (o.enforce_positivity && (abad & 2))) why = "Invalid diffusivity (validate_scalar)";
    else if (s.s_bad & 1) why = "Invalid source_term (validate_scalar)";
    if (!why.empty()) {
      stats[p].status = CDM_BAD_INPUT;
      set_error(why);
      bad = CDM_BAD_INPUT;
    }
  }
  if (o.tz && bad == CDM_OK) {
    // twilight_zone.jl:54-195 (update.jl:23-71, residuals.jl:49-99)
    std::string why;
    if (ndim != 2) why = "tz = true: the twilight-zone forcing is two-dimensional (twilight_zone.jl:70)";
    else if (precision == CDM_PREC_MIXED) why = "tz = true needs an FP64 precision (CDM_PREC_FP64 or _EXACT)";
    for (int p = 0; p < nprob && why.empty(); ++p)
      if (!ps[p].tz_mesh) why = "tz = true needs the mesh inputs of cdm_apt_set_twilight_zone first";
    if (!why.empty()) {
      for (int p = 0; p < nprob; ++p) stats[p].status = CDM_BAD_INPUT;
      set_error(why);
      bad = CDM_BAD_INPUT;
    }
  }
  if (bad != CDM_OK) {
    for (int p = 0; p < nprob; ++p) stats[p].time = now_seconds() - t0;
    return bad;
  }
  // a twilight-zone step restores the tuned kernel variant however it ends
  struct TzGuard {
    Engine* e;
    bool on;
    ~TzGuard() {
      if (on) e->end_tz_step();
    }
  } tz_guard{this, o.tz != 0};
  if (o.tz) {
    const int rb = begin_tz_step();
    if (rb != CDM_OK) return rb;
  }
  // T and rho may still be written by the caller's kernels
  CDM_CK(fence_caller());
  // copy!(solver.u, T); copy!(solver.u_prev, T)  (:229-230): Tⁿ into u_prev and both
  // iterates, every problem in one copy launch (host arrays cross into u_prev first)
  for (int p = 0; p < nprob; ++p) {
    ProbState& s = ps[p];
    CopyJob& j = h_cjobs[p];
    j.n = s.nfull;
    if (o.mem == CDM_MEM_DEVICE) {
      j.src = T[p];
      j.dst[0] = s.u_prev;
      j.dst[1] = s.u[0];
      j.dst[2] = s.u[1];
    } else {
      CDM_CK(stage_in(s.u_prev, T[p], s.nfull, o.mem, stream));
      j.src = s.u_prev;
      j.dst[0] = s.u[0];
      j.dst[1] = s.u[1];
      j.dst[2] = nullptr;
    }
  }
  {
    const int nb = plan_batch_copy(h_cjobs, nprob);
    CDM_CK(cudaMemcpyAsync(d_cjobs, h_cjobs, sizeof(CopyJob) * nprob, cudaMemcpyHostToDevice, stream));
    CDM_CK(launch_batch_copy(d_cjobs, nprob, nb, stream));
    prof.other_launches += 1;
  }
  std::vector<const double*> inits(nprob, nullptr);
  std::vector<int> guessed(nprob, 0);
  bool any_guess = false;
  for (int p = 0; p < nprob; ++p) {
    ProbState& s = ps[p];
    Problem& P = hp[p];
    std::memset(&P, 0, sizeof(P));
    const size_t bytes = (size_t)s.nfull * sizeof(double);
    // the iteration starts from Tⁿ (:229), a user array, or the network's prediction
    const double* init = s.u_prev;
    if (o.guess == CDM_GUESS_USER && s.has_guess) {
      init = s.guess;
    } else if (o.guess == CDM_GUESS_LEARNED) {
      const int lg = learned_guess(p, kappa[p]);
      if (lg < 0) return lg == -1 ? CDM_CUDA_ERROR : -lg;
      if (lg == 1) init = s.guess;
    } else if (o.guess == CDM_GUESS_EXTRAPOLATE) {
      keep_hist = true;
      const int lg = extrapolated_guess(p);
      if (lg < 0) return CDM_CUDA_ERROR;
      if (lg == 1) init = s.guess;
    }
    inits[p] = init;
    guessed[p] = init != s.u_prev;
    any_guess = any_guess || guessed[p];
    // a guessed start first runs the plain start's first iteration (probe below), from
    // the copies of Tⁿ made above
    const double* rp = rho[p];
    if (o.mem != CDM_MEM_DEVICE) {
      if (!s.rho_buf) CDM_CK(dalloc(&s.rho_buf, (size_t)s.nfull));
      CDM_CK(cudaMemcpyAsync(s.rho_buf, rho[p], bytes, cudaMemcpyHostToDevice, stream));
      rp = s.rho_buf;
    }
    P.ndim = ndim;
    P.ni = s.ni;
    P.nj = s.nj;
    P.nk = s.nk;
    P.nh = s.nh;
    P.nx = s.ni + 2 * s.nh;
    P.ny = s.nj + 2 * s.nh;
    P.nz = ndim == 3 ? s.nk + 2 * s.nh : 1;
    P.tiles_i = s.tiles_i;
    P.tiles_j = s.tiles_j;
    P.tiles_k = s.tiles_k;
    P.ntiles = s.ntiles;
    P.strip_h = s.strip_h;
    P.item0 = s.item0;
    P.mean = mean;
    P.subcycle = o.subcycle_conductivity ? 1 : 0;
    kappa_decompose(kappa[p].n, P.kmode, P.km, P.khalf);
    P.qpar = s.qpar;
    for (int l = 0; l < 6; ++l) {
      P.rule[l] = s.rule[l];
      P.val[l] = s.val[l];
    }
    double msp = s.spacing[0];
    for (int d = 1; d < ndim; ++d) msp = std::min(msp, s.spacing[d]);
    P.dt = dt[p];
    P.cp = cp[p];
    P.k0 = kappa[p].k0;
    P.kn = kappa[p].n;
    P.L = s.L;
    P.LL = s.L * s.L;
    P.Vpdtau = o.CFL * msp;  // :223
    P.VpL = P.Vpdtau * s.L;
    for (int b = 0; b < 2; ++b) {
      P.u[b] = s.u[b];
      for (int d = 0; d < 3; ++d) P.q[b][d] = s.q[b][d];
      P.d32[b] = s.d32[b];
      P.ub64[b] = s.ub64[b];
      for (int d = 0; d < 3; ++d) P.e32[b][d] = s.e32[b][d];
    }
    P.u_prev = s.u_prev;
    P.S = s.S;
    P.rho = rp;
    for (int k = 0; k < 9; ++k) {
      P.coef[k] = s.coef[k];
      P.coef32[k] = s.coef32[k];
    }
    P.partial = s.partial;
    P.ctrl = d_ctrl + p;
    P.ub32 = s.ub32;
    P.ab32 = s.ab32;
    P.R32 = s.R32;
    P.rho32 = s.rho32;
    P.tz = nullptr;
    if (o.tz) {
      // the forcing's α-independent terms at this step's t (twilight_zone.jl:69-183)
      TzMesh tm;
      tm.x = s.tz_mesh;
      tm.y = s.tz_mesh + s.nfull;
      tm.xxi = s.tz_mesh + 2 * s.nfull;
      tm.xeta = s.tz_mesh + 3 * s.nfull;
      tm.yxi = s.tz_mesh + 4 * s.nfull;
      tm.yeta = s.tz_mesh + 5 * s.nfull;
      tm.nnx = s.tz_nn[0];
      tm.nny = s.tz_nn[1];
      CDM_CK(launch_tz_terms(P, tm, rp, cp[p], o.t, o.no_t, s.tz_terms, stream));
      prof.other_launches += 1;
      P.tz = s.tz_terms;
    }
    if (ndim == 2 && s.nh > 1) {
      CDM_CK(launch_dirichlet_fill(P, s.u[0], stream));
      CDM_CK(launch_dirichlet_fill(P, s.u[1], stream));
      prof.other_launches += 2;
    }
    // control block (:206-221)
    Ctrl& C = h_ctrl[p];
    std::memset(&C, 0, sizeof(Ctrl));
    const int last = s.last_err_check;
    C.min_err_check = (int)std::nearbyint(last * 0.9);
    C.err_interval = std::max(1, (last - C.min_err_check) / 2);
    C.max_iter = o.max_iter;
    C.check_every = o.check_every;
    C.norm_kind = o.norm;
    C.rtol = o.rtol;
    C.atol = o.atol;
    C.init_L2 = INFINITY;
    C.rel = 2 * o.rtol;
    C.abs = 2 * o.atol;
    C.nfull = (double)s.nfull;
    C.sqrtN = std::sqrt((double)s.nfull);
    C.est_iter = wave_pace ? last : 0;
    predicted = std::min(predicted, o.check_every > 0 ? 0 : std::max(0, C.min_err_check - 1));
  }
  CDM_CK(cudaMemcpyAsync(d_probs, hp.data(), sizeof(Problem) * nprob, cudaMemcpyHostToDevice, stream));
  CDM_CK(cudaMemsetAsync(d_counters, 0, 4 * sizeof(unsigned int), stream));
  CDM_CK(cudaMemcpyAsync(d_ctrl, h_ctrl, sizeof(Ctrl) * nprob, cudaMemcpyHostToDevice, stream));
  int rc = CDM_OK;
  if (any_guess) rc = probe_plain_norm(guessed, inits, t0, timeout_s);
  if (rc == CDM_OK) {
    if (precision == CDM_PREC_MIXED) rc = step_mixed(&o, t0, timeout_s);
    else rc = run_iterations(&o, predicted, t0, timeout_s);
  }
  if (rc != CDM_OK) {
    for (int p = 0; p < nprob; ++p) {
      stats[p].status = rc;
      stats[p].time = now_seconds() - t0;
    }
    return rc;
  }
  // after the loop (:321-346)
  int worst = CDM_OK;
  int njobs = 0, nout = 0;
  std::vector<int64_t> red_n(nprob);
  for (int p = 0; p < nprob; ++p) {
    ProbState& s = ps[p];
    const Ctrl& C = h_ctrl[p];
    stats[p].rel_err = C.rel;
    stats[p].abs_err = C.abs;
    stats[p].niter = C.iter;
    stats[p].status = C.status;
    stats[p].n_checks = C.n_checks;
    stats[p].n_restarts = C.n_restarts;
    if (precision != CDM_PREC_MIXED) s.qpar = (s.qpar + C.iter) & 1;
    if (C.status != ST_OK) {
      worst = std::max(worst, C.status);
      if (C.status == ST_NONFINITE)
        set_error("Non-finite error detected! abs_error = " + std::to_string(C.abs) +
                  ", rel_error = " + std::to_string(C.rel));
      else
        set_error("Maximum iteration limit reached (" + std::to_string(o.max_iter) + ")");
      continue;
    }
    s.last_err_check = C.iter;
    // Tⁿ becomes the previous step of the next call's learned or extrapolated guess
    if (guess_net || keep_hist) {
      if (!s.t_hist) CDM_CK(dalloc(&s.t_hist, (size_t)s.nfull));
      CDM_CK(cudaMemcpyAsync(s.t_hist, s.u_prev, (size_t)s.nfull * sizeof(double), cudaMemcpyDeviceToDevice,
                             stream));
      s.has_hist = 1;
    }
    // result: the last ping-pong iterate (FP64 path) or the last restart's base (mixed)
    double* res = precision == CDM_PREC_MIXED ? s.ub64[(C.n_restarts - 1) & 1] : s.u[C.iter & 1];
    CDM_CK(launch_clamp(res, s.nfull, o.enforce_positivity, o.apply_cutoff, stream));
    h_jobs[njobs].p = p;
    h_jobs[njobs].u = res;
    h_jobs[njobs].J = s.cellJ;
    red_n[njobs++] = s.nfull;
    prof.other_launches += (o.enforce_positivity || o.apply_cutoff) ? 1 : 0;
    prof.cell_iters += s.ndomain * (int64_t)C.iter;
    if (o.mem == CDM_MEM_DEVICE) {  // into the caller's array in one copy launch below
      CopyJob& j = h_cjobs[nprob + nout++];
      j.src = res;
      j.dst[0] = T[p];
      j.dst[1] = j.dst[2] = nullptr;
      j.n = s.nfull;
    } else {
      CDM_CK(cudaMemcpyAsync(T[p], res, (size_t)s.nfull * sizeof(double), cudaMemcpyDeviceToHost, stream));
    }
  }
  if (nout > 0) {
    const int nb = plan_batch_copy(h_cjobs + nprob, nout);
    CDM_CK(cudaMemcpyAsync(d_cjobs + nprob, h_cjobs + nprob, sizeof(CopyJob) * nout, cudaMemcpyHostToDevice, stream));
    CDM_CK(launch_batch_copy(d_cjobs + nprob, nout, nb, stream));
    prof.other_launches += 1;
  }
  if (njobs > 0) {
    // next_dt and energy reductions of every problem in four launches
    const int nblocks = plan_step_reductions(h_jobs, njobs, red_n.data());
    CDM_CK(cudaMemcpyAsync(d_jobs, h_jobs, sizeof(RedJob) * njobs, cudaMemcpyHostToDevice, stream));
    CDM_CK(launch_step_reductions_batch(d_probs, d_jobs, njobs, nblocks, o.ndt_tol, d_bred, d_redout, stream));
    prof.other_launches += 4;
  }
  CDM_CK(cudaMemcpyAsync(h_redout, d_redout, sizeof(double) * 8 * nprob, cudaMemcpyDeviceToHost, stream));
  rc = wait_stream(timeout_s);
  if (rc != CDM_OK) return rc;
  prof.sweep_ms = collect_profile_ms();
  for (int p = 0; p < nprob; ++p) {
    const double* r = h_redout + 8 * p;
    if (stats[p].status == CDM_OK) {
      // next_dt (timestep_control.jl:43-54)
      if (o.calculate_next_dt) {
        const double cand = dt[p] * std::sqrt(std::fabs(o.maximum_u_change / r[1]));
        const double cap = o.timestep_growth_factor * dt[p];
        next_dt[p] = cand < cap ? cand : cap;
      } else {
        next_dt[p] = dt[p];
      }
      stats[p].energy_before = r[2];
      stats[p].energy_after = r[3];
      stats[p].source_work = dt[p] * r[4];
    } else {
      next_dt[p] = dt[p];
    }
    stats[p].time = now_seconds() - t0;
  }
  return worst;
}

}  // namespace cdm

// ============================================================================
// C ABI
using cdm::Engine;

struct cdm_apt {
  Engine e;
};
struct cdm_batch {
  Engine e;
};

extern "C" {

int cdm_apt_version(void) { return CDM_APT_ABI_VERSION; }

int cdm_selftest_bounded_wait(int device, double limit_s, int* expired) {
  if (!expired || !(limit_s > 0.0) || limit_s > 10.0) {
    cdm::set_error("cdm_selftest_bounded_wait: expired must not be NULL and 0 < limit_s <= 10");
    return CDM_BAD_INPUT;
  }
  *expired = 0;
  CDM_CK(cudaSetDevice(device));
  int* buf = nullptr;  // [0] the count nothing raises, [1] the error flag
  CDM_CK(cudaMalloc((void**)&buf, 2 * sizeof(int)));
  cudaError_t e = cudaMemset(buf, 0, 2 * sizeof(int));
  if (e == cudaSuccess) e = cdm::launch_wave_wait_probe(buf, (unsigned int*)(buf + 1), limit_s, nullptr);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  int flag = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&flag, buf + 1, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(buf);
  if (e != cudaSuccess) {
    cdm::set_error(std::string("cdm_selftest_bounded_wait: ") + cudaGetErrorString(e));
    return CDM_CUDA_ERROR;
  }
  *expired = flag != 0;
  return CDM_OK;
}

int cdm_selftest_fastmath(int device, const double* x, int n, double* out) {
  if (!x || !out || n <= 0 || n > (1 << 22)) {
    cdm::set_error("cdm_selftest_fastmath: x and out must not be NULL and 0 < n <= 2^22");
    return CDM_BAD_INPUT;
  }
  CDM_CK(cudaSetDevice(device));
  double* buf = nullptr;  // n inputs, then 3n results
  CDM_CK(cudaMalloc((void**)&buf, 4 * (size_t)n * sizeof(double)));
  cudaError_t e = cudaMemcpy(buf, x, (size_t)n * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cdm::launch_fastmath_probe(buf, n, buf + n, nullptr);
  if (e == cudaSuccess) e = cudaMemcpy(out, buf + n, 3 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(buf);
  if (e != cudaSuccess) {
    cdm::set_error(std::string("cdm_selftest_fastmath: ") + cudaGetErrorString(e));
    return CDM_CUDA_ERROR;
  }
  return CDM_OK;
}

const char* cdm_apt_last_error(void) { return cdm::g_error.c_str(); }

void cdm_step_opts_default(cdm_step_opts* o) {
  std::memset(o, 0, sizeof(*o));
  o->t = 0.0;
  o->tz = 0;
  o->tz_dim = 1;
  o->no_t = 1;
  o->max_iter = 1500;
  o->rtol = 1e-5;
  o->atol = std::sqrt(2.220446049250313e-16);
  o->error_check_interval = 2;
  o->apply_cutoff = 0;
  o->calculate_next_dt = 1;
  o->subcycle_conductivity = 1;
  o->enforce_positivity = 0;
  o->CFL = 1.0 / std::sqrt(3.0);
  o->ndt_tol = 1e-3;
  o->maximum_u_change = 0.05;
  o->timestep_growth_factor = 1.1;
  o->norm = CDM_NORM_MAX;
  o->check_every = 0;
  o->guess = CDM_GUESS_PREV;
  o->mem = CDM_MEM_HOST;
  o->iter_block = 0;
  o->use_graph = 1;
}

void cdm_apt_config_default(cdm_apt_config* c) {
  c->mean = CDM_MEAN_HARMONIC;
  c->precision = CDM_PREC_FP64;
  c->device = 0;
  c->stream = nullptr;
}

int cdm_apt_create(const cdm_mesh_desc* mesh, const cdm_bc* bcs, const cdm_apt_config* cfg, cdm_apt** out) {
  if (!mesh || !bcs || !out) {
    cdm::set_error("NULL argument");
    return CDM_BAD_INPUT;
  }
  *out = nullptr;
  cdm_apt* h = new cdm_apt();
  int rc = h->e.init(1, mesh, bcs, cfg);
  if (rc != CDM_OK) {
    delete h;
    return rc;
  }
  *out = h;
  return CDM_OK;
}

int cdm_apt_destroy(cdm_apt* h) {
  if (h) {
    cudaSetDevice(h->e.device);
    cudaStreamSynchronize(h->e.stream);
    delete h;
  }
  return CDM_OK;
}

int cdm_apt_set_source(cdm_apt* h, const double* S, int mem) {
  if (!h || !S) return CDM_BAD_INPUT;
  return h->e.set_source(0, S, mem);
}

int cdm_apt_step(cdm_apt* h, double* T, const double* rho, double cp, cdm_kappa kappa, double dt,
                 const cdm_step_opts* opts, cdm_stats* stats, double* next_dt) {
  if (!h || !stats || !next_dt) {
    cdm::set_error("NULL argument");
    return CDM_BAD_INPUT;
  }
  double* Ts[1] = {T};
  const double* rs[1] = {rho};
  return h->e.step(Ts, rs, &cp, &kappa, &dt, opts, stats, next_dt);
}

int cdm_apt_advance(cdm_apt* h, double* T, const double* rho, double cp, cdm_kappa kappa, double* t,
                    double t_end, int max_cycles, double* dt, double dt_max, const cdm_step_opts* opts,
                    cdm_stats* last, int* nsteps) {
  if (!h || !T || !rho || !t || !dt || !last || !nsteps) {
    cdm::set_error("NULL argument");
    return CDM_BAD_INPUT;
  }
  Engine& e = h->e;
  cdm_step_opts o;
  cdm_step_opts_default(&o);
  if (opts) o = *opts;
  *nsteps = 0;
  std::memset(last, 0, sizeof(cdm_stats));
  CDM_CK(cudaSetDevice(e.device));
  // host arrays are staged on the device once for the whole loop
  const cdm::ProbState& s = e.ps[0];
  const size_t bytes = (size_t)s.nfull * sizeof(double);
  double* Td = T;
  double* rd = const_cast<double*>(rho);
  const bool host = o.mem != CDM_MEM_DEVICE;
  if (host) {
    CDM_CK(cudaMalloc((void**)&Td, bytes));
    if (cudaMalloc((void**)&rd, bytes) != cudaSuccess) {
      cudaFree(Td);
      cdm::set_error("cdm_apt_advance: allocation failed");
      return CDM_CUDA_ERROR;
    }
    cudaMemcpyAsync(Td, T, bytes, cudaMemcpyHostToDevice, e.stream);
    cudaMemcpyAsync(rd, rho, bytes, cudaMemcpyHostToDevice, e.stream);
    o.mem = CDM_MEM_DEVICE;
  }
  int rc = CDM_OK;
  int iter = 0;
  double ndt = *dt;
  // the drivers' time loop (test/integrated/2d/gaussian/run.jl:192-231)
  while (true) {
    double* Ts[1] = {Td};
    const double* rs[1] = {rd};
    rc = e.step(Ts, rs, &cp, &kappa, dt, &o, last, &ndt);
    if (rc != CDM_OK) break;
    ++*nsteps;
    if (*t >= t_end) break;
    iter += 1;
    *t += *dt;
    if (iter >= max_cycles - 1) break;
    *dt = ndt < dt_max ? ndt : dt_max;
  }
  if (host) {
    cudaError_t ce = cudaMemcpyAsync(T, Td, bytes, cudaMemcpyDeviceToHost, e.stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e.stream);
    cudaFree(Td);
    cudaFree(rd);
    if (ce != cudaSuccess && rc == CDM_OK) {
      cdm::set_error(std::string("cdm_apt_advance: ") + cudaGetErrorString(ce));
      rc = CDM_CUDA_ERROR;
    }
  }
  return rc;
}

int cdm_apt_set_twilight_zone(cdm_apt* h, const cdm_tz_desc* d) {
  if (!h || !d) {
    cdm::set_error("NULL argument");
    return CDM_BAD_INPUT;
  }
  return h->e.set_twilight_zone(0, d);
}

int cdm_batch_set_twilight_zone(cdm_batch* b, int p, const cdm_tz_desc* d) {
  if (!b || !d || p < 0 || p >= (int)b->e.ps.size()) {
    cdm::set_error("bad arguments to cdm_batch_set_twilight_zone");
    return CDM_BAD_INPUT;
  }
  return b->e.set_twilight_zone(p, d);
}

int cdm_apt_set_guess(cdm_apt* h, const double* u0, int mem) {
  if (!h || !u0) return CDM_BAD_INPUT;
  return h->e.set_guess(0, u0, mem);
}

int cdm_apt_set_guess_net(cdm_apt* h, cdm_net* net, double log_jmean) {
  if (!h) return CDM_BAD_INPUT;
  h->e.guess_net = net;
  h->e.log_jmean = log_jmean;
  if (!net && !h->e.keep_hist)
    for (auto& s : h->e.ps) s.has_hist = 0;
  return CDM_OK;
}

int cdm_apt_get_state(cdm_apt* h, double* q, int* last_err_check) {
  if (!h || !q || !last_err_check) return CDM_BAD_INPUT;
  Engine& e = h->e;
  cdm::ProbState& s = e.ps[0];
  CDM_CK(cudaSetDevice(e.device));
  for (int d = 0; d < e.ndim; ++d)
    CDM_CK(cudaMemcpyAsync(q + d * s.nfull, s.q[s.qpar][d], sizeof(double) * s.nfull, cudaMemcpyDeviceToHost,
                           e.stream));
  CDM_CK(cudaStreamSynchronize(e.stream));
  *last_err_check = s.last_err_check;
  return CDM_OK;
}

int cdm_apt_set_state(cdm_apt* h, const double* q, int last_err_check) {
  if (!h || !q) return CDM_BAD_INPUT;
  Engine& e = h->e;
  cdm::ProbState& s = e.ps[0];
  CDM_CK(cudaSetDevice(e.device));
  for (int d = 0; d < e.ndim; ++d)
    CDM_CK(cudaMemcpyAsync(s.q[s.qpar][d], q + d * s.nfull, sizeof(double) * s.nfull, cudaMemcpyHostToDevice,
                           e.stream));
  CDM_CK(cudaStreamSynchronize(e.stream));
  s.last_err_check = last_err_check;
  return CDM_OK;
}

int cdm_apt_get_metric_cache(cdm_apt* h, double* cache) {
  if (!h || !cache) return CDM_BAD_INPUT;
  Engine& e = h->e;
  cdm::ProbState& s = e.ps[0];
  CDM_CK(cudaSetDevice(e.device));
  for (int d = 0; d < e.ndim; ++d)
    CDM_CK(cudaMemcpyAsync(cache + d * s.nfull, s.cache[d], sizeof(double) * s.nfull, cudaMemcpyDeviceToHost,
                           e.stream));
  CDM_CK(cudaStreamSynchronize(e.stream));
  return CDM_OK;
}

int cdm_apt_full_size(const cdm_apt* h, int64_t* nfull, int64_t* ndomain) {
  if (!h) return CDM_BAD_INPUT;
  if (nfull) *nfull = h->e.ps[0].nfull;
  if (ndomain) *ndomain = h->e.ps[0].ndomain;
  return CDM_OK;
}

int cdm_apt_get_profile(const cdm_apt* h, cdm_profile* out) {
  if (!h || !out) return CDM_BAD_INPUT;
  *out = h->e.prof;
  return CDM_OK;
}

int cdm_batch_get_profile(const cdm_batch* b, cdm_profile* out) {
  if (!b || !out) return CDM_BAD_INPUT;
  *out = b->e.prof;
  return CDM_OK;
}

int cdm_batch_create(int nprob, const cdm_mesh_desc* meshes, const cdm_bc* bcs, const cdm_apt_config* cfg,
                     cdm_batch** out) {
  if (!meshes || !bcs || !out || nprob < 1) {
    cdm::set_error("bad arguments to cdm_batch_create");
    return CDM_BAD_INPUT;
  }
  *out = nullptr;
  cdm_batch* b = new cdm_batch();
  int rc = b->e.init(nprob, meshes, bcs, cfg);
  if (rc != CDM_OK) {
    delete b;
    return rc;
  }
  *out = b;
  return CDM_OK;
}

int cdm_batch_destroy(cdm_batch* b) {
  if (b) {
    cudaSetDevice(b->e.device);
    cudaStreamSynchronize(b->e.stream);
    delete b;
  }
  return CDM_OK;
}

int cdm_batch_set_source(cdm_batch* b, int p, const double* S, int mem) {
  if (!b || !S || p < 0 || p >= (int)b->e.ps.size()) return CDM_BAD_INPUT;
  return b->e.set_source(p, S, mem);
}

int cdm_batch_step(cdm_batch* b, double* const* T, const double* const* rho, const double* cp,
                   const cdm_kappa* kappa, const double* dt, const cdm_step_opts* opts, cdm_stats* stats,
                   double* next_dt) {
  if (!b || !T || !rho || !cp || !kappa || !dt || !stats || !next_dt) {
    cdm::set_error("NULL argument");
    return CDM_BAD_INPUT;
  }
  return b->e.step(T, rho, cp, kappa, dt, opts, stats, next_dt);
}

}  // extern "C"
