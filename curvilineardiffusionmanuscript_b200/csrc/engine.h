// engine.h — host-side APT engine shared by the single-problem and batched C ABI.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include "cdm_apt.h"
#include "cdm_net.h"
#include "cdm_device.cuh"
#include "cdm_kernels.h"

namespace cdm {

void set_error(const std::string& msg);

#define CDM_CK(expr)                                                                      \
  do {                                                                                    \
    cudaError_t _e = (expr);                                                              \
    if (_e != cudaSuccess) {                                                              \
      ::cdm::set_error(std::string(#expr) + ": " + cudaGetErrorString(_e));               \
      return CDM_CUDA_ERROR;                                                              \
    }                                                                                     \
  } while (0)

// Host bookkeeping of one problem.
cudaError_t launch_flux_init2d(const Problem& P, const double* u, double* qx, double* qy, cudaStream_t s);

struct ProbState {
  int ndim = 2, ni = 0, nj = 0, nk = 1, nh = 1;
  int64_t nfull = 0, ndomain = 0;
  double L = 0, spacing[3] = {0, 0, 0};
  int rule[6] = {0, 0, 0, 0, 0, 0};
  double val[6] = {0, 0, 0, 0, 0, 0};
  int bc_kind[6] = {0, 0, 0, 0, 0, 0};
  int tiles_i = 1, tiles_j = 1, tiles_k = 1, ntiles = 1, strip_h = 1;
  int item0 = -1;  // wavefront schedule: first strip in the item list (-1: none)
  // device buffers owned by the engine
  double* u[2] = {nullptr, nullptr};
  double* q[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
  double* u_prev = nullptr;
  double* S = nullptr;
  double* rho_buf = nullptr;
  double* coef[9] = {nullptr};
  double* cache[3] = {nullptr, nullptr, nullptr};
  double* cellJ = nullptr;
  double* partial = nullptr;
  double* guess = nullptr;
  // state carried across steps
  int last_err_check = 0;
  int qpar = 0;
  int s_bad = 0;
  int has_guess = 0;
  double* t_hist = nullptr;  // Tⁿ of the previous step (learned guess input)
  int has_hist = 0;
  // mixed precision buffers
  float* d32[2] = {nullptr, nullptr};
  float* e32[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
  float* ub32 = nullptr;
  float* ab32 = nullptr;
  float* R32 = nullptr;
  float* rho32 = nullptr;
  float* coef32[9] = {nullptr};
  double* ub64[2] = {nullptr, nullptr};
  // twilight zone (cdm_apt_set_twilight_zone): centroids and forward metrics
  // (6 full-size arrays back to back), the step's forcing terms, mesh.nnodes
  double* tz_mesh = nullptr;
  double* tz_terms = nullptr;
  int tz_nn[2] = {0, 0};
};

struct Engine {
  int ndim = 2;
  int device = 0;
  int mean = 0;
  int precision = 0;
  cdm_net* guess_net = nullptr;  // attached learned-guess network (not owned)
  double log_jmean = 0.0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int variant = 0;
  int strip_h_override = 0;   // row-marching strip height chosen by the autotuner (0: heuristic)
  int tuned_iter_block = 8;   // iterations per graph block when cdm_step_opts.iter_block is 0
  std::vector<ProbState> ps;
  std::vector<Problem> hp;
  Problem* d_probs = nullptr;
  Ctrl* d_ctrl = nullptr;
  Ctrl* h_ctrl = nullptr;  // pinned mirror
  int2* d_items = nullptr;
  int nitems = 0;
  unsigned int* d_counters = nullptr;  // [0, 1] tile tickets of the persistent sweep; [2] wavefront
                                       // ticket, [3] wavefront wait-expired flag
  int* d_wave = nullptr;               // wavefront schedule: per problem, iterations done in the launch
  WavePlan wave_plan{};                // wavefront schedule: the launch's jobs (device, written per launch)
  int wave_pace = 1;                   // pace problems by their expected iteration counts (CDM_WAVE_PACE=0: off)
  unsigned int* h_wave_err = nullptr;  // pinned mirror of d_counters[3]
  int n_edge = 0;                      // items [0, n_edge) touch a domain boundary
  cudaStream_t side_stream = nullptr;  // boundary strips run here, concurrently
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  SweepStreams sweep_streams() const;
  cudaGraphExec_t mixed_graph = nullptr;  // 16 FP32 correction sweeps
  int* d_flags = nullptr;        // per problem: source validity bits
  double* d_red = nullptr;       // reduction scratch
  double* d_redout = nullptr;    // per problem 8 doubles
  RedJob* d_jobs = nullptr;      // batched end-of-step reductions: one job per problem
  RedJob* h_jobs = nullptr;      // pinned
  double* d_bred = nullptr;      // their partials
  CopyJob* d_cjobs = nullptr;    // batched copies in and out of a step: 2 x nprob jobs
  CopyJob* h_cjobs = nullptr;    // pinned
  double* h_redout = nullptr;    // pinned
  cudaEvent_t ev = nullptr;
  std::map<int, cudaGraphExec_t> graphs;
  std::map<int, cudaGraph_t> graph_defs;
  int graph_variant = -1;
  // profiling of the last step
  std::vector<cudaEvent_t> ev_pool;
  int ev_used = 0;
  cdm_profile prof{};
  int record_pair();           // returns index of a (start) event; end = start + 1
  double collect_profile_ms();

  ~Engine();
  int init(int nprob, const cdm_mesh_desc* meshes, const cdm_bc* bcs, const cdm_apt_config* cfg);
  int build_items();
  int set_source(int p, const double* S, int mem);
  int set_guess(int p, const double* u0, int mem);
  int step(double* const* T, const double* const* rho, const double* cp, const cdm_kappa* kappa,
           const double* dt, const cdm_step_opts* opts, cdm_stats* stats, double* next_dt);
  int run_iterations(const cdm_step_opts* o, int predicted, double t_start, double timeout_s);
  int launch_block(int K, bool use_graph);
  int retile_tail();
  int items_cap = 0;     // capacity of d_items
  bool retiled = false;  // the tail of the last step shortened strips (restored at the next step)
  cudaError_t launch_iters(int K);
  int wait_stream(double timeout_s);
  // Orders a private stream after the work the caller issued to the legacy
  // default stream before this call, so that the caller's device arrays are
  // complete when the library reads them.  A caller-supplied stream orders itself.
  cudaError_t fence_caller();
  cudaEvent_t ev_caller = nullptr;
  int free_graphs();
  // twilight zone: the step in progress adds the forcing (2D, exact row-marching kernel)
  bool tz_active = false;
  bool graph_tz = false;
  int tz_saved_variant = -1;  // tuned variant to restore after a twilight-zone step
  int set_twilight_zone(int p, const cdm_tz_desc* d);
  int begin_tz_step();
  int end_tz_step();
  // mixed precision (apt_mixed.cu)
  int mixed_alloc();
  int step_mixed(const cdm_step_opts* o, double t_start, double timeout_s);
  int learned_guess(int p, const cdm_kappa& kappa);
  int extrapolated_guess(int p);
  bool keep_hist = false;  // a step asked for the extrapolated start: keep Tⁿ for the next one
  int autotune(double* const* T, const double* const* rho, const double* cp, const cdm_kappa* kappa,
               const double* dt, const cdm_step_opts* opts, const char* cache_path, int* chosen);
  int probe_plain_norm(const std::vector<int>& guessed, const std::vector<const double*>& init, double t_start,
                       double timeout_s);
};

int resolve_ghost_rules(int ndim, const cdm_bc* bcs, int* rule, double* val);
double now_seconds();

}  // namespace cdm
