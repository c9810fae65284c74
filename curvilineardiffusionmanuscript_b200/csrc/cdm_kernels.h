// cdm_kernels.h — host-callable launchers of the device kernels.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace cdm {

struct Problem;
struct Ctrl;

struct TileShape {
  int tx, ty, tz, threads;
  int march;  // 1: 2D row-marching kernel, tx = threads per block (tx-2 owned columns);
              // 2: 3D plane-marching kernel, tx x ty owned cells per k-plane;
              // 3: the 2D row-marching kernel on the wavefront schedule
};

int num_tile_shapes(int ndim);
TileShape tile_shape(int ndim, int variant);

// tz: the problems carry twilight-zone forcing terms (Problem::tz)
cudaError_t launch_march2d_fp64(int variant, int tz, const Problem* probs, const int2* items, int nitems,
                                cudaStream_t s);
// streams of a sweep launch: boundary strips may run on `side`, concurrently
// with the interior strips on `main` (fork/join through the two events)
struct SweepStreams {
  cudaStream_t main;
  cudaStream_t side;
  cudaEvent_t ev_fork, ev_join;
};

// fast 2D kernel: items[0, n_edge) are boundary strips, items[n_edge, n_edge + n_int)
// interior strips claimed by persistent blocks through counters[0..1] (zero between launches)
cudaError_t launch_march2d_fast(int variant, int harmonic, const Problem* probs, const int2* items, int n_edge,
                                int n_int, unsigned int* counters, const SweepStreams& ss);
// strip classification: no ghost column and no ghost row (the FP32 sweep's interior
// kernel), and no ghost row only (the FP64 row-marching kernels' branch-free body)
bool march_tile_interior(int ni, int nj, int tiles_i, int strip_h, int tx, int tile);
bool march_tile_no_ghost_rows(int nj, int tiles_i, int strip_h, int tile);
// the same kernel on the wavefront schedule: up to K pseudo-iterations of every problem
// in one persistent launch of K rounds, each problem's next iteration starting when its
// own strips are done.  items: each problem's strips together from Problem::item0,
// boundary strips with bit 30 of the tile set.  pace = 1 spreads the iterations a
// problem is expected to have left (Ctrl::est_iter) evenly over the rounds; pace = 0
// (or no estimates) puts every problem in every round.  counters[2] is the launch's
// ticket, counters[3] a flag set when a bounded dependency wait ran out (left set; clear
// it before the next step); wave_count holds nprob ints; W holds the launch's jobs
// (written by the launch's prologue, room for cap >= K * nprob jobs).
// tx: threads per block (128 or 64; tx - 2 owned columns)
constexpr int kWaveMaxRounds = 64;
struct WavePlan {
  int* head;                 // [0] jobs, [1] tickets of the launch
  int* tb;                   // cap + 1: first ticket of each job, in ticket order
  int2* pj;                  // cap: (problem, its iteration of the launch) of each job
  unsigned long long* mask;  // nprob: the rounds each problem takes part in
  long long cap;
};
cudaError_t launch_march2d_wave(int tx, int harmonic, const Problem* probs, int nprob, const int2* items,
                                int nitems, int K, int pace, unsigned int* counters, int* wave_count,
                                const WavePlan& W, cudaStream_t s);
// blocks one wavefront launch of tx-thread blocks keeps resident on the current device
int march2d_wave_slots(int tx, int harmonic);
// one block whose thread 0 runs the wavefront's dependency wait on *count (which
// must stay 0) with a limit of limit_s seconds; sets *err when the wait runs out
cudaError_t launch_wave_wait_probe(const int* count, unsigned int* err, double limit_s, cudaStream_t s);
// rcp_nr, rcp_pos and 1/x of every x (3 results per x)
cudaError_t launch_fastmath_probe(const double* x, int n, double* out, cudaStream_t s);
// 3D plane-marching kernel (reciprocal form); items are (problem, column tile + strip),
// items[0, n_edge) tiles touching the (i, j) boundary, then n_int interior tiles
cudaError_t launch_march3d_fast(int harmonic, int tx, int ty, const Problem* probs, const int2* items, int n_edge,
                                int n_int, const SweepStreams& ss);
bool march3d_tile_interior(int ni, int nj, int tiles_i, int tiles_j, int tx, int ty, int tile);

// one fused FP64 pseudo-iteration over all items (problem, tile)
// exact = 1: operation-for-operation reference arithmetic (bit-identical to the
// CPU restatement); exact = 0: reciprocal form (last-bit differences)
// tz = 1 (2D row-marching exact form only): add the twilight-zone forcing
cudaError_t launch_sweep_fp64(int ndim, int variant, int exact, int harmonic, const Problem* probs,
                              const int2* items, int nitems, int n_edge, unsigned int* counters,
                              const SweepStreams& ss, int tz = 0);

// metric cache (mesh_metric_cache.jl:39-250) and the packed divergence
// coefficients derived from the cell-centre metrics and the cache
struct MeshPtrs {
  const double* inv[9];
  const double* edgeJ[3];
  const double* edgehat[3][9];
};
cudaError_t launch_metric_cache(const Problem& P, const MeshPtrs& m, double* cache[3], cudaStream_t s);
cudaError_t launch_coefficients(const Problem& P, const MeshPtrs& m, double* const cache[3], double* coef[9],
                                cudaStream_t s);

// twilight-zone forcing terms of every domain cell for time t (cdm_tz.cuh):
// centroids and forward metrics of the mesh, the step's density and cₚ;
// writes tz::kNumTerms full-size arrays to out (nx*ny apart)
struct TzMesh {
  const double* x;
  const double* y;
  const double* xxi;
  const double* xeta;
  const double* yxi;
  const double* yeta;
  int nnx, nny;
};
cudaError_t launch_tz_terms(const Problem& P, const TzMesh& m, const double* rho, double cp, double t, int no_t,
                            double* out, cudaStream_t s);

// finite-value check of a field on the domain and the first halo layer
// (validity_checks.jl:1-43); writes bit 0 (non-finite) / bit 1 (negative) to *flag
cudaError_t launch_validate(const Problem& P, const double* f, int* flag, cudaStream_t s);

// Dirichlet ghosts beyond the first layer (2D: every halo layer, boundary_operators.jl:143-150)
cudaError_t launch_dirichlet_fill(const Problem& P, double* u, cudaStream_t s);

// enforce_positivity / cutoff! over the full array (PseudoTransientSolver.jl:323-368)
cudaError_t launch_clamp(double* u, int64_t n, int positivity, int cutoff, cudaStream_t s);

// extrapolated start of a step: out = 2·Tⁿ − Tⁿ⁻¹ over the full array
cudaError_t launch_extrapolate(double* out, const double* Tn, const double* Tnm1, int64_t n, cudaStream_t s);

// next_dt reductions (timestep_control.jl:33-73) and the energy balance.
// out[0] = max(u_prev) (NaN-propagating), out[1] = max relative change,
// out[2] = sum rho*cp*T*J (T = u_prev) over the domain, out[3] = same for u,
// out[4] = sum S*J over the domain.  `scratch` holds >= 2*1024 doubles.
cudaError_t launch_step_reductions(const Problem& P, const double* u, const double* cellJ, double tol,
                                   double* scratch, double* out, cudaStream_t s);
// the same reductions for several problems in four launches: job j reduces problem p over
// blocks [b0, b0 + nb) of one grid; plan_step_reductions fills b0 and nb (a lone problem
// gets the single-problem partition, so its results are bit for bit those above) and
// returns the grid size; `scratch` holds >= 4 * that doubles, out[8p ...] as above
struct RedJob {
  int p, b0, nb;
  const double* u;
  const double* J;
};
int plan_step_reductions(RedJob* jobs, int njobs, const int64_t* nfull);
// batched device copies: job j copies src[0, n) to dst[0] and, where not NULL, dst[1]
// and dst[2]; plan_batch_copy fills b0 and nb and returns the grid size
struct CopyJob {
  const double* src;
  double* dst[3];
  int64_t n;
  int b0, nb;
};
int plan_batch_copy(CopyJob* jobs, int njobs);
cudaError_t launch_batch_copy(const CopyJob* jobs, int njobs, int nblocks, cudaStream_t s);
cudaError_t launch_step_reductions_batch(const Problem* probs, const RedJob* jobs, int njobs, int nblocks,
                                         double tol, double* scratch, double* out, cudaStream_t s);

}  // namespace cdm
