/*
 * cdm_apt.h — C ABI of the B200 accelerated pseudo-transient (APT) solver.
 *
 * This library is a drop-in for the APT path of CurvilinearDiffusion
 * (smillerc/CurvilinearDiffusionManuscript).  Every entry point below names the
 * reference function it replaces (path:line inside that project).  A Julia
 * `ccall` shim, or any other FFI, binds these symbols directly: the signatures
 * use only plain C types, pointers and sizes.
 *
 * Array layout (identical to `mesh.iterators.cell.full` of the reference):
 *   every cell-centred or face-centred field is a full-size array including
 *   `nhalo` halo layers per side, column-major (i fastest), i.e. element
 *   (i, j, k) of a 3D field lives at  i + nx*(j + ny*k)  with
 *   nx = ni + 2*nhalo, ny = nj + 2*nhalo, nz = nk + 2*nhalo (nz = 1 in 2D).
 *   Domain cell (0,0,0) sits at (nhalo, nhalo, nhalo).  Face arrays store the
 *   value at the i+1/2 (j+1/2, k+1/2) face of the cell with the same index.
 *
 * Errors: every call returns an int status (CDM_OK = 0).  No exception crosses
 * the ABI and nothing traps on the device.  `cdm_apt_last_error` returns a
 * human-readable message for the last failing call on this thread.
 *
 * Threading: a handle is not thread-safe; use one host thread per handle.  Each
 * handle owns a CUDA stream (or uses the one passed in its config).  Calls are
 * synchronous: they return after the device work of the call has finished.
 *
 * Stream order of device arguments: with a stream in the config, the library
 * reads the caller's device arrays in that stream's order, so the caller issues
 * the kernels that produce them there.  With a NULL stream, every call that
 * reads caller device memory first waits for the work already issued to the
 * legacy default stream; work on other streams must be finished by the caller.
 */
#ifndef CDM_APT_H
#define CDM_APT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CDM_APT_ABI_VERSION 1

/* ---- status codes (reference error paths in parentheses) ------------------ */
enum cdm_status {
  CDM_OK = 0,
  CDM_MAX_ITER = 1,   /* PseudoTransientSolver.jl:309-314  iter > max_iter        */
  CDM_NONFINITE = 2,  /* PseudoTransientSolver.jl:302-307  non-finite residual   */
  CDM_BAD_INPUT = 3,  /* validity_checks.jl:1-43 and argument checks              */
  CDM_CUDA_ERROR = 4, /* a CUDA runtime call failed                               */
  CDM_TIMEOUT = 5,    /* a bounded host wait expired                              */
  CDM_NO_DEVICE = 6   /* no usable sm_100 device                                  */
};

/* ---- enums ----------------------------------------------------------------- */
enum cdm_mem { CDM_MEM_HOST = 0, CDM_MEM_DEVICE = 1 };

/* boundary_operators.jl:9-17 */
enum cdm_bc_kind {
  CDM_BC_NEUMANN = 0,      /* ghost <- adjacent interior            (:55-82)   */
  CDM_BC_DIRICHLET = 1,    /* ghost <- value                        (:137-200) */
  CDM_BC_PERIODIC = 2,     /* ghost <- opposite interior, LO sides  (:220-263) */
  CDM_BC_NEG_SYMMETRY = 3  /* ghost <- -adjacent interior           (:157-175) */
};

/* averaging.jl:7-8, selected by the `mean` keyword (PseudoTransientSolver.jl:76-80) */
enum cdm_mean { CDM_MEAN_HARMONIC = 0, CDM_MEAN_ARITHMETIC = 1 };

/* residual norm (residuals.jl:1-22): the reference's GPU and CPU paths differ. */
enum cdm_norm {
  CDM_NORM_MAX = 0, /* GPU path: norm(res, Inf) / sqrt(length(res))   (:5)     */
  CDM_NORM_RMS = 1  /* CPU path: sqrt(sum(res.^2) / length(res))      (:12-22) */
};

enum cdm_precision {
  CDM_PREC_FP64 = 0,       /* plain FP64 APT, divisions in reciprocal form (last-bit
                              differences from the reference's expressions)          */
  CDM_PREC_MIXED = 1,      /* FP32 sweeps + FP64 residual / defect-correction restarts */
  CDM_PREC_FP64_EXACT = 2  /* plain FP64 APT evaluating the reference's expressions
                              operation for operation (bit-identical to the CPU
                              restatement of the reference)                          */
};

enum cdm_guess {
  CDM_GUESS_PREV = 0,   /* u = T^n, as PseudoTransientSolver.jl:229                */
  CDM_GUESS_USER = 1,   /* u = array given by cdm_apt_set_guess                    */
  CDM_GUESS_LEARNED = 2, /* u = T^n + network(T^n, T^{n-1}, kappa, J) (learned guess) */
  CDM_GUESS_EXTRAPOLATE = 3 /* u = 2 T^n - T^{n-1}, the previous call's T^n kept by the
                               handle (the first call starts from T^n); no counterpart in
                               the reference, which starts from T^n (PseudoTransientSolver.jl:229) */
};

/* conductivity model: replaces the Julia closure kappa(rho, T) of the drivers,
 * e.g. test/integrated/2d/gaussian/run.jl:129-135.  kappa = k0*|T|^n, and 0 when
 * T is not finite.  Integer and half-integer n are evaluated by products and
 * one sqrt; other n by pow(). */
typedef struct cdm_kappa {
  double k0;
  double n;
} cdm_kappa;

typedef struct cdm_bc {
  int kind;     /* enum cdm_bc_kind */
  double value; /* Dirichlet value (bc.val.u in 2D, bc.val in 3D)     */
} cdm_bc;

/* Mesh description: the fields of a CurvilinearGrids mesh that the APT path
 * reads (PseudoTransientSolver.jl:57-60,122-153; mesh_metric_cache.jl:51-85;
 * flux_divergence.jl:11-14).  Pointers live in `mem` space and are full-size
 * arrays in the layout above.  Only the first ndim components of each vector
 * are read.  The library copies what it needs; the caller keeps ownership. */
typedef struct cdm_mesh_desc {
  int ndim;           /* 2 or 3 */
  int ni, nj, nk;     /* domain cells per axis (nk ignored in 2D)  */
  int nhalo;          /* >= 1 */
  int mem;            /* enum cdm_mem for every pointer below      */
  /* cell_center_metrics.{xi,eta,zeta}.{x1,x2,x3}: index [3*a + c], a = xi/eta/zeta, c = x1/x2/x3 */
  const double* cell_inv[9];
  /* cell_center_metrics.J (cell area / volume) */
  const double* cell_J;
  /* edge_metrics.{i+1/2, j+1/2, k+1/2}.J and the J-scaled metrics
   * edge_metrics.f.{xi_hat, eta_hat, zeta_hat}.{x1,x2,x3} at index [3*a + c] */
  const double* edge_J[3];
  const double* edge_hat[3][9];
  /* physical dimensions (phys_dims, PseudoTransientSolver.jl:122-153).  When
   * L <= 0 or spacing[0] <= 0 they are computed from the domain node
   * coordinates node_x[0..ndim) ((ni+1) x (nj+1) [x (nk+1)], column-major,
   * host memory) and, in 2D, from cell_J as the reference does. */
  double L;
  double spacing[3];
  const double* node_x[3];
} cdm_mesh_desc;

/* PseudoTransientSolver(mesh, bcs; backend, mean, T)  (PseudoTransientSolver.jl:48-103) */
typedef struct cdm_apt_config {
  int mean;      /* enum cdm_mean, default CDM_MEAN_HARMONIC (:49)      */
  int precision; /* enum cdm_precision, default CDM_PREC_FP64            */
  int device;    /* CUDA device ordinal, default 0                       */
  void* stream;  /* cudaStream_t to use, or NULL for a private stream    */
} cdm_apt_config;

/* Keyword arguments of step! (PseudoTransientSolver.jl:188-202) and of next_dt
 * (timestep_control.jl:33-42), same names and defaults, plus extensions. */
typedef struct cdm_step_opts {
  double t;
  int tz, tz_dim, no_t;          /* tz = 1: add the twilight-zone forcing of
                                    define_forcing_wavy (twilight_zone.jl:54-195) at time t,
                                    time-independent when no_t (tz_dim is unused there, as in
                                    the reference); needs cdm_apt_set_twilight_zone, 2D and an
                                    FP64 precision (CDM_BAD_INPUT otherwise) */
  int max_iter;                  /* 1500 */
  double rtol;                   /* 1e-5 */
  double atol;                   /* sqrt(eps(Float64)) */
  int error_check_interval;      /* 2; accepted and unused, as in the reference */
  int apply_cutoff;              /* 0 */
  int calculate_next_dt;         /* 1 */
  int subcycle_conductivity;     /* 1 */
  int enforce_positivity;        /* 0 */
  double CFL;                    /* 1/sqrt(3) */
  double ndt_tol;                /* next_dt tol = 1e-3 */
  double maximum_u_change;       /* 0.05 */
  double timestep_growth_factor; /* 1.1 */
  /* extensions */
  int norm;        /* enum cdm_norm, default CDM_NORM_MAX                          */
  int check_every; /* 0: reference check schedule (:206-208, :280); k > 0: every k */
  int guess;       /* enum cdm_guess, default CDM_GUESS_PREV                       */
  int mem;         /* enum cdm_mem of the T / rho arrays passed to step            */
  int iter_block;  /* iterations launched between host polls (0 = auto)            */
  int use_graph;   /* capture iteration blocks in CUDA graphs (default 1)          */
} cdm_step_opts;

/* stats NamedTuple of step! (PseudoTransientSolver.jl:349) plus extensions */
typedef struct cdm_stats {
  double rel_err;
  double abs_err;
  int niter;
  int status;
  double time;             /* seconds, host wall clock of the call             */
  double energy_before;    /* sum(rho*cp*T*J) over the domain at t^n           */
  double energy_after;     /* same at t^{n+1}                                  */
  double source_work;      /* dt * sum(S*J) over the domain                    */
  int n_restarts;          /* mixed precision: FP64 defect-correction restarts */
  int n_checks;            /* residual evaluations                             */
} cdm_stats;

typedef struct cdm_apt cdm_apt; /* opaque solver handle */

/* device-time profile of the last step call (no reference counterpart: the
 * reference times stages with TimerOutputs, PseudoTransientSolver.jl:232-339) */
typedef struct cdm_profile {
  double sweep_ms;          /* CUDA-event time of the pseudo-iteration launches     */
  int64_t sweep_launches;   /* fused-sweep kernel launches (including early-exit
                               tails; the 2D boundary and interior kernels of an
                               iteration count separately)                         */
  int64_t other_launches;   /* every other kernel launched by the step              */
  int64_t cell_iters;       /* sum over problems of domain cells x pseudo-iterations */
  int64_t fp32_cell_iters;  /* mixed precision: cells x FP32 correction sweeps      */
  int64_t fp64_cell_evals;  /* mixed precision: cells x FP64 residual restarts      */
} cdm_profile;

/* ---- library ---------------------------------------------------------------- */
int cdm_apt_version(void);
const char* cdm_apt_last_error(void);
/* Diagnostic, no counterpart in the reference: runs the wavefront schedule's
 * bounded dependency wait (the spin of a block waiting for its problem's
 * previous iteration) on device `device` against a counter that nothing
 * raises, with a limit of limit_s seconds (0 < limit_s <= 10).  *expired = 1
 * when the wait gave up and raised the error flag, as the sweep does before
 * the host reports CDM_TIMEOUT; the context stays usable. */
int cdm_selftest_bounded_wait(int device, double limit_s, int* expired);
/* Diagnostic, no counterpart in the reference: the reciprocal ("fast") form's
 * Newton-refined reciprocals beside CUDA's correctly rounded division on device
 * `device`.  For the n host values x (0 < n <= 2^22), out (3n host doubles)
 * receives per value: the general refined reciprocal (0 and inf kept), the
 * refined reciprocal for positive normal arguments, 1/x. */
int cdm_selftest_fastmath(int device, const double* x, int n, double* out);
void cdm_step_opts_default(cdm_step_opts* opts);
void cdm_apt_config_default(cdm_apt_config* cfg);

/* ---- construction: PseudoTransientSolver(mesh, bcs; ...)  (PseudoTransientSolver.jl:48-103)
 * bcs has 2*ndim entries in the order ilo, ihi, jlo, jhi[, klo, khi]; the order
 * is significant exactly as in applybcs! (boundary_operators.jl:26-30).  The
 * metric cache (mesh_metric_cache.jl:2-37) is computed here on the device. */
int cdm_apt_create(const cdm_mesh_desc* mesh, const cdm_bc* bcs, const cdm_apt_config* cfg,
                   cdm_apt** out);
int cdm_apt_destroy(cdm_apt* h);

/* source_term (solver.source_term, PseudoTransientSolver.jl:31); full-size array in `mem` space */
int cdm_apt_set_source(cdm_apt* h, const double* S, int mem);

/* ---- one time step: step!(solver, mesh, T, rho, cp, kappa, dt; kwargs...)
 * (PseudoTransientSolver.jl:180-351), reached through
 * nonlinear_thermal_conduction_step! (nonlinear_thermal_conduction.jl:51-72).
 * T (full size, in/out) and rho (full size) live in opts->mem space.  On
 * return T holds the new temperature including the halo exactly as
 * copy!(T, solver.u) leaves it (:346); *next_dt receives next_dt(...) (:338-344)
 * or dt when calculate_next_dt == 0.  Returns stats->status. */
int cdm_apt_step(cdm_apt* h, double* T, const double* rho, double cp, cdm_kappa kappa, double dt,
                 const cdm_step_opts* opts, cdm_stats* stats, double* next_dt);

/* The drivers' time loop around nonlinear_thermal_conduction_step!
 * (test/integrated/2d/gaussian/run.jl:192-231), in one call: step with *dt;
 * stop if *t >= t_end (tested before t advances, as the drivers do); else
 * *t += *dt, count the cycle, stop at max_cycles - 1 cycles, and continue
 * with *dt = min(next_dt, dt_max).  T (updated in place) and rho are staged on
 * the device once when opts->mem is host.  On return *t and *dt are the
 * loop's time and next time step, *nsteps the steps taken and *last the
 * statistics of the last step; a failing step ends the loop with its status,
 * T holding the last successful step. */
int cdm_apt_advance(cdm_apt* h, double* T, const double* rho, double cp, cdm_kappa kappa, double* t,
                    double t_end, int max_cycles, double* dt, double dt_max, const cdm_step_opts* opts,
                    cdm_stats* last, int* nsteps);

/* ---- twilight zone: the mesh fields define_forcing_wavy reads beyond
 * cdm_mesh_desc (twilight_zone.jl:72-75, :115-118).  Full-size arrays in `mem`
 * space, copied by the call. */
typedef struct cdm_tz_desc {
  int mem;                   /* enum cdm_mem                                      */
  int nnodes[2];             /* mesh.nnodes: domain nodes per axis (ni+1, nj+1)   */
  const double* x;           /* centroid_coordinates.x                            */
  const double* y;           /* centroid_coordinates.y                            */
  const double* x_xi;        /* cell_center_metrics.x₁.ξ  (∂x/∂ξ)                 */
  const double* x_eta;       /* cell_center_metrics.x₁.η                          */
  const double* y_xi;        /* cell_center_metrics.x₂.ξ                          */
  const double* y_eta;       /* cell_center_metrics.x₂.η                          */
} cdm_tz_desc;

/* Inputs of the tz = true path of step! (compute_update!, update.jl:73-119, and
 * update_residual!, residuals.jl:105-160, which call _update_kernel_tz! and
 * _update_resid_kernel_tz!).  Each tz step evaluates the forcing with the
 * iteration's diffusivity, in the reference's operation order; it runs the
 * operation-for-operation FP64 kernel whatever the precision (the reciprocal
 * form has no forcing term), 2D only. */
int cdm_apt_set_twilight_zone(cdm_apt* h, const cdm_tz_desc* tz);

/* initial guess for the next step (CDM_GUESS_USER); full-size array */
int cdm_apt_set_guess(cdm_apt* h, const double* u0, int mem);

/* ---- checkpoint of the state that carries across steps: the damped fluxes q
 * (solver.q, :32) and last_err_check (:45).  `q` holds ndim full-size arrays
 * back to back (host memory). */
int cdm_apt_get_state(cdm_apt* h, double* q, int* last_err_check);
int cdm_apt_set_state(cdm_apt* h, const double* q, int last_err_check);

/* metric cache (mesh_metric_cache.jl:2-37) as computed on the device: ndim
 * full-size arrays back to back (host memory); domain cells only are written. */
int cdm_apt_get_metric_cache(cdm_apt* h, double* cache);

/* grid sizes */
int cdm_apt_full_size(const cdm_apt* h, int64_t* ncells_full, int64_t* ncells_domain);

/* profile of the last cdm_apt_step / cdm_batch_step */
int cdm_apt_get_profile(const cdm_apt* h, cdm_profile* out);

/* ---- batched solve: many independent problems of uneven size, one launch per
 * pseudo-iteration, iteration blocks captured in CUDA graphs.  Each problem is
 * one step!(...) call of the reference; all problems share cp-free options.
 * T[p], rho[p] are full-size arrays in opts->mem space. */
typedef struct cdm_batch cdm_batch;
int cdm_batch_create(int nprob, const cdm_mesh_desc* meshes, const cdm_bc* bcs /* nprob*2*ndim */,
                     const cdm_apt_config* cfg, cdm_batch** out);
int cdm_batch_destroy(cdm_batch* b);
int cdm_batch_set_source(cdm_batch* b, int p, const double* S, int mem);
/* cdm_apt_set_twilight_zone for problem p of a batch */
int cdm_batch_set_twilight_zone(cdm_batch* b, int p, const cdm_tz_desc* tz);
int cdm_batch_step(cdm_batch* b, double* const* T, const double* const* rho, const double* cp,
                   const cdm_kappa* kappa, const double* dt, const cdm_step_opts* opts,
                   cdm_stats* stats /* nprob */, double* next_dt /* nprob */);
/* Autotuner (no counterpart in the reference).  Times one complete step of
 * this batch per candidate — row-marching strip height h ∈ {8, 16, 32, 64} x
 * iteration-block length K ∈ {4, 8, 16} (graph-replayed iterations between
 * host polls), candidate index 3·index(h) + index(K); for 2D FP64 also the
 * tile kernels (32x16 and 32x8 tiles) x K, indices 12..17, and for the
 * reciprocal form the wavefront schedule with 128-thread blocks (variant 4) and
 * with 64-thread blocks (variant 5), each with h ∈ {16, 32, 64} x K ∈ {16, 32, 64},
 * indices 18 + 9·(variant − 4) + 3·index(h) + index(K); for 3D FP64 (reciprocal
 * form) the plane march on 32x8 column tiles (indices 0..11) and on 16x16 column
 * tiles (variant 3, indices 12 + 3·index(h) + index(K)) — from the given inputs
 * (arguments as cdm_batch_step; T is not modified and the solver state is
 * restored after every trial) and keeps the fastest for later steps.  With
 * cache_path not NULL the choice is read from / written to that JSON file,
 * keyed by the batch's sizes, precision and mean.  *chosen = -1 when nothing
 * is tuned (3D tile kernels).  cdm_step_opts.iter_block > 0 still overrides K. */
int cdm_batch_autotune(cdm_batch* b, double* const* T, const double* const* rho, const double* cp,
                       const cdm_kappa* kappa, const double* dt, const cdm_step_opts* opts,
                       const char* cache_path, int* chosen);
/* kernel variant (2D: 0 marching; 1 marching with 64-thread blocks; 2, 3 tile kernels;
 * 4, 5 marching on the wavefront schedule with 128- / 64-thread blocks; 3D: 0, 3 plane
 * march on 32x8 / 16x16 column tiles, 1, 2 tile kernels of the exact form), strip height
 * (0 = built-in heuristic) and iteration-block length in use */
int cdm_batch_tuning(const cdm_batch* b, int* variant, int* strip_h, int* iter_block);
/* apply a tuning without timing (e.g. one found by cdm_batch_autotune on another
 * run): 2D variant 0 (marching, strip_h 0 = heuristic), 1 (the same with 64-thread
 * blocks), 2 or 3 (tile kernels), 4 and 5 (marching on the wavefront schedule with
 * 128- / 64-thread blocks: iter_block pseudo-iterations of every problem in one
 * persistent launch, a problem's next iteration starting as soon as its own strips
 * are done; CDM_PREC_FP64 only); 3D variant 0 (plane march on 32x8 column tiles)
 * or 3 (on 16x16 column tiles, CDM_PREC_FP64 only); the 3D exact form keeps its tile
 * kernels (1, 2); the mixed path takes variant 0 only.
 * iter_block in [1, 64]. */
int cdm_batch_set_tuning(cdm_batch* b, int variant, int strip_h, int iter_block);
int cdm_batch_get_profile(const cdm_batch* b, cdm_profile* out);

/* ---- implicit comparator ------------------------------------------------
 * The reference's implicit scheme: backward Euler in the conservative
 * curvilinear form with the diffusivity taken at Tⁿ, one sparse linear system
 * per time step solved by a Krylov method.  2D (9-point) and 3D (27-point
 * stencil, 19 non-zero entries); Neumann, Dirichlet and periodic sides
 * (FixedNegSymmetryBC has no matrix rows in the reference; CDM_BAD_INPUT).
 * The system covers the domain plus one halo layer; the reference's GMRES +
 * ILU(0) is replaced by Jacobi-preconditioned BiCGSTAB with the same stopping
 * rule on the true residual, ||b - A x||_2 <= atol + rtol ||b - A x0||_2. */
typedef struct cdm_implicit cdm_implicit; /* opaque handle */

/* keyword arguments of nonlinear_thermal_conduction_step!(::ImplicitScheme)
 * (nonlinear_thermal_conduction.jl:4-16), _iterative_solve!
 * (ImplictSolver.jl:249-259) and next_dt (timestep_control.jl:33-42) */
typedef struct cdm_implicit_opts {
  double atol, rtol;             /* 1e-9, 1e-9                                   */
  int max_iter;                  /* Krylov iterations, 0 = 2 x rows (Krylov.jl)  */
  int enforce_positivity;        /* 1: cutoff of the solution                    */
  int apply_density_bc;          /* 1: the boundary rules applied to rho too      */
  double ndt_tol;                /* 1e-3                                          */
  double maximum_u_change;       /* 0.05                                          */
  double timestep_growth_factor; /* 1.1                                           */
  int mem;                       /* enum cdm_mem of T and rho                     */
} cdm_implicit_opts;

void cdm_implicit_opts_default(cdm_implicit_opts* opts);
/* ImplicitScheme(mesh, bcs; mean, backend)  (ImplictSolver.jl:49-160); reads
 * mesh.cell_J, edge_J[f] and edge_hat[f][3a + c] (the J-scaled face metrics)
 * for f, a, c < ndim, cfg->mean and cfg->device (precision is not used) */
int cdm_implicit_create(const cdm_mesh_desc* mesh, const cdm_bc* bcs /* 2 ndim */, const cdm_apt_config* cfg,
                        cdm_implicit** out);
int cdm_implicit_destroy(cdm_implicit* h);
/* scheme.source_term (ImplictSolver.jl:28): a full-size array, the domain and
 * its first halo layer are used */
int cdm_implicit_set_source(cdm_implicit* h, const double* S, int mem);
/* nonlinear_thermal_conduction_step!(scheme, mesh, T, ρ, cₚ, κ, Δt; ...)
 * (nonlinear_thermal_conduction.jl:4-48) with solve! = _iterative_solve!
 * (ImplictSolver.jl:249-330): applybcs! on T (and rho into a library copy:
 * the caller's rho is not modified), α = |κ/(ρcₚ)|, validate_scalar, assemble!,
 * Krylov solve (from zero on the first call, from the previous solution
 * after), cutoff, next_dt; T is overwritten on the domain and its first halo
 * layer.  stats: niter (BiCGSTAB iterations, two products with A each),
 * rel_err = abs_err = the final ||b - A x||_2 (the reference returns the
 * Krylov residual for both), status; the energy fields are 0. */
int cdm_implicit_step(cdm_implicit* h, double* T, const double* rho, double cp, cdm_kappa kappa, double dt,
                      const cdm_implicit_opts* opts, cdm_stats* stats, double* next_dt);
/* the system of the last step (no reference counterpart; for checks): A as 9
 * (2D) or 27 (3D) arrays of rows = (ni+2)(nj+2)[(nk+2)] values, entry
 * e = (di+1) + 3(dj+1) [+ 9(dk+1)] at offset (di, dj[, dk]) (offsets2d /
 * offsets3d, inner_operators.jl:19-49) on interior rows (0 on boundary rows,
 * whose constraint rows are the ones init_matrix.jl builds), and b */
int cdm_implicit_get_system(cdm_implicit* h, double* A, double* b);
/* device time of the last Krylov solve (CUDA events), products with A, rows */
int cdm_implicit_get_profile(const cdm_implicit* h, double* solve_ms, int64_t* spmv, int64_t* rows);

/* ---- allocation-free end-of-step reductions ------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory while they run (a Julia host whose CUDA.jl pool owns the device
 * memory, a service that forbids allocation on its latency path): computes,
 * from device arrays the caller owns, what cdm_apt_step computes after its
 * pseudo-time loop — next_dt and the energy balance — using a fixed scratch
 * array inside the library instead of cudaMalloc.  u_new, u_prev, rho, S
 * (may be NULL) and cell_J are full-size device arrays; out (host) receives
 * {next_dt, energy_before, energy_after, source_work} as in cdm_stats.
 * Limit: at most 134,217,728 cells in the full array (CDM_BAD_INPUT beyond).
 * Every array must be device (or managed) memory of the current device that
 * holds the full array within its allocation, and `stream` (cudaStream_t or
 * NULL) must belong to the current device: anything else is CDM_BAD_INPUT,
 * returned before any launch.  The call is synchronous (it returns the results
 * in host memory), so it cannot be made inside a stream capture at any time;
 * its wait is bounded by CDM_STEP_TIMEOUT_S (CDM_TIMEOUT).  The first call on a
 * device looks up the scratch's device address.  Calls that overlap on the
 * GPU race on the shared scratch. */
int cdm_step_reductions_noalloc(int ndim, int ni, int nj, int nk, int nhalo, const double* u_new,
                                const double* u_prev, const double* rho, const double* S,
                                const double* cell_J, double cp, double dt, double ndt_tol,
                                double maximum_u_change, double timestep_growth_factor, double* out,
                                void* stream);

#ifdef __cplusplus
}
#endif
#endif /* CDM_APT_H */
