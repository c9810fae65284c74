/* cdm_net.h — learned initial guess for the APT step (B200, sm_100a).
 *
 * No counterpart in the reference: the reference starts every step's
 * pseudo-time iteration from u = Tⁿ (copy!(solver.u, T),
 * src/pseudo_transient/PseudoTransientSolver.jl:229).  This network predicts
 * the step's solution from the two previous steps, κ(Tⁿ) and the cell
 * Jacobian J; the APT iteration then runs from that guess to the same
 * stopping point as from Tⁿ, so the guess changes the work, not the answer.
 *
 * Network: a 4-level U-Net of 3x3 convolutions with 32 channels, bf16
 * weights and activations, FP32 accumulation on the tensor cores.
 *   inputs (16 channels, 4 used):  log|Tⁿ|, (Tⁿ − Tⁿ⁻¹)/s, ¼·log κ(Tⁿ), log J − log J̄
 *   output (16 channels, 1 used):  y = (Tⁿ⁺¹ − 2Tⁿ + Tⁿ⁻¹)/s
 *   guess:                         u₀ = 2Tⁿ − Tⁿ⁻¹ + s·smooth(y)
 * with s the RMS over the domain of Tⁿ − Tⁿ⁻¹.  Layers (3x3, "same"):
 *   L0a 16→32, L0b 32→32 (skip S0) | 2x2 mean pool | L1 (skip S1) | pool |
 *   L2 (skip S2) | pool | L3 | upsample+S2 | L4 | upsample+S1 | L5 |
 *   upsample+S0 | L6 | L7 32→16 (linear);  ReLU after every layer but L7.
 * Parameter vector (FP32, in this order per layer): W[9][cin][cout], b[cout];
 * tap index = 3·dy + dx for input offset (dx − 1, dy − 1).
 *
 * Domain sizes given to the network must be multiples of 8.  All array
 * pointers are device pointers; full arrays use the layout of cdm_apt.h.
 */
#ifndef CDM_NET_H
#define CDM_NET_H

#include <stdint.h>

#include "cdm_apt.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cdm_net cdm_net;

/* create a network with He-initialised weights (seeded); stream NULL = own stream */
int cdm_net_create(int device, uint64_t seed, void* stream, cdm_net** out);
int cdm_net_destroy(cdm_net* net);
int cdm_net_num_params(const cdm_net* net, int64_t* n);
/* FP32 parameter vector (host memory) */
int cdm_net_get_params(cdm_net* net, float* params);
int cdm_net_set_params(cdm_net* net, const float* params);
/* FP32 gradient of the last cdm_net_backward / cdm_net_train_step (host memory) */
int cdm_net_get_grads(cdm_net* net, float* grads);

/* Forward pass on given input features x (bf16 bits, [B][H][W][16]); writes
 * y (FP32, [B][H][W][16]).  Device pointers. */
int cdm_net_forward(cdm_net* net, const uint16_t* x, int B, int H, int W, float* y);
/* Backward pass of the mean squared error of channel 0 of the last forward's
 * output against target ([B][H][W], FP32): fills the gradient, returns the loss. */
int cdm_net_backward(cdm_net* net, const float* target, float* loss);

/* A training batch: nsamp (≤ 1024) crops of crop x crop domain cells from APT
 * trajectories (three consecutive steps per sample). */
typedef struct {
  int nsamp;
  const double* const* tprev;  /* host array of nsamp device pointers, full arrays */
  const double* const* tcur;
  const double* const* tnext;
  const double* J;             /* device, full array (cell Jacobian)               */
  const int* ox;               /* host arrays: crop origins in domain cells         */
  const int* oy;
  int crop;                    /* multiple of 8                                     */
  int ni, nj, nhalo;           /* domain size and halo of the full arrays           */
  double k0, kn;               /* κ = k0·|T|^kn                                     */
  double log_jmean;            /* log of the mean cell Jacobian of the mesh         */
  double dt;                   /* > 0: weight the loss by 1 + D/16, D = κΔt/(ρcₚJ)  */
  double rho_cp;               /* ρcₚ of that weight (constant over the mesh)       */
} cdm_net_batch;

/* features → forward → loss → backward → Adam (β = 0.9, 0.999, ε = 1e-8) */
int cdm_net_train_step(cdm_net* net, const cdm_net_batch* batch, float lr, float* loss);

/* Passes (default 8) of the 3x3 binomial filter applied to the predicted
 * correction s·y before it is added to 2Tⁿ − Tⁿ⁻¹; 0 turns it off. */
int cdm_net_set_guess_smoothing(cdm_net* net, int passes);

/* guess u0 (full array; halo copied from tcur) for the domain of ni x nj cells */
int cdm_net_predict(cdm_net* net, const double* tprev, const double* tcur, const double* J, int ni, int nj,
                    int nhalo, double k0, double kn, double log_jmean, double* u0);

/* Attach a network to a solver handle (NULL detaches).  Steps run with
 * cdm_step_opts.guess = CDM_GUESS_LEARNED then start from the network's guess
 * once the handle has seen one previous successful step (2D meshes whose
 * sizes are multiples of 8; otherwise from Tⁿ).  Whenever a step starts from a
 * guess (learned or CDM_GUESS_USER), the relative criterion divides by the
 * residual norm that the start u = Tⁿ reaches at its first check (one FP64
 * iteration from Tⁿ computes it), so the step stops at the same absolute
 * residual as the plain start; in 2D the damped flux of a guessed start is
 * set to the plain flux of the guess.  The handle does not own the network. */
int cdm_apt_set_guess_net(cdm_apt* h, cdm_net* net, double log_jmean);

#ifdef __cplusplus
}
#endif

#endif /* CDM_NET_H */
