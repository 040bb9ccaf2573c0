// Launchers of the step's kernels. Every launcher covers all simulations of a batch
// (FpBatch: the device array of their SimParams and the work-list offsets) in one launch of a
// fixed grid, enqueues on `st` and does not synchronise. Fixed grids and per-simulation
// buffers read from SimParams keep a captured CUDA graph valid while the simulations grow.
#pragma once
#include <cuda_runtime.h>

#include "fp_types.h"

void fp_launch_allocation(const FpBatch& bt, bool solidsFresh, bool solidsAll, int sms, cudaStream_t st);
int fp_allocation_launches(bool solidsFresh, bool solidsAll);
// The measurement of every simulation into its host-mapped readback words.
void fp_launch_readback(const FpBatch& bt, int sms, cudaStream_t st);
void fp_launch_predict(const FpBatch& bt, int B, int vd, int sms, cudaStream_t st);
void fp_launch_correct(const FpBatch& bt, int B, int vd, int sms, cudaStream_t st);
void fp_launch_evolve(const FpBatch& bt, int B, int vd, int sms, cudaStream_t st);
// Coarse smoke (smoke_divisor > 1): advection with the donors' range (it reads only the
// start-of-step state), then evolution with source production and content flags (after the
// fine fields' evolution); simulations without coarse smoke skip both. B field cells a brick
// side, vd the velocity divisor, sd the finest smoke divisor among them.
void fp_launch_smoke_advect(const FpBatch& bt, int B, int vd, int sd, int sms, cudaStream_t st);
void fp_launch_smoke_evolve(const FpBatch& bt, int B, int vd, int sd, int sms, cudaStream_t st);
void fp_launch_curl(const FpBatch& bt, int B, int vd, int sms, cudaStream_t st);
void fp_launch_forces(const FpBatch& bt, int B, int vd, int sms, cudaStream_t st);
// Divergence with the finest level's first iterate into p0[pSel]; projection with p0[pSel].
void fp_launch_divergence(const FpBatch& bt, int pSel, int vd, int sms, cudaStream_t st);
void fp_launch_project(const FpBatch& bt, int pSel, int vd, int sms, cudaStream_t st);
void fp_launch_noise(float4* noise, cudaStream_t st);

// Multigrid (pressure.wgsl). Levels below the brick levels live in brick slots, the rest in
// tile slots. Buffers are named by selector, level * 4 + which: which 0 and 1 are the level's
// pressure pair, 2 its right-hand side (the divergence at level 0), 3 at level 0 the CG
// residual; -1 names none (a relaxation's `pin` of -1 starts from zero).
struct MgSel {
  int level;  // output level
  int rhs, pin, coarse, pout, cfirst;
  int cycle;  // V-cycle of the step: from the second on, simulations that converged skip
  // Relaxation: 0 weighted Jacobi (pin -> pout); 1 or 2 red-black Gauss-Seidel in place
  // (pin = pout) of the cells with x + y + z even (1) or odd (2).
  int colour;
};
inline int fp_mg_sel(int level, int which) { return level * 4 + which; }
void fp_launch_topology(const FpBatch& bt, bool anyAll, int sms, cudaStream_t st);
void fp_launch_relax(const FpBatch& bt, const MgSel& S, bool tiles, int B, int sms, cudaStream_t st);
void fp_launch_restrict(const FpBatch& bt, const MgSel& S, bool tiles, int B, int sms, cudaStream_t st);
void fp_launch_prolong(const FpBatch& bt, const MgSel& S, bool tiles, int B, int sms, cudaStream_t st);
// The bottom level's iterations, a CTA per simulation.
void fp_launch_bottom(const FpBatch& bt, const MgSel& S, int iterations, int sms, cudaStream_t st);
// The V-cycle from the second tile level down in one CTA per simulation (k_coarse): S.level is
// that level, S.rhs its right-hand side, S.pin its first iterate, S.pout its result, S.cfirst
// the bottom's result. Usable when every simulation's live tiles fit (fp_coarse_fits).
bool fp_coarse_fits(int liveTiles);
void fp_launch_coarse(const FpBatch& bt, const MgSel& S, int iterations, int sms, cudaStream_t st);
// After V-cycle `cycle`: the FP64 sums of squares of the finest level's residual (and, after
// the first, of its right-hand side) over the unknowns, then each simulation's convergence
// decision. A simulation that converged skips the later cycles.
void fp_launch_residual(const FpBatch& bt, int pSel, int cycle, int sms, cudaStream_t st);
// The red-black bottom: `sweeps` sweeps of the bottom level in place (S.pout), from zero when
// S.pin is -1, a CTA per simulation.
void fp_launch_bottom_rb(const FpBatch& bt, const MgSel& S, int sweeps, int sms, cudaStream_t st);
// Flexible CG on the finest level (FP_KRYLOV_FCG). `begin`: the start x = p0[pSel] into p0[2],
// the residual s = rhs + A x and its and the right-hand side's FP64 norms (V-cycle 0), then
// the convergence decision. `iterate`, after V-cycle `cycle` >= 1 left z = V(s) in p0[zSel]:
// the direction d = z + beta d (A-orthogonal to the previous), q = A d, the step
// x += alpha d, s += alpha q, the residual's norm and the decision.
void fp_launch_fcg_begin(const FpBatch& bt, int pSel, int sms, cudaStream_t st);
void fp_launch_fcg_iterate(const FpBatch& bt, int zSel, int cycle, int sms, cudaStream_t st);
int fp_fcg_iterate_launches(int cycle);
// After the projection: FP64 sums of squares of h x divergence and of the face velocities over
// the interior unknowns.
void fp_launch_post_divergence(const FpBatch& bt, int sms, cudaStream_t st);
// Size the staged brick-level multigrid kernels for bricks of B cells (once per brick size).
void fp_mg_configure(int B);
// Set the step kernels' shared-memory limits (before any launch or stream capture).
void fp_step_configure(int B);
