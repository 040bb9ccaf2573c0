// Launchers of the step's kernels. Every launcher takes the device copy of the simulation's
// SimParams and enqueues on `st`; none synchronises.
#pragma once
#include <cuda_runtime.h>

#include "fp_types.h"

void fp_launch_allocation(const SimParams* dP, int capacity, bool solids, int sms, cudaStream_t st);
void fp_launch_predict(const SimParams* dP, int B, int sms, cudaStream_t st);
void fp_launch_correct(const SimParams* dP, int B, int sms, cudaStream_t st);
void fp_launch_evolve(const SimParams* dP, int B, int sms, cudaStream_t st);
void fp_launch_curl(const SimParams* dP, int sms, cudaStream_t st);
void fp_launch_forces(const SimParams* dP, int B, int sms, cudaStream_t st);
void fp_launch_divergence(const SimParams* dP, float* pOut, int sms, cudaStream_t st);
void fp_launch_project(const SimParams* dP, const float* p, int sms, cudaStream_t st);
void fp_launch_noise(float4* noise, cudaStream_t st);

// Multigrid (pressure.wgsl). Levels below `brickLevels` live in brick slots, the rest in
// tile slots.
void fp_launch_topology(const SimParams* dP, int brickLevels, int bottom, bool all, int capacity, int sms,
                        cudaStream_t st);
void fp_launch_relax(const SimParams* dP, int level, bool tiles, const float* rhs, const float* pin, float* pout,
                     int capacity, int sms, cudaStream_t st);
void fp_launch_restrict(const SimParams* dP, int fine, bool tiles, const float* rhs, const float* p, float* crhs,
                        float* cfirst, int capacity, int sms, cudaStream_t st);
void fp_launch_prolong(const SimParams* dP, int level, bool tiles, const float* pin, const float* coarse, float* pout,
                       int capacity, int sms, cudaStream_t st);
void fp_launch_bottom(const SimParams* dP, int level, int iterations, const float* rhs, const float* pin, float* pout,
                      int capacity, cudaStream_t st);
// Most tile slots the one-CTA bottom solve holds in shared memory.
int fp_bottom_capacity();
// Size the staged brick-level multigrid kernels for bricks of B cells (once per brick size).
void fp_mg_configure(int B);
// Set the step kernels' shared-memory limits (before any launch or stream capture).
void fp_step_configure(int B);
