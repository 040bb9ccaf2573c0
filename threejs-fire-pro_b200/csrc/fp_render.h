// Device-side description of one render of a simulation (fp_sim_render): the camera, the
// render settings as the reference's RenderParams uniform holds them (volume-common.wgsl:4-10),
// the render box and the render pools.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "fp_types.h"

#define FP_BLACKBODY_SIZE 512

// Depths a half-resolution pass records (VolumeSlices.ts DEPTH_SLICES).
#define FP_SLICES 8

struct FpRender {
  float ivp[16];  // clip to world, column-major
  int width, height;
  float time;
  float optical[4], light[4], smoke[4], fire[4];
  float sceneLight[3], ambient[3];
  float flameOpacity;
  int shadowSamples, raySteps, filter;
  int lightShift;       // lighting texels per brick side = 1 << lightShift
  const int* boxes;     // the render boxes: lo xyz, hi xyz in bricks (inclusive), six ints each;
                        // boxes never overlap, each lies in one cluster of tiles
  int boxCount;
  float* renderField;   // [slot][4][cells]: smoothed smoke, heat, lifetime, fuel (coarse smoke:
                        // the simulation's fields as they are)
  float* renderSmoke;   // coarse smoke (smokeDiv > 1): [slot][smoke cells], the smoothed density
  float* lighting;      // [slot][4][texels]: glow RGB, sun transmittance
  uint8_t* occupancy;   // [slot]: bit 0 flame glow, bit 1 anything visible, in the block and halo
  const float4* lut;    // blackbody: peak-normalised linear RGB, log2 radiance
  float* image;         // width x height x 4
  const float* depth;   // the scene's depth buffer (width x height, clip z 0..1), or null
  float* slices;        // half resolution: sliceW x sliceH x FP_SLICES x 4, or null (full resolution)
  int sliceW, sliceH;
};

// Launchers (fp_render.cu): the render pools of every active brick in the box, then the march.
void fp_launch_render(const SimParams* dP, const FpRender& R, int sms, cudaStream_t st);
// Scene-light sums (scene-lights.wgsl): 8 floats per anchor added into `sums` (zeroed).
void fp_launch_collect_lights(const SimParams* dP, const FpRender& R, const float* anchors, int count, float* sums,
                              int sms, cudaStream_t st);
// The blackbody table (blackbody.ts:85-97) computed on the host, FP_BLACKBODY_SIZE entries.
void fp_blackbody_table(float* out4);
