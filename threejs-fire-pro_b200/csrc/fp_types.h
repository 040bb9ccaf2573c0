// Device-visible records of one simulation: the per-step parameters, the packed scene
// and the addresses of every table and pool. The host engine (fp_engine.cpp) fills a
// SimParams per simulation per step and copies it to the device; every kernel reads it.
//
// HBM layout (per simulation)
//   per tile slot      tileRec int4 (x,y,z,state), tileNbr int[27]
//   tile hash          int4 (x,y,z,slot) open addressing, power-of-two size
//   per brick id       pages, entries, state, activity (+ per tile), records int[28]
//   per pool slot      [slot][channel][cell] pools, cells x fastest in a brick:
//                        velocity x4 3ch, curl 4ch, scalars x3 4ch, expn, div 1ch,
//                        scalar bounds 8ch, velocity donors 3 x u16, solids bits
//   multigrid          level 0: p[2] (+ the CG iterate, residual, direction and A direction
//                        with FP_KRYLOV_FCG) and topology per slot; brick levels 1.. per slot;
//                        tile levels per tile slot
#pragma once
#include <stdint.h>

#define FP_MAX_LEVELS 8
#define FP_RECORD_WORDS 28
#define FP_FRESH_ENTRY 0x2000000
#define FP_FRESH_SLOT 0x80000000u

// Activity flags (fluid-content.wgsl:11-13) and brick state bits (fluid-allocation.wgsl:38-41).
#define FP_CONTENT 1u
#define FP_EXPANDS 2u
#define FP_MAY_EXPAND 4u
#define FP_BRICK_FREES 8u
#define FP_BRICK_REQUESTS 16u
#define FP_STORED_SOLID 64u

// Emitter (fluid-common.wgsl:34-40), 80 bytes as the reference packs it.
struct FpEmitter {
  float pos[3];
  float enabled;
  float size[3];
  float box;
  float flame, heat, smoke, response;
  float vel[3];
  float outward;
  float period, strength, fuel, pad;
};

// Collider (fluid-common.wgsl:45-51): kind 0 ellipsoid, 1 box, 2 mesh mask.
struct FpCollider {
  float center[3];
  float kind;
  float extent[4];
  float axes[3][4];  // columns
  int lo[3];
  int first;
  int size[4];
};

// Force rows (force-fields.wgsl:266-272).
struct FpForce {
  float axis[3];
  float strength;
  float center[3];
  float kind;
  float scale, lift, inward, pad0;
  float regionFirst, regionCount, hasMesh, targeted;
  float reserved[4];
};
struct FpRegion {
  float center[3];
  float box;  // 3 box, 1 sphere
  float size[4];
};

// MeshSource (fluid-common.wgsl:53-57): one field cell a mesh source's samples reach.
struct FpMeshSource {
  int cell[4];
  float scalar[4];  // flame lifetime, heat, smoke, fuel rates
  float motion[4];  // velocity x response, response
};

// FlameParams (flame-common.wgsl:2-6) and its ramps.
struct FpFlame {
  float dt, lifespan, smoke, heat;
  float expansion, pad[3];
  int counts[4];
  float knots[3][8][2];
};

// Work counters the allocation writes and every later kernel reads.
struct FpCounters {
  uint32_t active;     // computing bricks this step
  uint32_t fresh;      // slots granted this step
  int32_t freeCount;   // free stack height
  uint32_t failures;   // failed allocations since the last measurement
  uint32_t frees, requests, granted, pad;
};

// The pressure solve's measurements of one step (device). Sums are FP64: the norms decide
// convergence. The post-projection divergence is measured over the same unknowns.
#define FP_MAX_VCYCLES 16
struct FpSolver {
  double rhs2;                  // sum of squares of the right-hand side over the unknowns
  double res2[FP_MAX_VCYCLES];  // sum of squares of the residual after each V-cycle
  double div2, vel2;            // post-projection divergence x h, and face velocity: sums of squares
  double unknowns;              // unknown cells counted
  int cycles;                   // V-cycles run
  int converged;                // the latest norm met the tolerance: later cycles skip
  int measured;                 // the post-projection divergence was measured
  int pad;
  // flexible CG, per V-cycle: z.q (new preconditioned residual against the old A d), d.q, d.s
  double zq[FP_MAX_VCYCLES], dq[FP_MAX_VCYCLES], ds[FP_MAX_VCYCLES];
};

// The bounds-checked build (compiled with FP_BOUNDS): every index a kernel reads out of a table
// (a slot from an entry or a neighbour record, a tile from the directory or its hash, a brick id
// from a list) is checked against its table before use. A bad one is counted, the first one is
// kept (its site, value and limit), and the access is skipped: it reads as "no slot" or "no
// tile", so the kernel goes on and returns normally.
enum FpBoundsSite {
  FP_SITE_RECORD = 1,  // a neighbour record's slot (enterBrick)
  FP_SITE_ENTRY = 2,   // a brick entry's slot (brickSlot beyond the neighbours)
  FP_SITE_TILE_NBR = 3,  // a tile neighbour slot (tileAt)
  FP_SITE_HASH = 4,    // a tile slot from the hash (hashFind)
  FP_SITE_BRICK_ID = 5,  // a brick id from a work list (enterBrick)
  FP_SITE_LEVEL = 6,   // a multigrid cell's owner slot (cellAddress)
};
struct FpBounds {
  unsigned int count;  // violations seen
  int site;            // FpBoundsSite of the first
  long long index;     // the first bad index
  long long limit;     // the size of its table
};

struct SimParams {
  // what this step builds besides the fields (one launch covers many simulations, each
  // skipping the work its own flags leave out)
  int buildSolids;  // collider bits of granted slots, or of every slot with solidsAll
  int topoAll;      // multigrid topology of every slot and tile, not only granted slots
  int curlOn;       // vorticity confinement is on: the curl is computed
  uint32_t* readback;  // host-mapped: the counters, then a content word per tile slot
  // lattice
  int B, shift, N, W;  // cells per brick side, log2, cells per brick, solid words per slot
  int brickLevels, bottom;
  float h, invH, dt;
  // The two lattices of a simulation (velocityDivisor d, FluidSimulation.ts:365-373): the field
  // lattice (scalars, expansion, solids, mesh tables) and the velocity lattice (velocity, curl,
  // divergence, pressure and its levels) of B/d cells a brick side at spacing h d. A simulation
  // has a SimParams per lattice, alike but for the lattice fields above (`brickLevels` and
  // `bottom` are the velocity lattice's in both); `fview` and `vview` point at the two (at
  // itself when d = 1). Velocity kernels run on `vview`, field kernels on `fview`.
  const SimParams* fview;
  const SimParams* vview;
  int velDiv;     // d
  int solidSpan;  // field cells a side per cell of this lattice: d in the velocity view, else 1
  int fshift;     // the field lattice's log2 cells a brick side
  float fineH;    // the field lattice's spacing
  // dynamics (Params, fluid-common.wgsl:21-32)
  float buoyancy, cooling, smokeWeight, damping, dissipation, vorticity;
  float cutoff, time, seedF;
  uint32_t seedBits;
  int lifetimeZero, fuelEnabled;
  float ignition, burnRate;
  int ground, colliderCount, maccormack, solidsAll;
  int held;
  uint32_t slots;
  // directory
  int capacity;  // tile slots; brick ids = capacity * 64
  const int4* tileRec;
  const int* tileNbr;
  uint64_t* tileMask;  // per tile slot, each step: bit l when brick l of the tile computes
  const int* liveTiles;  // the live tile slots, ascending (liveCount of them)
  const int* tileIndex;  // per tile slot: its position in liveTiles, -1 when not live
  int liveCount;
  const int4* hash;
  uint32_t hashMask;
  // per brick id
  int* pages;
  int* entries;
  uint32_t* state;
  uint32_t* activity;
  int* records;
  uint32_t* blockCounts;  // per 256 ids: frees, requests, listedWithPage
  // lists
  uint32_t* active;  // ascending brick ids
  uint32_t* zeroList;  // granted: id, slot
  uint32_t* freeStack;
  FpCounters* counters;
  // pools
  float* vel;   // velocity at the start of the step
  float* velP;  // predictor, then the projected velocity
  float* velC;  // corrected
  float* velF;  // forced
  float* curl;
  float* fld;   // scalars at the start of the step
  float* fldP;  // predictor
  float* fldN;  // evolved
  float* expn;
  float* div;
  float* sb;
  uint16_t* donors;
  // coarse smoke (smoke_divisor d > 1, smoke.wgsl): density on 2^smokeShift cells a brick side
  // (smokeCells a slot) at spacing h d; smk the start of the step and smkN the evolved (the
  // scalars' storage width), smkP the FP32 predictor, smkB its donors' min and max [slot][2][cells]
  int smokeDiv, smokeShift, smokeCells;
  float* smk;
  float* smkP;
  float* smkN;
  float* smkB;
  uint32_t* solids;
  // multigrid
  float* p0[3];  // the finest level's pair, then the CG iterate (null without CG)
  int latest;  // p0 index of the previous solution
  // flexible CG on the finest level (FP_KRYLOV_FCG, null without): the residual rhs + A x, the
  // search direction d and A d
  float* kry[3];
  // storage precision (FP_PRECISION_MIXED): the scalar pools fld/fldP/fldN hold __half, the
  // multigrid levels above 0 (lp, lrhs) __nv_bfloat16; everything else FP32
  int scalarHalf, coarseBf16;
  // pressure solve: up to `vcycles` V-cycles, stopping once the FP64 RMS residual of the
  // finest level is at most `tolerance` x its RMS right-hand side (0: run them all)
  int vcycles;
  float tolerance;
  FpSolver* solver;  // device: this step's norms and state
  FpBounds* bounds;  // device: the bounds-checked build's record (unused otherwise)
  uint8_t* topo[FP_MAX_LEVELS];
  float* lp[FP_MAX_LEVELS][2];
  float* lrhs[FP_MAX_LEVELS];
  // scene
  const FpEmitter* emitters;
  const FpCollider* colliders;
  const uint32_t* masks;
  const FpForce* forces;
  const FpRegion* regions;
  const uint32_t* tileLists;  // 8-word header per tile slot, then indices
  // mesh emission (fluid-sources.wgsl:3-22): per brick id its table (-1 none), then per table
  // a record index per cell (0: none); meshCount records from 1 (0: no mesh emission)
  const int* meshTables;
  const FpMeshSource* meshSources;
  int meshCount;
  // mesh force targets (force-fields.wgsl:13-47): per brick id its first entry (~0u none), then
  // per covered brick a count and per force its index and a bit per velocity cell; null: none
  const uint32_t* forceCoverage;
  FpFlame flame;
  const float4* noise;  // 64^3 curl noise
};

// Work lists of one launch over a batch of simulations. Each list is the concatenation of
// the simulations' own lists; a row of prefix offsets (count + 1 entries) maps an item to its
// simulation. Rows of the host-known lists are written before the launch, the computing
// bricks and granted slots by the allocation on the device.
enum FpWork {
  FP_WORK_IDBLOCKS,  // blocks of 256 brick ids
  FP_WORK_TILES,     // live tile slots (through SimParams::liveTiles)
  FP_WORK_IDS,       // brick ids
  FP_WORK_ACTIVE,    // computing bricks
  FP_WORK_FRESH,     // slots granted this step
  FP_WORK_KINDS
};
struct FpBatch {
  const SimParams* sims;  // one per simulation of the launch
  uint32_t* work;         // work[0] = simulations; row k at work + 1 + k * stride
  int stride;             // most simulations + 1
};
