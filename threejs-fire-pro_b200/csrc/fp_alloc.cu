// Brick activation and compaction: deterministic slot allocation, the computing-brick list
// in ascending id order, neighbour records and collider bits. Restates
// src/engine/shaders/fluid-allocation.wgsl (buildBricks 129-175, freeBricks 179-195,
// allocateBricks 200-230, linkBricks 234-268, buildSolids 270-341, finishBricks 352-387).
//
// Integer work over brick ids; bound by latency, not bandwidth. Blocks of 256 ids each rank
// their frees and requests; a CTA per simulation scans its block totals; frees push and
// grants pop in brick-id order, so the free stack, pages and entries are bit-identical to
// the oracle. Every kernel covers all simulations of a batch (FpBatch) in one launch.
#include "fp_device.cuh"
#include "fp_launch.h"

namespace {

constexpr int RANK_BLOCK = 256;

// sourceNear (fluid-allocation.wgsl:90-108).
__device__ bool sourceNear(const SimParams& P, int tile, int bx, int by, int bz) {
  float size = (float)P.B * P.h;
  float lo[3] = {(float)bx * size, (float)by * size, (float)bz * size};
  float hi[3] = {((float)bx + 1.f) * size, ((float)by + 1.f) * size, ((float)bz + 1.f) * size};
  uint2 list = tileList(P, tile, 0);
  for (uint32_t i = 0; i < list.y; i++) {
    const FpEmitter& e = P.emitters[P.tileLists[list.x + i]];
    if (e.enabled < 0.5f) continue;
    bool inside = true;
    for (int a = 0; a < 3; a++) {
      // Rounded products and sums, never contracted: an integer decision the oracle repeats.
      float motion = fabsf(e.vel[a]) + fabsf(e.outward);
      // two velocity cells (spacing h d, exact) and a step of motion
      float pad = fminf(size, __fadd_rn(__fmul_rn(2.f, P.h * (float)P.velDiv), __fmul_rn(motion, P.dt)));
      float extent = fmaxf(e.size[a], 0.03f) + pad;
      if (!(e.pos[a] + extent > lo[a] && e.pos[a] - extent < hi[a])) inside = false;
    }
    if (inside) return true;
  }
  return false;
}

// Exclusive block scan of two counters; returns this thread's ranks and the block totals.
__device__ void blockScan2(uint32_t a, uint32_t b, uint32_t& ra, uint32_t& rb, uint32_t& ta, uint32_t& tb) {
  __shared__ uint32_t wa[RANK_BLOCK / 32], wb[RANK_BLOCK / 32];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t ma = __ballot_sync(0xffffffffu, a), mb = __ballot_sync(0xffffffffu, b);
  uint32_t below = (1u << lane) - 1u;
  uint32_t la = __popc(ma & below), lb = __popc(mb & below);
  if (lane == 0) {
    wa[warp] = __popc(ma);
    wb[warp] = __popc(mb);
  }
  __syncthreads();
  uint32_t oa = 0, ob = 0;
  ta = tb = 0;
  for (int w = 0; w < RANK_BLOCK / 32; w++) {
    if (w < warp) {
      oa += wa[w];
      ob += wb[w];
    }
    ta += wa[w];
    tb += wb[w];
  }
  ra = oa + la;
  rb = ob + lb;
  __syncthreads();
}

// Blocks of 256 brick ids of every simulation in the launch, grid-stride; `b` is the block
// within its simulation, `index` this thread's brick id.
__global__ void __launch_bounds__(RANK_BLOCK) k_build_bricks(FpBatch bt) {
  uint32_t blocks = workTotal(bt, FP_WORK_IDBLOCKS);
  for (uint32_t item = blockIdx.x; item < blocks; item += gridDim.x) {
    uint32_t b;
    const SimParams& P = workSim(bt, FP_WORK_IDBLOCKS, item, b);
    uint32_t count = (uint32_t)P.capacity * 64u;
    uint32_t index = b * RANK_BLOCK + threadIdx.x;
    uint32_t s = 0;
    bool keep = false;
    if (index < count) {
      int tile = (int)(index >> 6);
      int4 rec = __ldg(&P.tileRec[tile]);
      if (rec.w != 0) {
        int l = index & 63;
        int bx = rec.x * 4 + (l & 3), by = rec.y * 4 + ((l >> 2) & 3), bz = rec.z * 4 + (l >> 4);
        Home H;
        H.tile = tile;
        H.tx = rec.x;
        H.ty = rec.y;
        H.tz = rec.z;
        bool open = rec.w != 2;
        bool listed = false;
        for (int z = -1; z <= 1 && open && !listed; z++)
          for (int y = -1; y <= 1 && !listed; y++)
            for (int x = -1; x <= 1 && !listed; x++) {
              int nb = brickIdAt(P, H, bx + x, by + y, bz + z);
              if (nb < 0) continue;
              int toward = nbrIndex(-x, -y, -z);
              listed = ((P.activity[nb] >> 3u) & (1u << toward)) != 0u || (P.meshCount > 0 && P.meshTables[nb] >= 0);
            }
        if (open && !listed) listed = sourceNear(P, tile, bx, by, bz);
        int page = P.pages[index];
        bool wasListed = (P.state[index] & 1u) != 0u;
        s = (uint32_t)listed | ((uint32_t)wasListed << 2);
        if (!listed && page >= 0) s |= FP_BRICK_FREES;
        if (listed && page < 0) s |= FP_BRICK_REQUESTS;
        keep = listed && page >= 0;
      }
    }
    uint32_t rf, rr, tf, tr;
    blockScan2((s & FP_BRICK_FREES) != 0u, (s & FP_BRICK_REQUESTS) != 0u, rf, rr, tf, tr);
    uint32_t rk, tk, dummy, td;
    blockScan2(keep, 0u, rk, dummy, tk, td);
    if (threadIdx.x == 0) {
      P.blockCounts[b * 4 + 0] = tf;
      P.blockCounts[b * 4 + 1] = tr;
      P.blockCounts[b * 4 + 2] = tk;
    }
    if (index < count) P.state[index] = s | (rf << 8) | (rr << 16);
  }
}

// A CTA per simulation: exclusive offsets of frees, requests and computing bricks per block,
// and the step's totals (finishBricks' arithmetic, fluid-allocation.wgsl:352-358).
__global__ void __launch_bounds__(1024) k_scan_blocks(FpBatch bt) {
  __shared__ uint32_t sf[1024], sr[1024], sk[1024];
  __shared__ uint32_t carry[3];
  int sims = batchCount(bt);
  for (int sim = blockIdx.x; sim < sims; sim += gridDim.x) {
    const SimParams& P = bt.sims[sim];
    uint32_t count = (uint32_t)P.capacity * 64u;
    int blocks = (int)((count + RANK_BLOCK - 1) / RANK_BLOCK);
    if (threadIdx.x == 0) carry[0] = carry[1] = carry[2] = 0;
    __syncthreads();
    // Pass 1: frees and requests offsets.
    for (int base = 0; base < blocks; base += 1024) {
      int b = base + threadIdx.x;
      uint32_t f = b < blocks ? P.blockCounts[b * 4 + 0] : 0, r = b < blocks ? P.blockCounts[b * 4 + 1] : 0;
      sf[threadIdx.x] = f;
      sr[threadIdx.x] = r;
      __syncthreads();
      for (int off = 1; off < 1024; off <<= 1) {
        uint32_t a = threadIdx.x >= off ? sf[threadIdx.x - off] : 0, c = threadIdx.x >= off ? sr[threadIdx.x - off] : 0;
        __syncthreads();
        sf[threadIdx.x] += a;
        sr[threadIdx.x] += c;
        __syncthreads();
      }
      if (b < blocks) {
        P.blockCounts[b * 4 + 0] = carry[0] + sf[threadIdx.x] - f;  // exclusive
        P.blockCounts[b * 4 + 1] = carry[1] + sr[threadIdx.x] - r;
        P.blockCounts[b * 4 + 3] = r;  // keep the block's request count
      }
      __syncthreads();
      if (threadIdx.x == 1023) {
        carry[0] += sf[1023];
        carry[1] += sr[1023];
      }
      __syncthreads();
    }
    uint32_t frees = carry[0], requests = carry[1];
    int32_t freeCount = P.counters->freeCount;
    int32_t avail = freeCount + (int32_t)frees - P.held;
    uint32_t granted = (uint32_t)min((int32_t)requests, max(avail, 0));
    // Pass 2: computing bricks per block = kept + granted requests of the block.
    for (int base = 0; base < blocks; base += 1024) {
      int b = base + threadIdx.x;
      uint32_t k = 0;
      if (b < blocks) {
        uint32_t roff = P.blockCounts[b * 4 + 1], rcount = P.blockCounts[b * 4 + 3];
        uint32_t g = granted > roff ? min(granted - roff, rcount) : 0u;
        k = P.blockCounts[b * 4 + 2] + g;
      }
      sk[threadIdx.x] = k;
      __syncthreads();
      for (int off = 1; off < 1024; off <<= 1) {
        uint32_t a = threadIdx.x >= off ? sk[threadIdx.x - off] : 0;
        __syncthreads();
        sk[threadIdx.x] += a;
        __syncthreads();
      }
      if (b < blocks) P.blockCounts[b * 4 + 2] = carry[2] + sk[threadIdx.x] - k;
      __syncthreads();
      if (threadIdx.x == 1023) carry[2] += sk[1023];
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      FpCounters* C = P.counters;
      C->frees = frees;
      C->requests = requests;
      C->granted = granted;
      C->active = carry[2];
      C->fresh = granted;
    }
    __syncthreads();
  }
}

// freeBricks: push freed slots in brick order.
__global__ void __launch_bounds__(RANK_BLOCK) k_free_bricks(FpBatch bt) {
  uint32_t blocks = workTotal(bt, FP_WORK_IDBLOCKS);
  for (uint32_t item = blockIdx.x; item < blocks; item += gridDim.x) {
    uint32_t b;
    const SimParams& P = workSim(bt, FP_WORK_IDBLOCKS, item, b);
    uint32_t count = (uint32_t)P.capacity * 64u;
    uint32_t index = b * RANK_BLOCK + threadIdx.x;
    if (index >= count) continue;
    uint32_t s = P.state[index];
    if (!(s & FP_BRICK_FREES)) continue;
    uint32_t rank = P.blockCounts[b * 4 + 0] + ((s >> 8) & 255u);
    P.freeStack[P.counters->freeCount + (int32_t)rank] = (uint32_t)P.pages[index];
    P.pages[index] = -1;
  }
}

// allocateBricks: grants pop from the stack top in brick order; publish entries and the
// ascending list of computing bricks; restart each brick's activity flags.
__global__ void __launch_bounds__(RANK_BLOCK) k_allocate_bricks(FpBatch bt) {
  uint32_t blocks = workTotal(bt, FP_WORK_IDBLOCKS);
  for (uint32_t item = blockIdx.x; item < blocks; item += gridDim.x) {
    uint32_t b;
    const SimParams& P = workSim(bt, FP_WORK_IDBLOCKS, item, b);
    uint32_t count = (uint32_t)P.capacity * 64u;
    uint32_t index = b * RANK_BLOCK + threadIdx.x;
    bool act = false;
    int page = -1;
    bool fresh = false;
    uint32_t s = 0;
    if (index < count) {
      s = P.state[index];
      page = P.pages[index];
      if (s & FP_BRICK_REQUESTS) {
        uint32_t rank = P.blockCounts[b * 4 + 1] + ((s >> 16) & 255u);
        int32_t top = P.counters->freeCount + (int32_t)P.counters->frees - (int32_t)rank;
        if (top > P.held) {
          page = (int)P.freeStack[top - 1];
          P.pages[index] = page;
          P.zeroList[2 * rank] = index;
          P.zeroList[2 * rank + 1] = (uint32_t)page;
          fresh = true;
        }
      }
      act = page >= 0;
    }
    uint32_t ra, rb, ta, tb;
    blockScan2(act, 0u, ra, rb, ta, tb);
    if (index < count) {
      if (act) P.active[P.blockCounts[b * 4 + 2] + ra] = index;
      P.state[index] = (uint32_t)act;
      P.entries[index] = act ? (page | (fresh ? FP_FRESH_ENTRY : 0)) : -1;
      uint32_t flags = P.activity[index];
      P.activity[index] = (flags & FP_EXPANDS) ? FP_MAY_EXPAND : 0u;
    }
    // Tiles hold no content until this step's evolution records it.
    if (index < (uint32_t)P.capacity) P.activity[count + index] = 0u;
  }
}

// linkBricks: each slotted brick's 27 neighbour entries and its pressure-unknown flag.
__global__ void __launch_bounds__(RANK_BLOCK) k_link_bricks(FpBatch bt) {
  uint32_t blocks = workTotal(bt, FP_WORK_IDBLOCKS);
  for (uint32_t item = blockIdx.x; item < blocks; item += gridDim.x) {
    uint32_t b;
    const SimParams& P = workSim(bt, FP_WORK_IDBLOCKS, item, b);
    uint32_t count = (uint32_t)P.capacity * 64u;
    uint32_t index = b * RANK_BLOCK + threadIdx.x;
    if (index >= count || P.entries[index] < 0) continue;
    int tile = (int)(index >> 6);
    int4 rec = __ldg(&P.tileRec[tile]);
    int l = index & 63;
    int bx = rec.x * 4 + (l & 3), by = rec.y * 4 + ((l >> 2) & 3), bz = rec.z * 4 + (l >> 4);
    Home H;
    H.tile = tile;
    H.tx = rec.x;
    H.ty = rec.y;
    H.tz = rec.z;
    int w[27];
    for (int k = 0; k < 27; k++) {
      int nb = brickIdAt(P, H, bx + k % 3 - 1, by + (k / 3) % 3 - 1, bz + k / 9 - 1);
      w[k] = nb >= 0 ? P.entries[nb] : -1;
      P.records[(size_t)index * FP_RECORD_WORDS + k] = w[k];
    }
    int unknowns = 1;
    for (int k = 0; k < 8; k++) {
      int dx = -(k & 1), dy = -((k >> 1) & 1), dz = -((k >> 2) & 1);
      if (P.ground && by + dy < 0) continue;
      if (w[nbrIndex(dx, dy, dz)] < 0) unknowns = 0;
    }
    P.records[(size_t)index * FP_RECORD_WORDS + 27] = unknowns;
  }
}

// finishBricks' commit of each simulation's stack (fluid-allocation.wgsl:354-358), then the
// prefix offsets of the launch's computing bricks and granted slots. One CTA.
__global__ void __launch_bounds__(1024) k_finish_bricks(FpBatch bt) {
  __shared__ uint32_t sa[1024], sg[1024];
  __shared__ uint32_t carry[2];
  int sims = batchCount(bt);
  uint32_t* active = bt.work + 1 + FP_WORK_ACTIVE * bt.stride;
  uint32_t* fresh = bt.work + 1 + FP_WORK_FRESH * bt.stride;
  if (threadIdx.x == 0) carry[0] = carry[1] = 0;
  __syncthreads();
  for (int base = 0; base < sims; base += 1024) {
    int sim = base + threadIdx.x;
    uint32_t a = 0, g = 0;
    if (sim < sims) {
      FpCounters* C = bt.sims[sim].counters;
      int32_t fr = C->freeCount + (int32_t)C->frees;
      C->freeCount = fr - (int32_t)C->granted;
      C->failures += C->requests - C->granted;
      a = C->active;
      g = C->fresh;
    }
    sa[threadIdx.x] = a;
    sg[threadIdx.x] = g;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
      uint32_t x = threadIdx.x >= off ? sa[threadIdx.x - off] : 0, y = threadIdx.x >= off ? sg[threadIdx.x - off] : 0;
      __syncthreads();
      sa[threadIdx.x] += x;
      sg[threadIdx.x] += y;
      __syncthreads();
    }
    if (sim < sims) {
      active[sim] = carry[0] + sa[threadIdx.x] - a;
      fresh[sim] = carry[1] + sg[threadIdx.x] - g;
    }
    __syncthreads();
    if (threadIdx.x == 1023) {
      carry[0] += sa[1023];
      carry[1] += sg[1023];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    active[sims] = carry[0];
    fresh[sims] = carry[1];
  }
}

// insideCollider (fluid-allocation.wgsl:274-290).
__device__ bool insideCollider(const SimParams& P, const FpCollider& c, int x, int y, int z) {
  int kind = (int)c.kind;
  if (kind == 2) {
    int q[3] = {x - c.lo[0], y - c.lo[1], z - c.lo[2]};
    for (int a = 0; a < 3; a++)
      if (q[a] < 0 || q[a] >= c.size[a]) return false;
    uint32_t idx = (uint32_t)((q[2] * c.size[1] + q[1]) * c.size[0] + q[0]);
    return ((P.masks[c.first + (idx >> 5)] >> (idx & 31u)) & 1u) != 0u;
  }
  float w[3] = {((float)x + 0.5f) * P.h, ((float)y + 0.5f) * P.h, ((float)z + 0.5f) * P.h};
  float d[3];
  // Rounded products and sums, never contracted: the bits are compared with the oracle's.
  for (int a = 0; a < 3; a++) {
    float s = __fmul_rn(c.axes[a][0], w[0] - c.center[0]);
    s = __fadd_rn(s, __fmul_rn(c.axes[a][1], w[1] - c.center[1]));
    s = __fadd_rn(s, __fmul_rn(c.axes[a][2], w[2] - c.center[2]));
    d[a] = fabsf(s / c.extent[a]);
  }
  if (kind == 1) return d[0] < 1.f && d[1] < 1.f && d[2] < 1.f;
  float r = __fmul_rn(d[0], d[0]);
  r = __fadd_rn(r, __fmul_rn(d[1], d[1]));
  r = __fadd_rn(r, __fmul_rn(d[2], d[2]));
  return r < 1.f;
}

// buildSolids: a CTA per brick, a warp per word of 32 cells, a lane per cell (the word is the
// warp's ballot). ALL: every slotted brick of the simulations whose colliders changed;
// otherwise the slots granted this step in the simulations that have colliders.
template <bool ALL>
__global__ void __launch_bounds__(128) k_build_solids(FpBatch bt) {
  const int kind = ALL ? FP_WORK_IDS : FP_WORK_FRESH;
  uint32_t total = workTotal(bt, kind);
  for (uint32_t item = blockIdx.x; item < total; item += gridDim.x) {
    uint32_t i;
    const SimParams& P = workSim(bt, kind, item, i);
    if (!P.buildSolids || (P.solidsAll != 0) != ALL) continue;
    uint32_t id;
    int slot;
    if (ALL) {
      id = i;
      slot = entryPage(P.entries[id]);
    } else {
      id = P.zeroList[2 * i];
      slot = (int)P.zeroList[2 * i + 1];
    }
    if (slot < 0) continue;
    int tile = (int)(id >> 6);
    int4 rec = __ldg(&P.tileRec[tile]);
    int l = id & 63;
    int bx = rec.x * 4 + (l & 3), by = rec.y * 4 + ((l >> 2) & 3), bz = rec.z * 4 + (l >> 4);
    uint2 list = tileList(P, tile, 2);
    const int lane = threadIdx.x & 31, warps = blockDim.x >> 5;
    for (int word = threadIdx.x >> 5; word < P.W; word += warps) {
      const int bit = word * 32 + lane;
      const int x = bx * P.B + (bit & (P.B - 1)), y = by * P.B + ((bit >> P.shift) & (P.B - 1)),
                z = bz * P.B + (bit >> (2 * P.shift));
      bool inside = false;
      for (uint32_t j = 0; j < list.y && !inside; j++)
        inside = insideCollider(P, P.colliders[P.tileLists[list.x + j]], x, y, z);
      const uint32_t bits = __ballot_sync(0xffffffffu, inside);
      if (lane == 0) P.solids[(size_t)slot * P.W + word] = bits;
    }
  }
}

// A fresh slot starts as still, empty air (fluid-zeroing.wgsl:75-105). Pools every step
// rewrites before reading need no clearing.
__global__ void __launch_bounds__(256) k_zero_fresh(FpBatch bt) {
  uint32_t total = workTotal(bt, FP_WORK_FRESH);
  for (uint32_t item = blockIdx.x; item < total; item += gridDim.x) {
    uint32_t i;
    const SimParams& P = workSim(bt, FP_WORK_FRESH, item, i);
    size_t slot = P.zeroList[2 * i + 1];
    const int VN = P.vview->N;  // the velocity lattice's cells a slot
    float4* v = reinterpret_cast<float4*>(P.vel + slot * 3 * VN);
    // The scalar pool holds 4 channels of 4 bytes (FP32) or 2 bytes (FP16) a cell.
    const int scalarBytes = P.scalarHalf ? 2 : 4;
    float4* f = reinterpret_cast<float4*>(reinterpret_cast<char*>(P.fld) + slot * 4 * P.N * scalarBytes);
    float4* e = reinterpret_cast<float4*>(P.expn + slot * P.N);
    float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int k = threadIdx.x; k < 3 * VN / 4; k += blockDim.x) v[k] = z;
    for (int k = threadIdx.x; k < P.N * scalarBytes / 4; k += blockDim.x) f[k] = z;
    for (int k = threadIdx.x; k < P.N / 4; k += blockDim.x) e[k] = z;
    // Coarse smoke's state in the scalars' width (zeroSmokeBricks, smoke.wgsl:188-223); a
    // slot's cells are a multiple of 16 bytes (at least 8 cells).
    if (P.smokeDiv > 1) {
      float4* s = reinterpret_cast<float4*>(reinterpret_cast<char*>(P.smk) + slot * P.smokeCells * scalarBytes);
      for (int k = threadIdx.x; k < P.smokeCells * scalarBytes / 16; k += blockDim.x) s[k] = z;
    }
  }
}

// The measurement of each simulation (readActivity, FluidSimulation.ts:1701-1746): its
// counters, the previous step's pressure-solve measurements and a content word per tile slot,
// into host-mapped memory; then failed allocations count afresh and the solve's
// measurements start over. A CTA per simulation.
__global__ void __launch_bounds__(256) k_readback(FpBatch bt) {
  int sims = batchCount(bt);
  const int cw = (int)(sizeof(FpCounters) / 4), sw = (int)(sizeof(FpSolver) / 4);
  for (int sim = blockIdx.x; sim < sims; sim += gridDim.x) {
    const SimParams& P = bt.sims[sim];
    const uint32_t* counters = reinterpret_cast<const uint32_t*>(P.counters);
    const uint32_t* solver = reinterpret_cast<const uint32_t*>(P.solver);
    const uint32_t* tiles = P.activity + (size_t)P.capacity * 64;
    for (int k = threadIdx.x; k < cw + sw; k += blockDim.x) P.readback[k] = k < cw ? counters[k] : solver[k - cw];
    // The tile words, four a store where the host-mapped words allow it (a few transactions over
    // the bus rather than one a word).
    uint32_t* out = P.readback + cw + sw;
    const int n = P.capacity;
    if ((reinterpret_cast<uintptr_t>(out) & 15u) == 0 && (reinterpret_cast<uintptr_t>(tiles) & 15u) == 0) {
      for (int k = threadIdx.x; k < n / 4; k += blockDim.x)
        reinterpret_cast<uint4*>(out)[k] = reinterpret_cast<const uint4*>(tiles)[k];
      for (int k = (n / 4) * 4 + threadIdx.x; k < n; k += blockDim.x) out[k] = tiles[k];
    } else {
      for (int k = threadIdx.x; k < n; k += blockDim.x) out[k] = tiles[k];
    }
    __syncthreads();
    if (threadIdx.x == 0) P.counters->failures = 0;
    uint32_t* clear = reinterpret_cast<uint32_t*>(P.solver);
    for (int k = threadIdx.x; k < sw; k += blockDim.x) clear[k] = 0u;
    __syncthreads();
  }
}

}  // namespace

void fp_launch_allocation(const FpBatch& bt, bool solidsFresh, bool solidsAll, int sms, cudaStream_t st) {
  int grid = sms * 8;
  k_build_bricks<<<grid, RANK_BLOCK, 0, st>>>(bt);
  k_scan_blocks<<<sms, 1024, 0, st>>>(bt);
  k_free_bricks<<<grid, RANK_BLOCK, 0, st>>>(bt);
  k_allocate_bricks<<<grid, RANK_BLOCK, 0, st>>>(bt);
  k_link_bricks<<<grid, RANK_BLOCK, 0, st>>>(bt);
  k_finish_bricks<<<1, 1024, 0, st>>>(bt);
  if (solidsFresh) k_build_solids<false><<<sms * 4, 128, 0, st>>>(bt);
  if (solidsAll) k_build_solids<true><<<sms * 4, 128, 0, st>>>(bt);
  k_zero_fresh<<<sms * 2, 256, 0, st>>>(bt);
}

int fp_allocation_launches(bool solidsFresh, bool solidsAll) { return 7 + (solidsFresh ? 1 : 0) + (solidsAll ? 1 : 0); }

void fp_launch_readback(const FpBatch& bt, int sms, cudaStream_t st) { k_readback<<<sms, 256, 0, st>>>(bt); }
