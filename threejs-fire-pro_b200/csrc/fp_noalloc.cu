// Ordered compaction of brick ids with no device allocation.
//
// The same ranking the allocation uses to list the computing bricks in ascending id order
// (fp_alloc.cu: per-block counts, one CTA scans them, blocks scatter at their offsets), with
// its block-count scratch in a file-scope device array instead of memory the caller or the
// library allocates. It exists for callers that cannot call cudaMalloc at the point they
// compact: a render or game thread inside its frame budget (cudaMalloc and cudaFree may
// synchronise the device), an embedding host that owns every device byte through its own
// allocator or a fixed memory budget, and code between stream-capture begin and end.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/firepro.h"
#include "fp_error.h"

namespace {

constexpr unsigned RANK_BLOCK = 256;
constexpr unsigned MAX_BLOCKS = FP_COMPACT_MAX_IDS / RANK_BLOCK;

// One count, then one exclusive offset, per block of 256 ids: 64 KB that every GPU loading
// this library holds until the process exits. Every call shares it.
static __device__ __align__(256) uint32_t g_compactScratch[MAX_BLOCKS];

__global__ void __launch_bounds__(RANK_BLOCK) k_compact_count(const uint32_t* __restrict__ flags, uint32_t n,
                                                               uint32_t* __restrict__ scratch) {
  uint32_t i = blockIdx.x * RANK_BLOCK + threadIdx.x;
  int keep = i < n && flags[i] != 0u;
  int count = __syncthreads_count(keep);
  if (threadIdx.x == 0) scratch[blockIdx.x] = (uint32_t)count;
}

// One CTA: counts become exclusive offsets; the total goes to `count`.
__global__ void __launch_bounds__(1024) k_compact_offsets(uint32_t blocks, uint32_t* __restrict__ scratch,
                                                          uint32_t* __restrict__ count) {
  __shared__ uint32_t part[1024];
  __shared__ uint32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (uint32_t base = 0; base < blocks; base += 1024) {
    uint32_t b = base + threadIdx.x;
    uint32_t v = b < blocks ? scratch[b] : 0u;
    part[threadIdx.x] = v;
    __syncthreads();
    for (unsigned off = 1; off < 1024; off <<= 1) {
      uint32_t add = threadIdx.x >= off ? part[threadIdx.x - off] : 0u;
      __syncthreads();
      part[threadIdx.x] += add;
      __syncthreads();
    }
    if (b < blocks) scratch[b] = carry + part[threadIdx.x] - v;
    __syncthreads();
    if (threadIdx.x == 1023) carry += part[1023];
    __syncthreads();
  }
  if (threadIdx.x == 0) *count = carry;
}

__global__ void __launch_bounds__(RANK_BLOCK) k_compact_scatter(const uint32_t* __restrict__ flags, uint32_t n,
                                                                 const uint32_t* __restrict__ scratch,
                                                                 uint32_t* __restrict__ ids) {
  __shared__ uint32_t warpCount[RANK_BLOCK / 32];
  uint32_t i = blockIdx.x * RANK_BLOCK + threadIdx.x;
  bool keep = i < n && flags[i] != 0u;
  uint32_t mask = __ballot_sync(0xffffffffu, keep);
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) warpCount[warp] = __popc(mask);
  __syncthreads();
  uint32_t before = 0;
  for (int w = 0; w < warp; w++) before += warpCount[w];
  if (keep) ids[scratch[blockIdx.x] + before + __popc(mask & ((1u << lane) - 1u))] = i;
}

// The scratch array's device address, found once per device with that device current.
std::mutex g_mutex;
constexpr int MAX_DEVICES = 64;
uint32_t* g_scratchOf[MAX_DEVICES] = {};

}  // namespace

extern "C" int fp_compact_ids_noalloc(const uint32_t* flags, uint32_t n, uint32_t* ids, uint32_t* count,
                                      void* stream) {
  if (n > FP_COMPACT_MAX_IDS)
    return fp_set_error(FP_ELIMIT, "fp_compact_ids_noalloc: n = " + std::to_string(n) + " exceeds FP_COMPACT_MAX_IDS (" +
                                       std::to_string(FP_COMPACT_MAX_IDS) + ").");
  if (!count || (n > 0 && (!flags || !ids)))
    return fp_set_error(FP_EINVAL, "fp_compact_ids_noalloc needs device flags, ids and count.");
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return fp_set_error(FP_EDEVICE, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (device < 0 || device >= MAX_DEVICES) return fp_set_error(FP_EDEVICE, "device ordinal out of range");
  uint32_t* scratch;
  {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratchOf[device]) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_compactScratch);
      if (e != cudaSuccess)
        return fp_set_error(FP_EDEVICE, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      g_scratchOf[device] = static_cast<uint32_t*>(p);
    }
    scratch = g_scratchOf[device];
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  uint32_t blocks = (n + RANK_BLOCK - 1) / RANK_BLOCK;
  if (blocks) k_compact_count<<<blocks, RANK_BLOCK, 0, st>>>(flags, n, scratch);
  k_compact_offsets<<<1, 1024, 0, st>>>(blocks, scratch, count);
  if (blocks) k_compact_scatter<<<blocks, RANK_BLOCK, 0, st>>>(flags, n, scratch, ids);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fp_set_error(FP_EDEVICE, std::string("fp_compact_ids_noalloc: ") + cudaGetErrorString(e));
  return FP_OK;
}
