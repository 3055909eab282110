// Kernels used only by the batched form (many independent domains stepped
// together): the per-step bookkeeping and the per-domain scan of the cell
// counts. The push, sort and field kernels of a batched step are the batched
// wrappers in kernels_push.cuh, kernels_sort.cuh and kernels_field.cuh.
#pragma once
#include "device_common.cuh"

namespace pbd {

// Per-domain pieces of the bookkeeping.
struct BatchDomain {
  long long* jacc;       // 4 planes of int64 current accumulators
  long long nacc;        // their count (a multiple of 2)
  const int32_t* counts; // [ncells + 1] new-cell counts (last entry 0)
  int32_t* off;          // [ncells + 1] exclusive scan of counts
  int ncounts;           // ncells + 1
};

// Start of a batched step: zero every domain's accumulators (grid row
// blockIdx.y = domain), reset the counters of the persistent push and
// scatter blocks and advance the step index (-1 before the first step).
static __global__ void k_batch_begin(const BatchDomain* d, int* counters, int* step) {
  const BatchDomain a = d[blockIdx.y];
  longlong2* p = reinterpret_cast<longlong2*>(a.jacc);
  const long long n2 = a.nacc >> 1;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n2; k += (long long)gridDim.x * blockDim.x)
    p[k] = make_longlong2(0, 0);
  if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) {
    counters[0] = 0;
    counters[1] = 0;
    *step += 1;
  }
}

// Exclusive scan of every domain's cell counts, one block of SCB threads per
// domain (grid = domains). Chunks of SCB * SCI counts; thread t owns the SCI
// consecutive counts at t * SCI of the chunk.
constexpr int SCB = 1024, SCI = 8;

static __global__ void __launch_bounds__(SCB) k_scan_batched(const BatchDomain* d) {
  __shared__ int32_t wsum[SCB / 32];
  __shared__ int32_t carry_s;
  const BatchDomain a = d[blockIdx.x];
  const unsigned lane = lane_id();
  const int w = threadIdx.x >> 5;
  int32_t carry = 0;
  for (int c0 = 0; c0 < a.ncounts; c0 += SCB * SCI) {
    const int i0 = c0 + (int)threadIdx.x * SCI;
    int32_t v[SCI];
    int32_t s = 0;
#pragma unroll
    for (int k = 0; k < SCI; ++k) {
      v[k] = i0 + k < a.ncounts ? a.counts[i0 + k] : 0;
      s += v[k];
    }
    // inclusive scan of the thread sums: warp, then across warps
    int32_t x = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int32_t y = __shfl_up_sync(FULL, x, o);
      if ((int)lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    if (w == 0) {
      int32_t z = lane < SCB / 32 ? wsum[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int32_t y = __shfl_up_sync(FULL, z, o);
        if ((int)lane >= o) z += y;
      }
      if (lane < SCB / 32) wsum[lane] = z;
    }
    __syncthreads();
    int32_t run = carry + (w > 0 ? wsum[w - 1] : 0) + x - s;
#pragma unroll
    for (int k = 0; k < SCI; ++k) {
      if (i0 + k < a.ncounts) a.off[i0 + k] = run;
      run += v[k];
    }
    if (threadIdx.x == SCB - 1) carry_s = run;
    __syncthreads();
    carry = carry_s;
    __syncthreads();
  }
}

}  // namespace pbd
