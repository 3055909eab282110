// Device-side helpers shared by the kernels of the pbpic B200 step.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace pbd {

constexpr unsigned FULL = 0xffffffffu;
constexpr int NTHREADS = 256;  // threads per block of the particle kernels

// Threads per block of the push: FP32 (mixed) 128, five blocks per SM at 96
// registers (finer passes over a tile than two blocks of 256, 1.4 % faster
// step; 20 warps per SM against 16 at four blocks: 1.6 % faster single-domain
// step, 4.3 % faster batched step, with 84 B spilled); FP64 (plain)
// 128, three blocks per SM at 168 registers (12 warps per SM, against 8 for one
// 256-thread block at the 196 registers the kernel takes uncapped: a 23 % shorter
// step, with 4 bytes spilled).
#ifndef PBPIC_PUSH_THREADS_FP32
#define PBPIC_PUSH_THREADS_FP32 128
#endif
#ifndef PBPIC_PUSH_THREADS_FP64
#define PBPIC_PUSH_THREADS_FP64 128
#endif
template <class T>
struct PushThreads {
  static constexpr int value = sizeof(T) == 4 ? PBPIC_PUSH_THREADS_FP32 : PBPIC_PUSH_THREADS_FP64;
};

// Mixed form: the per-cell gather records hold each field's bilinear
// coefficients over the cell (1) or the cell's 4 nodes (0).
#ifndef PBPIC_CELL_COEF
#define PBPIC_CELL_COEF 1
#endif

// Current components (denjr record of pic2d.f90:65-67).
enum { JX = 0, JY = 1, JZ = 2, RHO = 3 };

// Fixed-point scale of the mixed form's current: a deposit value v becomes
// llrint(v * 2^32) (resolution 2.3e-10, far below the FP32 rounding of the
// terms). Deposit values are charge * cell-fraction * weight or charge *
// (uz/gamma) * weight; a single particle's value is below 1 in magnitude (it
// moves less than a cell per step), so it fits in 33 signed bits, and
// per-node sums of up to 2^30 particles stay below 2^63.
constexpr float FIX_SCALE = 4294967296.0f;  // 2^32
constexpr double FIX_INV = 1.0 / 4294967296.0;

// ---------------------------------------------------------------------------
// Arithmetic with explicit rounding. Every operation of the particle push
// goes through these, so the compiler cannot contract or reorder it: the same
// inputs give the same bits in every kernel that inlines the push. FMA selects
// whether a*b+c is one fused operation (mixed form) or a rounded multiply
// followed by a rounded add, the order the reference's expressions are
// written in (plain form).
// ---------------------------------------------------------------------------
template <class T, bool FMA>
struct M;

template <bool FMA>
struct M<float, FMA> {
  static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
  static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
  static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
  static __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
  static __device__ __forceinline__ float sqrt(float a) { return __fsqrt_rn(a); }
  static __device__ __forceinline__ float mad(float a, float b, float c) {
    return FMA ? __fmaf_rn(a, b, c) : __fadd_rn(__fmul_rn(a, b), c);
  }
  static __device__ __forceinline__ float abs(float a) { return fabsf(a); }
};

template <bool FMA>
struct M<double, FMA> {
  static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
  static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
  static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
  static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
  static __device__ __forceinline__ double sqrt(double a) { return __dsqrt_rn(a); }
  static __device__ __forceinline__ double mad(double a, double b, double c) {
    return FMA ? __fma_rn(a, b, c) : __dadd_rn(__dmul_rn(a, b), c);
  }
  static __device__ __forceinline__ double abs(double a) { return fabs(a); }
};

// ---------------------------------------------------------------------------
// Cell word of a particle: bit 31 = electron (q = -1), bits 16..30 = ix,
// bits 0..15 = iy (0-based cell). Ordering cell words with bit 31 masked is
// the reference's order by grid = my*(ix-1)+iy (pic2d.f90:422, 1303-1329).
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ int cw_ix(uint32_t w) { return (int)((w >> 16) & 0x7fffu); }
__host__ __device__ __forceinline__ int cw_iy(uint32_t w) { return (int)(w & 0xffffu); }
__host__ __device__ __forceinline__ int cw_sp(uint32_t w) { return (int)(w >> 31); }
__host__ __device__ __forceinline__ uint32_t cw_make(int ix, int iy, int sp) {
  return ((uint32_t)sp << 31) | ((uint32_t)ix << 16) | (uint32_t)iy;
}

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Block-wide sum of a double into thread 0 (blockDim.x a multiple of 32, <= 1024).
__device__ __forceinline__ double block_sum(double v, double* sm /* >= 32 */) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v += __shfl_down_sync(FULL, v, d);
  const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane_id() == 0) sm[w] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < nw; ++i) r += sm[i];
  __syncthreads();
  return r;
}

}  // namespace pbd
