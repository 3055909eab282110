// Stable counting sort of particles by cell (countingsort, pic2d.f90:1303-1329).
//
// The reference histograms the cell keys, turns the histogram into
// allocations by an exclusive scan, and scatters each particle to the next
// free slot of its cell in array order, which makes the sort stable. On the
// GPU the same permutation comes from:
//   1. a histogram of the dense cell keys (warp-aggregated atomics) and an
//      exclusive scan -> per-cell counts and offsets (ptlalloc);
//   2. a least-significant-digit radix sort of (key, index) pairs, 8 bits per
//      pass; every pass is a stable multisplit (per-block digit histograms,
//      a device-wide scan in digit-major order, and a scatter that ranks equal
//      digits by warp match + per-warp counters in array order), so the final
//      index order is exactly the stable order by cell;
//   3. a gather of every particle array through that permutation.
#pragma once
#include "device_common.cuh"

namespace pbd {

// --------------------------------------------------------------- scan
constexpr int SCAN_BT = 256, SCAN_IPT = 16, SCAN_TILE = SCAN_BT * SCAN_IPT;

// Exclusive scan of each SCAN_TILE chunk in place; chunk totals to sums[].
__global__ void __launch_bounds__(SCAN_BT) k_scan_local(int32_t* data, int64_t n, int32_t* sums) {
  __shared__ int32_t buf[SCAN_TILE];
  __shared__ int32_t ws[SCAN_BT / 32];
  const int t = threadIdx.x;
  const int64_t base = (int64_t)blockIdx.x * SCAN_TILE;
#pragma unroll
  for (int k = 0; k < SCAN_IPT; ++k) {
    const int64_t i = base + k * SCAN_BT + t;
    buf[k * SCAN_BT + t] = i < n ? data[i] : 0;
  }
  __syncthreads();
  int32_t local = 0;
#pragma unroll
  for (int k = 0; k < SCAN_IPT; ++k) {
    const int32_t x = buf[t * SCAN_IPT + k];
    buf[t * SCAN_IPT + k] = local;
    local += x;
  }
  // block-wide exclusive scan of the per-thread totals
  int32_t inc = local;
  const unsigned lane = lane_id();
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int32_t y = __shfl_up_sync(FULL, inc, d);
    if (lane >= (unsigned)d) inc += y;
  }
  if (lane == 31) ws[t >> 5] = inc;
  __syncthreads();
  if (t < 32) {
    int32_t w = t < SCAN_BT / 32 ? ws[t] : 0;
    int32_t wi = w;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int32_t y = __shfl_up_sync(FULL, wi, d);
      if (lane >= (unsigned)d) wi += y;
    }
    if (t < SCAN_BT / 32) ws[t] = wi - w;
  }
  __syncthreads();
  const int32_t excl = ws[t >> 5] + inc - local;
#pragma unroll
  for (int k = 0; k < SCAN_IPT; ++k) buf[t * SCAN_IPT + k] += excl;
  if (t == SCAN_BT - 1) sums[blockIdx.x] = excl + local;
  __syncthreads();
#pragma unroll
  for (int k = 0; k < SCAN_IPT; ++k) {
    const int64_t i = base + k * SCAN_BT + t;
    if (i < n) data[i] = buf[k * SCAN_BT + t];
  }
}

__global__ void k_scan_add(int32_t* data, int64_t n, const int32_t* sums) {
  const int64_t base = (int64_t)blockIdx.x * SCAN_TILE;
  const int32_t add = sums[blockIdx.x];
  for (int k = threadIdx.x; k < SCAN_TILE; k += blockDim.x) {
    const int64_t i = base + k;
    if (i < n) data[i] += add;
  }
}

// ------------------------------------------------------------ histogram
// keys[i] = dense cell of particle i (ix*my + iy); counts[key] += 1.
__global__ void k_cell_keys(const uint32_t* cell, int64_t n, int my, int32_t* keys, int32_t* counts) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool ok = i < n;
  int key = -1;
  if (ok) {
    const uint32_t w = cell[i];
    key = cw_ix(w) * my + cw_iy(w);
    if (keys) keys[i] = key;
  }
  const unsigned peers = __match_any_sync(FULL, key);
  if (ok && (lane_id() == (unsigned)(__ffs(peers) - 1))) atomicAdd(&counts[key], __popc(peers));
}

// Histogram of caller-provided keys, flagging keys outside [0, ncells).
__global__ void k_key_hist(const int32_t* keys, int64_t n, int32_t ncells, int32_t* counts, int* status) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool ok = i < n;
  int key = -1;
  if (ok) {
    key = keys[i];
    if (key < 0 || key >= ncells) {
      atomicOr(status, 8);
      key = -2;
    }
  }
  const unsigned peers = __match_any_sync(FULL, key);
  if (ok && key >= 0 && (lane_id() == (unsigned)(__ffs(peers) - 1))) atomicAdd(&counts[key], __popc(peers));
}

// ----------------------------------------------------------- radix sort
constexpr int RB = 256, RIPT = 16, RTILE = RB * RIPT, RWARPS = RB / 32;

// Per-block histogram of one 8-bit digit, written digit-major: hist[d * nblocks + b].
__global__ void __launch_bounds__(RB) k_radix_up(const int32_t* keys, int64_t n, int shift,
                                                 int32_t* hist, int nblocks) {
  __shared__ int32_t h[256];
  const int t = threadIdx.x;
  h[t] = 0;
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * RTILE;
#pragma unroll 4
  for (int k = 0; k < RIPT; ++k) {
    const int64_t i = base + k * RB + t;
    const int d = i < n ? ((keys[i] >> shift) & 255) : 256;
    const unsigned peers = __match_any_sync(FULL, d);
    if (d < 256 && lane_id() == (unsigned)(__ffs(peers) - 1)) atomicAdd(&h[d], __popc(peers));
  }
  __syncthreads();
  hist[(int64_t)t * nblocks + blockIdx.x] = h[t];
}

// Stable scatter of one digit. Warp w owns the contiguous index range
// [base + w*32*RIPT, base + (w+1)*32*RIPT), item k of lane l at offset k*32 + l,
// so (warp, item, lane) order is array order.
__global__ void __launch_bounds__(RB) k_radix_down(const int32_t* kin, const int32_t* vin, int64_t n,
                                                   int shift, const int32_t* hist_off, int nblocks,
                                                   int32_t* kout, int32_t* vout) {
  __shared__ int32_t cnt[RWARPS][257];
  const int t = threadIdx.x, w = t >> 5;
  const unsigned lane = lane_id(), lt = lanemask_lt();
  for (int e = t; e < RWARPS * 257; e += RB) (&cnt[0][0])[e] = 0;
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * RTILE + (int64_t)w * 32 * RIPT;
  int32_t key[RIPT], val[RIPT], pos[RIPT];
  int dig[RIPT];
#pragma unroll
  for (int k = 0; k < RIPT; ++k) {
    const int64_t i = base + k * 32 + lane;
    const bool ok = i < n;
    key[k] = ok ? kin[i] : 0;
    val[k] = ok ? (vin ? vin[i] : (int32_t)i) : 0;
    const int d = ok ? ((key[k] >> shift) & 255) : 256;
    const unsigned peers = __match_any_sync(FULL, d);
    const int before = cnt[w][d];
    __syncwarp();
    if ((peers & lt) == 0) cnt[w][d] = before + __popc(peers);
    __syncwarp();
    pos[k] = before + __popc(peers & lt);
    dig[k] = d;
  }
  __syncthreads();
  {
    const int d = t;  // RB == 256: one digit per thread
    int32_t run = hist_off[(int64_t)d * nblocks + blockIdx.x];
#pragma unroll
    for (int ww = 0; ww < RWARPS; ++ww) {
      const int32_t c = cnt[ww][d];
      cnt[ww][d] = run;
      run += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < RIPT; ++k) {
    if (dig[k] < 256) {
      const int32_t p = cnt[w][dig[k]] + pos[k];
      kout[p] = key[k];
      vout[p] = val[k];
    }
  }
}

// ----------------------------------------------------------------- gather
template <class T>
__global__ void k_gather(const int32_t* perm, int64_t n, const uint32_t* ci, const T* dxi, const T* dyi,
                         const T* uxi, const T* uyi, const T* uzi, const int32_t* pidi, uint32_t* co,
                         T* dxo, T* dyo, T* uxo, T* uyo, T* uzo, int32_t* pido) {
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
    const int32_t s = perm[j];
    co[j] = ci[s];
    dxo[j] = dxi[s];
    dyo[j] = dyi[s];
    uxo[j] = uxi[s];
    uyo[j] = uyi[s];
    uzo[j] = uzi[s];
    if (pido) pido[j] = pidi[s];
  }
}

// Tile ranges from cell offsets: tile t starts at cell (t / tpc)*my + (t % tpc)*ty.
__global__ void k_tile_off(const int32_t* off, int ntiles, int tpc, int ty, int my, int32_t n,
                           int32_t* tile_off) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t > ntiles) return;
  if (t == ntiles) {
    tile_off[t] = n;
    return;
  }
  const int ix = t / tpc;
  tile_off[t] = off[(int64_t)ix * my + (int64_t)(t - ix * tpc) * ty];
}

// Equal-count partition of positions (particles not sorted by cell).
__global__ void k_tile_off_uniform(int ntiles, int64_t n, int32_t* tile_off) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t <= ntiles) tile_off[t] = (int32_t)(n * t / ntiles);
}

}  // namespace pbd
