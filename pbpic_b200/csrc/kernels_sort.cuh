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
#include "kernels_push.cuh"

namespace pbd {

// --------------------------------------------------------------- scan
constexpr int SCAN_BT = 256, SCAN_IPT = 16, SCAN_TILE = SCAN_BT * SCAN_IPT;

// In-place exclusive scan of buf[0, SCAN_TILE) by a block of SCAN_BT threads
// (the values stored, a barrier passed); ws holds SCAN_BT/32 + 1 ints. Returns
// the chunk's total to every thread.
__device__ __forceinline__ int32_t block_scan_excl(int32_t* buf, int32_t* ws) {
  const int t = threadIdx.x;
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
    if (t == SCAN_BT / 32 - 1) ws[SCAN_BT / 32] = wi;
  }
  __syncthreads();
  const int32_t excl = ws[t >> 5] + inc - local;
#pragma unroll
  for (int k = 0; k < SCAN_IPT; ++k) buf[t * SCAN_IPT + k] += excl;
  __syncthreads();
  return ws[SCAN_BT / 32];
}

// Exclusive scan of each SCAN_TILE chunk of in[] into out[] (in may equal
// out); chunk totals to sums[].
static __global__ void __launch_bounds__(SCAN_BT) k_scan_local(const int32_t* in, int32_t* out, int64_t n,
                                                              int32_t* sums) {
  __shared__ int32_t buf[SCAN_TILE];
  __shared__ int32_t ws[SCAN_BT / 32 + 1];
  const int t = threadIdx.x;
  const int64_t base = (int64_t)blockIdx.x * SCAN_TILE;
#pragma unroll
  for (int k = 0; k < SCAN_IPT; ++k) {
    const int64_t i = base + k * SCAN_BT + t;
    buf[k * SCAN_BT + t] = i < n ? in[i] : 0;
  }
  __syncthreads();
  const int32_t total = block_scan_excl(buf, ws);
  if (t == 0) sums[blockIdx.x] = total;
#pragma unroll
  for (int k = 0; k < SCAN_IPT; ++k) {
    const int64_t i = base + k * SCAN_BT + t;
    if (i < n) out[i] = buf[k * SCAN_BT + t];
  }
}

static __global__ void k_scan_add(int32_t* data, int64_t n, const int32_t* sums) {
  const int64_t base = (int64_t)blockIdx.x * SCAN_TILE;
  const int32_t add = sums[blockIdx.x];
  for (int k = threadIdx.x; k < SCAN_TILE; k += blockDim.x) {
    const int64_t i = base + k;
    if (i < n) data[i] += add;
  }
}

// ------------------------------------------------------------ histogram
// keys[i] = dense cell of particle i (ix*my + iy); counts[key] += 1.
static __global__ void k_cell_keys(const uint32_t* cell, int64_t n, int my, int32_t* keys, int32_t* counts) {
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

// Sort of an array in which every cell's particles form one contiguous run
// (concatenated cell-sorted pieces with disjoint cells, e.g. a slab's own
// particles followed by its ghost bands): k_cell_runs counts the run starts
// of each cell and records the position of one, k_runs_ok flags a cell with
// more than one run, and k_run_scatter moves each particle to
// offset(cell) + (its index - the run start), the stable sort's position.
static __global__ void k_cell_runs(const uint32_t* cell, int64_t n, int my, int32_t* nruns, int32_t* runstart) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t w = cell[i];
    const int key = cw_ix(w) * my + cw_iy(w);
    int prev = -1;
    if (i > 0) {
      const uint32_t v = cell[i - 1];
      prev = cw_ix(v) * my + cw_iy(v);
    }
    if (key != prev) {
      atomicAdd(&nruns[key], 1);
      runstart[key] = (int32_t)i;
    }
  }
}

static __global__ void k_runs_ok(const int32_t* nruns, int64_t ncells, int* flag) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < ncells; c += (int64_t)gridDim.x * blockDim.x)
    if (nruns[c] > 1) atomicOr(flag, 1);
}

template <class T>
__global__ void k_run_scatter(int64_t n, int my, const int32_t* off, const int32_t* runstart, const uint32_t* ci,
                              const T* dxi, const T* dyi, const T* uxi, const T* uyi, const T* uzi,
                              const int32_t* pidi, uint32_t* co, T* dxo, T* dyo, T* uxo, T* uyo, T* uzo,
                              int32_t* pido) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t w = ci[i];
    const int key = cw_ix(w) * my + cw_iy(w);
    const int64_t d = (int64_t)off[key] + (i - runstart[key]);
    co[d] = w;
    dxo[d] = dxi[i];
    dyo[d] = dyi[i];
    uxo[d] = uxi[i];
    uyo[d] = uyi[i];
    uzo[d] = uzi[i];
    if (pido) pido[d] = pidi[i];
  }
}

// Histogram of caller-provided keys, flagging keys outside [0, ncells).
static __global__ void k_key_hist(const int32_t* keys, int64_t n, int32_t ncells, int32_t* counts, int* status) {
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
static __global__ void __launch_bounds__(RB) k_radix_up(const int32_t* keys, int64_t n, int shift,
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
static __global__ void __launch_bounds__(RB) k_radix_down(const int32_t* kin, const int32_t* vin, int64_t n,
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
static __global__ void k_tile_off(const int32_t* off, int ntiles, int tpc, int ty, int my, int32_t n,
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
static __global__ void k_tile_off_uniform(int ntiles, int64_t n, int32_t* tile_off) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t <= ntiles) tile_off[t] = (int32_t)(n * t / ntiles);
}

}  // namespace pbd

namespace pbd {

// ------------------------------------------------------- fused counting sort
// When the particles were sorted by cell before the push, a particle of tile T
// (a run of cells of one column) lands in T's window: the cells adjacent to T.
// The push counts the new cells per (tile, window bin); with those counts the
// stable counting sort needs no radix passes:
//   count(cell) = sum over the tiles whose window holds the cell,
//   slot(particle) = offset(cell) + [particles of earlier tiles in the cell]
//                  + [earlier particles of its own tile in the cell],
// where "earlier" is array order, i.e. tile order then position in the tile.

// Tiles whose window contains cell (cx, cy): the owners of its 3x3 neighbours.
__device__ __forceinline__ int tiles_of_cell(int cx, int cy, int mx, int my, int ybc, int ty, int tpc, int* tl) {
  int n = 0;
#pragma unroll
  for (int a = -1; a <= 1; ++a) {
    int x = cx + a;
    x = x < 0 ? x + mx : (x >= mx ? x - mx : x);
#pragma unroll
    for (int b = -1; b <= 1; ++b) {
      int y = cy + b;
      if (ybc == 0) {
        y = y < 0 ? y + my : (y >= my ? y - my : y);
      } else if (y < 0 || y >= my) {
        continue;
      }
      const int tt = x * tpc + y / ty;
      bool dup = false;
      for (int k = 0; k < n; ++k) dup |= tl[k] == tt;
      if (!dup) tl[n++] = tt;
    }
  }
  return n;
}

__device__ __forceinline__ int bin_in_tile(int cx, int cy, int tt, int mx, int my, int ybc, int ty, int tpc) {
  const int ixt = tt / tpc, y0 = (tt - ixt * tpc) * ty, y1 = min(y0 + ty, my);
  return window_bin(cx, cy, ixt, y0, y1, ty, mx, my, ybc);
}

struct FusedSortParams {
  int mx, my, ybc, ty, tpc, ntiles, nb;
  const int32_t* tilecnt;  // [ntiles][nb] from the push
  int32_t* counts;         // [mx*my + 1] per-cell counts (last entry 0)
  int32_t* off;            // exclusive scan of counts
  int32_t* base;           // [ntiles][nb] first slot of each (tile, bin)
};

// A cell whose 3x3 neighbours need no wrap or wall: the tiles whose windows hold it are the
// tile rows (cy-1)/ty .. (cy+1)/ty of columns cx-1, cx, cx+1, and its bin in the tile of column
// cx+dx and tile row tr is (1-dx, cy - tr*ty + 1) -- the same tiles and bins tiles_of_cell and
// bin_in_tile find, in tile order (column, then row).
__device__ __forceinline__ bool interior_cell(int cx, int cy, int mx, int my) {
  return cx >= 1 && cx <= mx - 2 && cy >= 1 && cy <= my - 2;
}
__device__ __forceinline__ int64_t interior_bin_index(const FusedSortParams& a, int cx, int cy, int dx, int tr) {
  return ((int64_t)(cx + dx) * a.tpc + tr) * a.nb + (1 - dx) * (a.ty + 2) + (cy - tr * a.ty + 1);
}

__device__ __forceinline__ void fused_counts_body(const FusedSortParams& a) {
  const int64_t ncells = (int64_t)a.mx * a.my;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c <= ncells; c += (int64_t)gridDim.x * blockDim.x) {
    if (c == ncells) {
      a.counts[c] = 0;
      continue;
    }
    const int cx = (int)(c / a.my), cy = (int)(c - (int64_t)cx * a.my);
    int32_t s = 0;
    if (interior_cell(cx, cy, a.mx, a.my)) {
      const int tlo = (cy - 1) / a.ty, thi = (cy + 1) / a.ty;
      for (int dx = -1; dx <= 1; ++dx)
        for (int tr = tlo; tr <= thi; ++tr) s += a.tilecnt[interior_bin_index(a, cx, cy, dx, tr)];
    } else {
      int tl[9];
      const int n = tiles_of_cell(cx, cy, a.mx, a.my, a.ybc, a.ty, a.tpc, tl);
      for (int k = 0; k < n; ++k) {
        const int b = bin_in_tile(cx, cy, tl[k], a.mx, a.my, a.ybc, a.ty, a.tpc);
        if (b >= 0) s += a.tilecnt[(int64_t)tl[k] * a.nb + b];
      }
    }
    a.counts[c] = s;
  }
}

__device__ __forceinline__ void fused_base_body(const FusedSortParams& a) {
  const int64_t n = (int64_t)a.ntiles * a.nb;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int tt = (int)(e / a.nb), b = (int)(e - (int64_t)tt * a.nb);
    int32_t base = 0;
    if (a.tilecnt[e] > 0) {
      const int ixt = tt / a.tpc, y0 = (tt - ixt * a.tpc) * a.ty;
      const int bx = b / (a.ty + 2), by = b - bx * (a.ty + 2);
      int cx = ixt - 1 + bx;
      cx = cx < 0 ? cx + a.mx : (cx >= a.mx ? cx - a.mx : cx);
      int cy = y0 - 1 + by;
      if (a.ybc == 0) cy = cy < 0 ? cy + a.my : (cy >= a.my ? cy - a.my : cy);
      const int64_t c = (int64_t)cx * a.my + cy;
      base = a.off[c];
      int tl[9];
      const int nt = tiles_of_cell(cx, cy, a.mx, a.my, a.ybc, a.ty, a.tpc, tl);
      for (int k = 0; k < nt; ++k) {
        if (tl[k] >= tt) continue;
        const int b2 = bin_in_tile(cx, cy, tl[k], a.mx, a.my, a.ybc, a.ty, a.tpc);
        if (b2 >= 0) base += a.tilecnt[(int64_t)tl[k] * a.nb + b2];
      }
    }
    a.base[e] = base;
  }
}

static __global__ void k_fused_counts(FusedSortParams a) { fused_counts_body(a); }

// After the chunk scan of the counts (k_scan_local) and the scan of the chunk
// totals, one thread per cell: the cell's offset (its chunk's prefix added)
// and the first slot of each (tile, bin) that holds the cell (the offset plus
// the cell's particles in earlier tiles, as fused_base_body).
static __global__ void k_fused_offsets(FusedSortParams a, const int32_t* sums) {
  const int64_t ncells = (int64_t)a.mx * a.my;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c <= ncells; c += (int64_t)gridDim.x * blockDim.x) {
    const int32_t o = a.off[c] + sums[c / SCAN_TILE];
    a.off[c] = o;
    if (c == ncells) continue;
    const int cx = (int)(c / a.my), cy = (int)(c - (int64_t)cx * a.my);
    if (interior_cell(cx, cy, a.mx, a.my)) {  // the (tile, bin) entries in tile order: a running sum
      const int tlo = (cy - 1) / a.ty, thi = (cy + 1) / a.ty;
      int32_t before = o;
      for (int dx = -1; dx <= 1; ++dx)
        for (int tr = tlo; tr <= thi; ++tr) {
          const int64_t e = interior_bin_index(a, cx, cy, dx, tr);
          a.base[e] = before;
          before += a.tilecnt[e];
        }
      continue;
    }
    int tl[9], bl[9], cl[9];
    const int nt = tiles_of_cell(cx, cy, a.mx, a.my, a.ybc, a.ty, a.tpc, tl);
    for (int k = 0; k < nt; ++k) {
      bl[k] = bin_in_tile(cx, cy, tl[k], a.mx, a.my, a.ybc, a.ty, a.tpc);
      cl[k] = bl[k] >= 0 ? a.tilecnt[(int64_t)tl[k] * a.nb + bl[k]] : 0;
    }
    for (int k = 0; k < nt; ++k) {
      if (bl[k] < 0) continue;
      int32_t before = o;
      for (int j = 0; j < nt; ++j)
        if (tl[j] < tl[k]) before += cl[j];
      a.base[(int64_t)tl[k] * a.nb + bl[k]] = before;
    }
  }
}

static __global__ void k_fused_counts_batched(const FusedSortParams* d) {
  __shared__ FusedSortParams a;
  if (threadIdx.x == 0) a = d[blockIdx.y];
  __syncthreads();
  fused_counts_body(a);
}

static __global__ void k_fused_base_batched(const FusedSortParams* d) {
  __shared__ FusedSortParams a;
  if (threadIdx.x == 0) a = d[blockIdx.y];
  __syncthreads();
  fused_base_body(a);
}

template <class T>
struct ScatterParams {
  int mx, my, ybc, ty, tpc, nb;
  const int32_t* tile_off;  // position ranges of the tiles (those the push used)
  const int32_t* base;      // [ntiles][nb]
  const uint32_t* ci;       // the pushed particles' cell words
  int32_t* perm;            // sorted slot -> element of ci
};

constexpr int SC_MAXNB = 3 * (64 + 2) + 1;  // window bins of the largest tile, plus a sentinel

// Per-warp bin counts and the block's running ranks of one tile.
struct ScatterSmem {
  int32_t cnt[8][SC_MAXNB];
  int32_t run[SC_MAXNB], sbase[SC_MAXNB];
};

// ------------------------------------------------- permutation-only sort
// The stable ranking of a tile's particles by new cell (warp match_any +
// per-warp counters, array order), from the cell words only: the
// particle at array element p of the tile gets its sorted slot d, and
// perm[d] = p. The particle data stay where they are; the next push reads
// them through perm (PushParams::src), and a gather (k_gather) applies perm
// when the arrays themselves must be in cell order.
#ifndef PBPIC_PERM_IPT
#define PBPIC_PERM_IPT 8  // particles per thread in one chunk of the ranking
#endif
constexpr int SP_IPT = PBPIC_PERM_IPT, SP_CHUNK = 256 * SP_IPT;

template <class T>
__device__ __forceinline__ void perm_tile(const ScatterParams<T>& a, const int t, ScatterSmem& sm) {
  int32_t(&cnt)[8][SC_MAXNB] = sm.cnt;
  int32_t* perm = a.perm;
  const int ixt = t / a.tpc, y0 = (t - ixt * a.tpc) * a.ty, y1 = min(y0 + a.ty, a.my);
  const int pbeg = a.tile_off[t], pend = a.tile_off[t + 1];
  const int w = threadIdx.x >> 5;
  const unsigned lane = lane_id(), lt = lanemask_lt();
  // the window wraps only for the first and last columns and, with periodic y, the first and last tile rows
  const bool edge = ixt == 0 || ixt == a.mx - 1 || (a.ybc == 0 && (y0 == 0 || y1 == a.my));
  const int nrow = y1 - y0 + 1;  // window rows 0..nrow
  for (int b = threadIdx.x; b < a.nb; b += blockDim.x) {
    sm.run[b] = 0;
    sm.sbase[b] = a.base[(int64_t)t * a.nb + b];
  }
  for (int c0 = pbeg; c0 < pend; c0 += SP_CHUNK) {
    for (int e = threadIdx.x; e < 8 * SC_MAXNB; e += blockDim.x) (&cnt[0][0])[e] = 0;
    __syncthreads();
    int bin[SP_IPT], pos[SP_IPT];
    uint32_t vc[SP_IPT];
    if (c0 + SP_CHUNK <= pend && !edge) {
      // a whole chunk of a tile whose window does not wrap: each bin straight from the cell steps
#pragma unroll
      for (int k = 0; k < SP_IPT; ++k) vc[k] = a.ci[c0 + w * (32 * SP_IPT) + k * 32 + (int)lane];
#pragma unroll
      for (int k = 0; k < SP_IPT; ++k) {
        const int bx = (int)cw_ix(vc[k]) - ixt + 1, by = (int)cw_iy(vc[k]) - y0 + 1;
        bin[k] = ((unsigned)bx <= 2u && (unsigned)by <= (unsigned)nrow) ? bx * (a.ty + 2) + by : a.nb;
      }
    } else {
#pragma unroll
      for (int k = 0; k < SP_IPT; ++k) {  // every load of the chunk before the ranking
        const int p = c0 + w * (32 * SP_IPT) + k * 32 + (int)lane;
        vc[k] = p < pend ? a.ci[p] : 0u;
      }
#pragma unroll
      for (int k = 0; k < SP_IPT; ++k) {
        const int p = c0 + w * (32 * SP_IPT) + k * 32 + (int)lane;
        int b = a.nb;  // sentinel: beyond the tile
        if (p < pend) {
          b = window_bin(cw_ix(vc[k]), cw_iy(vc[k]), ixt, y0, y1, a.ty, a.mx, a.my, a.ybc);
          if (b < 0) b = a.nb;  // cannot happen: the push kept every particle in its window
        }
        bin[k] = b;
      }
    }
#pragma unroll
    for (int k = 0; k < SP_IPT; ++k) {
      const int b = bin[k];
      const unsigned peers = __match_any_sync(FULL, b);
      const int before = cnt[w][b];
      __syncwarp();
      if ((peers & lt) == 0) cnt[w][b] = before + __popc(peers);
      __syncwarp();
      pos[k] = before + __popc(peers & lt);
    }
    __syncthreads();
    for (int b = threadIdx.x; b < a.nb; b += blockDim.x) {
      int32_t r = sm.run[b];
#pragma unroll
      for (int ww = 0; ww < 8; ++ww) {
        const int32_t c = cnt[ww][b];
        cnt[ww][b] = r;
        r += c;
      }
      sm.run[b] = r;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < SP_IPT; ++k) {
      if (bin[k] < a.nb) {
        const int p = c0 + w * (32 * SP_IPT) + k * 32 + (int)lane;
        perm[(int64_t)sm.sbase[bin[k]] + cnt[w][bin[k]] + pos[k]] = p;
      }
    }
    __syncthreads();
  }
}

template <class T>
__global__ void __launch_bounds__(256) k_fused_perm(ScatterParams<T> a) {
  __shared__ ScatterSmem sm;
  perm_tile(a, blockIdx.x, sm);
}

// The identity permutation: arrays already in cell order, read through perm.
static __global__ void k_iota(int32_t* perm, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    perm[i] = (int32_t)i;
}

// Batched permutation-only sort: persistent blocks over the (domain, tile) table.
template <class T>
__global__ void __launch_bounds__(256)
    k_fused_perm_batched(const ScatterParams<T>* descs, const int2* tiles, int ntiles, int* counter) {
  __shared__ ScatterSmem sm;
  __shared__ ScatterParams<T> a;
  __shared__ int next;
  while (true) {
    if (threadIdx.x == 0) next = atomicAdd(counter, 1);
    __syncthreads();
    const int t = next;
    if (t >= ntiles) break;
    const int2 it = tiles[t];
    if (threadIdx.x == 0) a = descs[it.x];
    __syncthreads();
    perm_tile(a, it.y, sm);
    __syncthreads();
  }
}

}  // namespace pbd

namespace pbd {

// Tile ranges of batched domains (grid row blockIdx.y = domain).
struct TileOffDesc {
  const int32_t* off;  // the domain's cell offsets (global positions)
  int ntiles, tpc, ty, my;
  int32_t end;         // global position after the domain's last particle
  int32_t* tile_off;
};

static __global__ void k_tile_off_batched(const TileOffDesc* d) {
  const TileOffDesc a = d[blockIdx.y];
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t <= a.ntiles; t += gridDim.x * blockDim.x) {
    if (t == a.ntiles) {
      a.tile_off[t] = a.end;
    } else {
      const int ix = t / a.tpc;
      a.tile_off[t] = a.off[(int64_t)ix * a.my + (int64_t)(t - ix * a.tpc) * a.ty];
    }
  }
}

}  // namespace pbd
