// Kernels of the y-slab decomposition (one rank per slab of cell rows, the
// reference's 1-D domain decomposition along y, pic2d.f90:206-212). Each rank
// steps an extended domain: its own rows plus ghost bands of rows copied
// from the neighbouring slabs. These kernels move particles and field rows in
// and out of such a domain and sum energies over its own rows:
//   k_band_flags / k_band_out    particles of a band of rows -> reference
//                                records, rows renumbered to the global grid
//   k_band_keep                  stable compaction to a band of rows
//   k_band_in                    reference records (global grid) -> appended
//   k_rows_get / k_rows_set      rows of the six field planes
//   k_kinetic_rows, k_field_energy_rows   energy sums over the own rows
// and, when the particles are sorted by cell, single-pass versions: a band
// copied column by column from the cell offsets (k_band_out_sorted), and the
// own rows merged with both received bands straight into cell order
// (k_band_assemble); both read through the sort's permutation when the
// particle arrays are held in permuted order.
#pragma once
#include "device_common.cuh"
#include "kernels_misc.cuh"

namespace pbd {

static __global__ void k_band_flags(int64_t n, const uint32_t* cell, int y_lo, int y_hi, int32_t* flags) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += (int64_t)gridDim.x * blockDim.x) {
    if (i == n) {
      flags[i] = 0;
      continue;
    }
    const int iy = cw_iy(cell[i]);
    flags[i] = (iy >= y_lo && iy < y_hi) ? 1 : 0;
  }
}

// Particles with a flag to out[pos[i]] as reference records of the global
// grid: grid = my_global * ix + (iy + row_offset) + 1, q = +1 ion / -1 electron.
template <class T, class R>
__global__ void k_band_out(int64_t n, const uint32_t* cell, const T* dx, const T* dy, const T* ux, const T* uy,
                           const T* uz, const int32_t* pid, const int32_t* pos, int my_global, int row_offset,
                           RefRec<R>* out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (pos[i + 1] == pos[i]) continue;  // not in the band
    const uint32_t w = cell[i];
    RefRec<R> r;
    r.dx = (R)dx[i];
    r.dy = (R)dy[i];
    r.ux = (R)ux[i];
    r.uy = (R)uy[i];
    r.uz = (R)uz[i];
    r.grid = my_global * cw_ix(w) + cw_iy(w) + row_offset + 1;
    r.q = cw_sp(w) ? -1 : 1;
    r.pid = pid ? pid[i] : 0;
    out[pos[i]] = r;
  }
}

// Stable compaction of the flagged particles into the other buffer.
template <class T>
__global__ void k_band_keep(int64_t n, const int32_t* pos, const uint32_t* ci, const T* dxi, const T* dyi,
                            const T* uxi, const T* uyi, const T* uzi, const int32_t* pidi, uint32_t* co, T* dxo,
                            T* dyo, T* uxo, T* uyo, T* uzo, int32_t* pido) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (pos[i + 1] == pos[i]) continue;
    const int64_t d = pos[i];
    co[d] = ci[i];
    dxo[d] = dxi[i];
    dyo[d] = dyi[i];
    uxo[d] = uxi[i];
    uyo[d] = uyi[i];
    uzo[d] = uzi[i];
    if (pido) pido[d] = pidi[i];
  }
}

// Reference records of the global grid appended at base: local row =
// global row - row_offset, which must fall in [0, my) (status bit 8 and the
// record is written as an empty electron at cell (0, 0) with zero momentum
// otherwise, so that the count stays consistent).
template <class T, class R>
__global__ void k_band_in(const RefRec<R>* in, int64_t n, int my_global, int row_offset, int mx, int my, int64_t base,
                          uint32_t* cell, T* dx, T* dy, T* ux, T* uy, T* uz, int32_t* pid, int* status) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const RefRec<R> r = in[i];
    const int g = r.grid - 1;
    const int ix = g / my_global, gy = g - ix * my_global;
    const int iy = gy - row_offset;
    const bool ok = g >= 0 && ix < mx && iy >= 0 && iy < my && (r.q == 1 || r.q == -1);
    const int64_t d = base + i;
    if (!ok) atomicOr(status, 8);
    cell[d] = ok ? cw_make(ix, iy, r.q < 0 ? 1 : 0) : cw_make(0, 0, 1);
    dx[d] = ok ? (T)r.dx : T(0);
    dy[d] = ok ? (T)r.dy : T(0);
    ux[d] = ok ? (T)r.ux : T(0);
    uy[d] = ok ? (T)r.uy : T(0);
    uz[d] = ok ? (T)r.uz : T(0);
    if (pid) pid[d] = r.pid;
  }
}

// Rows j0 .. j0+nrows-1 of the six planes <-> buf[(c * mx + i) * nrows + r].
template <class T>
struct Planes6 {
  T* f[6];
};

template <class T>
__global__ void k_rows_get(Planes6<T> p, int mx, int S, int j0, int nrows, T* buf) {
  const int64_t tot = (int64_t)6 * mx * nrows;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < tot; k += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(k / ((int64_t)mx * nrows));
    const int64_t rem = k - (int64_t)c * mx * nrows;
    const int i = (int)(rem / nrows), r = (int)(rem - (int64_t)i * nrows);
    buf[k] = p.f[c][(int64_t)i * S + j0 + r];
  }
}

template <class T>
__global__ void k_rows_set(Planes6<T> p, int mx, int S, int j0, int nrows, const T* buf) {
  const int64_t tot = (int64_t)6 * mx * nrows;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < tot; k += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(k / ((int64_t)mx * nrows));
    const int64_t rem = k - (int64_t)c * mx * nrows;
    const int i = (int)(rem / nrows), r = (int)(rem - (int64_t)i * nrows);
    p.f[c][(int64_t)i * S + j0 + r] = buf[k];
  }
}

// Kinetic energy of the particles in rows [y_lo, y_hi), as k_kinetic.
template <class T, bool MIXED>
__global__ void k_kinetic_rows(int64_t n, const uint32_t* cell, const T* ux, const T* uy, const T* uz, T ms_i,
                               int y_lo, int y_hi, double* part) {
  __shared__ double red[32];
  double ke[2] = {0, 0};
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t w = cell[i];
    const int iy = cw_iy(w);
    if (iy < y_lo || iy >= y_hi) continue;
    using A = M<T, MIXED>;
    const T a = ux[i], b = uy[i], c = uz[i];
    const T usq = A::mad(c, c, A::mad(b, b, A::mul(a, a)));
    const T g = A::sqrt(A::mad(c, c, A::mad(b, b, A::mad(a, a, T(1)))));
    const int sp = cw_sp(w);
    const T ms = sp ? T(1) : ms_i;
    const double e = MIXED ? (double)A::mul(A::div(usq, A::add(g, T(1))), ms) : (double)A::mul(A::sub(g, T(1)), ms);
    ke[sp ? 0 : 1] += e;
  }
  const double s0 = block_sum(ke[0], red), s1 = block_sum(ke[1], red);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = s0;
    part[2 * blockIdx.x + 1] = s1;
  }
}

// Field energy sums over node rows [y_lo, y_hi) of the node grid (the
// fieldsenergy sums of k_nodes); node rows equal to wall_lo or wall_hi
// (global walls) weigh 1/2.
template <class T>
__global__ void k_field_energy_rows(int mx, int my, const T* ng, int y_lo, int y_hi, int wall_lo, int wall_hi,
                                    double* part) {
  __shared__ double red[32];
  const int rows = y_hi - y_lo;
  const int64_t nn = (int64_t)mx * rows;
  double se = 0.0, sb = 0.0;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(k / rows), j = y_lo + (int)(k - (int64_t)(k / rows) * rows);
    const T* g = ng + ((int64_t)i * (my + 1) + j) * 8;
    const T e2 = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
    const T b2 = g[4] * g[4] + g[5] * g[5] + g[6] * g[6];
    const double w = (j == wall_lo || j == wall_hi) ? 0.5 : 1.0;
    se += w * (double)e2;
    sb += w * (double)b2;
  }
  se = block_sum(se, red);
  sb = block_sum(sb, red);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = se;
    part[2 * blockIdx.x + 1] = sb;
  }
}

}  // namespace pbd

namespace pbd {

// ----------------------------------------------- sorted fast paths of the slab
// When the particles are sorted by cell, the particles of rows [y_lo, y_hi)
// of column ix are the range [off[ix*my + y_lo], off[ix*my + y_hi]).

// Per column: the number of particles of rows [y_lo, y_hi) (colcnt[mx] = 0).
static __global__ void k_col_counts(const int32_t* off, int mx, int my, int y_lo, int y_hi, int32_t* colcnt) {
  for (int ix = blockIdx.x * blockDim.x + threadIdx.x; ix <= mx; ix += gridDim.x * blockDim.x)
    colcnt[ix] = ix == mx ? 0 : off[(int64_t)ix * my + y_hi] - off[(int64_t)ix * my + y_lo];
}

// Column of output index k: the last ix with start[ix] <= k (start: exclusive
// scan over mx columns, start[mx] = total).
__device__ __forceinline__ int column_of(const int32_t* start, int mx, int64_t k) {
  int lo = 0, hi = mx - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (start[mid] <= k) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// One 32-byte reference record with two 16-byte stores when the buffer is
// 16-byte aligned (FP64 records, 56 bytes, are stored as they are).
__device__ __forceinline__ void store_record(RefRec<float>* p, const RefRec<float>& r, bool al16) {
  if (al16) {
    uint4* d = reinterpret_cast<uint4*>(p);
    d[0] = make_uint4(__float_as_uint(r.dx), __float_as_uint(r.dy), __float_as_uint(r.ux), __float_as_uint(r.uy));
    d[1] = make_uint4(__float_as_uint(r.uz), (unsigned)r.grid, (unsigned)r.q, (unsigned)r.pid);
  } else {
    *p = r;
  }
}
__device__ __forceinline__ void store_record(RefRec<double>* p, const RefRec<double>& r, bool) { *p = r; }

// Band extraction from sorted particles: output k of column ix comes from
// off[ix*my + y_lo] + (k - colstart[ix]); same records as k_band_out. One
// block per column (grid-stride over the columns).
template <class T, class R>
__global__ void k_band_out_sorted(const int32_t* colstart, const int32_t* off, int mx, int my, int y_lo,
                                  const uint32_t* cell, const T* dx, const T* dy, const T* ux, const T* uy,
                                  const T* uz, const int32_t* pid, int my_global, int row_offset, RefRec<R>* out,
                                  const int32_t* perm, bool al16) {
  for (int ix = blockIdx.x; ix < mx; ix += gridDim.x) {
    const int64_t k0 = colstart[ix], k1 = colstart[ix + 1];
    const int64_t j0 = (int64_t)off[(int64_t)ix * my + y_lo] - k0;  // sorted position of output k: j0 + k
    for (int64_t k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
      const int64_t j = j0 + k;
      const int64_t i = perm ? (int64_t)perm[j] : j;
      const uint32_t w = cell[i];
      RefRec<R> r;
      r.dx = (R)dx[i];
      r.dy = (R)dy[i];
      r.ux = (R)ux[i];
      r.uy = (R)uy[i];
      r.uz = (R)uz[i];
      r.grid = my_global * cw_ix(w) + cw_iy(w) + row_offset + 1;
      r.q = cw_sp(w) ? -1 : 1;
      r.pid = pid ? pid[i] : 0;
      store_record(out + k, r, al16);
    }
  }
}

// Particles per output column: bottom band + own rows + top band.
static __global__ void k_col_sum3(const int32_t* a, const int32_t* b, const int32_t* c, int mx, int32_t* out) {
  for (int ix = blockIdx.x * blockDim.x + threadIdx.x; ix <= mx; ix += gridDim.x * blockDim.x)
    out[ix] = ix == mx ? 0 : a[ix] + b[ix] + c[ix];
}

// Per-column counts of band records (global grid) that come in column order:
// the first and one-past-last record of each column's run are found at the
// run boundaries (no atomics: neighbouring threads share a column), then
// cnt = last - first (both zero for an absent column).
template <class R>
__global__ void k_band_col_bounds(const RefRec<R>* in, int64_t n, int my_global, int mx, int32_t* first,
                                  int32_t* last) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int ix = (in[i].grid - 1) / my_global;
    if (ix < 0 || ix >= mx) continue;
    const int prev = i > 0 ? (in[i - 1].grid - 1) / my_global : -1;
    const int next = i + 1 < n ? (in[i + 1].grid - 1) / my_global : -1;
    if (prev != ix) first[ix] = (int32_t)i;
    if (next != ix) last[ix] = (int32_t)(i + 1);
  }
}

static __global__ void k_col_diff(const int32_t* first, const int32_t* last, int mx, int32_t* cnt) {
  for (int ix = blockIdx.x * blockDim.x + threadIdx.x; ix <= mx; ix += gridDim.x * blockDim.x)
    cnt[ix] = ix == mx ? 0 : last[ix] - first[ix];
}

// The slab's new particle array in cell order, column by column: the bottom
// band's particles of the column, the own rows' particles (sorted input,
// range from off), the top band's particles. Band records are in column order
// and, within a column, in cell order (they were extracted that way).
struct ReplaceSrc {
  const int32_t* off;      // cell offsets of the sorted input
  const int32_t* outstart; // [mx + 1] first output position of each column
  const int32_t* bstart;   // [mx + 1] first bottom-band record of each column
  const int32_t* bcnt;     // [mx] bottom-band records per column
  const int32_t* ocnt;     // [mx] own particles per column
  int mx, my, y_lo, my_global, off_bottom, off_top;
  const int32_t* tstart;   // [mx + 1] first top-band record of each column
};

template <class T, class R>
__global__ void k_band_assemble(int64_t total, ReplaceSrc s, const RefRec<R>* bot, const RefRec<R>* top,
                                const uint32_t* ci, const T* dxi, const T* dyi, const T* uxi, const T* uyi,
                                const T* uzi, const int32_t* pidi, uint32_t* co, T* dxo, T* dyo, T* uxo, T* uyo,
                                T* uzo, int32_t* pido, int* status, const int32_t* perm) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
    const int ix = column_of(s.outstart, s.mx, k);
    int64_t r = k - s.outstart[ix];
    const int nb = s.bcnt[ix], no = s.ocnt[ix];
    if (r >= nb && r < nb + no) {  // own particle (read through the sort's permutation when there is one)
      const int64_t j = (int64_t)s.off[(int64_t)ix * s.my + s.y_lo] + (r - nb);
      const int64_t i = perm ? (int64_t)perm[j] : j;
      co[k] = ci[i];
      dxo[k] = dxi[i];
      dyo[k] = dyi[i];
      uxo[k] = uxi[i];
      uyo[k] = uyi[i];
      uzo[k] = uzi[i];
      if (pido) pido[k] = pidi[i];
      continue;
    }
    const bool lower = r < nb;
    const RefRec<R> rec = lower ? bot[s.bstart[ix] + r] : top[s.tstart[ix] + (r - nb - no)];
    const int g = rec.grid - 1;
    const int gx = g / s.my_global, gy = g - gx * s.my_global;
    const int iy = gy - (lower ? s.off_bottom : s.off_top);
    const bool ok = gx == ix && iy >= 0 && iy < s.my && (rec.q == 1 || rec.q == -1);
    if (!ok) atomicOr(status, 8);
    co[k] = ok ? cw_make(ix, iy, rec.q < 0 ? 1 : 0) : cw_make(ix, s.y_lo, 1);
    dxo[k] = ok ? (T)rec.dx : T(0);
    dyo[k] = ok ? (T)rec.dy : T(0);
    uxo[k] = ok ? (T)rec.ux : T(0);
    uyo[k] = ok ? (T)rec.uy : T(0);
    uzo[k] = ok ? (T)rec.uz : T(0);
    if (pido) pido[k] = rec.pid;
  }
}

// Band assembly without moving the slab's own particles: the received band
// records are converted in place after the current particles (elements
// base .. base + nb + nt of the current arrays: the bottom band, then the top
// band), and the assembled cell order becomes a permutation -- each column's
// bottom band, own rows, top band, as k_band_assemble writes them -- which the
// next push reads through. The own particles stay where they are.
template <class T, class R>
__global__ void k_band_to_soa(int64_t nb, int64_t nt, ReplaceSrc s, const RefRec<R>* bot, const RefRec<R>* top,
                              int64_t base, uint32_t* co, T* dxo, T* dyo, T* uxo, T* uyo, T* uzo, int32_t* pido,
                              int* status) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nb + nt; k += (int64_t)gridDim.x * blockDim.x) {
    const bool lower = k < nb;
    const RefRec<R> rec = lower ? bot[k] : top[k - nb];
    const int g = rec.grid - 1;
    const int gx = g / s.my_global, gy = g - gx * s.my_global;
    const int iy = gy - (lower ? s.off_bottom : s.off_top);
    const bool ok = gx >= 0 && gx < s.mx && iy >= 0 && iy < s.my && (rec.q == 1 || rec.q == -1);
    if (!ok) atomicOr(status, 8);
    const int64_t e = base + k;
    co[e] = ok ? cw_make(gx, iy, rec.q < 0 ? 1 : 0) : cw_make(gx >= 0 && gx < s.mx ? gx : 0, s.y_lo, 1);
    dxo[e] = ok ? (T)rec.dx : T(0);
    dyo[e] = ok ? (T)rec.dy : T(0);
    uxo[e] = ok ? (T)rec.ux : T(0);
    uyo[e] = ok ? (T)rec.uy : T(0);
    uzo[e] = ok ? (T)rec.uz : T(0);
    if (pido) pido[e] = rec.pid;
  }
}

// Assembled position -> element of the current arrays, one block per column
// (its positions outstart[ix] .. outstart[ix+1]: bottom band, own rows, top band).
__global__ static void k_band_assemble_perm(ReplaceSrc s, int64_t base, int64_t nb_all, const int32_t* perm,
                                            int32_t* out) {
  for (int ix = blockIdx.x; ix < s.mx; ix += gridDim.x) {
    const int64_t k0 = s.outstart[ix], k1 = s.outstart[ix + 1];
    const int nb = s.bcnt[ix], no = s.ocnt[ix];
    const int64_t own0 = s.off[(int64_t)ix * s.my + s.y_lo];
    const int64_t b0 = base + s.bstart[ix], t0 = base + nb_all + s.tstart[ix];
    for (int64_t k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
      const int64_t r = k - k0;
      int64_t e;
      if (r < nb) {
        e = b0 + r;
      } else if (r < nb + no) {
        const int64_t j = own0 + (r - nb);
        e = perm ? (int64_t)perm[j] : j;
      } else {
        e = t0 + (r - nb - no);
      }
      out[k] = (int32_t)e;
    }
  }
}

// Cell counts of the assembled order: the own rows [y_lo, y_hi) keep their
// counts (from the offsets before the assembly), the ghost rows count the
// converted band records.
__global__ static void k_counts_own_rows(const int32_t* off, int64_t ncells, int my, int y_lo, int y_hi,
                                         int32_t* counts) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c <= ncells; c += (int64_t)gridDim.x * blockDim.x) {
    if (c == ncells) {
      counts[c] = 0;
      continue;
    }
    const int row = (int)(c % my);
    counts[c] = (row >= y_lo && row < y_hi) ? off[c + 1] - off[c] : 0;
  }
}

__global__ static void k_counts_band(int64_t n, const uint32_t* cell, int64_t base, int my, int32_t* counts) {
  // The records of a cell are one run (the bands arrive in cell order): the
  // run's first record adds -k and its last k + 1, so the count grows by the
  // run's length with two atomics per cell instead of one per record. A run
  // split in two (a record out of order) still adds both lengths.
  auto key = [&](int64_t k) { const uint32_t w = cell[base + k]; return (int64_t)cw_ix(w) * my + cw_iy(w); };
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = key(k);
    const bool first = k == 0 || key(k - 1) != c, last = k + 1 == n || key(k + 1) != c;
    if (first && last) atomicAdd(&counts[c], 1);
    else if (first) atomicAdd(&counts[c], (int32_t)-k);
    else if (last) atomicAdd(&counts[c], (int32_t)(k + 1));
  }
}

}  // namespace pbd
