// Particle push over cell-sorted particles, one warp per cell: the same
// per-particle step as k_push (push_one: gather pic2d.f90:938-963, Boris
// 964-1000, move 1002-1026, the zig-zag terms of currentdeposit 1226-1296, x
// wrap and y wrap or walls), organised for sorted input.
//
// A block takes one tile (a run of tile_rows cells of one column, as k_push).
// Its warps take the tile's cells one at a time from a shared counter. A warp
// walks its cell's particles 32 at a time, lane l taking sorted position
// start + 32 i + l, so that every load and store of the particle arrays is one
// coalesced 128-byte access per array (through the sort's permutation the
// elements of a cell are almost consecutive), and every lane of the warp is in
// the same cell:
//   - the cell's gather record (bilinear coefficients of the 6 fields) is
//     loaded once per cell (one broadcast record) and stays in registers;
//   - each lane sums the 17-value deposit stencil of its particles in
//     registers; at the end of the cell one transposing reduction over the
//     warp (five shuffle rounds that halve the values a lane holds) leaves
//     entry k of the cell's stencil in one lane, which adds it to the tile's
//     shared-memory window;
//   - a particle that crosses a cell edge adds its second zig-zag segment to
//     the window on its own (split 32-bit sums in the mixed form, as k_push)
//     and moves one count of the tile's new-cell histogram (the fused sort).
// The last pass over a cell leaves the lanes past its end idle (on average
// half a pass per cell).
//
// A particle whose cell word is not the warp's cell (the input was not
// sorted by the offsets it came with) is not pushed: it is written back
// unchanged and STATUS_UNSORTED is set. The handle only runs this kernel on
// particles sorted by its own counting sort.
//
// With PushParams::rankw the kernel also ranks every particle for the fused
// counting sort: its direction (the window bin of its new cell relative to its
// old cell, 9 values) and its rank among the particles of its cell with that
// direction in position order (a match over the warp's lanes and a running
// count per direction), as a rank word per position, and each row's count per
// direction. The particles landing in a bin before a given one are then those
// of earlier rows with the matching direction (at most 3 rows) plus its rank,
// which k_fused_perm_rw turns into the sorted slot with a few additions.
//
// Sums: the lanes add their particles in sorted order, the reduction adds in a
// fixed lane pattern, and the window holds integers in the mixed form, so the
// mixed form's result does not depend on timing (bit-reproducible run to run).
#pragma once
#include "kernels_push.cuh"

namespace pbd {

// The handle runs this kernel on sorted input (PBPIC_PUSH_CELLS = 0 builds the
// library with k_push alone, for comparison).
#ifndef PBPIC_PUSH_CELLS
#define PBPIC_PUSH_CELLS 1
#endif
// The per-cell push writes rank words for the fused sort (0: the sort ranks
// the pushed cell words itself, k_fused_perm).
#ifndef PBPIC_PUSH_RANKS
#define PBPIC_PUSH_RANKS 1
#endif
#ifndef PBPIC_CPUSH_THREADS
#define PBPIC_CPUSH_THREADS 128
#endif
#ifndef PBPIC_CPUSH_MINBLOCKS
#define PBPIC_CPUSH_MINBLOCKS 4
#endif
#ifndef PBPIC_CPUSH_MINBLOCKS_FP64
#define PBPIC_CPUSH_MINBLOCKS_FP64 3
#endif

// Element k of a compile-time-sized array, 0 past its end.
template <int L, class T>
__device__ __forceinline__ T tr_get(const T (&v)[L], int k) {
  return k < L ? v[k < L ? k : 0] : T(0);
}

// One round of the transposing warp reduction: lanes without bit O keep the
// first M = ceil(L/2) values and receive their partner's, lanes with bit O keep
// the rest (zero-padded to M) and receive their partner's.
template <int L, int O, class T>
__device__ __forceinline__ void tr_round(const T (&v)[L], T (&w)[(L + 1) / 2], bool upper) {
  constexpr int H = (L + 1) / 2;
#pragma unroll
  for (int k = 0; k < H; ++k) {
    const T lo = v[k];
    const T hi = tr_get<L>(v, H + k);
    const T send = upper ? lo : hi;
    const T keep = upper ? hi : lo;
    w[k] = add_rn(keep, __shfl_xor_sync(FULL, send, O));
  }
}

// Sum of the 17 stencil values over the warp: the lane with index
// reduce17_entry(lane) = k receives the warp's total of entry k.
template <class T>
__device__ __forceinline__ T warp_reduce17(const T (&v)[17], unsigned lane) {
  T a[9], b[5], c[3], d[2], e[1];
  tr_round<17, 16>(v, a, (lane & 16u) != 0);
  tr_round<9, 8>(a, b, (lane & 8u) != 0);
  tr_round<5, 4>(b, c, (lane & 4u) != 0);
  tr_round<3, 2>(c, d, (lane & 2u) != 0);
  tr_round<2, 1>(d, e, (lane & 1u) != 0);
  return e[0];
}

// Stencil entry a lane holds after warp_reduce17, -1 for none (15 lanes).
__host__ __device__ __forceinline__ int reduce17_entry(unsigned lane) {
  const int sizes[5] = {17, 9, 5, 3, 2};
  int start = 0, len = 17;
  for (int r = 0; r < 5; ++r) {
    const int h = (sizes[r] + 1) / 2;
    if (lane & (16u >> r)) {
      start += h;
      len = len > h ? len - h : 0;
    } else {
      len = len < h ? len : h;
    }
  }
  return len >= 1 ? start : -1;
}

template <class T, bool MIXED, bool COMPAT, bool GATHER>
__global__ void __launch_bounds__(PBPIC_CPUSH_THREADS, MIXED ? PBPIC_CPUSH_MINBLOCKS : PBPIC_CPUSH_MINBLOCKS_FP64)
    k_push_cells(PushParams<T> a) {
  using Acc = typename std::conditional<MIXED, long long, double>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[32];
  __shared__ int next_row;
  __shared__ int dcount[PBPIC_CPUSH_THREADS / 32][16];  // rank words: the warp's running counts per direction
  const int t = blockIdx.x;
  const int TY = a.tile_rows, WR = TY + 3, NB = 3 * (TY + 2);
  Acc* win = reinterpret_cast<Acc*>(smem_raw);
  int* hist = reinterpret_cast<int*>(win + 16 * WR);
  unsigned* clo = reinterpret_cast<unsigned*>(hist + NB);  // crossers (mixed form): jx, jy planes (8 * WR)
  int* chi = reinterpret_cast<int*>(clo + 8 * WR);
  const int ixt = t / a.tiles_per_col;
  const int y0 = (t - ixt * a.tiles_per_col) * TY;
  const int y1 = min(y0 + TY, a.my);
  for (int e = threadIdx.x; e < 16 * WR; e += blockDim.x) win[e] = Acc(0);
  if (MIXED)
    for (int e = threadIdx.x; e < 8 * WR; e += blockDim.x) {
      clo[e] = 0u;
      chi[e] = 0;
    }
  // new-cell counts of the tile's window, starting from the input's counts
  for (int e = threadIdx.x; e < NB; e += blockDim.x) {
    const int by = e - (TY + 2);
    int v = 0;
    if (by >= 1 && by <= y1 - y0) {
      const long long c = (long long)ixt * a.my + y0 + by - 1;
      v = a.cell_off[c + 1] - a.cell_off[c];
    }
    hist[e] = v;
  }
  if (threadIdx.x == 0) next_row = y0;
  __syncthreads();
  Acc* gacc = reinterpret_cast<Acc*>(a.jacc);
  const long long cbase = (long long)ixt * a.my;
  const bool split = MIXED && a.cell_off[cbase + y1] - a.cell_off[cbase + y0] <= 32767;
  const unsigned lane = lane_id();
  const int ent = reduce17_entry(lane);
  int sc = 0, sx = 0, sy = 0;
  stencil_node(ent >= 0 ? ent : 0, &sc, &sx, &sy);
  uint32_t* ocell = GATHER ? a.cell_o : a.cell;
  T *odx = GATHER ? a.dx_o : a.dx, *ody = GATHER ? a.dy_o : a.dy;
  T *oux = GATHER ? a.ux_o : a.ux, *ouy = GATHER ? a.uy_o : a.uy, *ouz = GATHER ? a.uz_o : a.uz;
  double ke_e = 0.0, ke_i = 0.0;
  int status = 0;
  while (true) {
    int iy = 0;
    if (lane == 0) iy = atomicAdd(&next_row, 1);
    iy = __shfl_sync(FULL, iy, 0);
    if (iy >= y1) break;
    const long long c = cbase + iy;
    const int pbeg = a.cell_off[c], pend = a.cell_off[c + 1];
    if (pbeg >= pend) {  // an empty row sends nothing anywhere
      if (a.rankw && lane < 9) a.ctab[((long long)t * TY + (iy - y0)) * 9 + lane] = 0;
      continue;
    }
    const int key = iy - y0;
    const uint32_t cw0 = cw_make(ixt, iy, 0);
    Node6<T> n00, n01, n10, n11;
    CellCoef cc;
    if constexpr (MIXED && PBPIC_CELL_COEF) {
      load_coef(a.cg + c * 24, cc);
    } else if constexpr (MIXED) {
      load_cell(a.cg + c * 24, n00, n01, n10, n11);
    } else {
      const T* g00 = a.ng + ((long long)ixt * (a.my + 1) + iy) * 8;
      const T* g10 = g00 + (long long)(a.my + 1) * 8;
      n00 = load_node(g00);
      n01 = load_node(g00 + 8);
      n10 = load_node(g10);
      n11 = load_node(g10 + 8);
    }
    T acc[17];
#pragma unroll
    for (int k = 0; k < 17; ++k) acc[k] = T(0);
    T pke_e = T(0), pke_i = T(0);
    const int w = threadIdx.x >> 5;
    if (a.rankw) {
      if (lane < 16) dcount[w][lane] = 0;
      __syncwarp();
    }
#pragma unroll 1
    for (int q = pbeg; q < pend; q += 32) {
      const int p = q + (int)lane;
      int dir = 15;  // rank words: this lane's direction (15: no particle)
      if (p < pend) {
        const int e = GATHER ? __ldg(a.src + p) : p;
        uint32_t wrd;
        T px, py, pux, puy, puz;
        if (GATHER) {  // the input is not written by this launch: read-only loads
          wrd = __ldg(a.cell + e);
          px = __ldg(a.dx + e);
          py = __ldg(a.dy + e);
          pux = __ldg(a.ux + e);
          puy = __ldg(a.uy + e);
          puz = __ldg(a.uz + e);
        } else {
          wrd = a.cell[e];
          px = a.dx[e];
          py = a.dy[e];
          pux = a.ux[e];
          puy = a.uy[e];
          puz = a.uz[e];
        }
        const int sp = cw_sp(wrd);
        if ((wrd & 0x7fffffffu) != cw0) {  // not this cell's particle: left as it is
          status |= 4;
          dir = 4;  // ranked with this cell's particles, where its count is
          ocell[p] = wrd;
          odx[p] = px;
          ody[p] = py;
          oux[p] = pux;
          ouy[p] = puy;
          ouz[p] = puz;
        } else {
          Pushed<T> o;
          if constexpr (MIXED && PBPIC_CELL_COEF)
            push_one_coef<COMPAT>(a, sp, ixt, iy, px, py, pux, puy, puz, cc, o);
          else
            push_one<T, MIXED, COMPAT>(a, sp, ixt, iy, px, py, pux, puy, puz, n00, n01, n10, n11, o);
          status |= o.status;
          const bool cross = o.dcx != 0 || o.dcy != 0;
          if (cross) {
            // new cell in the tile's window: column 1 + dcx, row new_iy - y0 + 1
            // (wrapped rows come back through +-my; a reflected particle keeps its row)
            int by = cw_iy(o.cw) - y0 + 1;
            by = by < 0 ? by + a.my : (by > y1 - y0 + 1 ? by - a.my : by);
            int b = (1 + o.dcx) * (TY + 2) + by;
            if (by < 0 || by > y1 - y0 + 1) {
              b = window_bin(cw_ix(o.cw), cw_iy(o.cw), ixt, y0, y1, TY, a.mx, a.my, a.ybc);
              if (b < 0) {  // only a corrupt offset can jump two cells: keep the particle in its cell
                status |= 1;
                o.cw = wrd;
                b = window_bin(ixt, iy, ixt, y0, y1, TY, a.mx, a.my, a.ybc);
              }
            }
            const int bo = (TY + 2) + key + 1;  // the old cell's bin
            if (b != bo) {
              atomicAdd(&hist[b], 1);
              atomicAdd(&hist[bo], -1);
            }
            dir = (b / (TY + 2)) * 3 + (b % (TY + 2) - key);
            // second zig-zag segment, attached to the new cell
            const int wx = 1 + o.dcx, wy = key + 1 + o.dcy;
            const int b0 = (JX * 4 + wx) * WR + wy, b1 = (JY * 4 + wx) * WR + wy;
            if (split) {
              cross_add(clo, chi, b0, to_acc<T, MIXED>(o.e[2]));
              cross_add(clo, chi, b0 + 1, to_acc<T, MIXED>(o.e[3]));
              cross_add(clo, chi, b1, to_acc<T, MIXED>(o.e[6]));
              cross_add(clo, chi, b1 + WR, to_acc<T, MIXED>(o.e[7]));
            } else {
              acc_add(&win[b0], to_acc<T, MIXED>(o.e[2]));
              acc_add(&win[b0 + 1], to_acc<T, MIXED>(o.e[3]));
              acc_add(&win[b1], to_acc<T, MIXED>(o.e[6]));
              acc_add(&win[b1 + WR], to_acc<T, MIXED>(o.e[7]));
            }
          }
          if constexpr (MIXED) {
            acc[0] = __fadd_rn(acc[0], __fmaf_rn(-o.ja, o.jw, o.ja));
            acc[1] = __fmaf_rn(o.ja, o.jw, acc[1]);
            acc[2] = __fadd_rn(acc[2], __fmaf_rn(-o.jb, o.jv, o.jb));
            acc[3] = __fmaf_rn(o.jb, o.jv, acc[3]);
            // jz: outer product of the x weights (x = -1, 0, 1) and y weights
            const T qs = __fmul_rn(o.quz, o.zdx), qz0 = __fsub_rn(o.quz, qs);
            const T qxm = o.di < 0 ? qs : T(0), qxp = o.di > 0 ? qs : T(0);
            const T ym = o.dj < 0 ? o.zdy : T(0), yp = o.dj > 0 ? o.zdy : T(0), yz0 = __fsub_rn(T(1), o.zdy);
            acc[4 + 0] = __fmaf_rn(qxm, ym, acc[4 + 0]);
            acc[4 + 1] = __fmaf_rn(qxm, yz0, acc[4 + 1]);
            acc[4 + 2] = __fmaf_rn(qxm, yp, acc[4 + 2]);
            acc[4 + 3] = __fmaf_rn(qz0, ym, acc[4 + 3]);
            acc[4 + 4] = __fmaf_rn(qz0, yz0, acc[4 + 4]);
            acc[4 + 5] = __fmaf_rn(qz0, yp, acc[4 + 5]);
            acc[4 + 6] = __fmaf_rn(qxp, ym, acc[4 + 6]);
            acc[4 + 7] = __fmaf_rn(qxp, yz0, acc[4 + 7]);
            acc[4 + 8] = __fmaf_rn(qxp, yp, acc[4 + 8]);
          } else {
            acc[0] += cross ? o.e[0] : o.e[0] + o.e[2];
            acc[1] += cross ? o.e[1] : o.e[1] + o.e[3];
            acc[2] += cross ? o.e[4] : o.e[4] + o.e[6];
            acc[3] += cross ? o.e[5] : o.e[5] + o.e[7];
            // jz: (0,0) <- e8, (di,0) <- e9, (0,dj) <- e10, (di,dj) <- e11 with di, dj = +-1
            const T zxm = o.di < 0 ? T(1) : T(0), zxp = o.di > 0 ? T(1) : T(0);
            const T zym = o.dj < 0 ? T(1) : T(0), zyp = o.dj > 0 ? T(1) : T(0);
            acc[4 + 0] += zxm * zym * o.e[11];
            acc[4 + 1] += zxm * o.e[9];
            acc[4 + 2] += zxm * zyp * o.e[11];
            acc[4 + 3] += zym * o.e[10];
            acc[4 + 4] += o.e[8];
            acc[4 + 5] += zyp * o.e[10];
            acc[4 + 6] += zxp * zym * o.e[11];
            acc[4 + 7] += zxp * o.e[9];
            acc[4 + 8] += zxp * zyp * o.e[11];
          }
          acc[13] += o.e[12];
          acc[14] += o.e[13];
          acc[15] += o.e[14];
          acc[16] += o.e[15];
          if (sp) pke_e += o.ke;
          else pke_i += o.ke;
          if (!cross) dir = 4;  // stays: window column 1, row key + 1
          ocell[p] = o.cw;
          odx[p] = o.dx;
          ody[p] = o.dy;
          oux[p] = o.ux;
          ouy[p] = o.uy;
          ouz[p] = o.uz;
        }
        if (GATHER && a.pid_o) a.pid_o[p] = __ldg(a.pid_i + e);
      }
      if (a.rankw) {  // stable rank among this cell's particles of the same direction
        const unsigned peers = __match_any_sync(FULL, dir);
        const int before = dir < 9 ? dcount[w][dir] : 0;
        __syncwarp();
        if (dir < 9 && (peers & lanemask_lt()) == 0) dcount[w][dir] = before + __popc(peers);
        __syncwarp();
        if (p < pend) {
          const int r = before + __popc(peers & lanemask_lt());
          if (r >= (1 << 22)) status |= 1;  // a cell of more than 4 M particles
          a.rankw[p] = (key << 26) | ((dir & 15) << 22) | (r & 0x3fffff);
        }
      }
    }
    if (a.rankw && lane < 9) a.ctab[((long long)t * TY + key) * 9 + lane] = dcount[w][lane];
    ke_e += (double)pke_e;
    ke_i += (double)pke_i;
    const T v = warp_reduce17(acc, lane);
    if (ent >= 0 && v != T(0)) acc_add(&win[(sc * 4 + 1 + sx) * WR + key + 1 + sy], to_acc<T, MIXED>(v));
  }
  __syncthreads();
  // Fold the window into the global current (as k_push).
  for (int e = threadIdx.x; e < 16 * WR; e += blockDim.x) {
    Acc val = win[e];
    if (MIXED && e < 8 * WR) val += (Acc)(((long long)chi[e] << 17) + (long long)clo[e]);
    if (val == Acc(0)) continue;
    const int cc = e / (4 * WR);
    const int r = e - cc * 4 * WR;
    const int wx = r / WR, wy = r - wx * WR;
    long long gi;
    int sg;
    if (map_current(cc, ixt - 1 + wx, y0 - 1 + wy, a.mx, a.my, a.S, a.ybc, a.compat, &gi, &sg))
      acc_add(&gacc[gi], sg < 0 ? -val : val);
  }
  for (int e = threadIdx.x; e < NB; e += blockDim.x) a.tilecnt[(long long)t * NB + e] = hist[e];
  const double se = block_sum(ke_e, red);
  const double si = block_sum(ke_i, red);
  if (threadIdx.x == 0) {
    a.ke_part[2 * t] = se;
    a.ke_part[2 * t + 1] = si;
  }
  status = __reduce_or_sync(FULL, status);
  if (lane == 0 && status) atomicOr(a.status, status);
}

}  // namespace pbd
