// Particle push: bilinear field gather, Boris rotation, move with cell
// crossing, Umeda zig-zag current deposit, x wrap and y wrap or wall
// reflection -- the particle loop of pusher (pic2d.f90:934-1063) and
// currentdeposit (pic2d.f90:1226-1296).
//
// Work decomposition: a tile is a run of `tile_rows` cells of one column
// (cells ix*my + y0 .. ix*my + y0 + tile_rows - 1, contiguous in the sorted
// order), and one block pushes the particles of one tile. Its current goes to
// a shared-memory window of 4 node columns (ix-1 .. ix+2) x (tile_rows + 3)
// node rows, which covers every node a particle of the tile can touch in one
// step. Non-crossing particles deposit a 17-value stencil relative to their
// cell; lanes of a warp that share a cell are summed by a segmented scan and
// only the last lane of each run adds to shared memory. Crossing particles add
// their 16 values individually. A particle outside its tile (the array is not
// sorted) adds straight to global memory. At the end the window is folded into
// the global current with the periodic wrap and the wall images.
#pragma once
#include <type_traits>
#include "device_common.cuh"

namespace pbd {

template <class T>
struct PushParams {
  int mx, my, S, ybc, compat;
  int tile_rows, tiles_per_col, ntiles;
  const int32_t* tile_off;  // [ntiles + 1] particle position ranges of the tiles
  uint32_t* cell;
  T *dx, *dy, *ux, *uy, *uz;
  const T* ng;  // node fields (mx+1) x (my+1) x 8: ex ey ez 0 bx by bz 0
  void* jacc;   // 4 planes (jx, jy, jz, rho) of mx x S accumulators
  T c0[2], c1[2], ms[2], qx[2], qy[2], q[2];  // per species: 0 ion, 1 electron
  T dtcva, idx, idy, cva;
  double* ke_part;  // [ntiles][2]: electron, ion kinetic energy of the tile
  int* status;
};

template <class T>
struct Node6 {
  T ex, ey, ez, bx, by, bz;
};

__device__ __forceinline__ Node6<float> load_node(const float* g) {
  float4 a = __ldg(reinterpret_cast<const float4*>(g));
  float4 b = __ldg(reinterpret_cast<const float4*>(g) + 1);
  return Node6<float>{a.x, a.y, a.z, b.x, b.y, b.z};
}
__device__ __forceinline__ Node6<double> load_node(const double* g) {
  const double2* p = reinterpret_cast<const double2*>(g);
  double2 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2), d = __ldg(p + 3);
  return Node6<double>{a.x, a.y, b.x, c.x, c.y, d.x};
}

// State of one particle after the push, and its 16 deposit terms.
template <class T>
struct Pushed {
  uint32_t cw;          // new cell word
  T dx, dy, ux, uy, uz; // new state (after reflection)
  int ix, iy;           // old cell
  int dcx, dcy, di, dj; // cell steps and jz quadrant
  T e[16];              // jx 4, jy 4, jz 4, rho 4 (see deposit_terms)
  double ke;
  int status;
};

// The push of one particle. `MIXED` selects fused multiply-adds; with
// MIXED == false every expression is evaluated in the reference's order with
// separately rounded operations.
template <class T, bool MIXED>
__device__ __forceinline__ void push_one(const PushParams<T>& a, uint32_t w, T px, T py, T pux,
                                         T puy, T puz, Pushed<T>& o) {
  using A = M<T, MIXED>;
  const int sp = cw_sp(w);
  const int ix = cw_ix(w), iy = cw_iy(w);
  const T half = T(0.5), one = T(1);
  // CIC weights, pic2d.f90:948-951
  const T axw = A::add(half, px), ayw = A::add(half, py);
  const T s1 = A::mul(axw, ayw);
  const T s2 = A::sub(axw, s1);
  const T s3 = A::sub(ayw, s1);
  const T s4 = A::sub(A::sub(A::sub(one, s1), s2), s3);
  // gather, pic2d.f90:952-963 (nodes ix..ix+1, iy..iy+1)
  const T* g00 = a.ng + ((long long)ix * (a.my + 1) + iy) * 8;
  const T* g10 = g00 + (long long)(a.my + 1) * 8;
  const Node6<T> n00 = load_node(g00), n01 = load_node(g00 + 8);
  const Node6<T> n10 = load_node(g10), n11 = load_node(g10 + 8);
#define PBD_GATHER(f) \
  A::mad(n11.f, s1, A::mad(n01.f, s3, A::mad(n10.f, s2, A::mul(n00.f, s4))))
  const T ex = PBD_GATHER(ex), ey = PBD_GATHER(ey), ez = PBD_GATHER(ez);
  const T bx = PBD_GATHER(bx), by = PBD_GATHER(by), bz = PBD_GATHER(bz);
#undef PBD_GATHER
  // Boris rotation, pic2d.f90:969-996
  const T c0 = sp ? a.c0[1] : a.c0[0], c1 = sp ? a.c1[1] : a.c1[0];
  const T umx = A::mad(c1, ex, pux), umy = A::mad(c1, ey, puy), umz = A::mad(c1, ez, puz);
  T gama = A::sqrt(A::mad(umz, umz, A::mad(umy, umy, A::mad(umx, umx, one))));
  const T c2 = A::div(c0, gama);
  const T tx = A::mul(c2, bx), ty = A::mul(c2, by), tz = A::mul(c2, bz);
  const T t2 = A::div(T(2), A::mad(tz, tz, A::mad(ty, ty, A::mad(tx, tx, one))));
  const T sx = A::mul(t2, tx), sy = A::mul(t2, ty), sz = A::mul(t2, tz);
  const bool cb = (a.compat & 1) != 0;  // rotate the pre-kick momentum (pic2d.f90:985-987)
  const T vx = cb ? pux : umx, vy = cb ? puy : umy, vz0 = cb ? puz : umz;
  const T u0x = A::add(umx, A::mad(vy, tz, -A::mul(vz0, ty)));
  const T u0y = A::add(umy, A::mad(vz0, tx, -A::mul(vx, tz)));
  const T u0z = A::add(umz, A::mad(vx, ty, -A::mul(vy, tx)));
  const T upx = A::add(umx, A::mad(u0y, sz, -A::mul(u0z, sy)));
  const T upy = A::add(umy, A::mad(u0z, sx, -A::mul(u0x, sz)));
  const T upz = A::add(umz, A::mad(u0x, sy, -A::mul(u0y, sx)));
  const T ux = A::mad(c1, ex, upx), uy = A::mad(c1, ey, upy), uz = A::mad(c1, ez, upz);
  const T usq = A::mad(uz, uz, A::mad(uy, uy, A::mul(ux, ux)));
  gama = A::sqrt(A::mad(uz, uz, A::mad(uy, uy, A::mad(ux, ux, one))));
  // move, pic2d.f90:1002-1023
  const T c3 = A::div(a.dtcva, gama);
  const T dx1 = A::mad(A::mul(c3, ux), a.idx, px);
  const T dy1 = A::mad(A::mul(c3, uy), a.idy, py);
  int dcx = 0, dcy = 0;
  T dx2 = dx1, dy2 = dy1;
  if (A::abs(dx1) > half) {
    dcx = dx1 >= T(0) ? 1 : -1;
    dx2 = A::add(dx1, dx1 >= T(0) ? -one : one);
  }
  if (A::abs(dy1) > half) {
    dcy = dy1 >= T(0) ? 1 : -1;
    dy2 = A::add(dy1, dy1 >= T(0) ? -one : one);
  }
  int st = 0;
  if (A::abs(dx1) > T(1.5) || A::abs(dy1) > T(1.5)) st |= 1;
  if (!(gama < T(3.0e38))) st |= 2;  // NaN or overflow
  // vz for jz: plain uses uz*cva/gama (pic2d.f90:1028); mixed keeps uz/gama
  // and applies cva when the fixed-point sum is converted.
  const T vz = MIXED ? A::div(uz, gama) : A::div(A::mul(uz, a.cva), gama);
  const T msp = sp ? a.ms[1] : a.ms[0];
  o.ke = MIXED ? (double)A::mul(A::div(usq, A::add(gama, one)), msp)
               : (double)A::mul(A::sub(gama, one), msp);

  // ---- charge-conserving deposit terms (pic2d.f90:1237-1295), indices
  // relative to the old cell: i1 = j1 = 0, i2 = dcx, j2 = dcy.
  const T qx = sp ? a.qx[1] : a.qx[0], qy = sp ? a.qy[1] : a.qy[0], qq = sp ? a.q[1] : a.q[0];
  const T im = A::mul(A::add(A::add(A::add(T(dcx), px), dx2), one), half);
  const T jm = A::mul(A::add(A::add(A::add(T(dcy), py), dy2), one), half);
  const T ir = fmin(T(dcx < 0 ? dcx : 0) + one, fmax(T(dcx > 0 ? dcx : 0), im));
  const T jr = fmin(T(dcy < 0 ? dcy : 0) + one, fmax(T(dcy > 0 ? dcy : 0), jm));
  const T fx1 = A::mul(qx, A::sub(A::sub(ir, px), half));
  const T fy1 = A::mul(qy, A::sub(A::sub(jr, py), half));
  const T fx2 = A::mul(qx, A::sub(A::add(A::add(T(dcx), dx2), half), ir));
  const T fy2 = A::mul(qy, A::sub(A::add(A::add(T(dcy), dy2), half), jr));
  const T wx1 = A::mul(A::add(A::add(ir, px), half), half);
  const T wy1 = A::mul(A::add(A::add(jr, py), half), half);
  const T wx2 = A::mul(A::add(A::add(A::sub(ir, T(dcx)), dx2), half), half);
  const T wy2 = A::mul(A::add(A::add(A::sub(jr, T(dcy)), dy2), half), half);
  o.e[0] = A::mul(fx1, A::sub(one, wy1));  // jx (0, 0)
  o.e[1] = A::mul(fx1, wy1);               // jx (0, 1)
  o.e[2] = A::mul(fx2, A::sub(one, wy2));  // jx (dcx, dcy)
  o.e[3] = A::mul(fx2, wy2);               // jx (dcx, dcy+1)
  o.e[4] = A::mul(fy1, A::sub(one, wx1));  // jy (0, 0)
  o.e[5] = A::mul(fy1, wx1);               // jy (1, 0)
  o.e[6] = A::mul(fy2, A::sub(one, wx2));  // jy (dcx, dcy)
  o.e[7] = A::mul(fy2, wx2);               // jy (dcx+1, dcy)
  T dimid = A::sub(im, half), djmid = A::sub(jm, half);
  const int di = dimid >= T(0) ? 1 : -1, dj = djmid >= T(0) ? 1 : -1;
  dimid = A::abs(dimid);
  djmid = A::abs(djmid);
  {
    const T z1 = A::mul(dimid, djmid);
    const T z2 = A::sub(dimid, z1);
    const T z3 = A::sub(djmid, z1);
    const T z4 = A::sub(A::sub(A::sub(one, z1), z2), z3);
    const T quz = A::mul(qq, vz);
    o.e[8] = A::mul(quz, z4);   // jz (0, 0)
    o.e[9] = A::mul(quz, z2);   // jz (di, 0)
    o.e[10] = A::mul(quz, z3);  // jz (0, dj)
    o.e[11] = A::mul(quz, z1);  // jz (di, dj)
  }
  {
    const bool cr = (a.compat & 4) != 0;  // mirrored weights (pic2d.f90:1285-1288)
    const T rx = cr ? A::sub(half, px) : A::add(half, px);
    const T ry = cr ? A::sub(half, py) : A::add(half, py);
    const T r1 = A::mul(rx, ry);
    const T r2 = A::sub(rx, r1);
    const T r3 = A::sub(ry, r1);
    const T r4 = A::sub(A::sub(A::sub(one, r1), r2), r3);
    o.e[12] = A::mul(r4, qq);  // rho (0, 0)
    o.e[13] = A::mul(r2, qq);  // rho (1, 0)
    o.e[14] = A::mul(r3, qq);  // rho (0, 1)
    o.e[15] = A::mul(r1, qq);  // rho (1, 1)
  }

  // ---- boundaries: x periodic (pic2d.f90:1032); y periodic (the 1-rank
  // exchange of pic2d.f90:1033-1146 reduces to a wrap) or specular walls.
  int nix = ix + dcx;
  nix = nix < 0 ? nix + a.mx : (nix >= a.mx ? nix - a.mx : nix);
  int niy = iy + dcy;
  T ruy = uy, rdy = dy2;
  if (a.ybc == 0) {
    niy = niy < 0 ? niy + a.my : (niy >= a.my ? niy - a.my : niy);
  } else if (niy < 0 || niy >= a.my) {
    niy = niy < 0 ? 0 : a.my - 1;
    rdy = -dy2;
    ruy = -uy;
  }
  o.cw = cw_make(nix, niy, sp);
  o.dx = dx2;
  o.dy = rdy;
  o.ux = ux;
  o.uy = ruy;
  o.uz = uz;
  o.ix = ix;
  o.iy = iy;
  o.dcx = dcx;
  o.dcy = dcy;
  o.di = di;
  o.dj = dj;
  o.status = st;
}

// Relative node (x, y) of deposit term k (old cell at (0, 0)).
__device__ __forceinline__ void term_node(int k, int dcx, int dcy, int di, int dj, int* x, int* y) {
  switch (k) {
    case 0: *x = 0; *y = 0; break;
    case 1: *x = 0; *y = 1; break;
    case 2: *x = dcx; *y = dcy; break;
    case 3: *x = dcx; *y = dcy + 1; break;
    case 4: *x = 0; *y = 0; break;
    case 5: *x = 1; *y = 0; break;
    case 6: *x = dcx; *y = dcy; break;
    case 7: *x = dcx + 1; *y = dcy; break;
    case 8: *x = 0; *y = 0; break;
    case 9: *x = di; *y = 0; break;
    case 10: *x = 0; *y = dj; break;
    case 11: *x = di; *y = dj; break;
    case 12: *x = 0; *y = 0; break;
    case 13: *x = 1; *y = 0; break;
    case 14: *x = 0; *y = 1; break;
    default: *x = 1; *y = 1; break;
  }
}

// Global node of unwrapped 0-based node (gx, gy) of component c: periodic x,
// periodic y or wall images (node rows of jx/rho mirror about rows 0 and my,
// half rows of jy/jz about -1/2 and my-1/2, jy changing sign). Returns false
// for the jy column the reference never folds (compat).
__device__ __forceinline__ bool map_current(int c, int gx, int gy, int mx, int my, int S, int ybc,
                                            int compat, long long* idx, int* sgn) {
  if (c == JY && (compat & 2) && gx == mx + 1) return false;
  int x = gx < 0 ? gx + mx : (gx >= mx ? gx - mx : gx);
  int y = gy, s = 1;
  if (ybc == 0) {
    y = gy < 0 ? gy + my : (gy >= my ? gy - my : gy);
  } else if (c == JX || c == RHO) {
    if (gy < 0) y = -gy;
    else if (gy > my) y = 2 * my - gy;
  } else {
    if (gy < 0) {
      y = -1 - gy;
      s = c == JY ? -1 : 1;
    } else if (gy > my - 1) {
      y = 2 * my - 1 - gy;
      s = c == JY ? -1 : 1;
    }
  }
  *idx = ((long long)c * mx + x) * S + y;
  *sgn = s;
  return true;
}

__device__ __forceinline__ void acc_add(double* p, double v) { atomicAdd(p, v); }
__device__ __forceinline__ void acc_add(long long* p, long long v) {
  atomicAdd(reinterpret_cast<unsigned long long*>(p), (unsigned long long)v);
}

template <class T, bool MIXED>
__device__ __forceinline__ typename std::conditional<MIXED, long long, double>::type to_acc(T v) {
  if constexpr (MIXED) {
    return __float2ll_rn(__fmul_rn((float)v, FIX_SCALE));
  } else {
    return (double)v;
  }
}

template <class T, bool MIXED>
__global__ void __launch_bounds__(NTHREADS) k_push(PushParams<T> a) {
  using Acc = typename std::conditional<MIXED, long long, double>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Acc* win = reinterpret_cast<Acc*>(smem_raw);  // [4 comps][4 cols][WR rows]
  __shared__ double red[32];
  const int TY = a.tile_rows, WR = TY + 3;
  const int t = blockIdx.x;
  const int ixt = t / a.tiles_per_col;
  const int y0 = (t - ixt * a.tiles_per_col) * TY;
  const int y1 = min(y0 + TY, a.my);
  for (int e = threadIdx.x; e < 16 * WR; e += blockDim.x) win[e] = Acc(0);
  __syncthreads();
  Acc* gacc = reinterpret_cast<Acc*>(a.jacc);
  const int pbeg = a.tile_off[t], pend = a.tile_off[t + 1];
  const unsigned lane = lane_id();
  double ke_e = 0.0, ke_i = 0.0;
  int status = 0;
  for (int base = pbeg; base < pend; base += NTHREADS) {
    const int p = base + (int)threadIdx.x;
    int key = -1 - (int)lane;  // unique negative: never merges, never deposits
    T v[17];
#pragma unroll
    for (int k = 0; k < 17; ++k) v[k] = T(0);
    if (p < pend) {
      Pushed<T> o;
      push_one<T, MIXED>(a, a.cell[p], a.dx[p], a.dy[p], a.ux[p], a.uy[p], a.uz[p], o);
      const bool inwin = o.ix == ixt && o.iy >= y0 && o.iy < y1;
      if (inwin && o.dcx == 0 && o.dcy == 0) {
        key = o.iy - y0;
        v[0] = o.e[0] + o.e[2];  // jx (0,0)
        v[1] = o.e[1] + o.e[3];  // jx (0,1)
        v[2] = o.e[4] + o.e[6];  // jy (0,0)
        v[3] = o.e[5] + o.e[7];  // jy (1,0)
        // jz on the 3x3 block around the cell: index 4 + (x+1)*3 + (y+1);
        // (0,0) <- e8, (di,0) <- e9, (0,dj) <- e10, (di,dj) <- e11, di, dj = +-1
#pragma unroll
        for (int xx = -1; xx <= 1; ++xx)
#pragma unroll
          for (int yy = -1; yy <= 1; ++yy) {
            T z = T(0);
            if (xx == 0 && yy == 0) z = o.e[8];
            if (xx != 0 && yy == 0 && xx == o.di) z = o.e[9];
            if (xx == 0 && yy != 0 && yy == o.dj) z = o.e[10];
            if (xx != 0 && yy != 0 && xx == o.di && yy == o.dj) z = o.e[11];
            v[4 + (xx + 1) * 3 + (yy + 1)] = z;
          }
        v[13] = o.e[12];
        v[14] = o.e[13];
        v[15] = o.e[14];
        v[16] = o.e[15];
      } else if (inwin) {
        const int wy0 = o.iy - y0 + 1;
#pragma unroll
        for (int k = 0; k < 16; ++k) {
          int rx, ry;
          term_node(k, o.dcx, o.dcy, o.di, o.dj, &rx, &ry);
          const int c = k >> 2;
          acc_add(&win[(c * 4 + 1 + rx) * WR + wy0 + ry], to_acc<T, MIXED>(o.e[k]));
        }
      } else {
        status |= 4;
#pragma unroll
        for (int k = 0; k < 16; ++k) {
          int rx, ry;
          term_node(k, o.dcx, o.dcy, o.di, o.dj, &rx, &ry);
          const int c = k >> 2;
          long long gi;
          int sg;
          if (map_current(c, o.ix + rx, o.iy + ry, a.mx, a.my, a.S, a.ybc, a.compat, &gi, &sg))
            acc_add(&gacc[gi], to_acc<T, MIXED>(sg < 0 ? -o.e[k] : o.e[k]));
        }
      }
      a.cell[p] = o.cw;
      a.dx[p] = o.dx;
      a.dy[p] = o.dy;
      a.ux[p] = o.ux;
      a.uy[p] = o.uy;
      a.uz[p] = o.uz;
      if (cw_sp(o.cw)) ke_e += o.ke;
      else ke_i += o.ke;
      status |= o.status;
    }
    // Sum the stencils of lanes that share a cell; the last lane of each run deposits.
    const int kprev = __shfl_up_sync(FULL, key, 1);
    const unsigned head = (lane == 0) || (kprev != key);
    warp_segmented_scan<T, 17>(v, head);
    const unsigned head_next = __shfl_down_sync(FULL, head, 1);
    if (key >= 0 && (lane == 31 || head_next)) {
      const int wy = key + 1;
      acc_add(&win[(0 * 4 + 1) * WR + wy], to_acc<T, MIXED>(v[0]));
      acc_add(&win[(0 * 4 + 1) * WR + wy + 1], to_acc<T, MIXED>(v[1]));
      acc_add(&win[(1 * 4 + 1) * WR + wy], to_acc<T, MIXED>(v[2]));
      acc_add(&win[(1 * 4 + 2) * WR + wy], to_acc<T, MIXED>(v[3]));
#pragma unroll
      for (int xx = 0; xx < 3; ++xx)
#pragma unroll
        for (int yy = 0; yy < 3; ++yy) {
          const T z = v[4 + xx * 3 + yy];
          if (z != T(0)) acc_add(&win[(2 * 4 + xx) * WR + wy - 1 + yy], to_acc<T, MIXED>(z));
        }
      acc_add(&win[(3 * 4 + 1) * WR + wy], to_acc<T, MIXED>(v[13]));
      acc_add(&win[(3 * 4 + 2) * WR + wy], to_acc<T, MIXED>(v[14]));
      acc_add(&win[(3 * 4 + 1) * WR + wy + 1], to_acc<T, MIXED>(v[15]));
      acc_add(&win[(3 * 4 + 2) * WR + wy + 1], to_acc<T, MIXED>(v[16]));
    }
  }
  __syncthreads();
  // Fold the window into the global current.
  for (int e = threadIdx.x; e < 16 * WR; e += blockDim.x) {
    const Acc val = win[e];
    if (val == Acc(0)) continue;
    const int c = e / (4 * WR);
    const int r = e - c * 4 * WR;
    const int wx = r / WR, wy = r - wx * WR;
    long long gi;
    int sg;
    if (map_current(c, ixt - 1 + wx, y0 - 1 + wy, a.mx, a.my, a.S, a.ybc, a.compat, &gi, &sg))
      acc_add(&gacc[gi], sg < 0 ? -val : val);
  }
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
