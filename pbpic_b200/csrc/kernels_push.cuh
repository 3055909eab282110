// Particle push: bilinear field gather, Boris rotation, move with cell
// crossing, Umeda zig-zag current deposit, x wrap and y wrap or wall
// reflection -- the particle loop of pusher (pic2d.f90:934-1063) and
// currentdeposit (pic2d.f90:1226-1296).
//
// Work decomposition: a tile is a run of `tile_rows` cells of one column
// (contiguous in the cell-sorted order); one block pushes the particles of one
// tile. Each thread takes 8 consecutive particles per pass (4 in the plain
// form), written in groups of 4 with 128-bit stores; they are read the same way
// in place, or one by one through the sort's permutation. The mixed form
// gathers a cell's 4 nodes from the cell's record (k_cell_records), the plain
// form from the node grid. Consecutive particles of a sorted array share their
// cell, so a thread sums the deposit stencils of its particles in registers
// before touching memory.
//
// Deposit: the zig-zag move of a particle splits at the relay point into a
// segment in the old cell and one in the new cell. Everything attached to the
// old cell -- the first segment's jx/jy (and the second's when the particle
// does not cross), jz on the 3x3 nodes around the cell, rho -- forms a
// 17-value stencil. At the end of a pass the lanes of a warp that share a
// cell (a run of lanes: the keys do not decrease across a sorted array) are
// summed: each lane stages its stencil in shared memory and 17 lanes add up
// the run's columns in lane order, one stencil entry each (a thread whose
// particles change cell keeps its first cell's part in a second column, joined
// to the run it continues). Each run's sum is added to a shared-memory window
// by 17 lanes at once. A crossing particle adds its second segment (4 values) on its own. The window (4 node columns x tile_rows + 3 node rows) is folded
// into the global current at the end, with the periodic wrap and the wall
// images. Particles outside their tile (array not sorted) add straight to
// global memory.
//
// The window holds int64 fixed-point sums (mixed form), and 64-bit shared
// atomics are slow. A crossing particle's four second-segment values (each
// below 2^32 in fixed point) therefore go to a separate pair of 32-bit
// windows: the low 17 bits to an unsigned sum and the rest (signed) to a
// second sum, both with native 32-bit atomics. With at most 32767 particles
// in the tile neither sum can overflow (32767 * (2^17 - 1) < 2^32 and
// 32767 * 2^15 < 2^31); larger tiles use the 64-bit window. Integer sums do
// not depend on the order of the atomics, so the result is the same bits
// either way.
//
// With GATHER the input is the previous step's arrays in their own order and
// the fused sort's permutation (sorted position -> element): the push reads
// each particle through it and writes the result in sorted position to a
// second set of arrays, so that the sort never moves the particle data.
//
// With HIST the kernel also counts the new cells of its particles in the
// tile's window (the 3x3 neighbourhood of the tile), the first half of the
// fused counting sort (kernels_sort.cuh). The input is sorted, so the counts
// start from its cell counts (cell_off) and only a crossing particle moves a
// count, from its old cell's bin to its new one.
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
  const T* ng;      // node fields (mx+1) x (my+1) x 8: ex ey ez 0 bx by bz 0
  const T* cg;      // mixed form: per-cell gather records mx x my x 24 (k_cell_records)
  void* jacc;       // 4 planes (jx, jy, jz, rho) of mx x S accumulators
  int32_t* tilecnt; // [ntiles][3*(tile_rows+2)] new-cell counts (HIST)
  const int32_t* cell_off;  // [mx*my + 1] cell offsets of the sorted input (HIST)
  // GATHER: particle p of the sorted order is element src[p] of the input
  // arrays above; its result goes to element p of the output arrays.
  const int32_t* src;
  uint32_t* cell_o;
  T *dx_o, *dy_o, *ux_o, *uy_o, *uz_o;
  const int32_t* pid_i;  // tracked ids, moved with the particles (null: none)
  int32_t* pid_o;
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

__device__ __forceinline__ Node6<double> load_node_staged(const double* g) {
  const double2* p = reinterpret_cast<const double2*>(g);
  const double2 a = p[0], b = p[1], c = p[2], d = p[3];
  return Node6<double>{a.x, a.y, b.x, c.x, c.y, d.x};
}

// Mixed form: a cell's gather record (k_cell_records) holds, per field (ex ey
// ez bx by bz, one aligned 16-byte group each), the bilinear coefficients
// (A, B, C, D) of the field over the cell, f(x, y) = A + B x + C y + D x y for
// the in-cell offsets x, y in [-1/2, 1/2): the same bilinear interpolation of
// the 4 nodes as pic2d.f90:948-963, 3 FMAs per field. PBPIC_CELL_COEF = 0
// (device_common.cuh) keeps the 4 nodes themselves instead.

struct CellCoef {
  float4 f[6];
};
__device__ __forceinline__ void load_coef(const float* r, CellCoef& c) {
  const float4* q = reinterpret_cast<const float4*>(r);
#pragma unroll
  for (int k = 0; k < 6; ++k) c.f[k] = __ldg(q + k);
}
// The same from the tile's records staged in shared memory.
__device__ __forceinline__ void load_coef_staged(const float* r, CellCoef& c) {
  const float4* q = reinterpret_cast<const float4*>(r);
#pragma unroll
  for (int k = 0; k < 6; ++k) c.f[k] = q[k];
}
__device__ __forceinline__ float coef_at(const float4& q, float x, float y) {
  return __fmaf_rn(__fmaf_rn(q.w, x, q.z), y, __fmaf_rn(q.y, x, q.x));
}

// The 4 gather nodes of a cell from its record: n00, n01, n10, n11, each ex ey
// ez bx by bz (6 aligned 16-byte loads from one address).
__device__ __forceinline__ void load_cell(const float* r, Node6<float>& n00, Node6<float>& n01, Node6<float>& n10,
                                          Node6<float>& n11) {
  const float4* q = reinterpret_cast<const float4*>(r);
  const float4 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2), d = __ldg(q + 3), e = __ldg(q + 4), f = __ldg(q + 5);
  n00 = Node6<float>{a.x, a.y, a.z, a.w, b.x, b.y};
  n01 = Node6<float>{b.z, b.w, c.x, c.y, c.z, c.w};
  n10 = Node6<float>{d.x, d.y, d.z, d.w, e.x, e.y};
  n11 = Node6<float>{e.z, e.w, f.x, f.y, f.z, f.w};
}

__device__ __forceinline__ void ld4(const float* p, float (&v)[4]) {
  const float4 x = *reinterpret_cast<const float4*>(p);
  v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
}
__device__ __forceinline__ void ld4(const double* p, double (&v)[4]) {
  const double2 a = reinterpret_cast<const double2*>(p)[0], b = reinterpret_cast<const double2*>(p)[1];
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
__device__ __forceinline__ void ld4(const uint32_t* p, uint32_t (&v)[4]) {
  const uint4 x = *reinterpret_cast<const uint4*>(p);
  v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
}
__device__ __forceinline__ void st4(float* p, const float (&v)[4]) {
  *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void st4(double* p, const double (&v)[4]) {
  reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
  reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
}
__device__ __forceinline__ void st4(uint32_t* p, const uint32_t (&v)[4]) {
  *reinterpret_cast<uint4*>(p) = make_uint4(v[0], v[1], v[2], v[3]);
}

// Bulk copy of a tile's gather records (mixed form) or node-grid columns
// (plain form) into shared memory (the copy engine's cp.async.bulk,
// completion counted on an mbarrier; no multicast). The wait is bounded: a
// copy that has not landed after PUSH_WAIT_TRIES polls raises
// PBPIC_STATUS_COPY_TIMEOUT and the push reads global memory instead.
#ifndef PBPIC_PUSH_STAGE_RECS
#define PBPIC_PUSH_STAGE_RECS 1
#endif
#ifndef PBPIC_PUSH_STAGE_NODES
#define PBPIC_PUSH_STAGE_NODES 1  // plain form: the tile's two node-grid columns
#endif
constexpr int PUSH_WAIT_TRIES = 1 << 22;
__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* b) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_addr(b)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
// Announces `bytes` of bulk copies on mbarrier b (after the block's earlier
// reads of the destination, ordered by a barrier, and this fence).
__device__ __forceinline__ void bulk_expect(uint64_t* b, unsigned bytes) {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_copy(void* dst, const void* src, unsigned bytes, uint64_t* b) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(b))
               : "memory");
}
__device__ __forceinline__ bool mbar_wait(uint64_t* b, unsigned parity) {
  for (int i = 0; i < PUSH_WAIT_TRIES; ++i) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_addr(b)), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

// Reciprocal square root and quotient of the push. Plain form, exact order
// (COMPAT instances): correctly rounded square roots and quotients, as the
// reference's expressions. Plain form otherwise: 1/gamma from CUDA's double
// rsqrt and the rotation's 2/(1 + t^2) by Newton steps from the hardware
// reciprocal estimate (push_two_over), so that the push's chain holds no FP64
// division instead of four quotients and two square roots (results within a
// few ulp of the exact order). Mixed form: the hardware reciprocal square root
// and fast division (deterministic, about 2 ulp).
__device__ __forceinline__ float push_rsqrt(float x) { return rsqrtf(x); }
__device__ __forceinline__ double push_rsqrt(double x) { return rsqrt(x); }
__device__ __forceinline__ float push_fdiv(float a, float b) { return __fdividef(a, b); }

// Plain form, fast mode: 2/x for x = 1 + |t|^2 >= 1 by Newton-Raphson
// refinement of the hardware reciprocal estimate (rcp.approx.ftz.f64): two
// steps y <- y + y (1 - x y), each squaring the relative error, then one
// residual correction of the quotient, q <- q + (2 - x q) y (Markstein's
// correction); a few ulp from the correctly rounded quotient at most.
__device__ __forceinline__ double push_two_over(double x) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  double e = __fma_rn(-x, y, 1.0);
  y = __fma_rn(y, e, y);
  e = __fma_rn(-x, y, 1.0);
  y = __fma_rn(y, e, y);
  const double q = __dmul_rn(2.0, y);
  return __fma_rn(__fma_rn(-x, q, 2.0), y, q);
}

// Outcome of pushing one particle.
template <class T>
struct Pushed {
  uint32_t cw;           // new cell word
  T dx, dy, ux, uy, uz;  // new state (after reflection)
  int dcx, dcy, di, dj;  // cell steps and jz quadrant
  T e[16];               // deposit terms: jx 4, jy 4, jz 4, rho 4 (the exact order fills all 16; the
                         // cell-relative form only the second segment's e[2], e[3], e[6], e[7] and
                         // the stencil quantities below)
  // mixed form, cell-stencil form of the same deposit: jx at (0,0), (0,1) is
  // ja*(1-jw), ja*jw (first segment only for a crossing particle, the whole
  // move otherwise), jy at (0,0), (1,0) is jb*(1-jv), jb*jv; jz is quz times
  // the outer product of the x and y midpoint weights (1-zdx at 0, zdx at
  // di; 1-zdy at 0, zdy at dj)
  T ja, jw, jb, jv, quz, zdx, zdy;
  T q, rw[4];            // charge and the rho weights of e[12..15] (e[12 + k] = q * rw[k])
  T ke;                  // kinetic energy (gamma - 1) ms
  int status;
};

template <class T, bool MIXED, bool COMPAT = true>
__device__ __forceinline__ void push_core(const PushParams<T>& a, int sp, int ix, int iy, T px, T py, T pux, T puy,
                                          T puz, T ex, T ey, T ez, T bx, T by, T bz, Pushed<T>& o);

// A species constant of the push (index 0 ion, 1 electron): an indexed read of
// the parameter array (PBPIC_PUSH_IDXCONST = 1) or a select of its two entries.
#ifndef PBPIC_PUSH_IDXCONST
#define PBPIC_PUSH_IDXCONST 0
#endif
#if PBPIC_PUSH_IDXCONST
#define PBD_SPECIES(arr, sp) (arr)[(sp)]
#else
#define PBD_SPECIES(arr, sp) ((sp) ? (arr)[1] : (arr)[0])
#endif

// Push of one particle whose gather nodes are n00 (ix,iy), n01 (ix,iy+1),
// n10 (ix+1,iy), n11 (ix+1,iy+1). MIXED is only instantiated with T = float.
// COMPAT = false compiles the step for a configuration without the compat
// switches of the push (the rho weights are then the gather weights) and, in
// the plain form, forms 1/gamma with rsqrt and contracts a*b+c into one
// fused multiply-add; COMPAT = true keeps the reference's correctly rounded
// quotients and square roots and its separately rounded products and sums,
// bit for bit.
template <class T, bool MIXED, bool COMPAT = true>
__device__ __forceinline__ void push_one(const PushParams<T>& a, int sp, int ix, int iy, T px, T py, T pux,
                                         T puy, T puz, const Node6<T>& n00, const Node6<T>& n01,
                                         const Node6<T>& n10, const Node6<T>& n11, Pushed<T>& o) {
  using A = M<T, MIXED || !COMPAT>;  // fused multiply-adds except in the exact order
  const T half = T(0.5), one = T(1);
  // CIC weights, pic2d.f90:948-951
  const T axw = A::add(half, px), ayw = A::add(half, py);
  const T s1 = A::mul(axw, ayw);
  const T s2 = A::sub(axw, s1);
  const T s3 = A::sub(ayw, s1);
  const T s4 = A::sub(A::sub(A::sub(one, s1), s2), s3);
  // gather, pic2d.f90:952-963, summed in the reference's order
#define PBD_GATHER(f) A::mad(n11.f, s1, A::mad(n01.f, s3, A::mad(n10.f, s2, A::mul(n00.f, s4))))
  const T ex = PBD_GATHER(ex), ey = PBD_GATHER(ey), ez = PBD_GATHER(ez);
  const T bx = PBD_GATHER(bx), by = PBD_GATHER(by), bz = PBD_GATHER(bz);
#undef PBD_GATHER
  push_core<T, MIXED, COMPAT>(a, sp, ix, iy, px, py, pux, puy, puz, ex, ey, ez, bx, by, bz, o);
}

// Mixed form, from the cell's bilinear coefficients.
template <bool COMPAT = true>
__device__ __forceinline__ void push_one_coef(const PushParams<float>& a, int sp, int ix, int iy, float px, float py,
                                              float pux, float puy, float puz, const CellCoef& c, Pushed<float>& o) {
  push_core<float, true, COMPAT>(a, sp, ix, iy, px, py, pux, puy, puz, coef_at(c.f[0], px, py),
                                 coef_at(c.f[1], px, py), coef_at(c.f[2], px, py), coef_at(c.f[3], px, py),
                                 coef_at(c.f[4], px, py), coef_at(c.f[5], px, py), o);
}

// Everything after the gather: Boris, move, deposit terms, boundaries.
template <class T, bool MIXED, bool COMPAT>
__device__ __forceinline__ void push_core(const PushParams<T>& a, int sp, int ix, int iy, T px, T py, T pux, T puy,
                                          T puz, T ex, T ey, T ez, T bx, T by, T bz, Pushed<T>& o) {
  using A = M<T, MIXED || !COMPAT>;  // fused multiply-adds except in the exact order
  const T half = T(0.5), one = T(1);
  // Boris rotation, pic2d.f90:969-996
  const T c0 = PBD_SPECIES(a.c0, sp), c1 = PBD_SPECIES(a.c1, sp);
  const T umx = A::mad(c1, ex, pux), umy = A::mad(c1, ey, puy), umz = A::mad(c1, ez, puz);
  const T g2m = A::mad(umz, umz, A::mad(umy, umy, A::mad(umx, umx, one)));
  T c2, t2;
  if constexpr (MIXED || !COMPAT) {
    c2 = A::mul(c0, push_rsqrt(g2m));
  } else {
    c2 = A::div(c0, A::sqrt(g2m));
  }
  const T tx = A::mul(c2, bx), ty = A::mul(c2, by), tz = A::mul(c2, bz);
  const T tsq1 = A::mad(tz, tz, A::mad(ty, ty, A::mad(tx, tx, one)));
  if constexpr (MIXED) {
    t2 = push_fdiv(T(2), tsq1);
  } else if constexpr (!COMPAT) {
    t2 = push_two_over(tsq1);
  } else {
    t2 = A::div(T(2), tsq1);
  }
  const T sx = A::mul(t2, tx), sy = A::mul(t2, ty), sz = A::mul(t2, tz);
  const bool cb = COMPAT && (a.compat & 1) != 0;  // rotate the pre-kick momentum (pic2d.f90:985-987)
  const T vx = cb ? pux : umx, vy = cb ? puy : umy, vz0 = cb ? puz : umz;
  T u0x, u0y, u0z, upx, upy, upz;
  if constexpr (MIXED || !COMPAT) {  // u' = u- + v x t and u+ = u- + u' x s as two fused multiply-adds a component
    u0x = A::mad(vy, tz, A::mad(-vz0, ty, umx));
    u0y = A::mad(vz0, tx, A::mad(-vx, tz, umy));
    u0z = A::mad(vx, ty, A::mad(-vy, tx, umz));
    upx = A::mad(u0y, sz, A::mad(-u0z, sy, umx));
    upy = A::mad(u0z, sx, A::mad(-u0x, sz, umy));
    upz = A::mad(u0x, sy, A::mad(-u0y, sx, umz));
  } else {
    u0x = A::add(umx, A::mad(vy, tz, -A::mul(vz0, ty)));
    u0y = A::add(umy, A::mad(vz0, tx, -A::mul(vx, tz)));
    u0z = A::add(umz, A::mad(vx, ty, -A::mul(vy, tx)));
    upx = A::add(umx, A::mad(u0y, sz, -A::mul(u0z, sy)));
    upy = A::add(umy, A::mad(u0z, sx, -A::mul(u0x, sz)));
    upz = A::add(umz, A::mad(u0x, sy, -A::mul(u0y, sx)));
  }
  const T ux = A::mad(c1, ex, upx), uy = A::mad(c1, ey, upy), uz = A::mad(c1, ez, upz);
  const T g2 = A::mad(uz, uz, A::mad(uy, uy, A::mad(ux, ux, one)));
  T c3, vz, gama;
  if constexpr (MIXED) {
    const T rg = push_rsqrt(g2);
    gama = A::mul(g2, rg);
    c3 = A::mul(a.dtcva, rg);
    vz = A::mul(uz, rg);  // uz/gamma; cva enters when the fixed-point sum is converted
  } else if constexpr (!COMPAT) {
    const T rg = push_rsqrt(g2);
    gama = A::mul(g2, rg);
    c3 = A::mul(a.dtcva, rg);              // pic2d.f90:1004
    vz = A::mul(A::mul(uz, a.cva), rg);    // pic2d.f90:1028
  } else {
    gama = A::sqrt(g2);
    c3 = A::div(a.dtcva, gama);            // pic2d.f90:1004
    vz = A::div(A::mul(uz, a.cva), gama);  // pic2d.f90:1028
  }
  // move, pic2d.f90:1005-1023
  const T dx1 = A::mad(A::mul(c3, ux), a.idx, px);
  const T dy1 = A::mad(A::mul(c3, uy), a.idy, py);
  // cell steps (pic2d.f90:1008-1023), also as floating-point values for the deposit
  const T fdcx = dx1 > half ? one : (dx1 < -half ? -one : T(0));
  const T fdcy = dy1 > half ? one : (dy1 < -half ? -one : T(0));
  const int dcx = dx1 > half ? 1 : (dx1 < -half ? -1 : 0);
  const int dcy = dy1 > half ? 1 : (dy1 < -half ? -1 : 0);
  const T dx2 = A::sub(dx1, fdcx);
  const T dy2 = A::sub(dy1, fdcy);
  int st = 0;
  if (A::abs(dx1) > T(1.5) || A::abs(dy1) > T(1.5)) st |= 1;
  if (!(gama < T(3.0e38))) st |= 2;  // NaN or overflow
  const T msp = PBD_SPECIES(a.ms, sp);
  if constexpr (MIXED) {  // (gamma - 1) = u^2 / (gamma + 1) avoids the cancellation of gamma - 1 in FP32
    const T usq = A::mad(uz, uz, A::mad(uy, uy, A::mul(ux, ux)));
    o.ke = A::mul(push_fdiv(usq, A::add(gama, one)), msp);
  } else {
    o.ke = A::mul(A::sub(gama, one), msp);  // pic2d.f90:1062
  }

  // ---- charge-conserving deposit terms (pic2d.f90:1237-1295), indices
  // relative to the old cell: i1 = j1 = 0, i2 = dcx, j2 = dcy.
  T qx, qy, qq;
  if constexpr (MIXED) {  // the mixed form's charges are the unit charges: +1 ion, -1 electron (the sign bit)
    qq = __uint_as_float(0x3f800000u | ((unsigned)sp << 31));
    qx = qq;
    qy = qq;
  } else {
    qx = PBD_SPECIES(a.qx, sp);
    qy = PBD_SPECIES(a.qy, sp);
    qq = PBD_SPECIES(a.q, sp);
  }
  T im, jm;
  if constexpr (MIXED || !COMPAT) {  // cell-relative form (the plain form's exact order below)
    // Positions in cell units from the old cell's lower-left node: start
    // xs = dx0 + 1/2, end xe = dx1 + 1/2 (= dcx + dx2 + 1/2). The relay point
    // is the midpoint for a particle that stays, else the face it crosses.
    const T xs = A::add(px, half), xe = A::add(dx1, half);
    const T ys = A::add(py, half), ye = A::add(dy1, half);
    im = A::mul(A::add(xs, xe), half);
    jm = A::mul(A::add(ys, ye), half);
    const T ir = dcx == 0 ? im : (dcx > 0 ? one : T(0));
    const T jr = dcy == 0 ? jm : (dcy > 0 ? one : T(0));
    const T fx1 = A::mul(qx, A::sub(ir, xs)), fx2 = A::mul(qx, A::sub(xe, ir));
    const T fy1 = A::mul(qy, A::sub(jr, ys)), fy2 = A::mul(qy, A::sub(ye, jr));
    const T wx1 = A::mul(A::add(ir, xs), half), wy1 = A::mul(A::add(jr, ys), half);
    const T wx2 = A::sub(A::mul(A::add(ir, xe), half), fdcx), wy2 = A::sub(A::mul(A::add(jr, ye), half), fdcy);
    o.e[2] = A::mad(-fx2, wy2, fx2);  // jx (dcx, dcy)
    o.e[3] = A::mul(fx2, wy2);        // jx (dcx, dcy+1)
    o.e[6] = A::mad(-fy2, wx2, fy2);  // jy (dcx, dcy)
    o.e[7] = A::mul(fy2, wx2);        // jy (dcx+1, dcy)
    const bool cr = dcx != 0 || dcy != 0;
    o.ja = cr ? fx1 : A::mul(qx, A::sub(xe, xs));
    o.jw = cr ? wy1 : jm;
    o.jb = cr ? fy1 : A::mul(qy, A::sub(ye, ys));
    o.jv = cr ? wx1 : im;
  } else {
    im = A::mul(A::add(A::add(A::add(fdcx, px), dx2), one), half);
    jm = A::mul(A::add(A::add(A::add(fdcy, py), dy2), one), half);
    const T ir = fmin(fmin(fdcx, T(0)) + one, fmax(fmax(fdcx, T(0)), im));
    const T jr = fmin(fmin(fdcy, T(0)) + one, fmax(fmax(fdcy, T(0)), jm));
    const T fx1 = A::mul(qx, A::sub(A::sub(ir, px), half));
    const T fy1 = A::mul(qy, A::sub(A::sub(jr, py), half));
    const T fx2 = A::mul(qx, A::sub(A::add(A::add(fdcx, dx2), half), ir));
    const T fy2 = A::mul(qy, A::sub(A::add(A::add(fdcy, dy2), half), jr));
    const T wx1 = A::mul(A::add(A::add(ir, px), half), half);
    const T wy1 = A::mul(A::add(A::add(jr, py), half), half);
    const T wx2 = A::mul(A::add(A::add(A::sub(ir, fdcx), dx2), half), half);
    const T wy2 = A::mul(A::add(A::add(A::sub(jr, fdcy), dy2), half), half);
    o.e[0] = A::mul(fx1, A::sub(one, wy1));  // jx (0, 0)
    o.e[1] = A::mul(fx1, wy1);               // jx (0, 1)
    o.e[2] = A::mul(fx2, A::sub(one, wy2));  // jx (dcx, dcy)
    o.e[3] = A::mul(fx2, wy2);               // jx (dcx, dcy+1)
    o.e[4] = A::mul(fy1, A::sub(one, wx1));  // jy (0, 0)
    o.e[5] = A::mul(fy1, wx1);               // jy (1, 0)
    o.e[6] = A::mul(fy2, A::sub(one, wx2));  // jy (dcx, dcy)
    o.e[7] = A::mul(fy2, wx2);               // jy (dcx+1, dcy)
  }
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
    o.quz = quz;
    o.zdx = dimid;
    o.zdy = djmid;
    if constexpr (!(MIXED || !COMPAT)) {
      o.e[8] = A::mul(quz, z4);   // jz (0, 0)
      o.e[9] = A::mul(quz, z2);   // jz (di, 0)
      o.e[10] = A::mul(quz, z3);  // jz (0, dj)
      o.e[11] = A::mul(quz, z1);  // jz (di, dj)
    }
  }
  {
    const bool cr = COMPAT && (a.compat & 4) != 0;  // mirrored weights (pic2d.f90:1285-1288)
    const T rx = cr ? A::sub(half, px) : A::add(half, px);
    const T ry = cr ? A::sub(half, py) : A::add(half, py);
    const T r1 = A::mul(rx, ry);
    const T r2 = A::sub(rx, r1);
    const T r3 = A::sub(ry, r1);
    const T r4 = A::sub(A::sub(A::sub(one, r1), r2), r3);
    if constexpr (!(MIXED || !COMPAT)) {
      o.e[12] = A::mul(r4, qq);  // rho (0, 0)
      o.e[13] = A::mul(r2, qq);  // rho (1, 0)
      o.e[14] = A::mul(r3, qq);  // rho (0, 1)
      o.e[15] = A::mul(r1, qq);  // rho (1, 1)
    }
    o.q = qq;
    o.rw[0] = r4;
    o.rw[1] = r2;
    o.rw[2] = r3;
    o.rw[3] = r1;
  }

  // ---- boundaries: x periodic (pic2d.f90:1032); y periodic (the 1-rank
  // exchange of pic2d.f90:1033-1146 reduces to a wrap) or specular walls.
  int nix = ix + dcx, niy = iy + dcy;
  T ruy = uy, rdy = dy2;
  if ((unsigned)nix >= (unsigned)a.mx || (unsigned)niy >= (unsigned)a.my) {  // a particle leaving the domain
    nix = nix < 0 ? nix + a.mx : (nix >= a.mx ? nix - a.mx : nix);
    if (a.ybc == 0) {
      niy = niy < 0 ? niy + a.my : (niy >= a.my ? niy - a.my : niy);
    } else if (niy < 0 || niy >= a.my) {
      niy = niy < 0 ? 0 : a.my - 1;
      rdy = -dy2;
      ruy = -uy;
    }
  }
  o.cw = cw_make(nix, niy, sp);
  o.dx = dx2;
  o.dy = rdy;
  o.ux = ux;
  o.uy = ruy;
  o.uz = uz;
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

// Component and relative node of entry k of the 17-value cell stencil:
// 0-1 jx (0,0),(0,1); 2-3 jy (0,0),(1,0); 4-12 jz (x,y) in [-1,1]^2 at
// 4 + (x+1)*3 + (y+1); 13-16 rho (0,0),(1,0),(0,1),(1,1).
__device__ __forceinline__ void stencil_node(int k, int* c, int* x, int* y) {
  if (k < 2) {
    *c = JX; *x = 0; *y = k;
  } else if (k < 4) {
    *c = JY; *x = k - 2; *y = 0;
  } else if (k < 13) {
    *c = JZ; *x = (k - 4) / 3 - 1; *y = (k - 4) % 3 - 1;
  } else {
    *c = RHO; *x = (k - 13) & 1; *y = (k - 13) >> 1;
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

// Bin of cell (cx, cy) in the window of the tile (ixt, rows y0..y1-1): the
// 3 x (y1-y0+2) cells adjacent to the tile, bin = bx*(tile_rows+2) + by.
// Returns -1 outside the window.
__device__ __forceinline__ int window_bin(int cx, int cy, int ixt, int y0, int y1, int ty, int mx, int my,
                                          int ybc) {
  int bx = cx - ixt + 1;
  bx = bx < 0 ? bx + mx : (bx >= mx ? bx - mx : bx);
  int by = cy - y0 + 1;
  if (ybc == 0) by = by < 0 ? by + my : (by >= my ? by - my : by);
  if (bx < 0 || bx > 2 || by < 0 || by > y1 - y0 + 1) return -1;
  return bx * (ty + 2) + by;
}

__device__ __forceinline__ void acc_add(double* p, double v) { atomicAdd(p, v); }
__device__ __forceinline__ void acc_add(long long* p, long long v) {
  atomicAdd(reinterpret_cast<unsigned long long*>(p), (unsigned long long)v);
}

// A crossing particle's value v (|v| < 2^32, fixed point) into the split
// 32-bit windows: v = hi * 2^17 + lo with 0 <= lo < 2^17.
__device__ __forceinline__ void cross_add(unsigned* lo, int* hi, int idx, long long v) {
  atomicAdd(&lo[idx], (unsigned)(v & 0x1ffff));
  atomicAdd(&hi[idx], (int)(v >> 17));
}
__device__ __forceinline__ void cross_add(unsigned*, int*, int, double) {}

template <class T, bool MIXED>
__device__ __forceinline__ typename std::conditional<MIXED, long long, double>::type to_acc(T v) {
  if constexpr (MIXED) {
    return __float2ll_rn(__fmul_rn((float)v, FIX_SCALE));
  } else {
    return (double)v;
  }
}

// Compile-time shape of the push loop: particles per thread per pass are
// 4 * PBPIC_PUSH_HALVES (read as float4 groups; PBPIC_PUSH_HALVES_FP64 for the
// plain form, where 4 particles a pass measured 1 % faster than 8 at three
// blocks per SM), PBPIC_PUSH_UNROLL selects whether the loop over the 4
// particles of a group is unrolled, and the MINBLOCKS values are the resident
// blocks per SM the register allocation must allow.
#ifndef PBPIC_PUSH_HALVES
#define PBPIC_PUSH_HALVES 2
#endif
#ifndef PBPIC_PUSH_UNROLL
#define PBPIC_PUSH_UNROLL 0
#endif
#ifndef PBPIC_PUSH_MINBLOCKS
#define PBPIC_PUSH_MINBLOCKS 5
#endif
#ifndef PBPIC_PUSH_HALVES_FP64
#define PBPIC_PUSH_HALVES_FP64 1
#endif
#ifndef PBPIC_PUSH_MINBLOCKS_FP64
#define PBPIC_PUSH_MINBLOCKS_FP64 3
#endif
#ifndef PBPIC_PUSH_NODECACHE
#define PBPIC_PUSH_NODECACHE 0
#endif

// Per-warp staging of the lanes' stencil sums (stride 33: conflict-free rows
// and columns), and a second column per lane for the first cell of a lane
// whose particles change cell inside a pass: static in the mixed form; the
// plain form's (FP64, twice the size) is in the dynamic shared memory, after
// the window and the histogram (push_first_offset).
template <class T, bool MIXED>
struct PushSmem {
  T stage[PushThreads<T>::value / 32][17][33];
  double red[32];
  uint64_t mbar;
};
template <>
struct PushSmem<float, true> {
  float stage[PushThreads<float>::value / 32][17][33];
  float first[PushThreads<float>::value / 32][17][33];
  double red[32];
  uint64_t mbar;  // completion of the tile records' bulk copy (tile_begin)
};

// Rare path: a particle outside its tile adds its 16 terms (staged in the
// thread's shared-memory column, stride 33) to global memory.
// (The geometry comes by value: a reference to the kernel's parameters would
// make every thread copy them to local memory.)
template <class T, bool MIXED>
__device__ __noinline__ void deposit_global(void* jacc, int mx, int my, int S, int ybc, int compat, const T* col,
                                            int ix, int iy, int dcx, int dcy, int di, int dj) {
  using Acc = typename std::conditional<MIXED, long long, double>::type;
  Acc* gacc = reinterpret_cast<Acc*>(jacc);
  for (int k = 0; k < 16; ++k) {
    int rx, ry;
    term_node(k, dcx, dcy, di, dj, &rx, &ry);
    long long gi;
    int sg;
    const T v = col[k * 33];
    if (map_current(k >> 2, ix + rx, iy + ry, mx, my, S, ybc, compat, &gi, &sg))
      acc_add(&gacc[gi], to_acc<T, MIXED>(sg < 0 ? -v : v));
  }
}

// Rare path: a thread's particles changed cell inside a pass; add the finished
// cell's stencil (staged in shared memory, stride 33) to the window.
template <class T, bool MIXED>
__device__ __noinline__ void flush_column(typename std::conditional<MIXED, long long, double>::type* win,
                                          const T* col, int key, int WR) {
  for (int k = 0; k < 17; ++k) {
    int c, x, y;
    stencil_node(k, &c, &x, &y);
    const T v = col[k * 33];
    if (v != T(0)) acc_add(&win[(c * 4 + 1 + x) * WR + key + 1 + y], to_acc<T, MIXED>(v));
  }
}

// The loop over the 4 particles of a group is not unrolled: each iteration
// takes element 0 and appends its result, so after 4 iterations the group
// holds the 4 results in order.
template <class V>
__device__ __forceinline__ void rot4(V (&v)[4], V x) {
  v[0] = v[1];
  v[1] = v[2];
  v[2] = v[3];
  v[3] = x;
}

// Byte offset of the plain form's second stage in the dynamic shared memory.
__host__ __device__ __forceinline__ size_t push_first_offset(int ty) {
  return ((size_t)16 * (ty + 3) * 8 + (size_t)3 * (ty + 2) * 4 + 15) & ~(size_t)15;
}

// Round-to-nearest add that the compiler keeps as written (no fusion into an FMA).
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }

// Shared-memory window of a tile push (smem_raw): the window (16*(ty+3)
// accumulators), the new-cell histogram (3*(ty+2) int), then the mixed form's
// crossers' windows (2 x 8*(ty+3) 32-bit sums) or the plain form's second stage.
template <class T, bool MIXED>
struct TileWin {
  using Acc = typename std::conditional<MIXED, long long, double>::type;
  int TY, WR, NB, ixt, y0, y1;
  Acc* win;
  int* hist;
  unsigned* clo;  // crossers: jx, jy planes (8 * WR)
  int* chi;
  const T* stg;    // staged in shared memory: the mixed form's gather records of rows y0..y1-1 (24 values
                   // a row), the plain form's node-grid columns ixt and ixt+1 of rows y0..y1 (8 a node)
  uint64_t* mbar;  // completion of their bulk copy
};

// Byte offset of the mixed form's staged records (after the split windows) and
// of their mbarrier (after the records of a 64-row tile).
__host__ __device__ __forceinline__ size_t push_rec_offset(int ty) {
  return ((size_t)16 * (ty + 3) * 8 + (size_t)3 * (ty + 2) * 4 + (size_t)16 * (ty + 3) * 4 + 15) & ~(size_t)15;
}
// ... and of the plain form's staged node columns (after its second stage).
__host__ __device__ __forceinline__ size_t push_node_offset(int ty) {
  return (push_first_offset(ty) + (size_t)(PushThreads<double>::value / 32) * 17 * 33 * 8 + 15) & ~(size_t)15;
}


// Clears the windows of tile t and starts its histogram from the input's cell
// counts: the input is sorted by cell, so every particle of a tile cell stays
// in that cell's bin unless it crosses, and each crossing particle moves one
// count.
template <class T, bool MIXED, bool HIST>
__device__ __forceinline__ TileWin<T, MIXED> tile_begin(const PushParams<T>& a, int t, unsigned char* smem_raw,
                                                        uint64_t* mbar) {
  using Acc = typename TileWin<T, MIXED>::Acc;
  TileWin<T, MIXED> w;
  w.TY = a.tile_rows;
  w.WR = w.TY + 3;
  w.NB = 3 * (w.TY + 2);
  w.win = reinterpret_cast<Acc*>(smem_raw);
  w.hist = reinterpret_cast<int*>(w.win + 16 * w.WR);
  w.clo = reinterpret_cast<unsigned*>(w.hist + w.NB);
  w.chi = reinterpret_cast<int*>(w.clo + 8 * w.WR);
  w.ixt = t / a.tiles_per_col;
  w.y0 = (t - w.ixt * a.tiles_per_col) * w.TY;
  w.y1 = min(w.y0 + w.TY, a.my);
  w.stg = reinterpret_cast<const T*>(smem_raw + (MIXED ? push_rec_offset(w.TY) : push_node_offset(w.TY)));
  w.mbar = mbar;
  if constexpr (MIXED && PBPIC_CELL_COEF && PBPIC_PUSH_STAGE_RECS) {
    // the records of cells (ixt, y0..y1-1) are contiguous: one copy of 96 B per row
    if (threadIdx.x == 0) {
      const unsigned bytes = (unsigned)(w.y1 - w.y0) * 96u;
      bulk_expect(w.mbar, bytes);
      bulk_copy(const_cast<T*>(w.stg), a.cg + ((long long)w.ixt * a.my + w.y0) * 24, bytes, w.mbar);
    }
  } else if constexpr (!MIXED && PBPIC_PUSH_STAGE_NODES) {
    // nodes (ixt, y0..y1) and (ixt+1, y0..y1): two contiguous runs of 64 B per node
    if (threadIdx.x == 0) {
      const unsigned bytes = (unsigned)(w.y1 - w.y0 + 1) * 64u;
      const T* g = a.ng + ((long long)w.ixt * (a.my + 1) + w.y0) * 8;
      bulk_expect(w.mbar, 2 * bytes);
      bulk_copy(const_cast<T*>(w.stg), g, bytes, w.mbar);
      bulk_copy(const_cast<T*>(w.stg) + (w.TY + 1) * 8, g + (long long)(a.my + 1) * 8, bytes, w.mbar);
    }
  }
  for (int e = threadIdx.x; e < 16 * w.WR; e += blockDim.x) w.win[e] = Acc(0);
  if (MIXED)
    for (int e = threadIdx.x; e < 8 * w.WR; e += blockDim.x) {
      w.clo[e] = 0u;
      w.chi[e] = 0;
    }
  if (HIST)
    for (int e = threadIdx.x; e < w.NB; e += blockDim.x) {
      const int by = e - (w.TY + 2);
      int v = 0;
      if (by >= 1 && by <= w.y1 - w.y0) {
        const long long c = (long long)w.ixt * a.my + w.y0 + by - 1;
        v = a.cell_off[c + 1] - a.cell_off[c];
      }
      w.hist[e] = v;
    }
  __syncthreads();
  return w;
}

// A crossing particle (old cell (ix, iy) in tile window w) moves one count of
// the histogram from its old cell's bin to its new cell's. Returns the status
// bits it raises (a jump of two cells, only from a corrupt offset, keeps the
// particle in its cell: *cw is reset to the old word).
template <class T, bool MIXED>
__device__ __forceinline__ int hist_move(const PushParams<T>& a, const TileWin<T, MIXED>& w, uint32_t old_cw,
                                         uint32_t* cw, int dcx, int ix, int iy) {
  int st = 0;
  // new cell in the tile's window: column 1 + dcx, row new_iy - y0 + 1
  // (wrapped rows come back through +-my; a reflected particle keeps its row)
  int by = cw_iy(*cw) - w.y0 + 1;
  by = by < 0 ? by + a.my : (by > w.y1 - w.y0 + 1 ? by - a.my : by);
  int b = (1 + dcx) * (w.TY + 2) + by;
  if (by < 0 || by > w.y1 - w.y0 + 1) {
    b = window_bin(cw_ix(*cw), cw_iy(*cw), w.ixt, w.y0, w.y1, w.TY, a.mx, a.my, a.ybc);
    if (b < 0) {
      st = 1;
      *cw = old_cw;
      b = window_bin(ix, iy, w.ixt, w.y0, w.y1, w.TY, a.mx, a.my, a.ybc);
    }
  }
  const int bo = (w.TY + 2) + iy - w.y0 + 1;  // the old cell's bin
  if (b != bo) {
    atomicAdd(&w.hist[b], 1);
    atomicAdd(&w.hist[bo], -1);
  }
  return st;
}

// End of a pass: sum the stencils of lanes that share a cell; 17 lanes add
// each run's sum to the window. stage: the warp's [17][33] staging rows;
// fw: the warp's [17][33] first parts; vals(k): this lane's stencil entry k.
template <class T, bool MIXED, class Vals>
__device__ __forceinline__ void pass_sums(const Vals& vals, int acc_key, int first_key, T (*stage)[33], const T* fw,
                                          typename std::conditional<MIXED, long long, double>::type* win, int WR,
                                          int sc, int sx, int sy) {
  const unsigned lane = lane_id();
  T* mycol = &stage[0][lane];
  const int key = acc_key >= 0 ? acc_key : -1 - (int)lane;
  const int kprev = __shfl_up_sync(FULL, key, 1);
  const unsigned head = (lane == 0) || (kprev != key);
  // Keys do not decrease across the lanes, so a run is the lanes head..tail
  // plus, when the next lane's first part has the run's cell, that part. The
  // 17 lanes sum the run's staged columns in lane order (a fixed order: the
  // result does not depend on timing). A first part that does not continue
  // the run ending at the previous lane is added on its own.
  const int fnext = __shfl_down_sync(FULL, first_key, 1);
  const unsigned heads = __ballot_sync(FULL, head);
  const unsigned head_next = __shfl_down_sync(FULL, head, 1);
  unsigned tails = __ballot_sync(FULL, acc_key >= 0 && (lane == 31 || head_next));
  const bool joined = lane > 0 && head && kprev == first_key;
  unsigned solo = __ballot_sync(FULL, first_key >= 0 && !joined);
#pragma unroll
  for (int k = 0; k < 17; ++k) mycol[k * 33] = vals(k);
  __syncwarp();
  while (tails) {
    const int src = __ffs(tails) - 1;
    tails &= tails - 1;
    const int start = 31 - __clz(heads & (0xffffffffu >> (31 - src)));
    const int kt = __shfl_sync(FULL, key, src);
    const int nf = __shfl_sync(FULL, fnext, src);
    if (lane < 17) {
      const T* row = &stage[lane][0];
      T v = row[start];
      for (int l = start + 1; l <= src; ++l) v = add_rn(v, row[l]);
      if (src < 31 && nf == kt) v = add_rn(v, fw[lane * 33 + src + 1]);
      if (v != T(0)) acc_add(&win[(sc * 4 + 1 + sx) * WR + kt + 1 + sy], to_acc<T, MIXED>(v));
    }
  }
  while (solo) {
    const int src = __ffs(solo) - 1;
    solo &= solo - 1;
    const int kt = __shfl_sync(FULL, first_key, src);
    if (lane < 17) {
      const T v = fw[lane * 33 + src];
      if (v != T(0)) acc_add(&win[(sc * 4 + 1 + sx) * WR + kt + 1 + sy], to_acc<T, MIXED>(v));
    }
  }
  __syncwarp();  // the stage is rewritten in the next pass
}

// End of a tile: fold the window into the global current, write the tile's
// histogram, kinetic energies and status.
template <class T, bool MIXED, bool HIST>
__device__ __forceinline__ void tile_end(const PushParams<T>& a, int t, const TileWin<T, MIXED>& w, double ke_e,
                                         double ke_i, int status, double* red) {
  using Acc = typename TileWin<T, MIXED>::Acc;
  Acc* gacc = reinterpret_cast<Acc*>(a.jacc);
  __syncthreads();
  for (int e = threadIdx.x; e < 16 * w.WR; e += blockDim.x) {
    Acc val = w.win[e];
    if (MIXED && e < 8 * w.WR) val += (Acc)(((long long)w.chi[e] << 17) + (long long)w.clo[e]);
    if (val == Acc(0)) continue;
    const int c = e / (4 * w.WR);
    const int r = e - c * 4 * w.WR;
    const int wx = r / w.WR, wy = r - wx * w.WR;
    long long gi;
    int sg;
    if (map_current(c, w.ixt - 1 + wx, w.y0 - 1 + wy, a.mx, a.my, a.S, a.ybc, a.compat, &gi, &sg))
      acc_add(&gacc[gi], sg < 0 ? -val : val);
  }
  if (HIST)
    for (int e = threadIdx.x; e < w.NB; e += blockDim.x) a.tilecnt[(long long)t * w.NB + e] = w.hist[e];
  const double se = block_sum(ke_e, red);
  const double si = block_sum(ke_i, red);
  if (threadIdx.x == 0) {
    a.ke_part[2 * t] = se;
    a.ke_part[2 * t + 1] = si;
  }
  status = __reduce_or_sync(FULL, status);
  if (lane_id() == 0 && status) atomicOr(a.status, status);
}

// Push of tile t of the domain `a`, by all threads of the block: G float4
// groups of particles per thread per pass (8 particles for G = 2).
// parity: the phase of sm.mbar this tile's record copy completes (the
// block's count of earlier tiles, mod 2).
template <class T, bool MIXED, bool HIST, int G, bool COMPAT = true, bool GATHER = false>
__device__ __forceinline__ void push_tile(const PushParams<T>& a, const int t, PushSmem<T, MIXED>& sm,
                                          unsigned char* smem_raw, unsigned parity) {
  constexpr int PT = 4 * G;  // particles per thread per pass
  constexpr bool STAGED = MIXED ? (PBPIC_CELL_COEF && PBPIC_PUSH_STAGE_RECS) : PBPIC_PUSH_STAGE_NODES;
  const TileWin<T, MIXED> tw = tile_begin<T, MIXED, HIST>(a, t, smem_raw, &sm.mbar);
  const int TY = tw.TY, WR = tw.WR, ixt = tw.ixt, y0 = tw.y0, y1 = tw.y1;
  bool staged = false;  // this thread reads the tile's records from shared memory
  if constexpr (STAGED) staged = mbar_wait(tw.mbar, parity);
  auto* win = tw.win;
  unsigned* clo = tw.clo;
  int* chi = tw.chi;
  const int pbeg = a.tile_off[t], pend = a.tile_off[t + 1];
  const bool split = MIXED && pend - pbeg <= 32767;  // crossers to the 32-bit windows
  const unsigned lane = lane_id();
  const int w = threadIdx.x >> 5;
  // [17][33] first parts of the lanes of warp w whose particles change cell
  // (the mixed form's static array keeps its addresses constant)
  T* fw;
  if constexpr (MIXED) fw = &sm.first[w][0][0];
  else fw = reinterpret_cast<T*>(smem_raw + push_first_offset(TY)) + w * 17 * 33;
  // this lane's entry of the stencil when it deposits a run's sum
  int sc = 0, sx = 0, sy = 0;
  stencil_node(lane < 17 ? (int)lane : 0, &sc, &sx, &sy);
  T* mycol = &sm.stage[w][0][lane];
  double ke_e = 0.0, ke_i = 0.0;
  int status = 0;
  if (STAGED && !staged) status |= PBPIC_STATUS_COPY_TIMEOUT;
  for (int q0 = pbeg & ~3; q0 < pend; q0 += PT * PushThreads<T>::value) {
    // thread-level accumulation of the stencils of particles sharing a cell
    T acc[17];
#pragma unroll
    for (int k = 0; k < 17; ++k) acc[k] = T(0);
    auto sval = [&](int k) -> T { return acc[k]; };  // stencil entry k of the thread's sums
    int acc_key = -1;
    int first_key = -1;  // cell of this pass's finished first part (in `fw`), or -1
    int cache_cell = -1;
    Node6<T> n00{}, n01{}, n10{}, n11{};
    CellCoef cc;  // mixed form with coefficient records
    T pke_e = T(0), pke_i = T(0);  // this pass's kinetic energy, per species
#pragma unroll 1
    for (int g = 0; g < G; ++g) {
      const int q = q0 + PT * (int)threadIdx.x + 4 * g;
      uint32_t cw[4];
      T px[4], py[4], pux[4], puy[4], puz[4];
      const bool full = q >= pbeg && q + 4 <= pend;
      int32_t sidx[4] = {0, 0, 0, 0};  // GATHER: input elements of the group
      if (GATHER) {
        if (full) {
          ld4(reinterpret_cast<const uint32_t*>(a.src) + q, reinterpret_cast<uint32_t(&)[4]>(sidx));
        } else {
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const int p = q + j;
            sidx[j] = (p >= pbeg && p < pend) ? a.src[p] : 0;
          }
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {  // the input is not written by this launch: read-only loads
          // (a position outside the tile has entry 0: element 0 is read and its values are not used)
          const int e = sidx[j];
          cw[j] = __ldg(a.cell + e);
          px[j] = __ldg(a.dx + e);
          py[j] = __ldg(a.dy + e);
          pux[j] = __ldg(a.ux + e);
          puy[j] = __ldg(a.uy + e);
          puz[j] = __ldg(a.uz + e);
        }
      } else if (full) {
        ld4(a.cell + q, cw);
        ld4(a.dx + q, px);
        ld4(a.dy + q, py);
        ld4(a.ux + q, pux);
        ld4(a.uy + q, puy);
        ld4(a.uz + q, puz);
      } else {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int p = q + j;
          const bool act = p >= pbeg && p < pend;
          cw[j] = act ? a.cell[p] : 0u;
          px[j] = act ? a.dx[p] : T(0);
          py[j] = act ? a.dy[p] : T(0);
          pux[j] = act ? a.ux[p] : T(0);
          puy[j] = act ? a.uy[p] : T(0);
          puz[j] = act ? a.uz[p] : T(0);
        }
      }
#if PBPIC_PUSH_UNROLL
#pragma unroll
#else
#pragma unroll 1
#endif
      for (int j = 0; j < 4; ++j) {
        const int p = q + j;
        if (!full && (p < pbeg || p >= pend)) {
          rot4(cw, cw[0]);
          rot4(px, px[0]);
          rot4(py, py[0]);
          rot4(pux, pux[0]);
          rot4(puy, puy[0]);
          rot4(puz, puz[0]);
          continue;
        }
        const uint32_t wrd = cw[0];
        const int sp = cw_sp(wrd), ix = cw_ix(wrd), iy = cw_iy(wrd);
        const int cid = (ix << 16) | iy;
        const bool inwin = ix == ixt && (unsigned)(iy - y0) < (unsigned)(y1 - y0);  // in this tile (sorted input)
        if (!PBPIC_PUSH_NODECACHE || cid != cache_cell) {
          if constexpr (MIXED && STAGED) {
            const int r = iy - y0;
            if (staged && inwin) load_coef_staged(tw.stg + r * 24, cc);
            else load_coef(a.cg + ((long long)ix * a.my + iy) * 24, cc);
          } else if constexpr (MIXED && PBPIC_CELL_COEF) {
            load_coef(a.cg + ((long long)ix * a.my + iy) * 24, cc);
          } else if constexpr (MIXED) {
            load_cell(a.cg + ((long long)ix * a.my + iy) * 24, n00, n01, n10, n11);
          } else if (STAGED && staged && inwin) {
            // FP64 from the tile's staged node columns
            const T* s00 = tw.stg + (iy - y0) * 8;
            const T* s10 = s00 + (TY + 1) * 8;
            n00 = load_node_staged(s00);
            n01 = load_node_staged(s00 + 8);
            n10 = load_node_staged(s10);
            n11 = load_node_staged(s10 + 8);
          } else {  // FP64: from the node grid (its records took more registers than they saved)
            const T* g00 = a.ng + ((long long)ix * (a.my + 1) + iy) * 8;
            const T* g10 = g00 + (long long)(a.my + 1) * 8;
            n00 = load_node(g00);
            n01 = load_node(g00 + 8);
            n10 = load_node(g10);
            n11 = load_node(g10 + 8);
          }
          cache_cell = cid;
        }
        Pushed<T> o;
        if constexpr (MIXED && PBPIC_CELL_COEF)
          push_one_coef<COMPAT>(a, sp, ix, iy, px[0], py[0], pux[0], puy[0], puz[0], cc, o);
        else
          push_one<T, MIXED, COMPAT>(a, sp, ix, iy, px[0], py[0], pux[0], puy[0], puz[0], n00, n01, n10, n11, o);
        status |= o.status;
        const bool cross = o.dcx != 0 || o.dcy != 0;
        if (inwin) {
          const int key = iy - y0;
          if (key != acc_key) {
            if (acc_key >= 0) {  // the thread's particles changed cell
              if (first_key < 0) {  // first change of the pass: keep the part for the run sums
                first_key = acc_key;
#pragma unroll
                for (int k = 0; k < 17; ++k) {
                  fw[k * 33 + lane] = sval(k);
                  acc[k] = T(0);
                }
              }
              if (acc_key >= 0 && acc_key != first_key) {  // a cell wholly inside this thread's pass
#pragma unroll
                for (int k = 0; k < 17; ++k) {
                  mycol[k * 33] = sval(k);
                  acc[k] = T(0);
                }
                flush_column<T, MIXED>(win, mycol, acc_key, WR);
              }
            }
            acc_key = key;
          }
          if constexpr (MIXED || !COMPAT) {  // FMA forms of the cell-relative terms
            using F = M<T, true>;
            acc[0] = F::add(acc[0], F::mad(-o.ja, o.jw, o.ja));
            acc[1] = F::mad(o.ja, o.jw, acc[1]);
            acc[2] = F::add(acc[2], F::mad(-o.jb, o.jv, o.jb));
            acc[3] = F::mad(o.jb, o.jv, acc[3]);
            // jz: outer product of the x weights (x = -1, 0, 1) and y weights
            const T qs = F::mul(o.quz, o.zdx), q0 = F::sub(o.quz, qs);
            const T qxm = o.di < 0 ? qs : T(0), qxp = o.di > 0 ? qs : T(0);
            const T ym = o.dj < 0 ? o.zdy : T(0), yp = o.dj > 0 ? o.zdy : T(0), y0 = F::sub(T(1), o.zdy);
            acc[4 + 0] = F::mad(qxm, ym, acc[4 + 0]);
            acc[4 + 1] = F::mad(qxm, y0, acc[4 + 1]);
            acc[4 + 2] = F::mad(qxm, yp, acc[4 + 2]);
            acc[4 + 3] = F::mad(q0, ym, acc[4 + 3]);
            acc[4 + 4] = F::mad(q0, y0, acc[4 + 4]);
            acc[4 + 5] = F::mad(q0, yp, acc[4 + 5]);
            acc[4 + 6] = F::mad(qxp, ym, acc[4 + 6]);
            acc[4 + 7] = F::mad(qxp, y0, acc[4 + 7]);
            acc[4 + 8] = F::mad(qxp, yp, acc[4 + 8]);
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
          if constexpr (MIXED) {  // unit charge: q * w + acc in one rounding, the same as acc + (q * w)
            using F = M<T, true>;
#pragma unroll
            for (int k = 0; k < 4; ++k) acc[13 + k] = F::mad(o.q, o.rw[k], acc[13 + k]);
          } else if constexpr (!COMPAT) {  // the products the exact order keeps in e[12..15]
#pragma unroll
            for (int k = 0; k < 4; ++k) acc[13 + k] += M<T, true>::mul(o.rw[k], o.q);
          } else {
            acc[13] += o.e[12];
            acc[14] += o.e[13];
            acc[15] += o.e[14];
            acc[16] += o.e[15];
          }
          if (cross) {  // new-cell count and second zig-zag segment, in one branch
            if (HIST) status |= hist_move<T, MIXED>(a, tw, wrd, &o.cw, o.dcx, ix, iy);
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
        } else {
          status |= 4;
          if constexpr (MIXED || !COMPAT) {  // the 16 terms from the stencil quantities (rare path only)
            using F = M<T, true>;
            const T z = T(0);
            mycol[0 * 33] = F::mad(-o.ja, o.jw, o.ja);
            mycol[1 * 33] = F::mul(o.ja, o.jw);
            mycol[2 * 33] = cross ? o.e[2] : z;
            mycol[3 * 33] = cross ? o.e[3] : z;
            mycol[4 * 33] = F::mad(-o.jb, o.jv, o.jb);
            mycol[5 * 33] = F::mul(o.jb, o.jv);
            mycol[6 * 33] = cross ? o.e[6] : z;
            mycol[7 * 33] = cross ? o.e[7] : z;
            const T qs = F::mul(o.quz, o.zdx), q0 = F::sub(o.quz, qs), y0 = F::sub(T(1), o.zdy);
            mycol[8 * 33] = F::mul(q0, y0);
            mycol[9 * 33] = F::mul(qs, y0);
            mycol[10 * 33] = F::mul(q0, o.zdy);
            mycol[11 * 33] = F::mul(qs, o.zdy);
#pragma unroll
            for (int k = 0; k < 4; ++k) mycol[(12 + k) * 33] = F::mul(o.q, o.rw[k]);
          } else {
#pragma unroll
            for (int k = 0; k < 16; ++k) mycol[k * 33] = o.e[k];
          }
          deposit_global<T, MIXED>(a.jacc, a.mx, a.my, a.S, a.ybc, a.compat, mycol, ix, iy, o.dcx, o.dcy, o.di, o.dj);
        }
        rot4(cw, o.cw);
        rot4(px, o.dx);
        rot4(py, o.dy);
        rot4(pux, o.ux);
        rot4(puy, o.uy);
        rot4(puz, o.uz);
        if (sp) pke_e += o.ke;
        else pke_i += o.ke;
      }
      uint32_t* ocell = GATHER ? a.cell_o : a.cell;
      T *odx = GATHER ? a.dx_o : a.dx, *ody = GATHER ? a.dy_o : a.dy;
      T *oux = GATHER ? a.ux_o : a.ux, *ouy = GATHER ? a.uy_o : a.uy, *ouz = GATHER ? a.uz_o : a.uz;
      if (full) {
        st4(ocell + q, cw);
        st4(odx + q, px);
        st4(ody + q, py);
        st4(oux + q, pux);
        st4(ouy + q, puy);
        st4(ouz + q, puz);
      } else {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int p = q + j;
          if (p >= pbeg && p < pend) {
            ocell[p] = cw[j];
            odx[p] = px[j];
            ody[p] = py[j];
            oux[p] = pux[j];
            ouy[p] = puy[j];
            ouz[p] = puz[j];
          }
        }
      }
      if (GATHER && a.pid_o) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int p = q + j;
          if (p >= pbeg && p < pend) a.pid_o[p] = __ldg(a.pid_i + sidx[j]);
        }
      }
    }
    ke_e += (double)pke_e;
    ke_i += (double)pke_i;
    pass_sums<T, MIXED>(sval, acc_key, first_key, sm.stage[w], fw, win, WR, sc, sx, sy);
  }
  // a copy that did not land in time must not be in flight when the block
  // moves on: wait for it again (bounded) before the shared memory is reused
  if (STAGED && !staged) mbar_wait(tw.mbar, parity);
  tile_end<T, MIXED, HIST>(a, t, tw, ke_e, ke_i, status, sm.red);
}

// Single domain: one block per tile. COMPAT = false when no compat switch is
// set; GATHER when the input is the previous step's arrays and the sort's
// permutation.
template <class T, bool MIXED, bool HIST, bool COMPAT, bool GATHER = false>
__global__ void __launch_bounds__(PushThreads<T>::value, MIXED ? PBPIC_PUSH_MINBLOCKS : PBPIC_PUSH_MINBLOCKS_FP64) k_push(PushParams<T> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ PushSmem<T, MIXED> sm;
  if (threadIdx.x == 0) mbar_init(&sm.mbar);  // thread 0 also starts the copy; the others wait after a barrier
  push_tile<T, MIXED, HIST, MIXED ? PBPIC_PUSH_HALVES : PBPIC_PUSH_HALVES_FP64, COMPAT, GATHER>(a, blockIdx.x, sm,
                                                                                              smem_raw, 0u);
}

// Batched domains: persistent blocks take (domain, tile) pairs from a global
// counter (reset to 0 before each launch) in the order of `tiles`.
template <class T, bool MIXED, bool HIST, int G, bool COMPAT, bool GATHER = false>
__global__ void __launch_bounds__(PushThreads<T>::value, MIXED ? PBPIC_PUSH_MINBLOCKS : PBPIC_PUSH_MINBLOCKS_FP64)
    k_push_batched(const PushParams<T>* descs, const int2* tiles, int ntiles, int* counter) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ PushSmem<T, MIXED> sm;
  __shared__ PushParams<T> a;
  __shared__ int next;
  if (threadIdx.x == 0) mbar_init(&sm.mbar);
  unsigned parity = 0;
  while (true) {
    if (threadIdx.x == 0) next = atomicAdd(counter, 1);
    __syncthreads();
    const int t = next;
    if (t >= ntiles) break;
    const int2 it = tiles[t];
    if (threadIdx.x == 0) a = descs[it.x];
    __syncthreads();
    push_tile<T, MIXED, HIST, G, COMPAT, GATHER>(a, it.y, sm, smem_raw, parity);
    parity ^= 1u;
    __syncthreads();
  }
}

}  // namespace pbd
