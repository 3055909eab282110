// Differentiable form: the forward step with per-particle weights and the
// discrete adjoint of the whole step.
//
// Forward step n -> n+1 (the plain push of kernels_push.cuh and the field
// solve of kernels_field.cuh):
//   G^n = N(E^n, B^n)                       node averages (linear)
//   (x, u)^{n+1}, J = Push((x, u)^n, G^n)   gather, Boris, move, zig-zag deposit
//   (E, B)^{n+1} = A (E, B)^n + C J         B half step, E full step, B half step
// The adjoint runs the steps backwards:
//   field adjoint: the transposed FDTD update (k_adj_bhalf, k_adj_efull), and
//                  the transposed node average (k_adj_nodes);
//   particle adjoint (k_dadjoint): recompute the push of each particle from its
//                  stored state, then the deposition adjoint as a gather of the
//                  current adjoint at the particle's stencil, the move adjoint,
//                  the reverse Boris rotation, and the field-gather adjoint as a
//                  scatter-add of the particle's field adjoint to its 4 nodes.
// Branch decisions (cell crossings, relay points, the jz quadrant, wall
// reflections) are piecewise constant and enter the adjoint as fixed.
// Adjoint quantities are accumulated in double precision.
#pragma once
#include "device_common.cuh"
#include "kernels_push.cuh"

namespace pbd {

template <class T>
struct DiffParams {
  PushParams<T> push;     // constants, geometry and the node grid of step n
  int64_t n;              // particles (pairs in load order: 2k ion, 2k+1 electron)
  int64_t nsheet;         // pairs k < nsheet are sheet particles (weight 1)
  double omega_bg;        // weight of background particles
  double in0;             // current normalisation
  const T* lam_in[5];     // adjoint of the state after the step (dx, dy, ux, uy, uz)
  T* lam_out[5];          // adjoint of the state before the step
  const double* jbar;     // adjoint of the normalised current, 3 planes of mx x S
  double* gbar;           // adjoint of the node fields (mx+1) x (my+1) x 8
  double* domega;         // d loss / d omega_bg (one double)
};

template <class T>
__device__ __forceinline__ double particle_weight(const DiffParams<T>& a, int64_t p) {
  return (p >> 1) < a.nsheet ? 1.0 : a.omega_bg;
}

// Forward push with weights: the plain push, current (jx, jy, jz) deposited
// into double accumulators (FP64) or int64 fixed point (FP32, deterministic).
template <class T>
__global__ void k_dpush(DiffParams<T> a) {
  const PushParams<T>& pp = a.push;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < a.n; p += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t w = pp.cell[p];
    const int sp = cw_sp(w), ix = cw_ix(w), iy = cw_iy(w);
    const T* g00 = pp.ng + ((long long)ix * (pp.my + 1) + iy) * 8;
    const T* g10 = g00 + (long long)(pp.my + 1) * 8;
    const Node6<T> n00 = load_node(g00), n01 = load_node(g00 + 8), n10 = load_node(g10), n11 = load_node(g10 + 8);
    Pushed<T> o;
    push_one<T, false>(pp, sp, ix, iy, pp.dx[p], pp.dy[p], pp.ux[p], pp.uy[p], pp.uz[p], n00, n01, n10, n11, o);
    const double om = particle_weight(a, p);
#pragma unroll
    for (int k = 0; k < 12; ++k) {
      int rx, ry;
      term_node(k, o.dcx, o.dcy, o.di, o.dj, &rx, &ry);
      long long gi;
      int sg;
      if (map_current(k >> 2, ix + rx, iy + ry, pp.mx, pp.my, pp.S, pp.ybc, 0, &gi, &sg)) {
        const double v = om * (double)o.e[k] * sg;
        if (sizeof(T) == 8) {
          atomicAdd(reinterpret_cast<double*>(pp.jacc) + gi, v);
        } else {
          atomicAdd(reinterpret_cast<unsigned long long*>(pp.jacc) + gi,
                    (unsigned long long)__double2ll_rn(v * (double)FIX_SCALE));
        }
      }
    }
    pp.cell[p] = o.cw;
    pp.dx[p] = o.dx;
    pp.dy[p] = o.dy;
    pp.ux[p] = o.ux;
    pp.uy[p] = o.uy;
    pp.uz[p] = o.uz;
  }
}

struct D3 {
  double x, y, z;
};
__device__ __forceinline__ D3 cross3(D3 a, D3 b) {
  return D3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ D3 add3(D3 a, D3 b) { return D3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D3 scale3(D3 a, double s) { return D3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ double dot3(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// Particle adjoint of one step (see the file comment).
template <class T>
__global__ void k_dadjoint(DiffParams<T> a) {
  const PushParams<T>& pp = a.push;
  __shared__ double red[32];
  double domega = 0.0;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < a.n; p += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t w = pp.cell[p];
    const int sp = cw_sp(w), ix = cw_ix(w), iy = cw_iy(w);
    const T* g00 = pp.ng + ((long long)ix * (pp.my + 1) + iy) * 8;
    const T* g10 = g00 + (long long)(pp.my + 1) * 8;
    const Node6<T> n00 = load_node(g00), n01 = load_node(g00 + 8), n10 = load_node(g10), n11 = load_node(g10 + 8);
    const T px = pp.dx[p], py = pp.dy[p];
    Pushed<T> o;  // the forward push, for the branch decisions and the deposit terms
    push_one<T, false>(pp, sp, ix, iy, px, py, pp.ux[p], pp.uy[p], pp.uz[p], n00, n01, n10, n11, o);
    const double om = particle_weight(a, p);
    // ---- forward quantities in double
    const double c0 = (double)(sp ? pp.c0[1] : pp.c0[0]), c1 = (double)(sp ? pp.c1[1] : pp.c1[0]);
    const double qx = (double)(sp ? pp.qx[1] : pp.qx[0]), qy = (double)(sp ? pp.qy[1] : pp.qy[0]);
    const double qq = (double)(sp ? pp.q[1] : pp.q[0]);
    const double ax = 0.5 + (double)px, ay = 0.5 + (double)py;
    const double W[4] = {(1 - ax) * (1 - ay), ax * (1 - ay), (1 - ax) * ay, ax * ay};  // n00 n10 n01 n11
    const Node6<T>* nodes[4] = {&n00, &n10, &n01, &n11};
    D3 E{0, 0, 0}, B{0, 0, 0};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      E = add3(E, scale3(D3{(double)nodes[k]->ex, (double)nodes[k]->ey, (double)nodes[k]->ez}, W[k]));
      B = add3(B, scale3(D3{(double)nodes[k]->bx, (double)nodes[k]->by, (double)nodes[k]->bz}, W[k]));
    }
    const D3 u{(double)pp.ux[p], (double)pp.uy[p], (double)pp.uz[p]};
    const D3 um = add3(u, scale3(E, c1));
    const double gm = sqrt(1.0 + dot3(um, um));
    const double c2 = c0 / gm;
    const D3 t = scale3(B, c2);
    const double t2 = 2.0 / (1.0 + dot3(t, t));
    const D3 s = scale3(t, t2);
    const D3 u0 = add3(um, cross3(um, t));
    const D3 up = add3(um, cross3(u0, s));
    const D3 u1 = add3(up, scale3(E, c1));
    const double g1 = sqrt(1.0 + dot3(u1, u1));
    const double dtcva = (double)pp.dtcva, cva = (double)pp.cva;
    const double c3 = dtcva / g1;
    const double idx = (double)pp.idx, idy = (double)pp.idy;
    const double x1 = (double)px + c3 * u1.x * idx, y1 = (double)py + c3 * u1.y * idy;
    const double vz = u1.z * cva / g1;
    const int dcx = o.dcx, dcy = o.dcy;
    // ---- adjoint of the state after the step; undo the wall reflection
    const bool refl = pp.ybc == 1 && (iy + dcy < 0 || iy + dcy >= pp.my);
    double lx1 = (double)a.lam_in[0][p];
    double ly1 = (double)a.lam_in[1][p] * (refl ? -1.0 : 1.0);
    D3 lu1{(double)a.lam_in[2][p], (double)a.lam_in[3][p] * (refl ? -1.0 : 1.0), (double)a.lam_in[4][p]};
    double lpx = 0.0, lpy = 0.0, lvz = 0.0;
    // ---- deposition adjoint: gather the current adjoint at the 12 terms
    double tb[12];
    double dom = 0.0;
#pragma unroll
    for (int k = 0; k < 12; ++k) {
      int rx, ry;
      term_node(k, dcx, o.dcy, o.di, o.dj, &rx, &ry);
      long long gi;
      int sg;
      tb[k] = 0.0;
      if (map_current(k >> 2, ix + rx, iy + ry, pp.mx, pp.my, pp.S, pp.ybc, 0, &gi, &sg)) {
        const double jb = a.jbar[gi] * a.in0 * sg;  // d loss / d (unweighted term k)
        tb[k] = jb * om;
        dom += jb * (double)o.e[k];
      }
    }
    if ((p >> 1) >= a.nsheet) domega += dom;
    {
      const double fdcx = dcx, fdcy = dcy;
      const double im = 0.5 * ((double)px + x1 + 1.0), jm = 0.5 * ((double)py + y1 + 1.0);
      const double ir = dcx == 0 ? im : (dcx > 0 ? 1.0 : 0.0);
      const double jr = dcy == 0 ? jm : (dcy > 0 ? 1.0 : 0.0);
      const double fx1 = qx * (ir - px - 0.5), fx2 = qx * (x1 + 0.5 - ir);
      const double fy1 = qy * (jr - py - 0.5), fy2 = qy * (y1 + 0.5 - jr);
      const double wx1 = 0.5 * (ir + px + 0.5), wy1 = 0.5 * (jr + py + 0.5);
      const double wx2 = 0.5 * (ir + x1 - 2 * fdcx + 0.5), wy2 = 0.5 * (jr + y1 - 2 * fdcy + 0.5);
      const double bfx1 = tb[0] * (1 - wy1) + tb[1] * wy1, bwy1 = (tb[1] - tb[0]) * fx1;
      const double bfx2 = tb[2] * (1 - wy2) + tb[3] * wy2, bwy2 = (tb[3] - tb[2]) * fx2;
      const double bfy1 = tb[4] * (1 - wx1) + tb[5] * wx1, bwx1 = (tb[5] - tb[4]) * fy1;
      const double bfy2 = tb[6] * (1 - wx2) + tb[7] * wx2, bwx2 = (tb[7] - tb[6]) * fy2;
      double bir = qx * bfx1 - qx * bfx2 + 0.5 * bwx1 + 0.5 * bwx2;
      double bjr = qy * bfy1 - qy * bfy2 + 0.5 * bwy1 + 0.5 * bwy2;
      lpx += -qx * bfx1 + 0.5 * bwx1;
      lx1 += qx * bfx2 + 0.5 * bwx2;
      lpy += -qy * bfy1 + 0.5 * bwy1;
      ly1 += qy * bfy2 + 0.5 * bwy2;
      double bim = dcx == 0 ? bir : 0.0;
      double bjm = dcy == 0 ? bjr : 0.0;
      // jz: CIC at the midpoint, z1 = ab, z2 = a(1-b), z3 = b(1-a), z4 = (1-a)(1-b)
      const double dmx = im - 0.5, dmy = jm - 0.5;
      const double av = fabs(dmx), bv = fabs(dmy);
      const double quz = qq * vz;
      const double z1 = av * bv, z2 = av * (1 - bv), z3 = bv * (1 - av), z4 = (1 - av) * (1 - bv);
      const double bquz = tb[8] * z4 + tb[9] * z2 + tb[10] * z3 + tb[11] * z1;
      const double bz1 = quz * tb[11], bz2 = quz * tb[9], bz3 = quz * tb[10], bz4 = quz * tb[8];
      const double ba = bz1 * bv + bz2 * (1 - bv) - bz3 * bv - bz4 * (1 - bv);
      const double bb = bz1 * av - bz2 * av + bz3 * (1 - av) - bz4 * (1 - av);
      bim += ba * (dmx >= 0 ? 1.0 : -1.0);
      bjm += bb * (dmy >= 0 ? 1.0 : -1.0);
      lpx += 0.5 * bim;
      lx1 += 0.5 * bim;
      lpy += 0.5 * bjm;
      ly1 += 0.5 * bjm;
      lvz += qq * bquz;
    }
    // ---- move adjoint: x1 = px + c3 ux idx, y1 = py + c3 uy idy, vz = uz cva / g1
    lpx += lx1;
    lpy += ly1;
    lu1.x += lx1 * c3 * idx;
    lu1.y += ly1 * c3 * idy;
    lu1.z += lvz * cva / g1;
    const double bc3 = lx1 * u1.x * idx + ly1 * u1.y * idy;
    const double bg1 = -bc3 * dtcva / (g1 * g1) - lvz * u1.z * cva / (g1 * g1);
    lu1 = add3(lu1, scale3(u1, bg1 / g1));
    // ---- reverse Boris rotation
    D3 lE = scale3(lu1, c1);
    const D3 lup = lu1;
    D3 lum = lup;
    const D3 lu0 = cross3(s, lup);
    const D3 ls = cross3(lup, u0);
    lum = add3(lum, add3(lu0, cross3(t, lu0)));
    D3 lt = cross3(lu0, um);
    lt = add3(lt, scale3(ls, t2));
    const double lt2 = dot3(ls, t);
    lt = add3(lt, scale3(t, -lt2 * t2 * t2));
    const double lc2 = dot3(lt, B);
    const D3 lB = scale3(lt, c2);
    const double lgm = -lc2 * c0 / (gm * gm);
    lum = add3(lum, scale3(um, lgm / gm));
    const D3 lu = lum;
    lE = add3(lE, scale3(lum, c1));
    // ---- field-gather adjoint: scatter to the 4 nodes; weights' adjoint to the offsets
    double bW[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const Node6<T>& nd = *nodes[k];
      bW[k] = lE.x * (double)nd.ex + lE.y * (double)nd.ey + lE.z * (double)nd.ez + lB.x * (double)nd.bx +
              lB.y * (double)nd.by + lB.z * (double)nd.bz;
    }
    const int nodeidx[4] = {0, 1, 0, 1};
    const int nodeidy[4] = {0, 0, 1, 1};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      double* g = a.gbar + ((long long)(ix + nodeidx[k]) * (pp.my + 1) + iy + nodeidy[k]) * 8;
      atomicAdd(g + 0, W[k] * lE.x);
      atomicAdd(g + 1, W[k] * lE.y);
      atomicAdd(g + 2, W[k] * lE.z);
      atomicAdd(g + 4, W[k] * lB.x);
      atomicAdd(g + 5, W[k] * lB.y);
      atomicAdd(g + 6, W[k] * lB.z);
    }
    // W = [(1-ax)(1-ay), ax(1-ay), (1-ax)ay, ax ay]
    lpx += -bW[0] * (1 - ay) + bW[1] * (1 - ay) - bW[2] * ay + bW[3] * ay;
    lpy += -bW[0] * (1 - ax) - bW[1] * ax + bW[2] * (1 - ax) + bW[3] * ax;
    a.lam_out[0][p] = (T)lpx;
    a.lam_out[1][p] = (T)lpy;
    a.lam_out[2][p] = (T)lu.x;
    a.lam_out[3][p] = (T)lu.y;
    a.lam_out[4][p] = (T)lu.z;
  }
  const double s = block_sum(domega, red);
  if (threadIdx.x == 0 && s != 0.0) atomicAdd(a.domega, s);
}

// ------------------------------------------------------------ field adjoint
struct AdjField {
  int mx, my, S, ybc;
  double dth, cdt, idx, idy;
  double *ex, *ey, *ez, *bx, *by, *bz;  // adjoint planes (mx x S)
  double* jbar;                          // 3 planes: adjoint of the normalised current
};

__device__ __forceinline__ void adj_half(double* f, int i, int j, int my, int S, int ybc, double odd_sign, double v) {
  if (ybc == 0) {
    j = j < 0 ? j + my : (j >= my ? j - my : j);
    atomicAdd(&f[(long long)i * S + j], v);
    return;
  }
  if (j < 0) atomicAdd(&f[(long long)i * S], odd_sign * v);
  else if (j >= my) atomicAdd(&f[(long long)i * S + my - 1], odd_sign * v);
  else atomicAdd(&f[(long long)i * S + j], v);
}

__device__ __forceinline__ void adj_node(double* f, int i, int j, int my, int S, int ybc, double v) {
  if (ybc == 0 && j >= my) j -= my;
  atomicAdd(&f[(long long)i * S + j], v);
}

// Transposed B half step: the forward reads E and adds to B, so the adjoint
// adds the transposed curl of the B adjoint to the E adjoint.
static __global__ void k_adj_bhalf(AdjField a) {
  const int rows = a.ybc == 0 ? a.my : a.my + 1;
  const long long n = (long long)a.mx * rows;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k / rows), j = (int)(k - (long long)i * rows);
    const long long o = (long long)i * a.S + j;
    const double bbx = a.bx[o];  // bx -= dth (ez(i,j) - ez(i,j-1)) idy
    adj_half(a.ez, i, j, a.my, a.S, a.ybc, -1.0, -a.dth * a.idy * bbx);
    adj_half(a.ez, i, j - 1, a.my, a.S, a.ybc, -1.0, a.dth * a.idy * bbx);
    if (j < a.my) {
      const int im = i == 0 ? a.mx - 1 : i - 1, ip = i + 1 == a.mx ? 0 : i + 1;
      const double bby = a.by[o];  // by += dth (ez(i,j) - ez(i-1,j)) idx
      atomicAdd(&a.ez[o], a.dth * a.idx * bby);
      atomicAdd(&a.ez[(long long)im * a.S + j], -a.dth * a.idx * bby);
      const double bbz = a.bz[o];  // bz += dth ((ex(i,j+1)-ex(i,j)) idy - (ey(i+1,j)-ey(i,j)) idx)
      adj_node(a.ex, i, j + 1, a.my, a.S, a.ybc, a.dth * a.idy * bbz);
      atomicAdd(&a.ex[o], -a.dth * a.idy * bbz);
      atomicAdd(&a.ey[(long long)ip * a.S + j], -a.dth * a.idx * bbz);
      atomicAdd(&a.ey[o], a.dth * a.idx * bbz);
    }
  }
}

// Transposed E full step: adds the transposed curl of the E adjoint to the B
// adjoint and sets the current adjoint; the wall rows of ex are set to zero
// by the forward step, so their adjoint does not flow back.
static __global__ void k_adj_efull(AdjField a) {
  const int rows = a.ybc == 0 ? a.my : a.my + 1;
  const long long n = (long long)a.mx * rows;
  const long long plane = (long long)a.mx * a.S;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k / rows), j = (int)(k - (long long)i * rows);
    const long long o = (long long)i * a.S + j;
    if (a.ybc == 1 && (j == 0 || j == a.my)) {
      a.jbar[o] = 0.0;
    } else {
      const double bex = a.ex[o];  // ex += cdt ((bz(i,j) - bz(i,j-1)) idy - jx)
      adj_half(a.bz, i, j, a.my, a.S, a.ybc, 1.0, a.cdt * a.idy * bex);
      adj_half(a.bz, i, j - 1, a.my, a.S, a.ybc, 1.0, -a.cdt * a.idy * bex);
      a.jbar[o] = -a.cdt * bex;
    }
    if (j < a.my) {
      const int im = i == 0 ? a.mx - 1 : i - 1, ip = i + 1 == a.mx ? 0 : i + 1;
      const double bey = a.ey[o];  // ey -= cdt ((bz(i,j) - bz(i-1,j)) idx + jy)
      atomicAdd(&a.bz[o], -a.cdt * a.idx * bey);
      atomicAdd(&a.bz[(long long)im * a.S + j], a.cdt * a.idx * bey);
      a.jbar[plane + o] = -a.cdt * bey;
      const double bez = a.ez[o];  // ez += cdt ((by(i+1,j)-by(i,j)) idx - (bx(i,j+1)-bx(i,j)) idy - jz)
      atomicAdd(&a.by[(long long)ip * a.S + j], a.cdt * a.idx * bez);
      atomicAdd(&a.by[o], -a.cdt * a.idx * bez);
      adj_node(a.bx, i, j + 1, a.my, a.S, a.ybc, -a.cdt * a.idy * bez);
      atomicAdd(&a.bx[o], a.cdt * a.idy * bez);
      a.jbar[2 * plane + o] = -a.cdt * bez;
    } else {
      a.jbar[plane + o] = 0.0;
      a.jbar[2 * plane + o] = 0.0;
    }
  }
}

static __global__ void k_zero_wall_ex(AdjField a) {
  if (a.ybc != 1) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.mx; i += gridDim.x * blockDim.x) {
    a.ex[(long long)i * a.S] = 0.0;
    a.ex[(long long)i * a.S + a.my] = 0.0;
  }
}

// Transposed node average: the node adjoint (mx+1) x (my+1) x 8 goes back to
// the Yee planes with the images and wraps of k_nodes.
static __global__ void k_adj_nodes(AdjField a, const double* gbar) {
  const int NX = a.mx + 1, NY = a.my + 1;
  const long long n = (long long)NX * NY;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int ia = (int)(k / NY), b = (int)(k - (long long)ia * NY);
    const int i = ia == a.mx ? 0 : ia;
    const int im = i == 0 ? a.mx - 1 : i - 1;
    const int bn = (a.ybc == 0 && b == a.my) ? 0 : b;
    const double* g = gbar + k * 8;
    if (g[0] != 0.0) {
      atomicAdd(&a.ex[(long long)i * a.S + bn], 0.5 * g[0]);
      atomicAdd(&a.ex[(long long)im * a.S + bn], 0.5 * g[0]);
    }
    if (g[4] != 0.0) {
      atomicAdd(&a.bx[(long long)i * a.S + bn], 0.5 * g[4]);
      atomicAdd(&a.bx[(long long)im * a.S + bn], 0.5 * g[4]);
    }
    if (g[1] != 0.0) {
      adj_half(a.ey, i, b, a.my, a.S, a.ybc, 1.0, 0.5 * g[1]);
      adj_half(a.ey, i, b - 1, a.my, a.S, a.ybc, 1.0, 0.5 * g[1]);
    }
    if (g[5] != 0.0) {
      adj_half(a.by, i, b, a.my, a.S, a.ybc, -1.0, 0.5 * g[5]);
      adj_half(a.by, i, b - 1, a.my, a.S, a.ybc, -1.0, 0.5 * g[5]);
    }
    if (g[2] != 0.0) {
      const double v = 0.25 * g[2];
      adj_half(a.ez, i, b, a.my, a.S, a.ybc, -1.0, v);
      adj_half(a.ez, im, b, a.my, a.S, a.ybc, -1.0, v);
      adj_half(a.ez, i, b - 1, a.my, a.S, a.ybc, -1.0, v);
      adj_half(a.ez, im, b - 1, a.my, a.S, a.ybc, -1.0, v);
    }
    if (g[6] != 0.0) {
      const double v = 0.25 * g[6];
      adj_half(a.bz, i, b, a.my, a.S, a.ybc, 1.0, v);
      adj_half(a.bz, im, b, a.my, a.S, a.ybc, 1.0, v);
      adj_half(a.bz, i, b - 1, a.my, a.S, a.ybc, 1.0, v);
      adj_half(a.bz, im, b - 1, a.my, a.S, a.ybc, 1.0, v);
    }
  }
}

// Magnetic-energy loss of one step, dt * 0.5 mime/(cva^2 in0) * sum w |B_node|^2
// over the energy nodes of k_nodes, and its seed for the node adjoint.
template <class T>
__global__ void k_loss_b(int mx, int my, int ybc, const T* ng, double scale, double* loss, double* gbar) {
  __shared__ double red[32];
  const int NX = mx + 1, NY = my + 1;
  const long long n = (long long)NX * NY;
  double s = 0.0;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int ia = (int)(k / NY), b = (int)(k - (long long)ia * NY);
    if (ia < mx && (ybc == 1 || b < my)) {
      const double wgt = (ybc == 1 && (b == 0 || b == my)) ? 0.5 : 1.0;
      const double bx = (double)ng[k * 8 + 4], by = (double)ng[k * 8 + 5], bz = (double)ng[k * 8 + 6];
      s += wgt * (bx * bx + by * by + bz * bz);
      if (gbar) {
        gbar[k * 8 + 4] += 2.0 * scale * wgt * bx;
        gbar[k * 8 + 5] += 2.0 * scale * wgt * by;
        gbar[k * 8 + 6] += 2.0 * scale * wgt * bz;
      }
    }
  }
  s = block_sum(s, red);
  if (threadIdx.x == 0 && loss) atomicAdd(loss, scale * s);
}

// The j.E loss of one step and its adjoint seeds: sum over the Yee entries
// (ex: node rows, off the walls; ey, ez: half rows) of J_k E_k, J the step's
// normalised current (jacc * jscale), E the fields the step starts from.
// With jbar/fbar_e, also adds scale * E to the current adjoint and scale * J to
// the E adjoint (3 planes each, mx x S).
template <class T, class Acc>
__global__ void k_loss_jdote(int mx, int my, int S, int ybc, const void* jacc, double jscale, const T* ex,
                             const T* ey, const T* ez, double scale, double* loss, double* jbar, double* fbar_e) {
  __shared__ double red[32];
  const Acc* J = reinterpret_cast<const Acc*>(jacc);
  const long long plane = (long long)mx * S;
  const int rows = ybc == 0 ? my : my + 1;
  const long long n = (long long)mx * rows;
  double s = 0.0;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k / rows), j = (int)(k - (long long)i * rows);
    const long long o = (long long)i * S + j;
    if (!(ybc == 1 && (j == 0 || j == my))) {
      const double jx = (double)J[o] * jscale, e = (double)ex[o];
      s += jx * e;
      if (jbar) {
        jbar[o] += scale * e;
        fbar_e[o] += scale * jx;
      }
    }
    if (j < my) {
      const double jy = (double)J[plane + o] * jscale, ey_ = (double)ey[o];
      const double jz = (double)J[2 * plane + o] * jscale, ez_ = (double)ez[o];
      s += jy * ey_ + jz * ez_;
      if (jbar) {
        jbar[plane + o] += scale * ey_;
        jbar[2 * plane + o] += scale * ez_;
        fbar_e[plane + o] += scale * jy;
        fbar_e[2 * plane + o] += scale * jz;
      }
    }
  }
  s = block_sum(s, red);
  if (threadIdx.x == 0 && loss) atomicAdd(loss, scale * s);
}

// d loss / d (Ti/Te) through the loaded momenta. The loader sets
// u = g uth(tau) + U(tau) (U: the sheet drift along z), so with g recovered
// from the loaded u, du/dtau = g duth/dtau + dU/dtau, contracted here with the
// adjoint of the initial momenta. Pair k = p/2: ion p even, electron p odd.
template <class T>
__global__ void k_dtau(int64_t n, int64_t nsheet, const T* ux, const T* uy, const T* uz, const T* lux, const T* luy,
                       const T* luz, double uthi, double uthe, double duthi, double duthe, double udi, double ude,
                       double dudi, double dude, double* out) {
  __shared__ double red[32];
  double acc = 0.0;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
    const bool el = (p & 1) != 0, sheet = (p >> 1) < nsheet;
    const double uth = el ? uthe : uthi, duth = el ? duthe : duthi;
    const double U = sheet ? (el ? ude : udi) : 0.0, dU = sheet ? (el ? dude : dudi) : 0.0;
    const double gx = (double)ux[p] / uth, gy = (double)uy[p] / uth, gz = ((double)uz[p] - U) / uth;
    acc += (double)lux[p] * gx * duth + (double)luy[p] * gy * duth + (double)luz[p] * (gz * duth + dU);
  }
  acc = block_sum(acc, red);
  if (threadIdx.x == 0) atomicAdd(out, acc);
}

}  // namespace pbd
