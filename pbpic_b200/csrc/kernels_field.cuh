// Yee-grid field solver (fieldsolver, pic2d.f90:678-860) and field energy
// (fieldsenergy, pic2d.f90:653-673).
//
// Storage: each of ex, ey, ez, bx, by, bz is one plane of mx x S values
// (S = my + 1), x-major with y fastest; entry (i, j) is the reference's
// emf(i+1, j+1). Locations in cell units (node (i, j) at (i, j)):
//   ex, bx at (i+1/2, j)      ("node rows": j = 0..my-1, with walls 0..my)
//   ey, by at (i, j+1/2)      ("half rows": j = 0..my-1)
//   ez, bz at (i+1/2, j+1/2)  (half rows)
// x is periodic. y is periodic (the reference's 1-rank ghost exchange,
// pic2d.f90:701-835, is a wrap) or bounded by perfectly conducting walls on
// node rows 0 and my: ex = 0 on the walls, and the ghost half rows are images
// (ez, by odd; ey, bz even). The reference stores the curl terms in its
// `fields` record; here they are recomputed from the fields, which gives the
// same interior values (the stored terms are refreshed from the same fields
// before every use).
#pragma once
#include "device_common.cuh"

namespace pbd {

template <class T>
struct FieldParams {
  int mx, my, S, ybc;
  T *ex, *ey, *ez, *bx, *by, *bz;
  T dth, cdt, idx, idy;  // dt/2, dt*cva^2 (pic2d.f90:43, 742)
  const void* jacc;      // 4 planes of accumulators (double or int64)
  double jscale[4];      // accumulator -> normalised current (in0, fixed-point scale)
  T* ng;                 // node grid (mx+1) x (my+1) x 8
  T* cg;                 // mixed form: per-cell gather records mx x my x 24 of the push
  double* fe_part;       // per-block field energy partial sums [grid][2]
  int nblk;              // batched launches: blocks that compute the partials
};

__device__ __forceinline__ int wrapx(int i, int mx) { return i < 0 ? i + mx : (i >= mx ? i - mx : i); }

// Value of a half-row component at row j in [-1, my]: wrap, or wall image
// with sign `odd_sign` (-1: odd image, +1: even image).
template <class T>
__device__ __forceinline__ T half_row(const T* f, int i, int j, int my, int S, int ybc, T odd_sign) {
  if (ybc == 0) {
    j = j < 0 ? j + my : (j >= my ? j - my : j);
    return f[(long long)i * S + j];
  }
  if (j < 0) return odd_sign * f[(long long)i * S];
  if (j >= my) return odd_sign * f[(long long)i * S + my - 1];
  return f[(long long)i * S + j];
}

// Node-row component at row j in [0, my]: wrap (row my is row 0) or the wall row.
template <class T>
__device__ __forceinline__ T node_row(const T* f, int i, int j, int my, int S, int ybc) {
  if (ybc == 0 && j >= my) j -= my;
  return f[(long long)i * S + j];
}

// B half step, pic2d.f90:688-690 / 801-803, with the curl of E as in 790-793.
template <class T>
__device__ __forceinline__ void bhalf_body(const FieldParams<T>& a) {
  const int rows = a.ybc == 0 ? a.my : a.my + 1;
  const long long n = (long long)a.mx * rows;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k / rows), j = (int)(k - (long long)i * rows);
    const long long o = (long long)i * a.S + j;
    // bx (node row j): dez_dy = (ez(i,j) - ez(i,j-1)) * idy
    {
      const T ezj = half_row(a.ez, i, j, a.my, a.S, a.ybc, T(-1));
      const T ezm = half_row(a.ez, i, j - 1, a.my, a.S, a.ybc, T(-1));
      const T d = (ezj - ezm) * a.idy;
      a.bx[o] = a.bx[o] - a.dth * d;
    }
    if (j < a.my) {
      const int im = wrapx(i - 1, a.mx), ip = wrapx(i + 1, a.mx);
      // by: dez_dx = (ez(i,j) - ez(i-1,j)) * idx
      const T dezdx = (a.ez[o] - a.ez[(long long)im * a.S + j]) * a.idx;
      a.by[o] = a.by[o] + a.dth * dezdx;
      // bz: dex_dy = (ex(i,j+1) - ex(i,j)) * idy, dey_dx = (ey(i+1,j) - ey(i,j)) * idx
      const T exn = node_row(a.ex, i, j + 1, a.my, a.S, a.ybc);
      const T dexdy = (exn - a.ex[o]) * a.idy;
      const T deydx = (a.ey[(long long)ip * a.S + j] - a.ey[o]) * a.idx;
      a.bz[o] = a.bz[o] + a.dth * (dexdy - deydx);
    }
  }
}

template <class T>
__global__ void k_bhalf(FieldParams<T> a) {
  bhalf_body(a);
}

template <class Acc>
__device__ __forceinline__ double jval(const void* jacc, long long idx) {
  return (double)reinterpret_cast<const Acc*>(jacc)[idx];
}

// E full step, pic2d.f90:742-744 with the curl of B as in 733-739.
template <class T, class Acc>
__device__ __forceinline__ void efull_body(const FieldParams<T>& a) {
  const int rows = a.ybc == 0 ? a.my : a.my + 1;
  const long long n = (long long)a.mx * rows;
  const long long plane = (long long)a.mx * a.S;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k / rows), j = (int)(k - (long long)i * rows);
    const long long o = (long long)i * a.S + j;
    // ex (node row j): dbz_dy = (bz(i,j) - bz(i,j-1)) * idy
    if (a.ybc == 1 && (j == 0 || j == a.my)) {
      a.ex[o] = T(0);  // tangential E on a perfect conductor
    } else {
      const T bzj = half_row(a.bz, i, j, a.my, a.S, a.ybc, T(1));
      const T bzm = half_row(a.bz, i, j - 1, a.my, a.S, a.ybc, T(1));
      const T dbzdy = (bzj - bzm) * a.idy;
      const T jx = (T)(jval<Acc>(a.jacc, o) * a.jscale[0]);
      a.ex[o] = a.ex[o] + a.cdt * (dbzdy - jx);
    }
    if (j < a.my) {
      const int im = wrapx(i - 1, a.mx), ip = wrapx(i + 1, a.mx);
      // ey: dbz_dx = (bz(i,j) - bz(i-1,j)) * idx
      const T dbzdx = (a.bz[o] - a.bz[(long long)im * a.S + j]) * a.idx;
      const T jy = (T)(jval<Acc>(a.jacc, plane + o) * a.jscale[1]);
      a.ey[o] = a.ey[o] - a.cdt * (dbzdx + jy);
      // ez: dby_dx = (by(i+1,j) - by(i,j)) * idx, dbx_dy = (bx(i,j+1) - bx(i,j)) * idy
      const T dbydx = (a.by[(long long)ip * a.S + j] - a.by[o]) * a.idx;
      const T bxn = node_row(a.bx, i, j + 1, a.my, a.S, a.ybc);
      const T dbxdy = (bxn - a.bx[o]) * a.idy;
      const T jz = (T)(jval<Acc>(a.jacc, 2 * plane + o) * a.jscale[2]);
      a.ez[o] = a.ez[o] + a.cdt * (dbydx - dbxdy - jz);
    }
  }
}

template <class T, class Acc>
__global__ void k_efull(FieldParams<T> a) {
  efull_body<T, Acc>(a);
}

// Node averages (emfgrid, pic2d.f90:838-845) and the field energy sums
// (pic2d.f90:659-670; with walls the two wall rows carry weight 1/2).
// Block `bid` of `nblk` writes partial sums `bid` (the partition of the sums,
// and so their rounding, depends only on nblk).
template <class T>
__device__ __forceinline__ void node_at(const FieldParams<T>& a, int ia, int b, T& e2, T& b2) {
  const int NY = a.my + 1;
  const int i = ia == a.mx ? 0 : ia;
  const int im = wrapx(i - 1, a.mx);
  const long long oi = (long long)i * a.S, om = (long long)im * a.S;
  const int bn = (a.ybc == 0 && b == a.my) ? 0 : b;  // node row
  const T ex = (a.ex[oi + bn] + a.ex[om + bn]) * T(0.5);
  const T bx = (a.bx[oi + bn] + a.bx[om + bn]) * T(0.5);
  const T ey = (half_row(a.ey, i, b, a.my, a.S, a.ybc, T(1)) +
                half_row(a.ey, i, b - 1, a.my, a.S, a.ybc, T(1))) * T(0.5);
  const T by = (half_row(a.by, i, b, a.my, a.S, a.ybc, T(-1)) +
                half_row(a.by, i, b - 1, a.my, a.S, a.ybc, T(-1))) * T(0.5);
  const T ez = (half_row(a.ez, i, b, a.my, a.S, a.ybc, T(-1)) +
                half_row(a.ez, im, b, a.my, a.S, a.ybc, T(-1)) +
                half_row(a.ez, i, b - 1, a.my, a.S, a.ybc, T(-1)) +
                half_row(a.ez, im, b - 1, a.my, a.S, a.ybc, T(-1))) * T(0.25);
  const T bz = (half_row(a.bz, i, b, a.my, a.S, a.ybc, T(1)) +
                half_row(a.bz, im, b, a.my, a.S, a.ybc, T(1)) +
                half_row(a.bz, i, b - 1, a.my, a.S, a.ybc, T(1)) +
                half_row(a.bz, im, b - 1, a.my, a.S, a.ybc, T(1))) * T(0.25);
  T* g = a.ng + ((long long)ia * NY + b) * 8;
  g[0] = ex;
  g[1] = ey;
  g[2] = ez;
  g[3] = T(0);
  g[4] = bx;
  g[5] = by;
  g[6] = bz;
  g[7] = T(0);
  e2 = ex * ex + ey * ey + ez * ez;
  b2 = bx * bx + by * by + bz * bz;
}

template <class T>
__device__ __forceinline__ void nodes_body(const FieldParams<T>& a, double* red, int bid, int nblk) {
  const int NX = a.mx + 1, NY = a.my + 1;
  const long long n = (long long)NX * NY;
  double se = 0.0, sb = 0.0;
  for (long long k = bid * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)nblk * blockDim.x) {
    const int ia = (int)(k / NY), b = (int)(k - (long long)ia * NY);
    T e2, b2;
    node_at(a, ia, b, e2, b2);
    if (ia < a.mx && (a.ybc == 1 || b < a.my)) {
      const double w = (a.ybc == 1 && (b == 0 || b == a.my)) ? 0.5 : 1.0;
      se += w * (double)e2;
      sb += w * (double)b2;
    }
  }
  const double te = block_sum(se, red);
  const double tb = block_sum(sb, red);
  if (threadIdx.x == 0) {
    a.fe_part[2 * bid] = te;
    a.fe_part[2 * bid + 1] = tb;
  }
}

// Node averages of node rows [b0, b1) only (after a few field rows were set),
// the same values as the whole-grid pass; no energy sums.
template <class T>
__global__ void k_nodes_rows(FieldParams<T> a, int b0, int b1) {
  const int R = b1 - b0;
  const long long n = (long long)(a.mx + 1) * R;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int ia = (int)(k / R), b = b0 + (int)(k - (long long)ia * R);
    T e2, b2;
    node_at(a, ia, b, e2, b2);
  }
}

template <class T>
__global__ void k_nodes(FieldParams<T> a) {
  __shared__ double red[32];
  nodes_body(a, red, blockIdx.x, gridDim.x);
}

// Gather records of the mixed-form push from the node grid: cell (cx, cy)
// gets, from its nodes (cx, cy), (cx, cy+1), (cx+1, cy), (cx+1, cy+1), the
// bilinear coefficients (A, B, C, D) of each of ex ey ez bx by bz over the cell
// (with PBPIC_CELL_COEF = 0 the 4 nodes themselves), as 6 contiguous 16-byte
// stores, so the push reads a cell's gather data with 6 loads from one address.
__device__ __forceinline__ void cell_record(const FieldParams<float>& a, int cx, int cy) {
  const long long c = (long long)cx * a.my + cy;
  const float4* g00 = reinterpret_cast<const float4*>(a.ng + ((long long)cx * (a.my + 1) + cy) * 8);
  const float4* g10 = g00 + 2 * (long long)(a.my + 1);
  const float4 p0 = g00[0], q0 = g00[1], p1 = g00[2], q1 = g00[3];  // nodes 00, 01: ex ey ez 0 | bx by bz 0
  const float4 p2 = g10[0], q2 = g10[1], p3 = g10[2], q3 = g10[3];  // nodes 10, 11
  float4* r = reinterpret_cast<float4*>(a.cg + c * 24);
#if PBPIC_CELL_COEF
  // per field: A = mean of the 4 nodes, B = x slope, C = y slope, D = twist
  auto coef = [](float n00, float n01, float n10, float n11) {
    const float sx0 = __fadd_rn(n00, n01), sx1 = __fadd_rn(n10, n11);
    const float sy0 = __fadd_rn(n00, n10), sy1 = __fadd_rn(n01, n11);
    return make_float4(__fmul_rn(0.25f, __fadd_rn(sx0, sx1)), __fmul_rn(0.5f, __fsub_rn(sx1, sx0)),
                       __fmul_rn(0.5f, __fsub_rn(sy1, sy0)), __fsub_rn(__fsub_rn(n11, n10), __fsub_rn(n01, n00)));
  };
  r[0] = coef(p0.x, p1.x, p2.x, p3.x);
  r[1] = coef(p0.y, p1.y, p2.y, p3.y);
  r[2] = coef(p0.z, p1.z, p2.z, p3.z);
  r[3] = coef(q0.x, q1.x, q2.x, q3.x);
  r[4] = coef(q0.y, q1.y, q2.y, q3.y);
  r[5] = coef(q0.z, q1.z, q2.z, q3.z);
#else
  r[0] = make_float4(p0.x, p0.y, p0.z, q0.x);
  r[1] = make_float4(q0.y, q0.z, p1.x, p1.y);
  r[2] = make_float4(p1.z, q1.x, q1.y, q1.z);
  r[3] = make_float4(p2.x, p2.y, p2.z, q2.x);
  r[4] = make_float4(q2.y, q2.z, p3.x, p3.y);
  r[5] = make_float4(p3.z, q3.x, q3.y, q3.z);
#endif
}

__device__ __forceinline__ void cell_records_body(const FieldParams<float>& a, int bid, int nblk) {
  const long long n = (long long)a.mx * a.my;
  for (long long c = bid * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)nblk * blockDim.x) {
    const int cx = (int)(c / a.my), cy = (int)(c - (long long)cx * a.my);
    cell_record(a, cx, cy);
  }
}

// Gather records of cell rows [r0, r1) only.
static __global__ void k_cell_records_rows(FieldParams<float> a, int r0, int r1) {
  const int R = r1 - r0;
  const long long n = (long long)a.mx * R;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int cx = (int)(k / R), cy = r0 + (int)(k - (long long)cx * R);
    cell_record(a, cx, cy);
  }
}

static __global__ void k_cell_records(FieldParams<float> a) { cell_records_body(a, blockIdx.x, gridDim.x); }

// Optional field filters, periodic y only: Marder divergence cleaning
// (divergenceclean, pic2d.f90:867-886) and the Cherenkov filter
// (suppresscerenkov, pic2d.f90:889-907), whose call the reference comments
// out right after the E update (pic2d.f90:754-755). Both act with E from
// before the update (the reference reads terms stored by the previous field
// solve) and with rho of this step's push: k_filter_prep computes the
// corrections before the update, k_filter_apply adds them after it.
template <class T>
struct FilterParams {
  int flags;             // bit 0 Marder, bit 1 Cherenkov
  T mdx, mdy;            // dt * d / dx, dt * d / dy          (pic2d.f90:874-875)
  T cdx, cdy;            // dt * cva2 * tau / dx, .. / dy       (pic2d.f90:896-897)
  T cva2;
  T* fc;                 // 5 planes of mx x my: Marder ex, ey; Cherenkov ex, ey, ez
};

template <class T, class Acc>
struct FilterOps {
  const FieldParams<T>& a;
  __device__ T ex(int i, int j) const { return a.ex[(long long)wrapx(i, a.mx) * a.S + wrapx(j, a.my)]; }
  __device__ T ey(int i, int j) const { return a.ey[(long long)wrapx(i, a.mx) * a.S + wrapx(j, a.my)]; }
  __device__ T ez(int i, int j) const { return a.ez[(long long)wrapx(i, a.mx) * a.S + wrapx(j, a.my)]; }
  __device__ T rho(int i, int j) const {
    const long long plane = (long long)a.mx * a.S;
    return (T)(jval<Acc>(a.jacc, 3 * plane + (long long)wrapx(i, a.mx) * a.S + wrapx(j, a.my)) * a.jscale[3]);
  }
  __device__ T marder_f(int i, int j, T cva2) const {  // dive - cva2 * rho at node (i, j)
    const T dive = (ex(i, j) - ex(i - 1, j)) * a.idx + (ey(i, j) - ey(i, j - 1)) * a.idy;
    return dive - cva2 * rho(i, j);
  }
  __device__ T dexdy(int i, int j) const { return (ex(i, j + 1) - ex(i, j)) * a.idy; }
  __device__ T deydx(int i, int j) const { return (ey(i + 1, j) - ey(i, j)) * a.idx; }
  __device__ T dezdx(int i, int j) const { return (ez(i, j) - ez(i - 1, j)) * a.idx; }
  __device__ T dezdy(int i, int j) const { return (ez(i, j) - ez(i, j - 1)) * a.idy; }
};

template <class T, class Acc>
__global__ void k_filter_prep(FieldParams<T> a, FilterParams<T> f) {
  const FilterOps<T, Acc> op{a};
  const long long pl = (long long)a.mx * a.my;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < pl; k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k / a.my), j = (int)(k - (long long)i * a.my);
    if (f.flags & 1) {
      const T m = op.marder_f(i, j, f.cva2);
      f.fc[k] = f.mdx * (op.marder_f(i + 1, j, f.cva2) - m);
      f.fc[pl + k] = f.mdy * (op.marder_f(i, j + 1, f.cva2) - m);
    }
    if (f.flags & 2) {
      f.fc[2 * pl + k] = f.cdy * (op.deydx(i, j) - op.deydx(i, j - 1) - op.dexdy(i, j) + op.dexdy(i, j - 1));
      f.fc[3 * pl + k] = f.cdx * (-op.deydx(i, j) + op.deydx(i - 1, j) + op.dexdy(i, j) - op.dexdy(i - 1, j));
      f.fc[4 * pl + k] = f.cdx * (op.dezdx(i + 1, j) - op.dezdx(i, j)) + f.cdy * (op.dezdy(i, j + 1) - op.dezdy(i, j));
    }
  }
}

template <class T>
__global__ void k_filter_apply(FieldParams<T> a, FilterParams<T> f) {
  const long long pl = (long long)a.mx * a.my;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < pl; k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k / a.my), j = (int)(k - (long long)i * a.my);
    const long long o = (long long)i * a.S + j;
    T ex = a.ex[o], ey = a.ey[o], ez = a.ez[o];
    if (f.flags & 1) {  // divergenceclean first, as the commented calls
      ex = ex + f.fc[k];
      ey = ey + f.fc[pl + k];
    }
    if (f.flags & 2) {
      ex = ex - f.fc[2 * pl + k];
      ey = ey - f.fc[3 * pl + k];
      ez = ez + f.fc[4 * pl + k];
    }
    a.ex[o] = ex;
    a.ey[o] = ey;
    a.ez[o] = ez;
  }
}

// Batched domains: grid row blockIdx.y works on domain blockIdx.y.
template <class T>
__global__ void k_bhalf_batched(const FieldParams<T>* d) {
  __shared__ FieldParams<T> a;
  if (threadIdx.x == 0) a = d[blockIdx.y];
  __syncthreads();
  bhalf_body(a);
}
template <class T, class Acc>
__global__ void k_efull_batched(const FieldParams<T>* d) {
  __shared__ FieldParams<T> a;
  if (threadIdx.x == 0) a = d[blockIdx.y];
  __syncthreads();
  efull_body<T, Acc>(a);
}
template <class T>
__global__ void k_nodes_batched(const FieldParams<T>* d) {
  __shared__ FieldParams<T> a;
  __shared__ double red[32];
  if (threadIdx.x == 0) a = d[blockIdx.y];
  __syncthreads();
  if ((int)blockIdx.x < a.nblk) nodes_body(a, red, blockIdx.x, a.nblk);
}
static __global__ void k_cell_records_batched(const FieldParams<float>* d) {
  __shared__ FieldParams<float> a;
  if (threadIdx.x == 0) a = d[blockIdx.y];
  __syncthreads();
  cell_records_body(a, blockIdx.x, gridDim.x);
}

// Sum the per-tile kinetic and per-block field partials in a fixed order and
// write one row (electron KE, ion KE, E energy, B energy) of the history.
// Either pointer may be null, in which case that half of the row is kept.
static __global__ void k_energy_row(const double* ke_part, int nke, const double* fe_part, int nfe,
                             double fe_scale, double fb_scale, double* row) {
  __shared__ double red[32];
  double s[4] = {0, 0, 0, 0};
  if (ke_part)
    for (int i = threadIdx.x; i < nke; i += blockDim.x) {
      s[0] += ke_part[2 * i];
      s[1] += ke_part[2 * i + 1];
    }
  if (fe_part)
    for (int i = threadIdx.x; i < nfe; i += blockDim.x) {
      s[2] += fe_part[2 * i];
      s[3] += fe_part[2 * i + 1];
    }
  for (int c = 0; c < 4; ++c) {
    const double t = block_sum(s[c], red);
    if (threadIdx.x == 0) {
      if (c < 2 && ke_part) row[c] = t;
      if (c == 2 && fe_part) row[2] = t * fe_scale;
      if (c == 3 && fe_part) row[3] = t * fb_scale;
    }
  }
}

// One energy row per domain (block blockIdx.x works on domain blockIdx.x),
// written to row *step of the domain's rows (same sums as k_energy_row).
struct EnergyRow {
  const double* ke_part;
  int nke;
  const double* fe_part;
  int nfe;
  double fe_scale, fb_scale;
  double* rows;
};

static __global__ void k_energy_rows_batched(const EnergyRow* d, const int* step) {
  __shared__ double red[32];
  const EnergyRow r = d[blockIdx.x];
  double* row = r.rows + 4 * (long long)(*step);
  double s[4] = {0, 0, 0, 0};
  for (int i = threadIdx.x; i < r.nke; i += blockDim.x) {
    s[0] += r.ke_part[2 * i];
    s[1] += r.ke_part[2 * i + 1];
  }
  for (int i = threadIdx.x; i < r.nfe; i += blockDim.x) {
    s[2] += r.fe_part[2 * i];
    s[3] += r.fe_part[2 * i + 1];
  }
  for (int c = 0; c < 4; ++c) {
    const double t = block_sum(s[c], red);
    if (threadIdx.x == 0) row[c] = c == 2 ? t * r.fe_scale : (c == 3 ? t * r.fb_scale : t);
  }
}

}  // namespace pbd
