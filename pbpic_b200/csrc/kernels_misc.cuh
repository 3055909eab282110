// Loading, format conversion and diagnostics kernels.
#pragma once
#include "device_common.cuh"
#include "pic_common.h"

namespace pbd {

// Device plasma loader: one thread per (ion, electron) pair, the same
// generator and arithmetic as the host loader in pic_common.h.
template <class T>
__global__ void k_load(pic::LoadParams L, int64_t npairs, int electrons_only, uint32_t* cell, T* dx,
                       T* dy, T* ux, T* uy, T* uz, int32_t* pid) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= npairs) return;
  pic::LoadedParticle pr[2];
  pic::load_pair(L, k, pr);
  for (int s = electrons_only ? 1 : 0; s < 2; ++s) {
    const int64_t o = electrons_only ? k : 2 * k + s;
    cell[o] = cw_make(pr[s].ix, pr[s].iy, s);
    dx[o] = (T)pr[s].ox;
    dy[o] = (T)pr[s].oy;
    ux[o] = (T)pr[s].ux;
    uy[o] = (T)pr[s].uy;
    uz[o] = (T)pr[s].uz;
    if (pid) pid[o] = (int32_t)(2 * k + s + 1);
  }
}

// The reference's particle record (pic2d.f90:47-50) with real kind R.
template <class R>
struct RefRec;
template <>
struct RefRec<float> {
  float dx, dy, ux, uy, uz;
  int32_t grid, q, pid;
};
template <>
struct RefRec<double> {
  double dx, dy, ux, uy, uz;
  int32_t grid, q, pid, pad;
};

template <class T, class R>
__global__ void k_aos_in(const RefRec<R>* in, int64_t n, int mx, int my, uint32_t* cell, T* dx, T* dy,
                         T* ux, T* uy, T* uz, int32_t* pid, int* status) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const RefRec<R> r = in[i];
    int g = r.grid - 1;
    if (g < 0 || g >= mx * my || (r.q != 1 && r.q != -1)) {
      atomicOr(status, 8);
      g = 0;
    }
    const int ix = g / my, iy = g - (g / my) * my;
    cell[i] = cw_make(ix, iy, r.q < 0 ? 1 : 0);
    dx[i] = (T)r.dx;
    dy[i] = (T)r.dy;
    ux[i] = (T)r.ux;
    uy[i] = (T)r.uy;
    uz[i] = (T)r.uz;
    if (pid) pid[i] = r.pid;
  }
}

// Record i is array element perm[i] (the sort's permutation, not yet applied to
// the arrays) or element i (perm null).
template <class T, class R>
__global__ void k_aos_out(RefRec<R>* out, int64_t n, int my, const int32_t* perm, const uint32_t* cell, const T* dx,
                          const T* dy, const T* ux, const T* uy, const T* uz, const int32_t* pid) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = perm ? (int64_t)perm[i] : i;
    const uint32_t w = cell[e];
    RefRec<R> r;
    r.dx = (R)dx[e];
    r.dy = (R)dy[e];
    r.ux = (R)ux[e];
    r.uy = (R)uy[e];
    r.uz = (R)uz[e];
    r.grid = my * cw_ix(w) + cw_iy(w) + 1;
    r.q = cw_sp(w) ? -1 : 1;
    r.pid = pid ? pid[e] : 0;
    if constexpr (sizeof(RefRec<R>) == 56) r.pad = 0;
    out[i] = r;
  }
}

// Kinetic energy per species of the current particles (pic2d.f90:554-568),
// one partial pair per block.
template <class T, bool MIXED>
__global__ void k_kinetic(int64_t n, const uint32_t* cell, const T* ux, const T* uy, const T* uz, T ms_i,
                          double* part) {
  __shared__ double red[32];
  double ke[2] = {0, 0};
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    using A = M<T, MIXED>;
    const T a = ux[i], b = uy[i], c = uz[i];
    const T usq = A::mad(c, c, A::mad(b, b, A::mul(a, a)));
    const T g = A::sqrt(A::mad(c, c, A::mad(b, b, A::mad(a, a, T(1)))));
    const int sp = cw_sp(cell[i]);
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

// Charge density of the current positions with the gather's CIC weights
// (pic2d.f90:948-951), unnormalised, into a double plane of mx x S.
template <class T>
__global__ void k_rho(int64_t n, int mx, int my, int S, int ybc, const uint32_t* cell, const T* dx,
                      const T* dy, double* rho) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t w = cell[i];
    const int ix = cw_ix(w), iy = cw_iy(w);
    const double q = cw_sp(w) ? -1.0 : 1.0;
    const double ax = 0.5 + (double)dx[i], ay = 0.5 + (double)dy[i];
    const double s1 = ax * ay, s2 = ax - s1, s3 = ay - s1, s4 = 1.0 - s1 - s2 - s3;
    const int ip = ix + 1 == mx ? 0 : ix + 1;
    int jp = iy + 1;
    if (jp == my && ybc == 0) jp = 0;  // periodic: node row my is row 0
    atomicAdd(&rho[(int64_t)ix * S + iy], q * s4);
    atomicAdd(&rho[(int64_t)ip * S + iy], q * s2);
    atomicAdd(&rho[(int64_t)ix * S + jp], q * s3);
    atomicAdd(&rho[(int64_t)ip * S + jp], q * s1);
  }
}

__device__ __forceinline__ void atomic_max_pos(double* addr, double v) {
  atomicMax(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}

// max |div E / cva^2 - in0 rho| over interior nodes; div E at node (i, j) is
// (ex(i,j) - ex(i-1,j))/dx + (ey(i,j) - ey(i,j-1))/dy.
template <class T>
__global__ void k_gauss(int mx, int my, int S, int ybc, int jlo, int jhi, const T* ex, const T* ey,
                        const double* rho, double idx, double idy, double icva2, double in0, double* out) {
  double m = 0.0;
  // node rows [jlo, jhi) of 0..my-1 (walls: interior rows 1..my-1)
  const int j0 = max(jlo, ybc == 0 ? 0 : 1), j1 = min(jhi, my);
  if (j1 <= j0) return;
  const int rows = j1 - j0;
  const int64_t nn = (int64_t)mx * rows;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(k / rows), j = j0 + (int)(k - (int64_t)(k / rows) * rows);
    const int im = i == 0 ? mx - 1 : i - 1;
    const int jm = j == 0 ? my - 1 : j - 1;
    const double dive = ((double)ex[(int64_t)i * S + j] - (double)ex[(int64_t)im * S + j]) * idx +
                        ((double)ey[(int64_t)i * S + j] - (double)ey[(int64_t)i * S + jm]) * idy;
    const double g = fabs(dive * icva2 - in0 * rho[(int64_t)i * S + j]);
    m = fmax(m, g);
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) m = fmax(m, __shfl_down_sync(FULL, m, d));
  if (lane_id() == 0) atomic_max_pos(out, m);
}

// 0.5 * sum_i |By(node i, row my/2)| * dx
template <class T>
__global__ void k_flux(int mx, int my, const T* ng, double dx, double* out) {
  __shared__ double red[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < mx; i += blockDim.x) s += fabs((double)ng[((int64_t)i * (my + 1) + my / 2) * 8 + 5]);
  s = block_sum(s, red);
  if (threadIdx.x == 0) *out = 0.5 * s * dx;
}

// Energy spectra (energyspectra, pic2d.f90:1957-1990): per species the
// number of particles with (gamma - 1) ms in ((k-1) de, k de], k = 1..nbins,
// gamma from the momenta in double. The reference's histogram is indexed
// (bin, species) on a (species, bin) array and can take bin 0 (quirk Q6);
// here it is counts[species][k-1] (species 0 electrons, 1 ions) and an
// energy of exactly 0 counts in bin 1. Block histograms in shared memory.
template <class T>
__global__ void k_spectra(int64_t n, const uint32_t* cell, const T* ux, const T* uy, const T* uz, double mime,
                          double de_e, double de_i, int nbins, unsigned long long* counts) {
  extern __shared__ unsigned int hs[];  // 2 * nbins
  for (int b = threadIdx.x; b < 2 * nbins; b += blockDim.x) hs[b] = 0u;
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double x = ux[i], y = uy[i], z = uz[i];  // explicit rounding: no contraction
    const double g2 = __dadd_rn(__dadd_rn(__dadd_rn(1.0, __dmul_rn(x, x)), __dmul_rn(y, y)), __dmul_rn(z, z));
    const double gama = __dsqrt_rn(g2);
    const int sp = cw_sp(cell[i]) ? 0 : 1;  // 0 electron, 1 ion (j = 1, 2 of the reference)
    const double ms = sp ? mime : 1.0, de = sp ? de_i : de_e;
    const double ene = __dmul_rn(__dsub_rn(gama, 1.0), ms);
    if (ene < __dmul_rn(de, (double)nbins)) {
      int k = (int)ceil(__ddiv_rn(ene, de));
      k = k < 1 ? 1 : (k > nbins ? nbins : k);
      atomicAdd(&hs[sp * nbins + k - 1], 1u);
    }
  }
  __syncthreads();
  for (int b = threadIdx.x; b < 2 * nbins; b += blockDim.x)
    if (hs[b]) atomicAdd(&counts[b], (unsigned long long)hs[b]);
}

// Node values along chosen node rows (all x) and node columns (all y), the
// cuts dispersioninfo stores for the field spectra (pic2d.f90:2124-2142):
// out = [nrows][mx][6] then [ncols][my][6] (ex ey ez bx by bz), double.
template <class T>
__global__ void k_field_cuts(int mx, int my, const T* ng, const int32_t* rows, int nrows, const int32_t* cols,
                             int ncols, double* out) {
  const int64_t nr = (int64_t)nrows * mx, nt = nr + (int64_t)ncols * my;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nt; k += (int64_t)gridDim.x * blockDim.x) {
    int i, j;
    if (k < nr) {
      j = rows[k / mx];
      i = (int)(k % mx);
    } else {
      i = cols[(k - nr) / my];
      j = (int)((k - nr) % my);
    }
    const T* g = ng + ((int64_t)i * (my + 1) + j) * 8;
    double* o = out + k * 6;
    o[0] = g[0];
    o[1] = g[1];
    o[2] = g[2];
    o[3] = g[4];
    o[4] = g[5];
    o[5] = g[6];
  }
}

}  // namespace pbd
