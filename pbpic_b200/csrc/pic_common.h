// Shared host/device definitions for the pbpic B200 step: the counter-based
// random number generator, a self-contained logarithm, the Gaussian sampler
// and the plasma loaders.
//
// Every function here compiles both for the GPU (nvcc, device code) and for
// the host (gcc). Double-precision arithmetic goes through the PIC_D* macros,
// which map to the explicitly rounded CUDA intrinsics on the device and to
// plain IEEE operations on the host (host code is compiled with
// -ffp-contract=off), so the GPU loader and a CPU loader produce bit-identical
// particles from the same seed.
//
// The reference seeds Fortran's random_number from /dev/urandom
// (src/programs/pic2d.f90:2486-2532), which is not reproducible; all seeded
// inputs of this implementation come from Philox4x64-10 instead (Salmon,
// Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11).
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define PIC_HD __host__ __device__ __forceinline__
#define PIC_UNROLL _Pragma("unroll")
#else
#define PIC_HD inline
#define PIC_UNROLL
#endif

#if defined(__CUDA_ARCH__)
#define PIC_DMUL(a, b) __dmul_rn((a), (b))
#define PIC_DADD(a, b) __dadd_rn((a), (b))
#define PIC_DSUB(a, b) __dsub_rn((a), (b))
#define PIC_DDIV(a, b) __ddiv_rn((a), (b))
#define PIC_DSQRT(a) __dsqrt_rn((a))
#else
#include <math.h>
#define PIC_DMUL(a, b) ((a) * (b))
#define PIC_DADD(a, b) ((a) + (b))
#define PIC_DSUB(a, b) ((a) - (b))
#define PIC_DDIV(a, b) ((a) / (b))
#define PIC_DSQRT(a) sqrt((a))
#endif

namespace pic {

// ---------------------------------------------------------------------------
// Philox4x64-10 (SC'11 paper, section 3). Multipliers and Weyl increments are
// the published ones. numpy.random.Philox implements the same generator; it
// increments its counter before each block, so numpy's block c equals
// philox4x64(counter = c + 1).
// ---------------------------------------------------------------------------
struct u64x4 {
  uint64_t v[4];
};

PIC_HD void mulhilo64(uint64_t a, uint64_t b, uint64_t* hi, uint64_t* lo) {
#if defined(__CUDA_ARCH__)
  *lo = a * b;
  *hi = __umul64hi(a, b);
#else
  unsigned __int128 p = (unsigned __int128)a * (unsigned __int128)b;
  *lo = (uint64_t)p;
  *hi = (uint64_t)(p >> 64);
#endif
}

PIC_HD u64x4 philox4x64(uint64_t c0, uint64_t c1, uint64_t c2, uint64_t c3,
                        uint64_t k0, uint64_t k1) {
  const uint64_t M0 = 0xD2E7470EE14C6C93ull, M1 = 0xCA5A826395121157ull;
  const uint64_t W0 = 0x9E3779B97F4A7C15ull, W1 = 0xBB67AE8584CAA73Bull;
  uint64_t x0 = c0, x1 = c1, x2 = c2, x3 = c3;
PIC_UNROLL
  for (int r = 0; r < 10; ++r) {
    uint64_t hi0, lo0, hi1, lo1;
    mulhilo64(M0, x0, &hi0, &lo0);
    mulhilo64(M1, x2, &hi1, &lo1);
    uint64_t y0 = hi1 ^ x1 ^ k0;
    uint64_t y2 = hi0 ^ x3 ^ k1;
    x0 = y0;
    x1 = lo1;
    x2 = y2;
    x3 = lo0;
    k0 += W0;
    k1 += W1;
  }
  u64x4 out;
  out.v[0] = x0;
  out.v[1] = x1;
  out.v[2] = x2;
  out.v[3] = x3;
  return out;
}

// Uniform double in [0, 1) from the top 53 bits.
PIC_HD double u01(uint64_t x) { return (double)(x >> 11) * 1.1102230246251565404e-16; }

// ---------------------------------------------------------------------------
// Natural logarithm of a positive normal double, written from the identity
//   log(m * 2^e) = e*ln2 + 2*atanh(s),  s = (m-1)/(m+1),  m in [sqrt(1/2), sqrt(2))
// with the atanh Taylor series s + s^3/3 + s^5/5 + ... summed by Horner's
// rule to s^25 (|s| <= 0.1716, so the first omitted term is below 1e-20).
// It is used only by the loaders; it exists so that the host and the device
// evaluate exactly the same sequence of IEEE operations.
// ---------------------------------------------------------------------------
PIC_HD double pic_log(double x) {
  uint64_t bits;
#if defined(__CUDA_ARCH__)
  bits = (uint64_t)__double_as_longlong(x);
#else
  __builtin_memcpy(&bits, &x, 8);
#endif
  int e = (int)((bits >> 52) & 0x7ff) - 1023;
  uint64_t mbits = (bits & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull;  // m in [1,2)
  double m;
#if defined(__CUDA_ARCH__)
  m = __longlong_as_double((long long)mbits);
#else
  __builtin_memcpy(&m, &mbits, 8);
#endif
  if (m > 1.4142135623730950488) {  // bring m into [sqrt(1/2), sqrt(2))
    m = PIC_DMUL(m, 0.5);
    e += 1;
  }
  double s = PIC_DDIV(PIC_DSUB(m, 1.0), PIC_DADD(m, 1.0));
  double s2 = PIC_DMUL(s, s);
  double p = 1.0 / 25.0;
  // Horner: p = 1/(2k+1) + s2 * p, k = 11 .. 0
  p = PIC_DADD(1.0 / 23.0, PIC_DMUL(s2, p));
  p = PIC_DADD(1.0 / 21.0, PIC_DMUL(s2, p));
  p = PIC_DADD(1.0 / 19.0, PIC_DMUL(s2, p));
  p = PIC_DADD(1.0 / 17.0, PIC_DMUL(s2, p));
  p = PIC_DADD(1.0 / 15.0, PIC_DMUL(s2, p));
  p = PIC_DADD(1.0 / 13.0, PIC_DMUL(s2, p));
  p = PIC_DADD(1.0 / 11.0, PIC_DMUL(s2, p));
  p = PIC_DADD(1.0 / 9.0, PIC_DMUL(s2, p));
  p = PIC_DADD(1.0 / 7.0, PIC_DMUL(s2, p));
  p = PIC_DADD(1.0 / 5.0, PIC_DMUL(s2, p));
  p = PIC_DADD(1.0 / 3.0, PIC_DMUL(s2, p));
  p = PIC_DADD(1.0, PIC_DMUL(s2, p));
  double logm = PIC_DMUL(PIC_DMUL(2.0, s), p);
  const double LN2 = 0.69314718055994530942;
  return PIC_DADD(PIC_DMUL((double)e, LN2), logm);
}

// ---------------------------------------------------------------------------
// Gaussian deviates by the Marsaglia polar method, the method the reference
// uses in gaussianrand (src/programs/pic2d.f90:2538-2552): draw v1, v2 uniform
// in (-1, 1) until 0 < r^2 < 1, then fac = sqrt(-2 log(r^2) / r^2).
// Each Philox block supplies two candidate pairs.
// ---------------------------------------------------------------------------
struct GaussStream {
  uint64_t k0, k1, c0, c1;  // key and the fixed counter words
  uint64_t block;           // next counter block
  double pend[4];
  int npend;
  double saved;
  int have_saved;
};

PIC_HD void gauss_init(GaussStream* g, uint64_t key0, uint64_t key1, uint64_t c0, uint64_t c1) {
  g->k0 = key0;
  g->k1 = key1;
  g->c0 = c0;
  g->c1 = c1;
  g->block = 0;
  g->npend = 0;
  g->have_saved = 0;
  g->saved = 0.0;
}

PIC_HD double gauss_next(GaussStream* g) {
  if (g->have_saved) {
    g->have_saved = 0;
    return g->saved;
  }
  for (int guard = 0; guard < 4096; ++guard) {
    if (g->npend == 0) {
      u64x4 r = philox4x64(g->c0, g->c1, g->block, 0, g->k0, g->k1);
      g->block += 1;
      g->pend[0] = u01(r.v[0]);
      g->pend[1] = u01(r.v[1]);
      g->pend[2] = u01(r.v[2]);
      g->pend[3] = u01(r.v[3]);
      g->npend = 4;
    }
    double a = g->pend[4 - g->npend];
    double b = g->pend[5 - g->npend];
    g->npend -= 2;
    double v1 = PIC_DSUB(PIC_DMUL(2.0, a), 1.0);
    double v2 = PIC_DSUB(PIC_DMUL(2.0, b), 1.0);
    double rsq = PIC_DADD(PIC_DMUL(v1, v1), PIC_DMUL(v2, v2));
    if (rsq >= 1.0 || rsq == 0.0) continue;
    double fac = PIC_DSQRT(PIC_DDIV(PIC_DMUL(-2.0, pic_log(rsq)), rsq));
    g->saved = PIC_DMUL(v2, fac);
    g->have_saved = 1;
    return PIC_DMUL(v1, fac);
  }
  return 0.0;  // unreachable in practice: 4096 rejected pairs has probability < 1e-2700
}

// ---------------------------------------------------------------------------
// Plasma loaders. Particles come in co-located (ion, electron) pairs, so the
// initial charge density is exactly zero and Gauss's law holds with E = 0.
// ---------------------------------------------------------------------------
enum LoadKind {
  LOAD_UNIFORM = 0,     // uniform Maxwellian, stratified: ppc pairs in every cell
  LOAD_HARRIS = 1,      // GEM Harris sheet (normal along y) plus uniform background
  LOAD_TWO_STREAM = 2,  // counter-drifting electron beams along x
  LOAD_WEIBEL = 3,      // bi-Maxwellian electrons, T_perp / T_par = anisotropy
  LOAD_DOUBLE_HARRIS = 4,  // two sheets normal to x at Lx/4, 3Lx/4 (pic2d.f90:357-578)
};

struct LoadParams {
  int32_t kind;
  int32_t mx, my;
  double dx, dy;           // cell size (d_i)
  int64_t npairs;          // number of (ion, electron) pairs to load
  int64_t nsheet;          // Harris: the first nsheet pairs belong to the sheet
  int32_t ppc;             // uniform loader: pairs per cell
  double uthe, uthi;       // thermal momenta u = gamma v / c (electron, ion), parallel
  double uthe_perp;        // Weibel: perpendicular electron thermal momentum
  double udrift_e, udrift_i;  // drift momenta (z for Harris, x for two-stream)
  double lambda;           // Harris half-thickness (d_i)
  uint64_t seed;
  double uthe_bg, uthi_bg;  // double Harris: background thermal momenta (x and y)
};

// One loaded particle in double precision, before conversion to storage type.
struct LoadedParticle {
  int32_t ix, iy;  // 0-based cell
  double ox, oy;   // offset from the cell centre, in [-0.5, 0.5)
  double ux, uy, uz;
};

PIC_HD void place(const LoadParams& L, double x, double y, LoadedParticle* p) {
  double fx = PIC_DDIV(x, L.dx), fy = PIC_DDIV(y, L.dy);
  int ix = (int)fx, iy = (int)fy;  // x, y >= 0 so truncation is floor
  if (ix > L.mx - 1) ix = L.mx - 1;
  if (iy > L.my - 1) iy = L.my - 1;
  if (ix < 0) ix = 0;
  if (iy < 0) iy = 0;
  p->ix = ix;
  p->iy = iy;
  p->ox = PIC_DSUB(PIC_DSUB(fx, (double)ix), 0.5);
  p->oy = PIC_DSUB(PIC_DSUB(fy, (double)iy), 0.5);
}

static const uint64_t PIC_LOAD_SALT = 0x5049434C4F414431ull;  // "PICLOAD1"

// Load pair k: out[0] is the ion (q = +1), out[1] the electron (q = -1).
PIC_HD void load_pair(const LoadParams& L, int64_t k, LoadedParticle out[2]) {
  const uint64_t key0 = L.seed, key1 = PIC_LOAD_SALT;
  double Lx = PIC_DMUL((double)L.mx, L.dx), Ly = PIC_DMUL((double)L.my, L.dy);
  LoadedParticle pos;
  if (L.kind == LOAD_UNIFORM || L.kind == LOAD_TWO_STREAM || L.kind == LOAD_WEIBEL) {
    u64x4 r = philox4x64((uint64_t)k, 0, 0, 0, key0, key1);
    if (L.kind == LOAD_UNIFORM && L.ppc > 0) {
      int64_t cell = k / L.ppc;  // stratified: cell index in sorted (y fastest) order
      pos.ix = (int32_t)(cell / L.my);
      pos.iy = (int32_t)(cell % L.my);
      pos.ox = PIC_DSUB(u01(r.v[0]), 0.5);
      pos.oy = PIC_DSUB(u01(r.v[1]), 0.5);
    } else {
      place(L, PIC_DMUL(u01(r.v[0]), Lx), PIC_DMUL(u01(r.v[1]), Ly), &pos);
    }
  } else if (L.kind == LOAD_DOUBLE_HARRIS) {
    if (k < L.nsheet) {
      // even pairs in the sheet at Lx/4, odd ones in the sheet at 3Lx/4; x from
      // the sech^2 profile by the logistic sampling of pic2d.f90:398-412 and
      // 453-466, redrawn outside the box; y uniform
      const double xc = PIC_DMUL((k & 1) ? 0.75 : 0.25, Lx);
      double x = xc, y = 0.0;
      for (uint64_t attempt = 0; attempt < 1024; ++attempt) {
        u64x4 r = philox4x64((uint64_t)k, 0, attempt, 0, key0, key1);
        double u = u01(r.v[0]);
        if (u < 1e-10) u = 1e-10;
        if (u > 1.0 - 1e-10) u = 1.0 - 1e-10;
        double t = pic_log(PIC_DDIV(u, PIC_DSUB(1.0, u)));
        x = PIC_DADD(xc, PIC_DMUL(PIC_DMUL(0.5, L.lambda), t));
        y = PIC_DMUL(u01(r.v[1]), Ly);
        if (x >= 0.0 && x < Lx) break;
        x = xc;
      }
      place(L, x, y, &pos);
    } else {
      u64x4 r = philox4x64((uint64_t)k, 0, 0, 0, key0, key1);
      place(L, PIC_DMUL(u01(r.v[0]), Lx), PIC_DMUL(u01(r.v[1]), Ly), &pos);
    }
  } else {  // LOAD_HARRIS
    if (k < L.nsheet) {
      // sech^2 profile centred at Ly/2 by inverting its CDF: y = (lambda/2) log(u/(1-u)),
      // the same logistic sampling as the reference (pic2d.f90:400-411); samples
      // outside the box are redrawn.
      double x = 0.0, y = 0.0;
      for (uint64_t attempt = 0; attempt < 1024; ++attempt) {
        u64x4 r = philox4x64((uint64_t)k, 0, attempt, 0, key0, key1);
        double u = u01(r.v[1]);
        if (u < 1e-10) u = 1e-10;
        if (u > 1.0 - 1e-10) u = 1.0 - 1e-10;
        double t = pic_log(PIC_DDIV(u, PIC_DSUB(1.0, u)));
        y = PIC_DADD(PIC_DMUL(0.5, Ly), PIC_DMUL(PIC_DMUL(0.5, L.lambda), t));
        x = PIC_DMUL(u01(r.v[0]), Lx);
        if (y >= 0.0 && y < Ly) break;
        y = PIC_DMUL(0.5, Ly);
      }
      place(L, x, y, &pos);
    } else {
      u64x4 r = philox4x64((uint64_t)k, 0, 0, 0, key0, key1);
      place(L, PIC_DMUL(u01(r.v[0]), Lx), PIC_DMUL(u01(r.v[1]), Ly), &pos);
    }
  }
  out[0] = pos;
  out[1] = pos;
  GaussStream gi, ge;
  gauss_init(&gi, key0, key1, (uint64_t)k, 1);
  gauss_init(&ge, key0, key1, (uint64_t)k, 2);
  double gi0 = gauss_next(&gi), gi1 = gauss_next(&gi), gi2 = gauss_next(&gi);
  double ge0 = gauss_next(&ge), ge1 = gauss_next(&ge), ge2 = gauss_next(&ge);
  switch (L.kind) {
    case LOAD_HARRIS: {
      bool sheet = k < L.nsheet;
      out[0].ux = PIC_DMUL(gi0, L.uthi);
      out[0].uy = PIC_DMUL(gi1, L.uthi);
      out[0].uz = PIC_DADD(PIC_DMUL(gi2, L.uthi), sheet ? L.udrift_i : 0.0);
      out[1].ux = PIC_DMUL(ge0, L.uthe);
      out[1].uy = PIC_DMUL(ge1, L.uthe);
      out[1].uz = PIC_DADD(PIC_DMUL(ge2, L.uthe), sheet ? L.udrift_e : 0.0);
      break;
    }
    case LOAD_DOUBLE_HARRIS: {  // pic2d.f90:436-448, 490-502, 539-551: no thermal motion along z
      const bool sheet = k < L.nsheet;
      const double sgn = (k & 1) ? -1.0 : 1.0;  // the second sheet drifts the other way
      const double ui = sheet ? L.uthi : L.uthi_bg, ue = sheet ? L.uthe : L.uthe_bg;
      out[0].ux = PIC_DMUL(gi0, ui);
      out[0].uy = PIC_DMUL(gi1, ui);
      out[0].uz = sheet ? PIC_DMUL(sgn, L.udrift_i) : 0.0;
      out[1].ux = PIC_DMUL(ge0, ue);
      out[1].uy = PIC_DMUL(ge1, ue);
      out[1].uz = sheet ? PIC_DMUL(sgn, L.udrift_e) : 0.0;
      break;
    }
    case LOAD_TWO_STREAM: {
      double sgn = (k & 1) ? -1.0 : 1.0;
      out[0].ux = 0.0;
      out[0].uy = 0.0;
      out[0].uz = 0.0;
      out[1].ux = PIC_DADD(PIC_DMUL(ge0, L.uthe), PIC_DMUL(sgn, L.udrift_e));
      out[1].uy = PIC_DMUL(ge1, L.uthe);
      out[1].uz = PIC_DMUL(ge2, L.uthe);
      break;
    }
    case LOAD_WEIBEL: {
      out[0].ux = 0.0;
      out[0].uy = 0.0;
      out[0].uz = 0.0;
      out[1].ux = PIC_DMUL(ge0, L.uthe);
      out[1].uy = PIC_DMUL(ge1, L.uthe_perp);
      out[1].uz = PIC_DMUL(ge2, L.uthe_perp);
      break;
    }
    default: {  // LOAD_UNIFORM
      out[0].ux = PIC_DMUL(gi0, L.uthi);
      out[0].uy = PIC_DMUL(gi1, L.uthi);
      out[0].uz = PIC_DMUL(gi2, L.uthi);
      out[1].ux = PIC_DMUL(ge0, L.uthe);
      out[1].uy = PIC_DMUL(ge1, L.uthe);
      out[1].uz = PIC_DMUL(ge2, L.uthe);
      break;
    }
  }
}

}  // namespace pic
