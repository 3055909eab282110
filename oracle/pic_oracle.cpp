// ===========================================================================
// ORACLE -- TEST INFRASTRUCTURE ONLY.
//
// A CPU restatement of the reference's 2-D electromagnetic PIC step
// (xiaocanli/pbpic, src/programs/pic2d.f90), written to check the CUDA
// library. Only tests/, __graft_entry__.smoke() and the cpu_baseline /
// --impl reference legs of bench.py may load it. The product never does.
//
// PARITY UNPINNED: the reference ships no golden vectors, known-answer tests
// or fixtures, and it cannot be built in this environment (no Fortran
// compiler, MPI or HDF5). This file restates its arithmetic line by line
// instead; tests/golden/ pins it against an independent line-by-line Python
// transcription and against physics invariants.
//
// Citation shorthand: F:<line> = src/programs/pic2d.f90:<line>.
//
// What is restated, with the reference's own array conventions
// (1-based cells, grid = my*(ix-1)+iy, guard extents emf(0:mx+1,0:my+1),
// denjr(0:mx+2,0:my+2), column-major storage):
//   pusher          F:912-1217  (gather, Boris, move, deposit call, x wrap,
//                                y crossing with the 1-rank MPI self exchange:
//                                compaction of holes and append, J
//                                normalisation, x fold and y guard fold)
//   currentdeposit  F:1226-1296 (Umeda zig-zag jx/jy, CIC jz at the midpoint,
//                                CIC rho at the old position)
//   fieldsolver     F:678-860   (B half step, E full step, B half step with
//                                stored curl terms, periodic copies and the
//                                1-rank ghost exchange; node averages)
//   fieldsenergy    F:653-673
//   countingsort    F:1303-1329
//   divergenceclean F:867-886, suppresscerenkov F:889-907 (off by default, as
//                   in the reference; periodic y only)
// Additions the reference lacks (the benchmark configurations need them):
//   conducting walls in y (particle reflection, image fold of the guard
//   current, PEC ghost values), switchable corrections of quirks Q1-Q3.
// Deviation kept on purpose: energy sums accumulate in double, not real(4)
// (the reference's real(4) accumulators lose digits over 1e6 particles).
//
// A second, OpenMP-parallel pusher/countingsort (omp_*) exists only as the
// timed CPU baseline: it follows the same arithmetic but keeps every particle
// in its array slot (in-place y wrap, as on the GPU) and sums thread-private
// current arrays.
// ===========================================================================
#include <stdint.h>
#include <string.h>
#include <math.h>
#include <algorithm>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../pbpic_b200/csrc/pic_common.h"
#include "../pbpic_b200/csrc/pic_fields_init.h"

extern "C" {

struct OrcParams {
  int32_t mx, my;
  double dx, dy, dt, cva, mime, in0;
  int32_t ybc;     // 0: periodic (the reference on 1 rank), 1: conducting walls
  int32_t compat;  // bit 0: Q1 Boris, bit 1: Q3 lost jy fold, bit 2: Q2 mirrored rho
};

// The reference's `type particle` (F:47-50) widened to double for exchange.
struct OrcParticle {
  double dx, dy, ux, uy, uz;
  int32_t grid, q, pid, pad;
};
}

namespace {

enum { COMPAT_BORIS = 1, COMPAT_FOLD = 2, COMPAT_RHO = 4 };

// record layouts (F:52-67)
enum { EX = 0, DEX_DY, EY, DEY_DX, EZ, DEZ_DX, DEZ_DY, DIVE, BX, DBX_DY, BY, DBY_DX, BZ, DBZ_DX, DBZ_DY, PAD1 };
enum { GEX = 0, GEY, GEZ, GPAD1, GBX, GBY, GBZ, GPAD2 };
enum { JX = 0, JY, JZ, RHO };

template <class T>
struct Ptl {
  T dx, dy, ux, uy, uz;
  int32_t grid, q, pid;
};

template <class T>
struct Sim {
  int mx, my, ybc, compat;
  T dx, dy, idx, idy, dt, dth, cva, cva2, mime, in0;
  std::vector<T> emf, emfgrid, denjr;
  std::vector<Ptl<T>> ptl, ptlsort;
  int64_t nptlact = 0, nptltot = 0;
  std::vector<int32_t> ptlalloc, counts;
  double ke[2] = {0, 0}, fe[2] = {0, 0};

  // accessors with the reference's lower bounds
  T& E(int c, int i, int j) { return emf[((size_t)j * (mx + 2) + i) * 16 + c]; }
  T& G(int c, int i, int j) { return emfgrid[((size_t)j * (mx + 2) + i) * 8 + c]; }
  T& D(int c, int i, int j) { return denjr[((size_t)j * (mx + 3) + i) * 4 + c]; }

  void init(const OrcParams& p) {
    mx = p.mx;
    my = p.my;
    ybc = p.ybc;
    compat = p.compat;
    dx = (T)p.dx;
    dy = (T)p.dy;
    idx = (T)1.0 / dx;  // F:16
    idy = (T)1.0 / dy;
    dt = (T)p.dt;
    dth = dt / (T)2.0;  // F:43
    cva = (T)p.cva;
    cva2 = cva * cva;   // F:21
    mime = (T)p.mime;
    in0 = (T)p.in0;
    emf.assign((size_t)(mx + 2) * (my + 2) * 16, (T)0);
    emfgrid.assign((size_t)(mx + 2) * (my + 2) * 8, (T)0);
    denjr.assign((size_t)(mx + 3) * (my + 3) * 4, (T)0);
    ptlalloc.assign((size_t)mx * my, 0);
    counts.assign((size_t)mx * my, 0);
  }

  // ----------------------------------------------------------------- deposit
  // currentdeposit, F:1226-1296
  void currentdeposit(int i1, int i2, int j1, int j2, T dx1, T dx2, T dy1, T dy2, int q0, T uz,
                      std::vector<T>* jbuf) {
    auto Dj = [&](int c, int i, int j) -> T& {
      return (*jbuf)[((size_t)j * (mx + 3) + i) * 4 + c];
    };
    T qx = (T)q0 * dx / dt;  // F:1237
    T qy = (T)q0 * dy / dt;
    T im = ((T)(i1 + i2) + dx1 + dx2 + (T)1) * (T)0.5;  // F:1239
    T jm = ((T)(j1 + j2) + dy1 + dy2 + (T)1) * (T)0.5;
    T ir = std::min((T)std::min(i1, i2) + (T)1.0, std::max((T)std::max(i1, i2) + (T)0.0, im));  // F:1241
    T jr = std::min((T)std::min(j1, j2) + (T)1.0, std::max((T)std::max(j1, j2) + (T)0.0, jm));
    T fx1 = qx * (ir - (T)i1 - dx1 - (T)0.5);  // F:1244-1247
    T fy1 = qy * (jr - (T)j1 - dy1 - (T)0.5);
    T fx2 = qx * ((T)i2 + dx2 + (T)0.5 - ir);
    T fy2 = qy * ((T)j2 + dy2 + (T)0.5 - jr);
    T wx1 = (ir - (T)i1 + dx1 + (T)0.5) * (T)0.5;  // F:1249-1252
    T wy1 = (jr - (T)j1 + dy1 + (T)0.5) * (T)0.5;
    T wx2 = (ir - (T)i2 + dx2 + (T)0.5) * (T)0.5;
    T wy2 = (jr - (T)j2 + dy2 + (T)0.5) * (T)0.5;
    Dj(JX, i1, j1) += fx1 * ((T)1.0 - wy1);  // F:1254-1261
    Dj(JX, i1, j1 + 1) += fx1 * wy1;
    Dj(JY, i1, j1) += fy1 * ((T)1.0 - wx1);
    Dj(JY, i1 + 1, j1) += fy1 * wx1;
    Dj(JX, i2, j2) += fx2 * ((T)1.0 - wy2);
    Dj(JX, i2, j2 + 1) += fx2 * wy2;
    Dj(JY, i2, j2) += fy2 * ((T)1.0 - wx2);
    Dj(JY, i2 + 1, j2) += fy2 * wx2;
    T dimid = im - (T)i1 - (T)0.5;  // F:1263-1270
    T djmid = jm - (T)j1 - (T)0.5;
    int di = dimid >= (T)0 ? 1 : -1;
    int dj = djmid >= (T)0 ? 1 : -1;
    dimid = std::fabs(dimid);
    djmid = std::fabs(djmid);
    T s1 = dimid * djmid;  // F:1272-1275
    T s2 = dimid - s1;
    T s3 = djmid - s1;
    T s4 = (T)1.0 - s1 - s2 - s3;
    T quz = (T)q0 * uz;  // F:1277-1281
    Dj(JZ, i1, j1) += quz * s4;
    Dj(JZ, i1 + di, j1) += quz * s2;
    Dj(JZ, i1, j1 + dj) += quz * s3;
    Dj(JZ, i1 + di, j1 + dj) += quz * s1;
    if (compat & COMPAT_RHO) {  // F:1285-1295, weights mirrored (Q2)
      s1 = ((T)0.5 - dx1) * ((T)0.5 - dy1);
      s2 = (T)0.5 - dx1 - s1;
      s3 = (T)0.5 - dy1 - s1;
    } else {  // CIC consistent with the gather weights F:948-951
      s1 = ((T)0.5 + dx1) * ((T)0.5 + dy1);
      s2 = (T)0.5 + dx1 - s1;
      s3 = (T)0.5 + dy1 - s1;
    }
    s4 = (T)1.0 - s1 - s2 - s3;
    Dj(RHO, i1, j1) += s4 * (T)q0;
    Dj(RHO, i1 + 1, j1) += s2 * (T)q0;
    Dj(RHO, i1, j1 + 1) += s3 * (T)q0;
    Dj(RHO, i1 + 1, j1 + 1) += s1 * (T)q0;
  }

  // ------------------------------------------------------------ push kernel
  // Body of the particle loop F:935-1062 for one particle. Returns the cell
  // step in y (iy1) so the caller can apply the y boundary.
  struct Moved {
    int ix, iy1;
    T gama, ms;
  };

  Moved push_one(Ptl<T>& p, std::vector<T>* jbuf) {
    T ux = p.ux, uy = p.uy, uz = p.uz;  // F:935-937
    int ix = (p.grid - 1) / my + 1;      // F:938-939
    int iy = (p.grid - 1) % my + 1;
    T s1 = ((T)0.5 + p.dx) * ((T)0.5 + p.dy);  // F:948-951
    T s2 = (T)0.5 + p.dx - s1;
    T s3 = (T)0.5 + p.dy - s1;
    T s4 = (T)1.0 - s1 - s2 - s3;
    auto gat = [&](int c) {  // F:952-963
      return G(c, ix, iy) * s4 + G(c, ix + 1, iy) * s2 + G(c, ix, iy + 1) * s3 +
             G(c, ix + 1, iy + 1) * s1;
    };
    T ex = gat(GEX), ey = gat(GEY), ez = gat(GEZ);
    T bx = gat(GBX), by = gat(GBY), bz = gat(GBZ);
    T ms = p.q > 0 ? mime : (T)1.0;  // F:964-968
    T c0 = (T)p.q * dt * mime / ms / (T)2.0;  // F:969-970
    T c1 = c0 / cva;
    T umx = ux + c1 * ex;  // F:971-974
    T umy = uy + c1 * ey;
    T umz = uz + c1 * ez;
    T gama = std::sqrt((T)1.0 + umx * umx + umy * umy + umz * umz);
    T c2 = c0 / gama;  // F:976-983
    T tx = c2 * bx, ty = c2 * by, tz = c2 * bz;
    T t2 = (T)2.0 / ((T)1.0 + tx * tx + ty * ty + tz * tz);
    T sx = t2 * tx, sy = t2 * ty, sz = t2 * tz;
    // F:985-987 rotate the pre-kick momentum (Q1); the Boris method rotates u-minus
    T vx = (compat & COMPAT_BORIS) ? ux : umx;
    T vy = (compat & COMPAT_BORIS) ? uy : umy;
    T vz = (compat & COMPAT_BORIS) ? uz : umz;
    T u0x = umx + (vy * tz - vz * ty);
    T u0y = umy + (vz * tx - vx * tz);
    T u0z = umz + (vx * ty - vy * tx);
    T upx = umx + (u0y * sz - u0z * sy);  // F:989-991
    T upy = umy + (u0z * sx - u0x * sz);
    T upz = umz + (u0x * sy - u0y * sx);
    ux = upx + c1 * ex;  // F:993-996
    uy = upy + c1 * ey;
    uz = upz + c1 * ez;
    gama = std::sqrt((T)1.0 + ux * ux + uy * uy + uz * uz);
    p.ux = ux;  // F:998-1000
    p.uy = uy;
    p.uz = uz;
    T dx0 = p.dx, dy0 = p.dy;  // F:1002-1006
    T c3 = dt * cva / gama;
    T dx1 = dx0 + c3 * ux * idx;
    T dy1 = dy0 + c3 * uy * idy;
    int dcellx, dcelly;
    if (std::fabs(dx1) > (T)0.5) {  // F:1008-1023
      dcellx = dx1 >= (T)0 ? 1 : -1;
      p.dx = dx1 + (-dx1 >= (T)0 ? (T)1.0 : (T)-1.0);
    } else {
      dcellx = 0;
      p.dx = dx1;
    }
    if (std::fabs(dy1) > (T)0.5) {
      dcelly = dy1 >= (T)0 ? 1 : -1;
      p.dy = dy1 + (-dy1 >= (T)0 ? (T)1.0 : (T)-1.0);
    } else {
      dcelly = 0;
      p.dy = dy1;
    }
    int ix1 = ix + dcellx;  // F:1025-1026
    int iy1 = iy + dcelly;
    T vzz = uz * cva / gama;  // F:1028-1030
    currentdeposit(ix, ix1, iy, iy1, dx0, p.dx, dy0, p.dy, p.q, vzz, jbuf);
    Moved m;
    m.ix = (ix1 + mx - 1) % mx + 1;  // F:1032
    m.iy1 = iy1;
    m.gama = gama;
    m.ms = ms;
    return m;
  }

  void add_ke(const Ptl<T>& p, T gama, T ms, double* acc) {
    int j = p.q > 0 ? 2 : 1;  // F:1061: j = ceiling(q*0.5+1)
    acc[j - 1] += (double)((gama - (T)1.0) * ms);
  }

  // J normalisation F:1066-1069 and the x fold F:1150-1169
  void normalise_and_fold_x() {
    for (size_t k = 0; k < denjr.size(); ++k) denjr[k] = denjr[k] * in0;
    for (int j = 0; j <= my + 2; ++j) {
      D(JX, 0, j) = D(JX, 0, j) + D(JX, mx, j);
      D(JX, 1, j) = D(JX, 1, j) + D(JX, mx + 1, j);
      D(JX, mx, j) = D(JX, 0, j);
      D(JX, mx + 1, j) = D(JX, 1, j);
      D(JY, 0, j) = D(JY, 0, j) + D(JY, mx, j);
      D(JY, 1, j) = D(JY, 1, j) + D(JY, mx + 1, j);
      if (!(compat & COMPAT_FOLD)) D(JY, 2, j) = D(JY, 2, j) + D(JY, mx + 2, j);  // F:1156 (Q3)
      D(JY, mx, j) = D(JY, 0, j);
      D(JY, mx + 1, j) = D(JY, 1, j);
      if (!(compat & COMPAT_FOLD)) D(JY, mx + 2, j) = D(JY, 2, j);
      D(JZ, 0, j) = D(JZ, 0, j) + D(JZ, mx, j);
      D(JZ, 1, j) = D(JZ, 1, j) + D(JZ, mx + 1, j);
      D(JZ, mx, j) = D(JZ, 0, j);
      D(JZ, mx + 1, j) = D(JZ, 1, j);
      D(RHO, 1, j) = D(RHO, 1, j) + D(RHO, mx + 1, j);
      D(RHO, mx + 1, j) = D(RHO, 1, j);
      D(RHO, 0, j) = D(RHO, mx, j);
    }
  }

  // y guard fold: the 1-rank self exchange F:1171-1216, or the conducting-wall
  // image fold (a guard-row deposit is mirrored into the domain: jx, jz and
  // rho keep their sign, the wall-normal jy flips it).
  void fold_y() {
    if (ybc == 0) {
      int n = mx + 2;
      std::vector<T> sendt(5 * n), sendb(5 * n);
      for (int i = 0; i <= mx + 1; ++i) {
        sendt[i] = D(JX, i, my + 1);
        sendt[n + i] = D(JX, i, my + 2);
        sendt[2 * n + i] = D(JY, i, my + 1);
        sendt[3 * n + i] = D(JZ, i, my + 1);
        sendt[4 * n + i] = D(RHO, i, my + 1);
        sendb[i] = D(JX, i, 0);
        sendb[n + i] = D(JX, i, 1);
        sendb[2 * n + i] = D(JY, i, 0);
        sendb[3 * n + i] = D(JZ, i, 0);
        sendb[4 * n + i] = D(RHO, i, 1);
      }
      const std::vector<T>& recvb = sendt;  // from the left neighbour = this rank
      const std::vector<T>& recvt = sendb;  // from the right neighbour = this rank
      for (int i = 0; i <= mx + 1; ++i) {
        D(JX, i, 1) = D(JX, i, 1) + recvb[i];
        D(JX, i, 2) = D(JX, i, 2) + recvb[n + i];
        D(JY, i, 1) = D(JY, i, 1) + recvb[2 * n + i];
        D(JZ, i, 1) = D(JZ, i, 1) + recvb[3 * n + i];
        D(RHO, i, 1) = D(RHO, i, 1) + recvb[4 * n + i];
        D(JX, i, my) = D(JX, i, my) + recvt[i];
        D(JX, i, my + 1) = D(JX, i, my + 1) + recvt[n + i];
        D(JY, i, my) = D(JY, i, my) + recvt[2 * n + i];
        D(JZ, i, my) = D(JZ, i, my) + recvt[3 * n + i];
        D(RHO, i, my + 1) = D(RHO, i, my + 1) + recvt[4 * n + i];
      }
    } else {
      // walls at node rows 1 and my+1; node rows mirror j -> 2-j and j -> 2(my+1)-j,
      // half rows (jy, jz at j+1/2) mirror j -> 1-j and j -> 2my+1-j.
      for (int i = 0; i <= mx + 2; ++i) {
        D(JX, i, 2) = D(JX, i, 2) + D(JX, i, 0);
        D(JX, i, my) = D(JX, i, my) + D(JX, i, my + 2);
        D(RHO, i, 2) = D(RHO, i, 2) + D(RHO, i, 0);
        D(RHO, i, my) = D(RHO, i, my) + D(RHO, i, my + 2);
        D(JY, i, 1) = D(JY, i, 1) - D(JY, i, 0);
        D(JY, i, my) = D(JY, i, my) - D(JY, i, my + 1);
        D(JZ, i, 1) = D(JZ, i, 1) + D(JZ, i, 0);
        D(JZ, i, my) = D(JZ, i, my) + D(JZ, i, my + 1);
        D(JX, i, 0) = D(JX, i, my + 2) = 0;
        D(RHO, i, 0) = D(RHO, i, my + 2) = 0;
        D(JY, i, 0) = D(JY, i, my + 1) = 0;
        D(JZ, i, 0) = D(JZ, i, my + 1) = 0;
      }
    }
  }

  // pusher, F:912-1217
  void pusher() {
    std::fill(denjr.begin(), denjr.end(), (T)0);  // F:173-176
    ke[0] = ke[1] = 0;
    std::vector<Ptl<T>> sendt, sendb;
    std::vector<int64_t> crossindex;
    for (int64_t i = 0; i < nptlact; ++i) {
      Ptl<T>& p = ptl[i];
      Moved m = push_one(p, &denjr);
      int ix = m.ix, iy;
      if (ybc == 0) {  // F:1033-1053
        if (m.iy1 > my) {
          iy = m.iy1 - my;
          p.grid = my * (ix - 1) + iy;
          sendt.push_back(p);
          p.pid = (int32_t)(nptltot + 1);
          crossindex.push_back(i);
        } else if (m.iy1 < 1) {
          iy = m.iy1 + my;
          p.grid = my * (ix - 1) + iy;
          sendb.push_back(p);
          p.pid = (int32_t)(nptltot + 1);
          crossindex.push_back(i);
        } else {
          iy = m.iy1;
          p.grid = my * (ix - 1) + iy;
        }
      } else {  // conducting walls: specular reflection
        iy = m.iy1;
        if (iy > my || iy < 1) {
          iy = iy > my ? my : 1;
          p.dy = -p.dy;
          p.uy = -p.uy;
        }
        p.grid = my * (ix - 1) + iy;
      }
      add_ke(p, m.gama, m.ms, ke);  // F:1061-1062
    }
    if (ybc == 0) {
      // compaction of the holes left by crossers, F:1072-1083 (0-based j)
      int64_t nptlcross = (int64_t)crossindex.size();
      int64_t j = nptlact - 1;
      for (int64_t k = 0; k < nptlcross; ++k) {
        while (j >= 0 && ptl[j].pid > nptltot) --j;
        if (j < crossindex[k]) break;
        ptl[crossindex[k]] = ptl[j];
        --j;
      }
      nptlact -= nptlcross;
      // 1 rank: the particles sent up come back from below and vice versa;
      // ptlrecvt (= own sendb) is appended first, then ptlrecvb (F:1138-1146)
      for (auto& p : sendb) ptl[nptlact++] = p;
      for (auto& p : sendt) ptl[nptlact++] = p;
    }
    normalise_and_fold_x();
    fold_y();
  }
  // ------------------------------------------------------------ field solver
  void periodic_x(int c) {  // F:693-698 and F:747-752
    for (int j = 0; j <= my + 1; ++j) {
      E(c, 0, j) = E(c, mx, j);
      E(c, 1, j) = E(c, mx + 1, j);
    }
  }
  // ghost rows in y: the 1-rank exchange (F:701-730) or the PEC images
  void ghost_y(int ca, int sa, int cb, int sb) {
    for (int i = 0; i <= mx + 1; ++i) {
      if (ybc == 0) {
        T ta = E(ca, i, my), tb = E(cb, i, my), ba = E(ca, i, 1), bb = E(cb, i, 1);
        E(ca, i, my + 1) = ba;
        E(cb, i, my + 1) = bb;
        E(ca, i, 0) = ta;
        E(cb, i, 0) = tb;
      } else {
        E(ca, i, 0) = (T)sa * E(ca, i, 1);
        E(ca, i, my + 1) = (T)sa * E(ca, i, my);
        E(cb, i, 0) = (T)sb * E(cb, i, 1);
        E(cb, i, my + 1) = (T)sb * E(cb, i, my);
      }
    }
  }

  void b_half() {  // F:688-690, F:801-803
    for (size_t k = 0; k < emf.size(); k += 16) {
      T* f = &emf[k];
      f[BX] = f[BX] - dth * f[DEZ_DY];
      f[BY] = f[BY] + dth * f[DEZ_DX];
      f[BZ] = f[BZ] + dth * (f[DEX_DY] - f[DEY_DX]);
    }
  }

  void curl_e() {  // F:790-798 (dive, a diagnostic with quirk Q4, is not restated)
    for (int j = 1; j <= my; ++j)
      for (int i = 0; i <= mx + 1; ++i) E(DEX_DY, i, j) = (E(EX, i, j + 1) - E(EX, i, j)) * idy;
    for (int j = 0; j <= my + 1; ++j)
      for (int i = 0; i <= mx; ++i) E(DEY_DX, i, j) = (E(EY, i + 1, j) - E(EY, i, j)) * idx;
    for (int j = 0; j <= my + 1; ++j)
      for (int i = 1; i <= mx + 1; ++i) E(DEZ_DX, i, j) = (E(EZ, i, j) - E(EZ, i - 1, j)) * idx;
    for (int j = 1; j <= my + 1; ++j)
      for (int i = 0; i <= mx + 1; ++i) E(DEZ_DY, i, j) = (E(EZ, i, j) - E(EZ, i, j - 1)) * idy;
    for (int j = 0; j <= my + 1; ++j) E(DEY_DX, mx + 1, j) = E(DEY_DX, 1, j);
  }

  void curl_b() {  // F:733-739
    for (int j = 1; j <= my; ++j)
      for (int i = 0; i <= mx + 1; ++i) E(DBX_DY, i, j) = (E(BX, i, j + 1) - E(BX, i, j)) * idy;
    for (int j = 0; j <= my + 1; ++j)
      for (int i = 0; i <= mx; ++i) E(DBY_DX, i, j) = (E(BY, i + 1, j) - E(BY, i, j)) * idx;
    for (int j = 0; j <= my + 1; ++j)
      for (int i = 1; i <= mx + 1; ++i) E(DBZ_DX, i, j) = (E(BZ, i, j) - E(BZ, i - 1, j)) * idx;
    for (int j = 1; j <= my + 1; ++j)
      for (int i = 0; i <= mx + 1; ++i) E(DBZ_DY, i, j) = (E(BZ, i, j) - E(BZ, i, j - 1)) * idy;
    for (int j = 0; j <= my + 1; ++j) E(DBY_DX, mx + 1, j) = E(DBY_DX, 1, j);
  }

  void e_full() {  // F:742-744; denjr(0:mx+1,0:my+1) pairs with emf (Q5)
    T c = dt * cva2;
    for (int j = 0; j <= my + 1; ++j)
      for (int i = 0; i <= mx + 1; ++i) {
        E(EX, i, j) = E(EX, i, j) + c * (E(DBZ_DY, i, j) - D(JX, i, j));
        E(EY, i, j) = E(EY, i, j) - c * (E(DBZ_DX, i, j) + D(JY, i, j));
        E(EZ, i, j) = E(EZ, i, j) + c * (E(DBY_DX, i, j) - E(DBX_DY, i, j) - D(JZ, i, j));
      }
    if (ybc == 1)  // perfect conductor: tangential Ex vanishes on the wall node rows
      for (int i = 0; i <= mx + 1; ++i) E(EX, i, 1) = E(EX, i, my + 1) = 0;
  }

  void node_average() {  // F:838-845
    for (int j = 0; j <= my + 1; ++j)
      for (int i = 1; i <= mx + 1; ++i) {
        G(GEX, i, j) = (E(EX, i, j) + E(EX, i - 1, j)) * (T)0.5;
        G(GBX, i, j) = (E(BX, i, j) + E(BX, i - 1, j)) * (T)0.5;
      }
    for (int j = 1; j <= my + 1; ++j)
      for (int i = 0; i <= mx + 1; ++i) {
        G(GEY, i, j) = (E(EY, i, j) + E(EY, i, j - 1)) * (T)0.5;
        G(GBY, i, j) = (E(BY, i, j) + E(BY, i, j - 1)) * (T)0.5;
      }
    for (int j = 1; j <= my + 1; ++j)
      for (int i = 1; i <= mx + 1; ++i) {
        G(GEZ, i, j) = (E(EZ, i, j) + E(EZ, i - 1, j) + E(EZ, i, j - 1) + E(EZ, i - 1, j - 1)) * (T)0.25;
        G(GBZ, i, j) = (E(BZ, i, j) + E(BZ, i - 1, j) + E(BZ, i, j - 1) + E(BZ, i - 1, j - 1)) * (T)0.25;
      }
  }

  // fieldsenergy F:653-673 (double sums; walls: trapezoid weights on the wall rows)
  void fieldsenergy() {
    double se = 0, sb = 0;
    int jmax = ybc == 0 ? my : my + 1;
    for (int j = 1; j <= jmax; ++j) {
      double w = (ybc == 1 && (j == 1 || j == my + 1)) ? 0.5 : 1.0;
      for (int i = 1; i <= mx; ++i) {
        T e = G(GEX, i, j) * G(GEX, i, j) + G(GEY, i, j) * G(GEY, i, j) + G(GEZ, i, j) * G(GEZ, i, j);
        T b = G(GBX, i, j) * G(GBX, i, j) + G(GBY, i, j) * G(GBY, i, j) + G(GBZ, i, j) * G(GBZ, i, j);
        se += w * (double)e;
        sb += w * (double)b;
      }
    }
    double c2 = (double)cva2, mi = (double)mime, n0 = (double)in0;
    fe[0] = 0.5 * se * mi / (c2 * c2 * n0);
    fe[1] = 0.5 * sb * mi / (c2 * n0);
  }

  // Optional field filters: Marder divergence cleaning (divergenceclean,
  // F:867-886) and the Cherenkov filter (suppresscerenkov, F:889-907). The
  // reference defines both and comments out their call, right after the E
  // update (F:754-755); both read terms it stored at the end of the previous
  // field solve, i.e. they act with E before this step's update (dive, the
  // curls of E) and with rho from this step's push. Restated for periodic y
  // (the reference's only boundary), in 0-based interior coordinates with
  // both axes wrapped, without the reference's index slips (Q4 in dive, the
  // stored rows the reference never sets).
  int filters = 0;  // bit 0 Marder, bit 1 Cherenkov
  double marder_d = 0.001, cer_tau = 0.125;
  std::vector<T> fc;  // corrections: Marder ex, ey; Cherenkov ex, ey, ez (5 x mx x my)

  int wxi(int i) const { return i < 0 ? i + mx : (i >= mx ? i - mx : i); }
  int wyi(int j) const { return j < 0 ? j + my : (j >= my ? j - my : j); }
  T e0(int c, int i, int j) { return E(c, wxi(i) + 1, wyi(j) + 1); }
  T rho0(int i, int j) { return D(RHO, wxi(i) + 1, wyi(j) + 1); }
  T marder_f(int i, int j) {  // dive - cva2 * rho at node (i, j)
    const T dive = (e0(EX, i, j) - e0(EX, i - 1, j)) * idx + (e0(EY, i, j) - e0(EY, i, j - 1)) * idy;
    return dive - cva2 * rho0(i, j);
  }
  T dexdy(int i, int j) { return (e0(EX, i, j + 1) - e0(EX, i, j)) * idy; }
  T deydx(int i, int j) { return (e0(EY, i + 1, j) - e0(EY, i, j)) * idx; }
  T dezdx(int i, int j) { return (e0(EZ, i, j) - e0(EZ, i - 1, j)) * idx; }
  T dezdy(int i, int j) { return (e0(EZ, i, j) - e0(EZ, i, j - 1)) * idy; }

  void filter_prepare() {
    const size_t pl = (size_t)mx * my;
    fc.assign(5 * pl, (T)0);
    const T mdx = dt * (T)marder_d / dx, mdy = dt * (T)marder_d / dy;  // F:873-875
    const T tau = (T)cer_tau * dt;                                     // F:895
    const T cdx = dt * cva2 * tau / dx, cdy = dt * cva2 * tau / dy;    // F:896-897
    for (int i = 0; i < mx; ++i)
      for (int j = 0; j < my; ++j) {
        const size_t k = (size_t)i * my + j;
        if (filters & 1) {
          const T f = marder_f(i, j);
          fc[k] = mdx * (marder_f(i + 1, j) - f);       // F:878-881
          fc[pl + k] = mdy * (marder_f(i, j + 1) - f);  // F:882-883
        }
        if (filters & 2) {
          fc[2 * pl + k] = cdy * (deydx(i, j) - deydx(i, j - 1) - dexdy(i, j) + dexdy(i, j - 1));   // F:898-900
          fc[3 * pl + k] = cdx * (-deydx(i, j) + deydx(i - 1, j) + dexdy(i, j) - dexdy(i - 1, j));  // F:901-903
          fc[4 * pl + k] = cdx * (dezdx(i + 1, j) - dezdx(i, j)) + cdy * (dezdy(i, j + 1) - dezdy(i, j));  // F:904-906
        }
      }
  }

  void filter_apply() {  // Marder first, then the Cherenkov filter, as the commented calls
    const size_t pl = (size_t)mx * my;
    for (int i = 0; i < mx; ++i)
      for (int j = 0; j < my; ++j) {
        const size_t k = (size_t)i * my + j;
        T& ex = E(EX, i + 1, j + 1);
        T& ey = E(EY, i + 1, j + 1);
        T& ez = E(EZ, i + 1, j + 1);
        if (filters & 1) {
          ex = ex + fc[k];
          ey = ey + fc[pl + k];
        }
        if (filters & 2) {
          ex = ex - fc[2 * pl + k];
          ey = ey - fc[3 * pl + k];
          ez = ez + fc[4 * pl + k];
        }
      }
    // keep the periodic guards equal to the corrected interior: the x guard
    // columns (the reference's periodic copy right after sets column 1 from
    // column mx+1) and the ex ghost rows, which the 1-rank exchange never sets
    for (int c : {EX, EY, EZ})
      for (int j = 1; j <= my; ++j) {
        E(c, 0, j) = E(c, mx, j);
        E(c, mx + 1, j) = E(c, 1, j);
      }
    for (int i = 0; i <= mx + 1; ++i) {
      E(EX, i, 0) = E(EX, i, my);
      E(EX, i, my + 1) = E(EX, i, 1);
    }
  }

  // fieldsolver F:678-860
  void fieldsolver() {
    if (filters) filter_prepare();
    b_half();
    periodic_x(BX);
    periodic_x(BY);
    periodic_x(BZ);
    ghost_y(BY, -1, BZ, 1);
    curl_b();
    e_full();
    if (filters) filter_apply();  // the commented calls of F:754-755
    periodic_x(EX);
    periodic_x(EY);
    periodic_x(EZ);
    ghost_y(EY, 1, EZ, -1);
    curl_e();
    b_half();
    ghost_y(BY, -1, BZ, 1);
    node_average();
    fieldsenergy();
  }

  // Derived state after loading primary fields: guards, curl terms, node averages.
  void refresh_derived() {
    // guard columns from the loaded interior (column 0 = mx, column mx+1 = 1)
    for (int c : {EX, EY, EZ, BX, BY, BZ})
      for (int j = 0; j <= my + 1; ++j) {
        E(c, 0, j) = E(c, mx, j);
        E(c, mx + 1, j) = E(c, 1, j);
      }
    if (ybc == 0) {
      ghost_y(EY, 1, EZ, -1);
      ghost_y(BY, -1, BZ, 1);
      for (int i = 0; i <= mx + 1; ++i) {  // bx, ex rows are never exchanged; the loader sets them
        E(EX, i, my + 1) = E(EX, i, 1);
        E(EX, i, 0) = E(EX, i, my);
        E(BX, i, my + 1) = E(BX, i, 1);
        E(BX, i, 0) = E(BX, i, my);
      }
    } else {
      ghost_y(EY, 1, EZ, -1);
      ghost_y(BY, -1, BZ, 1);
    }
    curl_e();
    node_average();
    fieldsenergy();
  }

  // countingsort F:1303-1329
  void countingsort() {
    std::fill(ptlalloc.begin(), ptlalloc.end(), 0);
    for (int64_t i = 0; i < nptlact; ++i) ptlalloc[ptl[i].grid - 1] += 1;
    counts = ptlalloc;
    int64_t k = 0;
    for (size_t i = 0; i < ptlalloc.size(); ++i) {
      int32_t j = ptlalloc[i];
      ptlalloc[i] = (int32_t)k;
      k += j;
    }
    if (ptlsort.size() < ptl.size()) ptlsort.resize(ptl.size());
    for (int64_t i = 0; i < nptlact; ++i) {
      int32_t j = ptl[i].grid - 1;
      int32_t kk = ptlalloc[j] + 1;
      ptlalloc[j] = kk;
      ptlsort[kk - 1] = ptl[i];
    }
    std::copy(ptlsort.begin(), ptlsort.begin() + nptlact, ptl.begin());
  }

  // ---------------------------------------------------- OpenMP CPU baseline
  // Same arithmetic as pusher(), parallel over particle chunks with private
  // current arrays; particles keep their slot (y wrap / reflection in place).
  std::vector<std::vector<T>> jpriv;
  void omp_pusher(int nthreads) {
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#else
    nthreads = 1;
#endif
    if ((int)jpriv.size() != nthreads) jpriv.assign(nthreads, std::vector<T>(denjr.size()));
    std::vector<double> kep(2 * nthreads, 0.0);
#pragma omp parallel num_threads(nthreads)
    {
#ifdef _OPENMP
      int t = omp_get_thread_num();
#else
      int t = 0;
#endif
      std::vector<T>& jb = jpriv[t];
      std::fill(jb.begin(), jb.end(), (T)0);
      int64_t lo = nptlact * t / nthreads, hi = nptlact * (t + 1) / nthreads;
      for (int64_t i = lo; i < hi; ++i) {
        Ptl<T>& p = ptl[i];
        Moved m = push_one(p, &jb);
        int iy = m.iy1;
        if (ybc == 0) {
          if (iy > my) iy -= my;
          else if (iy < 1) iy += my;
        } else if (iy > my || iy < 1) {
          iy = iy > my ? my : 1;
          p.dy = -p.dy;
          p.uy = -p.uy;
        }
        p.grid = my * (m.ix - 1) + iy;
        add_ke(p, m.gama, m.ms, &kep[2 * t]);
      }
    }
    size_t nj = denjr.size();
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (int64_t k = 0; k < (int64_t)nj; ++k) {
      T s = 0;
      for (int t = 0; t < nthreads; ++t) s += jpriv[t][k];
      denjr[k] = s;
    }
    ke[0] = ke[1] = 0;
    for (int t = 0; t < nthreads; ++t) {
      ke[0] += kep[2 * t];
      ke[1] += kep[2 * t + 1];
    }
    normalise_and_fold_x();
    fold_y();
  }

  // Stable counting sort, parallel: per-thread histograms over contiguous
  // chunks give each (thread, cell) its stable starting slot.
  void omp_countingsort(int nthreads) {
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#else
    nthreads = 1;
#endif
    size_t nc = (size_t)mx * my;
    std::vector<int64_t> h((size_t)nthreads * nc, 0);
#pragma omp parallel num_threads(nthreads)
    {
#ifdef _OPENMP
      int t = omp_get_thread_num();
#else
      int t = 0;
#endif
      int64_t lo = nptlact * t / nthreads, hi = nptlact * (t + 1) / nthreads;
      int64_t* ht = &h[(size_t)t * nc];
      for (int64_t i = lo; i < hi; ++i) ht[ptl[i].grid - 1] += 1;
    }
    int64_t run = 0;
    for (size_t c = 0; c < nc; ++c) {
      int64_t tot = 0;
      for (int t = 0; t < nthreads; ++t) {
        int64_t v = h[(size_t)t * nc + c];
        h[(size_t)t * nc + c] = run + tot;
        tot += v;
      }
      counts[c] = (int32_t)tot;
      run += tot;
    }
    if (ptlsort.size() < ptl.size()) ptlsort.resize(ptl.size());
#pragma omp parallel num_threads(nthreads)
    {
#ifdef _OPENMP
      int t = omp_get_thread_num();
#else
      int t = 0;
#endif
      int64_t lo = nptlact * t / nthreads, hi = nptlact * (t + 1) / nthreads;
      int64_t* ht = &h[(size_t)t * nc];
      for (int64_t i = lo; i < hi; ++i) ptlsort[ht[ptl[i].grid - 1]++] = ptl[i];
    }
    std::swap(ptl, ptlsort);
  }
};

struct Handle {
  int precision;  // 0 double, 1 float
  Sim<double> d;
  Sim<float> f;
};

template <class T>
void load_particles(Sim<T>& s, const OrcParticle* in, int64_t n, int64_t capacity) {
  s.ptl.assign(std::max<int64_t>(capacity, n), Ptl<T>{0, 0, 0, 0, 0, s.mx * s.my + 1, 0, 0});
  s.nptltot = (int64_t)s.ptl.size();
  for (int64_t i = 0; i < n; ++i) {
    Ptl<T>& p = s.ptl[i];
    p.dx = (T)in[i].dx;
    p.dy = (T)in[i].dy;
    p.ux = (T)in[i].ux;
    p.uy = (T)in[i].uy;
    p.uz = (T)in[i].uz;
    p.grid = in[i].grid;
    p.q = in[i].q;
    p.pid = in[i].pid;
  }
  s.nptlact = n;
}

template <class T>
int64_t get_particles(Sim<T>& s, OrcParticle* out, int64_t cap) {
  int64_t n = std::min<int64_t>(cap, s.nptlact);
  for (int64_t i = 0; i < n; ++i) {
    const Ptl<T>& p = s.ptl[i];
    out[i] = OrcParticle{(double)p.dx, (double)p.dy, (double)p.ux, (double)p.uy, (double)p.uz,
                         p.grid, p.q, p.pid, 0};
  }
  return s.nptlact;
}

// Canonical 0-based exchange layout shared with the tests: component arrays of
// shape (mx, my+1), x-major with y fastest; (i, j) here is reference (i+1, j+1).
template <class T>
void set_yee(Sim<T>& s, const double* f6) {
  size_t ny1 = (size_t)s.my + 1;
  const int comps[6] = {EX, EY, EZ, BX, BY, BZ};
  for (int c = 0; c < 6; ++c)
    for (int i = 0; i < s.mx; ++i)
      for (int j = 0; j <= s.my; ++j) {
        T v = (T)f6[((size_t)c * s.mx + i) * ny1 + j];
        bool node_row = comps[c] == EX || comps[c] == BX;
        if (j == s.my && !(node_row && s.ybc == 1)) continue;
        s.E(comps[c], i + 1, j + 1) = v;
      }
  s.refresh_derived();
}

template <class T>
void get_yee(Sim<T>& s, double* f6) {
  size_t ny1 = (size_t)s.my + 1;
  const int comps[6] = {EX, EY, EZ, BX, BY, BZ};
  for (int c = 0; c < 6; ++c)
    for (int i = 0; i < s.mx; ++i)
      for (int j = 0; j <= s.my; ++j) f6[((size_t)c * s.mx + i) * ny1 + j] = (double)s.E(comps[c], i + 1, j + 1);
}

// J after normalisation and folding, (4, mx, my+1) with the canonical layout.
template <class T>
void get_j(Sim<T>& s, double* j4) {
  size_t ny1 = (size_t)s.my + 1;
  for (int c = 0; c < 4; ++c)
    for (int i = 0; i < s.mx; ++i)
      for (int j = 0; j <= s.my; ++j) j4[((size_t)c * s.mx + i) * ny1 + j] = (double)s.D(c, i + 1, j + 1);
}

// emfgrid nodes 1..mx+1 x 1..my+1 as (mx+1, my+1, 8)
template <class T>
void get_grid(Sim<T>& s, double* g) {
  for (int i = 0; i <= s.mx; ++i)
    for (int j = 0; j <= s.my; ++j)
      for (int c = 0; c < 8; ++c) g[(((size_t)i * (s.my + 1)) + j) * 8 + c] = (double)s.G(c, i + 1, j + 1);
}

}  // namespace

extern "C" {

void* orc_create(const OrcParams* p, int precision) {
  Handle* h = new Handle();
  h->precision = precision;
  if (precision == 0) h->d.init(*p);
  else h->f.init(*p);
  return h;
}
void orc_destroy(void* h) { delete (Handle*)h; }

void orc_load_particles(void* h, const OrcParticle* in, int64_t n, int64_t capacity) {
  Handle* H = (Handle*)h;
  if (H->precision == 0) load_particles(H->d, in, n, capacity);
  else load_particles(H->f, in, n, capacity);
}
int64_t orc_get_particles(void* h, OrcParticle* out, int64_t cap) {
  Handle* H = (Handle*)h;
  return H->precision == 0 ? get_particles(H->d, out, cap) : get_particles(H->f, out, cap);
}
int64_t orc_nptl(void* h) {
  Handle* H = (Handle*)h;
  return H->precision == 0 ? H->d.nptlact : H->f.nptlact;
}
void orc_set_yee(void* h, const double* f6) {
  Handle* H = (Handle*)h;
  if (H->precision == 0) set_yee(H->d, f6);
  else set_yee(H->f, f6);
}
void orc_get_yee(void* h, double* f6) {
  Handle* H = (Handle*)h;
  if (H->precision == 0) get_yee(H->d, f6);
  else get_yee(H->f, f6);
}
void orc_get_j(void* h, double* j4) {
  Handle* H = (Handle*)h;
  if (H->precision == 0) get_j(H->d, j4);
  else get_j(H->f, j4);
}
void orc_get_grid(void* h, double* g) {
  Handle* H = (Handle*)h;
  if (H->precision == 0) get_grid(H->d, g);
  else get_grid(H->f, g);
}
void orc_pusher(void* h) {
  Handle* H = (Handle*)h;
  if (H->precision == 0) H->d.pusher();
  else H->f.pusher();
}
void orc_fieldsolver(void* h) {
  Handle* H = (Handle*)h;
  if (H->precision == 0) H->d.fieldsolver();
  else H->f.fieldsolver();
}
void orc_set_filters(void* h, int flags, double marder_d, double cer_tau) {
  Handle* H = (Handle*)h;
  if (H->precision == 0) {
    H->d.filters = flags;
    H->d.marder_d = marder_d;
    H->d.cer_tau = cer_tau;
  } else {
    H->f.filters = flags;
    H->f.marder_d = marder_d;
    H->f.cer_tau = cer_tau;
  }
}
void orc_countingsort(void* h, int32_t* counts_out) {
  Handle* H = (Handle*)h;
  if (H->precision == 0) {
    H->d.countingsort();
    if (counts_out) memcpy(counts_out, H->d.counts.data(), H->d.counts.size() * 4);
  } else {
    H->f.countingsort();
    if (counts_out) memcpy(counts_out, H->f.counts.data(), H->f.counts.size() * 4);
  }
}
void orc_omp_pusher(void* h, int nthreads) {
  Handle* H = (Handle*)h;
  if (H->precision == 0) H->d.omp_pusher(nthreads);
  else H->f.omp_pusher(nthreads);
}
void orc_omp_countingsort(void* h, int nthreads) {
  Handle* H = (Handle*)h;
  if (H->precision == 0) H->d.omp_countingsort(nthreads);
  else H->f.omp_countingsort(nthreads);
}
// out[0..3] = (electron KE, ion KE, E energy, B energy) of the last push / field solve
void orc_energies(void* h, double* out) {
  Handle* H = (Handle*)h;
  double* ke = H->precision == 0 ? H->d.ke : H->f.ke;
  double* fe = H->precision == 0 ? H->d.fe : H->f.fe;
  out[0] = ke[0];
  out[1] = ke[1];
  out[2] = fe[0];
  out[3] = fe[1];
}
int orc_omp_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// ------------------------------------------------------------------ loaders
// CPU loader with the same generator and arithmetic as the device loader.
void orc_load_pairs(const pic::LoadParams* L, int64_t k0, int64_t k1, OrcParticle* out) {
#pragma omp parallel for schedule(static)
  for (int64_t k = k0; k < k1; ++k) {
    pic::LoadedParticle pr[2];
    pic::load_pair(*L, k, pr);
    for (int s = 0; s < 2; ++s) {
      OrcParticle& o = out[2 * (k - k0) + s];
      o.dx = pr[s].ox;
      o.dy = pr[s].oy;
      o.ux = pr[s].ux;
      o.uy = pr[s].uy;
      o.uz = pr[s].uz;
      o.grid = L->my * pr[s].ix + pr[s].iy + 1;
      o.q = s == 0 ? 1 : -1;
      o.pid = (int32_t)(2 * k + s + 1);
      o.pad = 0;
    }
  }
}

void orc_philox(uint64_t c0, uint64_t c1, uint64_t c2, uint64_t c3, uint64_t k0, uint64_t k1,
                uint64_t* out4) {
  pic::u64x4 r = pic::philox4x64(c0, c1, c2, c3, k0, k1);
  for (int i = 0; i < 4; ++i) out4[i] = r.v[i];
}
double orc_log(double x) { return pic::pic_log(x); }

// Initial fields in the canonical (6, mx, my+1) layout.
void orc_init_fields(const pic::FieldInit* f, double* f6) {
  size_t ny1 = (size_t)f->my + 1;
  size_t plane = (size_t)f->mx * ny1;
  memset(f6, 0, 6 * plane * sizeof(double));
  for (int i = 0; i < f->mx; ++i)
    for (int j = 0; j <= f->my; ++j) {
      f6[3 * plane + i * ny1 + j] = pic::init_bx(*f, i, j);
      f6[4 * plane + i * ny1 + j] = pic::init_by(*f, i, j);
      f6[5 * plane + i * ny1 + j] = pic::init_bz(*f, i, j);
    }
}

}  // extern "C"
