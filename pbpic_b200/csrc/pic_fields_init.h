// Initial electromagnetic fields for the plasma loaders (host code only).
// Shared by the library and by the CPU oracle so that both start from the
// same fields. Positions are 0-based Yee locations:
//   bx(i,j) at (i+1/2, j), by(i,j) at (i, j+1/2), bz(i,j) at (i+1/2, j+1/2)
// in units of cells, with node (i,j) at x = i*dx, y = j*dy.
#pragma once
#include <math.h>

namespace pic {

struct FieldInit {
  int kind;          // LoadKind
  int mx, my;
  double dx, dy;
  double lambda;     // Harris half-thickness (d_i)
  double psi0;       // GEM flux perturbation amplitude (B0 d_i)
  double bguide;     // Harris guide field Bz (B0)
  double b0z;        // uniform Bz for the uniform / two-stream / Weibel plasmas (B0)
};

// GEM perturbation flux function psi = psi0 cos(2 pi (x - Lx/2)/Lx) cos(pi (y - Ly/2)/Ly);
// the perturbed field is B = z x grad(psi), i.e. dBx = -dpsi/dy, dBy = dpsi/dx.
inline double gem_psi(const FieldInit& f, double x, double y) {
  const double PI = 3.14159265358979323846;
  double Lx = f.mx * f.dx, Ly = f.my * f.dy;
  return f.psi0 * cos(2.0 * PI * (x - 0.5 * Lx) / Lx) * cos(PI * (y - 0.5 * Ly) / Ly);
}

// Bx at (i+1/2, j): Harris tanh profile plus the perturbation differenced from psi
// at the neighbouring cell centres, so that the discrete div B vanishes exactly.
inline double init_bx(const FieldInit& f, int i, int j) {
  if (f.kind != 1) return 0.0;
  double Ly = f.my * f.dy;
  double y = j * f.dy;
  double xc = (i + 0.5) * f.dx;
  double b = tanh((y - 0.5 * Ly) / f.lambda);
  double dpsi = gem_psi(f, xc, (j + 0.5) * f.dy) - gem_psi(f, xc, (j - 0.5) * f.dy);
  return b - dpsi / f.dy;
}

// By at (i, j+1/2). Double Harris (kind 4): the two sheets' profile at the node
// column x = i dx (initfields, pic2d.f90:606-610).
inline double init_by(const FieldInit& f, int i, int j) {
  if (f.kind == 4) {
    const double Lx = f.mx * f.dx, x = i * f.dx;
    return tanh((x - 0.25 * Lx) / f.lambda) - tanh((x - 0.75 * Lx) / f.lambda) - 1.0;
  }
  if (f.kind != 1) return 0.0;
  double yc = (j + 0.5) * f.dy;
  double dpsi = gem_psi(f, (i + 0.5) * f.dx, yc) - gem_psi(f, (i - 0.5) * f.dx, yc);
  return dpsi / f.dx;
}

// Bz at (i+1/2, j+1/2).
inline double init_bz(const FieldInit& f, int /*i*/, int /*j*/) {
  if (f.kind == 1 || f.kind == 4) return f.bguide;
  return f.b0z;
}

}  // namespace pic
