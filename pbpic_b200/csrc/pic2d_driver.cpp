// pic2d_driver: the reference's main program (program pic2d,
// src/programs/pic2d.f90:148-192) restated in C++ on the C ABI of the B200
// step. The module globals of `module parameters` (pic2d.f90:4-142) become a
// handle; the subroutines keep their names and call order:
//
//   init                     -> pbpic_create + pbpic_init_plasma  (pic2d.f90:160, 197-308)
//   countingsort             -> pbpic_sort                        (pic2d.f90:161, 1303-1329)
//   do itime = 1, ntime
//     pusher                 -> pbpic_push                        (pic2d.f90:177, 912-1217)
//     fieldsolver            -> pbpic_fieldsolve                  (pic2d.f90:178, 678-860)
//     every 50 steps: countingsort                                (pic2d.f90:180-182)
//     every ntdiag steps: energyinfo -> pbpic_energies            (pic2d.f90:183-187)
//   releasememory            -> pbpic_destroy                     (pic2d.f90:189, 2557-2582)
//
// Usage: pic2d_driver [--double-harris|--harris|--uniform] [--mx N] [--my N] [--ppc N]
//                     [--ntime N] [--sort-every N] [--ntdiag N] [--fp32|--fp64] [--seed N]
// The default is the reference's own run: its double Harris sheet on 256x256
// cells of 0.04 d_i, 64 pairs per cell, 30 steps (pic2d.f90:12-43, 357-648).
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "pbpic.h"

namespace {

enum Plasma { DOUBLE_HARRIS, HARRIS, UNIFORM };

struct Parameters {  // the run parameters of module parameters (pic2d.f90:12-43, 127-136)
  int mx = 256, my = 256, ppc = 64, ntime = 30, sort_every = 50, ntdiag = 10;
  int plasma = DOUBLE_HARRIS, precision = PBPIC_FP32_MIXED;
  double mime = 25.0, wpe_wce = 2.0;
  unsigned long long seed = 1;
};

pbpic_handle* h = nullptr;
Parameters prm;

void check(int rc, const char* what) {
  if (rc != PBPIC_OK) {
    fprintf(stderr, "%s failed (%d): %s\n", what, rc, pbpic_last_error());
    exit(1);
  }
}

// init (pic2d.f90:197-308): domain, fields and particles.
void init() {
  const double cva = prm.wpe_wce * sqrt(prm.mime);
  const double dx = 0.1, dy = 0.1;
  const double dt = 0.5 / (cva * sqrt(1.0 / (dx * dx) + 1.0 / (dy * dy)));  // CFL 0.5
  pbpic_loader ld;
  memset(&ld, 0, sizeof(ld));
  ld.ppc = prm.ppc;
  ld.seed = prm.seed;
  pbpic_config cfg;
  memset(&cfg, 0, sizeof(cfg));
  cfg.mx = prm.mx;
  cfg.my = prm.my;
  cfg.dx = dx;
  cfg.dy = dy;
  cfg.dt = dt;
  cfg.cva = cva;
  cfg.mime = prm.mime;
  cfg.precision = prm.precision;
  if (prm.plasma == DOUBLE_HARRIS) {
    // the reference's parameters (pic2d.f90:15-31, 42): dx = 0.04 d_i, c/v_A = 15,
    // dt = 0.045 / mime, sheet electrons at 0.092 c with Ti/Te = 5, the background
    // 10 times colder with Ti/Te = 1 and nb = 0.2, sheets of half-width 0.5 d_i
    // drifting at v_A
    const double ddx = 0.04, c_va = 15.0, vthec = 0.092, lam = 0.5, nb = 0.2;
    cfg.dx = cfg.dy = ddx;
    cfg.cva = c_va;
    cfg.dt = 0.045 / prm.mime;
    ld.kind = PBPIC_LOAD_DOUBLE_HARRIS;
    ld.vthe = vthec;
    ld.vthi = vthec * sqrt(5.0 / prm.mime);
    ld.vthe_bg = vthec * sqrt(0.1);
    ld.vthi_bg = ld.vthe_bg * sqrt(1.0 / prm.mime);
    ld.vdrift_i = 1.0 / c_va;
    ld.vdrift_e = -1.0 / c_va;
    ld.lambda = lam;
    ld.nb = nb;
    cfg.ybc = PBPIC_BC_PERIODIC;
    const double lx = prm.mx * ddx;
    cfg.in0 = (4.0 * lam + nb * lx) / (prm.ppc * lx);  // 1 / (n0 dx dy), n0 the sheet peak density
  } else if (prm.plasma == HARRIS) {
    // Harris sheet in pressure balance, Ti/Te = 5, lambda = 0.5 d_i, nb = 0.2 n0
    const double tite = 5.0, lam = 0.5, nb = 0.2;
    const double te = 1.0 / (2.0 * (1.0 + tite));
    ld.kind = PBPIC_LOAD_HARRIS;
    ld.vthe = sqrt(prm.mime * te) / cva;
    ld.vthi = ld.vthe * sqrt(tite / prm.mime);
    const double du = -1.0 / (lam * cva);
    ld.vdrift_i = du * tite / (1.0 + tite);
    ld.vdrift_e = -du / (1.0 + tite);
    ld.lambda = lam;
    ld.nb = nb;
    ld.psi0 = 0.1;
    cfg.ybc = PBPIC_BC_CONDUCTING;
    const double lx = prm.mx * dx, ly = prm.my * dy;
    cfg.in0 = lx * (2.0 * lam + nb * ly) / (dx * dy) / ((double)prm.ppc * prm.mx * prm.my);
  } else {
    ld.kind = PBPIC_LOAD_UNIFORM;
    ld.vthe = 0.1;
    ld.vthi = 0.1 / sqrt(prm.mime);
    ld.b0z = 1.0;
    cfg.ybc = PBPIC_BC_PERIODIC;
    cfg.in0 = 1.0 / prm.ppc;
  }
  cfg.capacity = 2ll * prm.ppc * prm.mx * prm.my;
  check(pbpic_create(&cfg, &h), "pbpic_create");
  check(pbpic_init_plasma(h, &ld), "pbpic_init_plasma");
}

void pusher() { check(pbpic_push(h), "pusher"); }
void fieldsolver() { check(pbpic_fieldsolve(h), "fieldsolver"); }
void countingsort() { check(pbpic_sort(h), "countingsort"); }

// energyinfo (pic2d.f90:1957-2115) without the HDF5 writer: print totene(:, itime).
void energyinfo(int itime) {
  double e[4];
  check(pbpic_energies(h, e), "energyinfo");
  printf("%6d  %.10e %.10e %.10e %.10e\n", itime, e[0], e[1], e[2], e[3]);
}

void releasememory() { check(pbpic_destroy(h), "releasememory"); }

void parse(int argc, char** argv) {
  for (int i = 1; i < argc; ++i) {
    auto next = [&](void) -> const char* {
      if (i + 1 >= argc) {
        fprintf(stderr, "missing value after %s\n", argv[i]);
        exit(2);
      }
      return argv[++i];
    };
    if (!strcmp(argv[i], "--double-harris")) prm.plasma = DOUBLE_HARRIS;
    else if (!strcmp(argv[i], "--harris")) prm.plasma = HARRIS;
    else if (!strcmp(argv[i], "--uniform")) prm.plasma = UNIFORM;
    else if (!strcmp(argv[i], "--mx")) prm.mx = atoi(next());
    else if (!strcmp(argv[i], "--my")) prm.my = atoi(next());
    else if (!strcmp(argv[i], "--ppc")) prm.ppc = atoi(next());
    else if (!strcmp(argv[i], "--ntime")) prm.ntime = atoi(next());
    else if (!strcmp(argv[i], "--sort-every")) prm.sort_every = atoi(next());
    else if (!strcmp(argv[i], "--ntdiag")) prm.ntdiag = atoi(next());
    else if (!strcmp(argv[i], "--fp32")) prm.precision = PBPIC_FP32_MIXED;
    else if (!strcmp(argv[i], "--fp64")) prm.precision = PBPIC_FP64_PLAIN;
    else if (!strcmp(argv[i], "--seed")) prm.seed = strtoull(next(), nullptr, 10);
    else {
      fprintf(stderr, "unknown option %s\n", argv[i]);
      exit(2);
    }
  }
}

}  // namespace

int main(int argc, char** argv) {
  parse(argc, argv);
  init();                       // pic2d.f90:160
  countingsort();               // pic2d.f90:161
  energyinfo(0);                // pic2d.f90:168
  for (int itime = 1; itime <= prm.ntime; ++itime) {  // pic2d.f90:171-188
    pusher();
    fieldsolver();
    if (prm.sort_every > 0 && itime % prm.sort_every == 0) countingsort();
    if (prm.ntdiag > 0 && itime % prm.ntdiag == 0) energyinfo(itime);
  }
  int32_t st = 0;
  check(pbpic_status(h, &st), "pbpic_status");
  if (st & (PBPIC_STATUS_CELL_JUMP | PBPIC_STATUS_NAN)) fprintf(stderr, "device status bits: %d\n", st);
  releasememory();              // pic2d.f90:189
  return st & (PBPIC_STATUS_CELL_JUMP | PBPIC_STATUS_NAN) ? 1 : 0;
}
