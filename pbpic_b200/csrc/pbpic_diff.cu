// Differentiable form of the step (include/pbpic.h, pbpic_diff_*): a
// checkpointed forward run of the GEM Harris sheet and the discrete adjoint of
// every step (kernels_adjoint.cuh), giving d loss / d (psi0, nb, Ti/Te).
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "../../include/pbpic.h"
#include "api_internal.h"
#include "kernels_adjoint.cuh"
#include "kernels_field.cuh"
#include "kernels_misc.cuh"
#include "pic_common.h"
#include "pic_fields_init.h"

using namespace pbd;

namespace {

#define DCK(call)                                                                                       \
  do {                                                                                                  \
    cudaError_t e_ = (call);                                                                            \
    if (e_ != cudaSuccess)                                                                              \
      return pbpic_internal_fail(PBPIC_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_));      \
  } while (0)
#define DLAUNCH(what)                                                                                   \
  do {                                                                                                  \
    pbpic_internal_count_launch();                                                                      \
    cudaError_t e_ = cudaGetLastError();                                                                \
    if (e_ != cudaSuccess)                                                                              \
      return pbpic_internal_fail(PBPIC_ECUDA, std::string(what) + ": " + cudaGetErrorString(e_));       \
  } while (0)
#define DTRY(...)                  \
  do {                             \
    int r_ = (__VA_ARGS__);        \
    if (r_ != PBPIC_OK) return r_; \
  } while (0)

int grid_of(int64_t n, int maxblocks = 148 * 8) {
  int64_t g = (n + 255) / 256;
  return (int)std::max<int64_t>(1, std::min<int64_t>(g, maxblocks));
}

// One stored state: particles and Yee fields.
struct Slot {
  void* p = nullptr;  // cell (4 B) then 5 component arrays of T
  void* f = nullptr;  // 6 planes of T
};

}  // namespace

struct pbpic_diff {
  pbpic_diff_config cfg;
  bool f32 = false;
  size_t tsz = 8;
  int mx = 0, my = 0, S = 0;
  int64_t n = 0, npairs = 0, nsheet = 0;
  double dx = 0, dy = 0, dt = 0, cva = 0, in0 = 0;
  int nseg = 0;
  std::vector<Slot> ck;   // checkpoints: state at steps 0, K, 2K, ...
  std::vector<Slot> seg;  // recomputed states of one segment (K + 1)
  Slot work;              // running state
  void* ng = nullptr;     // node grid of T
  void* jacc = nullptr;   // 4 planes of 8-byte accumulators
  double* fe_part = nullptr;
  int nfe = 0;
  void* lam[2][5] = {{nullptr}};
  double* fbar = nullptr;  // 6 adjoint planes (ex ey ez bx by bz)
  double* jbar = nullptr;  // 3 planes
  double* gbar = nullptr;  // node adjoint
  double* scal = nullptr;  // [0] loss, [1] d loss / d omega, [2] d loss / d tau
  void* jseg = nullptr;    // j.E loss: the current of each step of the recomputed segment (3 planes each)
  pbpic_diff_params last{};
  bool have_forward = false;
  std::vector<void*> allocs;
};

namespace {

int dmalloc(pbpic_diff* d, void** p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, std::max<size_t>(bytes, 16));
  if (e != cudaSuccess)
    return pbpic_internal_fail(PBPIC_ENOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  d->allocs.push_back(*p);
  return PBPIC_OK;
}

size_t part_bytes(const pbpic_diff* d) { return (size_t)d->n * (4 + 5 * d->tsz); }
size_t field_bytes(const pbpic_diff* d) { return (size_t)6 * d->mx * d->S * d->tsz; }
int64_t plane(const pbpic_diff* d) { return (int64_t)d->mx * d->S; }

template <class T>
struct View {
  uint32_t* cell;
  T* c[5];
  T* f[6];
};

template <class T>
View<T> view(const pbpic_diff* d, const Slot& s) {
  View<T> v;
  v.cell = (uint32_t*)s.p;
  T* base = (T*)((char*)s.p + (size_t)d->n * 4);
  for (int k = 0; k < 5; ++k) v.c[k] = base + (size_t)k * d->n;
  for (int k = 0; k < 6; ++k) v.f[k] = (T*)s.f + (size_t)k * plane(d);
  return v;
}

struct Harris {
  double vthe, vthi, ude, udi;  // thermal speeds and drifts (units of c)
};

Harris harris_speeds(const pbpic_diff* d, double tite) {
  const pbpic_diff_config& c = d->cfg;
  const double te = 1.0 / (2.0 * (1.0 + tite));
  Harris h;
  h.vthe = sqrt(c.mime * te) / d->cva;
  h.vthi = h.vthe * sqrt(tite / c.mime);
  const double du = -1.0 / (c.lambda * d->cva);
  h.udi = du * tite / (1.0 + tite);
  h.ude = -du / (1.0 + tite);
  return h;
}

double urel(double v) { return v / sqrt(1.0 - v * v); }
double durel(double v) { return 1.0 / pow(1.0 - v * v, 1.5); }

template <class T>
PushParams<T> push_params(const pbpic_diff* d, const Slot& s) {
  View<T> v = view<T>(d, s);
  PushParams<T> p;
  memset(&p, 0, sizeof(p));
  p.mx = d->mx;
  p.my = d->my;
  p.S = d->S;
  p.ybc = PBPIC_BC_CONDUCTING;
  p.compat = 0;
  p.cell = v.cell;
  p.dx = v.c[0];
  p.dy = v.c[1];
  p.ux = v.c[2];
  p.uy = v.c[3];
  p.uz = v.c[4];
  p.ng = (const T*)d->ng;
  p.cg = nullptr;  // the adjoint kernels gather from the node grid
  p.jacc = d->jacc;
  const T dt = (T)d->dt, mime = (T)d->cfg.mime, cva = (T)d->cva, dx = (T)d->dx, dy = (T)d->dy;
  for (int sp = 0; sp < 2; ++sp) {
    const T q = sp == 0 ? T(1) : T(-1);
    const T ms = sp == 0 ? mime : T(1);
    p.c0[sp] = q * dt * mime / ms / T(2);
    p.c1[sp] = p.c0[sp] / cva;
    p.ms[sp] = ms;
    p.q[sp] = q;
    p.qx[sp] = q * dx / dt;
    p.qy[sp] = q * dy / dt;
  }
  p.dtcva = dt * cva;
  p.idx = T(1) / dx;
  p.idy = T(1) / dy;
  p.cva = cva;
  return p;
}

template <class T>
FieldParams<T> field_params(const pbpic_diff* d, const Slot& s) {
  View<T> v = view<T>(d, s);
  FieldParams<T> a;
  a.mx = d->mx;
  a.my = d->my;
  a.S = d->S;
  a.ybc = PBPIC_BC_CONDUCTING;
  a.ex = v.f[0];
  a.ey = v.f[1];
  a.ez = v.f[2];
  a.bx = v.f[3];
  a.by = v.f[4];
  a.bz = v.f[5];
  const T dt = (T)d->dt, cva = (T)d->cva;
  a.dth = dt / T(2);
  a.cdt = dt * (cva * cva);
  a.idx = T(1) / (T)d->dx;
  a.idy = T(1) / (T)d->dy;
  a.jacc = d->jacc;
  for (int k = 0; k < 4; ++k) a.jscale[k] = d->f32 ? d->in0 * FIX_INV : d->in0;
  a.ng = (T*)d->ng;
  a.cg = nullptr;
  a.fe_part = d->fe_part;
  return a;
}

double loss_scale(const pbpic_diff* d) { return d->dt * 0.5 * d->cfg.mime / (d->cva * d->cva * d->in0); }

// j.E loss: dt * mime / (cva^2 in0) * sum J . E, the work done on the particles
// in the units of the field energy (the E update drains cva^2 J per unit time
// from fields whose energy is mime / (2 cva^4 in0) sum E^2).
double jdote_scale(const pbpic_diff* d) { return d->dt * d->cfg.mime / (d->cva * d->cva * d->in0); }
double jdote_jscale(const pbpic_diff* d) { return d->f32 ? d->in0 * FIX_INV : d->in0; }

// The j.E loss of the step whose current is in `jacc` and whose starting
// fields are the slot's; with jbar/fbar_e, its adjoint seeds.
template <class T>
int loss_jdote(pbpic_diff* d, const Slot& s, const void* jacc, double* loss, double* jbar, double* fbar_e) {
  View<T> v = view<T>(d, s);
  const int g = grid_of((int64_t)d->mx * (d->my + 1));
  if (d->f32)
    k_loss_jdote<T, long long><<<g, 256>>>(d->mx, d->my, d->S, PBPIC_BC_CONDUCTING, jacc, jdote_jscale(d), v.f[0],
                                           v.f[1], v.f[2], jdote_scale(d), loss, jbar, fbar_e);
  else
    k_loss_jdote<T, double><<<g, 256>>>(d->mx, d->my, d->S, PBPIC_BC_CONDUCTING, jacc, jdote_jscale(d), v.f[0],
                                        v.f[1], v.f[2], jdote_scale(d), loss, jbar, fbar_e);
  DLAUNCH("k_loss_jdote");
  return PBPIC_OK;
}

// Node grid of a slot's fields into d->ng.
template <class T>
int nodes(pbpic_diff* d, const Slot& s) {
  FieldParams<T> a = field_params<T>(d, s);
  k_nodes<T><<<d->nfe, 256>>>(a);
  DLAUNCH("k_nodes");
  return PBPIC_OK;
}

// One forward step of a slot in place; adds the step's loss to scal[0]. With
// the j.E loss and `jkeep`, also keeps the step's current (3 planes) there.
template <class T>
int step(pbpic_diff* d, const Slot& s, double omega, void* jkeep = nullptr) {
  DTRY(nodes<T>(d, s));
  DCK(cudaMemsetAsync(d->jacc, 0, (size_t)4 * plane(d) * 8));
  DiffParams<T> dp;
  memset(&dp, 0, sizeof(dp));
  dp.push = push_params<T>(d, s);
  dp.n = d->n;
  dp.nsheet = d->nsheet;
  dp.omega_bg = omega;
  dp.in0 = d->in0;
  k_dpush<T><<<grid_of(d->n, 148 * 16), 256>>>(dp);
  DLAUNCH("k_dpush");
  const bool jdote = d->cfg.loss == PBPIC_LOSS_JDOTE;
  if (jdote) {
    DTRY(loss_jdote<T>(d, s, d->jacc, d->scal, nullptr, nullptr));
    if (jkeep) DCK(cudaMemcpyAsync(jkeep, d->jacc, (size_t)3 * plane(d) * 8, cudaMemcpyDeviceToDevice));
  }
  FieldParams<T> a = field_params<T>(d, s);
  const int g = grid_of((int64_t)d->mx * (d->my + 1));
  k_bhalf<T><<<g, 256>>>(a);
  DLAUNCH("k_bhalf");
  if (d->f32) k_efull<T, long long><<<g, 256>>>(a);
  else k_efull<T, double><<<g, 256>>>(a);
  DLAUNCH("k_efull");
  k_bhalf<T><<<g, 256>>>(a);
  DLAUNCH("k_bhalf");
  DTRY(nodes<T>(d, s));
  if (!jdote) {
    k_loss_b<T><<<grid_of((int64_t)(d->mx + 1) * (d->my + 1)), 256>>>(d->mx, d->my, 1, (const T*)d->ng,
                                                                       loss_scale(d), d->scal, nullptr);
    DLAUNCH("k_loss_b");
  }
  return PBPIC_OK;
}

int copy_slot(pbpic_diff* d, const Slot& dst, const Slot& src) {
  DCK(cudaMemcpyAsync(dst.p, src.p, part_bytes(d), cudaMemcpyDeviceToDevice));
  DCK(cudaMemcpyAsync(dst.f, src.f, field_bytes(d), cudaMemcpyDeviceToDevice));
  return PBPIC_OK;
}

template <class T>
int load(pbpic_diff* d, const pbpic_diff_params* prm) {
  const pbpic_diff_config& c = d->cfg;
  Harris hs = harris_speeds(d, prm->ti_te);
  pic::LoadParams L;
  memset(&L, 0, sizeof(L));
  L.kind = pic::LOAD_HARRIS;
  L.mx = d->mx;
  L.my = d->my;
  L.dx = d->dx;
  L.dy = d->dy;
  L.ppc = c.ppc;
  L.npairs = d->npairs;
  L.nsheet = d->nsheet;
  L.uthe = urel(hs.vthe);
  L.uthi = urel(hs.vthi);
  L.uthe_perp = L.uthe;
  L.udrift_e = urel(hs.ude);
  L.udrift_i = urel(hs.udi);
  L.lambda = c.lambda;
  L.seed = c.seed;
  View<T> v = view<T>(d, d->work);
  k_load<T><<<(unsigned)((d->npairs + 255) / 256), 256>>>(L, d->npairs, 0, v.cell, v.c[0], v.c[1], v.c[2], v.c[3],
                                                           v.c[4], nullptr);
  DLAUNCH("k_load");
  pic::FieldInit fi;
  fi.kind = pic::LOAD_HARRIS;
  fi.mx = d->mx;
  fi.my = d->my;
  fi.dx = d->dx;
  fi.dy = d->dy;
  fi.lambda = c.lambda;
  fi.psi0 = prm->psi0;
  fi.bguide = 0.0;
  fi.b0z = 0.0;
  std::vector<T> yee((size_t)6 * plane(d), T(0));
  for (int i = 0; i < d->mx; ++i)
    for (int j = 0; j <= d->my; ++j) {
      yee[(size_t)3 * plane(d) + (size_t)i * d->S + j] = (T)pic::init_bx(fi, i, j);
      yee[(size_t)4 * plane(d) + (size_t)i * d->S + j] = (T)pic::init_by(fi, i, j);
      yee[(size_t)5 * plane(d) + (size_t)i * d->S + j] = (T)pic::init_bz(fi, i, j);
    }
  DCK(cudaMemcpy(d->work.f, yee.data(), yee.size() * sizeof(T), cudaMemcpyHostToDevice));
  return PBPIC_OK;
}

template <class T>
int forward(pbpic_diff* d, const pbpic_diff_params* prm, double* loss) {
  DTRY(load<T>(d, prm));
  DCK(cudaMemset(d->scal, 0, 4 * sizeof(double)));
  const int K = d->cfg.checkpoint_every, N = d->cfg.nsteps;
  const double omega = prm->nb / d->cfg.nb0;
  for (int it = 0; it < N; ++it) {
    if (it % K == 0) DTRY(copy_slot(d, d->ck[it / K], d->work));
    DTRY(step<T>(d, d->work, omega));
  }
  DCK(cudaMemcpy(loss, d->scal, sizeof(double), cudaMemcpyDeviceToHost));
  d->last = *prm;
  d->have_forward = true;
  return PBPIC_OK;
}

AdjField adj_field(pbpic_diff* d) {
  AdjField a;
  a.mx = d->mx;
  a.my = d->my;
  a.S = d->S;
  a.ybc = PBPIC_BC_CONDUCTING;
  a.dth = (double)(d->f32 ? (double)((float)d->dt / 2.0f) : d->dt / 2.0);
  const double cva = d->f32 ? (double)(float)d->cva : d->cva;
  const double dt = d->f32 ? (double)(float)d->dt : d->dt;
  a.cdt = dt * cva * cva;
  a.idx = 1.0 / d->dx;
  a.idy = 1.0 / d->dy;
  const int64_t pl = plane(d);
  a.ex = d->fbar;
  a.ey = d->fbar + pl;
  a.ez = d->fbar + 2 * pl;
  a.bx = d->fbar + 3 * pl;
  a.by = d->fbar + 4 * pl;
  a.bz = d->fbar + 5 * pl;
  a.jbar = d->jbar;
  return a;
}

template <class T>
int backward(pbpic_diff* d, double grad[3]) {
  if (!d->have_forward) return pbpic_internal_fail(PBPIC_ESTATE, "pbpic_diff_backward needs a forward call first");
  const int K = d->cfg.checkpoint_every, N = d->cfg.nsteps;
  const double omega = d->last.nb / d->cfg.nb0;
  const int64_t pl = plane(d);
  const size_t nodes_bytes = (size_t)(d->mx + 1) * (d->my + 1) * 8 * sizeof(double);
  const bool jdote = d->cfg.loss == PBPIC_LOSS_JDOTE;
  const size_t jbytes = (size_t)3 * pl * 8;
  for (int k = 0; k < 5; ++k) DCK(cudaMemset(d->lam[0][k], 0, (size_t)d->n * d->tsz));
  DCK(cudaMemset(d->fbar, 0, (size_t)6 * pl * sizeof(double)));
  DCK(cudaMemset(d->scal + 1, 0, 3 * sizeof(double)));
  int cur = 0;
  AdjField af = adj_field(d);
  const int gf = grid_of((int64_t)d->mx * (d->my + 1));
  const int gn = grid_of((int64_t)(d->mx + 1) * (d->my + 1));
  for (int sg = (N + K - 1) / K - 1; sg >= 0; --sg) {
    const int s0 = sg * K, s1 = std::min(N, s0 + K);
    DTRY(copy_slot(d, d->seg[0], d->ck[sg]));
    for (int m = 0; m < s1 - s0; ++m) {  // recompute the segment, keeping every state
      DTRY(copy_slot(d, d->seg[m + 1], d->seg[m]));
      DTRY(step<T>(d, d->seg[m + 1], omega, jdote ? (char*)d->jseg + m * jbytes : nullptr));
    }
    for (int it = s1 - 1; it >= s0; --it) {
      const int m = it - s0;
      if (!jdote) {  // magnetic loss of step it+1: seed the adjoint of the fields after the step
        DTRY(nodes<T>(d, d->seg[m + 1]));
        DCK(cudaMemsetAsync(d->gbar, 0, nodes_bytes));
        k_loss_b<T><<<gn, 256>>>(d->mx, d->my, 1, (const T*)d->ng, loss_scale(d), nullptr, d->gbar);
        DLAUNCH("k_loss_b");
        k_adj_nodes<<<gn, 256>>>(af, d->gbar);
        DLAUNCH("k_adj_nodes");
      }
      // transposed field solve: B half step, E full step, B half step in reverse
      k_adj_bhalf<<<gf, 256>>>(af);
      DLAUNCH("k_adj_bhalf");
      k_adj_efull<<<gf, 256>>>(af);
      DLAUNCH("k_adj_efull");
      // j.E loss of step it: E (the step's start) into the current adjoint, the
      // step's current into the adjoint of that E
      if (jdote) DTRY(loss_jdote<T>(d, d->seg[m], (char*)d->jseg + m * jbytes, nullptr, d->jbar, d->fbar));
      k_zero_wall_ex<<<grid_of(d->mx), 256>>>(af);
      DLAUNCH("k_zero_wall_ex");
      k_adj_bhalf<<<gf, 256>>>(af);
      DLAUNCH("k_adj_bhalf");
      // particle adjoint of the push of step it
      DTRY(nodes<T>(d, d->seg[m]));
      DCK(cudaMemsetAsync(d->gbar, 0, nodes_bytes));
      DiffParams<T> dp;
      memset(&dp, 0, sizeof(dp));
      dp.push = push_params<T>(d, d->seg[m]);
      dp.n = d->n;
      dp.nsheet = d->nsheet;
      dp.omega_bg = omega;
      dp.in0 = d->in0;
      for (int k = 0; k < 5; ++k) {
        dp.lam_in[k] = (const T*)d->lam[cur][k];
        dp.lam_out[k] = (T*)d->lam[1 - cur][k];
      }
      dp.jbar = d->jbar;
      dp.gbar = d->gbar;
      dp.domega = d->scal + 1;
      k_dadjoint<T><<<grid_of(d->n, 148 * 16), 256>>>(dp);
      DLAUNCH("k_dadjoint");
      k_adj_nodes<<<gn, 256>>>(af, d->gbar);
      DLAUNCH("k_adj_nodes");
      cur = 1 - cur;
    }
  }
  // d loss / d tau through the loaded momenta (checkpoint 0 holds the initial state)
  {
    const double tite = d->last.ti_te;
    Harris hs = harris_speeds(d, tite);
    const double dvthe = -hs.vthe / (2.0 * (1.0 + tite));
    const double dvthi = dvthe * sqrt(tite / d->cfg.mime) + hs.vthe * 0.5 / sqrt(tite * d->cfg.mime);
    const double du = -1.0 / (d->cfg.lambda * d->cva);
    const double dudi_v = du / ((1.0 + tite) * (1.0 + tite)), dude_v = du / ((1.0 + tite) * (1.0 + tite));
    View<T> v0 = view<T>(d, d->ck[0]);
    k_dtau<T><<<grid_of(d->n, 148 * 16), 256>>>(
        d->n, d->nsheet, v0.c[2], v0.c[3], v0.c[4], (const T*)d->lam[cur][2], (const T*)d->lam[cur][3],
        (const T*)d->lam[cur][4], urel(hs.vthi), urel(hs.vthe), durel(hs.vthi) * dvthi, durel(hs.vthe) * dvthe,
        urel(hs.udi), urel(hs.ude), durel(hs.udi) * dudi_v, durel(hs.ude) * dude_v, d->scal + 2);
    DLAUNCH("k_dtau");
  }
  double sc[3];
  DCK(cudaMemcpy(sc, d->scal + 1, 2 * sizeof(double), cudaMemcpyDeviceToHost));
  // d loss / d psi0: the initial B is linear in psi0
  std::vector<double> fb((size_t)2 * pl);
  DCK(cudaMemcpy(fb.data(), d->fbar + 3 * pl, fb.size() * sizeof(double), cudaMemcpyDeviceToHost));
  pic::FieldInit f1, f0;
  f1.kind = f0.kind = pic::LOAD_HARRIS;
  f1.mx = f0.mx = d->mx;
  f1.my = f0.my = d->my;
  f1.dx = f0.dx = d->dx;
  f1.dy = f0.dy = d->dy;
  f1.lambda = f0.lambda = d->cfg.lambda;
  f1.bguide = f0.bguide = 0.0;
  f1.b0z = f0.b0z = 0.0;
  f1.psi0 = 1.0;
  f0.psi0 = 0.0;
  double gpsi = 0.0;
  for (int i = 0; i < d->mx; ++i)
    for (int j = 0; j <= d->my; ++j) {
      const size_t o = (size_t)i * d->S + j;
      gpsi += fb[o] * (pic::init_bx(f1, i, j) - pic::init_bx(f0, i, j));
      if (j < d->my) gpsi += fb[pl + o] * (pic::init_by(f1, i, j) - pic::init_by(f0, i, j));
    }
  grad[0] = gpsi;
  grad[1] = sc[0] / d->cfg.nb0;
  grad[2] = sc[1];
  return PBPIC_OK;
}

}  // namespace

extern "C" {

int pbpic_diff_create(const pbpic_diff_config* cfg, pbpic_diff** out) {
  if (!cfg || !out) return pbpic_internal_fail(PBPIC_EINVAL, "null argument");
  *out = nullptr;
  const pbpic_diff_config& c = *cfg;
  if (c.mx < 3 || c.my < 3 || c.mx > 32767 || c.my > 65535 || c.ppc <= 0)
    return pbpic_internal_fail(PBPIC_EINVAL, "bad grid or ppc");
  if (c.precision != PBPIC_FP64_PLAIN && c.precision != PBPIC_FP32_MIXED)
    return pbpic_internal_fail(PBPIC_EINVAL, "unknown precision");
  if (c.nsteps <= 0 || c.checkpoint_every <= 0) return pbpic_internal_fail(PBPIC_EINVAL, "nsteps and checkpoint_every must be positive");
  if (c.loss != PBPIC_LOSS_MAGNETIC && c.loss != PBPIC_LOSS_JDOTE) return pbpic_internal_fail(PBPIC_EINVAL, "unknown loss");
  if (!(c.dx > 0 && c.mime > 0 && c.wpe_wce > 0 && c.lambda > 0 && c.nb0 > 0 && c.cfl > 0 && c.cfl < 1))
    return pbpic_internal_fail(PBPIC_EINVAL, "dx, mime, wpe_wce, lambda, nb0 must be positive and 0 < cfl < 1");
  if ((int64_t)2 * c.ppc * c.mx * c.my > 0x7fffff00ll) return pbpic_internal_fail(PBPIC_EINVAL, "too many particles");
  pbpic_diff* d = new pbpic_diff();
  d->cfg = c;
  d->f32 = c.precision == PBPIC_FP32_MIXED;
  d->tsz = d->f32 ? 4 : 8;
  d->mx = c.mx;
  d->my = c.my;
  d->S = c.my + 1;
  d->dx = d->dy = c.dx;
  d->cva = c.wpe_wce * sqrt(c.mime);
  d->dt = c.cfl / (d->cva * sqrt(2.0) / c.dx);
  d->npairs = (int64_t)c.ppc * c.mx * c.my;
  d->n = 2 * d->npairs;
  const double ly = c.my * c.dx, lx = c.mx * c.dx;
  d->nsheet = (int64_t)llround((double)d->npairs * (2.0 * c.lambda / (2.0 * c.lambda + c.nb0 * ly)));
  d->in0 = lx * (2.0 * c.lambda + c.nb0 * ly) / (c.dx * c.dx) / (double)d->npairs;
  d->nseg = (c.nsteps + c.checkpoint_every - 1) / c.checkpoint_every;
  int r = PBPIC_OK;
  auto A = [&](void** p, size_t b) {
    if (r == PBPIC_OK) r = dmalloc(d, p, b);
  };
  d->ck.resize(d->nseg);
  d->seg.resize(c.checkpoint_every + 1);
  for (auto& s : d->ck) {
    A(&s.p, part_bytes(d));
    A(&s.f, field_bytes(d));
  }
  for (auto& s : d->seg) {
    A(&s.p, part_bytes(d));
    A(&s.f, field_bytes(d));
  }
  A(&d->work.p, part_bytes(d));
  A(&d->work.f, field_bytes(d));
  A(&d->ng, (size_t)(c.mx + 1) * (c.my + 1) * 8 * d->tsz);
  A(&d->jacc, (size_t)4 * plane(d) * 8);
  d->nfe = grid_of((int64_t)(c.mx + 1) * (c.my + 1));
  A((void**)&d->fe_part, (size_t)d->nfe * 2 * sizeof(double));
  for (int b = 0; b < 2; ++b)
    for (int k = 0; k < 5; ++k) A(&d->lam[b][k], (size_t)d->n * d->tsz);
  A((void**)&d->fbar, (size_t)6 * plane(d) * sizeof(double));
  A((void**)&d->jbar, (size_t)3 * plane(d) * sizeof(double));
  A((void**)&d->gbar, (size_t)(c.mx + 1) * (c.my + 1) * 8 * sizeof(double));
  A((void**)&d->scal, 4 * sizeof(double));
  if (c.loss == PBPIC_LOSS_JDOTE) A(&d->jseg, (size_t)c.checkpoint_every * 3 * plane(d) * 8);
  if (r != PBPIC_OK) {
    pbpic_diff_destroy(d);
    return r;
  }
  *out = d;
  return PBPIC_OK;
}

int pbpic_diff_destroy(pbpic_diff* d) {
  if (!d) return PBPIC_OK;
  cudaDeviceSynchronize();
  for (void* p : d->allocs) cudaFree(p);
  delete d;
  return PBPIC_OK;
}

int pbpic_diff_forward(pbpic_diff* d, const pbpic_diff_params* params, double* loss) {
  if (!d || !params || !loss) return pbpic_internal_fail(PBPIC_EINVAL, "null argument");
  if (!(params->nb > 0 && params->ti_te > 0)) return pbpic_internal_fail(PBPIC_EINVAL, "nb and ti_te must be positive");
  return d->f32 ? forward<float>(d, params, loss) : forward<double>(d, params, loss);
}

int pbpic_diff_backward(pbpic_diff* d, double grad[3]) {
  if (!d || !grad) return pbpic_internal_fail(PBPIC_EINVAL, "null argument");
  int r = d->f32 ? backward<float>(d, grad) : backward<double>(d, grad);
  if (r == PBPIC_OK && cudaDeviceSynchronize() != cudaSuccess)
    return pbpic_internal_fail(PBPIC_ECUDA, "device error in the adjoint");
  return r;
}

}  // extern "C"
