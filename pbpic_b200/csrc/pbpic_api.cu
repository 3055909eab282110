// C ABI of the pbpic B200 step (include/pbpic.h): device state, kernel
// orchestration and host<->device transfers.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>
#include <errno.h>
#include <sys/stat.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/pbpic.h"
#include "api_internal.h"
#include "device_common.cuh"
#include "kernels_batch.cuh"
#include "kernels_field.cuh"
#include "kernels_misc.cuh"
#include "kernels_push.cuh"
#include "kernels_slab.cuh"
#include "kernels_sort.cuh"
#include "h5_writer.h"
#include "npy_io.h"
#include "pic_common.h"
#include "pic_fields_init.h"

using namespace pbd;

namespace {

thread_local std::string g_err = "";
std::atomic<long long> g_launches{0};  // kernels launched by this library (all handles)

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

#define CK(call)                                                                         \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess) return fail(PBPIC_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define CKLAUNCH(what)                                                                    \
  do {                                                                                    \
    g_launches.fetch_add(1, std::memory_order_relaxed);                                   \
    cudaError_t e_ = cudaGetLastError();                                                  \
    if (e_ != cudaSuccess) return fail(PBPIC_ECUDA, std::string(what) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define TRY(...)                   \
  do {                             \
    int r_ = (__VA_ARGS__);        \
    if (r_ != PBPIC_OK) return r_; \
  } while (0)

int grid_for(int64_t n, int block, int maxblocks = 148 * 16) {
  int64_t g = (n + block - 1) / block;
  if (g < 1) g = 1;
  if (g > maxblocks) g = maxblocks;
  return (int)g;
}

// ------------------------------------------------------------------ scan
// Exclusive scan of n int32 in place. scratch holds the chunk totals of every
// level: scan_scratch_ints(n) entries.
int64_t scan_scratch_ints(int64_t n) {
  int64_t tot = 0;
  while (true) {
    int64_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
    tot += nb + 1;
    if (nb <= 1) break;
    n = nb;
  }
  return tot;
}

int scan_excl(cudaStream_t s, int32_t* data, int64_t n, int32_t* scratch) {
  if (n <= 0) return PBPIC_OK;
  int64_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
  k_scan_local<<<(unsigned)nb, SCAN_BT, 0, s>>>(data, data, n, scratch);
  CKLAUNCH("k_scan_local");
  if (nb > 1) {
    TRY(scan_excl(s, scratch, nb, scratch + nb + 1));
    k_scan_add<<<(unsigned)nb, 256, 0, s>>>(data, n, scratch);
    CKLAUNCH("k_scan_add");
  }
  return PBPIC_OK;
}

// ------------------------------------------------------------ radix sort
int radix_passes(int32_t ncells) {
  int bits = 1;
  while (bits < 31 && (1ll << bits) < (int64_t)ncells) ++bits;
  return (bits + 7) / 8;
}

int64_t radix_hist_ints(int64_t n) { return 256 * ((n + RTILE - 1) / RTILE); }

// Stable LSD radix sort of keys k0[0..n) (values: the indices). Buffers k0/k1
// and v0/v1 ping-pong; returns the buffer holding the permutation.
int radix_sort(cudaStream_t s, int64_t n, int32_t ncells, int32_t* k0, int32_t* k1, int32_t* v0,
               int32_t* v1, int32_t* rhist, int32_t* scan_scratch, int32_t** perm) {
  const int passes = radix_passes(ncells);
  const int nblocks = (int)((n + RTILE - 1) / RTILE);
  int32_t *kin = k0, *kout = k1, *vin = nullptr, *vout = v1;
  int32_t* other_v = v0;
  for (int p = 0; p < passes; ++p) {
    k_radix_up<<<nblocks, RB, 0, s>>>(kin, n, 8 * p, rhist, nblocks);
    CKLAUNCH("k_radix_up");
    TRY(scan_excl(s, rhist, (int64_t)256 * nblocks, scan_scratch));
    k_radix_down<<<nblocks, RB, 0, s>>>(kin, vin, n, 8 * p, rhist, nblocks, kout, vout);
    CKLAUNCH("k_radix_down");
    std::swap(kin, kout);
    vin = vout;
    vout = other_v;
    other_v = vin;
  }
  *perm = vin;
  return PBPIC_OK;
}

template <class T>
struct DevT {
  static constexpr bool mixed = sizeof(T) == 4;
};

}  // namespace

int pbpic_internal_fail(int code, const std::string& msg) { return fail(code, msg); }
void pbpic_internal_count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

// ===================================================================== handle
struct pbpic_handle {
  pbpic_config cfg;
  bool mixed = false;
  size_t tsz = 8;
  cudaStream_t stream = 0;
  int S = 0, ncells = 0, TY = 0, tpc = 0, ntiles = 0;
  int64_t n = 0, cap = 0;
  uint32_t* cell[2] = {nullptr, nullptr};
  void* comp[2][5] = {{nullptr}};
  int32_t* pid[2] = {nullptr, nullptr};
  int cur = 0;
  void* f[6] = {nullptr};
  void* ng = nullptr;
  void* cg = nullptr;  // mixed form: per-cell gather records of the push (k_cell_records after k_nodes)
  void* jacc = nullptr;
  int32_t *counts = nullptr, *off = nullptr, *tile_off = nullptr;
  double *ke_part = nullptr, *fe_part = nullptr;
  int nfe = 0, nke = 0;
  double* hist = nullptr;
  int hist_rows = 0;
  int itime = 0;
  int* status = nullptr;
  int32_t *keys[2] = {nullptr, nullptr}, *vals[2] = {nullptr, nullptr};
  int32_t* rhist = nullptr;
  int32_t* scan_scratch = nullptr;
  bool sorted = false;
  bool fused_ok = false;    // grid admits the fused counting sort (distinct window cells)
  bool hist_valid = false;  // the last push counted new cells per tile on a sorted array
  bool defer_sort = false;  // pbpic_step: the push leaves its fused sort to run beside the field solve
  cudaStream_t side = nullptr;                       // pbpic_step: the field solve's stream
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;  // pbpic_step: push -> field solve, field solve -> next
  // The fused sort leaves the particle data in place and writes perm (sorted
  // position -> element); while `lazy`, the cell order is the arrays read
  // through perm. The next push reads through it; every other reader of the
  // particle arrays applies it first (materialize).
  int32_t* perm = nullptr;
  int32_t* perm2 = nullptr;  // the band assembly's permutation (swapped with perm)
  bool lazy = false;
  size_t push_optin = 0;    // dynamic shared memory the plain form's k_push may take
  int nb = 0;               // window bins per tile, 3*(TY+2)
  int tile_cap = 0;         // tiles the per-tile arrays hold
  int64_t bin_cap = 0;      // (tile, bin) entries tilecnt and tbase hold
  int32_t* tilecnt = nullptr;
  int32_t* tbase = nullptr;
  void* staging = nullptr;
  size_t staging_bytes = 0;
  double* rho = nullptr;
  double* dscalar = nullptr;
  int filters = 0;               // field filters (PBPIC_FILTER_*), periodic y only
  double marder_d = 0.001, cer_tau = 0.125;
  void* fc = nullptr;            // filter corrections, 5 x mx x my values of the precision
  int32_t* runbuf = nullptr;        // run-merge sort: run counts and run starts (2 x cells)
  int32_t* band_flags = nullptr;    // slab exchange: flags / positions (capacity + 2)
  int32_t* band_scratch = nullptr;  // and their scan's chunk totals
  int32_t* colbuf = nullptr;        // sorted slab paths: per-column counts and starts (8 x (mx + 1))
  int32_t* colscan = nullptr;       // and their scans' chunk totals
  // spectra written by pbpic_dump_h5 so far (time step, 2 x nbins counts): the
  // reference's spectra.h5 gains one group per call, so every call rewrites it
  // with all of them
  std::vector<std::pair<int32_t, std::vector<int32_t>>> h5_spectra;
  std::vector<void*> allocs;
};

namespace {

int dalloc(pbpic_handle* h, void** p, size_t bytes) {
  if (bytes == 0) bytes = 16;
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    *p = nullptr;
    return fail(PBPIC_ENOMEM, std::string("cudaMalloc(") + std::to_string(bytes) + "): " + cudaGetErrorString(e));
  }
  h->allocs.push_back(*p);
  return PBPIC_OK;
}

template <class P>
int dalloc(pbpic_handle* h, P** p, size_t bytes) {
  void* q = nullptr;
  int r = dalloc(h, &q, bytes);
  *p = (P*)q;
  return r;
}

int64_t plane_elems(const pbpic_handle* h) { return (int64_t)h->cfg.mx * h->S; }

// Dynamic shared memory of k_push: the tile's current window (16 x (ty+3)
// 8-byte accumulators), the new-cell histogram (3 x (ty+2) int) and, in the
// mixed form, the crossers' split 32-bit windows (2 x 8 x (ty+3)) and the
// tile's gather records staged by a bulk copy (96 B a row); with the static
// part this stays below the 48 KB a launch gets without opting in. The
// plain form adds the second stage of its run sums (a warp's 17 x 33 doubles
// per warp), which takes 256-thread blocks above 48 KB (push_smem_optin).
size_t push_smem_bytes(int ty, bool mixed) {
  if (!mixed) {
    if (PBPIC_PUSH_STAGE_NODES) return push_node_offset(ty) + (size_t)2 * (ty + 1) * 64;  // + staged node columns
    return push_first_offset(ty) + (size_t)(PushThreads<double>::value / 32) * 17 * 33 * sizeof(double);
  }
  if (PBPIC_CELL_COEF && PBPIC_PUSH_STAGE_RECS) return push_rec_offset(ty) + (size_t)ty * 96;  // + staged records
  return (size_t)16 * (ty + 3) * 8 + (size_t)3 * (ty + 2) * 4 + (size_t)16 * (ty + 3) * 4;
}

// Lets the plain form's k_push instantiations take more than 48 KB of shared
// memory. The limit belongs to the function and every handle on the device
// shares it, so it is set to what the tallest tile (64 rows) needs, never to a
// handle's own smaller figure (once per handle: a handle stays on one device).
template <class T, bool MIXED>
int push_smem_optin(pbpic_handle* h) {
  if constexpr (!MIXED) {
    const size_t smem = push_smem_bytes(64, false);
    if (h->push_optin >= smem) return PBPIC_OK;
    const void* fns[] = {(const void*)k_push<T, MIXED, true, false, true>, (const void*)k_push<T, MIXED, true, true, true>,
                         (const void*)k_push<T, MIXED, true, false>,       (const void*)k_push<T, MIXED, true, true>,
                         (const void*)k_push<T, MIXED, false, false>,      (const void*)k_push<T, MIXED, false, true>};
    for (const void* f : fns) CK(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    h->push_optin = smem;
  }
  return PBPIC_OK;
}

int ensure_staging(pbpic_handle* h, size_t bytes) {
  if (h->staging_bytes >= bytes) return PBPIC_OK;
  if (h->staging) {
    cudaFree(h->staging);
    h->allocs.erase(std::find(h->allocs.begin(), h->allocs.end(), h->staging));
    h->staging = nullptr;
  }
  TRY(dalloc(h, &h->staging, bytes));
  h->staging_bytes = bytes;
  return PBPIC_OK;
}

int ensure_hist(pbpic_handle* h, int rows) {
  if (rows <= h->hist_rows) return PBPIC_OK;
  int nr = std::max(rows, h->hist_rows * 2);
  double* nh = nullptr;
  TRY(dalloc(h, &nh, (size_t)nr * 4 * sizeof(double)));
  CK(cudaMemsetAsync(nh, 0, (size_t)nr * 4 * sizeof(double), h->stream));
  if (h->hist) {
    CK(cudaMemcpyAsync(nh, h->hist, (size_t)h->hist_rows * 4 * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    cudaFree(h->hist);
    h->allocs.erase(std::find(h->allocs.begin(), h->allocs.end(), (void*)h->hist));
  }
  h->hist = nh;
  h->hist_rows = nr;
  return PBPIC_OK;
}

template <class T>
T* P(pbpic_handle* h, int buf, int c) {
  return (T*)h->comp[buf][c];
}

// ------------------------------------------------------------- constants
template <class T, bool MIXED>
PushParams<T> push_params(pbpic_handle* h) {
  const pbpic_config& c = h->cfg;
  PushParams<T> p;
  p.mx = c.mx;
  p.my = c.my;
  p.S = h->S;
  p.ybc = c.ybc;
  p.compat = c.compat;
  p.tile_rows = h->TY;
  p.tiles_per_col = h->tpc;
  p.ntiles = h->ntiles;
  p.tile_off = h->tile_off;
  const int b = h->cur;
  p.cell = h->cell[b];
  p.dx = P<T>(h, b, 0);
  p.dy = P<T>(h, b, 1);
  p.ux = P<T>(h, b, 2);
  p.uy = P<T>(h, b, 3);
  p.uz = P<T>(h, b, 4);
  p.ng = (const T*)h->ng;
  p.cg = (const T*)h->cg;
  p.jacc = h->jacc;
  p.tilecnt = h->tilecnt;
  p.cell_off = h->off;
  p.src = nullptr;
  p.cell_o = nullptr;
  p.dx_o = p.dy_o = p.ux_o = p.uy_o = p.uz_o = nullptr;
  p.pid_i = nullptr;
  p.pid_o = nullptr;
  const T dt = (T)c.dt, mime = (T)c.mime, cva = (T)c.cva, dx = (T)c.dx, dy = (T)c.dy;
  for (int s = 0; s < 2; ++s) {
    const T q = s == 0 ? T(1) : T(-1);
    const T ms = s == 0 ? mime : T(1);
    p.c0[s] = q * dt * mime / ms / T(2);  // pic2d.f90:969
    p.c1[s] = p.c0[s] / cva;              // pic2d.f90:970
    p.ms[s] = ms;
    p.q[s] = q;
    p.qx[s] = MIXED ? q : q * dx / dt;  // pic2d.f90:1237-1238
    p.qy[s] = MIXED ? q : q * dy / dt;
  }
  p.dtcva = dt * cva;  // pic2d.f90:1004
  p.idx = T(1) / dx;   // pic2d.f90:16
  p.idy = T(1) / dy;
  p.cva = cva;
  p.ke_part = h->ke_part;
  p.status = h->status;
  return p;
}

template <class T, bool MIXED>
FieldParams<T> field_params(pbpic_handle* h) {
  const pbpic_config& c = h->cfg;
  FieldParams<T> a;
  a.mx = c.mx;
  a.my = c.my;
  a.S = h->S;
  a.ybc = c.ybc;
  a.ex = (T*)h->f[0];
  a.ey = (T*)h->f[1];
  a.ez = (T*)h->f[2];
  a.bx = (T*)h->f[3];
  a.by = (T*)h->f[4];
  a.bz = (T*)h->f[5];
  const T dt = (T)c.dt, cva = (T)c.cva;
  const T cva2 = cva * cva;  // pic2d.f90:21
  a.dth = dt / T(2);         // pic2d.f90:43
  a.cdt = dt * cva2;         // pic2d.f90:742
  a.idx = T(1) / (T)c.dx;
  a.idy = T(1) / (T)c.dy;
  a.jacc = h->jacc;
  if (MIXED) {
    a.jscale[0] = c.in0 * (c.dx / c.dt) * FIX_INV;
    a.jscale[1] = c.in0 * (c.dy / c.dt) * FIX_INV;
    a.jscale[2] = c.in0 * c.cva * FIX_INV;
    a.jscale[3] = c.in0 * FIX_INV;
  } else {
    for (int k = 0; k < 4; ++k) a.jscale[k] = c.in0;
  }
  a.ng = (T*)h->ng;
  a.cg = (T*)h->cg;
  a.fe_part = h->fe_part;
  return a;
}

double fe_scale(const pbpic_config& c) { return 0.5 * c.mime / (c.cva * c.cva * c.cva * c.cva * c.in0); }
double fb_scale(const pbpic_config& c) { return 0.5 * c.mime / (c.cva * c.cva * c.in0); }

// ------------------------------------------------------------ operations
template <class T, bool MIXED>
int nodes_and_field_energy(pbpic_handle* h, int row) {
  TRY(ensure_hist(h, row + 1));
  FieldParams<T> a = field_params<T, MIXED>(h);
  k_nodes<T><<<h->nfe, 256, 0, h->stream>>>(a);
  CKLAUNCH("k_nodes");
  if constexpr (MIXED) {
    k_cell_records<<<h->nfe, 256, 0, h->stream>>>(a);
    CKLAUNCH("k_cell_records");
  }
  k_energy_row<<<1, 256, 0, h->stream>>>(nullptr, 0, h->fe_part, h->nfe, fe_scale(h->cfg), fb_scale(h->cfg),
                                          h->hist + (size_t)row * 4);
  CKLAUNCH("k_energy_row");
  return PBPIC_OK;
}

// Node averages of node rows [b0, b1) and the gather records of the cells on
// them (cell row c reads node rows c and c + 1), after some field rows changed.
template <class T, bool MIXED>
int node_rows(pbpic_handle* h, int b0, int b1) {
  if (b1 <= b0) return PBPIC_OK;
  FieldParams<T> a = field_params<T, MIXED>(h);
  k_nodes_rows<T><<<grid_for((int64_t)(h->cfg.mx + 1) * (b1 - b0), 256), 256, 0, h->stream>>>(a, b0, b1);
  CKLAUNCH("k_nodes_rows");
  if constexpr (MIXED) {
    const int r0 = std::max(0, b0 - 1), r1 = std::min(h->cfg.my, b1);
    if (r1 > r0) {
      k_cell_records_rows<<<grid_for((int64_t)h->cfg.mx * (r1 - r0), 256), 256, 0, h->stream>>>(a, r0, r1);
      CKLAUNCH("k_cell_records_rows");
    }
  }
  return PBPIC_OK;
}

template <class T, bool MIXED>
int kinetic_row(pbpic_handle* h, int row) {
  TRY(ensure_hist(h, row + 1));
  const int b = h->cur;
  k_kinetic<T, MIXED><<<h->nke, 256, 0, h->stream>>>(h->n, h->cell[b], P<T>(h, b, 2), P<T>(h, b, 3),
                                                      P<T>(h, b, 4), (T)h->cfg.mime, h->ke_part);
  CKLAUNCH("k_kinetic");
  k_energy_row<<<1, 256, 0, h->stream>>>(h->ke_part, h->nke, nullptr, 0, 0, 0, h->hist + (size_t)row * 4);
  CKLAUNCH("k_energy_row");
  return PBPIC_OK;
}

// Apply the fused sort's permutation to the particle arrays (they are then in
// cell order themselves); a no-op unless the handle is lazy.
template <class T>
int materialize_t(pbpic_handle* h) {
  const int64_t n = h->n;
  const int b = h->cur, o = 1 - b;
  if (n > 0) {
    k_gather<T><<<grid_for(n, 256), 256, 0, h->stream>>>(h->perm, n, h->cell[b], P<T>(h, b, 0), P<T>(h, b, 1),
                                                          P<T>(h, b, 2), P<T>(h, b, 3), P<T>(h, b, 4), h->pid[b],
                                                          h->cell[o], P<T>(h, o, 0), P<T>(h, o, 1), P<T>(h, o, 2),
                                                          P<T>(h, o, 3), P<T>(h, o, 4), h->pid[o]);
    CKLAUNCH("k_gather");
    h->cur = o;
  }
  h->lazy = false;
  return PBPIC_OK;
}

int materialize(pbpic_handle* h) {
  if (!h->lazy) return PBPIC_OK;
  return h->mixed ? materialize_t<float>(h) : materialize_t<double>(h);
}

int set_unsorted_tiles(pbpic_handle* h) {
  k_tile_off_uniform<<<grid_for(h->ntiles + 1, 256, 1 << 20), 256, 0, h->stream>>>(h->ntiles, h->n, h->tile_off);
  CKLAUNCH("k_tile_off_uniform");
  h->sorted = false;
  h->hist_valid = false;
  h->lazy = false;
  return PBPIC_OK;
}

template <class T, bool MIXED>
int do_fused_sort(pbpic_handle* h);

template <class T, bool MIXED>
int do_sort(pbpic_handle* h) {
  if (h->hist_valid) return do_fused_sort<T, MIXED>(h);
  if (h->sorted) return PBPIC_OK;  // already in cell order (tables current)
  cudaStream_t s = h->stream;
  const int64_t n = h->n;
  CK(cudaMemsetAsync(h->counts, 0, (size_t)(h->ncells + 1) * 4, s));
  const int b = h->cur, o = 1 - b;
  if (n > 0) {
    k_cell_keys<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(h->cell[b], n, h->cfg.my, h->keys[0], h->counts);
    CKLAUNCH("k_cell_keys");
  }
  CK(cudaMemcpyAsync(h->off, h->counts, (size_t)(h->ncells + 1) * 4, cudaMemcpyDeviceToDevice, s));
  TRY(scan_excl(s, h->off, h->ncells + 1, h->scan_scratch));
  // one run per cell (concatenated sorted pieces): a single scatter suffices
  bool runs = false;
  if (n > 0) {
    if (!h->runbuf) TRY(dalloc(h, &h->runbuf, ((size_t)2 * h->ncells + 16) * 4));
    int32_t* nruns = h->runbuf;
    int32_t* runstart = h->runbuf + h->ncells;
    int* flag = (int*)(h->runbuf + 2 * (size_t)h->ncells);
    CK(cudaMemsetAsync(nruns, 0, (size_t)h->ncells * 4, s));
    CK(cudaMemsetAsync(flag, 0, 4, s));
    k_cell_runs<<<grid_for(n, 256), 256, 0, s>>>(h->cell[b], n, h->cfg.my, nruns, runstart);
    CKLAUNCH("k_cell_runs");
    k_runs_ok<<<grid_for(h->ncells, 256), 256, 0, s>>>(nruns, h->ncells, flag);
    CKLAUNCH("k_runs_ok");
    int many = 1;
    CK(cudaMemcpyAsync(&many, flag, 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (!many) {
      k_run_scatter<T><<<grid_for(n, 256), 256, 0, s>>>(n, h->cfg.my, h->off, runstart, h->cell[b], P<T>(h, b, 0),
                                                        P<T>(h, b, 1), P<T>(h, b, 2), P<T>(h, b, 3), P<T>(h, b, 4),
                                                        h->pid[b], h->cell[o], P<T>(h, o, 0), P<T>(h, o, 1),
                                                        P<T>(h, o, 2), P<T>(h, o, 3), P<T>(h, o, 4), h->pid[o]);
      CKLAUNCH("k_run_scatter");
      h->cur = o;
      runs = true;
    }
  }
  if (n > 0 && !runs) {
    int32_t* perm = nullptr;
    TRY(radix_sort(s, n, h->ncells, h->keys[0], h->keys[1], h->vals[0], h->vals[1], h->rhist, h->scan_scratch,
                   &perm));
    k_gather<T><<<grid_for(n, 256), 256, 0, s>>>(perm, n, h->cell[b], P<T>(h, b, 0), P<T>(h, b, 1), P<T>(h, b, 2),
                                                  P<T>(h, b, 3), P<T>(h, b, 4), h->pid[b], h->cell[o], P<T>(h, o, 0),
                                                  P<T>(h, o, 1), P<T>(h, o, 2), P<T>(h, o, 3), P<T>(h, o, 4),
                                                  h->pid[o]);
    CKLAUNCH("k_gather");
    h->cur = o;
  }
  k_tile_off<<<grid_for(h->ntiles + 1, 256, 1 << 20), 256, 0, s>>>(h->off, h->ntiles, h->tpc, h->TY, h->cfg.my,
                                                                  (int32_t)n, h->tile_off);
  CKLAUNCH("k_tile_off");
  h->sorted = true;
  h->hist_valid = false;
  return PBPIC_OK;
}

template <class T, bool MIXED>
int do_push(pbpic_handle* h) {
  const bool autosort = !(h->cfg.options & PBPIC_OPT_NO_AUTOSORT) && h->fused_ok;
  if (autosort && !h->sorted) TRY((do_sort<T, MIXED>(h)));
  cudaStream_t s = h->stream;
  TRY(ensure_hist(h, h->itime + 2));
  CK(cudaMemsetAsync(h->jacc, 0, (size_t)4 * plane_elems(h) * 8, s));
  PushParams<T> p = push_params<T, MIXED>(h);
  const size_t smem = push_smem_bytes(h->TY, MIXED);
  if (h->TY > 64) return fail(PBPIC_ESTATE, "k_push: tiles have at most 64 rows");
  TRY((push_smem_optin<T, MIXED>(h)));
  const bool hist = h->sorted && h->fused_ok;
  if (hist && !p.cell_off) return fail(PBPIC_EINVAL, "k_push: counting from the cell offsets needs them");
  if (MIXED && !p.cg) return fail(PBPIC_ESTATE, "k_push: no per-cell gather records");
  const int nt = PushThreads<T>::value;
  // the compat instances also carry the plain form's exact-order arithmetic
  const bool compat = h->cfg.compat != 0 || (!MIXED && (h->cfg.options & PBPIC_OPT_EXACT_FP64));
  if (h->lazy) {  // read through the sort's permutation, write in cell order to the other buffer
    if (!hist) return fail(PBPIC_ESTATE, "k_push: a permuted input needs the sort's tables");
    const int o = 1 - h->cur;
    p.src = h->perm;
    p.cell_o = h->cell[o];
    p.dx_o = P<T>(h, o, 0);
    p.dy_o = P<T>(h, o, 1);
    p.ux_o = P<T>(h, o, 2);
    p.uy_o = P<T>(h, o, 3);
    p.uz_o = P<T>(h, o, 4);
    p.pid_i = h->pid[h->cur];
    p.pid_o = h->pid[o];
    if (!compat) k_push<T, MIXED, true, false, true><<<h->ntiles, nt, smem, s>>>(p);
    else k_push<T, MIXED, true, true, true><<<h->ntiles, nt, smem, s>>>(p);
    CKLAUNCH("k_push");
    h->cur = o;
    h->lazy = false;
  } else {
    if (hist && !compat) k_push<T, MIXED, true, false><<<h->ntiles, nt, smem, s>>>(p);
    else if (hist) k_push<T, MIXED, true, true><<<h->ntiles, nt, smem, s>>>(p);
    else if (!compat) k_push<T, MIXED, false, false><<<h->ntiles, nt, smem, s>>>(p);
    else k_push<T, MIXED, false, true><<<h->ntiles, nt, smem, s>>>(p);
    CKLAUNCH("k_push");
  }
  k_energy_row<<<1, 256, 0, s>>>(h->ke_part, h->ntiles, nullptr, 0, 0, 0, h->hist + (size_t)(h->itime + 1) * 4);
  CKLAUNCH("k_energy_row");
  h->hist_valid = hist;
  h->sorted = false;
  if (autosort && !h->defer_sort) TRY((do_fused_sort<T, MIXED>(h)));
  return PBPIC_OK;
}

// Counting sort from the per-tile histograms of the last push (kernels_sort.cuh).
template <class T, bool MIXED>
int do_fused_sort(pbpic_handle* h) {
  cudaStream_t s = h->stream;
  const int64_t n = h->n;
  FusedSortParams f;
  f.mx = h->cfg.mx;
  f.my = h->cfg.my;
  f.ybc = h->cfg.ybc;
  f.ty = h->TY;
  f.tpc = h->tpc;
  f.ntiles = h->ntiles;
  f.nb = h->nb;
  f.tilecnt = h->tilecnt;
  f.counts = h->counts;
  f.off = h->off;
  f.base = h->tbase;
  // cell counts; their chunk scan into the offsets; the scan of the chunk
  // totals; one pass per cell adding the chunk prefixes and writing the
  // (tile, bin) first slots
  k_fused_counts<<<grid_for((int64_t)h->ncells + 1, 256), 256, 0, s>>>(f);
  CKLAUNCH("k_fused_counts");
  const int64_t nchunks = ((int64_t)h->ncells + 1 + SCAN_TILE - 1) / SCAN_TILE;
  k_scan_local<<<(unsigned)nchunks, SCAN_BT, 0, s>>>(h->counts, h->off, (int64_t)h->ncells + 1, h->scan_scratch);
  CKLAUNCH("k_scan_local");
  TRY(scan_excl(s, h->scan_scratch, nchunks, h->scan_scratch + nchunks + 1));
  k_fused_offsets<<<grid_for((int64_t)h->ncells + 1, 256), 256, 0, s>>>(f, h->scan_scratch);
  CKLAUNCH("k_fused_offsets");
  ScatterParams<T> sp{};  // the ranking reads the cell words and the tables only
  sp.mx = f.mx;
  sp.my = f.my;
  sp.ybc = f.ybc;
  sp.ty = f.ty;
  sp.tpc = f.tpc;
  sp.nb = f.nb;
  sp.tile_off = h->tile_off;
  sp.base = h->tbase;
  sp.ci = h->cell[h->cur];
  if (n > 0) {  // the sorted order as a permutation; the particle data stay in place
    if (!h->perm) TRY(dalloc(h, &h->perm, ((size_t)std::max<int64_t>(h->cap, 1) + 16) * 4));
    sp.perm = h->perm;
    k_fused_perm<T><<<h->ntiles, 256, 0, s>>>(sp);
    CKLAUNCH("k_fused_perm");
    h->lazy = true;
  }
  k_tile_off<<<grid_for(h->ntiles + 1, 256, 1 << 20), 256, 0, s>>>(h->off, h->ntiles, h->tpc, h->TY, h->cfg.my,
                                                                  (int32_t)n, h->tile_off);
  CKLAUNCH("k_tile_off");
  h->sorted = true;
  h->hist_valid = false;
  return PBPIC_OK;
}

template <class T, bool MIXED>
FilterParams<T> filter_params(pbpic_handle* h) {
  const pbpic_config& c = h->cfg;
  FilterParams<T> f;
  f.flags = h->filters;
  const T dt = (T)c.dt, cva = (T)c.cva, cva2 = cva * cva;
  const T d = (T)h->marder_d, tau = (T)h->cer_tau * dt;  // pic2d.f90:873, 895
  f.mdx = dt * d / (T)c.dx;
  f.mdy = dt * d / (T)c.dy;
  f.cdx = dt * cva2 * tau / (T)c.dx;
  f.cdy = dt * cva2 * tau / (T)c.dy;
  f.cva2 = cva2;
  f.fc = (T*)h->fc;
  return f;
}

template <class T, bool MIXED>
int do_fieldsolve(pbpic_handle* h) {
  cudaStream_t s = h->stream;
  FieldParams<T> a = field_params<T, MIXED>(h);
  const int rows = h->cfg.ybc == 0 ? h->cfg.my : h->cfg.my + 1;
  const int g = grid_for((int64_t)h->cfg.mx * rows, 256);
  FilterParams<T> fp = filter_params<T, MIXED>(h);
  const int gf = grid_for((int64_t)h->cfg.mx * h->cfg.my, 256);
  if (h->filters) {
    if (MIXED) k_filter_prep<T, long long><<<gf, 256, 0, s>>>(a, fp);
    else k_filter_prep<T, double><<<gf, 256, 0, s>>>(a, fp);
    CKLAUNCH("k_filter_prep");
  }
  k_bhalf<T><<<g, 256, 0, s>>>(a);
  CKLAUNCH("k_bhalf");
  if (MIXED) k_efull<T, long long><<<g, 256, 0, s>>>(a);
  else k_efull<T, double><<<g, 256, 0, s>>>(a);
  CKLAUNCH("k_efull");
  if (h->filters) {
    k_filter_apply<T><<<gf, 256, 0, s>>>(a, fp);
    CKLAUNCH("k_filter_apply");
  }
  k_bhalf<T><<<g, 256, 0, s>>>(a);
  CKLAUNCH("k_bhalf");
  TRY(nodes_and_field_energy<T, MIXED>(h, h->itime + 1));
  h->itime += 1;
  return PBPIC_OK;
}

// The loop body of the reference (pic2d.f90:171-188): push, field solve and,
// when due, the counting sort. The fused sort needs only the push's cell words
// and tile counts and the field solve only the push's current, so after the
// push the field solve runs on a second stream beside the sort and the handle's
// stream waits for it before the next step: each step costs push + the longer
// of the two. (The separate calls pbpic_push, pbpic_fieldsolve and pbpic_sort
// stay in order on the handle's stream.)
template <class T, bool MIXED>
int do_step(pbpic_handle* h, int nsteps, int sort_every) {
  const bool autosort = !(h->cfg.options & PBPIC_OPT_NO_AUTOSORT) && h->fused_ok;
  for (int s = 0; s < nsteps; ++s) {
    h->defer_sort = true;
    const int rp = do_push<T, MIXED>(h);
    h->defer_sort = false;
    TRY(rp);
    const bool due = autosort || (sort_every > 0 && (h->itime + 1) % sort_every == 0);
    if (!(due && h->hist_valid)) {
      TRY((do_fieldsolve<T, MIXED>(h)));
      if (sort_every > 0 && h->itime % sort_every == 0) TRY((do_sort<T, MIXED>(h)));
      continue;
    }
    if (!h->side) {
      CK(cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking));
      CK(cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming));
      CK(cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming));
    }
    CK(cudaEventRecord(h->ev_fork, h->stream));
    CK(cudaStreamWaitEvent(h->side, h->ev_fork, 0));
    const cudaStream_t main = h->stream;
    h->stream = h->side;
    const int rf = do_fieldsolve<T, MIXED>(h);
    h->stream = main;
    const int rs = rf == PBPIC_OK ? do_fused_sort<T, MIXED>(h) : rf;
    CK(cudaEventRecord(h->ev_join, h->side));  // joined on the error paths too
    CK(cudaStreamWaitEvent(h->stream, h->ev_join, 0));
    TRY(rs);
  }
  return PBPIC_OK;
}

template <class T, bool MIXED>
int do_load_fields(pbpic_handle* h, const double* yee6) {
  const int64_t pe = plane_elems(h);
  std::vector<T> tmp((size_t)pe);
  for (int c = 0; c < 6; ++c) {
    for (int64_t k = 0; k < pe; ++k) tmp[k] = (T)yee6[(size_t)c * pe + k];
    CK(cudaMemcpyAsync(h->f[c], tmp.data(), (size_t)pe * sizeof(T), cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
  }
  return nodes_and_field_energy<T, MIXED>(h, h->itime);
}

template <class T, bool MIXED>
int do_store_fields(pbpic_handle* h, double* yee6) {
  const int64_t pe = plane_elems(h);
  std::vector<T> tmp((size_t)pe);
  for (int c = 0; c < 6; ++c) {
    CK(cudaMemcpyAsync(tmp.data(), h->f[c], (size_t)pe * sizeof(T), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    for (int64_t k = 0; k < pe; ++k) yee6[(size_t)c * pe + k] = (double)tmp[k];
  }
  return PBPIC_OK;
}

template <class T, bool MIXED>
int do_store_grid(pbpic_handle* h, double* g8) {
  const size_t ne = (size_t)(h->cfg.mx + 1) * (h->cfg.my + 1) * 8;
  std::vector<T> tmp(ne);
  CK(cudaMemcpyAsync(tmp.data(), h->ng, ne * sizeof(T), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  for (size_t k = 0; k < ne; ++k) g8[k] = (double)tmp[k];
  return PBPIC_OK;
}

int do_store_denjr(pbpic_handle* h, double* j4) {
  const int64_t pe = plane_elems(h);
  std::vector<double> acc((size_t)(4 * pe));
  CK(cudaMemcpyAsync(acc.data(), h->jacc, (size_t)(4 * pe) * 8, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  const pbpic_config& c = h->cfg;
  double sc[4];
  if (h->mixed) {
    sc[0] = c.in0 * (c.dx / c.dt) * FIX_INV;
    sc[1] = c.in0 * (c.dy / c.dt) * FIX_INV;
    sc[2] = c.in0 * c.cva * FIX_INV;
    sc[3] = c.in0 * FIX_INV;
  } else {
    for (int k = 0; k < 4; ++k) sc[k] = c.in0;
  }
  for (int comp = 0; comp < 4; ++comp)
    for (int64_t k = 0; k < pe; ++k) {
      const size_t i = (size_t)comp * pe + k;
      double v;
      if (h->mixed) {
        long long q;
        memcpy(&q, &acc[i], 8);
        v = (double)q;
      } else {
        v = acc[i];
      }
      j4[i] = v * sc[comp];
    }
  return PBPIC_OK;
}

template <class T, bool MIXED, class R>
int do_load_aos(pbpic_handle* h, const RefRec<R>* host, int64_t n) {
  if (n < 0 || n > h->cap) return fail(PBPIC_ECAPACITY, "particle count exceeds the handle's capacity");
  const int b = h->cur;
  if (n > 0) {
    TRY(ensure_staging(h, (size_t)n * sizeof(RefRec<R>)));
    CK(cudaMemcpyAsync(h->staging, host, (size_t)n * sizeof(RefRec<R>), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemsetAsync(h->status, 0, sizeof(int), h->stream));
    k_aos_in<T, R><<<grid_for(n, 256), 256, 0, h->stream>>>((const RefRec<R>*)h->staging, n, h->cfg.mx, h->cfg.my,
                                                              h->cell[b], P<T>(h, b, 0), P<T>(h, b, 1),
                                                              P<T>(h, b, 2), P<T>(h, b, 3), P<T>(h, b, 4),
                                                              h->pid[b], h->status);
    CKLAUNCH("k_aos_in");
    int st = 0;
    CK(cudaMemcpyAsync(&st, h->status, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (st & 8) return fail(PBPIC_EINVAL, "particle record with grid outside 1..mx*my or q not +-1");
  }
  h->n = n;
  h->itime = 0;
  TRY(set_unsorted_tiles(h));
  return kinetic_row<T, MIXED>(h, 0);
}

template <class T, bool MIXED, class R>
int do_store_aos(pbpic_handle* h, RefRec<R>* host, int64_t cap, int64_t* nout) {
  // a pending permutation is read through, not applied: the records come out in cell order either way
  if (nout) *nout = h->n;
  const int64_t n = std::min<int64_t>(cap, h->n);
  if (n <= 0) return PBPIC_OK;
  const int b = h->cur;
  TRY(ensure_staging(h, (size_t)n * sizeof(RefRec<R>)));
  k_aos_out<T, R><<<grid_for(n, 256), 256, 0, h->stream>>>((RefRec<R>*)h->staging, n, h->cfg.my,
                                                             h->lazy ? h->perm : nullptr, h->cell[b],
                                                             P<T>(h, b, 0), P<T>(h, b, 1), P<T>(h, b, 2),
                                                             P<T>(h, b, 3), P<T>(h, b, 4), h->pid[b]);
  CKLAUNCH("k_aos_out");
  CK(cudaMemcpyAsync(host, h->staging, (size_t)n * sizeof(RefRec<R>), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return PBPIC_OK;
}

pic::LoadParams loader_params(const pbpic_handle* h, const pbpic_loader* ld) {
  const pbpic_config& c = h->cfg;
  pic::LoadParams L;
  memset(&L, 0, sizeof(L));
  L.kind = ld->kind;
  L.mx = c.mx;
  L.my = c.my;
  L.dx = c.dx;
  L.dy = c.dy;
  L.ppc = ld->ppc;
  L.npairs = (int64_t)ld->ppc * c.mx * c.my;
  auto u = [](double v) { return v / sqrt(1.0 - v * v); };  // pic2d.f90:383-387
  L.uthe = u(ld->vthe);
  L.uthi = u(ld->vthi);
  L.uthe_perp = L.uthe;
  if (ld->kind == PBPIC_LOAD_WEIBEL) {
    const double a = ld->anisotropy > 0 ? ld->anisotropy : 1.0;
    L.uthe_perp = u(ld->vthe);
    L.uthe = u(ld->vthe / sqrt(a));
  }
  L.udrift_e = u(ld->vdrift_e);
  L.udrift_i = u(ld->vdrift_i);
  L.lambda = ld->lambda;
  L.seed = ld->seed;
  L.uthe_bg = u(ld->vthe_bg);
  L.uthi_bg = u(ld->vthi_bg);
  if (ld->kind == PBPIC_LOAD_DOUBLE_HARRIS) {
    // two sheets of 2 lambda n0 Ly particles each on nb n0 Lx Ly of background;
    // an even count, one half per sheet (pic2d.f90:376-378)
    const double Lx = c.mx * c.dx;
    const double fs = 4.0 * ld->lambda / (4.0 * ld->lambda + ld->nb * Lx);
    L.nsheet = 2 * (int64_t)llround(0.5 * (double)L.npairs * fs);
  }
  if (ld->kind == PBPIC_LOAD_HARRIS) {
    const double Ly = c.my * c.dy;
    const double fs = 2.0 * ld->lambda / (2.0 * ld->lambda + ld->nb * Ly);
    L.nsheet = (int64_t)llround((double)L.npairs * fs);
  }
  return L;
}

int validate_loader(const pbpic_handle* h, const pbpic_loader* ld) {
  if (!ld) return fail(PBPIC_EINVAL, "null loader");
  if (ld->kind < 0 || ld->kind > 4) return fail(PBPIC_EINVAL, "unknown loader kind");
  if (ld->ppc <= 0) return fail(PBPIC_EINVAL, "loader ppc must be positive");
  if (ld->vthe < 0 || ld->vthe >= 1 || ld->vthi < 0 || ld->vthi >= 1) return fail(PBPIC_EINVAL, "thermal speeds must be in [0, c)");
  if (fabs(ld->vdrift_e) >= 1 || fabs(ld->vdrift_i) >= 1) return fail(PBPIC_EINVAL, "drift speeds must be below c");
  if ((ld->kind == PBPIC_LOAD_HARRIS || ld->kind == PBPIC_LOAD_DOUBLE_HARRIS) && (ld->lambda <= 0 || ld->nb < 0))
    return fail(PBPIC_EINVAL, "Harris loader needs lambda > 0 and nb >= 0");
  if (ld->kind == PBPIC_LOAD_DOUBLE_HARRIS && (ld->vthe_bg < 0 || ld->vthe_bg >= 1 || ld->vthi_bg < 0 || ld->vthi_bg >= 1))
    return fail(PBPIC_EINVAL, "background thermal speeds must be in [0, c)");
  (void)h;
  return PBPIC_OK;
}

template <class T, bool MIXED>
int do_init_plasma(pbpic_handle* h, const pbpic_loader* ld) {
  TRY(validate_loader(h, ld));
  pic::LoadParams L = loader_params(h, ld);
  const int64_t n = ld->immobile_ions ? L.npairs : 2 * L.npairs;
  if (n > h->cap) return fail(PBPIC_ECAPACITY, "loader produces more particles than the capacity");
  const int b = h->cur;
  if (L.npairs > 0) {
    k_load<T><<<(unsigned)((L.npairs + 255) / 256), 256, 0, h->stream>>>(
        L, L.npairs, ld->immobile_ions, h->cell[b], P<T>(h, b, 0), P<T>(h, b, 1), P<T>(h, b, 2), P<T>(h, b, 3),
        P<T>(h, b, 4), h->pid[b]);
    CKLAUNCH("k_load");
  }
  h->n = n;
  h->itime = 0;
  h->sorted = false;  // new particles, in load order
  h->hist_valid = false;
  h->lazy = false;
  // initial fields (initfields, pic2d.f90:583-648)
  pic::FieldInit fi;
  fi.kind = ld->kind;
  fi.mx = h->cfg.mx;
  fi.my = h->cfg.my;
  fi.dx = h->cfg.dx;
  fi.dy = h->cfg.dy;
  fi.lambda = ld->lambda;
  fi.psi0 = ld->psi0;
  fi.bguide = ld->bguide;
  fi.b0z = ld->b0z;
  const int64_t pe = plane_elems(h);
  std::vector<double> yee((size_t)(6 * pe), 0.0);
  for (int i = 0; i < fi.mx; ++i)
    for (int j = 0; j <= fi.my; ++j) {
      yee[(size_t)3 * pe + (size_t)i * h->S + j] = pic::init_bx(fi, i, j);
      yee[(size_t)4 * pe + (size_t)i * h->S + j] = pic::init_by(fi, i, j);
      yee[(size_t)5 * pe + (size_t)i * h->S + j] = pic::init_bz(fi, i, j);
    }
  TRY((do_load_fields<T, MIXED>(h, yee.data())));
  TRY((kinetic_row<T, MIXED>(h, 0)));
  TRY((do_sort<T, MIXED>(h)));
  return PBPIC_OK;
}

template <class T, bool MIXED>
int do_gauss(pbpic_handle* h, double* out, int jlo, int jhi) {
  TRY(materialize(h));
  cudaStream_t s = h->stream;
  const int64_t pe = plane_elems(h);
  CK(cudaMemsetAsync(h->rho, 0, (size_t)pe * 8, s));
  CK(cudaMemsetAsync(h->dscalar, 0, 8, s));
  const int b = h->cur;
  if (h->n > 0) {
    k_rho<T><<<grid_for(h->n, 256), 256, 0, s>>>(h->n, h->cfg.mx, h->cfg.my, h->S, h->cfg.ybc, h->cell[b],
                                                  P<T>(h, b, 0), P<T>(h, b, 1), h->rho);
    CKLAUNCH("k_rho");
  }
  const pbpic_config& c = h->cfg;
  k_gauss<T><<<grid_for(pe, 256), 256, 0, s>>>(c.mx, c.my, h->S, c.ybc, jlo, jhi, (const T*)h->f[0], (const T*)h->f[1],
                                                h->rho, 1.0 / c.dx, 1.0 / c.dy, 1.0 / (c.cva * c.cva), c.in0,
                                                h->dscalar);
  CKLAUNCH("k_gauss");
  CK(cudaMemcpyAsync(out, h->dscalar, 8, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return PBPIC_OK;
}

template <class T, bool MIXED>
int do_flux(pbpic_handle* h, double* out) {
  k_flux<T><<<1, 256, 0, h->stream>>>(h->cfg.mx, h->cfg.my, (const T*)h->ng, h->cfg.dx, h->dscalar);
  CKLAUNCH("k_flux");
  CK(cudaMemcpyAsync(out, h->dscalar, 8, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return PBPIC_OK;
}

#define DISPATCH(h, FN, ...) ((h)->mixed ? FN<float, true>(__VA_ARGS__) : FN<double, false>(__VA_ARGS__))

int check_handle(const pbpic_handle* h) {
  if (!h) return fail(PBPIC_EINVAL, "null handle");
  return PBPIC_OK;
}

}  // namespace

// ====================================================================== C ABI
extern "C" {

const char* pbpic_last_error(void) { return g_err.c_str(); }

int pbpic_kernel_launches(int64_t* count) {
  if (!count) return fail(PBPIC_EINVAL, "null argument");
  *count = g_launches.load(std::memory_order_relaxed);
  return PBPIC_OK;
}

int pbpic_create(const pbpic_config* cfg, pbpic_handle** out) {
  if (!cfg || !out) return fail(PBPIC_EINVAL, "null argument");
  *out = nullptr;
  const pbpic_config& c = *cfg;
  if (c.mx < 2 || c.my < 2 || c.mx > 32767 || c.my > 65535)
    return fail(PBPIC_EINVAL, "mx must be in [2, 32767] and my in [2, 65535]");
  if ((int64_t)c.mx * c.my > (1ll << 30)) return fail(PBPIC_EINVAL, "mx*my must not exceed 2^30 cells");
  if (!(c.dx > 0 && c.dy > 0 && c.dt > 0 && c.cva > 0 && c.mime > 0 && c.in0 > 0))
    return fail(PBPIC_EINVAL, "dx, dy, dt, cva, mime and in0 must be positive");
  if (c.ybc != PBPIC_BC_PERIODIC && c.ybc != PBPIC_BC_CONDUCTING) return fail(PBPIC_EINVAL, "unknown ybc");
  if (c.precision != PBPIC_FP64_PLAIN && c.precision != PBPIC_FP32_MIXED)
    return fail(PBPIC_EINVAL, "unknown precision");
  if (c.capacity < 0 || c.capacity > 0x7fffff00ll) return fail(PBPIC_EINVAL, "capacity must be in [0, 2^31)");
  if (c.compat & ~7) return fail(PBPIC_EINVAL, "unknown compat bits");
  if (c.options & ~(PBPIC_OPT_NO_AUTOSORT | PBPIC_OPT_EXACT_FP64)) return fail(PBPIC_EINVAL, "unknown option bits");
  const double cfl = c.cva * c.dt * sqrt(1.0 / (c.dx * c.dx) + 1.0 / (c.dy * c.dy));
  if (!(cfl < 1.0)) return fail(PBPIC_EINVAL, "time step violates the CFL condition c*dt*sqrt(1/dx^2+1/dy^2) < 1");
  if (c.cva * c.dt / std::min(c.dx, c.dy) >= 1.0)
    return fail(PBPIC_EINVAL, "a particle at c would cross more than one cell per step");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return fail(PBPIC_ECUDA, "no CUDA device");
  pbpic_handle* h = new pbpic_handle();
  h->cfg = c;
  h->mixed = c.precision == PBPIC_FP32_MIXED;
  h->tsz = h->mixed ? 4 : 8;
  h->S = c.my + 1;
  h->ncells = c.mx * c.my;
  if (c.tile_rows < 0 || c.tile_rows > 64) {
    delete h;
    return fail(PBPIC_EINVAL, "tile_rows must be in [0, 64]");
  }
  // Default tile: 64 rows; with periodic y at most my-2 rows, so that a tile's
  // window (the adjacent cells) holds distinct cells and the fused sort applies.
  const int ty_default = c.ybc == PBPIC_BC_PERIODIC ? std::max(1, std::min(64, c.my - 2)) : std::min(64, c.my);
  h->TY = c.tile_rows > 0 ? std::min(c.tile_rows, c.my) : ty_default;
  h->tpc = (c.my + h->TY - 1) / h->TY;
  h->ntiles = c.mx * h->tpc;
  h->nb = 3 * (h->TY + 2);
  h->fused_ok = c.mx >= 3 && (c.ybc == PBPIC_BC_CONDUCTING || c.my >= h->TY + 2);
  h->cap = c.capacity;
  const size_t capn = (size_t)std::max<int64_t>(c.capacity, 1);
  const int64_t pe = plane_elems(h);
  int r = PBPIC_OK;
  auto A = [&](auto** p, size_t bytes) {
    if (r == PBPIC_OK) r = dalloc(h, p, bytes);
  };
  for (int b = 0; b < 2; ++b) {
    // particle arrays carry 16 elements of padding: bulk copies read whole 16-byte units
    A(&h->cell[b], (capn + 16) * 4);
    for (int k = 0; k < 5; ++k) A(&h->comp[b][k], (capn + 16) * h->tsz);
    if (c.track_pid) A(&h->pid[b], (capn + 16) * 4);
    A(&h->keys[b], capn * 4);
    A(&h->vals[b], capn * 4);
  }
  for (int k = 0; k < 6; ++k) A(&h->f[k], (size_t)pe * h->tsz);
  A(&h->ng, (size_t)(c.mx + 1) * (c.my + 1) * 8 * h->tsz);
  if (h->mixed) A(&h->cg, (size_t)c.mx * c.my * 24 * h->tsz);
  A(&h->jacc, (size_t)4 * pe * 8);
  A(&h->counts, (size_t)(h->ncells + 1) * 4);
  A(&h->off, (size_t)(h->ncells + 1) * 4);
  A(&h->tile_off, (size_t)(h->ntiles + 1) * 4);
  A(&h->tilecnt, (size_t)h->ntiles * h->nb * 4);
  A(&h->tbase, (size_t)h->ntiles * h->nb * 4);
  A(&h->ke_part, (size_t)std::max(h->ntiles, 148 * 16) * 2 * 8);
  h->tile_cap = h->ntiles;
  h->bin_cap = (int64_t)h->ntiles * h->nb;
  h->nke = 148 * 8;
  h->nfe = grid_for((int64_t)(c.mx + 1) * (c.my + 1), 256, 148 * 8);
  A(&h->fe_part, (size_t)h->nfe * 2 * 8);
  A(&h->status, 16);
  A(&h->rhist, (size_t)radix_hist_ints((int64_t)capn) * 4);
  const int64_t sc = std::max(scan_scratch_ints(radix_hist_ints((int64_t)capn)), scan_scratch_ints(h->ncells + 1));
  A(&h->scan_scratch, (size_t)sc * 4);
  A(&h->rho, (size_t)pe * 8);
  A(&h->dscalar, 64);  // scalars of the diagnostics (up to 4 doubles)
  if (r != PBPIC_OK) {
    pbpic_destroy(h);
    return r;
  }
  for (int k = 0; k < 6; ++k) cudaMemset(h->f[k], 0, (size_t)pe * h->tsz);
  cudaMemset(h->ng, 0, (size_t)(c.mx + 1) * (c.my + 1) * 8 * h->tsz);
  if (h->cg) cudaMemset(h->cg, 0, (size_t)c.mx * c.my * 24 * h->tsz);
  cudaMemset(h->jacc, 0, (size_t)4 * pe * 8);
  cudaMemset(h->counts, 0, (size_t)(h->ncells + 1) * 4);
  cudaMemset(h->off, 0, (size_t)(h->ncells + 1) * 4);
  cudaMemset(h->status, 0, 16);
  if (ensure_hist(h, 64) != PBPIC_OK || set_unsorted_tiles(h) != PBPIC_OK) {
    pbpic_destroy(h);
    return PBPIC_ENOMEM;
  }
  if (cudaDeviceSynchronize() != cudaSuccess) {
    pbpic_destroy(h);
    return fail(PBPIC_ECUDA, "device initialisation failed");
  }
  *out = h;
  return PBPIC_OK;
}

int pbpic_destroy(pbpic_handle* h) {
  if (!h) return PBPIC_OK;
  cudaStreamSynchronize(h->stream);
  if (h->side) {
    cudaStreamSynchronize(h->side);
    cudaStreamDestroy(h->side);
  }
  if (h->ev_fork) cudaEventDestroy(h->ev_fork);
  if (h->ev_join) cudaEventDestroy(h->ev_join);
  for (void* p : h->allocs) cudaFree(p);
  delete h;
  return PBPIC_OK;
}

int pbpic_set_stream(pbpic_handle* h, void* stream) {
  TRY(check_handle(h));
  h->stream = (cudaStream_t)stream;
  return PBPIC_OK;
}

int pbpic_get_config(const pbpic_handle* h, pbpic_config* out) {
  TRY(check_handle(h));
  if (!out) return fail(PBPIC_EINVAL, "null argument");
  *out = h->cfg;
  return PBPIC_OK;
}

int pbpic_loader_count(const pbpic_handle* h, const pbpic_loader* ld, int64_t* n) {
  TRY(check_handle(h));
  TRY(validate_loader(h, ld));
  if (!n) return fail(PBPIC_EINVAL, "null argument");
  const int64_t pairs = (int64_t)ld->ppc * h->cfg.mx * h->cfg.my;
  *n = ld->immobile_ions ? pairs : 2 * pairs;
  return PBPIC_OK;
}

int pbpic_init_plasma(pbpic_handle* h, const pbpic_loader* ld) {
  TRY(check_handle(h));
  return DISPATCH(h, do_init_plasma, h, ld);
}

int pbpic_load_particles_f32(pbpic_handle* h, const pbpic_particle_f32* p, int64_t n) {
  TRY(check_handle(h));
  if (!p && n > 0) return fail(PBPIC_EINVAL, "null particles");
  const RefRec<float>* r = reinterpret_cast<const RefRec<float>*>(p);
  return h->mixed ? do_load_aos<float, true, float>(h, r, n) : do_load_aos<double, false, float>(h, r, n);
}

int pbpic_load_particles_f64(pbpic_handle* h, const pbpic_particle_f64* p, int64_t n) {
  TRY(check_handle(h));
  if (!p && n > 0) return fail(PBPIC_EINVAL, "null particles");
  const RefRec<double>* r = reinterpret_cast<const RefRec<double>*>(p);
  return h->mixed ? do_load_aos<float, true, double>(h, r, n) : do_load_aos<double, false, double>(h, r, n);
}

int pbpic_store_particles_f32(pbpic_handle* h, pbpic_particle_f32* p, int64_t cap, int64_t* n) {
  TRY(check_handle(h));
  if (!p && cap > 0) return fail(PBPIC_EINVAL, "null particles");
  RefRec<float>* r = reinterpret_cast<RefRec<float>*>(p);
  return h->mixed ? do_store_aos<float, true, float>(h, r, cap, n) : do_store_aos<double, false, float>(h, r, cap, n);
}

int pbpic_store_particles_f64(pbpic_handle* h, pbpic_particle_f64* p, int64_t cap, int64_t* n) {
  TRY(check_handle(h));
  if (!p && cap > 0) return fail(PBPIC_EINVAL, "null particles");
  RefRec<double>* r = reinterpret_cast<RefRec<double>*>(p);
  return h->mixed ? do_store_aos<float, true, double>(h, r, cap, n)
                  : do_store_aos<double, false, double>(h, r, cap, n);
}

int pbpic_load_particles_soa_f64(pbpic_handle* h, int64_t n, const int32_t* grid, const int32_t* q,
                                 const double* dx, const double* dy, const double* ux, const double* uy,
                                 const double* uz, const int32_t* pid) {
  TRY(check_handle(h));
  if (n > 0 && !(grid && q && dx && dy && ux && uy && uz)) return fail(PBPIC_EINVAL, "null array");
  std::vector<pbpic_particle_f64> tmp((size_t)std::max<int64_t>(n, 0));
  for (int64_t i = 0; i < n; ++i)
    tmp[i] = pbpic_particle_f64{dx[i], dy[i], ux[i], uy[i], uz[i], grid[i], q[i], pid ? pid[i] : 0, 0};
  return pbpic_load_particles_f64(h, tmp.data(), n);
}

int pbpic_store_particles_soa_f64(pbpic_handle* h, int64_t cap, int64_t* n, int32_t* grid, int32_t* q, double* dx,
                                  double* dy, double* ux, double* uy, double* uz, int32_t* pid) {
  TRY(check_handle(h));
  int64_t m = std::min<int64_t>(cap, h->n);
  std::vector<pbpic_particle_f64> tmp((size_t)std::max<int64_t>(m, 0));
  TRY(pbpic_store_particles_f64(h, tmp.data(), m, nullptr));
  if (n) *n = h->n;
  for (int64_t i = 0; i < m; ++i) {
    if (grid) grid[i] = tmp[i].grid;
    if (q) q[i] = tmp[i].q;
    if (dx) dx[i] = tmp[i].dx;
    if (dy) dy[i] = tmp[i].dy;
    if (ux) ux[i] = tmp[i].ux;
    if (uy) uy[i] = tmp[i].uy;
    if (uz) uz[i] = tmp[i].uz;
    if (pid) pid[i] = tmp[i].pid;
  }
  return PBPIC_OK;
}

int pbpic_num_particles(const pbpic_handle* h, int64_t* n) {
  TRY(check_handle(h));
  if (!n) return fail(PBPIC_EINVAL, "null argument");
  *n = h->n;
  return PBPIC_OK;
}

int pbpic_load_fields_f64(pbpic_handle* h, const double* yee6) {
  TRY(check_handle(h));
  if (!yee6) return fail(PBPIC_EINVAL, "null fields");
  return DISPATCH(h, do_load_fields, h, yee6);
}

int pbpic_store_fields_f64(pbpic_handle* h, double* yee6) {
  TRY(check_handle(h));
  if (!yee6) return fail(PBPIC_EINVAL, "null fields");
  return DISPATCH(h, do_store_fields, h, yee6);
}

int pbpic_store_emfgrid_f64(pbpic_handle* h, double* grid8) {
  TRY(check_handle(h));
  if (!grid8) return fail(PBPIC_EINVAL, "null buffer");
  return DISPATCH(h, do_store_grid, h, grid8);
}

int pbpic_store_denjr_f64(pbpic_handle* h, double* j4) {
  TRY(check_handle(h));
  if (!j4) return fail(PBPIC_EINVAL, "null buffer");
  return do_store_denjr(h, j4);
}

int pbpic_push(pbpic_handle* h) {
  TRY(check_handle(h));
  return DISPATCH(h, do_push, h);
}

int pbpic_fieldsolve(pbpic_handle* h) {
  TRY(check_handle(h));
  return DISPATCH(h, do_fieldsolve, h);
}

int pbpic_sort(pbpic_handle* h) {
  TRY(check_handle(h));
  return DISPATCH(h, do_sort, h);
}

int pbpic_step(pbpic_handle* h, int32_t nsteps, int32_t sort_every) {
  TRY(check_handle(h));
  if (nsteps < 0 || sort_every < 0) return fail(PBPIC_EINVAL, "nsteps and sort_every must be >= 0");
  return DISPATCH(h, do_step, h, nsteps, sort_every);
}

int pbpic_energy_spectra(pbpic_handle* h, double de_electron, double de_ion, int32_t nbins, int64_t* counts) {
  TRY(check_handle(h));
  if (!counts) return fail(PBPIC_EINVAL, "null buffer");
  if (!(de_electron > 0 && de_ion > 0) || nbins < 1 || nbins > 8192)
    return fail(PBPIC_EINVAL, "spectra need positive bin widths and 1..8192 bins");
  TRY(materialize(h));
  const size_t bytes = (size_t)2 * nbins * 8;
  TRY(ensure_staging(h, bytes));
  cudaStream_t s = h->stream;
  CK(cudaMemsetAsync(h->staging, 0, bytes, s));
  const int b = h->cur;
  if (h->n > 0) {
    const int g = grid_for(h->n, 256, 148 * 4);
    if (h->mixed)
      k_spectra<float><<<g, 256, (size_t)2 * nbins * 4, s>>>(h->n, h->cell[b], P<float>(h, b, 2), P<float>(h, b, 3),
                                                            P<float>(h, b, 4), h->cfg.mime, de_electron, de_ion, nbins,
                                                            (unsigned long long*)h->staging);
    else
      k_spectra<double><<<g, 256, (size_t)2 * nbins * 4, s>>>(h->n, h->cell[b], P<double>(h, b, 2),
                                                             P<double>(h, b, 3), P<double>(h, b, 4), h->cfg.mime,
                                                             de_electron, de_ion, nbins,
                                                             (unsigned long long*)h->staging);
    CKLAUNCH("k_spectra");
  }
  CK(cudaMemcpyAsync(counts, h->staging, bytes, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return PBPIC_OK;
}

int pbpic_field_cuts(pbpic_handle* h, const int32_t* rows, int32_t nrows, const int32_t* cols, int32_t ncols,
                     double* out) {
  TRY(check_handle(h));
  const pbpic_config& c = h->cfg;
  if (nrows < 0 || ncols < 0 || (nrows && !rows) || (ncols && !cols) || !out)
    return fail(PBPIC_EINVAL, "null or negative cut arguments");
  for (int k = 0; k < nrows; ++k)
    if (rows[k] < 0 || rows[k] > c.my) return fail(PBPIC_EINVAL, "cut row outside 0..my");
  for (int k = 0; k < ncols; ++k)
    if (cols[k] < 0 || cols[k] > c.mx) return fail(PBPIC_EINVAL, "cut column outside 0..mx");
  const int64_t nv = ((int64_t)nrows * c.mx + (int64_t)ncols * c.my) * 6;
  const size_t ib = (size_t)(nrows + ncols) * 4, vb = (size_t)nv * 8;
  TRY(ensure_staging(h, ib + vb + 16));
  cudaStream_t s = h->stream;
  int32_t* didx = (int32_t*)h->staging;
  double* dval = (double*)((char*)h->staging + ((ib + 15) & ~(size_t)15));
  if (nrows) CK(cudaMemcpyAsync(didx, rows, (size_t)nrows * 4, cudaMemcpyHostToDevice, s));
  if (ncols) CK(cudaMemcpyAsync(didx + nrows, cols, (size_t)ncols * 4, cudaMemcpyHostToDevice, s));
  if (nv > 0) {
    const int g = grid_for(nv / 6, 256);
    if (h->mixed)
      k_field_cuts<float><<<g, 256, 0, s>>>(c.mx, c.my, (const float*)h->ng, didx, nrows, didx + nrows, ncols, dval);
    else
      k_field_cuts<double><<<g, 256, 0, s>>>(c.mx, c.my, (const double*)h->ng, didx, nrows, didx + nrows, ncols, dval);
    CKLAUNCH("k_field_cuts");
    CK(cudaMemcpyAsync(out, dval, vb, cudaMemcpyDeviceToHost, s));
  }
  CK(cudaStreamSynchronize(s));
  return PBPIC_OK;
}

int pbpic_set_field_filters(pbpic_handle* h, int32_t flags, double marder_d, double cerenkov_tau) {
  TRY(check_handle(h));
  if (flags & ~(PBPIC_FILTER_MARDER | PBPIC_FILTER_CERENKOV)) return fail(PBPIC_EINVAL, "unknown filter bits");
  if (flags && h->cfg.ybc != PBPIC_BC_PERIODIC)
    return fail(PBPIC_EINVAL, "the field filters are defined for periodic y only, as in the reference");
  if (flags && !h->fc)
    TRY(dalloc(h, &h->fc, (size_t)5 * h->cfg.mx * h->cfg.my * h->tsz));
  h->filters = flags;
  h->marder_d = marder_d > 0 ? marder_d : 0.001;      // pic2d.f90:873
  h->cer_tau = cerenkov_tau > 0 ? cerenkov_tau : 0.125;  // pic2d.f90:895
  return PBPIC_OK;
}

int pbpic_synchronize(pbpic_handle* h) {
  TRY(check_handle(h));
  CK(cudaStreamSynchronize(h->stream));
  return PBPIC_OK;
}

int pbpic_energies(pbpic_handle* h, double out[4]) {
  TRY(check_handle(h));
  if (!out) return fail(PBPIC_EINVAL, "null argument");
  CK(cudaMemcpyAsync(out, h->hist + (size_t)h->itime * 4, 4 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return PBPIC_OK;
}

int pbpic_energy_history(pbpic_handle* h, double* out, int32_t max_rows, int32_t* n_rows) {
  TRY(check_handle(h));
  const int rows = std::min(max_rows, h->itime + 1);
  if (n_rows) *n_rows = h->itime + 1;
  if (rows > 0) {
    if (!out) return fail(PBPIC_EINVAL, "null buffer");
    CK(cudaMemcpyAsync(out, h->hist, (size_t)rows * 4 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
  }
  return PBPIC_OK;
}

int pbpic_time_step(const pbpic_handle* h, int32_t* itime) {
  TRY(check_handle(h));
  if (!itime) return fail(PBPIC_EINVAL, "null argument");
  *itime = h->itime;
  return PBPIC_OK;
}

int pbpic_cell_counts(pbpic_handle* h, int32_t* counts) {
  TRY(check_handle(h));
  if (!counts) return fail(PBPIC_EINVAL, "null buffer");
  CK(cudaMemcpyAsync(counts, h->counts, (size_t)h->ncells * 4, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return PBPIC_OK;
}

int pbpic_gauss_residual(pbpic_handle* h, double* out) {
  TRY(check_handle(h));
  if (!out) return fail(PBPIC_EINVAL, "null argument");
  return DISPATCH(h, do_gauss, h, out, 0, h->cfg.my);
}

int pbpic_gauss_residual_rows(pbpic_handle* h, int32_t y_lo, int32_t y_hi, double* out) {
  TRY(check_handle(h));
  if (!out) return fail(PBPIC_EINVAL, "null argument");
  if (y_lo < 0 || y_hi < y_lo || y_hi > h->cfg.my) return fail(PBPIC_EINVAL, "rows outside 0..my");
  return DISPATCH(h, do_gauss, h, out, (int)y_lo, (int)y_hi);
}

int pbpic_reconnected_flux(pbpic_handle* h, double* out) {
  TRY(check_handle(h));
  if (!out) return fail(PBPIC_EINVAL, "null argument");
  return DISPATCH(h, do_flux, h, out);
}

int pbpic_status(pbpic_handle* h, int32_t* bits) {
  TRY(check_handle(h));
  if (!bits) return fail(PBPIC_EINVAL, "null argument");
  int st = 0;
  CK(cudaMemcpyAsync(&st, h->status, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemsetAsync(h->status, 0, sizeof(int), h->stream));
  CK(cudaStreamSynchronize(h->stream));
  *bits = st;
  return PBPIC_OK;
}

int pbpic_counting_sort_keys(const int32_t* keys_dev, int64_t n, int32_t ncells, int32_t* perm_dev,
                             int32_t* counts_dev, void* stream) {
  if (n < 0 || n > 0x7fffff00ll || ncells <= 0) return fail(PBPIC_EINVAL, "bad n or ncells");
  if (n > 0 && (!keys_dev || !perm_dev)) return fail(PBPIC_EINVAL, "null device buffer");
  if (!counts_dev) return fail(PBPIC_EINVAL, "null counts buffer");
  cudaStream_t s = (cudaStream_t)stream;
  const size_t nn = (size_t)std::max<int64_t>(n, 1);
  const int64_t rh = radix_hist_ints((int64_t)nn);
  const int64_t sc = std::max(scan_scratch_ints(rh), (int64_t)16);
  const size_t bytes = nn * 4 * 4 + (size_t)rh * 4 + (size_t)sc * 4 + 16;
  char* buf = nullptr;
  CK(cudaMallocAsync((void**)&buf, bytes, s));
  int32_t* k0 = (int32_t*)buf;
  int32_t* k1 = k0 + nn;
  int32_t* v0 = k1 + nn;
  int32_t* v1 = v0 + nn;
  int32_t* rhist = v1 + nn;
  int32_t* scr = rhist + rh;
  int* status = (int*)(scr + sc);
  int rc = PBPIC_OK;
  int st = 0;
  do {
    if (cudaMemsetAsync(counts_dev, 0, (size_t)ncells * 4, s) != cudaSuccess ||
        cudaMemsetAsync(status, 0, 4, s) != cudaSuccess) {
      rc = fail(PBPIC_ECUDA, "cudaMemsetAsync failed");
      break;
    }
    if (n == 0) break;
    k_key_hist<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(keys_dev, n, ncells, counts_dev, status);
    g_launches.fetch_add(1, std::memory_order_relaxed);
    if (cudaGetLastError() != cudaSuccess) {
      rc = fail(PBPIC_ECUDA, "k_key_hist launch failed");
      break;
    }
    if (cudaMemcpyAsync(k0, keys_dev, (size_t)n * 4, cudaMemcpyDeviceToDevice, s) != cudaSuccess) {
      rc = fail(PBPIC_ECUDA, "key copy failed");
      break;
    }
    int32_t* perm = nullptr;
    rc = radix_sort(s, n, ncells, k0, k1, v0, v1, rhist, scr, &perm);
    if (rc != PBPIC_OK) break;
    if (cudaMemcpyAsync(perm_dev, perm, (size_t)n * 4, cudaMemcpyDeviceToDevice, s) != cudaSuccess) {
      rc = fail(PBPIC_ECUDA, "permutation copy failed");
      break;
    }
  } while (0);
  if (cudaMemcpyAsync(&st, status, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess && rc == PBPIC_OK)
    rc = fail(PBPIC_ECUDA, "status copy failed");
  cudaFreeAsync(buf, s);
  if (cudaStreamSynchronize(s) != cudaSuccess && rc == PBPIC_OK) rc = fail(PBPIC_ECUDA, "stream synchronize failed");
  if (rc == PBPIC_OK && (st & 8)) rc = fail(PBPIC_EINVAL, "key outside [0, ncells)");
  return rc;
}

}  // extern "C"

// ============================================================================
// pbpic_counting_sort_keys_static: the stateless counting sort without any
// device allocation, for callers that cannot call cudaMalloc: a host code whose
// device memory is owned up front by another allocator (for example a
// framework's caching allocator that has reserved the GPU), or a time loop that
// must not trigger the device-wide synchronisation of an allocation.
//
// Its scratch is the file-scope array below, sized for
// PBPIC_STATIC_SORT_MAX_KEYS keys. Every GPU that loads this library holds the
// array until the process exits. Host code cannot use the array's name as a
// device address, so the first call on each device (with that device current)
// looks the address up with cudaGetSymbolAddress and keeps it; make that first
// call before any stream capture. Each call copies the key-range status back
// to the host and waits for its stream, so it returns with the sort finished.
// All calls share the array and it keeps the
// last call's contents: the only word that must start at zero (the key-range
// status) is cleared on every call, and calls that overlap on the GPU (on
// different streams or host threads) race on the array.
// ============================================================================
namespace {

constexpr int64_t kStaticKeys = PBPIC_STATIC_SORT_MAX_KEYS;
constexpr int64_t kStaticHist = 256 * ((kStaticKeys + RTILE - 1) / RTILE);
constexpr int64_t kStaticScan = 1024;  // chunk totals of every scan level of the histogram (needs 19)
constexpr int64_t kStaticWords = 4 * kStaticKeys + kStaticHist + kStaticScan + 64;

static __device__ __align__(256) int32_t g_static_sort_scratch[kStaticWords];

std::mutex g_static_mu;
int32_t* g_static_addr[1024] = {};  // device address of the array, per device ordinal

int static_sort_scratch(int32_t** out) {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 1024) return fail(PBPIC_EINVAL, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_static_mu);
  if (!g_static_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_static_sort_scratch);
    if (e != cudaSuccess || !p)
      return fail(PBPIC_ECUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    g_static_addr[dev] = (int32_t*)p;
  }
  *out = g_static_addr[dev];
  return PBPIC_OK;
}

}  // namespace

extern "C" int pbpic_counting_sort_keys_static(const int32_t* keys_dev, int64_t n, int32_t ncells,
                                               int32_t* perm_dev, int32_t* counts_dev, void* stream) {
  if (n < 0 || ncells <= 0) return fail(PBPIC_EINVAL, "bad n or ncells");
  if (n > kStaticKeys)
    return fail(PBPIC_ECAPACITY, "n = " + std::to_string(n) + " exceeds the static scratch limit of " +
                                     std::to_string(kStaticKeys) + " keys (PBPIC_STATIC_SORT_MAX_KEYS)");
  if (n > 0 && (!keys_dev || !perm_dev)) return fail(PBPIC_EINVAL, "null device buffer");
  if (!counts_dev) return fail(PBPIC_EINVAL, "null counts buffer");
  if (scan_scratch_ints(radix_hist_ints(std::max<int64_t>(n, 1))) > kStaticScan)
    return fail(PBPIC_EINVAL, "static scan scratch too small");
  int32_t* base = nullptr;
  TRY(static_sort_scratch(&base));
  cudaStream_t s = (cudaStream_t)stream;
  int32_t* k0 = base;
  int32_t* k1 = k0 + kStaticKeys;
  int32_t* v0 = k1 + kStaticKeys;
  int32_t* v1 = v0 + kStaticKeys;
  int32_t* rhist = v1 + kStaticKeys;
  int32_t* scr = rhist + kStaticHist;
  int* status = (int*)(scr + kStaticScan);
  CK(cudaMemsetAsync(counts_dev, 0, (size_t)ncells * 4, s));
  CK(cudaMemsetAsync(status, 0, sizeof(int), s));
  if (n > 0) {
    k_key_hist<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(keys_dev, n, ncells, counts_dev, status);
    CKLAUNCH("k_key_hist");
    CK(cudaMemcpyAsync(k0, keys_dev, (size_t)n * 4, cudaMemcpyDeviceToDevice, s));
    int32_t* perm = nullptr;
    TRY(radix_sort(s, n, ncells, k0, k1, v0, v1, rhist, scr, &perm));
    CK(cudaMemcpyAsync(perm_dev, perm, (size_t)n * 4, cudaMemcpyDeviceToDevice, s));
  }
  int st = 0;
  CK(cudaMemcpyAsync(&st, status, sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (st & 8) return fail(PBPIC_EINVAL, "key outside [0, ncells)");
  return PBPIC_OK;
}

// ============================================================== batched form
// Many independent FP32 domains advanced together. Every domain is an
// ordinary handle (its own particles, fields and tables); a batched step runs
// each phase once for all domains:
//   k_batch_begin          zero the current accumulators, reset counters
//   k_push_batched         persistent blocks over the (domain, tile) table
//   k_fused_counts_batched, k_scan_batched, k_fused_base_batched,
//   k_fused_perm_batched (persistent), k_tile_off_batched
//                          the fused counting sort of every domain
//   k_bhalf/k_efull/k_bhalf/k_nodes_batched, k_cell_records_batched, k_energy_rows_batched
// Two consecutive steps (the particle buffers swap each step) are captured
// once in a CUDA graph and replayed. A domain stepped here goes through the
// same arithmetic as pbpic_step(h, n, 1) with the same tile rows and
// particles per thread, so its state is bit-identical to that run.
struct pbpic_batch {
  std::vector<pbpic_handle*> dom;
  cudaStream_t stream = nullptr;
  int groups = PBPIC_PUSH_HALVES;  // particles per thread / 4 in the push
  bool compat = true;              // some domain sets a compat switch (generic push)
  int64_t launches_per_pair = 0;
  cudaGraphExec_t graph = nullptr;
  // descriptor tables: host copies (kept alive for the asynchronous uploads) and device arrays
  std::vector<PushParams<float>> h_push;       // [2][D]: [0] the domains' current buffers, [1] swapped
  std::vector<ScatterParams<float>> h_scat;    // [2][D]
  std::vector<FusedSortParams> h_fsort;
  std::vector<FieldParams<float>> h_field;
  std::vector<TileOffDesc> h_toff;
  std::vector<BatchDomain> h_dom;
  std::vector<EnergyRow> h_erow;
  std::vector<int2> h_tiles;
  PushParams<float>* d_push = nullptr;
  ScatterParams<float>* d_scat = nullptr;
  FusedSortParams* d_fsort = nullptr;
  FieldParams<float>* d_field = nullptr;
  TileOffDesc* d_toff = nullptr;
  BatchDomain* d_dom = nullptr;
  EnergyRow* d_erow = nullptr;
  int2* d_tiles = nullptr;
  int* d_counters = nullptr;  // [0] push, [1] scatter, [2] step index
  int ntiles = 0, push_blocks = 0, scatter_blocks = 0;
  size_t push_smem = 0;
  int gx_zero = 1, gx_cells = 1, gx_bins = 1, gx_tiles = 1, gx_field = 1, gx_nodes = 1;
};

namespace {

void dfree(pbpic_handle* h, void* p) {
  if (!p) return;
  cudaFree(p);
  auto it = std::find(h->allocs.begin(), h->allocs.end(), p);
  if (it != h->allocs.end()) h->allocs.erase(it);
}

// Tile rows of a domain: ty, or the default for ty <= 0, capped so that the
// fused counting sort applies (with periodic y a tile's window must hold
// distinct rows).
int batch_tile_rows(const pbpic_handle* h, int ty) {
  const pbpic_config& c = h->cfg;
  const int cap = c.ybc == PBPIC_BC_PERIODIC ? std::max(1, std::min(64, c.my - 2)) : std::min(64, c.my);
  return ty > 0 ? std::min(ty, cap) : cap;
}

// Change a handle's tile rows, growing its per-tile arrays if needed, and
// recompute its tile ranges (from the cell offsets when sorted).
int retile(pbpic_handle* h, int ty) {
  if (ty == h->TY) return PBPIC_OK;
  TRY(materialize(h));
  const pbpic_config& c = h->cfg;
  const int tpc = (c.my + ty - 1) / ty;
  const int ntiles = c.mx * tpc;
  const int nb = 3 * (ty + 2);
  CK(cudaStreamSynchronize(h->stream));
  if (ntiles > h->tile_cap) {
    dfree(h, h->tile_off);
    dfree(h, h->ke_part);
    h->tile_off = nullptr;
    h->ke_part = nullptr;
    TRY(dalloc(h, &h->tile_off, (size_t)(ntiles + 1) * 4));
    TRY(dalloc(h, &h->ke_part, (size_t)std::max(ntiles, 148 * 16) * 2 * 8));
    h->tile_cap = ntiles;
  }
  if ((int64_t)ntiles * nb > h->bin_cap) {
    dfree(h, h->tilecnt);
    dfree(h, h->tbase);
    h->tilecnt = nullptr;
    h->tbase = nullptr;
    TRY(dalloc(h, &h->tilecnt, (size_t)ntiles * nb * 4));
    TRY(dalloc(h, &h->tbase, (size_t)ntiles * nb * 4));
    h->bin_cap = (int64_t)ntiles * nb;
  }
  h->TY = ty;
  h->tpc = tpc;
  h->ntiles = ntiles;
  h->nb = nb;
  h->fused_ok = c.mx >= 3 && (c.ybc == PBPIC_BC_CONDUCTING || c.my >= ty + 2);
  h->hist_valid = false;
  if (h->sorted) {
    k_tile_off<<<grid_for(h->ntiles + 1, 256, 1 << 20), 256, 0, h->stream>>>(h->off, h->ntiles, h->tpc, h->TY,
                                                                            c.my, (int32_t)h->n, h->tile_off);
    CKLAUNCH("k_tile_off");
  } else {
    TRY(set_unsorted_tiles(h));
  }
  return PBPIC_OK;
}

void drop_graph(pbpic_batch* b) {
  if (b->graph) cudaGraphExecDestroy(b->graph);
  b->graph = nullptr;
}

template <class X>
int upload(pbpic_batch* b, X* dst, const std::vector<X>& src) {
  if (src.empty()) return PBPIC_OK;
  CK(cudaMemcpyAsync(dst, src.data(), src.size() * sizeof(X), cudaMemcpyHostToDevice, b->stream));
  return PBPIC_OK;
}

// Build the (domain, tile) table, largest expected tiles first (rows x mean
// particles per cell), and the launch shapes. Called when tile rows change.
int batch_layout(pbpic_batch* b) {
  const int D = (int)b->dom.size();
  struct Item {
    double cost;
    int d, t;
  };
  std::vector<Item> items;
  size_t smem = 0;
  int64_t maxcells = 1, maxbins = 1, maxtiles = 1, maxfield = 1, maxacc = 1;
  int maxnfe = 1;
  for (int d = 0; d < D; ++d) {
    const pbpic_handle* h = b->dom[d];
    const double ppc = (double)h->n / (double)h->ncells;
    for (int t = 0; t < h->ntiles; ++t) {
      const int y0 = (t % h->tpc) * h->TY;
      const int rows = std::min(h->TY, h->cfg.my - y0);
      items.push_back({rows * ppc, d, t});
    }
    smem = std::max(smem, push_smem_bytes(h->TY, true));
    maxcells = std::max<int64_t>(maxcells, (int64_t)h->ncells + 1);
    maxbins = std::max<int64_t>(maxbins, (int64_t)h->ntiles * h->nb);
    maxtiles = std::max<int64_t>(maxtiles, (int64_t)h->ntiles + 1);
    const int rows = h->cfg.ybc == 0 ? h->cfg.my : h->cfg.my + 1;
    maxfield = std::max<int64_t>(maxfield, (int64_t)h->cfg.mx * rows);
    maxacc = std::max<int64_t>(maxacc, 2 * plane_elems(h));  // 16-byte stores of 4 planes
    maxnfe = std::max(maxnfe, h->nfe);
  }
  std::stable_sort(items.begin(), items.end(), [](const Item& x, const Item& y) { return x.cost > y.cost; });
  if (items.size() > (size_t)0x7fffffff) return fail(PBPIC_EINVAL, "too many tiles in the batch");
  b->h_tiles.resize(items.size());
  for (size_t k = 0; k < items.size(); ++k) b->h_tiles[k] = make_int2(items[k].d, items[k].t);
  b->ntiles = (int)items.size();
  b->push_smem = smem;
  if (b->d_tiles) cudaFree(b->d_tiles);
  b->d_tiles = nullptr;
  CK(cudaMalloc(&b->d_tiles, std::max<size_t>(1, items.size()) * sizeof(int2)));
  TRY(upload(b, b->d_tiles, b->h_tiles));
  int dev = 0, sms = 148;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  int per_sm = 1;
  b->compat = false;
  for (pbpic_handle* h : b->dom) b->compat |= h->cfg.compat != 0;
  const void* fn = b->groups == 1 ? (b->compat ? (const void*)k_push_batched<float, true, true, 1, true, true>
                                               : (const void*)k_push_batched<float, true, true, 1, false, true>)
                                  : (b->compat ? (const void*)k_push_batched<float, true, true, 2, true, true>
                                               : (const void*)k_push_batched<float, true, true, 2, false, true>);
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, PushThreads<float>::value, smem));
  b->push_blocks = std::max(1, std::min(b->ntiles, sms * std::max(1, per_sm)));
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fused_perm_batched<float>, 256, 0));
  b->scatter_blocks = std::max(1, std::min(b->ntiles, sms * std::max(1, per_sm)));
  b->gx_zero = grid_for(maxacc, 256, 1024);
  b->gx_cells = grid_for(maxcells, 256);
  b->gx_bins = grid_for(maxbins, 256);
  b->gx_tiles = grid_for(maxtiles, 256, 1 << 16);
  b->gx_field = grid_for(maxfield, 256);
  b->gx_nodes = maxnfe;
  (void)D;
  return PBPIC_OK;
}

// Descriptor tables from the domains' current state (buffers, histories).
int batch_descriptors(pbpic_batch* b) {
  const int D = (int)b->dom.size();
  b->h_push.resize(2 * D);
  b->h_scat.resize(2 * D);
  b->h_fsort.resize(D);
  b->h_field.resize(D);
  b->h_toff.resize(D);
  b->h_dom.resize(D);
  b->h_erow.resize(D);
  for (int d = 0; d < D; ++d) {
    pbpic_handle* h = b->dom[d];
    const int cur0 = h->cur;
    for (int par = 0; par < 2; ++par) {  // step of parity par: push i -> o through perm, then rank o
      h->cur = par == 0 ? cur0 : 1 - cur0;
      PushParams<float>& pp = b->h_push[par * D + d];
      pp = push_params<float, true>(h);
      if (!pp.cell_off) return fail(PBPIC_EINVAL, "batched push: no cell offsets");
      const int i = h->cur, o = 1 - i;
      pp.src = h->perm;
      pp.cell_o = h->cell[o];
      pp.dx_o = P<float>(h, o, 0);
      pp.dy_o = P<float>(h, o, 1);
      pp.ux_o = P<float>(h, o, 2);
      pp.uy_o = P<float>(h, o, 3);
      pp.uz_o = P<float>(h, o, 4);
      pp.pid_i = h->pid[i];
      pp.pid_o = h->pid[o];
      ScatterParams<float>& sp = b->h_scat[par * D + d];
      sp = ScatterParams<float>{};
      sp.mx = h->cfg.mx;
      sp.my = h->cfg.my;
      sp.ybc = h->cfg.ybc;
      sp.ty = h->TY;
      sp.tpc = h->tpc;
      sp.nb = h->nb;
      sp.tile_off = h->tile_off;
      sp.base = h->tbase;
      sp.ci = h->cell[o];
      sp.perm = h->perm;
    }
    h->cur = cur0;
    FusedSortParams& f = b->h_fsort[d];
    f.mx = h->cfg.mx;
    f.my = h->cfg.my;
    f.ybc = h->cfg.ybc;
    f.ty = h->TY;
    f.tpc = h->tpc;
    f.ntiles = h->ntiles;
    f.nb = h->nb;
    f.tilecnt = h->tilecnt;
    f.counts = h->counts;
    f.off = h->off;
    f.base = h->tbase;
    b->h_field[d] = field_params<float, true>(h);
    b->h_field[d].nblk = h->nfe;
    TileOffDesc& t = b->h_toff[d];
    t.off = h->off;
    t.ntiles = h->ntiles;
    t.tpc = h->tpc;
    t.ty = h->TY;
    t.my = h->cfg.my;
    t.end = (int32_t)h->n;
    t.tile_off = h->tile_off;
    BatchDomain& bd = b->h_dom[d];
    bd.jacc = (long long*)h->jacc;
    bd.nacc = 4 * plane_elems(h);
    bd.counts = h->counts;
    bd.off = h->off;
    bd.ncounts = h->ncells + 1;
    EnergyRow& e = b->h_erow[d];
    e.ke_part = h->ke_part;
    e.nke = h->ntiles;
    e.fe_part = h->fe_part;
    e.nfe = h->nfe;
    e.fe_scale = fe_scale(h->cfg);
    e.fb_scale = fb_scale(h->cfg);
    e.rows = h->hist + (size_t)(h->itime + 1) * 4;
  }
  TRY(upload(b, b->d_push, b->h_push));
  TRY(upload(b, b->d_scat, b->h_scat));
  TRY(upload(b, b->d_fsort, b->h_fsort));
  TRY(upload(b, b->d_field, b->h_field));
  TRY(upload(b, b->d_toff, b->h_toff));
  TRY(upload(b, b->d_dom, b->h_dom));
  TRY(upload(b, b->d_erow, b->h_erow));
  return PBPIC_OK;
}

// One batched step on descriptor set `par` (0: buffers as uploaded, 1: swapped).
int batch_enqueue_step(pbpic_batch* b, int par) {
  const int D = (int)b->dom.size();
  cudaStream_t s = b->stream;
  int* ctr = b->d_counters;
  k_batch_begin<<<dim3(b->gx_zero, D), 256, 0, s>>>(b->d_dom, ctr, ctr + 2);
  CKLAUNCH("k_batch_begin");
  const PushParams<float>* pp = b->d_push + (size_t)par * D;
  const unsigned nt = PushThreads<float>::value;
  if (b->groups == 1 && b->compat)
    k_push_batched<float, true, true, 1, true, true><<<b->push_blocks, nt, b->push_smem, s>>>(pp, b->d_tiles, b->ntiles, ctr);
  else if (b->groups == 1)
    k_push_batched<float, true, true, 1, false, true><<<b->push_blocks, nt, b->push_smem, s>>>(pp, b->d_tiles, b->ntiles, ctr);
  else if (b->compat)
    k_push_batched<float, true, true, 2, true, true><<<b->push_blocks, nt, b->push_smem, s>>>(pp, b->d_tiles, b->ntiles, ctr);
  else
    k_push_batched<float, true, true, 2, false, true><<<b->push_blocks, nt, b->push_smem, s>>>(pp, b->d_tiles, b->ntiles, ctr);
  CKLAUNCH("k_push_batched");
  k_fused_counts_batched<<<dim3(b->gx_cells, D), 256, 0, s>>>(b->d_fsort);
  CKLAUNCH("k_fused_counts_batched");
  k_scan_batched<<<D, SCB, 0, s>>>(b->d_dom);
  CKLAUNCH("k_scan_batched");
  k_fused_base_batched<<<dim3(b->gx_bins, D), 256, 0, s>>>(b->d_fsort);
  CKLAUNCH("k_fused_base_batched");
  k_fused_perm_batched<float><<<b->scatter_blocks, 256, 0, s>>>(b->d_scat + (size_t)par * D, b->d_tiles,
                                                                b->ntiles, ctr + 1);
  CKLAUNCH("k_fused_perm_batched");
  k_tile_off_batched<<<dim3(b->gx_tiles, D), 256, 0, s>>>(b->d_toff);
  CKLAUNCH("k_tile_off_batched");
  k_bhalf_batched<float><<<dim3(b->gx_field, D), 256, 0, s>>>(b->d_field);
  CKLAUNCH("k_bhalf_batched");
  k_efull_batched<float, long long><<<dim3(b->gx_field, D), 256, 0, s>>>(b->d_field);
  CKLAUNCH("k_efull_batched");
  k_bhalf_batched<float><<<dim3(b->gx_field, D), 256, 0, s>>>(b->d_field);
  CKLAUNCH("k_bhalf_batched");
  k_nodes_batched<float><<<dim3(b->gx_nodes, D), 256, 0, s>>>(b->d_field);
  CKLAUNCH("k_nodes_batched");
  k_cell_records_batched<<<dim3(b->gx_nodes, D), 256, 0, s>>>(b->d_field);
  CKLAUNCH("k_cell_records_batched");
  k_energy_rows_batched<<<D, 256, 0, s>>>(b->d_erow, ctr + 2);
  CKLAUNCH("k_energy_rows_batched");
  return PBPIC_OK;
}

// Capture two consecutive steps (set 0 then set 1) into a graph.
int batch_capture(pbpic_batch* b) {
  drop_graph(b);
  const long long before = g_launches.load();
  CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  int r = batch_enqueue_step(b, 0);
  if (r == PBPIC_OK) r = batch_enqueue_step(b, 1);
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(b->stream, &g);
  const long long captured = g_launches.load() - before;
  g_launches.fetch_sub(captured);  // counted again at each replay
  if (r != PBPIC_OK) {
    if (g) cudaGraphDestroy(g);
    return r;
  }
  if (e != cudaSuccess) return fail(PBPIC_ECUDA, std::string("stream capture of the batched step: ") + cudaGetErrorString(e));
  const cudaError_t ie = cudaGraphInstantiate(&b->graph, g, 0);
  cudaGraphDestroy(g);
  if (ie != cudaSuccess) {
    b->graph = nullptr;
    return fail(PBPIC_ECUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(ie));
  }
  b->launches_per_pair = captured;
  return PBPIC_OK;
}

int batch_set_tiles(pbpic_batch* b, const int32_t* tile_rows, int groups) {
  if (groups != 1 && groups != 2) return fail(PBPIC_EINVAL, "groups (particles per thread / 4) must be 1 or 2");
  for (size_t d = 0; d < b->dom.size(); ++d) {
    pbpic_handle* h = b->dom[d];
    TRY(retile(h, batch_tile_rows(h, tile_rows ? tile_rows[d] : 0)));
  }
  b->groups = groups;
  drop_graph(b);
  return batch_layout(b);
}

int batch_step(pbpic_batch* b, int nsteps) {
  if (nsteps <= 0) return PBPIC_OK;
  for (pbpic_handle* h : b->dom)
    if (h->filters) return fail(PBPIC_EINVAL, "the batched form does not apply field filters");
  // Every batched step reads through the domain's permutation (the push) and
  // writes a new one (the sort): a domain whose arrays are already in cell
  // order enters with the identity.
  for (pbpic_handle* h : b->dom) {
    if (!h->sorted) TRY(do_sort<float, true>(h));
    if (!h->perm) TRY(dalloc(h, &h->perm, ((size_t)std::max<int64_t>(h->cap, 1) + 16) * 4));
    if (!h->lazy) {
      if (h->n > 0) {
        k_iota<<<grid_for(h->n, 256), 256, 0, h->stream>>>(h->perm, h->n);
        CKLAUNCH("k_iota");
      }
      h->lazy = true;
    }
    TRY(ensure_hist(h, h->itime + nsteps + 2));
  }
  TRY(batch_descriptors(b));
  CK(cudaMemsetAsync(b->d_counters + 2, 0xff, sizeof(int), b->stream));  // step index -1
  if (nsteps >= 2 && !b->graph) TRY(batch_capture(b));
  for (int k = 0; k + 1 < nsteps; k += 2) {
    CK(cudaGraphLaunch(b->graph, b->stream));
    g_launches.fetch_add(b->launches_per_pair);
  }
  if (nsteps & 1) TRY(batch_enqueue_step(b, 0));
  for (pbpic_handle* h : b->dom) {
    if (nsteps & 1) h->cur = 1 - h->cur;
    h->itime += nsteps;
    h->sorted = true;
    h->hist_valid = false;
    h->lazy = true;  // the last step's permutation
  }
  return PBPIC_OK;
}

int check_batch(const pbpic_batch* b) {
  if (!b) return fail(PBPIC_EINVAL, "null batch");
  return PBPIC_OK;
}

}  // namespace

extern "C" {

int pbpic_batch_destroy(pbpic_batch* b) {
  if (!b) return PBPIC_OK;
  if (b->stream) cudaStreamSynchronize(b->stream);
  drop_graph(b);
  for (pbpic_handle* h : b->dom) {
    h->stream = 0;
    pbpic_destroy(h);
  }
  void* arrays[] = {b->d_push, b->d_scat, b->d_fsort, b->d_field, b->d_toff, b->d_dom, b->d_erow, b->d_tiles,
                    b->d_counters};
  for (void* p : arrays)
    if (p) cudaFree(p);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return PBPIC_OK;
}

int pbpic_batch_create(const pbpic_config* cfgs, const pbpic_loader* loaders, int32_t ndomains, pbpic_batch** out) {
  if (!cfgs || !loaders || !out) return fail(PBPIC_EINVAL, "null argument");
  *out = nullptr;
  if (ndomains < 1 || ndomains > 65535) return fail(PBPIC_EINVAL, "ndomains must be in [1, 65535]");
  for (int d = 0; d < ndomains; ++d) {
    const pbpic_config& c = cfgs[d];
    if (c.precision != PBPIC_FP32_MIXED) return fail(PBPIC_EINVAL, "the batched form runs FP32 mixed domains only");
    if (c.mx < 3 || (c.ybc == PBPIC_BC_PERIODIC && c.my < 3))
      return fail(PBPIC_EINVAL, "batched domains need mx >= 3, and my >= 3 with periodic y");
  }
  pbpic_batch* b = new pbpic_batch();
  auto bail = [&](int r) {
    pbpic_batch_destroy(b);
    return r;
  };
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
    b->stream = nullptr;
    return bail(fail(PBPIC_ECUDA, "cudaStreamCreateWithFlags failed"));
  }
  for (int d = 0; d < ndomains; ++d) {
    pbpic_config c = cfgs[d];
    const int64_t pairs = (int64_t)loaders[d].ppc * c.mx * c.my;
    const int64_t need = loaders[d].immobile_ions ? pairs : 2 * pairs;
    c.capacity = std::max<int64_t>(c.capacity, need);
    c.tile_rows = 0;
    pbpic_handle* h = nullptr;
    int r = pbpic_create(&c, &h);
    if (r != PBPIC_OK) return bail(r);
    h->cfg.tile_rows = cfgs[d].tile_rows;
    h->stream = b->stream;
    b->dom.push_back(h);
    r = do_init_plasma<float, true>(h, &loaders[d]);
    if (r != PBPIC_OK) {
      g_err = "domain " + std::to_string(d) + ": " + g_err;
      return bail(r);
    }
  }
  const size_t D = (size_t)ndomains;
  int r = PBPIC_OK;
  auto M = [&](auto** p, size_t bytes) {
    if (r == PBPIC_OK && cudaMalloc((void**)p, bytes) != cudaSuccess) {
      *p = nullptr;
      r = fail(PBPIC_ENOMEM, "cudaMalloc of the batch tables failed");
    }
  };
  M(&b->d_push, 2 * D * sizeof(PushParams<float>));
  M(&b->d_scat, 2 * D * sizeof(ScatterParams<float>));
  M(&b->d_fsort, D * sizeof(FusedSortParams));
  M(&b->d_field, D * sizeof(FieldParams<float>));
  M(&b->d_toff, D * sizeof(TileOffDesc));
  M(&b->d_dom, D * sizeof(BatchDomain));
  M(&b->d_erow, D * sizeof(EnergyRow));
  M(&b->d_counters, 4 * sizeof(int));
  if (r != PBPIC_OK) return bail(r);
  std::vector<int32_t> ty(D);
  for (size_t d = 0; d < D; ++d) ty[d] = cfgs[d].tile_rows;
  r = batch_set_tiles(b, ty.data(), PBPIC_PUSH_HALVES);
  if (r != PBPIC_OK) return bail(r);
  if (cudaStreamSynchronize(b->stream) != cudaSuccess) return bail(fail(PBPIC_ECUDA, "batch initialisation failed"));
  *out = b;
  return PBPIC_OK;
}

int pbpic_batch_num_domains(const pbpic_batch* b, int32_t* n) {
  TRY(check_batch(b));
  if (!n) return fail(PBPIC_EINVAL, "null argument");
  *n = (int32_t)b->dom.size();
  return PBPIC_OK;
}

int pbpic_batch_domain(pbpic_batch* b, int32_t d, pbpic_handle** h) {
  TRY(check_batch(b));
  if (!h) return fail(PBPIC_EINVAL, "null argument");
  if (d < 0 || d >= (int32_t)b->dom.size()) return fail(PBPIC_EINVAL, "domain index out of range");
  *h = b->dom[d];
  return PBPIC_OK;
}

int pbpic_batch_set_tiles(pbpic_batch* b, const int32_t* tile_rows, int32_t groups) {
  TRY(check_batch(b));
  return batch_set_tiles(b, tile_rows, groups);
}

int pbpic_batch_get_tiles(const pbpic_batch* b, int32_t* tile_rows, int32_t* groups) {
  TRY(check_batch(b));
  if (tile_rows)
    for (size_t d = 0; d < b->dom.size(); ++d) tile_rows[d] = b->dom[d]->TY;
  if (groups) *groups = b->groups;
  return PBPIC_OK;
}

int pbpic_batch_step(pbpic_batch* b, int32_t nsteps) {
  TRY(check_batch(b));
  if (nsteps < 0) return fail(PBPIC_EINVAL, "nsteps must be >= 0");
  return batch_step(b, nsteps);
}

int pbpic_batch_stream(const pbpic_batch* b, void** stream) {
  TRY(check_batch(b));
  if (!stream) return fail(PBPIC_EINVAL, "null argument");
  *stream = (void*)b->stream;
  return PBPIC_OK;
}

int pbpic_batch_synchronize(pbpic_batch* b) {
  TRY(check_batch(b));
  CK(cudaStreamSynchronize(b->stream));
  return PBPIC_OK;
}

int pbpic_batch_autotune(pbpic_batch* b, int32_t trial_steps, int32_t* tile_rows_out, int32_t* groups_out,
                         double* best_ms_per_step) {
  TRY(check_batch(b));
  if (trial_steps < 2) return fail(PBPIC_EINVAL, "trial_steps must be >= 2");
  const int pairs = trial_steps / 2;
  const int caps[] = {16, 32, 64};
  const int D = (int)b->dom.size();
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  double best = 1e300;
  int best_cap = 64, best_g = PBPIC_PUSH_HALVES;
  std::vector<int32_t> ty(D);
  int r = PBPIC_OK;
  for (int g = 1; g <= 2 && r == PBPIC_OK; ++g)
    for (int cap : caps) {
      for (int d = 0; d < D; ++d) ty[d] = cap;
      r = batch_set_tiles(b, ty.data(), g);
      if (r == PBPIC_OK) r = batch_step(b, 2);  // capture and warm up
      if (r == PBPIC_OK && cudaEventRecord(e0, b->stream) != cudaSuccess) r = fail(PBPIC_ECUDA, "cudaEventRecord");
      if (r == PBPIC_OK) r = batch_step(b, 2 * pairs);
      if (r == PBPIC_OK && cudaEventRecord(e1, b->stream) != cudaSuccess) r = fail(PBPIC_ECUDA, "cudaEventRecord");
      float ms = 0;
      if (r == PBPIC_OK && (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess))
        r = fail(PBPIC_ECUDA, "timing the autotuner trial failed");
      if (r != PBPIC_OK) break;
      const double per = ms / (2.0 * pairs);
      if (per < best) {
        best = per;
        best_cap = cap;
        best_g = g;
      }
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  TRY(r);
  for (int d = 0; d < D; ++d) ty[d] = best_cap;
  TRY(batch_set_tiles(b, ty.data(), best_g));
  if (tile_rows_out)
    for (int d = 0; d < D; ++d) tile_rows_out[d] = b->dom[d]->TY;
  if (groups_out) *groups_out = best_g;
  if (best_ms_per_step) *best_ms_per_step = best;
  return PBPIC_OK;
}

int pbpic_batch_energies(pbpic_batch* b, double* out) {
  TRY(check_batch(b));
  if (!out) return fail(PBPIC_EINVAL, "null argument");
  for (size_t d = 0; d < b->dom.size(); ++d) {
    const pbpic_handle* h = b->dom[d];
    CK(cudaMemcpyAsync(out + 4 * d, h->hist + (size_t)h->itime * 4, 4 * sizeof(double), cudaMemcpyDeviceToHost,
                       b->stream));
  }
  CK(cudaStreamSynchronize(b->stream));
  return PBPIC_OK;
}

}  // extern "C"

// ============================================================ dump / restart
// The state of a handle as a directory of .npy files named like the datasets
// of the reference's HDF5 dumps (particlesinfo, pic2d.f90:1358-1380, and
// fieldsinfo, pic2d.f90:1625-1644): particles/{dx,dy,ux,uy,uz,grid,q,pid},
// fields/{ex,ey,ez,bx,by,bz} (mx x (my+1), the layout of pbpic_store_fields),
// fields/{jx,jy,jz,rho} (the last push's current, as pbpic_store_denjr),
// totene (itime+1 x 4) and state.json (the run parameters, itime and counts).
// Particle and field values keep the handle's precision (<f4 mixed, <f8
// plain), so a restart reproduces the state exactly. HDF5 itself is not used.
namespace {

bool make_dir(const std::string& d) { return mkdir(d.c_str(), 0755) == 0 || errno == EEXIST; }

template <class T>
const char* npy_descr() {
  return sizeof(T) == 4 ? "<f4" : "<f8";
}

template <class T, bool MIXED>
int do_dump(pbpic_handle* h, const std::string& dir) {
  if (!make_dir(dir) || !make_dir(dir + "/particles") || !make_dir(dir + "/fields"))
    return fail(PBPIC_EINVAL, "cannot create the dump directory " + dir);
  const int64_t n = h->n;
  std::vector<pbpic_particle_f64> rec((size_t)std::max<int64_t>(n, 1));
  int64_t got = 0;
  TRY(pbpic_store_particles_f64(h, rec.data(), n, &got));
  std::vector<T> v((size_t)std::max<int64_t>(n, 1));
  std::vector<int32_t> iv((size_t)std::max<int64_t>(n, 1));
  const char* names[5] = {"dx", "dy", "ux", "uy", "uz"};
  for (int c = 0; c < 5; ++c) {
    for (int64_t i = 0; i < n; ++i) {
      const pbpic_particle_f64& r = rec[i];
      const double x = c == 0 ? r.dx : c == 1 ? r.dy : c == 2 ? r.ux : c == 3 ? r.uy : r.uz;
      v[i] = (T)x;  // exact: the values are the device's T values
    }
    if (!npyio::write(dir + "/particles/" + names[c] + ".npy", npy_descr<T>(), {n}, v.data(), (size_t)n * sizeof(T)))
      return fail(PBPIC_EINVAL, "cannot write " + dir + "/particles");
  }
  const char* inames[3] = {"grid", "q", "pid"};
  for (int c = 0; c < 3; ++c) {
    if (c == 2 && !h->cfg.track_pid) continue;
    for (int64_t i = 0; i < n; ++i) iv[i] = c == 0 ? rec[i].grid : c == 1 ? rec[i].q : rec[i].pid;
    if (!npyio::write(dir + "/particles/" + inames[c] + ".npy", "<i4", {n}, iv.data(), (size_t)n * 4))
      return fail(PBPIC_EINVAL, "cannot write " + dir + "/particles");
  }
  const int64_t pe = plane_elems(h);
  std::vector<double> f6((size_t)(6 * pe)), j4((size_t)(4 * pe));
  TRY((do_store_fields<T, MIXED>(h, f6.data())));
  TRY(do_store_denjr(h, j4.data()));
  const char* fnames[6] = {"ex", "ey", "ez", "bx", "by", "bz"};
  std::vector<T> plane((size_t)pe);
  for (int c = 0; c < 6; ++c) {
    for (int64_t k = 0; k < pe; ++k) plane[k] = (T)f6[(size_t)c * pe + k];
    if (!npyio::write(dir + "/fields/" + fnames[c] + ".npy", npy_descr<T>(), {h->cfg.mx, h->S}, plane.data(),
                      (size_t)pe * sizeof(T)))
      return fail(PBPIC_EINVAL, "cannot write " + dir + "/fields");
  }
  const char* jnames[4] = {"jx", "jy", "jz", "rho"};
  for (int c = 0; c < 4; ++c)
    if (!npyio::write(dir + "/fields/" + jnames[c] + ".npy", "<f8", {h->cfg.mx, h->S}, j4.data() + (size_t)c * pe,
                      (size_t)pe * 8))
      return fail(PBPIC_EINVAL, "cannot write " + dir + "/fields");
  const int rows = h->itime + 1;
  std::vector<double> hist((size_t)rows * 4);
  CK(cudaMemcpyAsync(hist.data(), h->hist, hist.size() * 8, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (!npyio::write(dir + "/totene.npy", "<f8", {rows, 4}, hist.data(), hist.size() * 8))
    return fail(PBPIC_EINVAL, "cannot write " + dir + "/totene.npy");
  const pbpic_config& c = h->cfg;
  if (!npyio::write_numbers(dir + "/state.json",
                            {{"format", 1}, {"mx", c.mx}, {"my", c.my}, {"dx", c.dx}, {"dy", c.dy}, {"dt", c.dt},
                             {"cva", c.cva}, {"mime", c.mime}, {"in0", c.in0}, {"ybc", c.ybc},
                             {"precision", c.precision}, {"compat", c.compat}, {"track_pid", c.track_pid},
                             {"itime", h->itime}, {"particles", (double)n}}))
    return fail(PBPIC_EINVAL, "cannot write " + dir + "/state.json");
  return PBPIC_OK;
}

// The reference's HDF5 dumps (particlesinfo pic2d.f90:1358-1380 and
// 1400-1560, fieldsinfo 1625-1830, energyinfo 2034-2112), written with
// h5_writer.h: root datasets, the reference's names and element types (its
// `real` is 4 bytes), Fortran dimensions (a, b) stored as C order (b, a).
template <class T, bool MIXED>
int do_dump_h5(pbpic_handle* h, const std::string& dir, double de_e, double de_i, int nbins) {
  if (!make_dir(dir)) return fail(PBPIC_EINVAL, "cannot create the dump directory " + dir);
  const pbpic_config& c = h->cfg;
  const int mx = c.mx, my = c.my;
  const int64_t n = h->n;
  std::string err;
  using h5w::Dataset;
  auto vec_writer = [](const void* p) {
    return [p](FILE* f, uint64_t bytes) { return fwrite(p, 1, bytes, f) == bytes; };
  };
  // ---- particles.h5: dx dy ux uy uz (real), grid q pid (integer) of length
  // the capacity, the particles first (zeros after them, unwritten in the
  // reference), and nptlact (one entry per rank: one rank here)
  std::vector<pbpic_particle_f32> rec((size_t)std::max<int64_t>(n, 1));
  int64_t got = 0;
  TRY(pbpic_store_particles_f32(h, rec.data(), n, &got));
  const uint64_t cap = (uint64_t)std::max<int64_t>(h->cap, n);
  std::vector<std::vector<uint32_t>> cols(8, std::vector<uint32_t>((size_t)cap, 0u));
  for (int64_t i = 0; i < n; ++i) {
    const pbpic_particle_f32& r = rec[i];
    memcpy(&cols[0][i], &r.dx, 4);
    memcpy(&cols[1][i], &r.dy, 4);
    memcpy(&cols[2][i], &r.ux, 4);
    memcpy(&cols[3][i], &r.uy, 4);
    memcpy(&cols[4][i], &r.uz, 4);
    memcpy(&cols[5][i], &r.grid, 4);
    memcpy(&cols[6][i], &r.q, 4);
    memcpy(&cols[7][i], &r.pid, 4);
  }
  const int32_t nptlact = (int32_t)n;
  {
    h5w::Group root;
    const char* names[8] = {"dx", "dy", "ux", "uy", "uz", "grid", "q", "pid"};
    for (int k = 0; k < 8; ++k)
      root.datasets.push_back(Dataset{names[k], k < 5 ? h5w::FLOAT : h5w::INT, 4, {cap}, vec_writer(cols[k].data())});
    root.datasets.push_back(Dataset{"nptlact", h5w::INT, 4, {1}, vec_writer(&nptlact)});
    if (!h5w::write_file(dir + "/particles.h5", root, &err)) return fail(PBPIC_EINVAL, err);
  }
  // particle number per cell (numdensity, pic2d.f90:1343-1353)
  std::vector<int32_t> num((size_t)mx * my, 0);
  for (int64_t i = 0; i < n; ++i) {
    const int64_t g = (int64_t)rec[i].grid - 1;
    if (g >= 0 && g < (int64_t)mx * my) num[(size_t)g] += 1;
  }
  cols.clear();
  rec.clear();
  // ---- fields%05d.h5: emf(0:mx+1, 1:my+1) and denjr(0:mx+1, 1:my+1) as
  // (my+1) x (mx+2): x ghosts 0 and mx+1 are the periodic copies of columns
  // mx and 1; the last row is the top ghost row (periodic y: a copy of row 1)
  const int64_t pe = plane_elems(h);
  std::vector<double> f6((size_t)(6 * pe)), j4((size_t)(4 * pe));
  TRY((do_store_fields<T, MIXED>(h, f6.data())));
  TRY(do_store_denjr(h, j4.data()));
  const int W = mx + 2, H = my + 1;
  auto at = [&](const double* plane, int iref, int jref) {  // reference (iref, jref), 0..mx+1, 1..my+1
    int i = iref - 1, j = jref - 1;
    i = i < 0 ? i + mx : (i >= mx ? i - mx : i);
    if (c.ybc == PBPIC_BC_PERIODIC && j == my) j = 0;
    return plane[(size_t)i * h->S + j];
  };
  std::vector<std::vector<float>> fl(11, std::vector<float>((size_t)W * H));
  std::vector<int32_t> numd((size_t)W * H, 0);
  for (int jr = 1; jr <= my + 1; ++jr)
    for (int ir = 0; ir <= mx + 1; ++ir) {
      const size_t o = (size_t)(jr - 1) * W + ir;
      for (int k = 0; k < 6; ++k) fl[k][o] = (float)at(f6.data() + (size_t)k * pe, ir, jr);
      // dive (emf%dive): div E at the node, (ex(i,j) - ex(i-1,j))/dx + (ey(i,j) - ey(i,j-1))/dy
      fl[6][o] = (float)((at(f6.data(), ir, jr) - at(f6.data(), ir - 1, jr)) / c.dx +
                         (at(f6.data() + pe, ir, jr) - at(f6.data() + pe, ir, jr == 1 ? my : jr - 1)) / c.dy);
      for (int k = 0; k < 4; ++k) fl[7 + k][o] = (float)at(j4.data() + (size_t)k * pe, ir, jr);
      if (ir >= 1 && ir <= mx && jr <= my) numd[o] = num[(size_t)(ir - 1) * my + (jr - 1)];
    }
  {
    h5w::Group root;
    const char* names[11] = {"ex", "ey", "ez", "bx", "by", "bz", "dive", "jx", "jy", "jz", "rho"};
    for (int k = 0; k < 11; ++k)
      root.datasets.push_back(Dataset{names[k], h5w::FLOAT, 4, {(uint64_t)H, (uint64_t)W}, vec_writer(fl[k].data())});
    root.datasets.push_back(Dataset{"num", h5w::INT, 4, {(uint64_t)H, (uint64_t)W}, vec_writer(numd.data())});
    char name[32];
    snprintf(name, sizeof(name), "/fields%05d.h5", h->itime);
    if (!h5w::write_file(dir + name, root, &err)) return fail(PBPIC_EINVAL, err);
  }
  // ---- spectra.h5: one group "%05d" per dumped time step with "spectra"
  // (integer, (2, nbins): electrons, ions), and "ebins" (real, bin upper edges)
  std::vector<int64_t> sp((size_t)2 * nbins);
  TRY(pbpic_energy_spectra(h, de_e, de_i, nbins, sp.data()));
  std::vector<int32_t> spc((size_t)2 * nbins);
  for (int b = 0; b < nbins; ++b) {
    spc[(size_t)2 * b] = (int32_t)sp[(size_t)b];
    spc[(size_t)2 * b + 1] = (int32_t)sp[(size_t)nbins + b];
  }
  auto same = std::find_if(h->h5_spectra.begin(), h->h5_spectra.end(),
                           [&](const std::pair<int32_t, std::vector<int32_t>>& e) { return e.first == h->itime; });
  if (same != h->h5_spectra.end()) same->second = spc;
  else h->h5_spectra.push_back({h->itime, spc});
  std::vector<float> ebins((size_t)2 * nbins);
  for (int b = 0; b < nbins; ++b) {
    ebins[(size_t)2 * b] = (float)((b + 1) * de_e);
    ebins[(size_t)2 * b + 1] = (float)((b + 1) * de_i);
  }
  {
    h5w::Group root;
    for (const auto& e : h->h5_spectra) {
      char gname[16];
      snprintf(gname, sizeof(gname), "%05d", e.first);
      h5w::Group g;
      g.name = gname;
      g.datasets.push_back(Dataset{"spectra", h5w::INT, 4, {(uint64_t)(e.second.size() / 2), 2}, vec_writer(e.second.data())});
      root.groups.push_back(g);
    }
    root.datasets.push_back(Dataset{"ebins", h5w::FLOAT, 4, {(uint64_t)nbins, 2}, vec_writer(ebins.data())});
    if (!h5w::write_file(dir + "/spectra.h5", root, &err)) return fail(PBPIC_EINVAL, err);
  }
  // ---- energy_tot.h5: tote, (4, ntime) energies of the steps so far
  const int rows = h->itime + 1;
  std::vector<double> hist((size_t)rows * 4);
  CK(cudaMemcpyAsync(hist.data(), h->hist, hist.size() * 8, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  std::vector<float> tote(hist.begin(), hist.end());
  {
    h5w::Group root;
    root.datasets.push_back(Dataset{"tote", h5w::FLOAT, 4, {(uint64_t)rows, 4}, vec_writer(tote.data())});
    if (!h5w::write_file(dir + "/energy_tot.h5", root, &err)) return fail(PBPIC_EINVAL, err);
  }
  return PBPIC_OK;
}

template <class T, bool MIXED>
int do_restart(pbpic_handle* h, const std::string& dir) {
  std::map<std::string, double> st;
  if (!npyio::read_numbers(dir + "/state.json", &st) || !st.count("itime") || !st.count("particles"))
    return fail(PBPIC_EINVAL, "cannot read " + dir + "/state.json");
  const pbpic_config& c = h->cfg;
  if ((int)st["mx"] != c.mx || (int)st["my"] != c.my || (int)st["ybc"] != c.ybc || (int)st["precision"] != c.precision)
    return fail(PBPIC_EINVAL, "the dump's mx, my, ybc or precision differ from the handle's");
  const int64_t n = (int64_t)st["particles"];
  const int itime = (int)st["itime"];
  if (n > h->cap) return fail(PBPIC_ECAPACITY, "the dump holds more particles than the handle's capacity");
  auto load = [&](const std::string& name, const char* descr, int64_t count, npyio::Array* a) -> int {
    const std::string err = npyio::read(dir + "/" + name + ".npy", a);
    if (!err.empty()) return fail(PBPIC_EINVAL, err);
    if (a->descr != descr || a->count() != count) return fail(PBPIC_EINVAL, dir + "/" + name + ".npy: unexpected dtype or shape");
    return PBPIC_OK;
  };
  std::vector<pbpic_particle_f64> rec((size_t)std::max<int64_t>(n, 1));
  const char* names[5] = {"dx", "dy", "ux", "uy", "uz"};
  for (int k = 0; k < 5; ++k) {
    npyio::Array a;
    TRY(load(std::string("particles/") + names[k], npy_descr<T>(), n, &a));
    const T* p = reinterpret_cast<const T*>(a.data.data());
    for (int64_t i = 0; i < n; ++i) {
      double* dst = k == 0 ? &rec[i].dx : k == 1 ? &rec[i].dy : k == 2 ? &rec[i].ux : k == 3 ? &rec[i].uy : &rec[i].uz;
      *dst = (double)p[i];
    }
  }
  const char* inames[3] = {"grid", "q", "pid"};
  for (int k = 0; k < 3; ++k) {
    npyio::Array a;
    if (k == 2) {
      for (int64_t i = 0; i < n; ++i) rec[i].pid = 0;
      if (!c.track_pid) continue;
      FILE* f = fopen((dir + "/particles/pid.npy").c_str(), "rb");
      if (!f) continue;  // dumped without particle ids
      fclose(f);
    }
    TRY(load(std::string("particles/") + inames[k], "<i4", n, &a));
    const int32_t* p = reinterpret_cast<const int32_t*>(a.data.data());
    for (int64_t i = 0; i < n; ++i) (k == 0 ? rec[i].grid : k == 1 ? rec[i].q : rec[i].pid) = p[i];
  }
  for (int64_t i = 0; i < n; ++i) rec[i].pad = 0;
  npyio::Array hist;
  TRY(load("totene", "<f8", (int64_t)(itime + 1) * 4, &hist));
  const int64_t pe = plane_elems(h);
  std::vector<double> f6((size_t)(6 * pe));
  const char* fnames[6] = {"ex", "ey", "ez", "bx", "by", "bz"};
  for (int k = 0; k < 6; ++k) {
    npyio::Array a;
    TRY(load(std::string("fields/") + fnames[k], npy_descr<T>(), pe, &a));
    const T* p = reinterpret_cast<const T*>(a.data.data());
    for (int64_t i = 0; i < pe; ++i) f6[(size_t)k * pe + i] = (double)p[i];
  }
  TRY(pbpic_load_particles_f64(h, rec.data(), n));
  h->itime = itime;
  TRY(ensure_hist(h, itime + 2));
  CK(cudaMemcpyAsync(h->hist, hist.data.data(), hist.data.size(), cudaMemcpyHostToDevice, h->stream));
  TRY((do_load_fields<T, MIXED>(h, f6.data())));
  TRY((do_sort<T, MIXED>(h)));
  CK(cudaStreamSynchronize(h->stream));
  return PBPIC_OK;
}

}  // namespace

extern "C" {

int pbpic_dump(pbpic_handle* h, const char* dir) {
  TRY(check_handle(h));
  if (!dir) return fail(PBPIC_EINVAL, "null directory");
  return DISPATCH(h, do_dump, h, std::string(dir));
}

int pbpic_dump_h5(pbpic_handle* h, const char* dir, double de_electron, double de_ion, int32_t nbins) {
  TRY(check_handle(h));
  if (!dir) return fail(PBPIC_EINVAL, "null directory");
  if (de_electron <= 0) de_electron = 0.005;
  if (de_ion <= 0) de_ion = de_electron;
  if (nbins <= 0) nbins = 1000;
  if (nbins > 8192) return fail(PBPIC_EINVAL, "spectra take 1..8192 bins");
  return DISPATCH(h, do_dump_h5, h, std::string(dir), de_electron, de_ion, (int)nbins);
}

int pbpic_restart(pbpic_handle* h, const char* dir) {
  TRY(check_handle(h));
  if (!dir) return fail(PBPIC_EINVAL, "null directory");
  return DISPATCH(h, do_restart, h, std::string(dir));
}

}  // extern "C"

// ================================================================ y slabs
// Device-side pieces of the y-slab decomposition (kernels_slab.cuh); the
// driver that exchanges ghost bands between ranks is pbpic_b200/slab.py.
namespace {

int band_buffers(pbpic_handle* h) {
  if (h->band_flags) return PBPIC_OK;
  const int64_t m = std::max<int64_t>(h->cap, 1) + 2;
  TRY(dalloc(h, &h->band_flags, (size_t)m * 4));
  TRY(dalloc(h, &h->band_scratch, (size_t)scan_scratch_ints(m) * 4));
  return PBPIC_OK;
}

// Positions of the particles in rows [y_lo, y_hi): exclusive scan of the
// flags in h->band_flags; returns their number.
int band_positions(pbpic_handle* h, int y_lo, int y_hi, int64_t* count) {
  TRY(band_buffers(h));
  cudaStream_t s = h->stream;
  const int64_t n = h->n;
  k_band_flags<<<grid_for(n + 1, 256), 256, 0, s>>>(n, h->cell[h->cur], y_lo, y_hi, h->band_flags);
  CKLAUNCH("k_band_flags");
  TRY(scan_excl(s, h->band_flags, n + 1, h->band_scratch));
  int32_t c = 0;
  CK(cudaMemcpyAsync(&c, h->band_flags + n, 4, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  *count = c;
  return PBPIC_OK;
}

int col_buffers(pbpic_handle* h) {
  if (h->colbuf) return PBPIC_OK;
  TRY(dalloc(h, &h->colbuf, (size_t)8 * (h->cfg.mx + 1) * 4));
  TRY(dalloc(h, &h->colscan, (size_t)scan_scratch_ints(h->cfg.mx + 1) * 4));
  return PBPIC_OK;
}

// Particles sorted by cell: a band of rows is one range per column (cell offsets).
template <class T, bool MIXED>
int band_extract_sorted(pbpic_handle* h, int y_lo, int y_hi, int my_global, int row_offset, void* dst, int64_t cap,
                        int64_t* nout) {
  TRY(col_buffers(h));
  cudaStream_t s = h->stream;
  const int mx = h->cfg.mx;
  int32_t* colstart = h->colbuf;
  k_col_counts<<<grid_for(mx + 1, 256), 256, 0, s>>>(h->off, mx, h->cfg.my, y_lo, y_hi, colstart);
  CKLAUNCH("k_col_counts");
  TRY(scan_excl(s, colstart, mx + 1, h->colscan));
  int32_t total = 0;
  CK(cudaMemcpyAsync(&total, colstart + mx, 4, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (nout) *nout = total;
  if (total > cap) return fail(PBPIC_ECAPACITY, "the band holds more particles than the destination");
  if (total > 0 && !dst) return fail(PBPIC_EINVAL, "null band destination");
  const int b = h->cur;
  if (total > 0) {
    k_band_out_sorted<T, T><<<std::min(mx, 148 * 16), 256, 0, s>>>(
        colstart, h->off, mx, h->cfg.my, y_lo, h->cell[b], P<T>(h, b, 0), P<T>(h, b, 1), P<T>(h, b, 2),
        P<T>(h, b, 3), P<T>(h, b, 4), h->pid[b], my_global, row_offset, (RefRec<T>*)dst,
        h->lazy ? h->perm : nullptr, ((uintptr_t)dst & 15) == 0);
    CKLAUNCH("k_band_out_sorted");
  }
  CK(cudaStreamSynchronize(s));
  return PBPIC_OK;
}

template <class T, bool MIXED>
int do_band_extract(pbpic_handle* h, int y_lo, int y_hi, int my_global, int row_offset, void* dst, int64_t cap,
                    int64_t* nout) {
  if (h->sorted) return band_extract_sorted<T, MIXED>(h, y_lo, y_hi, my_global, row_offset, dst, cap, nout);
  TRY(materialize(h));
  int64_t c = 0;
  TRY(band_positions(h, y_lo, y_hi, &c));
  if (nout) *nout = c;
  if (c > cap) return fail(PBPIC_ECAPACITY, "the band holds more particles than the destination");
  if (c > 0 && !dst) return fail(PBPIC_EINVAL, "null band destination");
  const int b = h->cur;
  if (h->n > 0 && c > 0) {
    k_band_out<T, T><<<grid_for(h->n, 256), 256, 0, h->stream>>>(h->n, h->cell[b], P<T>(h, b, 0), P<T>(h, b, 1),
                                                                 P<T>(h, b, 2), P<T>(h, b, 3), P<T>(h, b, 4),
                                                                 h->pid[b], h->band_flags, my_global, row_offset,
                                                                 (RefRec<T>*)dst);
    CKLAUNCH("k_band_out");
  }
  CK(cudaStreamSynchronize(h->stream));
  return PBPIC_OK;
}

template <class T, bool MIXED>
int do_band_keep(pbpic_handle* h, int y_lo, int y_hi) {
  TRY(materialize(h));
  int64_t c = 0;
  TRY(band_positions(h, y_lo, y_hi, &c));
  const int b = h->cur, o = 1 - b;
  if (h->n > 0) {
    k_band_keep<T><<<grid_for(h->n, 256), 256, 0, h->stream>>>(
        h->n, h->band_flags, h->cell[b], P<T>(h, b, 0), P<T>(h, b, 1), P<T>(h, b, 2), P<T>(h, b, 3), P<T>(h, b, 4),
        h->pid[b], h->cell[o], P<T>(h, o, 0), P<T>(h, o, 1), P<T>(h, o, 2), P<T>(h, o, 3), P<T>(h, o, 4), h->pid[o]);
    CKLAUNCH("k_band_keep");
    h->cur = o;
  }
  h->n = c;
  return set_unsorted_tiles(h);
}

template <class T, bool MIXED>
int do_band_append(pbpic_handle* h, const void* src, int64_t n, int my_global, int row_offset) {
  TRY(materialize(h));
  if (n < 0) return fail(PBPIC_EINVAL, "negative count");
  if (h->n + n > h->cap) return fail(PBPIC_ECAPACITY, "appending the band exceeds the capacity");
  if (n == 0) return PBPIC_OK;
  if (!src) return fail(PBPIC_EINVAL, "null band");
  cudaStream_t s = h->stream;
  const int b = h->cur;
  CK(cudaMemsetAsync(h->dscalar, 0, 4, s));
  k_band_in<T, T><<<grid_for(n, 256), 256, 0, s>>>((const RefRec<T>*)src, n, my_global, row_offset, h->cfg.mx,
                                                   h->cfg.my, h->n, h->cell[b], P<T>(h, b, 0), P<T>(h, b, 1),
                                                   P<T>(h, b, 2), P<T>(h, b, 3), P<T>(h, b, 4), h->pid[b],
                                                   (int*)h->dscalar);
  CKLAUNCH("k_band_in");
  int st = 0;
  CK(cudaMemcpyAsync(&st, h->dscalar, 4, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  h->n += n;
  TRY(set_unsorted_tiles(h));
  if (st & 8) return fail(PBPIC_EINVAL, "band record outside this domain's rows or with q not +-1");
  return PBPIC_OK;
}

// Own rows [y_lo, y_hi) plus the two received bands, in cell order, in one
// pass (particles sorted by cell on entry); otherwise compaction, appends and
// a sort.
template <class T, bool MIXED>
int do_band_replace(pbpic_handle* h, int y_lo, int y_hi, const void* bot, int64_t nb, int off_bottom,
                    const void* top, int64_t nt, int off_top, int my_global) {
  if (!h->sorted) {  // (a handle in permuted order is sorted: the path below reads through the permutation)
    TRY((do_band_keep<T, MIXED>(h, y_lo, y_hi)));
    TRY((do_band_append<T, MIXED>(h, bot, nb, my_global, off_bottom)));
    TRY((do_band_append<T, MIXED>(h, top, nt, my_global, off_top)));
    return do_sort<T, MIXED>(h);
  }
  if ((nb && !bot) || (nt && !top) || nb < 0 || nt < 0) return fail(PBPIC_EINVAL, "null or negative band");
  TRY(col_buffers(h));
  cudaStream_t s = h->stream;
  const int mx = h->cfg.mx, my = h->cfg.my;
  const size_t m1 = (size_t)mx + 1;
  int32_t *ocnt = h->colbuf, *bcnt = ocnt + m1, *tcnt = bcnt + m1, *bstart = tcnt + m1, *tstart = bstart + m1,
          *outstart = tstart + m1;
  k_col_counts<<<grid_for(mx + 1, 256), 256, 0, s>>>(h->off, mx, my, y_lo, y_hi, ocnt);
  CKLAUNCH("k_col_counts");
  int32_t *first = outstart + m1, *last = first + m1;
  for (int band = 0; band < 2; ++band) {  // per-column counts of the bands (column-ordered records)
    const void* src = band == 0 ? bot : top;
    const int64_t nr = band == 0 ? nb : nt;
    int32_t* cnt = band == 0 ? bcnt : tcnt;
    CK(cudaMemsetAsync(first, 0, 2 * m1 * 4, s));
    if (nr) {
      k_band_col_bounds<T><<<grid_for(nr, 256), 256, 0, s>>>((const RefRec<T>*)src, nr, my_global, mx, first, last);
      CKLAUNCH("k_band_col_bounds");
    }
    k_col_diff<<<grid_for(mx + 1, 256), 256, 0, s>>>(first, last, mx, cnt);
    CKLAUNCH("k_col_diff");
  }
  CK(cudaMemcpyAsync(bstart, bcnt, 2 * m1 * 4, cudaMemcpyDeviceToDevice, s));  // bstart, tstart
  k_col_sum3<<<grid_for(mx + 1, 256), 256, 0, s>>>(ocnt, bcnt, tcnt, mx, outstart);
  CKLAUNCH("k_col_sum3");
  TRY(scan_excl(s, bstart, (int64_t)m1, h->colscan));
  TRY(scan_excl(s, tstart, (int64_t)m1, h->colscan));
  TRY(scan_excl(s, outstart, (int64_t)m1, h->colscan));
  int32_t total = 0;
  CK(cudaMemcpyAsync(&total, outstart + mx, 4, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (total > h->cap) return fail(PBPIC_ECAPACITY, "the slab's particles and bands exceed the capacity");
  const int b = h->cur, o = 1 - b;
  const int64_t base = h->n;  // the bands' records go after the current particles
  const bool by_perm = base + nb + nt <= h->cap;
  ReplaceSrc rs;
  rs.off = h->off;
  rs.outstart = outstart;
  rs.bstart = bstart;
  rs.bcnt = bcnt;
  rs.ocnt = ocnt;
  rs.mx = mx;
  rs.my = my;
  rs.y_lo = y_lo;
  rs.my_global = my_global;
  rs.off_bottom = off_bottom;
  rs.off_top = off_top;
  rs.tstart = tstart;
  if (by_perm) {
    // the own particles stay in place: the bands are converted after them and
    // the assembled order is a permutation the next push reads through
    if (nb + nt > 0) {
      k_band_to_soa<T, T><<<grid_for(nb + nt, 256), 256, 0, s>>>(
          nb, nt, rs, (const RefRec<T>*)bot, (const RefRec<T>*)top, base, h->cell[b], P<T>(h, b, 0), P<T>(h, b, 1),
          P<T>(h, b, 2), P<T>(h, b, 3), P<T>(h, b, 4), h->pid[b], h->status);
      CKLAUNCH("k_band_to_soa");
    }
    const int64_t pcap = std::max<int64_t>(h->cap, 1) + 16;
    if (!h->perm) TRY(dalloc(h, &h->perm, (size_t)pcap * 4));
    if (!h->perm2) TRY(dalloc(h, &h->perm2, (size_t)pcap * 4));
    if (total > 0) {
      k_band_assemble_perm<<<std::min(mx, 148 * 16), 256, 0, s>>>(rs, base, nb, h->lazy ? h->perm : nullptr, h->perm2);
      CKLAUNCH("k_band_assemble_perm");
    }
    k_counts_own_rows<<<grid_for((int64_t)h->ncells + 1, 256), 256, 0, s>>>(h->off, h->ncells, my, y_lo, y_hi,
                                                                            h->counts);
    CKLAUNCH("k_counts_own_rows");
    if (nb + nt > 0) {
      k_counts_band<<<grid_for(nb + nt, 256), 256, 0, s>>>(nb + nt, h->cell[b], base, my, h->counts);
      CKLAUNCH("k_counts_band");
    }
    std::swap(h->perm, h->perm2);
    h->lazy = true;  // cell order = the current arrays read through perm
    h->n = total;
    CK(cudaMemcpyAsync(h->off, h->counts, (size_t)(h->ncells + 1) * 4, cudaMemcpyDeviceToDevice, s));
    TRY(scan_excl(s, h->off, h->ncells + 1, h->scan_scratch));
    k_tile_off<<<grid_for(h->ntiles + 1, 256, 1 << 20), 256, 0, s>>>(h->off, h->ntiles, h->tpc, h->TY, my, total,
                                                                    h->tile_off);
    CKLAUNCH("k_tile_off");
    h->sorted = true;
    h->hist_valid = false;
    return PBPIC_OK;
  }
  if (total > 0) {
    k_band_assemble<T, T><<<grid_for(total, 256), 256, 0, s>>>(
        total, rs, (const RefRec<T>*)bot, (const RefRec<T>*)top, h->cell[b], P<T>(h, b, 0), P<T>(h, b, 1),
        P<T>(h, b, 2), P<T>(h, b, 3), P<T>(h, b, 4), h->pid[b], h->cell[o], P<T>(h, o, 0), P<T>(h, o, 1),
        P<T>(h, o, 2), P<T>(h, o, 3), P<T>(h, o, 4), h->pid[o], h->status, h->lazy ? h->perm : nullptr);
    CKLAUNCH("k_band_assemble");
  }
  h->cur = o;
  h->lazy = false;  // the assembled arrays are in cell order themselves
  h->n = total;
  // cell offsets and tile ranges of the new (sorted) array
  CK(cudaMemsetAsync(h->counts, 0, (size_t)(h->ncells + 1) * 4, s));
  if (total > 0) {
    k_cell_keys<<<(unsigned)(((int64_t)total + 255) / 256), 256, 0, s>>>(h->cell[o], total, my, nullptr, h->counts);
    CKLAUNCH("k_cell_keys");
  }
  CK(cudaMemcpyAsync(h->off, h->counts, (size_t)(h->ncells + 1) * 4, cudaMemcpyDeviceToDevice, s));
  TRY(scan_excl(s, h->off, h->ncells + 1, h->scan_scratch));
  k_tile_off<<<grid_for(h->ntiles + 1, 256, 1 << 20), 256, 0, s>>>(h->off, h->ntiles, h->tpc, h->TY, my, total,
                                                                  h->tile_off);
  CKLAUNCH("k_tile_off");
  h->sorted = true;
  h->hist_valid = false;
  return PBPIC_OK;
}

template <class T, bool MIXED>
int do_field_rows(pbpic_handle* h, int j0, int nrows, void* buf, bool set) {
  if (j0 < 0 || nrows < 0 || j0 + nrows > h->S) return fail(PBPIC_EINVAL, "field rows outside 0..my");
  if (nrows == 0) return PBPIC_OK;
  if (!buf) return fail(PBPIC_EINVAL, "null buffer");
  Planes6<T> p;
  for (int c = 0; c < 6; ++c) p.f[c] = (T*)h->f[c];
  const int g = grid_for((int64_t)6 * h->cfg.mx * nrows, 256);
  if (set) {
    k_rows_set<T><<<g, 256, 0, h->stream>>>(p, h->cfg.mx, h->S, j0, nrows, (const T*)buf);
    CKLAUNCH("k_rows_set");
    // Node row b averages field rows b - 1 and b, so the rows set feed node
    // rows [j0, j0 + nrows]; with periodic y node row my repeats node row 0.
    const int my = h->cfg.my;
    const int b0 = std::max(0, (int)j0), b1 = std::min(my + 1, (int)(j0 + nrows + 1));
    TRY((node_rows<T, MIXED>(h, b0, b1)));
    if (h->cfg.ybc == PBPIC_BC_PERIODIC) {
      if (b0 == 0) TRY((node_rows<T, MIXED>(h, my, my + 1)));
      if (b1 == my + 1) TRY((node_rows<T, MIXED>(h, 0, 1)));
    }
  } else {
    k_rows_get<T><<<g, 256, 0, h->stream>>>(p, h->cfg.mx, h->S, j0, nrows, (T*)buf);
    CKLAUNCH("k_rows_get");
  }
  CK(cudaStreamSynchronize(h->stream));
  return PBPIC_OK;
}

template <class T, bool MIXED>
int do_energies_rows(pbpic_handle* h, int y_lo, int y_hi, int wall_lo, int wall_hi, double* out) {
  TRY(materialize(h));
  const pbpic_config& c = h->cfg;
  if (y_lo < 0 || y_hi > h->S || y_lo > y_hi) return fail(PBPIC_EINVAL, "rows outside 0..my");
  cudaStream_t s = h->stream;
  const int b = h->cur;
  k_kinetic_rows<T, MIXED><<<h->nke, 256, 0, s>>>(h->n, h->cell[b], P<T>(h, b, 2), P<T>(h, b, 3), P<T>(h, b, 4),
                                                   (T)c.mime, y_lo, std::min(y_hi, c.my), h->ke_part);
  CKLAUNCH("k_kinetic_rows");
  k_field_energy_rows<T><<<h->nfe, 256, 0, s>>>(c.mx, c.my, (const T*)h->ng, y_lo, y_hi, wall_lo, wall_hi,
                                               h->fe_part);
  CKLAUNCH("k_field_energy_rows");
  k_energy_row<<<1, 256, 0, s>>>(h->ke_part, h->nke, h->fe_part, h->nfe, fe_scale(c), fb_scale(c), h->dscalar);
  CKLAUNCH("k_energy_row");
  CK(cudaMemcpyAsync(out, h->dscalar, 4 * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return PBPIC_OK;
}

}  // namespace

extern "C" {

int pbpic_band_extract(pbpic_handle* h, int32_t y_lo, int32_t y_hi, int32_t my_global, int32_t row_offset,
                       void* dst_dev, int64_t cap, int64_t* n) {
  TRY(check_handle(h));
  if (y_lo < 0 || y_hi > h->cfg.my || y_lo > y_hi || my_global < 1) return fail(PBPIC_EINVAL, "bad band rows");
  return DISPATCH(h, do_band_extract, h, y_lo, y_hi, my_global, row_offset, dst_dev, cap, n);
}

int pbpic_band_keep(pbpic_handle* h, int32_t y_lo, int32_t y_hi) {
  TRY(check_handle(h));
  if (y_lo < 0 || y_hi > h->cfg.my || y_lo > y_hi) return fail(PBPIC_EINVAL, "bad band rows");
  return DISPATCH(h, do_band_keep, h, y_lo, y_hi);
}

int pbpic_band_append(pbpic_handle* h, const void* src_dev, int64_t n, int32_t my_global, int32_t row_offset) {
  TRY(check_handle(h));
  if (my_global < 1) return fail(PBPIC_EINVAL, "bad global row count");
  return DISPATCH(h, do_band_append, h, src_dev, n, my_global, row_offset);
}

int pbpic_band_replace(pbpic_handle* h, int32_t y_lo, int32_t y_hi, const void* bottom_dev, int64_t nb,
                       int32_t off_bottom, const void* top_dev, int64_t nt, int32_t off_top, int32_t my_global) {
  TRY(check_handle(h));
  if (y_lo < 0 || y_hi > h->cfg.my || y_lo > y_hi || my_global < 1) return fail(PBPIC_EINVAL, "bad band rows");
  return DISPATCH(h, do_band_replace, h, y_lo, y_hi, bottom_dev, nb, off_bottom, top_dev, nt, off_top, my_global);
}

int pbpic_field_rows_get(pbpic_handle* h, int32_t j0, int32_t nrows, void* dst_dev) {
  TRY(check_handle(h));
  return DISPATCH(h, do_field_rows, h, j0, nrows, dst_dev, false);
}

int pbpic_field_rows_set(pbpic_handle* h, int32_t j0, int32_t nrows, const void* src_dev) {
  TRY(check_handle(h));
  return DISPATCH(h, do_field_rows, h, j0, nrows, const_cast<void*>(src_dev), true);
}

int pbpic_energies_rows(pbpic_handle* h, int32_t y_lo, int32_t y_hi, int32_t wall_lo, int32_t wall_hi, double* out) {
  TRY(check_handle(h));
  if (!out) return fail(PBPIC_EINVAL, "null argument");
  return DISPATCH(h, do_energies_rows, h, y_lo, y_hi, wall_lo, wall_hi, out);
}

}  // extern "C"
