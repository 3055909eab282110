/*
 * pbpic.h -- C ABI of the B200 implementation of pbpic's 2-D electromagnetic
 * particle-in-cell time step (xiaocanli/pbpic, src/programs/pic2d.f90).
 *
 * The reference's step boundary is three argument-less Fortran subroutines
 * acting on module globals of `module parameters` (pic2d.f90:4-142):
 *     call pusher        (pic2d.f90:177, body 912-1217)
 *     call fieldsolver   (pic2d.f90:178, body 678-860)
 *     call countingsort  (pic2d.f90:161, 181, body 1303-1329)
 * Here the globals become a handle that owns the device state, and each
 * subroutine becomes one call. Every function returns 0 on success or a
 * negative PBPIC_E* code; pbpic_last_error() describes the last failure of the
 * calling thread. Calls are stream-ordered on the handle's stream (default:
 * the legacy default stream) and a handle must be used by one host thread at a
 * time. No type in these signatures depends on CUDA or PyTorch.
 *
 * Units follow the reference: lengths in ion inertial lengths d_i, time in
 * 1/Omega_ci, velocities in v_A, momenta u = gamma v / c, B in B0, E in v_A B0
 * (pic2d.f90:15-43, 969-1006).
 */
#ifndef PBPIC_H
#define PBPIC_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ----------------------------------------------------------------- errors */
#define PBPIC_OK 0
#define PBPIC_EINVAL (-1)    /* bad argument or configuration */
#define PBPIC_ECUDA (-2)     /* a CUDA call failed */
#define PBPIC_ENOMEM (-3)    /* device allocation failed */
#define PBPIC_ECAPACITY (-4) /* more particles than the handle's capacity */
#define PBPIC_ESTATE (-5)    /* call not valid in the handle's current state */

/* ------------------------------------------------------- configuration */
#define PBPIC_BC_PERIODIC 0   /* y periodic: the reference on one MPI rank (pic2d.f90:294-304) */
#define PBPIC_BC_CONDUCTING 1 /* y conducting walls: reflection + PEC (not in the reference) */

#define PBPIC_FP64_PLAIN 0 /* FP64 throughout; the drop-in form */
#define PBPIC_FP32_MIXED 1 /* FP32 push/deposit/FDTD, int64 fixed-point current, FP64 energies */

/* Reproduce reference quirks bit for bit (default: corrected behaviour). */
#define PBPIC_COMPAT_BORIS 1 /* rotate the pre-kick momentum (pic2d.f90:985-987) */
#define PBPIC_COMPAT_FOLD 2  /* drop jy deposited in column mx+2 (fold commented, pic2d.f90:1156) */
#define PBPIC_COMPAT_RHO 4   /* mirrored CIC weights for rho (pic2d.f90:1285-1295) */

/* Device status bits reported by pbpic_status(). */
#define PBPIC_STATUS_CELL_JUMP 1 /* a particle moved more than one cell in a step (pic2d.f90:1008-1023 assumes at most one) */
#define PBPIC_STATUS_NAN 2       /* a momentum became NaN or infinite */
#define PBPIC_STATUS_UNSORTED 4  /* a push met a particle outside its tile (informational) */
#define PBPIC_STATUS_BAD_RECORD 8   /* a band record fell outside this domain's rows (pbpic_band_replace) */
#define PBPIC_STATUS_COPY_TIMEOUT 16 /* a push's bulk copy of a tile's gather records or node columns did not land within its bounded wait (the push then read them from global memory) */

typedef struct pbpic_config {
  int32_t mx, my;      /* cells in x and y (nx, ny of pic2d.f90:12; one domain) */
  double dx, dy;       /* cell size, d_i (pic2d.f90:15) */
  double dt;           /* time step, 1/Omega_ci (pic2d.f90:42) */
  double cva;          /* c / v_A (pic2d.f90:20) */
  double mime;         /* m_i / m_e (pic2d.f90:19) */
  double in0;          /* 1 / (macro-particles per cell at density n0) (pic2d.f90:31) */
  int32_t ybc;         /* PBPIC_BC_* */
  int32_t precision;   /* PBPIC_FP64_PLAIN or PBPIC_FP32_MIXED */
  int32_t compat;      /* PBPIC_COMPAT_* bits */
  int32_t track_pid;   /* nonzero: carry the reference's per-particle pid through the step */
  int64_t capacity;    /* maximum number of particles (both species) */
  int32_t tile_rows;   /* cells per push tile along y (0: default) */
  int32_t options;     /* PBPIC_OPT_* bits */
} pbpic_config;

/* By default every push ends with the particles sorted by cell (the fused
 * counting sort from the push's own tile histograms, right after it): the
 * push needs cell-sorted tiles to run fast, so sorting every step costs less
 * than the push would lose on unsorted particles (at 1024x512 cells and 105 M
 * particles: 3.9 ms per step sorting every step, 13 ms with the reference's
 * sort every 50 steps). pbpic_sort on sorted particles does nothing. This
 * option leaves the sort to the caller, as the reference's pusher does. */
#define PBPIC_OPT_NO_AUTOSORT 1
/* Plain form only: evaluate the push's square roots and quotients correctly
 * rounded in the reference's order (pic2d.f90:969-1028), so that the particle
 * state after a step is bit-identical to an FP64 evaluation of the reference's
 * expressions. Without it 1/gamma comes from a reciprocal square root and the
 * state agrees with that evaluation to a few ulp (1e-15 relative), faster.
 * Any compat switch implies it. */
#define PBPIC_OPT_EXACT_FP64 2

/* The reference's `type particle` (pic2d.f90:47-50): 32 bytes. grid is the
 * 1-based cell my*(ix-1)+iy (y fastest), dx, dy the offset from the cell
 * centre in [-0.5, 0.5], q = +1 (ion) or -1 (electron). */
typedef struct pbpic_particle_f32 {
  float dx, dy, ux, uy, uz;
  int32_t grid, q, pid;
} pbpic_particle_f32;

/* The same record with double-precision reals (56 bytes with padding). */
typedef struct pbpic_particle_f64 {
  double dx, dy, ux, uy, uz;
  int32_t grid, q, pid, pad;
} pbpic_particle_f64;

/* Seeded plasma loader (the reference loads a double Harris sheet from
 * /dev/urandom, pic2d.f90:357-578; these loaders are seeded Philox4x64-10). */
#define PBPIC_LOAD_UNIFORM 0    /* uniform Maxwellian, ppc pairs in every cell, uniform Bz = b0z */
#define PBPIC_LOAD_HARRIS 1     /* GEM Harris sheet along y with background, psi0 perturbation */
#define PBPIC_LOAD_TWO_STREAM 2 /* counter-drifting electron beams along x */
#define PBPIC_LOAD_WEIBEL 3     /* electrons with T_perp / T_par = anisotropy */
/* The reference's own plasma (initparticles and initfields, pic2d.f90:357-648):
 * two current sheets normal to x at Lx/4 and 3Lx/4 (half-thickness lambda) on a
 * background nb, By = tanh((x - Lx/4)/lambda) - tanh((x - 3Lx/4)/lambda) - 1;
 * sheet pairs drift along z at vdrift_i / vdrift_e in the first sheet and the
 * opposite in the second, with thermal spread in x and y only (vthe, vthi);
 * background pairs have vthe_bg, vthi_bg in x and y and no z motion. */
#define PBPIC_LOAD_DOUBLE_HARRIS 4

typedef struct pbpic_loader {
  int32_t kind;
  int32_t ppc;          /* macro-particles per cell per species (average) */
  double vthe, vthi;    /* thermal speeds / c (electron, ion) */
  double vdrift_e;      /* electron drift / c: Harris along z, two-stream beams along +-x */
  double vdrift_i;      /* ion drift / c (Harris, along z) */
  double lambda;        /* Harris half-thickness, d_i */
  double nb;            /* Harris background density / n0 */
  double psi0;          /* GEM perturbation, B0 d_i */
  double bguide;        /* Harris guide field Bz, B0 */
  double b0z;           /* uniform Bz of the other loaders, B0 */
  double anisotropy;    /* Weibel T_perp / T_par */
  uint64_t seed;
  int32_t immobile_ions; /* nonzero: load electrons only (a fixed neutralising ion background) */
  int32_t reserved;
  double vthe_bg, vthi_bg; /* double Harris: background thermal speeds / c */
} pbpic_loader;

typedef struct pbpic_handle pbpic_handle;

/* ------------------------------------------------------------ lifecycle */
/* Replaces the allocation part of `init` (pic2d.f90:197-308). */
int pbpic_create(const pbpic_config* cfg, pbpic_handle** out);
int pbpic_destroy(pbpic_handle* h);
const char* pbpic_last_error(void);
/* Stream for all subsequent work of the handle (a cudaStream_t passed as void*). */
int pbpic_set_stream(pbpic_handle* h, void* stream);
int pbpic_get_config(const pbpic_handle* h, pbpic_config* out);

/* ------------------------------------------------------------- loading */
/* Seeded loading of particles and initial fields; replaces initparticles and
 * initfields (pic2d.f90:357-648). Leaves the particles sorted by cell. */
int pbpic_init_plasma(pbpic_handle* h, const pbpic_loader* ld);
/* Number of particles a loader produces for this handle's grid. */
int pbpic_loader_count(const pbpic_handle* h, const pbpic_loader* ld, int64_t* n);

/* Particles in the reference's record (ptl, pic2d.f90:70). Host buffers. */
int pbpic_load_particles_f32(pbpic_handle* h, const pbpic_particle_f32* p, int64_t n);
int pbpic_load_particles_f64(pbpic_handle* h, const pbpic_particle_f64* p, int64_t n);
int pbpic_store_particles_f32(pbpic_handle* h, pbpic_particle_f32* p, int64_t cap, int64_t* n);
int pbpic_store_particles_f64(pbpic_handle* h, pbpic_particle_f64* p, int64_t cap, int64_t* n);
/* Structure-of-arrays variants (host buffers); q[] holds +1 / -1; pid may be NULL. */
int pbpic_load_particles_soa_f64(pbpic_handle* h, int64_t n, const int32_t* grid, const int32_t* q,
                                 const double* dx, const double* dy, const double* ux,
                                 const double* uy, const double* uz, const int32_t* pid);
int pbpic_store_particles_soa_f64(pbpic_handle* h, int64_t cap, int64_t* n, int32_t* grid, int32_t* q,
                                  double* dx, double* dy, double* ux, double* uy, double* uz,
                                  int32_t* pid);
int pbpic_num_particles(const pbpic_handle* h, int64_t* n);

/* Primary Yee fields, host buffer of 6 planes (ex, ey, ez, bx, by, bz), each
 * mx x (my+1) values with y fastest; entry (i, j) is the reference's
 * emf(i+1, j+1) (pic2d.f90:71). Row my is used only for the node-row
 * components (ex, bx) with conducting walls. Loading recomputes the node
 * averages (emfgrid) and the field energy. */
int pbpic_load_fields_f64(pbpic_handle* h, const double* yee6);
int pbpic_store_fields_f64(pbpic_handle* h, double* yee6);
/* emfgrid (pic2d.f90:72) nodes 1..mx+1 x 1..my+1: (mx+1) x (my+1) x 8 values,
 * record (ex, ey, ez, 0, bx, by, bz, 0), y fastest. */
int pbpic_store_emfgrid_f64(pbpic_handle* h, double* grid8);
/* denjr (pic2d.f90:73) after normalisation by in0 and guard folding, 4 planes
 * (jx, jy, jz, rho) of mx x (my+1), y fastest, as left by the last push. */
int pbpic_store_denjr_f64(pbpic_handle* h, double* j4);

/* ---------------------------------------------------------------- step */
/* pusher (pic2d.f90:912-1217): zero the current, gather + Boris + move +
 * charge-conserving deposit + x wrap + y wrap or wall reflection + J fold,
 * kinetic energies into the history. */
int pbpic_push(pbpic_handle* h);
/* fieldsolver (pic2d.f90:678-860): B half step, E full step, B half step,
 * node averages, field energies into the history. */
int pbpic_fieldsolve(pbpic_handle* h);
/* countingsort (pic2d.f90:1303-1329): stable sort of the particles by cell. */
int pbpic_sort(pbpic_handle* h);
/* The reference time loop body (pic2d.f90:171-188) nsteps times:
 * push, fieldsolve, and a sort every sort_every steps (0: never). When a
 * step sorts, its field solve runs on a second stream of the library beside
 * the sort, and the handle's stream waits for it (an event) before the next
 * step: the results equal the three calls in order. */
int pbpic_step(pbpic_handle* h, int32_t nsteps, int32_t sort_every);
/* Wait for the handle's stream. */
int pbpic_synchronize(pbpic_handle* h);

/* ---------------------------------------------------------- diagnostics */
/* totene(1:4, itime) of the last completed step (pic2d.f90:122, 653-673,
 * 1055-1062): electron KE, ion KE, electric and magnetic energy in m_e c^2. */
int pbpic_energies(pbpic_handle* h, double out[4]);
/* Energy history rows 0..n-1 (row 0 is the initial state), 4 doubles per row. */
int pbpic_energy_history(pbpic_handle* h, double* out, int32_t max_rows, int32_t* n_rows);
/* Steps completed since loading (itime of pic2d.f90:171). */
int pbpic_time_step(const pbpic_handle* h, int32_t* itime);
/* Per-cell particle counts from the last sort (ptlalloc before the scan,
 * pic2d.f90:1310-1313), mx*my int32 in reference grid order. */
int pbpic_cell_counts(pbpic_handle* h, int32_t* counts);
/* Gauss's law residual max |div E / cva^2 - rho| over interior nodes, with rho
 * the CIC charge density (units of n0 e) of the current particle positions. */
int pbpic_gauss_residual(pbpic_handle* h, double* out);
/* The same over the node rows [y_lo, y_hi) only (a y slab's own rows; its
 * ghost rows hold the neighbours' values). No reference counterpart: the
 * reference has no Gauss diagnostic. */
int pbpic_gauss_residual_rows(pbpic_handle* h, int32_t y_lo, int32_t y_hi, double* out);
/* Reconnected flux: half the sum of |By| along the node row my/2 times dx. */
int pbpic_reconnected_flux(pbpic_handle* h, double* out);
/* Energy spectra (energyspectra, pic2d.f90:1957-1990): counts[0][k-1]
 * electrons and counts[1][k-1] ions with (gamma - 1) ms in ((k-1) de, k de],
 * k = 1..nbins (the reference: de = 0.005 electrons, 0.005 Ti/Te ions, 1000
 * bins). The reference's histogram indexing slip (bin, species) and its bin
 * 0 (quirk Q6) are not reproduced: an energy of 0 counts in bin 1. */
int pbpic_energy_spectra(pbpic_handle* h, double de_electron, double de_ion, int32_t nbins, int64_t* counts);
/* Node values (ex ey ez bx by bz, double) along node rows rows[0..nrows)
 * for all x and node columns cols[0..ncols) for all y, the cuts that
 * dispersioninfo keeps for the field spectra (pic2d.f90:2124-2142):
 * out = [nrows][mx][6] then [ncols][my][6]. Indices 0-based. */
int pbpic_field_cuts(pbpic_handle* h, const int32_t* rows, int32_t nrows, const int32_t* cols, int32_t ncols,
                     double* out);

/* Optional field filters, off by default as in the reference, which defines
 * them and comments out their call after the E update (pic2d.f90:754-755):
 * Marder divergence cleaning (divergenceclean, pic2d.f90:867-886; marder_d
 * is its constant, <= 0 selects the reference's 0.001) and the Cherenkov
 * filter (suppresscerenkov, pic2d.f90:889-907; tau = cerenkov_tau * dt,
 * <= 0 selects the reference's 0.125). Periodic y only. Not applied by the
 * batched form. */
#define PBPIC_FILTER_MARDER 1
#define PBPIC_FILTER_CERENKOV 2
int pbpic_set_field_filters(pbpic_handle* h, int32_t flags, double marder_d, double cerenkov_tau);

/* Device status bits (PBPIC_STATUS_*) accumulated since the last call; clears them. */
int pbpic_status(pbpic_handle* h, int32_t* bits);
/* Number of CUDA kernels this library has launched in the process (all handles). */
int pbpic_kernel_launches(int64_t* count);

/* ----------------------------------------------- stateless counting sort */
/* Stable counting sort of n cell keys in [0, ncells): perm[j] is the index of
 * the j-th key in sorted order and counts[c] the number of keys in cell c
 * (both device pointers). The same algorithm as pbpic_sort, exposed on raw
 * device buffers; allocates its scratch with cudaMalloc on each call.
 * stream is a cudaStream_t passed as void*. Replaces the ordering part of
 * countingsort (pic2d.f90:1303-1329). */
int pbpic_counting_sort_keys(const int32_t* keys_dev, int64_t n, int32_t ncells,
                             int32_t* perm_dev, int32_t* counts_dev, void* stream);

/* The same stable counting sort with no device allocation at all, for callers
 * that cannot call cudaMalloc: host code whose GPU memory is already owned by
 * another allocator (a framework's caching allocator that reserved the device),
 * or a time loop that must not pay for the synchronisation an allocation
 * implies. It has no counterpart in the reference. Its scratch is a static
 * device array inside the library, sized for PBPIC_STATIC_SORT_MAX_KEYS keys
 * (about 17 MB, held on every GPU that loads the library until the process
 * exits); larger n is rejected with PBPIC_ECAPACITY. The first call on a device
 * looks up the array's address and should come before any stream capture.
 * Each call reads the key-range check back to the host, so it returns only
 * after its stream has finished the sort. Calls share the array: calls that
 * overlap on the GPU race. */
#define PBPIC_STATIC_SORT_MAX_KEYS 1048576
int pbpic_counting_sort_keys_static(const int32_t* keys_dev, int64_t n, int32_t ncells,
                                    int32_t* perm_dev, int32_t* counts_dev, void* stream);

/* --------------------------------------------------------- dump / restart */
/* Writes the handle's state to directory `dir` (created if missing) as .npy
 * files named like the datasets of the reference's particle and field dumps
 * (particlesinfo / fieldsinfo, pic2d.f90:1358-1380, 1625-1644; HDF5 there):
 * particles/{dx,dy,ux,uy,uz,grid,q[,pid]}, fields/{ex,ey,ez,bx,by,bz} and
 * fields/{jx,jy,jz,rho} (mx x (my+1)), totene (itime+1 x 4) and state.json.
 * Values keep the handle's precision, so pbpic_restart reproduces the state
 * exactly. */
int pbpic_dump(pbpic_handle* h, const char* dir);
/* Writes the reference's own HDF5 dump files into directory `dir`, with its
 * file names, dataset names, element types (its `real` is 4 bytes) and
 * shapes, so that the reference's readers (restart, python/ and idl/ plots)
 * open them: particles.h5 (particlesinfo, pic2d.f90:1358-1560: dx dy ux uy uz
 * grid q pid of length the capacity, the particles first, and nptlact),
 * fields%05d.h5 for the current step (fieldsinfo, pic2d.f90:1625-1830: ex ey
 * ez bx by bz dive jx jy jz rho num over (0:mx+1, 1:my+1)), spectra.h5
 * (energyinfo, pic2d.f90:2034-2090: a group "%05d" per call so far with
 * "spectra", and "ebins"; bins of de_electron / de_ion, nbins of them; 0
 * selects 0.005, de_electron and 1000) and energy_tot.h5 ("tote"). Written by
 * a self-contained HDF5 writer (no HDF5 library: superblock version 0,
 * contiguous datasets). */
int pbpic_dump_h5(pbpic_handle* h, const char* dir, double de_electron, double de_ion, int32_t nbins);
/* Loads a dump into a handle created with the same mx, my, ybc and precision
 * and enough capacity, sets its time step and energy history, and sorts the
 * particles (stable, so a dump taken right after a sort continues bit for
 * bit). */
int pbpic_restart(pbpic_handle* h, const char* dir);

/* ----------------------------------------------------------------- y slabs */
/* Device-side pieces of the y-slab decomposition, the reference's 1-D domain
 * decomposition along y over MPI ranks (pic2d.f90:206-212; its ghost-row and
 * particle exchanges, pic2d.f90:701-835, 1072-1146). Each rank steps an
 * extended domain (its own rows plus ghost bands of neighbouring rows) and
 * exchanges, after each step, the ghost field rows and the particles of the
 * bands next to its neighbours (pbpic_b200/slab.py drives it). Bands travel
 * as reference particle records of the global grid (pbpic_particle_f32 for
 * the mixed form, _f64 for the plain form) in DEVICE memory: grid =
 * my_global * ix + (local row + row_offset) + 1. */
/* Copies the particles in local rows [y_lo, y_hi) to dst_dev (at most cap
 * records); *n = their number (ECAPACITY when above cap). Order kept. */
int pbpic_band_extract(pbpic_handle* h, int32_t y_lo, int32_t y_hi, int32_t my_global, int32_t row_offset,
                       void* dst_dev, int64_t cap, int64_t* n);
/* Keeps only the particles in local rows [y_lo, y_hi), in their order. */
int pbpic_band_keep(pbpic_handle* h, int32_t y_lo, int32_t y_hi);
/* Appends n records from device memory; local row = global row - row_offset. */
int pbpic_band_append(pbpic_handle* h, const void* src_dev, int64_t n, int32_t my_global, int32_t row_offset);
/* pbpic_band_keep(y_lo, y_hi), then both appends, then a sort, in one pass
 * when the particles are sorted by cell: the bands (device records, each in
 * the cell order band_extract produced) go below (bottom, local row = global
 * row - off_bottom) and above (top) the own rows. Leaves the particles sorted. */
int pbpic_band_replace(pbpic_handle* h, int32_t y_lo, int32_t y_hi, const void* bottom_dev, int64_t nb,
                       int32_t off_bottom, const void* top_dev, int64_t nt, int32_t off_top, int32_t my_global);
/* Rows j0 .. j0+nrows-1 of the six field planes to / from device memory as
 * [6][mx][nrows] values of the handle's precision; setting them recomputes
 * the node averages and the push's gather records that those rows feed (the
 * energy history is not rewritten). */
int pbpic_field_rows_get(pbpic_handle* h, int32_t j0, int32_t nrows, void* dst_dev);
int pbpic_field_rows_set(pbpic_handle* h, int32_t j0, int32_t nrows, const void* src_dev);
/* Energies (electron KE, ion KE, E, B) of the particles in rows [y_lo,
 * y_hi) and of the node rows [y_lo, y_hi); node rows wall_lo and wall_hi
 * (global walls; -1: none) weigh 1/2 as in the conducting-wall sums. */
int pbpic_energies_rows(pbpic_handle* h, int32_t y_lo, int32_t y_hi, int32_t wall_lo, int32_t wall_hi, double* out);

/* ------------------------------------------------------------ batched form */
/* Many independent domains of uneven grid size and particle count advanced
 * together. Every phase of a step runs once for all domains: persistent
 * blocks over one table of (domain, tile) pairs for the push and the
 * scatter of the counting sort, one grid row per domain for the rest. The
 * counting sort runs every step, and pairs of steps are replayed from a
 * captured CUDA graph on the batch's own stream. Domains are FP32 mixed.
 * Tile rows (per domain) and particles per thread are set by hand or by
 * pbpic_batch_autotune. A domain's particles, fields and energies after n
 * batched steps are bit-identical to pbpic_step(h, n, 1) on a handle with
 * the same tile rows and 8 particles per thread. No counterpart in the
 * reference, which runs one domain per MPI job. */
typedef struct pbpic_batch pbpic_batch;
/* Creates the domains and loads them (cfgs[d], loaders[d]); each capacity is
 * raised to the loader's particle count; cfgs[d].tile_rows 0 = default. */
int pbpic_batch_create(const pbpic_config* cfgs, const pbpic_loader* loaders, int32_t ndomains,
                       pbpic_batch** out);
int pbpic_batch_destroy(pbpic_batch* b);
int pbpic_batch_num_domains(const pbpic_batch* b, int32_t* n);
/* The handle of domain d, owned by the batch: any read of the single-domain
 * API works on it (store_particles_*, store_fields_f64, energies,
 * energy_history, gauss_residual, ...). Do not destroy it or set its stream. */
int pbpic_batch_domain(pbpic_batch* b, int32_t d, pbpic_handle** h);
/* tile_rows: one per domain, 0 = default (NULL: all defaults), capped at 64
 * and, with periodic y, at my - 2; groups: particles per thread / 4 (1 or 2). */
int pbpic_batch_set_tiles(pbpic_batch* b, const int32_t* tile_rows, int32_t groups);
int pbpic_batch_get_tiles(const pbpic_batch* b, int32_t* tile_rows, int32_t* groups);
/* Enqueues nsteps steps of every domain on the batch's stream. */
int pbpic_batch_step(pbpic_batch* b, int32_t nsteps);
/* The batch's CUDA stream (a cudaStream_t), for events and ordering. */
int pbpic_batch_stream(const pbpic_batch* b, void** stream);
int pbpic_batch_synchronize(pbpic_batch* b);
/* Times trial_steps steps (real steps of the run: every domain advances) for
 * each candidate tiling (tile rows capped at 16, 32, 64; groups 1, 2), keeps
 * the fastest and reports it. Either output may be NULL. The summation
 * order of the FP32 current, and so its rounding, depends on the tiling. */
int pbpic_batch_autotune(pbpic_batch* b, int32_t trial_steps, int32_t* tile_rows_out, int32_t* groups_out,
                         double* best_ms_per_step);
/* Energies (electron KE, ion KE, E, B) of every domain at its current step, ndomains x 4. */
int pbpic_batch_energies(pbpic_batch* b, double* out);

/* ------------------------------------------------------ differentiable form */
/* Gradients of a time-integrated loss of the GEM Harris sheet with respect to
 * the perturbation amplitude psi0, the background density nb and T_i/T_e, by
 * the discrete adjoint of the step (reverse Boris rotation, deposition adjoint
 * as a gather, field-gather adjoint as a scatter-add, transposed FDTD update),
 * with the particle state checkpointed every checkpoint_every steps and
 * recomputed between checkpoints. The particle set is loaded at the nominal
 * background density nb0; nb enters as the weight nb/nb0 of the background
 * particles, which makes the loss differentiable in nb. No counterpart in the
 * reference (which has no gradients). */
#define PBPIC_LOSS_MAGNETIC 0 /* sum over steps of dt * magnetic field energy */
/* sum over steps of the work the electric field does on the particles,
 * dt * mime / (cva^2 in0) * sum over the Yee grid of J^{n+1/2} . E^n (the
 * current a step deposits against the E it starts from; the rate at which the
 * current drains the field energy in the E update, pic2d.f90:742-744). The
 * reference's own j.E analysis (python/analysis_jdote.py) is a stub. */
#define PBPIC_LOSS_JDOTE 1

typedef struct pbpic_diff_config {
  int32_t mx, my;       /* cells; conducting walls in y, periodic in x */
  int32_t ppc;          /* macro-particles per cell per species */
  int32_t precision;    /* PBPIC_FP64_PLAIN or PBPIC_FP32_MIXED (FP32 forward, FP64 loss and adjoint sums) */
  double dx;            /* cell size (d_i), dy = dx */
  double mime, wpe_wce; /* mass ratio, omega_pe / omega_ce */
  double lambda, nb0;   /* sheet half-thickness (d_i), nominal background density */
  double cfl;           /* c dt sqrt(1/dx^2 + 1/dy^2) */
  int32_t nsteps, checkpoint_every, loss, reserved;
  uint64_t seed;
} pbpic_diff_config;

typedef struct pbpic_diff_params {
  double psi0;  /* GEM perturbation, B0 d_i */
  double nb;    /* background density / n0 */
  double ti_te; /* ion to electron temperature ratio */
} pbpic_diff_params;

typedef struct pbpic_diff pbpic_diff;
int pbpic_diff_create(const pbpic_diff_config* cfg, pbpic_diff** out);
int pbpic_diff_destroy(pbpic_diff* d);
/* Load the sheet for `params`, run nsteps keeping checkpoints, return the loss. */
int pbpic_diff_forward(pbpic_diff* d, const pbpic_diff_params* params, double* loss);
/* d loss / d (psi0, nb, ti_te) at the parameters of the last forward call. */
int pbpic_diff_backward(pbpic_diff* d, double grad[3]);

#ifdef __cplusplus
}
#endif
#endif /* PBPIC_H */
