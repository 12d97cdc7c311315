/*
 * mhit_b200.h -- C ABI of libmhit_b200.so, a B200 (sm_100a) implementation of the MHIT36
 * timestep loop (aroccon/MHIT36_mixedp, multi/main.f90:456-1042) on one GPU.
 *
 * The reference has no operator API: its hot path is the inline body of `do t=tstart,tfin`
 * in program main, acting on module arrays (multi/module.f90:51-71) and `param` scalars
 * (multi/module.f90:1-19, set by multi/readinput.f90:14-49).  Each entry point below names the
 * block of that loop (or of its setup / I/O) it replaces, so a Fortran host can call it through
 * ISO_C_BINDING in place of the loop body (see the bind(C) module in
 * mhit36_mixedp_b200/fortran/mhit_gpu.f90).
 *
 * Conventions
 *   - Arrays cross the boundary as host pointers to x-fastest (nx, ny, nz) float64 arrays with
 *     no halo: Fortran u(1:nx, 2:ny+1, 2:nz+1) of the reference, the layout of its field files
 *     (multi/readwrite.f90:28-46).
 *   - Every function returns an int status: MHIT_OK (0) or a negative MHIT_ERR_* code.  The
 *     library never calls exit(); mhit_last_error() describes the last failure of the calling
 *     thread.
 *   - One context = one box on one GPU with its own CUDA stream.  The library owns all device
 *     memory; host pointers are borrowed only for the duration of a call.  Calls on one
 *     context must not overlap; different contexts are independent.
 */
#ifndef MHIT_B200_H
#define MHIT_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define MHIT_ABI_VERSION 1

/* status codes */
#define MHIT_OK 0
#define MHIT_ERR_ARG (-1)      /* bad argument, unsupported size */
#define MHIT_ERR_CUDA (-2)     /* CUDA runtime failure (message in mhit_last_error) */
#define MHIT_ERR_NAN (-3)      /* NaN in the velocity (the reference has no such check) */
#define MHIT_ERR_CFL (-4)      /* CFL > 7 after a step: the reference stops (multi/main.f90:1006) */
#define MHIT_ERR_IO (-5)       /* file missing, short read or write */
#define MHIT_ERR_STATE (-6)    /* call out of order (e.g. particles on a context without them) */
#define MHIT_ERR_TIMEOUT (-7)  /* a bounded wait inside a kernel ran out (tensor-core z solve) */

/* Poisson precision (multi/main.f90:844,853-912) */
#define MHIT_POISSON_FP64 0    /* the intended FP64 solve of the main branch */
#define MHIT_POISSON_FP32 1    /* this branch: rhs cast to FP32, FP32 transforms, FP32 pressure */
#define MHIT_POISSON_FP32_REFINED 2 /* FP32 solve + one FP64 residual sweep (needs MHIT_LAP_MODIFIED):
                                       r = rhs - L_h p32 in FP64, L_h d = r in FP32, p = p32 + d */
#define MHIT_POISSON_FP32_INCREMENTAL 3 /* one FP32 solve for the increment over the previous
                                       step's pressure q (needs MHIT_LAP_MODIFIED): r = rhs - L_h q
                                       in FP64, L_h d = r in FP32, p = q + d in FP64 for the
                                       projection, q <- fl32(p) for the next step; q = 0 after an
                                       upload or an initial-condition call */

/* Laplacian symbol of the spectral divide */
#define MHIT_LAP_EXACT 0       /* exact integer k^2, as multi/main.f90:889 */
#define MHIT_LAP_MODIFIED 1    /* (2-2cos(k dx))/dx^2: discrete divergence ~ round-off */

/* tracer interpolation */
#define MHIT_INTERP_LINEAR1D 0 /* per-component 1-D linear, multi/particles.f90:114-117 */
#define MHIT_INTERP_TRILINEAR 1

/* Parameters: the 18 values of input.inp (multi/readinput.f90:14-35) that act on a step,
 * plus the grid size (compile-time `nx` in multi/module.f90:2) and the feature switches
 * (compile-time phiflag/partflag in multi/main.f90:55,57). */
typedef struct mhit_params {
  int nx, ny, nz;            /* each in {16,32,64,128,192,256,512,1024} */
  double dt, mu, rho;        /* input.inp lines 7-9 */
  double f1, f2, f3, k0;     /* ABC forcing, lines 10-13 */
  double radius, sigma, epsr;/* phase field, lines 14-16 */
  int phiflag;               /* 1: ACDI phase field on */
  int partflag;              /* 1: tracers on */
  int npart;                 /* number of tracers (line 17) */
  int poisson;               /* MHIT_POISSON_* */
  int laplacian;             /* MHIT_LAP_* */
  int interp;                /* MHIT_INTERP_* */
  int yz_shift;              /* 1: the reference's labelling of y/z planes (forcing/tracers) */
  int use_graph;             /* 1: replay steps from a captured CUDA graph */
  int device;                /* CUDA device ordinal */
  int acdi_clamp;            /* 0: reference psi (phi < -1e-16 gives NaN, multi/main.f90:527-528);
                                1: phi also clamped below at 0 before the log (opt-in deviation) */
  int zsolve_tc;             /* 1: the 512-point z solve of the FP32 modes as BF16x3 split DFT-matrix
                                GEMMs on the tensor cores (needs nz = 512 and a FP32 Poisson mode) */
} mhit_params;

/* Run control lines of input.inp (multi/readinput.f90:14-19, 34-35). */
typedef struct mhit_run {
  int restart, tstart, tfin, dump, inflow, inphi, inpart;
} mhit_run;

typedef struct mhit_diag {
  long long nstep;           /* steps taken by this context */
  double gumax;              /* signed max of u,v,w after the last step (multi/main.f90:1001) */
  double cfl;                /* gumax*dt/dx (multi/main.f90:1003) */
  double mean[3];            /* mean of u,v,w removed by the last projection (:967-981) */
  double maxdiv;             /* max |div u| of the current field (1/dx units) */
  double ke;                 /* 0.5 <u.u> */
  double dissipation;        /* 2 nu <S_ij S_ij>, post/compute_diss/main.f90:72-117, solver dx */
  int flags;                 /* bit0 NaN seen, bit1 CFL > 7 */
} mhit_diag;

typedef struct mhit_ctx mhit_ctx;

/* Library identification and the last error text of the calling thread. */
int mhit_abi_version(void);
const char* mhit_last_error(void);

/* Defaults: nx=ny=nz=64, reference input.inp values (multi/input.inp), FP64 Poisson,
 * exact k^2, linear1d, yz_shift=1, use_graph=1, device 0. */
int mhit_params_default(mhit_params* p);

/* Parse an input.inp file (positional, one value per line, Fortran list-directed reals such
 * as 1.0d0 accepted).  Replaces subroutine readinput (multi/readinput.f90:4-81).  Grid size
 * and switches in *p are left untouched; run may be NULL. */
int mhit_read_input(const char* path, mhit_params* p, mhit_run* run);

/* Allocate a context on p->device: fields, spectrum, tables (setup of multi/main.f90:186-310
 * without MPI/cuDecomp).  Fields start at zero, gumax=1 and the first step is Euler
 * (multi/main.f90:440-444). */
int mhit_init(const mhit_params* p, mhit_ctx** out);
void mhit_destroy(mhit_ctx* ctx);

/* Set the state (replaces the initial-condition block multi/main.f90:322-415 and readfield).
 * u,v,w: required.  phi: required iff phiflag.  Resets rhs_o, rhsphi_o, the mean, gumax=1 and
 * the Euler first step. */
int mhit_upload_fields(mhit_ctx* ctx, const double* u, const double* v, const double* w, const double* phi);

/* Initial conditions built on the device (the O(N^3) work of multi/main.f90:322-415 and of the
 * seeded benchmark fields; the one-dimensional tables are computed on the host).
 *
 * mhit_init_taylor_green: u = sin(x - dx/2) cos(y) cos(z), v = -cos(x) sin(y - dx/2) cos(z),
 *   w = 0 on the accumulated coordinates x(i) = x(i-1) + dx with the y/z labelling of
 *   yz_shift (multi/main.f90:210-214, 324-337).  Replaces u, v, w.
 * mhit_init_velocity_modes: u = Re sum_m c_m exp(i (m_x tx + m_y ty + m_z tz)) over the index
 *   wavenumbers -kmax..kmax per axis (kmax 1..16), with the index phases tx = i 2pi/nx,
 *   ty = (j + yz_shift) 2pi/ny, tz = (k + yz_shift) 2pi/nz and each component's own phase half a
 *   cell back (its face position: u at tx - pi/nx, ...), then scaled to the given rms.  In a
 *   cube the phases are the coordinates; in a box of nx dx by ny dx by nz dx the index
 *   wavenumber m_y is the physical m_y nx/ny.  modes holds 3 (2kmax+1)^3 complex amplitudes as
 *   (re, im) pairs, ordered [component][kz][ky][kx] with m from -kmax; the caller draws them (a
 *   seeded random solenoidal field: Gaussian amplitudes with k.c = 0).  Replaces u, v, w.
 * mhit_init_drops: phi = 0.5 (1 - tanh((r - radius)/(2 eps))), eps = epsr dx, r the periodic
 *   minimum-image distance in the box nx dx by ny dx by nz dx to the nearest of ndrops centres
 *   (x, y, z triples), cells at x = i dx, y = (j + yz_shift) dx, z = (k + yz_shift) dx; one
 *   centre at (pi, pi, pi) is the centred drop of multi/main.f90:370-382.  Replaces phi (needs
 *   phiflag = 1); the velocity keeps its values.
 * Each resets rhs_o, rhsphi_o, gumax = 1 and the Euler first step like mhit_upload_fields and
 * keeps the fields it does not replace; after an error return the fields it would have replaced
 * are undefined (upload or initialise them again). */
int mhit_init_taylor_green(mhit_ctx* ctx);
int mhit_init_velocity_modes(mhit_ctx* ctx, int kmax, const double* modes, double rms);
int mhit_init_drops(mhit_ctx* ctx, int ndrops, const double* centres, double radius);
/* The tracer table of particlegenerator (multi/particles.f90:37-76, inflag = 1) built on the
 * device: tags 1..npart, positions uniform in the box (2 pi by ny dx by nz dx), all velocities
 * and histories zero.  The reference draws from an unseeded RANDOM_NUMBER; here coordinate a
 * (0 x, 1 y, 2 z) of tracer i (0-based) is L_a * (top 53 bits of
 * splitmix64(seed + (3 i + a + 1) * 0x9E3779B97F4A7C15)) / 2^53, reproducible from the seed.
 * Replaces the table like mhit_upload_particles (needs partflag = 1). */
int mhit_init_particles(mhit_ctx* ctx, int npart, unsigned long long seed);

/* Tracer table, column-major (npart, 12) as the reference's part(nplocmax,12)
 * (multi/particles.f90:11-22): tag, x, y, z, u, v, w, phi, u1, v1, w1, phi1. */
int mhit_upload_particles(mhit_ctx* ctx, const double* part, int npart);
int mhit_download_particles(mhit_ctx* ctx, double* part, int npart);

/* Advance nsteps timesteps (one pass of multi/main.f90:456-1007 each).  Returns MHIT_ERR_CFL
 * or MHIT_ERR_NAN if the device flags were raised by any of these steps (checked once at the
 * end of the call). */
int mhit_step(mhit_ctx* ctx, int nsteps);

/* Copy the current state to host arrays (any pointer may be NULL).  u,v,w carry the mean
 * removal of multi/main.f90:977-981; p is the pressure of the last solve widened to FP64. */
int mhit_download_fields(mhit_ctx* ctx, double* u, double* v, double* w, double* p, double* phi);

/* Scalars of the last step plus max|div|, KE and dissipation of the current field. */
int mhit_diagnostics(mhit_ctx* ctx, mhit_diag* d);

/* Field files in the layout of multi/readwrite.f90 (raw float64, x fastest, no header).
 * fieldn: 1 u, 2 v, 3 w, 4 p, 5 phi (multi/readwrite.f90:21-25).
 * mhit_write_field writes <dir>/<name>_%08d.dat (writefield, :1-96); mhit_read_field reads
 * the file at path into field fieldn (readfield/readfield_restart, :107-318). */
int mhit_write_field(mhit_ctx* ctx, const char* dir, int t, int fieldn);
int mhit_read_field(mhit_ctx* ctx, const char* path, int fieldn);

/* Shell-summed kinetic-energy spectrum of the current velocity (no reference counterpart; the
 * reference's post-processing has dissipation and 1-D profiles only):
 *   E[k] = 1/2 sum over |kappa| in [k - 1/2, k + 1/2) of |u_kappa|^2 + |v_kappa|^2 + |w_kappa|^2,
 * u_kappa the FFT of the stored velocity (mean removed) divided by nx ny nz, kappa in units of
 * 2 pi / Lx (kappa_y = m_y nx/ny, kappa_z = m_z nx/nz), for k = 0..nbins-1 (nbins 1..4096).
 * Shells beyond nbins are dropped; with all shells, sum E = KE of mhit_diagnostics (Parseval).
 * Uses the FP64 transform passes of the Poisson solver (in the FP32 modes on an FP64 buffer
 * allocated on first use); the last bits depend on the order of shared-memory atomics. */
int mhit_energy_spectrum(mhit_ctx* ctx, double* E, int nbins);

/* Exact-resume checkpoint (no reference counterpart: the reference restarts from the field
 * files, multi/readwrite.f90:107-318, with an Euler step because rhs_o is not in them,
 * multi/main.f90:440-441).  The file holds everything the next step reads: u, v, w as stored
 * with the lazily removed mean, phi, rhs_o of u, v, w and phi, the pressure in the Poisson
 * precision, the device scalars (mean, gumax of the previous projection), the step count and the
 * tracer table; stepping a context that read it gives the same bits as never stopping.
 * mhit_read_checkpoint needs a context created with the same nx, ny, nz, phiflag, partflag and
 * Poisson mode (MHIT_ERR_ARG otherwise; MHIT_ERR_IO for a missing, short or foreign file).  A
 * read that fails after the header leaves the context's fields undefined: upload or read again. */
int mhit_write_checkpoint(mhit_ctx* ctx, const char* path);
int mhit_read_checkpoint(mhit_ctx* ctx, const char* path);

/* Droplet labelling (post/unionfind_periodic/main.f90): connected components of
 * phi >= thresh (the reference uses 0.5) with periodic boundaries, connectivity 6 (faces) or 26
 * (faces, edges, corners), and per drop the cell count, volume = cells dx^3, the centre as the
 * circular mean of the cell centres per axis in [0, L) and the mean of the stored u, v, w over
 * its cells (:276-336, :425-436).  Drops are numbered by their smallest cell index (k, j, i).
 * Fills min(maxdrops, total) entries of drops and sets *ndrops = total; labels (may be NULL)
 * receives the label field (0 background, 1..total), x fastest.  Needs phiflag = 1. */
typedef struct {
  long long cells;
  double volume;
  double x, y, z;
  double u, v, w;
} mhit_drop;
int mhit_label_drops(mhit_ctx* ctx, double thresh, int connectivity, mhit_drop* drops, int maxdrops, int* ndrops,
                     int* labels);

/* Measurement helpers (no reference counterpart; the reference times with cpu_time,
 * multi/main.f90:453,463,1009-1010).  mhit_time_steps runs nsteps on the context stream between
 * two CUDA events and returns the elapsed milliseconds.  mhit_profile_step runs one step with
 * an event pair around each kernel launch and returns per-stage milliseconds; names (may be
 * NULL) receives static strings; *nstages is in/out (capacity / count). */
int mhit_time_steps(mhit_ctx* ctx, int nsteps, double* ms);
int mhit_profile_step(mhit_ctx* ctx, double* ms, const char** names, int* nstages);
/* Number of kernels one step after the first launches: the kernel nodes of the captured step
 * graph (captured here if no step has needed it yet). */
int mhit_kernels_per_step(mhit_ctx* ctx, int* n);

/* Ensemble of independent boxes of uneven sizes (the reference runs one box per job; this is
 * the batched mode of its timestep loop).  Every box is a full context -- upload, download,
 * diagnostics and field files go through mhit_ensemble_box() and the single-box calls -- but
 * the boxes advance together: mhit_ensemble_step runs each step after the first as ONE CUDA
 * graph launch whose graph forks the boxes' step sequences onto concurrent streams ("lanes")
 * and joins them.  All boxes must be at the same step (upload all, then step all).
 * In the batched schedule (the default when every box has the same phiflag and acdi_clamp) the
 * phase and momentum stages of all boxes run as one persistent launch each, whose blocks take
 * (box, tile, z chunk) items from a device work queue; the Poisson passes and the projection of
 * each box follow on the lanes.  Both schedules give the same bits.
 * mhit_ensemble_autotune times the z-chunk of the phase and momentum kernels per box size and
 * the number of lanes, then the batched schedule with uniform z chunks, keeps the fastest, and
 * leaves every box zeroed: call it before the uploads.  mhit_ensemble_tuning reports the choices
 * (arrays of nbox ints, may be NULL); mhit_ensemble_batched reports the schedule and
 * mhit_ensemble_set_batched chooses it (1: batched, 0: per-box lanes). */
typedef struct mhit_ensemble mhit_ensemble;
int mhit_ensemble_create(const mhit_params* params, int nbox, mhit_ensemble** out);
void mhit_ensemble_destroy(mhit_ensemble* e);
int mhit_ensemble_box(mhit_ensemble* e, int b, mhit_ctx** ctx);
int mhit_ensemble_step(mhit_ensemble* e, int nsteps);
int mhit_ensemble_time_steps(mhit_ensemble* e, int nsteps, double* ms);
int mhit_ensemble_autotune(mhit_ensemble* e, int trials, int* nlanes);
int mhit_ensemble_tuning(mhit_ensemble* e, int* nlanes, int* zchunk_phase, int* zchunk_mom);
int mhit_ensemble_batched(mhit_ensemble* e, int* on);
int mhit_ensemble_set_batched(mhit_ensemble* e, int on);

/* Test hooks (no reference counterpart): run one stage of the step pipeline on the current
 * buffers, read an internal buffer widened to float64, and commit the staged step.  They let
 * a test compare each kernel with the matching block of multi/main.f90.  Stage order:
 * tracer (:477-508), phase (:522-636), momentum (:658-816), then the Poisson stages x-fwd,
 * y-fwd, z-solve, y-inv, x-inv (:833-923) and the projection (:942-1007).  A stage of a
 * disabled feature is a no-op.  Buffers: u,v,w of the current step (stored, before the lazy
 * mean removal), u*,v*,w* / phi^{n+1} of the step being built, the pressure, rhs_o, rhsphi_o,
 * and the spectrum (interleaved re,im with a row pitch, see mhit_debug_buffer_len). */
#define MHIT_STAGE_TRACER 0
#define MHIT_STAGE_PHASE 1
#define MHIT_STAGE_MOMENTUM 2
#define MHIT_STAGE_XFWD 3
#define MHIT_STAGE_YFWD 4
#define MHIT_STAGE_ZSOLVE 5
#define MHIT_STAGE_YINV 6
#define MHIT_STAGE_XINV 7
#define MHIT_STAGE_REFINE 8
#define MHIT_STAGE_CORRECT 9
#define MHIT_BUF_U 0
#define MHIT_BUF_V 1
#define MHIT_BUF_W 2
#define MHIT_BUF_UN 3
#define MHIT_BUF_VN 4
#define MHIT_BUF_WN 5
#define MHIT_BUF_P 6
#define MHIT_BUF_PHI 7
#define MHIT_BUF_PHIN 8
#define MHIT_BUF_RU 9
#define MHIT_BUF_RV 10
#define MHIT_BUF_RW 11
#define MHIT_BUF_RPHI 12
#define MHIT_BUF_SPEC 13
/* No-allocation field statistics.  This entry point has no counterpart in the reference.
 * For callers that cannot let the library allocate device memory -- a host whose device arrays
 * belong to its own runtime (OpenACC / CUDA Fortran) and only wants statistics of fields it
 * already holds, or a run with the GPU's memory nearly fully committed, where an extra cudaMalloc
 * can fail and a cudaFree synchronises the device.  Computes, from caller-owned device arrays
 * u, v, w (x-fastest nx*ny*nz float64), stats[0] = max|div u|, stats[1] = KE = 0.5 <u.u>,
 * stats[2] = 2 nu <S_ij S_ij> -- the formulas of mhit_diagnostics, applied to the arrays as
 * passed (no mean is removed; mhit_diagnostics first subtracts its context's lazily removed
 * mean, so the two agree on downloaded or zero-mean fields) -- into the caller's device array
 * stats[3], on `stream` (a cudaStream_t, NULL for the default stream).  A NaN in u, v or w
 * gives NaN in stats[0] and stats[1].
 * It calls no cudaMalloc/cudaFree: its only scratch is a file-scope device array with one slot
 * per z plane, so nz may not exceed MHIT_STATS_NOALLOC_MAX_PLANES (MHIT_ERR_ARG otherwise).
 * The first call on a device (and the first after the device's CUDA context changed, e.g. after
 * cudaDeviceReset) looks up that array's device address (cudaGetSymbolAddress, no allocation);
 * make that first call before any stream capture.  All calls share the array: calls whose
 * kernels overlap on the GPU race and must be serialised by the caller. */
#define MHIT_STATS_NOALLOC_MAX_PLANES 1024
int mhit_field_stats_noalloc(int nx, int ny, int nz, double nu, const double* u, const double* v, const double* w,
                             double* stats, void* stream);

int mhit_debug_run_stage(mhit_ctx* ctx, int stage);
int mhit_debug_commit_step(mhit_ctx* ctx);
/* Iteration bound of mhit_label_drops' union-find loops (0, the default: the cell count, which
 * no parent chain or link retry sequence can exceed).  A small bound makes a legitimate chain
 * run out, so a test can drive the bounded-loop error path (MHIT_ERR_STATE) without a fault. */
int mhit_debug_set_label_bound(mhit_ctx* ctx, long long bound);
/* 1 (the default): the momentum kernel fills the plane rings of the tiles that need no periodic
 * wrap with TMA boxes; 0: every tile copies 16-byte pairs per thread.  Both give the same bits
 * (a test compares them). */
int mhit_debug_set_mom_tma(mhit_ctx* ctx, int on);
/* 1: the inverse x transform runs inside the projection (one pass; the pressure of a step is
 * transformed into its array only when something reads it: a download, a field file, a
 * checkpoint, a debug read, or a call that reuses the spectrum buffer); 0: the two passes of
 * multi/main.f90:909-912 and :942-1003 run apart; -1 (the default): fused where it is the faster
 * (nx = 512).  The refinement sweep always runs them apart.  The results agree to rounding (a
 * test compares). */
int mhit_debug_set_fused_projection(mhit_ctx* ctx, int on);
long long mhit_debug_buffer_len(mhit_ctx* ctx, int which);
int mhit_debug_get_buffer(mhit_ctx* ctx, int which, double* out);

#ifdef __cplusplus
}
#endif
#endif /* MHIT_B200_H */
