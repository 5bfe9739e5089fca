/* diskgpu.h — C ABI of the B200 (sm_100a) diskfft time step.
 *
 * The library advances a razor-thin barotropic self-gravitating disk on a log-polar
 * grid: second-order van-Leer MUSCL transport plus Kalnajs softened log-spiral
 * self-gravity.  It is a drop-in for the time step of oklo/heavy-disks' `diskdisk`
 * (diskfft/src/diskmain.cpp, hydro.hpp, kalnajs.hpp).
 *
 * Conventions
 *   - Host buffers are caller-owned, FP64, row-major with index i*Nphi + j:
 *     i is the radial (log-spaced) cell, j the azimuthal cell (hydro.hpp:44).
 *   - Every call returns an int status: DG_OK (0), or a negative DG_ERR_* code.
 *     No exception crosses the ABI.  dg_last_error() gives a one-line reason.
 *   - One handle owns one disk on one CUDA device and one stream.  A handle is not
 *     thread-safe; different handles may be used from different threads.
 *   - The state lives in device memory between calls; set/get copy it.
 *
 * Precision
 *   DG_PREC_FP64   the plain method: FP64 state and FP64 FFT gravity.  Matches the
 *                  reference's FFTW+OpenMP run to <= 1e-10 relative.
 *   DG_PREC_MIXED  FP32 perturbation about an FP64 axisymmetric basic state; the
 *                  gravity convolution runs as split-BF16 tensor-core (tcgen05) DFT
 *                  products with FP32 accumulation.
 */
#ifndef DISKGPU_H
#define DISKGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DG_ABI_VERSION 1

/* status codes */
#define DG_OK 0
#define DG_ERR_INVALID (-1)     /* invalid argument or NULL pointer */
#define DG_ERR_CUDA (-2)        /* CUDA runtime error (message in dg_last_error) */
#define DG_ERR_NONFINITE (-3)   /* state or dt became non-finite / non-positive */
#define DG_ERR_UNSUPPORTED (-4) /* grid size or option not supported */
#define DG_ERR_NOMEM (-5)       /* device or host allocation failed */
#define DG_ERR_TIMEOUT (-6)     /* a bounded device wait gave up */
#define DG_ERR_STATE (-7)       /* call out of order (e.g. step before any state is set) */

#define DG_PREC_FP64 0
#define DG_PREC_MIXED 1

/* Physical and numerical parameters.  dg_params_default() fills the reference's
 * standard heavy disk and CLI defaults (diskmain.cpp:17-29). */
typedef struct dg_params {
  int Nu, Nphi;          /* radial and azimuthal cells (argv[1], argv[2]) */
  double Rin, Rout;      /* grid radii (0.25, 1.0) */
  double Kpoly;          /* P = K Sigma^gamma (0.25) */
  double gamma_gas;      /* (2.0) */
  double gmstar;         /* G M_* of the central star (0.6) */
  double G;              /* gravitational constant of the disk (1.0) */
  double eps;            /* scale-free Kalnajs softening (argv[3], 0.02) */
  int selfgrav;          /* 1: disk self-gravity on (argv[5]) */
  double amp;            /* m=2 seed amplitude (argv[6], 1e-3) */
  double phase0;         /* seed phase: Sigma0 (1 + amp cos 2(phi - phase0)); 0 = reference */
  double R0, w2, S0;     /* Gaussian disk Sigma0 = S0 exp(-(R-R0)^2/w2) (0.45, 0.05, 0.372) */
  int precision;         /* DG_PREC_FP64 or DG_PREC_MIXED */
  int device;            /* CUDA device ordinal; -1 = the calling thread's current device */
  int basic_state;       /* rotation curve of dg_init_standard: DG_BASIC_FFT (the reference's,
                            diskmain.cpp:41-56) or DG_BASIC_ELLIPTIC (complete elliptic integrals) */
} dg_params;

#define DG_BASIC_FFT 0
#define DG_BASIC_ELLIPTIC 1

/* One row of the mode table: diskmain.cpp:93-97 prints t, |C0|, |C2|, arg(C2). */
typedef struct dg_record {
  double t;
  double c0;    /* |C0| */
  double c2;    /* |C2| */
  double arg2;  /* arg(C2) = atan2(Im, Re) */
} dg_record;

typedef struct dg_handle dg_handle;

/* Fill *p with the reference defaults (diskmain.cpp:17-29). */
int dg_params_default(dg_params *p);

/* Create a disk (DiskHydro ctor hydro.hpp:28-43 + KalnajsSolver ctor kalnajs.hpp:25-42:
 * grid, device buffers, Green's-function table khat built once in FP64). */
int dg_create(const dg_params *p, dg_handle **out);
/* Release every device and host resource of the handle (NULL is a no-op). */
void dg_destroy(dg_handle *h);
/* Reason for the last non-zero status of this handle ("" if none). */
const char *dg_last_error(const dg_handle *h);
/* Static text for a status code. */
const char *dg_status_string(int status);

/* Grid: R (Nu), Rf (Nu+1), Vol (Nu) exactly as hydro.hpp:31-38.  Any pointer may be NULL. */
int dg_grid(const dg_handle *h, double *R, double *Rf, double *Vol);

/* Standard initial condition: self-gravitating equilibrium + m=2 seed (diskmain.cpp:34-63). */
int dg_init_standard(dg_handle *h);
/* Replace / read the state (DiskHydro::Sig, vR, vp; hydro.hpp:24). */
int dg_set_state(dg_handle *h, const double *Sig, const double *vR, const double *vp);
int dg_get_state(dg_handle *h, double *Sig, double *vR, double *vp);

/* DiskHydro::timestep(cfl) (hydro.hpp:48-61): dt = cfl / max_ij (sR + sphi). */
int dg_timestep(dg_handle *h, double cfl, double *dt);
/* One step with the disk's own self-gravity when selfgrav is on: the body of
 * diskmain.cpp:102-108 = potential -> forces -> DiskHydro::step(dt, gR, gp). */
int dg_step(dg_handle *h, double dt);
/* DiskHydro::step(dt, gR, gp) (hydro.hpp:63-70) with caller forces; gR and gp may both
 * be NULL (no self-gravity, hydro.hpp:86-88). */
int dg_step_forces(dg_handle *h, double dt, const double *gR, const double *gp);

/* KalnajsSolver::potential (kalnajs.hpp:48-63) of a caller surface density. */
int dg_potential(dg_handle *h, const double *Sig, double *Phi);
/* KalnajsSolver::forces (kalnajs.hpp:65-80). */
int dg_forces(dg_handle *h, const double *Phi, double *gR, double *gp);

/* Disk mass m_D = sum Sigma dA of the current state (diskmain.cpp:66-70). */
int dg_disk_mass(dg_handle *h, double *mD);
/* Fourier amplitudes C_m = sum Sigma e^{-i m phi} dA / m_D for m = 0..mmax of the current
 * state (diskmain.cpp:72-84, normalised by the m_D fixed at dg_init_standard / dg_set_state).
 * re_im receives 2*(mmax+1) doubles: Re C_0, Im C_0, Re C_1, ... */
int dg_modes(dg_handle *h, int mmax, double *re_im);
/* FP64 global sums: mass = sum Sigma dA, angmom = sum Sigma vphi R dA. */
int dg_conserved(dg_handle *h, double *mass, double *angmom);

/* The time loop of diskmain.cpp:88-110 run on the device: repeat
 * { record modes every dtout; dt = timestep(cfl); clip to tlim; gravity; step } while t < tlim,
 * with no host synchronisation inside a chunk of steps.  Records are written to rec
 * (up to max_rec); *n_rec, *t and *nsteps receive the counts and final time. */
int dg_advance(dg_handle *h, double tlim, double cfl, double dtout, dg_record *rec, int max_rec,
               int *n_rec, double *t, long long *nsteps);
/* Receiver of mode records for dg_advance_cb. */
typedef void (*dg_record_fn)(const dg_record *rec, void *user);
/* dg_advance that hands each record to fn(rec, user), in order, as soon as the host drains
 * it from the device (after every chunk of at most 64 device steps) instead of collecting
 * them: diskmain.cpp:93-98 prints and writes each record as it is made, and a long run
 * keeps the records it made before a failure.  *n_rec (may be NULL) receives the count. */
int dg_advance_cb(dg_handle *h, double tlim, double cfl, double dtout, dg_record_fn fn, void *user, int *n_rec,
                  double *t, long long *nsteps);
/* Simulation time and step count of the handle. */
int dg_time(dg_handle *h, double *t, long long *nsteps);

/* ---- Growth fit of the m = 2 mode (FP64, host only) ----
 * The reference derived gamma and Omega_p off-line from diskfft_modes.dat
 * (diskfft/README.md:26-29,37).  With the convention of Cm() (diskmain.cpp:72-84) a
 * pattern rotating at Omega_p has arg C2 = -2 Omega_p t + const, so gamma = d ln|C2|/dt
 * and Omega_p = -1/2 d arg C2/dt, arg C2 unwrapped over the records.
 *
 * Least squares over the records with tmin <= t <= tmax and |C2| > 0 (NaN for tmin or tmax
 * means no bound); *npoints receives the count.  DG_ERR_INVALID with fewer than two. */
int dg_fit_growth(const dg_record *rec, int n, double tmin, double tmax, double *gamma, double *omega_p,
                  int *npoints);
/* The two phases of a run through saturation, into out[6]:
 *   out[0..2] gamma, Omega_p and the record count of the linear phase: from t0 (past the
 *             seed's transient) until |C2|/|C0| first exceeds ratio_end (all records from
 *             t0 / 2 on when that window holds fewer than four);
 *   out[3..5] mean |C2|/|C0|, Omega_p and the record count of the saturated phase: from the
 *             first to the last record with |C2|/|C0| >= ratio_min (NaN, NaN, 0 if fewer
 *             than two).
 * Typical thresholds: t0 = 1, ratio_end = 0.05, ratio_min = 0.15. */
int dg_fit_phases(const dg_record *rec, int n, double t0, double ratio_end, double ratio_min, double *out);

/* ---- Parameter file of a sweep (the reference takes positional argv only, diskmain.cpp:17-23) ----
 * Plain text, one disk per line of blank-separated key=value pairs; '#' starts a comment.
 * Keys are the dg_params field names (precision also takes fp64 | mixed, basic_state
 * fft | elliptic).  A line may instead give a sweep point as Qmin, mass_ratio and
 * soft_over_r (all three, with gamma_gas or its default 2): it is mapped through
 * dg_params_physical first and any explicit field keys on the line apply after that.
 * Unset fields take dg_params_default.  dg_params_write writes every field (doubles as
 * %.17g), so reading the file back gives the same parameters bit for bit.  dg_params_read
 * fills up to max entries and sets *n; a malformed line, an unknown key or more disks than
 * max return DG_ERR_INVALID with the line number in dg_last_error(NULL). */
int dg_params_write(const char *path, const dg_params *p, int n);
int dg_params_read(const char *path, dg_params *p, int max, int *n);

/* Snapshot / restart (new: the reference keeps its state only in the process).  The file
 * holds the parameters, t, the next record time, m_D, the step count, the full FP64
 * fields and, for the mixed path, its basic state, so a restarted run continues bit for
 * bit.  dg_load needs a handle with the same grid, precision and physics parameters. */
int dg_save(dg_handle *h, const char *path);
int dg_load(dg_handle *h, const char *path);

/* Per-step Fourier diagnostics on the device (m = 0..mmax, mmax <= 8): with capacity > 0
 * every device step appends a row (t, Re C_0, Im C_0, ..., Re C_mmax, Im C_mmax) to a
 * ring of `capacity` rows; C_m is normalised by m_D as in diskmain.cpp:72-84.  capacity 0
 * turns it off.  dg_diagnostics_read copies up to max_rows rows (oldest first), sets *n
 * and empties the ring; rows written while the ring is full are dropped. */
int dg_set_diagnostics(dg_handle *h, int mmax, int capacity);
int dg_diagnostics_read(dg_handle *h, double *rows, int max_rows, int *n);

/* ---- Batched sweeps: many independent disks in one graph launch ---- */

typedef struct dg_batch dg_batch;
/* n disks (heterogeneous grids / parameters, one device) advanced together: each launch is
 * one CUDA graph with one branch per disk, each branch holding that disk's steps on its
 * own stream.  The disks are ordinary handles (dg_batch_disk) for state and diagnostics. */
int dg_batch_create(int n, const dg_params *params, dg_batch **out);
void dg_batch_destroy(dg_batch *b);
const char *dg_batch_last_error(const dg_batch *b);
int dg_batch_size(const dg_batch *b);
/* Borrowed handle of disk k (owned by the batch; do not destroy). */
dg_handle *dg_batch_disk(dg_batch *b, int k);
int dg_batch_init_standard(dg_batch *b);
/* dg_advance for every disk to the same tlim.  Each graph launch runs about
 * steps_per_launch steps of the disk with the smallest dt and proportionally more of the
 * others.  rec holds n * max_rec_per_disk records (disk k at k * max_rec_per_disk);
 * n_rec, t and nsteps receive n values each (any may be NULL). */
int dg_batch_advance(dg_batch *b, double tlim, double cfl, double dtout, int steps_per_launch, dg_record *rec,
                     int max_rec_per_disk, int *n_rec, double *t, long long *nsteps);

/* ---- Learned surrogate (no counterpart in the reference) ---- */

typedef struct dg_mlp dg_mlp;
/* MLP n_in -> depth hidden layers of `width` (SiLU) -> n_out (linear), trained and run by
 * the library's own CUDA kernels: BF16 weights in every product, FP32 activations and
 * accumulation, FP32 master weights updated by Adam.  Parameters are one flat FP32 vector,
 * per layer W (fan_out x fan_in, row-major) then b.  Host buffers, row-major samples. */
int dg_mlp_create(int n_in, int width, int depth, int n_out, unsigned long long seed, int device, dg_mlp **out);
void dg_mlp_destroy(dg_mlp *m);
const char *dg_mlp_last_error(const dg_mlp *m);
long long dg_mlp_num_params(const dg_mlp *m);
int dg_mlp_get_params(dg_mlp *m, float *params);
/* Also resets the Adam state. */
int dg_mlp_set_params(dg_mlp *m, const float *params);
int dg_mlp_forward(dg_mlp *m, int n, const float *x, float *y);
/* Mean-squared-error loss over n samples and its gradient w.r.t. the parameters (grad may
 * be NULL). */
int dg_mlp_loss_grad(dg_mlp *m, int n, const float *x, const float *t, float *loss, float *grad);
/* One Adam step (beta 0.9 / 0.999) on the batch; *loss receives the loss before the step. */
int dg_mlp_train_step(dg_mlp *m, int n, const float *x, const float *t, float lr, float *loss);

/* ---- FP64 host-side basic state (no device work) ---- */

/* Disk self-gravity force gR(R) (negative inward), vphi^2, kappa^2 and Toomre Q at radii
 * R[0..n) (increasing), from complete elliptic integrals with the Kalnajs kernel's
 * softening eps R R'.  It is the closed form of lka98/selfgravity.py:35-95 with that
 * softening; vphi^2 follows diskmain.cpp:55.  Any output pointer may be NULL. */
int dg_rotation_curve_elliptic(const dg_params *p, int n, const double *R, double *gR, double *vphi2,
                               double *kappa2, double *Q);
/* Map sweep parameters onto *p (other fields kept): eps = soft_over_r^2, gamma_gas, S0 so
 * that the disk mass is mass_ratio * M_* (G M_* = p->gmstar), and Kpoly so that the minimum
 * of the elliptic-integral Toomre Q (defined as in lka98/selfgravity.py:98-102) over the disk
 * body (Sigma0 >= 0.1 S0) equals Qmin.  K is capped at the largest value for which the
 * equilibrium exists over the body (vphi^2 > 0, kappa^2 > 0); *Qmin_achieved (may be NULL)
 * receives the minimum Q actually reached, which is below Qmin when the cap binds. */
int dg_params_physical(double Qmin, double mass_ratio, double soft_over_r, double gamma_gas, dg_params *p,
                       double *Qmin_achieved);

/* ---- GPU-side extensions (no counterpart in the CPU reference) ---- */

/* Run subsequent work of this handle on the caller's CUDA stream (a cudaStream_t passed
 * as void*; NULL restores the handle's own stream).  The caller keeps ownership. */
int dg_set_stream(dg_handle *h, void *stream);
/* Enqueue nsteps device-resident steps: dt = cfl / max(sR + sphi) is derived on the device
 * from the state each step produces (no tlim clip, no records, no host synchronisation).
 * With sync = 0 the call returns once the work is queued; a device-side error then shows
 * up at the next synchronising call. */
int dg_run_steps(dg_handle *h, int nsteps, double cfl, int sync);
/* Record the device loop's step graph now (64 steps; nothing runs).  dg_run_steps and
 * dg_advance otherwise record it at their first full chunk, so a caller that times that
 * call, or must not pay the recording at a later point, records it up front.  The graph
 * holds the handle's stream and kernel choices: call after dg_set_stream and after the
 * first state upload (which runs the autotuner). */
int dg_capture_graph(dg_handle *h);
/* One reference-style step on caller host buffers, in place: upload (Sig, vR, vp), then
 * timestep(cfl) -> potential -> forces -> step as diskmain.cpp:100-105, and download the
 * new state; *dt receives the dt used.  This is DiskHydro::step on host vectors. */
int dg_step_host(dg_handle *h, double cfl, double *Sig, double *vR, double *vp, double *dt);

/* Per-phase device timing with CUDA events on the handle's stream. */
#define DG_PROF_HYDRO 0         /* fused hydro kernel */
#define DG_PROF_GRAVITY 1       /* whole gravity convolution */
#define DG_PROF_CFL 2           /* standalone CFL reductions */
#define DG_PROF_GRAV_PHI_FWD 3  /* gravity, part: forward phi transform (FP64 FFT pass / phi DFT GEMM) */
#define DG_PROF_GRAV_U 4        /* gravity, part: radial convolution with khat */
#define DG_PROF_GRAV_PHI_INV 5  /* gravity, part: inverse phi transform and potential scaling */
#define DG_PROF_N 6
int dg_profile_enable(dg_handle *h, int on);
/* Accumulated milliseconds and launch counts per phase since the last read (resets). */
int dg_profile_read(dg_handle *h, double *ms, long long *count);
/* Number of this library's kernels one time step of the handle launches (gravity passes,
 * the fused hydro kernel and, after the mixed path's tile hydro forms, the one-warp step
 * finalisation); depends on precision, grid, hydro form and self-gravity. */
int dg_kernels_per_step(const dg_handle *h);
/* What the autotuner chose for this handle, as one line of text (NUL-terminated, cut to
 * len bytes): the hydro kernel form and the pipeline depth of each gravity product, with
 * the timings behind the choice.  No counterpart in the reference.  The tuner runs at the
 * first dg_set_state / dg_init_standard / dg_load of a mixed-precision handle and caches its
 * choices per process by grid; DISKGPU_TUNE=0 in the environment keeps the defaults. */
int dg_tuning_info(const dg_handle *h, char *buf, int len);

/* Allocation-free CFL time step.  No counterpart in the reference: it is the same
 * dt = cfl / max_ij (sR + sphi) as dg_timestep, for callers that must not allocate device
 * memory when they need it (a pool or framework owns all device memory, or a fixed-budget
 * loop must stay out of the allocator).  Sig, vR, vp (Nu x Nphi, FP64, row-major) and dt
 * (one double) are DEVICE pointers owned by the caller; the grid is rebuilt from Nu, Nphi,
 * Rin, Rout.  The call allocates nothing: its scratch is a static per-device array of 8192
 * row maxima (64 KiB, held by every device that loads the library until exit), so
 * Nu > 8192 returns DG_ERR_UNSUPPORTED.  The first call on a device looks up that array's
 * address and keeps it for the process (make it before any stream capture; do not call
 * again on a device after cudaDeviceReset).  Work is queued on `stream` (a cudaStream_t
 * as void*, NULL = default stream); the call does not synchronise.  A non-finite state
 * gives dt = NaN (the reference would skip the NaN).  All calls share the scratch: calls
 * that overlap on the GPU race. */
int dg_timestep_static(const double *Sig, const double *vR, const double *vp, int Nu, int Nphi, double Rin,
                       double Rout, double Kpoly, double gamma_gas, double cfl, double *dt, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* DISKGPU_H */
