/*
 * hydrocode_b200.h -- C ABI of the B200 (sm_100a) hydro + self-gravity step.
 *
 * Plain C types only: pointers, sizes, ints, doubles.  One context object
 * owns all device memory of one solver; the host keeps the reference's
 * array-of-structures State3D layout (5 doubles per cell, IDX3D row-major
 * with k fastest, hydro_solver_3d.h:12-21) at this boundary, while the device
 * stores structure-of-arrays fields.
 *
 * Every function returns HC_OK (0) or a negative HC_ERR_* code; the message
 * of the last error of the calling thread is available from hc_last_error().
 * A context is used by one host thread at a time (the reference solver is
 * single-threaded and non-reentrant, gravity_solver_3d.c:552).
 *
 * Reference interfaces these entry points replace (file:line in the
 * reference project):
 *   hc_create / hc_destroy            solver3d_create + gravity_solver_create,
 *                                     solver3d_destroy (hydro_solver_3d.c:33-128,
 *                                     gravity_solver_3d.c:49-131)
 *   hc_step                           godunov_step_3d (hydro_solver_3d.c:637-811),
 *                                     the body of the run loops (:2257-2275)
 *   hc_step_host                      the same step on a host State3D array
 *   hc_gravity_solve                  gravity_solve / gravity_solve_potential
 *                                     (gravity_solver_3d.c:905-911, :510-747)
 *   hc_gravity_acceleration           gravity_compute_acceleration (:753-899)
 *   hc_set_gravity_params             gravity_set_solver_params (:137-144)
 *   hc_set_gravity_bc                 gravity_set_boundary_type (:146-148)
 *   hc_get_diag                       gravity_get_diagnostics (:150-155)
 *   hc_set_state / hc_get_state       the U array the reference steps in place
 *   hc_get_phi / hc_get_accel         GravitySolver3D.phi / gx gy gz
 */
#ifndef HYDROCODE_B200_H
#define HYDROCODE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hc_ctx hc_ctx;

enum {
    HC_OK = 0,
    HC_NOT_CONVERGED = -1,   /* SOR hit max_iter (gravity_solver_3d.c:746) */
    HC_ERR_ARG = -2,
    HC_ERR_CUDA = -3,
    HC_ERR_NOMEM = -4,
    HC_ERR_STATE = -5,
    HC_ERR_TIMEOUT = -6,     /* a bounded device wait gave up */
    HC_ERR_NUMERIC = -7      /* non-finite value met */
};

/* Arithmetic of the step. */
enum {
    HC_FP64 = 0,    /* FP64 throughout, reference operation order, no FMA:
                       bit-identical to the reference C build */
    HC_FP32 = 1     /* FP32 hydro state and HLLC, FP64 potential with FP64
                       residual and FP32 SOR correction sweeps */
};

/* Order of the FP64 multipole moment sums. */
enum {
    HC_MOMENTS_SEQUENTIAL = 0,  /* the reference's (i,j,k) order: bit-exact */
    HC_MOMENTS_TREE = 1         /* deterministic parallel tree */
};

/* Warm start of each Poisson solve. */
enum {
    HC_WARM_PREVIOUS = 0,   /* previous step's potential (the reference) */
    HC_WARM_UNET = 1        /* learned 3D U-Net prediction, checked against
                               the previous potential */
};

typedef struct hc_config {
    int nx, ny, nz;
    double xmin, xmax, ymin, ymax, zmin, zmax;
    double gamma;            /* adiabatic index */
    double cfl;
    double G;                /* self-gravity on iff G > 0 (hydro_solver_3d.c:63) */
    int bc[6];               /* BCType (0 periodic, 1 reflective, 2 outflow):
                                xmin, xmax, ymin, ymax, zmin, zmax */
    int precision;           /* HC_FP64 / HC_FP32 */
    int moment_order;        /* HC_MOMENTS_* */
    int grav_bc;             /* GravBCType: 0 periodic, 1 isolated, 2 dirichlet */
    int lmax;                /* 0: reference monopole + Cartesian quadrupole;
                                1..12: real solid harmonics to degree lmax */
    double omega;            /* SOR relaxation (default 1.5) */
    double tol;              /* SOR tolerance on max |phi_GS - phi_old| */
    int max_iter;
    int sor_depth;           /* SOR kernels: 0 (default) colour-split sweeps;
                                -3 colour-split with the FP32 correction
                                sweeps staged by TMA where rows of one colour
                                hold at most 256 cells, a multiple of 4;
                                -2 colour-split, two FP32 correction
                                iterations per HBM pass (temporal blocking);
                                -1 natural-layout per-colour sweeps; >= 1
                                natural-layout wavefront passes of that many
                                iterations */
    int warm_start;          /* HC_WARM_* */
    int device;              /* CUDA device ordinal */
    int gravity_only;        /* 1: Poisson solver only (no hydro state); allows
                                nz == 1, the reference's 2D mode */
    int recon;               /* interface states: 0 (default) piecewise constant,
                                the reference's scheme; 1 MUSCL-Hancock
                                (minmod-limited linear primitives with a half-step
                                predictor), HC_FP64 only -- no reference
                                counterpart */
    double dx, dy, dz;       /* cell sizes; 0 (default): (max - min) / n as
                                hydro_solver_3d.c:55-57.  A slab of a larger
                                grid passes the whole grid's sizes so that its
                                arithmetic is the whole grid's bit for bit */
} hc_config;

typedef struct hc_diag {
    int last_iterations;     /* iterations of the last solve */
    double last_residual;    /* its final update norm */
    int last_status;         /* 0 converged, -1 not converged */
    int warm_start_used;     /* 1 if the learned start was taken */
    int outer_cycles;        /* mixed precision: FP64 residual evaluations */
    double dt;               /* dt of the last step */
    long long steps;         /* steps taken by this context */
    long long total_iterations;
    int overshoot;           /* temporal blocking crossed tol inside a pass */
    long long unet_accepted; /* solves that started from the learned prediction */
    long long unet_fallbacks;/* solves whose prediction was rejected (larger FP64
                                residual than the previous potential's) */
    double cons[5];          /* with hc_set_conservation_record on: FP64 sums of
                                rho, rho u, rho v, rho w, E over all cells after
                                the last step of the last hc_step call */
    /* learned-start outcome monitor (hc_set_unet_guard) */
    long long unet_probes;   /* plain solves run to measure the network */
    long long unet_wins;     /* comparisons the prediction won */
    long long unet_losses;   /* comparisons it lost (no fewer iterations) */
    long long unet_switch_offs;
    int unet_off;            /* 1 while the network is switched off */
} hc_diag;

/* Per-kernel-family device time (CUDA events on the context's stream),
 * accumulated since the last reset, in milliseconds. */
typedef struct hc_timing {
    double hydro_ms;         /* fused flux/update/source kernel */
    double bc_ms;            /* boundary source, periodic copies, BCs, CFL */
    double sor_ms;           /* SOR sweeps (and FP32 correction sweeps) */
    double residual_ms;      /* FP64 residual + correction update */
    double moments_ms;       /* multipole moments + boundary evaluation */
    double unet_ms;          /* learned warm start */
    long long hydro_launches;
    long long sor_launches;
    long long launches;      /* every kernel launched by this context */
} hc_timing;

void hc_config_default(hc_config *cfg);

hc_ctx *hc_create(const hc_config *cfg);
void hc_destroy(hc_ctx *ctx);

size_t hc_ncells(const hc_ctx *ctx);

/* Conserved state, host array of ncells State3D (5 doubles per cell). */
int hc_set_state(hc_ctx *ctx, const double *U_aos);
int hc_get_state(hc_ctx *ctx, double *U_aos);
/* Conserved state as 5 consecutive fields of ncells doubles. */
int hc_set_state_soa(hc_ctx *ctx, const double *q);
int hc_get_state_soa(hc_ctx *ctx, double *q);

/* nsteps godunov steps on the device-resident state; dt_out (nullable)
 * receives each step's dt.  Returns HC_OK, or HC_NOT_CONVERGED if any SOR
 * solve failed (the step still completes, as in the reference). */
int hc_step(hc_ctx *ctx, int nsteps, double *dt_out);

/* One step on a host State3D array: upload, step, download. */
int hc_step_host(hc_ctx *ctx, double *U_aos, double *dt_out);

/* Poisson solve for a host density (rho != NULL) or the current state's
 * density (rho == NULL).  with_accel: also form g on success, as
 * gravity_solve does. */
int hc_gravity_solve(hc_ctx *ctx, const double *rho, int with_accel);
int hc_gravity_acceleration(hc_ctx *ctx);
int hc_set_gravity_params(hc_ctx *ctx, double omega, int max_iter, double tol);
int hc_set_gravity_bc(hc_ctx *ctx, int grav_bc);

int hc_get_phi(hc_ctx *ctx, double *phi);
int hc_set_phi(hc_ctx *ctx, const double *phi);
int hc_get_accel(hc_ctx *ctx, double *gx, double *gy, double *gz);

/* Multipole data of the last solve: mom[0]=M, mom[1..3]=centre of mass,
 * then 9 Cartesian Q (lmax == 0) or (lmax+1)^2 solid-harmonic moments. */
int hc_get_moments(hc_ctx *ctx, double *mom, int cap);

/* FP64 sums over all cells of the 5 conserved fields (rho, rho u, rho v,
 * rho w, E; multiply by the cell volume for totals) of the device-resident
 * state, in either precision, formed on the device in a fixed order (the same
 * state gives the same bits) -- 40 bytes cross to the host, not the state.  No
 * reference counterpart: the reference reports no totals, yet its step is not
 * conservative (boundary cells are not flux-updated, hydro_solver_3d.c:729-731;
 * the gravity source is not in flux form, :597-631; floors add mass,
 * :765-768), so the drift of these sums measures a run's accuracy.
 * hc_set_conservation_record(ctx, 1): every hc_step call also forms them after
 * its last step and reports them in hc_diag.cons. */
int hc_conservation_sums(hc_ctx *ctx, double *out5);
int hc_set_conservation_record(hc_ctx *ctx, int on);

/* FP64 max |(lap_nbrs(phi) - 4 pi G rho)/factor - phi| over the interior. */
int hc_residual_norm(hc_ctx *ctx, double *out);

int hc_get_diag(hc_ctx *ctx, hc_diag *d);
int hc_get_timing(hc_ctx *ctx, hc_timing *t, int reset);
int hc_sync(hc_ctx *ctx);

/* Device time between two points of the context's stream (CUDA events on
 * that stream): hc_timer_start records the start, hc_timer_stop the end,
 * waits for it and returns the elapsed milliseconds. */
int hc_timer_start(hc_ctx *ctx);
int hc_timer_stop(hc_ctx *ctx, double *ms);

/* Learned warm start (no reference counterpart).  A 3D U-Net (16 channels, 4
 * pooling levels, LeakyReLU, 56,305 parameters; BF16 weights and activations,
 * FP32 accumulation on the tensor cores) maps the first FP64 residual of a
 * mixed-precision solve (HC_FP32, colour-split sweeps, grid dimensions
 * multiples of 32) to a correction of the previous potential:
 *   e0 = trilinear_up(net(pool2(delta) / rms)) * rms * kscale.
 * With warm_start = HC_WARM_UNET the solve starts from phi + e0 when that
 * lowers max|delta|, else from phi (counted in hc_diag); SOR then iterates to
 * the same tolerance either way.
 * Parameters: compact FP32 vector of hc_unet_param_count() values (per conv:
 * weights [co][tap][ci] then biases; the first conv has one input channel,
 * the last one output channel).  Files: "HCUNET01", int32 count, float32
 * kscale, float32 parameters.
 * Training on the device: hc_unet_collect(ctx, capacity) records one
 * (normalised residual, normalised converged correction) pair per
 * mixed-precision solve into a ring; hc_unet_train runs `steps` Adam steps
 * (lr, seeded sample order) of the relative squared error and returns the
 * mean loss of the last quarter of the steps.  hc_unet_loss_grad: one forward
 * and backward pass on host data at the network's level-0 dimensions (each a
 * multiple of 16; x normalised input, t target, nx*ny*nz values): loss, the
 * compact gradient and the output (each nullable). */
int hc_unet_param_count(void);
int hc_unet_init(hc_ctx *ctx, unsigned seed);
int hc_unet_load(hc_ctx *ctx, const float *params, int nparam, double kscale);
int hc_unet_save(hc_ctx *ctx, float *params, int nparam, double *kscale);
int hc_unet_load_file(hc_ctx *ctx, const char *path);
int hc_unet_save_file(hc_ctx *ctx, const char *path);
int hc_unet_collect(hc_ctx *ctx, int capacity);
int hc_unet_samples(hc_ctx *ctx);
int hc_unet_train(hc_ctx *ctx, int steps, double lr, unsigned seed, double *mean_loss);
int hc_unet_loss_grad(hc_ctx *ctx, int nx, int ny, int nz, const float *x, const float *t, double *loss,
                      float *grad, float *out);
/* Predictions per solve (1..8, default 1): after an accepted prediction the
 * network is applied again to the residual it left, until one is rejected. */
int hc_set_unet_passes(hc_ctx *ctx, int passes);
/* Outcome monitor of the learned start (consecutive_losses K >= 1; 0, the
 * default, turns it off).  The acceptance test of a prediction (max|delta|
 * lower than the previous potential's) cannot see smooth error, so an
 * accepted prediction may still cost SOR iterations.  The monitor compares
 * the iterations of consecutive solves of which one started from a
 * prediction and the other from the previous potential: a rejected
 * prediction, or a plain "probe" solve it schedules after a number of
 * predicted solves that grows with the network's advantage (64 solves and
 * doubling to 1024 once a prediction needed under a quarter of the plain
 * iterations; 16 under half; 4 otherwise; 2 after a loss).  After K
 * consecutive losses the network is switched off, retried after 16 solves
 * (doubling to 256 after each failed retry) and switched back on by a win.
 * The first solve of a context is not compared.  Its state (counters in
 * hc_diag) is not part of a checkpoint: a restarted run starts a fresh
 * monitor.  No reference counterpart. */
int hc_set_unet_guard(hc_ctx *ctx, int consecutive_losses);
/* Correction cycles of a mixed-precision solve that start from a prediction
 * (1..8, default 2): the first from the step's residual, the second from the
 * smooth residual the first cycle's sweeps left; each prediction is kept only
 * if it lowers max|delta|. */
int hc_set_unet_cycles(hc_ctx *ctx, int cycles);
/* With collection on (hc_unet_collect): the correction cycle whose starting
 * residual is recorded as a training sample (1..8, default 1; 0 records
 * nothing, which pauses collection between the solves to be sampled). */
int hc_set_unet_record_cycle(hc_ctx *ctx, int cycle);
/* Relaxation factor of the FP32 correction sweeps of a mixed-precision solve
 * (0 < omega < 2; 0 restores the default, the solve's own omega).  No
 * reference counterpart: the reference relaxes every sweep with the one omega
 * of gravity_set_solver_params (gravity_solver_3d.c:78, :137-144).  The
 * FP64 path ignores it, and the solve still stops on the reference's test
 * max|phi_GS - phi_old| < tol, which does not depend on omega. */
int hc_set_correction_omega(hc_ctx *ctx, double omega);

/* Binary checkpoint and restart.  No counterpart in the reference, whose
 * restart reads its own CSV output (hydro_solver_3d.c:2142-2351): 6 decimal
 * digits per value, so a restarted run drifts from the uninterrupted one.
 * hc_checkpoint_save packs, on the device, everything the next step reads
 * -- the conserved state in the context's precision, and with self-gravity
 * the potential (the next solve's starting iterate and boundary values) and
 * the potential of the last converged solve (from which g is formed) -- and
 * returns while a writer thread copies the packed buffer to the host on its
 * own stream and writes `path`; the context may keep stepping meanwhile.  One
 * write is in flight per context: the next save, a load, hc_checkpoint_wait
 * and hc_destroy wait for it, and hc_checkpoint_wait returns its status.
 * hc_checkpoint_load checks the header (grid, precision, gravity, domain,
 * gamma, G) and a checksum of the payload before it replaces anything; a run
 * restarted from it continues bit for bit as the uninterrupted run.  t and
 * step are stored for the caller and returned by the load (each nullable).
 * Layout: a 136-byte header (hydrocode_astro1_b200/checkpoint.py lists its
 * fields; magic "HCCKPT01"), then 5 state fields of nx*ny*nz
 * words (8 bytes for HC_FP64, 4 for HC_FP32; k fastest), then phi and the
 * last converged phi (nx*ny*nz doubles each) when G > 0. */
int hc_checkpoint_save(hc_ctx *ctx, const char *path, double t, long long step);
int hc_checkpoint_wait(hc_ctx *ctx);
int hc_checkpoint_load(hc_ctx *ctx, const char *path, double *t, long long *step);

/* Initial state of the stellar-profile (nstars = 1: every cell from the
 * profile at its distance to centre[0..2], at rest) or binary-star (nstars =
 * 2: inside one star -- r < R_star[s] -- its profile and velocity vel[3s..];
 * inside both the density-weighted mix; outside both the floors) set-ups,
 * built on the device from radial profile tables (r strictly increasing,
 * n[s] points, rho and specific internal energy u), as
 * hydro_solver_3d.c:927-1002 and :1133-1205 define them.  No reference
 * counterpart as an entry point: the reference loops over the cells on the
 * host.  The state equals what hc_set_state would set from the host-built
 * array, bit for bit, without that array or its upload. */
int hc_ic_profile_stars(hc_ctx *ctx, int nstars, const int *n, const double *const *r, const double *const *rho,
                        const double *const *u, const double *R_star, const double *centre, const double *vel);

/* Diagnostics of the tensor-core convolution kernels (no reference
 * counterpart), on host buffers.  Volumes are nx*ny*nz voxels of 16 BF16
 * channels (channels last), weights w[co][tap][ci] (16*27*16 BF16, tap =
 * (di+1)*9 + (dj+1)*3 + (dk+1)), bias[16] FP32.
 * hc_unet_conv_test: 3x3x3 zero-padded convolution; out_mode 0: +bias,
 * LeakyReLU(0.1) if act, BF16-rounded, 16 channels; 1: BF16, no bias; 2: FP32
 * channel 0 + bias[0]; 3: FP32 16 channels + bias; `out` receives FP32.
 * hc_unet_wgrad_test: dw[co][tap][ci] = sum_v dy[v][co] x[v+tap][ci] (FP32),
 * reduced over at most max_parts partial sums. */
int hc_unet_conv_test(int nx, int ny, int nz, const uint16_t *x, const uint16_t *w, const float *bias,
                      int out_mode, int act, float *out);
int hc_unet_wgrad_test(int nx, int ny, int nz, const uint16_t *x, const uint16_t *dy, int max_parts, float *dw);

/* Red-black SOR to tolerance on caller-owned DEVICE arrays, allocating
 * nothing.  No counterpart in the reference: it exists for callers that own
 * all device memory themselves (a fixed arena reserved at start-up, a pool
 * shared with other solvers, a budget that must not grow or fail with
 * out-of-memory mid-run) and for callers whose other streams must not see
 * the device-wide synchronisation that cudaMalloc/cudaFree can cause.
 *
 * phi (nx*ny*nz doubles, in/out) is iterated in place on the interior; its
 * boundary cells are held as given.  rho is read only.  Arithmetic and stop
 * rule are those of hc_gravity_solve (max |phi_GS - phi_old| < tol), so the
 * iterates match it bit for bit.  `stream` is a cudaStream_t (NULL: the
 * legacy default stream); the call returns after the solve has finished on
 * it, having synchronised only that stream.  On HC_NOT_CONVERGED, iterations
 * is max_iter and residual the last iteration's norm, as the context path
 * reports them.  Returns HC_OK, HC_NOT_CONVERGED, HC_ERR_ARG (max_iter
 * outside 1..HC_NOALLOC_MAX_ITER, a dimension below 3, null phi or rho,
 * non-positive cell sizes, omega outside (0, 2), tol not finite and
 * positive) or HC_ERR_CUDA (with hc_last_error() naming the failed call).
 *
 * Scratch: one residual slot per iteration plus two flags live in a fixed
 * file-scope device array of (HC_NOALLOC_MAX_ITER + 8) * 8 bytes (about
 * 512 KB) that every GPU loading this library holds until the process exits;
 * max_iter above HC_NOALLOC_MAX_ITER is rejected.  The first call on a device
 * looks up the array's device address (cudaGetSymbolAddress) with that device
 * current and loads the solver's kernels (with CUDA's lazy module loading that
 * load would otherwise happen at their first launch, and loading a module may
 * itself reserve device memory): make that first call at start-up, before any
 * stream capture and before the caller's memory budget is fixed.  Every call shares
 * the array and clears what it needs at its start, so calls that overlap on
 * the GPU (concurrent streams, threads) race: serialise them. */
#define HC_NOALLOC_MAX_ITER 65536
int hc_sor_solve_noalloc(double *phi, const double *rho, int nx, int ny, int nz,
                         double dx, double dy, double dz, double G, double omega,
                         int max_iter, double tol, void *stream,
                         int *iterations, double *residual);

/* Slab decomposition support (no reference counterpart; the reference runs
 * one grid in one process).  A grid split along i into slabs, one context per
 * slab with a ghost plane on each side that has a neighbour, steps as the
 * whole grid does when, between steps, (1) every slab's signal speed -- the
 * CFL maximum of |u_d| + c over its cells that the next step's dt is formed
 * from (hydro_solver_3d.c:422-450) -- is replaced by the maximum over the
 * slabs, and (2) each ghost plane receives the neighbour's plane.
 * hc_get_signal_speed forms it for a freshly set state; hc_set_signal_speed
 * replaces it (a value another slab of the same precision produced).
 * hc_copy_planes copies planes [i0, i0+count) of the 5 state fields to
 * (to_ctx = 0) or from (to_ctx = 1) a device buffer laid out field by field
 * (5 x count x ny x nz words of the context's precision).  With self-gravity
 * (G > 0) each context is also declared a slab (hc_set_slab) and the
 * Poisson solve runs across the slabs before each step, as below. */
int hc_get_signal_speed(hc_ctx *ctx, double *s);
int hc_set_signal_speed(hc_ctx *ctx, double s);
int hc_copy_planes(hc_ctx *ctx, int i0, int count, void *dev_buf, int to_ctx);

/* Self-gravity across slabs (FP64 contexts, isolated boundary, ny, nz >= 3;
 * the whole grid's gravity_solve_potential, gravity_solver_3d.c:510-747).
 * hc_set_slab declares that the context holds global planes
 * [ioff, ioff + nx) of a grid of gnx planes: its config's xmin/xmax are the
 * whole grid's (dx = (xmax - xmin) / gnx unless given), its own planes are
 * all but the ghost planes (local 0 when ioff > 0, local nx-1 when
 * ioff + nx < gnx), x faces exist only at global planes 0 and gnx-1, and
 * hc_step no longer solves: its source term uses the potential of the last
 * converged slab solve.  One solve, every step before hc_step, all slabs in
 * lock step:
 *   1. moments, pass 0 then pass 1.  hc_slab_moment_layout gives the form:
 *      sequential (lmax 0 with HC_MOMENTS_SEQUENTIAL): hc_slab_moments
 *      continues `width` sums in buf over the own planes (the first slab
 *      starts from zeros, each next slab from the previous slab's result),
 *      and every slab passes the last slab's sums to hc_slab_set_moments --
 *      the reference's sums bit for bit; otherwise hc_slab_moments writes
 *      `width` doubles per own plane and every slab passes all slabs'
 *      partials, concatenated in plane order (gnx planes), to
 *      hc_slab_set_moments -- the single context's tree order bit for bit;
 *   2. hc_slab_sor_begin;
 *   3. for iter = 0, 1, ... < max_iter: hc_slab_sor_sweep(iter, 0) and
 *      (iter, 1) -- the whole grid's red and black colours -- each followed
 *      by the ghost exchange of the potential (hc_slab_phi_planes: planes of
 *      the colour-split potential, both colours, [2][count][ny (nz+1)/2]
 *      doubles indexed by the whole grid's colour); after iteration 0 also hc_slab_sor_boundary and an
 *      exchange; then the maximum over the slabs of hc_slab_sor_norm(iter)
 *      -- stop with iter + 1 iterations when it is below tol;
 *   4. hc_slab_sor_end(iterations, that maximum, converged).
 * The result equals the single context's solve bit for bit (potential,
 * iterations, residual). */
int hc_set_slab(hc_ctx *ctx, int gnx, int ioff);
int hc_slab_moment_layout(hc_ctx *ctx, int pass, int *sequential, int *width);
int hc_slab_moments(hc_ctx *ctx, int pass, double *buf);
int hc_slab_set_moments(hc_ctx *ctx, int pass, const double *all, int nplanes);
int hc_slab_sor_begin(hc_ctx *ctx);
int hc_slab_sor_sweep(hc_ctx *ctx, int iter, int colour);
int hc_slab_sor_boundary(hc_ctx *ctx);
int hc_slab_sor_norm(hc_ctx *ctx, int iter, double *norm);
int hc_slab_sor_end(hc_ctx *ctx, int iterations, double residual, int converged);
int hc_slab_phi_planes(hc_ctx *ctx, int i0, int count, void *buf, int to_ctx);

/* Page-lock (pin) a host buffer for faster transfers, and release it. */
int hc_host_register(void *ptr, size_t bytes);
int hc_host_unregister(void *ptr);

const char *hc_last_error(void);
int hc_device_count(void);

#ifdef __cplusplus
}
#endif
#endif
