/*
 * hydro_solver_3d.h -- the reference's hydro solver API (hydro_solver_3d.h of
 * the reference project), served by the B200 library: the reference driver
 * main_3d.c compiles against this header and links the library unchanged.
 *
 * GodunovHLLC3D keeps the reference's fields in their order (:33-63); U,
 * gx, gy, gz are host mirrors of the device state, valid after the initial
 * condition is set and whenever output is written.  U_half and the flux arrays
 * of the reference are not used by the device step and stay NULL.  Trailing
 * fields hold the device context and the deck's added settings.
 *
 * Reference interfaces (hydro_solver_3d.h:69-95): solver3d_create,
 * solver3d_destroy, set_initial_conditions_3d,
 * set_initial_conditions_3d_from_deck, run_simulation_3d,
 * run_simulation_3d_restart, write_output_to_file_3d, write_output_vtk,
 * load_from_csv_restart, solver3d_create_from_deck.
 */
#ifndef HYDRO_SOLVER_3D_H
#define HYDRO_SOLVER_3D_H

#include <stdbool.h>
#include <stdio.h>

#include "gravity_solver_3d.h"
#include "input_deck.h"

#define RHO_FLOOR 1.0e-5
#define P_FLOOR 1.0e-6
#define IDX3D(i, j, k, ny, nz) (((i) * (ny) + (j)) * (nz) + (k))

typedef struct {
    double rho;
    double rhou;
    double rhov;
    double rhow;
    double E;
} State3D;

typedef struct {
    double rho;
    double u;
    double v;
    double w;
    double p;
} Primitive3D;

typedef struct GodunovHLLC3D {
    int nx, ny, nz;
    double xmin, xmax, ymin, ymax, zmin, zmax;
    double dx, dy, dz;
    double dt;
    double cfl;

    BCType bc_xmin, bc_xmax;
    BCType bc_ymin, bc_ymax;
    BCType bc_zmin, bc_zmax;

    ProblemType problem;
    double gamma;

    State3D *U;
    State3D *U_half;
    State3D *F_x;
    State3D *F_y;
    State3D *F_z;

    double *gx;
    double *gy;
    double *gz;

    GravitySolver3D *gravity_solver;
    bool enable_gravity;
    double G_const;

    /* ---- B200 library state (appended) ---- */
    struct hc_ctx *dev;      /* device context; created on first step */
    int host_dirty;          /* U on the host is newer than the device state */
    int device_dirty;        /* device state is newer than U on the host */
    int precision;           /* 0 fp64 (bit-exact), 1 fp32 */
    int moment_order;
    int lmax;
    int warm_start;
    int sor_depth;
    int max_steps;
    int log_every;
    char unet_weights[256];
    long long steps_taken;
    int checkpoint_every;      /* binary checkpoint every N steps of a run (0 = off) */
    char checkpoint_file[256];
    int ck_restored;           /* a binary checkpoint was loaded: its time is ck_t */
    double ck_t;
    int recon;                 /* 0 piecewise-constant states, 1 MUSCL-Hancock (fp64) */
    int device_ics;            /* profile-based set-ups built on the device: 1 always, 0 never,
                                  -1 (default) from 256^3 cells on */
    int ic_on_device;          /* the last set-up left the state on the device only */
    int unet_guard;            /* learned-start outcome monitor: consecutive losses (0 = off) */
} GodunovHLLC3D;

GodunovHLLC3D *solver3d_create(int nx, int ny, int nz,
                               double xmin, double xmax,
                               double ymin, double ymax,
                               double zmin, double zmax,
                               double G);
void solver3d_destroy(GodunovHLLC3D *solver);

void set_initial_conditions_3d(GodunovHLLC3D *solver, ProblemType problem);
void set_initial_conditions_3d_from_deck(GodunovHLLC3D *solver, const InputDeck *deck);

void run_simulation_3d(GodunovHLLC3D *solver, double t_end, double output_dt);
void run_simulation_3d_restart(GodunovHLLC3D *solver, double t_start, double t_end,
                               double output_dt, int start_output_count);

void write_output_to_file_3d(const GodunovHLLC3D *solver, int step);
void write_output_vtk(const GodunovHLLC3D *solver, int step);

int load_from_csv_restart(GodunovHLLC3D *solver, const char *filename);

GodunovHLLC3D *solver3d_create_from_deck(const InputDeck *deck);

/* ---- additions (no reference counterpart) ---- */
/* Advance nsteps godunov steps (godunov_step_3d is static in the reference);
 * returns 0, or -1 if a Poisson solve did not converge. */
int solver3d_step(GodunovHLLC3D *solver, int nsteps);
/* Copy the device state into U (and gx/gy/gz, the gravity potential). */
int solver3d_sync_host(GodunovHLLC3D *solver);
/* Binary checkpoint (hc_checkpoint_save): exact state, potentials and step
 * parity, with t and step; written in the background -- the next checkpoint,
 * a read and solver3d_destroy wait for it.  Returns 0 or -1 (message on
 * stderr).  load_from_csv_restart also accepts such a file (recognised by its
 * magic), and run_simulation_3d_restart then starts from the stored time. */
int solver3d_write_checkpoint(GodunovHLLC3D *solver, const char *path, double t, long long step);
/* Restore a binary checkpoint; *t and *step (nullable) receive the stored values. */
int solver3d_read_checkpoint(GodunovHLLC3D *solver, const char *path, double *t, long long *step);

#endif /* HYDRO_SOLVER_3D_H */
