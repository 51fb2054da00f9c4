/*
 * ref_harness.c -- test infrastructure, not product code.
 *
 * Builds the UNMODIFIED reference hydrocode (hydro_solver_3d.c,
 * gravity_solver_3d.c, input_deck.c) into a shared library so that the
 * tests, the golden-fixture generator and the CPU baseline of bench.py can
 * drive its static time step `godunov_step_3d` (hydro_solver_3d.c:637-811)
 * and the static multipole/boundary helpers of the gravity solver
 * (gravity_solver_3d.c:164-504) directly.  The reference sources are
 * #included from the reference tree by the recipe in oracle/Makefile; none
 * of them is copied here.  Output goes to oracle/_ref/ only.
 *
 * Every entry point below takes/returns the reference's own AoS layout
 * (State3D = 5 doubles per cell, IDX3D row-major with k fastest,
 * hydro_solver_3d.h:12-21).
 */
#include "hydro_solver_3d.c"
#include "gravity_solver_3d.c"
#include "input_deck.c"

void *ref_create(int nx, int ny, int nz,
                 double xmin, double xmax, double ymin, double ymax,
                 double zmin, double zmax, double G, double gamma, double cfl,
                 const int *bc6)
{
    GodunovHLLC3D *s = solver3d_create(nx, ny, nz, xmin, xmax, ymin, ymax,
                                       zmin, zmax, G);
    if (!s) return NULL;
    s->gamma = gamma;
    s->cfl = cfl;
    s->bc_xmin = (BCType)bc6[0]; s->bc_xmax = (BCType)bc6[1];
    s->bc_ymin = (BCType)bc6[2]; s->bc_ymax = (BCType)bc6[3];
    s->bc_zmin = (BCType)bc6[4]; s->bc_zmax = (BCType)bc6[5];
    s->problem = KELVIN_HELMHOLTZ_3D;
    return s;
}

void ref_destroy(void *h) { solver3d_destroy((GodunovHLLC3D *)h); }

int ref_has_gravity(void *h) { return ((GodunovHLLC3D *)h)->enable_gravity ? 1 : 0; }

void ref_enable_gravity(void *h, int on)
{
    GodunovHLLC3D *s = (GodunovHLLC3D *)h;
    s->enable_gravity = (on && s->gravity_solver) ? true : false;
}

void ref_set_grav(void *h, double omega, int max_iter, double tol, int bc_type)
{
    GodunovHLLC3D *s = (GodunovHLLC3D *)h;
    if (!s->gravity_solver) return;
    gravity_set_solver_params(s->gravity_solver, omega, max_iter, tol);
    gravity_set_boundary_type(s->gravity_solver, (GravBCType)bc_type);
}

static size_t ncell(const GodunovHLLC3D *s) { return (size_t)s->nx * s->ny * s->nz; }

void ref_set_state(void *h, const double *U)
{
    GodunovHLLC3D *s = (GodunovHLLC3D *)h;
    memcpy(s->U, U, ncell(s) * sizeof(State3D));
}

void ref_get_state(void *h, double *U)
{
    GodunovHLLC3D *s = (GodunovHLLC3D *)h;
    memcpy(U, s->U, ncell(s) * sizeof(State3D));
}

/* Run n reference time steps; record dt, SOR iterations and residual per step. */
int ref_steps(void *h, int n, double *dts, int *iters, double *resid)
{
    GodunovHLLC3D *s = (GodunovHLLC3D *)h;
    for (int q = 0; q < n; q++) {
        godunov_step_3d(s);
        if (dts) dts[q] = s->dt;
        if (s->gravity_solver) {
            if (iters) iters[q] = s->gravity_solver->last_iterations;
            if (resid) resid[q] = s->gravity_solver->last_residual;
        } else {
            if (iters) iters[q] = 0;
            if (resid) resid[q] = 0.0;
        }
    }
    return 0;
}

/* Hydro arrays g (copied out of the gravity solver by solve_gravity_field). */
void ref_get_hydro_g(void *h, double *gx, double *gy, double *gz)
{
    GodunovHLLC3D *s = (GodunovHLLC3D *)h;
    size_t n = ncell(s);
    memcpy(gx, s->gx, n * sizeof(double));
    memcpy(gy, s->gy, n * sizeof(double));
    memcpy(gz, s->gz, n * sizeof(double));
}

void ref_get_phi(void *h, double *phi)
{
    GodunovHLLC3D *s = (GodunovHLLC3D *)h;
    if (s->gravity_solver) memcpy(phi, s->gravity_solver->phi, ncell(s) * sizeof(double));
}

void ref_set_phi(void *h, const double *phi)
{
    GodunovHLLC3D *s = (GodunovHLLC3D *)h;
    if (s->gravity_solver) memcpy(s->gravity_solver->phi, phi, ncell(s) * sizeof(double));
}

void ref_get_grav_g(void *h, double *gx, double *gy, double *gz)
{
    GodunovHLLC3D *s = (GodunovHLLC3D *)h;
    if (!s->gravity_solver) return;
    size_t n = ncell(s);
    memcpy(gx, s->gravity_solver->gx, n * sizeof(double));
    memcpy(gy, s->gravity_solver->gy, n * sizeof(double));
    memcpy(gz, s->gravity_solver->gz, n * sizeof(double));
}

/* gravity_solve (gravity_solver_3d.c:905) on the solver's own gravity object. */
int ref_gravity_solve(void *h, const double *rho, int *iters, double *resid)
{
    GodunovHLLC3D *s = (GodunovHLLC3D *)h;
    if (!s->gravity_solver) return -2;
    int st = gravity_solve(s->gravity_solver, rho);
    gravity_get_diagnostics(s->gravity_solver, iters, resid);
    return st;
}

/* gravity_solve_potential alone (no acceleration). */
int ref_gravity_solve_potential(void *h, const double *rho, int *iters, double *resid)
{
    GodunovHLLC3D *s = (GodunovHLLC3D *)h;
    if (!s->gravity_solver) return -2;
    int st = gravity_solve_potential(s->gravity_solver, rho);
    gravity_get_diagnostics(s->gravity_solver, iters, resid);
    return st;
}

/* Monopole + quadrupole moments exactly as the reference boundary uses them:
 * out[0]=M, out[1..3]=centre of mass, out[4..12]=Q row-major. */
void ref_moments(void *h, const double *rho, double *out)
{
    GodunovHLLC3D *s = (GodunovHLLC3D *)h;
    if (!s->gravity_solver) return;
    double Q[3][3];
    compute_mass_moments(s->gravity_solver, rho, &out[0], &out[1], &out[2], &out[3]);
    compute_quadrupole_moment(s->gravity_solver, rho, out[1], out[2], out[3], Q);
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) out[4 + 3 * a + b] = Q[a][b];
}

/* apply_boundary_conditions (gravity_solver_3d.c:268) on the solver's phi. */
void ref_grav_boundary(void *h, const double *rho)
{
    GodunovHLLC3D *s = (GodunovHLLC3D *)h;
    if (!s->gravity_solver) return;
    s->gravity_solver->rho = (double *)rho;
    apply_boundary_conditions(s->gravity_solver);
}

void ref_grav_acceleration(void *h)
{
    GodunovHLLC3D *s = (GodunovHLLC3D *)h;
    if (s->gravity_solver) gravity_compute_acceleration(s->gravity_solver);
}

/* set_initial_conditions_3d_from_deck on a deck file (reference IC path). */
int ref_ic_from_deck(void *h, const char *deck_path)
{
    GodunovHLLC3D *s = (GodunovHLLC3D *)h;
    InputDeck *d = input_deck_create(deck_path);
    if (!d) return -1;
    set_initial_conditions_3d_from_deck(s, d);
    input_deck_destroy(d);
    return 0;
}

void ref_ic_problem(void *h, int problem)
{
    set_initial_conditions_3d((GodunovHLLC3D *)h, (ProblemType)problem);
}

/* The reference deck parser, field by field, for deck-format parity tests. */
int ref_parse_deck(const char *path, int *ints, double *dbls, char *strs)
{
    InputDeck *d = input_deck_create(path);
    if (!d) return -1;
    ints[0] = d->nx; ints[1] = d->ny; ints[2] = d->nz;
    ints[3] = (int)d->problem;
    ints[4] = (int)d->bc_xmin; ints[5] = (int)d->bc_xmax;
    ints[6] = (int)d->bc_ymin; ints[7] = (int)d->bc_ymax;
    ints[8] = (int)d->bc_zmin; ints[9] = (int)d->bc_zmax;
    ints[10] = d->restart ? 1 : 0; ints[11] = d->restart_step;
    ints[12] = d->binary_auto_orbit ? 1 : 0;
    ints[13] = d->enable_perturbations ? 1 : 0; ints[14] = d->perturbation_seed;
    ints[15] = d->perturb_velocity_modes; ints[16] = d->perturb_density_modes;
    ints[17] = d->enable_sph_harmonic_mode ? 1 : 0;
    ints[18] = d->sph_harmonic_l; ints[19] = d->sph_harmonic_m;
    ints[20] = d->enable_torus ? 1 : 0;
    double *o = dbls;
    *o++ = d->xmin; *o++ = d->xmax; *o++ = d->ymin; *o++ = d->ymax;
    *o++ = d->zmin; *o++ = d->zmax; *o++ = d->t_end; *o++ = d->output_dt;
    *o++ = d->cfl; *o++ = d->gamma; *o++ = d->G_const; *o++ = d->G_M_PNS;
    *o++ = d->L_nu; *o++ = d->g_strength; *o++ = d->L_heat; *o++ = d->restart_time;
    *o++ = d->star1_x; *o++ = d->star1_y; *o++ = d->star1_z;
    *o++ = d->star2_x; *o++ = d->star2_y; *o++ = d->star2_z;
    *o++ = d->star1_vx; *o++ = d->star1_vy; *o++ = d->star1_vz;
    *o++ = d->star2_vx; *o++ = d->star2_vy; *o++ = d->star2_vz;
    *o++ = d->binary_separation; *o++ = d->binary_orbital_velocity;
    *o++ = d->explosion_energy; *o++ = d->explosion_radius;
    *o++ = d->perturb_velocity_amplitude; *o++ = d->perturb_velocity_kmin;
    *o++ = d->perturb_velocity_kmax; *o++ = d->perturb_density_amplitude;
    *o++ = d->perturb_density_kmin; *o++ = d->perturb_density_kmax;
    *o++ = d->sph_harmonic_amp_rho; *o++ = d->sph_harmonic_amp_vel;
    *o++ = d->torus_major_radius; *o++ = d->torus_minor_radius;
    *o++ = d->torus_density; *o++ = d->torus_pressure;
    *o++ = d->torus_rotation_velocity;
    /* 6 strings of 256 bytes: output_dir, restart_file, star1, star2,
     * stellar_profile, explosion_type */
    memset(strs, 0, 6 * 256);
    strncpy(strs + 0 * 256, d->output_dir, 255);
    strncpy(strs + 1 * 256, d->restart_file, 255);
    strncpy(strs + 2 * 256, d->star1_profile, 255);
    strncpy(strs + 3 * 256, d->star2_profile, 255);
    strncpy(strs + 4 * 256, d->stellar_profile, 255);
    strncpy(strs + 5 * 256, d->explosion_type, 31);
    input_deck_destroy(d);
    return 0;
}
