/*
 * hydro_solver_3d.c -- the reference's hydro solver API (hydro_solver_3d.h)
 * on the B200 library: the reference driver main_3d.c runs unchanged on top
 * of it.  The time step runs on the device through the C ABI of
 * hydrocode_b200.h; the host keeps U (array of State3D) as the mirror used
 * for initial conditions, restart input and output files.
 *
 * Host/device traffic: the initial state (or restart) is uploaded once before
 * the first step; per step only dt comes back; the state is downloaded when
 * output is written.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "hydro_solver_3d.h"
#include "hydrocode_b200.h"
#include "ics.h"

#define MAXD(a, b) (((a) > (b)) ? (a) : (b))

static size_t ncells(const GodunovHLLC3D *s) { return (size_t)s->nx * s->ny * s->nz; }

GodunovHLLC3D *solver3d_create(int nx, int ny, int nz, double xmin, double xmax, double ymin,
                               double ymax, double zmin, double zmax, double G)
{
    GodunovHLLC3D *s = (GodunovHLLC3D *)calloc(1, sizeof(GodunovHLLC3D));
    if (!s) {
        fprintf(stderr, "Failed to allocate solver structure.\n");
        return NULL;
    }
    s->nx = nx; s->ny = ny; s->nz = nz;
    s->xmin = xmin; s->xmax = xmax; s->ymin = ymin; s->ymax = ymax; s->zmin = zmin; s->zmax = zmax;
    s->dx = (xmax - xmin) / nx;        /* hydro_solver_3d.c:55-57 */
    s->dy = (ymax - ymin) / ny;
    s->dz = (zmax - zmin) / nz;
    s->cfl = 0.4;                      /* :59-63 */
    s->dt = 0.0;
    s->gamma = 5.0 / 3.0;
    s->G_const = G;
    s->enable_gravity = (G > 0.0);
    s->bc_xmin = s->bc_xmax = s->bc_ymin = s->bc_ymax = s->bc_zmin = s->bc_zmax = BC_OUTFLOW;
    s->log_every = 10;
    s->device_ics = -1;   /* profile set-ups on the device from 256^3 cells on */
    s->unet_guard = 3;
    s->gravity_solver = NULL;
    if (s->enable_gravity) {
        s->gravity_solver = gravity_solver_create(nx, ny, nz, xmin, xmax, ymin, ymax, zmin, zmax, G);
        if (!s->gravity_solver) {
            fprintf(stderr, "Warning: Failed to create gravity solver. Disabling gravity.\n");
            s->enable_gravity = false;
        } else {
            gravity_set_boundary_type(s->gravity_solver, GRAV_BC_ISOLATED);
            s->gravity_solver->owned = 1;
            printf("Gravity solver initialized with G = %.6e\n", G);
        }
    }
    size_t n = ncells(s);
    s->U = (State3D *)calloc(n, sizeof(State3D));
    s->gx = (double *)calloc(n, sizeof(double));
    s->gy = (double *)calloc(n, sizeof(double));
    s->gz = (double *)calloc(n, sizeof(double));
    if (!s->U || !s->gx || !s->gy || !s->gz) {
        fprintf(stderr, "Failed to allocate solver arrays.\n");
        solver3d_destroy(s);
        return NULL;
    }
    s->host_dirty = 1;
    return s;
}

void solver3d_destroy(GodunovHLLC3D *s)
{
    if (!s) return;
    if (s->dev) hc_destroy(s->dev);
    free(s->U);
    free(s->gx); free(s->gy); free(s->gz);
    if (s->gravity_solver) {
        s->gravity_solver->owned = 0;
        if (s->gravity_solver->dev == s->dev) s->gravity_solver->dev = NULL;
        gravity_solver_destroy(s->gravity_solver);
    }
    free(s);
}

GodunovHLLC3D *solver3d_create_from_deck(const InputDeck *d)   /* hydro_solver_3d.c:130-156 */
{
    GodunovHLLC3D *s = solver3d_create(d->nx, d->ny, d->nz, d->xmin, d->xmax, d->ymin, d->ymax,
                                       d->zmin, d->zmax, d->G_const);
    if (!s) return NULL;
    s->cfl = d->cfl;
    s->gamma = d->gamma;
    s->problem = d->problem;
    s->bc_xmin = d->bc_xmin; s->bc_xmax = d->bc_xmax;
    s->bc_ymin = d->bc_ymin; s->bc_ymax = d->bc_ymax;
    s->bc_zmin = d->bc_zmin; s->bc_zmax = d->bc_zmax;
    s->precision = d->precision;
    s->moment_order = d->moment_order;
    s->lmax = d->grav_lmax;
    s->warm_start = d->warm_start;
    s->sor_depth = d->sor_depth;
    s->recon = d->recon;
    s->device_ics = d->device_ics;
    s->unet_guard = d->unet_guard;
    s->max_steps = d->max_steps;
    s->log_every = d->log_every > 0 ? d->log_every : 10;
    strncpy(s->unet_weights, d->unet_weights, sizeof s->unet_weights - 1);
    s->checkpoint_every = d->checkpoint_every;
    strncpy(s->checkpoint_file, d->checkpoint_file, sizeof s->checkpoint_file - 1);
    if (s->gravity_solver) {
        gravity_set_solver_params(s->gravity_solver, d->grav_omega, d->grav_max_iter, d->grav_tolerance);
        s->gravity_solver->lmax = d->grav_lmax;
        s->gravity_solver->moment_order = d->moment_order;
    }
    return s;
}

/* ---------------------------------------------------------------- device */
static int ensure_device(GodunovHLLC3D *s)
{
    if (s->dev) return 0;
    hc_config c;
    hc_config_default(&c);
    c.nx = s->nx; c.ny = s->ny; c.nz = s->nz;
    c.xmin = s->xmin; c.xmax = s->xmax; c.ymin = s->ymin; c.ymax = s->ymax;
    c.zmin = s->zmin; c.zmax = s->zmax;
    c.gamma = s->gamma;
    c.cfl = s->cfl;
    c.G = s->enable_gravity ? s->G_const : 0.0;
    c.bc[0] = s->bc_xmin; c.bc[1] = s->bc_xmax; c.bc[2] = s->bc_ymin;
    c.bc[3] = s->bc_ymax; c.bc[4] = s->bc_zmin; c.bc[5] = s->bc_zmax;
    c.precision = s->precision;
    c.moment_order = s->moment_order;
    c.lmax = s->lmax;
    c.warm_start = s->warm_start;
    c.sor_depth = s->sor_depth;
    c.recon = s->recon;
    if (s->gravity_solver) {
        c.omega = s->gravity_solver->omega;
        c.max_iter = s->gravity_solver->max_iterations;
        c.tol = s->gravity_solver->tolerance;
        c.grav_bc = (int)s->gravity_solver->bc_type;
        c.lmax = s->gravity_solver->lmax ? s->gravity_solver->lmax : s->lmax;
    }
    s->dev = hc_create(&c);
    if (!s->dev) {
        fprintf(stderr, "Error: could not create the device solver: %s\n", hc_last_error());
        return -1;
    }
    if (s->gravity_solver) {
        s->gravity_solver->dev = s->dev;
        s->gravity_solver->owned = 1;
    }
    if (s->warm_start && s->unet_weights[0]) {
        extern int hc_unet_load_file(struct hc_ctx * ctx, const char *path);
        if (hc_unet_load_file(s->dev, s->unet_weights) != HC_OK)
            fprintf(stderr, "Warning: learned warm start unavailable (%s); using the previous potential\n",
                    hc_last_error());
        else if (s->unet_guard > 0 && hc_set_unet_guard(s->dev, s->unet_guard) != HC_OK)
            fprintf(stderr, "Warning: learned-start monitor not set: %s\n", hc_last_error());
    }
    s->host_dirty = 1;
    return 0;
}

static int upload_if_dirty(GodunovHLLC3D *s)
{
    if (ensure_device(s)) return -1;
    if (s->host_dirty) {
        if (hc_set_state(s->dev, (const double *)s->U) != HC_OK) {
            fprintf(stderr, "Error: state upload failed: %s\n", hc_last_error());
            return -1;
        }
        s->host_dirty = 0;
        s->device_dirty = 0;
    }
    if (s->gravity_solver)
        hc_set_gravity_params(s->dev, s->gravity_solver->omega, s->gravity_solver->max_iterations,
                              s->gravity_solver->tolerance);
    if (s->gravity_solver) hc_set_gravity_bc(s->dev, (int)s->gravity_solver->bc_type);
    return 0;
}

int solver3d_sync_host(GodunovHLLC3D *s)
{
    if (!s->dev || !s->device_dirty) return 0;
    if (hc_get_state(s->dev, (double *)s->U) != HC_OK) {
        fprintf(stderr, "Error: state download failed: %s\n", hc_last_error());
        return -1;
    }
    /* g exists once a solve has run (or a checkpoint restored one); before the
     * first step the host arrays keep their initial zeros */
    if (s->enable_gravity && s->steps_taken > 0) {
        hc_get_accel(s->dev, s->gx, s->gy, s->gz);
        if (s->gravity_solver) {
            GravitySolver3D *g = s->gravity_solver;
            hc_get_phi(s->dev, g->phi);
            size_t n = ncells(s);
            memcpy(g->gx, s->gx, n * sizeof(double));
            memcpy(g->gy, s->gy, n * sizeof(double));
            memcpy(g->gz, s->gz, n * sizeof(double));
            hc_diag dg;
            hc_get_diag(s->dev, &dg);
            g->last_iterations = dg.last_iterations;
            g->last_residual = dg.last_residual;
        }
    }
    s->device_dirty = 0;
    return 0;
}

int solver3d_step(GodunovHLLC3D *s, int nsteps)
{
    if (upload_if_dirty(s)) return -2;
    int worst = 0;
    for (int q = 0; q < nsteps; q++) {
        double dt = 0.0;
        int rc = hc_step(s->dev, 1, &dt);
        if (rc != HC_OK && rc != HC_NOT_CONVERGED) {
            fprintf(stderr, "Error: device step failed: %s\n", hc_last_error());
            return -2;
        }
        if (rc == HC_NOT_CONVERGED) {
            fprintf(stderr, "Warning: Gravity solver did not converge fully.\n");
            worst = -1;
        }
        s->dt = dt;
        s->device_dirty = 1;
        s->steps_taken++;
    }
    return worst;
}

/* ---------------------------------------------------------------- checkpoints */
int solver3d_write_checkpoint(GodunovHLLC3D *s, const char *path, double t, long long step)
{
    if (upload_if_dirty(s)) return -1;
    if (hc_checkpoint_save(s->dev, path, t, step) != HC_OK) {
        fprintf(stderr, "Error: checkpoint %s: %s\n", path, hc_last_error());
        return -1;
    }
    return 0;
}

int solver3d_read_checkpoint(GodunovHLLC3D *s, const char *path, double *t, long long *step)
{
    if (ensure_device(s)) return -1;
    double tt = 0.0;
    long long st = 0;
    if (hc_checkpoint_load(s->dev, path, &tt, &st) != HC_OK) {
        fprintf(stderr, "Error: %s\n", hc_last_error());
        return -1;
    }
    s->host_dirty = 0;     /* the device state is the restored one */
    s->device_dirty = 1;
    s->ck_restored = 1;
    s->ck_t = tt;
    s->steps_taken = st;
    if (t) *t = tt;
    if (step) *step = st;
    return 0;
}

/* ---------------------------------------------------------------- ICs */
int hc_ic_stars_device(GodunovHLLC3D *s, int nstars, const int *n, const double *const *r,
                       const double *const *rho, const double *const *u, const double *R_star,
                       const double *centre, const double *vel)
{
    const long long cells = (long long)s->nx * s->ny * s->nz;
    if (s->device_ics == 0 || (s->device_ics < 0 && cells < (1LL << 24))) return -1;
    if (ensure_device(s)) return -1;
    if (hc_ic_profile_stars(s->dev, nstars, n, r, rho, u, R_star, centre, vel) != HC_OK) {
        fprintf(stderr, "Warning: device initial conditions failed (%s); building them on the host\n",
                hc_last_error());
        return -1;
    }
    s->ic_on_device = 1;
    return 0;
}

/* after a set-up: the host array is newer, unless the state was built on the device */
static void ic_done(GodunovHLLC3D *s)
{
    if (s->ic_on_device) {
        s->host_dirty = 0;
        s->device_dirty = 1;
    } else {
        s->host_dirty = 1;
        s->device_dirty = 0;
    }
    s->ic_on_device = 0;
}

void set_initial_conditions_3d(GodunovHLLC3D *s, ProblemType problem)
{
    s->ic_on_device = 0;
    hc_ic_problem(s, problem);
    ic_done(s);
}

void set_initial_conditions_3d_from_deck(GodunovHLLC3D *s, const InputDeck *d)
{
    s->ic_on_device = 0;
    hc_ic_from_deck(s, d);
    ic_done(s);
}

/* ---------------------------------------------------------------- output */
static Primitive3D prim(const GodunovHLLC3D *s, size_t c) { return hc_ic_cons_to_prim(s->U[c], s->gamma); }

void write_output_to_file_3d(const GodunovHLLC3D *solver, int step)   /* :2336-2374 */
{
    GodunovHLLC3D *s = (GodunovHLLC3D *)solver;
    solver3d_sync_host(s);
    char fn[256];
    sprintf(fn, "output/output_%06d.csv", step);
    FILE *fp = fopen(fn, "w");
    if (!fp) {
        fprintf(stderr, "Error: Could not open file %s for writing.\n", fn);
        return;
    }
    fprintf(fp, "x,y,z,rho,u,v,w,p,gx,gy,gz\n");
    int skip = 1;
    if (s->nx > 128) skip = 2;
    if (s->nx > 256) skip = 4;
    for (int i = 0; i < s->nx; i += skip)
        for (int j = 0; j < s->ny; j += skip)
            for (int k = 0; k < s->nz; k += skip) {
                size_t c = ((size_t)i * s->ny + j) * s->nz + k;
                double x = s->xmin + (i + 0.5) * s->dx;
                double y = s->ymin + (j + 0.5) * s->dy;
                double z = s->zmin + (k + 0.5) * s->dz;
                Primitive3D P = prim(s, c);
                double gx = s->enable_gravity ? s->gx[c] : 0.0;
                double gy = s->enable_gravity ? s->gy[c] : 0.0;
                double gz = s->enable_gravity ? s->gz[c] : 0.0;
                fprintf(fp, "%.6f,%.6f,%.6f,%.6e,%.6e,%.6e,%.6e,%.6e,%.6e,%.6e,%.6e\n", x, y, z, P.rho,
                        P.u, P.v, P.w, P.p, gx, gy, gz);
            }
    fclose(fp);
}

void write_output_vtk(const GodunovHLLC3D *solver, int step)   /* :2376-2435 */
{
    GodunovHLLC3D *s = (GodunovHLLC3D *)solver;
    solver3d_sync_host(s);
    char fn[256];
    sprintf(fn, "output/output_%06d.vtk", step);
    FILE *fp = fopen(fn, "w");
    if (!fp) {
        fprintf(stderr, "Error: Could not open file %s for writing.\n", fn);
        return;
    }
    size_t n = ncells(s);
    fprintf(fp, "# vtk DataFile Version 3.0\n");
    fprintf(fp, "3D Hydro Simulation Output\n");
    fprintf(fp, "ASCII\n");
    fprintf(fp, "DATASET STRUCTURED_POINTS\n");
    fprintf(fp, "DIMENSIONS %d %d %d\n", s->nx, s->ny, s->nz);
    fprintf(fp, "ORIGIN %f %f %f\n", s->xmin, s->ymin, s->zmin);
    fprintf(fp, "SPACING %f %f %f\n", s->dx, s->dy, s->dz);
    fprintf(fp, "POINT_DATA %d\n", s->nx * s->ny * s->nz);
    fprintf(fp, "SCALARS density float 1\n");
    fprintf(fp, "LOOKUP_TABLE default\n");
    for (size_t c = 0; c < n; c++) fprintf(fp, "%e\n", prim(s, c).rho);
    fprintf(fp, "SCALARS pressure float 1\n");
    fprintf(fp, "LOOKUP_TABLE default\n");
    for (size_t c = 0; c < n; c++) fprintf(fp, "%e\n", prim(s, c).p);
    fprintf(fp, "VECTORS velocity float\n");
    for (size_t c = 0; c < n; c++) {
        Primitive3D P = prim(s, c);
        fprintf(fp, "%e %e %e\n", P.u, P.v, P.w);
    }
    fclose(fp);
}

/* ---------------------------------------------------------------- restart */
int load_from_csv_restart(GodunovHLLC3D *s, const char *filename)   /* :2139-2235 */
{
    {   /* a binary checkpoint of this library: exact restart */
        FILE *b = fopen(filename, "rb");
        char magic[8] = { 0 };
        const int bin = b && fread(magic, 1, 8, b) == 8 && memcmp(magic, "HCCKPT01", 8) == 0;
        if (b) fclose(b);
        if (bin) {
            double t = 0.0;
            long long st = 0;
            if (solver3d_read_checkpoint(s, filename, &t, &st)) return -1;
            printf("Loaded binary checkpoint %s (t = %.17g, step %lld)\n", filename, t, st);
            return 0;
        }
    }
    FILE *fp = fopen(filename, "r");
    if (!fp) {
        fprintf(stderr, "Error: Could not open restart file '%s'\n", filename);
        return -1;
    }
    printf("Loading restart data from: %s\n", filename);
    char line[1024];
    if (!fgets(line, sizeof line, fp)) {
        fprintf(stderr, "Error: Could not read header from restart file\n");
        fclose(fp);
        return -1;
    }
    if (strstr(line, "rho") == NULL || strstr(line, "u") == NULL) {
        fprintf(stderr, "Error: Invalid header format in restart file\n");
        fprintf(stderr, "Expected: x,y,z,rho,u,v,w,p,gx,gy,gz\n");
        fclose(fp);
        return -1;
    }
    size_t n = ncells(s);
    memset(s->U, 0, n * sizeof(State3D));
    int points = 0;
    double x, y, z, rho, u, v, w, p, gx, gy, gz;
    while (fgets(line, sizeof line, fp)) {
        int got = sscanf(line, "%lf,%lf,%lf,%lf,%lf,%lf,%lf,%lf,%lf,%lf,%lf", &x, &y, &z, &rho, &u, &v,
                         &w, &p, &gx, &gy, &gz);
        if (got < 8) {
            got = sscanf(line, "%lf,%lf,%lf,%lf,%lf,%lf,%lf,%lf", &x, &y, &z, &rho, &u, &v, &w, &p);
            gx = gy = gz = 0.0;
        }
        if (got < 8) continue;
        int i = (int)((x - s->xmin) / s->dx);
        int j = (int)((y - s->ymin) / s->dy);
        int k = (int)((z - s->zmin) / s->dz);
        if (i >= 0 && i < s->nx && j >= 0 && j < s->ny && k >= 0 && k < s->nz) {
            size_t c = ((size_t)i * s->ny + j) * s->nz + k;
            Primitive3D P = { rho, u, v, w, p };
            s->U[c] = hc_ic_prim_to_cons(P, s->gamma);
            if (s->enable_gravity && got >= 11) {
                s->gx[c] = gx; s->gy[c] = gy; s->gz[c] = gz;
            }
            points++;
        }
    }
    fclose(fp);
    printf("Successfully loaded %d data points from restart file\n", points);
    if ((size_t)points < n / 10) {
        fprintf(stderr, "Warning: Only loaded %d points out of %zu cells. This may indicate:\n", points, n);
        fprintf(stderr, "  - The restart file was subsampled\n");
        fprintf(stderr, "  - Different grid resolution\n");
        fprintf(stderr, "  - Incomplete or corrupted file\n");
    }
    s->host_dirty = 1;
    s->device_dirty = 0;
    return 0;
}

/* ---------------------------------------------------------------- run loops */
static void run_loop(GodunovHLLC3D *s, double t, double t_end, double output_dt, int output_count,
                     double next_output_time)
{
    int step_counter = 0;
    while (t < t_end) {                                /* hydro_solver_3d.c:2257-2275 */
        if (solver3d_step(s, 1) < -1) {
            fprintf(stderr, "Error: stopping the run after a device failure.\n");
            break;
        }
        t += s->dt;
        step_counter++;
        if (t >= next_output_time) {
            write_output_to_file_3d(s, output_count);
            write_output_vtk(s, output_count);
            printf("Step %d, t = %.5f, dt = %.5e, Output %d\n", step_counter, t, s->dt, output_count);
            output_count++;
            next_output_time += output_dt;
        }
        if (step_counter % s->log_every == 0)
            printf("Step %d, t = %.5f, dt = %.5e\n", step_counter, t, s->dt);
        if (s->checkpoint_every > 0 && step_counter % s->checkpoint_every == 0)
            solver3d_write_checkpoint(s, s->checkpoint_file, t, s->steps_taken);   /* written in the background */
        if (s->max_steps > 0 && step_counter >= s->max_steps) break;
    }
    if (s->dev && hc_checkpoint_wait(s->dev) != HC_OK)
        fprintf(stderr, "Error: checkpoint %s: %s\n", s->checkpoint_file, hc_last_error());
    if (t - (next_output_time - output_dt) > 1e-6) {
        write_output_to_file_3d(s, output_count);
        write_output_vtk(s, output_count);
    }
    printf("Simulation completed: %d steps, final time: %.5f\n", step_counter, t);
}

void run_simulation_3d(GodunovHLLC3D *s, double t_end, double output_dt)   /* :2241-2284 */
{
    printf("Starting 3D simulation from t=0.0 to t=%.5f\n", t_end);
    printf("Grid: %d x %d x %d = %d cells\n", s->nx, s->ny, s->nz, s->nx * s->ny * s->nz);
    write_output_to_file_3d(s, 0);
    write_output_vtk(s, 0);
    run_loop(s, 0.0, t_end, output_dt, 1, output_dt);
}

void run_simulation_3d_restart(GodunovHLLC3D *s, double t_start, double t_end, double output_dt,
                               int start_output_count)   /* :2286-2330 */
{
    if (s->ck_restored && s->ck_t != t_start) {
        printf("Binary checkpoint: starting from its stored time t = %.17g (restart_time %.5f ignored)\n", s->ck_t,
               t_start);
        t_start = s->ck_t;
    }
    printf("Restarting 3D simulation from t=%.5f to t=%.5f\n", t_start, t_end);
    printf("Starting output count: %d\n", start_output_count);
    printf("Grid: %d x %d x %d = %d cells\n", s->nx, s->ny, s->nz, s->nx * s->ny * s->nz);
    write_output_to_file_3d(s, start_output_count);
    write_output_vtk(s, start_output_count);
    run_loop(s, t_start, t_end, output_dt, start_output_count + 1, t_start + output_dt);
}
