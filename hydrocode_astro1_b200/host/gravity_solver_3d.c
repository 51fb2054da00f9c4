/*
 * gravity_solver_3d.c -- the reference's gravity API (gravity_solver_3d.h)
 * on the B200 library.  The Poisson solve runs on the device through the C
 * ABI of hydrocode_b200.h, in FP64 with the reference's operation order, so
 * phi, the iteration count and the residual equal the reference's.
 *
 * Standalone use (a caller passes a host density): each call uploads rho and
 * the current host phi (the reference warm-starts from it), solves, and
 * copies phi back.  When a hydro solver owns this object the device context
 * of the hydro solver does the work and the host arrays are refreshed at
 * output time.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "gravity_solver_3d.h"
#include "hydrocode_b200.h"

static int is_quasi_2d(const GravitySolver3D *s)   /* gravity_solver_3d.c:26-43 */
{
    if (s->nz == 1) return 1;
    double ar = (s->xmax - s->xmin) / (s->zmax - s->zmin);
    return ar > 10.0 && s->nz > 1;
}

GravitySolver3D *gravity_solver_create(int nx, int ny, int nz, double xmin, double xmax,
                                       double ymin, double ymax, double zmin, double zmax,
                                       double G)
{
    GravitySolver3D *s = (GravitySolver3D *)calloc(1, sizeof(GravitySolver3D));
    if (!s) {
        fprintf(stderr, "Error: Failed to allocate gravity solver structure.\n");
        return NULL;
    }
    s->nx = nx; s->ny = ny; s->nz = nz;
    s->xmin = xmin; s->xmax = xmax;
    s->ymin = ymin; s->ymax = ymax;
    s->zmin = zmin; s->zmax = zmax;
    s->dx = (xmax - xmin) / nx;
    s->dy = (ymax - ymin) / ny;
    s->dz = (zmax - zmin) / nz;
    s->G = G;
    s->omega = 1.5;                 /* gravity_solver_3d.c:78-82 */
    s->max_iterations = 10000;
    s->tolerance = 1.0e-6;
    s->bc_type = GRAV_BC_ISOLATED;
    size_t n = (size_t)nx * ny * nz;
    s->phi = (double *)calloc(n, sizeof(double));
    s->gx = (double *)calloc(n, sizeof(double));
    s->gy = (double *)calloc(n, sizeof(double));
    s->gz = (double *)calloc(n, sizeof(double));
    if (!s->phi || !s->gx || !s->gy || !s->gz) {
        fprintf(stderr, "Error: Failed to allocate gravity solver arrays.\n");
        gravity_solver_destroy(s);
        return NULL;
    }
    printf("Gravity solver: Using multipole expansion boundary conditions\n");
    printf("  - Monopole + quadrupole terms for accurate isolated boundaries\n");
    printf("  - Eliminates artifacts from phi=0 assumption\n");
    if (is_quasi_2d(s)) {
        if (nz == 1) printf("Gravity solver: Initialized in TRUE 2D mode (nz=1)\n");
        else printf("Gravity solver: Initialized in QUASI-2D mode (aspect ratio %.1f:1)\n",
                    (xmax - xmin) / (zmax - zmin));
    }
    return s;
}

void gravity_solver_destroy(GravitySolver3D *s)
{
    if (!s) return;
    if (s->dev && !s->owned) hc_destroy(s->dev);
    free(s->phi); free(s->gx); free(s->gy); free(s->gz);
    free(s);   /* rho is borrowed */
}

void gravity_set_solver_params(GravitySolver3D *s, double omega, int max_iter, double tol)
{
    s->omega = omega;
    s->max_iterations = max_iter;
    s->tolerance = tol;
    if (s->dev && !s->owned) hc_set_gravity_params(s->dev, omega, max_iter, tol);
}

void gravity_set_boundary_type(GravitySolver3D *s, GravBCType bc)
{
    s->bc_type = bc;
    if (s->dev && !s->owned) hc_set_gravity_bc(s->dev, (int)bc);
}

void gravity_get_diagnostics(const GravitySolver3D *s, int *iterations, double *residual)
{
    if (iterations) *iterations = s->last_iterations;
    if (residual) *residual = s->last_residual;
}

static struct hc_ctx *standalone_ctx(GravitySolver3D *s)
{
    if (s->dev && !s->owned) return s->dev;
    hc_config c;
    hc_config_default(&c);
    c.nx = s->nx; c.ny = s->ny; c.nz = s->nz;
    c.xmin = s->xmin; c.xmax = s->xmax; c.ymin = s->ymin; c.ymax = s->ymax;
    c.zmin = s->zmin; c.zmax = s->zmax;
    c.G = s->G;
    c.gravity_only = 1;
    c.precision = HC_FP64;
    c.moment_order = s->moment_order;
    c.lmax = s->lmax;
    c.grav_bc = (int)s->bc_type;
    c.omega = s->omega;
    c.max_iter = s->max_iterations;
    c.tol = s->tolerance;
    struct hc_ctx *d = hc_create(&c);
    if (!d) {
        fprintf(stderr, "Error: gravity device context: %s\n", hc_last_error());
        return NULL;
    }
    if (s->owned) {
        /* a hydro-owned object used directly: keep its own context apart */
        fprintf(stderr, "Note: gravity_solve_potential on a hydro-owned solver uses a separate device context\n");
    }
    s->dev = d;
    s->owned = 0;
    return d;
}

int gravity_solve_potential(GravitySolver3D *s, const double *rho)
{
    static int first_call = 1;   /* gravity_solver_3d.c:552-564 */
    if (first_call) {
        if (s->nz == 1) {
            printf("Gravity solver: Using TRUE 2D Poisson equation\n");
        } else if (is_quasi_2d(s)) {
            printf("Gravity solver: Using QUASI-2D mode (WARNING: may have convergence issues)\n");
        } else {
            printf("Gravity solver: Using full 3D Poisson equation\n");
        }
        first_call = 0;
    }
    s->rho = (double *)rho;
    struct hc_ctx *d = standalone_ctx(s);
    if (!d) return -1;
    hc_set_gravity_params(d, s->omega, s->max_iterations, s->tolerance);
    hc_set_gravity_bc(d, (int)s->bc_type);
    if (hc_set_phi(d, s->phi) != HC_OK) {
        fprintf(stderr, "Error: %s\n", hc_last_error());
        return -1;
    }
    int rc = hc_gravity_solve(d, rho, 0);
    if (rc != HC_OK && rc != HC_NOT_CONVERGED) {
        fprintf(stderr, "Error: %s\n", hc_last_error());
        return -1;
    }
    hc_get_phi(d, s->phi);
    hc_diag dg;
    hc_get_diag(d, &dg);
    s->last_iterations = dg.last_iterations;
    s->last_residual = dg.last_residual;
    if (rc == HC_NOT_CONVERGED && is_quasi_2d(s) && s->nz > 1) {
        fprintf(stderr, "\nHINT: Convergence failure may be due to extreme aspect ratio.\n");
        fprintf(stderr, "      Try setting nz=1 and bc_zmin=bc_zmax=PERIODIC for true 2D simulation.\n");
    }
    return rc == HC_OK ? 0 : -1;
}

void gravity_compute_acceleration(GravitySolver3D *s)
{
    struct hc_ctx *d = standalone_ctx(s);
    if (!d) return;
    hc_set_phi(d, s->phi);
    hc_gravity_acceleration(d);
    hc_get_accel(d, s->gx, s->gy, s->gz);
}

int gravity_solve(GravitySolver3D *s, const double *rho)   /* gravity_solver_3d.c:905-911 */
{
    int st = gravity_solve_potential(s, rho);
    if (st == 0) gravity_compute_acceleration(s);
    return st;
}

void gravity_write_potential(const GravitySolver3D *s, const char *filename)   /* :913-943 */
{
    FILE *fp = fopen(filename, "w");
    if (!fp) {
        fprintf(stderr, "Error: Could not open file %s for writing potential.\n", filename);
        return;
    }
    fprintf(fp, "x,y,z,phi,rho,gx,gy,gz\n");
    for (int i = 0; i < s->nx; i++)
        for (int j = 0; j < s->ny; j++)
            for (int k = 0; k < s->nz; k++) {
                size_t c = ((size_t)i * s->ny + j) * s->nz + k;
                double x = s->xmin + (i + 0.5) * s->dx;
                double y = s->ymin + (j + 0.5) * s->dy;
                double z = s->zmin + (k + 0.5) * s->dz;
                double r = s->rho ? s->rho[c] : 0.0;
                fprintf(fp, "%.6f,%.6f,%.6f,%.6e,%.6e,%.6e,%.6e,%.6e\n", x, y, z, s->phi[c], r,
                        s->gx[c], s->gy[c], s->gz[c]);
            }
    fclose(fp);
    printf("Wrote gravitational potential to %s\n", filename);
}
