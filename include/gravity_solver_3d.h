/*
 * gravity_solver_3d.h -- the reference's self-gravity API (gravity_solver_3d.h
 * of the reference project), served by the B200 library.
 *
 * The struct keeps the reference's fields in their order (:17-43) so code that
 * reads them compiles unchanged; phi, gx, gy, gz are host mirrors of device
 * arrays, valid after gravity_solve_potential / gravity_compute_acceleration
 * return (standalone use) or after the owning hydro solver writes output.
 * One trailing field holds the device context.
 *
 * Reference interfaces (gravity_solver_3d.h:64-149):
 *   gravity_solver_create, gravity_solver_destroy, gravity_solve_potential,
 *   gravity_compute_acceleration, gravity_set_solver_params,
 *   gravity_set_boundary_type, gravity_get_diagnostics, gravity_solve,
 *   gravity_write_potential.
 */
#ifndef GRAVITY_SOLVER_3D_H
#define GRAVITY_SOLVER_3D_H

#include <stdbool.h>

#define IDX3D_GRAV(i, j, k, ny, nz) (((i) * (ny) + (j)) * (nz) + (k))

typedef enum {
    GRAV_BC_PERIODIC,
    GRAV_BC_ISOLATED,
    GRAV_BC_DIRICHLET
} GravBCType;

struct hc_ctx;

typedef struct GravitySolver3D {
    int nx, ny, nz;
    double dx, dy, dz;
    double xmin, xmax;
    double ymin, ymax;
    double zmin, zmax;

    double G;

    double *phi;
    double *rho;            /* borrowed density pointer, never freed */
    double *gx;
    double *gy;
    double *gz;

    double omega;
    int max_iterations;
    double tolerance;

    GravBCType bc_type;

    int last_iterations;
    double last_residual;

    /* ---- B200 library state (appended) ---- */
    struct hc_ctx *dev;     /* device context; NULL until first use */
    int owned;              /* 1 when a hydro solver owns the device side */
    int lmax;               /* 0: reference monopole + quadrupole */
    int moment_order;       /* 0 sequential (bit-exact), 1 tree */
} GravitySolver3D;

GravitySolver3D *gravity_solver_create(int nx, int ny, int nz,
                                       double xmin, double xmax,
                                       double ymin, double ymax,
                                       double zmin, double zmax,
                                       double G);
void gravity_solver_destroy(GravitySolver3D *solver);
int gravity_solve_potential(GravitySolver3D *solver, const double *rho_field);
void gravity_compute_acceleration(GravitySolver3D *solver);
void gravity_set_solver_params(GravitySolver3D *solver, double omega, int max_iter,
                               double tolerance);
void gravity_set_boundary_type(GravitySolver3D *solver, GravBCType bc_type);
void gravity_get_diagnostics(const GravitySolver3D *solver, int *iterations, double *residual);
int gravity_solve(GravitySolver3D *solver, const double *rho_field);
void gravity_write_potential(const GravitySolver3D *solver, const char *filename);

#endif /* GRAVITY_SOLVER_3D_H */
