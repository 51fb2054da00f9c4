/*
 * hc_oracle.h -- CPU oracle for the hydro + self-gravity time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * algorithm (hydro_solver_3d.c:158-811, gravity_solver_3d.c:164-911) on a
 * structure-of-arrays FP64 layout.  It exists to check the CUDA product path;
 * the product never links, loads or calls it.  Only tests/, the smoke check
 * of __graft_entry__.py and the cpu_baseline leg of bench.py may use it.
 *
 * Parity pin: tests/test_oracle_vs_reference.py checks it bit-for-bit against
 * the reference itself (oracle/_ref, built from the reference sources by
 * oracle/Makefile) and tests/test_golden.py against fixtures that the
 * reference produced (tests/golden/make_golden.py).
 */
#ifndef HC_ORACLE_H
#define HC_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hco_grid {
    int nx, ny, nz;
    double xmin, xmax, ymin, ymax, zmin, zmax;
    double dx, dy, dz;          /* (max-min)/n, as hydro_solver_3d.c:55-57 */
    double gamma, cfl, G;
    int bc[6];                  /* BCType per face: xmin,xmax,ymin,ymax,zmin,zmax */
    int gravity;                /* self-gravity on (the reference: G > 0) */
    int grav_bc;                /* GravBCType: 0 periodic, 1 isolated, 2 dirichlet */
    int lmax;                   /* 0: reference monopole+quadrupole; >0 spherical to lmax */
    double omega, tol;
    int max_iter;
    double *q[5];               /* rho, rhou, rhov, rhow, E : nx*ny*nz each */
    double *phi;                /* potential, persists between solves (warm start) */
    double *gx, *gy, *gz;       /* acceleration (stale if a solve fails) */
    double dt;
    int last_iter;
    double last_res;
    int recon;                  /* 0: the reference's piecewise-constant states; 1: MUSCL-Hancock
                                   (minmod-limited linear primitives, half-step predictor; no
                                   reference counterpart) */
} hco_grid;

/* One godunov_step_3d (hydro_solver_3d.c:637-811). Returns SOR status (0 ok,
 * -1 not converged, 1 gravity off). */
int hco_step(hco_grid *g);

/* compute_dt_3d (hydro_solver_3d.c:422-450): sets and returns g->dt. */
double hco_cfl_dt(hco_grid *g);
/* Its maximum signal speed max(|u_d| + c) over all cells (floor 1e-10). */
double hco_signal_max(const hco_grid *g);
/* One step with a given dt instead of the grid's own CFL dt: a slab of a
 * larger grid steps with the whole grid's dt. */
int hco_step_dt(hco_grid *g, double dt);
/* The same without the gravity solve: the source term uses g->gx/gy/gz as
 * they are (a slab whose potential was solved across all slabs). */
int hco_step_ext(hco_grid *g, double dt);

/* gravity_solve / gravity_solve_potential / gravity_compute_acceleration
 * (gravity_solver_3d.c:905, :510, :753). */
int hco_gravity_solve(hco_grid *g, const double *rho);
int hco_gravity_solve_potential(hco_grid *g, const double *rho);
void hco_gravity_acceleration(hco_grid *g);

/* compute_mass_moments + compute_quadrupole_moment (gravity_solver_3d.c:164-262):
 * out[0]=M, out[1..3]=COM, out[4..12]=Q row-major. */
void hco_moments_ref(const hco_grid *g, const double *rho, double *out);

/* apply_boundary_conditions (gravity_solver_3d.c:268-504) on g->phi. */
void hco_boundary(hco_grid *g, const double *rho);

/* Slabs (no reference counterpart; the reference steps one grid): a grid
 * that holds global planes [ioff, ioff + nx) of a grid of gnx planes along
 * x, with the whole grid's xmin, xmax and dx.
 *   hco_moments_acc   the moment sums of compute_mass_moments (pass 0) or
 *                     compute_quadrupole_moment (pass 1, about com) over the
 *                     local planes [i0, i1), continuing acc -- slabs chained
 *                     in plane order give the single grid's sums bit for bit;
 *   hco_moments_com   the centre of mass from the pass-0 sums;
 *   hco_boundary_mom  the monopole + quadrupole face values (mom as
 *                     hco_moments_ref's out) on the local planes [i0, i1);
 *   hco_sor_half      one half sweep of a local colour; its update norm. */
void hco_moments_acc(const hco_grid *g, const double *rho, int pass, int i0, int i1, int ioff,
                     const double *com, double *acc);
void hco_moments_com(const hco_grid *g, const double *acc, double *com);
void hco_boundary_mom(hco_grid *g, const double *mom, int ioff, int gnx, int i0, int i1);
double hco_sor_half(hco_grid *g, const double *rho, int colour);

/* Extension (no reference counterpart): multipole to degree lmax about the
 * centre of mass with real solid harmonics.  com[3]; cs[(lmax+1)^2] holds
 * C_lm for m>=0 at index l*l+l+m and S_lm at index l*l+l-m. */
void hco_multipole_lmax(const hco_grid *g, const double *rho, int lmax,
                        double *com, double *cs);
void hco_boundary_lmax(hco_grid *g, int lmax, const double *com, const double *cs);

/* Post-hoc FP64 residual norm: max over the interior of
 * |(lap_nbrs(phi) - 4 pi G rho)/factor - phi|, the quantity the reference's
 * update norm measures when evaluated at a fixed phi. */
double hco_residual_norm(const hco_grid *g, const double *phi, const double *rho);
double hco_sweep_norm(hco_grid *g, const double *phi, const double *rho);

#ifdef __cplusplus
}
#endif
#endif
