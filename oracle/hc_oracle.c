/*
 * hc_oracle.c -- CPU oracle (TEST INFRASTRUCTURE ONLY, never shipped).
 *
 * A structure-of-arrays FP64 restatement of the reference time step.  Each
 * arithmetic expression keeps the reference's operand order and rounding
 * points, because the reference is built as ISO C11 (no FMA contraction, no
 * reassociation): with the same order every result is bit-identical.  The
 * multipole moments are summed in the reference's sequential (i, j, k) order
 * for the same reason.  Citations are file:line in the reference project.
 */
#include "hc_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define RHO_FLOOR 1.0e-5   /* hydro_solver_3d.h:10 */
#define P_FLOOR 1.0e-6     /* hydro_solver_3d.h:11 */

enum { BCP = 0, BCR = 1, BCO = 2 };          /* BCType, input_deck.h:30-34 */
enum { GBC_PER = 0, GBC_ISO = 1, GBC_DIR = 2 }; /* GravBCType, gravity_solver_3d.h:10-14 */

/* MIN/MAX exactly as the reference macros (gravity_solver_3d.c:7-8): the
 * second operand wins ties and NaN comparisons. */
static inline double mx(double a, double b) { return a > b ? a : b; }
static inline double mn(double a, double b) { return a < b ? a : b; }

typedef struct { double d, m[3], e; } cons_t;
typedef struct { double d, v[3], p; } prim_t;

static inline size_t at(const hco_grid *g, int i, int j, int k)
{
    return ((size_t)i * g->ny + j) * g->nz + k;   /* IDX3D, hydro_solver_3d.h:12 */
}

static inline cons_t load(const hco_grid *g, size_t c)
{
    cons_t q = { g->q[0][c], { g->q[1][c], g->q[2][c], g->q[3][c] }, g->q[4][c] };
    return q;
}

static inline void store(hco_grid *g, size_t c, cons_t q)
{
    g->q[0][c] = q.d; g->q[1][c] = q.m[0]; g->q[2][c] = q.m[1];
    g->q[3][c] = q.m[2]; g->q[4][c] = q.e;
}

/* cons_to_prim_3d, hydro_solver_3d.c:162-175 */
static inline prim_t to_prim(cons_t q, double gam)
{
    prim_t w;
    w.d = mx(q.d, RHO_FLOOR);
    w.v[0] = q.m[0] / w.d;
    w.v[1] = q.m[1] / w.d;
    w.v[2] = q.m[2] / w.d;
    double kin = 0.5 * w.d * (w.v[0] * w.v[0] + w.v[1] * w.v[1] + w.v[2] * w.v[2]);
    w.p = mx((gam - 1.0) * (q.e - kin), P_FLOOR);
    return w;
}

/* prim_to_cons_3d, hydro_solver_3d.c:177-189 */
static inline cons_t to_cons(prim_t w, double gam)
{
    cons_t q;
    q.d = w.d;
    q.m[0] = w.d * w.v[0];
    q.m[1] = w.d * w.v[1];
    q.m[2] = w.d * w.v[2];
    double kin = 0.5 * w.d * (w.v[0] * w.v[0] + w.v[1] * w.v[1] + w.v[2] * w.v[2]);
    q.e = w.p / (gam - 1.0) + kin;
    return q;
}

/* sound_speed_3d, hydro_solver_3d.c:191-193 */
static inline double csound(prim_t w, double gam) { return sqrt(gam * w.p / w.d); }

/* compute_flux_{x,y,z}_3d, hydro_solver_3d.c:199-233, for normal axis a. */
static inline cons_t euler_flux(cons_t q, prim_t w, int a)
{
    cons_t f;
    f.d = q.m[a];
    for (int c = 0; c < 3; c++) f.m[c] = q.m[c] * w.v[a];
    f.m[a] = q.m[a] * w.v[a] + w.p;
    f.e = (q.e + w.p) * w.v[a];
    return f;
}

/* hllc_riemann_solver_{x,y,z}_3d, hydro_solver_3d.c:239-416.  The three
 * reference functions differ only in which velocity component is normal;
 * here the axis is a parameter. */
static cons_t hllc(cons_t qL, cons_t qR, int a, double gam)
{
    prim_t wL = to_prim(qL, gam), wR = to_prim(qR, gam);
    double cL = csound(wL, gam), cR = csound(wR, gam);
    double sL = mn(wL.v[a] - cL, wR.v[a] - cR);
    double sR = mx(wL.v[a] + cL, wR.v[a] + cR);
    if (sL >= 0.0) return euler_flux(qL, wL, a);
    if (sR <= 0.0) return euler_flux(qR, wR, a);

    double num = wR.p - wL.p + wL.d * wL.v[a] * (sL - wL.v[a]) - wR.d * wR.v[a] * (sR - wR.v[a]);
    double den = wL.d * (sL - wL.v[a]) - wR.d * (sR - wR.v[a]);
    double ss = num / den;

    /* left star state if the contact moves right (or is at rest) */
    int left = ss >= 0.0;
    cons_t qK = left ? qL : qR;
    prim_t wK = left ? wL : wR;
    double sK = left ? sL : sR;

    double fac = (sK - wK.v[a]) / (sK - ss);
    cons_t st;
    st.d = wK.d * fac;
    for (int c = 0; c < 3; c++) st.m[c] = st.d * (c == a ? ss : wK.v[c]);
    st.e = st.d * (qK.e / wK.d + (ss - wK.v[a]) * (ss + wK.p / (wK.d * (sK - wK.v[a]))));

    cons_t f = euler_flux(qK, wK, a);
    f.d = f.d + sK * (st.d - qK.d);
    for (int c = 0; c < 3; c++) f.m[c] = f.m[c] + sK * (st.m[c] - qK.m[c]);
    f.e = f.e + sK * (st.e - qK.e);
    return f;
}

/* The maximum signal speed of compute_dt_3d, hydro_solver_3d.c:422-442. */
double hco_signal_max(const hco_grid *g)
{
    double smax = 1.0e-10;
    size_t n = (size_t)g->nx * g->ny * g->nz;
    for (size_t c = 0; c < n; c++) {
        prim_t w = to_prim(load(g, c), g->gamma);
        double cs = csound(w, g->gamma);
        smax = mx(smax, fabs(w.v[0]) + cs);
        smax = mx(smax, fabs(w.v[1]) + cs);
        smax = mx(smax, fabs(w.v[2]) + cs);
    }
    return smax;
}

/* compute_dt_3d, hydro_solver_3d.c:422-450 */
double hco_cfl_dt(hco_grid *g)
{
    double smax = hco_signal_max(g);
    double tx = g->dx / smax, ty = g->dy / smax, tz = g->dz / smax;
    g->dt = g->cfl * mn(tx, mn(ty, tz));
    return g->dt;
}

/* ------------------------------------------------------------------------ */
/* Gravity                                                                   */
/* ------------------------------------------------------------------------ */

/* gravity_solver_3d.c:164-262: sequential sums over cells with rho > 0, in
 * (i,j,k) order over the local planes [i0, i1), continuing the sums in acc.
 * The grid holds global planes [ioff, ioff + nx); xmin and dx are the whole
 * grid's, so x = xmin + (i + ioff + 0.5) dx is the whole grid's coordinate
 * bit for bit.  pass 0: acc[0..3] = (M, sum dm x, sum dm y, sum dm z);
 * pass 1: acc[0..8] = Q_ij about com[0..2]. */
void hco_moments_acc(const hco_grid *g, const double *rho, int pass, int i0, int i1, int ioff,
                     const double *com, double *acc)
{
    const double dV = g->dx * g->dy * g->dz;
    for (int i = i0; i < i1; i++)
        for (int j = 0; j < g->ny; j++)
            for (int k = 0; k < g->nz; k++) {
                double r = rho[at(g, i, j, k)];
                if (!(r > 0.0)) continue;
                double dm = r * dV;
                if (pass == 0) {
                    double x = g->xmin + (i + ioff + 0.5) * g->dx;
                    double y = g->ymin + (j + 0.5) * g->dy;
                    double z = g->zmin + (k + 0.5) * g->dz;
                    acc[0] += dm; acc[1] += dm * x; acc[2] += dm * y; acc[3] += dm * z;
                } else {
                    double x = g->xmin + (i + ioff + 0.5) * g->dx - com[0];
                    double y = g->ymin + (j + 0.5) * g->dy - com[1];
                    double z = g->zmin + (k + 0.5) * g->dz - com[2];
                    double r2 = x * x + y * y + z * z;
                    acc[0] += dm * (3.0 * x * x - r2);
                    acc[1] += dm * (3.0 * x * y);
                    acc[2] += dm * (3.0 * x * z);
                    acc[3] += dm * (3.0 * y * x);
                    acc[4] += dm * (3.0 * y * y - r2);
                    acc[5] += dm * (3.0 * y * z);
                    acc[6] += dm * (3.0 * z * x);
                    acc[7] += dm * (3.0 * z * y);
                    acc[8] += dm * (3.0 * z * z - r2);
                }
            }
}

/* Centre of mass from the pass-0 sums (gravity_solver_3d.c:205-215): the
 * box centre when there is no mass. */
void hco_moments_com(const hco_grid *g, const double *acc, double *com)
{
    const double M = acc[0];
    if (M > 0.0) { com[0] = acc[1] / M; com[1] = acc[2] / M; com[2] = acc[3] / M; }
    else {
        com[0] = 0.5 * (g->xmin + g->xmax);
        com[1] = 0.5 * (g->ymin + g->ymax);
        com[2] = 0.5 * (g->zmin + g->zmax);
    }
}

void hco_moments_ref(const hco_grid *g, const double *rho, double *out)
{
    double acc[4] = { 0 }, com[3], Q[9] = { 0 };
    hco_moments_acc(g, rho, 0, 0, g->nx, 0, NULL, acc);
    hco_moments_com(g, acc, com);
    hco_moments_acc(g, rho, 1, 0, g->nx, 0, com, Q);
    out[0] = acc[0]; out[1] = com[0]; out[2] = com[1]; out[3] = com[2];
    memcpy(out + 4, Q, sizeof Q);
}

/* Monopole + quadrupole potential at one boundary point,
 * gravity_solver_3d.c:323-345 (identical in all six face blocks). */
static double mono_quad(double x, double y, double z, const double *mom, double G)
{
    double rx = x - mom[1], ry = y - mom[2], rz = z - mom[3];
    double r = sqrt(rx * rx + ry * ry + rz * rz);
    double ph = 0.0;
    if (r > 0.0) {
        const double *Q = mom + 4;
        ph = -G * mom[0] / r;
        double r5 = r * r * r * r * r;
        double Qr = Q[0] * rx * rx + Q[1] * rx * ry + Q[2] * rx * rz +
                    Q[3] * ry * rx + Q[4] * ry * ry + Q[5] * ry * rz +
                    Q[6] * rz * rx + Q[7] * rz * ry + Q[8] * rz * rz;
        ph += -G * Qr / (2.0 * r5);
    }
    return ph;
}

/* apply_boundary_conditions, gravity_solver_3d.c:268-504.  Face order x, y,
 * then z (z only when nz > 1); later faces overwrite shared edges. */
void hco_boundary(hco_grid *g, const double *rho)
{
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    double *phi = g->phi;
    if (g->grav_bc == GBC_PER) {
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) phi[at(g, 0, j, k)] = phi[at(g, nx - 1, j, k)];
        for (int i = 0; i < nx; i++)
            for (int k = 0; k < nz; k++) phi[at(g, i, 0, k)] = phi[at(g, i, ny - 1, k)];
        if (nz > 1)
            for (int i = 0; i < nx; i++)
                for (int j = 0; j < ny; j++) phi[at(g, i, j, 0)] = phi[at(g, i, j, nz - 1)];
        return;
    }
    if (g->grav_bc != GBC_ISO) return;  /* DIRICHLET: keep current values */
    if (g->lmax > 0) {
        int nm = (g->lmax + 1) * (g->lmax + 1);
        double com[3];
        double *cs = (double *)malloc(sizeof(double) * nm);
        hco_multipole_lmax(g, rho, g->lmax, com, cs);
        hco_boundary_lmax(g, g->lmax, com, cs);
        free(cs);
        return;
    }
    double mom[13];
    hco_moments_ref(g, rho, mom);
    hco_boundary_mom(g, mom, 0, nx, 0, nx);
}

/* The monopole + quadrupole face loops of apply_boundary_conditions
 * (gravity_solver_3d.c:302-498) over the local planes [i0, i1) of a grid
 * that holds global planes [ioff, ioff + nx) of gnx: the x faces where the
 * global planes 0 and gnx - 1 are held, then the y and z faces of those
 * planes, in the reference's order (later faces overwrite shared edges). */
void hco_boundary_mom(hco_grid *g, const double *mom, int ioff, int gnx, int i0, int i1)
{
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    double *phi = g->phi;
    const double G = g->G;
    const int xlo = ioff == 0 && i0 == 0, xhi = ioff + nx == gnx && i1 == nx;
    for (int j = 0; j < ny; j++)
        for (int k = 0; k < nz; k++) {
            double y = g->ymin + (j + 0.5) * g->dy, z = g->zmin + (k + 0.5) * g->dz;
            if (xlo) phi[at(g, 0, j, k)] = mono_quad(g->xmin + 0.5 * g->dx, y, z, mom, G);
            if (xhi) phi[at(g, nx - 1, j, k)] = mono_quad(g->xmax - 0.5 * g->dx, y, z, mom, G);
        }
    for (int i = i0; i < i1; i++)
        for (int k = 0; k < nz; k++) {
            double x = g->xmin + (i + ioff + 0.5) * g->dx, z = g->zmin + (k + 0.5) * g->dz;
            phi[at(g, i, 0, k)] = mono_quad(x, g->ymin + 0.5 * g->dy, z, mom, G);
            phi[at(g, i, ny - 1, k)] = mono_quad(x, g->ymax - 0.5 * g->dy, z, mom, G);
        }
    if (nz > 1)
        for (int i = i0; i < i1; i++)
            for (int j = 0; j < ny; j++) {
                double x = g->xmin + (i + ioff + 0.5) * g->dx, y = g->ymin + (j + 0.5) * g->dy;
                phi[at(g, i, j, 0)] = mono_quad(x, y, g->zmin + 0.5 * g->dz, mom, G);
                phi[at(g, i, j, nz - 1)] = mono_quad(x, y, g->zmax - 0.5 * g->dz, mom, G);
            }
}

/* ---- extension: real solid-harmonic multipole to degree lmax ------------
 * Q_l^m = r^l P_l^m(cos t) e^{i m p} (no Condon-Shortley phase) obeys
 *   Q_0^0 = 1, Q_m^m = (2m-1)(x+iy) Q_{m-1}^{m-1}, Q_{m+1}^m = (2m+1) z Q_m^m,
 *   (l-m) Q_l^m = (2l-1) z Q_{l-1}^m - (l+m-1) r^2 Q_{l-2}^m.
 * With N_lm = sqrt((2-d_m0)(l-m)!/(l+m)!) the addition theorem gives
 *   1/|r-r'| = sum_l sum_m N_lm^2 Re[Q_l^m(r') conj(Q_l^m(r))] / r^(2l+1),
 * so C_lm = sum dm N Re Q_l^m(r'), S_lm = sum dm N Im Q_l^m(r') and
 *   phi(r) = -G sum_l sum_m N (C_lm Re Q_l^m(r) + S_lm Im Q_l^m(r)) / r^(2l+1).
 * At lmax = 2 this equals the reference's monopole + traceless quadrupole
 * (gravity_solver_3d.c:332-345) up to rounding. */
#define HCO_LMAX_MAX 16
static void solid_harmonics(double x, double y, double z, int lmax, double *re, double *im)
{
    /* re/im indexed l*(lmax+1)+m */
    const int L = lmax + 1;
    double r2 = x * x + y * y + z * z;
    re[0] = 1.0; im[0] = 0.0;
    for (int m = 1; m <= lmax; m++) {
        double pr = re[(m - 1) * L + m - 1], pi = im[(m - 1) * L + m - 1];
        re[m * L + m] = (2 * m - 1) * (x * pr - y * pi);
        im[m * L + m] = (2 * m - 1) * (x * pi + y * pr);
    }
    for (int m = 0; m <= lmax; m++) {
        if (m + 1 <= lmax) {
            re[(m + 1) * L + m] = (2 * m + 1) * z * re[m * L + m];
            im[(m + 1) * L + m] = (2 * m + 1) * z * im[m * L + m];
        }
        for (int l = m + 2; l <= lmax; l++) {
            double a = (double)(2 * l - 1), b = (double)(l + m - 1), c = 1.0 / (double)(l - m);
            re[l * L + m] = (a * z * re[(l - 1) * L + m] - b * r2 * re[(l - 2) * L + m]) * c;
            im[l * L + m] = (a * z * im[(l - 1) * L + m] - b * r2 * im[(l - 2) * L + m]) * c;
        }
    }
}

static double norm_lm(int l, int m)
{
    double v = (m == 0) ? 1.0 : 2.0;
    for (int t = l - m + 1; t <= l + m; t++) v /= (double)t;
    return sqrt(v);
}

void hco_multipole_lmax(const hco_grid *g, const double *rho, int lmax,
                        double *com, double *cs)
{
    double mom[13];
    hco_moments_ref(g, rho, mom);   /* centre of mass as the reference */
    com[0] = mom[1]; com[1] = mom[2]; com[2] = mom[3];
    const int L = lmax + 1, nm = L * L;
    double re[(HCO_LMAX_MAX + 1) * (HCO_LMAX_MAX + 1)], im[(HCO_LMAX_MAX + 1) * (HCO_LMAX_MAX + 1)];
    double nrm[(HCO_LMAX_MAX + 1) * (HCO_LMAX_MAX + 1)];
    for (int l = 0; l <= lmax; l++)
        for (int m = 0; m <= l; m++) nrm[l * L + m] = norm_lm(l, m);
    for (int t = 0; t < nm; t++) cs[t] = 0.0;
    const double dV = g->dx * g->dy * g->dz;
    for (int i = 0; i < g->nx; i++)
        for (int j = 0; j < g->ny; j++)
            for (int k = 0; k < g->nz; k++) {
                double r = rho[at(g, i, j, k)];
                if (!(r > 0.0)) continue;
                double x = g->xmin + (i + 0.5) * g->dx - com[0];
                double y = g->ymin + (j + 0.5) * g->dy - com[1];
                double z = g->zmin + (k + 0.5) * g->dz - com[2];
                double dm = r * dV;
                solid_harmonics(x, y, z, lmax, re, im);
                for (int l = 0; l <= lmax; l++)
                    for (int m = 0; m <= l; m++) {
                        double w = dm * nrm[l * L + m];
                        cs[l * l + l + m] += w * re[l * L + m];
                        if (m > 0) cs[l * l + l - m] += w * im[l * L + m];
                    }
            }
}

static double eval_lmax(double x, double y, double z, int lmax, const double *com,
                        const double *cs, double G)
{
    const int L = lmax + 1;
    double re[(HCO_LMAX_MAX + 1) * (HCO_LMAX_MAX + 1)], im[(HCO_LMAX_MAX + 1) * (HCO_LMAX_MAX + 1)];
    double rx = x - com[0], ry = y - com[1], rz = z - com[2];
    double r2 = rx * rx + ry * ry + rz * rz;
    if (!(r2 > 0.0)) return 0.0;
    double r = sqrt(r2);
    solid_harmonics(rx, ry, rz, lmax, re, im);
    double sum = 0.0, inv = 1.0 / r, rpow = inv;   /* 1/r^(2l+1) */
    double inv2 = inv * inv;
    for (int l = 0; l <= lmax; l++) {
        double sl = 0.0;
        for (int m = 0; m <= l; m++) {
            double n = norm_lm(l, m);
            double t = cs[l * l + l + m] * re[l * L + m];
            if (m > 0) t += cs[l * l + l - m] * im[l * L + m];
            sl += n * t;
        }
        sum += sl * rpow;
        rpow *= inv2;
    }
    return -G * sum;
}

void hco_boundary_lmax(hco_grid *g, int lmax, const double *com, const double *cs)
{
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const double G = g->G;
    for (int j = 0; j < ny; j++)
        for (int k = 0; k < nz; k++) {
            double y = g->ymin + (j + 0.5) * g->dy, z = g->zmin + (k + 0.5) * g->dz;
            g->phi[at(g, 0, j, k)] = eval_lmax(g->xmin + 0.5 * g->dx, y, z, lmax, com, cs, G);
            g->phi[at(g, nx - 1, j, k)] = eval_lmax(g->xmax - 0.5 * g->dx, y, z, lmax, com, cs, G);
        }
    for (int i = 0; i < nx; i++)
        for (int k = 0; k < nz; k++) {
            double x = g->xmin + (i + 0.5) * g->dx, z = g->zmin + (k + 0.5) * g->dz;
            g->phi[at(g, i, 0, k)] = eval_lmax(x, g->ymin + 0.5 * g->dy, z, lmax, com, cs, G);
            g->phi[at(g, i, ny - 1, k)] = eval_lmax(x, g->ymax - 0.5 * g->dy, z, lmax, com, cs, G);
        }
    if (nz > 1)
        for (int i = 0; i < nx; i++)
            for (int j = 0; j < ny; j++) {
                double x = g->xmin + (i + 0.5) * g->dx, y = g->ymin + (j + 0.5) * g->dy;
                g->phi[at(g, i, j, 0)] = eval_lmax(x, y, g->zmin + 0.5 * g->dz, lmax, com, cs, G);
                g->phi[at(g, i, j, nz - 1)] = eval_lmax(x, y, g->zmax - 0.5 * g->dz, lmax, com, cs, G);
            }
}

/* One red or black half sweep, gravity_solver_3d.c:642-708 (3D) and
 * :577-633 (nz == 1).  Returns max |phi_GS - phi_old| over the colour. */
static double sor_color(hco_grid *g, const double *rho, int color,
                        double ix2, double iy2, double iz2, double fpg, double fac)
{
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const double om = g->omega;
    double *phi = g->phi;
    double res = 0.0;
    const size_t sj = (size_t)nz, si = (size_t)ny * nz;
    if (nz == 1) {
        for (int i = 1; i < nx - 1; i++)
            for (int j = 1; j < ny - 1; j++) {
                if ((i + j) % 2 != color) continue;
                size_t c = at(g, i, j, 0);
                double old = phi[c];
                double lap = (phi[c - si] + phi[c + si]) * ix2 + (phi[c - sj] + phi[c + sj]) * iy2;
                double nw = (lap - fpg * rho[c]) / fac;
                phi[c] = old + om * (nw - old);
                res = mx(res, fabs(nw - old));
            }
        return res;
    }
    for (int i = 1; i < nx - 1; i++)
        for (int j = 1; j < ny - 1; j++) {
            int k0 = ((i + j + 1) % 2 == color) ? 1 : 2;
            for (int k = k0; k < nz - 1; k += 2) {
                size_t c = at(g, i, j, k);
                double old = phi[c];
                double lap = (phi[c - si] + phi[c + si]) * ix2 +
                             (phi[c - sj] + phi[c + sj]) * iy2 +
                             (phi[c - 1] + phi[c + 1]) * iz2;
                double nw = (lap - fpg * rho[c]) / fac;
                phi[c] = old + om * (nw - old);
                res = mx(res, fabs(nw - old));
            }
        }
    return res;
}

static double sor_factor(const hco_grid *g, double *ix2, double *iy2, double *iz2)
{
    *ix2 = 1.0 / (g->dx * g->dx);
    *iy2 = 1.0 / (g->dy * g->dy);
    *iz2 = 1.0 / (g->dz * g->dz);
    return g->nz == 1 ? 2.0 * (*ix2 + *iy2) : 2.0 * (*ix2 + *iy2 + *iz2);
}

/* One half sweep of local colour `colour` (cells with (i + j + k) % 2 ==
 * colour in local indices) with the grid's coefficients; returns its update
 * norm.  A slab whose first plane is global plane ioff sweeps the whole
 * grid's colour c as local colour c ^ (ioff & 1). */
double hco_sor_half(hco_grid *g, const double *rho, int colour)
{
    double ix2, iy2, iz2;
    double fac = sor_factor(g, &ix2, &iy2, &iz2);
    return sor_color(g, rho, colour, ix2, iy2, iz2, 4.0 * M_PI * g->G, fac);
}

/* gravity_solve_potential, gravity_solver_3d.c:510-747.  The boundary is
 * evaluated after every iteration in the reference; density is fixed during
 * a solve, so the values are the same each time -- they are computed once,
 * after the first iteration, which keeps the first iteration's sweeps on the
 * previous boundary values exactly as the reference does. */
int hco_gravity_solve_potential(hco_grid *g, const double *rho)
{
    double ix2, iy2, iz2;
    double fac = sor_factor(g, &ix2, &iy2, &iz2);
    double fpg = 4.0 * M_PI * g->G;
    double res = 0.0;
    int it;
    for (it = 0; it < g->max_iter; it++) {
        double r0 = sor_color(g, rho, 0, ix2, iy2, iz2, fpg, fac);
        double r1 = sor_color(g, rho, 1, ix2, iy2, iz2, fpg, fac);
        res = mx(mx(0.0, r0), r1);
        if (it == 0) hco_boundary(g, rho);
        else if (g->grav_bc == GBC_PER) hco_boundary(g, rho);
        if (res < g->tol) {
            g->last_iter = it + 1;
            g->last_res = res;
            return 0;
        }
    }
    g->last_iter = it;
    g->last_res = res;
    return -1;
}

/* gravity_compute_acceleration, gravity_solver_3d.c:753-899 */
void hco_gravity_acceleration(hco_grid *g)
{
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const double *phi = g->phi;
    double *gx = g->gx, *gy = g->gy, *gz = g->gz;
    const size_t sj = (size_t)nz, si = (size_t)ny * nz;
    if (nz == 1) {
        for (int i = 1; i < nx - 1; i++)
            for (int j = 1; j < ny - 1; j++) {
                size_t c = at(g, i, j, 0);
                gx[c] = -(phi[c + si] - phi[c - si]) / (2.0 * g->dx);
                gy[c] = -(phi[c + sj] - phi[c - sj]) / (2.0 * g->dy);
                gz[c] = 0.0;
            }
        for (int j = 0; j < ny; j++) {
            size_t a = at(g, 0, j, 0), b = at(g, nx - 1, j, 0);
            gx[a] = gy[a] = gz[a] = 0.0;
            gx[b] = gy[b] = gz[b] = 0.0;
        }
        for (int i = 0; i < nx; i++) {
            size_t a = at(g, i, 0, 0), b = at(g, i, ny - 1, 0);
            gx[a] = gy[a] = gz[a] = 0.0;
            gx[b] = gy[b] = gz[b] = 0.0;
        }
        return;
    }
    for (int i = 1; i < nx - 1; i++)
        for (int j = 1; j < ny - 1; j++)
            for (int k = 1; k < nz - 1; k++) {
                size_t c = at(g, i, j, k);
                gx[c] = -(phi[c + si] - phi[c - si]) / (2.0 * g->dx);
                gy[c] = -(phi[c + sj] - phi[c - sj]) / (2.0 * g->dy);
                gz[c] = -(phi[c + 1] - phi[c - 1]) / (2.0 * g->dz);
            }
    /* boundary copies in the order x, y, z (gravity_solver_3d.c:842-897) */
    for (int j = 0; j < ny; j++)
        for (int k = 0; k < nz; k++) {
            size_t a = at(g, 0, j, k), b = at(g, 1, j, k);
            gx[a] = gx[b]; gy[a] = gy[b]; gz[a] = gz[b];
            a = at(g, nx - 1, j, k); b = at(g, nx - 2, j, k);
            gx[a] = gx[b]; gy[a] = gy[b]; gz[a] = gz[b];
        }
    for (int i = 0; i < nx; i++)
        for (int k = 0; k < nz; k++) {
            size_t a = at(g, i, 0, k), b = at(g, i, 1, k);
            gx[a] = gx[b]; gy[a] = gy[b]; gz[a] = gz[b];
            a = at(g, i, ny - 1, k); b = at(g, i, ny - 2, k);
            gx[a] = gx[b]; gy[a] = gy[b]; gz[a] = gz[b];
        }
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++) {
            size_t a = at(g, i, j, 0), b = at(g, i, j, 1);
            gx[a] = gx[b]; gy[a] = gy[b]; gz[a] = gz[b];
            a = at(g, i, j, nz - 1); b = at(g, i, j, nz - 2);
            gx[a] = gx[b]; gy[a] = gy[b]; gz[a] = gz[b];
        }
}

/* gravity_solve, gravity_solver_3d.c:905-911: acceleration only on success. */
int hco_gravity_solve(hco_grid *g, const double *rho)
{
    int st = hco_gravity_solve_potential(g, rho);
    if (st == 0) hco_gravity_acceleration(g);
    return st;
}

double hco_residual_norm(const hco_grid *g, const double *phi, const double *rho)
{
    double ix2, iy2, iz2;
    double fac = sor_factor(g, &ix2, &iy2, &iz2);
    double fpg = 4.0 * M_PI * g->G;
    const size_t sj = (size_t)g->nz, si = (size_t)g->ny * g->nz;
    double res = 0.0;
    for (int i = 1; i < g->nx - 1; i++)
        for (int j = 1; j < g->ny - 1; j++)
            for (int k = 1; k < g->nz - 1; k++) {
                size_t c = at(g, i, j, k);
                double lap = (phi[c - si] + phi[c + si]) * ix2 +
                             (phi[c - sj] + phi[c + sj]) * iy2 +
                             (phi[c - 1] + phi[c + 1]) * iz2;
                double nw = (lap - fpg * rho[c]) / fac;
                res = mx(res, fabs(nw - phi[c]));
            }
    return res;
}

/* The convergence test of gravity_solve_potential (gravity_solver_3d.c:
 * 702-714) applied to a given potential: the update norm max |phi_GS -
 * phi_old| of one red-black sweep started from phi (phi is not changed). */
double hco_sweep_norm(hco_grid *g, const double *phi, const double *rho)
{
    double ix2, iy2, iz2;
    double fac = sor_factor(g, &ix2, &iy2, &iz2);
    double fpg = 4.0 * M_PI * g->G;
    const size_t n = (size_t)g->nx * g->ny * g->nz;
    double *work = (double *)malloc(n * sizeof(double));
    memcpy(work, phi, n * sizeof(double));
    double *keep = g->phi;
    g->phi = work;
    double r0 = sor_color(g, rho, 0, ix2, iy2, iz2, fpg, fac);
    double r1 = sor_color(g, rho, 1, ix2, iy2, iz2, fpg, fac);
    g->phi = keep;
    free(work);
    return mx(mx(0.0, r0), r1);
}

/* ------------------------------------------------------------------------ */
/* The time step                                                             */
/* ------------------------------------------------------------------------ */

/* apply_boundary_conditions_3d, hydro_solver_3d.c:456-552: per face, a
 * reflective face negates the boundary cell's own normal velocity (through a
 * prim round trip), an outflow face copies the neighbour, periodic does
 * nothing here.  Axis order x, y, z; min face before max face. */
static void hydro_bc(hco_grid *g)
{
    const int n[3] = { g->nx, g->ny, g->nz };
    for (int a = 0; a < 3; a++) {
        int b = (a == 0) ? 1 : 0, c = (a == 2) ? 1 : 2;
        for (int u = 0; u < n[b]; u++)
            for (int v = 0; v < n[c]; v++) {
                for (int side = 0; side < 2; side++) {
                    int type = g->bc[2 * a + side];
                    int ib = side ? n[a] - 1 : 0, in = side ? n[a] - 2 : 1;
                    int idx[3], jdx[3];
                    idx[a] = ib; idx[b] = u; idx[c] = v;
                    jdx[a] = in; jdx[b] = u; jdx[c] = v;
                    size_t cb = at(g, idx[0], idx[1], idx[2]);
                    if (type == BCR) {
                        prim_t w = to_prim(load(g, cb), g->gamma);
                        w.v[a] = -w.v[a];
                        store(g, cb, to_cons(w, g->gamma));
                    } else if (type == BCO) {
                        store(g, cb, load(g, at(g, jdx[0], jdx[1], jdx[2])));
                    }
                }
            }
    }
}

/* ---- MUSCL-Hancock face states (no reference counterpart; the reference's
 * states are piecewise constant, hydro_solver_3d.c:654-724).  Per cell, on
 * primitives (rho, u, v, w, p):
 *   slopes  dW_a = minmod(W - W[-e_a], W[+e_a] - W), zero where the cell is
 *           on the domain boundary along axis a;
 *   half step (primitive Euler equations, normal velocity un = W.v[a])
 *           t_a = (un drho + rho du_a,  un du_c for c != a,  un du_a + dp/rho,
 *                  un dp + gamma p du_a),
 *           W* = W - h_x t_x - h_y t_y - h_z t_z,  h_a = 0.5 dt / d_a;
 *   faces   W* + dW_a/2 (the +a face), W* - dW_a/2 (the -a face);
 *   first order for the cell (W* = W, dW = 0) if W* or any face state has
 *           rho <= 0 or p <= 0.
 * The face flux is HLLC on the two face states turned into conserved states.
 * The CUDA path (hydro_plm.cu) forms the same values in the same order. */
static inline double minmod(double a, double b)
{
    return (a * b <= 0.0) ? 0.0 : (fabs(a) < fabs(b) ? a : b);
}

static inline void prim_arr(prim_t w, double *o)
{
    o[0] = w.d; o[1] = w.v[0]; o[2] = w.v[1]; o[3] = w.v[2]; o[4] = w.p;
}

static inline cons_t cons_of_arr(const double *o, double gam)
{
    prim_t w = { o[0], { o[1], o[2], o[3] }, o[4] };
    return to_cons(w, gam);
}

/* pl: 20 arrays of n values -- W* (5), then dW for axes x, y, z (5 each) */
static void plm_predict(const hco_grid *g, double *pl)
{
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const size_t n = (size_t)nx * ny * nz;
    const size_t str[3] = { (size_t)ny * nz, (size_t)nz, 1 };
    const int nn[3] = { nx, ny, nz };
    const double gam = g->gamma;
    const double h[3] = { 0.5 * g->dt / g->dx, 0.5 * g->dt / g->dy, 0.5 * g->dt / g->dz };
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                const size_t c = at(g, i, j, k);
                const int idx[3] = { i, j, k };
                double w[5], dw[3][5], t[3][5], ws[5];
                prim_arr(to_prim(load(g, c), gam), w);
                for (int a = 0; a < 3; a++) {
                    if (idx[a] >= 1 && idx[a] <= nn[a] - 2) {
                        double wm[5], wp[5];
                        prim_arr(to_prim(load(g, c - str[a]), gam), wm);
                        prim_arr(to_prim(load(g, c + str[a]), gam), wp);
                        for (int v = 0; v < 5; v++) dw[a][v] = minmod(w[v] - wm[v], wp[v] - w[v]);
                    } else {
                        for (int v = 0; v < 5; v++) dw[a][v] = 0.0;
                    }
                }
                for (int a = 0; a < 3; a++) {
                    const double un = w[1 + a];
                    t[a][0] = un * dw[a][0] + w[0] * dw[a][1 + a];
                    for (int cc = 0; cc < 3; cc++) t[a][1 + cc] = un * dw[a][1 + cc];
                    t[a][1 + a] = un * dw[a][1 + a] + dw[a][4] / w[0];
                    t[a][4] = un * dw[a][4] + gam * w[4] * dw[a][1 + a];
                }
                for (int v = 0; v < 5; v++) ws[v] = w[v] - h[0] * t[0][v] - h[1] * t[1][v] - h[2] * t[2][v];
                int ok = ws[0] > 0.0 && ws[4] > 0.0;
                for (int a = 0; a < 3; a++) {
                    ok = ok && (ws[0] + 0.5 * dw[a][0]) > 0.0 && (ws[4] + 0.5 * dw[a][4]) > 0.0;
                    ok = ok && (ws[0] - 0.5 * dw[a][0]) > 0.0 && (ws[4] - 0.5 * dw[a][4]) > 0.0;
                }
                if (!ok) {
                    for (int v = 0; v < 5; v++) {
                        ws[v] = w[v];
                        for (int a = 0; a < 3; a++) dw[a][v] = 0.0;
                    }
                }
                for (int v = 0; v < 5; v++) {
                    pl[v * n + c] = ws[v];
                    for (int a = 0; a < 3; a++) pl[(5 + 5 * a + v) * n + c] = dw[a][v];
                }
            }
}

/* flux through the face between cell cl and cl + e_a from the two face states */
static cons_t plm_flux(const hco_grid *g, const double *pl, size_t cl, size_t cr, int a)
{
    const size_t n = (size_t)g->nx * g->ny * g->nz;
    double L[5], R[5];
    for (int v = 0; v < 5; v++) {
        L[v] = pl[v * n + cl] + 0.5 * pl[(5 + 5 * a + v) * n + cl];
        R[v] = pl[v * n + cr] - 0.5 * pl[(5 + 5 * a + v) * n + cr];
    }
    return hllc(cons_of_arr(L, g->gamma), cons_of_arr(R, g->gamma), a, g->gamma);
}

static int step_impl(hco_grid *g, double dt_given, int solve);

int hco_step(hco_grid *g) { return step_impl(g, 0.0, 1); }

int hco_step_dt(hco_grid *g, double dt) { return step_impl(g, dt, 1); }

int hco_step_ext(hco_grid *g, double dt) { return step_impl(g, dt, 0); }

static int step_impl(hco_grid *g, double dt_given, int solve)
{
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const size_t n = (size_t)nx * ny * nz;
    const double gam = g->gamma;
    int st = 1;

    /* solve_gravity_field, hydro_solver_3d.c:558-591 (solve == 0: the caller
     * solved, and g->gx/gy/gz hold the acceleration the source uses) */
    if (g->gravity && solve) {
        double *rho = (double *)malloc(n * sizeof(double));
        memcpy(rho, g->q[0], n * sizeof(double));
        st = hco_gravity_solve(g, rho);
        free(rho);
    }

    if (dt_given > 0.0) g->dt = dt_given;
    else hco_cfl_dt(g);
    const double dt = g->dt, dx = g->dx, dy = g->dy, dz = g->dz;

    /* face fluxes F[a][c] = flux through the face between cell c and c+e_a,
     * for the faces the interior update reads (hydro_solver_3d.c:654-724).
     * The periodic wrap faces (:666-674 etc.) are never read by the update
     * loop, which stops at n-2, so they are not formed. */
    double *F[3][5];
    for (int a = 0; a < 3; a++)
        for (int v = 0; v < 5; v++) F[a][v] = (double *)calloc(n, sizeof(double));
    const size_t str[3] = { (size_t)ny * nz, (size_t)nz, 1 };
    double *pl = NULL;
    if (g->recon == 1) {
        pl = (double *)malloc(20 * n * sizeof(double));
        plm_predict(g, pl);
    }
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                size_t c = at(g, i, j, k);
                int lim[3] = { i < nx - 1, j < ny - 1, k < nz - 1 };
                for (int a = 0; a < 3; a++) {
                    if (!lim[a]) continue;
                    cons_t f = pl ? plm_flux(g, pl, c, c + str[a], a) : hllc(load(g, c), load(g, c + str[a]), a, gam);
                    F[a][0][c] = f.d; F[a][1][c] = f.m[0]; F[a][2][c] = f.m[1];
                    F[a][3][c] = f.m[2]; F[a][4][c] = f.e;
                }
            }

    /* interior update + floors, hydro_solver_3d.c:729-771 */
    for (int i = 1; i < nx - 1; i++)
        for (int j = 1; j < ny - 1; j++)
            for (int k = 1; k < nz - 1; k++) {
                size_t c = at(g, i, j, k);
                double u[5];
                for (int v = 0; v < 5; v++) {
                    double du = -(dt / dx) * (F[0][v][c] - F[0][v][c - str[0]])
                                - (dt / dy) * (F[1][v][c] - F[1][v][c - str[1]])
                                - (dt / dz) * (F[2][v][c] - F[2][v][c - str[2]]);
                    u[v] = g->q[v][c] + du;
                }
                cons_t q = { u[0], { u[1], u[2], u[3] }, u[4] };
                q.d = mx(q.d, RHO_FLOOR);
                prim_t w = to_prim(q, gam);
                w.p = mx(w.p, P_FLOOR);
                store(g, c, to_cons(w, gam));
            }
    for (int a = 0; a < 3; a++)
        for (int v = 0; v < 5; v++) free(F[a][v]);
    free(pl);

    /* apply_gravity_source_terms, hydro_solver_3d.c:597-631 (all cells) */
    if (g->gravity) {
        for (size_t c = 0; c < n; c++) {
            double r = g->q[0][c];
            double u = g->q[1][c] / r, v = g->q[2][c] / r, w = g->q[3][c] / r;
            double ax = g->gx[c], ay = g->gy[c], az = g->gz[c];
            g->q[1][c] += dt * r * ax;
            g->q[2][c] += dt * r * ay;
            g->q[3][c] += dt * r * az;
            double work = r * (u * ax + v * ay + w * az);
            g->q[4][c] += dt * work;
        }
    }

    /* periodic copies, hydro_solver_3d.c:779-807 */
    if (g->bc[0] == BCP && g->bc[1] == BCP)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) store(g, at(g, 0, j, k), load(g, at(g, nx - 1, j, k)));
    if (g->bc[2] == BCP && g->bc[3] == BCP)
        for (int i = 0; i < nx; i++)
            for (int k = 0; k < nz; k++) store(g, at(g, i, 0, k), load(g, at(g, i, ny - 1, k)));
    if (g->bc[4] == BCP && g->bc[5] == BCP)
        for (int i = 0; i < nx; i++)
            for (int j = 0; j < ny; j++) store(g, at(g, i, j, 0), load(g, at(g, i, j, nz - 1)));

    hydro_bc(g);
    return st;
}
