/*
 * ics.c -- initial conditions of the drop-in solver (host code, run once).
 *
 * The reference's problem set-ups (hydro_solver_3d.c:813-2133) computed with
 * the same formulas, operand order and libm calls, so a deck produces the
 * same initial state; plus the analytic set-ups SOD_3D, POLYTROPE_3D and
 * COLD_COLLAPSE_3D and an optional log-normal density perturbation drawn
 * from the reference's generator.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "hydro_solver_3d.h"
#include "ics.h"

#define MAXD(a, b) (((a) > (b)) ? (a) : (b))

/* ---------------------------------------------------------------- EOS */
static Primitive3D c2p(State3D U, double gam)   /* hydro_solver_3d.c:162-175 */
{
    Primitive3D P;
    P.rho = MAXD(U.rho, RHO_FLOOR);
    P.u = U.rhou / P.rho;
    P.v = U.rhov / P.rho;
    P.w = U.rhow / P.rho;
    double ke = 0.5 * P.rho * (P.u * P.u + P.v * P.v + P.w * P.w);
    P.p = (gam - 1.0) * (U.E - ke);
    P.p = MAXD(P.p, P_FLOOR);
    return P;
}

static State3D p2c(Primitive3D P, double gam)   /* hydro_solver_3d.c:177-189 */
{
    State3D U;
    U.rho = P.rho;
    U.rhou = P.rho * P.u;
    U.rhov = P.rho * P.v;
    U.rhow = P.rho * P.w;
    double ke = 0.5 * P.rho * (P.u * P.u + P.v * P.v + P.w * P.w);
    U.E = P.p / (gam - 1.0) + ke;
    return U;
}

State3D hc_ic_prim_to_cons(Primitive3D P, double gamma) { return p2c(P, gamma); }
Primitive3D hc_ic_cons_to_prim(State3D U, double gamma) { return c2p(U, gamma); }

static double cx(const GodunovHLLC3D *s, int i) { return s->xmin + (i + 0.5) * s->dx; }
static double cy(const GodunovHLLC3D *s, int j) { return s->ymin + (j + 0.5) * s->dy; }
static double cz(const GodunovHLLC3D *s, int k) { return s->zmin + (k + 0.5) * s->dz; }
static size_t at(const GodunovHLLC3D *s, int i, int j, int k)
{
    return ((size_t)i * s->ny + j) * s->nz + k;
}

/* ---------------------------------------------------------------- RNG */
/* LCG + Box-Muller of hydro_solver_3d.c:1522-1539 (state kept per caller). */
static unsigned long g_rng = 1;
void hc_ic_seed(int seed) { g_rng = (unsigned long)seed; }
double hc_ic_uniform(void)
{
    g_rng = (g_rng * 1664525UL + 1013904223UL) & 0xFFFFFFFFUL;
    return (double)g_rng / 4294967296.0;
}
double hc_ic_normal(void)
{
    double u1 = hc_ic_uniform();
    double u2 = hc_ic_uniform();
    return sqrt(-2.0 * log(u1 + 1e-10)) * cos(2.0 * M_PI * u2);
}

/* ---------------------------------------------------------------- profiles */
typedef struct {
    int n;
    double *r, *rho, *u;
    double R_star;
} Profile;

static void profile_free(Profile *p)
{
    if (!p) return;
    free(p->r); free(p->rho); free(p->u);
    free(p);
}

/* read_stellar_profile, hydro_solver_3d.c:825-879: rows "r rho u", lines
 * starting with '#' or of 5 characters or fewer skipped. */
static Profile *profile_read(const char *fn)
{
    FILE *fp = fopen(fn, "r");
    if (!fp) {
        fprintf(stderr, "Error: Could not open stellar profile file '%s'\n", fn);
        return NULL;
    }
    char line[512];
    int n = 0;
    while (fgets(line, sizeof line, fp))
        if (line[0] != '#' && strlen(line) > 5) n++;
    rewind(fp);
    printf("Reading stellar profile from %s...\n", fn);
    printf("  Found %d data points\n", n);
    Profile *p = (Profile *)calloc(1, sizeof *p);
    p->n = n;
    p->r = (double *)calloc(n > 0 ? n : 1, sizeof(double));
    p->rho = (double *)calloc(n > 0 ? n : 1, sizeof(double));
    p->u = (double *)calloc(n > 0 ? n : 1, sizeof(double));
    int i = 0;
    while (fgets(line, sizeof line, fp) && i < n)
        if (line[0] != '#' && strlen(line) > 5) {
            sscanf(line, "%lf %lf %lf", &p->r[i], &p->rho[i], &p->u[i]);
            i++;
        }
    fclose(fp);
    if (n == 0) {
        profile_free(p);
        fprintf(stderr, "Error: stellar profile '%s' has no data rows\n", fn);
        return NULL;
    }
    double thr = 1e-4 * p->rho[0];
    p->R_star = p->r[n - 1];
    for (int j = 0; j < n; j++)
        if (p->rho[j] < thr) { p->R_star = p->r[j]; break; }
    printf("  Stellar radius: R = %.4f\n", p->R_star);
    printf("  Central density: rho_c = %.4e\n", p->rho[0]);
    printf("  Central internal energy: u_c = %.4e\n", p->u[0]);
    return p;
}

/* interpolate_profile, hydro_solver_3d.c:889-925.  The bracketing interval
 * is found by bisection instead of a linear scan; for a table with
 * increasing radii it is the same interval, so the result is identical. */
static void profile_at(const Profile *p, double r, double *rho, double *u)
{
    if (r <= p->r[0]) { *rho = p->rho[0]; *u = p->u[0]; return; }
    if (r >= p->r[p->n - 1]) { *rho = 1e-6; *u = 1e-6; return; }
    int lo = 0, hi = p->n - 1;           /* r[lo] <= r < r[hi] */
    while (hi - lo > 1) {
        int mid = (lo + hi) / 2;
        if (r >= p->r[mid]) lo = mid; else hi = mid;
    }
    double f = (r - p->r[lo]) / (p->r[lo + 1] - p->r[lo]);
    *rho = p->rho[lo] + f * (p->rho[lo + 1] - p->rho[lo]);
    *u = p->u[lo] + f * (p->u[lo + 1] - p->u[lo]);
}

static double profile_mass(const Profile *p)   /* hydro_solver_3d.c:1041-1052 */
{
    double M = 0.0;
    for (int i = 0; i < p->n - 1; i++) {
        double r1 = p->r[i], r2 = p->r[i + 1];
        double dr = r2 - r1;
        double rm = 0.5 * (r1 + r2);
        double rhom = 0.5 * (p->rho[i] + p->rho[i + 1]);
        M += 4.0 * M_PI * rhom * rm * rm * dr;
    }
    return M;
}

/* ---------------------------------------------------------------- set-ups */
static void ic_uniform_fallback(GodunovHLLC3D *s)
{
    for (int i = 0; i < s->nx; i++)
        for (int j = 0; j < s->ny; j++)
            for (int k = 0; k < s->nz; k++) {
                Primitive3D P = { 1.0, 0.0, 0.0, 0.0, 1.0 };
                s->U[at(s, i, j, k)] = p2c(P, s->gamma);
            }
}

static void ic_stellar_profile(GodunovHLLC3D *s, const char *fn)   /* :927-1002 */
{
    Profile *p = profile_read(fn);
    if (!p) {
        fprintf(stderr, "Failed to read profile. Using uniform density instead.\n");
        ic_uniform_fallback(s);
        return;
    }
    double x0 = 0.5 * (s->xmin + s->xmax), y0 = 0.5 * (s->ymin + s->ymax), z0 = 0.5 * (s->zmin + s->zmax);
    {
        const double c[3] = { x0, y0, z0 };
        const double *r = p->r, *rho = p->rho, *u = p->u;
        if (hc_ic_stars_device(s, 1, &p->n, &r, &rho, &u, NULL, c, NULL) == 0) {
            profile_free(p);
            return;
        }
    }
    for (int i = 0; i < s->nx; i++)
        for (int j = 0; j < s->ny; j++)
            for (int k = 0; k < s->nz; k++) {
                double r = sqrt(pow(cx(s, i) - x0, 2) + pow(cy(s, j) - y0, 2) + pow(cz(s, k) - z0, 2));
                double rho, u;
                profile_at(p, r, &rho, &u);
                Primitive3D P;
                P.rho = rho; P.u = 0.0; P.v = 0.0; P.w = 0.0;
                P.p = (s->gamma - 1.0) * rho * u;
                P.rho = MAXD(P.rho, RHO_FLOOR);
                P.p = MAXD(P.p, P_FLOOR);
                s->U[at(s, i, j, k)] = p2c(P, s->gamma);
            }
    profile_free(p);
}

/* Two stars on the grid (hydro_solver_3d.c:1133-1205 and :1298-1370). */
static void place_two_stars(GodunovHLLC3D *s, const Profile *p1, const Profile *p2,
                            const double c1[3], const double c2[3],
                            const double v1[3], const double v2[3])
{
    const double gm1 = s->gamma - 1.0;
    {
        const int n[2] = { p1->n, p2->n };
        const double *r[2] = { p1->r, p2->r }, *rho[2] = { p1->rho, p2->rho }, *u[2] = { p1->u, p2->u };
        const double R[2] = { p1->R_star, p2->R_star };
        const double c[6] = { c1[0], c1[1], c1[2], c2[0], c2[1], c2[2] };
        const double v[6] = { v1[0], v1[1], v1[2], v2[0], v2[1], v2[2] };
        if (hc_ic_stars_device(s, 2, n, r, rho, u, R, c, v) == 0) return;
    }
    for (int i = 0; i < s->nx; i++)
        for (int j = 0; j < s->ny; j++)
            for (int k = 0; k < s->nz; k++) {
                double x = cx(s, i), y = cy(s, j), z = cz(s, k);
                double r1 = sqrt(pow(x - c1[0], 2) + pow(y - c1[1], 2) + pow(z - c1[2], 2));
                double r2 = sqrt(pow(x - c2[0], 2) + pow(y - c2[1], 2) + pow(z - c2[2], 2));
                double rho1, u1, rho2, u2;
                profile_at(p1, r1, &rho1, &u1);
                profile_at(p2, r2, &rho2, &u2);
                int in1 = r1 < p1->R_star, in2 = r2 < p2->R_star;
                Primitive3D P;
                if (in1 && !in2) {
                    P.rho = rho1; P.u = v1[0]; P.v = v1[1]; P.w = v1[2];
                    P.p = gm1 * rho1 * u1;
                } else if (in2 && !in1) {
                    P.rho = rho2; P.u = v2[0]; P.v = v2[1]; P.w = v2[2];
                    P.p = gm1 * rho2 * u2;
                } else if (in1 && in2) {
                    double rt = rho1 + rho2;
                    double w1 = rho1 / rt, w2 = rho2 / rt;
                    P.rho = rt;
                    P.u = w1 * v1[0] + w2 * v2[0];
                    P.v = w1 * v1[1] + w2 * v2[1];
                    P.w = w1 * v1[2] + w2 * v2[2];
                    double pp1 = gm1 * rho1 * u1, pp2 = gm1 * rho2 * u2;
                    P.p = pp1 + pp2;
                } else {
                    P.rho = RHO_FLOOR; P.u = 0.0; P.v = 0.0; P.w = 0.0; P.p = P_FLOOR;
                }
                P.rho = MAXD(P.rho, RHO_FLOOR);
                P.p = MAXD(P.p, P_FLOOR);
                s->U[at(s, i, j, k)] = p2c(P, s->gamma);
            }
}

static void ic_binary_dual(GodunovHLLC3D *s, const InputDeck *d)   /* :1008-1212 */
{
    Profile *p1 = profile_read(d->star1_profile);
    Profile *p2 = profile_read(d->star2_profile);
    if (!p1 || !p2) {
        fprintf(stderr, "Failed to read one or both profiles. Cannot create binary system.\n");
        profile_free(p1);
        profile_free(p2);
        return;
    }
    double M1 = profile_mass(p1), M2 = profile_mass(p2);
    double c1[3] = { d->star1_x, d->star1_y, d->star1_z }, c2[3] = { d->star2_x, d->star2_y, d->star2_z };
    double v1[3] = { d->star1_vx, d->star1_vy, d->star1_vz }, v2[3] = { d->star2_vx, d->star2_vy, d->star2_vz };
    if (d->binary_auto_orbit) {
        double sep = d->binary_separation;
        double Mt = M1 + M2;
        double r1c = sep * M2 / Mt, r2c = sep * M1 / Mt;
        c1[0] = -r1c; c1[1] = 0.0; c1[2] = 0.0;
        c2[0] = r2c; c2[1] = 0.0; c2[2] = 0.0;
        double vo = sqrt(s->G_const * Mt / sep);
        double a1 = vo * M2 / Mt, a2 = vo * M1 / Mt;
        v1[0] = 0.0; v1[1] = +a1; v1[2] = 0.0;
        v2[0] = 0.0; v2[1] = -a2; v2[2] = 0.0;
        printf("  Orbital velocity: v_orb = %.4e\n", vo);
    }
    place_two_stars(s, p1, p2, c1, c2, v1, v2);
    profile_free(p1);
    profile_free(p2);
}

static void ic_binary_legacy(GodunovHLLC3D *s, const char *fn)   /* :1218-1378 */
{
    Profile *p = profile_read(fn);
    if (!p) {
        fprintf(stderr, "Failed to read profile. Cannot create binary system.\n");
        return;
    }
    double M = profile_mass(p);
    double sep = 3.0 * p->R_star;
    double Mt = 2.0 * M;
    double vo = sqrt(s->G_const * Mt / sep);
    double a1 = vo * 0.5, a2 = vo * 0.5;
    double c1[3] = { -sep / 2.0, 0.0, 0.0 }, c2[3] = { sep / 2.0, 0.0, 0.0 };
    double v1[3] = { 0.0, +a1, 0.0 }, v2[3] = { 0.0, -a2, 0.0 };
    place_two_stars(s, p, p, c1, c2, v1, v2);
    profile_free(p);
}

static void ic_kh(GodunovHLLC3D *s)   /* :1384-1448 */
{
    const double rho1 = 2.0, rho2 = 1.0, v1 = -0.5, v2 = 0.5, p0 = 2.5, w0 = 0.1, A = 0.1;
    for (int i = 0; i < s->nx; i++)
        for (int j = 0; j < s->ny; j++)
            for (int k = 0; k < s->nz; k++) {
                double x = cx(s, i), y = cy(s, j), z = cz(s, k);
                Primitive3D P;
                double f = 0.5 * (1.0 + tanh((y - 0.0) / w0));
                P.rho = rho1 * f + rho2 * (1.0 - f);
                P.u = v1 * f + v2 * (1.0 - f);
                double env = exp(-y * y / (4.0 * w0 * w0));
                double kx = 2.0 * M_PI / 2.0, kz = 2.0 * M_PI / 2.0;
                P.v = A * sin(kx * x) * cos(kz * z) * env;
                P.w = 0.5 * A * cos(kx * x) * sin(kz * z) * env;
                P.p = p0;
                s->U[at(s, i, j, k)] = p2c(P, s->gamma);
            }
}

static void ic_blast(GodunovHLLC3D *s)   /* :1449-1495 */
{
    const double rho_a = 1.0, p_a = 1.0e-5, E = 1.0, rb = 0.1;
    double x0 = 0.5 * (s->xmin + s->xmax), y0 = 0.5 * (s->ymin + s->ymax), z0 = 0.5 * (s->zmin + s->zmax);
    double V = (4.0 / 3.0) * M_PI * rb * rb * rb;
    double pb = (s->gamma - 1.0) * E / V;
    for (int i = 0; i < s->nx; i++)
        for (int j = 0; j < s->ny; j++)
            for (int k = 0; k < s->nz; k++) {
                double x = cx(s, i), y = cy(s, j), z = cz(s, k);
                double r = sqrt((x - x0) * (x - x0) + (y - y0) * (y - y0) + (z - z0) * (z - z0));
                Primitive3D P = { rho_a, 0.0, 0.0, 0.0, r < rb ? pb : p_a };
                s->U[at(s, i, j, k)] = p2c(P, s->gamma);
            }
}

/* ---- additions ---- */
static void ic_sod(GodunovHLLC3D *s)
{
    for (int i = 0; i < s->nx; i++)
        for (int j = 0; j < s->ny; j++)
            for (int k = 0; k < s->nz; k++) {
                int left = cx(s, i) < 0.5 * (s->xmin + s->xmax);
                Primitive3D P = { left ? 1.0 : 0.125, 0.0, 0.0, 0.0, left ? 1.0 : 0.1 };
                s->U[at(s, i, j, k)] = p2c(P, s->gamma);
            }
}

/* n=1 polytrope M=1, R=0.35 (G from the solver), p = K rho^2 */
static void ic_polytrope(GodunovHLLC3D *s)
{
    const double M = 1.0, R = 0.35;
    double G = s->G_const > 0.0 ? s->G_const : 1.0;
    double x0 = 0.5 * (s->xmin + s->xmax), y0 = 0.5 * (s->ymin + s->ymax), z0 = 0.5 * (s->zmin + s->zmax);
    double rc = M_PI * M / (4.0 * R * R * R);
    double K = 2.0 * G * R * R / M_PI;
    for (int i = 0; i < s->nx; i++)
        for (int j = 0; j < s->ny; j++)
            for (int k = 0; k < s->nz; k++) {
                double dx = cx(s, i) - x0, dy = cy(s, j) - y0, dz = cz(s, k) - z0;
                double r = sqrt(dx * dx + dy * dy + dz * dz);
                double xi = M_PI * r / R;
                double prof = xi > 0.0 ? sin(xi) / xi : 1.0;
                double rho = r < R ? rc * prof : 0.0;
                rho = MAXD(rho, 1e-6 * rc);
                Primitive3D P = { rho, 0.0, 0.0, 0.0, K * rho * rho };
                s->U[at(s, i, j, k)] = p2c(P, s->gamma);
            }
}

/* rho ~ 1/r inside R=1 (softened at 2 cells), mass 1, e = 0.05 GM/R */
static void ic_cold_collapse(GodunovHLLC3D *s)
{
    const double M = 1.0, R = 1.0;
    double G = s->G_const > 0.0 ? s->G_const : 1.0;
    double soft = 2.0 * s->dx;
    double dV = s->dx * s->dy * s->dz;
    double msum = 0.0;
    for (int pass = 0; pass < 2; pass++)
        for (int i = 0; i < s->nx; i++)
            for (int j = 0; j < s->ny; j++)
                for (int k = 0; k < s->nz; k++) {
                    double x = cx(s, i), y = cy(s, j), z = cz(s, k);
                    double r = sqrt(x * x + y * y + z * z);
                    double rho = 1e-5;
                    if (r < R) {
                        rho = M / (2.0 * M_PI * R * R * MAXD(r, soft));
                        if (pass == 0) { msum += rho * dV; continue; }
                        rho *= M / msum;
                    } else if (pass == 0) continue;
                    double e = 0.05 * G * M / R;
                    Primitive3D P = { rho, 0.0, 0.0, 0.0, (s->gamma - 1.0) * rho * e };
                    s->U[at(s, i, j, k)] = p2c(P, s->gamma);
                }
}

/* ---- octant explosion, hydro_solver_3d.c:1864-2020 ---- */
static void ic_octant(GodunovHLLC3D *s, const char *fn, double E, double rexp, const char *type)
{
    Profile *p = profile_read(fn);
    if (!p) return;
    const double dV = s->dx * s->dy * s->dz;
    int count = 0;
    for (int i = 0; i < s->nx; i++)
        for (int j = 0; j < s->ny; j++)
            for (int k = 0; k < s->nz; k++) {
                double x = cx(s, i), y = cy(s, j), z = cz(s, k);
                if (x < 0.0 || y < 0.0 || z < 0.0) continue;
                if (sqrt(x * x + y * y + z * z) < rexp) count++;
            }
    int thermal = strcmp(type, "thermal") == 0;
    double e_cell = 0.0, vmag = 0.0;
    if (thermal) {
        e_cell = E / (double)count;
    } else {
        double mass = 0.0;
        for (int i = 0; i < s->nx; i++)
            for (int j = 0; j < s->ny; j++)
                for (int k = 0; k < s->nz; k++) {
                    double x = cx(s, i), y = cy(s, j), z = cz(s, k);
                    if (x < 0.0 || y < 0.0 || z < 0.0) continue;
                    double r = sqrt(x * x + y * y + z * z);
                    if (r < rexp) {
                        double rho, u;
                        profile_at(p, r, &rho, &u);
                        mass += rho * s->dx * s->dy * s->dz;
                    }
                }
        vmag = sqrt(2.0 * E / mass);
    }
    (void)dV;
    for (int i = 0; i < s->nx; i++)
        for (int j = 0; j < s->ny; j++)
            for (int k = 0; k < s->nz; k++) {
                double x = cx(s, i), y = cy(s, j), z = cz(s, k);
                Primitive3D P;
                if (x >= 0.0 && y >= 0.0 && z >= 0.0) {
                    double r = sqrt(x * x + y * y + z * z);
                    double rho, u;
                    profile_at(p, r, &rho, &u);
                    P.rho = rho; P.u = 0.0; P.v = 0.0; P.w = 0.0;
                    P.p = rho * u * (s->gamma - 1.0);
                    if (r < rexp) {
                        if (thermal) {
                            double ui = u;
                            ui += e_cell / (rho * s->dx * s->dy * s->dz);
                            P.p = rho * ui * (s->gamma - 1.0);
                        } else if (r > 1e-10) {
                            P.u = vmag * (x / r);
                            P.v = vmag * (y / r);
                            P.w = vmag * (z / r);
                        }
                    }
                } else {
                    P.rho = RHO_FLOOR; P.u = 0.0; P.v = 0.0; P.w = 0.0; P.p = P_FLOOR;
                }
                s->U[at(s, i, j, k)] = p2c(P, s->gamma);
            }
    profile_free(p);
}

/* legendre_Plm, hydro_solver_3d.c:1543-1573 (Condon-Shortley phase) */
static double plm(int l, int m, double x)
{
    if (m < 0 || m > l) return 0.0;
    if (x > 1.0) x = 1.0;
    if (x < -1.0) x = -1.0;
    double pmm = 1.0;
    if (m > 0) {
        double somx2 = sqrt((1.0 - x) * (1.0 + x));
        double fact = 1.0;
        for (int i = 1; i <= m; i++) {
            pmm *= -fact * somx2;
            fact += 2.0;
        }
    }
    if (l == m) return pmm;
    double pmmp1 = x * (2 * m + 1) * pmm;
    if (l == m + 1) return pmmp1;
    double pll = 0.0;
    for (int ll = m + 2; ll <= l; ll++) {
        pll = ((2 * ll - 1) * x * pmmp1 - (ll + m - 1) * pmm) / (ll - m);
        pmm = pmmp1;
        pmmp1 = pll;
    }
    return pll;
}

static double ylm_real(int l, int m, double th, double ph)   /* :1576-1590 */
{
    double Pl = plm(l, abs(m), cos(th));
    double nrm = sqrt((2.0 * l + 1.0) / (4.0 * M_PI));
    if (m > 0) return nrm * Pl * cos(m * ph);
    if (m < 0) return nrm * Pl * sin(abs(m) * ph);
    return nrm * Pl;
}

typedef struct { double kx, ky, kz, a0, a1, a2, ph; } Mode;

static void draw_modes(Mode *md, int n, double kmin, double kmax, int vec)
{
    for (int q = 0; q < n; q++) {
        double km = kmin + (kmax - kmin) * hc_ic_uniform();
        double phi = 2.0 * M_PI * hc_ic_uniform();
        double ct = 2.0 * hc_ic_uniform() - 1.0;
        double st = sqrt(1.0 - ct * ct);
        md[q].kx = km * st * cos(phi);
        md[q].ky = km * st * sin(phi);
        md[q].kz = km * ct;
        md[q].a0 = hc_ic_normal();
        if (vec) {
            md[q].a1 = hc_ic_normal();
            md[q].a2 = hc_ic_normal();
        }
        md[q].ph = 2.0 * M_PI * hc_ic_uniform();
    }
}

/* apply_{velocity,density}_perturbations, :1596-1754, and the spherical
 * harmonic mode, :1756-1815, on the octant x, y, z >= 0. */
static void perturb_octant(GodunovHLLC3D *s, const InputDeck *d)
{
    hc_ic_seed(d->perturbation_seed);
    const double gam = s->gamma;
    if (d->perturb_velocity_amplitude > 0.0 && d->perturb_velocity_modes > 0) {
        int n = d->perturb_velocity_modes;
        Mode *md = (Mode *)malloc(sizeof(Mode) * n);
        draw_modes(md, n, d->perturb_velocity_kmin, d->perturb_velocity_kmax, 1);
        for (int i = 0; i < s->nx; i++)
            for (int j = 0; j < s->ny; j++)
                for (int k = 0; k < s->nz; k++) {
                    double x = cx(s, i), y = cy(s, j), z = cz(s, k);
                    if (x < 0.0 || y < 0.0 || z < 0.0) continue;
                    size_t c = at(s, i, j, k);
                    Primitive3D P = c2p(s->U[c], gam);
                    double cs = sqrt(gam * P.p / P.rho);
                    double du = 0.0, dv = 0.0, dw = 0.0;
                    for (int q = 0; q < n; q++) {
                        double wv = cos(md[q].kx * x + md[q].ky * y + md[q].kz * z + md[q].ph);
                        du += md[q].a0 * wv;
                        dv += md[q].a1 * wv;
                        dw += md[q].a2 * wv;
                    }
                    double nrm = sqrt((double)n);
                    P.u += (du / nrm) * d->perturb_velocity_amplitude * cs;
                    P.v += (dv / nrm) * d->perturb_velocity_amplitude * cs;
                    P.w += (dw / nrm) * d->perturb_velocity_amplitude * cs;
                    s->U[c] = p2c(P, gam);
                }
        free(md);
    }
    if (d->perturb_density_amplitude > 0.0 && d->perturb_density_modes > 0) {
        int n = d->perturb_density_modes;
        Mode *md = (Mode *)malloc(sizeof(Mode) * n);
        draw_modes(md, n, d->perturb_density_kmin, d->perturb_density_kmax, 0);
        for (int i = 0; i < s->nx; i++)
            for (int j = 0; j < s->ny; j++)
                for (int k = 0; k < s->nz; k++) {
                    double x = cx(s, i), y = cy(s, j), z = cz(s, k);
                    if (x < 0.0 || y < 0.0 || z < 0.0) continue;
                    size_t c = at(s, i, j, k);
                    Primitive3D P = c2p(s->U[c], gam);
                    double dr = 0.0;
                    for (int q = 0; q < n; q++)
                        dr += md[q].a0 * cos(md[q].kx * x + md[q].ky * y + md[q].kz * z + md[q].ph);
                    double nrm = sqrt((double)n);
                    double f = 1.0 + (dr / nrm) * d->perturb_density_amplitude;
                    if (f < 0.1) f = 0.1;
                    P.rho *= f;
                    s->U[c] = p2c(P, gam);
                }
        free(md);
    }
    if (d->enable_sph_harmonic_mode) {
        for (int i = 0; i < s->nx; i++)
            for (int j = 0; j < s->ny; j++)
                for (int k = 0; k < s->nz; k++) {
                    double x = cx(s, i), y = cy(s, j), z = cz(s, k);
                    if (x < 0.0 || y < 0.0 || z < 0.0) continue;
                    double r = sqrt(x * x + y * y + z * z);
                    if (r < 1e-10) continue;
                    double th = acos(z / r), ph = atan2(y, x);
                    double Y = ylm_real(d->sph_harmonic_l, d->sph_harmonic_m, th, ph);
                    size_t c = at(s, i, j, k);
                    Primitive3D P = c2p(s->U[c], gam);
                    double cs = sqrt(gam * P.p / P.rho);
                    P.rho *= (1.0 + d->sph_harmonic_amp_rho * Y);
                    double vr = d->sph_harmonic_amp_vel * cs * Y;
                    P.u += vr * (x / r);
                    P.v += vr * (y / r);
                    P.w += vr * (z / r);
                    s->U[c] = p2c(P, gam);
                }
    }
}

static void add_torus(GodunovHLLC3D *s, const InputDeck *d)   /* :2026-2086 */
{
    double R = d->torus_major_radius, rr = d->torus_minor_radius;
    for (int i = 0; i < s->nx; i++)
        for (int j = 0; j < s->ny; j++)
            for (int k = 0; k < s->nz; k++) {
                double x = cx(s, i), y = cy(s, j), z = cz(s, k);
                if (x < 0.0 || y < 0.0 || z < 0.0) continue;
                double rc = sqrt(x * x + y * y);
                double td = sqrt((rc - R) * (rc - R) + z * z);
                if (td <= rr) {
                    Primitive3D P;
                    P.rho = d->torus_density;
                    P.p = d->torus_pressure;
                    if (rc > 1e-10) {
                        P.u = -d->torus_rotation_velocity * y / rc;
                        P.v = d->torus_rotation_velocity * x / rc;
                        P.w = 0.0;
                    } else {
                        P.u = 0.0; P.v = 0.0; P.w = 0.0;
                    }
                    s->U[at(s, i, j, k)] = p2c(P, s->gamma);
                }
            }
}

/* Multiplies rho (and the momenta and energy with it, at fixed velocity and
 * pressure) by exp(sigma N(0,1)) per cell, N from the reference generator
 * seeded with `seed`, cells in IDX3D order. */
void hc_ic_log_normal(GodunovHLLC3D *s, double sigma, int seed)
{
    if (!(sigma > 0.0)) return;
    hc_ic_seed(seed);
    size_t n = (size_t)s->nx * s->ny * s->nz;
    for (size_t c = 0; c < n; c++) {
        Primitive3D P = c2p(s->U[c], s->gamma);
        double f = exp(sigma * hc_ic_normal());
        P.rho *= f;
        s->U[c] = p2c(P, s->gamma);
    }
}

/* set_initial_conditions_3d, hydro_solver_3d.c:1383-1515 (problems without
 * a set-up leave the state untouched). */
void hc_ic_problem(GodunovHLLC3D *s, ProblemType problem)
{
    switch (problem) {
    case KELVIN_HELMHOLTZ_3D: ic_kh(s); break;
    case BLAST_WAVE_3D: ic_blast(s); break;
    case STELLAR_PROFILE_3D: ic_stellar_profile(s, "stellar_profile.txt"); break;
    case BINARY_STAR_3D: ic_binary_legacy(s, "stellar_profile.txt"); break;
    case SOD_3D: ic_sod(s); break;
    case POLYTROPE_3D: ic_polytrope(s); break;
    case COLD_COLLAPSE_3D: ic_cold_collapse(s); break;
    default: break;
    }
}

/* set_initial_conditions_3d_from_deck, hydro_solver_3d.c:2092-2133 */
void hc_ic_from_deck(GodunovHLLC3D *s, const InputDeck *d)
{
    const int want = s->device_ics;
    if (d->log_noise > 0.0) s->device_ics = 0;   /* the noise is applied to the host array */
    if (d->problem == STELLAR_OCTANT_EXPLOSION_3D) {
        ic_octant(s, d->stellar_profile, d->explosion_energy, d->explosion_radius, d->explosion_type);
        if (d->enable_perturbations) perturb_octant(s, d);
        if (d->enable_torus) add_torus(s, d);
    } else if (d->problem == BINARY_STAR_3D) {
        ic_binary_dual(s, d);
    } else {
        hc_ic_problem(s, d->problem);
    }
    if (d->log_noise > 0.0) hc_ic_log_normal(s, d->log_noise, d->perturbation_seed);
    s->device_ics = want;
}
