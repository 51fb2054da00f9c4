// ics_device.cu -- profile-based initial conditions built on the device.
//
// The stellar-profile and binary-star set-ups (hydro_solver_3d.c:927-1002
// and :1133-1205 / :1298-1370) interpolate a radial profile table (r, rho, u)
// at every cell.  The host code (host/ics.c) does that for the reference's
// drop-in API; for large grids the same values are formed here, one thread
// per cell, and written straight into the device state -- no host loop over
// the cells and no upload of the host array.  Operations and their order are
// those of host/ics.c (profile_at's bisection, p2c, the floors; the
// reference's pow(d, 2) is d*d, which is what GCC emits for it), compiled
// without FMA contraction, so the state equals the host-built one bit for bit.
#include <algorithm>
#include <cstring>

#include "../../include/hydrocode_b200.h"
#include "hc_internal.cuh"
#include "hc_math.cuh"

namespace hc {
namespace {

struct ProfDev {
    const double *r, *rho, *u;
    int n;
    double R;   // radius that decides "inside the star" (two-star rule)
};

// profile_at (host/ics.c): the bracketing interval by bisection
__device__ __forceinline__ void prof_at(const ProfDev &p, double r, double &rho, double &u)
{
    if (r <= p.r[0]) {
        rho = p.rho[0];
        u = p.u[0];
        return;
    }
    if (r >= p.r[p.n - 1]) {
        rho = 1e-6;
        u = 1e-6;
        return;
    }
    int lo = 0, hi = p.n - 1;
    while (hi - lo > 1) {
        const int mid = (lo + hi) / 2;
        if (r >= p.r[mid]) lo = mid;
        else hi = mid;
    }
    const double f = (r - p.r[lo]) / (p.r[lo + 1] - p.r[lo]);
    rho = p.rho[lo] + f * (p.rho[lo + 1] - p.rho[lo]);
    u = p.u[lo] + f * (p.u[lo + 1] - p.u[lo]);
}

struct StarArgs {
    Geom g;
    double gamma;
    int nstars;
    ProfDev p[2];
    double c[2][3], v[2][3];
    double *q64[5];
    float *q32[5];
};

__global__ void __launch_bounds__(256) stars_kernel(StarArgs a)
{
    const Geom g = a.g;
    const long long sI = (long long)g.ny * g.nz, sJ = g.nz;
    const double gm1 = a.gamma - 1.0;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.n;
         c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c / sI), j = (int)((c / sJ) % g.ny), k = (int)(c % sJ);
        const double x = g.xmin + (i + 0.5) * g.dx, y = g.ymin + (j + 0.5) * g.dy, z = g.zmin + (k + 0.5) * g.dz;
        double prho, pu, pv, pw, pp;
        if (a.nstars == 1) {   // ic_stellar_profile: every cell from the profile, at rest
            const double dx = x - a.c[0][0], dy = y - a.c[0][1], dz = z - a.c[0][2];
            const double r = sqrt(dx * dx + dy * dy + dz * dz);
            double rho, u;
            prof_at(a.p[0], r, rho, u);
            prho = rho;
            pu = 0.0;
            pv = 0.0;
            pw = 0.0;
            pp = (a.gamma - 1.0) * rho * u;
        } else {               // place_two_stars
            const double ax = x - a.c[0][0], ay = y - a.c[0][1], az = z - a.c[0][2];
            const double bx = x - a.c[1][0], by = y - a.c[1][1], bz = z - a.c[1][2];
            const double r1 = sqrt(ax * ax + ay * ay + az * az);
            const double r2 = sqrt(bx * bx + by * by + bz * bz);
            double rho1, u1, rho2, u2;
            prof_at(a.p[0], r1, rho1, u1);
            prof_at(a.p[1], r2, rho2, u2);
            const bool in1 = r1 < a.p[0].R, in2 = r2 < a.p[1].R;
            if (in1 && !in2) {
                prho = rho1;
                pu = a.v[0][0];
                pv = a.v[0][1];
                pw = a.v[0][2];
                pp = gm1 * rho1 * u1;
            } else if (in2 && !in1) {
                prho = rho2;
                pu = a.v[1][0];
                pv = a.v[1][1];
                pw = a.v[1][2];
                pp = gm1 * rho2 * u2;
            } else if (in1 && in2) {
                const double rt = rho1 + rho2;
                const double w1 = rho1 / rt, w2 = rho2 / rt;
                prho = rt;
                pu = w1 * a.v[0][0] + w2 * a.v[1][0];
                pv = w1 * a.v[0][1] + w2 * a.v[1][1];
                pw = w1 * a.v[0][2] + w2 * a.v[1][2];
                const double pp1 = gm1 * rho1 * u1, pp2 = gm1 * rho2 * u2;
                pp = pp1 + pp2;
            } else {
                prho = HC_RHO_FLOOR;
                pu = 0.0;
                pv = 0.0;
                pw = 0.0;
                pp = HC_P_FLOOR;
            }
        }
        prho = prho > HC_RHO_FLOOR ? prho : HC_RHO_FLOOR;   // MAXD of the host code
        pp = pp > HC_P_FLOOR ? pp : HC_P_FLOOR;
        // p2c (prim_to_cons_3d)
        const double U0 = prho, U1 = prho * pu, U2 = prho * pv, U3 = prho * pw;
        const double ke = 0.5 * prho * (pu * pu + pv * pv + pw * pw);
        const double U4 = pp / (a.gamma - 1.0) + ke;
        if (a.q64[0]) {
            a.q64[0][c] = U0; a.q64[1][c] = U1; a.q64[2][c] = U2; a.q64[3][c] = U3; a.q64[4][c] = U4;
        } else {
            a.q32[0][c] = (float)U0; a.q32[1][c] = (float)U1; a.q32[2][c] = (float)U2;
            a.q32[3][c] = (float)U3; a.q32[4][c] = (float)U4;
        }
    }
}

}  // namespace

// the profile tables are copied to `scratch` (3 sum(n) doubles, device)
cudaError_t ic_profile_stars(const Geom &g, double gamma, int nstars, const int *n, const double *const *r,
                             const double *const *rho, const double *const *u, const double *R_star,
                             const double *centre, const double *vel, double *const q64[5], float *const q32[5],
                             double *scratch, cudaStream_t s)
{
    StarArgs a;
    memset(&a, 0, sizeof a);
    a.g = g;
    a.gamma = gamma;
    a.nstars = nstars;
    size_t off = 0;
    for (int t = 0; t < nstars; t++) {
        const size_t bytes = (size_t)n[t] * sizeof(double);
        cudaError_t e = cudaMemcpyAsync(scratch + off, r[t], bytes, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(scratch + off + n[t], rho[t], bytes, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(scratch + off + 2 * n[t], u[t], bytes, cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) return e;
        a.p[t].r = scratch + off;
        a.p[t].rho = scratch + off + n[t];
        a.p[t].u = scratch + off + 2 * n[t];
        a.p[t].n = n[t];
        a.p[t].R = R_star ? R_star[t] : 0.0;
        for (int d = 0; d < 3; d++) {
            a.c[t][d] = centre[3 * t + d];
            a.v[t][d] = vel ? vel[3 * t + d] : 0.0;
        }
        off += 3 * (size_t)n[t];
    }
    for (int v = 0; v < 5; v++) {
        a.q64[v] = q64 ? q64[v] : nullptr;
        a.q32[v] = q32 ? q32[v] : nullptr;
    }
    const int blocks = (int)std::min<long long>((g.n + 255) / 256, 148LL * 16);
    stars_kernel<<<blocks, 256, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace hc
