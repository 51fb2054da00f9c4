// hydro_plm.cu -- opt-in MUSCL-Hancock reconstruction for the FP64 step
// (hc_config.recon = 1).  No reference counterpart: the reference forms its
// HLLC fluxes from piecewise-constant states (hydro_solver_3d.c:654-724);
// the default path keeps that, bit for bit.
//
// Per cell, on primitives W = (rho, u, v, w, p):
//   slopes    dW_a = minmod(W - W[-e_a], W[+e_a] - W), zero where the cell
//             lies on the domain boundary along axis a;
//   half step (primitive Euler equations, normal velocity un = W.v[a])
//             t_a = (un drho + rho du_a,  un du_c for c != a,
//                    un du_a + dp/rho,  un dp + gamma p du_a),
//             W* = W - h_x t_x - h_y t_y - h_z t_z,  h_a = dt / (2 d_a);
//   faces     W* + dW_a/2 on the +a face, W* - dW_a/2 on the -a face;
//   fallback  first order for the cell (W* = W, dW = 0) when W* or one of
//             its six face states has rho <= 0 or p <= 0.
// The flux through a face is HLLC on its two face states, each turned into a
// conserved state (and back to primitives with the usual floors, as the HLLC
// of the first-order path receives them).  The update, floors, gravity source
// and next-step CFL maximum of an interior cell are those of interior_kernel;
// the boundary cells, BCs and dt are the first-order path's kernels.
//
// Two kernels: plm_predict (every cell: W* and the three slopes into a
// 20-value-per-cell buffer) and plm_update (interior cells: six face fluxes,
// each face formed by both of its cells from the same values, so the update
// is conservative).  Compiled with -fmad=false and in the operand order of
// the CPU oracle (oracle/hc_oracle.c, plm_predict / plm_flux): the two agree
// bit for bit.
#include <algorithm>

#include "hc_internal.cuh"
#include "hc_math.cuh"
#include "hydro_kernels.cuh"

namespace hc {
namespace {

__device__ __forceinline__ double minmod(double a, double b)
{
    return (a * b <= 0.0) ? 0.0 : (fabs(a) < fabs(b) ? a : b);
}

__device__ __forceinline__ void prim_arr(const Prim<double> &w, double *o)
{
    o[0] = w.d;
    o[1] = w.v[0];
    o[2] = w.v[1];
    o[3] = w.v[2];
    o[4] = w.p;
}

__global__ void __launch_bounds__(256) plm_predict_kernel(HydroArgs a, double *__restrict__ pl)
{
    const Geom g = a.g;
    const long long n = g.n, sI = (long long)g.ny * g.nz, sJ = g.nz;
    const double *const *qin = reinterpret_cast<const double *const *>(a.qin);
    const double gam = a.gamma, gm1 = a.gamma - 1.0;
    const double dt = a.sc->dt;
    const double h[3] = { 0.5 * dt / g.dx, 0.5 * dt / g.dy, 0.5 * dt / g.dz };
    const long long str[3] = { sI, sJ, 1 };
    const int nn[3] = { g.nx, g.ny, g.nz };
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x) {
        const int idx[3] = { (int)(c / sI), (int)((c / sJ) % g.ny), (int)(c % sJ) };
        double w[5], dw[3][5], t[3][5], ws[5];
        prim_arr(to_prim(ld_cons(qin, c), gm1), w);
#pragma unroll
        for (int ax = 0; ax < 3; ax++) {
            if (idx[ax] >= 1 && idx[ax] <= nn[ax] - 2) {
                double wm[5], wp[5];
                prim_arr(to_prim(ld_cons(qin, c - str[ax]), gm1), wm);
                prim_arr(to_prim(ld_cons(qin, c + str[ax]), gm1), wp);
#pragma unroll
                for (int v = 0; v < 5; v++) dw[ax][v] = minmod(w[v] - wm[v], wp[v] - w[v]);
            } else {
#pragma unroll
                for (int v = 0; v < 5; v++) dw[ax][v] = 0.0;
            }
        }
#pragma unroll
        for (int ax = 0; ax < 3; ax++) {
            const double un = w[1 + ax];
            t[ax][0] = un * dw[ax][0] + w[0] * dw[ax][1 + ax];
#pragma unroll
            for (int cc = 0; cc < 3; cc++) t[ax][1 + cc] = un * dw[ax][1 + cc];
            t[ax][1 + ax] = un * dw[ax][1 + ax] + dw[ax][4] / w[0];
            t[ax][4] = un * dw[ax][4] + gam * w[4] * dw[ax][1 + ax];
        }
#pragma unroll
        for (int v = 0; v < 5; v++) ws[v] = w[v] - h[0] * t[0][v] - h[1] * t[1][v] - h[2] * t[2][v];
        bool ok = ws[0] > 0.0 && ws[4] > 0.0;
#pragma unroll
        for (int ax = 0; ax < 3; ax++) {
            ok = ok && (ws[0] + 0.5 * dw[ax][0]) > 0.0 && (ws[4] + 0.5 * dw[ax][4]) > 0.0;
            ok = ok && (ws[0] - 0.5 * dw[ax][0]) > 0.0 && (ws[4] - 0.5 * dw[ax][4]) > 0.0;
        }
        if (!ok) {
#pragma unroll
            for (int v = 0; v < 5; v++) {
                ws[v] = w[v];
#pragma unroll
                for (int ax = 0; ax < 3; ax++) dw[ax][v] = 0.0;
            }
        }
#pragma unroll
        for (int v = 0; v < 5; v++) {
            pl[v * n + c] = ws[v];
#pragma unroll
            for (int ax = 0; ax < 3; ax++) pl[(5 + 5 * ax + v) * n + c] = dw[ax][v];
        }
    }
}

// flux through the face between cells cl and cl + e_A from their face states
template <int A>
__device__ __forceinline__ Cons<double> plm_flux(const double *__restrict__ pl, long long n, long long cl,
                                                 long long cr, double gam, double gm1)
{
    Prim<double> L, R;
    L.d = pl[0 * n + cl] + 0.5 * pl[(5 + 5 * A + 0) * n + cl];
    L.v[0] = pl[1 * n + cl] + 0.5 * pl[(5 + 5 * A + 1) * n + cl];
    L.v[1] = pl[2 * n + cl] + 0.5 * pl[(5 + 5 * A + 2) * n + cl];
    L.v[2] = pl[3 * n + cl] + 0.5 * pl[(5 + 5 * A + 3) * n + cl];
    L.p = pl[4 * n + cl] + 0.5 * pl[(5 + 5 * A + 4) * n + cl];
    R.d = pl[0 * n + cr] - 0.5 * pl[(5 + 5 * A + 0) * n + cr];
    R.v[0] = pl[1 * n + cr] - 0.5 * pl[(5 + 5 * A + 1) * n + cr];
    R.v[1] = pl[2 * n + cr] - 0.5 * pl[(5 + 5 * A + 2) * n + cr];
    R.v[2] = pl[3 * n + cr] - 0.5 * pl[(5 + 5 * A + 3) * n + cr];
    R.p = pl[4 * n + cr] - 0.5 * pl[(5 + 5 * A + 4) * n + cr];
    const Cons<double> qL = to_cons(L, gm1), qR = to_cons(R, gm1);
    const Prim<double> wL = to_prim(qL, gm1), wR = to_prim(qR, gm1);
    return hllc<A>(qL, wL, csound(wL, gam), qR, wR, csound(wR, gam));
}

__global__ void __launch_bounds__(256) plm_update_kernel(HydroArgs a, const double *__restrict__ pl)
{
    const Geom g = a.g;
    const long long n = g.n, sI = (long long)g.ny * g.nz, sJ = g.nz;
    const int ni = g.nx - 2, nj = g.ny - 2, nk = g.nz - 2;
    const long long nint = (long long)ni * nj * nk;
    const double *const *qin = reinterpret_cast<const double *const *>(a.qin);
    double *const *qout = reinterpret_cast<double *const *>(a.qout);
    const double gam = a.gamma, gm1 = a.gamma - 1.0;
    const double dt = a.sc->dt;
    const double dtdx = dt / a.g.dx, dtdy = dt / a.g.dy, dtdz = dt / a.g.dz;
    const double idx2 = 2.0 * a.g.dx, idy2 = 2.0 * a.g.dy, idz2 = 2.0 * a.g.dz;
    double smax = 0.0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nint;
         t += (long long)gridDim.x * blockDim.x) {
        const int k = 1 + (int)(t % nk), j = 1 + (int)((t / nk) % nj), i = 1 + (int)(t / ((long long)nk * nj));
        const long long c = (long long)i * sI + (long long)j * sJ + k;
        const Cons<double> fxm = plm_flux<0>(pl, n, c - sI, c, gam, gm1);
        const Cons<double> fxp = plm_flux<0>(pl, n, c, c + sI, gam, gm1);
        const Cons<double> ym = plm_flux<1>(pl, n, c - sJ, c, gam, gm1);
        const Cons<double> yp = plm_flux<1>(pl, n, c, c + sJ, gam, gm1);
        const Cons<double> zm = plm_flux<2>(pl, n, c - 1, c, gam, gm1);
        const Cons<double> zp = plm_flux<2>(pl, n, c, c + 1, gam, gm1);
        // from here on as interior_kernel: update, floors, gravity source
        Cons<double> q = ld_cons(qin, c);
        q.d = q.d + (-dtdx * (fxp.d - fxm.d) - dtdy * (yp.d - ym.d) - dtdz * (zp.d - zm.d));
#pragma unroll
        for (int cc = 0; cc < 3; cc++)
            q.m[cc] = q.m[cc] + (-dtdx * (fxp.m[cc] - fxm.m[cc]) - dtdy * (yp.m[cc] - ym.m[cc]) -
                                 dtdz * (zp.m[cc] - zm.m[cc]));
        q.e = q.e + (-dtdx * (fxp.e - fxm.e) - dtdy * (yp.e - ym.e) - dtdz * (zp.e - zm.e));
        q.d = tmax(q.d, HC_RHO_FLOOR);
        Prim<double> w = to_prim(q, gm1);
        w.p = tmax(w.p, HC_P_FLOOR);
        q = to_cons(w, gm1);
        if (a.gravity) {
            const double *ph = a.phig;
            double ax = -(__ldg(ph + c + sI) - __ldg(ph + c - sI)) / idx2;
            double ay = -(__ldg(ph + c + sJ) - __ldg(ph + c - sJ)) / idy2;
            double az = -(__ldg(ph + c + 1) - __ldg(ph + c - 1)) / idz2;
            gravity_source(q, ax, ay, az, dt);
        }
        st_cons(qout, c, q);
        smax = tmax(smax, signal_speed(to_prim(q, gm1), gam));
    }
    block_max_to(smax, &a.sc->smax[a.step_parity ^ 1],
                 reinterpret_cast<unsigned int *>(&a.sc->smax[a.step_parity ^ 1]));
}

}  // namespace

cudaError_t fp64_plm_interior(const HydroArgs &a, double *pl, cudaStream_t s)
{
    if (a.g.nx < 3 || a.g.ny < 3 || a.g.nz < 3) return cudaErrorInvalidValue;
    const long long n = a.g.n, nint = (long long)(a.g.nx - 2) * (a.g.ny - 2) * (a.g.nz - 2);
    const int b1 = (int)std::min<long long>((n + 255) / 256, 148LL * 16);
    const int b2 = (int)std::min<long long>((nint + 255) / 256, 148LL * 16);
    plm_predict_kernel<<<b1, 256, 0, s>>>(a, pl);
    plm_update_kernel<<<b2, 256, 0, s>>>(a, pl);
    return cudaGetLastError();
}

}  // namespace hc
