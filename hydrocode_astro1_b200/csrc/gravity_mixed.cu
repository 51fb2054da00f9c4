// gravity_mixed.cu -- multipole boundary to degree lmax, and the
// mixed-precision Poisson solve (FP64 outer residual, FP32 SOR correction).
//
// Multipole (extension of gravity_solver_3d.c:164-345 beyond l = 2): with
// Q_l^m = r^l P_l^m(cos t) e^{i m p} (no Condon-Shortley phase),
//   Q_0^0 = 1, Q_m^m = (2m-1)(x+iy) Q_{m-1}^{m-1}, Q_{m+1}^m = (2m+1) z Q_m^m,
//   (l-m) Q_l^m = (2l-1) z Q_{l-1}^m - (l+m-1) r^2 Q_{l-2}^m,
// and N_lm = sqrt((2-d_m0)(l-m)!/(l+m)!), the exterior potential about the
// centre of mass is
//   phi(r) = -G sum_l sum_m N_lm (C_lm Re Q_l^m(r) + S_lm Im Q_l^m(r)) / r^(2l+1)
// with C_lm + i S_lm = sum_cells rho dV N_lm Q_l^m(r').  Coefficients are stored
// at l*l+l+m (C, m >= 0) and l*l+l-m (S, m > 0).  The sums are FP64 in a
// fixed order (rows, then blocks), so they are deterministic.
#include <algorithm>

#include "hc_internal.cuh"
#include "hc_math.cuh"
#include "sor_split.cuh"
#include "sor_split_tma.cuh"
#include "sor_wave_split.cuh"
#include "tmap.cuh"

#ifndef HC_MIXED_PAIR
#define HC_MIXED_PAIR 1   // pair forms of the FP64 residual / update where the layout allows
#endif

namespace hc {

int lmax_ncoef(int lmax) { return (lmax + 1) * (lmax + 1); }

namespace {

constexpr int LM_MAX = 12;
constexpr int LM_NC = (LM_MAX + 1) * (LM_MAX + 1);

__constant__ double c_norm[LM_NC];   // N_lm at l*(LM_MAX+1)+m

// Calls f(idx, value) for every coefficient of the solid harmonics at (x,y,z).
template <typename F>
__device__ __forceinline__ void solid_harmonics(double x, double y, double z, int lmax, F f)
{
    const double r2 = x * x + y * y + z * z;
    double smr = 1.0, smi = 0.0;     // Q_m^m
    for (int m = 0; m <= lmax; m++) {
        if (m > 0) {
            double a = (double)(2 * m - 1);
            double nr = a * (x * smr - y * smi);
            double ni = a * (x * smi + y * smr);
            smr = nr; smi = ni;
        }
        double pr = smr, pi = smi;          // Q_{l-1}^m
        double ppr = 0.0, ppi = 0.0;        // Q_{l-2}^m
        for (int l = m; l <= lmax; l++) {
            double cr, ci;
            if (l == m) { cr = smr; ci = smi; }
            else if (l == m + 1) { cr = (2 * m + 1) * z * smr; ci = (2 * m + 1) * z * smi; }
            else {
                double a = (double)(2 * l - 1), b = (double)(l + m - 1), inv = 1.0 / (double)(l - m);
                cr = (a * z * pr - b * r2 * ppr) * inv;
                ci = (a * z * pi - b * r2 * ppi) * inv;
            }
            if (l > m) { ppr = pr; ppi = pi; }
            pr = cr; pi = ci;
            if (l == m) { ppr = 0.0; ppi = 0.0; }
            double nrm = c_norm[l * (LM_MAX + 1) + m];
            f(l * l + l + m, nrm * cr);
            if (m > 0) f(l * l + l - m, nrm * ci);
        }
    }
}

// Row-factored moments.  For a fixed order m, Q_l^m = Q_m^m(x, y) p_l^m(z),
// where Q_m^m depends only on (x, y) -- constant along a row (i, j) -- and
// p_l^m is a real polynomial in z of degree l - m whose coefficients follow
// from the recursion with r^2 = rho2 + z^2, rho2 = x^2 + y^2:
//   p_m = 1,  p_{m+1} = (2m+1) z,
//   (l-m) p_l = (2l-1) z p_{l-1} - (l+m-1) (rho2 + z^2) p_{l-2}.
// Hence sum_k rho_k Q_l^m(x, y, z_k) = Q_m^m(x, y) sum_t c_lt Z_t, with the
// row's z-power sums Z_t = sum_k rho_k z_k^t (t <= lmax).  One pass over the
// density forms Z_t for every row (HBM-bound); a second, per (row, m), runs
// the coefficient recursion and accumulates the row's contribution.  The
// centre of mass comes first from the row sums of rho and rho z.
constexpr int LR_NT = 256;           // 8 warps; one row per warp at a time
constexpr int LR_ROWBLK = 128;       // rows per block of lmax_rows
constexpr int LR_UNROLL = 8;         // density loads in flight per lane

__device__ __forceinline__ double dens(const GravArgs &a, long long c)
{
    return a.rho ? a.rho[c] : (double)a.rho32[c];
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Centre of mass, COM_PP partials per own plane (one CTA each): (S0, x S0,
// y S0, S1) over its rows, S0 = sum_k rho, S1 = sum_k rho z (cells with
// rho > 0, as in every moment); warp w of part p takes rows
// p * 8 + w, + 8 COM_PP, ...
constexpr int COM_PP = 4;

__global__ void __launch_bounds__(LR_NT) lmax_com_partial(GravArgs a, double *parts)
{
    const Geom g = a.g;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = g.olo + (int)blockIdx.x / COM_PP, part = (int)blockIdx.x % COM_PP;
    double v0 = 0.0, vx = 0.0, vy = 0.0, vz = 0.0;
    for (int j = part * (LR_NT / 32) + warp; j < g.ny; j += COM_PP * (LR_NT / 32)) {
        const long long base = ((long long)i * g.ny + j) * g.nz;
        double s0 = 0.0, s1 = 0.0;
        for (int k0 = 0; k0 < g.nz; k0 += 32 * LR_UNROLL) {
            double rv[LR_UNROLL];
#pragma unroll
            for (int u = 0; u < LR_UNROLL; u++) {
                const int k = k0 + 32 * u + lane;
                rv[u] = k < g.nz ? dens(a, base + k) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < LR_UNROLL; u++) {
                if (rv[u] > 0.0) {
                    s0 += rv[u];
                    s1 += rv[u] * (g.zmin + (k0 + 32 * u + lane + 0.5) * g.dz);
                }
            }
        }
        s0 = warp_sum(s0);
        s1 = warp_sum(s1);
        v0 += s0;
        vx += (g.xmin + (i + g.ioff + 0.5) * g.dx) * s0;
        vy += (g.ymin + (j + 0.5) * g.dy) * s0;
        vz += s1;
    }
    __shared__ double red[LR_NT / 32][4];
    if (lane == 0) {
        red[warp][0] = v0;
        red[warp][1] = vx;
        red[warp][2] = vy;
        red[warp][3] = vz;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        double s = 0.0;
        for (int w = 0; w < LR_NT / 32; w++) s += red[w][threadIdx.x];
        parts[(long long)blockIdx.x * 4 + threadIdx.x] = s;
    }
}

// M = dV S0 and the centre of mass (box centre when there is no mass), as
// the reference's monopole pass stores them.  Warp q adds the partials of
// sum q (lane-strided, then a fixed butterfly).
__global__ void __launch_bounds__(128) lmax_com_final(GravArgs a, const double *parts, int nparts)
{
    __shared__ double v[4];
    const int q = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double s = 0.0;
    for (int b = lane; b < nparts; b += 32) s += parts[(long long)b * 4 + q];
    s = warp_sum(s);
    if (lane == 0) v[q] = s;
    __syncthreads();
    if (threadIdx.x != 0) return;
    const Geom g = a.g;
    a.sc->moments[0] = v[0] * (g.dx * g.dy * g.dz);
    if (v[0] > 0.0) {
        a.sc->moments[1] = v[1] / v[0];
        a.sc->moments[2] = v[2] / v[0];
        a.sc->moments[3] = v[3] / v[0];
    } else {
        a.sc->moments[1] = 0.5 * (g.xmin + g.xmax);
        a.sc->moments[2] = 0.5 * (g.ymin + g.ymax);
        a.sc->moments[3] = 0.5 * (g.zmin + g.zmax);
    }
}

// z-power sums about the centre of mass: zs[t * rows + row] = sum_k rho z^t
template <int LMAX>
__global__ void __launch_bounds__(LR_NT) lmax_zsums(GravArgs a, const double *com, double *zs)
{
    const Geom g = a.g;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long rows = (long long)g.nx * g.ny;
    const long long row1 = (long long)g.ohi * g.ny;
    const double z0 = g.zmin - com[2];
    for (long long row = (long long)g.olo * g.ny + (long long)blockIdx.x * (LR_NT / 32) + warp; row < row1;
         row += (long long)gridDim.x * (LR_NT / 32)) {
        const long long base = row * g.nz;
        double acc[LMAX + 1];
#pragma unroll
        for (int t = 0; t <= LMAX; t++) acc[t] = 0.0;
        for (int k0 = 0; k0 < g.nz; k0 += 32 * LR_UNROLL) {
            double rv[LR_UNROLL];
#pragma unroll
            for (int u = 0; u < LR_UNROLL; u++) {
                const int k = k0 + 32 * u + lane;
                rv[u] = k < g.nz ? dens(a, base + k) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < LR_UNROLL; u++) {
                if (rv[u] > 0.0) {
                    const double z = z0 + (k0 + 32 * u + lane + 0.5) * g.dz;
                    double w = rv[u];
                    acc[0] += w;
#pragma unroll
                    for (int t = 1; t <= LMAX; t++) {
                        w *= z;
                        acc[t] += w;
                    }
                }
            }
        }
#pragma unroll
        for (int t = 0; t <= LMAX; t++) acc[t] = warp_sum(acc[t]);
        if (lane == 0) {
#pragma unroll
            for (int t = 0; t <= LMAX; t++) zs[t * rows + row] = acc[t];
        }
    }
}

// Order m = blockIdx.y; block x covers rows q LR_ROWBLK .. of own plane
// olo + x / QR (q = x % QR, QR = ceil(ny / LR_ROWBLK)), one row per thread;
// the block's sums of dV N_lm Q_m^m sum_t c_lt Z_t go to its partial slots
// (l*l+l+m for the real part, l*l+l-m for the imaginary part), which
// lmax_final adds in block order.
template <int LMAX>
__global__ void __launch_bounds__(LR_ROWBLK) lmax_rows(GravArgs a, const double *com, const double *zs,
                                                       double *parts)
{
    const Geom g = a.g;
    const int m = blockIdx.y;
    const long long rows = (long long)g.nx * g.ny;
    const int QR = (g.ny + LR_ROWBLK - 1) / LR_ROWBLK;
    const int i = g.olo + (int)blockIdx.x / QR;
    const int j = ((int)blockIdx.x % QR) * LR_ROWBLK + threadIdx.x;
    const double xc = com[0], yc = com[1];
    double ar[LMAX + 1], ai[LMAX + 1];
#pragma unroll
    for (int d = 0; d <= LMAX; d++) ar[d] = ai[d] = 0.0;
    if (j < g.ny) {
        const long long row = (long long)i * g.ny + j;
        const double x = g.xmin + (i + g.ioff + 0.5) * g.dx - xc;
        const double y = g.ymin + (j + 0.5) * g.dy - yc;
        const double rho2 = x * x + y * y;
        double smr = 1.0, smi = 0.0;      // Q_m^m
        for (int q = 1; q <= m; q++) {
            const double f = (double)(2 * q - 1);
            const double nr = f * (x * smr - y * smi);
            const double ni = f * (x * smi + y * smr);
            smr = nr;
            smi = ni;
        }
        double Z[LMAX + 1];
#pragma unroll
        for (int t = 0; t <= LMAX; t++) Z[t] = (t <= LMAX - m) ? zs[t * rows + row] : 0.0;
        double c1[LMAX + 1], c2[LMAX + 1];   // coefficients of p_{l-1}, p_{l-2}
#pragma unroll
        for (int t = 0; t <= LMAX; t++) c1[t] = c2[t] = 0.0;
#pragma unroll
        for (int d = 0; d <= LMAX; d++) {
            if (d > LMAX - m) break;
            double c0[LMAX + 1];
#pragma unroll
            for (int t = 0; t <= LMAX; t++) c0[t] = 0.0;
            if (d == 0) {
                c0[0] = 1.0;
            } else if (d == 1) {
                c0[1] = (double)(2 * m + 1);
            } else {
                const int l = m + d;
                const double aa = (double)(2 * l - 1), bb = (double)(l + m - 1), inv = 1.0 / (double)d;
#pragma unroll
                for (int t = 0; t <= d; t++) {
                    const double v1 = t >= 1 ? c1[t - 1] : 0.0;
                    const double v3 = t >= 2 ? c2[t - 2] : 0.0;
                    c0[t] = (aa * v1 - bb * (rho2 * c2[t] + v3)) * inv;
                }
            }
            double S = 0.0;
#pragma unroll
            for (int t = 0; t <= d; t++) S += c0[t] * Z[t];
            ar[d] += smr * S;
            ai[d] += smi * S;
#pragma unroll
            for (int t = 0; t <= LMAX; t++) {
                c2[t] = c1[t];
                c1[t] = c0[t];
            }
        }
    }
    constexpr int NW = LR_ROWBLK / 32;
    __shared__ double red[NW][2 * (LMAX + 1)];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int d = 0; d <= LMAX; d++) {
        const double vr = warp_sum(ar[d]), vi = warp_sum(ai[d]);
        if (lane == 0) {
            red[warp][2 * d] = vr;
            red[warp][2 * d + 1] = vi;
        }
    }
    __syncthreads();
    const int q = threadIdx.x;
    if (q < 2 * (LMAX + 1)) {
        const int d = q >> 1, l = m + d;
        if (l <= LMAX && (m > 0 || !(q & 1))) {
            double s = 0.0;
            for (int w = 0; w < NW; w++) s += red[w][q];
            const double f = c_norm[l * (LM_MAX + 1) + m] * (g.dx * g.dy * g.dz);
            parts[(long long)blockIdx.x * LM_NC + l * l + l + ((q & 1) ? -m : m)] = f * s;
        }
    }
}

// one warp per coefficient: the blocks' partials, lane-strided, then a fixed
// butterfly (deterministic)
__global__ void __launch_bounds__(32) lmax_final(GravArgs a, const double *parts, int nparts)
{
    const int t = blockIdx.x, lane = threadIdx.x;
    double s = 0.0;
    for (int b = lane; b < nparts; b += 32) s += parts[(long long)b * LM_NC + t];
    s = warp_sum(s);
    if (lane == 0) a.mom[4 + t] = s;
    if (t == 0 && lane < 4) a.mom[lane] = a.sc->moments[lane];
}

__device__ __forceinline__ double eval_lmax(double x, double y, double z, int lmax,
                                            const double *mom, double G)
{
    double rx = x - mom[1], ry = y - mom[2], rz = z - mom[3];
    double r2 = rx * rx + ry * ry + rz * rz;
    if (!(r2 > 0.0)) return 0.0;
    const double inv2 = 1.0 / r2;
    double rp[LM_MAX + 1];
    rp[0] = 1.0 / sqrt(r2);
    for (int l = 1; l <= lmax; l++) rp[l] = rp[l - 1] * inv2;
    const double *cs = mom + 4;
    double sl[LM_MAX + 1];
    for (int l = 0; l <= lmax; l++) sl[l] = 0.0;
    solid_harmonics(rx, ry, rz, lmax, [&](int t, double v) {
        int l = (int)sqrt((double)t + 0.5);
        sl[l] += cs[t] * v;
    });
    double sum = 0.0;
    for (int l = 0; l <= lmax; l++) sum += sl[l] * rp[l];
    return -G * sum;
}

__global__ void boundary_lmax_kernel(GravArgs a)
{
    const Geom g = a.g;
    const bool zb = g.nz > 1;
    const long long nb = boundary_count(g.nx, g.ny, g.nz, zb);
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= nb) return;
    int i, j, k;
    boundary_cell(t, g.nx, g.ny, g.nz, zb, i, j, k);
    if (i < g.olo || i >= g.ohi) return;   // a ghost plane: the neighbour's cells
    double x = g.xmin + (i + g.ioff + 0.5) * g.dx, y = g.ymin + (j + 0.5) * g.dy, z = g.zmin + (k + 0.5) * g.dz;
    if (zb && (k == 0 || k == g.nz - 1)) z = (k == g.nz - 1) ? g.zmax - 0.5 * g.dz : g.zmin + 0.5 * g.dz;
    else if (j == 0 || j == g.ny - 1) y = (j == g.ny - 1) ? g.ymax - 0.5 * g.dy : g.ymin + 0.5 * g.dy;
    else x = (i + g.ioff == g.gnx - 1) ? g.xmax - 0.5 * g.dx : g.xmin + 0.5 * g.dx;
    a.phi[((long long)i * g.ny + j) * g.nz + k] = eval_lmax(x, y, z, a.lmax, a.mom, a.G);
}

bool g_norm_ready[64] = { false };

cudaError_t ensure_norm()
{
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && g_norm_ready[dev]) return cudaSuccess;
    double h[LM_NC];
    for (int l = 0; l <= LM_MAX; l++)
        for (int m = 0; m <= LM_MAX; m++) {
            double v = 0.0;
            if (m <= l) {
                v = (m == 0) ? 1.0 : 2.0;
                for (int t = l - m + 1; t <= l + m; t++) v /= (double)t;
                v = sqrt(v);
            }
            h[l * (LM_MAX + 1) + m] = v;
        }
    cudaError_t e = cudaMemcpyToSymbol(c_norm, h, sizeof h);
    if (e != cudaSuccess) return e;
    if (dev < 64) g_norm_ready[dev] = true;
    return cudaSuccess;
}

}  // namespace

// Row blocks per plane of lmax_rows.
static int rows_per_plane_blocks(const Geom &g) { return (g.ny + LR_ROWBLK - 1) / LR_ROWBLK; }

// Partial sums of the moment passes, per plane: 9 doubles (tree order of
// the quadrupole moments) or rows_per_plane_blocks x LM_NC (lmax rows).
static long long part_cap(const Geom &g)
{
    return std::max<long long>(64 * 1024, (long long)g.nx * rows_per_plane_blocks(g) * LM_NC);
}

long long grav_scratch_len(const Geom &g) { return part_cap(g) + (long long)g.nx * g.ny * (LM_MAX + 1); }

int lmax_slab_width(const Geom &g, int pass) { return pass == 0 ? 4 * COM_PP : rows_per_plane_blocks(g) * LM_NC; }

// Pass 0: the centre-of-mass partials of the own planes; pass 1: the rows'
// z-power sums about the centre of mass (in the scratch after the partials),
// then the harmonic partials of the own planes' row blocks.
cudaError_t grav_moments_lmax_parts(const GravArgs &a, int pass, double *parts, cudaStream_t s)
{
    if (a.lmax < 1 || a.lmax > LM_MAX) return cudaErrorInvalidValue;
    const int np = a.g.ohi - a.g.olo;
    if (np <= 0 || a.scratch_len < grav_scratch_len(a.g)) return cudaErrorInvalidValue;
    cudaError_t e = ensure_norm();
    if (e != cudaSuccess) return e;
    if (pass == 0) {
        lmax_com_partial<<<np * COM_PP, LR_NT, 0, s>>>(a, parts);
        return cudaGetLastError();
    }
    const double *com = a.sc->moments + 1;
    double *zs = a.scratch + part_cap(a.g);
    const long long rows = (long long)np * a.g.ny;
    const int nzb = (int)std::min<long long>((rows + LR_NT / 32 - 1) / (LR_NT / 32), 148LL * 8);
    const int nb = np * rows_per_plane_blocks(a.g);
    auto launch = [&](auto zk, auto rk) -> cudaError_t {
        zk<<<nzb, LR_NT, 0, s>>>(a, com, zs);
        rk<<<dim3(nb, a.lmax + 1), LR_ROWBLK, 0, s>>>(a, com, zs, parts);
        return cudaGetLastError();
    };
    switch (a.lmax) {
    case 1: return launch(lmax_zsums<1>, lmax_rows<1>);
    case 2: return launch(lmax_zsums<2>, lmax_rows<2>);
    case 3: return launch(lmax_zsums<3>, lmax_rows<3>);
    case 4: return launch(lmax_zsums<4>, lmax_rows<4>);
    case 5: return launch(lmax_zsums<5>, lmax_rows<5>);
    case 6: return launch(lmax_zsums<6>, lmax_rows<6>);
    case 7: return launch(lmax_zsums<7>, lmax_rows<7>);
    case 8: return launch(lmax_zsums<8>, lmax_rows<8>);
    case 9: return launch(lmax_zsums<9>, lmax_rows<9>);
    case 10: return launch(lmax_zsums<10>, lmax_rows<10>);
    case 11: return launch(lmax_zsums<11>, lmax_rows<11>);
    default: return launch(lmax_zsums<12>, lmax_rows<12>);
    }
}

// parts: the partials of nplanes planes of the whole grid, in plane order.
cudaError_t grav_moments_lmax_set(const GravArgs &a, int pass, const double *parts, int nplanes, cudaStream_t s)
{
    if (pass == 0) lmax_com_final<<<1, 128, 0, s>>>(a, parts, nplanes * COM_PP);
    else lmax_final<<<(a.lmax + 1) * (a.lmax + 1), 32, 0, s>>>(a, parts, nplanes * rows_per_plane_blocks(a.g));
    return cudaGetLastError();
}

// The centre of mass, the rows' z-power sums about it, then the
// solid-harmonic moments row by row, each from per-plane partials added in
// plane order.
cudaError_t grav_moments_lmax(const GravArgs &a, cudaStream_t s)
{
    const int np = a.g.ohi - a.g.olo;
    cudaError_t e = grav_moments_lmax_parts(a, 0, a.scratch, s);
    if (e == cudaSuccess) e = grav_moments_lmax_set(a, 0, a.scratch, np, s);
    if (e == cudaSuccess) e = grav_moments_lmax_parts(a, 1, a.scratch, s);
    if (e == cudaSuccess) e = grav_moments_lmax_set(a, 1, a.scratch, np, s);
    return e;
}

cudaError_t grav_boundary_lmax(const GravArgs &a, cudaStream_t s)
{
    cudaError_t e = ensure_norm();
    if (e != cudaSuccess) return e;
    long long nb = boundary_count(a.g.nx, a.g.ny, a.g.nz, a.g.nz > 1);
    boundary_lmax_kernel<<<(int)((nb + 127) / 128), 128, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace hc

// ---------------------------------------------------------------------------
// Mixed precision: FP64 outer residual, FP32 red-black SOR on the correction.
//   delta_i = (lap_nbrs(phi)_i - 4 pi G rho_i)/fac - phi_i      (FP64)
//   e_GS    = (cx (e_i-1 + e_i+1) + cy (..) + cz (..)) + delta,  e += w (e_GS - e)
// so phi + e satisfies the same fixed point as the reference's SOR iterate.
// ---------------------------------------------------------------------------
namespace hc {
namespace {

struct MixConst {
    double ix2, iy2, iz2, fpg, fac;
    float cx, cy, cz, om;
};

__host__ __device__ __forceinline__ MixConst mix_const(const GravArgs &a)
{
    MixConst c;
    c.ix2 = 1.0 / (a.g.dx * a.g.dx);
    c.iy2 = 1.0 / (a.g.dy * a.g.dy);
    c.iz2 = 1.0 / (a.g.dz * a.g.dz);
    c.fpg = 4.0 * M_PI * a.G;
    c.fac = 2.0 * (c.ix2 + c.iy2 + c.iz2);
    c.cx = (float)(c.ix2 / c.fac);
    c.cy = (float)(c.iy2 / c.fac);
    c.cz = (float)(c.iz2 / c.fac);
    c.om = (float)a.omega;
    return c;
}

template <int NT>
__device__ __forceinline__ double block_max_any(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = tmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    __shared__ double w[NT / 32];
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    if ((tid & 31) == 0) w[tid >> 5] = v;
    __syncthreads();
    double m = 0.0;
    if (tid == 0)
        for (int t = 0; t < NT / 32; t++) m = tmax(m, w[t]);
    return m;
}

// r32 / e32 in the natural layout, or colour-split (sp.cs > 0)
// One (i, j) row per block iteration, threads along k (no per-cell index
// division).  r32 / e32 in the natural layout, or colour-split (sp.cs > 0).
__global__ void __launch_bounds__(256) mixed_residual_kernel(GravArgs a, float *r32, float *e32, Split sp)
{
    const Geom g = a.g;
    const MixConst mc = mix_const(a);
    const double ifac = 1.0 / mc.fac;
    const long long sI = (long long)g.ny * g.nz, sJ = g.nz;
    const long long rows = (long long)g.nx * g.ny;
    double m = 0.0;
    for (long long row = blockIdx.x; row < rows; row += gridDim.x) {
        const int i = (int)(row / g.ny), j = (int)(row % g.ny);
        const bool inner = i >= 1 && i <= g.nx - 2 && j >= 1 && j <= g.ny - 2;
        const long long c0 = row * sJ;
        for (int k = threadIdx.x; k < g.nz; k += blockDim.x) {
            const long long c = c0 + k;
            const long long o = sp.cs ? sp.at(i, j, k) : c;
            float d = 0.f;
            if (inner && k >= 1 && k <= g.nz - 2) {
                const double *phi = a.phi;
                const double lap = (phi[c - sI] + phi[c + sI]) * mc.ix2 + (phi[c - sJ] + phi[c + sJ]) * mc.iy2 +
                                   (phi[c - 1] + phi[c + 1]) * mc.iz2;
                const double rr = a.rho ? a.rho[c] : (double)a.rho32[c];
                const double dd = (lap - mc.fpg * rr) * ifac - phi[c];
                m = tmax(m, fabs(dd));
                d = (float)dd;
            }
            r32[o] = d;
            e32[o] = 0.f;
        }
    }
    double b = block_max_any<256>(m);
    if (threadIdx.x == 0) atomic_max_nonneg((unsigned long long *)&a.sc->resnorm, b);
}

// phi += sign * e; max|e| into sc->resid_bits (the FP32 resolution check)
__global__ void __launch_bounds__(256) mixed_update_kernel(GravArgs a, const float *e32, Split sp, float sign)
{
    const long long rows = (long long)a.g.nx * a.g.ny;
    float m = 0.f;
    for (long long row = blockIdx.x; row < rows; row += gridDim.x) {
        const int i = (int)(row / a.g.ny), j = (int)(row % a.g.ny);
        const long long c0 = row * a.g.nz;
        for (int k = threadIdx.x; k < a.g.nz; k += blockDim.x) {
            const long long o = sp.cs ? sp.at(i, j, k) : c0 + k;
            const float e = sign * e32[o];
            a.phi[c0 + k] += (double)e;
            m = tmax(m, fabsf(e));
        }
    }
    const double b = block_max_any<256>((double)m);
    if (threadIdx.x == 0 && b > 0.0) atomic_max_nonneg(&a.sc->resid_bits, b);
}

// Pair forms of the residual and the update for the colour-split layout with
// even nz: thread m of a row takes the cells k = 2m and 2m+1 -- one of each
// colour, both at index m of their colour array -- so phi moves as 16-byte
// pairs and each colour array is written with unit stride.  Per cell the
// arithmetic is that of mixed_residual_kernel / mixed_update_kernel.
constexpr int PAIR_NT = 128;
__global__ void __launch_bounds__(PAIR_NT) mixed_residual_pair_kernel(GravArgs a, float *r32, float *e32, Split sp)
{
    const Geom g = a.g;
    const MixConst mc = mix_const(a);
    const double ifac = 1.0 / mc.fac;
    const long long sI = (long long)g.ny * g.nz, sJ = g.nz;
    const long long rows = (long long)g.nx * g.ny;
    const double *phi = a.phi;
    double mx = 0.0;
    for (long long row = blockIdx.x; row < rows; row += gridDim.x) {
        const int i = (int)(row / g.ny), j = (int)(row % g.ny);
        const bool inner = i >= 1 && i <= g.nx - 2 && j >= 1 && j <= g.ny - 2;
        const long long c0 = row * sJ;
        const int cc = (i + j) & 1;   // colour of k = 2m
        float *r0 = r32 + cc * sp.cs + row * sp.H, *r1 = r32 + (cc ^ 1) * sp.cs + row * sp.H;
        float *e0 = e32 + cc * sp.cs + row * sp.H, *e1 = e32 + (cc ^ 1) * sp.cs + row * sp.H;
        for (int m = threadIdx.x; m < sp.H; m += PAIR_NT) {
            const long long c = c0 + 2 * m;
            float d[2] = { 0.f, 0.f };
            if (inner) {
                const double2 pc = *reinterpret_cast<const double2 *>(phi + c);
                const double2 xm = *reinterpret_cast<const double2 *>(phi + c - sI);
                const double2 xp = *reinterpret_cast<const double2 *>(phi + c + sI);
                const double2 ym = *reinterpret_cast<const double2 *>(phi + c - sJ);
                const double2 yp = *reinterpret_cast<const double2 *>(phi + c + sJ);
                const double zl = m > 0 ? phi[c - 1] : 0.0, zr = 2 * m + 2 < g.nz ? phi[c + 2] : 0.0;
                double r0v, r1v;
                if (a.rho) {
                    const double2 rr = *reinterpret_cast<const double2 *>(a.rho + c);
                    r0v = rr.x;
                    r1v = rr.y;
                } else {
                    const float2 rr = *reinterpret_cast<const float2 *>(a.rho32 + c);
                    r0v = (double)rr.x;
                    r1v = (double)rr.y;
                }
                const int k = 2 * m;
                if (k >= 1 && k <= g.nz - 2) {
                    const double lap = (xm.x + xp.x) * mc.ix2 + (ym.x + yp.x) * mc.iy2 + (zl + pc.y) * mc.iz2;
                    const double dd = (lap - mc.fpg * r0v) * ifac - pc.x;
                    mx = tmax(mx, fabs(dd));
                    d[0] = (float)dd;
                }
                if (k + 1 >= 1 && k + 1 <= g.nz - 2) {
                    const double lap = (xm.y + xp.y) * mc.ix2 + (ym.y + yp.y) * mc.iy2 + (pc.x + zr) * mc.iz2;
                    const double dd = (lap - mc.fpg * r1v) * ifac - pc.y;
                    mx = tmax(mx, fabs(dd));
                    d[1] = (float)dd;
                }
            }
            r0[m] = d[0];
            r1[m] = d[1];
            e0[m] = 0.f;
            e1[m] = 0.f;
        }
    }
    const double b = block_max_any<PAIR_NT>(mx);
    if (threadIdx.x == 0) atomic_max_nonneg((unsigned long long *)&a.sc->resnorm, b);
}

__global__ void __launch_bounds__(PAIR_NT) mixed_update_pair_kernel(GravArgs a, const float *e32, Split sp, float sign)
{
    const long long rows = (long long)a.g.nx * a.g.ny;
    float mx = 0.f;
    for (long long row = blockIdx.x; row < rows; row += gridDim.x) {
        const int i = (int)(row / a.g.ny), j = (int)(row % a.g.ny);
        const int cc = (i + j) & 1;
        const float *f0 = e32 + cc * sp.cs + row * sp.H, *f1 = e32 + (cc ^ 1) * sp.cs + row * sp.H;
        double *prow = a.phi + row * a.g.nz;
        for (int m = threadIdx.x; m < sp.H; m += PAIR_NT) {
            const float ea = sign * f0[m], eb = sign * f1[m];
            double2 p = *reinterpret_cast<const double2 *>(prow + 2 * m);
            p.x += (double)ea;
            p.y += (double)eb;
            *reinterpret_cast<double2 *>(prow + 2 * m) = p;
            mx = tmax(mx, tmax(fabsf(ea), fabsf(eb)));
        }
    }
    const double b = block_max_any<PAIR_NT>((double)mx);
    if (threadIdx.x == 0 && b > 0.0) atomic_max_nonneg(&a.sc->resid_bits, b);
}

constexpr int S32_BX = 32, S32_BY = 8;

__global__ void __launch_bounds__(S32_BX * S32_BY)
sor32_color(GravArgs a, float *e, const float *r, int color, int iter, double thresh)
{
    if (*(volatile int *)&a.sc->done) return;
    if (color == 0 && iter > 0) {
        double prev = __longlong_as_double(*reinterpret_cast<const long long *>(a.res + iter - 1));
        if (prev < thresh) {
            if (threadIdx.x == 0 && threadIdx.y == 0) { a.sc->last_iter = iter; a.sc->done = 1; }
            return;
        }
    }
    const Geom g = a.g;
    const MixConst mc = mix_const(a);
    const int i = 1 + blockIdx.z;
    const int j = 1 + blockIdx.y * S32_BY + threadIdx.y;
    const int k0 = ((i + j + 1) % 2 == color) ? 1 : 2;
    const int k = k0 + 2 * (blockIdx.x * S32_BX + threadIdx.x);
    float rr = 0.f;
    if (j <= g.ny - 2 && k <= g.nz - 2) {
        const long long sI = (long long)g.ny * g.nz, sJ = g.nz;
        const long long c = i * sI + j * sJ + k;
        float old = e[c];
        float gs = (e[c - sI] + e[c + sI]) * mc.cx + (e[c - sJ] + e[c + sJ]) * mc.cy +
                   (e[c - 1] + e[c + 1]) * mc.cz + r[c];
        e[c] = old + mc.om * (gs - old);
        rr = fabsf(gs - old);
    }
    double m = block_max_any<S32_BX * S32_BY>((double)rr);
    if (threadIdx.x == 0 && threadIdx.y == 0) atomic_max_nonneg((unsigned long long *)(a.res + iter), m);
}

__global__ void check32_kernel(GravArgs a, int iter, double thresh)
{
    if (a.sc->done) return;
    if (iter > 0) {
        double prev = __longlong_as_double(*reinterpret_cast<const long long *>(a.res + iter - 1));
        if (prev < thresh) { a.sc->last_iter = iter; a.sc->done = 1; }
    }
}

}  // namespace

static Split split_or_natural(const GravArgs &a, bool split)
{
    Split sp = make_split(a.g);
    if (!split) sp.cs = 0;
    return sp;
}

// the pair kernels need the colour-split layout, even nz and 16-byte aligned rows
static bool pair_ok(const GravArgs &a, bool split)
{
    return HC_MIXED_PAIR && split && a.g.nz % 2 == 0 && ((uintptr_t)a.phi % 16) == 0 &&
           ((uintptr_t)(a.rho ? (const void *)a.rho : (const void *)a.rho32) % 16) == 0;
}

cudaError_t mixed_residual(const GravArgs &a, float *r32, float *e32, bool split, cudaStream_t s)
{
    if (pair_ok(a, split))
        mixed_residual_pair_kernel<<<148 * 32, PAIR_NT, 0, s>>>(a, r32, e32, make_split(a.g));
    else
        mixed_residual_kernel<<<148 * 16, 256, 0, s>>>(a, r32, e32, split_or_natural(a, split));
    return cudaGetLastError();
}

cudaError_t mixed_update(const GravArgs &a, const float *e32, bool split, float sign, cudaStream_t s)
{
    if (pair_ok(a, split))
        mixed_update_pair_kernel<<<148 * 32, PAIR_NT, 0, s>>>(a, e32, make_split(a.g), sign);
    else
        mixed_update_kernel<<<148 * 16, 256, 0, s>>>(a, e32, split_or_natural(a, split), sign);
    return cudaGetLastError();
}

// TMA-staged colour sweep (sor_split_tma.cuh) when the rows fit one bulk
// copy box and every stride is a multiple of 16 bytes; returns
// cudaErrorNotSupported (nothing launched) otherwise.
template <int NI, int NS>
static cudaError_t sweep_tma(float *base, const float *src, const Split &sp, const SorCoef<float> &cf, int colour,
                             double *res, int iter, double thresh, DevScalars *sc, cudaStream_t s)
{
    const size_t smem = (size_t)NS * stma::stage_floats<NI>(sp.H) * 4;
    // the limit is raised once per device, to what the longest rows this
    // instantiation takes need (HM cells per colour row)
    constexpr int HM = NI == 4 ? 128 : stma::HMAX;
    static std::atomic<unsigned long long> attr_set{0};
    cudaError_t e = set_smem_once(attr_set, (const void *)stma::sor_split_tma_kernel<NI, NS>,
                                  (int)((size_t)NS * stma::stage_floats<NI>(HM) * 4));
    if (e != cudaSuccess) return e;
    float *own = base + (size_t)colour * sp.cs;
    const float *oth = base + (size_t)(colour ^ 1) * sp.cs;
    const float *srcc = src + (size_t)colour * sp.cs;
    CUtensorMap mo, mw, ms;
    if (!tmap3(oth, 4, sp.nx, sp.ny, sp.H, sp.H, stma::TJ + 2, &mo, NI + 2) ||
        !tmap3(own, 4, sp.nx, sp.ny, sp.H, sp.H, stma::TJ, &mw, NI) ||
        !tmap3(srcc, 4, sp.nx, sp.ny, sp.H, sp.H, stma::TJ, &ms, NI))
        return cudaErrorNotSupported;
    stma::Tiles tl;
    tl.nx = sp.nx;
    tl.ny = sp.ny;
    tl.nz = sp.nz;
    tl.H = sp.H;
    tl.ti = (sp.nx - 2 + NI - 1) / NI;
    tl.tj = (sp.ny - 2 + stma::TJ - 1) / stma::TJ;
    static int sms_dev[64] = { 0 };
    int dev = 0;
    e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    int sms = (dev >= 0 && dev < 64) ? sms_dev[dev] : 0;
    if (!sms) {
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
        if (dev >= 0 && dev < 64) sms_dev[dev] = sms;
    }
    const int grid = std::min(tl.ti * tl.tj, sms);
    return launch_pdl_smem(stma::sor_split_tma_kernel<NI, NS>, dim3(grid), dim3(stma::NT), smem, s, mo, mw, ms, own,
                           tl, cf, colour, res, iter, thresh, sc);
}

cudaError_t mixed_sor32_split(const GravArgs &a, float *e32, const float *r32, int colour, int iter,
                              double thresh, cudaStream_t s)
{
    const MixConst mc = mix_const(a);
    SorCoef<float> cf;
    cf.cx = mc.cx;
    cf.cy = mc.cy;
    cf.cz = mc.cz;
    cf.om = mc.om;
    const Split sp = make_split(a.g);
    if (a.sweep_kind == 1 && sp.H % 4 == 0 && sp.H <= stma::HMAX && sp.nx >= 3 && sp.ny >= 3 &&
        ((uintptr_t)e32 | (uintptr_t)r32) % 16 == 0 && sp.cs % 4 == 0) {
        cudaError_t e = sp.H <= 128 ? sweep_tma<4, 2>(e32, r32, sp, cf, colour, a.res, iter, thresh, a.sc, s)
                                    : sweep_tma<2, 2>(e32, r32, sp, cf, colour, a.res, iter, thresh, a.sc, s);
        if (e != cudaErrorNotSupported) return e;
    }
    return launch_sor_split<float, float>(e32, r32, sp, cf, colour, a.res, iter, thresh, a.sc, s);
}

cudaError_t mixed_sor32(const GravArgs &a, float *e32, const float *r32, int color, int iter,
                        double thresh, cudaStream_t s)
{
    int nhalf = (a.g.nz - 1) / 2;
    dim3 grid((nhalf + S32_BX - 1) / S32_BX, (a.g.ny - 2 + S32_BY - 1) / S32_BY, a.g.nx - 2);
    sor32_color<<<grid, dim3(S32_BX, S32_BY), 0, s>>>(a, e32, r32, color, iter, thresh);
    return cudaGetLastError();
}

cudaError_t mixed_check(const GravArgs &a, int iter, double thresh, cudaStream_t s)
{
    check32_kernel<<<1, 1, 0, s>>>(a, iter, thresh);
    return cudaGetLastError();
}

// Tiling of the two-iteration passes: the largest window (BJ <= 8 owned rows)
// that fits shared memory, and the row tiles x plane chunks that fill the SMs
// with one CTA each at the least recomputed halo.
static bool wave_split_plan(const Geom &g, int &BJ, int &L, int &jt, int &ch)
{
    const Split sp = make_split(g);
    if (g.nz < 3 || g.nx < 3 || g.ny < 3 || sp.H % 4) return false;
    int dev = 0, nsm = 148, optin = 227 * 1024;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    double best = 1e300;
    bool ok = false;
    for (int bj = 8; bj >= 4; bj--) {
        if (wave_split_smem(bj + 2 * WV_NH, sp.H) + 2 * (WV_THREADS / 32) * sizeof(float) > (size_t)optin) continue;
        const int t = (g.ny - 2 + bj - 1) / bj;
        const int c = std::max(1, (int)std::lround((double)nsm / t));
        const int l = (g.nx - 2 + c - 1) / c;
        const int cc = (g.nx - 2 + l - 1) / l;
        const long long ctas = (long long)t * cc;
        const long long waves = (ctas + nsm - 1) / nsm;
        const double eff = (double)ctas / (double)(waves * nsm);
        const double halo = (4.0 * bj + 12.0) / (4.0 * bj) * (l + 6.0) / l;
        const double cost = halo / eff;
        if (cost < best) {
            best = cost;
            BJ = bj;
            L = l;
            jt = t;
            ch = cc;
            ok = true;
        }
    }
    return ok;
}

bool mixed_wave_split_ok(const Geom &g)
{
    int BJ, L, jt, ch;
    return wave_split_plan(g, BJ, L, jt, ch);
}

cudaError_t mixed_sor32_split_pass(const GravArgs &a, const float *ein, float *eout, const float *r32, int iter0,
                                   double thresh, cudaStream_t s)
{
    int BJ = 0, L = 0, jt = 0, ch = 0;
    if (!wave_split_plan(a.g, BJ, L, jt, ch)) return cudaErrorInvalidValue;
    const Split sp = make_split(a.g);
    if (sp.cs + 2LL * sp.ny * sp.H >= (1LL << 31)) return cudaErrorInvalidValue;
    const size_t smem = wave_split_smem(BJ + 2 * WV_NH, sp.H);
    static size_t attr_bytes[64] = { 0 };
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 64 || smem > attr_bytes[dev]) {
        cudaError_t e = cudaFuncSetAttribute(sor_wave_split_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        if (dev < 64) attr_bytes[dev] = smem;
    }
    const MixConst mc = mix_const(a);
    SorCoef<float> cf;
    cf.cx = mc.cx;
    cf.cy = mc.cy;
    cf.cz = mc.cz;
    cf.om = mc.om;
    sor_wave_split_kernel<<<dim3(jt, ch), WV_THREADS, smem, s>>>(ein, eout, r32, sp, cf, BJ, L, a.res, iter0, thresh,
                                                                 a.sc);
    return cudaGetLastError();
}

}  // namespace hc

// ---------------------------------------------------------------------------
// FP32 correction sweeps with temporal blocking: 4 iterations per HBM pass.
// ---------------------------------------------------------------------------
#include "sor_wavefront.cuh"
#include "sor_wavefront_tma.cuh"
#include "tmap.cuh"

namespace hc {
bool wf_tma_enabled();
namespace {
constexpr int WF32_TJ = 16, WF32_TK = 64, WF32_NT = 512;
template <int TT>
cudaError_t pass32(const GravArgs &a, const float *in, float *out, const float *r32, int iter0,
                   double thresh, cudaStream_t s)
{
    constexpr size_t sm = sor_wavefront_smem<float, TT, WF32_TJ, WF32_TK>();
    auto kern = sor_wavefront_kernel<float, float, TT, WF32_TJ, WF32_TK, WF32_NT>;
    static std::atomic<unsigned long long> attr_set{0};
    cudaError_t e = set_smem_once(attr_set, (const void *)kern, (int)sm);
    if (e != cudaSuccess) return e;
    SorCoef<float> cf;
    double ix2 = 1.0 / (a.g.dx * a.g.dx), iy2 = 1.0 / (a.g.dy * a.g.dy), iz2 = 1.0 / (a.g.dz * a.g.dz);
    double fac = 2.0 * (ix2 + iy2 + iz2);
    cf.cx = (float)(ix2 / fac);
    cf.cy = (float)(iy2 / fac);
    cf.cz = (float)(iz2 / fac);
    cf.om = (float)a.omega;
    const int tj = (a.g.ny + WF32_TJ - 1) / WF32_TJ, tk = (a.g.nz + WF32_TK - 1) / WF32_TK;
    const int nint = a.g.nx - 2;
    long long want = 148LL * 2 * 3;
    int chunks = (int)std::max(1LL, std::min((long long)nint / 24, (want + tj * tk - 1) / (tj * tk)));
    chunks = std::max(chunks, 1);
    int chunk = (nint + chunks - 1) / chunks;
    chunks = (nint + chunk - 1) / chunk;
    dim3 grid(tk, tj, chunks);
    using SH = wtma::Shape<float, TT, WF32_TJ, WF32_TK>;
    CUtensorMap tin, tsrc;
    // FP32 bulk copies start on 16 bytes: k0 - 2T must be a multiple of 4
    if (TT >= 2 && wf_tma_enabled() && tmap3(in, 4, a.g.nx, a.g.ny, a.g.nz, SH::SK, SH::SJ, &tin) &&
        tmap3(r32, 4, a.g.nx, a.g.ny, a.g.nz, SH::SK, SH::SJ, &tsrc)) {
        auto kt = wtma::sor_wavefront_tma_kernel<float, float, TT, WF32_TJ, WF32_TK, WF32_NT>;
        static std::atomic<unsigned long long> attr_t{0};
        e = set_smem_once(attr_t, (const void *)kt, (int)SH::SMEM);
        if (e != cudaSuccess) return e;
        kt<<<grid, WF32_NT, SH::SMEM, s>>>(tin, tsrc, out, a.g, cf, a.res, iter0, thresh, a.sc, chunk);
        return cudaGetLastError();
    }
    kern<<<grid, WF32_NT, sm, s>>>(in, out, r32, a.g, cf, a.res, iter0, thresh, a.sc, chunk);
    return cudaGetLastError();
}
}  // namespace

cudaError_t mixed_sor32_pass(const GravArgs &a, const float *in, float *out, const float *r32, int iter0,
                             int depth, double thresh, cudaStream_t s)
{
    switch (depth) {
    case 1: return pass32<1>(a, in, out, r32, iter0, thresh, s);
    case 2: return pass32<2>(a, in, out, r32, iter0, thresh, s);
    case 4: return pass32<4>(a, in, out, r32, iter0, thresh, s);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace hc
