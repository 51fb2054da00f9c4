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
// at l*l+l+m (C, m >= 0) and l*l+l-m (S, m > 0).  The sums are FP64 and use a
// fixed-shape tree, so they are deterministic.
#include <algorithm>

#include "hc_internal.cuh"
#include "hc_math.cuh"
#include "sor_split.cuh"

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

__constant__ double c_rinv[LM_MAX + 1];   // 1 / d for d = l - m >= 2 (index d)

// Solid-harmonic moments, one order m per warp: block b takes the (i,j) rows
// b, b + gridDim, ..., lane L the cells k = L, L+32, ... of each row, and
// accumulates, in registers, dm N_lm Q_l^m
// for l = m..lmax with the recursion of solid_harmonics (same operations, the
// division by l-m replaced by the identical product with 1/(l-m) computed on
// the host); a fixed butterfly reduction per warp writes this block's partial
// sums, which lmax_final adds in block order.
template <int LMAX>
__global__ void __launch_bounds__(32 * (LMAX + 1)) lmax_partial(GravArgs a, const double *com)
{
    const Geom g = a.g;
    constexpr int lmax = LMAX;
    const int m = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (m > lmax) return;
    const double dV = g.dx * g.dy * g.dz;
    const long long snz = g.nz;
    const double xc = com[0], yc = com[1], zc = com[2];
    double ar[LMAX + 1], ai[LMAX + 1];
#pragma unroll
    for (int d = 0; d <= LMAX; d++) ar[d] = ai[d] = 0.0;
    const long long rows = (long long)g.nx * g.ny;
    for (long long row = blockIdx.x; row < rows; row += gridDim.x) {
      const int i = (int)(row / g.ny), j = (int)(row % g.ny);
      const double x = g.xmin + (i + 0.5) * g.dx - xc;
      const double y = g.ymin + (j + 0.5) * g.dy - yc;
      for (int k = lane; k < g.nz; k += 32) {
        const long long c = row * snz + k;
        const double r = a.rho ? a.rho[c] : (double)a.rho32[c];
        if (!(r > 0.0)) continue;
        const double z = g.zmin + (k + 0.5) * g.dz - zc;
        const double dm = r * dV;
        const double r2 = x * x + y * y + z * z;
        double smr = 1.0, smi = 0.0;      // Q_m^m
        for (int q = 1; q <= m; q++) {
            const double f = (double)(2 * q - 1);
            const double nr = f * (x * smr - y * smi);
            const double ni = f * (x * smi + y * smr);
            smr = nr;
            smi = ni;
        }
        double pr = smr, pi = smi, ppr = 0.0, ppi = 0.0;
        {
            const double nrm = c_norm[m * (LM_MAX + 1) + m];
            ar[0] += dm * (nrm * smr);
            ai[0] += dm * (nrm * smi);
        }
#pragma unroll
        for (int d = 1; d <= LMAX; d++) {
            const int l = m + d;
            if (l > lmax) break;
            double cr, ci;
            if (d == 1) {
                cr = (2 * m + 1) * z * smr;
                ci = (2 * m + 1) * z * smi;
            } else {
                const double aa = (double)(2 * l - 1), bb = (double)(l + m - 1), inv = c_rinv[d];
                cr = (aa * z * pr - bb * r2 * ppr) * inv;
                ci = (aa * z * pi - bb * r2 * ppi) * inv;
            }
            ppr = pr;
            ppi = pi;
            pr = cr;
            pi = ci;
            const double nrm = c_norm[l * (LM_MAX + 1) + m];
            ar[d] += dm * (nrm * cr);
            ai[d] += dm * (nrm * ci);
        }
      }
    }
#pragma unroll
    for (int d = 0; d <= LMAX; d++) {
        double vr = ar[d], vi = ai[d];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            vr += __shfl_xor_sync(0xffffffffu, vr, o);
            vi += __shfl_xor_sync(0xffffffffu, vi, o);
        }
        const int l = m + d;
        if (lane == 0 && l <= lmax) {
            a.scratch[(long long)blockIdx.x * LM_NC + l * l + l + m] = vr;
            if (m > 0) a.scratch[(long long)blockIdx.x * LM_NC + l * l + l - m] = vi;
        }
    }
}

__global__ void lmax_final(GravArgs a, int nparts)
{
    const int nc = (a.lmax + 1) * (a.lmax + 1);
    for (int t = threadIdx.x; t < nc; t += blockDim.x) {
        double s = 0.0;
        for (int b = 0; b < nparts; b++) s += a.scratch[(long long)b * LM_NC + t];
        a.mom[4 + t] = s;
    }
    if (threadIdx.x == 0) {
        a.mom[0] = a.sc->moments[0];
        a.mom[1] = a.sc->moments[1];
        a.mom[2] = a.sc->moments[2];
        a.mom[3] = a.sc->moments[3];
    }
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
    double x = g.xmin + (i + 0.5) * g.dx, y = g.ymin + (j + 0.5) * g.dy, z = g.zmin + (k + 0.5) * g.dz;
    if (zb && (k == 0 || k == g.nz - 1)) z = (k == g.nz - 1) ? g.zmax - 0.5 * g.dz : g.zmin + 0.5 * g.dz;
    else if (j == 0 || j == g.ny - 1) y = (j == g.ny - 1) ? g.ymax - 0.5 * g.dy : g.ymin + 0.5 * g.dy;
    else x = (i == g.nx - 1) ? g.xmax - 0.5 * g.dx : g.xmin + 0.5 * g.dx;
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
    double rinv[LM_MAX + 1];
    for (int d = 0; d <= LM_MAX; d++) rinv[d] = d > 0 ? 1.0 / (double)d : 0.0;
    e = cudaMemcpyToSymbol(c_rinv, rinv, sizeof rinv);
    if (e == cudaSuccess && dev < 64) g_norm_ready[dev] = true;
    return e;
}

}  // namespace

// centre of mass first (tree), then the solid-harmonic moments about it
cudaError_t grav_moments_lmax(const GravArgs &a, cudaStream_t s)
{
    if (a.lmax < 1 || a.lmax > LM_MAX) return cudaErrorInvalidValue;

    cudaError_t e = ensure_norm();
    if (e != cudaSuccess) return e;
    GravArgs t = a;
    e = grav_moments_tree(t, s);       // M, COM, Q (Q unused here)
    if (e != cudaSuccess) return e;
    // blocks: every SM filled to its occupancy for this l_max
    static int nb_cache[LM_MAX + 1] = { 0 };
    int nb = nb_cache[a.lmax];
    auto launch = [&](auto kern) -> cudaError_t {
        if (!nb) {
            int per = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, 32 * (a.lmax + 1), 0) != cudaSuccess ||
                per < 1)
                per = 1;
            nb = std::min(148 * per, (int)(a.scratch_len / LM_NC));
            nb_cache[a.lmax] = nb;
        }
        kern<<<nb, 32 * (a.lmax + 1), 0, s>>>(a, a.sc->moments + 1);
        return cudaGetLastError();
    };
    switch (a.lmax) {
    case 1: e = launch(lmax_partial<1>); break;
    case 2: e = launch(lmax_partial<2>); break;
    case 3: e = launch(lmax_partial<3>); break;
    case 4: e = launch(lmax_partial<4>); break;
    case 5: e = launch(lmax_partial<5>); break;
    case 6: e = launch(lmax_partial<6>); break;
    case 7: e = launch(lmax_partial<7>); break;
    case 8: e = launch(lmax_partial<8>); break;
    case 9: e = launch(lmax_partial<9>); break;
    case 10: e = launch(lmax_partial<10>); break;
    case 11: e = launch(lmax_partial<11>); break;
    default: e = launch(lmax_partial<12>); break;
    }
    if (e != cudaSuccess) return e;
    lmax_final<<<1, 256, 0, s>>>(a, nb);
    return cudaGetLastError();
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

cudaError_t mixed_residual(const GravArgs &a, float *r32, float *e32, bool split, cudaStream_t s)
{
    mixed_residual_kernel<<<148 * 16, 256, 0, s>>>(a, r32, e32, split_or_natural(a, split));
    return cudaGetLastError();
}

cudaError_t mixed_update(const GravArgs &a, const float *e32, bool split, float sign, cudaStream_t s)
{
    mixed_update_kernel<<<148 * 16, 256, 0, s>>>(a, e32, split_or_natural(a, split), sign);
    return cudaGetLastError();
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
    return launch_sor_split<float, float>(e32, r32, make_split(a.g), cf, colour, a.res, iter, thresh, a.sc, s);
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
    static int attr_dev = -1;
    int dev = 0;
    cudaGetDevice(&dev);
    if (attr_dev != dev) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        attr_dev = dev;
    }
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
        static int attr_t = -1;
        if (attr_t != dev) {
            cudaError_t e = cudaFuncSetAttribute(kt, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SH::SMEM);
            if (e != cudaSuccess) return e;
            attr_t = dev;
        }
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
