// sor_wavefront.cuh -- red-black SOR with temporal blocking: T full
// iterations (2T half sweeps) per pass over HBM.
//
// A CTA owns a TJ x TK column of (j,k) and streams along i.  Shared memory
// holds a window of 2T+2 planes of the tile plus a 2T-cell ring.  At stream
// position i, half sweep h (h = 2l + colour, level l = 0..T-1) updates plane
// i-h in place; the dependency check is:
//   red_l  at p reads black at p-1,p,p+1 after black_{l-1} and before black_l
//   black_l at p reads red at p-1,p,p+1 after red_l and before red_{l+1}
// which the h-ordered loop satisfies.  Half sweep h covers the tile plus a
// ring of 2T-1-h cells, so the ring cells it reads always hold the previous
// half sweep's values; the outermost ring is input only.  Planes leave the
// window finished after black_{T-1} and are written to the output buffer.
//
// The pass is out of place (phi_in -> phi_out), so CTAs never read another
// CTA's partially updated cells.  Within a colour the updates are independent
// and each cell sees exactly the neighbour values the sequential red-black
// sweep gives it, so the iterates are the same -- in FP64 bit for bit.
//
// The update norm max |phi_GS - phi_old| of each level is reduced with a warp
// max and one atomic per CTA into that iteration's slot.  A pass starts only
// if the previous iteration's slot is not below the stop threshold.
#pragma once
#include "hc_internal.cuh"
#include "hc_math.cuh"

namespace hc {

template <typename T> struct SorCoef;
template <> struct SorCoef<double> {
    double ix2, iy2, iz2, fpg, fac, om;
    __device__ __forceinline__ double update(double old, double xm, double xp, double ym, double yp,
                                             double zm, double zp, double src, double &r) const
    {
        // gravity_solver_3d.c:654-671, operand order kept
        double lap = (xm + xp) * ix2 + (ym + yp) * iy2 + (zm + zp) * iz2;
        double nw = (lap - fpg * src) / fac;
        r = fabs(nw - old);
        return old + om * (nw - old);
    }
};
// FP32 correction sweep: e_GS = cx (e_x- + e_x+) + cy (..) + cz (..) + delta.
// The multiply-adds are written out (fmaf), so every FP32 sweep kernel --
// scalar, vector, streaming and the two-iteration pass -- rounds each update
// the same way and they produce the same iterates bit for bit, whatever the
// compiler would contract in each.
template <> struct SorCoef<float> {
    float cx, cy, cz, om;
    __device__ __forceinline__ float update(float old, float xm, float xp, float ym, float yp,
                                            float zm, float zp, float src, float &r) const
    {
        const float gs = __fadd_rn(__fmaf_rn(__fadd_rn(zm, zp), cz,
                                             __fmaf_rn(__fadd_rn(ym, yp), cy, __fmul_rn(__fadd_rn(xm, xp), cx))),
                                   src);
        const float d = __fsub_rn(gs, old);
        r = fabsf(d);
        return __fmaf_rn(om, d, old);
    }
};

template <typename T, typename S, int T_, int TJ, int TK, int NT>
__global__ void __launch_bounds__(NT)
sor_wavefront_kernel(const T *__restrict__ in, T *__restrict__ out, const S *__restrict__ src,
                     Geom g, SorCoef<T> cf, double *res, int iter0, double thresh, DevScalars *sc,
                     int chunk)
{
    constexpr int R = 2 * T_;                 // input ring
    constexpr int SJ = TJ + 2 * R, SK = TK + 2 * R;
    constexpr int NP = 2 * T_ + 2;            // planes in the window
    extern __shared__ __align__(16) unsigned char smraw[];
    T *win = reinterpret_cast<T *>(smraw);   // NP x SJ x SK, plane slot = p % NP

    if (*(volatile int *)&sc->done) return;
    if (iter0 > 0) {
        double prev = __longlong_as_double(*reinterpret_cast<const long long *>(res + iter0 - 1));
        if (prev < thresh) {
            if (threadIdx.x == 0) { sc->last_iter = iter0; sc->done = 1; }
            return;
        }
    }
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const long long sI = (long long)ny * nz, sJ = nz;
    const int k0 = blockIdx.x * TK, j0 = blockIdx.y * TJ;
    const int P0 = 1 + blockIdx.z * chunk;               // first output plane
    const int P1 = min(nx - 1, P0 + chunk);              // one past the last
    if (P0 >= P1) return;
    const int tid = threadIdx.x;

    auto slot = [&](int p) { return win + (size_t)(((p % NP) + NP) % NP) * SJ * SK; };
    constexpr int NW = NT / 32;
    const int lane = tid & 31, warp = tid >> 5;
    auto load_plane = [&](int p) {
        T *w = slot(p);
        const bool pin = (p >= 0 && p < nx);
        for (int sj = warp; sj < SJ; sj += NW) {
            const int gj = j0 - R + sj;
            const bool jin = pin && gj >= 0 && gj < ny;
            const T *row = in + (jin ? p * sI + gj * sJ : 0);
            for (int sk = lane; sk < SK; sk += 32) {
                const int gk = k0 - R + sk;
                w[sj * SK + sk] = (jin && gk >= 0 && gk < nz) ? row[gk] : (T)0;
            }
        }
    };

    float rmax[T_];
#pragma unroll
    for (int l = 0; l < T_; l++) rmax[l] = 0.f;
    double rmaxd[T_];
#pragma unroll
    for (int l = 0; l < T_; l++) rmaxd[l] = 0.0;

    const int L0 = P0 - 2 * T_ + 1;     // first plane red_0 processes
    // prime the window: planes L0-1 .. L0 (h = 0 at step L0 also needs L0+1)
    load_plane(L0 - 1);
    load_plane(L0);
    const int last_step = P1 - 1 + 2 * T_ - 1;
    for (int i = L0; i <= last_step; i++) {
        load_plane(i + 1);
        __syncthreads();
#pragma unroll
        for (int h = 0; h < 2 * T_; h++) {
            const int p = i - h;
            const int lh = max(1, L0 + h);
            // red_0 runs up to plane P1-1+2T-1, each later half sweep one less
            const int uh = min(nx - 2, P1 - 1 + 2 * T_ - 1 - h);
            if (p >= lh && p <= uh) {
                const int ring = 2 * T_ - 1 - h;
                const int color = h & 1;
                const int rj = TJ + 2 * ring, rk = TK + 2 * ring;
                const int rk2 = (rk + 1) / 2;
                T *wc = slot(p), *wm = slot(p - 1), *wp = slot(p + 1);
                for (int jj = warp; jj < rj; jj += NW) {
                    const int gj = j0 - ring + jj;
                    if (gj < 1 || gj > ny - 2) continue;
                    const int kstart = k0 - ring;
                    // first k >= kstart with (p + gj + k) % 2 == color
                    const int kpar = ((p + gj + kstart) & 1) ^ color;
                    const S *srow = src + p * sI + gj * sJ;
                    const int sj = gj - j0 + R;
                    for (int kk = lane; kk < rk2; kk += 32) {
                        const int gk = kstart + kpar + 2 * kk;
                        if (gk >= kstart + rk || gk < 1 || gk > nz - 2) continue;
                        const int s = sj * SK + (gk - k0 + R);
                        T r;
                        T old = wc[s];
                        T nv = cf.update(old, wm[s], wp[s], wc[s - SK], wc[s + SK], wc[s - 1], wc[s + 1],
                                         (T)srow[gk], r);
                        wc[s] = nv;
                        if (sizeof(T) == 8) rmaxd[h >> 1] = tmax(rmaxd[h >> 1], (double)r);
                        else rmax[h >> 1] = tmax(rmax[h >> 1], (float)r);
                    }
                }
            }
            __syncthreads();
        }
        // plane i-2T+1 is final: write the tile interior
        const int po = i - 2 * T_ + 1;
        if (po >= P0 && po < P1) {
            const T *w = slot(po);
            for (int jj = warp; jj < TJ; jj += NW) {
                const int gj = j0 + jj;
                if (gj < 1 || gj > ny - 2) continue;
                for (int kk = lane; kk < TK; kk += 32) {
                    const int gk = k0 + kk;
                    if (gk >= 1 && gk <= nz - 2) out[po * sI + gj * sJ + gk] = w[(jj + R) * SK + kk + R];
                }
            }
        }
        // the slot of plane i-2T is reused by plane i+2 at the next load
        __syncthreads();
    }
#pragma unroll
    for (int l = 0; l < T_; l++) {
        double v = (sizeof(T) == 8) ? rmaxd[l] : (double)rmax[l];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = tmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        if ((tid & 31) == 0 && v > 0.0)
            atomic_max_nonneg((unsigned long long *)(res + iter0 + l), v);
    }
}

template <typename T, int T_, int TJ, int TK>
constexpr size_t sor_wavefront_smem()
{
    return sizeof(T) * (size_t)(2 * T_ + 2) * (TJ + 4 * T_) * (TK + 4 * T_);
}

}  // namespace hc
