// sor_wavefront_tma.cuh -- the temporally blocked red-black SOR pass of
// sor_wavefront.cuh with its operands staged by TMA one plane ahead.
//
// Same schedule and arithmetic as sor_wavefront_kernel (see there for the
// dependency argument): T iterations per pass, half sweep h at plane i-h,
// out of place.  Differences: the potential plane and the source plane (rho,
// or the FP32 residual) of the next stream step are fetched by two
// cp.async.bulk.tensor loads into ring buffers while the current step's half
// sweeps run, completing on one mbarrier per step; the half sweeps read only
// shared memory.  Out-of-range planes, rows and columns arrive as zeros from
// the tensor copy; the update still skips every cell outside the interior.
#pragma once
#include <cuda.h>

#include "hc_internal.cuh"
#include "hc_math.cuh"
#include "sor_wavefront.cuh"

namespace hc {
namespace wtma {

__device__ __forceinline__ unsigned saddr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool bar_wait(uint64_t *bar, unsigned parity)
{
    const unsigned a = saddr(bar);
    for (int it = 0; it < (1 << 22); it++) {
        unsigned ok;
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(ok)
                     : "r"(a), "r"(parity)
                     : "memory");
        if (ok) return true;
        if (it > 64) __nanosleep(32);
    }
    return false;
}

__device__ __forceinline__ void tma3(const CUtensorMap *tm, void *dst, uint64_t *bar, int x, int y, int z)
{
    asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(saddr(dst)),
                 "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(z), "r"(saddr(bar))
                 : "memory");
}

template <typename T, int T_, int TJ, int TK>
struct Shape {
    static constexpr int R = 2 * T_;
    static constexpr int SJ = TJ + 2 * R, SK = TK + 2 * R;
    static constexpr int PLANE = SJ * SK;                                  // elements
    static constexpr int PLANE_P = ((PLANE * (int)sizeof(T) + 127) / 128) * 128 / (int)sizeof(T);
    static constexpr int NPP = 2 * T_ + 3;     // potential planes: 2T+2 in use + 1 in flight
    static constexpr int NPS = 2 * T_ + 1;     // source planes: 2T in use + 1 in flight
    static constexpr size_t SMEM = sizeof(T) * (size_t)PLANE_P * (NPP + NPS) + 64;
};

template <typename T, typename S, int T_, int TJ, int TK, int NT>
__global__ void __launch_bounds__(NT)
sor_wavefront_tma_kernel(const __grid_constant__ CUtensorMap tm_in, const __grid_constant__ CUtensorMap tm_src,
                         T *__restrict__ out, Geom g, SorCoef<T> cf, double *res, int iter0, double thresh,
                         DevScalars *sc, int chunk)
{
    static_assert(sizeof(S) == sizeof(T), "source staged with the potential's element size");
    using SH = Shape<T, T_, TJ, TK>;
    constexpr int R = SH::R, SJ = SH::SJ, SK = SH::SK, PP = SH::PLANE_P;
    constexpr int NPP = SH::NPP, NPS = SH::NPS;
    constexpr int NW = NT / 32;
    extern __shared__ __align__(128) unsigned char smraw[];
    T *win = reinterpret_cast<T *>(smraw);                 // NPP potential planes
    S *swin = reinterpret_cast<S *>(win + (size_t)NPP * PP); // NPS source planes
    uint64_t *bar = reinterpret_cast<uint64_t *>(swin + (size_t)NPS * PP);   // 2 barriers

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
    const int P0 = 1 + blockIdx.z * chunk;
    const int P1 = min(nx - 1, P0 + chunk);
    if (P0 >= P1) return;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    auto pslot = [&](int p) { return win + (size_t)(((p % NPP) + NPP) % NPP) * PP; };
    auto sslot = [&](int p) { return swin + (size_t)(((p % NPS) + NPS) % NPS) * PP; };
    constexpr unsigned BYTES = (unsigned)(SJ * SK * sizeof(T));

    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(&bar[0])));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(&bar[1])));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    // step i consumes potential plane i+1 and source plane i; both arrive on
    // bar[i & 1].  `np`/`ns` = number of potential/source planes in the copy.
    auto issue = [&](int i, bool pot, int pplane, bool src, int splane) {
        if (tid != 0) return;
        uint64_t *b = &bar[i & 1];
        unsigned bytes = (pot ? BYTES : 0u) + (src ? BYTES : 0u);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(b)), "r"(bytes)
                     : "memory");
        if (pot) tma3(&tm_in, pslot(pplane), b, k0 - R, j0 - R, pplane);
        if (src) tma3(&tm_src, sslot(splane), b, k0 - R, j0 - R, splane);
    };
    unsigned phase[2] = { 0u, 0u };
    bool ok = true;

    float rmax[T_];
    double rmaxd[T_];
#pragma unroll
    for (int l = 0; l < T_; l++) { rmax[l] = 0.f; rmaxd[l] = 0.0; }

    const int L0 = P0 - 2 * T_ + 1;
    const int last_step = P1 - 1 + 2 * T_ - 1;
    // prologue: potential planes L0-1, L0 and the first step's (L0+1, src L0)
    issue(L0 - 1, true, L0 - 1, false, 0);     // on bar[(L0-1)&1]
    // (L0-1) and (L0+1) share a barrier: wait before its next use
    ok = bar_wait(&bar[(L0 - 1) & 1], phase[(L0 - 1) & 1]) && ok;
    phase[(L0 - 1) & 1] ^= 1u;
    // every thread must have observed that phase before the barrier is armed
    // again: a thread still polling parity 0 after the next phase completed
    // would wait for the phase after that
    __syncthreads();
    issue(L0 + 1, true, L0, false, 0);         // potential plane L0 on bar[(L0+1)&1]
    ok = bar_wait(&bar[(L0 + 1) & 1], phase[(L0 + 1) & 1]) && ok;
    phase[(L0 + 1) & 1] ^= 1u;
    issue(L0, true, L0 + 1, true, L0);         // step L0's data on bar[L0&1]

    for (int i = L0; i <= last_step; i++) {
        ok = bar_wait(&bar[i & 1], phase[i & 1]) && ok;
        phase[i & 1] ^= 1u;
        __syncthreads();   // every thread is past the previous step's reads
        if (i + 1 <= last_step) issue(i + 1, true, i + 2, true, i + 1);
#pragma unroll
        for (int h = 0; h < 2 * T_; h++) {
            const int p = i - h;
            const int lh = max(1, L0 + h);
            const int uh = min(nx - 2, P1 - 1 + 2 * T_ - 1 - h);
            if (p >= lh && p <= uh) {
                const int ring = 2 * T_ - 1 - h;
                const int color = h & 1;
                const int rj = TJ + 2 * ring, rk = TK + 2 * ring;
                const int rk2 = (rk + 1) / 2;
                T *wc = pslot(p);
                const T *wm = pslot(p - 1), *wp = pslot(p + 1);
                const S *ws = sslot(p);
                for (int jj = warp; jj < rj; jj += NW) {
                    const int gj = j0 - ring + jj;
                    if (gj < 1 || gj > ny - 2) continue;
                    const int kstart = k0 - ring;
                    const int kpar = ((p + gj + kstart) & 1) ^ color;
                    const int sj = gj - j0 + R;
                    for (int kk = lane; kk < rk2; kk += 32) {
                        const int gk = kstart + kpar + 2 * kk;
                        if (gk >= kstart + rk || gk < 1 || gk > nz - 2) continue;
                        const int s = sj * SK + (gk - k0 + R);
                        T r;
                        const T old = wc[s];
                        const T nv = cf.update(old, wm[s], wp[s], wc[s - SK], wc[s + SK], wc[s - 1], wc[s + 1],
                                               (T)ws[s], r);
                        wc[s] = nv;
                        if (sizeof(T) == 8) rmaxd[h >> 1] = tmax(rmaxd[h >> 1], (double)r);
                        else rmax[h >> 1] = tmax(rmax[h >> 1], (float)r);
                    }
                }
            }
            __syncthreads();
        }
        const int po = i - 2 * T_ + 1;
        if (po >= P0 && po < P1) {
            const T *w = pslot(po);
            for (int jj = warp; jj < TJ; jj += NW) {
                const int gj = j0 + jj;
                if (gj < 1 || gj > ny - 2) continue;
                for (int kk = lane; kk < TK; kk += 32) {
                    const int gk = k0 + kk;
                    if (gk >= 1 && gk <= nz - 2) out[po * sI + gj * sJ + gk] = w[(jj + R) * SK + kk + R];
                }
            }
        }
    }
#pragma unroll
    for (int l = 0; l < T_; l++) {
        double v = (sizeof(T) == 8) ? rmaxd[l] : (double)rmax[l];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = tmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (lane == 0 && v > 0.0) atomic_max_nonneg((unsigned long long *)(res + iter0 + l), v);
    }
    if (!ok && tid == 0) atomicExch(&sc->err, HC_ERR_TIMEOUT);
}

}  // namespace wtma
}  // namespace hc
