// hydro_fp32_tma.cuh -- the FP32 fused hydro kernel with TMA-staged planes.
//
// A CTA owns a 32(k) x 8(j) column of cells and streams along i.  Plane
// tiles with a one-cell halo in j and a 4-cell halo in k (so every bulk copy
// starts on a 16-byte boundary) are fetched by one 4D cp.async.bulk.tensor per
// plane -- all five conserved fields at once -- into a double buffer, one
// plane ahead, completing on an mbarrier.  Per plane each cell's primitives
// are formed once into 48-byte shared records; each thread forms the x face
// ahead of its cell (carried in registers to the next plane), the y and z
// faces ahead of its cell (shared), and the CTA's edge warps the faces behind
// the tile.  The update, density/pressure floors, gravity source (g from the
// FP64 potential), and the next step's CFL max follow in registers.
//
// Arithmetic per hydro_solver_3d.c:162-416, in FP32 with hardware reciprocal
// and square root (this file is compiled with --use_fast_math).
#pragma once
#include <cuda.h>

#include "hc_internal.cuh"
#include "hc_math.cuh"
#include "mbar.cuh"

namespace hc {
namespace tma32 {

constexpr int TK = 32, TJ = 8, NT = TK * TJ;
constexpr int RK = TK + 8;          // raw tile: k0-4 .. k0+TK+3
constexpr int RJ = TJ + 2;          // raw tile: j0-1 .. j0+TJ
constexpr int RAWF = RJ * RK;       // floats per field per plane
constexpr int SK = TK + 2, SJ = TJ + 2, NS = SK * SJ;
constexpr unsigned RAW_BYTES = 5u * RAWF * 4u;
constexpr int RAWP = ((5 * RAWF + 31) / 32) * 32;   // buffer stride: 128-byte aligned

struct __align__(16) Rec {
    float4 a;   // rho, mx, my, mz   (raw conserved)
    float4 b;   // E, u, v, w
    float4 c;   // p, cs, rho_hat, 1/rho_hat
};
struct Flux { float d, m0, m1, m2, e; };

__device__ __forceinline__ Rec make_rec(float d, float mx, float my, float mz, float E, float gm1,
                                        float gam)
{
    Rec r;
    float dh = tmax(d, (float)HC_RHO_FLOOR);
    float inv = 1.0f / dh;
    float u = mx * inv, v = my * inv, w = mz * inv;
    float kin = 0.5f * dh * (u * u + v * v + w * w);
    float p = tmax(gm1 * (E - kin), (float)HC_P_FLOOR);
    float cs = sqrtf(gam * p * inv);
    r.a = make_float4(d, mx, my, mz);
    r.b = make_float4(E, u, v, w);
    r.c = make_float4(p, cs, dh, inv);
    return r;
}

template <int A> __device__ __forceinline__ float vel(const Rec &r) { return A == 0 ? r.b.y : (A == 1 ? r.b.z : r.b.w); }

// HLLC flux along axis A (hydro_solver_3d.c:239-300), branch-free side choice
template <int A>
__device__ __forceinline__ Flux hllc(const Rec &L, const Rec &R)
{
    const float uL = vel<A>(L), uR = vel<A>(R);
    const float dL = L.c.z, dR = R.c.z, pL = L.c.x, pR = R.c.x;
    const float sL = tmin(uL - L.c.y, uR - R.c.y);
    const float sR = tmax(uL + L.c.y, uR + R.c.y);
    const float num = pR - pL + dL * uL * (sL - uL) - dR * uR * (sR - uR);
    const float den = dL * (sL - uL) - dR * (sR - uR);
    const float ss = __fdividef(num, den);
    const bool supl = sL >= 0.f;
    const bool supr = !supl && (sR <= 0.f);
    const bool left = supl || (!supr && ss >= 0.f);
    // Select the upwind side value by value: a reference bound to one of two
    // register-resident records (the x faces) gave wrong conserved
    // components on sm_100a, selects do not.
    const float sK = left ? sL : sR;
    const float uK = left ? uL : uR, dK = left ? dL : dR, pK = left ? pL : pR;
    const float iK = left ? L.c.w : R.c.w, EK = left ? L.b.x : R.b.x;
    const float qd = left ? L.a.x : R.a.x, q0 = left ? L.a.y : R.a.y;
    const float q1 = left ? L.a.z : R.a.z, q2 = left ? L.a.w : R.a.w;
    const float v0 = left ? L.b.y : R.b.y, v1 = left ? L.b.z : R.b.z, v2 = left ? L.b.w : R.b.w;
    // F(U_K)
    Flux f;
    f.d = A == 0 ? q0 : (A == 1 ? q1 : q2);
    f.m0 = q0 * uK + (A == 0 ? pK : 0.f);
    f.m1 = q1 * uK + (A == 1 ? pK : 0.f);
    f.m2 = q2 * uK + (A == 2 ? pK : 0.f);
    f.e = (EK + pK) * uK;
    if (!(supl || supr)) {
        const float fac = __fdividef(sK - uK, sK - ss);
        const float sd = dK * fac;
        const float se = sd * (EK * iK + (ss - uK) * (ss + __fdividef(pK * iK, sK - uK)));
        f.d += sK * (sd - qd);
        f.m0 += sK * (sd * (A == 0 ? ss : v0) - q0);
        f.m1 += sK * (sd * (A == 1 ? ss : v1) - q1);
        f.m2 += sK * (sd * (A == 2 ? ss : v2) - q2);
        f.e += sK * (se - EK);
    }
    return f;
}

using hc::mbar_expect_tx;
using hc::mbar_init;
using hc::mbar_wait;
using hc::smem_addr;

// One 4D bulk tensor load: box {RK, RJ, 1, 5} at (k, j, i, 0).
__device__ __forceinline__ void tma_plane(const CUtensorMap *tm, float *dst, uint64_t *bar, int k, int j, int i)
{
    asm volatile("cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_addr(dst)),
                 "l"(reinterpret_cast<uint64_t>(tm)), "r"(k), "r"(j), "r"(i), "r"(0), "r"(smem_addr(bar))
                 : "memory");
}

__global__ void __launch_bounds__(NT, 4)
interior_tma_kernel(const __grid_constant__ CUtensorMap tmap, HydroArgs a, int ilen)
{
    __shared__ __align__(128) float raw[2][RAWP];
    __shared__ __align__(16) Rec P[NS];
    __shared__ Flux FY[(TJ + 1) * TK];
    __shared__ Flux FZ[TJ * (TK + 1)];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ float wmax[NT / 32];

    const int nx = a.g.nx, ny = a.g.ny, nz = a.g.nz;
    const long long sI = (long long)ny * nz, sJ = nz;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TK + tx;
    const int k0 = blockIdx.x * TK, j0 = blockIdx.y * TJ;
    const int k = k0 + tx, j = j0 + ty;
    const int ib = 1 + blockIdx.z * ilen;
    const int ie = min(nx - 1, ib + ilen);   // exclusive
    if (ib >= ie) return;
    float *const *qout = reinterpret_cast<float *const *>(a.qout);
    const float gam = (float)a.gamma, gm1 = (float)(a.gamma - 1.0);
    const float dt = (float)a.sc->dt;
    const float dtdx = dt / (float)a.g.dx, dtdy = dt / (float)a.g.dy, dtdz = dt / (float)a.g.dz;
    const float hx = (float)(0.5 / a.g.dx), hy = (float)(0.5 / a.g.dy), hz = (float)(0.5 / a.g.dz);
    const bool own_int = (j >= 1) && (j <= ny - 2) && (k >= 1) && (k <= nz - 2);

    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    unsigned use[2] = { 0u, 0u };
    bool ok = true;
    // plane p lives in raw[(p - ib + 1) & 1]
    auto issue = [&](int p) {
        if (tid == 0) {
            const int b = (p - ib + 1) & 1;
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_expect_tx(&bar[b], RAW_BYTES);
            tma_plane(&tmap, raw[b], &bar[b], k0 - 4, j0 - 1, p);
        }
    };
    auto wait = [&](int p) {
        const int b = (p - ib + 1) & 1;
        ok = mbar_wait(&bar[b], use[b] & 1) && ok;
        use[b]++;
    };
    auto rec_at = [&](const float *r, int rj, int rk) {
        const int o = rj * RK + rk;
        return make_rec(r[o], r[RAWF + o], r[2 * RAWF + o], r[3 * RAWF + o], r[4 * RAWF + o], gm1, gam);
    };
    auto build_P = [&](const float *r) {
        for (int s = tid; s < NS; s += NT) {
            const int sj = s / SK, sk = s - sj * SK;
            P[s] = rec_at(r, sj, sk + 3);
        }
    };
    // the NH = 2 SK + 2 TJ records around the tile: rows 0 and SJ-1, then the
    // first and last column of rows 1..TJ
    constexpr int NH = 2 * SK + 2 * TJ;
    auto build_halo = [&](const float *r) {
        if (tid < NH) {
            int sj, sk;
            if (tid < 2 * SK) {
                sj = (tid < SK) ? 0 : SJ - 1;
                sk = tid % SK;
            } else {
                const int q = tid - 2 * SK;
                sj = 1 + (q >> 1);
                sk = (q & 1) ? SK - 1 : 0;
            }
            P[sj * SK + sk] = rec_at(r, sj, sk + 3);
        }
    };

    issue(ib - 1);
    issue(ib);
    wait(ib - 1);
    Rec me_prev = rec_at(raw[0], ty + 1, tx + 4);
    wait(ib);
    build_P(raw[1]);
    __syncthreads();
    if (ib + 1 <= ie) issue(ib + 1);             // into the buffer of plane ib-1, consumed
    Rec me = P[(ty + 1) * SK + tx + 1];
    Flux fxm = hllc<0>(me_prev, me);

    float smax = 0.f;
    for (int i = ib; i < ie; i++) {
        if (i + 2 <= ie) issue(i + 2);           // buffer of plane i, already consumed
        wait(i + 1);
        const float *rn = raw[(i + 2 - ib) & 1];
        const Rec nx1 = rec_at(rn, ty + 1, tx + 4);
        const Flux fxp = hllc<0>(me, nx1);
        {
            const Rec &c0 = P[(ty + 1) * SK + tx + 1];
            FY[(ty + 1) * TK + tx] = hllc<1>(c0, P[(ty + 2) * SK + tx + 1]);
            FZ[ty * (TK + 1) + tx + 1] = hllc<2>(c0, P[(ty + 1) * SK + tx + 2]);
            if (ty == 0) {
                FY[tx] = hllc<1>(P[tx + 1], c0);
            } else if (ty == 1 && tx < TJ) {
                FZ[tx * (TK + 1)] = hllc<2>(P[(tx + 1) * SK], P[(tx + 1) * SK + 1]);
            }
        }
        __syncthreads();
        // plane i+1 for the next iteration: this thread's own record is nx1;
        // threads 0..NH-1 form the halo ring's records
        P[(ty + 1) * SK + tx + 1] = nx1;
        build_halo(rn);
        if (own_int && k < nz && j < ny) {
            const Flux &yp = FY[(ty + 1) * TK + tx], &ym = FY[ty * TK + tx];
            const Flux &zp = FZ[ty * (TK + 1) + tx + 1], &zm = FZ[ty * (TK + 1) + tx];
            float d = me.a.x + (-dtdx * (fxp.d - fxm.d) - dtdy * (yp.d - ym.d) - dtdz * (zp.d - zm.d));
            float mx = me.a.y + (-dtdx * (fxp.m0 - fxm.m0) - dtdy * (yp.m0 - ym.m0) - dtdz * (zp.m0 - zm.m0));
            float my = me.a.z + (-dtdx * (fxp.m1 - fxm.m1) - dtdy * (yp.m1 - ym.m1) - dtdz * (zp.m1 - zm.m1));
            float mz = me.a.w + (-dtdx * (fxp.m2 - fxm.m2) - dtdy * (yp.m2 - ym.m2) - dtdz * (zp.m2 - zm.m2));
            float E = me.b.x + (-dtdx * (fxp.e - fxm.e) - dtdy * (yp.e - ym.e) - dtdz * (zp.e - zm.e));
            // floors: rho floor then prim round trip (hydro_solver_3d.c:765-768)
            d = tmax(d, (float)HC_RHO_FLOOR);
            float inv = 1.0f / d;
            float u = mx * inv, v = my * inv, w = mz * inv;
            float kin = 0.5f * d * (u * u + v * v + w * w);
            float p = tmax(gm1 * (E - kin), (float)HC_P_FLOOR);
            mx = d * u; my = d * v; mz = d * w;
            E = p / gm1 + kin;
            const long long c = (long long)i * sI + (long long)j * sJ + k;
            if (a.gravity) {
                // g = -grad(phi) from the FP64 potential (gravity_solver_3d.c:832-834)
                const double *ph = a.phig;
                float ax = (float)(__ldg(ph + c - sI) - __ldg(ph + c + sI)) * hx;
                float ay = (float)(__ldg(ph + c - sJ) - __ldg(ph + c + sJ)) * hy;
                float az = (float)(__ldg(ph + c - 1) - __ldg(ph + c + 1)) * hz;
                // apply_gravity_source_terms (:612-628): pre-source velocities
                float work = d * (u * ax + v * ay + w * az);
                mx += dt * d * ax;
                my += dt * d * ay;
                mz += dt * d * az;
                E += dt * work;
                u = mx * inv; v = my * inv; w = mz * inv;
                kin = 0.5f * d * (u * u + v * v + w * w);
                p = tmax(gm1 * (E - kin), (float)HC_P_FLOOR);
            }
            qout[0][c] = d; qout[1][c] = mx; qout[2][c] = my; qout[3][c] = mz; qout[4][c] = E;
            const float cs = sqrtf(gam * p * inv);
            smax = tmax(smax, tmax(fabsf(u), tmax(fabsf(v), fabsf(w))) + cs);
        }
        __syncthreads();
        fxm = fxp;
        me = nx1;
    }
    // block max -> one atomic (next step's CFL)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) smax = tmax(smax, __shfl_xor_sync(0xffffffffu, smax, o));
    if ((tid & 31) == 0) wmax[tid >> 5] = smax;
    __syncthreads();
    if (tid == 0) {
        float m = 0.f;
        for (int t = 0; t < NT / 32; t++) m = tmax(m, wmax[t]);
        atomic_max_nonneg(reinterpret_cast<unsigned int *>(&a.sc->smax[a.step_parity ^ 1]), m);
        if (!ok) atomicExch(&a.sc->err, HC_ERR_TIMEOUT);
    }
}

}  // namespace tma32
}  // namespace hc
