// hc_math.cuh -- per-cell Euler / HLLC arithmetic shared by the FP64 and
// FP32 hydro kernels.
//
// The FP64 instantiation is compiled with -fmad=false and keeps the
// reference's operand order at every rounding point, so each value equals the
// reference C build bit for bit (hydro_solver_3d.c:162-416).  The FP32
// instantiation uses the same formulas in float.
#pragma once
#include <cuda_runtime.h>

#define HC_RHO_FLOOR 1.0e-5   // hydro_solver_3d.h:10
#define HC_P_FLOOR 1.0e-6     // hydro_solver_3d.h:11

namespace hc {

// MIN/MAX of the reference (second operand on ties and NaN), not fmin/fmax.
template <typename T> __device__ __forceinline__ T tmax(T a, T b) { return a > b ? a : b; }
template <typename T> __device__ __forceinline__ T tmin(T a, T b) { return a < b ? a : b; }

template <typename T> struct Cons { T d, m[3], e; };
template <typename T> struct Prim { T d, v[3], p; };

// cons_to_prim_3d, hydro_solver_3d.c:162-175
template <typename T>
__device__ __forceinline__ Prim<T> to_prim(const Cons<T> &q, T gm1)
{
    Prim<T> w;
    w.d = tmax(q.d, (T)HC_RHO_FLOOR);
    w.v[0] = q.m[0] / w.d;
    w.v[1] = q.m[1] / w.d;
    w.v[2] = q.m[2] / w.d;
    T kin = (T)0.5 * w.d * (w.v[0] * w.v[0] + w.v[1] * w.v[1] + w.v[2] * w.v[2]);
    w.p = tmax(gm1 * (q.e - kin), (T)HC_P_FLOOR);
    return w;
}

// prim_to_cons_3d, hydro_solver_3d.c:177-189
template <typename T>
__device__ __forceinline__ Cons<T> to_cons(const Prim<T> &w, T gm1)
{
    Cons<T> q;
    q.d = w.d;
    q.m[0] = w.d * w.v[0];
    q.m[1] = w.d * w.v[1];
    q.m[2] = w.d * w.v[2];
    T kin = (T)0.5 * w.d * (w.v[0] * w.v[0] + w.v[1] * w.v[1] + w.v[2] * w.v[2]);
    q.e = w.p / gm1 + kin;
    return q;
}

// sound_speed_3d, hydro_solver_3d.c:191-193
template <typename T>
__device__ __forceinline__ T csound(const Prim<T> &w, T gam) { return sqrt(gam * w.p / w.d); }

// compute_flux_{x,y,z}_3d, hydro_solver_3d.c:199-233, normal axis A.
template <int A, typename T>
__device__ __forceinline__ Cons<T> euler_flux(const Cons<T> &q, const Prim<T> &w)
{
    Cons<T> f;
    f.d = q.m[A];
#pragma unroll
    for (int c = 0; c < 3; c++) f.m[c] = (c == A) ? (q.m[c] * w.v[A] + w.p) : (q.m[c] * w.v[A]);
    f.e = (q.e + w.p) * w.v[A];
    return f;
}

// hllc_riemann_solver_{x,y,z}_3d, hydro_solver_3d.c:239-416, branch-free:
// the side (left/right) is selected first, then one flux and one star state
// are formed.  For the selected branch the operations are those of the
// reference, so the result is the same bits.
template <int A, typename T>
__device__ __forceinline__ Cons<T> hllc(const Cons<T> &qL, const Prim<T> &wL, T cL,
                                        const Cons<T> &qR, const Prim<T> &wR, T cR)
{
    T sL = tmin(wL.v[A] - cL, wR.v[A] - cR);
    T sR = tmax(wL.v[A] + cL, wR.v[A] + cR);
    T num = wR.p - wL.p + wL.d * wL.v[A] * (sL - wL.v[A]) - wR.d * wR.v[A] * (sR - wR.v[A]);
    T den = wL.d * (sL - wL.v[A]) - wR.d * (sR - wR.v[A]);
    T ss = num / den;
    const bool sup_l = sL >= (T)0;
    const bool sup_r = !sup_l && (sR <= (T)0);
    const bool left = sup_l || (!sup_r && ss >= (T)0);
    const bool star = !(sup_l || sup_r);

    Cons<T> qK;
    Prim<T> wK;
    qK.d = left ? qL.d : qR.d;
    qK.e = left ? qL.e : qR.e;
    wK.d = left ? wL.d : wR.d;
    wK.p = left ? wL.p : wR.p;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        qK.m[c] = left ? qL.m[c] : qR.m[c];
        wK.v[c] = left ? wL.v[c] : wR.v[c];
    }
    T sK = left ? sL : sR;

    Cons<T> f = euler_flux<A>(qK, wK);
    if (star) {
        T fac = (sK - wK.v[A]) / (sK - ss);
        T sd = wK.d * fac;
        T se = sd * (qK.e / wK.d + (ss - wK.v[A]) * (ss + wK.p / (wK.d * (sK - wK.v[A]))));
        f.d = f.d + sK * (sd - qK.d);
#pragma unroll
        for (int c = 0; c < 3; c++) {
            T sm = sd * ((c == A) ? ss : wK.v[c]);
            f.m[c] = f.m[c] + sK * (sm - qK.m[c]);
        }
        f.e = f.e + sK * (se - qK.e);
    }
    return f;
}

// Largest signal speed of a cell, as compute_dt_3d reduces it
// (hydro_solver_3d.c:429-439).
template <typename T>
__device__ __forceinline__ T signal_speed(const Prim<T> &w, T gam)
{
    T cs = csound(w, gam);
    T s = fabs(w.v[0]) + cs;
    s = tmax(s, fabs(w.v[1]) + cs);
    s = tmax(s, fabs(w.v[2]) + cs);
    return s;
}

// The gravity source for one cell, apply_gravity_source_terms
// (hydro_solver_3d.c:612-628): pre-source velocities, no density floor.
template <typename T, typename G>
__device__ __forceinline__ void gravity_source(Cons<T> &q, G ax, G ay, G az, T dt)
{
    T r = q.d;
    T u = q.m[0] / r, v = q.m[1] / r, w = q.m[2] / r;
    q.m[0] += dt * r * (T)ax;
    q.m[1] += dt * r * (T)ay;
    q.m[2] += dt * r * (T)az;
    T work = r * (u * (T)ax + v * (T)ay + w * (T)az);
    q.e += dt * work;
}

}  // namespace hc
