// hydro_fp32_pk.cuh -- the FP32 fused hydro kernel in packed FP32x2 arithmetic.
//
// The single-plane kernel (hydro_fp32_tma.cuh) is bound by instruction issue:
// three HLLC solves, two primitive recoveries, the update, floors and the
// gravity source cost about 600 thread instructions per cell against 48 bytes
// of HBM traffic.  Here each thread owns one (j, k) column of a 32(k) x 8(j)
// tile over TWO consecutive planes (i, i+1) per step, and every per-cell
// quantity is a float2 holding the two planes' values.  Each add, multiply
// and fused multiply-add then acts on both cells in one sm_100 packed
// instruction (add/sub/mul/fma .f32x2); only selects, comparisons, min/max
// and the special-function reciprocals and square roots stay per cell.
//
// Layout and data movement:
//   * One 4D cp.async.bulk.tensor per step fetches a plane PAIR of all five
//     conserved fields (box 40(k) x 10(j) x 2(i) x 5, k from k0-4 so every
//     copy starts on a 16-byte boundary) into a double buffer, one pair
//     ahead, completing on an mbarrier with bounded waits.
//   * The y and z faces of a pair are natural pairs: (plane i, plane i+1) at
//     the same (j, k).  Cell records live in shared memory as six float4
//     planes of structure-of-arrays (conflict-free 16-byte accesses, each
//     carrying both planes of two quantities); face fluxes likewise.
//   * The x faces i+1/2 and i+3/2 of the pair are the packed HLLC of the
//     current pair (i, i+1) against the shifted pair (i+1, i+2), all in
//     registers; the face i-1/2 is the previous step's upper face.
// Per cell the arithmetic is that of the single-plane kernel (the reference's
// hydro_solver_3d.c:162-416 and :729-771, the gravity source of :597-631, in
// FP32 with hardware reciprocal and square root); the HLLC star flux is
// written as F_K + S_K (U*_K - U_K) expanded per component (same terms,
// different FP32 rounding order).
#pragma once
#include <cuda.h>

#include "hc_internal.cuh"
#include "hc_math.cuh"
#include "mbar.cuh"

namespace hc {
namespace pk {

constexpr int TK = 32, TJ = 8, NT = TK * TJ;
constexpr int RK = TK + 8;          // raw tile: k0-4 .. k0+TK+3
constexpr int RJ = TJ + 2;          // raw tile: j0-1 .. j0+TJ
constexpr int RAWF = RJ * RK;       // floats per field per plane
constexpr int RAWB = 5 * 2 * RAWF;  // floats per plane-pair buffer
constexpr unsigned RAW_BYTES = (unsigned)RAWB * 4u;
constexpr int SK = TK + 2, SJ = TJ + 2, NS = SK * SJ;
constexpr int NFY = (TJ + 1) * TK, NFZ = TJ * (TK + 1);
constexpr int NH = 2 * SK + 2 * TJ;   // halo records around the tile

// shared-memory layout (bytes)
constexpr size_t OFF_RAW = 0;
constexpr size_t OFF_P = OFF_RAW + 2 * (size_t)RAW_BYTES;
constexpr size_t OFF_FYA = OFF_P + 6 * (size_t)NS * 16;
constexpr size_t OFF_FYB = OFF_FYA + (size_t)NFY * 16;
constexpr size_t OFF_FYE = OFF_FYB + (size_t)NFY * 16;
constexpr size_t OFF_FZA = OFF_FYE + (size_t)NFY * 8;
constexpr size_t OFF_FZB = OFF_FZA + (size_t)NFZ * 16;
constexpr size_t OFF_FZE = OFF_FZB + (size_t)NFZ * 16;
constexpr size_t OFF_BAR = (OFF_FZE + (size_t)NFZ * 8 + 15) / 16 * 16;
constexpr size_t OFF_WMAX = OFF_BAR + 16;
constexpr size_t SMEM = OFF_WMAX + (NT / 32) * 4;

// ---------------------------------------------------------------- packed arithmetic
// sm_100 packed FP32x2 operations (CUDA's __fadd2_rn / __fmul2_rn / __ffma2_rn
// intrinsics, which leave the register pairing to the compiler); a - b is
// the fused b * (-1) + a, rounded once like a subtraction.
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 sp2(float s) { return make_float2(s, s); }
__device__ __forceinline__ float2 max2(float2 a, float2 b) { return make_float2(tmax(a.x, b.x), tmax(a.y, b.y)); }
__device__ __forceinline__ float2 min2(float2 a, float2 b) { return make_float2(tmin(a.x, b.x), tmin(a.y, b.y)); }
__device__ __forceinline__ float2 maxs2(float2 a, float s) { return make_float2(tmax(a.x, s), tmax(a.y, s)); }
__device__ __forceinline__ float2 rcp2(float2 a) { return make_float2(1.0f / a.x, 1.0f / a.y); }
__device__ __forceinline__ float2 sqrt2(float2 a) { return make_float2(sqrtf(a.x), sqrtf(a.y)); }
__device__ __forceinline__ float2 div2(float2 a, float2 b)
{
    return make_float2(__fdividef(a.x, b.x), __fdividef(a.y, b.y));
}
__device__ __forceinline__ float2 sel2(bool px, bool py, float2 a, float2 b)
{
    return make_float2(px ? a.x : b.x, py ? a.y : b.y);
}
// (a.y, b.x): the pair shifted by one plane
__device__ __forceinline__ float2 shf(float2 a, float2 b) { return make_float2(a.y, b.x); }

// ---------------------------------------------------------------- records and fluxes
// One cell in two planes: raw conserved state, primitives, sound speed,
// floored density and its reciprocal.
struct R2 {
    float2 d, mx, my, mz, E, u, v, w, p, c, dh, inv;
};
struct F2 {
    float2 d, m0, m1, m2, e;
};

struct Consts {
    float2 gm1, rgm1, gam, half;
};

__device__ __forceinline__ R2 make_rec2(float2 d, float2 mx, float2 my, float2 mz, float2 E, const Consts &K)
{
    R2 r;
    r.d = d; r.mx = mx; r.my = my; r.mz = mz; r.E = E;
    r.dh = maxs2(d, (float)HC_RHO_FLOOR);
    r.inv = rcp2(r.dh);
    r.u = mul2(mx, r.inv);
    r.v = mul2(my, r.inv);
    r.w = mul2(mz, r.inv);
    float2 s = mul2(r.u, r.u);
    s = fma2(r.v, r.v, s);
    s = fma2(r.w, r.w, s);
    const float2 kin = mul2(mul2(K.half, r.dh), s);
    r.p = maxs2(mul2(K.gm1, sub2(E, kin)), (float)HC_P_FLOOR);
    r.c = sqrt2(mul2(mul2(K.gam, r.p), r.inv));
    return r;
}

// record of the cell at offset o of a raw plane-pair buffer (field f, plane q
// at f*2*RAWF + q*RAWF)
__device__ __forceinline__ R2 rec_raw(const float *r, int o, const Consts &K)
{
    return make_rec2(make_float2(r[o], r[RAWF + o]), make_float2(r[2 * RAWF + o], r[3 * RAWF + o]),
                     make_float2(r[4 * RAWF + o], r[5 * RAWF + o]), make_float2(r[6 * RAWF + o], r[7 * RAWF + o]),
                     make_float2(r[8 * RAWF + o], r[9 * RAWF + o]), K);
}

// shared records: six float4 planes of NS each
__device__ __forceinline__ void put_rec(float4 *P, int s, const R2 &r)
{
    P[s] = make_float4(r.d.x, r.d.y, r.mx.x, r.mx.y);
    P[NS + s] = make_float4(r.my.x, r.my.y, r.mz.x, r.mz.y);
    P[2 * NS + s] = make_float4(r.E.x, r.E.y, r.u.x, r.u.y);
    P[3 * NS + s] = make_float4(r.v.x, r.v.y, r.w.x, r.w.y);
    P[4 * NS + s] = make_float4(r.p.x, r.p.y, r.c.x, r.c.y);
    P[5 * NS + s] = make_float4(r.dh.x, r.dh.y, r.inv.x, r.inv.y);
}
__device__ __forceinline__ R2 get_rec(const float4 *P, int s)
{
    R2 r;
    float4 t = P[s];
    r.d = make_float2(t.x, t.y); r.mx = make_float2(t.z, t.w);
    t = P[NS + s];
    r.my = make_float2(t.x, t.y); r.mz = make_float2(t.z, t.w);
    t = P[2 * NS + s];
    r.E = make_float2(t.x, t.y); r.u = make_float2(t.z, t.w);
    t = P[3 * NS + s];
    r.v = make_float2(t.x, t.y); r.w = make_float2(t.z, t.w);
    t = P[4 * NS + s];
    r.p = make_float2(t.x, t.y); r.c = make_float2(t.z, t.w);
    t = P[5 * NS + s];
    r.dh = make_float2(t.x, t.y); r.inv = make_float2(t.z, t.w);
    return r;
}
__device__ __forceinline__ void put_flux(float4 *A, float4 *B, float2 *E, int s, const F2 &f)
{
    A[s] = make_float4(f.d.x, f.d.y, f.m0.x, f.m0.y);
    B[s] = make_float4(f.m1.x, f.m1.y, f.m2.x, f.m2.y);
    E[s] = f.e;
}
__device__ __forceinline__ F2 get_flux(const float4 *A, const float4 *B, const float2 *E, int s)
{
    F2 f;
    float4 t = A[s];
    f.d = make_float2(t.x, t.y); f.m0 = make_float2(t.z, t.w);
    t = B[s];
    f.m1 = make_float2(t.x, t.y); f.m2 = make_float2(t.z, t.w);
    f.e = E[s];
    return f;
}

// the same cell one plane further: (a.y, b.x) of every quantity
__device__ __forceinline__ R2 shift(const R2 &a, const R2 &b)
{
    R2 r;
    r.d = shf(a.d, b.d); r.mx = shf(a.mx, b.mx); r.my = shf(a.my, b.my); r.mz = shf(a.mz, b.mz);
    r.E = shf(a.E, b.E); r.u = shf(a.u, b.u); r.v = shf(a.v, b.v); r.w = shf(a.w, b.w);
    r.p = shf(a.p, b.p); r.c = shf(a.c, b.c); r.dh = shf(a.dh, b.dh); r.inv = shf(a.inv, b.inv);
    return r;
}

template <int A> __device__ __forceinline__ float2 velA(const R2 &r) { return A == 0 ? r.u : (A == 1 ? r.v : r.w); }

// HLLC flux along axis A for two faces at once (hydro_solver_3d.c:239-416):
// Davis speeds, contact speed S*, upwind side K, F = F_K + S_K (U*_K - U_K)
// in the star region and F = F_K outside it.
template <int A>
__device__ __forceinline__ F2 hllc2(const R2 &L, const R2 &R)
{
    const float2 uL = velA<A>(L), uR = velA<A>(R);
    const float2 sL = min2(sub2(uL, L.c), sub2(uR, R.c));
    const float2 sR = max2(add2(uL, L.c), add2(uR, R.c));
    const float2 gL = sub2(sL, uL), gR = sub2(sR, uR);         // S - u
    const float2 qL = mul2(L.dh, gL), qR = mul2(R.dh, gR);     // rho (S - u)
    float2 num = fma2(qL, uL, sub2(R.p, L.p));
    num = sub2(num, mul2(qR, uR));
    const float2 ss = div2(num, sub2(qL, qR));
    // upwind side and region, per face
    const bool supl_x = sL.x >= 0.f, supl_y = sL.y >= 0.f;
    const bool supr_x = !supl_x && sR.x <= 0.f, supr_y = !supl_y && sR.y <= 0.f;
    const bool lx = supl_x || (!supr_x && ss.x >= 0.f), ly = supl_y || (!supr_y && ss.y >= 0.f);
    const bool starx = !(supl_x || supr_x), stary = !(supl_y || supr_y);
    const float2 sK = sel2(lx, ly, sL, sR), uK = sel2(lx, ly, uL, uR);
    const float2 gK = sel2(lx, ly, gL, gR), qK = sel2(lx, ly, qL, qR);
    const float2 pK = sel2(lx, ly, L.p, R.p), iK = sel2(lx, ly, L.inv, R.inv);
    const float2 EK = sel2(lx, ly, L.E, R.E), dK = sel2(lx, ly, L.d, R.d);
    const float2 mxK = sel2(lx, ly, L.mx, R.mx), myK = sel2(lx, ly, L.my, R.my), mzK = sel2(lx, ly, L.mz, R.mz);
    const float2 vxK = sel2(lx, ly, L.u, R.u), vyK = sel2(lx, ly, L.v, R.v), vzK = sel2(lx, ly, L.w, R.w);
    // star-region weight: S_K inside, 0 outside (then F = F_K exactly)
    const float2 zero = sp2(0.f);
    const float2 sKw = sel2(starx, stary, sK, zero);
    const float2 a = sel2(starx, stary, mul2(sK, div2(qK, sub2(sK, ss))), zero);   // S_K rho*_K
    const float2 uw = sub2(uK, sKw);
    F2 f;
    const float2 mA = A == 0 ? mxK : (A == 1 ? myK : mzK);
    f.d = sub2(add2(mA, a), mul2(sKw, dK));
    const float2 fA = fma2(mA, uw, fma2(a, ss, pK));
    f.m0 = A == 0 ? fA : fma2(mxK, uw, mul2(a, vxK));
    f.m1 = A == 1 ? fA : fma2(myK, uw, mul2(a, vyK));
    f.m2 = A == 2 ? fA : fma2(mzK, uw, mul2(a, vzK));
    // E*/rho*: E_K/rho_K + (S* - u_K)(S* + p_K / (rho_K (S_K - u_K)))
    const float2 t1 = add2(ss, div2(mul2(pK, iK), gK));
    const float2 t3 = fma2(EK, iK, mul2(sub2(ss, uK), t1));
    f.e = fma2(a, t3, fma2(EK, uw, mul2(pK, uK)));
    return f;
}

// One 4D bulk tensor load of a plane pair: box {RK, RJ, 2, 5} at (k, j, i, 0).
__device__ __forceinline__ void tma_pair(const CUtensorMap *tm, float *dst, uint64_t *bar, int k, int j, int i)
{
    asm volatile("cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_addr(dst)),
                 "l"(reinterpret_cast<uint64_t>(tm)), "r"(k), "r"(j), "r"(i), "r"(0), "r"(smem_addr(bar))
                 : "memory");
}

__global__ void __launch_bounds__(NT, 2)
interior_pk_kernel(const __grid_constant__ CUtensorMap tmap, HydroArgs a, int ilen)
{
    extern __shared__ __align__(128) unsigned char smem[];
    float *raw0 = reinterpret_cast<float *>(smem + OFF_RAW);
    float4 *P = reinterpret_cast<float4 *>(smem + OFF_P);
    float4 *FYa = reinterpret_cast<float4 *>(smem + OFF_FYA), *FYb = reinterpret_cast<float4 *>(smem + OFF_FYB);
    float2 *FYe = reinterpret_cast<float2 *>(smem + OFF_FYE);
    float4 *FZa = reinterpret_cast<float4 *>(smem + OFF_FZA), *FZb = reinterpret_cast<float4 *>(smem + OFF_FZB);
    float2 *FZe = reinterpret_cast<float2 *>(smem + OFF_FZE);
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + OFF_BAR);
    float *wmax = reinterpret_cast<float *>(smem + OFF_WMAX);

    const int nx = a.g.nx, ny = a.g.ny, nz = a.g.nz;
    const long long sI = (long long)ny * nz, sJ = nz;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TK + tx;
    const int k0 = blockIdx.x * TK, j0 = blockIdx.y * TJ;
    const int k = k0 + tx, j = j0 + ty;
    const int ib = 1 + blockIdx.z * ilen;
    const int ie = min(nx - 1, ib + ilen);   // exclusive
    if (ib >= ie) return;
    float *const *qout = reinterpret_cast<float *const *>(a.qout);
    Consts K;
    K.gm1 = sp2((float)(a.gamma - 1.0));
    K.rgm1 = sp2((float)(1.0 / (a.gamma - 1.0)));
    K.gam = sp2((float)a.gamma);
    K.half = sp2(0.5f);
    const float dt = (float)a.sc->dt;
    const float2 ndtdx = sp2(-dt / (float)a.g.dx), ndtdy = sp2(-dt / (float)a.g.dy), ndtdz = sp2(-dt / (float)a.g.dz);
    const float2 dt2 = sp2(dt);
    const float2 hx = sp2((float)(0.5 / a.g.dx));
    const float hy = (float)(0.5 / a.g.dy), hz = (float)(0.5 / a.g.dz);
    const bool own_int = (j >= 1) && (j <= ny - 2) && (k >= 1) && (k <= nz - 2);
    const int own_s = (ty + 1) * SK + tx + 1;          // this thread's record slot
    const int own_o = (ty + 1) * RK + tx + 4;          // its offset in a raw plane

    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    unsigned use[2] = { 0u, 0u };
    bool ok = true;
    // plane pair q = planes (ib + 2q, ib + 2q + 1), q >= -1, in buffer (q + 1) & 1
    auto buf = [&](int q) { return raw0 + ((q + 1) & 1) * RAWB; };
    auto issue = [&](int q) {
        if (tid == 0) {
            const int b = (q + 1) & 1;
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_expect_tx(&bar[b], RAW_BYTES);
            tma_pair(&tmap, raw0 + b * RAWB, &bar[b], k0 - 4, j0 - 1, ib + 2 * q);
        }
    };
    auto wait = [&](int q) {
        const int b = (q + 1) & 1;
        ok = mbar_wait(&bar[b], use[b] & 1) && ok;
        use[b]++;
    };
    // the NH halo records are formed by threads HB .. HB+NH-1 (warps 3-5),
    // the faces behind the tile by warps 6 and 7: the extra work of a step
    // spread over warps that the barriers would otherwise hold up
    constexpr int HB = 96;
    static_assert(HB + NH <= 6 * 32, "halo records fit warps 3-5");
    auto build_halo = [&](const float *r) {
        const int h = tid - HB;
        if (h >= 0 && h < NH) {
            int sj, sk;
            if (h < 2 * SK) {
                sj = (h < SK) ? 0 : SJ - 1;
                sk = h % SK;
            } else {
                const int q = h - 2 * SK;
                sj = 1 + (q >> 1);
                sk = (q & 1) ? SK - 1 : 0;
            }
            put_rec(P, sj * SK + sk, rec_raw(r, sj * RK + sk + 3, K));
        }
    };

    // prologue: the face below the chunk, then the first pair's records
    issue(-1);
    issue(0);
    wait(-1);
    const R2 Pm = rec_raw(buf(-1), own_o, K);
    wait(0);
    R2 C = rec_raw(buf(0), own_o, K);
    float ftop[5];   // the face ib - 1/2 (.y of the prologue's pair of faces)
    {
        const F2 f = hllc2<0>(Pm, shift(Pm, C));
        ftop[0] = f.d.y; ftop[1] = f.m0.y; ftop[2] = f.m1.y; ftop[3] = f.m2.y; ftop[4] = f.e.y;
    }
    put_rec(P, own_s, C);
    build_halo(buf(0));
    // gravity: the potential of planes i-1 and i at (j, k), carried
    const double *ph = a.phig;
    const bool gin = a.gravity && own_int;
    const long long c0 = (long long)j * sJ + k;
    double phm = 0.0, ph0 = 0.0;
    if (gin) {
        phm = __ldg(ph + (long long)(ib - 1) * sI + c0);
        ph0 = __ldg(ph + (long long)ib * sI + c0);
    }
    __syncthreads();
    issue(1);    // into the buffer of pair -1, consumed

    float smax = 0.f;
    int s = 0;
    for (int i = ib; i < ie; i += 2, s++) {
        if (i + 2 < ie) issue(s + 2);          // into the buffer of pair s, consumed
        wait(s + 1);
        const float *rn = buf(s + 1);
        const R2 N = rec_raw(rn, own_o, K);
        const bool v1 = i + 1 < ie;            // the pair's second plane is in this chunk
        // x faces i+1/2 (.x) and i+3/2 (.y)
        const F2 fx = hllc2<0>(C, shift(C, N));
        // y and z faces ahead of the cell, and the CTA's faces behind the tile
        put_flux(FYa, FYb, FYe, (ty + 1) * TK + tx, hllc2<1>(C, get_rec(P, (ty + 2) * SK + tx + 1)));
        put_flux(FZa, FZb, FZe, ty * (TK + 1) + tx + 1, hllc2<2>(C, get_rec(P, own_s + 1)));
        if (ty == TJ - 1) {          // the y faces below the tile's first row
            put_flux(FYa, FYb, FYe, tx, hllc2<1>(get_rec(P, tx + 1), get_rec(P, SK + tx + 1)));
        } else if (ty == TJ - 2 && tx < TJ) {   // the z faces before the tile's first column
            put_flux(FZa, FZb, FZe, tx * (TK + 1),
                     hllc2<2>(get_rec(P, (tx + 1) * SK), get_rec(P, (tx + 1) * SK + 1)));
        }
        // the potential of planes i+1 (and i+2), the y, z neighbours of i (and i+1);
        // plane i+2 exists whenever plane i+1 is in the chunk (i+2 <= ie <= nx-1)
        double php = 0.0, ph2 = 0.0, pym0 = 0.0, pyp0 = 0.0, pzm0 = 0.0, pzp0 = 0.0;
        double pym1 = 0.0, pyp1 = 0.0, pzm1 = 0.0, pzp1 = 0.0;
        const long long cc = (long long)i * sI + c0;
        if (gin) {
            php = __ldg(ph + cc + sI);
            pym0 = __ldg(ph + cc - sJ);
            pyp0 = __ldg(ph + cc + sJ);
            pzm0 = __ldg(ph + cc - 1);
            pzp0 = __ldg(ph + cc + 1);
            if (v1) {
                ph2 = __ldg(ph + cc + 2 * sI);
                pym1 = __ldg(ph + cc + sI - sJ);
                pyp1 = __ldg(ph + cc + sI + sJ);
                pzm1 = __ldg(ph + cc + sI - 1);
                pzp1 = __ldg(ph + cc + sI + 1);
            }
        }
        __syncthreads();
        // the next pair's records: this thread's own, and the halo ring
        put_rec(P, own_s, N);
        build_halo(rn);
        if (own_int) {
            const F2 ym = get_flux(FYa, FYb, FYe, ty * TK + tx);
            const F2 yp = get_flux(FYa, FYb, FYe, (ty + 1) * TK + tx);
            const F2 zm = get_flux(FZa, FZb, FZe, ty * (TK + 1) + tx);
            const F2 zp = get_flux(FZa, FZb, FZe, ty * (TK + 1) + tx + 1);
            // faces below the pair: (i-1/2, i+1/2)
            const float2 xd = make_float2(ftop[0], fx.d.x), x0 = make_float2(ftop[1], fx.m0.x);
            const float2 x1 = make_float2(ftop[2], fx.m1.x), x2 = make_float2(ftop[3], fx.m2.x);
            const float2 xe = make_float2(ftop[4], fx.e.x);
            auto upd = [&](float2 q, float2 fxp, float2 fxm, float2 fyp, float2 fym, float2 fzp, float2 fzm) {
                float2 t = mul2(ndtdx, sub2(fxp, fxm));
                t = fma2(ndtdy, sub2(fyp, fym), t);
                t = fma2(ndtdz, sub2(fzp, fzm), t);
                return add2(q, t);
            };
            float2 d = upd(C.d, fx.d, xd, yp.d, ym.d, zp.d, zm.d);
            float2 mx = upd(C.mx, fx.m0, x0, yp.m0, ym.m0, zp.m0, zm.m0);
            float2 my = upd(C.my, fx.m1, x1, yp.m1, ym.m1, zp.m1, zm.m1);
            float2 mz = upd(C.mz, fx.m2, x2, yp.m2, ym.m2, zp.m2, zm.m2);
            float2 E = upd(C.E, fx.e, xe, yp.e, ym.e, zp.e, zm.e);
            // floors: rho floor then the prim round trip (hydro_solver_3d.c:765-768)
            d = maxs2(d, (float)HC_RHO_FLOOR);
            const float2 inv = rcp2(d);
            float2 u = mul2(mx, inv), v = mul2(my, inv), w = mul2(mz, inv);
            float2 q2 = fma2(w, w, fma2(v, v, mul2(u, u)));
            float2 kin = mul2(mul2(K.half, d), q2);
            float2 p = maxs2(mul2(K.gm1, sub2(E, kin)), (float)HC_P_FLOOR);
            mx = mul2(d, u);
            my = mul2(d, v);
            mz = mul2(d, w);
            E = fma2(p, K.rgm1, kin);
            if (a.gravity) {
                // g = -grad(phi) from the FP64 potential (gravity_solver_3d.c:832-834)
                const float2 ax = mul2(make_float2((float)(phm - php), (float)(ph0 - ph2)), hx);
                const float2 ay = make_float2((float)(pym0 - pyp0) * hy, (float)(pym1 - pyp1) * hy);
                const float2 az = make_float2((float)(pzm0 - pzp0) * hz, (float)(pzm1 - pzp1) * hz);
                // apply_gravity_source_terms (:612-628): pre-source velocities
                const float2 work = mul2(d, fma2(w, az, fma2(v, ay, mul2(u, ax))));
                const float2 dtd = mul2(dt2, d);
                mx = fma2(dtd, ax, mx);
                my = fma2(dtd, ay, my);
                mz = fma2(dtd, az, mz);
                E = fma2(dt2, work, E);
                u = mul2(mx, inv);
                v = mul2(my, inv);
                w = mul2(mz, inv);
                q2 = fma2(w, w, fma2(v, v, mul2(u, u)));
                kin = mul2(mul2(K.half, d), q2);
                p = maxs2(mul2(K.gm1, sub2(E, kin)), (float)HC_P_FLOOR);
            }
            const long long c = (long long)i * sI + c0;
            qout[0][c] = d.x; qout[1][c] = mx.x; qout[2][c] = my.x; qout[3][c] = mz.x; qout[4][c] = E.x;
            const float2 cs = sqrt2(mul2(mul2(K.gam, p), inv));
            smax = tmax(smax, tmax(fabsf(u.x), tmax(fabsf(v.x), fabsf(w.x))) + cs.x);
            if (v1) {
                qout[0][c + sI] = d.y; qout[1][c + sI] = mx.y; qout[2][c + sI] = my.y; qout[3][c + sI] = mz.y;
                qout[4][c + sI] = E.y;
                smax = tmax(smax, tmax(fabsf(u.y), tmax(fabsf(v.y), fabsf(w.y))) + cs.y);
            }
        }
        __syncthreads();
        ftop[0] = fx.d.y; ftop[1] = fx.m0.y; ftop[2] = fx.m1.y; ftop[3] = fx.m2.y; ftop[4] = fx.e.y;
        C = N;
        phm = php;
        ph0 = ph2;
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

}  // namespace pk
}  // namespace hc
