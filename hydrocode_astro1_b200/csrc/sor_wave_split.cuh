// sor_wave_split.cuh -- two red-black SOR iterations per pass over HBM on
// the colour-split layout (temporal blocking), FP32 correction sweeps.
//
// Layout: as sor_split.cuh (colour c at c*cs + (i*ny + j)*H + m).  A pass
// reads the iterate from P and writes the iterate two iterations later to Q
// (out of place: no CTA ever reads another CTA's partial results).  The four
// half-sweeps of the pass, h = 0 (red, iteration q0), 1 (black, q0),
// 2 (red, q0+1), 3 (black, q0+1), run as a wavefront along i: at step s,
// half-sweep h updates plane s - h, in increasing h.  Half-sweep h at plane p
// needs h-1 at planes p-1..p+1 (done at steps <= s, p+1 earlier in the same
// step) and its own colour at p from h-2 -- exactly the values of the
// sequential sweep, so the iterates are those of two plain iterations.
//
// A CTA owns rows [j0, j0+BJ) of planes [P0, P1) and whole rows in m (no z
// halo).  Half-sweep h also updates the 3-h rows and planes around them that
// later half-sweeps read (recomputed by the neighbouring CTAs too, with the
// same inputs, so the values are identical); the window holds BJ + 8 rows.
// Plane rings in shared memory: red/black iterate (7 slots each) and
// red/black source (5 slots each), filled with cp.async 16-byte copies two
// steps ahead of use (the slots written are dead by then: a red/black plane
// is last read 4 steps after its first use, a source plane 2 steps after).
// Final values of owned cells go from registers to Q.  The update norm of
// each iteration is the max over all updated cells (halo cells repeat values
// of other CTAs, so the max is that of the sequential sweep).
#pragma once
#include "hc_internal.cuh"
#include "hc_math.cuh"
#include "sor_split.cuh"

namespace hc {

constexpr int WV_NH = 4;              // half-sweeps per pass (two iterations)
constexpr int WV_D = 2;               // prefetch distance in steps
constexpr int WV_NE = 5 + WV_D;       // iterate ring slots per colour
constexpr int WV_NS = 3 + WV_D;       // source ring slots per colour
constexpr int WV_THREADS = 512;

__device__ __forceinline__ void wv_cp16(float *smem, const float *gmem)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void wv_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void wv_wait_prev() { asm volatile("cp.async.wait_group %0;" ::"n"(WV_D - 1) : "memory"); }
__device__ __forceinline__ void wv_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
__device__ __forceinline__ int wv_mod(int a, int n) { return ((a % n) + n) % n; }

// dynamic shared memory of one CTA for window rows NR and row length H
inline size_t wave_split_smem(int NR, int H) { return (size_t)(2 * WV_NE + 2 * WV_NS) * NR * H * sizeof(float); }

__global__ void __launch_bounds__(WV_THREADS, 1)
sor_wave_split_kernel(const float *__restrict__ P, float *__restrict__ Q, const float *__restrict__ R, Split sp,
                      SorCoef<float> cf, int BJ, int L, double *res, int iter0, double thresh, DevScalars *sc)
{
    extern __shared__ __align__(16) float wsm[];
    __shared__ float wred[2][WV_THREADS / 32];
    if (*(volatile int *)&sc->done) return;
    if (iter0 > 0) {
        const double prev = __longlong_as_double(*reinterpret_cast<const volatile long long *>(res + iter0 - 1));
        if (prev < thresh) {
            if (threadIdx.x == 0) {
                sc->last_iter = iter0;
                sc->done = 1;
            }
            return;
        }
    }
    const int H = sp.H, NR = BJ + 2 * WV_NH;
    const int pf = NR * H;   // floats per slot
    float *Er = wsm, *Eb = Er + WV_NE * pf, *Sr = Eb + WV_NE * pf, *Sb = Sr + WV_NS * pf;
    const long long cs = sp.cs;
    const int j0 = 1 + blockIdx.x * BJ, j1 = min(sp.ny - 1, j0 + BJ);   // owned rows [j0, j1)
    const int P0 = 1 + blockIdx.y * L, P1 = min(sp.nx - 1, P0 + L);     // owned planes [P0, P1)
    const int wlo = j0 - WV_NH;                                          // grid row of window row 0
    const int ra = max(0, -wlo), rb = min(NR, sp.ny - wlo);              // window rows inside the grid
    const int S0 = P0 - (WV_NH - 1), S1 = P1 - 1 + (WV_NH - 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nvec = H / 4, nchunk = (nvec + 31) / 32;

    // rows [ra, rb) of plane p of one colour array into a ring slot
    auto issue = [&](const float *g, float *slot, int p) {
        if (p < 0 || p > sp.nx - 1) return;
        const float *src = g + ((long long)p * sp.ny + wlo + ra) * H;
        float *dst = slot + ra * H;
        const int n4 = (rb - ra) * nvec;
        for (int t = threadIdx.x; t < n4; t += WV_THREADS) wv_cp16(dst + 4 * t, src + 4 * t);
    };
    // the planes first used at step s: red iterate s, black iterate s+1,
    // red source s, black source s-1
    auto load_step = [&](int s) {
        issue(P, Er + wv_mod(s, WV_NE) * pf, s);
        issue(P + cs, Eb + wv_mod(s + 1, WV_NE) * pf, s + 1);
        issue(R, Sr + wv_mod(s, WV_NS) * pf, s);
        issue(R + cs, Sb + wv_mod(s - 1, WV_NS) * pf, s - 1);
    };
    issue(P + cs, Eb + wv_mod(S0 - 1, WV_NE) * pf, S0 - 1);
    issue(P + cs, Eb + wv_mod(S0, WV_NE) * pf, S0);
#pragma unroll
    for (int d = 0; d < WV_D; d++) {
        load_step(S0 + d);
        wv_commit();
    }
    float rmax0 = 0.f, rmax1 = 0.f;
    for (int s = S0; s <= S1; s++) {
        wv_wait_prev();
        __syncthreads();
        if (s + WV_D <= S1) load_step(s + WV_D);
        wv_commit();
#pragma unroll
        for (int h = 0; h < WV_NH; h++) {
            const int e = WV_NH - 1 - h;
            const int p = s - h;
            const int pl = max(1, P0 - e), ph = min(sp.nx - 2, P1 - 1 + e);
            if (h > 0) __syncthreads();
            if (p < pl || p > ph) continue;   // uniform over the CTA
            const int c = h & 1;
            const int jl = max(1, j0 - e), jh = min(sp.ny - 2, j1 - 1 + e);
            float *own = (c ? Eb : Er) + wv_mod(p, WV_NE) * pf;
            const float *oth = (c ? Er : Eb);
            const float *xm = oth + wv_mod(p - 1, WV_NE) * pf, *xc = oth + wv_mod(p, WV_NE) * pf;
            const float *xp = oth + wv_mod(p + 1, WV_NE) * pf;
            const float *srcp = (c ? Sb : Sr) + wv_mod(p, WV_NS) * pf;
            const bool fin = h >= WV_NH - 2 && p >= P0 && p < P1;
            float *qrow = Q + c * cs + (long long)p * sp.ny * H;
            const int ntask = (jh - jl + 1) * nchunk;
            for (int task = warp; task < ntask; task += WV_THREADS / 32) {
                const int j = jl + task / nchunk;
                const int v = (task % nchunk) * 32 + lane;
                if (v >= nvec) continue;
                const int r = j - wlo, m0 = 4 * v, o = r * H + m0;
                const int sp_ = (p + j + c) & 1;
                float4 ow = *reinterpret_cast<const float4 *>(own + o);
                const float4 a = *reinterpret_cast<const float4 *>(xm + o);
                const float4 b = *reinterpret_cast<const float4 *>(xp + o);
                const float4 ym = *reinterpret_cast<const float4 *>(xc + o - H);
                const float4 yp = *reinterpret_cast<const float4 *>(xc + o + H);
                const float4 z = *reinterpret_cast<const float4 *>(xc + o);
                const float4 sr = *reinterpret_cast<const float4 *>(srcp + o);
                // z neighbour outside the vector: m0-1 (s = 0) or m0+4 (s = 1), inside the row
                const float ze = sp_ ? (m0 + 4 < H ? xc[o + 4] : 0.f) : (m0 > 0 ? xc[o - 1] : 0.f);
                const float A[4] = { a.x, a.y, a.z, a.w }, B[4] = { b.x, b.y, b.z, b.w };
                const float YM[4] = { ym.x, ym.y, ym.z, ym.w }, YP[4] = { yp.x, yp.y, yp.z, yp.w };
                const float Z[4] = { z.x, z.y, z.z, z.w }, SR[4] = { sr.x, sr.y, sr.z, sr.w };
                float W[4] = { ow.x, ow.y, ow.z, ow.w };
                float rm = 0.f;
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const int k = 2 * (m0 + q) + sp_;
                    if (k >= 1 && k <= sp.nz - 2) {
                        const float zm = sp_ ? Z[q] : (q == 0 ? ze : Z[q - 1]);
                        const float zp = sp_ ? (q == 3 ? ze : Z[q + 1]) : Z[q];
                        float rr;
                        W[q] = cf.update(W[q], A[q], B[q], YM[q], YP[q], zm, zp, SR[q], rr);
                        rm = fmaxf(rm, rr);
                    }
                }
                ow = make_float4(W[0], W[1], W[2], W[3]);
                *reinterpret_cast<float4 *>(own + o) = ow;
                if (h < 2) rmax0 = fmaxf(rmax0, rm);
                else rmax1 = fmaxf(rmax1, rm);
                if (fin && j >= j0 && j < j1) *reinterpret_cast<float4 *>(qrow + (long long)j * H + m0) = ow;
            }
        }
    }
    wv_wait_all();
    // per-iteration update norms: warp max, then one atomic per CTA and iteration
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        rmax0 = fmaxf(rmax0, __shfl_xor_sync(0xffffffffu, rmax0, off));
        rmax1 = fmaxf(rmax1, __shfl_xor_sync(0xffffffffu, rmax1, off));
    }
    if (lane == 0) {
        wred[0][warp] = rmax0;
        wred[1][warp] = rmax1;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        float b = 0.f;
        for (int w = 0; w < WV_THREADS / 32; w++) b = fmaxf(b, wred[threadIdx.x][w]);
        unsigned long long *slot = (unsigned long long *)(res + iter0 + threadIdx.x);
        if (b > 0.f && (unsigned long long)__double_as_longlong((double)b) > *(volatile unsigned long long *)slot)
            atomic_max_nonneg(slot, (double)b);
    }
}

}  // namespace hc
