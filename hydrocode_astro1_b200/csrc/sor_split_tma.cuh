// sor_split_tma.cuh -- one FP32 colour sweep on the colour-split layout with
// its operands staged by TMA.
//
// The vector sweep (sor_split_vec_kernel) issues all its loads from
// registers and is bound by memory latency: many short CTAs, each with a
// few 16-byte loads per thread in flight.  Here a persistent grid (one CTA
// per SM) walks over tiles of NI planes x TJ rows x a whole colour row (H
// cells); each tile's three operands -- the other colour with a one-plane
// and one-row halo, the own colour and the source -- arrive as three bulk
// tensor copies into shared memory, NS tiles in flight per CTA on mbarriers
// (bounded waits), so tens of kilobytes per SM stream in while the current
// tile is swept.  The cells are updated from shared memory and stored with
// 16-byte vector stores.
//
// Neighbours of a cell of colour c at (i, j, m), k = 2m + s with
// s = (i + j + c) & 1, are of the other colour: x and y at the same m in the
// rows (i+-1, j) and (i, j+-1); z at m-1 / m (s = 0) or m / m+1 (s = 1) in
// its own row.  A whole row is one tile column, so the z neighbours never
// cross a tile (the cells at m = 0, s = 0 and m = H-1, s = 1 are boundary or
// padding cells, not updated).  The update is SorCoef<float>::update with
// the vector kernel's operands, so the iterates are the same bits; cells of
// a stored vector that are not updated (k = 0, nz-1, the padding slot) are
// stored back unchanged.
#pragma once
#include <cuda.h>

#include "hc_internal.cuh"
#include "mbar.cuh"
#include "sor_split.cuh"

namespace hc {
namespace stma {

constexpr int TJ = 8;        // rows of a tile (one warp each)
constexpr int NT = 32 * TJ;
constexpr int HMAX = 256;    // row length limit of one bulk copy box

struct Tiles {
    int nx, ny, nz, H;
    int ti, tj;              // tiles along i (planes 1..nx-2) and j (rows 1..ny-2)
};

// One pipeline stage: other (NI+2) x (TJ+2) rows, own NI x TJ rows, source
// NI x TJ rows of H floats, each region starting on a 128-byte boundary.
__host__ __device__ __forceinline__ int pad32(int n) { return (n + 31) / 32 * 32; }
template <int NI>
__host__ __device__ __forceinline__ int stage_floats(int H)
{
    return pad32((NI + 2) * (TJ + 2) * H) + 2 * pad32(NI * TJ * H);
}

__device__ __forceinline__ void tma3(const CUtensorMap *tm, float *dst, uint64_t *bar, int x, int y, int z)
{
    asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_addr(dst)),
                 "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
                 : "memory");
}

template <int NI, int NS>
__global__ void __launch_bounds__(NT, 1)
sor_split_tma_kernel(const __grid_constant__ CUtensorMap m_oth, const __grid_constant__ CUtensorMap m_own,
                     const __grid_constant__ CUtensorMap m_src, float *__restrict__ own, Tiles tl, SorCoef<float> cf,
                     int colour, double *res, int iter, double thresh, DevScalars *sc)
{
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t bar[NS];
    __shared__ double wmax[NT / 32];
    pdl_wait_and_release();
    if (*(volatile int *)&sc->done) return;
    if (colour == 0 && iter > 0) {
        const double prev = __longlong_as_double(*reinterpret_cast<const volatile long long *>(res + iter - 1));
        if (prev < thresh) {
            if (threadIdx.x == 0) {
                sc->last_iter = iter;
                sc->done = 1;
            }
            return;
        }
    }
    const int H = tl.H;
    const int OTH = pad32((NI + 2) * (TJ + 2) * H), OWN = pad32(NI * TJ * H);
    const int STAGE = OTH + 2 * OWN;
    float *stage0 = reinterpret_cast<float *>(smem);
    // bytes the three copies of a stage deliver (the padding is not copied)
    const unsigned bytes = (unsigned)((NI + 2) * (TJ + 2) * H + 2 * NI * TJ * H) * 4u;
    const int ntiles = tl.ti * tl.tj;
    const int tid = threadIdx.x, lane = tid & 31, r = tid >> 5;
    if (tid == 0) {
        for (int b = 0; b < NS; b++) mbar_init(&bar[b], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    // this CTA's tiles: blockIdx.x + t * gridDim.x, t < mine; colour-1
    // sweeps take the tiles in reverse order (the L2 still holds the tiles
    // the colour-0 sweep ended with)
    const int mine = ((int)blockIdx.x < ntiles) ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    auto tile_of = [&](int t) {
        const int g = (int)blockIdx.x + t * (int)gridDim.x;
        return colour ? ntiles - 1 - g : g;
    };
    auto issue = [&](int t) {
        if (tid == 0 && t < mine) {
            const int g = tile_of(t);
            const int i0 = 1 + (g / tl.tj) * NI, j0 = 1 + (g % tl.tj) * TJ;
            const int b = t % NS;
            float *st = stage0 + (size_t)b * STAGE;
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_expect_tx(&bar[b], bytes);
            tma3(&m_oth, st, &bar[b], 0, j0 - 1, i0 - 1);
            tma3(&m_own, st + OTH, &bar[b], 0, j0, i0);
            tma3(&m_src, st + OTH + OWN, &bar[b], 0, j0, i0);
        }
    };
    for (int t = 0; t < NS; t++) issue(t);
    unsigned phase = 0u;   // bit b: parity of the next wait on bar[b]
    bool ok = true;
    float rmax = 0.f;
    const long long sI = (long long)tl.ny * H, sJ = H;
    for (int t = 0; t < mine; t++) {
        const int b = t % NS;
        ok = mbar_wait(&bar[b], (phase >> b) & 1u) && ok;
        phase ^= 1u << b;
        const float *st = stage0 + (size_t)b * STAGE;
        const float *O = st, *W = st + OTH, *S = st + OTH + OWN;
        const int g = tile_of(t);
        const int i0 = 1 + (g / tl.tj) * NI, j0 = 1 + (g % tl.tj) * TJ;
        const int j = j0 + r;
        if (j <= tl.ny - 2) {   // uniform over the warp
#pragma unroll
            for (int q = 0; q < NI; q++) {
                const int i = i0 + q;
                if (i > tl.nx - 2) break;
                const int s = (i + j + colour) & 1;
                const float *o_c = O + ((q + 1) * (TJ + 2) + r + 1) * H;   // other colour, same plane and row
                const float *o_xm = O + (q * (TJ + 2) + r + 1) * H;
                const float *o_xp = O + ((q + 2) * (TJ + 2) + r + 1) * H;
                const float *o_ym = O + ((q + 1) * (TJ + 2) + r) * H;
                const float *o_yp = O + ((q + 1) * (TJ + 2) + r + 2) * H;
                const float *w_r = W + (q * TJ + r) * H;
                const float *s_r = S + (q * TJ + r) * H;
                float *g_row = own + (long long)i * sI + (long long)j * sJ;
                for (int m0 = 4 * lane; m0 < H; m0 += 128) {
                    const float4 ow = *reinterpret_cast<const float4 *>(w_r + m0);
                    const float4 sr = *reinterpret_cast<const float4 *>(s_r + m0);
                    const float4 xm = *reinterpret_cast<const float4 *>(o_xm + m0);
                    const float4 xp = *reinterpret_cast<const float4 *>(o_xp + m0);
                    const float4 ym = *reinterpret_cast<const float4 *>(o_ym + m0);
                    const float4 yp = *reinterpret_cast<const float4 *>(o_yp + m0);
                    const float4 zc = *reinterpret_cast<const float4 *>(o_c + m0);
                    // the z neighbour outside the vector: m0-1 (s = 0) or m0+4 (s = 1),
                    // clamped into the row where it feeds no update
                    const float ze = s ? o_c[min(m0 + 4, H - 1)] : o_c[max(m0 - 1, 0)];
                    const float owv[4] = { ow.x, ow.y, ow.z, ow.w }, srv[4] = { sr.x, sr.y, sr.z, sr.w };
                    const float xmv[4] = { xm.x, xm.y, xm.z, xm.w }, xpv[4] = { xp.x, xp.y, xp.z, xp.w };
                    const float ymv[4] = { ym.x, ym.y, ym.z, ym.w }, ypv[4] = { yp.x, yp.y, yp.z, yp.w };
                    const float zv[4] = { zc.x, zc.y, zc.z, zc.w };
                    float nv[4];
#pragma unroll
                    for (int e = 0; e < 4; e++) {
                        const int k = 2 * (m0 + e) + s;
                        nv[e] = owv[e];
                        if (k >= 1 && k <= tl.nz - 2) {
                            const float zm = s ? zv[e] : (e == 0 ? ze : zv[e - 1]);
                            const float zp = s ? (e == 3 ? ze : zv[e + 1]) : zv[e];
                            float rr;
                            nv[e] = cf.update(owv[e], xmv[e], xpv[e], ymv[e], ypv[e], zm, zp, srv[e], rr);
                            rmax = tmax(rmax, rr);
                        }
                    }
                    *reinterpret_cast<float4 *>(g_row + m0) = make_float4(nv[0], nv[1], nv[2], nv[3]);
                }
            }
        }
        __syncthreads();            // every thread is done with this stage
        issue(t + NS);
    }
    double v = (double)rmax;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v = tmax(v, __shfl_xor_sync(0xffffffffu, v, off));
    if (lane == 0) wmax[r] = v;
    __syncthreads();
    if (tid == 0) {
        double m = 0.0;
#pragma unroll
        for (int w = 0; w < NT / 32; w++) m = tmax(m, wmax[w]);
        unsigned long long *slot = (unsigned long long *)(res + iter);
        if (m > 0.0 && (unsigned long long)__double_as_longlong(m) > *(volatile unsigned long long *)slot)
            atomic_max_nonneg(slot, m);
        if (!ok) atomicExch(&sc->err, HC_ERR_TIMEOUT);
    }
}

}  // namespace stma
}  // namespace hc
