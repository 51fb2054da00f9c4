// unet_conv.cuh -- 3x3x3 "same" convolutions of 16-channel BF16 volumes on
// the 5th-generation tensor cores (tcgen05, TMEM accumulators).
//
// Activations: channels-last (NDHWC), 16 BF16 channels = 32 bytes per voxel,
// voxel index v = (i*ny + j)*nz + k.  Weights: W[co][tap][ci] BF16 with
// tap = (di+1)*9 + (dj+1)*3 + (dk+1), i.e. the GEMM operand B with K = tap*16+ci
// contiguous (K-major).
//
// Forward (and input gradient) as an implicit GEMM:
//   Y[v][co] = sum_{tap,ci} X[v + off(tap)][ci] * W[co][tap][ci]
//   M = 128 voxels per CTA, N = 16 output channels, K = 27*16 = 432 in seven
//   chunks of four taps (64 columns, the last zero-padded).  The four warps
//   gather each A chunk (one 16-byte vector = 8 channels of one neighbour per
//   store) into a K-major canonical tile, double-buffered; one thread issues
//   four tcgen05.mma (K = 16 each) per chunk and commits them to the chunk
//   buffer's mbarrier; the accumulator (128 lanes x 16 FP32 columns) is read
//   back with tcgen05.ld for the epilogue (bias, LeakyReLU, BF16 store).
//   The input gradient is the same GEMM with W'[ci][tap][co] = W[co][26-tap][ci].
//
// Weight gradient as a GEMM over voxels:
//   dW[co][tap][ci] = sum_v dY[v][co] * X[v + off(tap)][ci]
//   D (M = (tap, ci) rows in four 128-row tiles, N = 16) += A * B^T with
//   K = 64 voxels per chunk; A[(tap,ci)][v] and B[co][v] are gathered
//   MN-major (8 consecutive channels of one voxel = one 16-byte row), so the
//   instruction descriptor sets a_major = b_major = 1.  Each CTA accumulates
//   its voxel range in TMEM (4 x 16 columns) and writes FP32 partial sums;
//   a second kernel adds the partials in a fixed order (deterministic).
//
// Every mbarrier wait is bounded; a wait that gives up sets the error flag,
// and the CTA still frees its TMEM before returning.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "tc.cuh"

namespace hc {
namespace unet {

constexpr int CH = 16;          // channels of every hidden volume
constexpr int NTAP = 27;
constexpr int TM = 128;         // voxels per CTA (GEMM M)
constexpr int KC = 64;          // K columns per chunk (4 taps x 16 channels)
constexpr int NCHUNK = 7;       // ceil(27/4)
constexpr int WELEM = CH * NTAP * CH;   // 6912 weights of one conv

struct Dims {
    int nx, ny, nz;
    long long n;                // voxels
};

__device__ __forceinline__ void voxel_ijk(const Dims &d, long long v, int &i, int &j, int &k)
{
    k = (int)(v % d.nz);
    long long t = v / d.nz;
    j = (int)(t % d.ny);
    i = (int)(t / d.ny);
}

// neighbour of (i,j,k) through tap, or -1 outside the volume
__device__ __forceinline__ long long neighbour(const Dims &d, int i, int j, int k, int tap)
{
    const int di = tap / 9 - 1, dj = (tap / 3) % 3 - 1, dk = tap % 3 - 1;
    const int a = i + di, b = j + dj, c = k + dk;
    if (a < 0 || a >= d.nx || b < 0 || b >= d.ny || c < 0 || c >= d.nz) return -1;
    return ((long long)a * d.ny + b) * d.nz + c;
}

__device__ __forceinline__ float leaky(float x) { return x > 0.f ? x : 0.1f * x; }

struct ConvSmem {
    __align__(128) unsigned char a[2][TM * KC * 2];        // 2 x 16 KB
    __align__(128) unsigned char b[NCHUNK][CH * KC * 2];   // 7 x 2 KB
    __align__(8) uint64_t bar[2];
    uint32_t tmem;
};

// out_mode: 0 = BF16 16 channels (+bias, LeakyReLU if act), 1 = BF16 16
// channels, no bias/activation (input gradient), 2 = FP32 channel 0 only
// (+bias[0], no activation: the network output), 3 = FP32 16 channels +bias
// (no rounding: the kernel's accumulators, for tests).
__global__ void __launch_bounds__(128)
conv3_kernel(const __nv_bfloat16 *__restrict__ x, const __nv_bfloat16 *__restrict__ w,
             const float *__restrict__ bias, void *__restrict__ out, Dims d, int out_mode, int act, int *err)
{
    extern __shared__ __align__(128) unsigned char smraw[];
    ConvSmem &sm = *reinterpret_cast<ConvSmem *>(smraw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const long long v0 = (long long)blockIdx.x * TM;

    if (warp == 0) {
        tc::tmem_alloc(&sm.tmem, 32);
        tc::fence_before();
    }
    if (tid == 0) {
        tc::bar_init(&sm.bar[0], 1);
        tc::bar_init(&sm.bar[1], 1);
    }
    // weights -> B tiles (K-major canonical, 16 rows x 64 columns per chunk)
    for (int t = tid; t < NCHUNK * CH * (KC / 8); t += blockDim.x) {
        const int c = t / (CH * (KC / 8));
        const int rem = t % (CH * (KC / 8));
        const int co = rem / (KC / 8), kg = rem % (KC / 8);   // kg: 8-column group
        const int tap = c * 4 + kg / 2, half = kg & 1;
        uint4 val = make_uint4(0, 0, 0, 0);
        if (tap < NTAP) val = *reinterpret_cast<const uint4 *>(w + ((size_t)co * NTAP + tap) * CH + half * 8);
        *reinterpret_cast<uint4 *>(sm.b[c] + tc::kmajor_off(co, kg * 8, KC)) = val;
    }
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = sm.tmem;
    constexpr uint32_t IDESC = tc::idesc_bf16(TM, CH);
    bool ok = true;

    // this thread gathers row r = tid of every A chunk
    const long long v = v0 + tid;
    const bool vin = v < d.n;
    int vi = 0, vj = 0, vk = 0;
    if (vin) voxel_ijk(d, v, vi, vj, vk);

    for (int c = 0; c < NCHUNK; c++) {
        const int buf = c & 1;
        if (c >= 2) ok = tc::bar_wait(&sm.bar[buf], ((c - 2) >> 1) & 1) && ok;   // MMAs of chunk c-2 done
        unsigned char *A = sm.a[buf];
#pragma unroll
        for (int tl = 0; tl < 4; tl++) {
            const int tap = c * 4 + tl;
            long long nb = -1;
            if (vin && tap < NTAP) nb = neighbour(d, vi, vj, vk, tap);
#pragma unroll
            for (int half = 0; half < 2; half++) {
                uint4 val = make_uint4(0, 0, 0, 0);
                if (nb >= 0) val = *reinterpret_cast<const uint4 *>(x + nb * CH + half * 8);
                *reinterpret_cast<uint4 *>(A + tc::kmajor_off(tid, tl * 16 + half * 8, KC)) = val;
            }
        }
        tc::fence_smem_to_async();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after();
            const uint32_t sa = tc::smem_u32(A), sb = tc::smem_u32(sm.b[c]);
#pragma unroll
            for (int s = 0; s < 4; s++) {
                const uint64_t da = tc::sdesc(sa + s * 256, 128, 16 * KC);
                const uint64_t db = tc::sdesc(sb + s * 256, 128, 16 * KC);
                tc::mma_bf16(tmem, da, db, IDESC, (c > 0 || s > 0) ? 1u : 0u);
            }
            tc::mma_commit(&sm.bar[buf]);
        }
    }
    // the last commit (chunk 6, buffer 0, its 4th phase) covers every MMA;
    // chunk 5's commit on buffer 1 is waited for too, so no arrive is pending
    ok = tc::bar_wait(&sm.bar[0], ((NCHUNK - 1) >> 1) & 1) && ok;
    ok = tc::bar_wait(&sm.bar[1], ((NCHUNK - 2) >> 1) & 1) && ok;
    tc::fence_after();
    float acc[16];
    tc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16), acc);
    const long long vo = v0 + warp * 32 + lane;   // TMEM lane = row of D
    if (vo < d.n) {
        if (out_mode == 2) {
            reinterpret_cast<float *>(out)[vo] = acc[0] + bias[0];
        } else if (out_mode == 3) {
            float *o = reinterpret_cast<float *>(out) + vo * CH;
#pragma unroll
            for (int t = 0; t < 16; t++) o[t] = acc[t] + bias[t];
        } else {
            __align__(16) __nv_bfloat16 h[16];
#pragma unroll
            for (int t = 0; t < 16; t++) {
                float y = acc[t];
                if (out_mode == 0) {
                    y += bias[t];
                    if (act) y = leaky(y);
                }
                h[t] = __float2bfloat16(y);
            }
            uint4 *o = reinterpret_cast<uint4 *>(reinterpret_cast<__nv_bfloat16 *>(out) + vo * CH);
            o[0] = *reinterpret_cast<const uint4 *>(&h[0]);
            o[1] = *reinterpret_cast<const uint4 *>(&h[8]);
        }
    }
    tc::fence_before();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, 32);
    if (!ok && tid == 0) atomicExch(err, -6);
}

// ---------------------------------------------------------------- weight gradient
constexpr int WG_NT = 256;
constexpr int WG_MT = 4;                   // 128-row tiles: taps 0-7, 8-15, 16-23, 24-26
struct WgradSmem {
    __align__(128) unsigned char a[2][WG_MT][TM * KC * 2];   // 2 x 4 x 16 KB
    __align__(128) unsigned char b[2][CH * KC * 2];          // 2 x 2 KB
    __align__(8) uint64_t bar[2];
    uint32_t tmem;
};

// byte offset of (mn, k) in an MN-major no-swizzle tile with KC columns:
// 8 consecutive mn = one 16-byte row, 8 rows (k) per core matrix
__host__ __device__ __forceinline__ uint32_t mnmajor_off(int mn, int k, int kc)
{
    return (uint32_t)((mn >> 3) * (16 * kc) + (k >> 3) * 128 + (k & 7) * 16 + (mn & 7) * 2);
}

// partial[cta][tap][ci][co] over the CTA's voxel chunks [c0, c1)
__global__ void __launch_bounds__(WG_NT)
wgrad_kernel(const __nv_bfloat16 *__restrict__ x, const __nv_bfloat16 *__restrict__ dy, float *__restrict__ partial,
             Dims d, int chunks_per_cta, int *err)
{
    extern __shared__ __align__(128) unsigned char smraw[];
    WgradSmem &sm = *reinterpret_cast<WgradSmem *>(smraw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const long long nchunk = (d.n + KC - 1) / KC;
    const long long c0 = (long long)blockIdx.x * chunks_per_cta;
    const long long c1 = min(nchunk, c0 + chunks_per_cta);

    if (warp == 0) {
        tc::tmem_alloc(&sm.tmem, 64);
        tc::fence_before();
    }
    if (tid == 0) {
        tc::bar_init(&sm.bar[0], 1);
        tc::bar_init(&sm.bar[1], 1);
    }
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = sm.tmem;
    constexpr uint32_t IDESC = tc::idesc_bf16(TM, CH) | (1u << 15) | (1u << 16);
    bool ok = true;
    int issued = 0;

    for (long long c = c0; c < c1; c++) {
        const int q = (int)(c - c0), buf = q & 1;
        if (q >= 2) ok = tc::bar_wait(&sm.bar[buf], ((q - 2) >> 1) & 1) && ok;
        // A: 4 tiles x (8 taps x 2 halves) x 64 voxels of 16-byte rows; B: 2 halves x 64
        for (int t = tid; t < KC * (32 * 2 + 2); t += WG_NT) {
            const int kk = t % KC, slot = t / KC;      // slot 0..63: (tap 0..31, half); 64..65: dy halves
            const long long v = c * KC + kk;
            uint4 val = make_uint4(0, 0, 0, 0);
            if (slot < 64) {
                const int tap = slot >> 1, half = slot & 1;
                if (v < d.n && tap < NTAP) {
                    int i, j, k;
                    voxel_ijk(d, v, i, j, k);
                    const long long nb = neighbour(d, i, j, k, tap);
                    if (nb >= 0) val = *reinterpret_cast<const uint4 *>(x + nb * CH + half * 8);
                }
                const int tile = tap >> 3, row = (tap & 7) * 16 + half * 8;
                *reinterpret_cast<uint4 *>(sm.a[buf][tile] + mnmajor_off(row, kk, KC)) = val;
            } else {
                const int half = slot - 64;
                if (v < d.n) val = *reinterpret_cast<const uint4 *>(dy + v * CH + half * 8);
                *reinterpret_cast<uint4 *>(sm.b[buf] + mnmajor_off(half * 8, kk, KC)) = val;
            }
        }
        tc::fence_smem_to_async();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after();
            const uint32_t sb = tc::smem_u32(sm.b[buf]);
#pragma unroll
            for (int tile = 0; tile < WG_MT; tile++) {
                const uint32_t sa = tc::smem_u32(sm.a[buf][tile]);
#pragma unroll
                for (int s = 0; s < 4; s++) {
                    const uint64_t da = tc::sdesc(sa + s * 256, 128, 16 * KC);
                    const uint64_t db = tc::sdesc(sb + s * 256, 128, 16 * KC);
                    tc::mma_bf16(tmem + tile * 16, da, db, IDESC, (q > 0 || s > 0) ? 1u : 0u);
                }
            }
            tc::mma_commit(&sm.bar[buf]);
        }
        issued = q + 1;
    }
    float *p = partial + (size_t)blockIdx.x * (WG_MT * TM * CH);
    if (issued > 0) {
        const int ql = issued - 1;
        ok = tc::bar_wait(&sm.bar[ql & 1], (ql >> 1) & 1) && ok;   // the last commit covers all
        if (ql >= 1) ok = tc::bar_wait(&sm.bar[(ql - 1) & 1], ((ql - 1) >> 1) & 1) && ok;
        tc::fence_after();
#pragma unroll
        for (int tile = 0; tile < WG_MT; tile++) {
            if (warp < 4) {   // warps 0-3 own TMEM lanes 0-127
                float acc[16];
                tc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + tile * 16, acc);
                const int row = tile * TM + warp * 32 + lane;   // (tap, ci) = (row / 16, row % 16)
#pragma unroll
                for (int co = 0; co < 16; co++) p[(size_t)row * CH + co] = acc[co];
            }
        }
    } else {
        for (int t = tid; t < WG_MT * TM * CH; t += WG_NT) p[t] = 0.f;
    }
    tc::fence_before();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, 64);
    if (!ok && tid == 0) atomicExch(err, -6);
}

// dW[co][tap][ci] = sum over CTAs of partial[cta][tap*16+ci][co], fixed order
__global__ void wgrad_reduce_kernel(const float *__restrict__ partial, int nparts, float *__restrict__ dw)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;   // (co, tap, ci)
    if (e >= WELEM) return;
    const int co = e / (NTAP * CH), tap = (e / CH) % NTAP, ci = e % CH;
    const int row = tap * CH + ci;
    float s = 0.f;
    for (int p = 0; p < nparts; p++) s += partial[(size_t)p * (WG_MT * TM * CH) + (size_t)row * CH + co];
    dw[e] = s;
}


// ---------------------------------------------------------------------------
// Halo-tile convolution (forward / input gradient) without an im2col copy.
//
// A CTA owns a 16 (j) x 8 (k) column of output voxels and marches along i.
// Each input plane of the column plus its halo (18 x 10 voxels) is fetched by
// two cp.async.bulk.tensor loads (one per 8-channel half, zero-filled outside
// the volume) into a 4-slot ring laid out [half][j][k][8 ch]: 8 consecutive k
// of one half are 128 contiguous bytes, i.e. one core matrix of a K-major
// operand.  The A operand of tap (a,b,c) for output plane i is therefore a
// descriptor into the halo of plane i+a-1 starting at row (b, c): SBO = 160
// bytes (next j), LBO = one half-plane (2944-byte stride, channels 8..15).  Each
// output plane is 27 MMAs (M=128 voxels, N=16, K=16 channels) accumulated in
// one of two TMEM buffers; the epilogue of plane p-1 runs while the MMAs of
// plane p execute, and the halo slot of plane p-2 is refilled once the MMAs
// of plane p-1 have completed.
// ---------------------------------------------------------------------------
constexpr int HT_J = 16, HT_K = 8;                  // output tile
constexpr int HH_J = HT_J + 2, HH_K = HT_K + 2;     // halo tile
constexpr int HALF_BYTES = HH_J * HH_K * 16;        // 2880 loaded per channel half
constexpr int HALF_STRIDE = 2944;                   // 128-byte aligned stride (the descriptor LBO)
constexpr int SLOT_BYTES = 2 * HALF_STRIDE;         // 5888
constexpr int NSLOT = 4;

struct HaloSmem {
    __align__(128) unsigned char slot[NSLOT][SLOT_BYTES];
    __align__(128) unsigned char w[NTAP][512];      // B per tap: 16 co x 16 ci, K-major
    __align__(8) uint64_t tbar[NSLOT];
    __align__(8) uint64_t mbar[2];
    uint32_t tmem;
};

__device__ __forceinline__ void halo_load(const CUtensorMap *tm, HaloSmem &sm, int slot, int k0, int j0, int i)
{
    uint64_t *bar = &sm.tbar[slot];
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc::smem_u32(bar)),
                 "r"((unsigned)(2 * HALF_BYTES))
                 : "memory");
#pragma unroll
    for (int h = 0; h < 2; h++)
        asm volatile("cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes"
                     " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(tc::smem_u32(sm.slot[slot] + h * HALF_STRIDE)),
                     "l"(reinterpret_cast<uint64_t>(tm)), "r"(8 * h), "r"(k0 - 1), "r"(j0 - 1), "r"(i),
                     "r"(tc::smem_u32(bar))
                     : "memory");
}

__global__ void __launch_bounds__(128)
conv3_halo_kernel(const __grid_constant__ CUtensorMap tmx, const __nv_bfloat16 *__restrict__ w,
                  const float *__restrict__ bias, void *__restrict__ out, Dims d, int out_mode, int act, int chunk,
                  int *err)
{
    extern __shared__ __align__(128) unsigned char smraw[];
    HaloSmem &sm = *reinterpret_cast<HaloSmem *>(smraw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int k0 = blockIdx.x * HT_K, j0 = blockIdx.y * HT_J;
    const int i0 = blockIdx.z * chunk, i1 = min(d.nx, i0 + chunk);
    if (i0 >= i1) return;
    const int np = i1 - i0;

    if (warp == 0) {
        tc::tmem_alloc(&sm.tmem, 32);
        tc::fence_before();
    }
    if (tid == 0) {
        for (int q = 0; q < NSLOT; q++) tc::bar_init(&sm.tbar[q], 1);
        tc::bar_init(&sm.mbar[0], 1);
        tc::bar_init(&sm.mbar[1], 1);
    }
    // weights: B of tap t, row co, K = ci: (co/8)*256 + (ci/8)*128 + (co%8)*16 + (ci%8)*2
    for (int q = tid; q < NTAP * CH * 2; q += blockDim.x) {
        const int tap = q / (CH * 2), rem = q % (CH * 2), co = rem >> 1, half = rem & 1;
        const uint4 v = *reinterpret_cast<const uint4 *>(w + ((size_t)co * NTAP + tap) * CH + half * 8);
        *reinterpret_cast<uint4 *>(sm.w[tap] + (co >> 3) * 256 + half * 128 + (co & 7) * 16) = v;
    }
    tc::fence_smem_to_async();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = sm.tmem;
    constexpr uint32_t IDESC = tc::idesc_bf16(TM, CH);
    bool ok = true;
    unsigned tph[NSLOT] = { 0, 0, 0, 0 }, mph[2] = { 0, 0 };
    auto slot_of = [](int plane) { return (plane + 4) & 3; };   // plane >= -1

    if (tid == 0) {
        halo_load(&tmx, sm, slot_of(i0 - 1), k0, j0, i0 - 1);
        halo_load(&tmx, sm, slot_of(i0), k0, j0, i0);
        halo_load(&tmx, sm, slot_of(i0 + 1), k0, j0, i0 + 1);
    }
    auto wait_plane = [&](int plane) {
        const int sl = slot_of(plane);
        ok = tc::bar_wait(&sm.tbar[sl], tph[sl] & 1) && ok;
        tph[sl]++;
    };
    auto epilogue = [&](int p) {
        const int b = p & 1;
        ok = tc::bar_wait(&sm.mbar[b], mph[b] & 1) && ok;
        mph[b]++;
        tc::fence_after();
        float acc[16];
        tc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + b * 16, acc);
        const int r = warp * 32 + lane, jj = r >> 3, kk = r & 7;
        const int j = j0 + jj, k = k0 + kk, i = i0 + p;
        if (j < d.ny && k < d.nz) {
            const long long vo = ((long long)i * d.ny + j) * d.nz + k;
            if (out_mode == 2) {
                reinterpret_cast<float *>(out)[vo] = acc[0] + bias[0];
            } else if (out_mode == 3) {
                float *o = reinterpret_cast<float *>(out) + vo * CH;
#pragma unroll
                for (int t = 0; t < 16; t++) o[t] = acc[t] + bias[t];
            } else {
                __align__(16) __nv_bfloat16 h[16];
#pragma unroll
                for (int t = 0; t < 16; t++) {
                    float y = acc[t];
                    if (out_mode == 0) {
                        y += bias[t];
                        if (act) y = leaky(y);
                    }
                    h[t] = __float2bfloat16(y);
                }
                uint4 *o = reinterpret_cast<uint4 *>(reinterpret_cast<__nv_bfloat16 *>(out) + vo * CH);
                o[0] = *reinterpret_cast<const uint4 *>(&h[0]);
                o[1] = *reinterpret_cast<const uint4 *>(&h[8]);
            }
        }
    };

    wait_plane(i0 - 1);
    wait_plane(i0);
    for (int p = 0; p < np; p++) {
        const int i = i0 + p;
        wait_plane(i + 1);
        if (tid == 0) {
            tc::fence_after();
            const uint32_t wb = tc::smem_u32(sm.w[0]);
#pragma unroll 1
            for (int a = 0; a < 3; a++) {
                const uint32_t base = tc::smem_u32(sm.slot[slot_of(i + a - 1)]);
#pragma unroll
                for (int bc = 0; bc < 9; bc++) {
                    const int b = bc / 3, c = bc % 3, tap = a * 9 + bc;
                    const uint64_t da = tc::sdesc(base + (b * HH_K + c) * 16, HALF_STRIDE, HH_K * 16);
                    const uint64_t db = tc::sdesc(wb + tap * 512, 128, 256);
                    tc::mma_bf16(tmem + (p & 1) * 16, da, db, IDESC, tap > 0 ? 1u : 0u);
                }
            }
            tc::mma_commit(&sm.mbar[p & 1]);
        }
        if (p >= 1) epilogue(p - 1);   // also: the MMAs of plane p-1 are done
        if (tid == 0 && p + 2 < np + 1) halo_load(&tmx, sm, slot_of(i + 2), k0, j0, i + 2);
        tc::fence_before();
        __syncthreads();   // TMEM buffer of plane p-1 read by all before plane p+1 reuses it
    }
    epilogue(np - 1);
    // the last halo load (plane i1) was consumed by the last plane; planes past it were not issued
    tc::fence_before();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, 32);
    if (!ok && tid == 0) atomicExch(err, -6);
}

}  // namespace unet
}  // namespace hc
