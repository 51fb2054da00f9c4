// unet_ops.cuh -- the non-GEMM kernels of the warm-start U-Net: 2x average
// pooling and nearest upsampling with skip addition (and their transposes
// fused with the LeakyReLU derivative), bias gradients, the loss, Adam, and
// the kernels that move between the solver's grid and the network's
// half-resolution input/output.
//
// Volumes: 16 BF16 channels per voxel (channels last), handled as two
// 16-byte halves of 8 channels.  A level-(l+1) voxel (I,J,K) is the average
// of the 8 level-l voxels (2I+a, 2J+b, 2K+c).
#pragma once
#include <cuda_bf16.h>

#include "hc_internal.cuh"
#include "sor_split.cuh"
#include "unet_conv.cuh"

namespace hc {
namespace unet {

__device__ __forceinline__ void ld8(const __nv_bfloat16 *p, float (&f)[8])
{
    const uint4 u = *reinterpret_cast<const uint4 *>(p);
    const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&u);
#pragma unroll
    for (int t = 0; t < 4; t++) {
        const float2 v = __bfloat1622float2(h[t]);
        f[2 * t] = v.x;
        f[2 * t + 1] = v.y;
    }
}

__device__ __forceinline__ void st8(__nv_bfloat16 *p, const float (&f)[8])
{
    uint4 u;
    __nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(&u);
#pragma unroll
    for (int t = 0; t < 4; t++) h[t] = __floats2bfloat162_rn(f[2 * t], f[2 * t + 1]);
    *reinterpret_cast<uint4 *>(p) = u;
}

__device__ __forceinline__ float dleaky(float y) { return y > 0.f ? 1.f : 0.1f; }

__device__ __forceinline__ long long vidx(const Dims &d, int i, int j, int k)
{
    return ((long long)i * d.ny + j) * d.nz + k;
}

#define UNET_LOOP(n) for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (n); \
                          t += (long long)gridDim.x * blockDim.x)

// out (coarse, dc) = average of 8 children of in (fine, 2 dc)
__global__ void pool2_kernel(const __nv_bfloat16 *__restrict__ in, __nv_bfloat16 *__restrict__ out, Dims dc)
{
    const Dims df{ 2 * dc.nx, 2 * dc.ny, 2 * dc.nz, 8 * dc.n };
    UNET_LOOP(dc.n * 2)
    {
        const long long v = t >> 1;
        const int half = (int)(t & 1);
        int I, J, K;
        voxel_ijk(dc, v, I, J, K);
        float s[8] = { 0, 0, 0, 0, 0, 0, 0, 0 };
        for (int c = 0; c < 8; c++) {
            float f[8];
            ld8(in + vidx(df, 2 * I + (c >> 2), 2 * J + ((c >> 1) & 1), 2 * K + (c & 1)) * CH + half * 8, f);
#pragma unroll
            for (int q = 0; q < 8; q++) s[q] += f[q];
        }
#pragma unroll
        for (int q = 0; q < 8; q++) s[q] *= 0.125f;
        st8(out + v * CH + half * 8, s);
    }
}

// out (fine, df) = nearest upsample of coarse (df/2) + skip (fine)
__global__ void up_add_kernel(const __nv_bfloat16 *__restrict__ coarse, const __nv_bfloat16 *__restrict__ skip,
                              __nv_bfloat16 *__restrict__ out, Dims df)
{
    const Dims dc{ df.nx / 2, df.ny / 2, df.nz / 2, df.n / 8 };
    UNET_LOOP(df.n * 2)
    {
        const long long v = t >> 1;
        const int half = (int)(t & 1);
        int i, j, k;
        voxel_ijk(df, v, i, j, k);
        float a[8], b[8];
        ld8(coarse + vidx(dc, i >> 1, j >> 1, k >> 1) * CH + half * 8, a);
        ld8(skip + v * CH + half * 8, b);
#pragma unroll
        for (int q = 0; q < 8; q++) a[q] += b[q];
        st8(out + v * CH + half * 8, a);
    }
}

// dz = g * LeakyReLU'(y)
__global__ void act_back_kernel(const __nv_bfloat16 *__restrict__ g, const __nv_bfloat16 *__restrict__ y,
                                __nv_bfloat16 *__restrict__ dz, long long n)
{
    UNET_LOOP(n * 2)
    {
        float a[8], b[8];
        ld8(g + t * 8, a);
        ld8(y + t * 8, b);
#pragma unroll
        for (int q = 0; q < 8; q++) a[q] *= dleaky(b[q]);
        st8(dz + t * 8, a);
    }
}

// transpose of the nearest upsample (sum of the 8 children of gfine), times
// LeakyReLU'(ycoarse): dz (coarse, dc)
__global__ void downsum_act_kernel(const __nv_bfloat16 *__restrict__ gfine, const __nv_bfloat16 *__restrict__ ycoarse,
                                   __nv_bfloat16 *__restrict__ dz, Dims dc)
{
    const Dims df{ 2 * dc.nx, 2 * dc.ny, 2 * dc.nz, 8 * dc.n };
    UNET_LOOP(dc.n * 2)
    {
        const long long v = t >> 1;
        const int half = (int)(t & 1);
        int I, J, K;
        voxel_ijk(dc, v, I, J, K);
        float s[8] = { 0, 0, 0, 0, 0, 0, 0, 0 };
        for (int c = 0; c < 8; c++) {
            float f[8];
            ld8(gfine + vidx(df, 2 * I + (c >> 2), 2 * J + ((c >> 1) & 1), 2 * K + (c & 1)) * CH + half * 8, f);
#pragma unroll
            for (int q = 0; q < 8; q++) s[q] += f[q];
        }
        float y[8];
        ld8(ycoarse + v * CH + half * 8, y);
#pragma unroll
        for (int q = 0; q < 8; q++) s[q] *= dleaky(y[q]);
        st8(dz + v * CH + half * 8, s);
    }
}

// transpose of the average pool (parent gradient / 8 to each child) added to
// the skip gradient, times LeakyReLU'(yfine): dz (fine, df)
__global__ void poolback_add_act_kernel(const __nv_bfloat16 *__restrict__ gskip,
                                        const __nv_bfloat16 *__restrict__ gcoarse,
                                        const __nv_bfloat16 *__restrict__ yfine, __nv_bfloat16 *__restrict__ dz, Dims df)
{
    const Dims dc{ df.nx / 2, df.ny / 2, df.nz / 2, df.n / 8 };
    UNET_LOOP(df.n * 2)
    {
        const long long v = t >> 1;
        const int half = (int)(t & 1);
        int i, j, k;
        voxel_ijk(df, v, i, j, k);
        float a[8], b[8], y[8];
        ld8(gskip + v * CH + half * 8, a);
        ld8(gcoarse + vidx(dc, i >> 1, j >> 1, k >> 1) * CH + half * 8, b);
        ld8(yfine + v * CH + half * 8, y);
#pragma unroll
        for (int q = 0; q < 8; q++) a[q] = (a[q] + 0.125f * b[q]) * dleaky(y[q]);
        st8(dz + v * CH + half * 8, a);
    }
}

// per-block channel sums of dz -> partial[block][16]
constexpr int BG_NT = 256;
__global__ void __launch_bounds__(BG_NT) bias_grad_kernel(const __nv_bfloat16 *__restrict__ dz, long long n,
                                                          float *__restrict__ partial)
{
    float s[8] = { 0, 0, 0, 0, 0, 0, 0, 0 };
    // thread t handles half (t & 1) of voxels t/2, t/2 + stride, ...
    const int half = threadIdx.x & 1;
    for (long long v = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 1; v < n;
         v += ((long long)gridDim.x * blockDim.x) >> 1) {
        float f[8];
        ld8(dz + v * CH + half * 8, f);
#pragma unroll
        for (int q = 0; q < 8; q++) s[q] += f[q];
    }
    // reduce over the threads with the same half, fixed order
    __shared__ float red[BG_NT][8];
#pragma unroll
    for (int q = 0; q < 8; q++) red[threadIdx.x][q] = s[q];
    __syncthreads();
    if (threadIdx.x < 16) {
        const int h = threadIdx.x >> 3, q = threadIdx.x & 7;
        float tot = 0.f;
        for (int r = h; r < BG_NT; r += 2) tot += red[r][q];
        partial[blockIdx.x * CH + h * 8 + q] = tot;
    }
}

__global__ void sum_partials_kernel(const float *__restrict__ partial, int nparts, float *__restrict__ out, int width)
{
    const int c = threadIdx.x;
    if (c >= width) return;
    float s = 0.f;
    for (int p = 0; p < nparts; p++) s += partial[p * width + c];
    out[c] = s;
}

// ---------------------------------------------------------------- solver side
// pooled[v0] = average of the 8 grid cells of net voxel v0 of the residual
// (colour-split FP32, zero on boundary cells); sumsq += pooled^2
// The sum of squares goes to one partial per block (part[blockIdx.x]; 256
// threads), added in a fixed order by sum_parts_kernel: the same input gives
// the same bits (no atomics on one address).
__global__ void in_pool_kernel(const float *__restrict__ r32, Split sp, Dims d0, float *__restrict__ pooled,
                               double *__restrict__ part)
{
    __shared__ double ws[8];
    double local = 0.0;
    UNET_LOOP(d0.n)
    {
        int I, J, K;
        voxel_ijk(d0, t, I, J, K);
        float s = 0.f;
        for (int c = 0; c < 8; c++) {
            const int i = 2 * I + (c >> 2), j = 2 * J + ((c >> 1) & 1), k = 2 * K + (c & 1);
            s += r32[sp.at(i, j, k)];
        }
        s *= 0.125f;
        pooled[t] = s;
        local += (double)s * s;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = local;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) b += ws[w];
        part[blockIdx.x] = b;
    }
}

// out = sum of part[0..n) in a fixed order (one warp)
__global__ void sum_parts_kernel(const double *__restrict__ part, int n, double *__restrict__ out)
{
    double acc = 0.0;
    for (int b = threadIdx.x; b < n; b += 32) acc += part[b];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (threadIdx.x == 0) *out = acc;
}

// x0 (16 channels, channel 0 = pooled / rms, others 0)
__global__ void in_norm_kernel(const float *__restrict__ pooled, const double *__restrict__ sumsq, long long n0,
                               __nv_bfloat16 *__restrict__ x0, float *__restrict__ xnorm)
{
    const double ms = *sumsq / (double)n0;
    const float inv = ms > 0.0 ? (float)(1.0 / sqrt(ms)) : 0.f;
    UNET_LOOP(n0 * 2)
    {
        const long long v = t >> 1;
        float f[8] = { 0, 0, 0, 0, 0, 0, 0, 0 };
        if ((t & 1) == 0) {
            f[0] = pooled[v] * inv;
            if (xnorm) xnorm[v] = f[0];
        }
        st8(x0 + t * 8, f);
    }
}

// x0 from a stored normalised single-channel sample
__global__ void in_expand_kernel(const float *__restrict__ x, long long n0, __nv_bfloat16 *__restrict__ x0)
{
    UNET_LOOP(n0 * 2)
    {
        float f[8] = { 0, 0, 0, 0, 0, 0, 0, 0 };
        if ((t & 1) == 0) f[0] = x[t >> 1];
        st8(x0 + t * 8, f);
    }
}

// trilinear weights of fine index i (cell centres) on the coarse axis of n0
__device__ __forceinline__ void lin_coarse(int i, int n0, int &a, int &b, float &wb)
{
    // coarse coordinate of the fine centre: (i + 0.5) / 2 - 0.5
    const int q = i >> 1;
    if (i & 1) {   // (q + 0.25): between q and q+1
        a = q;
        b = min(q + 1, n0 - 1);
        wb = 0.25f;
    } else {       // (q - 0.25): between q-1 and q
        a = max(q - 1, 0);
        b = q;
        wb = 0.75f;
    }
}

// e (colour-split FP32, whole grid) = trilinear upsample of the network output
// times rms * kscale; zero on boundary cells.  A CTA takes OUT_UP_ROWS
// consecutive (i, j) rows; per row the coarse rows and weights in i and j are
// fixed, and thread m writes the cells k = 2m (colour (i+j)&1) and k = 2m+1
// (the other colour), both at index m of their colour array.  Their k
// neighbours in the coarse rows are columns m-1, m (k = 2m, weight 0.75 on m)
// and m, m+1 (k = 2m+1, weight 0.25 on m+1), clamped at the ends: each lane
// loads column m of the four coarse rows and takes m-1 and m+1 from its
// neighbour lanes; both cells are formed in the order k, then j, then i.
constexpr int OUT_UP_ROWS = 16;
__global__ void out_up_kernel(const float *__restrict__ out0, Dims d0, const double *__restrict__ sumsq, float kscale,
                              Split sp, float *__restrict__ e)
{
    const double ms = *sumsq / (double)d0.n;
    const float sc = (float)sqrt(ms) * kscale;
    const long long rows = (long long)sp.nx * sp.ny;
    const int n0 = d0.nz;
    for (int q = 0; q < OUT_UP_ROWS; q++) {
        const long long row = (long long)blockIdx.x * OUT_UP_ROWS + q;   // i * ny + j
        if (row >= rows) break;
        const int i = (int)(row / sp.ny), j = (int)(row - (long long)i * sp.ny);
        const bool rin = i >= 1 && i <= sp.nx - 2 && j >= 1 && j <= sp.ny - 2;
        int ia, ib, ja, jb;
        float wi, wj;
        lin_coarse(i, d0.nx, ia, ib, wi);
        lin_coarse(j, d0.ny, ja, jb, wj);
        const float *p00 = out0 + vidx(d0, ia, ja, 0), *p01 = out0 + vidx(d0, ia, jb, 0);
        const float *p10 = out0 + vidx(d0, ib, ja, 0), *p11 = out0 + vidx(d0, ib, jb, 0);
        const int cc = (i + j) & 1;   // colour of k = 2m
        float *e0 = e + cc * sp.cs + row * sp.H, *e1 = e + (cc ^ 1) * sp.cs + row * sp.H;
        // whole warps run every pass (lanes past the row end hold the clamped
        // last coarse values), so the coarse neighbours m-1 and m+1 come from
        // the adjacent lanes; the lanes at a warp's edges load them
        const int lane = threadIdx.x & 31;
        const int Hw = (sp.H + 31) & ~31;
        for (int m = threadIdx.x; m < Hw; m += blockDim.x) {
            const int mc = min(m, n0 - 1);
            const int km = max(m - 1, 0), kp = min(m + 1, n0 - 1);
            const float b00 = p00[mc], b01 = p01[mc], b10 = p10[mc], b11 = p11[mc];
            float a00 = __shfl_up_sync(0xffffffffu, b00, 1), a01 = __shfl_up_sync(0xffffffffu, b01, 1);
            float a10 = __shfl_up_sync(0xffffffffu, b10, 1), a11 = __shfl_up_sync(0xffffffffu, b11, 1);
            float c00 = __shfl_down_sync(0xffffffffu, b00, 1), c01 = __shfl_down_sync(0xffffffffu, b01, 1);
            float c10 = __shfl_down_sync(0xffffffffu, b10, 1), c11 = __shfl_down_sync(0xffffffffu, b11, 1);
            if (lane == 0 || m == 0) {
                a00 = p00[km]; a01 = p01[km]; a10 = p10[km]; a11 = p11[km];
            }
            if (lane == 31 || m + 1 >= n0) {
                c00 = p00[kp]; c01 = p01[kp]; c10 = p10[kp]; c11 = p11[kp];
            }
            if (m >= sp.H) continue;
            const int k0 = 2 * m, k1 = 2 * m + 1;
            const bool in0 = rin && k0 >= 1 && k0 <= sp.nz - 2, in1 = rin && k1 >= 1 && k1 <= sp.nz - 2;
            float v0 = 0.f, v1 = 0.f;
            if (in0 || in1) {
                if (in0) {   // lin_coarse(2m): (m-1, m), weight 0.75 on m
                    const float wk = 0.75f;
                    const float s00 = a00 * (1.f - wk) + b00 * wk, s01 = a01 * (1.f - wk) + b01 * wk;
                    const float s10 = a10 * (1.f - wk) + b10 * wk, s11 = a11 * (1.f - wk) + b11 * wk;
                    const float t0 = s00 * (1.f - wj) + s01 * wj, t1 = s10 * (1.f - wj) + s11 * wj;
                    v0 = (t0 * (1.f - wi) + t1 * wi) * sc;
                }
                if (in1) {   // lin_coarse(2m+1): (m, m+1), weight 0.25 on m+1
                    const float wk = 0.25f;
                    const float s00 = b00 * (1.f - wk) + c00 * wk, s01 = b01 * (1.f - wk) + c01 * wk;
                    const float s10 = b10 * (1.f - wk) + c10 * wk, s11 = b11 * (1.f - wk) + c11 * wk;
                    const float t0 = s00 * (1.f - wj) + s01 * wj, t1 = s10 * (1.f - wj) + s11 * wj;
                    v1 = (t0 * (1.f - wi) + t1 * wi) * sc;
                }
            }
            e0[m] = v0;
            if (k1 < sp.nz) e1[m] = v1;
        }
    }
}

// training target: pooled (phi - phi0) / (rms * kscale) at the net voxels;
// sumt2 += target^2
__global__ void target_kernel(const double *__restrict__ phi, const double *__restrict__ phi0, Geom g, Dims d0,
                              const double *__restrict__ sumsq, float kscale, float *__restrict__ tgt,
                              double *__restrict__ sumt2)
{
    const double ms = *sumsq / (double)d0.n;
    const double inv = ms > 0.0 ? 1.0 / (sqrt(ms) * kscale) : 0.0;
    const long long sI = (long long)g.ny * g.nz, sJ = g.nz;
    double local = 0.0;
    UNET_LOOP(d0.n)
    {
        int I, J, K;
        voxel_ijk(d0, t, I, J, K);
        double s = 0.0;
        for (int c = 0; c < 8; c++) {
            const long long o = (2 * I + (c >> 2)) * sI + (2 * J + ((c >> 1) & 1)) * sJ + 2 * K + (c & 1);
            s += phi[o] - phi0[o];
        }
        const float v = (float)(0.125 * s * inv);
        tgt[t] = v;
        local += (double)v * v;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(sumt2, local);
}

// relative squared error: loss += (out - t)^2 / sumt2; dy channel 0 = its gradient
__global__ void loss_kernel(const float *__restrict__ out0, const float *__restrict__ tgt, long long n0, double sumt2,
                            __nv_bfloat16 *__restrict__ dy, double *__restrict__ loss)
{
    const float inv = sumt2 > 0.0 ? (float)(1.0 / sumt2) : 0.f;
    double local = 0.0;
    UNET_LOOP(n0 * 2)
    {
        const long long v = t >> 1;
        float f[8] = { 0, 0, 0, 0, 0, 0, 0, 0 };
        if ((t & 1) == 0) {
            const float r = out0[v] - tgt[v];
            f[0] = 2.f * r * inv;
            local += (double)r * r;
        }
        st8(dy + t * 8, f);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, local * (sumt2 > 0.0 ? 1.0 / sumt2 : 0.0));
}

// One of the 48 symmetries of the cube applied to a level-0 volume: output
// voxel (i0,i1,i2) reads input coordinate c[perm[a]] = flip[a] ? n-1-i_a : i_a
// (perm and flips packed in `sym`: bits 0-1, 2-3, 4-5 = perm, bits 6-8 = flips).
// Requires a cubic volume when perm is not the identity.
__global__ void symmetry_kernel(const float *__restrict__ in, float *__restrict__ out, Dims d, int sym)
{
    const int p[3] = { sym & 3, (sym >> 2) & 3, (sym >> 4) & 3 };
    const int n[3] = { d.nx, d.ny, d.nz };
    UNET_LOOP(d.n)
    {
        int o[3];
        voxel_ijk(d, t, o[0], o[1], o[2]);
        int c[3];
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const int v = ((sym >> (6 + a)) & 1) ? n[a] - 1 - o[a] : o[a];
            c[p[a]] = v;
        }
        out[t] = in[vidx(d, c[0], c[1], c[2])];
    }
}

__global__ void adam_kernel(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                            float *__restrict__ v, int n, float lr, float b1, float b2, float eps, float c1, float c2)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const float gt = g[t];
    const float mt = b1 * m[t] + (1.f - b1) * gt;
    const float vt = b2 * v[t] + (1.f - b2) * gt * gt;
    m[t] = mt;
    v[t] = vt;
    p[t] -= lr * (mt / c1) / (sqrtf(vt / c2) + eps);
}

// master FP32 weights of one conv -> BF16 forward layout [co][tap][ci] and
// input-gradient layout [ci][26-tap][co]
// The network's first convolution on the CUDA cores.  It has one input
// channel (the normalised pooled residual): not a GEMM worth the tensor
// cores, whose kernel would pad it to 16 channels and read a padded input
// volume.  A thread computes DK = 4 consecutive voxels along k of one (i, j)
// row: for each of the 9 (di, dj) neighbour rows it reads the 6 voxels
// k0-1 .. k0+4 once and applies the 3 k taps to all 4 outputs.  The weights
// of the tap in use sit in shared memory (read by broadcast); the
// multiply-adds are sm_100 packed FP32x2 operations.  The inputs are those of
// the tensor-core path -- the same BF16 values -- and FP32 accumulation, in
// another order, so outputs may differ from it in the last place.
constexpr int DK = 4;

// e0 = LeakyReLU(conv0(x) + bias), x = BF16(xin * s) with s = 1 / rms of xin
// (sumsq != NULL: rms^2 = *sumsq / n) or s = 1; zero padding; BF16 out, 16
// channels.  w: the BF16 weights [co][tap][ci] of the conv (ci = 0 used).
__global__ void __launch_bounds__(128) conv_first_kernel(const float *__restrict__ xin,
                                                         const double *__restrict__ sumsq, Dims d,
                                                         const __nv_bfloat16 *__restrict__ w,
                                                         const float *__restrict__ bias, __nv_bfloat16 *__restrict__ out)
{
    __shared__ float2 ws[NTAP][CH / 2];
    __shared__ float bs[CH];
    for (int q = threadIdx.x; q < NTAP * CH; q += blockDim.x) {
        const int tap = q / CH, co = q % CH;
        reinterpret_cast<float *>(&ws[tap][0])[co] = __bfloat162float(w[((size_t)co * NTAP + tap) * CH]);
    }
    if (threadIdx.x < CH) bs[threadIdx.x] = bias[threadIdx.x];
    __syncthreads();
    float sc = 1.f;
    if (sumsq) {
        const double ms = *sumsq / (double)d.n;
        sc = ms > 0.0 ? (float)(1.0 / sqrt(ms)) : 0.f;
    }
    const int nkb = d.nz / DK;
    const long long cols = (long long)nkb * d.ny * d.nx;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < cols;
         t += (long long)gridDim.x * blockDim.x) {
        const int kb = (int)(t % nkb);
        const long long r = t / nkb;
        const int j = (int)(r % d.ny), i = (int)(r / d.ny);
        const int k0 = kb * DK;
        float2 acc[DK][CH / 2];
#pragma unroll
        for (int kk = 0; kk < DK; kk++)
#pragma unroll
            for (int c = 0; c < CH / 2; c++) acc[kk][c] = make_float2(0.f, 0.f);
#pragma unroll 1
        for (int dij = 0; dij < 9; dij++) {
            const int a = i + dij / 3 - 1, b = j + dij % 3 - 1;
            if (a < 0 || a >= d.nx || b < 0 || b >= d.ny) continue;
            const float *row = xin + ((long long)a * d.ny + b) * d.nz;
            float x[DK + 2];
#pragma unroll
            for (int m = 0; m < DK + 2; m++) {
                const int k = k0 - 1 + m;
                x[m] = (k >= 0 && k < d.nz) ? __bfloat162float(__float2bfloat16(row[k] * sc)) : 0.f;
            }
#pragma unroll
            for (int dk = 0; dk < 3; dk++) {
                const float2 *wt = ws[dij * 3 + dk];
#pragma unroll
                for (int c = 0; c < CH / 2; c++) {
                    const float2 wc = wt[c];
#pragma unroll
                    for (int kk = 0; kk < DK; kk++) acc[kk][c] = __ffma2_rn(make_float2(x[kk + dk], x[kk + dk]), wc, acc[kk][c]);
                }
            }
        }
#pragma unroll
        for (int kk = 0; kk < DK; kk++) {
            float f0[8], f1[8];
#pragma unroll
            for (int c = 0; c < 4; c++) {
                f0[2 * c] = leaky(acc[kk][c].x + bs[2 * c]);
                f0[2 * c + 1] = leaky(acc[kk][c].y + bs[2 * c + 1]);
                f1[2 * c] = leaky(acc[kk][c + 4].x + bs[8 + 2 * c]);
                f1[2 * c + 1] = leaky(acc[kk][c + 4].y + bs[8 + 2 * c + 1]);
            }
            __nv_bfloat16 *o = out + vidx(d, i, j, k0 + kk) * CH;
            st8(o, f0);
            st8(o + 8, f1);
        }
    }
}

__global__ void pack_weights_kernel(const float *__restrict__ wm, __nv_bfloat16 *__restrict__ wf,
                                    __nv_bfloat16 *__restrict__ wt)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= WELEM) return;
    const int co = e / (NTAP * CH), tap = (e / CH) % NTAP, ci = e % CH;
    const __nv_bfloat16 b = __float2bfloat16(wm[e]);
    wf[e] = b;
    wt[((size_t)ci * NTAP + (NTAP - 1 - tap)) * CH + co] = b;
}

#undef UNET_LOOP

}  // namespace unet
}  // namespace hc
