// conservation.cu -- FP64 global sums of the conserved fields on the device.
//
// The reference's step is not exactly conservative: boundary cells are never
// flux-updated (hydro_solver_3d.c:729-731), the gravity source acts on every
// cell and is not in flux form (:597-631), and the floors add mass
// (:765-768).  The drift of total mass, momentum and energy is therefore the
// accuracy measure of a run, and it is formed here in FP64 from the
// device-resident state (FP64 or FP32 fields) without copying the state to
// the host.
//
// Order: the n cells are cut into CONS_BLOCKS contiguous pieces of fixed
// length (a function of n alone); in a piece, thread t adds the cells
// t, t + 256, ... in increasing order, the 32 lanes of a warp are combined by
// a fixed xor-shuffle tree and the 8 warps in index order; the block partials
// are added by the same scheme in a second kernel.  The result therefore does
// not depend on the device, the launch or the run: the same state gives the
// same bits.
#include <cuda_runtime.h>

#include "hc_internal.cuh"

namespace hc {
namespace {

constexpr int CONS_NT = 256;

template <typename T>
__global__ void __launch_bounds__(CONS_NT) cons_partial_kernel(ConsFields<T> q, long long n, long long piece,
                                                              double *partial)
{
    const long long lo = (long long)blockIdx.x * piece;
    const long long hi = (lo + piece < n) ? lo + piece : n;
    __shared__ double ws[5][CONS_NT / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll 1
    for (int f = 0; f < 5; f++) {
        const T *p = q.f[f];
        double acc = 0.0;
        long long c = lo + threadIdx.x;
        // four independent loads in flight, added in index order
        for (; c + 3 * CONS_NT < hi; c += 4 * CONS_NT) {
            const double a0 = (double)p[c], a1 = (double)p[c + CONS_NT];
            const double a2 = (double)p[c + 2 * CONS_NT], a3 = (double)p[c + 3 * CONS_NT];
            acc += a0;
            acc += a1;
            acc += a2;
            acc += a3;
        }
        for (; c < hi; c += CONS_NT) acc += (double)p[c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) ws[f][w] = acc;
    }
    __syncthreads();
    if (threadIdx.x < 5) {
        double s = 0.0;
        for (int t = 0; t < CONS_NT / 32; t++) s += ws[threadIdx.x][t];
        partial[(long long)threadIdx.x * CONS_BLOCKS + blockIdx.x] = s;
    }
}

// one warp per field
__global__ void cons_final_kernel(const double *partial, double *out)
{
    const int f = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (f >= 5) return;
    double acc = 0.0;
    for (int b = lane; b < CONS_BLOCKS; b += 32) acc += partial[(long long)f * CONS_BLOCKS + b];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) out[f] = acc;
}

}  // namespace

template <typename T>
cudaError_t cons_sums(const ConsFields<T> &q, long long n, double *partial, double *out, cudaStream_t s)
{
    const long long piece = (n + CONS_BLOCKS - 1) / CONS_BLOCKS;
    cons_partial_kernel<T><<<CONS_BLOCKS, CONS_NT, 0, s>>>(q, n, piece, partial);
    cons_final_kernel<<<1, 160, 0, s>>>(partial, out);
    return cudaGetLastError();
}

template cudaError_t cons_sums<double>(const ConsFields<double> &, long long, double *, double *, cudaStream_t);
template cudaError_t cons_sums<float>(const ConsFields<float> &, long long, double *, double *, cudaStream_t);

}  // namespace hc
