// hydro_fp32.cu -- FP32 instantiation of the hydro step kernels (FP32 state
// and HLLC arithmetic; the potential and g stay FP64).
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>

#include "hydro_kernels.cuh"
#include "hydro_fp32_pk.cuh"
#include "hydro_fp32_tma.cuh"

namespace hc {

namespace {
constexpr int TK = 32, TJ = 8;
__global__ void set_smax32(DevScalars *sc, int slot)
{
    sc->smax[slot] = (unsigned long long)__float_as_uint(1.0e-10f);
}
__global__ void cvt_to32(const double *a0, const double *a1, const double *a2, const double *a3,
                         const double *a4, float *b0, float *b1, float *b2, float *b3, float *b4,
                         long long n)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x) {
        b0[c] = (float)a0[c]; b1[c] = (float)a1[c]; b2[c] = (float)a2[c];
        b3[c] = (float)a3[c]; b4[c] = (float)a4[c];
    }
}
__global__ void cvt_to64(const float *a, double *b, long long n)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x)
        b[c] = (double)a[c];
}
inline int grid_for(long long n, int bs) { return (int)((n + bs - 1) / bs); }
}  // namespace

cudaError_t fp32_cfl_full(const HydroArgs &a, cudaStream_t s)
{
    set_smax32<<<1, 1, 0, s>>>(a.sc, a.step_parity);
    cfl_full_kernel<float><<<148 * 8, 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t fp32_dt(const HydroArgs &a, cudaStream_t s)
{
    dt_kernel<float><<<1, 1, 0, s>>>(a);
    return cudaGetLastError();
}

// TMA tensor map over the five FP32 fields of a state buffer:
// dims (k, j, i, field), box (40, 10, planes, 5) -- one (planes = 1) or two
// (planes = 2) plane tiles with halo.
static cudaError_t encode_state_map(const HydroArgs &a, CUtensorMap *tm, unsigned planes = 1)
{
    static PFN_cuTensorMapEncodeTiled_v12000 enc = nullptr;
    if (!enc) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn) return cudaErrorNotSupported;
        enc = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    }
    const cuuint64_t n = (cuuint64_t)a.g.n;
    cuuint64_t dims[4] = { (cuuint64_t)a.g.nz, (cuuint64_t)a.g.ny, (cuuint64_t)a.g.nx, 5 };
    cuuint64_t strides[3] = { (cuuint64_t)a.g.nz * 4, (cuuint64_t)a.g.ny * a.g.nz * 4, n * 4 };
    cuuint32_t box[4] = { (cuuint32_t)tma32::RK, (cuuint32_t)tma32::RJ, planes, 5 };
    cuuint32_t es[4] = { 1, 1, 1, 1 };
    CUresult r = enc(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<void *>(a.qin[0]), dims, strides, box,
                     es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

static bool tma_usable(const HydroArgs &a)
{
    static int off = -1;
    if (off < 0) {
        const char *e = getenv("HC_NO_TMA");
        off = (e && atoi(e) != 0) ? 1 : 0;
    }
    // row and field strides must be multiples of 16 bytes; fields contiguous
    return !off && (a.g.nz % 4) == 0 &&
           (const float *)a.qin[1] == (const float *)a.qin[0] + a.g.n &&
           (const float *)a.qin[4] == (const float *)a.qin[0] + 4 * a.g.n &&
           ((uintptr_t)a.qin[0] % 16) == 0;
}

// Interior kernel: "pk" (default; packed FP32x2, two planes per thread),
// "tma" (one plane per thread) or "plain" (no TMA), by HC_HYDRO32.
static int hydro32_choice()
{
    static int v = -1;
    if (v < 0) {
        const char *e = getenv("HC_HYDRO32");
        v = (e && !strcmp(e, "tma")) ? 1 : (e && !strcmp(e, "plain")) ? 2 : 0;
    }
    return v;
}

// Chunks along i for the packed kernel: the CTAs of all chunks run in waves
// of `slots`; a chunk of L planes (L even) costs about L/2 + 1 plane-pair
// steps (one for its prologue).  The chunk count minimising waves x steps.
static int pk_chunks(long long tiles, int nint, long long slots)
{
    int best = 1;
    double best_cost = 1e300;
    const int max_ch = std::max(1, nint / 8);
    for (int ch = 1; ch <= max_ch; ch++) {
        int ilen = (nint + ch - 1) / ch;
        ilen += ilen & 1;
        const int n = (nint + ilen - 1) / ilen;
        const long long waves = (tiles * n + slots - 1) / slots;
        const double cost = (double)waves * (ilen / 2 + 1);
        if (cost < best_cost - 1e-9) {
            best_cost = cost;
            best = n;
        }
    }
    return best;
}

static cudaError_t pk_interior(const HydroArgs &a, cudaStream_t s)
{
    CUtensorMap tm;
    cudaError_t e = encode_state_map(a, &tm, 2);
    if (e != cudaSuccess) return e;
    static std::atomic<unsigned long long> attr_set{0};
    e = set_smem_once(attr_set, (const void *)pk::interior_pk_kernel, (int)pk::SMEM);
    if (e != cudaSuccess) return e;
    static int slots_dev[64] = { 0 };
    int dev = 0;
    e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    int slots = (dev >= 0 && dev < 64) ? slots_dev[dev] : 0;
    if (!slots) {
        int per_sm = 0, sms = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pk::interior_pk_kernel, pk::NT, pk::SMEM);
        if (e != cudaSuccess) return e;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
        slots = std::max(1, per_sm) * sms;
        if (dev >= 0 && dev < 64) slots_dev[dev] = slots;
    }
    const long long tiles = (long long)((a.g.nz + pk::TK - 1) / pk::TK) * ((a.g.ny + pk::TJ - 1) / pk::TJ);
    const int nint = a.g.nx - 2;
    const int ch = pk_chunks(tiles, nint, slots);
    int ilen = (nint + ch - 1) / ch;
    ilen += ilen & 1;
    const int n = (nint + ilen - 1) / ilen;
    dim3 grid((a.g.nz + pk::TK - 1) / pk::TK, (a.g.ny + pk::TJ - 1) / pk::TJ, n);
    pk::interior_pk_kernel<<<grid, dim3(pk::TK, pk::TJ), pk::SMEM, s>>>(tm, a, ilen);
    return cudaGetLastError();
}

cudaError_t fp32_interior(const HydroArgs &a, int chunks, cudaStream_t s)
{
    if (hydro32_choice() == 0 && tma_usable(a)) {
        cudaError_t e = pk_interior(a, s);
        if (e != cudaErrorInvalidValue) return e;   // the map could not be encoded: next kernel
    }
    if (hydro32_choice() <= 1 && tma_usable(a)) {
        CUtensorMap tm;
        cudaError_t e = encode_state_map(a, &tm);
        if (e == cudaSuccess) {
            // 4 CTAs per SM, about 4 waves
            long long tiles = (long long)((a.g.nz + tma32::TK - 1) / tma32::TK) * ((a.g.ny + tma32::TJ - 1) / tma32::TJ);
            long long want = 148LL * 4 * 4;
            int nint = a.g.nx - 2;
            int ch = (int)std::max(1LL, std::min((want + tiles - 1) / tiles, (long long)std::max(1, nint / 8)));
            int ilen = (nint + ch - 1) / ch;
            ch = (nint + ilen - 1) / ilen;
            dim3 grid((a.g.nz + tma32::TK - 1) / tma32::TK, (a.g.ny + tma32::TJ - 1) / tma32::TJ, ch);
            tma32::interior_tma_kernel<<<grid, dim3(tma32::TK, tma32::TJ), 0, s>>>(tm, a, ilen);
            return cudaGetLastError();
        }
    }
    constexpr size_t sm = interior_smem<float, TK, TJ>();
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(interior_kernel<float, TK, TJ>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    int nint = a.g.nx - 2;
    int ilen = (nint + chunks - 1) / chunks;
    chunks = (nint + ilen - 1) / ilen;
    dim3 grid((a.g.nz + TK - 1) / TK, (a.g.ny + TJ - 1) / TJ, chunks);
    interior_kernel<float, TK, TJ><<<grid, dim3(TK, TJ), sm, s>>>(a, ilen);
    return cudaGetLastError();
}

cudaError_t fp32_boundary_source(const HydroArgs &a, cudaStream_t s)
{
    long long nb = boundary_count(a.g.nx, a.g.ny, a.g.nz, true);
    boundary_source_kernel<float><<<grid_for(nb, 256), 256, 0, s>>>(a);
    return cudaGetLastError();
}

static long long face_count(const HydroArgs &a, int axis)
{
    const int n[3] = { a.g.nx, a.g.ny, a.g.nz };
    return (long long)((axis == 0) ? n[1] : n[0]) * ((axis == 2) ? n[1] : n[2]);
}

cudaError_t fp32_periodic(const HydroArgs &a, int axis, cudaStream_t s)
{
    periodic_kernel<float><<<grid_for(face_count(a, axis), 256), 256, 0, s>>>(a, axis);
    return cudaGetLastError();
}

cudaError_t fp32_bc(const HydroArgs &a, int axis, cudaStream_t s)
{
    bc_kernel<float><<<grid_for(face_count(a, axis), 256), 256, 0, s>>>(a, axis);
    return cudaGetLastError();
}

cudaError_t fp32_cfl_boundary(const HydroArgs &a, cudaStream_t s)
{
    long long nb = boundary_count(a.g.nx, a.g.ny, a.g.nz, true);
    int blocks = (int)std::min<long long>(grid_for(nb, 256), 148 * 4);
    cfl_boundary_kernel<float><<<blocks, 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t fp32_from_fp64(const double *const q64[5], float *const q32[5], long long n, cudaStream_t s)
{
    cvt_to32<<<148 * 8, 256, 0, s>>>(q64[0], q64[1], q64[2], q64[3], q64[4], q32[0], q32[1], q32[2],
                                     q32[3], q32[4], n);
    return cudaGetLastError();
}

cudaError_t fp32_to_fp64(const float *const q32[5], double *const q64[5], long long n, cudaStream_t s)
{
    for (int v = 0; v < 5; v++) cvt_to64<<<148 * 8, 256, 0, s>>>(q32[v], q64[v], n);
    return cudaGetLastError();
}

namespace {
__global__ void aos64_to_soa32(const double *aos, float *q0, float *q1, float *q2, float *q3, float *q4,
                               long long n)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x) {
        const double *p = aos + 5 * c;
        q0[c] = (float)p[0]; q1[c] = (float)p[1]; q2[c] = (float)p[2];
        q3[c] = (float)p[3]; q4[c] = (float)p[4];
    }
}
__global__ void soa32_to_aos64(const float *q0, const float *q1, const float *q2, const float *q3,
                               const float *q4, double *aos, long long n)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x) {
        double *p = aos + 5 * c;
        p[0] = q0[c]; p[1] = q1[c]; p[2] = q2[c]; p[3] = q3[c]; p[4] = q4[c];
    }
}
}  // namespace

cudaError_t fp32_from_aos64(const double *aos, float *const q[5], long long n, cudaStream_t s)
{
    aos64_to_soa32<<<148 * 8, 256, 0, s>>>(aos, q[0], q[1], q[2], q[3], q[4], n);
    return cudaGetLastError();
}

cudaError_t fp32_to_aos64(const float *const q[5], double *aos, long long n, cudaStream_t s)
{
    soa32_to_aos64<<<148 * 8, 256, 0, s>>>(q[0], q[1], q[2], q[3], q[4], aos, n);
    return cudaGetLastError();
}

cudaError_t f32_to_f64(const float *a, double *b, long long n, cudaStream_t s)
{
    cvt_to64<<<148 * 8, 256, 0, s>>>(a, b, n);
    return cudaGetLastError();
}

}  // namespace hc
