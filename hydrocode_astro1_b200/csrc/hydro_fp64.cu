// hydro_fp64.cu -- FP64 instantiation of the hydro step kernels.
// Built with -fmad=false: with the reference's operand order and no fused
// multiply-add, every value is bit-identical to the reference C build.
#include "hydro_kernels.cuh"

namespace hc {

namespace {
constexpr int TK = 32, TJ = 8;
__global__ void set_smax64(DevScalars *sc, int slot)
{
    sc->smax[slot] = (unsigned long long)__double_as_longlong(1.0e-10);
}
__global__ void aos_to_soa64(const double *aos, double *q0, double *q1, double *q2, double *q3,
                             double *q4, long long n)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x) {
        const double *p = aos + 5 * c;
        q0[c] = p[0]; q1[c] = p[1]; q2[c] = p[2]; q3[c] = p[3]; q4[c] = p[4];
    }
}
__global__ void soa_to_aos64(const double *q0, const double *q1, const double *q2,
                             const double *q3, const double *q4, double *aos, long long n)
{
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x) {
        double *p = aos + 5 * c;
        p[0] = q0[c]; p[1] = q1[c]; p[2] = q2[c]; p[3] = q3[c]; p[4] = q4[c];
    }
}
inline int grid_for(long long n, int bs) { return (int)((n + bs - 1) / bs); }
}  // namespace

cudaError_t fp64_cfl_full(const HydroArgs &a, cudaStream_t s)
{
    set_smax64<<<1, 1, 0, s>>>(a.sc, a.step_parity);
    cfl_full_kernel<double><<<148 * 8, 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t fp64_dt(const HydroArgs &a, cudaStream_t s)
{
    dt_kernel<double><<<1, 1, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t fp64_interior(const HydroArgs &a, int chunks, cudaStream_t s)
{
    constexpr size_t sm = interior_smem<double, TK, TJ>();
    static std::atomic<unsigned long long> attr_set{0};
    cudaError_t e = set_smem_once(attr_set, (const void *)interior_kernel<double, TK, TJ>, (int)sm);
    if (e != cudaSuccess) return e;
    int nint = a.g.nx - 2;
    int ilen = (nint + chunks - 1) / chunks;
    chunks = (nint + ilen - 1) / ilen;
    dim3 grid((a.g.nz + TK - 1) / TK, (a.g.ny + TJ - 1) / TJ, chunks);
    interior_kernel<double, TK, TJ><<<grid, dim3(TK, TJ), sm, s>>>(a, ilen);
    return cudaGetLastError();
}

cudaError_t fp64_boundary_source(const HydroArgs &a, cudaStream_t s)
{
    long long nb = boundary_count(a.g.nx, a.g.ny, a.g.nz, true);
    boundary_source_kernel<double><<<grid_for(nb, 256), 256, 0, s>>>(a);
    return cudaGetLastError();
}

static long long face_count(const HydroArgs &a, int axis)
{
    const int n[3] = { a.g.nx, a.g.ny, a.g.nz };
    return (long long)((axis == 0) ? n[1] : n[0]) * ((axis == 2) ? n[1] : n[2]);
}

cudaError_t fp64_periodic(const HydroArgs &a, int axis, cudaStream_t s)
{
    periodic_kernel<double><<<grid_for(face_count(a, axis), 256), 256, 0, s>>>(a, axis);
    return cudaGetLastError();
}

cudaError_t fp64_bc(const HydroArgs &a, int axis, cudaStream_t s)
{
    bc_kernel<double><<<grid_for(face_count(a, axis), 256), 256, 0, s>>>(a, axis);
    return cudaGetLastError();
}

cudaError_t fp64_cfl_boundary(const HydroArgs &a, cudaStream_t s)
{
    long long nb = boundary_count(a.g.nx, a.g.ny, a.g.nz, true);
    int blocks = (int)std::min<long long>(grid_for(nb, 256), 148 * 4);
    cfl_boundary_kernel<double><<<blocks, 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t fp64_aos_to_soa(const double *aos, double *const q[5], long long n, cudaStream_t s)
{
    aos_to_soa64<<<148 * 8, 256, 0, s>>>(aos, q[0], q[1], q[2], q[3], q[4], n);
    return cudaGetLastError();
}

cudaError_t fp64_soa_to_aos(const double *const q[5], double *aos, long long n, cudaStream_t s)
{
    soa_to_aos64<<<148 * 8, 256, 0, s>>>(q[0], q[1], q[2], q[3], q[4], aos, n);
    return cudaGetLastError();
}

}  // namespace hc
