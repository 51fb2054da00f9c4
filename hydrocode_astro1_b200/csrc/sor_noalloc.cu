// sor_noalloc.cu -- red-black SOR to tolerance on caller-owned device arrays,
// without allocating any memory.
//
// Who needs this: a host code that embeds the Poisson solve in its own time
// loop and owns all device memory itself -- a fixed arena reserved at start-up,
// a memory pool shared with other solvers, or a budget that must not grow (or
// fail with out-of-memory) in the middle of a run.  cudaMalloc/cudaFree can
// also synchronise the whole device, which such a caller's other streams must
// not see.  hc_sor_solve_noalloc therefore calls no cudaMalloc, cudaFree or
// allocating library routine: the caller passes phi (in/out) and rho, and the
// only scratch -- one residual slot per iteration plus three words of flags -- is the
// file-scope array below, a fixed 512 KB per GPU that loads the library,
// held until the process exits.
//
// The arithmetic is that of the context path (red-black sweeps of
// gravity_solver_3d.c:642-708 with its stop rule, :715), so the iterates are
// the same bit for bit.  The boundary cells of phi are kept as given.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "hc_internal.cuh"
#include "hc_math.cuh"

namespace {

// Slot t (t < HC_NOALLOC_MAX_ITER) holds the bits of iteration t's max update;
// [HC_NOALLOC_MAX_ITER] is the stop flag, [HC_NOALLOC_MAX_ITER + 1] the
// iteration count at which the solve stopped, [HC_NOALLOC_MAX_ITER + 2] the
// bits of the last executed iteration's update norm (written by check_kernel,
// so the host reads flags and residual with one copy on the caller's stream).
static __device__ __align__(256) unsigned long long g_sor_scratch[HC_NOALLOC_MAX_ITER + 8];

struct Sor {
    double *phi;
    const double *rho;
    int nx, ny, nz;
    double ix2, iy2, iz2, fpg, fac, om, tol;
    unsigned long long *scr;
};

__device__ __forceinline__ double slot(const Sor &a, int t)
{
    return __longlong_as_double((long long)a.scr[t]);
}

__global__ void clear_kernel(unsigned long long *scr, int n)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) scr[t] = 0ull;
    if (blockIdx.x == 0 && threadIdx.x < 8) scr[HC_NOALLOC_MAX_ITER + threadIdx.x] = 0ull;
}

// iteration `iter` starts only if iteration iter-1 left the update norm >= tol
__device__ __forceinline__ bool stop_here(const Sor &a, int iter)
{
    volatile unsigned long long *flags = a.scr + HC_NOALLOC_MAX_ITER;
    if (flags[0]) return true;
    if (iter > 0 && slot(a, iter - 1) < a.tol) {
        if (threadIdx.x == 0 && threadIdx.y == 0) {
            a.scr[HC_NOALLOC_MAX_ITER + 1] = (unsigned long long)iter;
            a.scr[HC_NOALLOC_MAX_ITER] = 1ull;
        }
        return true;
    }
    return false;
}

constexpr int BX = 32, BY = 8;

__global__ void __launch_bounds__(BX * BY) colour_kernel(Sor a, int color, int iter)
{
    if (stop_here(a, color == 0 ? iter : -1)) return;
    const int i = 1 + blockIdx.z;
    const int j = 1 + blockIdx.y * BY + threadIdx.y;
    const int k0 = ((i + j + 1) % 2 == color) ? 1 : 2;
    const int k = k0 + 2 * (blockIdx.x * BX + threadIdx.x);
    double r = 0.0;
    if (j <= a.ny - 2 && k <= a.nz - 2) {
        const long long sI = (long long)a.ny * a.nz, sJ = a.nz;
        const long long c = i * sI + j * sJ + k;
        double *phi = a.phi;
        double old = phi[c];
        double lap = (phi[c - sI] + phi[c + sI]) * a.ix2 + (phi[c - sJ] + phi[c + sJ]) * a.iy2 +
                     (phi[c - 1] + phi[c + 1]) * a.iz2;
        double nw = (lap - a.fpg * a.rho[c]) / a.fac;
        phi[c] = old + a.om * (nw - old);
        r = fabs(nw - old);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r = hc::tmax(r, __shfl_xor_sync(0xffffffffu, r, o));
    __shared__ double w[BX * BY / 32];
    const int tid = threadIdx.y * BX + threadIdx.x;
    if ((tid & 31) == 0) w[tid >> 5] = r;
    __syncthreads();
    if (tid == 0) {
        double m = 0.0;
        for (int t = 0; t < BX * BY / 32; t++) m = hc::tmax(m, w[t]);
        atomicMax(a.scr + iter, (unsigned long long)__double_as_longlong(m));
    }
}

// End of a batch of `iter` queued iterations: sets the stop flag if the last
// one converged, then records the norm of the last iteration that ran.
__global__ void check_kernel(Sor a, int iter)
{
    stop_here(a, iter);
    const unsigned long long *flags = a.scr + HC_NOALLOC_MAX_ITER;
    const int used = flags[0] ? (int)flags[1] : iter;
    a.scr[HC_NOALLOC_MAX_ITER + 2] = a.scr[used - 1];
}

// Device address of the scratch array, looked up once per device with that
// device current (in host code the symbol name is only a host-side stand-in).
std::mutex g_mu;
unsigned long long *g_scr_dev[64] = { nullptr };

cudaError_t scratch_for_current_device(unsigned long long **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scr_dev[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_sor_scratch);
        if (e != cudaSuccess) return e;
        // load the three kernels now (lazy module loading would otherwise do
        // it, and may allocate, at their first launch)
        cudaFuncAttributes fa;
        if ((e = cudaFuncGetAttributes(&fa, clear_kernel)) != cudaSuccess) return e;
        if ((e = cudaFuncGetAttributes(&fa, colour_kernel)) != cudaSuccess) return e;
        if ((e = cudaFuncGetAttributes(&fa, check_kernel)) != cudaSuccess) return e;
        g_scr_dev[dev] = static_cast<unsigned long long *>(p);
    }
    *out = g_scr_dev[dev];
    return cudaSuccess;
}

}  // namespace

int hc_internal_set_error(int code, const char *msg);

// HC_ERR_CUDA with `what` and the CUDA error's text as the message.
static int cuda_fail(const char *what, cudaError_t e)
{
    char msg[256];
    snprintf(msg, sizeof msg, "hc_sor_solve_noalloc: %s: %s", what, cudaGetErrorString(e));
    return hc_internal_set_error(HC_ERR_CUDA, msg);
}

extern "C" int hc_sor_solve_noalloc(double *phi, const double *rho, int nx, int ny, int nz, double dx,
                                    double dy, double dz, double G, double omega, int max_iter,
                                    double tol, void *stream, int *iterations, double *residual)
{
    if (!phi || !rho) return hc_internal_set_error(HC_ERR_ARG, "hc_sor_solve_noalloc: null phi or rho");
    if (nx < 3 || ny < 3 || nz < 3)
        return hc_internal_set_error(HC_ERR_ARG, "hc_sor_solve_noalloc: every dimension needs at least 3 cells");
    if (max_iter < 1 || max_iter > HC_NOALLOC_MAX_ITER)
        return hc_internal_set_error(HC_ERR_ARG, "hc_sor_solve_noalloc: max_iter must be in 1..65536 "
                                                 "(the fixed scratch holds one slot per iteration)");
    if (!(dx > 0.0) || !(dy > 0.0) || !(dz > 0.0))
        return hc_internal_set_error(HC_ERR_ARG, "hc_sor_solve_noalloc: cell sizes must be positive");
    if (!(omega > 0.0 && omega < 2.0))
        return hc_internal_set_error(HC_ERR_ARG, "hc_sor_solve_noalloc: omega must lie in (0, 2)");
    if (!(tol > 0.0) || !std::isfinite(tol))
        return hc_internal_set_error(HC_ERR_ARG, "hc_sor_solve_noalloc: tol must be finite and positive");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Sor a;
    a.phi = phi;
    a.rho = rho;
    a.nx = nx; a.ny = ny; a.nz = nz;
    // gravity_solver_3d.c:519-545
    a.ix2 = 1.0 / (dx * dx);
    a.iy2 = 1.0 / (dy * dy);
    a.iz2 = 1.0 / (dz * dz);
    a.fpg = 4.0 * M_PI * G;
    a.fac = 2.0 * (a.ix2 + a.iy2 + a.iz2);
    a.om = omega;
    a.tol = tol;
    cudaError_t e = scratch_for_current_device(&a.scr);
    if (e != cudaSuccess)
        return cuda_fail("scratch address lookup failed", e);

    clear_kernel<<<64, 256, 0, s>>>(a.scr, max_iter + 1);
    const dim3 grid(((nz - 1) / 2 + BX - 1) / BX, (ny - 2 + BY - 1) / BY, nx - 2);
    const dim3 block(BX, BY);
    int it = 0, batch = 16;
    // stop flag, stopping iteration, bits of the last executed iteration's norm
    unsigned long long flags[3] = { 0ull, 0ull, 0ull };
    while (true) {
        const int end = (max_iter - it < batch) ? max_iter : it + batch;
        for (int q = it; q < end; q++) {
            colour_kernel<<<grid, block, 0, s>>>(a, 0, q);
            colour_kernel<<<grid, block, 0, s>>>(a, 1, q);
        }
        check_kernel<<<1, 1, 0, s>>>(a, end);
        if ((e = cudaGetLastError()) != cudaSuccess)
            return cuda_fail("kernel launch failed", e);
        if ((e = cudaMemcpyAsync(flags, a.scr + HC_NOALLOC_MAX_ITER, sizeof flags, cudaMemcpyDeviceToHost,
                                 s)) != cudaSuccess ||
            (e = cudaStreamSynchronize(s)) != cudaSuccess)
            return cuda_fail("reading the stop flag failed", e);
        if (flags[0] || end >= max_iter) break;
        it = end;
        batch = batch < 256 ? 2 * batch : 256;
    }
    const int used = flags[0] ? (int)flags[1] : max_iter;
    if (iterations) *iterations = used;
    if (residual) memcpy(residual, &flags[2], sizeof(double));
    return flags[0] ? HC_OK : HC_NOT_CONVERGED;
}
