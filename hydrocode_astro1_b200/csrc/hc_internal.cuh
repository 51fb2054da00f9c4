// hc_internal.cuh -- device context and kernel entry points shared by the
// translation units of the B200 hydro + gravity library.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>

#include "../../include/hydrocode_b200.h"

namespace hc {

// Raises a kernel's dynamic shared-memory limit once per device: `done` holds
// one bit per device ordinal (below 64; beyond that the attribute is set on
// every call).  Two threads may both set it the first time, which is harmless.
inline cudaError_t set_smem_once(std::atomic<unsigned long long> &done, const void *fn, int bytes)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned long long bit = (dev >= 0 && dev < 64) ? (1ull << dev) : 0ull;
    if (bit && (done.load(std::memory_order_acquire) & bit)) return cudaSuccess;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess && bit) done.fetch_or(bit, std::memory_order_release);
    return e;
}

}  // namespace hc


namespace hc {

// Grid geometry as the kernels see it.
struct Geom {
    int nx, ny, nz;
    long long n;               // nx*ny*nz
    double xmin, xmax, ymin, ymax, zmin, zmax;
    double dx, dy, dz;         // (max-min)/n, hydro_solver_3d.c:55-57
    // A slab of a grid split along x: the context holds global planes
    // [ioff, ioff + nx) of gnx; its own planes are local [olo, ohi), the
    // others ghost copies of a neighbour's.  xmin/xmax/dx are then the whole
    // grid's, x = xmin + (i + ioff + 0.5) dx.  A whole grid: 0, nx, 0, nx.
    int ioff, gnx, olo, ohi;
};

// Bitwise-ordered atomic max of a non-negative double (the bit pattern of a
// non-negative IEEE double grows with its value).
__device__ __forceinline__ void atomic_max_nonneg(unsigned long long *slot, double v)
{
    atomicMax(slot, (unsigned long long)__double_as_longlong(v));
}
__device__ __forceinline__ void atomic_max_nonneg(unsigned int *slot, float v)
{
    atomicMax(slot, (unsigned int)__float_as_uint(v));
}

// Device scalars of one context (one cudaMalloc'd struct).
struct DevScalars {
    unsigned long long smax[2];   // CFL max signal speed (bits), ping-pong per step
    double dt;                    // current step dt
    int done;                     // SOR converged / stopped flag
    int last_iter;                // iterations of the finished solve
    int overshoot;                // temporal blocking passed tol inside a pass
    int err;                      // sticky device error code
    unsigned long long resid_bits; // scratch
    double moments[4 + 9];        // M, COM, Q (reference mode)
    double resnorm;               // post-hoc residual
    double cons[5];               // FP64 sums of rho, rho u, rho v, rho w, E
};

// Boundary-cell enumeration: index t in [0, nb) -> (i,j,k) on the faces.
// zb: whether the z faces are boundary (false in the nz == 1 gravity mode).
__host__ __device__ __forceinline__ long long boundary_count(int nx, int ny, int nz, bool zb)
{
    if (zb) return 2LL * ny * nz + 2LL * (nx - 2) * nz + 2LL * (nx - 2) * (ny - 2);
    return (2LL * ny + 2LL * (nx - 2)) * nz;
}
__device__ __forceinline__ void boundary_cell(long long t, int nx, int ny, int nz, bool zb,
                                              int &i, int &j, int &k)
{
    long long a = 2LL * ny * nz;
    if (t < a) {
        i = (t < (long long)ny * nz) ? 0 : nx - 1;
        long long r = t % ((long long)ny * nz);
        j = (int)(r / nz); k = (int)(r % nz);
        return;
    }
    t -= a;
    long long b = 2LL * (nx - 2) * nz;
    if (t < b) {
        j = (t < (long long)(nx - 2) * nz) ? 0 : ny - 1;
        long long r = t % ((long long)(nx - 2) * nz);
        i = 1 + (int)(r / nz); k = (int)(r % nz);
        return;
    }
    t -= b;
    // z faces (only when zb)
    k = (t < (long long)(nx - 2) * (ny - 2)) ? 0 : nz - 1;
    long long r = t % ((long long)(nx - 2) * (ny - 2));
    i = 1 + (int)(r / (ny - 2)); j = 1 + (int)(r % (ny - 2));
}

}  // namespace hc

// ---------------------------------------------------------------------------
// Launchers implemented in the kernel translation units (host functions).
// All take the context's stream and return cudaError_t of the launch.
// ---------------------------------------------------------------------------
namespace hc {

struct HydroArgs {
    Geom g;
    double gamma, cfl;
    int bc[6];
    int gravity;
    const void *qin[5];     // double* or float* per precision
    void *qout[5];
    const double *phig;     // potential used for g (last converged)
    DevScalars *sc;
    int step_parity;        // smax slot read = parity, written = parity^1
};

// FP64 (bit-exact) hydro path -- hydro_fp64.cu
cudaError_t fp64_cfl_full(const HydroArgs &a, cudaStream_t s);
cudaError_t fp64_dt(const HydroArgs &a, cudaStream_t s);
cudaError_t fp64_interior(const HydroArgs &a, int chunks, cudaStream_t s);
cudaError_t fp64_boundary_source(const HydroArgs &a, cudaStream_t s);
cudaError_t fp64_periodic(const HydroArgs &a, int axis, cudaStream_t s);
cudaError_t fp64_bc(const HydroArgs &a, int axis, cudaStream_t s);
cudaError_t fp64_cfl_boundary(const HydroArgs &a, cudaStream_t s);
cudaError_t fp64_aos_to_soa(const double *aos, double *const q[5], long long n, cudaStream_t s);
cudaError_t fp64_soa_to_aos(const double *const q[5], double *aos, long long n, cudaStream_t s);
// profile-based initial state on the device -- ics_device.cu
cudaError_t ic_profile_stars(const Geom &g, double gamma, int nstars, const int *n, const double *const *r,
                             const double *const *rho, const double *const *u, const double *R_star,
                             const double *centre, const double *vel, double *const q64[5], float *const q32[5],
                             double *scratch, cudaStream_t s);
// opt-in MUSCL-Hancock interior update (FP64) -- hydro_plm.cu; pl: 20 n doubles of scratch
cudaError_t fp64_plm_interior(const HydroArgs &a, double *pl, cudaStream_t s);

// FP64 global sums of the 5 conserved fields (fixed order) -- conservation.cu.
// partial: 5 * CONS_BLOCKS doubles of scratch; out: 5 doubles (device).
constexpr int CONS_BLOCKS = 1184;
template <typename T>
struct ConsFields {
    const T *f[5];
};
template <typename T>
cudaError_t cons_sums(const ConsFields<T> &q, long long n, double *partial, double *out, cudaStream_t s);

// FP32 hydro path -- hydro_fp32.cu
cudaError_t fp32_cfl_full(const HydroArgs &a, cudaStream_t s);
cudaError_t fp32_dt(const HydroArgs &a, cudaStream_t s);
cudaError_t fp32_interior(const HydroArgs &a, int chunks, cudaStream_t s);
cudaError_t fp32_boundary_source(const HydroArgs &a, cudaStream_t s);
cudaError_t fp32_periodic(const HydroArgs &a, int axis, cudaStream_t s);
cudaError_t fp32_bc(const HydroArgs &a, int axis, cudaStream_t s);
cudaError_t fp32_cfl_boundary(const HydroArgs &a, cudaStream_t s);
cudaError_t fp32_from_fp64(const double *const q64[5], float *const q32[5], long long n, cudaStream_t s);
cudaError_t fp32_to_fp64(const float *const q32[5], double *const q64[5], long long n, cudaStream_t s);
cudaError_t f32_to_f64(const float *a, double *b, long long n, cudaStream_t s);
cudaError_t fp32_from_aos64(const double *aos, float *const q[5], long long n, cudaStream_t s);
cudaError_t fp32_to_aos64(const float *const q[5], double *aos, long long n, cudaStream_t s);

struct GravArgs {
    Geom g;
    double G, omega, tol;
    int max_iter;
    int sweep_kind;           // FP32 correction colour sweeps: 0 register vector sweeps,
                              // 1 TMA-staged where the layout allows
    int grav_bc;
    int lmax;
    int moment_order;
    double *phi;
    const double *rho;        // FP64 density (parity path)
    const float *rho32;       // FP32 density (mixed path) -- used when rho == NULL
    double *res;              // per-iteration residual slots (bits), max_iter+1
    DevScalars *sc;
    double *scratch;          // moment partial sums
    long long scratch_len;
    double *mom;              // multipole results: 4 + ncoef
    double *gx, *gy, *gz;
};

// FP64 gravity (bit-exact) -- gravity_fp64.cu
cudaError_t grav_moments_sequential(const GravArgs &a, cudaStream_t s);
cudaError_t grav_moments_tree(const GravArgs &a, cudaStream_t s);
// Moments of a slab (own planes [a.g.olo, a.g.ohi)).  Sequential order:
// pass 0 / 1 continues the sums acc[0..4) / acc[0..9) (device memory) over
// the own planes in cell order; grav_moments_seq_set stores the finished
// sums (pass 0: M and the centre of mass; pass 1: Q).  Tree order: one
// partial (9 doubles) per own plane into parts; grav_moments_tree_set adds
// nparts partials of the whole grid in plane order.
cudaError_t grav_moments_seq_slab(const GravArgs &a, int pass, double *acc, cudaStream_t s);
cudaError_t grav_moments_seq_set(const GravArgs &a, int pass, const double *acc, cudaStream_t s);
cudaError_t grav_moments_tree_parts(const GravArgs &a, int pass, double *parts, cudaStream_t s);
cudaError_t grav_moments_tree_set(const GravArgs &a, int pass, const double *parts, int nparts, cudaStream_t s);
cudaError_t grav_boundary_ref(const GravArgs &a, cudaStream_t s);
cudaError_t grav_boundary_periodic(const GravArgs &a, cudaStream_t s);
cudaError_t grav_sor_color(const GravArgs &a, int color, int iter, cudaStream_t s);
cudaError_t grav_sor_wavefront(const GravArgs &a, int iter0, int depth, cudaStream_t s);
cudaError_t grav_check(const GravArgs &a, int iter, cudaStream_t s);
cudaError_t grav_accel(const GravArgs &a, cudaStream_t s);
cudaError_t grav_residual_norm(const GravArgs &a, const double *phi, cudaStream_t s);
cudaError_t grav_reset_slots(const GravArgs &a, int from, int count, cudaStream_t s);

// Multipole to lmax and mixed precision -- gravity_mixed.cu
cudaError_t grav_moments_lmax(const GravArgs &a, cudaStream_t s);
cudaError_t grav_boundary_lmax(const GravArgs &a, cudaStream_t s);
int lmax_ncoef(int lmax);
// Moment scratch of a context (doubles): per-plane partials, then the rows'
// z-power sums.
long long grav_scratch_len(const Geom &g);
// lmax moments of a slab: pass 0 writes the centre-of-mass partials, pass 1
// the rows' harmonic partials, lmax_slab_width(g, pass) doubles per own
// plane; grav_moments_lmax_set adds the partials of nplanes planes of the
// whole grid in plane order (pass 0: M and the centre of mass; pass 1: the
// coefficients).
int lmax_slab_width(const Geom &g, int pass);
cudaError_t grav_moments_lmax_parts(const GravArgs &a, int pass, double *parts, cudaStream_t s);
cudaError_t grav_moments_lmax_set(const GravArgs &a, int pass, const double *parts, int nplanes, cudaStream_t s);

}  // namespace hc

namespace hc {
// split: r32 / e32 in the colour-split layout of sor_split.cuh
cudaError_t mixed_residual(const GravArgs &a, float *r32, float *e32, bool split, cudaStream_t s);
cudaError_t mixed_update(const GravArgs &a, const float *e32, bool split, float sign, cudaStream_t s);
cudaError_t mixed_sor32_split(const GravArgs &a, float *e32, const float *r32, int colour, int iter,
                              double thresh, cudaStream_t s);
cudaError_t mixed_sor32(const GravArgs &a, float *e32, const float *r32, int color, int iter,
                        double thresh, cudaStream_t s);
cudaError_t mixed_check(const GravArgs &a, int iter, double thresh, cudaStream_t s);
// two FP32 correction iterations per pass on the colour-split layout, ein -> eout
bool mixed_wave_split_ok(const Geom &g);
cudaError_t mixed_sor32_split_pass(const GravArgs &a, const float *ein, float *eout, const float *r32, int iter0,
                                   double thresh, cudaStream_t s);
}  // namespace hc

namespace hc {
cudaError_t grav_sor_pass64(const GravArgs &a, const double *in, double *out, int iter0, cudaStream_t s);
// colour-split FP64 SOR (sor_split.cuh): elements of a split field, natural
// -> split copies of phi (and rho), boundary cells only, split -> natural phi,
// one colour sweep
long long split_len(const Geom &g);
cudaError_t grav_split_fields(const GravArgs &a, double *phs, double *rhs, cudaStream_t s);
cudaError_t grav_split_boundary(const GravArgs &a, double *phs, cudaStream_t s);
cudaError_t grav_unsplit(const GravArgs &a, const double *phs, cudaStream_t s);
cudaError_t grav_sor_split(const GravArgs &a, double *phs, const double *rhs, int colour, int iter, cudaStream_t s);
cudaError_t mixed_sor32_pass(const GravArgs &a, const float *in, float *out, const float *r32, int iter0,
                             int depth, double thresh, cudaStream_t s);
}  // namespace hc

// Learned warm start (unet.cu): a 3D U-Net on the half-resolution grid that
// predicts the correction of a mixed-precision solve from its first residual.
namespace hc {
struct UNetState;
int unet_param_count();
UNetState *unet_create(int dev);
void unet_destroy(UNetState *u);
bool unet_has_weights(const UNetState *u);
float unet_kscale(const UNetState *u);
int unet_set_params(UNetState *u, const float *compact, int n, float kscale, cudaStream_t s);
int unet_get_params(UNetState *u, float *compact, int n, cudaStream_t s);
int unet_init(UNetState *u, unsigned seed, cudaStream_t s);
int unet_collect(UNetState *u, int capacity);
int unet_samples(const UNetState *u);
bool unet_collecting(const UNetState *u);
int unet_begin_solve(UNetState *u, const GravArgs &a, const float *r32, float *e_out, bool record, cudaStream_t s);
int unet_end_solve(UNetState *u, const GravArgs &a, bool converged, cudaStream_t s);
int unet_train(UNetState *u, int steps, double lr, unsigned seed, double *mean_loss, cudaStream_t s);
int unet_loss_grad(UNetState *u, int n0x, int n0y, int n0z, const float *x, const float *t, double *loss, float *grad,
                   float *out, cudaStream_t s);
}  // namespace hc
