// gravity_fp64.cu -- FP64 Poisson solve of the reference gravity solver.
// Built with -fmad=false so that every value keeps the reference's rounding
// (gravity_solver_3d.c:164-911).
//
//   moments      M, centre of mass and the Cartesian quadrupole Q_ij over
//                cells with rho > 0 (:164-262).  HC_MOMENTS_SEQUENTIAL sums in
//                the reference's (i,j,k) order on one CTA -- bit-exact;
//                HC_MOMENTS_TREE is a fixed-shape (deterministic) tree.
//   boundary     monopole + quadrupole potential on the six faces (:302-498),
//                each face cell given the value of the face loop that writes
//                it last (x, then y, then z); periodic copies (:273-301).
//   SOR          red-black sweeps (:642-708, :577-633 for nz == 1); the
//                per-iteration max |phi_GS - phi_old| is reduced with a warp
//                max and one atomic per block into a per-iteration slot, and
//                the next iteration's first kernel stops the solve when the
//                slot is below tol (:715) -- no host round trip per iteration.
//   acceleration g = -grad phi with the boundary copies (:753-899).
#include <algorithm>

#include "hc_internal.cuh"
#include "hc_math.cuh"

namespace hc {

namespace {

__device__ __forceinline__ double slot_val(const double *res, int it)
{
    return __longlong_as_double(*reinterpret_cast<const long long *>(res + it));
}

template <int NT>
__device__ __forceinline__ double block_max_d(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = tmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    __shared__ double w[NT / 32];
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    if ((tid & 31) == 0) w[tid >> 5] = v;
    __syncthreads();
    double m = 0.0;
    if (tid == 0) {
        for (int t = 0; t < NT / 32; t++) m = tmax(m, w[t]);
    }
    return m;   // valid in thread 0
}

// ---------------------------------------------------------------- moments
constexpr int SEQ_CH = 1024;
constexpr int SEQ_NT = 256;

// Bit-exact moments: terms per cell are formed in parallel into shared
// memory, then one thread per accumulator adds them in cell order.

// The terms of cell c: pass 0 (dm, dm x, dm y, dm z), pass 1 the quadrupole
// terms about com (gravity_solver_3d.c:181-190, :236-255); zero where rho <= 0.
__device__ __forceinline__ void seq_terms(const GravArgs &a, int pass, long long c, const double *com, double *t)
{
    const Geom &g = a.g;
    const double r = a.rho ? a.rho[c] : (double)a.rho32[c];
    if (!(r > 0.0)) return;
    const long long snz = g.nz, sjk = (long long)g.ny * g.nz;
    const int i = (int)(c / sjk), j = (int)((c / snz) % g.ny), k = (int)(c % snz);
    const double dm = r * (g.dx * g.dy * g.dz);
    if (pass == 0) {
        double x = g.xmin + (i + g.ioff + 0.5) * g.dx;
        double y = g.ymin + (j + 0.5) * g.dy;
        double z = g.zmin + (k + 0.5) * g.dz;
        t[0] = dm; t[1] = dm * x; t[2] = dm * y; t[3] = dm * z;
    } else {
        double x = g.xmin + (i + g.ioff + 0.5) * g.dx - com[0];
        double y = g.ymin + (j + 0.5) * g.dy - com[1];
        double z = g.zmin + (k + 0.5) * g.dz - com[2];
        double r2 = x * x + y * y + z * z;
        t[0] = dm * (3.0 * x * x - r2);
        t[1] = dm * (3.0 * x * y);
        t[2] = dm * (3.0 * x * z);
        t[3] = dm * (3.0 * y * x);
        t[4] = dm * (3.0 * y * y - r2);
        t[5] = dm * (3.0 * y * z);
        t[6] = dm * (3.0 * z * x);
        t[7] = dm * (3.0 * z * y);
        t[8] = dm * (3.0 * z * z - r2);
    }
}

// One pass over the cells [c0, c1) in order: thread q < nv returns acc plus
// term q of every cell, added one by one.
__device__ double seq_pass(const GravArgs &a, int pass, long long c0, long long c1, const double *com,
                           double *term, double acc)
{
    const int tid = threadIdx.x;
    const int nv = pass == 0 ? 4 : 9;
    for (long long base = c0; base < c1; base += SEQ_CH) {
        for (int e = tid; e < SEQ_CH; e += SEQ_NT) {
            const long long c = base + e;
            double t[9] = { 0, 0, 0, 0, 0, 0, 0, 0, 0 };
            if (c < c1) seq_terms(a, pass, c, com, t);
            for (int q = 0; q < nv; q++) term[q * SEQ_CH + e] = t[q];
        }
        __syncthreads();
        if (tid < nv) {
            const double *tt = term + tid * SEQ_CH;
            const int m = (int)min((long long)SEQ_CH, c1 - base);
            for (int e = 0; e < m; e++) acc += tt[e];
        }
        __syncthreads();
    }
    return acc;
}

__device__ __forceinline__ void centre_of_mass(const Geom &g, const double *acc, double *out)
{
    const double M = acc[0];
    out[0] = M;
    if (M > 0.0) {
        out[1] = acc[1] / M; out[2] = acc[2] / M; out[3] = acc[3] / M;
    } else {
        out[1] = 0.5 * (g.xmin + g.xmax);
        out[2] = 0.5 * (g.ymin + g.ymax);
        out[3] = 0.5 * (g.zmin + g.zmax);
    }
}

__global__ void __launch_bounds__(SEQ_NT) moments_seq_kernel(GravArgs a)
{
    extern __shared__ double term[];   // 9 x SEQ_CH
    __shared__ double accs[9];
    __shared__ double mc[4];
    const int tid = threadIdx.x;
    const long long n = a.g.n;
    double acc = seq_pass(a, 0, 0, n, nullptr, term, 0.0);
    if (tid < 4) accs[tid] = acc;
    __syncthreads();
    if (tid == 0) centre_of_mass(a.g, accs, mc);
    __syncthreads();
    acc = seq_pass(a, 1, 0, n, mc + 1, term, 0.0);
    if (tid < 4) a.sc->moments[tid] = mc[tid];
    if (tid < 9) a.sc->moments[4 + tid] = acc;
}

// A slab's share of the sequential sums: the own planes, continuing acc.
__global__ void __launch_bounds__(SEQ_NT) moments_seq_slab_kernel(GravArgs a, int pass, double *acc)
{
    extern __shared__ double term[];
    const int tid = threadIdx.x;
    const int nv = pass == 0 ? 4 : 9;
    const long long sjk = (long long)a.g.ny * a.g.nz;
    double v = tid < nv ? acc[tid] : 0.0;
    v = seq_pass(a, pass, a.g.olo * sjk, a.g.ohi * sjk, a.sc->moments + 1, term, v);
    if (tid < nv) acc[tid] = v;
}

__global__ void moments_seq_set_kernel(GravArgs a, int pass, const double *acc)
{
    if (threadIdx.x != 0) return;
    if (pass == 0) centre_of_mass(a.g, acc, a.sc->moments);
    else
        for (int t = 0; t < 9; t++) a.sc->moments[4 + t] = acc[t];
}

// Deterministic tree: one CTA per plane (thread-strided cells, warp and
// block sums in a fixed order), then the planes' partials added in plane
// order -- a fixed order that a grid split into slabs of planes reproduces.
constexpr int TREE_NT = 256;

__global__ void __launch_bounds__(TREE_NT) moments_tree_partial(GravArgs a, int pass, double *parts)
{
    const Geom g = a.g;
    const long long sjk = (long long)g.ny * g.nz;
    const long long c0 = (long long)(g.olo + blockIdx.x) * sjk;
    const int nv = pass == 0 ? 4 : 9;
    const double *com = a.sc->moments + 1;
    double acc[9] = { 0, 0, 0, 0, 0, 0, 0, 0, 0 };
    for (long long c = c0 + threadIdx.x; c < c0 + sjk; c += TREE_NT) {
        double t[9] = { 0, 0, 0, 0, 0, 0, 0, 0, 0 };
        seq_terms(a, pass, c, com, t);
        for (int q = 0; q < nv; q++) acc[q] += t[q];
    }
    __shared__ double red[TREE_NT / 32][9];
    for (int q = 0; q < nv; q++) {
        double v = acc[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][q] = v;
    }
    __syncthreads();
    if (threadIdx.x < nv) {
        double s = 0.0;
        for (int w = 0; w < TREE_NT / 32; w++) s += red[w][threadIdx.x];
        parts[(long long)blockIdx.x * 9 + threadIdx.x] = s;
    }
}

__global__ void moments_tree_final(GravArgs a, int pass, const double *parts, int nparts)
{
    const int q = threadIdx.x;
    const int nv = pass == 0 ? 4 : 9;
    __shared__ double v[9];
    if (q < nv) {
        double s = 0.0;
        for (int b = 0; b < nparts; b++) s += parts[(long long)b * 9 + q];
        v[q] = s;
    }
    __syncthreads();
    if (q != 0) return;
    if (pass == 0) {
        centre_of_mass(a.g, v, a.sc->moments);
    } else {
        for (int t = 0; t < 9; t++) a.sc->moments[4 + t] = v[t];
    }
}

// ---------------------------------------------------------------- boundary
// gravity_solver_3d.c:327-345 for one boundary point.
__device__ __forceinline__ double mono_quad(double x, double y, double z, const double *mom,
                                            double G)
{
    double rx = x - mom[1], ry = y - mom[2], rz = z - mom[3];
    double r = sqrt(rx * rx + ry * ry + rz * rz);
    double ph = 0.0;
    if (r > 0.0) {
        const double *Q = mom + 4;
        ph = -G * mom[0] / r;
        double r5 = r * r * r * r * r;
        double Qr = Q[0] * rx * rx + Q[1] * rx * ry + Q[2] * rx * rz +
                    Q[3] * ry * rx + Q[4] * ry * ry + Q[5] * ry * rz +
                    Q[6] * rz * rx + Q[7] * rz * ry + Q[8] * rz * rz;
        double pq = -G * Qr / (2.0 * r5);
        ph += pq;
    }
    return ph;
}

// Evaluation point of a boundary cell as written by the last face loop that
// touches it: z faces (nz > 1) after y faces after x faces.
__device__ __forceinline__ void face_point(const Geom &g, int i, int j, int k, bool zb,
                                           double &x, double &y, double &z)
{
    x = g.xmin + (i + g.ioff + 0.5) * g.dx;
    y = g.ymin + (j + 0.5) * g.dy;
    z = g.zmin + (k + 0.5) * g.dz;
    if (zb && (k == 0 || k == g.nz - 1)) {
        z = (k == g.nz - 1) ? g.zmax - 0.5 * g.dz : g.zmin + 0.5 * g.dz;
    } else if (j == 0 || j == g.ny - 1) {
        y = (j == g.ny - 1) ? g.ymax - 0.5 * g.dy : g.ymin + 0.5 * g.dy;
    } else {
        x = (i + g.ioff == g.gnx - 1) ? g.xmax - 0.5 * g.dx : g.xmin + 0.5 * g.dx;
    }
}

__global__ void boundary_ref_kernel(GravArgs a)
{
    const Geom g = a.g;
    const bool zb = g.nz > 1;
    const long long nb = boundary_count(g.nx, g.ny, g.nz, zb);
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= nb) return;
    int i, j, k;
    boundary_cell(t, g.nx, g.ny, g.nz, zb, i, j, k);
    if (i < g.olo || i >= g.ohi) return;   // a ghost plane: the neighbour's cells
    double x, y, z;
    face_point(g, i, j, k, zb, x, y, z);
    a.phi[((long long)i * g.ny + j) * g.nz + k] = mono_quad(x, y, z, a.sc->moments, a.G);
}

__global__ void periodic_phi_kernel(GravArgs a, int axis)
{
    const Geom g = a.g;
    const int n[3] = { g.nx, g.ny, g.nz };
    const int nu = (axis == 0) ? n[1] : n[0], nv = (axis == 2) ? n[1] : n[2];
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)nu * nv) return;
    const int u = (int)(t / nv), v = (int)(t % nv);
    const long long sI = (long long)g.ny * g.nz, sJ = g.nz;
    long long c0, c1;
    if (axis == 0) { c0 = u * sJ + v; c1 = (n[0] - 1) * sI + u * sJ + v; }
    else if (axis == 1) { c0 = u * sI + v; c1 = u * sI + (n[1] - 1) * sJ + v; }
    else { c0 = u * sI + v * sJ; c1 = u * sI + v * sJ + n[2] - 1; }
    a.phi[c0] = a.phi[c1];
}

// ---------------------------------------------------------------- SOR
struct SorConst {
    double ix2, iy2, iz2, fpg, fac;
};

__device__ __forceinline__ SorConst sor_const(const GravArgs &a)
{
    SorConst c;
    c.ix2 = 1.0 / (a.g.dx * a.g.dx);
    c.iy2 = 1.0 / (a.g.dy * a.g.dy);
    c.iz2 = 1.0 / (a.g.dz * a.g.dz);
    c.fpg = 4.0 * M_PI * a.G;
    c.fac = (a.g.nz == 1) ? 2.0 * (c.ix2 + c.iy2) : 2.0 * (c.ix2 + c.iy2 + c.iz2);
    return c;
}

// Stop rule of gravity_solver_3d.c:715, evaluated on the device: iteration
// `iter` starts only if iteration iter-1 left the update norm >= tol.
__device__ __forceinline__ bool sor_should_stop(const GravArgs &a, int iter)
{
    if (*(volatile int *)&a.sc->done) return true;
    if (iter > 0 && slot_val(a.res, iter - 1) < a.tol) {
        if (threadIdx.x == 0 && threadIdx.y == 0) {
            a.sc->last_iter = iter;
            a.sc->done = 1;
        }
        return true;
    }
    return false;
}

constexpr int SOR_BX = 32, SOR_BY = 8;

__global__ void __launch_bounds__(SOR_BX * SOR_BY) sor_color3d(GravArgs a, int color, int iter)
{
    if (sor_should_stop(a, color == 0 ? iter : -1)) return;
    const Geom g = a.g;
    const int i = 1 + blockIdx.z;
    const int j = 1 + blockIdx.y * SOR_BY + threadIdx.y;
    const int k0 = ((i + j + 1) % 2 == color) ? 1 : 2;
    const int k = k0 + 2 * (blockIdx.x * SOR_BX + threadIdx.x);
    const SorConst sc = sor_const(a);
    double r = 0.0;
    if (j <= g.ny - 2 && k <= g.nz - 2) {
        const long long sI = (long long)g.ny * g.nz, sJ = g.nz;
        const long long c = i * sI + j * sJ + k;
        double *phi = a.phi;
        double old = phi[c];
        double lap = (phi[c - sI] + phi[c + sI]) * sc.ix2 + (phi[c - sJ] + phi[c + sJ]) * sc.iy2 +
                     (phi[c - 1] + phi[c + 1]) * sc.iz2;
        double nw = (lap - sc.fpg * a.rho[c]) / sc.fac;
        phi[c] = old + a.omega * (nw - old);
        r = fabs(nw - old);
    }
    double m = block_max_d<SOR_BX * SOR_BY>(r);
    if (threadIdx.x == 0 && threadIdx.y == 0) atomic_max_nonneg((unsigned long long *)(a.res + iter), m);
}

__global__ void __launch_bounds__(256) sor_color2d(GravArgs a, int color, int iter)
{
    if (sor_should_stop(a, color == 0 ? iter : -1)) return;
    const Geom g = a.g;
    const SorConst sc = sor_const(a);
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long cnt = (long long)(g.nx - 2) * (g.ny - 2);
    double r = 0.0;
    if (t < cnt) {
        int i = 1 + (int)(t / (g.ny - 2)), j = 1 + (int)(t % (g.ny - 2));
        if ((i + j) % 2 == color) {
            const long long sI = g.ny, c = (long long)i * sI + j;
            double *phi = a.phi;
            double old = phi[c];
            double lap = (phi[c - sI] + phi[c + sI]) * sc.ix2 + (phi[c - 1] + phi[c + 1]) * sc.iy2;
            double nw = (lap - sc.fpg * a.rho[c]) / sc.fac;
            phi[c] = old + a.omega * (nw - old);
            r = fabs(nw - old);
        }
    }
    double m = block_max_d<256>(r);
    if (threadIdx.x == 0) atomic_max_nonneg((unsigned long long *)(a.res + iter), m);
}

__global__ void check_kernel(GravArgs a, int iter) { sor_should_stop(a, iter); }

// ---------------------------------------------------------------- accel
__global__ void accel_kernel(GravArgs a)
{
    const Geom g = a.g;
    const long long sI = (long long)g.ny * g.nz, sJ = g.nz;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.n;
         c += (long long)gridDim.x * blockDim.x) {
        int i = (int)(c / sI), j = (int)((c / sJ) % g.ny), k = (int)(c % sJ);
        const double *phi = a.phi;
        if (g.nz == 1) {
            if (i >= 1 && i <= g.nx - 2 && j >= 1 && j <= g.ny - 2) {
                a.gx[c] = -(phi[c + sI] - phi[c - sI]) / (2.0 * g.dx);
                a.gy[c] = -(phi[c + sJ] - phi[c - sJ]) / (2.0 * g.dy);
            } else {
                a.gx[c] = 0.0; a.gy[c] = 0.0;
            }
            a.gz[c] = 0.0;
            continue;
        }
        int ci = min(max(i, 1), g.nx - 2), cj = min(max(j, 1), g.ny - 2), ck = min(max(k, 1), g.nz - 2);
        long long cc = ci * sI + cj * sJ + ck;
        a.gx[c] = -(phi[cc + sI] - phi[cc - sI]) / (2.0 * g.dx);
        a.gy[c] = -(phi[cc + sJ] - phi[cc - sJ]) / (2.0 * g.dy);
        a.gz[c] = -(phi[cc + 1] - phi[cc - 1]) / (2.0 * g.dz);
    }
}

__global__ void residual_kernel(GravArgs a, const double *phi)
{
    const Geom g = a.g;
    const SorConst sc = sor_const(a);
    const long long sI = (long long)g.ny * g.nz, sJ = g.nz;
    double m = 0.0;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.n;
         c += (long long)gridDim.x * blockDim.x) {
        int i = (int)(c / sI), j = (int)((c / sJ) % g.ny), k = (int)(c % sJ);
        if (i < 1 || i > g.nx - 2 || j < 1 || j > g.ny - 2 || k < 1 || k > g.nz - 2) continue;
        double lap = (phi[c - sI] + phi[c + sI]) * sc.ix2 + (phi[c - sJ] + phi[c + sJ]) * sc.iy2 +
                     (phi[c - 1] + phi[c + 1]) * sc.iz2;
        double rr = a.rho ? a.rho[c] : (double)a.rho32[c];
        double nw = (lap - sc.fpg * rr) / sc.fac;
        m = tmax(m, fabs(nw - phi[c]));
    }
    double b = block_max_d<256>(m);
    if (threadIdx.x == 0) atomic_max_nonneg((unsigned long long *)&a.sc->resnorm, b);
}

__global__ void zero_slots(double *res, int from, int count)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += gridDim.x * blockDim.x)
        res[from + t] = 0.0;
}

inline int grid_for(long long n, int bs) { return (int)((n + bs - 1) / bs); }

}  // namespace

cudaError_t grav_moments_sequential(const GravArgs &a, cudaStream_t s)
{
    const size_t sm = 9 * SEQ_CH * sizeof(double);
    static std::atomic<unsigned long long> attr_set{0};
    cudaError_t e = set_smem_once(attr_set, (const void *)moments_seq_kernel, (int)sm);
    if (e != cudaSuccess) return e;
    moments_seq_kernel<<<1, SEQ_NT, sm, s>>>(a);
    return cudaGetLastError();
}

cudaError_t grav_moments_seq_slab(const GravArgs &a, int pass, double *acc, cudaStream_t s)
{
    const size_t sm = 9 * SEQ_CH * sizeof(double);
    static std::atomic<unsigned long long> attr_set{0};
    cudaError_t e = set_smem_once(attr_set, (const void *)moments_seq_slab_kernel, (int)sm);
    if (e != cudaSuccess) return e;
    moments_seq_slab_kernel<<<1, SEQ_NT, sm, s>>>(a, pass, acc);
    return cudaGetLastError();
}

cudaError_t grav_moments_seq_set(const GravArgs &a, int pass, const double *acc, cudaStream_t s)
{
    moments_seq_set_kernel<<<1, 32, 0, s>>>(a, pass, acc);
    return cudaGetLastError();
}

cudaError_t grav_moments_tree_parts(const GravArgs &a, int pass, double *parts, cudaStream_t s)
{
    if (a.g.ohi <= a.g.olo) return cudaErrorInvalidValue;
    moments_tree_partial<<<a.g.ohi - a.g.olo, TREE_NT, 0, s>>>(a, pass, parts);
    return cudaGetLastError();
}

cudaError_t grav_moments_tree_set(const GravArgs &a, int pass, const double *parts, int nparts, cudaStream_t s)
{
    moments_tree_final<<<1, 32, 0, s>>>(a, pass, parts, nparts);
    return cudaGetLastError();
}

cudaError_t grav_moments_tree(const GravArgs &a, cudaStream_t s)
{
    if (a.scratch_len < (long long)a.g.nx * 9) return cudaErrorInvalidValue;
    for (int pass = 0; pass < 2; pass++) {
        cudaError_t e = grav_moments_tree_parts(a, pass, a.scratch, s);
        if (e != cudaSuccess) return e;
        e = grav_moments_tree_set(a, pass, a.scratch, a.g.ohi - a.g.olo, s);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t grav_boundary_ref(const GravArgs &a, cudaStream_t s)
{
    long long nb = boundary_count(a.g.nx, a.g.ny, a.g.nz, a.g.nz > 1);
    boundary_ref_kernel<<<grid_for(nb, 256), 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t grav_boundary_periodic(const GravArgs &a, cudaStream_t s)
{
    const int n[3] = { a.g.nx, a.g.ny, a.g.nz };
    for (int axis = 0; axis < 3; axis++) {
        if (axis == 2 && a.g.nz <= 1) break;
        long long cnt = (long long)((axis == 0) ? n[1] : n[0]) * ((axis == 2) ? n[1] : n[2]);
        periodic_phi_kernel<<<grid_for(cnt, 256), 256, 0, s>>>(a, axis);
    }
    return cudaGetLastError();
}

cudaError_t grav_sor_color(const GravArgs &a, int color, int iter, cudaStream_t s)
{
    if (a.g.nz == 1) {
        long long cnt = (long long)(a.g.nx - 2) * (a.g.ny - 2);
        sor_color2d<<<grid_for(cnt, 256), 256, 0, s>>>(a, color, iter);
    } else {
        int nhalf = (a.g.nz - 1) / 2;   // cells of one colour per row, upper bound
        dim3 grid(grid_for(nhalf, SOR_BX), grid_for(a.g.ny - 2, SOR_BY), a.g.nx - 2);
        sor_color3d<<<grid, dim3(SOR_BX, SOR_BY), 0, s>>>(a, color, iter);
    }
    return cudaGetLastError();
}

cudaError_t grav_check(const GravArgs &a, int iter, cudaStream_t s)
{
    check_kernel<<<1, 1, 0, s>>>(a, iter);
    return cudaGetLastError();
}

cudaError_t grav_accel(const GravArgs &a, cudaStream_t s)
{
    accel_kernel<<<148 * 8, 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t grav_residual_norm(const GravArgs &a, const double *phi, cudaStream_t s)
{
    residual_kernel<<<148 * 8, 256, 0, s>>>(a, phi);
    return cudaGetLastError();
}

cudaError_t grav_reset_slots(const GravArgs &a, int from, int count, cudaStream_t s)
{
    if (count <= 0) return cudaSuccess;
    zero_slots<<<std::min(grid_for(count, 256), 1024), 256, 0, s>>>(a.res, from, count);
    return cudaGetLastError();
}

}  // namespace hc

// ---------------------------------------------------------------------------
// One full red-black iteration per pass over HBM (wavefront, out of place).
// ---------------------------------------------------------------------------
#include "sor_wavefront.cuh"
#include "sor_wavefront_tma.cuh"
#include "tmap.cuh"

namespace hc {
namespace {
constexpr int WF64_T = 1, WF64_TJ = 16, WF64_TK = 64, WF64_NT = 256;
}

// HC_NO_TMA=1 selects the plain-load kernels (A/B comparisons).
bool wf_tma_enabled()
{
    static int on = -1;
    if (on < 0) {
        const char *e = getenv("HC_NO_TMA");
        on = (e && atoi(e) != 0) ? 0 : 1;
    }
    return on == 1;
}

cudaError_t grav_sor_pass64(const GravArgs &a, const double *in, double *out, int iter0, cudaStream_t s)
{
    constexpr size_t sm = sor_wavefront_smem<double, WF64_T, WF64_TJ, WF64_TK>();
    auto kern = sor_wavefront_kernel<double, double, WF64_T, WF64_TJ, WF64_TK, WF64_NT>;
    static std::atomic<unsigned long long> attr_set{0};
    cudaError_t e = set_smem_once(attr_set, (const void *)kern, (int)sm);
    if (e != cudaSuccess) return e;
    SorCoef<double> cf;
    cf.ix2 = 1.0 / (a.g.dx * a.g.dx);
    cf.iy2 = 1.0 / (a.g.dy * a.g.dy);
    cf.iz2 = 1.0 / (a.g.dz * a.g.dz);
    cf.fpg = 4.0 * M_PI * a.G;
    cf.fac = 2.0 * (cf.ix2 + cf.iy2 + cf.iz2);
    cf.om = a.omega;
    const int tj = (a.g.ny + WF64_TJ - 1) / WF64_TJ, tk = (a.g.nz + WF64_TK - 1) / WF64_TK;
    const int nint = a.g.nx - 2;
    // about 3 waves of 4 CTAs per SM; at least 16 planes per chunk
    long long want = 148LL * 4 * 3;
    int chunks = (int)std::max(1LL, std::min((long long)nint / 16, (want + tj * tk - 1) / (tj * tk)));
    chunks = std::max(chunks, 1);
    int chunk = (nint + chunks - 1) / chunks;
    chunks = (nint + chunk - 1) / chunk;
    dim3 grid(tk, tj, chunks);
    // operands staged by TMA where the layout allows it (16-byte row stride)
    using SH = wtma::Shape<double, WF64_T, WF64_TJ, WF64_TK>;
    CUtensorMap tin, tsrc;
    if (wf_tma_enabled() && tmap3(in, 8, a.g.nx, a.g.ny, a.g.nz, SH::SK, SH::SJ, &tin) &&
        tmap3(a.rho, 8, a.g.nx, a.g.ny, a.g.nz, SH::SK, SH::SJ, &tsrc)) {
        auto kt = wtma::sor_wavefront_tma_kernel<double, double, WF64_T, WF64_TJ, WF64_TK, WF64_NT>;
        static std::atomic<unsigned long long> attr_t{0};
        e = set_smem_once(attr_t, (const void *)kt, (int)SH::SMEM);
        if (e != cudaSuccess) return e;
        kt<<<grid, WF64_NT, SH::SMEM, s>>>(tin, tsrc, out, a.g, cf, a.res, iter0, a.tol, a.sc, chunk);
        return cudaGetLastError();
    }
    kern<<<grid, WF64_NT, sm, s>>>(in, out, a.rho, a.g, cf, a.res, iter0, a.tol, a.sc, chunk);
    return cudaGetLastError();
}

}  // namespace hc

// ---------------------------------------------------------------------------
// Colour-split SOR (the default FP64 solve for nz >= 3)
// ---------------------------------------------------------------------------
#include "sor_split.cuh"

namespace hc {

long long split_len(const Geom &g)
{
    const Split sp = make_split(g);
    return 2 * sp.cs;
}

cudaError_t grav_split_fields(const GravArgs &a, double *phs, double *rhs, cudaStream_t s)
{
    const Split sp = make_split(a.g);
    const unsigned rows = (unsigned)((long long)a.g.nx * a.g.ny);
    const int nt = a.g.nz >= 256 ? 256 : 128;
    split_copy_kernel<double, double><<<rows, nt, 0, s>>>(a.phi, phs, sp);
    if (rhs) split_copy_kernel<double, double><<<rows, nt, 0, s>>>(a.rho, rhs, sp);
    return cudaGetLastError();
}

cudaError_t grav_split_boundary(const GravArgs &a, double *phs, cudaStream_t s)
{
    const Split sp = make_split(a.g);
    split_boundary_kernel<double><<<148 * 4, 256, 0, s>>>(a.phi, phs, sp);
    return cudaGetLastError();
}

cudaError_t grav_unsplit(const GravArgs &a, const double *phs, cudaStream_t s)
{
    const Split sp = make_split(a.g);
    const unsigned rows = (unsigned)((long long)a.g.nx * a.g.ny);
    unsplit_copy_kernel<double><<<rows, a.g.nz >= 256 ? 256 : 128, 0, s>>>(phs, a.phi, sp);
    return cudaGetLastError();
}

cudaError_t grav_sor_split(const GravArgs &a, double *phs, const double *rhs, int colour, int iter, cudaStream_t s)
{
    SorCoef<double> cf;
    cf.ix2 = 1.0 / (a.g.dx * a.g.dx);
    cf.iy2 = 1.0 / (a.g.dy * a.g.dy);
    cf.iz2 = 1.0 / (a.g.dz * a.g.dz);
    cf.fpg = 4.0 * M_PI * a.G;
    cf.fac = 2.0 * (cf.ix2 + cf.iy2 + cf.iz2);
    cf.om = a.omega;
    return launch_sor_split<double, double>(phs, rhs, make_split(a.g), cf, colour, a.res, iter, a.tol, a.sc, s);
}

}  // namespace hc
