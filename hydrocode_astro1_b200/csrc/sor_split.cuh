// sor_split.cuh -- red-black SOR sweeps on a colour-split layout.
//
// The red and the black cells of a field are stored in two separate arrays,
// each a dense (i, j, m) block: cell (i, j, k) has colour c = (i+j+k) & 1 and
// lives at  c*cs + (i*ny + j)*H + (k >> 1),  H = (nz+1)/2,  cs = nx*ny*H.
// A colour sweep then reads the other colour's array, its own array and the
// source (all unit-stride along m) and writes its own array with full-sector
// stores: 4 x 1/2 x sizeof(T) bytes per cell per colour, no stride-2 access
// and no partially written sectors.
//
// Neighbours of a cell of colour c at (i, j, m) with k = 2m + s,
// s = (i + j + c) & 1, are all of the other colour:
//   x+-1, y+-1 : same m in the rows (i+-1, j) and (i, j+-1)
//   z-1 / z+1  : m-1 / m (s = 0) or m / m+1 (s = 1) in row (i, j)
// Each thread updates one (j, m) column over a few planes, loading all their
// operands before the first update.  Within a colour the updates are
// independent, so the iterates are those of the reference's sweep
// (gravity_solver_3d.c:566-728) bit for bit in FP64 (same operand order,
// SorCoef<double>).
//
// The update norm max |phi_GS - phi_old| of the sweep is reduced per CTA
// into the iteration's slot with one atomic.  A red sweep whose previous
// iteration's slot is already below the stop threshold sets the done flag
// instead of sweeping; every later sweep of the batch then returns at once.
#pragma once
#include <cstdint>
#include <type_traits>
#include "hc_internal.cuh"
#include "hc_math.cuh"
#include "sor_wavefront.cuh"

// vector sweeps (sor_split_vec_kernel) where the row length allows them
#ifndef HC_SPLIT_VEC
#define HC_SPLIT_VEC 1
#endif
#ifndef HC_SPLIT_VEC64
#define HC_SPLIT_VEC64 0   // FP64: the scalar kernel is faster (119 vs 158 us per iteration at 256^3)
#endif
#ifndef HC_SPLIT_VEC_NI
#define HC_SPLIT_VEC_NI 2
#endif
#ifndef HC_SPLIT_VEC_MINB32
#define HC_SPLIT_VEC_MINB32 4
#endif
#ifndef HC_SPLIT_VEC_MINB64
#define HC_SPLIT_VEC_MINB64 2
#endif
#ifndef HC_SOR_PDL
#define HC_SOR_PDL 1
#endif
#ifndef HC_SPLIT_SNAKE
#define HC_SPLIT_SNAKE 1
#endif

namespace hc {

struct Split {
    int nx, ny, nz, H;
    long long cs;   // elements per colour
    __host__ __device__ __forceinline__ long long at(int i, int j, int k) const
    {
        return (long long)((i + j + k) & 1) * cs + ((long long)i * ny + j) * H + (k >> 1);
    }
};

inline Split make_split(const Geom &g)
{
    Split s;
    s.nx = g.nx;
    s.ny = g.ny;
    s.nz = g.nz;
    s.H = (g.nz + 1) / 2;
    s.cs = (long long)g.nx * g.ny * s.H;
    return s;
}

#ifndef HC_SPLIT_BY
#define HC_SPLIT_BY 8
#endif
constexpr int SPLIT_BX = 32, SPLIT_BY = HC_SPLIT_BY;   // rows of a CTA

// Programmatic dependent launch: a sweep launched with programmatic stream
// serialisation may be scheduled while the previous sweep's last CTAs still
// run; griddepcontrol.wait holds it until that grid has completed and its
// writes are visible, so nothing is read early.  Releasing the dependents at
// once lets the next sweep's CTAs take SM slots as this grid's last wave
// drains (they cannot crowd out this grid: its last CTAs are already
// resident when the release of every CTA completes).  In a kernel launched
// without the attribute both instructions do nothing.
__device__ __forceinline__ void pdl_wait_and_release()
{
#if HC_SOR_PDL
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
#endif
}

template <typename K, typename... Args>
cudaError_t launch_pdl_smem(K kernel, dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args... args)
{
#if HC_SOR_PDL
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
#else
    kernel<<<grid, block, smem, s>>>(args...);
    return cudaGetLastError();
#endif
}

template <typename K, typename... Args>
cudaError_t launch_pdl(K kernel, dim3 grid, dim3 block, cudaStream_t s, Args... args)
{
    return launch_pdl_smem(kernel, grid, block, 0, s, args...);
}

// One thread owns the column (j, m) over NI consecutive planes i0..i0+NI-1:
// every operand of the NI updates is loaded first (6 NI + 2 independent
// loads in flight per thread), then the updates run and are stored.  Offsets
// are 32-bit (a colour array holds < 2^31 cells).  Loads need no clamping:
// the z neighbour across a row end is a real cell of the adjacent row (rows
// j-1 and j+1 exist for 1 <= j <= ny-2) and feeds only boundary cells, and a
// CTA whose planes reach past nx-2 takes the guarded tail path.
template <typename T, typename S, int NI, int MINB = 1>
__global__ void __launch_bounds__(SPLIT_BX * SPLIT_BY, MINB)
sor_split_kernel(T *__restrict__ own, const T *__restrict__ oth, const S *__restrict__ src, Split sp,
                 SorCoef<T> cf, int colour, double *res, int iter, double thresh, DevScalars *sc)
{
    __shared__ double wmax[SPLIT_BX * SPLIT_BY / 32];
    pdl_wait_and_release();
    if (*(volatile int *)&sc->done) return;
    if (colour == 0 && iter > 0) {
        const double prev = __longlong_as_double(*reinterpret_cast<const volatile long long *>(res + iter - 1));
        if (prev < thresh) {
            if (threadIdx.x == 0 && threadIdx.y == 0) {
                sc->last_iter = iter;
                sc->done = 1;
            }
            return;
        }
    }
    const int m = blockIdx.x * SPLIT_BX + threadIdx.x;
    const int j = blockIdx.y * SPLIT_BY + threadIdx.y;
    const int i0 = 1 + blockIdx.z * NI;
    T rmax = (T)0;
    if (j >= 1 && j <= sp.ny - 2 && m < sp.H) {
        const int sJ = sp.H, sI = sp.ny * sp.H;
        const int o0 = i0 * sI + j * sJ + m;
        const int s0 = (i0 + j + colour) & 1;
        // interior in k for s = 0 (k = 2m) and s = 1 (k = 2m+1)
        const bool ok0 = m >= 1 && 2 * m <= sp.nz - 2;
        const bool ok1 = 2 * m + 1 <= sp.nz - 2;
        const int nq = min(NI, sp.nx - 1 - i0);   // planes i0 .. i0+nq-1 are interior
        const T *ox = oth + o0;
        const S *sx = src + o0;
        T *wx = own + o0;
        T x[NI + 2], ym[NI], yp[NI], zo[NI], ow[NI];
        S sr[NI];
        if (nq == NI) {
#pragma unroll
            for (int q = 0; q < NI + 2; q++) x[q] = ox[(q - 1) * sI];
#pragma unroll
            for (int q = 0; q < NI; q++) {
                const int s = s0 ^ (q & 1);
                ym[q] = ox[q * sI - sJ];
                yp[q] = ox[q * sI + sJ];
                zo[q] = ox[q * sI + (s ? 1 : -1)];
                ow[q] = wx[q * sI];
                sr[q] = sx[q * sI];
            }
        } else {
#pragma unroll
            for (int q = 0; q < NI + 2; q++) x[q] = (q <= nq + 1) ? ox[(q - 1) * sI] : (T)0;
#pragma unroll
            for (int q = 0; q < NI; q++) {
                const int s = s0 ^ (q & 1);
                if (q < nq) {
                    ym[q] = ox[q * sI - sJ];
                    yp[q] = ox[q * sI + sJ];
                    zo[q] = ox[q * sI + (s ? 1 : -1)];
                    ow[q] = wx[q * sI];
                    sr[q] = sx[q * sI];
                } else {
                    ym[q] = yp[q] = zo[q] = ow[q] = (T)0;
                    sr[q] = (S)0;
                }
            }
        }
#pragma unroll
        for (int q = 0; q < NI; q++) {
            const int s = s0 ^ (q & 1);
            if (q < nq && (s ? ok1 : ok0)) {
                const T zm = s ? x[q + 1] : zo[q];
                const T zp = s ? zo[q] : x[q + 1];
                T r;
                wx[q * sI] = cf.update(ow[q], x[q], x[q + 2], ym[q], yp[q], zm, zp, (T)sr[q], r);
                rmax = tmax(rmax, r);
            }
        }
    }
    double v = (double)rmax;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v = tmax(v, __shfl_xor_sync(0xffffffffu, v, off));
    const int tid = threadIdx.y * SPLIT_BX + threadIdx.x;
    if ((tid & 31) == 0) wmax[tid >> 5] = v;
    __syncthreads();
    if (tid == 0) {
        double b = 0.0;
#pragma unroll
        for (int w = 0; w < SPLIT_BX * SPLIT_BY / 32; w++) b = tmax(b, wmax[w]);
        // most CTAs find the slot already at or above their value
        unsigned long long *slot = (unsigned long long *)(res + iter);
        if (b > 0.0 && (unsigned long long)__double_as_longlong(b) > *(volatile unsigned long long *)slot)
            atomic_max_nonneg(slot, b);
    }
}

// V consecutive elements of a colour row, loaded and stored as one 16-byte
// vector (float4 / double2)
template <typename T>
struct alignas(16) Pack {
    static constexpr int V = 16 / sizeof(T);
    T v[V];
};

// Vector form of sor_split_kernel, for rows whose length H is a multiple of
// V = 16 / sizeof(T): a lane owns the V consecutive cells m0 .. m0+V-1 of its
// row over NI planes, so every operand is one 16-byte load (4x fewer load
// instructions than the scalar kernel for FP32).  A warp spans 32 V cells of
// one row; the z neighbour outside the lane's vector (m0-1 for s = 0, m0+V
// for s = 1) comes from the adjacent lane by a shuffle, or -- at a warp edge
// inside the row -- from an extra scalar load issued with the others.  The
// per-cell update is the scalar kernel's, operand for operand, and cells
// that are not updated (k = 0, nz-1, the padding slot of odd nz) are stored
// back unchanged.  Sweeps of colour 1 visit the planes in descending order
// (each sweep starts where the previous one ended, where the L2 still holds
// the shared colour arrays); the order does not change any result.
template <typename T, int NI, int MINB>
__global__ void __launch_bounds__(SPLIT_BX * SPLIT_BY, MINB)
sor_split_vec_kernel(T *__restrict__ own, const T *__restrict__ oth, const T *__restrict__ src, Split sp,
                     SorCoef<T> cf, int colour, double *res, int iter, double thresh, DevScalars *sc)
{
    constexpr int V = Pack<T>::V;
    using P = Pack<T>;
    __shared__ double wmax[SPLIT_BX * SPLIT_BY / 32];
    pdl_wait_and_release();
    if (*(volatile int *)&sc->done) return;
    if (colour == 0 && iter > 0) {
        const double prev = __longlong_as_double(*reinterpret_cast<const volatile long long *>(res + iter - 1));
        if (prev < thresh) {
            if (threadIdx.x == 0 && threadIdx.y == 0) {
                sc->last_iter = iter;
                sc->done = 1;
            }
            return;
        }
    }
    const int lane = threadIdx.x;
    const int m0 = (blockIdx.x * SPLIT_BX + lane) * V;
    const int j = blockIdx.y * SPLIT_BY + threadIdx.y;
#if HC_SPLIT_SNAKE
    const int bz = colour ? (int)gridDim.z - 1 - (int)blockIdx.z : (int)blockIdx.z;
#else
    const int bz = blockIdx.z;
#endif
    const int i0 = 1 + bz * NI;
    T rmax = (T)0;
    if (j >= 1 && j <= sp.ny - 2) {   // uniform over the warp (one row)
        const bool act = m0 < sp.H;
        const int sJ = sp.H, sI = sp.ny * sp.H;
        const int o0 = i0 * sI + j * sJ + (act ? m0 : 0);
        const int s0 = (i0 + j + colour) & 1;
        const int nq = min(NI, sp.nx - 1 - i0);   // planes i0 .. i0+nq-1 are interior
        const P *ox = reinterpret_cast<const P *>(oth + o0);
        const P *sx = reinterpret_cast<const P *>(src + o0);
        P *wx = reinterpret_cast<P *>(own + o0);
        const int vI = sI / V, vJ = sJ / V;
        P x[NI + 2], ym[NI], yp[NI], ow[NI], sr[NI];
        T ze[NI];
        const P zero = {};
#pragma unroll
        for (int q = 0; q < NI + 2; q++) x[q] = (act && q <= nq + 1) ? ox[(q - 1) * vI] : zero;
#pragma unroll
        for (int q = 0; q < NI; q++) {
            const int s = s0 ^ (q & 1);
            const bool ld = act && q < nq;
            ym[q] = ld ? ox[q * vI - vJ] : zero;
            yp[q] = ld ? ox[q * vI + vJ] : zero;
            ow[q] = ld ? wx[q * vI] : zero;
            sr[q] = ld ? sx[q * vI] : zero;
            const bool edge = s ? (lane == SPLIT_BX - 1 && m0 + V < sp.H) : (lane == 0 && m0 > 0);
            ze[q] = (ld && edge) ? oth[o0 + q * sI + (s ? V : -1)] : (T)0;
        }
#pragma unroll
        for (int q = 0; q < NI; q++) {
            const int s = s0 ^ (q & 1);
            const T nb = s ? __shfl_down_sync(0xffffffffu, x[q + 1].v[0], 1)
                           : __shfl_up_sync(0xffffffffu, x[q + 1].v[V - 1], 1);
            if (lane != (s ? SPLIT_BX - 1 : 0)) ze[q] = nb;
        }
#pragma unroll
        for (int q = 0; q < NI; q++) {
            const int s = s0 ^ (q & 1);
            if (act && q < nq) {
#pragma unroll
                for (int e = 0; e < V; e++) {
                    const int k = 2 * (m0 + e) + s;
                    if (k >= 1 && k <= sp.nz - 2) {
                        const T zm = s ? x[q + 1].v[e] : (e == 0 ? ze[q] : x[q + 1].v[e - 1]);
                        const T zp = s ? (e == V - 1 ? ze[q] : x[q + 1].v[e + 1]) : x[q + 1].v[e];
                        T r;
                        ow[q].v[e] = cf.update(ow[q].v[e], x[q].v[e], x[q + 2].v[e], ym[q].v[e], yp[q].v[e], zm, zp,
                                               sr[q].v[e], r);
                        rmax = tmax(rmax, r);
                    }
                }
                wx[q * vI] = ow[q];
            }
        }
    }
    double v = (double)rmax;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v = tmax(v, __shfl_xor_sync(0xffffffffu, v, off));
    const int tid = threadIdx.y * SPLIT_BX + threadIdx.x;
    if ((tid & 31) == 0) wmax[tid >> 5] = v;
    __syncthreads();
    if (tid == 0) {
        double b = 0.0;
#pragma unroll
        for (int w = 0; w < SPLIT_BX * SPLIT_BY / 32; w++) b = tmax(b, wmax[w]);
        unsigned long long *slot = (unsigned long long *)(res + iter);
        if (b > 0.0 && (unsigned long long)__double_as_longlong(b) > *(volatile unsigned long long *)slot)
            atomic_max_nonneg(slot, b);
    }
}

// natural (k fastest) -> colour-split copy; one CTA per row (i, j)
template <typename A, typename B>
__global__ void split_copy_kernel(const A *__restrict__ nat, B *__restrict__ spl, Split sp)
{
    const long long row = blockIdx.x;   // i*ny + j
    const int i = (int)(row / sp.ny), j = (int)(row % sp.ny);
    const A *r = nat + row * sp.nz;
    for (int k = threadIdx.x; k < sp.nz; k += blockDim.x) spl[sp.at(i, j, k)] = (B)r[k];
}

// colour-split -> natural copy; one CTA per row (i, j)
template <typename T>
__global__ void unsplit_copy_kernel(const T *__restrict__ spl, T *__restrict__ nat, Split sp)
{
    const long long row = blockIdx.x;
    const int i = (int)(row / sp.ny), j = (int)(row % sp.ny);
    T *r = nat + row * sp.nz;
    for (int k = threadIdx.x; k < sp.nz; k += blockDim.x) r[k] = spl[sp.at(i, j, k)];
}

// boundary cells only (the Dirichlet values of the solve)
template <typename T>
__global__ void split_boundary_kernel(const T *__restrict__ nat, T *__restrict__ spl, Split sp)
{
    const long long nb = boundary_count(sp.nx, sp.ny, sp.nz, true);
    const long long sI = (long long)sp.ny * sp.nz, sJ = sp.nz;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nb;
         t += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        boundary_cell(t, sp.nx, sp.ny, sp.nz, true, i, j, k);
        spl[sp.at(i, j, k)] = nat[i * sI + j * sJ + k];
    }
}

template <typename T, typename S>
cudaError_t launch_sor_split(T *base, const S *src, const Split &sp, const SorCoef<T> &cf, int colour,
                             double *res, int iter, double thresh, DevScalars *sc, cudaStream_t s)
{
    constexpr int NI = sizeof(T) == 8 ? 4 : 8;   // fastest at 256^3: FP64 55.6, FP32 28.8 us per sweep
    constexpr int MINB = sizeof(T) == 8 ? 1 : 4;
    if (sp.cs + 2LL * sp.ny * sp.H >= (1LL << 31)) return cudaErrorInvalidValue;   // 32-bit offsets
    T *own = base + (size_t)colour * sp.cs;
    const T *oth = base + (size_t)(colour ^ 1) * sp.cs;
#if HC_SPLIT_VEC
    constexpr int V = Pack<T>::V;
    if (std::is_same<T, S>::value && (HC_SPLIT_VEC64 || sizeof(T) == 4) && sp.H % V == 0 &&
        ((uintptr_t)base | (uintptr_t)src) % 16 == 0) {
        constexpr int VNI = HC_SPLIT_VEC_NI, VMINB = sizeof(T) == 8 ? HC_SPLIT_VEC_MINB64 : HC_SPLIT_VEC_MINB32;
        dim3 grid((sp.H / V + SPLIT_BX - 1) / SPLIT_BX, (sp.ny + SPLIT_BY - 1) / SPLIT_BY, (sp.nx - 2 + VNI - 1) / VNI);
        return launch_pdl(sor_split_vec_kernel<T, VNI, VMINB>, grid, dim3(SPLIT_BX, SPLIT_BY), s, own, oth,
                          reinterpret_cast<const T *>(src) + (size_t)colour * sp.cs, sp, cf, colour, res, iter, thresh,
                          sc);
    }
#endif
    dim3 grid((sp.H + SPLIT_BX - 1) / SPLIT_BX, (sp.ny + SPLIT_BY - 1) / SPLIT_BY, (sp.nx - 2 + NI - 1) / NI);
    return launch_pdl(sor_split_kernel<T, S, NI, MINB>, grid, dim3(SPLIT_BX, SPLIT_BY), s, own, oth,
                      src + (size_t)colour * sp.cs, sp, cf, colour, res, iter, thresh, sc);
}

}  // namespace hc
