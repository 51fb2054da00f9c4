// hydro_kernels.cuh -- the godunov step as CUDA kernels, templated on the
// state type.  Included by hydro_fp64.cu (T = double, compiled -fmad=false so
// that results are bit-identical to the reference) and hydro_fp32.cu.
//
// One step (godunov_step_3d, hydro_solver_3d.c:637-811) is:
//   dt kernel          dt = cfl*min(d/smax) from the max signal speed that
//                      the previous step's kernels reduced (compute_dt_3d,
//                      :422-450, evaluated on the same final state)
//   interior kernel    per interior cell: three HLLC face fluxes per axis
//                      shared through shared memory, flux difference update
//                      (:729-764), floors (:765-768), gravity source (:597-631)
//                      with g = -grad(phi) formed in place, next-step CFL max
//   boundary source    the gravity source on the six faces (never flux-updated,
//                      :729-731) with g copied from the nearest interior cell
//                      (gravity_solver_3d.c:842-897)
//   periodic / bc      hydro_solver_3d.c:779-807 then :456-552, axis by axis
//   boundary CFL       max signal speed of the final face cells
// The state is double-buffered: every kernel reads step-n values and writes
// the step-(n+1) buffer, which is what the reference's separate flux arrays
// give it.
#pragma once
#include "hc_internal.cuh"
#include "hc_math.cuh"

namespace hc {

template <typename T>
__device__ __forceinline__ Cons<T> ld_cons(const T *const *q, long long c)
{
    Cons<T> r;
    r.d = q[0][c]; r.m[0] = q[1][c]; r.m[1] = q[2][c]; r.m[2] = q[3][c]; r.e = q[4][c];
    return r;
}
template <typename T>
__device__ __forceinline__ void st_cons(T *const *q, long long c, const Cons<T> &r)
{
    q[0][c] = r.d; q[1][c] = r.m[0]; q[2][c] = r.m[1]; q[3][c] = r.m[2]; q[4][c] = r.e;
}

template <typename T> struct AccT { typedef double type; };

template <typename T>
__device__ __forceinline__ void block_max_to(T v, unsigned long long *slot64, unsigned int *slot32)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = tmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    __shared__ T wmax[32];
    const int nt = blockDim.x * blockDim.y;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    if ((tid & 31) == 0) wmax[tid >> 5] = v;
    __syncthreads();
    if (tid < 32) {
        T m = (tid < (nt + 31) / 32) ? wmax[tid] : (T)0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = tmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (tid == 0) {
            if (sizeof(T) == 8) atomic_max_nonneg(slot64, (double)m);
            else atomic_max_nonneg(slot32, (float)m);
        }
    }
}

// Per-cell values a face flux needs: conserved state, primitives, sound speed.
template <typename T> struct CellS {
    Cons<T> q;
    Prim<T> w;
    T c;
};

template <typename T>
__device__ __forceinline__ CellS<T> make_cell(const Cons<T> &q, T gm1, T gam)
{
    CellS<T> s;
    s.q = q;
    s.w = to_prim(q, gm1);
    s.c = csound(s.w, gam);
    return s;
}

// --------------------------------------------------------------------------
// interior kernel
// --------------------------------------------------------------------------
template <typename T, int TK, int TJ>
__global__ void __launch_bounds__(TK * TJ)
interior_kernel(HydroArgs a, int ilen)
{
    constexpr int SK = TK + 2, SJ = TJ + 2, NS = SK * SJ;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    CellS<T> *P = reinterpret_cast<CellS<T> *>(smem_raw);            // plane i, tile+halo
    Cons<T> *Qn = reinterpret_cast<Cons<T> *>(P + NS);                 // plane i+1 raw
    Cons<T> *FY = Qn + NS;                                              // (TJ+1) x TK
    Cons<T> *FZ = FY + (TJ + 1) * TK;                                   // TJ x (TK+1)

    const int nx = a.g.nx, ny = a.g.ny, nz = a.g.nz;
    const long long sI = (long long)ny * nz, sJ = nz;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TK + tx;
    const int k0 = blockIdx.x * TK, j0 = blockIdx.y * TJ;
    const int k = k0 + tx, j = j0 + ty;
    const int ib = 1 + blockIdx.z * ilen;
    const int ie = min(nx - 1, ib + ilen);   // exclusive; interior is [1, nx-2]
    if (ib >= ie) return;

    const T *const *qin = reinterpret_cast<const T *const *>(a.qin);
    T *const *qout = reinterpret_cast<T *const *>(a.qout);
    const T gam = (T)a.gamma, gm1 = (T)(a.gamma - 1.0);
    const T dt = (T)a.sc->dt;
    const T dtdx = dt / (T)a.g.dx, dtdy = dt / (T)a.g.dy, dtdz = dt / (T)a.g.dz;
    const double idx2 = 2.0 * a.g.dx, idy2 = 2.0 * a.g.dy, idz2 = 2.0 * a.g.dz;
    const bool own_in = (j < ny) && (k < nz);
    const bool own_int = (j >= 1) && (j <= ny - 2) && (k >= 1) && (k <= nz - 2);

    auto load_plane = [&](int i, Cons<T> *dst) {
        for (int s = tid; s < NS; s += TK * TJ) {
            int sj = s / SK, sk = s - sj * SK;
            int gj = j0 - 1 + sj, gk = k0 - 1 + sk;
            Cons<T> q;
            if (gj >= 0 && gj < ny && gk >= 0 && gk < nz) {
                q = ld_cons(qin, (long long)i * sI + gj * sJ + gk);
            } else {
                q.d = (T)1; q.m[0] = q.m[1] = q.m[2] = (T)0; q.e = (T)1;
            }
            dst[s] = q;
        }
    };
    auto prims_plane = [&]() {
        for (int s = tid; s < NS; s += TK * TJ) P[s] = make_cell(Qn[s], gm1, gam);
    };

    // prologue: plane ib-1 (own cell only) and plane ib (tile + halo)
    CellS<T> me_prev;
    {
        Cons<T> q;
        if (own_in) q = ld_cons(qin, (long long)(ib - 1) * sI + j * sJ + k);
        else { q.d = (T)1; q.m[0] = q.m[1] = q.m[2] = (T)0; q.e = (T)1; }
        me_prev = make_cell(q, gm1, gam);
    }
    load_plane(ib, Qn);
    __syncthreads();
    prims_plane();
    __syncthreads();
    CellS<T> me = P[(ty + 1) * SK + tx + 1];
    Cons<T> fxm = hllc<0>(me_prev.q, me_prev.w, me_prev.c, me.q, me.w, me.c);

    T smax = (T)0;
    for (int i = ib; i < ie; i++) {
        // next plane raw state (tile + halo)
        load_plane(i + 1, Qn);
        __syncthreads();
        CellS<T> nx1 = make_cell(Qn[(ty + 1) * SK + tx + 1], gm1, gam);
        Cons<T> fxp = hllc<0>(me.q, me.w, me.c, nx1.q, nx1.w, nx1.c);
        {
            const CellS<T> &a0 = P[(ty + 1) * SK + tx + 1];
            const CellS<T> &ay = P[(ty + 2) * SK + tx + 1];
            const CellS<T> &az = P[(ty + 1) * SK + tx + 2];
            FY[(ty + 1) * TK + tx] = hllc<1>(a0.q, a0.w, a0.c, ay.q, ay.w, ay.c);
            FZ[ty * (TK + 1) + tx + 1] = hllc<2>(a0.q, a0.w, a0.c, az.q, az.w, az.c);
            if (ty == 0) {
                const CellS<T> &b0 = P[tx + 1];
                FY[tx] = hllc<1>(b0.q, b0.w, b0.c, a0.q, a0.w, a0.c);
            } else if (ty == 1 && tx < TJ) {
                const CellS<T> &c0 = P[(tx + 1) * SK];
                const CellS<T> &c1 = P[(tx + 1) * SK + 1];
                FZ[tx * (TK + 1)] = hllc<2>(c0.q, c0.w, c0.c, c1.q, c1.w, c1.c);
            }
        }
        __syncthreads();
        // P is free again: prepare plane i+1 for the next iteration
        prims_plane();

        if (own_in && own_int) {
            const Cons<T> &yp = FY[(ty + 1) * TK + tx], &ym = FY[ty * TK + tx];
            const Cons<T> &zp = FZ[ty * (TK + 1) + tx + 1], &zm = FZ[ty * (TK + 1) + tx];
            Cons<T> q = me.q;
            q.d = q.d + (-dtdx * (fxp.d - fxm.d) - dtdy * (yp.d - ym.d) - dtdz * (zp.d - zm.d));
#pragma unroll
            for (int c = 0; c < 3; c++)
                q.m[c] = q.m[c] + (-dtdx * (fxp.m[c] - fxm.m[c]) - dtdy * (yp.m[c] - ym.m[c]) -
                                   dtdz * (zp.m[c] - zm.m[c]));
            q.e = q.e + (-dtdx * (fxp.e - fxm.e) - dtdy * (yp.e - ym.e) - dtdz * (zp.e - zm.e));
            // floors: rho floor, then a prim round trip (hydro_solver_3d.c:765-768)
            q.d = tmax(q.d, (T)HC_RHO_FLOOR);
            Prim<T> w = to_prim(q, gm1);
            w.p = tmax(w.p, (T)HC_P_FLOOR);
            q = to_cons(w, gm1);
            const long long c = (long long)i * sI + j * sJ + k;
            if (a.gravity) {
                const double *ph = a.phig;
                double ax = -(__ldg(ph + c + sI) - __ldg(ph + c - sI)) / idx2;
                double ay = -(__ldg(ph + c + sJ) - __ldg(ph + c - sJ)) / idy2;
                double az = -(__ldg(ph + c + 1) - __ldg(ph + c - 1)) / idz2;
                gravity_source(q, ax, ay, az, dt);
            }
            st_cons(qout, c, q);
            smax = tmax(smax, signal_speed(to_prim(q, gm1), gam));
        }
        __syncthreads();
        fxm = fxp;
        me = nx1;
    }
    block_max_to(smax, &a.sc->smax[a.step_parity ^ 1],
                 reinterpret_cast<unsigned int *>(&a.sc->smax[a.step_parity ^ 1]));
}

template <typename T, int TK, int TJ>
constexpr size_t interior_smem()
{
    return sizeof(CellS<T>) * (TK + 2) * (TJ + 2) + sizeof(Cons<T>) * (TK + 2) * (TJ + 2) +
           sizeof(Cons<T>) * ((TJ + 1) * TK + TJ * (TK + 1));
}

// --------------------------------------------------------------------------
// small kernels
// --------------------------------------------------------------------------
template <typename T>
__global__ void dt_kernel(HydroArgs a)
{
    unsigned long long *slots = a.sc->smax;
    T smax;
    if (sizeof(T) == 8) smax = (T)__longlong_as_double((long long)slots[a.step_parity]);
    else smax = (T)__uint_as_float((unsigned int)slots[a.step_parity]);
    T tx = (T)a.g.dx / smax, ty = (T)a.g.dy / smax, tz = (T)a.g.dz / smax;
    T dtv = (T)a.cfl * tmin(tx, tmin(ty, tz));
    a.sc->dt = (double)dtv;
    // initial max speed of compute_dt_3d (hydro_solver_3d.c:423)
    if (sizeof(T) == 8) slots[a.step_parity ^ 1] = (unsigned long long)__double_as_longlong(1.0e-10);
    else slots[a.step_parity ^ 1] = (unsigned long long)__float_as_uint(1.0e-10f);
}

template <typename T>
__global__ void cfl_full_kernel(HydroArgs a)
{
    const T *const *q = reinterpret_cast<const T *const *>(a.qin);
    const T gam = (T)a.gamma, gm1 = (T)(a.gamma - 1.0);
    T m = (T)0;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < a.g.n;
         c += (long long)gridDim.x * blockDim.x)
        m = tmax(m, signal_speed(to_prim(ld_cons(q, c), gm1), gam));
    block_max_to(m, &a.sc->smax[a.step_parity],
                 reinterpret_cast<unsigned int *>(&a.sc->smax[a.step_parity]));
}

template <typename T>
__global__ void boundary_source_kernel(HydroArgs a)
{
    const int nx = a.g.nx, ny = a.g.ny, nz = a.g.nz;
    const long long nb = boundary_count(nx, ny, nz, true);
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= nb) return;
    int i, j, k;
    boundary_cell(t, nx, ny, nz, true, i, j, k);
    const long long sI = (long long)ny * nz, sJ = nz;
    const long long c = i * sI + j * sJ + k;
    const T *const *qin = reinterpret_cast<const T *const *>(a.qin);
    T *const *qout = reinterpret_cast<T *const *>(a.qout);
    Cons<T> q = ld_cons(qin, c);
    if (a.gravity) {
        // g on a boundary cell equals g of the nearest interior cell after the
        // x, y, z copy passes of gravity_compute_acceleration (:842-897)
        int ci = min(max(i, 1), nx - 2), cj = min(max(j, 1), ny - 2), ck = min(max(k, 1), nz - 2);
        long long cc = ci * sI + cj * sJ + ck;
        const double *ph = a.phig;
        double ax = -(ph[cc + sI] - ph[cc - sI]) / (2.0 * a.g.dx);
        double ay = -(ph[cc + sJ] - ph[cc - sJ]) / (2.0 * a.g.dy);
        double az = -(ph[cc + 1] - ph[cc - 1]) / (2.0 * a.g.dz);
        gravity_source(q, ax, ay, az, (T)a.sc->dt);
    }
    st_cons(qout, c, q);
}

// index of (u,v) on the face plane normal to `axis`
__device__ __forceinline__ long long face_index(int axis, int side_idx, int u, int v, int ny, int nz)
{
    const long long sI = (long long)ny * nz, sJ = nz;
    if (axis == 0) return side_idx * sI + u * sJ + v;
    if (axis == 1) return u * sI + side_idx * sJ + v;
    return u * sI + v * sJ + side_idx;
}

template <typename T>
__global__ void periodic_kernel(HydroArgs a, int axis)
{
    const int n[3] = { a.g.nx, a.g.ny, a.g.nz };
    const int nu = (axis == 0) ? n[1] : n[0], nv = (axis == 2) ? n[1] : n[2];
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)nu * nv) return;
    const int u = (int)(t / nv), v = (int)(t % nv);
    T *const *q = reinterpret_cast<T *const *>(a.qout);
    long long c0 = face_index(axis, 0, u, v, n[1], n[2]);
    long long c1 = face_index(axis, n[axis] - 1, u, v, n[1], n[2]);
    Cons<T> s = ld_cons(reinterpret_cast<const T *const *>(a.qout), c1);
    st_cons(q, c0, s);
}

template <typename T>
__global__ void bc_kernel(HydroArgs a, int axis)
{
    const int n[3] = { a.g.nx, a.g.ny, a.g.nz };
    const int nu = (axis == 0) ? n[1] : n[0], nv = (axis == 2) ? n[1] : n[2];
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)nu * nv) return;
    const int u = (int)(t / nv), v = (int)(t % nv);
    T *const *q = reinterpret_cast<T *const *>(a.qout);
    const T *const *qc = reinterpret_cast<const T *const *>(a.qout);
    const T gm1 = (T)(a.gamma - 1.0);
    for (int side = 0; side < 2; side++) {
        int type = a.bc[2 * axis + side];
        int ib = side ? n[axis] - 1 : 0, in = side ? n[axis] - 2 : 1;
        long long cb = face_index(axis, ib, u, v, n[1], n[2]);
        if (type == 1) {            // BC_REFLECTIVE: negate own normal velocity
            Prim<T> w = to_prim(ld_cons(qc, cb), gm1);
            w.v[axis] = -w.v[axis];
            st_cons(q, cb, to_cons(w, gm1));
        } else if (type == 2) {     // BC_OUTFLOW: copy the neighbour
            st_cons(q, cb, ld_cons(qc, face_index(axis, in, u, v, n[1], n[2])));
        }
    }
}

template <typename T>
__global__ void cfl_boundary_kernel(HydroArgs a)
{
    const int nx = a.g.nx, ny = a.g.ny, nz = a.g.nz;
    const long long nb = boundary_count(nx, ny, nz, true);
    const T gam = (T)a.gamma, gm1 = (T)(a.gamma - 1.0);
    const T *const *q = reinterpret_cast<const T *const *>(a.qout);
    T m = (T)0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nb;
         t += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        boundary_cell(t, nx, ny, nz, true, i, j, k);
        long long c = ((long long)i * ny + j) * nz + k;
        m = tmax(m, signal_speed(to_prim(ld_cons(q, c), gm1), gam));
    }
    block_max_to(m, &a.sc->smax[a.step_parity ^ 1],
                 reinterpret_cast<unsigned int *>(&a.sc->smax[a.step_parity ^ 1]));
}

}  // namespace hc
