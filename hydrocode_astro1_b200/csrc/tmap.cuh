// tmap.cuh -- host-side TMA tensor maps over 3D fields (k fastest), cached
// by base pointer, for the bulk-tensor plane loads of the SOR passes.
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

namespace hc {

// Encodes (or returns the cached) map of a 3D array dims (nz, ny, nx) with a
// box of (bk, bj, bi).  Returns false if the driver entry point is missing or
// the layout breaks a TMA rule (16-byte base and row strides).
inline bool tmap3(const void *base, int elem_bytes, int nx, int ny, int nz, int bk, int bj, CUtensorMap *out,
                  int bi = 1)
{
    static std::mutex mu;
    static PFN_cuTensorMapEncodeTiled_v12000 enc = nullptr;
    struct Ent { const void *b; int e, nx, ny, nz, bk, bj, bi; CUtensorMap m; };
    static Ent cache[32];
    static int used = 0, next = 0;
    if ((uintptr_t)base % 16 != 0 || ((long long)nz * elem_bytes) % 16 != 0) return false;
    std::lock_guard<std::mutex> lk(mu);
    for (int t = 0; t < used; t++) {
        const Ent &c = cache[t];
        if (c.b == base && c.e == elem_bytes && c.nx == nx && c.ny == ny && c.nz == nz && c.bk == bk && c.bj == bj &&
            c.bi == bi) {
            *out = c.m;
            return true;
        }
    }
    if (!enc) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn)
            return false;
        enc = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    }
    cuuint64_t dims[3] = { (cuuint64_t)nz, (cuuint64_t)ny, (cuuint64_t)nx };
    cuuint64_t strides[2] = { (cuuint64_t)nz * elem_bytes, (cuuint64_t)ny * nz * elem_bytes };
    cuuint32_t box[3] = { (cuuint32_t)bk, (cuuint32_t)bj, (cuuint32_t)bi };
    cuuint32_t es[3] = { 1, 1, 1 };
    CUtensorMap m;
    CUresult r = enc(&m, elem_bytes == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
                     const_cast<void *>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return false;
    Ent &c = cache[next];
    c = Ent{ base, elem_bytes, nx, ny, nz, bk, bj, bi, m };
    next = (next + 1) % 32;
    if (used < 32) used++;
    *out = m;
    return true;
}

}  // namespace hc
