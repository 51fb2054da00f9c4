// unet.cu -- the learned warm start: launchers of the tcgen05 convolution
// kernels (unet_conv.cuh) and their C-ABI test hooks.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "../../include/hydrocode_b200.h"
#include "unet_conv.cuh"

namespace hc {
namespace unet {

cudaError_t conv3(const __nv_bfloat16 *x, const __nv_bfloat16 *w, const float *bias, void *out, const Dims &d,
                  int out_mode, int act, int *err, cudaStream_t s)
{
    const unsigned blocks = (unsigned)((d.n + TM - 1) / TM);
    conv3_kernel<<<blocks, 128, sizeof(ConvSmem), s>>>(x, w, bias, out, d, out_mode, act, err);
    return cudaGetLastError();
}

// partial: nparts * WG_MT*TM*CH floats, nparts <= max_parts
cudaError_t wgrad(const __nv_bfloat16 *x, const __nv_bfloat16 *dy, float *dw, float *partial, int max_parts,
                  const Dims &d, int *err, cudaStream_t s)
{
    static int attr_dev = -1;
    int dev = 0;
    cudaGetDevice(&dev);
    if (attr_dev != dev) {
        cudaError_t e = cudaFuncSetAttribute(wgrad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)sizeof(WgradSmem));
        if (e != cudaSuccess) return e;
        attr_dev = dev;
    }
    const long long nchunk = (d.n + KC - 1) / KC;
    int parts = (int)std::min<long long>(max_parts, nchunk);
    const int per = (int)((nchunk + parts - 1) / parts);
    parts = (int)((nchunk + per - 1) / per);
    wgrad_kernel<<<parts, WG_NT, sizeof(WgradSmem), s>>>(x, dy, partial, d, per, err);
    wgrad_reduce_kernel<<<(WELEM + 255) / 256, 256, 0, s>>>(partial, parts, dw);
    return cudaGetLastError();
}

}  // namespace unet
}  // namespace hc

using namespace hc;

namespace {
struct DevBuf {
    void *p = nullptr;
    ~DevBuf() { cudaFree(p); }
    cudaError_t alloc(size_t n) { return cudaMalloc(&p, n); }
};
}  // namespace

// Diagnostic: one convolution of a 16-channel BF16 volume (host buffers).
extern "C" int hc_unet_conv_test(int nx, int ny, int nz, const uint16_t *x, const uint16_t *w, const float *bias,
                                 int out_mode, int act, float *out)
{
    if (nx < 1 || ny < 1 || nz < 1 || !x || !w || !bias || !out || out_mode < 0 || out_mode > 3) return HC_ERR_ARG;
    unet::Dims d{ nx, ny, nz, (long long)nx * ny * nz };
    const size_t nv = (size_t)d.n;
    DevBuf dx, dw, db, dout, derr;
    const size_t out_bytes = (out_mode == 2) ? nv * 4 : (out_mode == 3 ? nv * 16 * 4 : nv * 16 * 2);
    if (dx.alloc(nv * 32) || dw.alloc(unet::WELEM * 2) || db.alloc(64) || dout.alloc(out_bytes) || derr.alloc(4))
        return HC_ERR_NOMEM;
    cudaMemcpy(dx.p, x, nv * 32, cudaMemcpyHostToDevice);
    cudaMemcpy(dw.p, w, unet::WELEM * 2, cudaMemcpyHostToDevice);
    cudaMemcpy(db.p, bias, 64, cudaMemcpyHostToDevice);
    cudaMemset(derr.p, 0, 4);
    if (unet::conv3((const __nv_bfloat16 *)dx.p, (const __nv_bfloat16 *)dw.p, (const float *)db.p, dout.p, d, out_mode,
                    act, (int *)derr.p, 0) != cudaSuccess)
        return HC_ERR_CUDA;
    if (cudaDeviceSynchronize() != cudaSuccess) return HC_ERR_CUDA;
    int e = 0;
    cudaMemcpy(&e, derr.p, 4, cudaMemcpyDeviceToHost);
    if (out_mode == 2 || out_mode == 3) {
        cudaMemcpy(out, dout.p, out_bytes, cudaMemcpyDeviceToHost);
    } else {
        std::vector<uint16_t> h(nv * 16);
        cudaMemcpy(h.data(), dout.p, out_bytes, cudaMemcpyDeviceToHost);
        for (size_t t = 0; t < nv * 16; t++) {
            uint32_t b = (uint32_t)h[t] << 16;
            memcpy(&out[t], &b, 4);
        }
    }
    return e ? e : HC_OK;
}

// Diagnostic: weight gradient dW[co][tap][ci] of one convolution (host buffers).
extern "C" int hc_unet_wgrad_test(int nx, int ny, int nz, const uint16_t *x, const uint16_t *dy, int max_parts,
                                  float *dw)
{
    if (nx < 1 || ny < 1 || nz < 1 || !x || !dy || !dw || max_parts < 1) return HC_ERR_ARG;
    unet::Dims d{ nx, ny, nz, (long long)nx * ny * nz };
    const size_t nv = (size_t)d.n;
    DevBuf dx, ddy, ddw, dpart, derr;
    if (dx.alloc(nv * 32) || ddy.alloc(nv * 32) || ddw.alloc(unet::WELEM * 4) ||
        dpart.alloc((size_t)max_parts * unet::WG_MT * unet::TM * unet::CH * 4) || derr.alloc(4))
        return HC_ERR_NOMEM;
    cudaMemcpy(dx.p, x, nv * 32, cudaMemcpyHostToDevice);
    cudaMemcpy(ddy.p, dy, nv * 32, cudaMemcpyHostToDevice);
    cudaMemset(derr.p, 0, 4);
    if (unet::wgrad((const __nv_bfloat16 *)dx.p, (const __nv_bfloat16 *)ddy.p, (float *)ddw.p, (float *)dpart.p,
                    max_parts, d, (int *)derr.p, 0) != cudaSuccess)
        return HC_ERR_CUDA;
    if (cudaDeviceSynchronize() != cudaSuccess) return HC_ERR_CUDA;
    int e = 0;
    cudaMemcpy(&e, derr.p, 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(dw, ddw.p, unet::WELEM * 4, cudaMemcpyDeviceToHost);
    return e ? e : HC_OK;
}
