// unet.cu -- the learned warm start: launchers of the tcgen05 convolution
// kernels (unet_conv.cuh) and their C-ABI test hooks.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <atomic>

#include <algorithm>
#include <cstdlib>
#include <mutex>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "../../include/hydrocode_b200.h"
#include "hc_internal.cuh"
#include "unet_conv.cuh"

#ifndef HC_HALO_MIN_PLANES
#define HC_HALO_MIN_PLANES 1   // fewest output planes a halo-convolution CTA walks: 1 keeps the
                                 // chains of the small levels short (U-Net 1.185 -> 1.127 ms per step
                                 // at 256^3 against 4)
#endif

namespace hc {
namespace unet {

// 4D BF16 tensor map (c = 16, k, j, i) of a channels-last volume with a
// {8, 10, 18, 1} box (one channel half of a halo plane), cached by pointer
// and dimensions.  false if the driver entry point is missing or the layout
// breaks a TMA rule.
static bool halo_map(const __nv_bfloat16 *x, const Dims &d, CUtensorMap *out)
{
    static std::mutex mu;
    static PFN_cuTensorMapEncodeTiled_v12000 enc = nullptr;
    struct Ent { const void *p; int nx, ny, nz; CUtensorMap m; };
    static Ent cache[64];
    static int used = 0, next = 0;
    if ((uintptr_t)x % 16) return false;
    std::lock_guard<std::mutex> lk(mu);
    for (int t = 0; t < used; t++)
        if (cache[t].p == x && cache[t].nx == d.nx && cache[t].ny == d.ny && cache[t].nz == d.nz) {
            *out = cache[t].m;
            return true;
        }
    if (!enc) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn)
            return false;
        enc = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    }
    cuuint64_t dims[4] = { (cuuint64_t)CH, (cuuint64_t)d.nz, (cuuint64_t)d.ny, (cuuint64_t)d.nx };
    cuuint64_t strides[3] = { (cuuint64_t)CH * 2, (cuuint64_t)d.nz * CH * 2, (cuuint64_t)d.ny * d.nz * CH * 2 };
    cuuint32_t box[4] = { 8, (cuuint32_t)HH_K, (cuuint32_t)HH_J, 1 };
    cuuint32_t es[4] = { 1, 1, 1, 1 };
    CUtensorMap m;
    if (enc(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<__nv_bfloat16 *>(x), dims, strides, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
    cache[next] = Ent{ x, d.nx, d.ny, d.nz, m };
    next = (next + 1) % 64;
    if (used < 64) used++;
    *out = m;
    return true;
}

static bool halo_enabled()
{
    static int on = -1;
    if (on < 0) {
        const char *e = getenv("HC_NO_TMA");
        on = (e && atoi(e) != 0) ? 0 : 1;
    }
    return on == 1;
}

cudaError_t conv3(const __nv_bfloat16 *x, const __nv_bfloat16 *w, const float *bias, void *out, const Dims &d,
                  int out_mode, int act, int *err, cudaStream_t s)
{
    CUtensorMap tm;
    if (halo_enabled() && halo_map(x, d, &tm)) {
        static std::atomic<unsigned long long> attr_set{0};
        cudaError_t e = hc::set_smem_once(attr_set, (const void *)conv3_halo_kernel, (int)sizeof(HaloSmem));
        if (e != cudaSuccess) return e;
        const int tk = (d.nz + HT_K - 1) / HT_K, tj = (d.ny + HT_J - 1) / HT_J;
        // 6 CTAs per SM (shared-memory limit): as many plane chunks as fit one
        // wave (rounding up would leave a second, nearly empty wave); at least
        // HC_HALO_MIN_PLANES planes per CTA
        const long long want = 148LL * 6;
        int chunks = (int)std::max(1LL, std::min((long long)(d.nx + HC_HALO_MIN_PLANES - 1) / HC_HALO_MIN_PLANES,
                                                 want / ((long long)tk * tj)));
        const int chunk = (d.nx + chunks - 1) / chunks;
        chunks = (d.nx + chunk - 1) / chunk;
        conv3_halo_kernel<<<dim3(tk, tj, chunks), 128, sizeof(HaloSmem), s>>>(tm, w, bias, out, d, out_mode, act,
                                                                              chunk, err);
        return cudaGetLastError();
    }
    const unsigned blocks = (unsigned)((d.n + TM - 1) / TM);
    conv3_kernel<<<blocks, 128, sizeof(ConvSmem), s>>>(x, w, bias, out, d, out_mode, act, err);
    return cudaGetLastError();
}

// partial: nparts * WG_MT*TM*CH floats, nparts <= max_parts
cudaError_t wgrad(const __nv_bfloat16 *x, const __nv_bfloat16 *dy, float *dw, float *partial, int max_parts,
                  const Dims &d, int *err, cudaStream_t s)
{
    static std::atomic<unsigned long long> attr_set{0};
    cudaError_t e = hc::set_smem_once(attr_set, (const void *)wgrad_kernel, (int)sizeof(WgradSmem));
    if (e != cudaSuccess) return e;
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

// ---------------------------------------------------------------------------
// The network: a 3D U-Net on the half-resolution grid of the solve, with
// NLEV = 4 pooling levels (level l has grid / 2^(l+1) cells per side):
//   x0 (channel 0 = 2x-pooled FP64 residual / its RMS)
//   e0 = f(conv0 x0);  e_l = f(conv_l pool e_{l-1})          l = 1..NLEV
//   d_l = f(conv_{2 NLEV - l} (up h + e_l)), h = e_NLEV then d_{l+1},  l = NLEV-1..0
//   out = conv_{2 NLEV + 1} d0 (channel 0)
// f = LeakyReLU(0.1); pool = 2x average; up = 2x nearest.  16 channels at
// every level; 2 NLEV + 2 = 10 convolutions, 56,305 trainable parameters.
// The correction of the solve is  e = trilinear_up(out) * RMS(pooled residual) * kscale.
// ---------------------------------------------------------------------------
#include "unet_ops.cuh"

namespace hc {

namespace unet {
constexpr int NLEV = 4;                           // pooling levels
constexpr int NCONV = 2 * NLEV + 2;
constexpr int PFULL = WELEM + CH;                 // weights + bias of one conv, full layout
constexpr int NFULL = NCONV * PFULL;
constexpr int NPARAM = (CH * NTAP + CH) + (NCONV - 2) * (WELEM + CH) + (NTAP * CH + 1);   // 56305
constexpr int MAX_PARTS = 148;
}  // namespace unet

using namespace unet;

struct UNetState {
    int dev = 0;
    float kscale = 30.f;
    bool have_weights = false;
    int adam_t = 0;
    // parameters (full layout, FP32) and Adam moments, gradients
    float *pm = nullptr, *pg = nullptr, *am = nullptr, *av = nullptr;
    __nv_bfloat16 *wf = nullptr, *wt = nullptr;    // NCONV x WELEM each
    // buffers for one grid size
    int gx = 0, gy = 0, gz = 0;
    Dims L[NLEV + 1];
    __nv_bfloat16 *x0;
    // per level: encoder output e, its pooled input p (l >= 1), decoder input
    // sum s and output d (l < NLEV), gradient buffers ga, gb (skip), gc
    __nv_bfloat16 *e[NLEV + 1], *p[NLEV + 1], *sm[NLEV + 1], *d[NLEV + 1];
    __nv_bfloat16 *ga[NLEV + 1], *gb[NLEV + 1], *gc[NLEV + 1];
    float *out0 = nullptr, *pooled = nullptr, *xnorm = nullptr, *partial = nullptr, *bpart = nullptr;
    double *scal = nullptr;       // [0] sumsq of the input, [1] sum t^2, [2] loss
    double *rpart = nullptr;      // per-block partial sums of the input's squares (NRPART)
    int *err = nullptr;
    void *act_mem = nullptr;
    // training samples: normalised inputs and targets at level 0
    int cap = 0, count = 0, next = 0, slot = -1;
    float *sx = nullptr, *st = nullptr;
    std::vector<double> st2;
    double *phi0 = nullptr;
    long long phi0_n = 0;
    std::vector<void *> fixed;
};

namespace {
int dalloc(void **p, size_t bytes)
{
    if (cudaMalloc(p, bytes) != cudaSuccess) {
        *p = nullptr;
        return HC_ERR_NOMEM;
    }
    return HC_OK;
}
constexpr int NRPART = 148 * 16;   // the most blocks nblk() gives
inline unsigned nblk(long long n, int nt = 256)
{
    long long b = (n + nt - 1) / nt;
    return (unsigned)std::max<long long>(1, std::min<long long>(b, 148LL * 16));
}
__nv_bfloat16 *wf_of(UNetState *u, int l) { return u->wf + (size_t)l * WELEM; }
__nv_bfloat16 *wt_of(UNetState *u, int l) { return u->wt + (size_t)l * WELEM; }
float *bias_of(UNetState *u, int l) { return u->pm + (size_t)l * PFULL + WELEM; }

// compact <-> full parameter layouts (host)
void compact_to_full(const float *c, std::vector<float> &f)
{
    f.assign(NFULL, 0.f);
    size_t q = 0;
    for (int l = 0; l < NCONV; l++) {
        float *w = f.data() + (size_t)l * PFULL, *b = w + WELEM;
        if (l == 0) {
            for (int co = 0; co < CH; co++)
                for (int tap = 0; tap < NTAP; tap++) w[(co * NTAP + tap) * CH] = c[q++];
            for (int co = 0; co < CH; co++) b[co] = c[q++];
        } else if (l == NCONV - 1) {
            for (int tap = 0; tap < NTAP; tap++)
                for (int ci = 0; ci < CH; ci++) w[tap * CH + ci] = c[q++];
            b[0] = c[q++];
        } else {
            for (int e = 0; e < WELEM; e++) w[e] = c[q++];
            for (int co = 0; co < CH; co++) b[co] = c[q++];
        }
    }
}
void full_to_compact(const std::vector<float> &f, float *c)
{
    size_t q = 0;
    for (int l = 0; l < NCONV; l++) {
        const float *w = f.data() + (size_t)l * PFULL, *b = w + WELEM;
        if (l == 0) {
            for (int co = 0; co < CH; co++)
                for (int tap = 0; tap < NTAP; tap++) c[q++] = w[(co * NTAP + tap) * CH];
            for (int co = 0; co < CH; co++) c[q++] = b[co];
        } else if (l == NCONV - 1) {
            for (int tap = 0; tap < NTAP; tap++)
                for (int ci = 0; ci < CH; ci++) c[q++] = w[tap * CH + ci];
            c[q++] = b[0];
        } else {
            for (int e = 0; e < WELEM; e++) c[q++] = w[e];
            for (int co = 0; co < CH; co++) c[q++] = b[co];
        }
    }
}

cudaError_t pack_all(UNetState *u, cudaStream_t s)
{
    for (int l = 0; l < NCONV; l++)
        pack_weights_kernel<<<(WELEM + 255) / 256, 256, 0, s>>>(u->pm + (size_t)l * PFULL, wf_of(u, l), wt_of(u, l));
    return cudaGetLastError();
}

void free_grid(UNetState *u)
{
    cudaFree(u->act_mem);
    u->act_mem = nullptr;
    u->gx = u->gy = u->gz = 0;
}

// Buffers for a solve grid of gx x gy x gz cells (each a multiple of 16).
int ensure_grid(UNetState *u, int gx, int gy, int gz)
{
    constexpr int MULT = 2 << NLEV;   // every level has integer dims
    if (gx % MULT || gy % MULT || gz % MULT) return HC_ERR_ARG;
    if (u->gx == gx && u->gy == gy && u->gz == gz) return HC_OK;
    free_grid(u);
    size_t nbf = 0;
    for (int l = 0; l <= NLEV; l++) {
        const int f = 2 << l;
        u->L[l] = Dims{ gx / f, gy / f, gz / f, (long long)(gx / f) * (gy / f) * (gz / f) };
        nbf += (size_t)u->L[l].n * CH * (l == 0 ? 8 : 7);
    }
    const size_t nf = 3 * (size_t)u->L[0].n + (size_t)MAX_PARTS * WG_MT * TM * CH + 148 * 16 * CH;
    const size_t bytes = nbf * 2 + nf * 4 + (4 + NRPART) * sizeof(double) + 256 * 4;
    if (dalloc(&u->act_mem, bytes)) return HC_ERR_NOMEM;
    char *p = (char *)u->act_mem;
    auto take_bf = [&](size_t n) { __nv_bfloat16 *r = (__nv_bfloat16 *)p; p += n * 2; return r; };
    for (int l = 0; l <= NLEV; l++) {
        const size_t v = (size_t)u->L[l].n * CH;
        if (l == 0) u->x0 = take_bf(v);
        u->e[l] = take_bf(v);
        u->p[l] = l ? take_bf(v) : nullptr;
        u->sm[l] = take_bf(v);
        u->d[l] = take_bf(v);
        u->ga[l] = take_bf(v);
        u->gb[l] = take_bf(v);
        u->gc[l] = take_bf(v);
    }
    auto take_f = [&](size_t n) { float *r = (float *)p; p += n * 4; return r; };
    u->out0 = take_f(u->L[0].n); u->pooled = take_f(u->L[0].n); u->xnorm = take_f(u->L[0].n);
    u->partial = take_f((size_t)MAX_PARTS * WG_MT * TM * CH);
    u->bpart = take_f(148 * 16 * CH);
    p = (char *)(((uintptr_t)p + 15) & ~(uintptr_t)15);
    u->scal = (double *)p; p += 4 * sizeof(double);
    u->rpart = (double *)p; p += NRPART * sizeof(double);
    u->err = (int *)p;
    u->gx = gx; u->gy = gy; u->gz = gz;
    // samples of another grid size are dropped
    cudaFree(u->sx); cudaFree(u->st);
    u->sx = u->st = nullptr;
    u->count = u->next = 0;
    u->slot = -1;
    u->st2.clear();
    if (u->cap > 0) {
        if (dalloc((void **)&u->sx, (size_t)u->cap * u->L[0].n * 4) ||
            dalloc((void **)&u->st, (size_t)u->cap * u->L[0].n * 4))
            return HC_ERR_NOMEM;
        u->st2.assign(u->cap, 0.0);
    }
    cudaMemset(u->err, 0, 4);
    return HC_OK;
}

cudaError_t conv_fwd(UNetState *u, int l, const __nv_bfloat16 *x, void *out, int lev, int mode, cudaStream_t s)
{
    return conv3(x, wf_of(u, l), bias_of(u, l), out, u->L[lev], mode, mode == 0 ? 1 : 0, u->err, s);
}
cudaError_t conv_dgrad(UNetState *u, int l, const __nv_bfloat16 *dy, __nv_bfloat16 *dx, int lev, cudaStream_t s)
{
    return conv3(dy, wt_of(u, l), bias_of(u, l), dx, u->L[lev], 1, 0, u->err, s);
}
cudaError_t conv_wgrad(UNetState *u, int l, const __nv_bfloat16 *x, const __nv_bfloat16 *dz, int lev, cudaStream_t s)
{
    float *g = u->pg + (size_t)l * PFULL;
    cudaError_t e = wgrad(x, dz, g, u->partial, MAX_PARTS, u->L[lev], u->err, s);
    if (e != cudaSuccess) return e;
    const unsigned nb = std::min<unsigned>(148, nblk(u->L[lev].n * 2, BG_NT));
    bias_grad_kernel<<<nb, BG_NT, 0, s>>>(dz, u->L[lev].n, u->bpart);
    sum_partials_kernel<<<1, 32, 0, s>>>(u->bpart, nb, g + WELEM, CH);
    return cudaGetLastError();
}

// Forward pass from the single-channel input in u->pooled, scaled by 1 / rms
// (sumsq != NULL: its sum of squares) or taken as is (sumsq == NULL).
cudaError_t forward(UNetState *u, const double *sumsq, cudaStream_t s)
{
    const Dims *L = u->L;
    cudaError_t e;
    // one thread per DK voxels along k, 128-thread blocks (136 registers: 64
    // packed accumulators)
    const unsigned nfirst = (unsigned)std::min<long long>((L[0].n / DK + 127) / 128, 148LL * 12);
    conv_first_kernel<<<nfirst, 128, 0, s>>>(u->pooled, sumsq, L[0], wf_of(u, 0), bias_of(u, 0), u->e[0]);
    for (int l = 1; l <= NLEV; l++) {
        pool2_kernel<<<nblk(L[l].n * 2), 256, 0, s>>>(u->e[l - 1], u->p[l], L[l]);
        if ((e = conv_fwd(u, l, u->p[l], u->e[l], l, 0, s))) return e;
    }
    const __nv_bfloat16 *h = u->e[NLEV];
    for (int l = NLEV - 1; l >= 0; l--) {
        up_add_kernel<<<nblk(L[l].n * 2), 256, 0, s>>>(h, u->e[l], u->sm[l], L[l]);
        if ((e = conv_fwd(u, 2 * NLEV - l, u->sm[l], u->d[l], l, 0, s))) return e;
        h = u->d[l];
    }
    // the output convolution (16 -> 1 channel) on the tensor cores: the
    // CUDA-core conv_last_kernel measured 283 us per 128^3 launch against
    // ~80 us here
    return conv_fwd(u, NCONV - 1, u->d[0], u->out0, 0, 2, s);
}

// gradients of the loss whose output gradient is in ga[0] (channel 0)
cudaError_t backward(UNetState *u, cudaStream_t s)
{
    const Dims *L = u->L;
    cudaError_t e;
    // output conv (no activation), then the decoder from level 0 down
    if ((e = conv_wgrad(u, NCONV - 1, u->d[0], u->ga[0], 0, s))) return e;
    if ((e = conv_dgrad(u, NCONV - 1, u->ga[0], u->gc[0], 0, s))) return e;
    act_back_kernel<<<nblk(L[0].n * 2), 256, 0, s>>>(u->gc[0], u->d[0], u->ga[0], L[0].n);   // dz of d0
    for (int l = 0; l < NLEV; l++) {
        const int c = 2 * NLEV - l;
        if ((e = conv_wgrad(u, c, u->sm[l], u->ga[l], l, s))) return e;
        if ((e = conv_dgrad(u, c, u->ga[l], u->gb[l], l, s))) return e;   // d(sum): skip part kept in gb
        // through the upsample into the level below: d_{l+1}, or e_NLEV at the bottom
        const __nv_bfloat16 *yb = (l + 1 < NLEV) ? u->d[l + 1] : u->e[NLEV];
        downsum_act_kernel<<<nblk(L[l + 1].n * 2), 256, 0, s>>>(u->gb[l], yb, u->ga[l + 1], L[l + 1]);
    }
    // encoder from the bottom: ga[l] holds dz of e_l
    for (int l = NLEV; l >= 1; l--) {
        if ((e = conv_wgrad(u, l, u->p[l], u->ga[l], l, s))) return e;
        if ((e = conv_dgrad(u, l, u->ga[l], u->gc[l], l, s))) return e;   // d(pooled input)
        poolback_add_act_kernel<<<nblk(L[l - 1].n * 2), 256, 0, s>>>(u->gb[l - 1], u->gc[l], u->e[l - 1],
                                                                       u->ga[l - 1], L[l - 1]);
    }
    return conv_wgrad(u, 0, u->x0, u->ga[0], 0, s);
}

// loss (relative squared error) of the current output against target t,
// with its gradient into ga[0]; adds loss into scal[2]
cudaError_t loss_grad(UNetState *u, const float *t, double sumt2, cudaStream_t s)
{
    loss_kernel<<<nblk(u->L[0].n * 2), 256, 0, s>>>(u->out0, t, u->L[0].n, sumt2, u->ga[0], u->scal + 2);
    return cudaGetLastError();
}

cudaError_t adam_step(UNetState *u, float lr, cudaStream_t s)
{
    u->adam_t++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - powf(b1, (float)u->adam_t), c2 = 1.f - powf(b2, (float)u->adam_t);
    adam_kernel<<<(NFULL + 255) / 256, 256, 0, s>>>(u->pm, u->pg, u->am, u->av, NFULL, lr, b1, b2, 1e-8f, c1, c2);
    return pack_all(u, s);
}

int read_err(UNetState *u, cudaStream_t s)
{
    int e = 0;
    if (cudaMemcpyAsync(&e, u->err, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess) return HC_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return HC_ERR_CUDA;
    if (e) {
        cudaMemsetAsync(u->err, 0, 4, s);
        return HC_ERR_TIMEOUT;
    }
    return HC_OK;
}
}  // namespace

int unet_param_count() { return NPARAM; }

UNetState *unet_create(int dev)
{
    UNetState *u = new UNetState();
    u->dev = dev;
    void *m = nullptr;
    const size_t bytes = (size_t)4 * NFULL * 4 + (size_t)2 * NCONV * WELEM * 2;
    if (dalloc(&m, bytes)) {
        delete u;
        return nullptr;
    }
    u->fixed.push_back(m);
    u->pm = (float *)m;
    u->pg = u->pm + NFULL;
    u->am = u->pg + NFULL;
    u->av = u->am + NFULL;
    u->wf = (__nv_bfloat16 *)(u->av + NFULL);
    u->wt = u->wf + (size_t)NCONV * WELEM;
    cudaMemset(m, 0, bytes);
    return u;
}

void unet_destroy(UNetState *u)
{
    if (!u) return;
    free_grid(u);
    cudaFree(u->sx);
    cudaFree(u->st);
    cudaFree(u->phi0);
    for (void *p : u->fixed) cudaFree(p);
    delete u;
}

bool unet_has_weights(const UNetState *u) { return u && u->have_weights; }
float unet_kscale(const UNetState *u) { return u->kscale; }

int unet_set_params(UNetState *u, const float *compact, int n, float kscale, cudaStream_t s)
{
    if (n != NPARAM || !compact || !(kscale > 0.f)) return HC_ERR_ARG;
    std::vector<float> f;
    compact_to_full(compact, f);
    if (cudaMemcpyAsync(u->pm, f.data(), (size_t)NFULL * 4, cudaMemcpyHostToDevice, s) != cudaSuccess) return HC_ERR_CUDA;
    cudaMemsetAsync(u->am, 0, (size_t)2 * NFULL * 4, s);   // am, av adjacent
    u->adam_t = 0;
    u->kscale = kscale;
    if (pack_all(u, s) != cudaSuccess) return HC_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return HC_ERR_CUDA;
    u->have_weights = true;
    return HC_OK;
}

int unet_get_params(UNetState *u, float *compact, int n, cudaStream_t s)
{
    if (n != NPARAM || !compact) return HC_ERR_ARG;
    std::vector<float> f(NFULL);
    if (cudaMemcpyAsync(f.data(), u->pm, (size_t)NFULL * 4, cudaMemcpyDeviceToHost, s) != cudaSuccess) return HC_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return HC_ERR_CUDA;
    full_to_compact(f, compact);
    return HC_OK;
}

// uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights and biases
int unet_init(UNetState *u, unsigned seed, cudaStream_t s)
{
    std::mt19937 rng(seed);
    std::vector<float> c(NPARAM);
    size_t q = 0;
    for (int l = 0; l < NCONV; l++) {
        const int fan = NTAP * (l == 0 ? 1 : CH);
        const float b = 1.f / std::sqrt((float)fan);
        std::uniform_real_distribution<float> U(-b, b);
        const int nw = (l == 0 || l == NCONV - 1) ? CH * NTAP : WELEM;
        const int nb = (l == NCONV - 1) ? 1 : CH;
        for (int t = 0; t < nw + nb; t++) c[q++] = U(rng);
    }
    return unet_set_params(u, c.data(), NPARAM, 30.f, s);
}

int unet_collect(UNetState *u, int capacity)
{
    if (capacity < 0) return HC_ERR_ARG;
    cudaFree(u->sx);
    cudaFree(u->st);
    u->sx = u->st = nullptr;
    u->cap = capacity;
    u->count = u->next = 0;
    u->slot = -1;
    u->st2.assign(capacity, 0.0);
    if (capacity > 0 && u->gx) {
        if (dalloc((void **)&u->sx, (size_t)capacity * u->L[0].n * 4) ||
            dalloc((void **)&u->st, (size_t)capacity * u->L[0].n * 4))
            return HC_ERR_NOMEM;
    }
    return HC_OK;
}

int unet_samples(const UNetState *u) { return u ? u->count : 0; }
bool unet_collecting(const UNetState *u) { return u && u->cap > 0; }

// At the start of a mixed-precision solve, after the first FP64 residual
// (r32, colour split): prepare the network input and, when `e_out` is given,
// predict the correction into it (colour split, zero on boundary cells).
// When collecting, also record the input and a copy of phi for the target.
int unet_begin_solve(UNetState *u, const GravArgs &a, const float *r32, float *e_out, bool record, cudaStream_t s)
{
    int rc = ensure_grid(u, a.g.nx, a.g.ny, a.g.nz);
    if (rc) return rc;
    const Split sp = make_split(a.g);
    const unsigned npool = nblk(u->L[0].n);
    in_pool_kernel<<<npool, 256, 0, s>>>(r32, sp, u->L[0], u->pooled, u->rpart);
    sum_parts_kernel<<<1, 32, 0, s>>>(u->rpart, (int)npool, u->scal);
    const bool collect = record && u->cap > 0 && u->sx;
    u->slot = collect ? u->next : -1;
    float *xs = collect ? u->sx + (size_t)u->slot * u->L[0].n : nullptr;
    // the normalised input as a training sample (the prediction reads the
    // pooled residual and its scale directly)
    if (collect) in_norm_kernel<<<nblk(u->L[0].n * 2), 256, 0, s>>>(u->pooled, u->scal, u->L[0].n, u->x0, xs);
    if (collect) {
        if (u->phi0_n != a.g.n) {
            cudaFree(u->phi0);
            if (dalloc((void **)&u->phi0, (size_t)a.g.n * 8)) return HC_ERR_NOMEM;
            u->phi0_n = a.g.n;
        }
        cudaMemcpyAsync(u->phi0, a.phi, (size_t)a.g.n * 8, cudaMemcpyDeviceToDevice, s);
    }
    if (e_out) {
        if (!u->have_weights) return HC_ERR_STATE;
        if (forward(u, u->scal, s) != cudaSuccess) return HC_ERR_CUDA;
        out_up_kernel<<<(unsigned)(((long long)a.g.nx * a.g.ny + OUT_UP_ROWS - 1) / OUT_UP_ROWS), 128, 0, s>>>(
            u->out0, u->L[0], u->scal, u->kscale, sp, e_out);
    }
    return cudaGetLastError() == cudaSuccess ? HC_OK : HC_ERR_CUDA;
}

// At the end of a converged solve: the recorded sample's target.
int unet_end_solve(UNetState *u, const GravArgs &a, bool converged, cudaStream_t s)
{
    if (u->slot < 0) return HC_OK;
    const int slot = u->slot;
    u->slot = -1;
    if (!converged) return HC_OK;
    cudaMemsetAsync(u->scal + 1, 0, sizeof(double), s);
    target_kernel<<<nblk(u->L[0].n), 256, 0, s>>>(a.phi, u->phi0, a.g, u->L[0], u->scal, u->kscale,
                                                  u->st + (size_t)slot * u->L[0].n, u->scal + 1);
    double t2 = 0.0;
    if (cudaMemcpyAsync(&t2, u->scal + 1, sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess) return HC_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return HC_ERR_CUDA;
    if (!(t2 > 0.0)) return HC_OK;   // nothing to learn from a zero correction
    u->st2[slot] = t2;
    u->next = (u->next + 1) % u->cap;
    u->count = std::min(u->count + 1, u->cap);
    return HC_OK;
}

// `steps` Adam steps (learning rate decayed from lr to 0 on a cosine), each on
// one stored sample (a seeded random order) under a random symmetry of the
// box (48 for a cubic grid, 8 flips otherwise); mean loss of the last quarter
int unet_train(UNetState *u, int steps, double lr, unsigned seed, double *mean_loss, cudaStream_t s)
{
    if (steps < 0 || !(lr > 0.0)) return HC_ERR_ARG;
    if (u->count == 0) return HC_ERR_STATE;
    std::mt19937 rng(seed);
    const long long n0 = u->L[0].n;
    double acc = 0.0;
    int nacc = 0;
    const int tail = std::max(1, steps / 4);
    cudaMemsetAsync(u->scal + 2, 0, sizeof(double), s);
    const Dims &d0 = u->L[0];
    const bool cube = d0.nx == d0.ny && d0.ny == d0.nz;
    static const int perms[6][3] = { { 0, 1, 2 }, { 0, 2, 1 }, { 1, 0, 2 }, { 1, 2, 0 }, { 2, 0, 1 }, { 2, 1, 0 } };
    for (int k = 0; k < steps; k++) {
        const int smp = (int)(rng() % (unsigned)u->count);
        // a random symmetry of the (cubic) box: the map residual -> correction
        // commutes with it, so the transformed pair is another valid sample
        const int pi = cube ? (int)(rng() % 6u) : 0, flips = (int)(rng() % 8u);
        const int sym = perms[pi][0] | (perms[pi][1] << 2) | (perms[pi][2] << 4) | (flips << 6);
        symmetry_kernel<<<nblk(n0), 256, 0, s>>>(u->sx + (size_t)smp * n0, u->pooled, d0, sym);
        symmetry_kernel<<<nblk(n0), 256, 0, s>>>(u->st + (size_t)smp * n0, u->xnorm, d0, sym);
        in_expand_kernel<<<nblk(n0 * 2), 256, 0, s>>>(u->pooled, n0, u->x0);
        if (forward(u, nullptr, s) != cudaSuccess) return HC_ERR_CUDA;
        if (k == steps - tail) cudaMemsetAsync(u->scal + 2, 0, sizeof(double), s);
        if (loss_grad(u, u->xnorm, u->st2[smp], s) != cudaSuccess) return HC_ERR_CUDA;
        if (backward(u, s) != cudaSuccess) return HC_ERR_CUDA;
        // cosine decay of the learning rate over this call's steps
        const double lrk = lr * 0.5 * (1.0 + std::cos(3.14159265358979 * k / std::max(1, steps)));
        if (adam_step(u, (float)lrk, s) != cudaSuccess) return HC_ERR_CUDA;
        if (k >= steps - tail) nacc++;
    }
    int rc = read_err(u, s);
    if (rc) return rc;
    if (cudaMemcpyAsync(&acc, u->scal + 2, sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess) return HC_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return HC_ERR_CUDA;
    u->have_weights = true;
    if (mean_loss) *mean_loss = nacc ? acc / nacc : 0.0;
    return HC_OK;
}

// One forward + backward on host data at level-0 dims (x: normalised input,
// t: target, n0 values each): the loss and the compact gradient.
int unet_loss_grad(UNetState *u, int n0x, int n0y, int n0z, const float *x, const float *t, double *loss,
                   float *grad, float *out, cudaStream_t s)
{
    int rc = ensure_grid(u, 2 * n0x, 2 * n0y, 2 * n0z);
    if (rc) return rc;
    const long long n0 = u->L[0].n;
    float *dx = u->pooled, *dt = u->xnorm;   // free level-0 FP32 buffers
    cudaMemcpyAsync(dx, x, n0 * 4, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dt, t, n0 * 4, cudaMemcpyHostToDevice, s);
    double t2 = 0.0;
    for (long long v = 0; v < n0; v++) t2 += (double)t[v] * t[v];
    in_expand_kernel<<<nblk(n0 * 2), 256, 0, s>>>(dx, n0, u->x0);
    if (forward(u, nullptr, s) != cudaSuccess) return HC_ERR_CUDA;
    cudaMemsetAsync(u->scal + 2, 0, sizeof(double), s);
    cudaMemsetAsync(u->pg, 0, (size_t)NFULL * 4, s);
    if (loss_grad(u, dt, t2, s) != cudaSuccess) return HC_ERR_CUDA;
    if (backward(u, s) != cudaSuccess) return HC_ERR_CUDA;
    rc = read_err(u, s);
    if (rc) return rc;
    std::vector<float> g(NFULL);
    cudaMemcpyAsync(g.data(), u->pg, (size_t)NFULL * 4, cudaMemcpyDeviceToHost, s);
    if (out) cudaMemcpyAsync(out, u->out0, n0 * 4, cudaMemcpyDeviceToHost, s);
    if (loss) cudaMemcpyAsync(loss, u->scal + 2, sizeof(double), cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return HC_ERR_CUDA;
    if (grad) full_to_compact(g, grad);
    return HC_OK;
}

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
