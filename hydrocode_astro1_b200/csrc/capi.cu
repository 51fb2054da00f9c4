// capi.cu -- the C ABI (include/hydrocode_b200.h): device context, the step
// and Poisson-solve orchestration on one CUDA stream.
//
// Memory: one context owns its buffers (cudaMalloc at create, freed at
// destroy).  State lives in structure-of-arrays form, double-buffered so a
// step reads step-n values and writes step n+1 (the reference achieves the
// same with its separate flux arrays).  The host is crossed only for the
// per-step dt, the SOR stop flag every few dozen iterations, and explicit
// state/potential transfers.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "hc_internal.cuh"
#include "unet_guard.h"

#ifndef HC_CYCLE_REDUCTION
#define HC_CYCLE_REDUCTION 1.0e-4   // residual reduction a correction cycle's sweeps aim for
#endif
#ifndef HC_LAST_CYCLE_TARGET
#define HC_LAST_CYCLE_TARGET 0.95   // the last cycle's sweeps stop below this fraction of tol
#endif

using namespace hc;

// ---------------------------------------------------------------- errors
static thread_local char g_err[512] = "";

static int set_err(int code, const char *fmt, ...) __attribute__((format(printf, 2, 3)));
static int set_err(int code, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
    return code;
}

#define CK(call)                                                                         \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess) {                                                         \
            (void)cudaGetLastError(); /* a non-sticky error must not fail later calls */  \
            return set_err(HC_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call,        \
                           cudaGetErrorString(e_));                                      \
        }                                                                                \
    } while (0)

extern "C" const char *hc_last_error(void) { return g_err; }

extern "C" int hc_device_count(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    return n;
}

// ---------------------------------------------------------------- context
struct EvPair {
    cudaEvent_t a, b;
    int fam;
};

enum { FAM_HYDRO = 0, FAM_BC, FAM_SOR, FAM_RES, FAM_MOM, FAM_UNET, FAM_N };

struct hc_ctx {
    hc_config cfg;
    Geom g;
    int dev;
    cudaStream_t s;
    int gravity;                 // self-gravity enabled
    // state
    double *q64[2][5];
    float *q32[2][5];
    int cur;
    int parity;
    int cfl_valid;
    // gravity
    double *phi, *phig, *rho_ext, *phi2;
    double *phs, *rhs;           // colour-split potential and density (FP64 solve)
    double *plm;                 // MUSCL-Hancock face-state buffer (20 values per cell; recon = 1)
    float *e32, *r32, *e32b;     // mixed precision correction (ping-pong) / residual
    double *gx, *gy, *gz;
    double *res;
    int res_cap;
    double *scratch;
    long long scratch_len;
    double *mom;
    // scalars
    DevScalars *sc;
    DevScalars *hsc;             // pinned mirror
    double *stage;               // AoS staging buffer on the device
    double *hdt;                 // pinned dt ring
    int hdt_cap;
    double *hslots;              // pinned copy of recent SOR update norms
    // diagnostics + timing
    hc_diag diag;
    double fam_ms[FAM_N];
    long long launches, hydro_launches, sor_launches;
    std::vector<EvPair> pend;
    std::vector<cudaEvent_t> evpool;
    // learned warm start
    UNetState *unet;
    // user timer
    cudaEvent_t t0, t1;
    int timer_on;
    int debug;                   // HC_DEBUG=1: per-solve progress on stderr
    int unet_passes;             // learned-start predictions per solve (>= 1)
    int unet_cycles;             // correction cycles that start from a prediction (0: 2)
    int unet_record_cycle;       // the cycle whose residual is recorded for training (0: 1; -1: none)
    double corr_omega;           // relaxation of the FP32 correction sweeps (0: the solve's omega)
    UnetGuard guard;             // learned-start outcome monitor (hc_set_unet_guard)
    double *cons_part;           // conservation sums: 5 * CONS_BLOCKS block partials
    int cons_record;             // 1: sums after every step, reported in hc_diag.cons
    // a slab of a grid split along x (hc_set_slab): the Poisson solve runs
    // across the slabs through the hc_slab_* entry points, not in hc_step
    int slab;
    double *slab_buf;            // moment sums / per-plane partials of the slab protocol
    long long slab_buf_len;
    // checkpoints: device packing buffer, copy stream, writer thread
    unsigned char *ck_dev;
    size_t ck_dev_bytes;
    unsigned char *ck_host[2];   // pinned chunks
    cudaStream_t ck_stream;
    cudaEvent_t ck_ev[3];
    std::thread *ck_thread;
    int ck_status;
    char ck_err[256];
};

static cudaEvent_t ev_get(hc_ctx *c)
{
    if (!c->evpool.empty()) {
        cudaEvent_t e = c->evpool.back();
        c->evpool.pop_back();
        return e;
    }
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    return e;
}

struct FamTimer {
    hc_ctx *c;
    EvPair p;
    FamTimer(hc_ctx *c_, int fam) : c(c_)
    {
        p.a = ev_get(c);
        p.b = ev_get(c);
        p.fam = fam;
        if (p.a) cudaEventRecord(p.a, c->s);
    }
    ~FamTimer()
    {
        if (p.b) cudaEventRecord(p.b, c->s);
        if (p.a && p.b) c->pend.push_back(p);
    }
};

static void resolve_timers(hc_ctx *c)
{
    for (auto &p : c->pend) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) c->fam_ms[p.fam] += ms;
        c->evpool.push_back(p.a);
        c->evpool.push_back(p.b);
    }
    c->pend.clear();
}

// Waits for the context's stream and reports the sticky device error code
// (set by a kernel whose bounded wait ran out), clearing it.
static int sync_ctx(hc_ctx *c)
{
    CK(cudaMemcpyAsync(&c->hsc->err, &c->sc->err, sizeof(int), cudaMemcpyDeviceToHost, c->s));
    CK(cudaStreamSynchronize(c->s));
    resolve_timers(c);
    if (c->hsc->err) {
        const int e = c->hsc->err;
        c->hsc->err = 0;
        CK(cudaMemsetAsync(&c->sc->err, 0, sizeof(int), c->s));
        return set_err(e, "a bounded wait in a device kernel gave up");
    }
    return HC_OK;
}

extern "C" void hc_config_default(hc_config *cfg)
{
    memset(cfg, 0, sizeof *cfg);
    cfg->nx = cfg->ny = cfg->nz = 64;
    cfg->xmin = cfg->ymin = cfg->zmin = 0.0;
    cfg->xmax = cfg->ymax = cfg->zmax = 1.0;
    cfg->gamma = 5.0 / 3.0;   // hydro_solver_3d.c:61
    cfg->cfl = 0.4;           // hydro_solver_3d.c:59
    cfg->G = 0.0;
    for (int t = 0; t < 6; t++) cfg->bc[t] = 2;
    cfg->precision = HC_FP64;
    cfg->moment_order = HC_MOMENTS_SEQUENTIAL;
    cfg->grav_bc = 1;          // ISOLATED, hydro_solver_3d.c:78
    cfg->lmax = 0;
    cfg->omega = 1.5;          // gravity_solver_3d.c:78-80
    cfg->max_iter = 10000;
    cfg->tol = 1.0e-6;
    cfg->sor_depth = 0;
    cfg->warm_start = HC_WARM_PREVIOUS;
    cfg->device = 0;
}

static void free_ctx(hc_ctx *c)
{
    if (!c) return;
    if (c->dev >= 0) cudaSetDevice(c->dev);
    for (int b = 0; b < 2; b++)
        for (int v = 0; v < 5; v++) {
            if (c->q64[b][v] && v == 0) cudaFree(c->q64[b][0]);
            if (c->q32[b][v] && v == 0) cudaFree(c->q32[b][0]);
        }
    cudaFree(c->phi); cudaFree(c->phig); cudaFree(c->rho_ext); cudaFree(c->phi2);
    cudaFree(c->phs); cudaFree(c->rhs); cudaFree(c->plm); cudaFree(c->slab_buf);
    cudaFree(c->e32); cudaFree(c->r32); cudaFree(c->e32b);
    cudaFree(c->gx); cudaFree(c->gy); cudaFree(c->gz);
    cudaFree(c->res); cudaFree(c->scratch); cudaFree(c->mom); cudaFree(c->cons_part);
    cudaFree(c->sc); cudaFree(c->stage);
    if (c->hsc) cudaFreeHost(c->hsc);
    if (c->hdt) cudaFreeHost(c->hdt);
    if (c->hslots) cudaFreeHost(c->hslots);
    resolve_timers(c);
    for (auto e : c->evpool) cudaEventDestroy(e);
    if (c->t0) cudaEventDestroy(c->t0);
    if (c->t1) cudaEventDestroy(c->t1);
    if (c->ck_thread) {
        c->ck_thread->join();
        delete c->ck_thread;
    }
    cudaFree(c->ck_dev);
    for (int b = 0; b < 2; b++)
        if (c->ck_host[b]) cudaFreeHost(c->ck_host[b]);
    for (int e = 0; e < 3; e++)
        if (c->ck_ev[e]) cudaEventDestroy(c->ck_ev[e]);
    if (c->ck_stream) cudaStreamDestroy(c->ck_stream);
    if (c->s) cudaStreamDestroy(c->s);
    unet_destroy(c->unet);
    delete c;
}

static int dmalloc(void **p, size_t bytes)
{
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        *p = nullptr;
        return set_err(HC_ERR_NOMEM, "cudaMalloc(%zu bytes) failed: %s", bytes, cudaGetErrorString(e));
    }
    return HC_OK;
}

static int ensure_res(hc_ctx *c, int max_iter)
{
    int need = std::max(max_iter, 1) + 16;   // slack for blocked passes
    if (c->res && c->res_cap >= need) return HC_OK;
    cudaFree(c->res);
    c->res = nullptr;
    int cap = std::max(need, 1024);
    int rc = dmalloc((void **)&c->res, sizeof(double) * cap);
    if (rc) return rc;
    c->res_cap = cap;
    return HC_OK;
}

extern "C" hc_ctx *hc_create(const hc_config *cfg)
{
    if (!cfg) { set_err(HC_ERR_ARG, "null config"); return nullptr; }
    const hc_config &k = *cfg;
    if (k.nx < 3 || k.ny < 3 || (k.nz < 3 && !(k.gravity_only && k.nz == 1))) {
        set_err(HC_ERR_ARG, "grid %dx%dx%d: every dimension needs at least 3 cells "
                "(nz == 1 only for a gravity-only context)", k.nx, k.ny, k.nz);
        return nullptr;
    }
    if (k.gravity_only && !(k.G > 0.0)) {
        set_err(HC_ERR_ARG, "gravity-only context needs G > 0");
        return nullptr;
    }
    if (k.precision != HC_FP64 && k.precision != HC_FP32) {
        set_err(HC_ERR_ARG, "unknown precision %d", k.precision);
        return nullptr;
    }
    if (k.lmax < 0 || k.lmax > 12) {
        set_err(HC_ERR_ARG, "lmax %d outside 0..12", k.lmax);
        return nullptr;
    }
    if (k.recon != 0 && k.recon != 1) {
        set_err(HC_ERR_ARG, "unknown reconstruction %d (0 piecewise constant, 1 MUSCL-Hancock)", k.recon);
        return nullptr;
    }
    if (k.recon == 1 && k.precision != HC_FP64) {
        set_err(HC_ERR_ARG, "MUSCL-Hancock reconstruction runs in HC_FP64 only");
        return nullptr;
    }
    if (!(k.xmax > k.xmin) || !(k.ymax > k.ymin) || !(k.zmax > k.zmin)) {
        set_err(HC_ERR_ARG, "empty domain");
        return nullptr;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        set_err(HC_ERR_CUDA, "no CUDA device available");
        return nullptr;
    }
    if (k.device < 0 || k.device >= ndev) {
        set_err(HC_ERR_ARG, "device %d not present (%d devices)", k.device, ndev);
        return nullptr;
    }
    const char *fail = getenv("HC_FAIL_ALLOC");   // host-side fault injection for tests
    if (fail && atoi(fail) != 0) {
        set_err(HC_ERR_NOMEM, "allocation failure injected by HC_FAIL_ALLOC");
        return nullptr;
    }
    hc_ctx *c = new hc_ctx();
    memset(c->q64, 0, sizeof c->q64);
    memset(c->q32, 0, sizeof c->q32);
    c->cfg = k;
    c->dev = k.device;
    if (cudaSetDevice(c->dev) != cudaSuccess) { set_err(HC_ERR_CUDA, "cudaSetDevice"); delete c; return nullptr; }
    Geom &g = c->g;
    g.nx = k.nx; g.ny = k.ny; g.nz = k.nz;
    g.n = (long long)k.nx * k.ny * k.nz;
    g.xmin = k.xmin; g.xmax = k.xmax; g.ymin = k.ymin; g.ymax = k.ymax; g.zmin = k.zmin; g.zmax = k.zmax;
    g.dx = k.dx > 0.0 ? k.dx : (k.xmax - k.xmin) / k.nx;
    g.dy = k.dy > 0.0 ? k.dy : (k.ymax - k.ymin) / k.ny;
    g.dz = k.dz > 0.0 ? k.dz : (k.zmax - k.zmin) / k.nz;
    g.ioff = 0; g.gnx = k.nx; g.olo = 0; g.ohi = k.nx;
    c->gravity = k.G > 0.0;
    const size_t n = (size_t)g.n;
    int rc = HC_OK;
    if (cudaStreamCreateWithFlags(&c->s, cudaStreamNonBlocking) != cudaSuccess) {
        set_err(HC_ERR_CUDA, "stream create");
        free_ctx(c);
        return nullptr;
    }
    for (int b = 0; b < 2 && !rc && !k.gravity_only; b++) {
        if (k.precision == HC_FP64) {
            double *base = nullptr;
            rc = dmalloc((void **)&base, 5 * n * sizeof(double));
            for (int v = 0; v < 5 && !rc; v++) c->q64[b][v] = base + v * n;
        } else {
            float *base = nullptr;
            rc = dmalloc((void **)&base, 5 * n * sizeof(float));
            for (int v = 0; v < 5 && !rc; v++) c->q32[b][v] = base + v * n;
        }
    }
    if (!rc) rc = dmalloc((void **)&c->sc, sizeof(DevScalars));
    if (!rc && c->gravity) {
        rc = dmalloc((void **)&c->phi, n * sizeof(double));
        if (!rc) rc = dmalloc((void **)&c->phig, n * sizeof(double));
        if (!rc) rc = ensure_res(c, k.max_iter);
        // tree partials (592x9), lmax partials (<= 387x169), then the lmax
        // z-power sums (13 per (i, j) row)
        c->scratch_len = grav_scratch_len(c->g);
        if (!rc) rc = dmalloc((void **)&c->scratch, c->scratch_len * sizeof(double));
        if (!rc) rc = dmalloc((void **)&c->mom, 4 * 1024 * sizeof(double));
        if (!rc && k.precision == HC_FP32) {
            // sized for the colour-split layout (>= n cells)
            const size_t ns = (size_t)std::max<long long>(split_len(c->g), (long long)n);
            rc = dmalloc((void **)&c->e32, ns * sizeof(float));
            if (!rc) rc = dmalloc((void **)&c->r32, ns * sizeof(float));
            if (!rc) rc = dmalloc((void **)&c->e32b, ns * sizeof(float));
        }
    }
    if (!rc && cudaMallocHost((void **)&c->hsc, sizeof(DevScalars)) != cudaSuccess)
        rc = set_err(HC_ERR_NOMEM, "pinned scalars");
    if (rc) { free_ctx(c); return nullptr; }
    // zero state and potential (calloc in the reference, gravity_solver_3d.c:87)
    cudaMemsetAsync(c->sc, 0, sizeof(DevScalars), c->s);
    for (int b = 0; b < 2; b++) {
        if (c->q64[b][0]) cudaMemsetAsync(c->q64[b][0], 0, 5 * n * sizeof(double), c->s);
        if (c->q32[b][0]) cudaMemsetAsync(c->q32[b][0], 0, 5 * n * sizeof(float), c->s);
    }
    if (c->e32b) {
        const size_t ns = (size_t)std::max<long long>(split_len(c->g), (long long)n);
        cudaMemsetAsync(c->e32, 0, ns * sizeof(float), c->s);
        cudaMemsetAsync(c->e32b, 0, ns * sizeof(float), c->s);
    }
    if (c->phi) {
        cudaMemsetAsync(c->phi, 0, n * sizeof(double), c->s);
        cudaMemsetAsync(c->phig, 0, n * sizeof(double), c->s);
    }
    if (cudaStreamSynchronize(c->s) != cudaSuccess) {
        set_err(HC_ERR_CUDA, "init memset");
        free_ctx(c);
        return nullptr;
    }
    c->cur = 0;
    c->parity = 0;
    c->cfl_valid = 0;
    const char *dbg = getenv("HC_DEBUG");
    c->debug = dbg && atoi(dbg) != 0;
    return c;
}

extern "C" void hc_destroy(hc_ctx *c) { free_ctx(c); }

extern "C" size_t hc_ncells(const hc_ctx *c) { return c ? (size_t)c->g.n : 0; }

// ---------------------------------------------------------------- state I/O
static int ensure_stage(hc_ctx *c)
{
    if (c->stage) return HC_OK;
    return dmalloc((void **)&c->stage, 5 * (size_t)c->g.n * sizeof(double));
}

static int upload_soa64(hc_ctx *c, const double *q)
{
    const size_t n = (size_t)c->g.n;
    if (c->cfg.precision == HC_FP64) {
        for (int v = 0; v < 5; v++)
            CK(cudaMemcpyAsync(c->q64[c->cur][v], q + v * n, n * sizeof(double), cudaMemcpyHostToDevice, c->s));
    } else {
        int rc = ensure_stage(c);
        if (rc) return rc;
        CK(cudaMemcpyAsync(c->stage, q, 5 * n * sizeof(double), cudaMemcpyHostToDevice, c->s));
        double *src[5];
        for (int v = 0; v < 5; v++) src[v] = c->stage + v * n;
        CK(fp32_from_fp64(src, c->q32[c->cur], c->g.n, c->s));
    }
    c->cfl_valid = 0;
    return HC_OK;
}

extern "C" int hc_set_state(hc_ctx *c, const double *U)
{
    if (c && c->cfg.gravity_only) return set_err(HC_ERR_STATE, "gravity-only context has no hydro state");
    if (!c || !U) return set_err(HC_ERR_ARG, "null argument");
    CK(cudaSetDevice(c->dev));
    int rc = ensure_stage(c);
    if (rc) return rc;
    const size_t n = (size_t)c->g.n;
    CK(cudaMemcpyAsync(c->stage, U, 5 * n * sizeof(double), cudaMemcpyHostToDevice, c->s));
    if (c->cfg.precision == HC_FP64) CK(fp64_aos_to_soa(c->stage, c->q64[c->cur], c->g.n, c->s));
    else CK(fp32_from_aos64(c->stage, c->q32[c->cur], c->g.n, c->s));
    c->cfl_valid = 0;
    c->launches += 1;
    return sync_ctx(c);
}

extern "C" int hc_get_state(hc_ctx *c, double *U)
{
    if (c && c->cfg.gravity_only) return set_err(HC_ERR_STATE, "gravity-only context has no hydro state");
    if (!c || !U) return set_err(HC_ERR_ARG, "null argument");
    CK(cudaSetDevice(c->dev));
    int rc = ensure_stage(c);
    if (rc) return rc;
    const size_t n = (size_t)c->g.n;
    if (c->cfg.precision == HC_FP64) CK(fp64_soa_to_aos(c->q64[c->cur], c->stage, c->g.n, c->s));
    else CK(fp32_to_aos64(c->q32[c->cur], c->stage, c->g.n, c->s));
    CK(cudaMemcpyAsync(U, c->stage, 5 * n * sizeof(double), cudaMemcpyDeviceToHost, c->s));
    return sync_ctx(c);
}

extern "C" int hc_set_state_soa(hc_ctx *c, const double *q)
{
    if (c && c->cfg.gravity_only) return set_err(HC_ERR_STATE, "gravity-only context has no hydro state");
    if (!c || !q) return set_err(HC_ERR_ARG, "null argument");
    CK(cudaSetDevice(c->dev));
    int rc = upload_soa64(c, q);
    if (rc) return rc;
    return sync_ctx(c);
}

extern "C" int hc_get_state_soa(hc_ctx *c, double *q)
{
    if (c && c->cfg.gravity_only) return set_err(HC_ERR_STATE, "gravity-only context has no hydro state");
    if (!c || !q) return set_err(HC_ERR_ARG, "null argument");
    CK(cudaSetDevice(c->dev));
    const size_t n = (size_t)c->g.n;
    if (c->cfg.precision == HC_FP64) {
        for (int v = 0; v < 5; v++)
            CK(cudaMemcpyAsync(q + v * n, c->q64[c->cur][v], n * sizeof(double), cudaMemcpyDeviceToHost, c->s));
    } else {
        int rc = ensure_stage(c);
        if (rc) return rc;
        double *dst[5];
        for (int v = 0; v < 5; v++) dst[v] = c->stage + v * n;
        CK(fp32_to_fp64(c->q32[c->cur], dst, c->g.n, c->s));
        CK(cudaMemcpyAsync(q, c->stage, 5 * n * sizeof(double), cudaMemcpyDeviceToHost, c->s));
    }
    return sync_ctx(c);
}

// ---------------------------------------------------------------- gravity
static GravArgs grav_args(hc_ctx *c, const double *rho, const float *rho32)
{
    GravArgs a;
    memset(&a, 0, sizeof a);
    a.g = c->g;
    a.G = c->cfg.G;
    a.omega = c->cfg.omega;
    a.tol = c->cfg.tol;
    a.max_iter = c->cfg.max_iter;
    a.sweep_kind = c->cfg.sor_depth == -3 ? 1 : 0;   // 1: TMA-staged FP32 correction sweeps
    a.grav_bc = c->cfg.grav_bc;
    a.lmax = c->cfg.lmax;
    a.moment_order = c->cfg.moment_order;
    a.phi = c->phi;
    a.rho = rho;
    a.rho32 = rho32;
    a.res = c->res;
    a.sc = c->sc;
    a.scratch = c->scratch;
    a.scratch_len = c->scratch_len;
    a.mom = c->mom;
    a.gx = c->gx; a.gy = c->gy; a.gz = c->gz;
    return a;
}

// Multipole moments + boundary values of the current density.
static int grav_boundary_values(hc_ctx *c, const GravArgs &a)
{
    if (a.grav_bc == 0) {
        CK(grav_boundary_periodic(a, c->s));
        c->launches += 3;
        return HC_OK;
    }
    if (a.grav_bc != 1) return HC_OK;   // DIRICHLET keeps the current values
    FamTimer t(c, FAM_MOM);
    if (a.lmax == 0) {
        CK(grav_boundary_ref(a, c->s));
        c->launches += 1;
    } else {
        CK(grav_boundary_lmax(a, c->s));
        c->launches += 1;
    }
    return HC_OK;
}

static int grav_moments(hc_ctx *c, const GravArgs &a)
{
    if (a.grav_bc != 1) return HC_OK;
    FamTimer t(c, FAM_MOM);
    if (a.lmax == 0) {
        if (a.moment_order == HC_MOMENTS_SEQUENTIAL && a.rho) {
            CK(grav_moments_sequential(a, c->s));
            c->launches += 1;
        } else {
            CK(grav_moments_tree(a, c->s));
            c->launches += 4;
        }
    } else {
        CK(grav_moments_lmax(a, c->s));
        c->launches += 4;
    }
    return HC_OK;
}

// Iterations to queue before the next host poll of an SOR solve: from the
// update norms of the last polled iterations (slots[0..nb)), the geometric
// rate r over up to 32 iterations predicts the iterations left to reach
// thresh; queue 10% more plus two, between 8 and 512.  Without a usable
// rate, double the previous batch (at most 256).  Queued sweeps past the stop
// only cost early-exit launches, so the prediction trades those against polls.
static int next_batch(const double *slots, int nb, double thresh, int prev)
{
    int w = std::min(32, nb - 1);
    while (w >= 4 && !(slots[nb - 1 - w] > 0.0)) w /= 2;
    const double last = slots[nb - 1];
    if (w >= 4 && last > 0.0 && slots[nb - 1 - w] > last) {
        const double rate = std::pow(last / slots[nb - 1 - w], 1.0 / w);
        if (rate > 0.0 && rate < 0.9999) {
            const double rem = std::log(thresh / last) / std::log(rate);
            if (rem <= 0.0) return 8;
            return (int)std::min(512.0, std::max(8.0, 1.1 * rem + 2.0));
        }
    }
    return std::min(prev * 2, 256);
}

// Red-black SOR to tolerance, FP64 (gravity_solve_potential,
// gravity_solver_3d.c:510-747).  Returns 0 / -1 like the reference, or a
// negative HC_ERR_* code.
static int sor_fp64(hc_ctx *c, const double *rho)
{
    GravArgs a = grav_args(c, rho, nullptr);
    int rc = ensure_res(c, a.max_iter);
    if (rc) return rc;
    a.res = c->res;
    CK(cudaMemsetAsync(&c->sc->done, 0, 2 * sizeof(int), c->s));    // done, last_iter
    CK(grav_reset_slots(a, 0, std::max(a.max_iter, 1), c->s));
    rc = grav_moments(c, a);
    if (rc) return rc;
    if (a.max_iter <= 0) {
        c->diag.last_iterations = 0;
        c->diag.last_residual = 0.0;
        return -1;
    }
    // sor_depth 0 (default): colour-split sweeps, in place on a split copy of
    // phi and rho; -1: one kernel per colour on the natural layout, in place
    // (the reference's sweeps); >= 1: one wavefront pass per iteration, out of
    // place between phi (buf 0) and phi2 (buf 1): iteration t reads buf[t%2],
    // writes buf[(t+1)%2].  All three give the same iterates.
    const bool split = c->cfg.sor_depth == 0 && c->g.nz >= 3;
    const bool wave = c->cfg.sor_depth >= 1 && c->g.nz >= 3;
    double *buf[2] = { c->phi, c->phi2 };
    if (split) {
        const size_t ns = (size_t)split_len(c->g);
        if (!c->phs) rc = dmalloc((void **)&c->phs, ns * sizeof(double));
        if (!rc && !c->rhs) rc = dmalloc((void **)&c->rhs, ns * sizeof(double));
        if (rc) return rc;
        CK(grav_split_fields(a, c->phs, c->rhs, c->s));
        c->launches += 2;
    }
    if (wave) {
        if (!c->phi2) {
            rc = dmalloc((void **)&c->phi2, (size_t)c->g.n * sizeof(double));
            if (rc) return rc;
            buf[1] = c->phi2;
        }
        // both buffers carry the current boundary cells
        CK(cudaMemcpyAsync(c->phi2, c->phi, (size_t)c->g.n * sizeof(double), cudaMemcpyDeviceToDevice, c->s));
    }
    auto one_iter = [&](int q) -> int {
        if (split) {
            CK(grav_sor_split(a, c->phs, c->rhs, 0, q, c->s));
            CK(grav_sor_split(a, c->phs, c->rhs, 1, q, c->s));
            c->launches += 2;
            c->sor_launches += 2;
        } else if (wave) {
            CK(grav_sor_pass64(a, buf[q & 1], buf[(q + 1) & 1], q, c->s));
            c->launches += 1;
            c->sor_launches += 1;
        } else {
            CK(grav_sor_color(a, 0, q, c->s));
            CK(grav_sor_color(a, 1, q, c->s));
            c->launches += 2;
            c->sor_launches += 2;
        }
        return HC_OK;
    };
    {
        FamTimer t(c, FAM_SOR);
        rc = one_iter(0);
        if (rc) return rc;
    }
    // the first iteration swept with the previous boundary; now the new one
    if (wave) {
        GravArgs b = a;
        b.phi = buf[1];
        rc = grav_boundary_values(c, b);
        if (rc) return rc;
    }
    rc = grav_boundary_values(c, a);
    if (rc) return rc;
    if (split) {
        CK(grav_split_boundary(a, c->phs, c->s));
        c->launches += 1;
    }
    int it = 1, done = 0, last = 0;
    int batch = 16;
    while (true) {
        int end = std::min(a.max_iter, it + batch);
        {
            FamTimer t(c, FAM_SOR);
            for (int q = it; q < end; q++) {
                rc = one_iter(q);
                if (rc) return rc;
            }
            CK(grav_check(a, end, c->s));
        }
        c->launches += 1;
        CK(cudaMemcpyAsync(&c->hsc->done, &c->sc->done, 2 * sizeof(int), cudaMemcpyDeviceToHost, c->s));
        const int nb = std::min(end - it, 512);
        if (!c->hslots && cudaMallocHost((void **)&c->hslots, 512 * sizeof(double)) != cudaSuccess)
            return set_err(HC_ERR_NOMEM, "pinned slot buffer");
        CK(cudaMemcpyAsync(c->hslots, c->res + (end - nb), nb * sizeof(double), cudaMemcpyDeviceToHost, c->s));
        rc = sync_ctx(c);
        if (rc) return rc;
        done = c->hsc->done;
        last = c->hsc->last_iter;
        if (done || end >= a.max_iter) break;
        it = end;
        batch = next_batch(c->hslots, nb, a.tol, batch);
    }
    int used = done ? last : a.max_iter;
    if (wave && (used & 1)) std::swap(c->phi, c->phi2);   // result in buf[used % 2]
    if (split) {
        CK(grav_unsplit(a, c->phs, c->s));
        c->launches += 1;
    }
    double rv = 0.0;
    CK(cudaMemcpy(&rv, c->res + (used - 1), sizeof(double), cudaMemcpyDeviceToHost));
    c->diag.last_iterations = used;
    c->diag.last_residual = rv;
    c->diag.total_iterations += used;
    return done ? 0 : -1;
}

static bool guard_allows_prediction(hc_ctx *c) { return unet_guard_allows(c->guard); }
static void guard_record(hc_ctx *c, bool predicted, int iters) { unet_guard_record(c->guard, predicted, iters); }

// Mixed-precision Poisson solve: FP64 residual of the full potential, FP32
// red-black SOR on the correction, FP64 update; repeated until the FP64
// update norm max|delta| is below tol.  Iteration budget: max_iter inner
// sweeps in total.
int hc_sor_mixed(hc_ctx *c, const float *rho32)
{
    GravArgs a = grav_args(c, nullptr, rho32);
    // only the correction sweeps relax (the FP64 residual and update do not),
    // so a.omega here is theirs; the stopping test max|phi_GS - phi_old| < tol
    // does not depend on it
    if (c->corr_omega > 0.0) a.omega = c->corr_omega;
    // sor_depth 0 (default): colour-split sweeps on e and r (-3: the FP32
    // correction sweeps staged by TMA where the layout allows); -2: colour-split,
    // two iterations per HBM pass (temporal blocking, out of place between
    // e32 and e32b; colour-split sweeps where the tiling does not fit); -1:
    // one in-place kernel per colour on the natural layout; >= 1: wavefront
    // passes of that many FP32 iterations per HBM pass on the natural layout
    const bool split = (c->cfg.sor_depth == 0 || c->cfg.sor_depth == -2 || c->cfg.sor_depth == -3) && c->g.nz >= 3;
    const bool wave2 = split && c->cfg.sor_depth == -2 && mixed_wave_split_ok(c->g);
    const int depth = wave2 ? 2 : (split ? -1 : c->cfg.sor_depth);
    int rc = ensure_res(c, a.max_iter);
    if (rc) return rc;
    a.res = c->res;
    rc = grav_moments(c, a);
    if (rc) return rc;
    rc = grav_boundary_values(c, a);
    if (rc) return rc;
    int total = 0, cycles = 0, status = -1;
    double dmax = 0.0;
    // FP64 residual delta of phi into r32 (e32 zeroed); returns max|delta|
    auto residual = [&](double *out) -> int {
        {
            FamTimer t(c, FAM_RES);
            CK(cudaMemsetAsync(&c->sc->resnorm, 0, sizeof(double), c->s));
            CK(mixed_residual(a, c->r32, c->e32, split, c->s));
            c->launches++;
        }
        CK(cudaMemcpyAsync(&c->hsc->resnorm, &c->sc->resnorm, sizeof(double), cudaMemcpyDeviceToHost, c->s));
        int r = sync_ctx(c);
        if (r) return r;
        *out = c->hsc->resnorm;
        return HC_OK;
    };
    c->diag.warm_start_used = 0;
    bool recorded = false;
    const bool guard_ok = c->cfg.warm_start == HC_WARM_UNET ? guard_allows_prediction(c) : true;
    while (true) {
        const double prev_dmax = cycles ? dmax : 1e300;
        rc = residual(&dmax);
        if (rc) return rc;
        cycles++;
        // Learned warm start (the first unet_cycles correction cycles,
        // colour-split layout): the network predicts the correction from this
        // residual; phi + e0 is kept only if its FP64 residual is smaller, else
        // phi is restored.  The first cycle's residual is the step's (rough,
        // after the hydro update); the second's is what the first cycle's
        // sweeps left (smooth), where the prediction removes the slow modes
        // that the remaining sweeps would spend most of their iterations on.
        // With sample collection on, the residual and phi at the start of
        // cycle unet_record_cycle are recorded for training.
        const int ucycles = c->unet_cycles > 0 ? c->unet_cycles : 2;
        const int rcycle = c->unet_record_cycle > 0 ? c->unet_record_cycle : (c->unet_record_cycle < 0 ? 0 : 1);
        if ((cycles <= ucycles || cycles == rcycle) && split && c->unet && std::isfinite(dmax)) {
            const bool predict = cycles <= ucycles && c->cfg.warm_start == HC_WARM_UNET && guard_ok &&
                                 unet_has_weights(c->unet);
            const bool rec = cycles == rcycle && unet_collecting(c->unet);
            if (predict || rec) {
                {
                    FamTimer t(c, FAM_UNET);
                    rc = unet_begin_solve(c->unet, a, c->r32, predict ? c->e32b : nullptr, rec, c->s);
                    c->launches += predict ? 40 : 3;
                }
                if (rc) return set_err(rc, "learned warm start: grid dimensions must be multiples of 32");
                if (rec) recorded = true;
            }
            // passes after the first predict from the residual the previous
            // accepted pass left, until one is rejected
            for (int pass = 0; predict && pass < std::max(1, c->unet_passes); pass++) {
                if (pass > 0) {
                    FamTimer t(c, FAM_UNET);
                    rc = unet_begin_solve(c->unet, a, c->r32, c->e32b, false, c->s);
                    if (rc) return set_err(rc, "learned warm start failed");
                    c->launches += 40;
                }
                CK(mixed_update(a, c->e32b, split, 1.0f, c->s));
                double d1 = 0.0;
                rc = residual(&d1);
                if (rc) return rc;
                c->launches += 2;
                if (c->debug) fprintf(stderr, "[hc] learned start %d: max|delta| %.3e -> %.3e\n", pass, dmax, d1);
                if (std::isfinite(d1) && d1 < dmax) {
                    dmax = d1;
                    if (pass == 0 && cycles == 1) {
                        c->diag.warm_start_used = 1;
                        c->diag.unet_accepted++;
                    }
                    continue;
                }
                CK(mixed_update(a, c->e32b, split, -1.0f, c->s));
                rc = residual(&dmax);
                if (rc) return rc;
                c->launches += 2;
                if (pass == 0 && cycles == 1) c->diag.unet_fallbacks++;
                break;
            }
        }
        if (c->debug) fprintf(stderr, "[hc] mixed cycle %d: max|delta| %.3e after %d sweeps\n", cycles, dmax, total);
        if (!std::isfinite(dmax)) return set_err(HC_ERR_NUMERIC, "non-finite Poisson residual");
        if (dmax < a.tol) { status = 0; break; }
        if (total >= a.max_iter) break;
        // a correction cycle that does not halve the residual means the FP32
        // sweeps cannot resolve it: report non-convergence instead of looping
        if (dmax > 0.5 * prev_dmax) {
            if (c->debug) fprintf(stderr, "[hc] mixed solve stalled at %.3e\n", dmax);
            break;
        }
        // one cycle reduces the residual 1e4-fold at most: FP32 resolves the
        // correction e to ~1e-7 |e|, and |e| can exceed max|delta| by the
        // grid's condition number on a cold start.  In the last cycle the
        // sweeps run to the reference's own test -- a red-black sweep whose
        // update norm max |phi_GS - phi_old| is below tol -- with a margin
        // for the FP32 rounding of that norm (checked below): to 0.95 tol.
        const double tol_last = a.tol * HC_LAST_CYCLE_TARGET;
        const double thresh = std::max(tol_last, HC_CYCLE_REDUCTION * dmax);
        const int budget = a.max_iter - total;
        CK(cudaMemsetAsync(&c->sc->done, 0, 2 * sizeof(int), c->s));
        CK(grav_reset_slots(a, 0, budget + 8, c->s));
        float *eb[2] = { c->e32, c->e32b };
        // the passes write every interior cell of their output; its boundary
        // cells (zero for the correction) come from here
        if (wave2) CK(cudaMemsetAsync(c->e32b, 0, (size_t)split_len(c->g) * sizeof(float), c->s));
        int it = 0, done = 0, last = 0, batch = 16, processed = 0, best_it = 0;
        double best = 1e300;
        if (!c->hslots && cudaMallocHost((void **)&c->hslots, 512 * sizeof(double)) != cudaSuccess)
            return set_err(HC_ERR_NOMEM, "pinned slot buffer");
        while (true) {
            int end = std::min(budget, it + batch);
            {
                FamTimer t(c, FAM_SOR);
                if (wave2) {
                    for (int q = it; q < end; q += 2) {
                        CK(mixed_sor32_split_pass(a, eb[(q / 2) & 1], eb[((q / 2) + 1) & 1], c->r32, q, thresh, c->s));
                        c->launches += 1;
                        c->sor_launches += 1;
                    }
                    end = it + ((end - it + 1) / 2) * 2;
                } else if (split) {
                    for (int q = it; q < end; q++) {
                        CK(mixed_sor32_split(a, c->e32, c->r32, 0, q, thresh, c->s));
                        CK(mixed_sor32_split(a, c->e32, c->r32, 1, q, thresh, c->s));
                    }
                    c->launches += 2 * (end - it);
                    c->sor_launches += 2 * (end - it);
                } else if (depth < 0) {
                    for (int q = it; q < end; q++) {
                        CK(mixed_sor32(a, c->e32, c->r32, 0, q, thresh, c->s));
                        CK(mixed_sor32(a, c->e32, c->r32, 1, q, thresh, c->s));
                    }
                    c->launches += 2 * (end - it);
                    c->sor_launches += 2 * (end - it);
                } else {
                    // passes start at multiples of depth; the last may overrun the
                    // budget by < depth iterations (slots are sized for it)
                    for (int q = it; q < end; q += depth) {
                        CK(mixed_sor32_pass(a, eb[(q / depth) & 1], eb[((q / depth) + 1) & 1], c->r32, q,
                                            depth, thresh, c->s));
                        c->launches += 1;
                        c->sor_launches += 1;
                    }
                    end = it + ((end - it + depth - 1) / depth) * depth;
                }
                CK(mixed_check(a, end, thresh, c->s));
                c->launches += 1;
            }
            processed = end;
            CK(cudaMemcpyAsync(&c->hsc->done, &c->sc->done, 2 * sizeof(int), cudaMemcpyDeviceToHost, c->s));
            const int nb = std::min(end - it, 512);
            CK(cudaMemcpyAsync(c->hslots, c->res + (end - nb), nb * sizeof(double), cudaMemcpyDeviceToHost, c->s));
            rc = sync_ctx(c);
            if (rc) return rc;
            done = c->hsc->done;
            last = c->hsc->last_iter;
            if (done || end >= budget) break;
            // stagnation guard: FP32 round-off floor reached before thresh
            for (int q = 0; q < nb; q++) {
                double v = c->hslots[q];
                if (v > 0.0 && v < 0.995 * best) { best = v; best_it = end - nb + q; }
            }
            if (end - best_it > 2048) {
                if (c->debug) fprintf(stderr, "[hc] inner sweeps stagnated at %.3e (thresh %.3e)\n", best, thresh);
                break;
            }
            it = end;
            batch = next_batch(c->hslots, nb, thresh, batch);
        }
        const int used = done ? last : processed;
        total += used;
        // the correction is in eb[passes % 2] for the blocked sweeps
        const float *efinal = ((split && !wave2) || depth < 0) ? c->e32 : eb[(used / depth) & 1];
        {
            FamTimer t(c, FAM_RES);
            CK(cudaMemsetAsync(&c->sc->resid_bits, 0, sizeof(unsigned long long), c->s));
            CK(mixed_update(a, efinal, split, 1.0f, c->s));
            c->launches++;
        }
        // Converged by the reference's criterion when the last sweep's update
        // norm (on e, which equals that of phi + e in exact arithmetic) is
        // below tol with room for its FP32 rounding -- the FP32 Gauss-Seidel
        // value of a cell sums its six neighbours' e (weights adding up to 1)
        // and delta, so it is off from the FP64 one by a few units in the
        // last place of max|e|; 4 ulp are allowed -- and FP32 resolves e
        // finely enough that an update of size tol cannot round away:
        // max|e| 2^-22 < tol.  Otherwise another correction cycle starts
        // from the FP64 residual of the updated potential.
        if (done && thresh == tol_last) {
            double snorm = 0.0;
            CK(cudaMemcpyAsync(&c->hsc->resnorm, c->res + (last - 1), sizeof(double), cudaMemcpyDeviceToHost,
                               c->s));
            CK(cudaMemcpyAsync(&c->hsc->resid_bits, &c->sc->resid_bits, sizeof(unsigned long long),
                               cudaMemcpyDeviceToHost, c->s));
            rc = sync_ctx(c);
            if (rc) return rc;
            snorm = c->hsc->resnorm;
            double emax;
            memcpy(&emax, &c->hsc->resid_bits, sizeof emax);
            if (c->debug)
                fprintf(stderr, "[hc] mixed cycle %d: sweep norm %.3e, max|e| %.3e after %d sweeps\n", cycles, snorm,
                        emax, total);
            if (snorm + 4.0 * emax * 0x1p-23 < a.tol && emax * 0x1p-22 < a.tol) {
                dmax = snorm;
                status = 0;
                break;
            }
        }
    }
    c->diag.last_iterations = total;
    c->diag.last_residual = dmax;
    c->diag.outer_cycles = cycles;
    c->diag.total_iterations += total;
    if (c->cfg.warm_start == HC_WARM_UNET && unet_has_weights(c->unet)) {
        guard_record(c, c->diag.warm_start_used != 0, total);
        const UnetGuard &g = c->guard;
        c->diag.unet_probes = g.probes;
        c->diag.unet_wins = g.wins;
        c->diag.unet_losses = g.loss_total;
        c->diag.unet_switch_offs = g.switch_offs;
        c->diag.unet_off = g.off;
    }
    if (recorded) {
        rc = unet_end_solve(c->unet, a, status == 0, c->s);
        if (rc) return set_err(rc, "learned warm start: recording a training sample failed");
    }
    return status;
}

static int gravity_solve_dev(hc_ctx *c, const double *rho64, const float *rho32)
{
    int st;
    if (c->cfg.precision == HC_FP64 || rho64) {
        st = sor_fp64(c, rho64);
    } else {
        st = hc_sor_mixed(c, rho32);
    }
    if (st < -1) return st;
    c->diag.last_status = st;
    if (st == 0) CK(cudaMemcpyAsync(c->phig, c->phi, (size_t)c->g.n * sizeof(double), cudaMemcpyDeviceToDevice, c->s));
    else
        fprintf(stderr, "Warning: Gravity solver did not converge in %d iterations.\n"
                        "         Final residual: %.3e (tolerance: %.3e)\n",
                c->diag.last_iterations, c->diag.last_residual, c->cfg.tol);
    return st;
}

extern "C" int hc_gravity_solve(hc_ctx *c, const double *rho, int with_accel)
{
    if (!c) return set_err(HC_ERR_ARG, "null context");
    if (!c->gravity) return set_err(HC_ERR_STATE, "gravity disabled (G <= 0)");
    if (c->slab) return set_err(HC_ERR_STATE, "a slab solves through the hc_slab_* entry points");
    CK(cudaSetDevice(c->dev));
    const size_t n = (size_t)c->g.n;
    int st;
    if (rho) {
        if (!c->rho_ext) {
            int rc = dmalloc((void **)&c->rho_ext, n * sizeof(double));
            if (rc) return rc;
        }
        CK(cudaMemcpyAsync(c->rho_ext, rho, n * sizeof(double), cudaMemcpyHostToDevice, c->s));
        st = gravity_solve_dev(c, c->rho_ext, nullptr);
    } else if (c->cfg.gravity_only) {
        return set_err(HC_ERR_ARG, "gravity-only context: pass a density");
    } else if (c->cfg.precision == HC_FP64) {
        st = gravity_solve_dev(c, c->q64[c->cur][0], nullptr);
    } else {
        st = gravity_solve_dev(c, nullptr, c->q32[c->cur][0]);
    }
    if (st < -1) return st;
    (void)with_accel;   // g is formed from the converged potential on demand
    int rc = sync_ctx(c);
    if (rc) return rc;
    return st == 0 ? HC_OK : HC_NOT_CONVERGED;
}

static int ensure_accel(hc_ctx *c)
{
    const size_t n = (size_t)c->g.n;
    int rc = HC_OK;
    if (!c->gx) rc = dmalloc((void **)&c->gx, n * sizeof(double));
    if (!rc && !c->gy) rc = dmalloc((void **)&c->gy, n * sizeof(double));
    if (!rc && !c->gz) rc = dmalloc((void **)&c->gz, n * sizeof(double));
    return rc;
}

extern "C" int hc_gravity_acceleration(hc_ctx *c)
{
    // gravity_compute_acceleration on the current potential: it becomes the
    // potential that the step's source term uses.
    if (!c || !c->gravity) return set_err(HC_ERR_STATE, "gravity disabled");
    CK(cudaSetDevice(c->dev));
    CK(cudaMemcpyAsync(c->phig, c->phi, (size_t)c->g.n * sizeof(double), cudaMemcpyDeviceToDevice, c->s));
    return sync_ctx(c);
}

extern "C" int hc_get_accel(hc_ctx *c, double *gx, double *gy, double *gz)
{
    if (!c || !gx || !gy || !gz) return set_err(HC_ERR_ARG, "null argument");
    if (!c->gravity) return set_err(HC_ERR_STATE, "gravity disabled");
    CK(cudaSetDevice(c->dev));
    int rc = ensure_accel(c);
    if (rc) return rc;
    GravArgs a = grav_args(c, nullptr, nullptr);
    a.phi = c->phig;
    CK(grav_accel(a, c->s));
    const size_t n = (size_t)c->g.n;
    CK(cudaMemcpyAsync(gx, c->gx, n * sizeof(double), cudaMemcpyDeviceToHost, c->s));
    CK(cudaMemcpyAsync(gy, c->gy, n * sizeof(double), cudaMemcpyDeviceToHost, c->s));
    CK(cudaMemcpyAsync(gz, c->gz, n * sizeof(double), cudaMemcpyDeviceToHost, c->s));
    return sync_ctx(c);
}

extern "C" int hc_get_phi(hc_ctx *c, double *phi)
{
    if (!c || !phi) return set_err(HC_ERR_ARG, "null argument");
    if (!c->gravity) return set_err(HC_ERR_STATE, "gravity disabled");
    CK(cudaSetDevice(c->dev));
    CK(cudaMemcpyAsync(phi, c->phi, (size_t)c->g.n * sizeof(double), cudaMemcpyDeviceToHost, c->s));
    return sync_ctx(c);
}

extern "C" int hc_set_phi(hc_ctx *c, const double *phi)
{
    if (!c || !phi) return set_err(HC_ERR_ARG, "null argument");
    if (!c->gravity) return set_err(HC_ERR_STATE, "gravity disabled");
    CK(cudaSetDevice(c->dev));
    CK(cudaMemcpyAsync(c->phi, phi, (size_t)c->g.n * sizeof(double), cudaMemcpyHostToDevice, c->s));
    return sync_ctx(c);
}

extern "C" int hc_get_moments(hc_ctx *c, double *mom, int cap)
{
    if (!c || !mom || cap < 13) return set_err(HC_ERR_ARG, "bad argument");
    if (!c->gravity) return set_err(HC_ERR_STATE, "gravity disabled");
    CK(cudaSetDevice(c->dev));
    if (c->cfg.lmax == 0) {
        CK(cudaMemcpyAsync(c->hsc->moments, c->sc->moments, sizeof(double) * 13, cudaMemcpyDeviceToHost, c->s));
        int rc = sync_ctx(c);
        if (rc) return rc;
        memcpy(mom, c->hsc->moments, sizeof(double) * 13);
        return HC_OK;
    }
    int nc = 4 + lmax_ncoef(c->cfg.lmax);
    if (cap < nc) return set_err(HC_ERR_ARG, "need %d doubles", nc);
    CK(cudaMemcpyAsync(mom, c->mom, sizeof(double) * nc, cudaMemcpyDeviceToHost, c->s));
    return sync_ctx(c);
}

extern "C" int hc_set_gravity_params(hc_ctx *c, double omega, int max_iter, double tol)
{
    if (!c) return set_err(HC_ERR_ARG, "null context");
    c->cfg.omega = omega;
    c->cfg.max_iter = max_iter;
    c->cfg.tol = tol;
    if (c->gravity) {
        CK(cudaSetDevice(c->dev));
        return ensure_res(c, max_iter);
    }
    return HC_OK;
}

extern "C" int hc_set_gravity_bc(hc_ctx *c, int bc)
{
    if (!c || bc < 0 || bc > 2) return set_err(HC_ERR_ARG, "bad gravity bc");
    c->cfg.grav_bc = bc;
    return HC_OK;
}

extern "C" int hc_residual_norm(hc_ctx *c, double *out)
{
    if (!c || !out) return set_err(HC_ERR_ARG, "null argument");
    if (!c->gravity) return set_err(HC_ERR_STATE, "gravity disabled");
    CK(cudaSetDevice(c->dev));
    if (c->cfg.gravity_only && !c->rho_ext) return set_err(HC_ERR_STATE, "no density solved for yet");
    GravArgs a = c->cfg.gravity_only ? grav_args(c, c->rho_ext, nullptr)
                 : c->cfg.precision == HC_FP64 ? grav_args(c, c->q64[c->cur][0], nullptr)
                                               : grav_args(c, nullptr, c->q32[c->cur][0]);
    CK(cudaMemsetAsync(&c->sc->resnorm, 0, sizeof(double), c->s));
    CK(grav_residual_norm(a, c->phi, c->s));
    CK(cudaMemcpyAsync(&c->hsc->resnorm, &c->sc->resnorm, sizeof(double), cudaMemcpyDeviceToHost, c->s));
    int rc = sync_ctx(c);
    if (rc) return rc;
    *out = c->hsc->resnorm;
    return HC_OK;
}

// ---------------------------------------------------------------- step
static HydroArgs hydro_args(hc_ctx *c)
{
    HydroArgs a;
    memset(&a, 0, sizeof a);
    a.g = c->g;
    a.gamma = c->cfg.gamma;
    a.cfl = c->cfg.cfl;
    for (int t = 0; t < 6; t++) a.bc[t] = c->cfg.bc[t];
    a.gravity = c->gravity;
    const int nxt = c->cur ^ 1;
    for (int v = 0; v < 5; v++) {
        if (c->cfg.precision == HC_FP64) {
            a.qin[v] = c->q64[c->cur][v];
            a.qout[v] = c->q64[nxt][v];
        } else {
            a.qin[v] = c->q32[c->cur][v];
            a.qout[v] = c->q32[nxt][v];
        }
    }
    a.phig = c->phig;
    a.sc = c->sc;
    a.step_parity = c->parity;
    return a;
}

static int interior_chunks(const hc_ctx *c)
{
    long long tiles = (long long)((c->g.nz + 31) / 32) * ((c->g.ny + 7) / 8);
    long long want = 148LL * 2 * 4;   // ~4 waves of 2 resident blocks per SM
    long long ch = (want + tiles - 1) / tiles;
    ch = std::max(1LL, std::min(ch, (long long)(c->g.nx - 2)));
    // keep at least 8 planes per chunk so the prologue plane stays cheap
    ch = std::min(ch, std::max(1LL, (long long)(c->g.nx - 2) / 8));
    return (int)ch;
}

// One godunov step on the device state (no host synchronisation).
static int step_once(hc_ctx *c, int *grav_status)
{
    if (c->cfg.gravity_only) return set_err(HC_ERR_STATE, "gravity-only context has no hydro state");
    const bool f64 = c->cfg.precision == HC_FP64;
    if (!c->cfl_valid) {
        HydroArgs a = hydro_args(c);
        FamTimer t(c, FAM_BC);
        CK(f64 ? fp64_cfl_full(a, c->s) : fp32_cfl_full(a, c->s));
        c->launches += 2;
        c->cfl_valid = 1;
    }
    *grav_status = 1;
    if (c->gravity && c->slab) {
        *grav_status = c->diag.last_status;   // the solve ran across the slabs
    } else if (c->gravity) {
        int st = f64 ? gravity_solve_dev(c, c->q64[c->cur][0], nullptr)
                     : gravity_solve_dev(c, nullptr, c->q32[c->cur][0]);
        if (st < -1) return st;
        *grav_status = st;
    }
    HydroArgs a = hydro_args(c);
    {
        FamTimer t(c, FAM_BC);
        CK(f64 ? fp64_dt(a, c->s) : fp32_dt(a, c->s));
    }
    {
        FamTimer t(c, FAM_HYDRO);
        if (f64 && c->cfg.recon == 1) {
            if (!c->plm && dmalloc((void **)&c->plm, 20 * (size_t)c->g.n * sizeof(double)))
                return set_err(HC_ERR_NOMEM, "MUSCL-Hancock face-state buffer");
            CK(fp64_plm_interior(a, c->plm, c->s));
            c->launches += 1;
        } else {
            CK(f64 ? fp64_interior(a, interior_chunks(c), c->s) : fp32_interior(a, interior_chunks(c), c->s));
        }
    }
    {
        FamTimer t(c, FAM_BC);
        CK(f64 ? fp64_boundary_source(a, c->s) : fp32_boundary_source(a, c->s));
        c->launches += 3;
        for (int ax = 0; ax < 3; ax++)
            if (c->cfg.bc[2 * ax] == 0 && c->cfg.bc[2 * ax + 1] == 0) {
                CK(f64 ? fp64_periodic(a, ax, c->s) : fp32_periodic(a, ax, c->s));
                c->launches++;
            }
        for (int ax = 0; ax < 3; ax++) {
            CK(f64 ? fp64_bc(a, ax, c->s) : fp32_bc(a, ax, c->s));
            c->launches++;
        }
        CK(f64 ? fp64_cfl_boundary(a, c->s) : fp32_cfl_boundary(a, c->s));
        c->launches++;
    }
    c->hydro_launches++;
    c->cur ^= 1;
    c->parity ^= 1;
    c->diag.steps++;
    return HC_OK;
}

static int launch_cons_sums(hc_ctx *c);

static int ensure_hdt(hc_ctx *c, int n)
{
    if (c->hdt && c->hdt_cap >= n) return HC_OK;
    if (c->hdt) cudaFreeHost(c->hdt);
    c->hdt = nullptr;
    int cap = std::max(n, 64);
    if (cudaMallocHost((void **)&c->hdt, cap * sizeof(double)) != cudaSuccess)
        return set_err(HC_ERR_NOMEM, "pinned dt buffer");
    c->hdt_cap = cap;
    return HC_OK;
}

extern "C" int hc_step(hc_ctx *c, int nsteps, double *dt_out)
{
    if (!c || nsteps < 0) return set_err(HC_ERR_ARG, "bad argument");
    CK(cudaSetDevice(c->dev));
    int rc = ensure_hdt(c, nsteps);
    if (rc) return rc;
    int worst = 0;
    for (int q = 0; q < nsteps; q++) {
        int gs = 1;
        rc = step_once(c, &gs);
        if (rc) return rc;
        if (gs == -1) worst = -1;
        CK(cudaMemcpyAsync(c->hdt + q, &c->sc->dt, sizeof(double), cudaMemcpyDeviceToHost, c->s));
    }
    if (c->cons_record && nsteps > 0) {
        rc = launch_cons_sums(c);
        if (rc) return rc;
        CK(cudaMemcpyAsync(c->hsc->cons, c->sc->cons, sizeof c->hsc->cons, cudaMemcpyDeviceToHost, c->s));
    }
    rc = sync_ctx(c);
    if (rc) return rc;
    if (nsteps > 0) c->diag.dt = c->hdt[nsteps - 1];
    if (c->cons_record && nsteps > 0)
        for (int v = 0; v < 5; v++) c->diag.cons[v] = c->hsc->cons[v];
    if (dt_out)
        for (int q = 0; q < nsteps; q++) dt_out[q] = c->hdt[q];
    return worst ? HC_NOT_CONVERGED : HC_OK;
}

extern "C" int hc_step_host(hc_ctx *c, double *U, double *dt_out)
{
    if (c && c->cfg.gravity_only) return set_err(HC_ERR_STATE, "gravity-only context has no hydro state");
    if (!c || !U) return set_err(HC_ERR_ARG, "null argument");
    CK(cudaSetDevice(c->dev));
    int rc = ensure_stage(c);
    if (rc) return rc;
    rc = ensure_hdt(c, 1);
    if (rc) return rc;
    const size_t n = (size_t)c->g.n;
    CK(cudaMemcpyAsync(c->stage, U, 5 * n * sizeof(double), cudaMemcpyHostToDevice, c->s));
    if (c->cfg.precision == HC_FP64) CK(fp64_aos_to_soa(c->stage, c->q64[c->cur], c->g.n, c->s));
    else CK(fp32_from_aos64(c->stage, c->q32[c->cur], c->g.n, c->s));
    c->cfl_valid = 0;
    int gs = 1;
    rc = step_once(c, &gs);
    if (rc) return rc;
    CK(cudaMemcpyAsync(c->hdt, &c->sc->dt, sizeof(double), cudaMemcpyDeviceToHost, c->s));
    if (c->cfg.precision == HC_FP64) CK(fp64_soa_to_aos(c->q64[c->cur], c->stage, c->g.n, c->s));
    else CK(fp32_to_aos64(c->q32[c->cur], c->stage, c->g.n, c->s));
    CK(cudaMemcpyAsync(U, c->stage, 5 * n * sizeof(double), cudaMemcpyDeviceToHost, c->s));
    rc = sync_ctx(c);
    if (rc) return rc;
    c->diag.dt = c->hdt[0];
    if (dt_out) *dt_out = c->hdt[0];
    return gs == -1 ? HC_NOT_CONVERGED : HC_OK;
}

// FP64 sums of the current state's 5 conserved fields into sc->cons (no sync).
static int launch_cons_sums(hc_ctx *c)
{
    if (!c->cons_part && dmalloc((void **)&c->cons_part, 5 * (size_t)CONS_BLOCKS * sizeof(double)))
        return set_err(HC_ERR_NOMEM, "conservation-sum partials");
    if (c->cfg.precision == HC_FP64) {
        ConsFields<double> q;
        for (int v = 0; v < 5; v++) q.f[v] = c->q64[c->cur][v];
        CK(cons_sums(q, c->g.n, c->cons_part, c->sc->cons, c->s));
    } else {
        ConsFields<float> q;
        for (int v = 0; v < 5; v++) q.f[v] = c->q32[c->cur][v];
        CK(cons_sums(q, c->g.n, c->cons_part, c->sc->cons, c->s));
    }
    c->launches += 2;
    return HC_OK;
}

extern "C" int hc_conservation_sums(hc_ctx *c, double *out)
{
    if (!c || !out) return set_err(HC_ERR_ARG, "null argument");
    if (c->cfg.gravity_only) return set_err(HC_ERR_STATE, "gravity-only context has no hydro state");
    CK(cudaSetDevice(c->dev));
    int rc = launch_cons_sums(c);
    if (rc) return rc;
    CK(cudaMemcpyAsync(c->hsc->cons, c->sc->cons, sizeof c->hsc->cons, cudaMemcpyDeviceToHost, c->s));
    rc = sync_ctx(c);
    if (rc) return rc;
    for (int v = 0; v < 5; v++) out[v] = c->hsc->cons[v];
    return HC_OK;
}

extern "C" int hc_set_conservation_record(hc_ctx *c, int on)
{
    if (!c || (on != 0 && on != 1)) return set_err(HC_ERR_ARG, "bad argument");
    if (c->cfg.gravity_only && on) return set_err(HC_ERR_STATE, "gravity-only context has no hydro state");
    c->cons_record = on;
    return HC_OK;
}

extern "C" int hc_get_diag(hc_ctx *c, hc_diag *d)
{
    if (!c || !d) return set_err(HC_ERR_ARG, "null argument");
    *d = c->diag;
    return HC_OK;
}

extern "C" int hc_get_timing(hc_ctx *c, hc_timing *t, int reset)
{
    if (!c || !t) return set_err(HC_ERR_ARG, "null argument");
    int rc = sync_ctx(c);
    if (rc) return rc;
    t->hydro_ms = c->fam_ms[FAM_HYDRO];
    t->bc_ms = c->fam_ms[FAM_BC];
    t->sor_ms = c->fam_ms[FAM_SOR];
    t->residual_ms = c->fam_ms[FAM_RES];
    t->moments_ms = c->fam_ms[FAM_MOM];
    t->unet_ms = c->fam_ms[FAM_UNET];
    t->hydro_launches = c->hydro_launches;
    t->sor_launches = c->sor_launches;
    t->launches = c->launches;
    if (reset) {
        for (int f = 0; f < FAM_N; f++) c->fam_ms[f] = 0.0;
        c->hydro_launches = c->sor_launches = c->launches = 0;
    }
    return HC_OK;
}

extern "C" int hc_sync(hc_ctx *c)
{
    if (!c) return set_err(HC_ERR_ARG, "null context");
    CK(cudaSetDevice(c->dev));
    return sync_ctx(c);
}

extern "C" int hc_timer_start(hc_ctx *c)
{
    if (!c) return set_err(HC_ERR_ARG, "null context");
    CK(cudaSetDevice(c->dev));
    if (!c->t0) CK(cudaEventCreate(&c->t0));
    if (!c->t1) CK(cudaEventCreate(&c->t1));
    CK(cudaEventRecord(c->t0, c->s));
    c->timer_on = 1;
    return HC_OK;
}

extern "C" int hc_timer_stop(hc_ctx *c, double *ms)
{
    if (!c || !ms) return set_err(HC_ERR_ARG, "null argument");
    if (!c->timer_on) return set_err(HC_ERR_STATE, "timer not started");
    CK(cudaSetDevice(c->dev));
    CK(cudaEventRecord(c->t1, c->s));
    CK(cudaEventSynchronize(c->t1));
    float f = 0.f;
    CK(cudaEventElapsedTime(&f, c->t0, c->t1));
    *ms = f;
    c->timer_on = 0;
    return sync_ctx(c);
}

// ---------------------------------------------------------------- slabs
extern "C" int hc_get_signal_speed(hc_ctx *c, double *s)
{
    if (!c || !s) return set_err(HC_ERR_ARG, "null argument");
    if (c->cfg.gravity_only) return set_err(HC_ERR_STATE, "gravity-only context has no hydro state");
    CK(cudaSetDevice(c->dev));
    const bool f64 = c->cfg.precision == HC_FP64;
    if (!c->cfl_valid) {
        HydroArgs a = hydro_args(c);
        FamTimer t(c, FAM_BC);
        CK(f64 ? fp64_cfl_full(a, c->s) : fp32_cfl_full(a, c->s));
        c->launches += 2;
        c->cfl_valid = 1;
    }
    CK(cudaMemcpyAsync(&c->hsc->smax[c->parity], &c->sc->smax[c->parity], sizeof(unsigned long long),
                       cudaMemcpyDeviceToHost, c->s));
    int rc = sync_ctx(c);
    if (rc) return rc;
    const unsigned long long b = c->hsc->smax[c->parity];
    double v;
    if (f64) {
        memcpy(&v, &b, sizeof v);
    } else {
        const unsigned int lo = (unsigned int)b;
        float f;
        memcpy(&f, &lo, sizeof f);
        v = f;
    }
    *s = v;
    return HC_OK;
}

extern "C" int hc_set_signal_speed(hc_ctx *c, double s)
{
    if (!c || !(s > 0.0) || !std::isfinite(s)) return set_err(HC_ERR_ARG, "signal speed must be finite and positive");
    if (c->cfg.gravity_only) return set_err(HC_ERR_STATE, "gravity-only context has no hydro state");
    CK(cudaSetDevice(c->dev));
    unsigned long long b = 0;
    if (c->cfg.precision == HC_FP64) {
        memcpy(&b, &s, sizeof b);
    } else {
        const float f = (float)s;
        if ((double)f != s) return set_err(HC_ERR_ARG, "FP32 context: the signal speed must be an FP32 value");
        unsigned int lo;
        memcpy(&lo, &f, sizeof lo);
        b = lo;
    }
    c->hsc->smax[c->parity] = b;
    CK(cudaMemcpyAsync(&c->sc->smax[c->parity], &c->hsc->smax[c->parity], sizeof b, cudaMemcpyHostToDevice, c->s));
    c->cfl_valid = 1;
    return sync_ctx(c);
}

extern "C" int hc_copy_planes(hc_ctx *c, int i0, int count, void *buf, int to_ctx)
{
    if (!c || !buf) return set_err(HC_ERR_ARG, "null argument");
    if (c->cfg.gravity_only) return set_err(HC_ERR_STATE, "gravity-only context has no hydro state");
    if (i0 < 0 || count < 0 || i0 + count > c->g.nx || (to_ctx != 0 && to_ctx != 1))
        return set_err(HC_ERR_ARG, "planes [%d, %d) outside 0..%d", i0, i0 + count, c->g.nx);
    CK(cudaSetDevice(c->dev));
    const size_t word = c->cfg.precision == HC_FP64 ? 8 : 4;
    const size_t plane = (size_t)c->g.ny * c->g.nz;
    const size_t bytes = (size_t)count * plane * word;
    for (int v = 0; v < 5; v++) {
        char *field = c->cfg.precision == HC_FP64 ? reinterpret_cast<char *>(c->q64[c->cur][v])
                                                  : reinterpret_cast<char *>(c->q32[c->cur][v]);
        char *f = field + (size_t)i0 * plane * word;
        char *b = static_cast<char *>(buf) + (size_t)v * bytes;
        CK(cudaMemcpyAsync(to_ctx ? f : b, to_ctx ? b : f, bytes, cudaMemcpyDefault, c->s));
    }
    return sync_ctx(c);
}

// ---------------------------------------------------------------- slabs: gravity
// The Poisson solve of a grid split along x into slabs (FP64, isolated
// boundary), driven across the slabs by the caller: the moment sums of the
// own planes (chained in plane order, or per-plane partials gathered in
// plane order), the red-black half sweeps with the ghost planes exchanged
// after each, and the maximum of the slabs' update norms as the stop test
// (gravity_solver_3d.c:510-747 on the whole grid).
extern "C" int hc_set_slab(hc_ctx *c, int gnx, int ioff)
{
    if (!c) return set_err(HC_ERR_ARG, "null context");
    const int nx = c->g.nx;
    if (ioff < 0 || gnx < nx || ioff + nx > gnx)
        return set_err(HC_ERR_ARG, "planes [%d, %d) outside a grid of %d", ioff, ioff + nx, gnx);
    const int olo = ioff > 0 ? 1 : 0, ohi = ioff + nx < gnx ? nx - 1 : nx;
    if (ohi - olo < 1) return set_err(HC_ERR_ARG, "a slab needs an own plane");
    if (c->gravity) {
        if (c->cfg.precision != HC_FP64) return set_err(HC_ERR_STATE, "slab gravity: FP64 contexts");
        if (c->cfg.grav_bc != 1) return set_err(HC_ERR_STATE, "slab gravity: isolated boundary only");
        if (c->g.nz < 3 || c->g.ny < 3) return set_err(HC_ERR_STATE, "slab gravity: ny, nz >= 3");
        if (c->cfg.lmax == 0 && c->cfg.moment_order != HC_MOMENTS_SEQUENTIAL &&
            c->cfg.moment_order != HC_MOMENTS_TREE)
            return set_err(HC_ERR_STATE, "slab gravity: sequential or tree moments");
    }
    Geom &g = c->g;
    g.ioff = ioff;
    g.gnx = gnx;
    g.olo = olo;
    g.ohi = ohi;
    if (!(c->cfg.dx > 0.0)) g.dx = (c->cfg.xmax - c->cfg.xmin) / gnx;
    c->slab = 1;
    return HC_OK;
}

static bool slab_sequential(const hc_ctx *c)
{
    return c->cfg.lmax == 0 && c->cfg.moment_order == HC_MOMENTS_SEQUENTIAL;
}

// Doubles per own plane of a pass's partials (or, sequential, the sums).
static int slab_width(const hc_ctx *c, int pass)
{
    if (slab_sequential(c)) return pass == 0 ? 4 : 9;
    if (c->cfg.lmax == 0) return 9;   // tree partials: 9 slots per plane in both passes
    return lmax_slab_width(c->g, pass);
}

static int slab_ready(hc_ctx *c)
{
    if (!c) return set_err(HC_ERR_ARG, "null context");
    if (!c->slab || !c->gravity) return set_err(HC_ERR_STATE, "not a self-gravitating slab (hc_set_slab)");
    if (c->cfg.gravity_only) return set_err(HC_ERR_STATE, "gravity-only context");
    CK(cudaSetDevice(c->dev));
    return HC_OK;
}

static int slab_buffer(hc_ctx *c, long long need)
{
    if (c->slab_buf && c->slab_buf_len >= need) return HC_OK;
    cudaFree(c->slab_buf);
    c->slab_buf = nullptr;
    int rc = dmalloc((void **)&c->slab_buf, (size_t)need * sizeof(double));
    if (rc) return rc;
    c->slab_buf_len = need;
    return HC_OK;
}

extern "C" int hc_slab_moment_layout(hc_ctx *c, int pass, int *sequential, int *width)
{
    int rc = slab_ready(c);
    if (rc) return rc;
    if ((pass != 0 && pass != 1) || !sequential || !width) return set_err(HC_ERR_ARG, "bad argument");
    *sequential = slab_sequential(c) ? 1 : 0;
    *width = slab_width(c, pass);
    return HC_OK;
}

extern "C" int hc_slab_moments(hc_ctx *c, int pass, double *buf)
{
    int rc = slab_ready(c);
    if (rc) return rc;
    if ((pass != 0 && pass != 1) || !buf) return set_err(HC_ERR_ARG, "bad argument");
    GravArgs a = grav_args(c, c->q64[c->cur][0], nullptr);
    const int w = slab_width(c, pass);
    const int np = c->g.ohi - c->g.olo;
    const long long count = slab_sequential(c) ? w : (long long)np * w;
    rc = slab_buffer(c, count);
    if (rc) return rc;
    {
        FamTimer t(c, FAM_MOM);
        if (slab_sequential(c)) {
            CK(cudaMemcpyAsync(c->slab_buf, buf, count * sizeof(double), cudaMemcpyHostToDevice, c->s));
            CK(grav_moments_seq_slab(a, pass, c->slab_buf, c->s));
        } else if (c->cfg.lmax == 0) {
            CK(grav_moments_tree_parts(a, pass, c->slab_buf, c->s));
        } else {
            CK(grav_moments_lmax_parts(a, pass, c->slab_buf, c->s));
        }
        c->launches += 1;
    }
    CK(cudaMemcpyAsync(buf, c->slab_buf, count * sizeof(double), cudaMemcpyDeviceToHost, c->s));
    return sync_ctx(c);
}

extern "C" int hc_slab_set_moments(hc_ctx *c, int pass, const double *all, int nplanes)
{
    int rc = slab_ready(c);
    if (rc) return rc;
    if ((pass != 0 && pass != 1) || !all) return set_err(HC_ERR_ARG, "bad argument");
    const int w = slab_width(c, pass);
    if (!slab_sequential(c) && nplanes != c->g.gnx)
        return set_err(HC_ERR_ARG, "partials of %d planes for a grid of %d", nplanes, c->g.gnx);
    const long long count = slab_sequential(c) ? w : (long long)nplanes * w;
    rc = slab_buffer(c, count);
    if (rc) return rc;
    GravArgs a = grav_args(c, c->q64[c->cur][0], nullptr);
    FamTimer t(c, FAM_MOM);
    CK(cudaMemcpyAsync(c->slab_buf, all, count * sizeof(double), cudaMemcpyHostToDevice, c->s));
    if (slab_sequential(c)) CK(grav_moments_seq_set(a, pass, c->slab_buf, c->s));
    else if (c->cfg.lmax == 0) CK(grav_moments_tree_set(a, pass, c->slab_buf, nplanes, c->s));
    else CK(grav_moments_lmax_set(a, pass, c->slab_buf, nplanes, c->s));
    c->launches += 1;
    return sync_ctx(c);
}

extern "C" int hc_slab_sor_begin(hc_ctx *c)
{
    int rc = slab_ready(c);
    if (rc) return rc;
    GravArgs a = grav_args(c, c->q64[c->cur][0], nullptr);
    rc = ensure_res(c, a.max_iter);
    if (rc) return rc;
    a.res = c->res;
    const size_t ns = (size_t)split_len(c->g);
    if (!c->phs) rc = dmalloc((void **)&c->phs, ns * sizeof(double));
    if (!rc && !c->rhs) rc = dmalloc((void **)&c->rhs, ns * sizeof(double));
    if (rc) return rc;
    if (!c->hslots && cudaMallocHost((void **)&c->hslots, 512 * sizeof(double)) != cudaSuccess)
        return set_err(HC_ERR_NOMEM, "pinned slot buffer");
    CK(cudaMemsetAsync(&c->sc->done, 0, 2 * sizeof(int), c->s));
    CK(grav_reset_slots(a, 0, std::max(a.max_iter, 1), c->s));
    CK(grav_split_fields(a, c->phs, c->rhs, c->s));
    c->launches += 3;
    return HC_OK;
}

// One half sweep of the whole grid's colour (local colour colour ^ ioff).
extern "C" int hc_slab_sor_sweep(hc_ctx *c, int iter, int colour)
{
    int rc = slab_ready(c);
    if (rc) return rc;
    if (iter < 0 || iter >= c->cfg.max_iter || (colour != 0 && colour != 1) || !c->phs)
        return set_err(HC_ERR_ARG, "bad sweep (iteration %d, colour %d)", iter, colour);
    GravArgs a = grav_args(c, c->q64[c->cur][0], nullptr);
    a.res = c->res;
    a.tol = -1.0;   // the stop test is the caller's, over all slabs
    FamTimer t(c, FAM_SOR);
    CK(grav_sor_split(a, c->phs, c->rhs, colour ^ (c->g.ioff & 1), iter, c->s));
    c->launches += 1;
    c->sor_launches += 1;
    return HC_OK;
}

extern "C" int hc_slab_sor_boundary(hc_ctx *c)
{
    int rc = slab_ready(c);
    if (rc) return rc;
    if (!c->phs) return set_err(HC_ERR_STATE, "hc_slab_sor_begin first");
    GravArgs a = grav_args(c, c->q64[c->cur][0], nullptr);
    rc = grav_boundary_values(c, a);
    if (rc) return rc;
    CK(grav_split_boundary(a, c->phs, c->s));
    c->launches += 1;
    return HC_OK;
}

extern "C" int hc_slab_sor_norm(hc_ctx *c, int iter, double *norm)
{
    int rc = slab_ready(c);
    if (rc) return rc;
    if (iter < 0 || iter >= c->cfg.max_iter || !norm) return set_err(HC_ERR_ARG, "bad argument");
    if (!c->hslots) return set_err(HC_ERR_STATE, "hc_slab_sor_begin first");
    CK(cudaMemcpyAsync(c->hslots, c->res + iter, sizeof(double), cudaMemcpyDeviceToHost, c->s));
    rc = sync_ctx(c);
    if (rc) return rc;
    *norm = c->hslots[0];
    return HC_OK;
}

extern "C" int hc_slab_sor_end(hc_ctx *c, int iterations, double residual, int converged)
{
    int rc = slab_ready(c);
    if (rc) return rc;
    if (!c->phs) return set_err(HC_ERR_STATE, "hc_slab_sor_begin first");
    GravArgs a = grav_args(c, c->q64[c->cur][0], nullptr);
    CK(grav_unsplit(a, c->phs, c->s));
    c->launches += 1;
    c->diag.last_iterations = iterations;
    c->diag.last_residual = residual;
    c->diag.total_iterations += iterations;
    c->diag.last_status = converged ? 0 : -1;
    if (converged) CK(cudaMemcpyAsync(c->phig, c->phi, (size_t)c->g.n * sizeof(double), cudaMemcpyDeviceToDevice, c->s));
    return sync_ctx(c);
}

// Planes [i0, i0 + count) of the colour-split potential, both colours:
// buf holds [2][count][ny * ((nz + 1) / 2)] doubles indexed by the whole
// grid's colour.  The context's colour arrays are split by the local parity
// (i + j + k) & 1, which is the global colour xor (ioff & 1); a row keeps the
// same position k >> 1 in either, so slabs of either offset parity exchange
// through the same buffer.
extern "C" int hc_slab_phi_planes(hc_ctx *c, int i0, int count, void *buf, int to_ctx)
{
    int rc = slab_ready(c);
    if (rc) return rc;
    if (!buf || !c->phs || i0 < 0 || count < 0 || i0 + count > c->g.nx || (to_ctx != 0 && to_ctx != 1))
        return set_err(HC_ERR_ARG, "bad argument");
    const size_t plane = (size_t)c->g.ny * ((c->g.nz + 1) / 2);
    const size_t cs = (size_t)c->g.nx * plane, bytes = (size_t)count * plane * sizeof(double);
    for (int q = 0; q < 2; q++) {
        double *f = c->phs + (q ^ (c->g.ioff & 1)) * cs + (size_t)i0 * plane;
        char *b = static_cast<char *>(buf) + q * bytes;
        CK(cudaMemcpyAsync(to_ctx ? (void *)f : (void *)b, to_ctx ? (const void *)b : (const void *)f, bytes,
                           cudaMemcpyDefault, c->s));
    }
    return sync_ctx(c);
}

extern "C" int hc_host_register(void *ptr, size_t bytes)
{
    if (!ptr || !bytes) return set_err(HC_ERR_ARG, "null buffer");
    CK(cudaHostRegister(ptr, bytes, cudaHostRegisterDefault));
    return HC_OK;
}

extern "C" int hc_host_unregister(void *ptr)
{
    if (!ptr) return set_err(HC_ERR_ARG, "null buffer");
    CK(cudaHostUnregister(ptr));
    return HC_OK;
}

// Error reporting for entry points defined in other translation units.
int hc_internal_set_error(int code, const char *msg)
{
    return set_err(code, "%s", msg);
}

// ---------------------------------------------------------------- learned warm start
static int ensure_unet(hc_ctx *c)
{
    if (c->unet) return HC_OK;
    CK(cudaSetDevice(c->dev));
    c->unet = unet_create(c->dev);
    return c->unet ? HC_OK : set_err(HC_ERR_NOMEM, "U-Net parameter buffers");
}

extern "C" int hc_unet_param_count(void) { return unet_param_count(); }

extern "C" int hc_unet_init(hc_ctx *c, unsigned seed)
{
    if (!c) return set_err(HC_ERR_ARG, "null context");
    int rc = ensure_unet(c);
    return rc ? rc : unet_init(c->unet, seed, c->s);
}

extern "C" int hc_unet_load(hc_ctx *c, const float *params, int nparam, double kscale)
{
    if (!c) return set_err(HC_ERR_ARG, "null context");
    int rc = ensure_unet(c);
    if (rc) return rc;
    rc = unet_set_params(c->unet, params, nparam, (float)kscale, c->s);
    return rc ? set_err(rc, "hc_unet_load: expected %d parameters and kscale > 0", unet_param_count()) : HC_OK;
}

extern "C" int hc_unet_save(hc_ctx *c, float *params, int nparam, double *kscale)
{
    if (!c || !c->unet || !unet_has_weights(c->unet)) return set_err(HC_ERR_STATE, "no U-Net weights");
    if (kscale) *kscale = unet_kscale(c->unet);
    return unet_get_params(c->unet, params, nparam, c->s);
}

// file: "HCUNET01", int32 parameter count, float32 kscale, float32 parameters
extern "C" int hc_unet_save_file(hc_ctx *c, const char *path)
{
    const int n = unet_param_count();
    std::vector<float> p(n);
    double k = 0.0;
    int rc = hc_unet_save(c, p.data(), n, &k);
    if (rc) return rc;
    FILE *f = fopen(path, "wb");
    if (!f) return set_err(HC_ERR_ARG, "cannot write %s", path);
    const float kf = (float)k;
    bool ok = fwrite("HCUNET01", 1, 8, f) == 8 && fwrite(&n, 4, 1, f) == 1 && fwrite(&kf, 4, 1, f) == 1 &&
              fwrite(p.data(), 4, n, f) == (size_t)n;
    ok = (fclose(f) == 0) && ok;
    return ok ? HC_OK : set_err(HC_ERR_ARG, "short write to %s", path);
}

extern "C" int hc_unet_load_file(hc_ctx *c, const char *path)
{
    FILE *f = fopen(path, "rb");
    if (!f) return set_err(HC_ERR_ARG, "cannot read %s", path);
    char magic[8];
    int n = 0;
    float k = 0.f;
    bool ok = fread(magic, 1, 8, f) == 8 && memcmp(magic, "HCUNET01", 8) == 0 && fread(&n, 4, 1, f) == 1 &&
              fread(&k, 4, 1, f) == 1 && n == unet_param_count();
    std::vector<float> p(ok ? n : 0);
    ok = ok && fread(p.data(), 4, n, f) == (size_t)n;
    fclose(f);
    if (!ok) return set_err(HC_ERR_ARG, "%s is not a U-Net weight file of %d parameters", path, unet_param_count());
    return hc_unet_load(c, p.data(), n, k);
}

extern "C" int hc_unet_collect(hc_ctx *c, int capacity)
{
    if (!c || capacity < 0) return set_err(HC_ERR_ARG, "bad argument");
    int rc = ensure_unet(c);
    if (rc) return rc;
    rc = unet_collect(c->unet, capacity);
    return rc ? set_err(rc, "sample buffers") : HC_OK;
}

extern "C" int hc_unet_samples(hc_ctx *c) { return (c && c->unet) ? unet_samples(c->unet) : 0; }

extern "C" int hc_unet_train(hc_ctx *c, int steps, double lr, unsigned seed, double *mean_loss)
{
    if (!c || !c->unet) return set_err(HC_ERR_STATE, "no U-Net");
    CK(cudaSetDevice(c->dev));
    int rc;
    {
        FamTimer t(c, FAM_UNET);
        rc = unet_train(c->unet, steps, lr, seed, mean_loss, c->s);
    }
    if (rc == HC_ERR_STATE) return set_err(rc, "no training samples (hc_unet_collect, then solve)");
    if (rc) return set_err(rc, "U-Net training failed");
    return sync_ctx(c);
}

extern "C" int hc_unet_loss_grad(hc_ctx *c, int nx, int ny, int nz, const float *x, const float *t, double *loss,
                                 float *grad, float *out)
{
    if (!c || !c->unet || !x || !t || nx < 2 || ny < 2 || nz < 2 || nx % 16 || ny % 16 || nz % 16)
        return set_err(HC_ERR_ARG, "bad argument (level-0 dimensions must be multiples of 16)");
    CK(cudaSetDevice(c->dev));
    const int rc = unet_loss_grad(c->unet, nx, ny, nz, x, t, loss, grad, out, c->s);
    return rc ? set_err(rc, "U-Net loss/gradient failed") : HC_OK;
}

extern "C" int hc_set_unet_passes(hc_ctx *c, int passes)
{
    if (!c || passes < 1 || passes > 8) return set_err(HC_ERR_ARG, "passes must be 1..8");
    c->unet_passes = passes;
    return HC_OK;
}

extern "C" int hc_set_unet_guard(hc_ctx *c, int consecutive_losses)
{
    if (!c || consecutive_losses < 0 || consecutive_losses > 64)
        return set_err(HC_ERR_ARG, "consecutive_losses must be 0..64");
    c->guard = UnetGuard();
    c->guard.K = consecutive_losses;
    return HC_OK;
}

extern "C" int hc_set_unet_cycles(hc_ctx *c, int cycles)
{
    if (!c || cycles < 1 || cycles > 8) return set_err(HC_ERR_ARG, "cycles must be 1..8");
    c->unet_cycles = cycles;
    return HC_OK;
}

extern "C" int hc_set_unet_record_cycle(hc_ctx *c, int cycle)
{
    if (!c || cycle < 0 || cycle > 8) return set_err(HC_ERR_ARG, "cycle must be 0..8");
    c->unet_record_cycle = cycle == 0 ? -1 : cycle;   // -1: record nothing
    return HC_OK;
}

extern "C" int hc_set_correction_omega(hc_ctx *c, double omega)
{
    if (!c || !(omega == 0.0 || (omega > 0.0 && omega < 2.0)))
        return set_err(HC_ERR_ARG, "correction omega must be 0 (the solve's omega) or in (0, 2)");
    c->corr_omega = omega;
    return HC_OK;
}

// ---------------------------------------------------------------- checkpoints
// Binary checkpoint of everything the next step reads: the conserved state
// in the context's own precision (bit for bit), and with self-gravity the
// potential (the next solve's starting iterate and boundary values) and the
// potential of the last converged solve (g); plus the step parity.  The CFL
// signal speed is recomputed from the state on load (a max: the same value).
// File: CkptHeader, then the payload -- 5 state fields (nx*ny*nz words each,
// k fastest), phi, phig -- with an FNV-1a 64 checksum of the payload in the
// header.  Saving packs the payload into one device buffer on the compute
// stream (device to device), then a writer thread copies it to the host on
// its own stream through two pinned 64 MB chunks and writes the file while
// the context keeps stepping.
namespace {
struct CkptHeader {
    char magic[8];      // "HCCKPT01"
    int32_t version, header_bytes;
    int32_t nx, ny, nz, precision, gravity, parity;
    int64_t step;
    double t, lo[3], hi[3], gamma, G;
    uint64_t payload_bytes, checksum;
};
constexpr size_t CK_CHUNK = (size_t)64 << 20;

uint64_t fnv1a(uint64_t h, const unsigned char *p, size_t n)
{
    for (size_t i = 0; i < n; i++) {
        h ^= p[i];
        h *= 1099511628211ULL;
    }
    return h;
}
constexpr uint64_t FNV_OFFSET = 14695981039346656037ULL;

size_t ck_payload_bytes(const hc_ctx *c)
{
    const size_t n = (size_t)c->g.n;
    return 5 * n * (c->cfg.precision == HC_FP64 ? 8 : 4) + (c->gravity ? 2 * n * 8 : 0);
}

void ck_fill_header(const hc_ctx *c, CkptHeader &h)
{
    memset(&h, 0, sizeof h);
    memcpy(h.magic, "HCCKPT01", 8);
    h.version = 1;
    h.header_bytes = (int32_t)sizeof(CkptHeader);
    h.nx = c->g.nx;
    h.ny = c->g.ny;
    h.nz = c->g.nz;
    h.precision = c->cfg.precision;
    h.gravity = c->gravity;
    h.parity = c->parity;
    h.lo[0] = c->cfg.xmin; h.lo[1] = c->cfg.ymin; h.lo[2] = c->cfg.zmin;
    h.hi[0] = c->cfg.xmax; h.hi[1] = c->cfg.ymax; h.hi[2] = c->cfg.zmax;
    h.gamma = c->cfg.gamma;
    h.G = c->cfg.G;
    h.payload_bytes = ck_payload_bytes(c);
}

int ck_buffers(hc_ctx *c, size_t bytes)
{
    if (!c->ck_dev || c->ck_dev_bytes < bytes) {
        cudaFree(c->ck_dev);
        c->ck_dev = nullptr;
        c->ck_dev_bytes = 0;
        if (dmalloc((void **)&c->ck_dev, bytes)) return set_err(HC_ERR_NOMEM, "checkpoint packing buffer");
        c->ck_dev_bytes = bytes;
    }
    for (int b = 0; b < 2; b++)
        if (!c->ck_host[b] && cudaMallocHost((void **)&c->ck_host[b], CK_CHUNK) != cudaSuccess)
            return set_err(HC_ERR_NOMEM, "pinned checkpoint chunks");
    if (!c->ck_stream && cudaStreamCreateWithFlags(&c->ck_stream, cudaStreamNonBlocking) != cudaSuccess)
        return set_err(HC_ERR_CUDA, "checkpoint stream");
    for (int e = 0; e < 3; e++)
        if (!c->ck_ev[e] && cudaEventCreateWithFlags(&c->ck_ev[e], cudaEventDisableTiming) != cudaSuccess)
            return set_err(HC_ERR_CUDA, "checkpoint events");
    return HC_OK;
}

// writer thread: chunk k is copied into pinned buffer k % 2 while chunk k-1
// is hashed and written
void ck_writer(hc_ctx *c, std::string path, CkptHeader h)
{
    auto fail = [&](int code, const char *what) {
        c->ck_status = code;
        snprintf(c->ck_err, sizeof c->ck_err, "checkpoint %s: %s", path.c_str(), what);
    };
    if (cudaSetDevice(c->dev) != cudaSuccess) return fail(HC_ERR_CUDA, "cudaSetDevice");
    FILE *f = fopen(path.c_str(), "wb");
    if (!f) return fail(HC_ERR_ARG, "cannot open for writing");
    bool ok = fwrite(&h, sizeof h, 1, f) == 1;
    const size_t bytes = h.payload_bytes;
    const size_t nch = (bytes + CK_CHUNK - 1) / CK_CHUNK;
    uint64_t hash = FNV_OFFSET;
    for (size_t k = 0; ok && k <= nch; k++) {
        if (k < nch) {
            const size_t off = k * CK_CHUNK, len = std::min(CK_CHUNK, bytes - off);
            if (cudaMemcpyAsync(c->ck_host[k & 1], c->ck_dev + off, len, cudaMemcpyDeviceToHost, c->ck_stream) !=
                    cudaSuccess ||
                cudaEventRecord(c->ck_ev[k & 1], c->ck_stream) != cudaSuccess) {
                fclose(f);
                return fail(HC_ERR_CUDA, "device-to-host copy");
            }
        }
        if (k >= 1) {
            const size_t q = k - 1, off = q * CK_CHUNK, len = std::min(CK_CHUNK, bytes - off);
            if (cudaEventSynchronize(c->ck_ev[q & 1]) != cudaSuccess) {
                fclose(f);
                return fail(HC_ERR_CUDA, "device-to-host copy");
            }
            hash = fnv1a(hash, c->ck_host[q & 1], len);
            ok = fwrite(c->ck_host[q & 1], 1, len, f) == len;
        }
    }
    h.checksum = hash;
    ok = ok && fseek(f, 0, SEEK_SET) == 0 && fwrite(&h, sizeof h, 1, f) == 1;
    ok = (fclose(f) == 0) && ok;
    if (!ok) fail(HC_ERR_ARG, "write failed");
}
}  // namespace

extern "C" int hc_checkpoint_wait(hc_ctx *c)
{
    if (!c) return set_err(HC_ERR_ARG, "null argument");
    if (c->ck_thread) {
        c->ck_thread->join();
        delete c->ck_thread;
        c->ck_thread = nullptr;
    }
    const int st = c->ck_status;
    c->ck_status = HC_OK;
    if (st) return set_err(st, "%s", c->ck_err);
    return HC_OK;
}

extern "C" int hc_checkpoint_save(hc_ctx *c, const char *path, double t, long long step)
{
    if (c && c->cfg.gravity_only) return set_err(HC_ERR_STATE, "gravity-only context has no hydro state");
    if (!c || !path) return set_err(HC_ERR_ARG, "null argument");
    CK(cudaSetDevice(c->dev));
    int rc = hc_checkpoint_wait(c);   // one write in flight per context
    if (rc) return rc;
    const size_t n = (size_t)c->g.n, bytes = ck_payload_bytes(c);
    rc = ck_buffers(c, bytes);
    if (rc) return rc;
    const bool f64 = c->cfg.precision == HC_FP64;
    const size_t w = f64 ? 8 : 4;
    for (int v = 0; v < 5; v++) {
        const void *src = f64 ? (const void *)c->q64[c->cur][v] : (const void *)c->q32[c->cur][v];
        CK(cudaMemcpyAsync(c->ck_dev + v * n * w, src, n * w, cudaMemcpyDeviceToDevice, c->s));
    }
    if (c->gravity) {
        CK(cudaMemcpyAsync(c->ck_dev + 5 * n * w, c->phi, n * 8, cudaMemcpyDeviceToDevice, c->s));
        CK(cudaMemcpyAsync(c->ck_dev + 5 * n * w + n * 8, c->phig, n * 8, cudaMemcpyDeviceToDevice, c->s));
    }
    CK(cudaEventRecord(c->ck_ev[2], c->s));
    CK(cudaStreamWaitEvent(c->ck_stream, c->ck_ev[2], 0));
    CkptHeader h;
    ck_fill_header(c, h);
    h.t = t;
    h.step = step;
    c->ck_status = HC_OK;
    try {
        c->ck_thread = new std::thread(ck_writer, c, std::string(path), h);
    } catch (...) {
        return set_err(HC_ERR_STATE, "cannot start the checkpoint writer thread");
    }
    return HC_OK;
}

extern "C" int hc_checkpoint_load(hc_ctx *c, const char *path, double *t, long long *step)
{
    if (c && c->cfg.gravity_only) return set_err(HC_ERR_STATE, "gravity-only context has no hydro state");
    if (!c || !path) return set_err(HC_ERR_ARG, "null argument");
    CK(cudaSetDevice(c->dev));
    int rc = hc_checkpoint_wait(c);
    if (rc) return rc;
    FILE *f = fopen(path, "rb");
    if (!f) return set_err(HC_ERR_ARG, "checkpoint: cannot open file");
    CkptHeader h, want;
    ck_fill_header(c, want);
    auto bad = [&](const char *what) {
        fclose(f);
        return set_err(HC_ERR_ARG, "%s", what);
    };
    if (fread(&h, sizeof h, 1, f) != 1 || memcmp(h.magic, "HCCKPT01", 8) != 0 || h.version != 1 ||
        h.header_bytes != (int32_t)sizeof(CkptHeader))
        return bad("checkpoint: not a version-1 checkpoint file");
    if (h.nx != want.nx || h.ny != want.ny || h.nz != want.nz || h.precision != want.precision ||
        h.gravity != want.gravity || h.payload_bytes != want.payload_bytes)
        return bad("checkpoint: grid, precision or gravity differ from this context");
    for (int a = 0; a < 3; a++)
        if (h.lo[a] != want.lo[a] || h.hi[a] != want.hi[a]) return bad("checkpoint: domain differs from this context");
    if (h.gamma != want.gamma || h.G != want.G) return bad("checkpoint: gamma or G differ from this context");
    const size_t bytes = h.payload_bytes;
    rc = ck_buffers(c, bytes);
    if (rc) {
        fclose(f);
        return rc;
    }
    // whole payload into the packing buffer first: a short or corrupt file
    // leaves the context's state untouched
    uint64_t hash = FNV_OFFSET;
    const size_t nch = (bytes + CK_CHUNK - 1) / CK_CHUNK;
    for (size_t k = 0; k < nch; k++) {
        const size_t off = k * CK_CHUNK, len = std::min(CK_CHUNK, bytes - off);
        unsigned char *buf = c->ck_host[k & 1];
        // the copy out of this buffer (chunk k - 2) is done
        cudaError_t e = k >= 2 ? cudaEventSynchronize(c->ck_ev[k & 1]) : cudaSuccess;
        if (e != cudaSuccess) {
            fclose(f);
            return set_err(HC_ERR_CUDA, "checkpoint load: %s", cudaGetErrorString(e));
        }
        if (fread(buf, 1, len, f) != len) {
            cudaStreamSynchronize(c->ck_stream);
            return bad("checkpoint: file is shorter than its header says");
        }
        hash = fnv1a(hash, buf, len);
        e = cudaMemcpyAsync(c->ck_dev + off, buf, len, cudaMemcpyHostToDevice, c->ck_stream);
        if (e == cudaSuccess) e = cudaEventRecord(c->ck_ev[k & 1], c->ck_stream);
        if (e != cudaSuccess) {
            fclose(f);
            return set_err(HC_ERR_CUDA, "checkpoint load: %s", cudaGetErrorString(e));
        }
    }
    fclose(f);
    CK(cudaStreamSynchronize(c->ck_stream));
    if (hash != h.checksum) return set_err(HC_ERR_ARG, "checkpoint: payload checksum mismatch");
    const size_t n = (size_t)c->g.n;
    const bool f64 = c->cfg.precision == HC_FP64;
    const size_t w = f64 ? 8 : 4;
    for (int v = 0; v < 5; v++) {
        void *dst = f64 ? (void *)c->q64[c->cur][v] : (void *)c->q32[c->cur][v];
        CK(cudaMemcpyAsync(dst, c->ck_dev + v * n * w, n * w, cudaMemcpyDeviceToDevice, c->s));
    }
    if (c->gravity) {
        CK(cudaMemcpyAsync(c->phi, c->ck_dev + 5 * n * w, n * 8, cudaMemcpyDeviceToDevice, c->s));
        CK(cudaMemcpyAsync(c->phig, c->ck_dev + 5 * n * w + n * 8, n * 8, cudaMemcpyDeviceToDevice, c->s));
    }
    c->parity = h.parity;
    c->cfl_valid = 0;
    if (t) *t = h.t;
    if (step) *step = h.step;
    return sync_ctx(c);
}

// ---------------------------------------------------------------- device ICs
extern "C" int hc_ic_profile_stars(hc_ctx *c, int nstars, const int *n, const double *const *r,
                                   const double *const *rho, const double *const *u, const double *R_star,
                                   const double *centre, const double *vel)
{
    if (c && c->cfg.gravity_only) return set_err(HC_ERR_STATE, "gravity-only context has no hydro state");
    if (!c || (nstars != 1 && nstars != 2) || !n || !r || !rho || !u || !centre ||
        (nstars == 2 && (!R_star || !vel)))
        return set_err(HC_ERR_ARG, "bad argument (1 or 2 stars; two stars need R_star and vel)");
    size_t tot = 0;
    for (int t = 0; t < nstars; t++) {
        if (n[t] < 2 || !r[t] || !rho[t] || !u[t]) return set_err(HC_ERR_ARG, "a profile needs >= 2 points");
        for (int q = 0; q + 1 < n[t]; q++)
            if (!(r[t][q + 1] > r[t][q])) return set_err(HC_ERR_ARG, "profile radii must increase");
        tot += 3 * (size_t)n[t];
    }
    CK(cudaSetDevice(c->dev));
    double *tmp = nullptr;
    if (dmalloc((void **)&tmp, tot * sizeof(double))) return set_err(HC_ERR_NOMEM, "profile tables");
    const bool f64 = c->cfg.precision == HC_FP64;
    cudaError_t e = ic_profile_stars(c->g, c->cfg.gamma, nstars, n, r, rho, u, R_star, centre, vel,
                                     f64 ? c->q64[c->cur] : nullptr, f64 ? nullptr : c->q32[c->cur], tmp, c->s);
    int rc = e == cudaSuccess ? sync_ctx(c) : set_err(HC_ERR_CUDA, "%s", cudaGetErrorString(e));
    cudaFree(tmp);
    c->cfl_valid = 0;
    c->launches += 1;
    return rc;
}
