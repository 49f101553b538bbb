// xts_abi.cu -- the extern "C" entry points of include/xtsrcmaps_b200.h: argument
// checks, host<->device staging, the cached device workspace and error strings.
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "xts_geom.cuh"
#include "xts_internal.cuh"

namespace xts {

static thread_local char g_err[512] = "";
static std::mutex g_mu;  // serialises calls that share the workspace
xts_tuning g_tuning = {0, 0, 0, 0, 0};

int set_error(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

int cuda_error(cudaError_t e, const char* what) {
    int code = (e == cudaErrorMemoryAllocation) ? XTS_ERR_OOM : XTS_ERR_CUDA;
    return set_error(code, "%s: %s", what, cudaGetErrorString(e));
}

constexpr int N_CHUNK_EV = 16;  // source chunks of a pipelined host-mode map

struct Ctx {
    int device = -1;
    cudaStream_t stream = nullptr;
    cudaStream_t copy_stream = nullptr;    // device-to-host copies of finished map chunks
    cudaStream_t geo_stream = nullptr;     // map geometry of the fused call, beside exposure and PSF
    cudaStream_t prio_stream = nullptr;    // exposure and PSF of the fused call, at the highest priority
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
    cudaEvent_t pfork_ev = nullptr, pjoin_ev = nullptr;
    cudaEvent_t pipe_a[2] = {}, pipe_b[2] = {};  // chunk pipeline of the window path
    cudaEvent_t chunk_ev[N_CHUNK_EV] = {};
    void* buf[N_SLOTS] = {};
    size_t cap[N_SLOTS] = {};
};
static Ctx g_ctx;

int ensure_device() {
    if (g_ctx.device >= 0) {
        cudaError_t e = cudaSetDevice(g_ctx.device);
        return e == cudaSuccess ? XTS_OK : cuda_error(e, "cudaSetDevice");
    }
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return set_error(XTS_ERR_NODEV, "no CUDA device visible");
    }
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceProp prop;
    XTS_CUDA(cudaGetDeviceProperties(&prop, dev));
    if (prop.major != 10)
        return set_error(XTS_ERR_NODEV, "device %d is sm_%d%d; this library is built for sm_100a",
                         dev, prop.major, prop.minor);
    XTS_CUDA(cudaSetDevice(dev));
    XTS_CUDA(cudaStreamCreateWithFlags(&g_ctx.stream, cudaStreamNonBlocking));
    if (!g_ctx.copy_stream) XTS_CUDA(cudaStreamCreateWithFlags(&g_ctx.copy_stream, cudaStreamNonBlocking));
    if (!g_ctx.geo_stream) XTS_CUDA(cudaStreamCreateWithFlags(&g_ctx.geo_stream, cudaStreamNonBlocking));
    if (!g_ctx.prio_stream) {
        int least = 0, greatest = 0;
        XTS_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        XTS_CUDA(cudaStreamCreateWithPriority(&g_ctx.prio_stream, cudaStreamNonBlocking, greatest));
    }
    if (!g_ctx.fork_ev) XTS_CUDA(cudaEventCreateWithFlags(&g_ctx.fork_ev, cudaEventDisableTiming));
    if (!g_ctx.join_ev) XTS_CUDA(cudaEventCreateWithFlags(&g_ctx.join_ev, cudaEventDisableTiming));
    if (!g_ctx.pfork_ev) XTS_CUDA(cudaEventCreateWithFlags(&g_ctx.pfork_ev, cudaEventDisableTiming));
    if (!g_ctx.pjoin_ev) XTS_CUDA(cudaEventCreateWithFlags(&g_ctx.pjoin_ev, cudaEventDisableTiming));
    for (int i = 0; i < 2; ++i) {
        if (!g_ctx.pipe_a[i]) XTS_CUDA(cudaEventCreateWithFlags(&g_ctx.pipe_a[i], cudaEventDisableTiming));
        if (!g_ctx.pipe_b[i]) XTS_CUDA(cudaEventCreateWithFlags(&g_ctx.pipe_b[i], cudaEventDisableTiming));
    }
    for (int i = 0; i < N_CHUNK_EV; ++i)
        if (!g_ctx.chunk_ev[i]) XTS_CUDA(cudaEventCreateWithFlags(&g_ctx.chunk_ev[i], cudaEventDisableTiming));
    g_ctx.device = dev;
    return XTS_OK;
}

cudaStream_t default_stream() { return g_ctx.stream; }

void pipe_events(cudaEvent_t a[2], cudaEvent_t b[2]) {
    for (int i = 0; i < 2; ++i) {
        a[i] = g_ctx.pipe_a[i];
        b[i] = g_ctx.pipe_b[i];
    }
}

void* workspace(int slot, size_t bytes) {
    bytes = align_up(bytes ? bytes : 1, 256);
    if (g_ctx.cap[slot] >= bytes) return g_ctx.buf[slot];
    if (g_ctx.buf[slot]) {
        cudaStreamSynchronize(g_ctx.stream);
        cudaDeviceSynchronize();
        cudaFree(g_ctx.buf[slot]);
        g_ctx.buf[slot] = nullptr;
        g_ctx.cap[slot] = 0;
    }
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_error(XTS_ERR_OOM, "cudaMalloc(%zu) for workspace slot %d: %s", bytes, slot,
                  cudaGetErrorString(e));
        return nullptr;
    }
    g_ctx.buf[slot] = p;
    g_ctx.cap[slot] = bytes;
    return p;
}

static void release_all() {
    if (g_ctx.device < 0) return;
    cudaSetDevice(g_ctx.device);
    cudaDeviceSynchronize();
    for (int i = 0; i < N_SLOTS; ++i) {
        if (g_ctx.buf[i]) cudaFree(g_ctx.buf[i]);
        g_ctx.buf[i] = nullptr;
        g_ctx.cap[i] = 0;
    }
}

// Kernel timing -------------------------------------------------------------
struct ProfRec { const char* name; cudaEvent_t a, b; };
static bool g_prof_on = false;
static bool g_prof_keep = false;  // records survive reads (launches captured into a CUDA graph)
static ProfRec g_prof[4096];
static int g_prof_n = 0;
static cudaEvent_t g_prof_pool[8192];
static int g_prof_pool_n = 0, g_prof_pool_used = 0;

static cudaEvent_t prof_event() {
    if (g_prof_pool_used < g_prof_pool_n) return g_prof_pool[g_prof_pool_used++];
    if (g_prof_pool_n >= 8192) return nullptr;
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) { cudaGetLastError(); return nullptr; }
    g_prof_pool[g_prof_pool_n++] = e;
    g_prof_pool_used = g_prof_pool_n;
    return e;
}

// Inside a stream capture the event becomes an event-record node of the graph,
// re-recorded on every replay.
static void prof_record(cudaEvent_t ev, cudaStream_t st) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusActive)
        cudaEventRecordWithFlags(ev, st, cudaEventRecordExternal);
    else
        cudaEventRecord(ev, st);
}

void prof_mark(const char* name, cudaStream_t st, bool begin) {
    if (!g_prof_on) return;
    if (begin) {
        if (g_prof_n >= 4096) return;
        cudaEvent_t a = prof_event(), b = prof_event();
        if (!a || !b) return;
        g_prof[g_prof_n] = {name, a, b};
        prof_record(a, st);
    } else {
        if (g_prof_n >= 4096 || !g_prof[g_prof_n].name) return;
        prof_record(g_prof[g_prof_n].b, st);
        ++g_prof_n;
        if (g_prof_n < 4096) g_prof[g_prof_n].name = nullptr;
    }
}

// Staging helpers ----------------------------------------------------------
struct Stager {
    bool dev;
    cudaStream_t st;
    int next_in = S_IN0, next_out = S_OUT0;
    int rc = XTS_OK;
    struct Pending { void* host; const void* dptr; size_t bytes; };
    Pending pend[8];
    int npend = 0;

    template <typename T>
    const T* in(const T* p, size_t n) {
        if (rc || dev || !p || n == 0) return p;
        if (next_in > S_IN17) { rc = set_error(XTS_ERR_ARG, "too many staged inputs"); return nullptr; }
        void* d = workspace(next_in++, n * sizeof(T));
        if (!d) { rc = XTS_ERR_OOM; return nullptr; }
        cudaError_t e = cudaMemcpyAsync(d, p, n * sizeof(T), cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) { rc = cuda_error(e, "cudaMemcpyAsync H2D"); return nullptr; }
        return (const T*)d;
    }
    template <typename T>
    T* out(T* p, size_t n) {
        if (rc || dev || !p || n == 0) return p;
        if (next_out > S_OUT15 || npend == 8) { rc = set_error(XTS_ERR_ARG, "too many staged outputs"); return nullptr; }
        void* d = workspace(next_out++, n * sizeof(T));
        if (!d) { rc = XTS_ERR_OOM; return nullptr; }
        pend[npend++] = {p, d, n * sizeof(T)};
        return (T*)d;
    }
    // drop a pending copy-out (the caller copies that output itself)
    void unpend(const void* host) {
        for (int i = 0; i < npend; ++i)
            if (pend[i].host == host) {
                for (int j = i + 1; j < npend; ++j) pend[j - 1] = pend[j];
                --npend;
                return;
            }
    }
    // scratch output the caller did not ask for
    template <typename T>
    T* scratch(size_t n) {
        if (rc) return nullptr;
        if (next_out > S_OUT15) { rc = set_error(XTS_ERR_ARG, "too many staged outputs"); return nullptr; }
        void* d = workspace(next_out++, n * sizeof(T));
        if (!d) rc = XTS_ERR_OOM;
        return (T*)d;
    }
    int finish(int launch_rc) {
        if (rc) return rc;
        if (launch_rc) return launch_rc;
        if (dev) return XTS_OK;
        for (int i = 0; i < npend; ++i) {
            cudaError_t e = cudaMemcpyAsync(pend[i].host, pend[i].dptr, pend[i].bytes,
                                            cudaMemcpyDeviceToHost, st);
            if (e != cudaSuccess) return cuda_error(e, "cudaMemcpyAsync D2H");
        }
        XTS_CUDA(cudaStreamSynchronize(st));
        return XTS_OK;
    }
};

// Pipelined copy-out of a host-mode model map: each finished chunk of sources
// gets an event on the compute stream; once every chunk is launched, the copy
// stream waits for each event in turn and copies that chunk (copies into
// pageable memory block the calling thread, so they are issued only after all
// kernels are queued).
struct ChunkCopy {
    char* host = nullptr;
    const char* dev = nullptr;
    size_t bytes_per_source = 0;
    int n = 0;
    int s0[N_CHUNK_EV], ns[N_CHUNK_EV];
    int issue(cudaStream_t st) {
        for (int i = 0; i < n; ++i) {
            XTS_CUDA(cudaStreamWaitEvent(g_ctx.copy_stream, g_ctx.chunk_ev[i], 0));
            const size_t off = (size_t)s0[i] * bytes_per_source;
            XTS_CUDA(cudaMemcpyAsync(host + off, dev + off, (size_t)ns[i] * bytes_per_source,
                                     cudaMemcpyDeviceToHost, g_ctx.copy_stream));
        }
        return XTS_OK;
    }
};

static int chunk_done(void* ctx, int s0, int n, cudaStream_t st) {
    ChunkCopy* c = (ChunkCopy*)ctx;
    if (c->n > 0 && c->n == N_CHUNK_EV) {  // merge into the last chunk (its event is re-recorded)
        c->ns[c->n - 1] = s0 + n - c->s0[c->n - 1];
        XTS_CUDA(cudaEventRecord(g_ctx.chunk_ev[c->n - 1], st));
        return XTS_OK;
    }
    c->s0[c->n] = s0;
    c->ns[c->n] = n;
    XTS_CUDA(cudaEventRecord(g_ctx.chunk_ev[c->n], st));
    c->n++;
    return XTS_OK;
}

static int srcmap_kernel(unsigned flags) {
    return (flags & XTS_TCGEN05) ? SRCMAP_TCGEN05 : (flags & XTS_CUDA_CORES) ? SRCMAP_ONEPASS : SRCMAP_WINDOWS;
}

// The model-map step with its outputs staged by sg.  In host mode the map is
// copied out by source chunks on the copy stream while later chunks are
// computed (window path); the other outputs are copied at the end.
static int run_srcmap(Stager& sg, SrcmapDev& a, void* model_map, size_t npix, bool f64) {
    const int S = a.S, E = a.E;
    ChunkCopy cc;
    if (!sg.dev && !sg.rc && S > 0 && npix * E > 0) {
        cc.host = (char*)model_map;
        cc.dev = (const char*)a.out;
        cc.bytes_per_source = npix * E * (f64 ? 8 : 4);
        sg.unpend(model_map);  // the map is not in the final copy list
        a.chunk_sources = (S + 7) / 8;  // about 8 chunks (at most N_CHUNK_EV events are used)
        a.on_chunk = chunk_done;
        a.on_chunk_ctx = &cc;
    }
    int rc = sg.rc ? sg.rc : launch_srcmap(a, sg.st);
    if (cc.host && rc == XTS_OK) {
        if (cc.n == 0) rc = chunk_done(&cc, 0, S, sg.st);  // path without chunk hooks: one chunk
        if (rc == XTS_OK) rc = cc.issue(sg.st);
    }
    rc = sg.finish(rc);
    if (cc.host && cc.n) {
        cudaError_t e = cudaStreamSynchronize(g_ctx.copy_stream);
        if (rc == XTS_OK && e != cudaSuccess) rc = cuda_error(e, "map copy-out");
    }
    if (rc == XTS_OK && !sg.dev && S > 0) rc = srcmap_status(sg.st);
    return rc;
}

static bool grid_ok(const xts_grid* g, int n_par) {
    return g && g->cosths && g->logEs && g->params && g->n_cos >= 2 && g->n_e >= 2 &&
           g->n_par == n_par;
}

static xts_grid stage_grid(Stager& sg, const xts_grid* g) {
    xts_grid d = *g;
    d.cosths = sg.in(g->cosths, (size_t)g->n_cos);
    d.logEs = sg.in(g->logEs, (size_t)g->n_e);
    d.params = sg.in(g->params, (size_t)g->n_cos * g->n_e * g->n_par);
    return d;
}

// Host mode: the per-source path needs only the livetime rows at the sources'
// NESTED pixels, so those rows are gathered on the host (pixels computed on the
// device from the staged positions) and only they are uploaded, instead of the
// whole cubes ([12 nside^2, C] floats each).  Device mode uploads nothing and
// reads the cubes in place.  The gathered rows must outlive the call's copies.
struct CubeRows {
    std::vector<float> x, w;
};
static void stage_cubes(Stager& sg, const xts_expcube* cube, const xts_expcube* wcube, const double* src_d, int S,
                        ExposureDev& ea, CubeRows& rows) {
    const int C = cube->nbrbins;
    const long long nhp = 12LL * cube->nside * cube->nside;
    if (sg.dev || S <= 0 || sg.rc) {
        ea.cube = sg.in(cube->cosbins, (size_t)nhp * C);
        ea.wcube = sg.in(wcube->cosbins, (size_t)nhp * C);
        return;
    }
    long long* pix_d = (long long*)workspace(W_SRCPIX, sizeof(long long) * (size_t)S);
    if (!pix_d) { sg.rc = XTS_ERR_OOM; return; }
    std::vector<long long> pix((size_t)S);
    int rc = launch_src_pixels(src_d, S, cube->nside, pix_d, sg.st);
    if (rc) { sg.rc = rc; return; }
    cudaError_t e = cudaMemcpyAsync(pix.data(), pix_d, sizeof(long long) * (size_t)S, cudaMemcpyDeviceToHost, sg.st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(sg.st);
    if (e != cudaSuccess) { sg.rc = cuda_error(e, "source pixels"); return; }
    rows.x.assign((size_t)S * C, NAN);
    rows.w.assign((size_t)S * C, NAN);
    for (int s = 0; s < S; ++s)
        if (pix[s] >= 0 && pix[s] < nhp) {
            memcpy(&rows.x[(size_t)s * C], cube->cosbins + (size_t)pix[s] * C, sizeof(float) * C);
            memcpy(&rows.w[(size_t)s * C], wcube->cosbins + (size_t)pix[s] * C, sizeof(float) * C);
        }
    ea.cube = sg.in(rows.x.data(), (size_t)S * C);
    ea.wcube = sg.in(rows.w.data(), (size_t)S * C);
    ea.gathered = true;
}

}  // namespace xts

using namespace xts;

#define XTS_ENTER()                                        \
    std::lock_guard<std::mutex> lock__(g_mu);              \
    do {                                                   \
        int rc__ = ensure_device();                        \
        if (rc__) return rc__;                             \
    } while (0)

extern "C" {

int xts_version(void) { return 100; }

const char* xts_last_error(void) { return g_err; }

int xts_init(int device) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (g_ctx.device >= 0 && g_ctx.device != device) release_all();
    if (g_ctx.device == device) return XTS_OK;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
        cudaGetLastError();
        return set_error(XTS_ERR_NODEV, "device %d not available (%d visible)", device, n);
    }
    XTS_CUDA(cudaSetDevice(device));
    g_ctx.device = -1;
    if (g_ctx.stream) { cudaStreamDestroy(g_ctx.stream); g_ctx.stream = nullptr; }
    if (g_ctx.copy_stream) { cudaStreamDestroy(g_ctx.copy_stream); g_ctx.copy_stream = nullptr; }
    if (g_ctx.geo_stream) { cudaStreamDestroy(g_ctx.geo_stream); g_ctx.geo_stream = nullptr; }
    if (g_ctx.prio_stream) { cudaStreamDestroy(g_ctx.prio_stream); g_ctx.prio_stream = nullptr; }
    if (g_ctx.fork_ev) { cudaEventDestroy(g_ctx.fork_ev); g_ctx.fork_ev = nullptr; }
    if (g_ctx.join_ev) { cudaEventDestroy(g_ctx.join_ev); g_ctx.join_ev = nullptr; }
    if (g_ctx.pfork_ev) { cudaEventDestroy(g_ctx.pfork_ev); g_ctx.pfork_ev = nullptr; }
    if (g_ctx.pjoin_ev) { cudaEventDestroy(g_ctx.pjoin_ev); g_ctx.pjoin_ev = nullptr; }
    for (int i = 0; i < 2; ++i) {
        if (g_ctx.pipe_a[i]) { cudaEventDestroy(g_ctx.pipe_a[i]); g_ctx.pipe_a[i] = nullptr; }
        if (g_ctx.pipe_b[i]) { cudaEventDestroy(g_ctx.pipe_b[i]); g_ctx.pipe_b[i] = nullptr; }
    }
    for (int i = 0; i < N_CHUNK_EV; ++i)
        if (g_ctx.chunk_ev[i]) { cudaEventDestroy(g_ctx.chunk_ev[i]); g_ctx.chunk_ev[i] = nullptr; }
    return ensure_device();
}

void xts_release(void) {
    std::lock_guard<std::mutex> lock(g_mu);
    release_all();
}

int xts_profile_enable(int on) {
    std::lock_guard<std::mutex> lock(g_mu);
    g_prof_on = on != 0;
    g_prof_keep = on == 2;
    g_prof_n = 0;
    g_prof_pool_used = 0;
    g_prof[0].name = nullptr;
    return XTS_OK;
}

int xts_profile_read(char* buf, int buflen) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!buf || buflen < 3) return set_error(XTS_ERR_ARG, "profile_read: buffer too small");
    const char* names[64];
    int counts[64];
    double ms[64];
    int nk = 0;
    for (int i = 0; i < g_prof_n; ++i) {
        cudaError_t e = cudaEventSynchronize(g_prof[i].b);
        if (e != cudaSuccess) return cuda_error(e, "cudaEventSynchronize");
        float t = 0.f;
        cudaEventElapsedTime(&t, g_prof[i].a, g_prof[i].b);
        int k = 0;
        while (k < nk && strcmp(names[k], g_prof[i].name) != 0) ++k;
        if (k == nk) {
            if (nk == 64) continue;
            names[nk] = g_prof[i].name; counts[nk] = 0; ms[nk] = 0.; ++nk;
        }
        counts[k] += 1;
        ms[k] += t;
    }
    int len = snprintf(buf, buflen, "{");
    for (int k = 0; k < nk && len < buflen; ++k)
        len += snprintf(buf + len, buflen - len, "%s\"%s\": [%d, %.6f]", k ? ", " : "", names[k],
                        counts[k], ms[k]);
    if (len < buflen) len += snprintf(buf + len, buflen - len, "}");
    if (!g_prof_keep) {
        g_prof_n = 0;
        g_prof_pool_used = 0;
        g_prof[0].name = nullptr;
    }
    return len < buflen ? len : set_error(XTS_ERR_ARG, "profile_read: buffer too small");
}

int xts_livetime_efficiency_factors(const double* logEs, int E, const float* p0, const float* p1,
                                    double* ltf, unsigned flags, void* stream) {
    XTS_ENTER();
    if (E <= 0 || !logEs || !p0 || !p1 || !ltf)
        return set_error(XTS_ERR_ARG, "livetime_efficiency_factors: bad arguments");
    Stager sg{(flags & XTS_DEVICE_PTRS) != 0, stream ? (cudaStream_t)stream : g_ctx.stream};
    const double* d_loge = sg.in(logEs, (size_t)E);
    const float* d_p0 = sg.in(p0, 6);
    const float* d_p1 = sg.in(p1, 6);
    double* d_out = sg.out(ltf, (size_t)2 * E);
    int rc = sg.rc ? sg.rc : launch_ltf(d_loge, E, d_p0, d_p1, d_out, sg.st);
    return sg.finish(rc);
}

int xts_normalize_rpsf(double* params, int Mc, int Me, const double* grid_logEs, float scale0,
                       float scale1, float scale_index, unsigned flags, void* stream) {
    XTS_ENTER();
    if (!params || !grid_logEs || Mc <= 0 || Me <= 0)
        return set_error(XTS_ERR_ARG, "normalize_rpsf: bad arguments");
    Stager sg{(flags & XTS_DEVICE_PTRS) != 0, stream ? (cudaStream_t)stream : g_ctx.stream};
    size_t n = (size_t)Mc * Me * 6;
    double* d_par = const_cast<double*>(sg.in((const double*)params, n));
    const double* d_glog = sg.in(grid_logEs, (size_t)Me);
    if (!sg.dev && !sg.rc) sg.pend[sg.npend++] = {params, d_par, n * sizeof(double)};
    int rc = sg.rc ? sg.rc
                   : launch_normalize_rpsf(d_par, Mc, Me, d_glog, scale0, scale1, scale_index, sg.st);
    return sg.finish(rc);
}

int xts_compute_exposure(const xts_expcube* cube, const xts_expcube* wcube, const double* logEs,
                         int E, const double* src_sph, int S, const xts_grid* aeff_front,
                         const xts_grid* aeff_back, const double* front_ltf,
                         const xts_exposure_out* out, unsigned flags, void* stream) {
    XTS_ENTER();
    if (!cube || !wcube || !cube->cosbins || !wcube->cosbins || !logEs || E <= 0 || S < 0 ||
        (S > 0 && !src_sph) || !front_ltf || !out)
        return set_error(XTS_ERR_ARG, "compute_exposure: null argument or bad size");
    if (cube->nside <= 0 || (cube->nside & (cube->nside - 1)) || cube->nbrbins <= 0 ||
        wcube->nside != cube->nside || wcube->nbrbins != cube->nbrbins)
        return set_error(XTS_ERR_ARG, "compute_exposure: livetime cubes need a power-of-two nside and equal shapes");
    if (!grid_ok(aeff_front, 1) || !grid_ok(aeff_back, 1))
        return set_error(XTS_ERR_ARG, "compute_exposure: effective-area grids need n_par == 1");
    int C = cube->nbrbins;
    Stager sg{(flags & XTS_DEVICE_PTRS) != 0, stream ? (cudaStream_t)stream : g_ctx.stream};
    ExposureDev a;
    a.src_sph = sg.in(src_sph, (size_t)2 * S); a.S = S;
    CubeRows rows;
    stage_cubes(sg, cube, wcube, a.src_sph, S, a, rows);
    a.nside = cube->nside; a.C = C; a.cosmin = cube->cosmin; a.thetabin = cube->thetabin;
    a.logEs = sg.in(logEs, (size_t)E); a.E = E;
    a.af = stage_grid(sg, aeff_front);
    a.ab = stage_grid(sg, aeff_back);
    a.ltf = sg.in(front_ltf, (size_t)2 * E);
    a.exp_costhetas = out->exp_costhetas ? sg.out(out->exp_costhetas, (size_t)C) : sg.scratch<double>(C);
    a.front_aeff = out->front_aeff ? sg.out(out->front_aeff, (size_t)C * E) : sg.scratch<double>((size_t)C * E);
    a.back_aeff = out->back_aeff ? sg.out(out->back_aeff, (size_t)C * E) : sg.scratch<double>((size_t)C * E);
    a.ecb = out->src_exposure_cosbins ? sg.out(out->src_exposure_cosbins, (size_t)S * C) : sg.scratch<double>((size_t)S * C);
    a.wecb = out->src_weighted_exposure_cosbins ? sg.out(out->src_weighted_exposure_cosbins, (size_t)S * C) : sg.scratch<double>((size_t)S * C);
    a.exposure = out->exposure ? sg.out(out->exposure, (size_t)S * E) : sg.scratch<double>((size_t)S * E);
    int rc = sg.rc ? sg.rc : launch_exposure(a, sg.st);
    return sg.finish(rc);
}

int xts_exposure_contract(const double* ecb, const double* wecb, int S, int C, const double* af,
                          const double* ab, const double* ltf, int E, double* exposure,
                          unsigned flags, void* stream) {
    XTS_ENTER();
    if (S < 0 || C <= 0 || E <= 0 || !af || !ab || !ltf || (S > 0 && (!ecb || !wecb || !exposure)))
        return set_error(XTS_ERR_ARG, "exposure_contract: null argument or bad size");
    Stager sg{(flags & XTS_DEVICE_PTRS) != 0, stream ? (cudaStream_t)stream : g_ctx.stream};
    const double* d_ecb = sg.in(ecb, (size_t)S * C);
    const double* d_wecb = sg.in(wecb, (size_t)S * C);
    const double* d_af = sg.in(af, (size_t)C * E);
    const double* d_ab = sg.in(ab, (size_t)C * E);
    const double* d_ltf = sg.in(ltf, (size_t)2 * E);
    double* d_out = sg.out(exposure, (size_t)S * E);
    int rc = sg.rc ? sg.rc
                   : launch_exposure_contract(d_ecb, d_wecb, S, C, d_af, d_ab, d_ltf, E, d_out,
                                              sg.st);
    return sg.finish(rc);
}

int xts_compute_psf_data(const xts_grid* psf_front, const xts_grid* psf_back,
                         const double* exp_costhetas, int C, const double* logEs, int E,
                         const double* front_aeff, const double* back_aeff, const double* ecb,
                         const double* wecb, int S, const double* front_ltf,
                         const double* exposure, double* upsf, double* partial, unsigned flags,
                         void* stream) {
    XTS_ENTER();
    if (!grid_ok(psf_front, 6) || !grid_ok(psf_back, 6))
        return set_error(XTS_ERR_ARG, "compute_psf_data: King grids need n_par == 6");
    if (!exp_costhetas || C <= 0 || !logEs || E <= 0 || !front_aeff || !back_aeff || S < 0 ||
        (S > 0 && (!ecb || !wecb || !exposure || !upsf || !partial)) || !front_ltf)
        return set_error(XTS_ERR_ARG, "compute_psf_data: null argument or bad size");
    Stager sg{(flags & XTS_DEVICE_PTRS) != 0, stream ? (cudaStream_t)stream : g_ctx.stream};
    PsfDev a;
    a.pf = stage_grid(sg, psf_front);
    a.pb = stage_grid(sg, psf_back);
    a.costh = sg.in(exp_costhetas, (size_t)C); a.C = C;
    a.logEs = sg.in(logEs, (size_t)E); a.E = E;
    a.af = sg.in(front_aeff, (size_t)C * E);
    a.ab = sg.in(back_aeff, (size_t)C * E);
    a.ecb = sg.in(ecb, (size_t)S * C);
    a.wecb = sg.in(wecb, (size_t)S * C); a.S = S;
    a.ltf = sg.in(front_ltf, (size_t)2 * E);
    a.exposure = sg.in(exposure, (size_t)S * E);
    a.upsf = sg.out(upsf, (size_t)S * ND * E);
    a.partial = sg.out(partial, (size_t)S * ND * E);
    int rc = sg.rc ? sg.rc : launch_psf(a, sg.st);
    return sg.finish(rc);
}

int xts_point_src_model_map_wcs(const xts_wcs* wcs, const double* src_sph, int S,
                                const double* exposure, const double* upsf, const double* partial,
                                int E, void* model_map, xts_srcmap_info* info, unsigned flags,
                                void* stream) {
    XTS_ENTER();
    if (!wcs || wcs->naxis1 <= 0 || wcs->naxis2 <= 0 || (wcs->proj != 0 && wcs->proj != 1) ||
        wcs->cdelt1 == 0. || wcs->cdelt2 == 0.)
        return set_error(XTS_ERR_ARG, "point_src_model_map_wcs: bad WCS (CAR/AIT, nonzero CDELT)");
    if (S < 0 || E <= 0 || (S > 0 && (!src_sph || !exposure || !upsf || !partial || !model_map)))
        return set_error(XTS_ERR_ARG, "point_src_model_map_wcs: null argument or bad size");
    if ((long long)wcs->naxis1 * wcs->naxis2 > (1LL << 31) - 1 || S > 65535)
        return set_error(XTS_ERR_ARG, "point_src_model_map_wcs: map or source count too large");
    bool f64 = (flags & XTS_OUT_F64) != 0;
    size_t npix = (size_t)wcs->naxis1 * wcs->naxis2;
    // the FP32 write passes store with TMA bulk copies, which need a 16-byte aligned base
    if ((flags & XTS_DEVICE_PTRS) && !f64 && ((uintptr_t)model_map & 15))
        return set_error(XTS_ERR_ARG, "point_src_model_map_wcs: device model_map must be 16-byte aligned");
    Stager sg{(flags & XTS_DEVICE_PTRS) != 0, stream ? (cudaStream_t)stream : g_ctx.stream};
    SrcmapDev a;
    a.wcs = *wcs;
    a.src_sph = sg.in(src_sph, (size_t)2 * S); a.S = S;
    a.exposure = sg.in(exposure, (size_t)S * E);
    a.upsf = sg.in(upsf, (size_t)S * ND * E);
    a.partial = sg.in(partial, (size_t)S * ND * E); a.E = E;
    a.out_f64 = f64;
    a.out = f64 ? (void*)sg.out((double*)model_map, (size_t)S * npix * E)
                : (void*)sg.out((float*)model_map, (size_t)S * npix * E);
    a.inv_integ = info ? sg.out(info->inv_map_integral, (size_t)S * E) : nullptr;
    a.correction = info ? sg.out(info->correction, (size_t)S * E) : nullptr;
    a.radius = info ? sg.out(info->psf_radius, (size_t)S) : nullptr;
    a.in_fov = info ? sg.out(info->in_fov, (size_t)S) : nullptr;
    a.kernel = srcmap_kernel(flags);
    // the map geometry and the window passes on the geometry stream (forked here,
    // after the inputs are staged), so the chunks of the window path pipeline
    if (sg.rc == XTS_OK && S > 0) {
        XTS_CUDA(cudaEventRecord(g_ctx.fork_ev, sg.st));
        XTS_CUDA(cudaStreamWaitEvent(g_ctx.geo_stream, g_ctx.fork_ev, 0));
        a.geo_stream = g_ctx.geo_stream;
        a.join_ev = g_ctx.join_ev;
    }
    return run_srcmap(sg, a, model_map, npix, f64);
}

int xts_exposure_map(const xts_expcube* cube, const xts_expcube* wcube, const double* logEs, int E,
                     const xts_grid* aeff_front, const xts_grid* aeff_back, const double* front_ltf,
                     double* exposure_map, unsigned flags, void* stream) {
    XTS_ENTER();
    if (!cube || !wcube || !cube->cosbins || !wcube->cosbins || !logEs || E <= 0 || !front_ltf || !exposure_map)
        return set_error(XTS_ERR_ARG, "exposure_map: null argument or bad size");
    if (cube->nside <= 0 || (cube->nside & (cube->nside - 1)) || cube->nbrbins <= 0 ||
        wcube->nside != cube->nside || wcube->nbrbins != cube->nbrbins)
        return set_error(XTS_ERR_ARG, "exposure_map: livetime cubes need a power-of-two nside and equal shapes");
    if (!grid_ok(aeff_front, 1) || !grid_ok(aeff_back, 1))
        return set_error(XTS_ERR_ARG, "exposure_map: effective-area grids need n_par == 1");
    const int C = cube->nbrbins;
    if (!exposure_map_supported(C, E))
        return set_error(XTS_ERR_ARG, "exposure_map: needs nbrbins <= 64 and a multiple of 4, E <= 256");
    const long long npix = 12LL * cube->nside * cube->nside;
    Stager sg{(flags & XTS_DEVICE_PTRS) != 0, stream ? (cudaStream_t)stream : g_ctx.stream};
    ExposureDev ea;
    ea.cube = sg.in(cube->cosbins, (size_t)npix * C);
    ea.wcube = sg.in(wcube->cosbins, (size_t)npix * C);
    ea.nside = cube->nside; ea.C = C; ea.cosmin = cube->cosmin; ea.thetabin = cube->thetabin;
    ea.logEs = sg.in(logEs, (size_t)E); ea.E = E;
    ea.src_sph = nullptr; ea.S = 0;
    ea.af = stage_grid(sg, aeff_front);
    ea.ab = stage_grid(sg, aeff_back);
    ea.ltf = sg.in(front_ltf, (size_t)2 * E);
    ea.exp_costhetas = sg.scratch<double>(C);
    ea.front_aeff = sg.scratch<double>((size_t)C * E);
    ea.back_aeff = sg.scratch<double>((size_t)C * E);
    ea.ecb = ea.wecb = ea.exposure = nullptr;
    double* out = sg.out(exposure_map, (size_t)npix * E);
    int* status = (int*)workspace(W_MISC, 64);
    int rc = sg.rc ? sg.rc : (status ? XTS_OK : XTS_ERR_OOM);
    if (rc == XTS_OK) {
        cudaError_t e = cudaMemsetAsync(status, 0, sizeof(int), sg.st);
        if (e != cudaSuccess) rc = cuda_error(e, "cudaMemsetAsync");
    }
    if (rc == XTS_OK) rc = launch_exposure(ea, sg.st);  // cos-theta bins and effective-area tables
    if (rc == XTS_OK)
        rc = launch_exposure_map_tc(ea.cube, ea.wcube, npix, C, ea.front_aeff, ea.back_aeff, ea.ltf, E, out, status,
                                    sg.st);
    rc = sg.finish(rc);
    if (rc == XTS_OK && !sg.dev) rc = srcmap_status(sg.st);
    return rc;
}

int xts_point_src_model_map_wcs_adaptive(const xts_wcs* wcs, const double* src_sph, int S,
                                         const double* exposure, const double* upsf,
                                         const double* partial, int E, double rtol, int max_depth,
                                         float* model_map, xts_srcmap_info* info, unsigned flags,
                                         void* stream) {
    XTS_ENTER();
    if (!wcs || wcs->naxis1 <= 0 || wcs->naxis2 <= 0 || (wcs->proj != 0 && wcs->proj != 1) ||
        wcs->cdelt1 == 0. || wcs->cdelt2 == 0.)
        return set_error(XTS_ERR_ARG, "point_src_model_map_wcs_adaptive: bad WCS (CAR/AIT, nonzero CDELT)");
    if (S < 0 || E <= 0 || E > 256 || (S > 0 && (!src_sph || !exposure || !upsf || !partial || !model_map)))
        return set_error(XTS_ERR_ARG, "point_src_model_map_wcs_adaptive: null argument or bad size (E <= 256)");
    if (!(rtol >= 1e-6 && rtol <= 1.0) || max_depth < 0 || max_depth > 16)
        return set_error(XTS_ERR_ARG, "point_src_model_map_wcs_adaptive: rtol must lie in [1e-6, 1] and "
                                      "max_depth in [0, 16]");
    if ((long long)wcs->naxis1 * wcs->naxis2 * E > 0xffffffffLL || S > 65535)
        return set_error(XTS_ERR_ARG, "point_src_model_map_wcs_adaptive: map or source count too large");
    if (flags & ~(unsigned)XTS_DEVICE_PTRS)
        return set_error(XTS_ERR_ARG, "point_src_model_map_wcs_adaptive: only XTS_DEVICE_PTRS applies");
    const size_t npix = (size_t)wcs->naxis1 * wcs->naxis2;
    Stager sg{(flags & XTS_DEVICE_PTRS) != 0, stream ? (cudaStream_t)stream : g_ctx.stream};
    SrcmapDev a;
    a.wcs = *wcs;
    a.src_sph = sg.in(src_sph, (size_t)2 * S); a.S = S;
    a.exposure = sg.in(exposure, (size_t)S * E);
    a.upsf = sg.in(upsf, (size_t)S * ND * E);
    a.partial = sg.in(partial, (size_t)S * ND * E); a.E = E;
    a.out_f64 = false;
    a.out = sg.out(model_map, (size_t)S * npix * E);
    a.inv_integ = info ? sg.out(info->inv_map_integral, (size_t)S * E) : nullptr;
    a.correction = info ? sg.out(info->correction, (size_t)S * E) : nullptr;
    a.radius = info ? sg.out(info->psf_radius, (size_t)S) : nullptr;
    a.in_fov = info ? sg.out(info->in_fov, (size_t)S) : nullptr;
    a.kernel = SRCMAP_WINDOWS;
    a.adaptive = true;
    a.rtol = rtol;
    a.max_depth = max_depth;
    return run_srcmap(sg, a, model_map, npix, false);
}

// ------------------------------------------------------------------ surrogate network
static int mlp_ok(const xts_mlp* net, const char* who) {
    if (!net || !net->params || !net->wbf16) return set_error(XTS_ERR_ARG, "%s: network parameters missing", who);
    for (int k = 0; k < XTS_MLP_IN; ++k)
        if (!(net->in_sd[k] > 0.f) || !std::isfinite(net->in_mu[k]))
            return set_error(XTS_ERR_ARG, "%s: feature standardisation %d must be finite with sd > 0", who, k);
    if (!(net->out_sd > 0.f) || !std::isfinite(net->out_mu))
        return set_error(XTS_ERR_ARG, "%s: target standardisation must be finite with sd > 0", who);
    return XTS_OK;
}

static int* mlp_status_word(cudaStream_t st) {
    int* status = (int*)workspace(W_MLP_ST, 64);
    if (status && cudaMemsetAsync(status, 0, sizeof(int), st) != cudaSuccess) return nullptr;
    return status;
}

int xts_gemm_bf16(const unsigned short* A, int a_trans, const unsigned short* B, int b_trans, int M, int K,
                  float* C, int c_trans, int accumulate, void* stream) {
    XTS_ENTER();
    if (!A || !B || !C) return set_error(XTS_ERR_ARG, "gemm_bf16: null operand");
    cudaStream_t st = stream ? (cudaStream_t)stream : g_ctx.stream;
    int* status = mlp_status_word(st);
    if (!status) return XTS_ERR_OOM;
    int rc = launch_gemm_bf16(A, a_trans, B, b_trans, M, K, C, c_trans, accumulate, status, st);
    if (rc) return rc;
    return mlp_check_status(status, st);
}

int xts_mlp_forward(const xts_mlp* net, const float* X, long long n, float* y, void* stream) {
    XTS_ENTER();
    int rc = mlp_ok(net, "mlp_forward");
    if (rc) return rc;
    if (n < 0 || (n > 0 && (!X || !y))) return set_error(XTS_ERR_ARG, "mlp_forward: null argument or n < 0");
    cudaStream_t st = stream ? (cudaStream_t)stream : g_ctx.stream;
    int* status = mlp_status_word(st);
    if (!status) return XTS_ERR_OOM;
    if ((rc = launch_mlp_forward(net, X, n, y, status, st))) return rc;
    return mlp_check_status(status, st);
}

int xts_mlp_grads(const xts_mlp* net, const float* X, const float* Y, long long n, float* grads, float* loss,
                  void* stream) {
    XTS_ENTER();
    int rc = mlp_ok(net, "mlp_grads");
    if (rc) return rc;
    if (!X || !Y || !grads) return set_error(XTS_ERR_ARG, "mlp_grads: null argument");
    cudaStream_t st = stream ? (cudaStream_t)stream : g_ctx.stream;
    int* status = mlp_status_word(st);
    if (!status) return XTS_ERR_OOM;
    return launch_mlp_grads(net, X, Y, n, grads, loss, status, st);
}

int xts_mlp_train_step(const xts_mlp* net, const float* X, const float* Y, long long n, float* grads,
                       float* adam_m, float* adam_v, int step, float lr, float* loss, void* stream) {
    XTS_ENTER();
    int rc = mlp_ok(net, "mlp_train_step");
    if (rc) return rc;
    if (!X || !Y || !grads || !adam_m || !adam_v) return set_error(XTS_ERR_ARG, "mlp_train_step: null argument");
    if (!(lr > 0.f) || !std::isfinite(lr)) return set_error(XTS_ERR_ARG, "mlp_train_step: lr must be > 0");
    cudaStream_t st = stream ? (cudaStream_t)stream : g_ctx.stream;
    int* status = mlp_status_word(st);
    if (!status) return XTS_ERR_OOM;
    if ((rc = launch_mlp_train_step(net, X, Y, n, grads, adam_m, adam_v, step, lr, loss, status, st))) return rc;
    return mlp_check_status(status, st);
}

int xts_surrogate_samples(const double* upsf, const double* logEs, int S, int E, long long n,
                          unsigned long long seed, double rho_min, float* X, float* Y, void* stream) {
    XTS_ENTER();
    if (n > 0 && (!upsf || !logEs || !X || !Y)) return set_error(XTS_ERR_ARG, "surrogate_samples: null argument");
    cudaStream_t st = stream ? (cudaStream_t)stream : g_ctx.stream;
    int rc = launch_surrogate_samples(upsf, logEs, S, E, n, seed, rho_min, X, Y, st);
    if (rc) return rc;
    XTS_CUDA(cudaStreamSynchronize(st));
    return XTS_OK;
}

int xts_point_src_model_map_wcs_surrogate(const xts_wcs* wcs, const double* src_sph, int S,
                                          const double* exposure, const double* upsf,
                                          const double* partial, const double* logEs, int E,
                                          const xts_mlp* net, double check_tol, float* model_map,
                                          xts_srcmap_info* info, xts_surrogate_stats* stats, void* stream) {
    XTS_ENTER();
    int rc = mlp_ok(net, "point_src_model_map_wcs_surrogate");
    if (rc) return rc;
    if (!wcs || wcs->naxis1 <= 0 || wcs->naxis2 <= 0 || (wcs->proj != 0 && wcs->proj != 1) ||
        wcs->cdelt1 == 0. || wcs->cdelt2 == 0.)
        return set_error(XTS_ERR_ARG, "point_src_model_map_wcs_surrogate: bad WCS (CAR/AIT, nonzero CDELT)");
    if (S < 0 || E <= 0 || E > 256 ||
        (S > 0 && (!src_sph || !exposure || !upsf || !partial || !logEs || !model_map)))
        return set_error(XTS_ERR_ARG, "point_src_model_map_wcs_surrogate: null argument or bad size (E <= 256)");
    if ((long long)wcs->naxis1 * wcs->naxis2 * E > 0xffffffffLL || S > 65535)
        return set_error(XTS_ERR_ARG, "point_src_model_map_wcs_surrogate: map or source count too large");
    if (!(check_tol > 0.)) return set_error(XTS_ERR_ARG, "point_src_model_map_wcs_surrogate: check_tol must be > 0");
    const size_t npix = (size_t)wcs->naxis1 * wcs->naxis2;
    Stager sg{true, stream ? (cudaStream_t)stream : g_ctx.stream};
    SrcmapDev a;
    a.wcs = *wcs;
    a.src_sph = src_sph; a.S = S;
    a.exposure = exposure;
    a.upsf = upsf;
    a.partial = partial; a.E = E;
    a.out_f64 = false;
    a.out = model_map;
    a.inv_integ = info ? info->inv_map_integral : nullptr;
    a.correction = info ? info->correction : nullptr;
    a.radius = info ? info->psf_radius : nullptr;
    a.in_fov = info ? info->in_fov : nullptr;
    a.kernel = SRCMAP_WINDOWS;
    a.surrogate = net;
    a.logEs = logEs;
    a.check_tol = check_tol;
    a.sur_stats = stats;
    if (stats) memset(stats, 0, sizeof(*stats));
    return run_srcmap(sg, a, model_map, npix, false);
}

int xts_surrogate_last_stats(xts_surrogate_stats* stats, void* stream) {
    XTS_ENTER();
    return surrogate_last_stats(stats, stream ? (cudaStream_t)stream : g_ctx.stream);
}

// The fused exposure -> mean PSF -> model map call; with net, the surrogate's map.
static int fused_maps(const xts_expcube* cube, const xts_expcube* wcube, const double* logEs,
                      int E, const double* src_sph, int S, const xts_grid* aeff_front,
                      const xts_grid* aeff_back, const xts_grid* psf_front,
                      const xts_grid* psf_back, const double* front_ltf, const xts_wcs* wcs,
                      void* model_map, xts_srcmap_info* info, unsigned flags, void* stream,
                      const xts_mlp* net, double check_tol, xts_surrogate_stats* stats) {
    if (!cube || !wcube || !cube->cosbins || !wcube->cosbins || !logEs || E <= 0 || S < 0 ||
        (S > 0 && (!src_sph || !model_map)) || !front_ltf)
        return set_error(XTS_ERR_ARG, "point_source_maps: null argument or bad size");
    if (cube->nside <= 0 || (cube->nside & (cube->nside - 1)) || cube->nbrbins <= 0 ||
        wcube->nside != cube->nside || wcube->nbrbins != cube->nbrbins)
        return set_error(XTS_ERR_ARG, "point_source_maps: livetime cubes need a power-of-two nside and equal shapes");
    if (!grid_ok(aeff_front, 1) || !grid_ok(aeff_back, 1))
        return set_error(XTS_ERR_ARG, "point_source_maps: effective-area grids need n_par == 1");
    if (!grid_ok(psf_front, 6) || !grid_ok(psf_back, 6))
        return set_error(XTS_ERR_ARG, "point_source_maps: King grids need n_par == 6");
    if (!wcs || wcs->naxis1 <= 0 || wcs->naxis2 <= 0 || (wcs->proj != 0 && wcs->proj != 1) ||
        wcs->cdelt1 == 0. || wcs->cdelt2 == 0.)
        return set_error(XTS_ERR_ARG, "point_source_maps: bad WCS (CAR/AIT, nonzero CDELT)");
    if ((long long)wcs->naxis1 * wcs->naxis2 > (1LL << 31) - 1 || S > 65535)
        return set_error(XTS_ERR_ARG, "point_source_maps: map or source count too large");
    const bool f64 = (flags & XTS_OUT_F64) != 0;
    const size_t npix = (size_t)wcs->naxis1 * wcs->naxis2;
    if ((flags & XTS_DEVICE_PTRS) && !f64 && ((uintptr_t)model_map & 15))
        return set_error(XTS_ERR_ARG, "point_source_maps: device model_map must be 16-byte aligned");
    const int C = cube->nbrbins;
    Stager sg{(flags & XTS_DEVICE_PTRS) != 0, stream ? (cudaStream_t)stream : g_ctx.stream};
    // The map geometry (pixel grids, solid angles, source boundaries, the window
    // pass) needs only the source list and the WCS: it runs on the geometry
    // stream from here on, beside the livetime-cube upload, the exposure and the
    // mean PSF, and joins the launching stream before the correction factors.
    const double* src_d = sg.in(src_sph, (size_t)2 * S);
    const bool fork = sg.rc == XTS_OK && S > 0;
    if (fork) {
        XTS_CUDA(cudaEventRecord(g_ctx.fork_ev, sg.st));
        XTS_CUDA(cudaStreamWaitEvent(g_ctx.geo_stream, g_ctx.fork_ev, 0));
    }
    // (a) exposure; its outputs stay in device memory
    ExposureDev ea;
    ea.src_sph = src_d; ea.S = S;
    CubeRows rows;
    stage_cubes(sg, cube, wcube, src_d, S, ea, rows);
    ea.nside = cube->nside; ea.C = C; ea.cosmin = cube->cosmin; ea.thetabin = cube->thetabin;
    ea.logEs = sg.in(logEs, (size_t)E); ea.E = E;
    ea.af = stage_grid(sg, aeff_front);
    ea.ab = stage_grid(sg, aeff_back);
    ea.ltf = sg.in(front_ltf, (size_t)2 * E);
    ea.exp_costhetas = sg.scratch<double>(C);
    ea.front_aeff = sg.scratch<double>((size_t)C * E);
    ea.back_aeff = sg.scratch<double>((size_t)C * E);
    ea.ecb = sg.scratch<double>((size_t)S * C);
    ea.wecb = sg.scratch<double>((size_t)S * C);
    ea.exposure = sg.scratch<double>((size_t)S * E);
    // (b) mean PSF tables
    PsfDev pa;
    pa.pf = stage_grid(sg, psf_front);
    pa.pb = stage_grid(sg, psf_back);
    pa.costh = ea.exp_costhetas; pa.C = C;
    pa.logEs = ea.logEs; pa.E = E;
    pa.af = ea.front_aeff; pa.ab = ea.back_aeff;
    pa.ecb = ea.ecb; pa.wecb = ea.wecb; pa.S = S;
    pa.ltf = ea.ltf; pa.exposure = ea.exposure;
    pa.upsf = sg.scratch<double>((size_t)S * ND * E);
    pa.partial = sg.scratch<double>((size_t)S * ND * E);
    // (c)+(d) model maps
    SrcmapDev ma;
    ma.wcs = *wcs;
    ma.src_sph = ea.src_sph; ma.S = S;
    ma.exposure = ea.exposure; ma.upsf = pa.upsf; ma.partial = pa.partial; ma.E = E;
    ma.out_f64 = f64;
    ma.out = f64 ? (void*)sg.out((double*)model_map, (size_t)S * npix * E)
                 : (void*)sg.out((float*)model_map, (size_t)S * npix * E);
    ma.inv_integ = info ? sg.out(info->inv_map_integral, (size_t)S * E) : nullptr;
    ma.correction = info ? sg.out(info->correction, (size_t)S * E) : nullptr;
    ma.radius = info ? sg.out(info->psf_radius, (size_t)S) : nullptr;
    ma.in_fov = info ? sg.out(info->in_fov, (size_t)S) : nullptr;
    ma.kernel = srcmap_kernel(flags);
    if (net) {
        ma.surrogate = net;
        ma.logEs = ea.logEs;
        ma.check_tol = check_tol;
        ma.sur_stats = stats;
        if (stats) memset(stats, 0, sizeof(*stats));
    }
    if (fork) { ma.geo_stream = g_ctx.geo_stream; ma.join_ev = g_ctx.join_ev; }
    int rc = sg.rc;
    // exposure and mean PSF on the library's highest-priority stream: the window pass
    // (one short block per work item, on the geometry stream) fills the GPU, and these
    // kernels' blocks are then scheduled ahead of its pending ones as slots free up
    if (rc == XTS_OK) {
        cudaStream_t ps = g_ctx.prio_stream;
        XTS_CUDA(cudaEventRecord(g_ctx.pfork_ev, sg.st));
        XTS_CUDA(cudaStreamWaitEvent(ps, g_ctx.pfork_ev, 0));
        rc = launch_exposure(ea, ps);
        if (rc == XTS_OK) rc = launch_psf(pa, ps);
        XTS_CUDA(cudaEventRecord(g_ctx.pjoin_ev, ps));
        XTS_CUDA(cudaStreamWaitEvent(sg.st, g_ctx.pjoin_ev, 0));
    }
    if (rc != XTS_OK) {
        if (fork) StreamJoin{g_ctx.geo_stream, sg.st, g_ctx.join_ev}.join();
        return sg.finish(rc);
    }
    return run_srcmap(sg, ma, model_map, npix, f64);
}

int xts_point_source_maps(const xts_expcube* cube, const xts_expcube* wcube, const double* logEs,
                          int E, const double* src_sph, int S, const xts_grid* aeff_front,
                          const xts_grid* aeff_back, const xts_grid* psf_front,
                          const xts_grid* psf_back, const double* front_ltf, const xts_wcs* wcs,
                          void* model_map, xts_srcmap_info* info, unsigned flags, void* stream) {
    XTS_ENTER();
    return fused_maps(cube, wcube, logEs, E, src_sph, S, aeff_front, aeff_back, psf_front, psf_back, front_ltf, wcs,
                      model_map, info, flags, stream, nullptr, 0., nullptr);
}

int xts_point_source_maps_surrogate(const xts_expcube* cube, const xts_expcube* wcube, const double* logEs,
                                    int E, const double* src_sph, int S, const xts_grid* aeff_front,
                                    const xts_grid* aeff_back, const xts_grid* psf_front,
                                    const xts_grid* psf_back, const double* front_ltf, const xts_wcs* wcs,
                                    const xts_mlp* net, double check_tol, float* model_map,
                                    xts_srcmap_info* info, xts_surrogate_stats* stats, unsigned flags,
                                    void* stream) {
    XTS_ENTER();
    int rc = mlp_ok(net, "point_source_maps_surrogate");
    if (rc) return rc;
    if (!(check_tol > 0.)) return set_error(XTS_ERR_ARG, "point_source_maps_surrogate: check_tol must be > 0");
    if (flags & (XTS_OUT_F64 | XTS_CUDA_CORES | XTS_TCGEN05))
        return set_error(XTS_ERR_ARG, "point_source_maps_surrogate: FP32 maps of the window path only");
    if (!srcmap_adaptive_supported(E))
        return set_error(XTS_ERR_ARG, "point_source_maps_surrogate: E must be in 1..256");
    return fused_maps(cube, wcube, logEs, E, src_sph, S, aeff_front, aeff_back, psf_front, psf_back, front_ltf, wcs,
                      model_map, info, flags, stream, net, check_tol, stats);
}

int xts_make_psf_kernel(const xts_wcs* kernel_wcs, int Nk, const double* upsf, int E, double* kernel,
                        unsigned flags, void* stream) {
    XTS_ENTER();
    if (!kernel_wcs || Nk <= 0 || !(Nk & 1) || E <= 0 || !upsf || !kernel || (long long)Nk * Nk > (1LL << 30))
        return set_error(XTS_ERR_ARG, "make_psf_kernel: null argument or bad size (Nk odd and positive)");
    if ((kernel_wcs->proj != 0 && kernel_wcs->proj != 1) || kernel_wcs->cdelt1 == 0. || kernel_wcs->cdelt2 == 0.)
        return set_error(XTS_ERR_ARG, "make_psf_kernel: bad WCS (CAR/AIT, nonzero CDELT)");
    Stager sg{(flags & XTS_DEVICE_PTRS) != 0, stream ? (cudaStream_t)stream : g_ctx.stream};
    const double* u = sg.in(upsf, (size_t)ND * E);
    double* k = sg.out(kernel, (size_t)E * Nk * Nk);
    int rc = sg.rc ? sg.rc : make_psf_kernel(*kernel_wcs, Nk, u, E, k, sg.st);
    return sg.finish(rc);
}

int xts_convolve_map_psf(const double* image, int E, int H, int W, const double* kernel, int K, double* out,
                         unsigned flags, void* stream) {
    XTS_ENTER();
    if (!image || !kernel || !out || E <= 0 || H <= 0 || W <= 0 || K <= 0)
        return set_error(XTS_ERR_ARG, "convolve_map_psf: null argument or bad size");
    const long long PH = (long long)H + K - 1, PW = (long long)W + K - 1;
    if (PH > (1 << 20) || PW > (1 << 20) || (long long)E * PH * PW > (1LL << 31))
        return set_error(XTS_ERR_ARG, "convolve_map_psf: padded cube too large");
    Stager sg{(flags & XTS_DEVICE_PTRS) != 0, stream ? (cudaStream_t)stream : g_ctx.stream};
    const double* im = sg.in(image, (size_t)E * H * W);
    const double* ke = sg.in(kernel, (size_t)E * K * K);
    double* o = sg.out(out, (size_t)E * PH * PW);
    int rc = sg.rc ? sg.rc : convolve_map_psf(im, E, H, W, ke, K, o, sg.st);
    return sg.finish(rc);
}

static bool wcs_ok(const xts_wcs* w);

int xts_set_tuning(const xts_tuning* t) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!t) {
        g_tuning = xts_tuning{0, 0, 0, 0, 0};
        return XTS_OK;
    }
    if (t->window_blocks_per_sm < 0 || t->window_blocks_per_sm > 4 || t->write_blocks_per_sm < 0 || t->write_blocks_per_sm > 2 ||
        t->queue_blocks_per_sm < 0 || t->queue_blocks_per_sm > 4 || t->mlp_blocks_per_sm < 0 ||
        t->mlp_blocks_per_sm > 2 || t->chunk_sources < 0)
        return set_error(XTS_ERR_ARG, "set_tuning: a field is outside its range");
    g_tuning = *t;
    return XTS_OK;
}

int xts_get_tuning(xts_tuning* t) {
    if (!t) return set_error(XTS_ERR_ARG, "get_tuning: null argument");
    std::lock_guard<std::mutex> lock(g_mu);
    *t = g_tuning;
    return XTS_OK;
}

int xts_cutout_windows(const xts_wcs* wcs, const double* src_sph, const double* radius_deg, int S,
                       xts_cutout* cut, long long* total_pixels) {
    if (!wcs_ok(wcs) || S < 0 || (S > 0 && (!src_sph || !radius_deg || !cut)))
        return set_error(XTS_ERR_ARG, "cutout_windows: bad WCS or null argument");
    const WcsDev w = make_wcs(*wcs);
    const long H = wcs->naxis1, W = wcs->naxis2;
    long long off = 0;
    for (int s = 0; s < S; ++s) {
        if (!(radius_deg[s] >= 0.) || !std::isfinite(radius_deg[s]))
            return set_error(XTS_ERR_ARG, "cutout_windows: radius %d must be finite and >= 0", s);
        double ra = src_sph[2 * s], p1 = 0., p2 = 0.;
        ra = ra > 180. ? ra - 360. : (ra < -180. ? ra + 360. : ra);
        sph2pix(w, ra, src_sph[2 * s + 1], &p1, &p2);
        xts_cutout c{0, 0, 0, 0, off};
        if (std::isfinite(p1) && std::isfinite(p2) && fabs(p1) < 1e9 && fabs(p2) < 1e9) {
            const long n1 = (long)ceil(radius_deg[s] / fabs(wcs->cdelt1));
            const long n2 = (long)ceil(radius_deg[s] / fabs(wcs->cdelt2));
            const long i = lround(p1) - 1, j = lround(p2) - 1;
            const long h0 = std::max(0L, i - n1), h1 = std::min(H, i + n1 + 1);
            const long w0 = std::max(0L, j - n2), w1 = std::min(W, j + n2 + 1);
            if (h1 > h0 && w1 > w0) {
                c.h0 = (int)h0; c.nh = (int)(h1 - h0);
                c.w0 = (int)w0; c.nw = (int)(w1 - w0);
            }
        }
        cut[s] = c;
        off += (long long)c.nh * c.nw;
    }
    if (total_pixels) *total_pixels = off;
    return XTS_OK;
}

int xts_point_src_model_map_cutouts(const xts_wcs* wcs, const double* src_sph, int S, const xts_cutout* cut,
                                    const double* exposure, const double* upsf, const double* partial, int E,
                                    float* model_map, xts_srcmap_info* info, unsigned flags, void* stream) {
    XTS_ENTER();
    if (!wcs_ok(wcs))
        return set_error(XTS_ERR_ARG, "point_src_model_map_cutouts: bad WCS (CAR/AIT, nonzero CDELT)");
    if (S < 0 || E <= 0 || E > 52 || (S > 0 && (!src_sph || !cut || !exposure || !upsf || !partial || !model_map)))
        return set_error(XTS_ERR_ARG, "point_src_model_map_cutouts: null argument or bad size (E <= 52)");
    if ((long long)wcs->naxis1 * wcs->naxis2 > (1LL << 30) || S > 65535)
        return set_error(XTS_ERR_ARG, "point_src_model_map_cutouts: map or source count too large");
    if (flags & ~(unsigned)XTS_DEVICE_PTRS)
        return set_error(XTS_ERR_ARG, "point_src_model_map_cutouts: only XTS_DEVICE_PTRS applies");
    const bool dev = (flags & XTS_DEVICE_PTRS) != 0;
    long long total = 0;
    if (!dev) {  // host windows: check them and size the staged map
        for (int s = 0; s < S; ++s) {
            const xts_cutout& c = cut[s];
            if (c.nh < 0 || c.nw < 0 || c.h0 < 0 || c.w0 < 0 || c.h0 + c.nh > wcs->naxis1 ||
                c.w0 + c.nw > wcs->naxis2 || c.offset != total)
                return set_error(XTS_ERR_ARG, "point_src_model_map_cutouts: window %d outside the map or out of order",
                                 s);
            total += (long long)c.nh * c.nw;
        }
    }
    Stager sg{dev, stream ? (cudaStream_t)stream : g_ctx.stream};
    SrcmapDev a;
    a.wcs = *wcs;
    a.src_sph = sg.in(src_sph, (size_t)2 * S); a.S = S;
    a.cut = sg.in(cut, (size_t)S);
    a.exposure = sg.in(exposure, (size_t)S * E);
    a.upsf = sg.in(upsf, (size_t)S * ND * E);
    a.partial = sg.in(partial, (size_t)S * ND * E); a.E = E;
    a.out_f64 = false;
    a.out = sg.out(model_map, (size_t)(dev ? 1 : total) * E);
    a.inv_integ = info ? sg.out(info->inv_map_integral, (size_t)S * E) : nullptr;
    a.correction = info ? sg.out(info->correction, (size_t)S * E) : nullptr;
    a.radius = info ? sg.out(info->psf_radius, (size_t)S) : nullptr;
    a.in_fov = info ? sg.out(info->in_fov, (size_t)S) : nullptr;
    int rc = sg.rc ? sg.rc : (S > 0 ? launch_srcmap(a, sg.st) : XTS_OK);
    rc = sg.finish(rc);
    if (rc == XTS_OK && !dev && S > 0) rc = srcmap_status(sg.st);
    return rc;
}

static bool wcs_ok(const xts_wcs* w) {
    return w && w->naxis1 > 0 && w->naxis2 > 0 && (w->proj == 0 || w->proj == 1) && w->cdelt1 != 0. &&
           w->cdelt2 != 0.;
}

int xts_rebin_wcs(const xts_wcs* in, double target_pix_size, xts_wcs* out) {
    if (!wcs_ok(in) || !out || !(target_pix_size > 0.) || !std::isfinite(target_pix_size))
        return set_error(XTS_ERR_ARG, "rebin_wcs: bad WCS or target pixel size");
    return rebin_wcs(*in, target_pix_size, out);
}

int xts_allsky_crop_range(const xts_wcs* allsky_wcs, const xts_wcs* roi_wcs, long range[4]) {
    if (!wcs_ok(allsky_wcs) || !wcs_ok(roi_wcs) || !range)
        return set_error(XTS_ERR_ARG, "allsky_crop_range: bad WCS (CAR/AIT, nonzero CDELT) or null range");
    return allsky_crop_range(*allsky_wcs, *roi_wcs, range);
}

int xts_crop_allsky(const float* allsky, int E0, long NY, long NX, const long range[4], float* out, unsigned flags,
                    void* stream) {
    XTS_ENTER();
    if (!allsky || !out || !range || E0 <= 0 || NY <= 0 || NX <= 0)
        return set_error(XTS_ERR_ARG, "crop_allsky: null argument or bad size");
    if (range[0] < 1 || range[0] > NX || range[1] < 1 || range[1] > NX || range[2] < 1 || range[3] > NY ||
        range[2] > range[3])
        return set_error(XTS_ERR_ARG, "crop_allsky: range outside the all-sky image");
    const long nx = range[1] >= range[0] ? range[1] - range[0] + 1 : NX - range[0] + 1 + range[1];
    const long ny = range[3] - range[2] + 1;
    Stager sg{(flags & XTS_DEVICE_PTRS) != 0, stream ? (cudaStream_t)stream : g_ctx.stream};
    const float* sky = sg.in(allsky, (size_t)E0 * NY * NX);
    float* o = sg.out(out, (size_t)E0 * ny * nx);
    int rc = sg.rc ? sg.rc : crop_allsky(sky, E0, NY, NX, range, o, sg.st);
    return sg.finish(rc);
}

int xts_trilerp_ehw(const float* src, int E0, int H0, int W0, float* dst, int E1, int H1, int W1, unsigned flags,
                    void* stream) {
    XTS_ENTER();
    if (!src || !dst || E0 <= 0 || H0 <= 0 || W0 <= 0 || E1 <= 0 || H1 <= 0 || W1 <= 0 ||
        (long long)E1 * H1 * W1 > (1LL << 40))
        return set_error(XTS_ERR_ARG, "trilerp_ehw: null argument or bad size");
    Stager sg{(flags & XTS_DEVICE_PTRS) != 0, stream ? (cudaStream_t)stream : g_ctx.stream};
    const float* sp = sg.in(src, (size_t)E0 * H0 * W0);
    float* dp = sg.out(dst, (size_t)E1 * H1 * W1);
    int rc = sg.rc ? sg.rc : trilerp_ehw(sp, E0, H0, W0, dp, E1, H1, W1, sg.st);
    return sg.finish(rc);
}

int xts_scale_model_map(const xts_wcs* wcs, const double* src_sph, int S, const double* exposure, const double* upsf,
                        const double* partial, int E, float* model_map, xts_srcmap_info* info, unsigned flags,
                        void* stream) {
    XTS_ENTER();
    if (!wcs_ok(wcs))
        return set_error(XTS_ERR_ARG, "scale_model_map: bad WCS (CAR/AIT, nonzero CDELT)");
    if (S < 0 || E <= 0 || E > 256 || (S > 0 && (!src_sph || !exposure || !upsf || !partial || !model_map)))
        return set_error(XTS_ERR_ARG, "scale_model_map: null argument or bad size (E <= 256)");
    if ((long long)wcs->naxis1 * wcs->naxis2 * E > 0xffffffffLL || S > 65535)
        return set_error(XTS_ERR_ARG, "scale_model_map: map or source count too large");
    if (flags & ~(unsigned)XTS_DEVICE_PTRS)
        return set_error(XTS_ERR_ARG, "scale_model_map: only XTS_DEVICE_PTRS applies");
    const size_t npix = (size_t)wcs->naxis1 * wcs->naxis2;
    Stager sg{(flags & XTS_DEVICE_PTRS) != 0, stream ? (cudaStream_t)stream : g_ctx.stream};
    SrcmapDev a;
    a.wcs = *wcs;
    a.src_sph = sg.in(src_sph, (size_t)2 * S); a.S = S;
    a.exposure = sg.in(exposure, (size_t)S * E);
    a.upsf = sg.in(upsf, (size_t)S * ND * E);
    a.partial = sg.in(partial, (size_t)S * ND * E); a.E = E;
    a.out_f64 = false;
    float* m = sg.out(model_map, (size_t)S * npix * E);  // pixel means in, model map out
    if (!sg.dev && !sg.rc && m && S > 0) {
        cudaError_t e = cudaMemcpyAsync(m, model_map, sizeof(float) * S * npix * E, cudaMemcpyHostToDevice, sg.st);
        if (e != cudaSuccess) return cuda_error(e, "cudaMemcpyAsync H2D");
    }
    a.out = m;
    a.inv_integ = info ? sg.out(info->inv_map_integral, (size_t)S * E) : nullptr;
    a.correction = info ? sg.out(info->correction, (size_t)S * E) : nullptr;
    a.radius = info ? sg.out(info->psf_radius, (size_t)S) : nullptr;
    a.in_fov = info ? sg.out(info->in_fov, (size_t)S) : nullptr;
    a.means_given = true;
    int rc = sg.rc ? sg.rc : launch_srcmap(a, sg.st);
    return sg.finish(rc);
}

int xts_write_src_model(const char* filename, const void* model_map, int S, int H, int W, int E,
                        const char* const* names, unsigned flags, void* stream) {
    XTS_ENTER();
    if (!filename || S < 0 || H <= 0 || W <= 0 || E <= 0 || (S > 0 && !model_map))
        return set_error(XTS_ERR_ARG, "write_src_model: null argument or bad size");
    if (W > 65535 || S > (1 << 30))
        return set_error(XTS_ERR_ARG, "write_src_model: W must be at most 65535");
    return write_src_model(filename, model_map, S, H, W, E, names, (flags & XTS_DEVICE_PTRS) != 0,
                           (flags & XTS_OUT_F64) != 0, (flags & XTS_FITS_F32) == 0,
                           stream ? (cudaStream_t)stream : g_ctx.stream);
}

}  // extern "C"
