// xts_internal.cuh -- shared definitions of the CUDA library: constants of the
// algorithm, error plumbing, the cached device workspace and the launchers each
// stage exports to the C-ABI layer.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/xtsrcmaps_b200.h"

#define XTS_HD __host__ __device__

namespace xts {

// misc/misc.hxx:15-43 -- constants are part of the algorithm.
constexpr double PI = 3.141592653589793238462643383279502884197;
constexpr double TWOPI = 6.283185307179586476925286766559005768394;
constexpr double HALFPI = 1.570796326794896619231321691639751442099;
constexpr double INV_HALFPI = 0.6366197723675813430755350534900574;
constexpr double D2R = 0.017453292519943295769236907684886127134;
constexpr double R2D = 57.295779513082320876798154814105170332405;
constexpr double SEP_STEP = 0.033731417579011382769913057686378448039204491;  // ln(7e5)/399
constexpr double RECIPSTEP = 29.645952402019046699874076387601854602589360539942632073727038565;
constexpr double REDM1 = 29.148763300179999028597222671574207003288142769360422095500496366;  // 1/(e^step - 1)
constexpr double LN_1E4 = 9.2103403719761827360719658187374568304044059545150919;
constexpr int ND = XTS_ND;

// Error plumbing ---------------------------------------------------------------
int set_error(int code, const char* fmt, ...);
int cuda_error(cudaError_t e, const char* what);

#define XTS_CUDA(call)                                         \
    do {                                                       \
        cudaError_t e__ = (call);                              \
        if (e__ != cudaSuccess) return ::xts::cuda_error(e__, #call); \
    } while (0)

#define XTS_CHECK_LAUNCH(name)                                 \
    do {                                                       \
        cudaError_t e__ = cudaGetLastError();                  \
        if (e__ != cudaSuccess) return ::xts::cuda_error(e__, name); \
    } while (0)

// Launch shapes chosen by the autotuner (xts_set_tuning); fields are 0 for the default.
extern xts_tuning g_tuning;

// Optional per-kernel timing (xts_profile_enable): CUDA events recorded on the
// launching stream around each kernel.  A no-op while profiling is off.
void prof_mark(const char* name, cudaStream_t st, bool begin);

// Launch a kernel, time it when profiling is on, and check the launch.
#define XTS_LAUNCH(name, st, ...)                              \
    do {                                                       \
        ::xts::prof_mark(name, st, true);                      \
        __VA_ARGS__;                                           \
        ::xts::prof_mark(name, st, false);                     \
        XTS_CHECK_LAUNCH(name);                                \
    } while (0)

// Grow-only device workspace, one buffer per slot ------------------------------
enum Slot {
    // staged inputs / outputs (host-pointer mode)
    S_IN0, S_IN1, S_IN2, S_IN3, S_IN4, S_IN5, S_IN6, S_IN7, S_IN8, S_IN9, S_IN10, S_IN11,
    S_IN12, S_IN13, S_IN14, S_IN15, S_IN16, S_IN17,
    S_OUT0, S_OUT1, S_OUT2, S_OUT3, S_OUT4, S_OUT5, S_OUT6, S_OUT7, S_OUT8, S_OUT9, S_OUT10,
    S_OUT11, S_OUT12, S_OUT13, S_OUT14, S_OUT15,
    // internal scratch
    W_CORNERS, W_CENTERS, W_OMEGA, W_LUT, W_PARTSUM, W_SRCINFO, W_SCALE, W_PSFTAB,
    W_KING, W_MISC, W_WIN, W_WMETA, W_SPARSE, W_MISC2, W_EXPMAP,
    W_FITS_IN, W_FITS_OUT, W_FITS_SUM, W_FFT_A, W_FFT_B, W_FFT_C, W_FFT_WORK, W_SRCPIX, W_CUT_ITEMS, W_ADAPT_MEAN,
    W_MLP_Z, W_MLP_H, W_MLP_DZ, W_MLP_DH, W_MLP_Y, W_MLP_ST, W_MLP_PART, W_MLP_PART2, W_SUR_X, W_SUR_AUX, W_SUR_Y, W_SUR_IDX, W_SUR_ERR, W_SUR_SEG,
    N_SLOTS
};
void* workspace(int slot, size_t bytes);  // nullptr + error set on OOM
cudaStream_t default_stream();
int ensure_device();

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Per-source geometry produced by the boundary-radius kernel (c6).
struct SrcInfo {
    double dir[3];
    double radius_deg;
    double radius_rad;
    int in_fov;
    int pad;
};

// Stage launchers (device pointers, enqueue on `st`) ----------------------------
struct ExposureDev {
    const float* cube; const float* wcube; long long nside; int C; double cosmin; int thetabin;
    const double* logEs; int E;
    const double* src_sph; int S;
    xts_grid af, ab;  // device pointers inside
    const double* ltf;
    double* exp_costhetas; double* front_aeff; double* back_aeff;
    double* ecb; double* wecb; double* exposure;
    bool gathered = false;  // cube, wcube hold only the sources' rows, [S][C] in source order
};
int launch_exposure(const ExposureDev& a, cudaStream_t st);
int launch_src_pixels(const double* src_sph, int S, long long nside, long long* pix, cudaStream_t st);
int launch_exposure_contract(const double* ecb, const double* wecb, int S, int C, const double* af,
                             const double* ab, const double* ltf, int E, double* out, cudaStream_t st);

int launch_ltf(const double* logEs, int E, const float* p0, const float* p1, double* ltf,
               cudaStream_t st);
int launch_normalize_rpsf(double* params, int Mc, int Me, const double* glog, float s0,
                          float s1, float si, cudaStream_t st);

struct PsfDev {
    xts_grid pf, pb;  // device pointers inside
    const double* costh; int C;
    const double* logEs; int E;
    const double* af; const double* ab;
    const double* ecb; const double* wecb; int S;
    const double* ltf; const double* exposure;
    double* upsf; double* partial;
};
int launch_psf(const PsfDev& a, cudaStream_t st);

struct SrcmapDev {
    xts_wcs wcs;
    const double* src_sph; int S;
    const double* exposure; const double* upsf; const double* partial; int E;
    void* out; bool out_f64;
    double* inv_integ; double* correction; double* radius; int* in_fov;  // optional (may be null)
    int kernel;  // FP32 write pass: SRCMAP_WINDOWS, SRCMAP_ONEPASS or SRCMAP_TCGEN05
    // Optional: sources per chunk of the write pass, and a hook called on the
    // launching stream after each chunk's maps are enqueued (pipelined copy-out).
    int chunk_sources = 0;
    int (*on_chunk)(void* ctx, int s0, int n, cudaStream_t st) = nullptr;
    void* on_chunk_ctx = nullptr;
    // adaptive Genz-Malik cubature in place of the 12-point rule (FP32 map)
    bool adaptive = false;
    double rtol = 1e-4;
    int max_depth = 6;
    // Optional: a stream for the map geometry (grids, solid angles, boundaries and
    // the first chunk's window pass), which needs neither the exposure nor uPsf;
    // it already waits for the source list, and joins the launching stream through
    // join_ev before the first kernel that reads uPsf.
    cudaStream_t geo_stream = nullptr;
    cudaEvent_t join_ev = nullptr;
    // a.out holds FP32 pixel means on entry: only the scalings of c7-c10 and d2 are
    // applied (the diffuse map's final steps)
    bool means_given = false;
    // per-source cutout windows [S] (device), or NULL for the dense map
    const xts_cutout* cut = nullptr;
    // pixel means from the surrogate network (with the 12-point rule as fallback)
    const xts_mlp* surrogate = nullptr;
    const double* logEs = nullptr;  // [E] log10 energies (the network's fourth feature)
    double check_tol = 1e-4;
    xts_surrogate_stats* sur_stats = nullptr;
};

// Two pairs of events for the chunk pipeline of the window path (library-owned).
void pipe_events(cudaEvent_t a[2], cudaEvent_t b[2]);

// The geometry stream joins the launching stream once: at join(), or when it
// goes out of scope (error paths, so that a stream capture never ends unjoined).
struct StreamJoin {
    cudaStream_t from, into;
    cudaEvent_t ev;
    bool pending = true;
    StreamJoin(cudaStream_t f, cudaStream_t i, cudaEvent_t e) : from(f), into(i), ev(e), pending(f != i && e) {}
    int join() {
        if (!pending) return XTS_OK;
        pending = false;
        cudaError_t e = cudaEventRecord(ev, from);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(into, ev, 0);
        return e == cudaSuccess ? XTS_OK : cuda_error(e, "geometry stream join");
    }
    ~StreamJoin() { join(); }
};
enum { SRCMAP_WINDOWS = 0, SRCMAP_ONEPASS = 1, SRCMAP_TCGEN05 = 2 };
int launch_srcmap(const SrcmapDev& a, cudaStream_t st);
int launch_map_integral_fast(const double* corners, const double* centers, const double* omega,
                             const SrcInfo* info, int S, int H, int W, int nch, double* hist,
                             cudaStream_t st);
int launch_srcmap_tc(const double* corners, const double* omega, const SrcInfo* info,
                     const double* upsf, const double* scale, int S, int H, int W, int E, float* out,
                     int* status, cudaStream_t st);
int srcmap_status(cudaStream_t st);
int launch_correction(const double* hist, int nch, const SrcInfo* info, int S, const double* upsf,
                      const double* partial, const double* exposure, int E, double* scale,
                      double* inv_integ, double* correction, double* radius, int* in_fov,
                      cudaStream_t st, float* lut = nullptr, int Epad = 0);  // lut: scaled FP32 table too
bool srcmap_win_supported(int E);
int make_psf_kernel(const xts_wcs& wcs, int Nk, const double* upsf, int E, double* kernel, cudaStream_t st);
int convolve_map_psf(const double* image, int E, int H, int W, const double* kernel, int K, double* out,
                     cudaStream_t st);
int allsky_crop_range(const xts_wcs& sky, const xts_wcs& roi, long range[4]);
int crop_allsky(const float* sky, int E0, long NY, long NX, const long range[4], float* out, cudaStream_t st);
int trilerp_ehw(const float* src, int E0, int H0, int W0, float* dst, int E1, int H1, int W1, cudaStream_t st);
int rebin_wcs(const xts_wcs& in, double target, xts_wcs* out);
int write_src_model(const char* filename, const void* model_map, int S, int H, int W, int E,
                    const char* const* names, bool dev_ptrs, bool f64in, bool f64out, cudaStream_t st);
bool exposure_map_supported(int C, int E);
int launch_exposure_map_tc(const float* cube, const float* wcube, long long npix, int C, const double* front_aeff,
                           const double* back_aeff, const double* ltf, int E, double* out, int* status,
                           cudaStream_t st);
bool srcmap_adaptive_supported(int E);
int launch_adaptive_map(const double* corners, const double* centers, const double* omega, const SrcInfo* info,
                        const double* upsf, int S, int H, int W, int E, double rtol, int max_depth, int nch,
                        double* sums, double* mean64, int* status, cudaStream_t st);
int launch_mean_integral64(const double* centers, const double* omega, const SrcInfo* info, const double* mean, int S,
                           int H, int W, int E, int nch, double* sums, cudaStream_t st);
int launch_scale_map64(const double* mean, float* out, const double* omega, const double* scale, int S, int npix,
                       int E, cudaStream_t st);
int launch_scale_map(float* out, const double* omega, const double* scale, int S, int npix, int E,
                     cudaStream_t st);
// c7 sums [S][nch][E] of pixel means [S][H*W][E] times solid angle over the pixels
// inside each source's boundary radius (E <= 256)
int mean_integral_chunks(int S, int npix);  // blocks per source of launch_mean_integral
int launch_mean_integral(const double* centers, const double* omega, const SrcInfo* info, const float* mean, int S,
                         int H, int W, int E, int nch, double* sums, cudaStream_t st);
// map of pixel means -> model map: c7 sums, c9 correction, c8/c10 scalings with the solid angle
// finish_mean_map for sources [s0, s0 + ns) only
int finish_mean_map_range(const SrcmapDev& a, int s0, int ns, const double* centers, const double* omega,
                          const SrcInfo* info, double* scale, cudaStream_t st);
int finish_mean_map(const SrcmapDev& a, const double* centers, const double* omega, const SrcInfo* info,
                    double* scale, int nch, cudaStream_t st);
// the surrogate network (xts_mlp.cu) and the surrogate model map (xts_surrogate.cu)
int launch_gemm_bf16(const void* A, int a_trans, const void* B, int b_trans, int M, int K, float* C, int c_trans,
                     int accumulate, int* status, cudaStream_t st);
int launch_mlp_forward(const xts_mlp* net, const float* X, long long n, float* y, int* status, cudaStream_t st);
// the same with the row count read on the device (at most n_max rows; no host sync)
int launch_mlp_forward_dev(const xts_mlp* net, const float* X, const unsigned long long* n_dev, long long n_max,
                           float* y, int* status, cudaStream_t st,
                           long long ldx = 0);  // X row-major [n][5] (0) or feature-major [5][ldx]
int launch_mlp_grads(const xts_mlp* net, const float* X, const float* Y, long long n, float* grads, float* loss,
                     int* status, cudaStream_t st);
int launch_mlp_train_step(const xts_mlp* net, const float* X, const float* Y, long long n, float* grads,
                          float* m, float* v, int step, float lr, float* loss, int* status, cudaStream_t st);
int mlp_check_status(int* status, cudaStream_t st);
int launch_surrogate_samples(const double* upsf, const double* logEs, int S, int E, long long n,
                             unsigned long long seed, double rho_min, float* X, float* Y, cudaStream_t st);
int launch_srcmap_surrogate(const SrcmapDev& a, const double* corners, const double* centers, const double* omega,
                            const SrcInfo* info, double* scale, int nch, cudaStream_t st);
int surrogate_last_stats(xts_surrogate_stats* stats, cudaStream_t st);
int launch_srcmap_win(const double* corners, const double* centers, const double* omega,
                      const SrcInfo* info, int S, int H, int W, int E,
                      const double* upsf, const double* partial, const double* exposure,
                      double* scale, double* inv_integ, double* correction, double* radius,
                      int* in_fov, int* status, float* out, int chunk_sources,
                      int (*on_chunk)(void*, int, int, cudaStream_t), void* on_chunk_ctx,
                      StreamJoin& geo,  // the first chunk's window pass runs on geo.from
                      cudaStream_t st,  // 0, or XTS_ERR_TIMEOUT if a bounded device wait gave up
                      bool means_only = false);  // the rule's pixel means (the table uPsf unscaled): no
                                                 // map integral, correction or scale outputs
int launch_srcmap_win_cut(const double* corners, const double* centers, const double* omega, const SrcInfo* info,
                          const xts_cutout* cut, int S, int H, int W, int E, const double* upsf,
                          const double* partial, const double* exposure, double* scale, double* inv_integ,
                          double* correction, double* radius, int* in_fov, int* status, float* out, cudaStream_t st);
int launch_srcmap_fast(const double* corners, const double* omega, const SrcInfo* info,
                       const double* upsf, const double* scale, int S, int H, int W, int E,
                       float* out, cudaStream_t st);

}  // namespace xts
