// xts_noalloc.cu -- the mean-PSF step for callers that cannot allocate device
// memory.
//
// Some hosts of this library must not call cudaMalloc once they are running: a
// caller that records its GPU work into a CUDA graph or a stream capture, a
// real-time or embedded host that reserves all device memory up front, or an
// application whose own memory pool owns the device.  xts_compute_psf_data
// allocates (and caches) its scratch tables on first use; this entry point keeps
// that scratch in a fixed file-scope device array instead, so a call needs no
// allocation at all: the caller passes device pointers for every input and
// output, and the King and psf*aeff tables live in g_noalloc_scratch.
//
// Limits and sharing:
//   * the scratch holds at most XTS_NOALLOC_SCRATCH_DOUBLES doubles: the King
//     tables, 401 * (Mc*Me front + Mc*Me back), rounded up to a multiple of 32,
//     then the psf*aeff table, C * 401 * E; larger shapes are rejected with
//     XTS_ERR_ARG before anything is launched;
//   * every GPU that loads the library holds the 8 MiB array until the process
//     exits;
//   * all calls share the array; each call overwrites every scratch element it
//     reads, so nothing has to start at zero, but calls that overlap on the GPU
//     (different streams, or different host threads without ordering) race on
//     it and must be serialised by the caller;
//   * the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current; make that first call
//     before any stream capture begins (a first call on a capturing stream is
//     refused with XTS_ERR_ARG).  The address is cached per device index and
//     is not valid after cudaDeviceReset.
#include <mutex>

#include "xts_internal.cuh"

namespace xts {

int launch_psf_scratch(const PsfDev& a, double* king, double* pa, cudaStream_t st);  // xts_psf.cu

constexpr size_t NOALLOC_SCRATCH_DOUBLES = XTS_NOALLOC_SCRATCH_DOUBLES;

static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_SCRATCH_DOUBLES];

static double* g_noalloc_ptr[64] = {};
static std::mutex g_noalloc_mu;

// Device address of the scratch array on the current device (looked up once per
// device index; the cached address does not survive cudaDeviceReset or a
// re-created primary context, after which the process must not call this entry
// point again).  The first lookup on a device is refused while `st` is being
// captured, with a message naming the rule, instead of failing inside the capture.
static int noalloc_scratch(cudaStream_t st, double** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_error(e, "cudaGetDevice");
    if (dev < 0 || dev >= 64) return set_error(XTS_ERR_ARG, "device index %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        e = cudaStreamIsCapturing(st, &cs);
        if (e != cudaSuccess) return cuda_error(e, "cudaStreamIsCapturing");
        if (cs != cudaStreamCaptureStatusNone)
            return set_error(XTS_ERR_ARG,
                             "compute_psf_data_noalloc: the first call on device %d must come before any "
                             "stream capture (it looks up the scratch array's device address)", dev);
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_error(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        g_noalloc_ptr[dev] = (double*)p;
    }
    *out = g_noalloc_ptr[dev];
    return XTS_OK;
}

}  // namespace xts

using namespace xts;

extern "C" int xts_compute_psf_data_noalloc(const xts_grid* psf_front, const xts_grid* psf_back,
                                            const double* exp_costhetas, int C, const double* logEs,
                                            int E, const double* front_aeff, const double* back_aeff,
                                            const double* ecb, const double* wecb, int S,
                                            const double* front_ltf, const double* exposure,
                                            double* upsf, double* partial, void* stream) {
    auto grid_ok = [](const xts_grid* g) {
        return g && g->cosths && g->logEs && g->params && g->n_cos >= 2 && g->n_e >= 2 && g->n_par == 6;
    };
    if (!grid_ok(psf_front) || !grid_ok(psf_back))
        return set_error(XTS_ERR_ARG, "compute_psf_data_noalloc: King grids need n_par == 6");
    if (!exp_costhetas || C <= 0 || !logEs || E <= 0 || !front_aeff || !back_aeff || S < 0 ||
        (S > 0 && (!ecb || !wecb || !exposure || !upsf || !partial)) || !front_ltf)
        return set_error(XTS_ERR_ARG, "compute_psf_data_noalloc: null argument or bad size");
    size_t king_n = (size_t)ND * ((size_t)psf_front->n_cos * psf_front->n_e +
                                  (size_t)psf_back->n_cos * psf_back->n_e);
    size_t pa_n = (size_t)C * ND * E;
    // the psf*aeff table starts at the next multiple of 32 doubles (256 bytes)
    // after the King tables; the limit counts that padding
    const size_t pa_off = (king_n + 31) & ~(size_t)31;
    if (pa_off + pa_n > NOALLOC_SCRATCH_DOUBLES)
        return set_error(XTS_ERR_ARG,
                         "compute_psf_data_noalloc: needs %zu scratch doubles (King %zu, padded to %zu, + "
                         "psf*aeff %zu), the fixed scratch holds %zu; use xts_compute_psf_data",
                         pa_off + pa_n, king_n, pa_off, pa_n, (size_t)NOALLOC_SCRATCH_DOUBLES);
    double* scratch = nullptr;
    int rc = noalloc_scratch((cudaStream_t)stream, &scratch);
    if (rc) return rc;
    PsfDev a;
    a.pf = *psf_front;
    a.pb = *psf_back;
    a.costh = exp_costhetas; a.C = C;
    a.logEs = logEs; a.E = E;
    a.af = front_aeff; a.ab = back_aeff;
    a.ecb = ecb; a.wecb = wecb; a.S = S;
    a.ltf = front_ltf; a.exposure = exposure;
    a.upsf = upsf; a.partial = partial;
    return launch_psf_scratch(a, scratch, scratch + pa_off, (cudaStream_t)stream);
}
