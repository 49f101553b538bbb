/*
 * xtsrcmaps_b200.h -- C-ABI of the B200 (sm_100a) point-source model-map path.
 *
 * The reference (xtsrcmaps) has no plugin or FFI layer; its seam is three C++
 * namespace functions called from xtsrcmaps/main.cxx:28-30.  Each entry point
 * below replaces one of them (or one of the finer routines they call) with the
 * same inputs, outputs, tensor layouts and meaning, as plain pointers and sizes.
 *
 * Layouts: row-major, last index contiguous, exactly the reference's
 * Fermi::Tensor layout (tensor/tensor.hpp:113-122).  S = sources, C = cos-theta
 * bins of the livetime cube, E = energies, D = 401 PSF separations, H x W map
 * (H = NAXIS1, the longitude axis; observation/observation.cxx:28-29).
 *
 * Pointers: by default every array argument is a HOST pointer; the library
 * stages it into device memory, runs the kernels on its stream and copies the
 * results back before returning.  With XTS_DEVICE_PTRS every array argument is
 * a device pointer on the current CUDA device, the call is asynchronous on the
 * given stream (NULL = the library's stream) and nothing is copied.
 *
 * Errors: every entry point returns XTS_OK (0) or a negative XTS_ERR_* code and
 * never exits the process; xts_last_error() gives a message for the calling
 * thread.  The reference instead asserts or calls exit(1) (misc/misc.hxx:41-48).
 */
#ifndef XTSRCMAPS_B200_H
#define XTSRCMAPS_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define XTS_ND 401 /* psf/psf.hxx:20 sep_arr_len */

enum xts_status {
    XTS_OK = 0,
    XTS_ERR_ARG = -1,     /* bad shape, null pointer or unsupported option */
    XTS_ERR_CUDA = -2,    /* a CUDA runtime call failed */
    XTS_ERR_OOM = -3,     /* device allocation failed */
    XTS_ERR_TIMEOUT = -4, /* a bounded device-side wait gave up */
    XTS_ERR_NODEV = -5,   /* no usable sm_100 device */
    XTS_ERR_IO = -6       /* a file could not be opened or written */
};

enum xts_flags {
    XTS_DEVICE_PTRS = 1u << 0, /* array arguments are device pointers */
    XTS_OUT_F64 = 1u << 1,     /* model map written as double (default float) */
    /* 1u << 2 is reserved */
    XTS_CUDA_CORES = 1u << 3,    /* FP32 source maps by the single-pass CUDA-core kernel (geometry and
                                    map integral in separate passes; default: the two-pass window path) */
    XTS_TCGEN05 = 1u << 4,       /* FP32 source maps with the window-times-table product on tcgen05
                                    tensor cores (3xTF32); default: the two-pass window path */
    XTS_FITS_F32 = 1u << 5       /* xts_write_src_model: BITPIX -32 images (default -64, as the reference) */
};

/* FITS celestial WCS (sky_geom/sky_geom.hxx:17-25, WcsConfig). */
typedef struct xts_wcs {
    long   naxis1, naxis2;
    double crpix1, crpix2;
    double crval1, crval2;
    double cdelt1, cdelt2;
    double crota2;  /* degrees */
    int    proj;    /* 0 = CAR, 1 = AIT */
    int    galactic;
} xts_wcs;

/* One padded IRF grid (irf/irf_types.hxx:11-16, IrfData3). */
typedef struct xts_grid {
    const double* cosths;  /* [Mc] */
    int           n_cos;
    const double* logEs;   /* [Me] */
    int           n_e;
    const double* params;  /* [Mc, Me, n_par] */
    int           n_par;
    double        min_cos_theta;
} xts_grid;

/* Livetime cube (observation/obs_types.hxx:24-32, ExposureCubeData). */
typedef struct xts_expcube {
    const float* cosbins;  /* [12 nside^2, nbrbins], HEALPix NESTED, equatorial */
    long         nside;
    int          nbrbins;
    double       cosmin;
    int          thetabin; /* THETABIN != "COSTHETA" */
} xts_expcube;

/* Outputs of the exposure step (exposure/exposure.hxx:19-26, XtExp). */
typedef struct xts_exposure_out {
    double* exp_costhetas;                 /* [C] */
    double* front_aeff;                    /* [C, E] */
    double* back_aeff;                     /* [C, E] */
    double* src_exposure_cosbins;          /* [S, C] */
    double* src_weighted_exposure_cosbins; /* [S, C] */
    double* exposure;                      /* [S, E] */
} xts_exposure_out;

/* Optional per-map results of the model-map step.  Any pointer may be NULL. */
typedef struct xts_srcmap_info {
    double* inv_map_integral; /* [S, E] 1 / sum over pixels within radius (0 stays 0) */
    double* correction;       /* [S, E] containment correction factor */
    double* psf_radius;       /* [S] degrees */
    int*    in_fov;           /* [S] */
} xts_srcmap_info;

/* Library state ------------------------------------------------------------ */
int         xts_init(int device);       /* select the device, create the stream */
void        xts_release(void);          /* free every cached device buffer */
const char* xts_last_error(void);
int         xts_version(void);

/* Launch shapes the autotuner chooses by measurement (no counterpart in the
 * reference, whose equivalents are compile-time: model_map.psf_boundary_radius.cxx:25,
 * misc/simdwidth.hpp).  0 in a field keeps its default.  Applies to the calls made
 * after it on every device of the process. */
typedef struct xts_tuning {
    int window_blocks_per_sm; /* window pass of the dense map: its work items (one block each) are
                                 sized for about 16 per block at this many resident blocks per SM
                                 (1..4; default: as many as fit) */
    int write_blocks_per_sm;  /* write pass: persistent blocks per SM (1..2; default: as many as fit) */
    int queue_blocks_per_sm;  /* cutout window pass (work queue): blocks per SM (1..4; default: as many as fit) */
    int mlp_blocks_per_sm;    /* surrogate network inference: 0 (default) four tiles in flight per SM in
                                 one block of four warpgroups; 1..2 the two-warpgroup kernel at that
                                 many blocks per SM */
    int chunk_sources;        /* dense map: sources per chunk of the window and write passes; the
                                 window pass of chunk k + 1 runs beside the write pass of chunk k
                                 (0: one chunk while the window records fit 4 GiB) */
} xts_tuning;
int xts_set_tuning(const xts_tuning* t);  /* NULL restores the defaults */
int xts_get_tuning(xts_tuning* t);

/* Kernel timing for profiling and the roofline report (no counterpart in the
 * reference, which has no tracing).  While enabled, every kernel the library
 * launches is bracketed by CUDA events on its stream.  xts_profile_read waits
 * for the recorded kernels, writes a JSON object
 * {"kernel": [launches, total_ms], ...} into buf and clears the record; it
 * returns the length written or a negative error code.  With on = 2 the record
 * is kept across reads: launches captured into a CUDA graph carry their events
 * as event-record nodes, and each read reports the graph's latest replay. */
int xts_profile_enable(int on);
int xts_profile_read(char* buf, int buflen);

/* Irf::livetime_efficiency_factors (irf/irf.cxx:70-109) -> ltf [2, E]. */
int xts_livetime_efficiency_factors(const double* logEs, int E, const float* p0,
                                    const float* p1, double* ltf, unsigned flags,
                                    void* stream);

/* irf_private::normalize_rpsf (irf/irf.normalize_rpsf.cpp:11-61): normalises a
 * King parameter grid [Mc, Me, 6] in place. */
int xts_normalize_rpsf(double* params, int Mc, int Me, const double* grid_logEs,
                       float scale0, float scale1, float scale_index,
                       unsigned flags, void* stream);

/* Exposure::compute_exposure<T> (exposure/exposure.hxx:44-88): steps a1-a5.
 * front_ltf is Irf::XtIrf::front_LTF [2, E]; C = exp_cube->nbrbins.  With host
 * pointers only the cube rows at the sources' NESTED pixels are copied to the
 * device (as in xts_point_source_maps); device-pointer cubes are read in place. */
int xts_compute_exposure(const xts_expcube* exp_cube, const xts_expcube* wexp_cube,
                         const double* logEs, int E, const double* src_sph, int S,
                         const xts_grid* aeff_front, const xts_grid* aeff_back,
                         const double* front_ltf, const xts_exposure_out* out,
                         unsigned flags, void* stream);

/* Exposure::exposure (exposure/exposure.cxx:159-263, with the DGEMMs of
 * exposure/exposure.contract.cpp:13-42): step a5 alone, from the gathered
 * livetime rows ecb, wecb [S, C] and the Aeff tables [C, E] -> exposure [S, E]. */
int xts_exposure_contract(const double* src_exposure_cosbins,
                          const double* src_weighted_exposure_cosbins, int S, int C,
                          const double* front_aeff, const double* back_aeff,
                          const double* front_ltf, int E, double* exposure,
                          unsigned flags, void* stream);

/* The exposure of every HEALPix pixel of the livetime cube [12 nside^2, E]: the
 * contraction of Exposure::exposure (exposure/exposure.cxx:159-263, DGEMMs of
 * exposure/exposure.contract.cpp:13-42) applied to all cube rows instead of the
 * rows gathered at the sources (exposure/exposure.cxx:42-63), so a source's
 * exposure is the map row at its NESTED pixel.  Computed on tcgen05 tensor
 * cores as 3xTF32 with FP32 accumulation (relative error ~1e-6; the per-source
 * xts_compute_exposure stays FP64).  Needs nbrbins <= 64 and a multiple of 4. */
int xts_exposure_map(const xts_expcube* exp_cube, const xts_expcube* wexp_cube,
                     const double* logEs, int E, const xts_grid* aeff_front,
                     const xts_grid* aeff_back, const double* front_ltf,
                     double* exposure_map, unsigned flags, void* stream);

/* Psf::compute_psf_data (psf/psf.compute_psf_data.cxx:7-33, which calls
 * psf/psf.psf_lookup_table_and_partial_integrals.cxx:8-57): steps b3-b7.
 * psf grids are normalised King grids [Mc, Me, 6]; outputs uPsf and
 * partial_psf_integral [S, 401, E]. */
int xts_compute_psf_data(const xts_grid* psf_front, const xts_grid* psf_back,
                         const double* exp_costhetas, int C, const double* logEs,
                         int E, const double* front_aeff, const double* back_aeff,
                         const double* src_exposure_cosbins,
                         const double* src_weighted_exposure_cosbins, int S,
                         const double* front_ltf, const double* exposure,
                         double* upsf, double* partial, unsigned flags, void* stream);

/* xts_compute_psf_data for callers that cannot allocate device memory.  This
 * entry point has no counterpart in the reference: it exists for hosts that must
 * not call cudaMalloc while they run (work recorded into a stream capture, a
 * service whose memory pool owns the device, a real-time loop).  Every pointer
 * is a DEVICE pointer (no flags argument; XTS_DEVICE_PTRS is implied) and the
 * launches go to `stream` (NULL = the legacy default stream) on the current
 * device, without xts_init.  The King and psf*aeff scratch tables live in one
 * fixed 8 MiB device array that the library holds on every GPU that loads it
 * until the process exits: shapes needing more than XTS_NOALLOC_SCRATCH_DOUBLES
 * doubles, 401 * (Mc*Me front + Mc*Me back) rounded up to a multiple of 32, plus
 * C * 401 * E, fail with XTS_ERR_ARG and launch nothing.  All calls share that
 * array and the last call's contents stay in it; calls that overlap on the GPU
 * race on it, so order them on one stream.  The first call on a device looks the
 * array up (cudaGetSymbolAddress) and must come before any stream capture (on a
 * capturing stream it is refused with XTS_ERR_ARG); the looked-up address is not
 * valid after cudaDeviceReset. */
#define XTS_NOALLOC_SCRATCH_DOUBLES (1u << 20)
int xts_compute_psf_data_noalloc(const xts_grid* psf_front, const xts_grid* psf_back,
                                 const double* exp_costhetas, int C, const double* logEs,
                                 int E, const double* front_aeff, const double* back_aeff,
                                 const double* src_exposure_cosbins,
                                 const double* src_weighted_exposure_cosbins, int S,
                                 const double* front_ltf, const double* exposure,
                                 double* upsf, double* partial, void* stream);

/* ModelMap::point_src_model_map_wcs (model_map/model_map.point_src_model_map_wcs.cxx:6-45,
 * reached from ModelMap::compute_srcmaps<PointSource>, model_map.compute_src_maps.cxx:6-22):
 * steps c1-c10 and d1.  model_map is [S, H, W, E], float unless XTS_OUT_F64. */
int xts_point_src_model_map_wcs(const xts_wcs* wcs, const double* src_sph, int S,
                                const double* exposure, const double* upsf,
                                const double* partial, int E, void* model_map,
                                xts_srcmap_info* info, unsigned flags, void* stream);

/* Per-source cutouts (no counterpart in the reference, which writes every source's
 * map over the whole H x W grid, model_map/mm_cubature/cubature.implementation.cxx:33):
 * source s's map covers the window of rows h0 .. h0 + nh - 1 and columns
 * w0 .. w0 + nw - 1 of the map, stored [nh][nw][E] from value offset * E of a
 * ragged output (offset = the pixels of all earlier windows). */
typedef struct xts_cutout {
    int h0, w0, nh, nw;
    long long offset;
} xts_cutout;

/* Cutout windows for radii radius_deg [S]: the source's pixel (p1, p2) =
 * sph2pix(src) (1-based), n = ceil(radius / |CDELTn|), rows round(p1) - 1 - n ..
 * round(p1) - 1 + n clipped to the map (columns likewise; an empty window when the
 * clipped range is empty).  Host pointers; total_pixels = the sum of nh * nw. */
int xts_cutout_windows(const xts_wcs* wcs, const double* src_sph, const double* radius_deg, int S,
                       xts_cutout* cut, long long* total_pixels);

/* ModelMap::point_src_model_map_wcs (model_map/model_map.point_src_model_map_wcs.cxx:6-45)
 * on per-source cutouts: source s's map is the reference's model map of the
 * sub-map its window describes (the WCS with CRPIX shifted by the window's origin):
 * its boundary radius and in-FOV flag (3.5 pixel buffer) are those of the window,
 * its map integral runs over the window's pixels within that radius, and the
 * correction follows from them (model_map.psf_boundary_radius.cxx:9-62,
 * model_map.map_integral.cxx:4-48, model_map.map_correction_factor.cxx:3-53).
 * model_map is float [sum of nh * nw, E] in source order (cut[s].offset); cut is
 * [S] (device with XTS_DEVICE_PTRS).  The window pass runs as one persistent launch
 * over a work queue of (source, 256-pixel tile) items, the write pass as one
 * persistent launch over the same items. */
int xts_point_src_model_map_cutouts(const xts_wcs* wcs, const double* src_sph, int S, const xts_cutout* cut,
                                    const double* exposure, const double* upsf, const double* partial, int E,
                                    float* model_map, xts_srcmap_info* info, unsigned flags, void* stream);

/* The model map of xts_point_src_model_map_wcs with adaptive cubature of each
 * pixel in place of the fixed 12-point rule: the Genz-Malik degree-7/5 rule on
 * the pixel (17 points), regions halved along the dimension with the larger
 * fourth difference until max_e |R5 - R7| / |R7| <= rtol or max_depth levels.
 * This is the design of the reference's uncompiled math/genz_malik.hxx:18-195,
 * math/genz_malik.cxx:66-217 and model_map/model_map.pixel_mean_psf_genz.cxx:21-108,
 * with rectangular sub-regions and the estimate kept at the depth limit.  The
 * map is float [S, H, W, E]; rtol in [1e-6, 1], max_depth in [0, 16] (the
 * reference's design uses 6); only XTS_DEVICE_PTRS applies. */
int xts_point_src_model_map_wcs_adaptive(const xts_wcs* wcs, const double* src_sph, int S,
                                         const double* exposure, const double* upsf,
                                         const double* partial, int E, double rtol, int max_depth,
                                         float* model_map, xts_srcmap_info* info, unsigned flags,
                                         void* stream);

/* The three calls of xtsrcmaps/main.cxx:28-30 in one: Exposure::compute_exposure
 * (exposure/exposure.hxx:44-88), Psf::compute_psf_data (psf/psf.compute_psf_data.cxx:7-33)
 * and ModelMap::compute_srcmaps<PointSource> (model_map/model_map.compute_src_maps.cxx:6-22),
 * with the exposure and mean-PSF tables kept in device memory between the steps.
 * Inputs are those of xts_compute_exposure plus the normalised King grids of
 * xts_compute_psf_data and the map WCS; outputs those of
 * xts_point_src_model_map_wcs.  With host pointers the maps are copied out in
 * chunks of sources while later chunks are still being computed. */
int xts_point_source_maps(const xts_expcube* exp_cube, const xts_expcube* wexp_cube,
                          const double* logEs, int E, const double* src_sph, int S,
                          const xts_grid* aeff_front, const xts_grid* aeff_back,
                          const xts_grid* psf_front, const xts_grid* psf_back,
                          const double* front_ltf, const xts_wcs* wcs, void* model_map,
                          xts_srcmap_info* info, unsigned flags, void* stream);

/* Fermi::fits::write_src_model (xtsrcmaps/fits/fits.write_src_model.cxx:10-66, the
 * commented-out call at main.cxx:40): the maps [S, H, W, E] (float, or double with
 * XTS_OUT_F64) written to a FITS file.  Primary HDU without data, HDUNAME =
 * 'PRIMARY'; then per source an IMAGE extension, EXTNAME = names[s] (NULL names
 * or entries: "SRC%05d"), NAXIS1 = H, NAXIS2 = W, NAXIS3 = E holding
 * img[e][w][h] = map[s][h][w][e] (the reference's SHWE -> SEHW reorder), BITPIX
 * -64 (XTS_FITS_F32: -32), with CHECKSUM and DATASUM.  The reorder, conversion,
 * byte order and data sums run on the device; the file is complete when the call
 * returns.  XTS_DEVICE_PTRS: model_map is a device pointer.  Names: printable
 * ASCII, at most 68 characters (a quote counts twice). */
int xts_write_src_model(const char* filename, const void* model_map, int S, int H, int W, int E,
                        const char* const* names, unsigned flags, void* stream);

/* Psf::make_kernel (psf/psf.make_kernel.cpp:8-90), a step of the reference's
 * work-in-progress diffuse-source map: the mean PSF of one source (upsf [401, E],
 * one source's slice of the uPsf table) sampled at the centres (h + 1, w + 1) of an
 * Nk x Nk grid described by kernel_wcs, by separation from the grid's reference
 * point (CRVAL), with the row and weight of the point-source cubature's logsep rule;
 * each energy plane normalised to unit sum.  kernel is [E, Nk, Nk], Nk odd.  The
 * reference weights the lower row by t and the upper by 1 - t there
 * (make_kernel.cpp:43-45), the reverse of its cubature; this uses the cubature's
 * (1 - t, t). */
int xts_make_psf_kernel(const xts_wcs* kernel_wcs, int Nk, const double* upsf, int E, double* kernel,
                        unsigned flags, void* stream);

/* FFT::convolve_map_psf (model_map/mm_fft/fft.convolve_map_psf.cpp:7-43, over
 * fftw_convolve_3d, math/convolve/fft/fft.fftw_convolve_CHW.cpp:7-90): for every
 * energy plane the full linear 2-D convolution of image [E, H, W] with kernel
 * [E, K, K], out [E, H + K - 1, W + K - 1], FP64, by cuFFT.  The reference's
 * transform is 3-D over (energy, h, w) and its scale factor is misparenthesised;
 * this is the per-plane convolution those lines are written for. */
int xts_convolve_map_psf(const double* image, int E, int H, int W, const double* kernel, int K, double* out,
                         unsigned flags, void* stream);

/* rebin_wcs_config (sky_geom/sky_geom.hxx:352-371, through rebin_skygeom :373-377), a
 * step of the diffuse-source map: the WCS of the same region at pixel size
 * target_pix_size (deg): CDELTn = +-target with the input's signs, NAXISn =
 * round(NAXISn * |CDELTn_in| / target), CRPIXn scaled by the same factor, the
 * rest unchanged.  The reference stores CRPIX2 into CDELT2 (:367); this writes the
 * rebinned CDELT2.  Host function (no device work). */
int xts_rebin_wcs(const xts_wcs* in, double target_pix_size, xts_wcs* out);

/* The all-sky pixel range of fits::read_allsky_cropped
 * (fits/fits.read_allsky_cropped.cpp:150-194): the ROI pixels (1, 1) and (NAXIS1,
 * NAXIS2) through the ROI WCS, longitude wrapped into [0, 360) and latitude clamped,
 * then through the all-sky WCS, rounded and bounded to [1, NAXISn].  range =
 * {x_first, x_last, y_first, y_last}, 1-based and inclusive (first = min, last =
 * max, as the reference).  Host function. */
int xts_allsky_crop_range(const xts_wcs* allsky_wcs, const xts_wcs* roi_wcs, long range[4]);

/* The block of an all-sky cube allsky [E0][NY][NX] (NAXIS1 = NX fastest) inside
 * range: out [E0][ny][nx], ny = y_last - y_first + 1, nx = x_last - x_first + 1, or,
 * for x_first > x_last, the columns x_first..NX then 1..x_last across the image's
 * longitude seam (what readSegmentsAcrossBoundary, fits.read_allsky_cropped.cpp:119-147,
 * is written for).  FP32 as the FITS image. */
int xts_crop_allsky(const float* allsky, int E0, long NY, long NX, const long range[4], float* out,
                    unsigned flags, void* stream);

/* Fermi::math::trilerpEHW (math/trilerp.hpp:7-59): trilinear resampling of src
 * [E0][H0][W0] onto dst [E1][H1][W1] with corner-aligned axes (scale (n0 - 1) /
 * (n1 - 1); 0 where n1 = 1, which the reference divides by), FP32 arithmetic in the
 * reference's order (h, then w, then e). */
int xts_trilerp_ehw(const float* src, int E0, int H0, int W0, float* dst, int E1, int H1, int W1,
                    unsigned flags, void* stream);

/* The final scalings of ModelMap::diffuse_src_model_map_wcs
 * (model_map/model_map.diffuse_src_model_map_wcs.cxx:76-95), which are those of
 * point_src_model_map_wcs after its cubature (model_map.point_src_model_map_wcs.cxx:24-42):
 * model_map [S, H, W, E] float holds pixel means on entry; on return
 * mean * solid angle * exposure * correction, with the map integral over the
 * pixels whose centre lies within each source's boundary radius (c6, c7) and the
 * containment correction (c9) as the point-source path computes them. */
int xts_scale_model_map(const xts_wcs* wcs, const double* src_sph, int S, const double* exposure,
                        const double* upsf, const double* partial, int E, float* model_map,
                        xts_srcmap_info* info, unsigned flags, void* stream);

/* Learned surrogate of the pixel cubature ---------------------------------------
 * No counterpart in the reference.  A multilayer perceptron 5 -> 128 -> 128 ->
 * 128 -> 1 with tanh-form GELU after each hidden layer maps five features of a
 * (source, pixel, energy) value to y = ln(m / u_c) * rho^2, where m is the
 * 12-point rule mean of the mean PSF over the pixel (the quantity of
 * cubature_convolve_map_psf, model_map/mm_cubature/cubature.implementation.cxx:21-55,
 * before the solid angle), u_c the mean PSF at the pixel centre and rho the
 * centre's separation in pixel sizes.  Features, in order: log10 rho; the
 * centre's offset between the two rows of the 401-row separation table that
 * bracket it (its logsep interpolation weight); log10 of the pixel's solid angle
 * in deg^2; log10 of the energy in MeV; the log slope ln(U[i] / U[i-1]) / step
 * of the mean PSF's table segment holding the centre.  The hidden layers run on tcgen05 tensor
 * cores with BF16 operands and FP32 accumulators in tensor memory; the input and
 * output layers and the GELUs on CUDA cores in FP32 (weights rounded to BF16).
 * All pointers are device pointers on the library's current device. */
#define XTS_MLP_IN 5
#define XTS_MLP_HID 128
#define XTS_MLP_W1 0                                     /* [128][5] */
#define XTS_MLP_B1 (XTS_MLP_W1 + XTS_MLP_HID * XTS_MLP_IN)  /* [128] */
#define XTS_MLP_W2 (XTS_MLP_B1 + XTS_MLP_HID)                /* [128 out][128 in] */
#define XTS_MLP_B2 (XTS_MLP_W2 + XTS_MLP_HID * XTS_MLP_HID)
#define XTS_MLP_W3 (XTS_MLP_B2 + XTS_MLP_HID)
#define XTS_MLP_B3 (XTS_MLP_W3 + XTS_MLP_HID * XTS_MLP_HID)
#define XTS_MLP_W4 (XTS_MLP_B3 + XTS_MLP_HID)                /* [128] */
#define XTS_MLP_B4 (XTS_MLP_W4 + XTS_MLP_HID)                /* [1] */
#define XTS_MLP_NPARAM (XTS_MLP_B4 + 1)
#define XTS_MLP_CELL_NR 32
#define XTS_MLP_CELL_NS 16

typedef struct xts_mlp {
    float* params;          /* [XTS_MLP_NPARAM] FP32 master parameters (device) */
    unsigned short* wbf16;  /* [2][128][128] BF16 copies of W2 and W3 (device), kept by the update */
    float in_mu[XTS_MLP_IN], in_sd[XTS_MLP_IN];  /* feature standardisation x' = (x - mu) / sd */
    float out_mu, out_sd;                       /* target standardisation */
    float lo[XTS_MLP_IN], hi[XTS_MLP_IN];       /* accepted feature range (the training range) */
    float rho_min;          /* centres closer than rho_min pixel sizes take the 12-point rule */
    /* Error cells: feature 0 (log10 rho) in XTS_MLP_CELL_NR bins over [cell_lo[0], cell_hi[0]]
     * times feature 4 (segment log slope) in XTS_MLP_CELL_NS bins over [cell_lo[1], cell_hi[1]].
     * cell_ok (device, [XTS_MLP_CELL_NR * XTS_MLP_CELL_NS]) holds 1 in cell i * XTS_MLP_CELL_NS + j
     * where the network's largest relative error on held-out samples of that cell stayed
     * within the bound it was calibrated for; the network takes a value only in such a
     * cell.  NULL: no cell restriction. */
    float cell_lo[2], cell_hi[2];
    const unsigned char* cell_ok;
} xts_mlp;

/* C = A B^T in FP32 from BF16 operands on tcgen05: A [M][K] (a_trans: stored
 * [K][M]), B [128][K] (b_trans: stored [K][128]), C [M][128] (c_trans: stored
 * [128][M]); M a multiple of 128, K of 64.  accumulate: C += A B^T (atomic
 * adds, K split over the blocks), else C = A B^T. */
int xts_gemm_bf16(const unsigned short* A, int a_trans, const unsigned short* B, int b_trans, int M, int K,
                  float* C, int c_trans, int accumulate, void* stream);

/* Network output y (de-standardised) for n feature rows X [n][5]. */
int xts_mlp_forward(const xts_mlp* net, const float* X, long long n, float* y, void* stream);

/* Gradient of the loss L = (1/n) sum (y' - (Y - out_mu) / out_sd)^2 (y' the
 * standardised output) with respect to the FP32 parameters, grads
 * [XTS_MLP_NPARAM] (overwritten); loss [1] (may be NULL).  n a multiple of 128, at most
 * 2^24 rows per call. */
int xts_mlp_grads(const xts_mlp* net, const float* X, const float* Y, long long n, float* grads, float* loss,
                  void* stream);

/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on a batch: grads, adam_m,
 * adam_v [XTS_MLP_NPARAM] (grads zero on entry, left zero), step >= 1; the BF16
 * copies are refreshed.  loss [1] accumulates the batch loss (may be NULL).  n as for
 * xts_mlp_grads. */
int xts_mlp_train_step(const xts_mlp* net, const float* X, const float* Y, long long n, float* grads,
                       float* adam_m, float* adam_v, int step, float lr, float* loss, void* stream);

/* Training samples from mean-PSF tables upsf [S][401][E] and energies logEs [E]:
 * per sample a source, an energy, a separation log-uniform in
 * [max(0.001, rho_min * size), 30] deg, a pixel of size uniform in [0.025, 0.2]
 * deg with aspect ratio in [0.8, 1.25] and a uniform orientation, placed on the
 * sphere; X [n][5] its features and Y [n] its target, both from the FP64 rule
 * the model map uses (a hash of seed and sample index drives every draw). */
int xts_surrogate_samples(const double* upsf, const double* logEs, int S, int E, long long n,
                          unsigned long long seed, double rho_min, float* X, float* Y, void* stream);

/* Counts of a surrogate model map. */
typedef struct xts_surrogate_stats {
    long long values;        /* S * H * W * E */
    long long accepted;      /* values served by the network (maps that passed the check, checked pixels excluded) */
    long long checked;       /* values the network took in the checked pixels, where the 12-point rule's stay */
    int maps_fallback;       /* sources whose check failed: all their values by the rule */
    float max_check_err;     /* largest relative difference seen by the check */
    long long evaluated;     /* rows the network evaluated (before the check) */
} xts_surrogate_stats;

/* The model map of xts_point_src_model_map_wcs with the pixel means taken from
 * the network wherever the centre lies at least rho_min pixel sizes from the
 * source, every feature is inside [lo, hi] and the value's error cell is marked
 * cell_ok; the other values take the 12-point rule (the plain map's FP32 window
 * and write passes over the unscaled mean PSF for E <= 52, the FP64 rule per value
 * above).  At every 16th pixel the rule's values stay and the network's are
 * compared with them; a source whose largest relative difference there exceeds
 * check_tol is redone entirely by the FP64 rule.  Map integral, correction and scalings as
 * xts_point_src_model_map_wcs.  Device pointers; model_map float [S, H, W, E].
 * With stats NULL the call neither synchronises nor allocates once its buffers
 * have grown (it can be captured into a CUDA graph); xts_surrogate_last_stats
 * then gives the counts of the latest call, and with stats given they are
 * filled before the call returns. */
int xts_point_src_model_map_wcs_surrogate(const xts_wcs* wcs, const double* src_sph, int S,
                                          const double* exposure, const double* upsf,
                                          const double* partial, const double* logEs, int E,
                                          const xts_mlp* net,
                                          double check_tol, float* model_map, xts_srcmap_info* info,
                                          xts_surrogate_stats* stats, void* stream);

/* xts_point_source_maps with the model map of the surrogate
 * (xts_point_src_model_map_wcs_surrogate) in place of the plain cubature: the
 * three calls of main.cxx:28-30 in one, FP32 maps.  Host or device pointers as
 * xts_point_source_maps (flags XTS_DEVICE_PTRS); with host pointers the map is
 * copied to the host in about eight groups of sources, each group finished
 * (checks, map integral, correction, scaling) and copied while the next is
 * computed.  stats: as xts_point_src_model_map_wcs_surrogate. */
int xts_point_source_maps_surrogate(const xts_expcube* exp_cube, const xts_expcube* wexp_cube,
                                    const double* logEs, int E, const double* src_sph, int S,
                                    const xts_grid* aeff_front, const xts_grid* aeff_back,
                                    const xts_grid* psf_front, const xts_grid* psf_back,
                                    const double* front_ltf, const xts_wcs* wcs, const xts_mlp* net,
                                    double check_tol, float* model_map, xts_srcmap_info* info,
                                    xts_surrogate_stats* stats, unsigned flags, void* stream);

/* Counts of the latest xts_point_src_model_map_wcs_surrogate call on the
 * library's device (waits for that call's work on `stream`); XTS_ERR_TIMEOUT if
 * one of its bounded tensor-core waits gave up. */
int xts_surrogate_last_stats(xts_surrogate_stats* stats, void* stream);

#ifdef __cplusplus
}
#endif
#endif
