// xts_diffuse.cu -- the two numeric steps of the reference's diffuse-source model
// map (model_map/model_map.diffuse_src_model_map_wcs.cxx:8-97, work in progress
// there and commented out of main.cxx): the PSF kernel image of one mean PSF
// (Psf::make_kernel, psf/psf.make_kernel.cpp:8-90) and the per-energy convolution
// of a map cube with it (FFT::convolve_map_psf, model_map/mm_fft/fft.convolve_map_psf.cpp:7-43,
// over fftw_convolve_3d, math/convolve/fft/fft.fftw_convolve_CHW.cpp:7-90).
//
// Kernel image: one thread per kernel pixel evaluates the FP64 separation of the
// pixel centre (h + 1, w + 1) from the grid's reference direction, the LUT row and
// weight of the keys-fixed logsep rule (row clamped to 400, extrapolated below
// 1e-4 deg), and the interpolated mean PSF for every energy; a second pass
// normalises each energy plane to unit sum (FP64 sums in a fixed order).
//
// Convolution: the full linear convolution, [E, H + K - 1, W + K - 1] as the
// reference returns it, computed per energy plane with cuFFT: both operands are
// zero-padded into one batched real-to-complex transform of a size whose factors
// are 2, 3, 5 and 7, the spectra are multiplied (with the 1 / (NH * NW) of the
// inverse transform folded in) by a kernel of this file, and the inverse
// transform's plane is cropped.  Two defects of the reference's work-in-progress
// code are not reproduced: its transform is 3-D over (energy, h, w), which mixes
// energy planes, and its normalisation `1.0 / paddedH * paddedW * C` multiplies
// where it means to divide.
//
// The steps before them: the all-sky cube's block under the ROI
// (fits::read_allsky_cropped, fits/fits.read_allsky_cropped.cpp:150-230: the
// pixel range on the host, the block gathered on the device, wrapped at the
// image's longitude seam as readSegmentsAcrossBoundary :119-147 intends), the
// WCS at the target pixel size (rebin_wcs_config, sky_geom/sky_geom.hxx:352-371)
// and the trilinear resampling onto it (Fermi::math::trilerpEHW,
// math/trilerp.hpp:7-59, in FP32 as the reference's float tensors).
#include <cufft.h>
#include <math.h>

#include "xts_geom.cuh"
#include "xts_internal.cuh"

namespace xts {

// -------------------------------------------------------------- kernel image
__global__ void k_psf_kernel(WcsDev w, double rx, double ry, double rz, int Nk, const double* __restrict__ upsf,
                             int E, double* __restrict__ kernel) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= Nk * Nk) return;
    const int h = k / Nk, wc = k - h * Nk;
    double d[3];
    pix2dir(w, h + 1.0, wc + 1.0, d);
    const double ref[3] = {rx, ry, rz};
    const double s = R2D * dir_diff(ref, d);  // degrees (SkyGeom::srcpixoff)
    const double j = s < 1e-4 ? 1.0 : 1.0 + RECIPSTEP * (LN_1E4 + log(s));
    int i = 1 + (int)j;
    i = i > 400 ? 400 : (i < 2 ? 2 : i);
    const double t = REDM1 * (s * 1e4 * exp(SEP_STEP * (2. - i)) - 1.);
    const double* yl = upsf + (size_t)(i - 1) * E;
    const double* yr = upsf + (size_t)i * E;
    for (int e = 0; e < E; ++e) kernel[((size_t)e * Nk + h) * Nk + wc] = (1.0 - t) * yl[e] + t * yr[e];
}

// One block per energy plane: sum in a fixed order, then scale to unit sum.
__global__ void __launch_bounds__(256) k_kernel_normalise(double* kernel, int n) {
    __shared__ double red[8];
    double* p = kernel + (size_t)blockIdx.x * n;
    double s = 0.;
    for (int k = threadIdx.x; k < n; k += blockDim.x) s += p[k];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    double tot = 0.;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) tot += red[k];
    const double inv = 1.0 / tot;
    for (int k = threadIdx.x; k < n; k += blockDim.x) p[k] *= inv;
}

int make_psf_kernel(const xts_wcs& wcs, int Nk, const double* upsf, int E, double* kernel, cudaStream_t st) {
    const WcsDev w = make_wcs(wcs);
    double rd[3];
    sph2dir(wcs.crval1, wcs.crval2, rd);  // SkyGeom::refdir(): the reference point
    const int n = Nk * Nk;
    XTS_LAUNCH("k_psf_kernel", st, k_psf_kernel<<<(n + 127) / 128, 128, 0, st>>>(w, rd[0], rd[1], rd[2], Nk, upsf, E,
                                                                                 kernel));
    XTS_LAUNCH("k_kernel_normalise", st, k_kernel_normalise<<<E, 256, 0, st>>>(kernel, n));
    return XTS_OK;
}

// -------------------------------------------------------------- convolution
static int fft_size(int n) {  // smallest m >= n whose prime factors are 2, 3, 5 and 7
    for (int m = n;; ++m) {
        int r = m;
        for (int p : {2, 3, 5, 7})
            while (r % p == 0) r /= p;
        if (r == 1) return m;
    }
}

// Zero-padded copies of the image planes and the kernel planes, [E][NH][NW] each.
__global__ void k_fft_pad(const double* __restrict__ image, int H, int W, const double* __restrict__ kernel, int K,
                          int NH, int NW, double* __restrict__ pimg, double* __restrict__ pker, long long total) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= total) return;
    const long long plane = (long long)NH * NW;
    const int e = (int)(k / plane);
    const int r = (int)(k - (long long)e * plane), i = r / NW, j = r - i * NW;
    pimg[k] = (i < H && j < W) ? image[((size_t)e * H + i) * W + j] : 0.0;
    pker[k] = (i < K && j < K) ? kernel[((size_t)e * K + i) * K + j] : 0.0;
}

__global__ void k_fft_cmul(double2* __restrict__ a, const double2* __restrict__ b, long long n, double scale) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const double2 x = a[k], y = b[k];
    a[k] = make_double2((x.x * y.x - x.y * y.y) * scale, (x.x * y.y + x.y * y.x) * scale);
}

__global__ void k_fft_crop(const double* __restrict__ r, int NH, int NW, int PH, int PW, double* __restrict__ out,
                           long long total) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= total) return;
    const long long plane = (long long)PH * PW;
    const int e = (int)(k / plane);
    const int q = (int)(k - (long long)e * plane), i = q / PW, j = q - i * PW;
    out[k] = r[((size_t)e * NH + i) * NW + j];
}

struct FftPlans {
    int NH = 0, NW = 0, E = 0, device = -1;
    cufftHandle fwd = 0, inv = 0;
    bool ok = false;
};
static FftPlans g_fft;

static int fft_plans(int NH, int NW, int E, size_t* work) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (!(g_fft.ok && g_fft.NH == NH && g_fft.NW == NW && g_fft.E == E && g_fft.device == dev)) {
        if (g_fft.ok) {
            cufftDestroy(g_fft.fwd);
            cufftDestroy(g_fft.inv);
            g_fft.ok = false;
        }
        int n[2] = {NH, NW};
        const int NC = NW / 2 + 1;
        int inembed[2] = {NH, NW}, onembed[2] = {NH, NC};
        size_t w1 = 0, w2 = 0;
        if (cufftCreate(&g_fft.fwd) != CUFFT_SUCCESS || cufftCreate(&g_fft.inv) != CUFFT_SUCCESS)
            return set_error(XTS_ERR_CUDA, "cufftCreate failed");
        cufftSetAutoAllocation(g_fft.fwd, 0);
        cufftSetAutoAllocation(g_fft.inv, 0);
        if (cufftMakePlanMany(g_fft.fwd, 2, n, inembed, 1, NH * NW, onembed, 1, NH * NC, CUFFT_D2Z, E, &w1) !=
                CUFFT_SUCCESS ||
            cufftMakePlanMany(g_fft.inv, 2, n, onembed, 1, NH * NC, inembed, 1, NH * NW, CUFFT_Z2D, E, &w2) !=
                CUFFT_SUCCESS) {
            cufftDestroy(g_fft.fwd);
            cufftDestroy(g_fft.inv);
            return set_error(XTS_ERR_CUDA, "cufftMakePlanMany failed (%d x %d, batch %d)", NH, NW, E);
        }
        g_fft.NH = NH; g_fft.NW = NW; g_fft.E = E; g_fft.device = dev; g_fft.ok = true;
        *work = w1 > w2 ? w1 : w2;
        return XTS_OK;
    }
    size_t w1 = 0, w2 = 0;
    cufftGetSize(g_fft.fwd, &w1);
    cufftGetSize(g_fft.inv, &w2);
    *work = w1 > w2 ? w1 : w2;
    return XTS_OK;
}

// Buffers: A holds the padded image planes, then the kernel spectrum; B the padded
// kernel planes, then the inverse transform; C the image spectrum.
int convolve_map_psf(const double* image, int E, int H, int W, const double* kernel, int K, double* out,
                     cudaStream_t st) {
    const int PH = H + K - 1, PW = W + K - 1;
    const int NH = fft_size(PH), NW = fft_size(PW), NC = NW / 2 + 1;
    size_t work = 0;
    int rc = fft_plans(NH, NW, E, &work);
    if (rc) return rc;
    const size_t real_n = (size_t)E * NH * NW, cplx_n = (size_t)E * NH * NC;
    double* A = (double*)workspace(W_FFT_A, sizeof(double2) * cplx_n);
    double* B = (double*)workspace(W_FFT_B, sizeof(double) * real_n);
    double2* C = (double2*)workspace(W_FFT_C, sizeof(double2) * cplx_n);
    void* wk = workspace(W_FFT_WORK, work ? work : 16);
    if (!A || !B || !C || !wk) return XTS_ERR_OOM;
    if (cufftSetWorkArea(g_fft.fwd, wk) != CUFFT_SUCCESS || cufftSetWorkArea(g_fft.inv, wk) != CUFFT_SUCCESS ||
        cufftSetStream(g_fft.fwd, st) != CUFFT_SUCCESS || cufftSetStream(g_fft.inv, st) != CUFFT_SUCCESS)
        return set_error(XTS_ERR_CUDA, "cufft work area or stream");
    const long long rt = (long long)real_n, cn = (long long)cplx_n, on = (long long)E * PH * PW;
    XTS_LAUNCH("k_fft_pad", st, k_fft_pad<<<(unsigned)((rt + 255) / 256), 256, 0, st>>>(image, H, W, kernel, K, NH, NW,
                                                                                      A, B, rt));
    if (cufftExecD2Z(g_fft.fwd, A, C) != CUFFT_SUCCESS) return set_error(XTS_ERR_CUDA, "cufftExecD2Z (image)");
    if (cufftExecD2Z(g_fft.fwd, B, (double2*)A) != CUFFT_SUCCESS)
        return set_error(XTS_ERR_CUDA, "cufftExecD2Z (kernel)");
    XTS_LAUNCH("k_fft_cmul", st, k_fft_cmul<<<(unsigned)((cn + 255) / 256), 256, 0, st>>>(
                                     C, (const double2*)A, cn, 1.0 / ((double)NH * NW)));
    if (cufftExecZ2D(g_fft.inv, C, B) != CUFFT_SUCCESS) return set_error(XTS_ERR_CUDA, "cufftExecZ2D");
    XTS_LAUNCH("k_fft_crop", st, k_fft_crop<<<(unsigned)((on + 255) / 256), 256, 0, st>>>(B, NH, NW, PH, PW, out, on));
    return XTS_OK;
}

// -------------------------------------------------------------- all-sky crop
// fits.read_allsky_cropped.cpp:155-194: the ROI's pixels (1, 1) and (NAXIS1,
// NAXIS2) to (lon, lat), longitude wrapped into [0, 360) and latitude clamped,
// to all-sky pixels, rounded and bounded to [1, NAXISn]; first = min, last = max.
int allsky_crop_range(const xts_wcs& sky, const xts_wcs& roi, long range[4]) {
    const WcsDev ws = make_wcs(sky), wr = make_wcs(roi);
    double lon[2], lat[2], px[2], py[2];
    pix2sph(wr, 1.0, 1.0, &lon[0], &lat[0]);
    pix2sph(wr, (double)roi.naxis1, (double)roi.naxis2, &lon[1], &lat[1]);
    for (int k = 0; k < 2; ++k) {
        lon[k] = fmod(lon[k] + 360.0, 360.0);
        lat[k] = lat[k] > 90.0 ? 90.0 : (lat[k] < -90.0 ? -90.0 : lat[k]);
        sph2pix(ws, lon[k], lat[k], &px[k], &py[k]);
    }
    auto bound = [](double v, long mx) {
        const long r = lround(v);
        return r < 1 ? 1L : (r > mx ? mx : r);
    };
    range[0] = bound(px[0] < px[1] ? px[0] : px[1], sky.naxis1);
    range[1] = bound(px[0] < px[1] ? px[1] : px[0], sky.naxis1);
    range[2] = bound(py[0] < py[1] ? py[0] : py[1], sky.naxis2);
    range[3] = bound(py[0] < py[1] ? py[1] : py[0], sky.naxis2);
    return XTS_OK;
}

// out[e][y][x] = allsky[e][y0 + y][(x0 + x) mod NX] (0-based x0 = range[0] - 1):
// columns past the image's last column continue at its first (the seam).
__global__ void k_crop_allsky(const float* __restrict__ sky, long NY, long NX, long x0, long y0, long nx, long ny,
                              long long total, float* __restrict__ out) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= total) return;
    const long long plane = (long long)nx * ny;
    const long long e = k / plane;
    const long long r = k - e * plane;
    const long y = (long)(r / nx), x = (long)(r - (long long)y * nx);
    long xs = x0 + x;
    if (xs >= NX) xs -= NX;
    out[k] = sky[((size_t)e * NY + (y0 + y)) * NX + xs];
}

int crop_allsky(const float* sky, int E0, long NY, long NX, const long range[4], float* out, cudaStream_t st) {
    const long x0 = range[0] - 1, y0 = range[2] - 1;
    const long nx = range[1] >= range[0] ? range[1] - range[0] + 1 : NX - range[0] + 1 + range[1];
    const long ny = range[3] - range[2] + 1;
    const long long total = (long long)E0 * nx * ny;
    if (total == 0) return XTS_OK;
    XTS_LAUNCH("k_crop_allsky", st, k_crop_allsky<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(
                                        sky, NY, NX, x0, y0, nx, ny, total, out));
    return XTS_OK;
}

// -------------------------------------------------------------- trilinear resampling
// math/trilerp.hpp:7-59 in FP32: corner-aligned scales (src - 1) / (dst - 1) per
// axis (0 when dst is 1, where the reference divides by zero), lower index
// floor(k * scale), upper index min(lower + 1, src - 1); h, then w, then e.
__global__ void k_trilerp_ehw(const float* __restrict__ src, int E0, int H0, int W0, float* __restrict__ dst,
                              int E1, int H1, int W1, float se, float sh, float sw) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long total = (long long)E1 * H1 * W1;
    if (k >= total) return;
    const int j = (int)(k % W1);
    const int i = (int)((k / W1) % H1);
    const int kk = (int)(k / ((long long)W1 * H1));
    const float e = (float)kk * se, h = (float)i * sh, w = (float)j * sw;
    const int e0 = (int)e, h0 = (int)h, w0 = (int)w;
    const int e1 = min(e0 + 1, E0 - 1), h1 = min(h0 + 1, H0 - 1), w1 = min(w0 + 1, W0 - 1);
    const float fe = e - (float)e0, fh = h - (float)h0, fw = w - (float)w0;
    const float ce = 1.f - fe, ch = 1.f - fh, cw = 1.f - fw;
    auto at = [&](int a, int b, int c) { return src[((size_t)a * H0 + b) * W0 + c]; };
    const float c00 = ch * at(e0, h0, w0) + fh * at(e0, h1, w0);
    const float c01 = ch * at(e1, h0, w0) + fh * at(e1, h1, w0);
    const float c10 = ch * at(e0, h0, w1) + fh * at(e0, h1, w1);
    const float c11 = ch * at(e1, h0, w1) + fh * at(e1, h1, w1);
    const float c0 = cw * c00 + fw * c10;
    const float c1 = cw * c01 + fw * c11;
    dst[k] = ce * c0 + fe * c1;
}

int trilerp_ehw(const float* src, int E0, int H0, int W0, float* dst, int E1, int H1, int W1, cudaStream_t st) {
    auto scale = [](int a, int b) { return b > 1 ? (float)(a - 1) / (float)(b - 1) : 0.f; };
    const long long total = (long long)E1 * H1 * W1;
    if (total == 0) return XTS_OK;
    XTS_LAUNCH("k_trilerp_ehw", st, k_trilerp_ehw<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(
                                        src, E0, H0, W0, dst, E1, H1, W1, scale(E0, E1), scale(H0, H1), scale(W0, W1)));
    return XTS_OK;
}

// -------------------------------------------------------------- rebinned WCS
// sky_geom.hxx:352-371: CDELTn = +-target (the input's sign), scale_n = |CDELTn_in /
// CDELTn|, NAXISn = round(NAXISn_in * scale_n), CRPIXn = CRPIXn_in * scale_n; the
// reference writes CRPIX2 into CDELT2 (:367), the rebinned CDELT2 is written here.
int rebin_wcs(const xts_wcs& in, double target, xts_wcs* out) {
    *out = in;
    const double c1 = in.cdelt1 < 0. ? -target : target, c2 = in.cdelt2 < 0. ? -target : target;
    const double s1 = fabs(in.cdelt1 / c1), s2 = fabs(in.cdelt2 / c2);
    out->cdelt1 = c1;
    out->cdelt2 = c2;
    out->naxis1 = lround((double)in.naxis1 * s1);
    out->naxis2 = lround((double)in.naxis2 * s2);
    out->crpix1 = in.crpix1 * s1;
    out->crpix2 = in.crpix2 * s2;
    return XTS_OK;
}

}  // namespace xts
