// xts_exposure.cu -- step (a) of the point-source path (exposure) and the two
// IRF set-up routines that feed it (livetime-efficiency factors, King PSF
// normalisation).
//
//   a1 exp_costhetas        exposure/exposure.cxx:29-40
//   a2 src_cosbins (gather) exposure/exposure.cxx:42-63 + healpix/healpix.cxx:181-229
//   a3 aeff_value           irf/irf.aeff_value.cxx:11-55, math/bilerp.cxx:6-27
//   a4 LTF                  irf/irf.cxx:70-109
//   a5 exposure contraction exposure/exposure.cxx:159-263, exposure/exposure.contract.cpp:13-42
//   b1 normalize_rpsf       irf/irf.normalize_rpsf.cpp:11-61, irf/irf.hxx:22-77
#include <math.h>

#include "xts_geom.cuh"
#include "xts_internal.cuh"

namespace xts {

// math/bilerp.cxx:6-27: upper_bound index, weight and complement.  The
// reference asserts the value lies inside the grid; the index is clamped to the
// last interval here instead of reading past the end.
__device__ inline void lerp_pars(const double* g, int n, double v, bool has_lb, double lb,
                                 double* wgt, double* cmpl, int* idx) {
    if (has_lb && v < lb) { *wgt = 0.; *cmpl = 0.; *idx = 1; return; }
    int lo = 0, hi = n;  // first i with g[i] > v
    while (lo < hi) { int m = (lo + hi) >> 1; if (v < g[m]) hi = m; else lo = m + 1; }
    int i = lo < 1 ? 1 : (lo > n - 1 ? n - 1 : lo);
    double t = (v - g[i - 1]) / (g[i] - g[i - 1]);
    *wgt = t; *cmpl = 1. - t; *idx = i;
}

// a1 + a3: cos-theta bin centres and the front/back effective-area tables [C, E].
__global__ void k_exposure_tables(int C, double cosmin, int thetabin, const double* logEs, int E,
                                  xts_grid af, xts_grid ab, double* costh, double* front,
                                  double* back) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= C * E) return;
    int c = i / E, e = i - c * E;
    double f = ((double)c + 0.5) / C;
    f = thetabin ? f * f : f;
    double ct = 1. - f * (1. - cosmin);
    if (e == 0) costh[c] = ct;
    const xts_grid* gs[2] = {&af, &ab};
    double* outs[2] = {front, back};
    for (int k = 0; k < 2; ++k) {
        const xts_grid& g = *gs[k];
        double cw, cc, ew, ec; int ci, ei;
        lerp_pars(g.cosths, g.n_cos, ct, true, g.min_cos_theta, &cw, &cc, &ci);
        lerp_pars(g.logEs, g.n_e, logEs[e], false, 0., &ew, &ec, &ei);
        int Me = g.n_e;
        const double* P = g.params;
        double xx = cc * ec * P[(ci - 1) * Me + (ei - 1)];
        double xy = cc * ew * P[(ci - 1) * Me + ei];
        double yx = cw * ec * P[ci * Me + (ei - 1)];
        double yy = cw * ew * P[ci * Me + ei];
        outs[k][i] = 1e4 * (xx + xy + yx + yy);
    }
}

// The NESTED pixel of each source (exposure/exposure.cxx:42-63), -1 when the
// position is not finite.
__device__ __forceinline__ long long src_pixel(const double* src_sph, int s, long long nside) {
    const double theta = HALFPI - src_sph[2 * s + 1] * D2R;
    const double phi = D2R * src_sph[2 * s];
    const long long pix = ang2pix_nest(theta, phi, nside);
    return pix < 0 || pix >= 12 * nside * nside ? -1 : pix;
}

__global__ void k_src_pixels(const double* src_sph, int S, long long nside, long long* pix) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < S) pix[s] = src_pixel(src_sph, s, nside);
}

int launch_src_pixels(const double* src_sph, int S, long long nside, long long* pix, cudaStream_t st) {
    if (S > 0)
        XTS_LAUNCH("k_src_pixels", st, k_src_pixels<<<(S + 127) / 128, 128, 0, st>>>(src_sph, S, nside, pix));
    return XTS_OK;
}

// a2: livetime rows of each source's NESTED pixel, float -> double [S, C].  With
// `gathered` the cubes hold only those rows already, [S][C] in source order.
__global__ void k_src_cosbins(const double* src_sph, int S, const float* cube, const float* wcube,
                              long long nside, int C, int gathered, double* ecb, double* wecb) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S * C) return;
    int s = i / C, c = i - s * C;
    const long long pix = gathered ? s : src_pixel(src_sph, s, nside);
    if (pix < 0) {  // non-finite source position
        ecb[i] = wecb[i] = __longlong_as_double(0x7ff8000000000000ll);
        return;
    }
    ecb[i] = (double)cube[pix * C + c];
    wecb[i] = (double)wcube[pix * C + c];
}

// a5 on FP64 cores: E[s,e] = ((X.Af L0 + X.Ab L0) + W.Af L1) + W.Ab L1.
__global__ void k_exposure_f64(const double* ecb, const double* wecb, int S, int C,
                               const double* af, const double* ab, const double* ltf, int E,
                               double* out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S * E) return;
    int s = i / E, e = i - s * E;
    double ef = 0, wf = 0, eb = 0, wb = 0;
#pragma unroll 8
    for (int c = 0; c < C; ++c) {  // unrolled: eight rows of loads in flight, sums still in c order
        double x = ecb[s * C + c], w = wecb[s * C + c];
        double a = af[c * E + e], b = ab[c * E + e];
        ef = fma(x, a, ef); wf = fma(w, a, wf);
        eb = fma(x, b, eb); wb = fma(w, b, wb);
    }
    double l0 = ltf[e], l1 = ltf[E + e];
    out[i] = ((ef * l0 + eb * l0) + wf * l1) + wb * l1;
}

int launch_exposure_contract(const double* ecb, const double* wecb, int S, int C, const double* af,
                             const double* ab, const double* ltf, int E, double* out,
                             cudaStream_t st) {
    int n = S * E;
    if (n == 0) return XTS_OK;
    XTS_LAUNCH("k_exposure_f64", st, k_exposure_f64<<<(n + 127) / 128, 128, 0, st>>>(ecb, wecb, S, C, af, ab, ltf, E, out));
    return XTS_OK;
}

int launch_exposure(const ExposureDev& a, cudaStream_t st) {
    int n = a.C * a.E;
    XTS_LAUNCH("k_exposure_tables", st, k_exposure_tables<<<(n + 127) / 128, 128, 0, st>>>(a.C, a.cosmin, a.thetabin, a.logEs, a.E,
                                                      a.af, a.ab, a.exp_costhetas, a.front_aeff,
                                                      a.back_aeff));
    n = a.S * a.C;
    if (n > 0) {
        XTS_LAUNCH("k_src_cosbins", st, k_src_cosbins<<<(n + 127) / 128, 128, 0, st>>>(a.src_sph, a.S, a.cube, a.wcube, a.nside,
                                                      a.C, a.gathered ? 1 : 0, a.ecb, a.wecb));
    }
    return launch_exposure_contract(a.ecb, a.wecb, a.S, a.C, a.front_aeff, a.back_aeff, a.ltf, a.E,
                                    a.exposure, st);
}

// a4: piecewise-linear efficiency in log E.  Row 1 from p0, row 0 from p1, and
// the break offsets b1, b2 in float, as the reference's float parameters give.
__device__ inline double ltf_single(const float* p, double logE) {
    float a0 = p[0], b0 = p[1], a1 = p[2], lb1 = p[3], a2 = p[4], lb2 = p[5];
    float b1f = __fadd_rn(__fmul_rn(__fsub_rn(a0, a1), lb1), b0);
    float b2f = __fadd_rn(__fmul_rn(__fsub_rn(a1, a2), lb2), b1f);
    double b1 = b1f, b2 = b2f;
    return logE < lb1 ? (double)a0 * logE + (double)b0
         : logE < lb2 ? (double)a1 * logE + b1
                      : (double)a2 * logE + b2;
}

__global__ void k_ltf(const double* logEs, int E, const float* p0, const float* p1, double* out) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    out[E + e] = ltf_single(p0, logEs[e]);
    out[e] = ltf_single(p1, logEs[e]);
}

int launch_ltf(const double* logEs, int E, const float* p0, const float* p1, double* ltf,
               cudaStream_t st) {
    XTS_LAUNCH("k_ltf", st, k_ltf<<<(E + 63) / 64, 64, 0, st>>>(logEs, E, p0, p1, ltf));
    return XTS_OK;
}

// b1: King normalisation.  64-point Gauss-Legendre below 120 MeV, analytic
// integral to 90 degrees above (irf/irf.normalize_rpsf.cpp:39-61).
__constant__ double c_gl_nodes[64];
__constant__ double c_gl_weights[64];

__device__ inline double king_f(double u, double g) {
    if (g == 1) g = 1.001;
    return (1. - 1. / g) * pow(1. + u / g, -g);
}

__device__ inline double evaluate_king(double sep, double sf, const double* p) {  // irf/irf.hxx:22-45
    double ncore = p[0], ntail = p[1], score = p[2] * sf, stail = p[3] * sf;
    double rc = sep / score, uc = rc * rc / 2.;
    double rt = sep / stail, ut = rt * rt / 2.;
    return ncore * king_f(uc, p[4]) + ntail * ncore * king_f(ut, p[5]);
}

__device__ inline double base_integral(double radius, double sf, const double* p) {  // irf/irf.hxx:48-77
    double ncore = p[0], ntail = p[1], score = p[2] * sf, stail = p[3] * sf;
    double sep = radius * D2R;
    double rc = sep / score, uc = rc * rc / 2.;
    double rt = sep / stail, ut = rt * rt / 2.;
    double fc = 1. - pow(1. + uc / p[4], 1. - p[4]);
    double ft = 1. - pow(1. + ut / p[5], 1. - p[5]);
    return ncore * fc * TWOPI * score * score + ntail * ncore * ft * TWOPI * stail * stail;
}

__global__ void k_normalize_rpsf(double* params, int Mc, int Me, const double* glog, float sp0,
                                 float sp1, float si) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Mc * Me) return;
    int e = i % Me;
    double* p = params + (size_t)i * 6;
    double energy = pow(10.0, glog[e]);
    double tt = pow(energy * 1.e-2, (double)si);
    double sf = sqrt((double)sp0 * tt * tt + (double)sp1);
    double norm;
    if (energy < 120.) {
        double acc = 0.;
        for (int k = 0; k < 64; ++k) {
            double v = 45. * c_gl_nodes[k] + 45.;
            double x = evaluate_king(v * D2R, sf, p);
            double y = sin(v * D2R) * TWOPI * D2R;
            acc += c_gl_weights[k] * (x * y);
        }
        norm = acc * 45.;
    } else {
        norm = base_integral(90.0, sf, p);
    }
    p[0] /= norm;
    p[2] *= sf;
    p[3] *= sf;
    p[4] = p[4] == 1. ? 1.001 : p[4];
    p[5] = p[5] == 1. ? 1.001 : p[5];
}

// Gauss-Legendre nodes by Newton iteration on the Legendre recurrence
// (math/gauss_legendre.hxx:37-62), computed once on the host.
static int upload_gauss_legendre(cudaStream_t st) {
    static bool done = false;
    static int dev_done = -1;
    int dev = -1;
    cudaGetDevice(&dev);
    if (done && dev_done == dev) return XTS_OK;
    double nodes[64], wts[64];
    const int N = 64;
    for (int i = 1; i <= N; ++i) {
        double x = cos(PI * (i - 0.25) / (N + 0.5)), dp = 0.;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = x;
            for (int j = 2; j <= N; ++j) { double p2 = ((2 * j - 1) * x * p1 - (j - 1) * p0) / j; p0 = p1; p1 = p2; }
            dp = N * (x * p1 - p0) / (x * x - 1);
            double dx = p1 / dp;
            x -= dx;
            if (fabs(dx) <= 1e-15) break;
        }
        nodes[i - 1] = x;
        wts[i - 1] = 2.0 / ((1. - x * x) * dp * dp);
    }
    XTS_CUDA(cudaMemcpyToSymbolAsync(c_gl_nodes, nodes, sizeof(nodes), 0, cudaMemcpyHostToDevice, st));
    XTS_CUDA(cudaMemcpyToSymbolAsync(c_gl_weights, wts, sizeof(wts), 0, cudaMemcpyHostToDevice, st));
    XTS_CUDA(cudaStreamSynchronize(st));
    done = true;
    dev_done = dev;
    return XTS_OK;
}

int launch_normalize_rpsf(double* params, int Mc, int Me, const double* glog, float s0, float s1,
                          float si, cudaStream_t st) {
    int rc = upload_gauss_legendre(st);
    if (rc) return rc;
    float sp0 = s0 * s0, sp1 = s1 * s1;
    int n = Mc * Me;
    XTS_LAUNCH("k_normalize_rpsf", st, k_normalize_rpsf<<<(n + 63) / 64, 64, 0, st>>>(params, Mc, Me, glog, sp0, sp1, si));
    return XTS_OK;
}

}  // namespace xts
