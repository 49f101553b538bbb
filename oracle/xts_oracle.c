/*
 * xts_oracle.c -- FP64 CPU restatement of the xtsrcmaps point-source model-map
 * path.  TEST INFRASTRUCTURE ONLY: the product library never links or calls it;
 * tests, smoke() and the CPU baseline of bench.py use it as the checker.
 *
 * Reference files are cited relative to the xtsrcmaps source tree.  The
 * restatement follows the reference's arithmetic order where that order is
 * visible in the source, including its documented quirks:
 *   - back-side exposure reuses the front livetime-efficiency factors
 *     (exposure/exposure.cxx:202-240, psf/psf.psf_lookup_table_and_partial_integrals.cxx:151-156);
 *   - cubature points are bilinear blends of corner unit vectors, not renormalised
 *     (model_map/mm_cubature/points_weights.hpp:93-107);
 *   - the pixel LUT kernel uses the *intended* semantics of
 *     convolve_pixel_psf_logsep (model_map/mm_cubature/convolve_pixel_psf_logsep.hpp:23-96):
 *     the shipped code never stores its column keys (keys[index] = psfidx is
 *     missing), so every point reads rows -1 and 0 of the table.  Here the key is
 *     stored; the result equals convolve_pixel_psf_searchsep inside [3e-4, 60] deg
 *     and keeps logsep's clamp (row 400) and its extrapolation below 1e-4 deg;
 *   - solid angles use pixel-centre quads shifted by half a pixel
 *     (math/solid_angle.hpp:42-79);
 *   - map_integral tests pixel centres against the radius (model_map.map_integral.cxx:26-37);
 *   - the containment correction integrates the whole separation bin above the
 *     radius (model_map.map_correction_factor.cxx:109-125);
 *   - the in-FOV test keeps a 3.5 pixel buffer (model_map.psf_boundary_radius.cxx:272-279).
 * Where the reference computes in float (IRF efficiency and scale parameters are
 * stored as float) the float steps are reproduced with explicit float casts.
 *
 * WCS: the reference calls wcslib; this file restates the FITS-WCS algorithm of
 * Calabretta & Greisen (2002, A&A 395, 1077) for CAR and AIT with the default
 * LONPOLE/LATPOLE rule for theta0 = 0 projections.
 */
#include "xts_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* misc/misc.hxx:15-43 */
static const double PI_ = 3.141592653589793238462643383279502884197;
static const double TWOPI = 6.283185307179586476925286766559005768394;
static const double HALFPI = 1.570796326794896619231321691639751442099;
static const double INV_HALFPI = 0.6366197723675813430755350534900574;
static const double D2R = 0.017453292519943295769236907684886127134;
static const double R2D = 57.295779513082320876798154814105170332405;
static const double SEP_STEP = 0.033731417579011382769913057686378448039204491;
static const double RECIPSTEP = 29.645952402019046699874076387601854602589360539942632073727038565;
static const double REDM1 = 29.148763300179999028597222671574207003288142769360422095500496366;
static const double LN_1E4 = 9.2103403719761827360719658187374568304044059545150919;

/* psf/psf.hxx:24-31: sep[0] = 0, sep[i+1] = 1e-4 * exp(i * ln(7e5)/399) */
void xo_separations(double* seps) {
    double xstep = log(70. / 1e-4) / (400 - 1.);
    seps[0] = 0.0;
    for (int i = 0; i < 400; ++i) seps[i + 1] = 1e-4 * exp(i * xstep);
}

/* ======================================================================== */
/* Geometry                                                                  */
/* ======================================================================== */

/* Celestial coordinates of the native pole for theta0 = 0 projections (CAR,
 * AIT): LONPOLE = 0 if dec0 >= theta0 else 180, LATPOLE = +90
 * (Calabretta & Greisen 2002, sect. 2.4).  The reference sets the same
 * keywords through wcsset() (sky_geom/sky_geom.hxx:79-125). */
static void native_pole(const xo_wcs* w, double* ap, double* dp, double* pp) {
    double a0 = w->crval1 > 180. ? w->crval1 - 360. : w->crval1; /* sky_geom.hxx:110 */
    double d0 = w->crval2;
    if (d0 >= 0.) { *pp = 0.;   *dp = 90. - d0; *ap = a0 - 180.; }
    else          { *pp = 180.; *dp = 90. + d0; *ap = a0; }
}

void xo_sph2dir(double ra, double dec, double* v) { /* sky_geom.hxx:281-287 */
    double cr = cos(ra * D2R), cd = cos(dec * D2R);
    double sr = sin(ra * D2R), sd = sin(dec * D2R);
    v[0] = cr * cd; v[1] = sr * cd; v[2] = sd;
}

void xo_wcs_pix2sph(const xo_wcs* w, double p1, double p2, double* ra, double* dec) {
    double dp1 = p1 - w->crpix1, dp2 = p2 - w->crpix2;
    double x, y;
    if (w->crota2 == 0.0) { x = w->cdelt1 * dp1; y = w->cdelt2 * dp2; }
    else {
        double cr = cos(w->crota2 * D2R), sr = sin(w->crota2 * D2R);
        x = w->cdelt1 * cr * dp1 - w->cdelt2 * sr * dp2;
        y = w->cdelt1 * sr * dp1 + w->cdelt2 * cr * dp2;
    }
    double phi, theta; /* native, degrees */
    if (w->proj == 0) { phi = x; theta = y; }
    else {
        double X = x * D2R, Y = y * D2R;
        double z2 = 1.0 - 0.0625 * X * X - 0.25 * Y * Y;
        double z = sqrt(z2 > 0. ? z2 : 0.);
        phi = 2.0 * atan2(0.5 * X * z, 2.0 * z2 - 1.0) * R2D;
        double s = Y * z;
        theta = asin(s > 1. ? 1. : (s < -1. ? -1. : s)) * R2D;
    }
    double ap, dp, pp;
    native_pole(w, &ap, &dp, &pp);
    double st = sin(theta * D2R), ct = cos(theta * D2R);
    double sdp = sin(dp * D2R), cdp = cos(dp * D2R);
    double dphi = (phi - pp) * D2R;
    double xr = st * cdp - ct * sdp * cos(dphi);
    double yr = -ct * sin(dphi);
    double a = ap + atan2(yr, xr) * R2D;
    double zs = st * sdp + ct * cdp * cos(dphi);
    double d = asin(zs > 1. ? 1. : (zs < -1. ? -1. : zs)) * R2D;
    while (a < 0.) a += 360.;   /* sky_geom.hxx:246-248 */
    while (a >= 360.) a -= 360.;
    *ra = a; *dec = d;
}

void xo_wcs_sph2pix(const xo_wcs* w, double ra, double dec, double* p1, double* p2) {
    double ap, dp, pp;
    native_pole(w, &ap, &dp, &pp);
    double sd = sin(dec * D2R), cd = cos(dec * D2R);
    double sdp = sin(dp * D2R), cdp = cos(dp * D2R);
    double da = (ra - ap) * D2R;
    double xr = sd * cdp - cd * sdp * cos(da);
    double yr = -cd * sin(da);
    double phi = pp + atan2(yr, xr) * R2D;
    double zs = sd * sdp + cd * cdp * cos(da);
    double theta = asin(zs > 1. ? 1. : (zs < -1. ? -1. : zs)) * R2D;
    while (phi > 180.) phi -= 360.;
    while (phi <= -180.) phi += 360.;
    double x, y;
    if (w->proj == 0) { x = phi; y = theta; }
    else {
        double ct = cos(theta * D2R);
        double g = R2D * sqrt(2.0 / (1.0 + ct * cos(0.5 * phi * D2R)));
        x = 2.0 * g * ct * sin(0.5 * phi * D2R);
        y = g * sin(theta * D2R);
    }
    double dp1, dp2;
    if (w->crota2 == 0.0) { dp1 = x / w->cdelt1; dp2 = y / w->cdelt2; }
    else {
        double cr = cos(w->crota2 * D2R), sr = sin(w->crota2 * D2R);
        dp1 = (cr * x + sr * y) / w->cdelt1;
        dp2 = (-sr * x + cr * y) / w->cdelt2;
    }
    *p1 = w->crpix1 + dp1; *p2 = w->crpix2 + dp2;
}

void xo_pix2dir(const xo_wcs* w, double p1, double p2, double* v) { /* sky_geom.hxx:277 */
    double ra, dec;
    xo_wcs_pix2sph(w, p1, p2, &ra, &dec);
    xo_sph2dir(ra, dec, v);
}

double xo_dir_diff(const double* a, const double* b) { /* sky_geom.hxx:305-310 */
    double x = a[0] - b[0], y = a[1] - b[1], z = a[2] - b[2];
    return 2. * asin(0.5 * sqrt(x * x + y * y + z * z));
}

/* HEALPix NESTED (Gorski et al. 2005); healpix/healpix.cxx:181-229 */
static long long spread_bits(long long v) {
    long long r = 0;
    for (int b = 0; b < 32; ++b) r |= ((v >> b) & 1LL) << (2 * b);
    return r;
}
static long long compress_bits(long long v) {
    long long r = 0;
    for (int b = 0; b < 32; ++b) r |= ((v >> (2 * b)) & 1LL) << b;
    return r;
}
static int ilog2ll(long long v) { int r = 0; while (v > 1) { v >>= 1; ++r; } return r; }

long long xo_ang2pix_nest(double theta, double phi, long long nside) {
    int have_sth = (theta < 0.01) || (theta > PI_ - 0.01);
    double sth = have_sth ? sin(theta) : 0.;
    double z = cos(theta), za = fabs(z);
    double tt = phi * INV_HALFPI; /* fmodulo(., 4) */
    if (tt >= 0) tt = (tt < 4.0) ? tt : fmod(tt, 4.0);
    else { double t = fmod(tt, 4.0) + 4.0; tt = (t == 4.0) ? 0. : t; }
    int order = ilog2ll(nside);
    long long ix, iy, face;
    if (za <= 2.0 / 3.0) {
        double t1 = nside * (0.5 + tt), t2 = nside * (z * 0.75);
        long long jp = (long long)(t1 - t2), jm = (long long)(t1 + t2);
        long long ifp = jp >> order, ifm = jm >> order;
        face = (ifp == ifm) ? (ifp | 4) : ((ifp < ifm) ? ifp : (ifm + 8));
        ix = jm & (nside - 1);
        iy = nside - (jp & (nside - 1)) - 1;
    } else {
        long long ntt = (long long)tt; if (ntt > 3) ntt = 3;
        double tp = tt - ntt;
        double tmp = ((za < 0.99) || !have_sth) ? nside * sqrt(3 * (1 - za))
                                                : nside * sth / sqrt((1. + za) / 3.);
        long long jp = (long long)(tp * tmp), jm = (long long)((1.0 - tp) * tmp);
        if (jp > nside - 1) jp = nside - 1;
        if (jm > nside - 1) jm = nside - 1;
        if (z >= 0) { face = ntt; ix = nside - jm - 1; iy = nside - jp - 1; }
        else { face = ntt + 8; ix = jp; iy = jm; }
    }
    return (face << (2 * order)) + spread_bits(ix) + (spread_bits(iy) << 1);
}

/* healpix/healpix.cxx:136-179 */
void xo_pix2ang_nest(long long pix, long long nside, double* theta, double* phi) {
    static const long long jrll[] = {2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4};
    static const long long jpll[] = {1, 3, 5, 7, 0, 2, 4, 6, 1, 3, 5, 7};
    long long npface = nside * nside, npix = 12 * npface;
    double fact2 = 4. / npix, fact1 = (nside << 1) * fact2;
    int order = ilog2ll(nside);
    long long face = pix >> (2 * order), t = pix & (npface - 1);
    long long ix = compress_bits(t), iy = compress_bits(t >> 1);
    long long jr = (jrll[face] << order) - ix - iy - 1, r;
    double z, sth = 0.; int have = 0;
    if (jr < nside) { r = jr; double tmp = (double)(r * r) * fact2; z = 1 - tmp;
        if (z > 0.99) { sth = sqrt(tmp * (2. - tmp)); have = 1; } }
    else if (jr > 3 * nside) { r = nside * 4 - jr; double tmp = (double)(r * r) * fact2; z = tmp - 1;
        if (z < -0.99) { sth = sqrt(tmp * (2. - tmp)); have = 1; } }
    else { r = nside; z = (2 * nside - jr) * fact1; }
    long long tt = jpll[face] * r + ix - iy;
    if (tt < 0) tt += 8 * r;
    *phi = (r == nside) ? 0.75 * HALFPI * tt * fact1 : (0.5 * HALFPI * tt) / r;
    *theta = have ? atan2(sth, z) : acos(z);
}

/* ======================================================================== */
/* Step (a): exposure                                                        */
/* ======================================================================== */

/* exposure/exposure.cxx:29-40 */
void xo_costhetas(int nbins, double cosmin, int thetabin, double* out) {
    for (int i = 0; i < nbins; ++i) {
        double f = ((double)i + 0.5) / nbins;
        f = thetabin ? f * f : f;
        out[i] = 1. - f * (1. - cosmin);
    }
}

/* exposure/exposure.cxx:42-63 */
void xo_src_cosbins(const double* src_sph, int S, const float* cube, long long nside,
                    int C, double* out) {
    for (int s = 0; s < S; ++s) {
        double theta = HALFPI - src_sph[2 * s + 1] * D2R;
        double phi = D2R * src_sph[2 * s];
        long long pix = xo_ang2pix_nest(theta, phi, nside);
        for (int c = 0; c < C; ++c) out[(size_t)s * C + c] = (double)cube[(size_t)pix * C + c];
    }
}

/* math/bilerp.cxx:6-27: upper_bound search, weight, complement, index.  The
 * reference asserts the value lies inside the grid; the oracle clamps the index
 * to the last interval instead of reading past the end. */
static void lerp_pars(const double* g, int n, double v, int has_lb, double lb,
                      double* wgt, double* cmpl, int* idx) {
    if (has_lb && v < lb) { *wgt = 0.; *cmpl = 0.; *idx = 1; return; }
    int i = 0;
    while (i < n && !(v < g[i])) ++i; /* upper_bound */
    if (i < 1) i = 1;
    if (i > n - 1) i = n - 1;
    double t = (v - g[i - 1]) / (g[i] - g[i - 1]);
    *wgt = t; *cmpl = 1. - t; *idx = i;
}

/* irf/irf.aeff_value.cxx:11-55 */
void xo_aeff_value(const double* costh, int C, const double* logEs, int E,
                   const xo_grid* A, double* out) {
    int Me = A->n_e;
    for (int c = 0; c < C; ++c) {
        double cw, cc; int ci;
        lerp_pars(A->cosths, A->n_cos, costh[c], 1, A->min_cos_theta, &cw, &cc, &ci);
        for (int e = 0; e < E; ++e) {
            double ew, ec; int ei;
            lerp_pars(A->logEs, A->n_e, logEs[e], 0, 0., &ew, &ec, &ei);
            const double* P = A->params; /* n_par == 1 */
            double xx = cc * ec * P[(size_t)(ci - 1) * Me + (ei - 1)];
            double xy = cc * ew * P[(size_t)(ci - 1) * Me + ei];
            double yx = cw * ec * P[(size_t)ci * Me + (ei - 1)];
            double yy = cw * ew * P[(size_t)ci * Me + ei];
            out[(size_t)c * E + e] = 1e4 * (xx + xy + yx + yy);
        }
    }
}

/* irf/irf.cxx:70-109.  Row 1 comes from p0 and row 0 from p1 ("intentionally").
 * The break offsets b1, b2 are computed in float, as in the reference where the
 * parameters are std::array<float, 6>. */
static double ltf_single(const float* p, double logE) {
    float a0 = p[0], b0 = p[1], a1 = p[2], lb1 = p[3], a2 = p[4], lb2 = p[5];
    volatile float t1 = (a0 - a1) * lb1;
    double b1 = (double)(float)(t1 + b0);
    volatile float t2 = (a1 - a2) * lb2;
    double b2 = (double)(float)(t2 + (float)b1);
    return logE < lb1 ? a0 * logE + b0 : logE < lb2 ? a1 * logE + b1 : a2 * logE + b2;
}
void xo_livetime_efficiency_factors(const double* logEs, int E, const float* p0,
                                    const float* p1, double* out) {
    for (int e = 0; e < E; ++e) {
        out[E + e] = ltf_single(p0, logEs[e]);
        out[e] = ltf_single(p1, logEs[e]);
    }
}

/* exposure/exposure.cxx:159-263 + exposure/exposure.contract.cpp:13-42 */
void xo_exposure(const double* ecb, const double* wecb, int S, int C,
                 const double* af, const double* ab, const double* ltf, int E,
                 double* out) {
    for (int s = 0; s < S; ++s)
        for (int e = 0; e < E; ++e) {
            double ef = 0, wf = 0, eb = 0, wb = 0;
            for (int c = 0; c < C; ++c) {
                double x = ecb[(size_t)s * C + c], w = wecb[(size_t)s * C + c];
                ef += x * af[(size_t)c * E + e];
                wf += w * af[(size_t)c * E + e];
                eb += x * ab[(size_t)c * E + e];
                wb += w * ab[(size_t)c * E + e];
            }
            ef *= ltf[e]; wf *= ltf[E + e]; eb *= ltf[e]; wb *= ltf[E + e];
            out[(size_t)s * E + e] = ((ef + eb) + wf) + wb;
        }
}

/* ======================================================================== */
/* Step (b): mean PSF                                                        */
/* ======================================================================== */

/* 64-point Gauss-Legendre nodes and weights on [-1, 1] by Newton iteration on
 * the Legendre recurrence (math/gauss_legendre.hxx:37-62). */
void xo_gauss_legendre_64(double* nodes, double* weights) {
    const int N = 64;
    for (int i = 1; i <= N; ++i) {
        double x = cos(PI_ * (i - 0.25) / (N + 0.5));
        double dp = 0.;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = x;
            for (int j = 2; j <= N; ++j) {
                double p2 = ((2 * j - 1) * x * p1 - (j - 1) * p0) / j;
                p0 = p1; p1 = p2;
            }
            dp = N * (x * p1 - p0) / (x * x - 1);
            double dx = p1 / dp;
            x -= dx;
            if (fabs(dx) <= 1e-15) break;
        }
        nodes[i - 1] = x;
        weights[i - 1] = 2.0 / ((1. - x * x) * dp * dp);
    }
}

/* irf/irf.hxx:22-45 */
static double king_f(double u, double g) {
    if (g == 1) g = 1.001;
    return (1. - 1. / g) * pow(1. + u / g, -g);
}
double xo_evaluate_king(double sep, double sf, const double* p) {
    double ncore = p[0], ntail = p[1], score = p[2] * sf, stail = p[3] * sf;
    double rc = sep / score, uc = rc * rc / 2.;
    double rt = sep / stail, ut = rt * rt / 2.;
    return ncore * king_f(uc, p[4]) + ntail * ncore * king_f(ut, p[5]);
}

/* irf/irf.hxx:48-77 */
double xo_psf_base_integral(double radius, double sf, const double* p) {
    double ncore = p[0], ntail = p[1], score = p[2] * sf, stail = p[3] * sf;
    double sep = radius * D2R;
    double rc = sep / score, uc = rc * rc / 2.;
    double rt = sep / stail, ut = rt * rt / 2.;
    double fc = 1. - pow(1. + uc / p[4], 1. - p[4]);
    double ft = 1. - pow(1. + ut / p[5], 1. - p[5]);
    return ncore * fc * TWOPI * score * score + ntail * ncore * ft * TWOPI * stail * stail;
}

/* irf/irf.normalize_rpsf.cpp:11-61 */
void xo_normalize_rpsf(double* params, int Mc, int Me, const double* glog,
                       float scale0, float scale1, float scale_index) {
    double nodes[64], wts[64];
    xo_gauss_legendre_64(nodes, wts);
    float sp0 = scale0 * scale0, sp1 = scale1 * scale1, si = scale_index;
    for (int c = 0; c < Mc; ++c)
        for (int e = 0; e < Me; ++e) {
            double* p = params + ((size_t)c * Me + e) * 6;
            double energy = pow(10.0, glog[e]);
            double tt = pow(energy * 1.e-2, si);
            double sf = sqrt(sp0 * tt * tt + sp1);
            double norm;
            if (energy < 120.) {
                double acc = 0.;
                for (int k = 0; k < 64; ++k) {
                    double v = 45. * nodes[k] + 45.;
                    double x = xo_evaluate_king(v * D2R, sf, p);
                    double y = sin(v * D2R) * TWOPI * D2R;
                    acc += wts[k] * (x * y);
                }
                norm = acc * 45.;
            } else {
                norm = xo_psf_base_integral(90.0, sf, p);
            }
            p[0] /= norm;
            p[2] *= sf;
            p[3] *= sf;
            p[4] = p[4] == 1. ? 1.001 : p[4];
            p[5] = p[5] == 1. ? 1.001 : p[5];
        }
}

/* psf/psf.king.cxx:9-43 -> [D, Mc, Me] */
void xo_king(const xo_grid* g, double* out) {
    double seps[XO_ND];
    xo_separations(seps);
    int Mc = g->n_cos, Me = g->n_e;
    for (int d = 0; d < XO_ND; ++d)
        for (int c = 0; c < Mc; ++c)
            for (int e = 0; e < Me; ++e)
                out[((size_t)d * Mc + c) * Me + e] =
                    xo_evaluate_king(seps[d] * D2R, 1.0, g->params + ((size_t)c * Me + e) * 6);
}

/* psf/psf.bilerp.cxx:6-52 -> [C, D, E] */
void xo_psf_bilerp(const double* costh, int C, const double* logEs, int E,
                   const xo_grid* g, const double* K, double* out) {
    int Mc = g->n_cos, Me = g->n_e;
    for (int c = 0; c < C; ++c) {
        double cw, cc; int ci;
        lerp_pars(g->cosths, Mc, costh[c], 0, 0., &cw, &cc, &ci);
        for (int e = 0; e < E; ++e) {
            double ew, ec; int ei;
            lerp_pars(g->logEs, Me, logEs[e], 0, 0., &ew, &ec, &ei);
            for (int d = 0; d < XO_ND; ++d) {
                const double* Kd = K + (size_t)d * Mc * Me;
                out[((size_t)c * XO_ND + d) * E + e] =
                    cc * ec * Kd[(ci - 1) * Me + ei - 1] + cc * ew * Kd[(ci - 1) * Me + ei] +
                    cw * ec * Kd[ci * Me + ei - 1] + cw * ew * Kd[ci * Me + ei];
            }
        }
    }
}

/* psf/psf.corrected_exposure_psf.cxx:12-120 */
void xo_corrected_exposure_psf(const double* P, const double* A, const double* ecb,
                               const double* wecb, int S, int C, int E,
                               const double* ltf, double* out) {
    size_t DE = (size_t)XO_ND * E;
    double* pa = (double*)malloc(sizeof(double) * C * DE);
    for (int c = 0; c < C; ++c)
        for (int d = 0; d < XO_ND; ++d)
            for (int e = 0; e < E; ++e)
                pa[(size_t)c * DE + (size_t)d * E + e] =
                    P[(size_t)c * DE + (size_t)d * E + e] * A[(size_t)c * E + e];
    for (int s = 0; s < S; ++s)
        for (size_t j = 0; j < DE; ++j) {
            double x = 0., w = 0.;
            for (int c = 0; c < C; ++c) {
                x += ecb[(size_t)s * C + c] * pa[(size_t)c * DE + j];
                w += wecb[(size_t)s * C + c] * pa[(size_t)c * DE + j];
            }
            int e = (int)(j % E);
            out[(size_t)s * DE + j] = x * ltf[e] + w * ltf[E + e];
        }
    free(pa);
}

/* psf/psf.mean_psf.cxx:6-33 */
void xo_mean_psf(const double* f, const double* b, const double* expo, int S, int E,
                 double* out) {
    for (int s = 0; s < S; ++s)
        for (int d = 0; d < XO_ND; ++d)
            for (int e = 0; e < E; ++e) {
                size_t i = ((size_t)s * XO_ND + d) * E + e;
                out[i] = (f[i] + b[i]) / expo[(size_t)s * E + e];
            }
}

/* psf/psf.partial_total_integral.cxx:8-52 */
void xo_partial_total_integral(const double* u, int S, int E, double* part, double* tot) {
    double seps[XO_ND];
    xo_separations(seps);
    for (int s = 0; s < S; ++s)
        for (int e = 0; e < E; ++e) {
            const double* us = u + (size_t)s * XO_ND * E;
            double* ps = part + (size_t)s * XO_ND * E;
            double cum = 0.0;
            ps[e] = 0.0;
            for (int d = 1; d < XO_ND; ++d) {
                double t1 = D2R * seps[d - 1], t2 = D2R * seps[d];
                double y1 = TWOPI * us[(size_t)(d - 1) * E + e] * sin(t1);
                double y2 = TWOPI * us[(size_t)d * E + e] * sin(t2);
                double m = (y2 - y1) / (t2 - t1);
                double b = y1 - t1 * m;
                double v = 0.5 * m * (t2 * t2 - t1 * t1) + b * (t2 - t1);
                cum += v;
                ps[(size_t)d * E + e] = cum;
            }
            tot[(size_t)s * E + e] = cum;
            if (cum != 0.)
                for (int d = 0; d < XO_ND; ++d) ps[(size_t)d * E + e] /= cum;
        }
}

/* psf/psf.normalize.cxx:7-24 */
void xo_normalize(double* u, const double* tot, int S, int E) {
    for (int s = 0; s < S; ++s)
        for (int d = 0; d < XO_ND; ++d)
            for (int e = 0; e < E; ++e) u[((size_t)s * XO_ND + d) * E + e] /= tot[(size_t)s * E + e];
}

/* psf/psf.psf_lookup_table_and_partial_integrals.cxx:8-57 */
void xo_compute_psf_data(const xo_grid* pf, const xo_grid* pb, const double* costh,
                         int C, const double* logEs, int E, const double* af,
                         const double* ab, const double* ecb, const double* wecb, int S,
                         const double* ltf, const double* expo, double* upsf,
                         double* partial) {
    size_t DE = (size_t)XO_ND * E;
    double* kf = (double*)malloc(sizeof(double) * XO_ND * pf->n_cos * pf->n_e);
    double* kb = (double*)malloc(sizeof(double) * XO_ND * pb->n_cos * pb->n_e);
    double* of = (double*)malloc(sizeof(double) * C * DE);
    double* ob = (double*)malloc(sizeof(double) * C * DE);
    double* cf = (double*)malloc(sizeof(double) * S * DE);
    double* cb = (double*)malloc(sizeof(double) * S * DE);
    double* tot = (double*)malloc(sizeof(double) * S * E);
    xo_king(pf, kf);
    xo_king(pb, kb);
    xo_psf_bilerp(costh, C, logEs, E, pf, kf, of);
    xo_psf_bilerp(costh, C, logEs, E, pb, kb, ob);
    xo_corrected_exposure_psf(of, af, ecb, wecb, S, C, E, ltf, cf);
    xo_corrected_exposure_psf(ob, ab, ecb, wecb, S, C, E, ltf, cb);
    xo_mean_psf(cf, cb, expo, S, E, upsf);
    xo_partial_total_integral(upsf, S, E, partial, tot);
    xo_normalize(upsf, tot, S, E);
    free(kf); free(kb); free(of); free(ob); free(cf); free(cb); free(tot);
}

/* ======================================================================== */
/* Steps (c)+(d): model map                                                  */
/* ======================================================================== */

/* Sommariva & Festa's degree-7, 12-point symmetric rule on [-1,1]^2 (Padova
 * "cub_square_lowcard" tables), as listed in
 * model_map/mm_cubature/cubature.hpp:209-225: (u, v, weight) triples. */
static const double SQUARE_DEG7[36] = {
    3.9383136101878902e-01, -3.6699793434042738e-01, 5.2092862230230441e-01,
    8.0196847620659251e-01, 8.0992592975809186e-01, 2.3740240561379911e-01,
    -1.8327327664247231e-02, 9.2596092593108370e-01, 2.4166897208389651e-01,
    3.6699793434042738e-01, 3.9383136101878902e-01, 5.2092862230230441e-01,
    -8.0992592975809186e-01, 8.0196847620659251e-01, 2.3740240561379911e-01,
    -9.2596092593108370e-01, -1.8327327664247231e-02, 2.4166897208389651e-01,
    -3.9383136101878902e-01, 3.6699793434042738e-01, 5.2092862230230441e-01,
    -8.0196847620659251e-01, -8.0992592975809186e-01, 2.3740240561379911e-01,
    1.8327327664247231e-02, -9.2596092593108370e-01, 2.4166897208389651e-01,
    -3.6699793434042738e-01, -3.9383136101878902e-01, 5.2092862230230441e-01,
    8.0992592975809186e-01, -8.0196847620659251e-01, 2.3740240561379911e-01,
    9.2596092593108370e-01, 1.8327327664247231e-02, 2.4166897208389651e-01,
};

/* model_map/mm_cubature/points_weights.hpp:5-56 (looping h < Nh; the reference
 * loops h < Nw and is only defined for square maps). */
void xo_square_ptswts(const xo_wcs* w, long Nh, long Nw, double* out) {
    for (long h = 0; h < Nh; ++h)
        for (long x = 0; x < Nw; ++x) {
            double ph = 1. + h, pw = 1. + x, a[3], b[3], c[3], d[3];
            xo_pix2dir(w, ph - 0.5, pw - 0.5, a); /* LL */
            xo_pix2dir(w, ph - 0.5, pw + 0.5, b); /* LR */
            xo_pix2dir(w, ph + 0.5, pw + 0.5, c); /* UR */
            xo_pix2dir(w, ph + 0.5, pw - 0.5, d); /* UL */
            double* o = out + ((size_t)h * Nw + x) * 48;
            for (int p = 0; p < 12; ++p) {
                double u = SQUARE_DEG7[3 * p], v = SQUARE_DEG7[3 * p + 1];
                double nn = (1.0 - u) * (1.0 - v), pn = (1.0 + u) * (1.0 - v);
                double pp = (1.0 + u) * (1.0 + v), np = (1.0 - u) * (1.0 + v);
                for (int k = 0; k < 3; ++k)
                    o[4 * p + k] = 0.25 * (nn * a[k] + pn * b[k] + pp * c[k] + np * d[k]);
                o[4 * p + 3] = 0.25 * SQUARE_DEG7[3 * p + 2];
            }
        }
}

/* model_map/mm_cubature/convolve_pixel_psf_logsep.hpp:23-96 with the column key
 * stored (see the file header). */
void xo_convolve_pixel_logsep(double* map_e, int E, const double* pw,
                              const double* lut, const double* src) {
    double va[12], vb[12];
    int keys[12], keylen = 0;
    for (int p = 0; p < 12; ++p) {
        double x = pw[4 * p] - src[0], y = pw[4 * p + 1] - src[1], z = pw[4 * p + 2] - src[2];
        double w = pw[4 * p + 3];
        double s = 2.0 * R2D * asin(0.5 * sqrt(x * x + y * y + z * z));
        double j = s < 1e-4 ? 1. : 1. + RECIPSTEP * (LN_1E4 + log(s));
        int idx = 1 + (int)(unsigned short)j;
        if (idx > 400) idx = 400;
        double t = REDM1 * (s * 1e4 * exp(SEP_STEP * (2. - idx)) - 1.);
        int k = 0;
        while (k < keylen && keys[k] != idx) ++k;
        if (k == keylen) { keys[keylen] = idx; va[keylen] = 0.; vb[keylen] = 0.; ++keylen; }
        va[k] += (1.0 - t) * w;
        vb[k] += t * w;
    }
    for (int k = 0; k < keylen; ++k) {
        const double* YL = lut + (size_t)E * (keys[k] - 1);
        const double* YR = lut + (size_t)E * keys[k];
        for (int e = 0; e < E; ++e) map_e[e] += (va[k] * YL[e]) + (vb[k] * YR[e]);
    }
}

/* model_map/mm_cubature/cubature.implementation.cxx:21-55 */
void xo_cubature_map(const xo_wcs* w, long Nh, long Nw, const double* src_sph, int S,
                     const double* upsf, int E, double* out) {
    double* pw = (double*)malloc(sizeof(double) * Nh * Nw * 48);
    xo_square_ptswts(w, Nh, Nw, pw);
    memset(out, 0, sizeof(double) * (size_t)S * Nh * Nw * E);
    for (int s = 0; s < S; ++s) {
        double src[3];
        xo_sph2dir(src_sph[2 * s], src_sph[2 * s + 1], src);
        for (long x = 0; x < Nw; ++x)
            for (long h = 0; h < Nh; ++h)
                xo_convolve_pixel_logsep(out + (((size_t)s * Nh + h) * Nw + x) * E, E,
                                         pw + ((size_t)h * Nw + x) * 48,
                                         upsf + (size_t)s * XO_ND * E, src);
    }
    free(pw);
}

/* math/solid_angle.hpp:42-79 */
static void sub3(const double* a, const double* b, double* o) { o[0] = a[0] - b[0]; o[1] = a[1] - b[1]; o[2] = a[2] - b[2]; }
static double norm3(const double* v) { return sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }
static double quad_half(const double* P, const double* Q, const double* R) {
    double u[3], v[3], c[3];
    sub3(P, Q, u); sub3(P, R, v);
    double nu = norm3(u), nv = norm3(v);
    u[0] /= nu; u[1] /= nu; u[2] /= nu; v[0] /= nv; v[1] /= nv; v[2] /= nv;
    c[0] = u[1] * v[2] - u[2] * v[1]; c[1] = u[2] * v[0] - u[0] * v[2]; c[2] = u[0] * v[1] - u[1] * v[0];
    return xo_dir_diff(P, Q) * xo_dir_diff(P, R) * norm3(c);
}
void xo_solid_angle(const xo_wcs* w, long Nh, long Nw, double* out) {
    for (long h = 0; h < Nh; ++h) {
        double ph = 1. + h;
        for (long x = 0; x < Nw; ++x) {
            double pw = 1. + x, A[3], B[3], C[3], D[3];
            xo_pix2dir(w, ph, pw, A);
            xo_pix2dir(w, ph, pw + 1., B);
            xo_pix2dir(w, ph + 1., pw + 1., C);
            xo_pix2dir(w, ph + 1., pw, D);
            out[h * Nw + x] = 0.5 * (quad_half(A, B, D) + quad_half(C, B, D));
        }
    }
}

/* model_map/model_map.psf_boundary_radius.cxx:9-62 */
void xo_psf_boundary_radius(const xo_wcs* w, long Nh, long Nw, const double* src_sph,
                            int S, double* radius, int* in_fov) {
    const double buf = 3.5;
    for (int s = 0; s < S; ++s) {
        double ra = src_sph[2 * s], dec = src_sph[2 * s + 1], p1, p2, sd[3], pd[3];
        double r = ra > 180. ? ra - 360. : (ra < -180. ? ra + 360. : ra);
        xo_wcs_sph2pix(w, r, dec, &p1, &p2);
        in_fov[s] = p1 > buf && p1 < (Nh - buf) && p2 > buf && p2 < (Nw - buf);
        xo_sph2dir(ra, dec, sd);
        double mn = 360.;
        for (long h = 0; h <= Nh; ++h) {
            xo_pix2dir(w, h + 0.5, 0.5, pd);
            double d = R2D * xo_dir_diff(sd, pd); mn = mn < d ? mn : d;
            xo_pix2dir(w, h + 0.5, Nw + 0.5, pd);
            d = R2D * xo_dir_diff(sd, pd); mn = mn < d ? mn : d;
        }
        for (long x = 0; x <= Nw; ++x) {
            xo_pix2dir(w, 0.5, x + 0.5, pd);
            double d = R2D * xo_dir_diff(sd, pd); mn = mn < d ? mn : d;
            xo_pix2dir(w, Nh + 0.5, x + 0.5, pd);
            d = R2D * xo_dir_diff(sd, pd); mn = mn < d ? mn : d;
        }
        radius[s] = mn;
    }
}

/* model_map/model_map.map_integral.cxx:4-48 (returns 1/sum, 0 stays 0) */
void xo_map_integral(const double* map, const xo_wcs* w, long Nh, long Nw,
                     const double* src_sph, int S, int E, const double* radius,
                     const int* in_fov, double* inv) {
    memset(inv, 0, sizeof(double) * S * E);
    double* cen = (double*)malloc(sizeof(double) * Nh * Nw * 3);
    for (long h = 0; h < Nh; ++h)
        for (long x = 0; x < Nw; ++x) xo_pix2dir(w, h + 1.0, x + 1.0, cen + (h * Nw + x) * 3);
    for (int s = 0; s < S; ++s) {
        if (!in_fov[s]) continue;
        double sd[3];
        xo_sph2dir(src_sph[2 * s], src_sph[2 * s + 1], sd);
        for (long h = 0; h < Nh; ++h)
            for (long x = 0; x < Nw; ++x) {
                double rad = xo_dir_diff(sd, cen + (h * Nw + x) * 3);
                if (rad <= D2R * radius[s])
                    for (int e = 0; e < E; ++e)
                        inv[(size_t)s * E + e] += map[(((size_t)s * Nh + h) * Nw + x) * E + e];
            }
    }
    for (int i = 0; i < S * E; ++i) inv[i] = inv[i] != 0. ? 1.0 / inv[i] : inv[i];
    free(cen);
}

/* psf/psf.fast_separation_lower_index.cxx:5-22 + model_map.map_correction_factor.cxx:3-53 */
void xo_map_correction_factor(const double* inv, const double* radius, const int* in_fov,
                              const double* upsf, const double* partial, int S, int E,
                              double* factor) {
    double seps[XO_ND];
    xo_separations(seps);
    for (int s = 0; s < S; ++s) {
        if (!in_fov[s]) { for (int e = 0; e < E; ++e) factor[(size_t)s * E + e] = 1.0; continue; }
        double v0 = radius[s];
        int li = v0 < 1. ? 1 : (int)floor(1. + log(1e4 * v0) * RECIPSTEP);
        int d = li >= XO_ND - 2 ? XO_ND - 2 : li;
        double t1 = seps[d] * D2R, t2 = seps[d + 1] * D2R;
        for (int e = 0; e < E; ++e) {
            const double* U = upsf + (size_t)s * XO_ND * E;
            double y1 = TWOPI * U[(size_t)d * E + e] * sin(t1);
            double y2 = TWOPI * U[(size_t)(d + 1) * E + e] * sin(t2);
            double m = (y2 - y1) / (t2 - t1);
            double b = y1 - t1 * m;
            double v = 0.5 * m * (t2 * t2 - t1 * t1) + b * (t2 - t1);
            double integ = v + partial[(size_t)s * XO_ND * E + (size_t)d * E + e];
            integ = integ > 1.0 ? 1.0 : integ;
            factor[(size_t)s * E + e] = integ * inv[(size_t)s * E + e];
        }
    }
}

/* model_map/model_map.point_src_model_map_wcs.cxx:6-45 */
/* Steps after the cubature (model_map.point_src_model_map_wcs.cxx:22-44): solid
 * angle, boundary radius, map integral, exposure, correction factor. */
static void finish_model_map(const xo_wcs* w, const double* src_sph, int S, const double* expo,
                             const double* upsf, const double* partial, int E, double* out,
                             double* inv, double* factor, double* radius, int* in_fov) {
    long Nh = w->naxis1, Nw = w->naxis2;
    double* om = (double*)malloc(sizeof(double) * Nh * Nw);
    xo_solid_angle(w, Nh, Nw, om);
    for (int s = 0; s < S; ++s)
        for (long p = 0; p < Nh * Nw; ++p)
            for (int e = 0; e < E; ++e) out[((size_t)s * Nh * Nw + p) * E + e] *= om[p];
    xo_psf_boundary_radius(w, Nh, Nw, src_sph, S, radius, in_fov);
    xo_map_integral(out, w, Nh, Nw, src_sph, S, E, radius, in_fov, inv);
    for (int s = 0; s < S; ++s)
        for (long p = 0; p < Nh * Nw; ++p)
            for (int e = 0; e < E; ++e) out[((size_t)s * Nh * Nw + p) * E + e] *= expo[(size_t)s * E + e];
    xo_map_correction_factor(inv, radius, in_fov, upsf, partial, S, E, factor);
    for (int s = 0; s < S; ++s)
        for (long p = 0; p < Nh * Nw; ++p)
            for (int e = 0; e < E; ++e) out[((size_t)s * Nh * Nw + p) * E + e] *= factor[(size_t)s * E + e];
    free(om);
}

void xo_point_src_model_map_wcs(const xo_wcs* w, const double* src_sph, int S,
                                const double* expo, const double* upsf,
                                const double* partial, int E, double* out,
                                double* inv, double* factor, double* radius, int* in_fov) {
    xo_cubature_map(w, w->naxis1, w->naxis2, src_sph, S, upsf, E, out);
    finish_model_map(w, src_sph, S, expo, upsf, partial, E, out, inv, factor, radius, in_fov);
}

/* ---- adaptive cubature: the published Genz-Malik degree-7/5 rule for d = 2
 * (A.C. Genz, A.A. Malik, J. Comput. Appl. Math. 6 (1980) 295-302; weights as
 * updated by Bernstein, Espelid and Genz), the design the reference lays out in
 * math/genz_malik.hxx:18-85 and math/genz_malik.cxx:66-217 (not compiled there).
 * Differences from that code, which follow the published algorithm instead:
 * sub-regions are rectangles with a half-width per dimension (region_split at
 * genz_malik.cxx:189-217 halves one scalar half-width for both dimensions while
 * splitting only one), and regions still above the tolerance at the depth limit
 * keep their estimate (integrate_region at genz_malik.hxx:150-194 drops them).
 * The integrand is the keys-fixed logsep interpolation of the mean PSF at the
 * pixel's bilinear blend of its corner unit vectors, as for the 12-point rule. */
static const double GM_L2 = 0.35856858280031809199064515390793749545406372969943071; /* sqrt(9/70) */
static const double GM_L4 = 0.94868329805051379959966806332981556011586654179756505; /* sqrt(9/10) */
static const double GM_L5 = 0.68824720161168529772162873429362352512689535661564885; /* sqrt(9/19) */

/* point offsets in half-widths along (dimension 0, dimension 1) */
static const signed char GM_OFF[17][2] = {
    {0, 0},
    {-2, 0}, {0, -2}, {2, 0}, {0, 2},         /* +-l2 on one axis  (code 2) */
    {-4, 0}, {0, -4}, {4, 0}, {0, 4},         /* +-l4 on one axis  (code 4) */
    {-4, -4}, {4, -4}, {-4, 4}, {4, 4},       /* (+-l4, +-l4) */
    {-5, -5}, {-5, 5}, {5, -5}, {5, 5},       /* (+-l5, +-l5) */
};

void xo_gm_rule(double* w7 /*[17]*/, double* w5 /*[17]*/, double* lam /*[6] by code*/) {
    const double a = (12824. - 9120. * 2. + 400. * 4.) / 19683., b = 980. / 6561.;
    const double c = (1820. - 400. * 2.) / 19683., d = 200. / 19683., f = 6859. / 19683. / 4.;
    const double a5 = (729. - 950. * 2. + 50. * 4.) / 729., b5 = 245. / 486.;
    const double c5 = (265. - 100. * 2.) / 1458., d5 = 25. / 729.;
    for (int p = 0; p < 17; ++p) {
        w7[p] = p == 0 ? a : p < 5 ? b : p < 9 ? c : p < 13 ? d : f;
        w5[p] = p == 0 ? a5 : p < 5 ? b5 : p < 9 ? c5 : p < 13 ? d5 : 0.;
    }
    for (int k = 0; k < 6; ++k) lam[k] = 0.;
    lam[2] = GM_L2; lam[4] = GM_L4; lam[5] = GM_L5;
}

/* mean PSF over one pixel [E] by adaptive Genz-Malik cubature; returns the
 * number of regions evaluated.  abcd: corner unit vectors LL, LR, UR, UL;
 * dimension 0 runs along the map's first axis (h), dimension 1 along w. */
int xo_adaptive_pixel(const double* abcd /*[4][3]*/, const double* lut /*[D,E]*/, int E,
                      const double* src, double rtol, int max_depth, double* mean /*[E]*/) {
    double w7[17], w5[17], lam[6];
    xo_gm_rule(w7, w5, lam);
    struct { double c0, c1, h0, h1; int depth; } stack[64];
    int top = 0, nreg = 0;
    stack[top].c0 = 0.; stack[top].c1 = 0.; stack[top].h0 = 1.; stack[top].h1 = 1.; stack[top].depth = 0; ++top;
    double* f = (double*)malloc(sizeof(double) * 17 * E);
    for (int e = 0; e < E; ++e) mean[e] = 0.;
    while (top > 0) {
        --top;
        const double c0 = stack[top].c0, c1 = stack[top].c1, h0 = stack[top].h0, h1 = stack[top].h1;
        const int depth = stack[top].depth;
        ++nreg;
        for (int p = 0; p < 17; ++p) {
            const int o0 = GM_OFF[p][0], o1 = GM_OFF[p][1];
            const double x0 = c0 + (o0 < 0 ? -lam[-o0] : lam[o0]) * h0;   /* v: along h */
            const double x1 = c1 + (o1 < 0 ? -lam[-o1] : lam[o1]) * h1;   /* u: along w */
            const double u = x1, v = x0;
            const double nn = (1.0 - u) * (1.0 - v), pn = (1.0 + u) * (1.0 - v);
            const double pp = (1.0 + u) * (1.0 + v), np = (1.0 - u) * (1.0 + v);
            double q[3];
            for (int k = 0; k < 3; ++k)
                q[k] = 0.25 * (nn * abcd[k] + pn * abcd[3 + k] + pp * abcd[6 + k] + np * abcd[9 + k]) - src[k];
            const double sd = 2.0 * R2D * asin(0.5 * sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]));
            const double j = sd < 1e-4 ? 1. : 1. + RECIPSTEP * (LN_1E4 + log(sd));
            int idx = 1 + (int)(unsigned short)j;
            if (idx > 400) idx = 400;
            const double t = REDM1 * (sd * 1e4 * exp(SEP_STEP * (2. - idx)) - 1.);
            const double* YL = lut + (size_t)E * (idx - 1);
            const double* YR = lut + (size_t)E * idx;
            for (int e = 0; e < E; ++e) f[p * E + e] = (1.0 - t) * YL[e] + t * YR[e];
        }
        const double area = h0 * h1;  /* fraction of the pixel */
        double rel = 0.;
        for (int e = 0; e < E; ++e) {
            double v7 = 0., v5 = 0.;
            for (int p = 0; p < 17; ++p) { v7 += w7[p] * f[p * E + e]; v5 += w5[p] * f[p * E + e]; }
            const double err = fabs(v5 - v7);
            const double r = v7 != 0. ? err / fabs(v7) : (err != 0. ? INFINITY : 0.);
            if (r > rel) rel = r;
        }
        if (rel <= rtol || depth >= max_depth) {
            for (int e = 0; e < E; ++e) {
                double v7 = 0.;
                for (int p = 0; p < 17; ++p) v7 += w7[p] * f[p * E + e];
                mean[e] += area * v7;
            }
            continue;
        }
        /* split the dimension with the larger fourth divided difference */
        double dd[2] = {0., 0.};
        for (int e = 0; e < E; ++e) {
            const double f0 = 2. * f[e];
            dd[0] += fabs((f[1 * E + e] + f[3 * E + e] - f0) - (1. / 7.) * (f[5 * E + e] + f[7 * E + e] - f0));
            dd[1] += fabs((f[2 * E + e] + f[4 * E + e] - f0) - (1. / 7.) * (f[6 * E + e] + f[8 * E + e] - f0));
        }
        const int dim = dd[0] >= dd[1] ? 0 : 1;
        for (int side = 1; side >= -1; side -= 2) {  /* the lower half is evaluated first */
            stack[top].c0 = c0; stack[top].c1 = c1; stack[top].h0 = h0; stack[top].h1 = h1;
            stack[top].depth = depth + 1;
            if (dim == 0) { stack[top].h0 = 0.5 * h0; stack[top].c0 = c0 + side * 0.5 * h0; }
            else { stack[top].h1 = 0.5 * h1; stack[top].c1 = c1 + side * 0.5 * h1; }
            ++top;
        }
    }
    free(f);
    return nreg;
}

void xo_adaptive_cubature_map(const xo_wcs* w, const double* src_sph, int S, const double* upsf,
                              int E, double rtol, int max_depth, double* out /*[S,H,W,E]*/,
                              int* nregions /*[S,H,W] or NULL*/) {
    long Nh = w->naxis1, Nw = w->naxis2;
    for (int s = 0; s < S; ++s) {
        double src[3];
        xo_sph2dir(src_sph[2 * s], src_sph[2 * s + 1], src);
        for (long h = 0; h < Nh; ++h)
            for (long x = 0; x < Nw; ++x) {
                double abcd[12];
                const double ph = 1. + h, pw = 1. + x;
                xo_pix2dir(w, ph - 0.5, pw - 0.5, abcd);     /* LL */
                xo_pix2dir(w, ph - 0.5, pw + 0.5, abcd + 3); /* LR */
                xo_pix2dir(w, ph + 0.5, pw + 0.5, abcd + 6); /* UR */
                xo_pix2dir(w, ph + 0.5, pw - 0.5, abcd + 9); /* UL */
                const size_t k = ((size_t)s * Nh + h) * Nw + x;
                const int n = xo_adaptive_pixel(abcd, upsf + (size_t)s * XO_ND * E, E, src, rtol,
                                                max_depth, out + k * E);
                if (nregions) nregions[k] = n;
            }
    }
}

void xo_point_src_model_map_wcs_adaptive(const xo_wcs* w, const double* src_sph, int S,
                                         const double* expo, const double* upsf,
                                         const double* partial, int E, double rtol, int max_depth,
                                         double* out, double* inv, double* factor, double* radius,
                                         int* in_fov, int* nregions) {
    xo_adaptive_cubature_map(w, src_sph, S, upsf, E, rtol, max_depth, out, nregions);
    finish_model_map(w, src_sph, S, expo, upsf, partial, E, out, inv, factor, radius, in_fov);
}
