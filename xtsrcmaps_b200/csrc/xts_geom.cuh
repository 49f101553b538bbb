// xts_geom.cuh -- FP64 sky geometry for the device: FITS-WCS (CAR, AIT), unit
// vectors, great-circle separations and HEALPix NESTED ang2pix.
//
// The reference calls wcslib through SkyGeom (sky_geom/sky_geom.hxx:79-310);
// here the FITS-WCS algorithm of Calabretta & Greisen (2002, A&A 395, 1077) is
// written out for the two projections the path uses, with the default
// LONPOLE/LATPOLE rule for theta0 = 0 projections.  HEALPix follows Gorski et
// al. (2005), as healpix/healpix.cxx:181-229 does.
#pragma once

#include "xts_internal.cuh"

namespace xts {

struct WcsDev {
    double crpix1, crpix2, cdelt1, cdelt2;
    double cosr, sinr;       // CROTA2
    int rotated;
    int proj;                // 0 CAR, 1 AIT
    double alpha_p, phi_p;   // celestial longitude of the native pole, LONPOLE (deg)
    double sin_dp, cos_dp;   // native pole latitude
};

XTS_HD inline WcsDev make_wcs(const xts_wcs& w) {
    WcsDev d;
    d.crpix1 = w.crpix1; d.crpix2 = w.crpix2;
    d.cdelt1 = w.cdelt1; d.cdelt2 = w.cdelt2;
    d.rotated = w.crota2 != 0.0;
    d.cosr = cos(w.crota2 * D2R); d.sinr = sin(w.crota2 * D2R);
    d.proj = w.proj;
    double a0 = w.crval1 > 180. ? w.crval1 - 360. : w.crval1;  // sky_geom.hxx:110
    double d0 = w.crval2, dp;
    if (d0 >= 0.) { d.phi_p = 0.;   dp = 90. - d0; d.alpha_p = a0 - 180.; }
    else          { d.phi_p = 180.; dp = 90. + d0; d.alpha_p = a0; }
    d.sin_dp = sin(dp * D2R); d.cos_dp = cos(dp * D2R);
    return d;
}

XTS_HD inline double clamp1(double x) { return x > 1. ? 1. : (x < -1. ? -1. : x); }

// sky_geom.hxx:281-287
XTS_HD inline void sph2dir(double ra, double dec, double* v) {
    double cr = cos(ra * D2R), cd = cos(dec * D2R), sr = sin(ra * D2R), sd = sin(dec * D2R);
    v[0] = cr * cd; v[1] = sr * cd; v[2] = sd;
}

// sky_geom.hxx:237-250 (wcsp2s): 1-based pixel -> (ra, dec) degrees, ra in [0, 360)
XTS_HD inline void pix2sph(const WcsDev& w, double p1, double p2, double* ra, double* dec) {
    double dp1 = p1 - w.crpix1, dp2 = p2 - w.crpix2, x, y;
    if (!w.rotated) { x = w.cdelt1 * dp1; y = w.cdelt2 * dp2; }
    else {
        x = w.cdelt1 * w.cosr * dp1 - w.cdelt2 * w.sinr * dp2;
        y = w.cdelt1 * w.sinr * dp1 + w.cdelt2 * w.cosr * dp2;
    }
    double phi, theta;
    if (w.proj == 0) { phi = x; theta = y; }
    else {
        double X = x * D2R, Y = y * D2R;
        double z2 = 1.0 - 0.0625 * X * X - 0.25 * Y * Y;
        double z = sqrt(z2 > 0. ? z2 : 0.);
        phi = 2.0 * atan2(0.5 * X * z, 2.0 * z2 - 1.0) * R2D;
        theta = asin(clamp1(Y * z)) * R2D;
    }
    double st = sin(theta * D2R), ct = cos(theta * D2R);
    double dphi = (phi - w.phi_p) * D2R;
    double cdp = cos(dphi), sdp = sin(dphi);
    double xr = st * w.cos_dp - ct * w.sin_dp * cdp;
    double yr = -ct * sdp;
    double a = w.alpha_p + atan2(yr, xr) * R2D;
    double dd = asin(clamp1(st * w.sin_dp + ct * w.cos_dp * cdp)) * R2D;
    while (a < 0.) a += 360.;
    while (a >= 360.) a -= 360.;
    *ra = a; *dec = dd;
}

// sky_geom.hxx:179-206 (wcss2p): (ra, dec) -> 1-based pixel
XTS_HD inline void sph2pix(const WcsDev& w, double ra, double dec, double* p1, double* p2) {
    double sd = sin(dec * D2R), cd = cos(dec * D2R);
    double da = (ra - w.alpha_p) * D2R;
    double cda = cos(da), sda = sin(da);
    double xr = sd * w.cos_dp - cd * w.sin_dp * cda;
    double yr = -cd * sda;
    double phi = w.phi_p + atan2(yr, xr) * R2D;
    double theta = asin(clamp1(sd * w.sin_dp + cd * w.cos_dp * cda)) * R2D;
    while (phi > 180.) phi -= 360.;
    while (phi <= -180.) phi += 360.;
    double x, y;
    if (w.proj == 0) { x = phi; y = theta; }
    else {
        double ct = cos(theta * D2R);
        double g = R2D * sqrt(2.0 / (1.0 + ct * cos(0.5 * phi * D2R)));
        x = 2.0 * g * ct * sin(0.5 * phi * D2R);
        y = g * sin(theta * D2R);
    }
    double dp1, dp2;
    if (!w.rotated) { dp1 = x / w.cdelt1; dp2 = y / w.cdelt2; }
    else {
        dp1 = (w.cosr * x + w.sinr * y) / w.cdelt1;
        dp2 = (-w.sinr * x + w.cosr * y) / w.cdelt2;
    }
    *p1 = w.crpix1 + dp1; *p2 = w.crpix2 + dp2;
}

XTS_HD inline void pix2dir(const WcsDev& w, double p1, double p2, double* v) {
    double ra, dec;
    pix2sph(w, p1, p2, &ra, &dec);
    sph2dir(ra, dec, v);
}

// sky_geom.hxx:305-310: 2 asin(|a - b| / 2), radians
XTS_HD inline double dir_diff(const double* a, const double* b) {
    double x = a[0] - b[0], y = a[1] - b[1], z = a[2] - b[2];
    return 2. * asin(0.5 * sqrt(x * x + y * y + z * z));
}

// ---------------------------------------------------------------- HEALPix
XTS_HD inline unsigned long long spread_bits(unsigned long long v) {
    v &= 0xffffffffull;
    v = (v | (v << 16)) & 0x0000ffff0000ffffull;
    v = (v | (v << 8)) & 0x00ff00ff00ff00ffull;
    v = (v | (v << 4)) & 0x0f0f0f0f0f0f0f0full;
    v = (v | (v << 2)) & 0x3333333333333333ull;
    v = (v | (v << 1)) & 0x5555555555555555ull;
    return v;
}

XTS_HD inline int ilog2_ll(long long v) { int r = 0; while (v > 1) { v >>= 1; ++r; } return r; }

// healpix/healpix.cxx:181-229 (NESTED ordering)
XTS_HD inline long long ang2pix_nest(double theta, double phi, long long nside) {
    bool have_sth = (theta < 0.01) || (theta > PI - 0.01);
    double sth = have_sth ? sin(theta) : 0.;
    double z = cos(theta), za = fabs(z);
    double tt = phi * INV_HALFPI;
    if (tt >= 0) tt = (tt < 4.0) ? tt : fmod(tt, 4.0);
    else { double t = fmod(tt, 4.0) + 4.0; tt = (t == 4.0) ? 0. : t; }
    int order = ilog2_ll(nside);
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
    return (face << (2 * order)) + (long long)spread_bits(ix) + ((long long)spread_bits(iy) << 1);
}

}  // namespace xts
