// Interface-compatible stand-in for the reference's Fermi::SkyGeom
// (xtsrcmaps/sky_geom/sky_geom.hxx:17-380), used only to compile the reference's
// own model-map translation units into the CPU checker under oracle/_ref.
//
// TEST INFRASTRUCTURE ONLY.  The reference class wraps wcslib, which is not in
// this image, and its pix2dir passes a std::array where a std::pair is expected
// (sky_geom.hxx:277-279), which g++ 13 rejects once the cubature instantiates
// it.  This class keeps the member names, argument types and the reference's
// conventions (CRVAL1 > 180 stored as CRVAL1 - 360; RA from pix2sph folded into
// [0, 360); longitudes beyond +-180 wrapped before sph2pix) and computes the
// CAR/AIT projections with the oracle's FP64 restatement of FITS-WCS
// (Calabretta & Greisen 2002), xo_wcs_pix2sph / xo_wcs_sph2pix.
#pragma once

#include "xtsrcmaps/misc/misc.hxx"

#include <array>
#include <cmath>
#include <concepts>
#include <string>
#include <utility>

#include "xts_oracle.h"

namespace Fermi {

struct WcsConfig {
    std::array<long, 3>   naxes;
    std::array<double, 3> crpix;
    std::array<double, 3> crval;
    std::array<double, 3> cdelt;
    double                axis_rot;
    std::string           proj_name;
    bool                  is_galactic;
};

template <typename T>
class SkyGeom {
    xo_wcs              m_w {};
    std::string         m_proj_name;
    bool                m_is_galactic { false };
    std::array<long, 2> m_naxes { 0, 0 };
    double              m_crval[2] { 0., 0. };
    double              m_crpix[2] { 0., 0. };
    double              m_cdelt[2] { 0., 0. };

  public:
    SkyGeom() = default;

    SkyGeom(long naxis1, long naxis2, std::string const& proj_name, bool is_galactic,
            double crpix1, double crpix2, double crval1, double crval2, double cdelt1,
            double cdelt2, double axis_rot)
        : m_proj_name(proj_name), m_is_galactic(is_galactic), m_naxes({ naxis1, naxis2 }) {
        m_w.naxis1 = naxis1;
        m_w.naxis2 = naxis2;
        m_w.crpix1 = m_crpix[0] = crpix1;
        m_w.crpix2 = m_crpix[1] = crpix2;
        m_w.crval1 = m_crval[0] = crval1 > 180. ? crval1 - 360. : crval1;
        m_w.crval2 = m_crval[1] = crval2;
        m_w.cdelt1 = m_cdelt[0] = cdelt1;
        m_w.cdelt2 = m_cdelt[1] = cdelt2;
        m_w.crota2 = axis_rot;
        m_w.proj = proj_name == "AIT" ? 1 : 0;
        m_w.galactic = is_galactic ? 1 : 0;
    }

    SkyGeom(WcsConfig const& c)
        : SkyGeom(c.naxes[0], c.naxes[1], c.proj_name, c.is_galactic, c.crpix[0], c.crpix[1],
                  c.crval[0], c.crval[1], c.cdelt[0], c.cdelt[1], c.axis_rot) {}

    long const*   naxes() const { return &m_naxes[0]; }
    double const* crval() const { return m_crval; }
    double const* crpix() const { return m_crpix; }
    double const* cdelt() const { return m_cdelt; }
    double        axis_rot() const { return m_w.crota2; }

    auto sph2pix(std::array<T, 2> const& ss) const -> std::array<T, 2> {
        double p1, p2;
        to_pix(ss[0], ss[1], &p1, &p2);
        return { static_cast<T>(p1), static_cast<T>(p2) };
    }
    auto sph2pix(std::pair<T, T> const& ss) const -> std::pair<T, T> {
        double p1, p2;
        to_pix(ss.first, ss.second, &p1, &p2);
        return { static_cast<T>(p1), static_cast<T>(p2) };
    }
    auto pix2sph(std::array<T, 2> const& px) const -> std::array<T, 2> { return pix2sph(px[0], px[1]); }
    auto pix2sph(T const first, T const second) const -> std::array<T, 2> {
        double ra, dec;
        xo_wcs_pix2sph(&m_w, first, second, &ra, &dec);
        while (ra < 0) ra += 360.;
        while (ra >= 360) ra -= 360.;
        return { static_cast<T>(ra), static_cast<T>(dec) };
    }
    auto dir2sph(std::array<T, 3> const& dir) const -> std::array<T, 2> {
        T ra = std::atan2(dir[1], dir[0]) * rad2deg;
        while (ra < 0) ra += 360.;
        while (ra > 360) ra -= 360.;
        return { ra, static_cast<T>(std::asin(dir[2]) * rad2deg) };
    }
    auto pix2dir(std::array<T, 2> const& px) const -> std::array<T, 3> {
        auto const s = pix2sph(px);
        return sph2dir(std::pair<T, T> { s[0], s[1] });
    }
    auto sph2dir(std::pair<T, T> const& s) const -> std::array<T, 3> {
        T const cr = std::cos(s.first * deg2rad), cd = std::cos(s.second * deg2rad);
        T const sr = std::sin(s.first * deg2rad), sd = std::sin(s.second * deg2rad);
        return { cr * cd, sr * cd, sd };
    }
    // psf_boundary_radius.cxx:37-55 passes arrays; a template so that braced
    // lists (cubature.implementation.cxx:41, map_integral.cxx:25) still pick the pair
    template <typename A>
        requires std::same_as<A, std::array<T, 2>>
    auto sph2dir(A const& s) const -> std::array<T, 3> {
        return sph2dir(std::pair<T, T> { s[0], s[1] });
    }
    auto refpix() const -> std::array<T, 2> { return { m_crpix[0], m_crpix[1] }; }
    auto refsph() const -> std::array<T, 2> { return { m_crval[0], m_crval[1] }; }

    static inline auto dir_diff(std::array<T, 3> const& L, std::array<T, 3> const& R) -> T {
        T const a = L[0] - R[0], b = L[1] - R[1], c = L[2] - R[2];
        return 2. * std::asin(0.5 * std::sqrt(a * a + b * b + c * c));
    }
    auto srcpixoff(std::array<T, 3> const& src, std::array<T, 3> const& pix) const -> T {
        return dir_diff(src, pix) * rad2deg;
    }
    auto wcs_config() const -> WcsConfig {
        return { { m_naxes[0], m_naxes[1], 1l }, { m_crpix[0], m_crpix[1], 1.0 },
                 { m_crval[0], m_crval[1], 1.0 }, { m_cdelt[0], m_cdelt[1], 1.0 },
                 m_w.crota2, m_proj_name, m_is_galactic };
    }

  private:
    void to_pix(double s1, double s2, double* p1, double* p2) const {
        if (s1 > 180) s1 -= 360.;
        if (s1 < -180) s1 += 360.;
        xo_wcs_sph2pix(&m_w, s1, s2, p1, p2);
    }
};

}  // namespace Fermi
