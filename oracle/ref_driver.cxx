// ref_driver.cxx -- flat-array C entry points over the reference's own
// translation units, compiled in place from the reference tree into
// oracle/_ref/libxts_ref.so by oracle/build_ref.sh.
//
// TEST INFRASTRUCTURE ONLY: the CPU checker and the timed CPU reference arm.
// Nothing in the product path loads this library.
//
// What runs is the reference's code: Exposure::costhetas, map, src_cosbins and
// exposure (exposure/exposure.cxx, exposure.contract.cpp, healpix/healpix.cxx),
// Psf::psf_lookup_table_and_partial_integrals and the functions it calls
// (psf/psf.*.cxx), and ModelMap::point_src_model_map_wcs with everything it
// calls (model_map/model_map.*.cxx, mm_cubature/cubature.implementation.cxx).
// Three things are supplied here because the image lacks what the reference
// builds against: the WCS projections (a SkyGeom stand-in over the oracle's
// CAR/AIT, oracle/ref_overlay), cblas_dgemm (below, plain FP64 loops) and the
// effective-area evaluation Irf::aeff_value, whose translation unit needs
// <mdspan> (callers pass the Aeff tables, e.g. from the oracle's xo_aeff_value).
// The cubature uses convolve_pixel_psf_logsep with its missing key store added
// by the build recipe (the shipped kernel never writes keys[] and reads row -1).
#include <omp.h>

#include <cstring>
#include <string>
#include <vector>

#include "cblas.h"
#include "xtsrcmaps/exposure/exposure.hxx"
#include "xtsrcmaps/model_map/model_map.hxx"
#include "xtsrcmaps/psf/psf.hxx"
#include "xtsrcmaps/sky_geom/sky_geom.hxx"
#include "xts_oracle.h"

extern "C" void cblas_dgemm(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE ta, enum CBLAS_TRANSPOSE tb,
                            int M, int N, int K, double alpha, const double* A, int lda, const double* B,
                            int ldb, double beta, double* C, int ldc) {
    // row-major only (the reference's call sites), C = alpha op(A) op(B) + beta C;
    // rows in parallel, standing in for the threaded BLAS the reference links
    if (order != CblasRowMajor) return;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < M; ++i) {
        std::vector<double> acc((size_t)N, 0.0);
        for (int k = 0; k < K; ++k) {
            const double a = ta == CblasNoTrans ? A[(size_t)i * lda + k] : A[(size_t)k * lda + i];
            if (tb == CblasNoTrans) {
                const double* b = B + (size_t)k * ldb;
                for (int j = 0; j < N; ++j) acc[j] += a * b[j];
            } else {
                for (int j = 0; j < N; ++j) acc[j] += a * B[(size_t)j * ldb + k];
            }
        }
        double* c = C + (size_t)i * ldc;
        for (int j = 0; j < N; ++j) c[j] = alpha * acc[j] + (beta == 0.0 ? 0.0 : beta * c[j]);
    }
}

namespace {

using Fermi::Tensor;

Tensor<double, 2> t2(const double* p, size_t a, size_t b) {
    return Tensor<double, 2>(p, p + a * b, std::array<size_t, 2> { a, b });
}
Tensor<double, 3> t3(const double* p, size_t a, size_t b, size_t c) {
    return Tensor<double, 3>(p, p + a * b * c, std::array<size_t, 3> { a, b, c });
}

Fermi::Irf::IrfData3 grid(const xo_grid& g) {
    Fermi::Irf::IrfData3 d;
    d.cosths = Tensor<double, 1>(g.cosths, g.cosths + g.n_cos, std::array<size_t, 1> { (size_t)g.n_cos });
    d.logEs = Tensor<double, 1>(g.logEs, g.logEs + g.n_e, std::array<size_t, 1> { (size_t)g.n_e });
    d.params = t3(g.params, g.n_cos, g.n_e, g.n_par);
    d.minCosTheta = g.min_cos_theta;
    return d;
}

Fermi::Obs::ExposureCubeData cube(const float* cosbins, long nside, int C, double cosmin, int thetabin) {
    Fermi::Obs::ExposureCubeData c;
    c.cosbins.assign(cosbins, cosbins + (size_t)12 * nside * nside * C);
    c.nside = (unsigned)nside;
    c.nbrbins = (unsigned)C;
    c.cosmin = cosmin;
    c.ordering = "NESTED";
    c.coordsys = "EQU";
    c.thetabin = thetabin != 0;
    return c;
}

}  // namespace

extern "C" {

// OpenMP threads of the reference code (its cubature runs sources in parallel,
// cubature.implementation.cxx:39, schedule(static, 16)).
int xr_set_threads(int n) {
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
}

// Exposure::costhetas + map + src_cosbins + exposure (exposure.hxx:44-88 without
// aeff_value): outputs costh [C], ecb/wecb [S, C], exposure [S, E].
int xr_exposure(const float* cosbins, const float* wcosbins, long nside, int C, double cosmin,
                int thetabin, const double* src_sph, int S, const double* front_aeff,
                const double* back_aeff, const double* ltf, int E, double* costh, double* ecb,
                double* wecb, double* exposure) {
    auto const ec = cube(cosbins, nside, C, cosmin, thetabin);
    auto const wc = cube(wcosbins, nside, C, cosmin, thetabin);
    auto const ct = Fermi::Exposure::costhetas(ec);
    auto const src = t2(src_sph, S, 2);
    auto const x = Fermi::Exposure::src_cosbins(src, Fermi::Exposure::map(ec));
    auto const w = Fermi::Exposure::src_cosbins(src, Fermi::Exposure::map(wc));
    auto const e = Fermi::Exposure::exposure(x, w, t2(front_aeff, C, E), t2(back_aeff, C, E), t2(ltf, 2, E));
    std::copy(ct.begin(), ct.end(), costh);
    std::memcpy(ecb, x.data(), sizeof(double) * S * C);
    std::memcpy(wecb, w.data(), sizeof(double) * S * C);
    std::memcpy(exposure, e.data(), sizeof(double) * S * E);
    return 0;
}

// Psf::psf_lookup_table_and_partial_integrals (psf.psf_lookup_table_and_partial_integrals.cxx:8-57):
// normalised King grids -> uPsf, partial [S, 401, E].
int xr_psf(const xo_grid* rpsf_front, const xo_grid* rpsf_back, const double* costh, int C,
           const double* logEs, int E, const double* front_aeff, const double* back_aeff,
           const double* ecb, const double* wecb, int S, const double* ltf, const double* exposure,
           double* upsf, double* partial) {
    Fermi::Irf::psf::Pass8FB d;
    d.front.rpsf = grid(*rpsf_front);
    d.back.rpsf = grid(*rpsf_back);
    auto [u, p] = Fermi::Psf::psf_lookup_table_and_partial_integrals(
        d, std::vector<double>(costh, costh + C), std::vector<double>(logEs, logEs + E), t2(front_aeff, C, E),
        t2(back_aeff, C, E), t2(ecb, S, C), t2(wecb, S, C), t2(ltf, 2, E), t2(exposure, S, E));
    std::memcpy(upsf, u.data(), sizeof(double) * S * XO_ND * E);
    std::memcpy(partial, p.data(), sizeof(double) * S * XO_ND * E);
    return 0;
}

// ModelMap::point_src_model_map_wcs (model_map.point_src_model_map_wcs.cxx:6-45) -> [S, H, W, E].
int xr_point_src_model_map_wcs(const xo_wcs* w, const double* src_sph, int S, const double* exposure,
                               const double* upsf, const double* partial, int E, double* out) {
    Fermi::SkyGeom<double> g(w->naxis1, w->naxis2, w->proj == 1 ? "AIT" : "CAR", w->galactic != 0, w->crpix1,
                             w->crpix2, w->crval1, w->crval2, w->cdelt1, w->cdelt2, w->crota2);
    std::vector<std::string> names((size_t)S);
    auto const m = Fermi::ModelMap::point_src_model_map_wcs(
        (size_t)w->naxis1, (size_t)w->naxis2, g, t2(src_sph, S, 2), names, t2(exposure, S, E),
        t3(upsf, S, XO_ND, E), t3(partial, S, XO_ND, E));
    std::memcpy(out, m.data(), sizeof(double) * (size_t)S * w->naxis1 * w->naxis2 * E);
    return 0;
}

}  // extern "C"
