/*
 * xts_oracle.h -- FP64 CPU oracle for the xtsrcmaps point-source model-map path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or calls
 * this code.  It is imported by the test-suite, by __graft_entry__.smoke() and by
 * bench.py's CPU baseline leg, where it acts as the checker (never as the thing
 * measured on the GPU and never as a fallback).
 *
 * Every function restates one reference routine (paths relative to the
 * xtsrcmaps source tree) in plain C99 with double precision throughout.  All
 * tensors are row-major with the last index contiguous, as in the reference
 * Fermi::Tensor (tensor/tensor.hpp:113-122).
 *
 * Shapes: S sources, C cos-theta bins of the livetime cube, E energies,
 * D = 401 PSF separations, H x W map pixels (H = NAXIS1, W = NAXIS2).
 */
#ifndef XTS_ORACLE_H
#define XTS_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define XO_ND 401

/* FITS-WCS description of a celestial map (sky_geom/sky_geom.hxx:17-25). */
typedef struct xo_wcs {
    long   naxis1, naxis2;
    double crpix1, crpix2;
    double crval1, crval2;
    double cdelt1, cdelt2;
    double crota2;        /* degrees */
    int    proj;          /* 0 = CAR, 1 = AIT */
    int    galactic;      /* labels only, the arithmetic is identical */
} xo_wcs;

/* One IRF grid after irf/irf.prepare_grid.cpp:26-102 (padded axes). */
typedef struct xo_grid {
    const double* cosths;  /* [Mc] */
    int           n_cos;
    const double* logEs;   /* [Me] */
    int           n_e;
    const double* params;  /* [Mc, Me, n_par] */
    int           n_par;
    double        min_cos_theta;
} xo_grid;

/* ---- separations & constants (psf/psf.hxx:20-43, misc/misc.hxx:11-39) ---- */
void xo_separations(double* seps /*[401]*/);

/* ---- geometry ---- */
void xo_wcs_pix2sph(const xo_wcs* w, double p1, double p2, double* ra, double* dec);
void xo_wcs_sph2pix(const xo_wcs* w, double ra, double dec, double* p1, double* p2);
void xo_sph2dir(double ra, double dec, double* dir3);
void xo_pix2dir(const xo_wcs* w, double p1, double p2, double* dir3);
double xo_dir_diff(const double* a, const double* b);
long long xo_ang2pix_nest(double theta, double phi, long long nside);
void xo_pix2ang_nest(long long pix, long long nside, double* theta, double* phi);

/* ---- step (a): exposure ---- */
void xo_costhetas(int nbins, double cosmin, int thetabin, double* out /*[C]*/);
void xo_src_cosbins(const double* src_sph, int S, const float* cube /*[npix,C]*/,
                    long long nside, int C, double* out /*[S,C]*/);
void xo_aeff_value(const double* costh, int C, const double* logEs, int E,
                   const xo_grid* aeff, double* out /*[C,E]*/);
void xo_livetime_efficiency_factors(const double* logEs, int E, const float* p0,
                                    const float* p1, double* out /*[2,E]*/);
void xo_exposure(const double* ecb, const double* wecb, int S, int C,
                 const double* aeff_f, const double* aeff_b, const double* ltf,
                 int E, double* out /*[S,E]*/);

/* ---- step (b): mean PSF ---- */
void xo_gauss_legendre_64(double* nodes, double* weights);
double xo_evaluate_king(double sep, double sf, const double* pars);
double xo_psf_base_integral(double radius_deg, double sf, const double* pars);
void xo_normalize_rpsf(double* params /*[Mc,Me,6]*/, int Mc, int Me,
                       const double* grid_logEs /*[Me]*/, float scale0,
                       float scale1, float scale_index);
void xo_king(const xo_grid* psf, double* out /*[D,Mc,Me]*/);
void xo_psf_bilerp(const double* costh, int C, const double* logEs, int E,
                   const xo_grid* psf, const double* kings, double* out /*[C,D,E]*/);
void xo_corrected_exposure_psf(const double* obs_psf /*[C,D,E]*/,
                               const double* aeff /*[C,E]*/, const double* ecb,
                               const double* wecb, int S, int C, int E,
                               const double* ltf, double* out /*[S,D,E]*/);
void xo_mean_psf(const double* front, const double* back, const double* expo,
                 int S, int E, double* out);
void xo_partial_total_integral(const double* upsf, int S, int E,
                               double* partial, double* total);
void xo_normalize(double* upsf, const double* total, int S, int E);
void xo_compute_psf_data(const xo_grid* psf_front, const xo_grid* psf_back,
                         const double* costh, int C, const double* logEs, int E,
                         const double* aeff_f, const double* aeff_b,
                         const double* ecb, const double* wecb, int S,
                         const double* ltf, const double* expo,
                         double* upsf /*[S,D,E]*/, double* partial /*[S,D,E]*/);

/* ---- steps (c)+(d): point-source model map ---- */
void xo_square_ptswts(const xo_wcs* w, long Nh, long Nw, double* out /*[H,W,48]*/);
void xo_convolve_pixel_logsep(double* map_e, int E, const double* pw48,
                              const double* lut /*[D,E]*/, const double* src3);
void xo_cubature_map(const xo_wcs* w, long Nh, long Nw, const double* src_sph, int S,
                     const double* upsf, int E, double* out /*[S,H,W,E]*/);
void xo_solid_angle(const xo_wcs* w, long Nh, long Nw, double* out /*[H,W]*/);
void xo_psf_boundary_radius(const xo_wcs* w, long Nh, long Nw, const double* src_sph,
                            int S, double* radius, int* in_fov);
void xo_map_integral(const double* map, const xo_wcs* w, long Nh, long Nw,
                     const double* src_sph, int S, int E, const double* radius,
                     const int* in_fov, double* inv_integ /*[S,E]*/);
void xo_map_correction_factor(const double* inv_integ, const double* radius,
                              const int* in_fov, const double* upsf,
                              const double* partial, int S, int E,
                              double* factor /*[S,E]*/);
void xo_point_src_model_map_wcs(const xo_wcs* w, const double* src_sph, int S,
                                const double* expo, const double* upsf,
                                const double* partial, int E,
                                double* out /*[S,H,W,E]*/, double* inv_integ,
                                double* factor, double* radius, int* in_fov);

/* ---- row d3: adaptive Genz-Malik cubature (see xts_oracle.c) ---- */
void xo_gm_rule(double* w7 /*[17]*/, double* w5 /*[17]*/, double* lam /*[6]*/);
int xo_adaptive_pixel(const double* abcd /*[4][3]*/, const double* lut /*[D,E]*/, int E,
                      const double* src3, double rtol, int max_depth, double* mean /*[E]*/);
void xo_adaptive_cubature_map(const xo_wcs* w, const double* src_sph, int S, const double* upsf,
                              int E, double rtol, int max_depth, double* out /*[S,H,W,E]*/,
                              int* nregions /*[S,H,W] or NULL*/);
void xo_point_src_model_map_wcs_adaptive(const xo_wcs* w, const double* src_sph, int S,
                                         const double* expo, const double* upsf,
                                         const double* partial, int E, double rtol, int max_depth,
                                         double* out, double* inv_integ, double* factor,
                                         double* radius, int* in_fov, int* nregions);

#ifdef __cplusplus
}
#endif
#endif
