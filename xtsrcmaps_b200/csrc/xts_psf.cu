// xts_psf.cu -- step (b): exposure-weighted mean King PSF tables.
//
//   b2 separations            psf/psf.hxx:24-31
//   b3 King table [D,Mc,Me]   psf/psf.king.cxx:9-43
//   b4 bilerp -> [C,D,E]      psf/psf.bilerp.cxx:6-52
//   b5 corrected_exposure_psf psf/psf.corrected_exposure_psf.cxx:12-120
//   b6 mean_psf               psf/psf.mean_psf.cxx:6-33
//   b7 partial/total, normalise psf/psf.partial_total_integral.cxx:8-52, psf/psf.normalize.cxx:7-24
//
// Front and back both use the front livetime-efficiency factors
// (psf.psf_lookup_table_and_partial_integrals.cxx:151-156), so the two sides'
// psf*aeff tables are summed before the contraction over cos-theta:
//   mean[s,d,e] = (sum_c (X[s,c] L0[e] + W[s,c] L1[e]) (Pf Af + Pb Ab)[c,d,e]) / exposure[s,e]
// which is the reference's four DGEMMs and three sums reassociated.
#include <math.h>

#include "xts_internal.cuh"

namespace xts {

__device__ __forceinline__ double sep_deg(int d) {  // psf/psf.hxx:24-31
    const double xstep = log(70. / 1e-4) / (400 - 1.);
    return d == 0 ? 0.0 : 1e-4 * exp((d - 1) * xstep);
}

__device__ inline double king_f2(double u, double g) {
    if (g == 1) g = 1.001;
    return (1. - 1. / g) * pow(1. + u / g, -g);
}

// b3: K[side][d][c][e] = evaluate_king(sep[d] rad, 1, params[c,e,:]) (irf/irf.hxx:22-45)
__global__ void k_king(xts_grid pf, xts_grid pb, double* kf, double* kb) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int side = blockIdx.y;
    const xts_grid& g = side ? pb : pf;
    int McMe = g.n_cos * g.n_e;
    if (i >= ND * McMe) return;
    int d = i / McMe, ce = i - d * McMe;
    const double* p = g.params + (size_t)ce * 6;
    double sep = sep_deg(d) * D2R;
    double ncore = p[0], ntail = p[1], score = p[2], stail = p[3];
    double rc = sep / score, uc = rc * rc / 2.;
    double rt = sep / stail, ut = rt * rt / 2.;
    (side ? kb : kf)[i] = ncore * king_f2(uc, p[4]) + ntail * ncore * king_f2(ut, p[5]);
}

__device__ inline void lerp_pars2(const double* g, int n, double v, double* wgt, double* cmpl,
                                  int* idx) {
    int lo = 0, hi = n;
    while (lo < hi) { int m = (lo + hi) >> 1; if (v < g[m]) hi = m; else lo = m + 1; }
    int i = lo < 1 ? 1 : (lo > n - 1 ? n - 1 : lo);
    double t = (v - g[i - 1]) / (g[i] - g[i - 1]);
    *wgt = t; *cmpl = 1. - t; *idx = i;
}

// b4 + the aeff product of b5, both sides summed: PA[c][d][e].  The bilinear
// weights depend on (side, e) and (side, c) only: each block looks them up once
// for all energies and its (at most two) cos-theta bins into shared memory.
static size_t psf_aeff_smem(int E) { return sizeof(double) * (4 * (size_t)E + 8) + sizeof(int) * (2 * (size_t)E + 4); }

__global__ void k_psf_aeff(xts_grid pf, xts_grid pb, const double* kf, const double* kb,
                           const double* costh, int C, const double* logEs, int E,
                           const double* af, const double* ab, double* pa) {
    extern __shared__ double sh[];
    double* sew = sh;              // [2][E] energy weight, complement
    double* sec = sew + 2 * E;
    double* scw = sec + 2 * E;     // [2 sides][2 bins] cos-theta weight, complement
    double* scc = scw + 4;
    int* sei = (int*)(scc + 4);    // [2][E], [2][2] indices
    int* sci = sei + 2 * E;
    const int i0 = blockIdx.x * blockDim.x;
    const int cfirst = i0 / (ND * E);
    for (int k = threadIdx.x; k < 2 * E + 4; k += blockDim.x) {
        if (k < 2 * E) {
            const int side = k / E, e = k - side * E;
            const xts_grid& g = side ? pb : pf;
            lerp_pars2(g.logEs, g.n_e, logEs[e], &sew[k], &sec[k], &sei[k]);
        } else {
            const int j = k - 2 * E, side = j >> 1, c = cfirst + (j & 1);
            const xts_grid& g = side ? pb : pf;
            if (c < C) lerp_pars2(g.cosths, g.n_cos, costh[c], &scw[j], &scc[j], &sci[j]);
        }
    }
    __syncthreads();
    int i = i0 + threadIdx.x;
    if (i >= C * ND * E) return;
    int e = i % E;
    int cd = i / E;
    int d = cd % ND, c = cd / ND;
    double v = 0.;
    for (int side = 0; side < 2; ++side) {
        const xts_grid& g = side ? pb : pf;
        const double* K = (side ? kb : kf) + (size_t)d * g.n_cos * g.n_e;
        const int jc = 2 * side + (c - cfirst), je = side * E + e;
        const double cw = scw[jc], cc = scc[jc], ew = sew[je], ec = sec[je];
        const int ci = sci[jc], ei = sei[je];
        int Me = g.n_e;
        double b = cc * ec * K[(ci - 1) * Me + ei - 1] + cc * ew * K[(ci - 1) * Me + ei] +
                   cw * ec * K[ci * Me + ei - 1] + cw * ew * K[ci * Me + ei];
        v += b * (side ? ab : af)[c * E + e];
    }
    pa[i] = v;
}

// b5 + b6: mean[s, de] by a register-tiled FP64 contraction over cos-theta:
// each block takes MP_TS sources and MP_CPT * 128 columns (d, e); each thread
// keeps MP_TS x MP_CPT pairs of accumulators (exposure and weighted exposure
// sides), reads its MP_CPT columns of psf*aeff once per cos-theta bin (coalesced,
// from L2) and the sources' cos-theta rows from shared memory (broadcast), so
// every shared load feeds 2 * MP_CPT FMAs and every column load 2 * MP_TS.
constexpr int PSF_TILE_S = 8;   // sources per block
constexpr int PSF_CPT = 4;      // columns per thread
constexpr int PSF_MAX_C = 64;

__global__ void __launch_bounds__(128) k_mean_psf(const double* __restrict__ pa, int C, int E,
                                                  const double* __restrict__ ecb, const double* __restrict__ wecb,
                                                  int S, const double* __restrict__ ltf,
                                                  const double* __restrict__ expo, double* __restrict__ out) {
    __shared__ double2 sxw[PSF_MAX_C][PSF_TILE_S];  // (exposure, weighted exposure) cos-theta rows
    const int s0 = blockIdx.y * PSF_TILE_S;
    const int ns = min(PSF_TILE_S, S - s0);
    for (int k = threadIdx.x; k < PSF_TILE_S * C; k += blockDim.x) {
        const int s = k / C, c = k - s * C;
        const bool ok = s < ns;
        sxw[c][s] = make_double2(ok ? ecb[(size_t)(s0 + s) * C + c] : 0., ok ? wecb[(size_t)(s0 + s) * C + c] : 0.);
    }
    __syncthreads();
    const int DE = ND * E;
    const int j0 = blockIdx.x * (128 * PSF_CPT) + threadIdx.x;
    double x[PSF_TILE_S][PSF_CPT], w[PSF_TILE_S][PSF_CPT];
#pragma unroll
    for (int s = 0; s < PSF_TILE_S; ++s)
#pragma unroll
        for (int q = 0; q < PSF_CPT; ++q) { x[s][q] = 0.; w[s][q] = 0.; }
#pragma unroll 2
    for (int c = 0; c < C; ++c) {
        double col[PSF_CPT];
#pragma unroll
        for (int q = 0; q < PSF_CPT; ++q) {
            const int j = j0 + 128 * q;
            col[q] = j < DE ? __ldg(pa + (size_t)c * DE + j) : 0.;
        }
#pragma unroll
        for (int s = 0; s < PSF_TILE_S; ++s) {
            const double2 xw = sxw[c][s];
#pragma unroll
            for (int q = 0; q < PSF_CPT; ++q) {
                x[s][q] = fma(xw.x, col[q], x[s][q]);
                w[s][q] = fma(xw.y, col[q], w[s][q]);
            }
        }
    }
#pragma unroll
    for (int q = 0; q < PSF_CPT; ++q) {
        const int j = j0 + 128 * q;
        if (j >= DE) continue;
        const int e = j % E;
        const double l0 = ltf[e], l1 = ltf[E + e];
#pragma unroll
        for (int s = 0; s < PSF_TILE_S; ++s)
            if (s < ns)
                out[(size_t)(s0 + s) * DE + j] = (x[s][q] * l0 + w[s][q] * l1) / expo[(size_t)(s0 + s) * E + e];
    }
}

// b7: per (s, e) exact integral of the linear interpolant of 2 pi u(theta) sin(theta)
// over each separation bin (psf.partial_total_integral.cxx:8-52), prefix sum,
// normalised partials, then uPsf /= total (psf.normalize.cxx:7-24).  One warp per
// (source, energy): each lane integrates a run of 13 bins, the runs are joined by
// a shuffle scan, and every lane normalises its own rows.  The reference forms
// the bin integral as 0.5 m (t2^2 - t1^2) + b (t2 - t1) with the slope m and
// intercept b of the interpolant; that is exactly the trapezoid
// 0.5 (t2 - t1)(y1 + y2), used here without its division (the two agree to a
// few ulp), and the normalisation multiplies by 1/total.
constexpr int PSCAN_ROWS = (ND - 1 + 31) / 32;  // bins per lane

__global__ void __launch_bounds__(256) k_partial_scan(double* upsf, double* partial, int E) {
    __shared__ double th[ND], st[ND], hdt[ND];  // theta (rad), 2 pi sin(theta), half bin widths
    for (int d = threadIdx.x; d < ND; d += blockDim.x) {
        th[d] = D2R * sep_deg(d);
        st[d] = TWOPI * sin(th[d]);
    }
    __syncthreads();
    for (int d = 1 + threadIdx.x; d < ND; d += blockDim.x) hdt[d] = 0.5 * (th[d] - th[d - 1]);
    __syncthreads();
    const int s = blockIdx.x, lane = threadIdx.x & 31;
    const int e = blockIdx.y * 8 + (threadIdx.x >> 5);
    if (e >= E) return;  // whole warp
    double* u = upsf + (size_t)s * ND * E + e;
    double* p = partial + (size_t)s * ND * E + e;
    const int d0 = 1 + lane * PSCAN_ROWS;
    const int d1 = min(ND, d0 + PSCAN_ROWS);
    double cum[PSCAN_ROWS];
    double run = 0.0;
    if (d0 < ND) {
        double y1 = u[(size_t)(d0 - 1) * E] * st[d0 - 1];
#pragma unroll
        for (int k = 0; k < PSCAN_ROWS; ++k) {
            const int d = d0 + k;
            if (d < d1) {
                const double y2 = u[(size_t)d * E] * st[d];
                run = fma(hdt[d], y1 + y2, run);
                y1 = y2;
            }
            cum[k] = run;
        }
    }
    double incl = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    const double base = incl - run;
    const double tot = __shfl_sync(0xffffffffu, incl, 31);
    const double inv = 1.0 / tot;  // +-inf when the total is 0: u / 0 as in the reference
    if (lane == 0) {
        p[0] = 0.0;
        u[0] = u[0] * inv;
    }
#pragma unroll
    for (int k = 0; k < PSCAN_ROWS; ++k) {
        const int d = d0 + k;
        if (d < d1) {
            const double c = base + cum[k];
            p[(size_t)d * E] = tot != 0. ? c * inv : c;
            u[(size_t)d * E] = u[(size_t)d * E] * inv;
        }
    }
}

int launch_psf(const PsfDev& a, cudaStream_t st) {
    if (a.C > PSF_MAX_C) return set_error(XTS_ERR_ARG, "compute_psf_data: C=%d exceeds %d", a.C, PSF_MAX_C);
    if (psf_aeff_smem(a.E) > 48 * 1024) return set_error(XTS_ERR_ARG, "compute_psf_data: E=%d exceeds 1200", a.E);
    size_t kf_n = (size_t)ND * a.pf.n_cos * a.pf.n_e, kb_n = (size_t)ND * a.pb.n_cos * a.pb.n_e;
    double* king = (double*)workspace(W_KING, sizeof(double) * (kf_n + kb_n));
    double* pa = (double*)workspace(W_PSFTAB, sizeof(double) * (size_t)a.C * ND * a.E);
    if (!king || !pa) return XTS_ERR_OOM;
    int mx = (int)(kf_n > kb_n ? kf_n : kb_n);
    XTS_LAUNCH("k_king", st, k_king<<<dim3((mx + 127) / 128, 2), 128, 0, st>>>(a.pf, a.pb, king, king + kf_n));
    int n = a.C * ND * a.E;
    XTS_LAUNCH("k_psf_aeff", st, k_psf_aeff<<<(n + 127) / 128, 128, psf_aeff_smem(a.E), st>>>(a.pf, a.pb, king, king + kf_n,
                                               a.costh, a.C, a.logEs, a.E, a.af, a.ab, pa));
    if (a.S == 0) return XTS_OK;
    int DE = ND * a.E;
    dim3 g((DE + 128 * PSF_CPT - 1) / (128 * PSF_CPT), (a.S + PSF_TILE_S - 1) / PSF_TILE_S);
    XTS_LAUNCH("k_mean_psf", st, k_mean_psf<<<g, 128, 0, st>>>(pa, a.C, a.E, a.ecb, a.wecb, a.S, a.ltf, a.exposure, a.upsf));
    XTS_LAUNCH("k_partial_integral", st, k_partial_scan<<<dim3(a.S, (a.E + 7) / 8), 256, 0, st>>>(a.upsf, a.partial, a.E));
    return XTS_OK;
}

// The same launches with caller-provided scratch: king holds both sides' King
// tables (401 * (Mc * Me front + Mc * Me back) doubles), pa the summed psf * aeff
// table (C * 401 * E doubles).  Nothing here allocates.
int launch_psf_scratch(const PsfDev& a, double* king, double* pa, cudaStream_t st) {
    if (a.C > PSF_MAX_C) return set_error(XTS_ERR_ARG, "compute_psf_data: C=%d exceeds %d", a.C, PSF_MAX_C);
    if (psf_aeff_smem(a.E) > 48 * 1024) return set_error(XTS_ERR_ARG, "compute_psf_data: E=%d exceeds 1200", a.E);
    size_t kf_n = (size_t)ND * a.pf.n_cos * a.pf.n_e, kb_n = (size_t)ND * a.pb.n_cos * a.pb.n_e;
    int mx = (int)(kf_n > kb_n ? kf_n : kb_n);
    XTS_LAUNCH("k_king", st, k_king<<<dim3((mx + 127) / 128, 2), 128, 0, st>>>(a.pf, a.pb, king, king + kf_n));
    int n = a.C * ND * a.E;
    XTS_LAUNCH("k_psf_aeff", st, k_psf_aeff<<<(n + 127) / 128, 128, psf_aeff_smem(a.E), st>>>(a.pf, a.pb, king, king + kf_n,
                                               a.costh, a.C, a.logEs, a.E, a.af, a.ab, pa));
    if (a.S == 0) return XTS_OK;
    int DE = ND * a.E;
    dim3 g((DE + 128 * PSF_CPT - 1) / (128 * PSF_CPT), (a.S + PSF_TILE_S - 1) / PSF_TILE_S);
    XTS_LAUNCH("k_mean_psf", st, k_mean_psf<<<g, 128, 0, st>>>(pa, a.C, a.E, a.ecb, a.wecb, a.S, a.ltf, a.exposure, a.upsf));
    XTS_LAUNCH("k_partial_integral", st, k_partial_scan<<<dim3(a.S, (a.E + 7) / 8), 256, 0, st>>>(a.upsf, a.partial, a.E));
    return XTS_OK;
}

}  // namespace xts
