// xts_point.cuh -- per-rule-point geometry shared by the source-map kernels:
// the separation tables, the 12-point rule in bilinear form, the LUT row and
// interpolation weight of one rule point, and TMA bulk-store helpers.
//
//   * The 12 rule points of square_ptswts (points_weights.hpp:93-107) are the
//     bilinear blend p(u,v) = A + B u + C v + D uv of the pixel's corner unit
//     vectors, so p - src is formed from four per-pixel FP64 vectors without
//     rounding p itself; its squared chord q = |p - src|^2 is FP64.
//   * The LUT column of convolve_pixel_psf_logsep (convolve_pixel_psf_logsep.hpp:39-55),
//     idx = 1 + floor(1 + ln(1e4 s)/step) clamped to [2, 400], is found by
//     comparing q with the FP64 squared chords of the 401 table separations
//     (an FP32 log gives the starting guess).
//   * The interpolation weight t = (s - S[idx-1]) / (S[idx] - S[idx-1]) is
//     (g - 1)/(e^step - 1) with g = s / S[idx-1] = asin(x sqrt(1+d))/asin(x),
//     d = q/Q[idx-1] - 1 formed in FP64; g - 1 = d P_k(d) with a per-row
//     degree-4 polynomial fitted on the host (max error 5e-12 on g - 1).  Points
//     outside the tabulated range (s < 1e-4 deg, s >= 70 deg) take the
//     reference's own FP64 formula.
#pragma once

#include <math.h>
#include <string.h>

#include "xts_geom.cuh"
#include "xts_internal.cuh"

namespace xts {

// Bins of the squared chord q by its FP64 exponent and top SB_BITS mantissa bits
// (32 bins per binade, q from 2^-39 to 8): a bin is narrower in ln q (at most
// ln(33/32) = 0.031) than any table row (0.0586 at 70 deg, 0.0672 at small
// angles), so it holds at most one row boundary and its row is k0 or k0 + 1.
struct SepBin {
    int k0, pad;  // lower row of the bin's low edge, clamped to [1, 399]
    double thr;   // q[k0 + 1] (+inf when k0 = 399): q >= thr selects row k0 + 1
};
constexpr int SB_EXP0 = 984;  // biased FP64 exponent of the first bin
constexpr int SB_BITS = 5;
constexpr int NSB = (1025 - SB_EXP0 + 1) << SB_BITS;

// Separation tables shared by every launch (see build_septab).
struct SepTab {
    double q[ND + 1];      // squared chord of S[k] (k = 0..400), q[401] = +inf guard
    float coef[ND][8];     // row k (= idx - 1): {1/q[k], c0..c4 of P_k(z), q[k] as two words},
                           // z = (d - DPOLY_C)/DPOLY_H
    SepBin bins[NSB];
};
// centre and half-width of the fitted d range, [-0.002, 0.146]: two table rows (the
// ratio q[k + 2] / q[k] - 1 is at most 0.1445), so one row's polynomial also gives
// t for the points of the next row (t error below 1e-8 over the range)
constexpr float DPOLY_C = 0.072f;
constexpr float DPOLY_H = 0.074f;

constexpr int RW = 8;   // dense row window per pixel
constexpr int WST = 9;  // padded stride of a window in shared memory (bank-conflict free)

static SepTab* g_septab_dev[64] = {};  // per translation unit and device

static int build_septab(cudaStream_t st, const SepTab** out) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return set_error(XTS_ERR_ARG, "device index %d out of range", dev);
    if (g_septab_dev[dev]) { *out = g_septab_dev[dev]; return XTS_OK; }
    static SepTab h;
    const long double D2Rl = 0.017453292519943295769236907684886127134L;
    const double xstep = log(70. / 1e-4) / (400 - 1.);
    long double S[ND];
    for (int k = 0; k < ND; ++k) S[k] = k == 0 ? 0.0L : (long double)(1e-4 * exp((k - 1) * xstep));
    for (int k = 0; k < ND; ++k) {
        long double ch = 2.0L * sinl(0.5L * S[k] * D2Rl);
        h.q[k] = (double)(ch * ch);
    }
    h.q[ND] = INFINITY;
    for (int k = 0; k < ND; ++k) {
        for (int j = 0; j < 8; ++j) h.coef[k][j] = 0.f;
        if (k == 0) continue;
        long double qk = 2.0L * sinl(0.5L * S[k] * D2Rl);
        qk *= qk;
        long double xlo = sinl(0.5L * S[k] * D2Rl), a0 = asinl(xlo);
        // Chebyshev interpolation of f(d) = (g(d) - 1)/d at 5 nodes, z in [-1, 1]
        const int N = 5;
        long double fz[N], zn[N];
        for (int i = 0; i < N; ++i) {
            zn[i] = cosl(3.14159265358979323846264338327950288L * (i + 0.5L) / N);
            long double d = (long double)DPOLY_C + (long double)DPOLY_H * zn[i];
            fz[i] = (asinl(xlo * sqrtl(1.0L + d)) / a0 - 1.0L) / d;
        }
        long double cc[N];
        for (int j = 0; j < N; ++j) {
            long double s = 0;
            for (int i = 0; i < N; ++i) s += fz[i] * cosl(j * acosl(zn[i]));
            cc[j] = s * (j == 0 ? 1.0L : 2.0L) / N;
        }
        // T0=1, T1=z, T2=2z^2-1, T3=4z^3-3z, T4=8z^4-8z^2+1 -> monomials in z
        long double m[N] = {cc[0] - cc[2] + cc[4], cc[1] - 3 * cc[3], 2 * cc[2] - 8 * cc[4], 4 * cc[3], 8 * cc[4]};
        h.coef[k][0] = (float)(1.0L / qk);
        for (int j = 0; j < N; ++j) h.coef[k][1 + j] = (float)m[j];
        memcpy(&h.coef[k][6], &h.q[k], sizeof(double));
    }
    for (int b = 0; b < NSB; ++b) {
        const double qa = ldexp(1.0 + (double)(b & ((1 << SB_BITS) - 1)) / (1 << SB_BITS),
                                SB_EXP0 + (b >> SB_BITS) - 1023);
        int k = 0;
        while (k < ND - 1 && h.q[k + 1] <= qa) ++k;  // largest k with q[k] <= qa
        k = k < 1 ? 1 : (k > 399 ? 399 : k);
        h.bins[b].k0 = k;
        h.bins[b].pad = 0;
        h.bins[b].thr = k < 399 ? h.q[k + 1] : INFINITY;
    }
    SepTab* d = nullptr;
    XTS_CUDA(cudaMalloc(&d, sizeof(SepTab)));
    XTS_CUDA(cudaMemcpyAsync(d, &h, sizeof(SepTab), cudaMemcpyHostToDevice, st));
    XTS_CUDA(cudaStreamSynchronize(st));
    g_septab_dev[dev] = d;
    *out = d;
    return XTS_OK;
}

// Rule in the bilinear form: u, v, u*v and 0.25 * weight per point (and that
// weight rounded to FP32).
static __constant__ double c_rule_uv[12][4];
static __constant__ float c_rule_w32[12];
static __constant__ double c_rule_q[12][3];  // u, u*u, v (biquadratic chord form)
static __constant__ float c_rule_f[12][4];   // u, u*u, v in FP32 (chord offsets from the centre), pad
// The rule's points come in mirror pairs (p + 6 = -p, same weight): for pair p < 6,
// u, v, uv, u^2, v^2, u^2 v, u v^2, u^2 v^2 in FP32, so the chord offset of the pair is
// E +- O with E the even and O the odd part of the biquadratic form.
static __constant__ float c_pair[6][8];
static __constant__ float c_rule_wsum;       // sum of the 12 FP32 weights

static int upload_rule_uv(cudaStream_t st) {
    static int dev_done = -1;
    int dev = -1;
    cudaGetDevice(&dev);
    if (dev_done == dev) return XTS_OK;
    // Sommariva & Festa degree-7 12-point rule (model_map/mm_cubature/cubature.hpp:209-225)
    static const double R[36] = {
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
    double b[12][4];
    for (int p = 0; p < 12; ++p) {
        b[p][0] = R[3 * p]; b[p][1] = R[3 * p + 1]; b[p][2] = R[3 * p] * R[3 * p + 1];
        b[p][3] = 0.25 * R[3 * p + 2];
    }
    float w32[12], bf[12][4];
    double bq[12][3];
    for (int p = 0; p < 12; ++p) {
        w32[p] = (float)b[p][3];
        bq[p][0] = R[3 * p]; bq[p][1] = R[3 * p] * R[3 * p]; bq[p][2] = R[3 * p + 1];
        bf[p][0] = (float)bq[p][0]; bf[p][1] = (float)bq[p][1]; bf[p][2] = (float)bq[p][2]; bf[p][3] = 0.f;
    }
    float pr[6][8], wsum = 0.f;
    for (int p = 0; p < 6; ++p) {
        const double u = R[3 * p], v = R[3 * p + 1];
        const double k[8] = {u, v, u * v, u * u, v * v, u * u * v, u * v * v, u * u * v * v};
        for (int j = 0; j < 8; ++j) pr[p][j] = (float)k[j];
    }
    for (int p = 0; p < 12; ++p) wsum += w32[p];
    XTS_CUDA(cudaMemcpyToSymbolAsync(c_pair, pr, sizeof(pr), 0, cudaMemcpyHostToDevice, st));
    XTS_CUDA(cudaMemcpyToSymbolAsync(c_rule_wsum, &wsum, sizeof(wsum), 0, cudaMemcpyHostToDevice, st));
    XTS_CUDA(cudaMemcpyToSymbolAsync(c_rule_f, bf, sizeof(bf), 0, cudaMemcpyHostToDevice, st));
    XTS_CUDA(cudaMemcpyToSymbolAsync(c_rule_uv, b, sizeof(b), 0, cudaMemcpyHostToDevice, st));
    XTS_CUDA(cudaMemcpyToSymbolAsync(c_rule_w32, w32, sizeof(w32), 0, cudaMemcpyHostToDevice, st));
    XTS_CUDA(cudaMemcpyToSymbolAsync(c_rule_q, bq, sizeof(bq), 0, cudaMemcpyHostToDevice, st));
    XTS_CUDA(cudaStreamSynchronize(st));
    dev_done = dev;
    return XTS_OK;
}

// ------------------------------------------------------------------ TMA bulk stores
__device__ __forceinline__ void bulk_store(void* gdst, const void* ssrc, unsigned bytes) {
    unsigned s = (unsigned)__cvta_generic_to_shared(ssrc);
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;\n"
                 :: "l"(gdst), "r"(s), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void bulk_wait_read() {
    asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory");
}
__device__ __forceinline__ void bulk_wait_all() {
    asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory");
}
__device__ __forceinline__ void fence_async_shared() {
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

// ------------------------------------------------------------------ mbarriers and bulk loads
constexpr int WAIT_LIMIT = 1 << 21;  // try_wait polls before a wait is declared failed

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

// Bounded wait for the phase with the given parity; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity) {
    for (int i = 0; i < WAIT_LIMIT; ++i) {
        unsigned done;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
                     : "=r"(done) : "r"(bar), "r"(parity) : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(bar), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// One TMA bulk copy global -> shared (16-byte aligned ends, bytes % 16 == 0) that
// completes on the mbarrier, which this thread arms with the byte count.
__device__ __forceinline__ void bulk_load(void* sdst, const void* gsrc, unsigned bytes, unsigned bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(bar), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(smem_u32(sdst)), "l"(gsrc), "r"(bytes), "r"(bar) : "memory");
}

// ------------------------------------------------------------------ one rule point
// Interpolation weight outside the tabulated range (s < 1e-4 deg or s >= 70 deg):
// the reference's own FP64 formula (convolve_pixel_psf_logsep.hpp:45-47).  Kept
// out of line: it runs for a handful of points per map.
static __device__ __noinline__ float t_exact(double q, int idx) {
    const double sdeg = 2.0 * R2D * asin(0.5 * sqrt(q));
    return (float)(REDM1 * (sdeg * 1e4 * exp(SEP_STEP * (2. - idx)) - 1.));
}

// Row idx in [2, 400] and interpolation weight of one rule point from its FP64
// squared chord q.  The FP32 starting guess is within one row of the bracket
// (|error| < 0.3 rows up to 70 deg, where the row is clamped to 400); one
// branch-free correction against the FP64 squared chords gives the
// reference's row.  sq: [ND + 1] squared chords; coef: [ND][2] float4.
__device__ __forceinline__ int point_row(double q, const double* sq, const float4* coef, float* t_out) {
    const float qf = (float)q;
    // ln s_deg ~ ln(180/pi) + ln(q)/2 + q/24;  j = 1 + (ln 1e4 + ln s_deg)/step
    const float lns = fmaf(0.34657359f, __log2f(fmaxf(qf, 1e-37f)), fmaf(qf, 1.f / 24.f, 4.0482950f));
    const float jf = fmaf(29.645952f, lns, 1.f + 29.645952f * 9.2103404f);
    int idx = 1 + (int)fminf(fmaxf(jf, 1.f), 399.f);  // [2, 400]
    const double qa = sq[idx - 1], qb = sq[idx];
    const int dn = (q < qa) & (idx > 2);
    const int up = (q >= qb) & (idx < 400);
    idx += up - dn;
    const double qlo = up ? qb : (dn ? sq[idx - 1] : qa);
    const float4 c0 = coef[2 * (idx - 1)], c1 = coef[2 * (idx - 1) + 1];
    const float dl = (float)(q - qlo) * c0.x;  // q / q_lo - 1
    if (dl >= -0.002f && dl <= 0.072f) {
        const float zz = fmaf(dl, 1.f / DPOLY_H, -DPOLY_C / DPOLY_H);
        const float P = fmaf(fmaf(fmaf(fmaf(c1.y, zz, c1.x), zz, c0.w), zz, c0.z), zz, c0.y);
        *t_out = (float)REDM1 * (dl * P);
    } else {
        *t_out = t_exact(q, idx);
    }
    return idx;
}

// The same row and weight by the bin table: one 16-byte load of the bin of q
// (exponent and top mantissa bits), one FP64 compare, and the row's record
// (1/q_k, t polynomial, q_k).  bins: [NSB]; coef: [ND][2] float4 with q_k in the
// last two words.
__device__ __forceinline__ int point_row_bin(double q, const SepBin* bins, const float4* coef, float* t_out) {
    int b = (__double2hiint(q) >> (20 - SB_BITS)) - (SB_EXP0 << SB_BITS);
    b = min(max(b, 0), NSB - 1);
    const SepBin sb = bins[b];
    const int k = sb.k0 + (q >= sb.thr);
    const float4 c0 = coef[2 * k], c1 = coef[2 * k + 1];
    const double qlo = __hiloint2double(__float_as_int(c1.w), __float_as_int(c1.z));
    const float dl = (float)(q - qlo) * c0.x;  // q / q_lo - 1
    if (dl >= -0.002f && dl <= 0.072f) {
        const float zz = fmaf(dl, 1.f / DPOLY_H, -DPOLY_C / DPOLY_H);
        const float P = fmaf(fmaf(fmaf(fmaf(c1.y, zz, c1.x), zz, c0.w), zz, c0.z), zz, c0.y);
        *t_out = (float)REDM1 * (dl * P);
    } else {
        *t_out = t_exact(q, k + 1);
    }
    return k + 1;
}

// point_row_bin without the out-of-range branch: t is NaN for points outside
// 1e-4 deg .. 70 deg (the caller evaluates those with t_exact), so a run of
// these lookups has no call in it and the compiler can overlap them.
__device__ __forceinline__ int point_row_bin_nc(double q, const SepBin* bins, const float4* coef, float* t_out) {
    int b = (__double2hiint(q) >> (20 - SB_BITS)) - (SB_EXP0 << SB_BITS);
    b = min(max(b, 0), NSB - 1);
    const SepBin sb = bins[b];
    const int k = sb.k0 + (q >= sb.thr);
    const float4 c0 = coef[2 * k], c1 = coef[2 * k + 1];
    const double qlo = __hiloint2double(__float_as_int(c1.w), __float_as_int(c1.z));
    const float dl = (float)(q - qlo) * c0.x;
    const float zz = fmaf(dl, 1.f / DPOLY_H, -DPOLY_C / DPOLY_H);
    const float P = fmaf(fmaf(fmaf(fmaf(c1.y, zz, c1.x), zz, c0.w), zz, c0.z), zz, c0.y);
    *t_out = (dl >= -0.002f && dl <= 0.072f) ? (float)REDM1 * (dl * P) : __int_as_float(0x7fffffff);
    return k + 1;
}

// Bilinear form of the rule points of pixel (h, w) relative to the source.
struct PixGeom { double Ax, Ay, Az, Bx, By, Bz, Cx, Cy, Cz, Dx, Dy, Dz; };

__device__ __forceinline__ PixGeom pixel_geom(const double* corners, int W1, int h, int w, const SrcInfo& si) {
    const double* a = corners + 3 * (h * W1 + w);            // LL (h+0.5, w+0.5)
    const double* b = corners + 3 * (h * W1 + w + 1);        // LR
    const double* c = corners + 3 * ((h + 1) * W1 + w + 1);  // UR
    const double* d = corners + 3 * ((h + 1) * W1 + w);      // UL
    PixGeom g;
    g.Ax = 0.25 * ((a[0] + b[0]) + (c[0] + d[0])) - si.dir[0];
    g.Ay = 0.25 * ((a[1] + b[1]) + (c[1] + d[1])) - si.dir[1];
    g.Az = 0.25 * ((a[2] + b[2]) + (c[2] + d[2])) - si.dir[2];
    g.Bx = 0.25 * ((b[0] + c[0]) - (a[0] + d[0]));
    g.By = 0.25 * ((b[1] + c[1]) - (a[1] + d[1]));
    g.Bz = 0.25 * ((b[2] + c[2]) - (a[2] + d[2]));
    g.Cx = 0.25 * ((c[0] + d[0]) - (a[0] + b[0]));
    g.Cy = 0.25 * ((c[1] + d[1]) - (a[1] + b[1]));
    g.Cz = 0.25 * ((c[2] + d[2]) - (a[2] + b[2]));
    g.Dx = 0.25 * ((a[0] + c[0]) - (b[0] + d[0]));
    g.Dy = 0.25 * ((a[1] + c[1]) - (b[1] + d[1]));
    g.Dz = 0.25 * ((a[2] + c[2]) - (b[2] + d[2]));
    return g;
}

__device__ __forceinline__ double point_q(const PixGeom& g, int p) {
    const double u = c_rule_uv[p][0], v = c_rule_uv[p][1], uv = c_rule_uv[p][2];
    const double x = fma(g.Dx, uv, fma(g.Cx, v, fma(g.Bx, u, g.Ax)));
    const double y = fma(g.Dy, uv, fma(g.Cy, v, fma(g.By, u, g.Ay)));
    const double z = fma(g.Dz, uv, fma(g.Cz, v, fma(g.Bz, u, g.Az)));
    return fma(x, x, fma(y, y, z * z));
}

// q(u, v) = |A + Bu + Cv + Duv|^2 of one pixel as a biquadratic polynomial,
// evaluated per rule point by Horner in v: q = P0(u) + v (P1(u) + v P2(u)), each
// P a quadratic in u (8 FP64 FMAs per point, dependency depth 4).
struct PixQ { double a0, a1, a2, a3, a4, a5, a6, a7, a8; };

__device__ __forceinline__ PixQ pixel_q(const PixGeom& g) {
    PixQ c;
    c.a0 = fma(g.Ax, g.Ax, fma(g.Ay, g.Ay, g.Az * g.Az));
    c.a1 = 2.0 * fma(g.Ax, g.Bx, fma(g.Ay, g.By, g.Az * g.Bz));
    c.a4 = fma(g.Bx, g.Bx, fma(g.By, g.By, g.Bz * g.Bz));
    c.a2 = 2.0 * fma(g.Ax, g.Cx, fma(g.Ay, g.Cy, g.Az * g.Cz));
    c.a3 = 2.0 * (fma(g.Ax, g.Dx, fma(g.Ay, g.Dy, g.Az * g.Dz)) + fma(g.Bx, g.Cx, fma(g.By, g.Cy, g.Bz * g.Cz)));
    c.a6 = 2.0 * fma(g.Bx, g.Dx, fma(g.By, g.Dy, g.Bz * g.Dz));
    c.a5 = fma(g.Cx, g.Cx, fma(g.Cy, g.Cy, g.Cz * g.Cz));
    c.a7 = 2.0 * fma(g.Cx, g.Dx, fma(g.Cy, g.Dy, g.Cz * g.Dz));
    c.a8 = fma(g.Dx, g.Dx, fma(g.Dy, g.Dy, g.Dz * g.Dz));
    return c;
}

__device__ __forceinline__ double point_q2(const PixQ& c, int p) {
    const double u = c_rule_q[p][0], uu = c_rule_q[p][1], v = c_rule_q[p][2];
    const double p0 = fma(c.a4, uu, fma(c.a1, u, c.a0));
    const double p1 = fma(c.a6, uu, fma(c.a3, u, c.a2));
    const double p2 = fma(c.a8, uu, fma(c.a7, u, c.a5));
    return fma(fma(p2, v, p1), v, p0);
}

// Scaled FP32 table Y'[s][d][e] = uPsf * (exposure * correction), energies
// padded to Epad with zeros (scale NULL: uPsf itself); launched as
// lut_scaled_grid(S) x 256 threads.  With hi/lo given, also the 3xTF32 split:
// hi = tf32(Y'), lo = Y' - hi.
static __global__ void k_lut_scaled(const double* upsf, const double* scale, int S, int E, int Epad,
                             float* lut, float* hi, float* lo) {
    const unsigned sd = blockIdx.x * 8 + (threadIdx.x >> 5);  // (source, row), one warp per row
    if (sd >= (unsigned)S * ND) return;
    const unsigned s = sd / ND;
    for (int e = threadIdx.x & 31; e < Epad; e += 32) {
        const size_t k = (size_t)sd * Epad + e;
        const float v = e < E ? (float)(upsf[(size_t)sd * E + e] * (scale ? scale[(size_t)s * E + e] : 1.0)) : 0.f;
        if (lut) lut[k] = v;
        if (hi) {
            unsigned hb;
            asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(hb) : "f"(v));
            const float h = __uint_as_float(hb);
            hi[k] = h;
            lo[k] = v - h;
        }
    }
}

// Launch shape of k_lut_scaled: 256 threads, one warp per (source, row).
static inline unsigned lut_scaled_grid(int S) { return (unsigned)(((size_t)S * ND + 7) / 8); }

}  // namespace xts
