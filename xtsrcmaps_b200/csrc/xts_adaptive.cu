// xts_adaptive.cu -- adaptive cubature of the pixel-mean PSF (the design of the
// reference's uncompiled math/genz_malik.hxx:18-195):
// the published Genz-Malik degree-7/5 rule for two dimensions (A.C. Genz,
// A.A. Malik, J. Comput. Appl. Math. 6 (1980) 295-302; weights as updated by
// Bernstein, Espelid and Genz), the design the reference lays out in
// math/genz_malik.hxx:18-85 and math/genz_malik.cxx:66-217 (not compiled there),
// with rectangular sub-regions and the estimate kept at the depth limit.
//
// Work is scheduled by region, not by pixel, so that pixels needing many regions
// (next to the source) do not hold up the others.  One persistent launch (a
// cooperative grid, every block resident) runs all levels: level 0 evaluates
// every (source, pixel)'s whole-pixel region and writes accepted pixels' means;
// an unaccepted region pushes its two halves onto a device-side queue; after a
// grid-wide barrier (bounded waits) the next level takes the previous level's
// queue, one region per thread, and accepted regions add area * R7 into their
// pixel's FP64 mean with FP64 atomics (order-free to within a few FP64 ulps).
// The queue has a fixed capacity; a region whose halves do not fit is accepted
// as it is.
//
// Decisions near the threshold are taken in FP64: when the FP32 estimate of
// max_e |R5 - R7| / |R7| lies within 5 % of rtol, or the two fourth differences
// that choose the split dimension are within 0.1 % of each other (or within their
// FP32 error, 4e-6 of the summed values), the region is
// evaluated again point by point in FP64 from the FP64 mean PSF, with the
// reference design's arithmetic (math/genz_malik.hxx:127-195) and no fused
// multiply-adds, and that evaluation decides (and gives the value).
//
// A region's 17 points give LUT rows and interpolation weights exactly as the
// 12-point rule's do (xts_point.cuh: FP64 chord of the corner-vector blend,
// exact row, per-row t polynomial).  When they span at most AW consecutive rows,
// four row windows are formed (the degree-7 value, degree-5 minus degree-7, and
// the two fourth divided differences that choose the split dimension) and dotted
// with the source's FP32 mean-PSF rows for every energy; otherwise the points
// are evaluated one by one.  A region is accepted when
// max_e |R5 - R7| / |R7| <= rtol or at the depth limit; otherwise it is halved
// along the dimension with the larger summed fourth difference.
//
// k_adaptive_integral then sums mean * solid angle over the pixels inside the
// boundary radius (FP64, fixed order), k_correction_sums forms the scales, and
// k_scale_map64 writes value = mean * solid angle * exposure * correction.
#include "xts_point.cuh"

namespace xts {

constexpr int AT = 256;     // threads per block
constexpr int AW = 8;       // rows of a region window

// Points of the rule in half-widths along (dimension 0 = map axis h, dimension 1
// = map axis w) and the coefficients of the four windows per point.
struct GmRule {
    float off0[17], off1[17];
    float w7[17], wd[17], d0[17], d1[17];
};
static __constant__ GmRule c_gm;
struct GmRule64 { double off0[17], off1[17], w7[17], w5[17]; };  // the same rule in FP64
static __constant__ GmRule64 c_gm64;
static int upload_gm(cudaStream_t st) {
    static int dev_done = -1;
    int dev = -1;
    cudaGetDevice(&dev);
    if (dev_done == dev) return XTS_OK;
    const double l2 = 0.35856858280031809199064515390793749545406372969943071;  // sqrt(9/70)
    const double l4 = 0.94868329805051379959966806332981556011586654179756505;  // sqrt(9/10)
    const double l5 = 0.68824720161168529772162873429362352512689535661564885;  // sqrt(9/19)
    // centre; +-l2 on each axis; +-l4 on each axis; (+-l4, +-l4); (+-l5, +-l5)
    const double o[17][2] = {{0, 0},     {-l2, 0},   {0, -l2},  {l2, 0},   {0, l2},   {-l4, 0},
                             {0, -l4},   {l4, 0},    {0, l4},   {-l4, -l4}, {l4, -l4}, {-l4, l4},
                             {l4, l4},   {-l5, -l5}, {-l5, l5}, {l5, -l5},  {l5, l5}};
    const double a7 = (12824. - 9120. * 2. + 400. * 4.) / 19683., b7 = 980. / 6561.;
    const double c7 = (1820. - 400. * 2.) / 19683., d7 = 200. / 19683., f7 = 6859. / 19683. / 4.;
    const double a5 = (729. - 950. * 2. + 50. * 4.) / 729., b5 = 245. / 486.;
    const double c5 = (265. - 100. * 2.) / 1458., d5 = 25. / 729.;
    GmRule g;
    GmRule64 g64;
    for (int p = 0; p < 17; ++p) {
        const double w7 = p == 0 ? a7 : p < 5 ? b7 : p < 9 ? c7 : p < 13 ? d7 : f7;
        const double w5 = p == 0 ? a5 : p < 5 ? b5 : p < 9 ? c5 : p < 13 ? d5 : 0.;
        g64.off0[p] = o[p][0];
        g64.off1[p] = o[p][1];
        g64.w7[p] = w7;
        g64.w5[p] = w5;
        g.off0[p] = (float)o[p][0];
        g.off1[p] = (float)o[p][1];
        g.w7[p] = (float)w7;
        g.wd[p] = (float)(w5 - w7);
        // fourth differences: (f(-l2) + f(+l2) - 2 f0) - (l2/l4)^2 (f(-l4) + f(+l4) - 2 f0)
        double e0 = 0., e1 = 0.;
        if (p == 0) e0 = e1 = -2. + 2. / 7.;
        if (p == 1 || p == 3) e0 = 1.;
        if (p == 5 || p == 7) e0 = -1. / 7.;
        if (p == 2 || p == 4) e1 = 1.;
        if (p == 6 || p == 8) e1 = -1. / 7.;
        g.d0[p] = (float)e0;
        g.d1[p] = (float)e1;
    }
    XTS_CUDA(cudaMemcpyToSymbolAsync(c_gm, &g, sizeof(g), 0, cudaMemcpyHostToDevice, st));
    XTS_CUDA(cudaMemcpyToSymbolAsync(c_gm64, &g64, sizeof(g64), 0, cudaMemcpyHostToDevice, st));
    XTS_CUDA(cudaStreamSynchronize(st));
    dev_done = dev;
    return XTS_OK;
}

// One queued region: its pixel (source * npix + pixel) and its rectangle in the
// pixel's [-1, 1]^2 parameter square.
struct QRegion { int sp; float c0, c1, h0, h1; };

constexpr size_t AO_SQ = 0;
constexpr size_t AO_COEF = (8 * (ND + 1) + 15) / 16 * 16;
constexpr size_t AO_WIN = AO_COEF + sizeof(float4) * 2 * ND;  // [4][AW][AT] floats
constexpr size_t A_SMEM = AO_WIN + sizeof(float) * 4 * AW * AT;

__device__ __forceinline__ float4 f4fma(float a, const float4& y, const float4& c) {
    return make_float4(fmaf(a, y.x, c.x), fmaf(a, y.y, c.y), fmaf(a, y.z, c.z), fmaf(a, y.w, c.w));
}
__device__ __forceinline__ float f4c(const float4& v, int c) { return c == 0 ? v.x : c == 1 ? v.y : c == 2 ? v.z : v.w; }

// The region again in FP64, point by point, with the reference design's arithmetic
// (math/genz_malik.hxx:127-195 as restated by the oracle): the rule points blended
// from the pixel's corner vectors, s = 2 asin(|p - src| / 2), the logsep row and
// weight, f = (1 - t) U[i - 1] + t U[i], R7 and R5 summed over the points in order,
// no fused multiply-adds.  Decides the region and, when it is accepted, adds (or,
// at level 0, stores) area * R7 into mean[e]; otherwise sets *dim.
__device__ __noinline__ bool gm_region64(const double* __restrict__ corners, int W1, int h, int w, const double* src,
                                         double c0, double c1, double h0, double h1, bool last,
                                         const double* __restrict__ U, int E, double rtol, double* mean, bool atomic,
                                         int* dim) {
    const double* a = corners + 3 * ((size_t)h * W1 + w);            // LL
    const double* b = corners + 3 * ((size_t)h * W1 + w + 1);        // LR
    const double* c = corners + 3 * ((size_t)(h + 1) * W1 + w + 1);  // UR
    const double* d = corners + 3 * ((size_t)(h + 1) * W1 + w);      // UL
    int ix[17];
    double tt[17];
    for (int p = 0; p < 17; ++p) {
        const double x1 = __dadd_rn(c1, __dmul_rn(c_gm64.off1[p], h1));
        const double x0 = __dadd_rn(c0, __dmul_rn(c_gm64.off0[p], h0));
        const double u = x1, v = x0;
        const double nn = __dmul_rn(__dsub_rn(1.0, u), __dsub_rn(1.0, v));
        const double pn = __dmul_rn(__dadd_rn(1.0, u), __dsub_rn(1.0, v));
        const double pp = __dmul_rn(__dadd_rn(1.0, u), __dadd_rn(1.0, v));
        const double np = __dmul_rn(__dsub_rn(1.0, u), __dadd_rn(1.0, v));
        double q2 = 0.;
        for (int k = 0; k < 3; ++k) {
            const double bl = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(nn, a[k]), __dmul_rn(pn, b[k])), __dmul_rn(pp, c[k])),
                                        __dmul_rn(np, d[k]));
            const double qk = __dsub_rn(__dmul_rn(0.25, bl), src[k]);
            q2 = __dadd_rn(q2, __dmul_rn(qk, qk));
        }
        const double sd = 2.0 * R2D * asin(0.5 * sqrt(q2));
        const double j = sd < 1e-4 ? 1. : __dadd_rn(1., __dmul_rn(RECIPSTEP, __dadd_rn(LN_1E4, log(sd))));
        int idx = 1 + (int)(unsigned short)j;
        idx = idx > 400 ? 400 : idx;
        ix[p] = idx;
        tt[p] = __dmul_rn(REDM1, __dsub_rn(__dmul_rn(__dmul_rn(sd, 1e4), exp(__dmul_rn(SEP_STEP, 2. - idx))), 1.));
    }
    double rel = 0., dd0 = 0., dd1 = 0.;
    const double area = __dmul_rn(h0, h1);
    for (int e = 0; e < E; ++e) {
        double v7 = 0., v5 = 0., f[9];
        for (int p = 0; p < 17; ++p) {
            const double fv = __dadd_rn(__dmul_rn(__dsub_rn(1.0, tt[p]), U[(size_t)(ix[p] - 1) * E + e]),
                                        __dmul_rn(tt[p], U[(size_t)ix[p] * E + e]));
            if (p < 9) f[p] = fv;
            v7 = __dadd_rn(v7, __dmul_rn(c_gm64.w7[p], fv));
            v5 = __dadd_rn(v5, __dmul_rn(c_gm64.w5[p], fv));
        }
        const double err = fabs(__dsub_rn(v5, v7));
        const double r = v7 != 0. ? err / fabs(v7) : (err != 0. ? INFINITY : 0.);
        rel = r > rel ? r : rel;
        const double f0 = __dmul_rn(2., f[0]);
        dd0 = __dadd_rn(dd0, fabs(__dsub_rn(__dsub_rn(__dadd_rn(f[1], f[3]), f0),
                                            __dmul_rn(1. / 7., __dsub_rn(__dadd_rn(f[5], f[7]), f0)))));
        dd1 = __dadd_rn(dd1, fabs(__dsub_rn(__dsub_rn(__dadd_rn(f[2], f[4]), f0),
                                            __dmul_rn(1. / 7., __dsub_rn(__dadd_rn(f[6], f[8]), f0)))));
    }
    if (!(rel <= rtol || last)) {
        *dim = dd0 >= dd1 ? 0 : 1;
        return false;
    }
    for (int e = 0; e < E; ++e) {
        double v7 = 0.;
        for (int p = 0; p < 17; ++p) {
            const double fv = __dadd_rn(__dmul_rn(__dsub_rn(1.0, tt[p]), U[(size_t)(ix[p] - 1) * E + e]),
                                        __dmul_rn(tt[p], U[(size_t)ix[p] * E + e]));
            v7 = __dadd_rn(v7, __dmul_rn(c_gm64.w7[p], fv));
        }
        if (atomic) atomicAdd(mean + e, __dmul_rn(area, v7));
        else mean[e] = __dmul_rn(area, v7);
    }
    return true;
}

// Evaluates one region.  Returns true when it is accepted, after adding
// area * R7 into mean[e] (FP64; atomically when `atomic`, else stored: level 0,
// one region per pixel); otherwise sets *dim.  Y is the source's FP32 mean-PSF
// table with rows of EP = E rounded up to 4 floats (zeros past E), read four
// energies at a time, U the source's FP64 table for decisions near the threshold
// (gm_region64).  The values are added during the acceptance check, so an
// accepted region (most of them) is evaluated once; a split region's values are
// taken back out (FP64 atomics; at level 0, cleared).
__device__ __noinline__ bool gm_region(const PixGeom& g, float c0, float c1, float h0, float h1, bool last,
                                       const double* sq, const float4* scoef, float* wk, const float* Y,
                                       const double* U, const double* corners, int W1, int h, int w,
                                       const double* src, int E, int EP, float rtol, double* mean, bool atomic,
                                       int* dim) {
    int ix[17];
    float tt[17];
    int rmin = ND, rmax = 0;
#pragma unroll
    for (int p = 0; p < 17; ++p) {
        const double u = c1 + c_gm.off1[p] * h1;  // along w
        const double v = c0 + c_gm.off0[p] * h0;  // along h
        const double x = fma(g.Dx, u * v, fma(g.Cx, v, fma(g.Bx, u, g.Ax)));
        const double y = fma(g.Dy, u * v, fma(g.Cy, v, fma(g.By, u, g.Ay)));
        const double z = fma(g.Dz, u * v, fma(g.Cz, v, fma(g.Bz, u, g.Az)));
        ix[p] = point_row(fma(x, x, fma(y, y, z * z)), sq, scoef, &tt[p]);
        rmin = min(rmin, ix[p] - 1);
        rmax = max(rmax, ix[p]);
    }
    const float area = h0 * h1;  // fraction of the pixel
    const int nr = rmax - rmin + 1;
    const bool windowed = nr <= AW;
    float w7[AW], wd[AW], e0[AW], e1[AW];
    if (windowed) {  // the four row windows of this region
#pragma unroll
        for (int j = 0; j < 4 * AW; ++j) wk[j * AT] = 0.f;
#pragma unroll
        for (int p = 0; p < 17; ++p) {
            const int r = ix[p] - 1 - rmin;
            const float a = 1.f - tt[p], b = tt[p];
            wk[(0 * AW + r) * AT] += a * c_gm.w7[p];
            wk[(0 * AW + r + 1) * AT] += b * c_gm.w7[p];
            wk[(1 * AW + r) * AT] += a * c_gm.wd[p];
            wk[(1 * AW + r + 1) * AT] += b * c_gm.wd[p];
            wk[(2 * AW + r) * AT] += a * c_gm.d0[p];
            wk[(2 * AW + r + 1) * AT] += b * c_gm.d0[p];
            wk[(3 * AW + r) * AT] += a * c_gm.d1[p];
            wk[(3 * AW + r + 1) * AT] += b * c_gm.d1[p];
        }
#pragma unroll
        for (int j = 0; j < AW; ++j) {
            w7[j] = wk[(0 * AW + j) * AT];
            wd[j] = wk[(1 * AW + j) * AT];
            e0[j] = wk[(2 * AW + j) * AT];
            e1[j] = wk[(3 * AW + j) * AT];
        }
    }
    const float* y0 = Y + (size_t)rmin * EP;
    const int EQ4 = EP >> 2;
    // R7, R5 - R7 and the two fourth differences at energies 4qd .. 4qd + 3: from
    // the windows, or point by point when the rows are too far apart
    auto rule = [&](int qd, float4& v7, float4& vd, float4& a0, float4& a1) {
        v7 = vd = a0 = a1 = make_float4(0.f, 0.f, 0.f, 0.f);
        if (windowed) {
#pragma unroll
            for (int j = 0; j < AW; ++j) {
                if (j < nr) {
                    const float4 yv = __ldg((const float4*)(y0 + (size_t)j * EP) + qd);
                    v7 = f4fma(w7[j], yv, v7);
                    vd = f4fma(wd[j], yv, vd);
                    a0 = f4fma(e0[j], yv, a0);
                    a1 = f4fma(e1[j], yv, a1);
                }
            }
        } else {
            for (int p = 0; p < 17; ++p) {
                const float4* yl = (const float4*)(Y + (size_t)(ix[p] - 1) * EP) + qd;
                const float4 lo = __ldg(yl), hi = __ldg(yl + EQ4);
                const float4 f = make_float4(fmaf(tt[p], hi.x - lo.x, lo.x), fmaf(tt[p], hi.y - lo.y, lo.y),
                                             fmaf(tt[p], hi.z - lo.z, lo.z), fmaf(tt[p], hi.w - lo.w, lo.w));
                v7 = f4fma(c_gm.w7[p], f, v7);
                vd = f4fma(c_gm.wd[p], f, vd);
                a0 = f4fma(c_gm.d0[p], f, a0);
                a1 = f4fma(c_gm.d1[p], f, a1);
            }
        }
    };
    float rel = 0.f, dd0 = 0.f, dd1 = 0.f, sx7 = 0.f;
    if (!last) {
        for (int qd = 0; qd < EQ4; ++qd) {
            float4 v7, vd, a0, a1;
            rule(qd, v7, vd, a0, a1);
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const int e = 4 * qd + c;
                if (e < E) {
                    const float x7 = f4c(v7, c), xd = f4c(vd, c);
                    const float r = fabsf(xd) <= rtol * fabsf(x7) ? fabsf(xd) / fmaxf(fabsf(x7), 1e-38f)
                                                                 : (x7 != 0.f ? fabsf(xd) / fabsf(x7) : 3.4e38f);
                    rel = fmaxf(rel, r);
                    dd0 += fabsf(f4c(a0, c));
                    dd1 += fabsf(f4c(a1, c));
                    sx7 += fabsf(x7);
                    // added now, so an accepted region needs no second pass; a split
                    // region is taken back out below
                    if (atomic) atomicAdd(mean + e, (double)(area * x7));
                    else mean[e] = (double)(area * x7);
                }
            }
        }
        // the FP32 estimate's decision, unless it is too close to call
        const bool near_tol = fabsf(rel - rtol) <= fmaxf(0.05f * rtol, 4e-6f);
        const bool accept = rel <= rtol;
        if (accept && !near_tol) return true;
        // the fourth differences cancel most of the values they are formed from, so
        // their FP32 error is measured against the values (sx7), not against themselves
        const bool near_dim = !accept && fabsf(dd0 - dd1) <= 1e-3f * (dd0 + dd1) + 4e-6f * sx7;
        for (int qd = 0; qd < EQ4; ++qd) {  // take the FP32 values back out
            float4 v7, vd, a0, a1;
            rule(qd, v7, vd, a0, a1);
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const int e = 4 * qd + c;
                if (e < E) {
                    if (atomic) atomicAdd(mean + e, -(double)(area * f4c(v7, c)));
                    else mean[e] = 0.;
                }
            }
        }
        if (near_tol || near_dim)
            return gm_region64(corners, W1, h, w, src, c0, c1, h0, h1, false, U, E, (double)rtol, mean, atomic, dim);
        *dim = dd0 >= dd1 ? 0 : 1;
        return false;
    }
    {  // the depth limit: accepted without a check
        for (int qd = 0; qd < EQ4; ++qd) {
            float4 v7, vd, a0, a1;
            rule(qd, v7, vd, a0, a1);
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const int e = 4 * qd + c;
                if (e < E) {
                    if (atomic) atomicAdd(mean + e, (double)(area * f4c(v7, c)));
                    else mean[e] = (double)(area * f4c(v7, c));
                }
            }
        }
        return true;
    }
}

// Pushes the two halves of a region (lower half first in the queue), or returns
// false when the queue is full.
__device__ __forceinline__ bool push_halves(QRegion* q, int* qcount, int qcap, int sp, float c0, float c1,
                                            float h0, float h1, int dim) {
    const int k = atomicAdd(qcount, 2);
    if (k + 2 > qcap) return false;
    QRegion a {sp, c0, c1, h0, h1}, b = a;
    if (dim == 0) {
        a.h0 = b.h0 = 0.5f * h0;
        a.c0 = c0 - 0.5f * h0;
        b.c0 = c0 + 0.5f * h0;
    } else {
        a.h1 = b.h1 = 0.5f * h1;
        a.c1 = c1 - 0.5f * h1;
        b.c1 = c1 + 0.5f * h1;
    }
    q[k] = a;
    q[k + 1] = b;
    return true;
}

__device__ __forceinline__ void load_tables(const SepTab* septab, double* sq, float4* scoef) {
    for (int k = threadIdx.x; k < ND + 1; k += blockDim.x) sq[k] = septab->q[k];
    for (int k = threadIdx.x; k < 2 * ND; k += blockDim.x) scoef[k] = ((const float4*)septab->coef)[k];
    __syncthreads();
}

// Grid-wide barrier of a cooperative launch: the last block to arrive resets the
// count and advances the generation; the others poll it with a bounded wait.
// Returns false (in every thread of the block) when the wait ran out.
constexpr int GRID_WAIT_LIMIT = 1 << 24;  // polls of ~100 ns: about a second or more

__device__ __forceinline__ bool grid_barrier(unsigned* bar, unsigned nblocks, unsigned* gen) {
    __syncthreads();
    bool ok = true;
    if (threadIdx.x == 0) {
        const unsigned g = *gen;
        __threadfence();
        const unsigned arrived = atomicAdd(&bar[0], 1u) + 1u;
        if (arrived == nblocks) {
            atomicExch(&bar[0], 0u);
            __threadfence();
            atomicAdd(&bar[1], 1u);
        } else {
            int it = 0;
            while (atomicAdd(&bar[1], 0u) == g && ++it < GRID_WAIT_LIMIT) __nanosleep(100);
            ok = it < GRID_WAIT_LIMIT;
        }
        __threadfence();
        *gen = g + 1u;
    }
    return __syncthreads_and(ok);
}

// All levels in one persistent launch (cooperative: every block resident).  Level
// 0: item k = (source, pixel) k, the whole pixel as one region; level L >= 1: item k
// = region k of level L - 1's queue.  Levels are separated by grid barriers.
__global__ void __launch_bounds__(AT, 2)
k_adaptive_levels(const double* __restrict__ corners, const SrcInfo* __restrict__ info,
                  const SepTab* __restrict__ septab, const float* __restrict__ lut, const double* __restrict__ upsf,
                  int S, int H, int W, int E, float rtol, int max_depth, double* __restrict__ mean,
                  QRegion* __restrict__ q, long long qcap, int* __restrict__ counts, unsigned* __restrict__ bar,
                  int* __restrict__ status) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ unsigned gen_s;
    double* sq = (double*)(smem + AO_SQ);
    float4* scoef = (float4*)(smem + AO_COEF);
    float* wk = (float*)(smem + AO_WIN) + threadIdx.x;
    if (threadIdx.x == 0) gen_s = atomicAdd(&bar[1], 0u);
    load_tables(septab, sq, scoef);
    const int npix = H * W, W1 = W + 1;
    const int EP = (E + 3) & ~3;
    const long long stride = (long long)gridDim.x * AT;
    for (int level = 0; level <= max_depth; ++level) {
        const bool last = level >= max_depth;
        QRegion* qout = q + (size_t)(level & 1) * qcap;
        int* qout_count = counts + level;
        if (level == 0) {
            const long long n = (long long)S * npix;
            for (long long k = (long long)blockIdx.x * AT + threadIdx.x; k < n; k += stride) {
                const int s = (int)(k / npix), pix = (int)(k - (long long)s * npix);
                const SrcInfo si = info[s];
                const int h = pix / W, w = pix - h * W;
                const PixGeom g = pixel_geom(corners, W1, h, w, si);
                double* m = mean + (size_t)k * E;
                int dim = 0;
                const float* Y = lut + (size_t)s * ND * EP;
                const double* U = upsf + (size_t)s * ND * E;
                if (gm_region(g, 0.f, 0.f, 1.f, 1.f, last, sq, scoef, wk, Y, U, corners, W1, h, w, si.dir, E, EP,
                              rtol, m, false, &dim))
                    continue;
                if (!push_halves(qout, qout_count, (int)qcap, (int)k, 0.f, 0.f, 1.f, 1.f, dim))
                    gm_region(g, 0.f, 0.f, 1.f, 1.f, true, sq, scoef, wk, Y, U, corners, W1, h, w, si.dir, E, EP,
                              rtol, m, false, &dim);  // queue full: keep the estimate
            }
        } else {
            const QRegion* qin = q + (size_t)((level - 1) & 1) * qcap;
            const long long n = min((long long)counts[level - 1], qcap);
            for (long long k = (long long)blockIdx.x * AT + threadIdx.x; k < n; k += stride) {
                const QRegion r = qin[k];
                const int s = r.sp / npix, pix = r.sp - s * npix;
                const SrcInfo si = info[s];
                const int h = pix / W, w = pix - h * W;
                const PixGeom g = pixel_geom(corners, W1, h, w, si);
                const float* Y = lut + (size_t)s * ND * EP;
                const double* U = upsf + (size_t)s * ND * E;
                double* m = mean + (size_t)r.sp * E;
                int dim = 0;
                if (gm_region(g, r.c0, r.c1, r.h0, r.h1, last, sq, scoef, wk, Y, U, corners, W1, h, w, si.dir, E, EP,
                              rtol, m, true, &dim))
                    continue;
                if (!push_halves(qout, qout_count, (int)qcap, r.sp, r.c0, r.c1, r.h0, r.h1, dim))
                    gm_region(g, r.c0, r.c1, r.h0, r.h1, true, sq, scoef, wk, Y, U, corners, W1, h, w, si.dir, E,
                              EP, rtol, m, true, &dim);
            }
        }
        if (level == max_depth) break;
        if (!grid_barrier(bar, gridDim.x, &gen_s)) {
            if (threadIdx.x == 0) atomicExch(status, 1);
            return;
        }
    }
}

// c7 on the adaptive map: per block (chunk, source) the FP64 sums over pixels
// inside the boundary radius of mean * solid angle, in a fixed order.
template <typename T>
__global__ void __launch_bounds__(AT) k_adaptive_integral(const double* __restrict__ centers,
                                                          const double* __restrict__ omega,
                                                          const SrcInfo* __restrict__ info,
                                                          const T* __restrict__ mean, int H, int W, int E,
                                                          int nch, double* __restrict__ sums_out) {
    __shared__ double part[AT];
    const int s = blockIdx.y, t = threadIdx.x;
    const SrcInfo si = info[s];
    const int npix = H * W, W1 = W + 1;
    double ch2 = 2.0 * sin(0.5 * si.radius_rad);
    ch2 *= ch2;
    // thread (g, e): energy e over pixels g, g + G, ... of the block's range
    const int G = AT / E, g = t / E, e = t - g * E;
    const int p_lo = (int)((long long)npix * blockIdx.x / nch), p_hi = (int)((long long)npix * (blockIdx.x + 1) / nch);
    double acc = 0.;
    if (si.in_fov && t < G * E) {
        for (int pix = p_lo + g; pix < p_hi; pix += G) {
            const int h = pix / W, w = pix - h * W;
            const double* c = centers + 3 * (h * W1 + w);
            const double x = si.dir[0] - c[0], y = si.dir[1] - c[1], z = si.dir[2] - c[2];
            const double d2 = x * x + y * y + z * z;
            bool inside;
            if (d2 < ch2 * (1.0 - 1e-12)) inside = true;
            else if (d2 > ch2 * (1.0 + 1e-12)) inside = false;
            else inside = dir_diff(si.dir, c) <= si.radius_rad;
            if (inside) acc += (double)mean[((size_t)s * npix + pix) * E + e] * omega[pix];
        }
    }
    part[t] = acc;
    __syncthreads();
    for (int ee = t; ee < E; ee += AT) {
        double v = 0.;
        for (int gg = 0; gg < G; ++gg) v += part[gg * E + ee];
        sums_out[((size_t)s * nch + blockIdx.x) * E + ee] = v;
    }
}

// The adaptive map from its FP64 means: value = mean * omega * exposure * correction.
__global__ void k_scale_map64(const double* __restrict__ mean, float* __restrict__ out,
                              const double* __restrict__ omega, const double* __restrict__ scale, int npix, int E) {
    __shared__ double sc[256];
    const int s = blockIdx.y;
    for (int e = threadIdx.x; e < E; e += blockDim.x) sc[e] = scale[(size_t)s * E + e];
    __syncthreads();
    const unsigned n = (unsigned)npix * (unsigned)E;
    const double* m = mean + (size_t)s * n;
    float* o = out + (size_t)s * n;
    for (unsigned k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const unsigned pix = k / (unsigned)E;
        o[k] = (float)(m[k] * omega[pix] * sc[k - pix * (unsigned)E]);
    }
}

// c8 + c10 and the solid angle: value = mean * omega * exposure * correction.
// out[s][pix][e] *= omega[pix] (FP64 product rounded to FP32) * scale[s][e]; four
// consecutive values per thread (one 16-byte load and store, one division), the
// source's first values up to a 16-byte boundary and its last ones one by one.
__device__ __forceinline__ float scale_value(float v, const double* omega, const float* sc, unsigned pix,
                                             unsigned e) {
    return (float)((double)v * omega[pix]) * sc[e];
}
__global__ void k_scale_map(float* __restrict__ out, const double* __restrict__ omega,
                            const double* __restrict__ scale, int npix, int E) {
    __shared__ float sc[256];
    const int s = blockIdx.y;
    for (int e = threadIdx.x; e < E; e += blockDim.x) sc[e] = (float)scale[(size_t)s * E + e];
    __syncthreads();
    const unsigned n = (unsigned)npix * (unsigned)E, uE = (unsigned)E;
    float* o = out + (size_t)s * n;
    const unsigned mis = (unsigned)(((uintptr_t)o >> 2) & 3u);  // o is 4-byte aligned
    const unsigned head = min((4u - mis) & 3u, n);
    const unsigned nq = (n - head) >> 2, tail0 = head + 4 * nq;
    const unsigned tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
    if (tid < head) o[tid] = scale_value(o[tid], omega, sc, tid / uE, tid % uE);
    if (tid < n - tail0) {
        const unsigned k = tail0 + tid;
        o[k] = scale_value(o[k], omega, sc, k / uE, k % uE);
    }
    float4* o4 = reinterpret_cast<float4*>(o + head);
    for (unsigned q = tid; q < nq; q += nth) {
        const unsigned k = head + 4 * q;
        unsigned pix = k / uE, e = k - pix * uE;
        float4 v = o4[q];
        float* f = reinterpret_cast<float*>(&v);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            f[i] = scale_value(f[i], omega, sc, pix, e);
            if (++e == uE) { e = 0; ++pix; }
        }
        o4[q] = v;
    }
}

bool srcmap_adaptive_supported(int E) { return E >= 1 && E <= 256; }

int launch_adaptive_map(const double* corners, const double* centers, const double* omega, const SrcInfo* info,
                        const double* upsf, int S, int H, int W, int E, double rtol, int max_depth, int nch,
                        double* sums, double* mean64, int* status, cudaStream_t st) {
    int rc = upload_gm(st);
    if (rc) return rc;
    const SepTab* tab = nullptr;
    rc = build_septab(st, &tab);
    if (rc) return rc;
    const int npix = H * W;
    // the mean PSF rows in FP32, [S][401][E]
    const int EP = (E + 3) & ~3;  // table rows padded to whole float4s
    float* lut = (float*)workspace(W_LUT, sizeof(float) * (size_t)S * ND * EP + 16);
    // two region queues (ping-pong), their counters per level and the grid barrier
    long long cap = 4LL * S * npix;
    cap = cap < (1 << 20) ? (1 << 20) : cap;
    cap = cap > (1 << 26) ? (1 << 26) : cap;
    QRegion* q = (QRegion*)workspace(W_SPARSE, sizeof(QRegion) * 2 * (size_t)cap + 16);
    int* counts = (int*)workspace(W_WMETA, sizeof(int) * 64);
    if (!lut || !q || !counts) return XTS_ERR_OOM;
    unsigned* bar = (unsigned*)(counts + 32);
    XTS_LAUNCH("k_lut_scaled", st, k_lut_scaled<<<lut_scaled_grid(S), 256, 0, st>>>(upsf, nullptr, S, E, EP, lut,
                                                                                       nullptr, nullptr));
    XTS_CUDA(cudaFuncSetAttribute(k_adaptive_levels, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)A_SMEM));
    XTS_CUDA(cudaMemsetAsync(counts, 0, sizeof(int) * 64, st));
    int dev = 0, nsm = 148, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    XTS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_adaptive_levels, AT, A_SMEM));
    const unsigned G = (unsigned)(nsm * (per_sm > 0 ? per_sm : 1));
    // one cooperative launch: every block resident, so the grid barriers between levels complete
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(G);
    cfg.blockDim = dim3(AT);
    cfg.dynamicSmemBytes = A_SMEM;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const float rtol_f = (float)rtol;
    cudaError_t le = cudaSuccess;
    XTS_LAUNCH("k_adaptive_map", st, le = cudaLaunchKernelEx(&cfg, k_adaptive_levels, corners, info, tab,
                                                             (const float*)lut, upsf, S, H, W, E, rtol_f, max_depth,
                                                             mean64, q, cap, counts, bar, status));
    if (le != cudaSuccess) return cuda_error(le, "cooperative launch of k_adaptive_levels");
    (void)centers; (void)omega; (void)nch; (void)sums;  // the c7 sums: launch_mean_integral, by the caller
    return XTS_OK;
}

// The map integral of FP32 pixel means: block (c, s) takes pixels
// [c npix / nc, (c + 1) npix / nc) of source s; warp w of the block the runs of 32
// pixels w, w + 8, ... of that range.  Per run each lane tests one pixel against the
// source's boundary; then, for the inside pixels in order, lane l adds energies l,
// l + 32, ... (a pixel's E means are contiguous, so the loads coalesce).  Per block the
// warps' partial sums are added in a fixed order into sums[s][c][e].
constexpr int MI_WARPS = 8;
constexpr int MI_EQ = 8;  // energies per lane: E <= 256
__global__ void __launch_bounds__(32 * MI_WARPS) k_mean_integral(const double* __restrict__ centers,
                                                                 const double* __restrict__ omega,
                                                                 const SrcInfo* __restrict__ info,
                                                                 const float* __restrict__ mean, int H, int W, int E,
                                                                 int nc, double* __restrict__ sums_out) {
    __shared__ double part[MI_WARPS][AT];
    const int s = blockIdx.y, t = threadIdx.x, lane = t & 31, wp = t >> 5;
    const SrcInfo si = info[s];
    const int npix = H * W, W1 = W + 1;
    double ch2 = 2.0 * sin(0.5 * si.radius_rad);
    ch2 *= ch2;
    const int p_lo = (int)((long long)npix * blockIdx.x / nc), p_hi = (int)((long long)npix * (blockIdx.x + 1) / nc);
    const int nq = (E + 31) >> 5;
    double acc[MI_EQ];
#pragma unroll
    for (int q = 0; q < MI_EQ; ++q) acc[q] = 0.;
    if (si.in_fov) {
        const float* m = mean + (size_t)s * npix * E;
        // 32 pixels per round: each lane tests its own pixel against the boundary, then
        // the warp sums the inside pixels' rows (lane = energy), two rows per step so
        // that two loads are in flight
        for (int pix0 = p_lo + 32 * wp; pix0 < p_hi; pix0 += 32 * MI_WARPS) {
            const int pix = pix0 + lane;
            bool inside = false;
            double om = 0.;
            if (pix < p_hi) {
                const int h = pix / W, w = pix - h * W;
                const double* c = centers + 3 * (h * W1 + w);
                const double x = si.dir[0] - c[0], y = si.dir[1] - c[1], z = si.dir[2] - c[2];
                const double d2 = x * x + y * y + z * z;
                if (d2 < ch2 * (1.0 - 1e-12)) inside = true;
                else if (d2 > ch2 * (1.0 + 1e-12)) inside = false;
                else inside = dir_diff(si.dir, c) <= si.radius_rad;
                if (inside) om = omega[pix];
            }
            unsigned mask = __ballot_sync(0xffffffffu, inside);
            while (mask) {
                const int l1 = __ffs(mask) - 1;
                mask &= mask - 1;
                const int l2 = mask ? __ffs(mask) - 1 : -1;
                if (l2 >= 0) mask &= mask - 1;
                const double om1 = __shfl_sync(0xffffffffu, om, l1);
                const double om2 = __shfl_sync(0xffffffffu, om, l2 < 0 ? l1 : l2);
                const float* mp1 = m + (size_t)(pix0 + l1) * E;
                const float* mp2 = m + (size_t)(pix0 + (l2 < 0 ? l1 : l2)) * E;
                float v1[MI_EQ], v2[MI_EQ];
#pragma unroll
                for (int q = 0; q < MI_EQ; ++q) {
                    const int e = lane + 32 * q;
                    const bool on = q < nq && e < E;
                    v1[q] = on ? mp1[e] : 0.f;
                    v2[q] = on && l2 >= 0 ? mp2[e] : 0.f;
                }
#pragma unroll
                for (int q = 0; q < MI_EQ; ++q) {
                    acc[q] += (double)v1[q] * om1;
                    if (l2 >= 0) acc[q] += (double)v2[q] * om2;
                }
            }
        }
    }
#pragma unroll
    for (int q = 0; q < MI_EQ; ++q) {
        const int e = lane + 32 * q;
        if (q < nq && e < E) part[wp][e] = acc[q];
    }
    __syncthreads();
    for (int e = t; e < E; e += 32 * MI_WARPS) {
        double v = 0.;
        for (int k = 0; k < MI_WARPS; ++k) v += part[k][e];
        sums_out[((size_t)s * nc + blockIdx.x) * E + e] = v;
    }
}

// Chunks of the FP32 mean-map integral per source: enough blocks for every SM.
int mean_integral_chunks(int S, int npix) {
    int nc = (2400 + (S > 0 ? S : 1) - 1) / (S > 0 ? S : 1);
    const int mx = (npix + 255) / 256;
    return nc < 1 ? 1 : (nc > mx ? mx : nc);
}

int launch_mean_integral(const double* centers, const double* omega, const SrcInfo* info, const float* mean, int S,
                         int H, int W, int E, int nch, double* sums, cudaStream_t st) {
    if (E < 1 || E > AT) return set_error(XTS_ERR_ARG, "map integral of pixel means: E (%d) above %d", E, AT);
    XTS_LAUNCH("k_mean_integral", st, k_mean_integral<<<dim3(nch, S), 32 * MI_WARPS, 0, st>>>(
                                          centers, omega, info, mean, H, W, E, nch, sums));
    return XTS_OK;
}

int launch_mean_integral64(const double* centers, const double* omega, const SrcInfo* info, const double* mean, int S,
                           int H, int W, int E, int nch, double* sums, cudaStream_t st) {
    if (E < 1 || E > AT) return set_error(XTS_ERR_ARG, "map integral of pixel means: E (%d) above %d", E, AT);
    XTS_LAUNCH("k_adaptive_integral", st, k_adaptive_integral<double><<<dim3(nch, S), AT, 0, st>>>(
                                              centers, omega, info, mean, H, W, E, nch, sums));
    return XTS_OK;
}

int launch_scale_map64(const double* mean, float* out, const double* omega, const double* scale, int S, int npix,
                       int E, cudaStream_t st) {
    const unsigned n = (unsigned)npix * (unsigned)E;
    unsigned gx = (n + 255) / 256;
    if (gx > 1024) gx = 1024;
    XTS_LAUNCH("k_scale_map", st, k_scale_map64<<<dim3(gx, S), 256, 0, st>>>(mean, out, omega, scale, npix, E));
    return XTS_OK;
}

int launch_scale_map(float* out, const double* omega, const double* scale, int S, int npix, int E,
                     cudaStream_t st) {
    const unsigned n = (unsigned)npix * (unsigned)E;
    unsigned gx = (n + 255) / 256;
    if (gx > 1024) gx = 1024;
    XTS_LAUNCH("k_scale_map", st, k_scale_map<<<dim3(gx, S), 256, 0, st>>>(out, omega, scale, npix, E));
    return XTS_OK;
}

}  // namespace xts
