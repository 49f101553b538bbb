// xts_srcmap_fast.cu -- the FP32 source-map write pass (d1 + d2 + c8 + c10) as
// an issue- and store-efficient sm_100a kernel.
//
// Per pixel (phase 1, one thread per pixel, FP64 where the geometry needs it):
//   * the 12 rule points of square_ptswts (points_weights.hpp:93-107) are the
//     bilinear blend p(u,v) = A + B u + C v + D uv of the pixel's corner unit
//     vectors, so p - src is formed from four per-pixel FP64 vectors without
//     ever rounding p itself; its squared chord q = |p - src|^2 is FP64;
//   * the LUT column of convolve_pixel_psf_logsep (convolve_pixel_psf_logsep.hpp:39-55),
//     idx = 1 + floor(1 + ln(1e4 s)/step) clamped to [2, 400], is found by
//     comparing q with the FP64 squared chords of the 401 table separations
//     (an FP32 log only provides the starting guess);
//   * the interpolation weight t = (s - S[idx-1]) / (S[idx] - S[idx-1]) is
//     (g - 1)/(e^step - 1) with g = s / S[idx-1] = asin(x sqrt(1+d))/asin(x),
//     d = q/Q[idx-1] - 1 formed in FP64; g - 1 = d P_k(d) with a per-row
//     degree-4 polynomial fitted on the host (max error 5e-12 on g - 1).  Points
//     outside the tabulated range (s < 1e-4 deg, s >= 70 deg) take the
//     reference's own FP64 formula;
//   * the points' weights (1-t) w and t w are accumulated into a dense window
//     of at most 8 consecutive table rows, then multiplied by the pixel's solid
//     angle.  Pixels whose points span more rows (the few next to the source)
//     are evaluated directly by their thread.
// Phase 2 walks the tile's output in flat (pixel, energy) order: each value is
// sum_j W[p][j] * Y'[rbase + j][e], where Y' = uPsf * exposure * correction in
// FP32 (the per-(source, energy) scale folded into the table), read through L1.
// Values are staged in shared memory and written with one TMA bulk store
// (cp.async.bulk.global.shared::cta) per tile.
#include <math.h>

#include "xts_geom.cuh"
#include "xts_internal.cuh"

namespace xts {

// Separation tables shared by every launch (see build_septab).
struct SepTab {
    double q[ND + 1];      // squared chord of S[k] (k = 0..400), q[401] = +inf guard
    float coef[ND][8];     // row k (= idx - 1): {1/q[k], c0..c4 of P_k(z)}, z = (d - D0)/DS
};
constexpr float DPOLY_C = 0.035f;   // centre and half-width of the fitted d range
constexpr float DPOLY_H = 0.037f;

static SepTab* g_septab_dev[64] = {};

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
        // Chebyshev interpolation of f(d) = (g(d) - 1)/d at 5 nodes in z in [-1, 1]
        const int N = 5;
        long double fz[N], zn[N];
        for (int i = 0; i < N; ++i) {
            zn[i] = cosl(3.14159265358979323846264338327950288L * (i + 0.5L) / N);
            long double d = (long double)DPOLY_C + (long double)DPOLY_H * zn[i];
            fz[i] = (asinl(xlo * sqrtl(1.0L + d)) / a0 - 1.0L) / d;
        }
        // Chebyshev coefficients, then monomial coefficients in z
        long double cc[N];
        for (int j = 0; j < N; ++j) {
            long double s = 0;
            for (int i = 0; i < N; ++i) s += fz[i] * cosl(j * acosl(zn[i]));
            cc[j] = s * (j == 0 ? 1.0L : 2.0L) / N;
        }
        // T0=1, T1=z, T2=2z^2-1, T3=4z^3-3z, T4=8z^4-8z^2+1
        long double m[N] = {cc[0] - cc[2] + cc[4], cc[1] - 3 * cc[3], 2 * cc[2] - 8 * cc[4], 4 * cc[3], 8 * cc[4]};
        h.coef[k][0] = (float)(1.0L / qk);
        for (int j = 0; j < N; ++j) h.coef[k][1 + j] = (float)m[j];
    }
    SepTab* d = nullptr;
    XTS_CUDA(cudaMalloc(&d, sizeof(SepTab)));
    XTS_CUDA(cudaMemcpyAsync(d, &h, sizeof(SepTab), cudaMemcpyHostToDevice, st));
    XTS_CUDA(cudaStreamSynchronize(st));
    g_septab_dev[dev] = d;
    *out = d;
    return XTS_OK;
}

// Rule in the bilinear form: u, v, u*v and 0.25 * weight per point.
__constant__ double c_rule_uv[12][4];

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
    XTS_CUDA(cudaMemcpyToSymbolAsync(c_rule_uv, b, sizeof(b), 0, cudaMemcpyHostToDevice, st));
    XTS_CUDA(cudaStreamSynchronize(st));
    dev_done = dev;
    return XTS_OK;
}

// Scaled FP32 table Y'[s][d][e] = uPsf * (exposure * correction), energies padded.
__global__ void k_lut_scaled(const double* upsf, const double* scale, int S, int E, int Epad,
                             float* lut) {
    size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    size_t n = (size_t)S * ND * Epad;
    if (k >= n) return;
    int e = (int)(k % Epad);
    size_t sd = k / Epad;
    int s = (int)(sd / ND);
    lut[k] = e < E ? (float)(upsf[sd * E + e] * scale[(size_t)s * E + e]) : 0.f;
}

constexpr int FT = 256;   // pixels per tile == threads per block
constexpr int RW = 8;     // dense row window per pixel
constexpr int WST = 9;    // padded stride of the window (bank-conflict free)

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

// Shared-memory layout (byte offsets, each 16-byte aligned).
constexpr size_t OFF_SQ = 0;
constexpr size_t OFF_COEF = (8 * (ND + 1) + 15) / 16 * 16;
constexpr size_t OFF_WIN = OFF_COEF + sizeof(float4) * 2 * ND;
constexpr size_t OFF_META = OFF_WIN + (sizeof(float) * FT * WST + 15) / 16 * 16;
constexpr size_t OFF_STAGE = OFF_META + sizeof(int) * FT;

size_t srcmap_fast_smem(int E) { return OFF_STAGE + sizeof(float) * ((size_t)FT * E + 8); }

// Interpolation weight outside the tabulated range (s < 1e-4 deg or s >= 70 deg):
// the reference's own FP64 formula (convolve_pixel_psf_logsep.hpp:45-47).  Kept
// out of line: it runs for a handful of points per map.
__device__ __noinline__ float t_exact(double q, int idx) {
    const double sdeg = 2.0 * R2D * asin(0.5 * sqrt(q));
    return (float)(REDM1 * (sdeg * 1e4 * exp(SEP_STEP * (2. - idx)) - 1.));
}

// Row and interpolation weight of one rule point from its FP64 squared chord q.
// The FP32 starting guess is within one row of the bracket (|error| < 0.3 rows
// up to 70 deg, where the row is clamped to 400 anyway); one branch-free
// correction against the FP64 squared chords gives the reference's row.
__device__ __forceinline__ int point_row(double q, const double* sq, const float4* scoef, float* t_out) {
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
    const float4 c0 = scoef[2 * (idx - 1)], c1 = scoef[2 * (idx - 1) + 1];
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

// Bilinear form of the rule points of pixel (h, w) relative to the source:
// p(u, v) - src = A + B u + C v + D uv (points_weights.hpp:93-107).
struct PixGeom { double Ax, Ay, Az, Bx, By, Bz, Cx, Cy, Cz, Dx, Dy, Dz; };

__device__ __forceinline__ PixGeom pixel_geom(const double* corners, int W1, int h, int w, const SrcInfo& si) {
    const double* a = corners + 3 * (h * W1 + w);            // LL
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

__global__ void __launch_bounds__(FT, 3)
k_srcmap_fast(const double* __restrict__ corners, const double* __restrict__ omega,
              const SrcInfo* __restrict__ info, const float* __restrict__ lut,
              const SepTab* __restrict__ septab, int H, int W, int E, int Epad, int nchunk,
              float* __restrict__ out) {
    extern __shared__ __align__(16) unsigned char smem[];
    double* sq = (double*)(smem + OFF_SQ);       // [ND + 1] squared chords
    float4* scoef = (float4*)(smem + OFF_COEF);  // [ND][2]
    float* wwin = (float*)(smem + OFF_WIN);      // [FT][WST] row-window weights
    int* meta = (int*)(smem + OFF_META);         // [FT]: rbase | nrows << 16
    float* stage = (float*)(smem + OFF_STAGE);   // [FT * E + 8] output tile

    const int s = blockIdx.y;
    for (int k = threadIdx.x; k < ND + 1; k += FT) sq[k] = septab->q[k];
    for (int k = threadIdx.x; k < 2 * ND; k += FT) scoef[k] = ((const float4*)septab->coef)[k];
    const SrcInfo si = info[s];
    const int npix = H * W, W1 = W + 1;
    const int ntiles = (npix + FT - 1) / FT;
    const float* Y = lut + (size_t)s * ND * Epad;
    const int t = threadIdx.x;
    float* wr = wwin + t * WST;
    __syncthreads();

    for (int tile = blockIdx.x; tile < ntiles; tile += nchunk) {
        const int p0 = tile * FT;
        const int np = min(FT, npix - p0);
        const long long g0 = ((long long)s * npix + p0) * E;  // first flat output
        const int m = (int)(g0 & 3);                          // staging residue
        const int nflat = np * E;

        // ---------------- phase 1: this thread's pixel (overlaps the previous tile's store).
        // The RW-row window is anchored on the pixel centre's row; a point whose
        // rows fall outside it makes the pixel "wide" (only next to the source).
        int nrows = 0, rbase = 0;
        bool wide = false;
        const int pix = p0 + t;
        if (t < np) {
            const int h = pix / W, w = pix - h * W;
            const PixGeom g = pixel_geom(corners, W1, h, w, si);
            float tc;
            const int ic = point_row(fma(g.Ax, g.Ax, fma(g.Ay, g.Ay, g.Az * g.Az)), sq, scoef, &tc);
            rbase = min(max(ic - 1 - RW / 2, 0), ND - RW);
#pragma unroll
            for (int j = 0; j < RW; ++j) wr[j] = 0.f;
            int lo = RW, hi = -1;
#pragma unroll
            for (int p = 0; p < 12; ++p) {
                float tt;
                const int r = point_row(point_q(g, p), sq, scoef, &tt) - 1 - rbase;
                if (r >= 0 && r < RW - 1) {  // thread-private window in shared memory
                    const float wgt = (float)c_rule_uv[p][3];
                    wr[r] = fmaf(1.f - tt, wgt, wr[r]);
                    wr[r + 1] = fmaf(tt, wgt, wr[r + 1]);
                    lo = min(lo, r);
                    hi = max(hi, r + 1);
                } else {
                    wide = true;
                }
            }
            if (!wide) {
                const float om = (float)omega[pix];
                nrows = hi - lo + 1;
                for (int j = 0; j < nrows; ++j) wr[j] = wr[j + lo] * om;
                rbase += lo;
            }
        }
        if (t == 0) bulk_wait_read();  // the previous tile's bulk store has read the stage
        meta[t] = (rbase & 0xffff) | (nrows << 16);
        __syncthreads();

        // wide pixels: evaluated point by point by their own thread, compensated sum
        if (wide) {
            const int h = pix / W, w = pix - h * W;
            const PixGeom g = pixel_geom(corners, W1, h, w, si);
            const float om = (float)omega[pix];
            float* dst = stage + m + t * E;
            for (int e0 = 0; e0 < E; e0 += 4) {
                float acc[4] = {0.f, 0.f, 0.f, 0.f}, comp[4] = {0.f, 0.f, 0.f, 0.f};
                for (int p = 0; p < 12; ++p) {
                    float tt;
                    const int idx = point_row(point_q(g, p), sq, scoef, &tt);
                    const float wgt = (float)c_rule_uv[p][3];
                    const float* yl = Y + (size_t)(idx - 1) * Epad + e0;
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const float term = fmaf((1.f - tt) * wgt, __ldg(yl + k), tt * wgt * __ldg(yl + Epad + k));
                        const float s2 = acc[k] + term;
                        comp[k] += fabsf(acc[k]) >= fabsf(term) ? (acc[k] - s2) + term : (term - s2) + acc[k];
                        acc[k] = s2;
                    }
                }
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    if (e0 + k < E) dst[e0 + k] = (acc[k] + comp[k]) * om;
            }
        }

        // ---------------- phase 2: flat (pixel, energy) order, four independent outputs per thread
        {
            const int dp = FT / E, de = FT - dp * E;
            int f = t, p = t / E;
            int e = t - p * E;
            while (f < nflat) {
                float res[4];
                int fo[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    fo[k] = -1;
                    res[k] = 0.f;
                    if (f < nflat) {
                        const int mt = meta[p];
                        const int nr = mt >> 16;
                        const float* wk = wwin + p * WST;
                        const float* yp = Y + (size_t)(short)(mt & 0xffff) * Epad + e;
                        float a = 0.f;
                        for (int j = 0; j < nr; ++j) a = fmaf(wk[j], __ldg(yp + j * Epad), a);
                        res[k] = a;
                        fo[k] = nr ? f : -1;  // nr == 0: wide pixel, already staged
                    }
                    f += FT;
                    p += dp;
                    e += de;
                    if (e >= E) { e -= E; ++p; }
                }
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    if (fo[k] >= 0) stage[m + fo[k]] = res[k];
            }
        }
        fence_async_shared();
        __syncthreads();
        // ---------------- store: TMA bulk for the 16-byte aligned body, threads for the edges
        const long long ga = (g0 + 3) & ~3LL, gb = (g0 + nflat) & ~3LL;
        if (t == 0 && gb > ga)
            bulk_store(out + ga, stage + m + (int)(ga - g0), (unsigned)((gb - ga) * 4));
        if (t < 8) {
            const long long g = t < 4 ? g0 + t : gb + (t - 4);
            const bool head = t < 4 && g < ga && g < g0 + nflat;
            const bool tail = t >= 4 && g >= gb && g >= ga && g < g0 + nflat;
            if (head || tail) out[g] = stage[m + (int)(g - g0)];
        }
        __syncthreads();
    }
    if (t == 0) bulk_wait_all();
    __syncthreads();
}

// c7 map integral, FP64, without atomics in the common case.  For each tile of
// 256 pixels of one in-FOV source, every pixel whose centre lies within the
// boundary radius (the reference's test 2 asin(|d|/2) <= radius, evaluated on the
// squared chord with an exact fallback next to the threshold) builds its FP64
// row window (interpolation weights times solid angle); then one thread per
// table row sums the tile's windows in a fixed order into the block's row
// histogram.  Pixels whose points leave the window (next to the source) add
// their 24 weights with shared-memory atomics.  The caller folds the block
// histograms with the mean-PSF table: sum_pix omega value(pix, e) = sum_r H[r] U[r][e].
constexpr size_t MI_OFF_SQ = 0;
constexpr size_t MI_OFF_COEF = (8 * (ND + 1) + 15) / 16 * 16;
constexpr size_t MI_OFF_HIST = MI_OFF_COEF + sizeof(float4) * 2 * ND;
constexpr size_t MI_OFF_WTS = MI_OFF_HIST + (8 * ND + 15) / 16 * 16;
constexpr size_t MI_OFF_BASE = MI_OFF_WTS + sizeof(double) * FT * RW;
constexpr size_t MI_SMEM = MI_OFF_BASE + sizeof(int) * (FT + 4);

__global__ void __launch_bounds__(FT) k_map_integral_fast(const double* __restrict__ corners, const double* __restrict__ centers,
                                                          const double* __restrict__ omega, const SrcInfo* __restrict__ info,
                                                          const SepTab* __restrict__ septab, int H, int W, int nch,
                                                          double* __restrict__ hist_out) {
    extern __shared__ __align__(16) unsigned char smem[];
    double* sq = (double*)(smem + MI_OFF_SQ);
    float4* scoef = (float4*)(smem + MI_OFF_COEF);
    double* hist = (double*)(smem + MI_OFF_HIST);
    double* wts = (double*)(smem + MI_OFF_WTS);  // [FT][RW]
    int* wbase = (int*)(smem + MI_OFF_BASE);     // [FT], plus [FT] = row min, [FT+1] = row max
    const int s = blockIdx.y, t = threadIdx.x;
    const SrcInfo si = info[s];
    double* out = hist_out + ((size_t)s * nch + blockIdx.x) * ND;
    if (!si.in_fov) {
        for (int r = t; r < ND; r += FT) out[r] = 0.;
        return;
    }
    for (int k = t; k < ND + 1; k += FT) sq[k] = septab->q[k];
    for (int k = t; k < 2 * ND; k += FT) scoef[k] = ((const float4*)septab->coef)[k];
    for (int r = t; r < ND; r += FT) hist[r] = 0.;
    double ch2 = 2.0 * sin(0.5 * si.radius_rad);
    ch2 *= ch2;
    const int npix = H * W, W1 = W + 1;
    const int ntiles = (npix + FT - 1) / FT;
    __syncthreads();
    for (int tile = blockIdx.x; tile < ntiles; tile += nch) {
        if (t == 0) { wbase[FT] = ND; wbase[FT + 1] = -1; }
        const int pix = tile * FT + t;
        int rb = -1;
        bool inside = false;
        if (pix < npix) {
            const int h = pix / W, w = pix - h * W;
            const double* c = centers + 3 * (h * W1 + w);
            const double x = si.dir[0] - c[0], y = si.dir[1] - c[1], z = si.dir[2] - c[2];
            const double d2 = x * x + y * y + z * z;
            if (d2 < ch2 * (1.0 - 1e-12)) inside = true;
            else if (d2 > ch2 * (1.0 + 1e-12)) inside = false;
            else inside = dir_diff(si.dir, c) <= si.radius_rad;
        }
        __syncthreads();
        if (!__syncthreads_or(inside)) continue;
        if (inside) {
            const int h = pix / W, w = pix - h * W;
            const PixGeom g = pixel_geom(corners, W1, h, w, si);
            const double om = omega[pix];
            float tc;
            const int ic = point_row(fma(g.Ax, g.Ax, fma(g.Ay, g.Ay, g.Az * g.Az)), sq, scoef, &tc);
            const int base = min(max(ic - 1 - RW / 2, 0), ND - RW);
            double* wd = wts + t * RW;
#pragma unroll
            for (int j = 0; j < RW; ++j) wd[j] = 0.;
            bool wide = false;
#pragma unroll
            for (int p = 0; p < 12; ++p) {
                float tt;
                const int idx = point_row(point_q(g, p), sq, scoef, &tt);
                const int r = idx - 1 - base;
                const double wgt = c_rule_uv[p][3];
                const double wa = (double)(1.f - tt) * wgt * om, wb = (double)tt * wgt * om;
                if (r >= 0 && r < RW - 1) {
                    wd[r] += wa;
                    wd[r + 1] += wb;
                } else {
                    wide = true;
                    atomicAdd(&hist[idx - 1], wa);
                    atomicAdd(&hist[idx], wb);
                }
            }
            rb = base;
            atomicMin(&wbase[FT], base);
            atomicMax(&wbase[FT + 1], base + RW - 1);
        }
        wbase[t] = rb;
        __syncthreads();
        const int rmin = wbase[FT], rmax = wbase[FT + 1];
        // 8 threads per row, each over 32 pixels, combined in a fixed shuffle order
        const int sub = t & 7;
        for (int r0 = rmin; r0 <= rmax; r0 += FT / 8) {
            const int r = r0 + (t >> 3);
            double acc = 0.;
            if (r <= rmax) {
                for (int p = sub * 32; p < sub * 32 + 32; ++p) {
                    const int b0 = wbase[p];
                    const int k = r - b0;
                    if (b0 >= 0 && k >= 0 && k < RW) acc += wts[p * RW + k];
                }
            }
            acc += __shfl_xor_sync(0xffffffffu, acc, 1);
            acc += __shfl_xor_sync(0xffffffffu, acc, 2);
            acc += __shfl_xor_sync(0xffffffffu, acc, 4);
            if (sub == 0 && r <= rmax) hist[r] += acc;
        }
        __syncthreads();
    }
    __syncthreads();
    for (int r = t; r < ND; r += FT) out[r] = hist[r];
}

int launch_map_integral_fast(const double* corners, const double* centers, const double* omega,
                             const SrcInfo* info, int S, int H, int W, int nch, double* hist,
                             cudaStream_t st) {
    int rc = upload_rule_uv(st);
    if (rc) return rc;
    const SepTab* tab = nullptr;
    rc = build_septab(st, &tab);
    if (rc) return rc;
    XTS_CUDA(cudaFuncSetAttribute(k_map_integral_fast, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MI_SMEM));
    XTS_LAUNCH("k_map_integral", st, k_map_integral_fast<<<dim3(nch, S), FT, MI_SMEM, st>>>(corners, centers, omega, info, tab, H, W, nch, hist));
    return XTS_OK;
}

int launch_srcmap_fast(const double* corners, const double* omega, const SrcInfo* info,
                       const double* upsf, const double* scale, int S, int H, int W, int E,
                       float* out, cudaStream_t st) {
    int rc = upload_rule_uv(st);
    if (rc) return rc;
    const SepTab* tab = nullptr;
    rc = build_septab(st, &tab);
    if (rc) return rc;
    int Epad = (E + 3) & ~3;
    float* lut = (float*)workspace(W_LUT, sizeof(float) * (size_t)S * ND * Epad + 16);
    if (!lut) return XTS_ERR_OOM;
    size_t n = (size_t)S * ND * Epad;
    XTS_LAUNCH("k_lut_scaled", st, k_lut_scaled<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(upsf, scale, S, E, Epad, lut));
    size_t smem = srcmap_fast_smem(E);
    if (smem > 227 * 1024) return set_error(XTS_ERR_ARG, "E=%d too large for the fast source-map kernel", E);
    XTS_CUDA(cudaFuncSetAttribute(k_srcmap_fast, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    int per_sm = 0;
    XTS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_srcmap_fast, FT, smem));
    if (per_sm < 1) per_sm = 1;
    int npix = H * W, ntiles = (npix + FT - 1) / FT;
    int target = nsm * per_sm * 4;
    int nchunk = (target + S - 1) / S;
    if (nchunk > ntiles) nchunk = ntiles;
    if (nchunk < 1) nchunk = 1;
    dim3 grid(nchunk, S);
    XTS_LAUNCH("k_srcmap", st, k_srcmap_fast<<<grid, FT, smem, st>>>(corners, omega, info, lut, tab, H, W, E, Epad, nchunk, out));
    return XTS_OK;
}

}  // namespace xts
