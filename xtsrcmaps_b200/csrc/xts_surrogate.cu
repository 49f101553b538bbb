// xts_surrogate.cu -- the surrogate model map: pixel means of the mean PSF from
// the network of xts_mlp.cu, with the 12-point rule of the plain path as the
// fallback and as the check; and the training samples the network learns from.
//
// For a source and a pixel in bilinear form p(u, v) = src + A + B u + C v + D uv
// (the corners' unit vectors blended as square_ptswts, points_weights.hpp:5-56):
//   * centre separation theta_c = 2 asin(|A| / 2), cell solid angle 4 |B x C|,
//     size delta = sqrt(solid angle), rho = theta_c / delta;
//   * the centre's offset t_c in the separation table: its logsep interpolation
//     weight between the bracketing rows (the mean PSF is the piecewise-linear
//     interpolant of 401 rows, whose curvature error, up to ~4e-3 of u between
//     rows, depends on where the pixel falls between them);
//   * per energy: u_c = the mean PSF at theta_c, the log slope
//     ln(U[i] / U[i-1]) / step of the table segment holding theta_c, and the
//     rule mean m = sum_p w_p u(theta_p) over the 12 points (the plain path's
//     cubature, cubature.implementation.cxx:21-55, with the logsep row and weight
//     of convolve_pixel_psf_logsep.hpp:39-55, keys fixed).
// The network's target is y = ln(m / u_c) rho^2; a value is m = u_c exp(y / rho^2).
// All of this is FP64 up to the network's FP32 input.
//
// The map: first the rule's pixel means for every value, by the plain path's
// window and write passes over the unscaled FP32 table (xts_srcmap_win.cu).  Then,
// per chunk of sources, k_sur_features writes the features of the values the
// network may take (inside the training range and a served error cell), compacted;
// the network runs on the compacted rows only; k_sur_assemble puts its values into
// the map, except at every SUR_CHECK_EVERY-th pixel, where the rule's value stays and
// the relative difference to the network's is recorded per source.  Sources whose
// check fails are redone by the FP64 rule (k_sur_fallback), and the map integral,
// correction and scalings follow as for the adaptive map.
#include <cfloat>
#include <vector>

#include "xts_point.cuh"

namespace xts {

constexpr int SUR_CHECK_EVERY = 16;         // every 16th pixel's values are also taken by the rule
constexpr long long SUR_CHUNK_VALUES = 1ll << 26;  // values per pass of the network (sources chunked)

__device__ __forceinline__ int sur_row(double sdeg, double* t) {
    const double j = sdeg < 1e-4 ? 1. : 1. + RECIPSTEP * (LN_1E4 + log(sdeg));
    int idx = 1 + (int)j;
    idx = idx > 400 ? 400 : (idx < 2 ? 2 : idx);
    *t = REDM1 * (sdeg * 1e4 * exp(SEP_STEP * (2. - idx)) - 1.);
    return idx;
}

__device__ __forceinline__ double sur_lerp(const double* U, int E, int e, int idx, double t) {
    return (1.0 - t) * U[(size_t)(idx - 1) * E + e] + t * U[(size_t)idx * E + e];
}

struct SurPix {
    int idx[12];
    double tt[12];
    int ic;
    double tc;
    float f0, f1, f2;
    double rho;
};

// the 12 rule points' rows and weights
__device__ __forceinline__ void sur_points(const PixGeom& g, SurPix& sp) {
    const PixQ c = pixel_q(g);
#pragma unroll
    for (int p = 0; p < 12; ++p) sp.idx[p] = sur_row(2.0 * R2D * asin(0.5 * sqrt(point_q2(c, p))), &sp.tt[p]);
}

// the centre's separation, row and offset, and the pixel features
__device__ __forceinline__ void sur_centre_geom(const PixGeom& g, SurPix& sp) {
    const double alen = sqrt(fma(g.Ax, g.Ax, fma(g.Ay, g.Ay, g.Az * g.Az)));
    const double thc = 2.0 * asin(0.5 * alen);  // radians
    const double cx = g.By * g.Cz - g.Bz * g.Cy, cy = g.Bz * g.Cx - g.Bx * g.Cz, cz = g.Bx * g.Cy - g.By * g.Cx;
    const double om = 4.0 * sqrt(cx * cx + cy * cy + cz * cz);
    const double delta = sqrt(om);
    sp.rho = thc / delta;
    sp.ic = sur_row(R2D * thc, &sp.tc);
    sp.f0 = (float)log10(sp.rho);
    sp.f1 = (float)sp.tc;
    sp.f2 = (float)log10(om * R2D * R2D);
}

__device__ __forceinline__ void sur_pixel(const PixGeom& g, SurPix& sp) {
    sur_points(g, sp);
    sur_centre_geom(g, sp);
}

__device__ __forceinline__ double sur_rule(const SurPix& sp, const double* U, int E, int e) {
    double m = 0.;
#pragma unroll
    for (int p = 0; p < 12; ++p) m += c_rule_uv[p][3] * sur_lerp(U, E, e, sp.idx[p], sp.tt[p]);
    return m;
}

// log slope ln(hi / lo) / step of a table segment, in FP32 (a network input)
__device__ __forceinline__ float sur_slope(double lo, double hi) {
    return (lo > 0. && hi > 0.) ? logf((float)hi / (float)lo) * (float)(1.0 / SEP_STEP) : 0.f;
}

// centre value and the log slope of its table segment at energy e
__device__ __forceinline__ double sur_centre(const SurPix& sp, const double* U, int E, int e, double* slope) {
    const double lo = U[(size_t)(sp.ic - 1) * E + e], hi = U[(size_t)sp.ic * E + e];
    *slope = sur_slope(lo, hi);
    return (1.0 - sp.tc) * lo + sp.tc * hi;
}

// ------------------------------------------------------------------ samples
__device__ __forceinline__ unsigned long long splitmix(unsigned long long& s) {
    unsigned long long z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__device__ __forceinline__ double uni(unsigned long long& s) { return (double)(splitmix(s) >> 11) * 0x1.0p-53; }

__global__ void k_sur_samples(const double* __restrict__ upsf, const double* __restrict__ logEs, int S, int E,
                              long long n, unsigned long long seed, double rho_min, float* __restrict__ X,
                              float* __restrict__ Y) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    unsigned long long st = seed ^ ((unsigned long long)i * 0xD1B54A32D192ED03ull);
    splitmix(st);
    const int s = min((int)(uni(st) * S), S - 1);
    const int e = min((int)(uni(st) * E), E - 1);
    const double size = 0.025 + 0.175 * uni(st);             // degrees
    const double asp = exp(log(1.25) * (2.0 * uni(st) - 1.0));
    const double lo = fmax(0.001, rho_min * size);
    const double th = lo * exp(uni(st) * log(30.0 / lo)) * D2R;
    const double al = uni(st) * HALFPI;
    const double ha = 0.5 * size * sqrt(asp) * D2R, hb = 0.5 * size / sqrt(asp) * D2R;
    // source at the pole; the pixel centre at polar angle th, axes rotated by al
    const double c[3] = {sin(th), 0.0, cos(th)};
    const double e1[3] = {cos(th), 0.0, -sin(th)}, e2[3] = {0.0, 1.0, 0.0};
    const double ca = cos(al), sa = sin(al);
    double U[3], V[3], k[4][3];
    for (int q = 0; q < 3; ++q) { U[q] = ca * e1[q] + sa * e2[q]; V[q] = -sa * e1[q] + ca * e2[q]; }
    const double su[4] = {-1, 1, 1, -1}, sv[4] = {-1, -1, 1, 1};  // LL, LR, UR, UL
    for (int j = 0; j < 4; ++j) {
        double nn = 0.;
        for (int q = 0; q < 3; ++q) {
            k[j][q] = c[q] + su[j] * ha * U[q] + sv[j] * hb * V[q];
            nn += k[j][q] * k[j][q];
        }
        nn = 1.0 / sqrt(nn);
        for (int q = 0; q < 3; ++q) k[j][q] *= nn;
    }
    const double src[3] = {0.0, 0.0, 1.0};
    PixGeom g;
    const double *a = k[0], *b = k[1], *cc = k[2], *d = k[3];
    g.Ax = 0.25 * ((a[0] + b[0]) + (cc[0] + d[0])) - src[0];
    g.Ay = 0.25 * ((a[1] + b[1]) + (cc[1] + d[1])) - src[1];
    g.Az = 0.25 * ((a[2] + b[2]) + (cc[2] + d[2])) - src[2];
    g.Bx = 0.25 * ((b[0] + cc[0]) - (a[0] + d[0]));
    g.By = 0.25 * ((b[1] + cc[1]) - (a[1] + d[1]));
    g.Bz = 0.25 * ((b[2] + cc[2]) - (a[2] + d[2]));
    g.Cx = 0.25 * ((cc[0] + d[0]) - (a[0] + b[0]));
    g.Cy = 0.25 * ((cc[1] + d[1]) - (a[1] + b[1]));
    g.Cz = 0.25 * ((cc[2] + d[2]) - (a[2] + b[2]));
    g.Dx = 0.25 * ((a[0] + cc[0]) - (b[0] + d[0]));
    g.Dy = 0.25 * ((a[1] + cc[1]) - (b[1] + d[1]));
    g.Dz = 0.25 * ((a[2] + cc[2]) - (b[2] + d[2]));
    SurPix sp;
    sur_pixel(g, sp);
    const double* Us = upsf + (size_t)s * ND * E;
    double slope;
    const double uc = sur_centre(sp, Us, E, e, &slope);
    const double m = sur_rule(sp, Us, E, e);
    X[i * 5 + 0] = sp.f0;
    X[i * 5 + 1] = sp.f1;
    X[i * 5 + 2] = sp.f2;
    X[i * 5 + 3] = (float)logEs[e];
    X[i * 5 + 4] = (float)slope;
    Y[i] = (float)(log(m / uc) * sp.rho * sp.rho);
}

int launch_surrogate_samples(const double* upsf, const double* logEs, int S, int E, long long n,
                             unsigned long long seed, double rho_min, float* X, float* Y, cudaStream_t st) {
    if (S < 1 || E < 1 || n < 0 || !(rho_min >= 0.))
        return set_error(XTS_ERR_ARG, "surrogate samples: S %d, E %d, n %lld, rho_min %g", S, E, n, rho_min);
    if (n == 0) return XTS_OK;
    int rc = upload_rule_uv(st);
    if (rc) return rc;
    XTS_LAUNCH("k_sur_samples", st, k_sur_samples<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(
                                        upsf, logEs, S, E, n, seed, rho_min, X, Y));
    return XTS_OK;
}

// ------------------------------------------------------------------ model map
struct SurRange {
    float lo[5], hi[5], rho_min;
    float c0, cs0, c1, cs1;          // cell bins: a = (f0 - c0) * cs0, b = (slope - c1) * cs1
    const unsigned char* cell_ok;    // [NR * NS] device, or NULL
};
constexpr int SUR_NCELL = XTS_MLP_CELL_NR * XTS_MLP_CELL_NS;

__device__ __forceinline__ const unsigned char* sur_cells_to_shared(const SurRange& rg, unsigned char* sh) {
    if (!rg.cell_ok) return nullptr;
    for (int k = threadIdx.x; k < SUR_NCELL; k += blockDim.x) sh[k] = rg.cell_ok[k];
    return sh;
}

constexpr int SF_PIX = 128;
constexpr int SF_THREADS = 256;

struct SurPixS {
    float f0, f1, f2, eps;
    double tc;
    int ic;
    int crow;  // error-cell row of log10 rho (0 without cells); -1: the network takes none of the pixel's values
    int tc01;  // the centre's offset tc lies in [0, 1]
};

// Per (segment row ic, energy) of the sources of a chunk: whether the network may take
// a value whose centre falls in that table segment -- the energy and the segment's log
// slope inside the training range and the slope inside the error-cell grid -- as
// code = slope cell column | sign class << 8 (sign class 1: both rows positive, so
// u_c > 0 for tc in [0, 1]; 2: neither positive, u_c <= 0; 0: u_c decided per value),
// or -1; and the slope itself.  seg, slope: [ns][ND][E] (row 0 unused).
__global__ void k_sur_segments(const double* __restrict__ upsf, const double* __restrict__ logEs, int ns, int E,
                               SurRange rg, short* __restrict__ seg, float* __restrict__ slope) {
    const long long n = (long long)ns * ND * E;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int e = (int)(i % E);
        const long long jr = i / E;
        const int r = (int)(jr % ND);
        if (r == 0) { seg[i] = -1; slope[i] = 0.f; continue; }
        const double lo = upsf[i - E], hi = upsf[i];
        const float sl = sur_slope(lo, hi);
        const float le = (float)logEs[e];
        bool ok = le >= rg.lo[3] && le <= rg.hi[3] && sl >= rg.lo[4] && sl <= rg.hi[4];
        int b = 0;
        if (rg.cell_ok) {
            const float bf = (sl - rg.c1) * rg.cs1;
            ok = ok && bf >= 0.f && bf < (float)XTS_MLP_CELL_NS;
            b = ok ? (int)bf : 0;
        }
        const int cls = (lo > 4.0 * DBL_MIN && hi > 4.0 * DBL_MIN) ? 1 : ((lo <= 0. && hi <= 0.) ? 2 : 0);
        seg[i] = ok ? (short)(b | (cls << 8)) : (short)-1;
        slope[i] = sl;
    }
}

__device__ __forceinline__ bool sur_geo_ok(const SurPix& q, const SurRange& rg) {
    return q.rho >= rg.rho_min && q.f0 >= rg.lo[0] && q.f0 <= rg.hi[0] && q.f1 >= rg.lo[1] && q.f1 <= rg.hi[1] &&
           q.f2 >= rg.lo[2] && q.f2 <= rg.hi[2];
}

// The network takes a value iff its pixel's geometric features lie in the training
// range (rho >= rho_min among them), the centre value u_c = (1 - tc) U[ic - 1] + tc U[ic]
// is positive, log10 E and the log slope of the centre's table segment lie in range, and
// the error cell (log10 rho, slope) is one the network was calibrated to serve: the pixel
// part is phase 1's crow, the (segment, energy) part k_sur_segments' code.

// Per block: SF_PIX pixels of one source of a chunk.  Phase 1, one thread per
// pixel: the centre and the features that do not depend on energy, into shared
// memory.  Pass 1, one thread per (pixel, energy) value in the maps' order: whether
// the network takes the value (a bit in shared memory).  The block then reserves
// room for its accepted values in the compacted network input with one atomic, and
// pass 2 writes each accepted value's five features, aux = (u_c, 1 / rho^2) and its
// chunk-relative value index there.
__global__ void __launch_bounds__(SF_THREADS) k_sur_features(const double* __restrict__ corners,
                                                             const SrcInfo* __restrict__ info,
                                                             const double* __restrict__ upsf,
                                                             const double* __restrict__ logEs, int s0, int H, int W,
                                                             int E, SurRange rg, float* __restrict__ X,
                                                             float2* __restrict__ aux, unsigned* __restrict__ vidx,
                                                             unsigned long long* __restrict__ n_acc,
                                                             unsigned long long* __restrict__ accepted,
                                                             const short* __restrict__ seg,
                                                             const float* __restrict__ slope, long long ldx) {
    __shared__ SurPixS sp[SF_PIX];
    __shared__ unsigned okbits[SF_PIX * 256 / 32];  // one bit per (pixel, energy) value, E <= 256
    __shared__ unsigned wpre[SF_PIX * 256 / 32];    // accepted values before each word
    __shared__ unsigned wsum[SF_THREADS / 32];
    __shared__ unsigned long long base_s;
    __shared__ unsigned char cells_s[SUR_NCELL];
    const int s = s0 + blockIdx.y, t = threadIdx.x, lane = t & 31, wp = t >> 5;
    const int npix = H * W, p0 = blockIdx.x * SF_PIX;
    const int np = min(SF_PIX, npix - p0);
    const int nv = np * E;
    const unsigned char* cells = sur_cells_to_shared(rg, cells_s);
    if (t < np) {
        const int pix = p0 + t, h = pix / W, w = pix - h * W;
        SurPix q;
        sur_centre_geom(pixel_geom(corners, W + 1, h, w, info[s]), q);
        SurPixS& o = sp[t];
        o.f0 = q.f0; o.f1 = q.f1; o.f2 = q.f2;
        o.eps = (float)(1.0 / (q.rho * q.rho));
        o.tc = q.tc;
        o.ic = q.ic;
        o.tc01 = q.tc >= 0. && q.tc <= 1.;
        int crow = sur_geo_ok(q, rg) ? 0 : -1;
        if (crow == 0 && cells) {
            const float a = (q.f0 - rg.c0) * rg.cs0;
            crow = (a >= 0.f && a < (float)XTS_MLP_CELL_NR) ? (int)a : -1;
        }
        o.crow = crow;
    }
    __syncthreads();
    const double* U = upsf + (size_t)s * ND * E;
    const short* sg = seg + (size_t)blockIdx.y * ND * E;
    const size_t vb = ((size_t)blockIdx.y * npix + p0) * E;  // first value of the block (chunk-relative)
    unsigned cnt = 0;
    // the value of thread t in round i is k = t + 256 i: its pixel and energy by steps
    const int dq = SF_THREADS / E, dr = SF_THREADS - dq * E;
    int lp = t / E, e = t - lp * E;
    for (int k0 = t - lane; k0 < nv; k0 += SF_THREADS) {  // a warp takes 32 consecutive values
        const int k = k0 + lane;
        bool ok = false;
        if (k < nv) {
            const SurPixS& o = sp[lp];
            if (o.crow >= 0) {
                const int code = sg[(size_t)o.ic * E + e];
                if (code >= 0) {
                    const int cls = code >> 8;
                    bool pos;
                    if (o.tc01 && cls == 1) pos = true;
                    else if (o.tc01 && cls == 2) pos = false;
                    else {
                        const double lo = U[(size_t)(o.ic - 1) * E + e], hi = U[(size_t)o.ic * E + e];
                        pos = (1.0 - o.tc) * lo + o.tc * hi > 0.;
                    }
                    ok = pos && (!cells || cells[o.crow * XTS_MLP_CELL_NS + (code & 255)] != 0);
                }
            }
        }
        const unsigned bits = __ballot_sync(0xffffffffu, ok);
        if (lane == 0) okbits[k0 >> 5] = bits;
        cnt += ok;
        lp += dq;
        e += dr;
        if (e >= E) { e -= E; ++lp; }
    }
    // the block's accepted values in value order: exclusive prefix counts of the
    // acceptance words, one reservation per block
    __syncthreads();
    const int nw = (nv + 31) >> 5, cpt = (nw + SF_THREADS - 1) / SF_THREADS;
    const int w0 = t * cpt, w1 = min(nw, w0 + cpt);
    unsigned mine = 0;
    for (int w = w0; w < w1; ++w) mine += __popc(okbits[w]);
    unsigned inc = mine;
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned v = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += v;
    }
    if (lane == 31) wsum[wp] = inc;
    __syncthreads();
    unsigned before = 0, total = 0;
    for (int w = 0; w < SF_THREADS / 32; ++w) {
        before += w < wp ? wsum[w] : 0u;
        total += wsum[w];
    }
    unsigned run = before + inc - mine;
    for (int w = w0; w < w1; ++w) {
        wpre[w] = run;
        run += __popc(okbits[w]);
    }
    if (t == 0) {
        base_s = total ? atomicAdd(n_acc, (unsigned long long)total) : 0ull;
        if (total) atomicAdd(accepted + s, (unsigned long long)total);
    }
    __syncthreads();
    (void)cnt;
    // pass 2: a warp's accepted lanes write consecutive rows (feature-major X [5][ldx])
    const unsigned long long base = base_s;
    const float* slp = slope + (size_t)blockIdx.y * ND * E;
    lp = t / E;
    e = t - lp * E;
    for (int k0 = t - lane; k0 < nv; k0 += SF_THREADS) {
        const unsigned word = okbits[k0 >> 5];
        if ((word >> lane) & 1u) {
            const unsigned long long j = base + wpre[k0 >> 5] + __popc(word & ((1u << lane) - 1u));
            const SurPixS& o = sp[lp];
            const double lo = U[(size_t)(o.ic - 1) * E + e], hi = U[(size_t)o.ic * E + e];
            const double uc = (1.0 - o.tc) * lo + o.tc * hi;
            X[j] = o.f0;
            X[ldx + j] = o.f1;
            X[2 * ldx + j] = o.f2;
            X[3 * ldx + j] = (float)logEs[e];
            X[4 * ldx + j] = slp[(size_t)o.ic * E + e];
            aux[j] = make_float2((float)uc, o.eps);
            vidx[j] = (unsigned)(vb + k0 + lane);
        }
        lp += dq;
        e += dr;
        if (e >= E) { e -= E; ++lp; }
    }
}

// The network's values into the map: row i of the compacted input is chunk value
// vidx[i]; n_acc rows (counted on the device), at most n_max.  At every
// SUR_CHECK_EVERY-th pixel the map keeps the rule's value and the relative
// difference of the network's is recorded: the largest per source in err and the
// count in chk (s0: the chunk's first source; per_src = H W E values per source).
__global__ void k_sur_assemble(const float2* __restrict__ aux, const unsigned* __restrict__ vidx,
                               const float* __restrict__ y, const unsigned long long* __restrict__ n_acc,
                               long long n_max, int s0, long long per_src, int E, float* __restrict__ mean,
                               float* __restrict__ err, unsigned long long* __restrict__ chk) {
    const long long n = min(n_max, (long long)*n_acc);
    const long long stride = (long long)gridDim.x * blockDim.x;
    const unsigned ps = (unsigned)per_src;
    for (long long i0 = (long long)blockIdx.x * blockDim.x; i0 < n; i0 += stride) {
        const long long i = i0 + threadIdx.x;
        const bool live = i < n;
        int sl = -1;  // the chunk-relative source of a checked value
        float r = 0.f;
        if (live) {
            const unsigned v = vidx[i];
            const float2 a = aux[i];
            const float m = a.x * expf(y[i] * a.y);
            const unsigned j = v / ps;  // chunk values fit 32 bits
            const unsigned pix = (v - j * ps) / (unsigned)E;
            if (pix % SUR_CHECK_EVERY == 0) {
                const float rule = mean[v];
                const float d = rule != 0.f ? fabsf(m - rule) / fabsf(rule) : fabsf(m);
                r = d != d ? 3.4e38f : d;
                sl = (int)j;
            } else {
                mean[v] = m;
            }
        }
        // per warp: lanes of the same source merged before one atomic each
        if (!__any_sync(0xffffffffu, sl >= 0)) continue;
        const unsigned grp = __match_any_sync(0xffffffffu, sl);
        float worst = r;
        for (int o = 0; o < 32; ++o) {
            const float ro = __shfl_sync(0xffffffffu, r, o);
            if ((grp >> o) & 1u) worst = fmaxf(worst, ro);
        }
        if (sl >= 0 && (threadIdx.x & 31) == __ffs(grp) - 1) {
            if (worst > 0.f) atomicMax((int*)(err + s0 + sl), __float_as_int(worst));  // non-negative floats order as ints
            atomicAdd(chk + s0 + sl, (unsigned long long)__popc(grp));  // the group's lanes are its checked values
        }
    }
}

// Every source listed (the rule for every value when the window path does not
// take the map's energy count).
__global__ void k_sur_all_list(int S, int* __restrict__ list, int* __restrict__ list_n) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < S; s += gridDim.x * blockDim.x) list[s] = s;
    if (blockIdx.x == 0 && threadIdx.x == 0) *list_n = S;
}

// Sources whose check exceeded tol, in source order: list [S], count list_n[0].
__global__ void k_sur_fail_list(const float* __restrict__ err, int S, float tol, int* __restrict__ list,
                                int* __restrict__ list_n) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int n = 0;
    for (int s = 0; s < S; ++s)
        if (!(err[s] <= tol)) list[n++] = s;
    *list_n = n;
}

// Every value of the listed sources by the rule: a persistent grid over
// (listed source, 128-pixel tile) items, the list's length read on the device.
__global__ void __launch_bounds__(128) k_sur_fallback(const double* __restrict__ corners, const SrcInfo* __restrict__ info,
                                                      const double* __restrict__ upsf, const int* __restrict__ list,
                                                      const int* __restrict__ list_n, int H, int W, int E,
                                                      float* __restrict__ mean) {
    const int npix = H * W, ntile = (npix + 127) / 128;
    const long long items = (long long)(*list_n) * ntile;
    for (long long it = blockIdx.x; it < items; it += gridDim.x) {
        const int s = list[it / ntile];
        const int pix = (int)(it % ntile) * 128 + threadIdx.x;
        if (pix >= npix) continue;
        const int h = pix / W, w = pix - h * W;
        SurPix sp;
        sur_pixel(pixel_geom(corners, W + 1, h, w, info[s]), sp);
        const double* U = upsf + (size_t)s * ND * E;
        for (int e = 0; e < E; ++e) mean[((size_t)s * npix + pix) * E + e] = (float)sur_rule(sp, U, E, e);
    }
}

// The latest call's device counters, for xts_surrogate_last_stats.
struct SurLast {
    bool valid = false;
    int S = 0;
    long long per_src = 0;
    float tol = 0.f;
    const float* err = nullptr;
    const unsigned long long* acc = nullptr;
    const unsigned long long* chk = nullptr;
    int* status = nullptr;
};
static SurLast g_sur_last;

int surrogate_last_stats(xts_surrogate_stats* stats, cudaStream_t st) {
    if (!stats) return set_error(XTS_ERR_ARG, "surrogate_last_stats: null argument");
    memset(stats, 0, sizeof(*stats));
    if (!g_sur_last.valid) return XTS_OK;
    const SurLast& L = g_sur_last;
    const int S = L.S;
    std::vector<float> herr(S > 0 ? S : 1);
    std::vector<unsigned long long> hacc(S > 0 ? S : 1), hchk(S > 0 ? S : 1);
    XTS_CUDA(cudaMemcpyAsync(herr.data(), L.err, sizeof(float) * S, cudaMemcpyDeviceToHost, st));
    XTS_CUDA(cudaMemcpyAsync(hacc.data(), L.acc, sizeof(unsigned long long) * S, cudaMemcpyDeviceToHost, st));
    XTS_CUDA(cudaMemcpyAsync(hchk.data(), L.chk, sizeof(unsigned long long) * S, cudaMemcpyDeviceToHost, st));
    int rc = mlp_check_status(L.status, st);  // synchronises the stream
    if (rc) return rc;
    float worst = 0.f;
    long long accepted = 0, evaluated = 0, checked = 0;
    int nfail = 0;
    for (int s = 0; s < S; ++s) {
        worst = herr[s] > worst ? herr[s] : worst;
        evaluated += (long long)hacc[s];
        checked += (long long)hchk[s];
        if (!(herr[s] <= L.tol)) ++nfail;
        else accepted += (long long)(hacc[s] - hchk[s]);
    }
    stats->values = (long long)S * L.per_src;
    stats->accepted = accepted;  // the checked pixels' and the redone maps' values are the rule's
    stats->checked = checked;
    stats->maps_fallback = nfail;
    stats->max_check_err = worst;
    stats->evaluated = evaluated;
    return XTS_OK;
}

int launch_srcmap_surrogate(const SrcmapDev& a, const double* corners, const double* centers, const double* omega,
                            const SrcInfo* info, double* scale, int nch, cudaStream_t st) {
    const xts_mlp* net = a.surrogate;
    const int H = (int)a.wcs.naxis1, W = (int)a.wcs.naxis2, S = a.S, E = a.E;
    const long long npix = (long long)H * W;
    if (!net->params || !net->wbf16) return set_error(XTS_ERR_ARG, "surrogate map: network parameters missing");
    for (int k = 0; k < XTS_MLP_IN; ++k)
        if (!(net->in_sd[k] > 0.f)) return set_error(XTS_ERR_ARG, "surrogate map: in_sd[%d] must be > 0", k);
    if (!(net->out_sd > 0.f)) return set_error(XTS_ERR_ARG, "surrogate map: out_sd must be > 0");
    if (net->cell_ok && !(net->cell_hi[0] > net->cell_lo[0] && net->cell_hi[1] > net->cell_lo[1]))
        return set_error(XTS_ERR_ARG, "surrogate map: error-cell ranges must be increasing");
    int rc = upload_rule_uv(st);
    if (rc) return rc;
    const long long per_src = npix * E;
    int sc = (int)(SUR_CHUNK_VALUES / (per_src > 0 ? per_src : 1));
    sc = sc < 1 ? 1 : (sc > S ? S : sc);
    const long long nmax = per_src * sc;
    float* X = (float*)workspace(W_SUR_X, sizeof(float) * 5 * (size_t)nmax + 16);
    float2* aux = (float2*)workspace(W_SUR_AUX, sizeof(float2) * (size_t)nmax + 16);
    float* yv = (float*)workspace(W_SUR_Y, sizeof(float) * (size_t)nmax + 16);
    unsigned* vidx = (unsigned*)workspace(W_SUR_IDX, sizeof(unsigned) * (size_t)nmax + 16);
    // per chunk: the segment codes [sc][ND][E] (short) and slopes (float)
    const size_t nseg = (size_t)sc * ND * E;
    char* segbuf = (char*)workspace(W_SUR_SEG, align_up(sizeof(short) * nseg, 256) + sizeof(float) * nseg + 16);
    if (!segbuf) return XTS_ERR_OOM;
    short* seg = (short*)segbuf;
    float* slope = (float*)(segbuf + align_up(sizeof(short) * nseg, 256));
    if (!vidx) return XTS_ERR_OOM;
    // per source: largest check difference, values the network evaluated, values
    // checked; then the compacted row count, the status word, the failed-source
    // count and list
    const size_t o_cnt = align_up(sizeof(float) * S, 16), o_chk = o_cnt + align_up(8 * (size_t)S, 16);
    const size_t o_ctr = o_chk + align_up(8 * (size_t)S, 16);
    const size_t o_list = o_ctr + 64;
    char* misc = (char*)workspace(W_SUR_ERR, o_list + sizeof(int) * (size_t)S + 16);
    if (!X || !aux || !yv || !misc) return XTS_ERR_OOM;
    float* err = (float*)misc;
    unsigned long long* acc_d = (unsigned long long*)(misc + o_cnt);
    unsigned long long* chk_d = (unsigned long long*)(misc + o_chk);
    unsigned long long* counts = (unsigned long long*)(misc + o_ctr);  // [1] compacted rows
    int* status = (int*)(counts + 4);
    int* list_n = status + 1;
    int* list_d = (int*)(misc + o_list);
    XTS_CUDA(cudaMemsetAsync(misc, 0, o_list, st));
    SurRange rg;
    for (int k = 0; k < 5; ++k) { rg.lo[k] = net->lo[k]; rg.hi[k] = net->hi[k]; }
    rg.rho_min = net->rho_min;
    rg.cell_ok = net->cell_ok;
    rg.c0 = net->cell_lo[0];
    rg.c1 = net->cell_lo[1];
    rg.cs0 = net->cell_ok ? (float)XTS_MLP_CELL_NR / (net->cell_hi[0] - net->cell_lo[0]) : 0.f;
    rg.cs1 = net->cell_ok ? (float)XTS_MLP_CELL_NS / (net->cell_hi[1] - net->cell_lo[1]) : 0.f;
    float* mean = (float*)a.out;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    // the rule's pixel means for every value (the window and write passes of the plain
    // path over the unscaled table); the network's values replace them below
    if (srcmap_win_supported(E)) {
        int* wstatus = (int*)workspace(W_MISC, 64);
        if (!wstatus) return XTS_ERR_OOM;
        XTS_CUDA(cudaMemsetAsync(wstatus, 0, sizeof(int), st));
        StreamJoin same(st, st, nullptr);
        rc = launch_srcmap_win(corners, centers, omega, info, S, H, W, E, a.upsf, a.partial, a.exposure, nullptr,
                               nullptr, nullptr, nullptr, nullptr, wstatus, mean, 0, nullptr, nullptr, same, st, true);
        if (rc) return rc;
    } else {  // more energies than the write pass holds: the FP64 rule per value
        XTS_LAUNCH("k_sur_all_list", st, k_sur_all_list<<<(unsigned)((S + 255) / 256), 256, 0, st>>>(S, list_d, list_n));
        XTS_LAUNCH("k_sur_fallback", st, k_sur_fallback<<<(unsigned)(4 * nsm), 128, 0, st>>>(
                                              corners, info, a.upsf, list_d, list_n, H, W, E, mean));
    }
    // With host copy-out hooks (a host-mode call), the sources go in groups of about
    // a.chunk_sources: each group is finished (failed maps redone, map integral,
    // correction, scaling) and handed to the hook, so its copy to the host overlaps
    // the next group's work.  Without hooks, one group.
    const int gsz = a.on_chunk && a.chunk_sources > 0 ? a.chunk_sources : S;
    for (int g0 = 0; g0 < S; g0 += gsz) {
        const int g1 = S - g0 < gsz ? S : g0 + gsz;
        for (int s0 = g0; s0 < g1; s0 += sc) {
            const int ns = g1 - s0 < sc ? g1 - s0 : sc;
            const long long n = per_src * ns;
            const dim3 gf((unsigned)((npix + SF_PIX - 1) / SF_PIX), (unsigned)ns);
            XTS_CUDA(cudaMemsetAsync(counts + 1, 0, sizeof(unsigned long long), st));
            XTS_LAUNCH("k_sur_segments", st, k_sur_segments<<<(unsigned)(4 * nsm), 256, 0, st>>>(
                                                 a.upsf + (size_t)s0 * ND * E, a.logEs, ns, E, rg, seg, slope));
            XTS_LAUNCH("k_sur_features", st, k_sur_features<<<gf, SF_THREADS, 0, st>>>(
                                                 corners, info, a.upsf, a.logEs, s0, H, W, E, rg, X, aux, vidx,
                                                 counts + 1, acc_d, seg, slope, nmax));
            // the network on the compacted rows; their count stays on the device
            if ((rc = launch_mlp_forward_dev(net, X, counts + 1, n, yv, status, st, nmax))) return rc;
            float* m0 = mean + (size_t)s0 * per_src;
            XTS_LAUNCH("k_sur_assemble", st, k_sur_assemble<<<(unsigned)(8 * nsm), 256, 0, st>>>(
                                                 aux, vidx, yv, counts + 1, n, s0, per_src, E, m0, err, chk_d));
        }
        // the group's maps whose check failed are redone by the rule, listed and
        // scheduled on the device
        const int gn = g1 - g0;
        XTS_LAUNCH("k_sur_fail_list", st, k_sur_fail_list<<<1, 32, 0, st>>>(err + g0, gn, (float)a.check_tol, list_d,
                                                                            list_n));
        XTS_LAUNCH("k_sur_fallback", st, k_sur_fallback<<<(unsigned)(4 * nsm), 128, 0, st>>>(
                                              corners, info + g0, a.upsf + (size_t)g0 * ND * E, list_d, list_n, H, W,
                                              E, mean + (size_t)g0 * per_src));
        if (gsz < S) {
            if ((rc = finish_mean_map_range(a, g0, gn, centers, omega, info, scale, st))) return rc;
            if ((rc = a.on_chunk(a.on_chunk_ctx, g0, gn, st))) return rc;
        }
    }
    g_sur_last.valid = true;
    g_sur_last.S = S;
    g_sur_last.per_src = per_src;
    g_sur_last.tol = (float)a.check_tol;
    g_sur_last.err = err;
    g_sur_last.acc = acc_d;
    g_sur_last.chk = chk_d;
    g_sur_last.status = status;
    if (a.sur_stats && (rc = surrogate_last_stats(a.sur_stats, st))) return rc;
    if (gsz < S) return XTS_OK;
    return finish_mean_map(a, centers, omega, info, scale, nch, st);
}

}  // namespace xts
