// xts_srcmap.cu -- steps (c) and (d): pixel geometry, per-pixel cubature of the
// mean PSF, per-map normalisation and the scaled source-map write.
//
//   c1 pix2dir / dir_diff             sky_geom/sky_geom.hxx:237-310
//   c2 square_ptswts (12-point rule)  model_map/mm_cubature/points_weights.hpp:5-56
//   c3 separation + LUT column        model_map/mm_cubature/convolve_pixel_psf_logsep.hpp:39-55
//   d1 pixel cubature                 model_map/mm_cubature/cubature.implementation.cxx:21-55
//   d2 scale_map_by_solid_angle       model_map.scale_map_by_solid_angle.cxx:5-26, math/solid_angle.hpp:42-79
//   c6 psf_boundary_radius            model_map.psf_boundary_radius.cxx:9-62
//   c7 map_integral                   model_map.map_integral.cxx:4-48
//   c8 scale_map_by_exposure          model_map.scale_map_by_exposure.cxx:4-28
//   c9 map_correction_factor          model_map.map_correction_factor.cxx:3-53,
//                                     psf/psf.fast_separation_lower_index.cxx:5-22
//   c10 scale_map_by_correction       model_map.scale_map_by_correction_factor.cxx:4-27
//
// The LUT kernel follows the intended semantics of convolve_pixel_psf_logsep:
// the shipped code never stores its column keys (keys[index] = psfidx is
// missing), so every point would read rows -1 and 0 of the table.  Here the key
// is stored, which equals convolve_pixel_psf_searchsep inside [3e-4, 60] deg and
// keeps logsep's row-400 clamp and its extrapolation below 1e-4 deg.
//
// The map is written once: a first pass gives the map integral of every in-FOV
// source from the pixels whose centre lies within the boundary radius (FP64 row
// histograms: k_map_integral_hist here for the FP64 path, the window pass of
// xts_srcmap_win.cu for the default FP32 path); k_correction_hist folds them in a
// fixed order into 1/sum and the containment factor; the write pass then stores
// value * omega * exposure * factor.  Computing the integral before the write
// costs less than writing the raw map and reading it back.
#include <math.h>

#include <type_traits>

#include "xts_geom.cuh"
#include "xts_internal.cuh"

namespace xts {

// Sommariva & Festa degree-7 12-point rule on [-1,1]^2 (Padova
// "cub_square_lowcard"), as tabulated in model_map/mm_cubature/cubature.hpp:209-225.
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

constexpr int NPTS = 12;
// Per point: 0.25*(1-u)(1-v), 0.25*(1+u)(1-v), 0.25*(1+u)(1+v), 0.25*(1-u)(1+v)
// (corner weights for LL, LR, UR, UL) and 0.25*w.  Scaling by 0.25 is exact, so
// these reproduce points_weights.hpp:96-107 bit for bit.
__constant__ double c_blend[NPTS][5];

static int upload_rule(cudaStream_t st) {
    static int dev_done = -1;
    int dev = -1;
    cudaGetDevice(&dev);
    if (dev_done == dev) return XTS_OK;
    double b[NPTS][5];
    for (int p = 0; p < NPTS; ++p) {
        double u = SQUARE_DEG7[3 * p], v = SQUARE_DEG7[3 * p + 1];
        b[p][0] = 0.25 * ((1.0 - u) * (1.0 - v));
        b[p][1] = 0.25 * ((1.0 + u) * (1.0 - v));
        b[p][2] = 0.25 * ((1.0 + u) * (1.0 + v));
        b[p][3] = 0.25 * ((1.0 - u) * (1.0 + v));
        b[p][4] = 0.25 * SQUARE_DEG7[3 * p + 2];
    }
    XTS_CUDA(cudaMemcpyToSymbolAsync(c_blend, b, sizeof(b), 0, cudaMemcpyHostToDevice, st));
    XTS_CUDA(cudaStreamSynchronize(st));
    dev_done = dev;
    return XTS_OK;
}

// ---------------------------------------------------------------- geometry grids
// corners[i][j] = pix2dir(i + 0.5, j + 0.5), centres[i][j] = pix2dir(i + 1, j + 1),
// i in [0, H], j in [0, W] (1-based FITS pixels).
__device__ inline double quad_half(const double* P, const double* Q, const double* R) {
    double u[3] = {P[0] - Q[0], P[1] - Q[1], P[2] - Q[2]};
    double v[3] = {P[0] - R[0], P[1] - R[1], P[2] - R[2]};
    double nu = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    double nv = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    for (int k = 0; k < 3; ++k) { u[k] /= nu; v[k] /= nv; }
    double c0 = u[1] * v[2] - u[2] * v[1], c1 = u[2] * v[0] - u[0] * v[2], c2 = u[0] * v[1] - u[1] * v[0];
    return dir_diff(P, Q) * dir_diff(P, R) * sqrt(c0 * c0 + c1 * c1 + c2 * c2);
}

// d1 + d2 in one launch, by 8x8 tiles of the (H+1) x (W+1) point grid: the
// tile's corner points and its centre points with a one-point halo (9x9) are
// evaluated by one thread each (145 pix2dir per block, one round), then the
// solid angles of the tile's pixels come from the centres in shared memory.
constexpr int GT = 8;                                    // grid points per tile side (one wave of blocks)
constexpr int GEO_THREADS = (GT + 1) * (GT + 1) + GT * GT;  // 145 tasks, one per thread

__global__ void __launch_bounds__(GEO_THREADS) k_map_geometry(WcsDev w, int H, int W, double* corners,
                                                             double* centers, double* omega) {
    __shared__ double cen[(GT + 1) * (GT + 1)][3];
    const int i0 = blockIdx.y * GT, j0 = blockIdx.x * GT, W1 = W + 1, t = threadIdx.x;
    double v[3];
    if (t < (GT + 1) * (GT + 1)) {  // centre (i0 + li, j0 + lj) = pix2dir(i + 1, j + 1)
        const int li = t / (GT + 1), lj = t - li * (GT + 1), i = i0 + li, j = j0 + lj;
        if (i <= H && j <= W) {
            pix2dir(w, i + 1.0, j + 1.0, v);
            cen[t][0] = v[0]; cen[t][1] = v[1]; cen[t][2] = v[2];
            if (li < GT && lj < GT) {
                double* c = centers + 3 * ((size_t)i * W1 + j);
                c[0] = v[0]; c[1] = v[1]; c[2] = v[2];
            }
        }
    } else {  // corner (i0 + li, j0 + lj) = pix2dir(i + 0.5, j + 0.5)
        const int k = t - (GT + 1) * (GT + 1), li = k / GT, lj = k - li * GT, i = i0 + li, j = j0 + lj;
        if (i <= H && j <= W) {
            pix2dir(w, i + 0.5, j + 0.5, v);
            double* c = corners + 3 * ((size_t)i * W1 + j);
            c[0] = v[0]; c[1] = v[1]; c[2] = v[2];
        }
    }
    __syncthreads();
    // d2: solid angle of pixel (h, w) from the quad of 1-based pixel centres
    // (h+1,w+1), (h+1,w+2), (h+2,w+2), (h+2,w+1), i.e. grid centres (h,w) .. (h+1,w+1)
    if (t < GT * GT) {
        const int li = t / GT, lj = t - li * GT, h = i0 + li, wc = j0 + lj;
        if (h < H && wc < W) {
            const int a = li * (GT + 1) + lj;
            omega[(size_t)h * W + wc] = 0.5 * (quad_half(cen[a], cen[a + 1], cen[a + GT + 1]) +
                                               quad_half(cen[a + GT + 2], cen[a + 1], cen[a + GT + 1]));
        }
    }
}

// c6: in-FOV flag (3.5 pixel buffer) and the minimum distance to the map edge,
// sampled at the corner grid's border.  The separation 2 asin(|a - b| / 2) is
// monotone in the squared chord, so the block finds the smallest squared chord
// over the border first and evaluates the separation only for the points within
// 1e-12 of it (the minimum of those is the minimum over the whole border).  One
// block per source.
__device__ __forceinline__ void border_point(int k, int H, int W, int* i, int* j) {
    if (k < H + 1) { *i = k; *j = 0; }
    else if (k < 2 * (H + 1)) { *i = k - (H + 1); *j = W; }
    else if (k < 2 * (H + 1) + W + 1) { *i = 0; *j = k - 2 * (H + 1); }
    else { *i = H; *j = k - 2 * (H + 1) - (W + 1); }
}

template <typename Op>
__device__ __forceinline__ double block_reduce(double x, double* red, Op op) {
    for (int o = 16; o > 0; o >>= 1) x = op(x, __shfl_xor_sync(0xffffffffu, x, o));
    __syncthreads();  // red is reused between reductions
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = x;
    __syncthreads();
    x = red[0];
    for (int k = 1; k < (int)(blockDim.x + 31) / 32; ++k) x = op(x, red[k]);
    return x;
}

// With cut given, source s's map is its cutout window: the border is the window's
// (corner rows h0 .. h0 + nh, columns w0 .. w0 + nw) and the in-FOV buffer is
// measured from the window's edges; an empty window is out of the FOV.
__global__ void __launch_bounds__(256) k_boundary_chord(WcsDev w, const double* src_sph, int Hf, int Wf,
                                                        const double* corners, SrcInfo* info,
                                                        const xts_cutout* cut) {
    __shared__ double red[32];
    const int s = blockIdx.x, W1 = Wf + 1;
    int h0 = 0, w0 = 0, H = Hf, W = Wf;
    if (cut) {
        const xts_cutout c = cut[s];
        h0 = c.h0; w0 = c.w0; H = c.nh; W = c.nw;
    }
    const int nb = 2 * (H + 1) + 2 * (W + 1);
    const double ra = src_sph[2 * s], dec = src_sph[2 * s + 1];
    double sd[3];
    sph2dir(ra, dec, sd);
    if (H <= 0 || W <= 0) {  // empty cutout (block-uniform)
        if (threadIdx.x == 0) {
            SrcInfo si;
            si.dir[0] = sd[0]; si.dir[1] = sd[1]; si.dir[2] = sd[2];
            si.radius_deg = 0.; si.radius_rad = 0.; si.in_fov = 0; si.pad = 0;
            info[s] = si;
        }
        return;
    }
    auto chord2 = [&](int k) {
        int i, j;
        border_point(k, H, W, &i, &j);
        const double* c = corners + 3 * ((size_t)(h0 + i) * W1 + (w0 + j));
        const double x = sd[0] - c[0], y = sd[1] - c[1], z = sd[2] - c[2];
        return x * x + y * y + z * z;
    };
    double m = INFINITY;
    for (int k = threadIdx.x; k < nb; k += blockDim.x) m = fmin(m, chord2(k));
    m = block_reduce(m, red, [](double a, double b) { return fmin(a, b); });
    double mn = 360.;
    const double lim = m * (1.0 + 1e-12);
    for (int k = threadIdx.x; k < nb; k += blockDim.x)
        if (chord2(k) <= lim) {
            int i, j;
            border_point(k, H, W, &i, &j);
            const double d = R2D * dir_diff(sd, corners + 3 * ((size_t)(h0 + i) * W1 + (w0 + j)));
            mn = mn < d ? mn : d;
        }
    mn = block_reduce(mn, red, [](double a, double b) { return a < b ? a : b; });
    if (threadIdx.x == 0) {
        double r = ra > 180. ? ra - 360. : (ra < -180. ? ra + 360. : ra), p1, p2;
        sph2pix(w, r, dec, &p1, &p2);
        p1 -= h0;  // pixel coordinates of the (window's) sub-map
        p2 -= w0;
        const double buf = 3.5;
        SrcInfo si;
        si.dir[0] = sd[0]; si.dir[1] = sd[1]; si.dir[2] = sd[2];
        si.radius_deg = mn;
        si.radius_rad = D2R * mn;
        si.in_fov = p1 > buf && p1 < (H - buf) && p2 > buf && p2 < (W - buf);
        si.pad = 0;
        info[s] = si;
    }
}

// ---------------------------------------------------------------- cubature core
// c2 + c3 for one pixel: the 12 rule points, their LUT columns and the
// collapsed interpolation weights, in order of first appearance.
__device__ __forceinline__ int pixel_columns(const double* corners, int W1, int h, int w,
                                             const double* src, int* keys, double* va, double* vb) {
    const double* a = corners + 3 * (h * W1 + w);            // LL (h+0.5, w+0.5)
    const double* b = corners + 3 * (h * W1 + w + 1);        // LR (h+0.5, w+1.5)
    const double* c = corners + 3 * ((h + 1) * W1 + w + 1);  // UR (h+1.5, w+1.5)
    const double* d = corners + 3 * ((h + 1) * W1 + w);      // UL (h+1.5, w+0.5)
    double A[3] = {a[0], a[1], a[2]}, B[3] = {b[0], b[1], b[2]};
    double Cc[3] = {c[0], c[1], c[2]}, D[3] = {d[0], d[1], d[2]};
    int n = 0;
#pragma unroll
    for (int p = 0; p < NPTS; ++p) {
        double nn = c_blend[p][0], pn = c_blend[p][1], pp = c_blend[p][2], np = c_blend[p][3];
        double wt = c_blend[p][4];
        double x = (nn * A[0] + pn * B[0] + pp * Cc[0] + np * D[0]) - src[0];
        double y = (nn * A[1] + pn * B[1] + pp * Cc[1] + np * D[1]) - src[1];
        double z = (nn * A[2] + pn * B[2] + pp * Cc[2] + np * D[2]) - src[2];
        double s = 2.0 * R2D * asin(0.5 * sqrt(x * x + y * y + z * z));
        double j = s < 1e-4 ? 1. : 1. + RECIPSTEP * (LN_1E4 + log(s));
        int idx = 1 + (int)j;
        idx = idx > 400 ? 400 : (idx < 2 ? 2 : idx);  // the lower clamp only catches non-finite input
        double t = REDM1 * (s * 1e4 * exp(SEP_STEP * (2. - idx)) - 1.);
        int k = 0;
        while (k < n && keys[k] != idx) ++k;
        if (k == n) { keys[n] = idx; va[n] = 0.; vb[n] = 0.; ++n; }
        va[k] += (1.0 - t) * wt;
        vb[k] += t * wt;
    }
    return n;
}

constexpr int TP = 128;  // pixels per tile (flat h*W + w order)

struct PixCols32 { float va[NPTS], vb[NPTS]; short key[NPTS]; int n; };
struct PixCols64 { double va[NPTS], vb[NPTS]; short key[NPTS]; int n; };


// d1 + d2 + c8 + c10: evaluate every pixel of a tile and write the scaled map.
// Phase 1: one thread per pixel computes its columns (FP64 separations).
// Phase 2: threads walk the tile's output in flat (pixel, energy) order so
// global stores are coalesced.
template <bool F64>
__global__ void __launch_bounds__(TP) k_srcmap(const double* corners, const double* omega,
                                               const SrcInfo* info, const float* lut32,
                                               const double* upsf, const double* scale, int H,
                                               int W, int E, int Epad, void* outp) {
    __shared__ typename std::conditional<F64, PixCols64, PixCols32>::type cols[TP];
    __shared__ double som[TP];
    int tile = blockIdx.x, s = blockIdx.y;
    int npix = H * W, W1 = W + 1;
    int pix0 = tile * TP;
    int npt = min(TP, npix - pix0);
    SrcInfo si = info[s];
    if (threadIdx.x < npt) {
        int pix = pix0 + threadIdx.x;
        int h = pix / W, w = pix - h * W;
        int keys[NPTS]; double va[NPTS], vb[NPTS];
        int n = pixel_columns(corners, W1, h, w, si.dir, keys, va, vb);
        for (int k = 0; k < n; ++k) {
            cols[threadIdx.x].key[k] = (short)keys[k];
            cols[threadIdx.x].va[k] = va[k];
            cols[threadIdx.x].vb[k] = vb[k];
        }
        cols[threadIdx.x].n = n;
        som[threadIdx.x] = omega[pix];
    }
    __syncthreads();
    const double* sc = scale + (size_t)s * E;
    size_t base = ((size_t)s * npix + pix0) * E;
    int nout = npt * E;
    if (F64) {
        const double* U = upsf + (size_t)s * ND * E;
        double* out = (double*)outp + base;
        for (int f = threadIdx.x; f < nout; f += blockDim.x) {
            int p = f / E, e = f - p * E;
            const PixCols64& c = *(const PixCols64*)&cols[p];
            double raw = 0.;
            for (int k = 0; k < c.n; ++k)
                raw += (c.va[k] * U[(size_t)(c.key[k] - 1) * E + e]) + (c.vb[k] * U[(size_t)c.key[k] * E + e]);
            out[f] = ((raw * som[p]) * sc[e]);
        }
    } else {
        const float* Y = lut32 + (size_t)s * ND * Epad;
        float* out = (float*)outp + base;
        for (int f = threadIdx.x; f < nout; f += blockDim.x) {
            int p = f / E, e = f - p * E;
            const PixCols32& c = *(const PixCols32*)&cols[p];
            // compensated (Neumaier) sum over the pixel's columns
            float acc = 0.f, comp = 0.f;
            for (int k = 0; k < c.n; ++k) {
                float term = fmaf(c.va[k], __ldg(Y + (c.key[k] - 1) * Epad + e), c.vb[k] * __ldg(Y + c.key[k] * Epad + e));
                float t = acc + term;
                comp += fabsf(acc) >= fabsf(term) ? (acc - t) + term : (term - t) + acc;
                acc = t;
            }
            out[f] = (float)((double)(acc + comp) * (som[p] * sc[e]));
        }
    }
}

// c7 as a row histogram: sum_pix omega * value(pix, e) = sum_r Hist[r] * uPsf[r][e]
// with Hist[r] = sum over pixels in the radius of omega * (interpolation weight
// on row r).  Each block accumulates one chunk of pixels of one in-FOV source
// into a shared FP64 histogram; k_correction_hist folds the chunks.
__global__ void __launch_bounds__(256) k_map_integral_hist(const double* corners, const double* centers,
                                                           const double* omega, const SrcInfo* info,
                                                           int H, int W, int nch, double* hist_out) {
    __shared__ double hist[ND];
    int s = blockIdx.y, ch = blockIdx.x;
    SrcInfo si = info[s];
    double* out = hist_out + ((size_t)s * nch + ch) * ND;
    if (!si.in_fov) {
        for (int r = threadIdx.x; r < ND; r += blockDim.x) out[r] = 0.;
        return;
    }
    for (int r = threadIdx.x; r < ND; r += blockDim.x) hist[r] = 0.;
    __syncthreads();
    // chord^2 of the radius; pixels within a relative 1e-12 of it take the
    // reference's own test 2 asin(|d|/2) <= radius
    double ch2 = 2.0 * sin(0.5 * si.radius_rad);
    ch2 *= ch2;
    int npix = H * W, W1 = W + 1;
    for (int pix = ch * blockDim.x + threadIdx.x; pix < npix; pix += nch * blockDim.x) {
        int h = pix / W, w = pix - h * W;
        const double* c = centers + 3 * (h * W1 + w);
        double x = si.dir[0] - c[0], y = si.dir[1] - c[1], z = si.dir[2] - c[2];
        double d2 = x * x + y * y + z * z;
        bool inside;
        if (d2 < ch2 * (1.0 - 1e-12)) inside = true;
        else if (d2 > ch2 * (1.0 + 1e-12)) inside = false;
        else inside = dir_diff(si.dir, c) <= si.radius_rad;
        if (!inside) continue;
        int keys[NPTS]; double va[NPTS], vb[NPTS];
        int n = pixel_columns(corners, W1, h, w, si.dir, keys, va, vb);
        double om = omega[pix];
        for (int k = 0; k < n; ++k) {
            atomicAdd(&hist[keys[k] - 1], va[k] * om);
            atomicAdd(&hist[keys[k]], vb[k] * om);
        }
    }
    __syncthreads();
    for (int r = threadIdx.x; r < ND; r += blockDim.x) out[r] = hist[r];
}

// c9 map_correction_factor (model_map.map_correction_factor.cxx:3-53): the PSF
// integral out to the boundary radius over the whole bin at the radius's lower
// index (fast_separation_lower_index, psf.fast_separation_lower_index.cxx:5-22,
// with its `v < 1.` rule), capped at 1, times 1/map integral; 1 out of FOV.
__device__ double containment(const SrcInfo& si, const double* U, const double* partial_s, int E, int e) {
    const double v0 = si.radius_deg;
    const int li = v0 < 1. ? 1 : (int)floor(1. + log(1e4 * v0) * RECIPSTEP);
    const int d = li >= ND - 2 ? ND - 2 : li;
    const double xstep = log(70. / 1e-4) / (400 - 1.);
    const double t1 = (d == 0 ? 0. : 1e-4 * exp((d - 1) * xstep)) * D2R;
    const double t2 = (1e-4 * exp(d * xstep)) * D2R;
    const double y1 = TWOPI * U[(size_t)d * E + e] * sin(t1);
    const double y2 = TWOPI * U[(size_t)(d + 1) * E + e] * sin(t2);
    const double m = (y2 - y1) / (t2 - t1);
    const double b = y1 - t1 * m;
    const double v = 0.5 * m * (t2 * t2 - t1 * t1) + b * (t2 - t1);
    const double integ = v + partial_s[(size_t)d * E + e];
    return integ > 1.0 ? 1.0 : integ;
}

__device__ double correction_factor(const SrcInfo& si, const double* U, const double* partial_s, int E, int e,
                                    double inv) {
    return si.in_fov ? containment(si, U, partial_s, E, e) * inv : 1.0;
}

// c7 (1/sum) + c9 (containment factor) + c8/c10 folded into one per-(s,e) scale.
// Block (s, group of 8 energies): fold the source's chunk histograms, then one
// warp per energy.  With lut given, the block also writes its 8 energies of the
// source's scaled FP32 table lut[s][r][e] = uPsf * scale (energies E..Epad-1 zero).
__global__ void __launch_bounds__(256) k_correction_hist(const double* hist_in, int nch, const SrcInfo* info,
                                                         const double* upsf, const double* partial,
                                                         const double* expo, int E, double* scale,
                                                         double* inv_out, double* fac_out,
                                                         double* rad_out, int* fov_out, float* lut, int Epad) {
    __shared__ double hsum[ND];
    __shared__ double ssc[8];
    int s = blockIdx.x;
    SrcInfo si = info[s];
    for (int r = threadIdx.x; r < ND; r += blockDim.x) {
        double v = 0.;
#pragma unroll 4
        for (int c = 0; c < nch; ++c) v += hist_in[((size_t)s * nch + c) * ND + r];  // loads in flight, sum in c order
        hsum[r] = v;
    }
    __syncthreads();
    const double* U = upsf + (size_t)s * ND * E;
    // one warp per energy (8 energies per block): lanes split the rows, then a
    // fixed shuffle order
    const int lane = threadIdx.x & 31, wq = threadIdx.x >> 5;
    const int e = blockIdx.y * 8 + wq;
    if (e < E) {
        int i = s * E + e;
        // the containment integral does not depend on the map integral: formed
        // first, so its transcendental chain overlaps the dot product's loads
        const double integ = si.in_fov ? containment(si, U, partial + (size_t)s * ND * E, E, e) : 1.0;
        double sum = 0.;
        if (si.in_fov) {
#pragma unroll 13
            for (int r = lane; r < ND; r += 32) sum = fma(hsum[r], U[(size_t)r * E + e], sum);
            for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
        }
        if (lane == 0) {
            const double inv = sum != 0. ? 1.0 / sum : sum;
            const double factor = si.in_fov ? integ * inv : 1.0;
            scale[i] = expo[i] * factor;
            ssc[wq] = scale[i];
            if (inv_out) inv_out[i] = inv;
            if (fac_out) fac_out[i] = factor;
            if (e == 0) {
                if (rad_out) rad_out[s] = si.radius_deg;
                if (fov_out) fov_out[s] = si.in_fov;
            }
        }
    }
    if (!lut) return;
    __syncthreads();
    const int e0 = blockIdx.y * 8, ne = min(8, Epad - e0);
    for (int k = threadIdx.x; k < ND * ne; k += blockDim.x) {
        const int r = k / ne, j = k - r * ne, ee = e0 + j;
        lut[((size_t)s * ND + r) * Epad + ee] = ee < E ? (float)(U[(size_t)r * E + ee] * ssc[j]) : 0.f;
    }
}

int launch_correction(const double* hist, int nch, const SrcInfo* info, int S, const double* upsf,
                      const double* partial, const double* exposure, int E, double* scale,
                      double* inv_integ, double* correction, double* radius, int* in_fov,
                      cudaStream_t st, float* lut, int Epad) {
    const int ny = ((lut && Epad > E ? Epad : E) + 7) / 8;
    XTS_LAUNCH("k_correction", st, k_correction_hist<<<dim3(S, ny), 256, 0, st>>>(hist, nch, info, upsf, partial, exposure, E,
                                                                        scale, inv_integ, correction, radius, in_fov,
                                                                        lut, Epad));
    return XTS_OK;
}

// c7 + c9 for the adaptive map, whose per-block FP64 sums over the pixels inside
// the boundary radius [S][nch][E] are folded in a fixed order.
__global__ void __launch_bounds__(256) k_correction_sums(const double* sums, int nch, const SrcInfo* info,
                                                         const double* upsf, const double* partial,
                                                         const double* expo, int E, double* scale,
                                                         double* inv_out, double* fac_out,
                                                         double* rad_out, int* fov_out) {
    const int s = blockIdx.x;
    const SrcInfo si = info[s];
    const double* U = upsf + (size_t)s * ND * E;
    for (int e = threadIdx.x; e < E; e += blockDim.x) {
        const int i = s * E + e;
        double sum = 0.;
        if (si.in_fov)
            for (int c = 0; c < nch; ++c) sum += sums[((size_t)s * nch + c) * E + e];
        const double inv = sum != 0. ? 1.0 / sum : sum;
        const double factor = correction_factor(si, U, partial + (size_t)s * ND * E, E, e, inv);
        scale[i] = expo[i] * factor;
        if (inv_out) inv_out[i] = inv;
        if (fac_out) fac_out[i] = factor;
        if (e == 0) {
            if (rad_out) rad_out[s] = si.radius_deg;
            if (fov_out) fov_out[s] = si.in_fov;
        }
    }
}

// The model map with adaptive cubature: pixel means * solid angle, map integral
// sums, correction, then one scaling pass over the map.
static int launch_srcmap_adaptive(const SrcmapDev& a, const double* corners, const double* centers,
                                  const double* omega, const SrcInfo* info, double* scale, int nch,
                                  cudaStream_t st) {
    const int H = (int)a.wcs.naxis1, W = (int)a.wcs.naxis2, S = a.S, E = a.E;
    const int npix = H * W;
    double* sums = (double*)workspace(W_PARTSUM, sizeof(double) * (size_t)S * nch * E + 8);
    double* mean64 = (double*)workspace(W_ADAPT_MEAN, sizeof(double) * (size_t)S * npix * E + 8);
    int* status = (int*)workspace(W_MISC, 64);
    if (!sums || !mean64 || !status) return XTS_ERR_OOM;
    XTS_CUDA(cudaMemsetAsync(status, 0, sizeof(int), st));
    int rc = launch_adaptive_map(corners, centers, omega, info, a.upsf, S, H, W, E, a.rtol, a.max_depth, nch,
                                 sums, mean64, status, st);
    if (rc) return rc;
    // c7 from the FP64 means, c9, then the scalings into the FP32 map
    if ((rc = launch_mean_integral64(centers, omega, info, mean64, S, H, W, E, nch, sums, st))) return rc;
    XTS_LAUNCH("k_correction", st, k_correction_sums<<<S, 128, 0, st>>>(sums, nch, info, a.upsf, a.partial,
                                                                        a.exposure, E, scale, a.inv_integ,
                                                                        a.correction, a.radius, a.in_fov));
    return launch_scale_map64(mean64, (float*)a.out, omega, scale, S, npix, E, st);
}

// A map of pixel means [S][H*W][E] (a.out, FP32) -> the model map: the map
// integral sums over the pixels inside the boundary radius, the correction, and
// value = mean * solid angle * exposure * correction.
int finish_mean_map_range(const SrcmapDev& a, int s0, int ns, const double* centers, const double* omega,
                          const SrcInfo* info, double* scale, cudaStream_t st) {
    const int H = (int)a.wcs.naxis1, W = (int)a.wcs.naxis2, E = a.E;
    if (ns <= 0) return XTS_OK;
    const size_t npix = (size_t)H * W, oE = (size_t)s0 * E, oT = (size_t)s0 * ND * E;
    const int nc = mean_integral_chunks(ns, (int)npix);
    double* sums = (double*)workspace(W_PARTSUM, sizeof(double) * (size_t)ns * nc * E + 8);
    if (!sums) return XTS_ERR_OOM;
    float* out = (float*)a.out + (size_t)s0 * npix * E;
    int rc = launch_mean_integral(centers, omega, info + s0, out, ns, H, W, E, nc, sums, st);
    if (rc) return rc;
    XTS_LAUNCH("k_correction", st, k_correction_sums<<<ns, 128, 0, st>>>(
                                       sums, nc, info + s0, a.upsf + oT, a.partial + oT, a.exposure + oE, E, scale + oE,
                                       a.inv_integ ? a.inv_integ + oE : nullptr, a.correction ? a.correction + oE : nullptr,
                                       a.radius ? a.radius + s0 : nullptr, a.in_fov ? a.in_fov + s0 : nullptr));
    return launch_scale_map(out, omega, scale + oE, ns, (int)npix, E, st);
}

int finish_mean_map(const SrcmapDev& a, const double* centers, const double* omega, const SrcInfo* info,
                    double* scale, int nch, cudaStream_t st) {
    (void)nch;
    return finish_mean_map_range(a, 0, a.S, centers, omega, info, scale, st);
}

int srcmap_status(cudaStream_t st) {
    int* status = (int*)workspace(W_MISC, 64);
    if (!status) return XTS_ERR_OOM;
    int v = 0;
    XTS_CUDA(cudaMemcpyAsync(&v, status, sizeof(int), cudaMemcpyDeviceToHost, st));
    XTS_CUDA(cudaStreamSynchronize(st));
    if (v) {
        cudaMemsetAsync(status, 0, sizeof(int), st);
        return set_error(XTS_ERR_TIMEOUT, "a bounded device-side wait gave up (tensor-memory or TMA pipeline)");
    }
    return XTS_OK;
}

int launch_srcmap(const SrcmapDev& a, cudaStream_t st) {
    // map geometry on the geometry stream when one is given; it joins the launching
    // stream before uPsf is read, and on every early return
    StreamJoin geo(a.geo_stream && a.join_ev ? a.geo_stream : st, st, a.join_ev);
    cudaStream_t gs = geo.from;
    int rc = upload_rule(st);
    if (rc) return rc;
    int H = (int)a.wcs.naxis1, W = (int)a.wcs.naxis2, S = a.S, E = a.E;
    WcsDev w = make_wcs(a.wcs);
    size_t ng = (size_t)(H + 1) * (W + 1);
    int npix = H * W;
    int ntiles = (npix + TP - 1) / TP;
    int Epad = (E + 3) & ~3;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    int nch = S > 0 ? (4 * nsm + S - 1) / S : 1;
    int maxch = (npix + 255) / 256;
    nch = nch < 1 ? 1 : (nch > maxch ? maxch : nch);
    double* corners = (double*)workspace(W_CORNERS, sizeof(double) * 3 * ng);
    double* centers = (double*)workspace(W_CENTERS, sizeof(double) * 3 * ng);
    double* omega = (double*)workspace(W_OMEGA, sizeof(double) * npix);
    SrcInfo* info = (SrcInfo*)workspace(W_SRCINFO, sizeof(SrcInfo) * (S > 0 ? S : 1));
    double* hist = (double*)workspace(W_PARTSUM, sizeof(double) * (size_t)S * nch * ND + 8);
    double* scale = (double*)workspace(W_SCALE, sizeof(double) * (size_t)S * E + 8);
    if (!corners || !centers || !omega || !info || !hist || !scale) return XTS_ERR_OOM;
    const dim3 gg((unsigned)((W + GT) / GT), (unsigned)((H + GT) / GT));  // tiles over the (H+1) x (W+1) grid
    XTS_LAUNCH("k_map_geometry", gs, k_map_geometry<<<gg, GEO_THREADS, 0, gs>>>(w, H, W, corners, centers, omega));
    if (S == 0) return XTS_OK;
    XTS_LAUNCH("k_boundary", gs, k_boundary_chord<<<S, 256, 0, gs>>>(w, a.src_sph, H, W, corners, info, a.cut));
    if (a.cut) {
        if ((rc = geo.join())) return rc;
        if (a.out_f64 || !srcmap_win_supported(E))
            return set_error(XTS_ERR_ARG, "cutout maps: FP32 maps with E <= %d only", 52);
        int* status = (int*)workspace(W_MISC, 64);
        if (!status) return XTS_ERR_OOM;
        XTS_CUDA(cudaMemsetAsync(status, 0, sizeof(int), st));
        return launch_srcmap_win_cut(corners, centers, omega, info, a.cut, S, H, W, E, a.upsf, a.partial,
                                     a.exposure, scale, a.inv_integ, a.correction, a.radius, a.in_fov, status,
                                     (float*)a.out, st);
    }
    if (a.means_given) {
        if ((rc = geo.join())) return rc;
        if (a.out_f64 || !srcmap_adaptive_supported(E))
            return set_error(XTS_ERR_ARG, "scale_model_map: FP32 maps with E <= 256 only");
        return finish_mean_map(a, centers, omega, info, scale, nch, st);
    }
    if (a.surrogate) {
        if ((rc = geo.join())) return rc;
        if (a.out_f64 || !srcmap_adaptive_supported(E))
            return set_error(XTS_ERR_ARG, "surrogate map: FP32 maps with E <= 256 only");
        return launch_srcmap_surrogate(a, corners, centers, omega, info, scale, nch, st);
    }
    if (a.adaptive) {
        if ((rc = geo.join())) return rc;
        if (a.out_f64 || !srcmap_adaptive_supported(E))
            return set_error(XTS_ERR_ARG, "adaptive cubature: FP32 maps with E <= 256 only");
        return launch_srcmap_adaptive(a, corners, centers, omega, info, scale, nch, st);
    }
    if (!a.out_f64 && a.kernel == SRCMAP_WINDOWS && srcmap_win_supported(E)) {
        int* status = (int*)workspace(W_MISC, 64);
        if (!status) return XTS_ERR_OOM;
        XTS_CUDA(cudaMemsetAsync(status, 0, sizeof(int), st));
        return launch_srcmap_win(corners, centers, omega, info, S, H, W, E, a.upsf, a.partial,
                                 a.exposure, scale, a.inv_integ, a.correction, a.radius, a.in_fov, status,
                                 (float*)a.out, a.chunk_sources, a.on_chunk, a.on_chunk_ctx, geo, st);
    }
    if ((rc = geo.join())) return rc;
    if (a.out_f64) {  // the reference's own per-point FP64 arithmetic throughout
        XTS_LAUNCH("k_map_integral_f64", st, k_map_integral_hist<<<dim3(nch, S), 256, 0, st>>>(corners, centers, omega, info, H, W, nch, hist));
    } else {
        rc = launch_map_integral_fast(corners, centers, omega, info, S, H, W, nch, hist, st);
        if (rc) return rc;
    }
    rc = launch_correction(hist, nch, info, S, a.upsf, a.partial, a.exposure, E, scale, a.inv_integ,
                           a.correction, a.radius, a.in_fov, st);
    if (rc) return rc;
    if (a.out_f64) {
        XTS_LAUNCH("k_srcmap_f64", st, k_srcmap<true><<<dim3(ntiles, S), TP, 0, st>>>(corners, omega, info, nullptr, a.upsf, scale,
                                                                                        H, W, E, Epad, a.out));
        return XTS_OK;
    }
    if (a.kernel == SRCMAP_TCGEN05 && E <= 128) {
        int* status = (int*)workspace(W_MISC, 64);
        if (!status) return XTS_ERR_OOM;
        XTS_CUDA(cudaMemsetAsync(status, 0, sizeof(int), st));
        rc = launch_srcmap_tc(corners, omega, info, a.upsf, scale, S, H, W, E, (float*)a.out, status, st);
        if (rc) return rc;
        return XTS_OK;
    }
    return launch_srcmap_fast(corners, omega, info, a.upsf, scale, S, H, W, E, (float*)a.out, st);
}

}  // namespace xts
