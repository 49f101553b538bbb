// xts_srcmap_win.cu -- the FP32 source-map path in two passes over the pixels.
//
// Pass A, k_pixel_windows (geometry, once per pixel and source): the 12 rule
// points of the pixel give LUT rows and interpolation weights (xts_point.cuh);
// their weights times the pixel's solid angle are summed into a dense window of
// at most RW consecutive table rows.  For pixels inside the boundary radius of
// an in-FOV source the window also enters the block's FP64 row histogram, whose
// dot product with uPsf is the map integral of c7 (model_map.map_integral.cxx:4-48):
//     sum_pix omega * value(pix, e) = sum_r Hist[r] * uPsf[r][e].
// The rule points' squared chords are FP32 offsets from the pixel centre's FP64
// squared chord (the biquadratic form of xts_point.cuh), compared with the
// window's row edges, also as FP32 offsets from the centre: one FP64 table
// search per pixel, none per point.  The histogram takes each window row of a
// pixel inside the radius by one FP64 shared-memory atomic add.  Every pixel's
// window is written once as a 16-byte record (3 FP32 weights and the first row /
// row count), with the 8 weights of a window longer than 3 rows in a 32-byte
// extension.  Pixels whose points leave the 8-row window (those next to the
// source) are "wide": they get a sparse record of their 24 (row, weight) pairs
// from a shared pool instead, or, if the pool is full, are evaluated point by
// point in pass B.
//
// Pass B, k_srcmap_win (the write pass, d1 + d2 + c8 + c10): the source's scaled
// table Y' = uPsf * exposure * correction (FP32, [401][EQ] float4, EQ odd so
// different rows fall in different shared-memory bank groups) is brought into
// shared memory by one TMA bulk copy; each thread reads its pixel's window
// record and forms value[e] = sum_j W[j] * Y'[row_j][e] for all energies in
// registers (rows rbase + j, or the 24 rows of a sparse record).  Values are
// staged and written by one TMA bulk store per tile, so the pass streams the
// window records in and the map out; the next tile's records are loaded while
// the current one is computed.
#include "xts_point.cuh"

namespace xts {

// ============================================================================ pass A
constexpr int WT = 256;  // pixels per tile == threads per block
constexpr int NSG = 4;   // sources per group: one pixel's source-independent geometry serves NSG sources

constexpr size_t WA_OFF_BINS = 0;
constexpr size_t WA_OFF_COEF = sizeof(SepBin) * NSB;
constexpr size_t WA_OFF_HIST = WA_OFF_COEF + sizeof(float4) * 2 * ND;
constexpr size_t WA_OFF_WTS = WA_OFF_HIST + (8 * NSG * ND + 15) / 16 * 16;
constexpr size_t WA_OFF_SRC = WA_OFF_WTS + sizeof(float) * WT * RW;
constexpr size_t WA_SMEM = WA_OFF_SRC + sizeof(SrcInfo) * NSG;

constexpr int NSP = 24;  // entries of a sparse record: 12 points x 2 rows
constexpr int META_OVERFLOW = -0x7fffffff - 1;  // wide pixel without a sparse record
constexpr int REC_ROWS = 3;  // window rows held by the 16-byte main record
constexpr float EMSTEP = (float)(REDM1 / (REDM1 + 1.0));  // e^-step: t in row k + 1 = (t in row k - 1) e^-step

// Per (source, pixel) the main record rec = {w0, w1, w2, meta}: meta >= 0 is the
// window's first row (bits 0-15) and row count (bits 16-23), with the weights of
// windows longer than REC_ROWS rows in ext (two float4, w0..w7); meta < 0 marks a
// wide pixel (sparse record -1 - meta, or META_OVERFLOW).
struct PassA {
    const SepBin* sbin;    // shared: row bins
    const float4* scoef;   // shared: per-row records
    double* hist;          // shared: the block's map-integral rows ([NSG][ND] in the dense pass)
    float* wts;            // shared: [RW][WT] windows
    float4* rec;
    float4* ext;
    float2* sparse;
    int sparse_cap;
    int* sparse_count;
};

// Shared tables of pass A, loaded by every block (the histogram is zeroed by the caller).
__device__ __forceinline__ PassA pass_a_tables(unsigned char* smem, const SepTab* septab, float4* rec, float4* ext,
                                               float2* sparse, int sparse_cap, int* sparse_count) {
    PassA A;
    A.sbin = (const SepBin*)(smem + WA_OFF_BINS);
    A.scoef = (const float4*)(smem + WA_OFF_COEF);
    A.hist = (double*)(smem + WA_OFF_HIST);
    A.wts = (float*)(smem + WA_OFF_WTS);
    A.rec = rec; A.ext = ext; A.sparse = sparse; A.sparse_cap = sparse_cap; A.sparse_count = sparse_count;
    SepBin* sb = (SepBin*)(smem + WA_OFF_BINS);
    float4* sc = (float4*)(smem + WA_OFF_COEF);
    for (int k = threadIdx.x; k < NSB; k += WT) sb[k] = septab->bins[k];
    for (int k = threadIdx.x; k < 2 * ND; k += WT) sc[k] = ((const float4*)septab->coef)[k];
    return A;
}

// Source-independent geometry of one pixel: its rule points are the bilinear
// blend P(u, v) = M + B u + C v + D uv of the corners, so relative to a source s
// with A = M - s the squared chord is q(u, v) = |A + B u + C v + D uv|^2, whose
// coefficients split into source-dependent ones (|A|^2, 2 A.B, 2 A.C, 2 A.D) and
// the rest (|B|^2, |C|^2, 2 B.C, 2 B.D, 2 C.D, |D|^2).  The latter enter each
// mirror pair's chord offset through eb (even part) and ob (odd part), formed once
// per pixel for a group of sources.
struct PixBase {
    double m[3];      // M, the corners' average (FP64)
    double c[3];      // pixel centre (boundary-radius test)
    float b2[3], c2[3], d2[3];  // 2B, 2C, 2D
    float bc2;        // 2 B.C
    float eb[6], ob[6];
    float om;         // solid angle
};

__device__ __forceinline__ PixBase pixel_base(const double* __restrict__ corners, const double* __restrict__ centers,
                                              const double* __restrict__ omega, int W1, int h, int w, size_t om_idx) {
    const double* a = corners + 3 * (h * W1 + w);            // LL
    const double* b = corners + 3 * (h * W1 + w + 1);        // LR
    const double* c = corners + 3 * ((h + 1) * W1 + w + 1);  // UR
    const double* d = corners + 3 * ((h + 1) * W1 + w);      // UL
    PixBase P;
    double B[3], C[3], D[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        P.m[i] = 0.25 * ((a[i] + b[i]) + (c[i] + d[i]));
        B[i] = 0.25 * ((b[i] + c[i]) - (a[i] + d[i]));
        C[i] = 0.25 * ((c[i] + d[i]) - (a[i] + b[i]));
        D[i] = 0.25 * ((a[i] + c[i]) - (b[i] + d[i]));
        P.b2[i] = (float)(2.0 * B[i]);
        P.c2[i] = (float)(2.0 * C[i]);
        P.d2[i] = (float)(2.0 * D[i]);
    }
    const double* pc = centers + 3 * ((size_t)h * W1 + w);
    P.c[0] = pc[0]; P.c[1] = pc[1]; P.c[2] = pc[2];
    const float q4 = (float)fma(B[0], B[0], fma(B[1], B[1], B[2] * B[2]));
    const float q5 = (float)fma(C[0], C[0], fma(C[1], C[1], C[2] * C[2]));
    const float q6 = (float)(2.0 * fma(B[0], D[0], fma(B[1], D[1], B[2] * D[2])));
    const float q7 = (float)(2.0 * fma(C[0], D[0], fma(C[1], D[1], C[2] * D[2])));
    const float q8 = (float)fma(D[0], D[0], fma(D[1], D[1], D[2] * D[2]));
    P.bc2 = (float)(2.0 * fma(B[0], C[0], fma(B[1], C[1], B[2] * C[2])));
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        P.eb[k] = fmaf(q8, c_pair[k][7], fmaf(q5, c_pair[k][4], q4 * c_pair[k][3]));
        P.ob[k] = fmaf(q7, c_pair[k][6], q6 * c_pair[k][5]);
    }
    P.om = omega ? (float)omega[om_idx] : 1.f;  // omega NULL: the pixel means (unit solid angle)
    return P;
}

// Lower table row of the squared chord q: one bin load and one FP64 compare.
__device__ __forceinline__ int row_lower(double q, const SepBin* bins) {
    int b = (__double2hiint(q) >> (20 - SB_BITS)) - (SB_EXP0 << SB_BITS);
    b = min(max(b, 0), NSB - 1);
    const SepBin sb = bins[b];
    return sb.k0 + (q >= sb.thr);
}

// One (source, pixel): the pixel's window for source si, record index kk.  Pixels
// whose centre lies within the boundary radius (squared chord ch2) add their window
// rows to hist (the source's map-integral rows); the rows they touch widen
// [*rlo, *rhi] when those are given.  (h, w) and W1 locate the pixel's corners for
// the rare wide pixel, which is redone in FP64 point by point.
__device__ __forceinline__ void window_source(const PixBase& P, const SrcInfo& si, double ch2,
                                              const double* __restrict__ corners, int W1, int h, int w,
                                              size_t kk, const PassA& A, double* hist, int* rlo, int* rhi) {
    const int t = threadIdx.x;
    const double Ax = P.m[0] - si.dir[0], Ay = P.m[1] - si.dir[1], Az = P.m[2] - si.dir[2];
    const double a0 = fma(Ax, Ax, fma(Ay, Ay, Az * Az));  // q at the centre of the blend
    bool inside = false;
    if (si.in_fov) {
        const double x = si.dir[0] - P.c[0], y = si.dir[1] - P.c[1], z = si.dir[2] - P.c[2];
        const double d2 = x * x + y * y + z * z;
        if (d2 < ch2 * (1.0 - 1e-12)) inside = true;
        else if (d2 > ch2 * (1.0 + 1e-12)) inside = false;
        else inside = dir_diff(si.dir, P.c) <= si.radius_rad;
    }
    // q(point) - a0 in FP32: 2 A.B u + 2 A.C v + (2 A.D + 2 B.C) uv + the pixel's part
    const float ax = (float)Ax, ay = (float)Ay, az = (float)Az;
    const float f1 = fmaf(ax, P.b2[0], fmaf(ay, P.b2[1], az * P.b2[2]));
    const float f2 = fmaf(ax, P.c2[0], fmaf(ay, P.c2[1], az * P.c2[2]));
    const float f3 = fmaf(ax, P.d2[0], fmaf(ay, P.d2[1], fmaf(az, P.d2[2], P.bc2)));
    float dqs[12];
    float mn = INFINITY, mx = -INFINITY;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const float E = fmaf(f3, c_pair[k][2], P.eb[k]);
        const float O = fmaf(f2, c_pair[k][1], fmaf(f1, c_pair[k][0], P.ob[k]));
        dqs[k] = E + O;
        dqs[k + 6] = E - O;
        mn = fminf(mn, fminf(dqs[k], dqs[k + 6]));
        mx = fmaxf(mx, fmaxf(dqs[k], dqs[k + 6]));
    }
    const float om = P.om;
    auto edge = [&](int k) {  // q[k] - a0 in FP32
        const float4 cw = A.scoef[2 * k + 1];
        return (float)(__hiloint2double(__float_as_int(cw.w), __float_as_int(cw.z)) - a0);
    };
    // Most pixels' points lie in the centre's table row, or in it and one
    // neighbour.  Then one row's polynomial (fitted over two rows) gives every
    // point's t relative to the lower row kl, u = t - 1; a point past the upper
    // edge eb has t' = u e^-step in row kl + 1.  With T = sum w u over all points
    // and S2 = sum w u over those past eb, the three row weights are
    //     s0 = om (S2 - T),  s2 = om e^-step S2,  s1 = om sum(w) - s0 - s2.
    const int kc = row_lower(a0, A.sbin);  // the centre's lower table row
    if (kc >= 2 && kc <= ND - 4) {
        const float em1 = edge(kc - 1), e0 = edge(kc), e1 = edge(kc + 1), e2 = edge(kc + 2);
        // rows kc (and kc + 1), or kc - 1 and kc; eb = +inf for one row.  The case is
        // made opaque to the compiler: specialising the point loop per case would run
        // up to three copies of it per warp, each with a part of the lanes.
        const bool up = mn >= e0 && mx < e2, dn = mn >= em1 && mx < e1;
        int kl = up ? kc : (dn ? kc - 1 : -1);
        float eb = (mn >= e0 && mx < e1) ? INFINITY : (up ? e1 : e0);
        float eL = up ? e0 : em1;
        asm volatile("" : "+r"(kl), "+f"(eb), "+f"(eL));
        if (kl >= 0) {  // (warp-divergent: a warp's pixels usually agree)
            const float4 c0 = A.scoef[2 * kl], c1 = A.scoef[2 * kl + 1];
            // zz = (dl - C)/H and REDM1 dl, dl = q / q_kl - 1 = (dq - eL) / q_kl, as FMAs in dq
            const float kz = c0.x * (1.f / DPOLY_H), z0 = fmaf(-eL, kz, -DPOLY_C / DPOLY_H);
            const float kr = c0.x * (float)REDM1, r0 = -eL * kr;
            float T = 0.f, S2 = 0.f;
#pragma unroll
            for (int p = 0; p < 12; ++p) {
                const float dq = dqs[p];
                const float zz = fmaf(dq, kz, z0);
                const float P4 = fmaf(fmaf(fmaf(fmaf(c1.y, zz, c1.x), zz, c0.w), zz, c0.z), zz, c0.y);
                const float u = fmaf(fmaf(dq, kr, r0), P4, -1.f);
                const float wp = c_rule_w32[p];
                T = fmaf(wp, u, T);
                S2 = fmaf(dq >= eb ? wp : 0.f, u, S2);
            }
            const float s0 = om * (S2 - T), s2 = om * (EMSTEP * S2);
            const float s1 = fmaf(om, c_rule_wsum, -s0) - s2;
            const bool two = eb != INFINITY;
            const int nent = two ? 3 : 2;
            if (inside) {
                atomicAdd(&hist[kl], (double)s0);
                atomicAdd(&hist[kl + 1], (double)s1);
                if (two) atomicAdd(&hist[kl + 2], (double)s2);
                if (rlo) {
                    atomicMin(rlo, kl);
                    atomicMax(rhi, kl + nent - 1);
                }
            }
            A.rec[kk] = make_float4(s0, s1, s2, __int_as_float(kl | (nent << 16)));
            return;
        }
    }
    // General path: the window of RW rows around the centre's row, the row edges
    // as FP32 offsets from a0.
    const int base = min(max(kc - RW / 2, 0), ND - RW);
    float d[RW];
#pragma unroll
    for (int j = 0; j < RW; ++j) d[j] = edge(base + j);
    float* wd = A.wts + t;  // slot j at wd[j * WT]: lanes hit consecutive words
#pragma unroll
    for (int j = 0; j < RW; ++j) wd[j * WT] = 0.f;
    bool wide = false;
    int lo = RW, hi = -1;
#pragma unroll
    for (int p = 0; p < 12; ++p) {
        const float dq = dqs[p];
        int r = 0;
        float dlo = d[0];
#pragma unroll
        for (int j = 1; j < RW; ++j) {
            const bool ge = dq >= d[j];
            r += ge;
            dlo = ge ? d[j] : dlo;
        }
        const int k = base + r;  // the point's lower table row
        const float wo = c_rule_w32[p] * om;
        if (dq >= d[0] && r < RW - 1 && k >= 1) {
            const float4 c0 = A.scoef[2 * k], c1 = A.scoef[2 * k + 1];
            const float dl = (dq - dlo) * c0.x;  // q / q_k - 1
            float tt;
            if (dl >= -0.002f && dl <= 0.072f) {
                const float zz = fmaf(dl, 1.f / DPOLY_H, -DPOLY_C / DPOLY_H);
                const float P4 = fmaf(fmaf(fmaf(fmaf(c1.y, zz, c1.x), zz, c0.w), zz, c0.z), zz, c0.y);
                tt = (float)REDM1 * (dl * P4);
            } else {
                tt = t_exact(a0 + (double)dq, k + 1);
            }
            wd[r * WT] += (1.f - tt) * wo;
            wd[(r + 1) * WT] += tt * wo;
            lo = min(lo, r);
            hi = max(hi, r + 1);
        } else {
            wide = true;
        }
    }
    if (!wide) {
        // map integral (c7): the window's rows of a pixel inside the radius
        if (inside) {
#pragma unroll
            for (int j = 0; j < RW; ++j)
                if (j >= lo && j <= hi) atomicAdd(&hist[base + j], (double)wd[j * WT]);
            if (rlo) {
                atomicMin(rlo, base + lo);
                atomicMax(rhi, base + hi);
            }
        }
        const int nent = hi - lo + 1;
        float f[RW];
#pragma unroll
        for (int j = 0; j < RW; ++j) f[j] = j < nent ? wd[min(j + lo, RW - 1) * WT] : 0.f;
        const int meta = (base + lo) | (nent << 16);
        A.rec[kk] = make_float4(f[0], f[1], f[2], __int_as_float(meta));
        if (nent > REC_ROWS) {
            A.ext[2 * kk] = make_float4(f[0], f[1], f[2], f[3]);
            A.ext[2 * kk + 1] = make_float4(f[4], f[5], f[6], f[7]);
        }
    } else {
        // a wide pixel (next to the source): its 12 points again with FP64 chords
        // from the corners, for its sparse record and its map-integral rows alike
        const PixQ g = pixel_q(pixel_geom(corners, W1, h, w, si));
        int meta = META_OVERFLOW;
        const int slot = atomicAdd(A.sparse_count, 1);
        float2* sr = slot < A.sparse_cap ? A.sparse + (size_t)slot * NSP : nullptr;
        for (int p = 0; p < 12; ++p) {
            float tt;
            const int idx = point_row_bin(point_q2(g, p), A.sbin, A.scoef, &tt);
            const float wo = c_rule_w32[p] * om;
            const float wa = (1.f - tt) * wo, wb = tt * wo;
            if (sr) {
                sr[2 * p] = make_float2(wa, __int_as_float(idx - 1));
                sr[2 * p + 1] = make_float2(wb, __int_as_float(idx));
            }
            if (inside) {
                atomicAdd(&hist[idx - 1], (double)wa);
                atomicAdd(&hist[idx], (double)wb);
                if (rlo) {
                    atomicMin(rlo, idx - 1);
                    atomicMax(rhi, idx);
                }
            }
        }
        if (sr) meta = -1 - slot;
        A.rec[kk] = make_float4(0.f, 0.f, 0.f, __int_as_float(meta));
    }
}

__device__ __forceinline__ double boundary_chord2(const SrcInfo& si) {
    const double c = 2.0 * sin(0.5 * si.radius_rad);
    return c * c;
}

// The dense map: block b takes item b = (g, p), part p of the P parts of group g (NSG
// sources; tiles [p nt / P, (p + 1) nt / P) of WT pixels), forms each pixel's
// source-independent geometry once and the windows of the group's sources from it,
// and adds the item's non-zero rows to hist_out[s] (cleared before the launch) with
// FP64 atomics.  Items are small (about 16 per resident block), so blocks retire
// steadily: the hardware balances them, and kernels of a higher-priority stream
// (exposure and PSF beside this pass) get their slots as they free up.
__global__ void __launch_bounds__(WT, 3) k_pixel_windows(const double* __restrict__ corners, const double* __restrict__ centers,
                                                      const double* __restrict__ omega, const SrcInfo* __restrict__ info,
                                                      const SepTab* __restrict__ septab, int S, int H, int W,
                                                      int P,
                                                      double* __restrict__ hist_out, float4* __restrict__ rec,
                                                      float4* __restrict__ ext, float2* __restrict__ sparse,
                                                      int sparse_cap, int* __restrict__ sparse_count) {
    extern __shared__ __align__(16) unsigned char smem[];
    const PassA A = pass_a_tables(smem, septab, rec, ext, sparse, sparse_cap, sparse_count);
    SrcInfo* ssrc = (SrcInfo*)(smem + WA_OFF_SRC);
    const int t = threadIdx.x;
    const int npix = H * W, W1 = W + 1;
    const int nt = (npix + WT - 1) / WT;
    const int item = blockIdx.x;
    const int g = item / P, p = item - g * P, s0 = g * NSG, ns = min(NSG, S - s0);
    if (t < ns) ssrc[t] = info[s0 + t];
    for (int r = t; r < NSG * ND; r += WT) A.hist[r] = 0.;
    __syncthreads();
    const int ta = (int)((long long)p * nt / P), tb = (int)((long long)(p + 1) * nt / P);
    for (int tile = ta; tile < tb; ++tile) {
        const int pix = tile * WT + t;
        if (pix >= npix) continue;
        const int h = pix / W, w = pix - h * W;
        const PixBase Q = pixel_base(corners, centers, omega, W1, h, w, (size_t)pix);
        for (int j = 0; j < ns; ++j) {
            const SrcInfo& si = ssrc[j];
            window_source(Q, si, boundary_chord2(si), corners, W1, h, w, (size_t)(s0 + j) * npix + pix, A,
                          A.hist + j * ND, nullptr, nullptr);
        }
    }
    __syncthreads();
    for (int r = t; r < ns * ND; r += WT) {
        const double v = A.hist[r];
        if (v != 0.) atomicAdd(hist_out + (size_t)s0 * ND + r, v);
    }
}

// Cutouts: one persistent launch over a work queue of (source, tile) items, tile
// = WT consecutive pixels of the source's window (row-major, nw wide).  A block
// takes the next item from the queue (one atomic), builds its pixels' records
// and the item's map-integral rows in shared memory, and adds the rows it touched
// to hist_out[s] with FP64 atomics.  item_src[i] is the source of item i, tile_off[s]
// its first item and tile_off[S] the number of items.
__global__ void __launch_bounds__(WT, 3) k_pixel_windows_cut(const double* __restrict__ corners,
                                                          const double* __restrict__ centers,
                                                          const double* __restrict__ omega,
                                                          const SrcInfo* __restrict__ info,
                                                          const xts_cutout* __restrict__ cut,
                                                          const int* __restrict__ item_src,
                                                          const long long* __restrict__ tile_off,
                                                          unsigned long long* __restrict__ queue,
                                                          const SepTab* __restrict__ septab, int S, int W,
                                                          double* __restrict__ hist_out, float4* __restrict__ rec,
                                                          float4* __restrict__ ext, float2* __restrict__ sparse,
                                                          int sparse_cap, int* __restrict__ sparse_count) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ long long item_s;
    __shared__ int rmin_s, rmax_s;
    const PassA A = pass_a_tables(smem, septab, rec, ext, sparse, sparse_cap, sparse_count);
    const int t = threadIdx.x, W1 = W + 1;
    for (int r = t; r < ND; r += WT) A.hist[r] = 0.;
    const long long n_items = tile_off[S];
    for (;;) {
        if (t == 0) {
            item_s = (long long)atomicAdd(queue, 1ull);
            rmin_s = ND;
            rmax_s = -1;
        }
        __syncthreads();  // also orders the previous item's flush before this item's adds
        const long long item = item_s;
        if (item >= n_items) break;
        const int s = item_src[item];
        const xts_cutout cw = cut[s];
        const SrcInfo si = info[s];
        const double ch2 = boundary_chord2(si);
        const long long npix = (long long)cw.nh * cw.nw;
        const long long pix = (item - tile_off[s]) * WT + t;
        if (pix < npix) {
            const int i = (int)(pix / cw.nw), j = (int)(pix - (long long)i * cw.nw);
            const int h = cw.h0 + i, w = cw.w0 + j;
            const PixBase P = pixel_base(corners, centers, omega, W1, h, w, (size_t)h * W + w);
            window_source(P, si, ch2, corners, W1, h, w, (size_t)(cw.offset + pix), A, A.hist, &rmin_s, &rmax_s);
        }
        __syncthreads();
        for (int r = rmin_s + t; r <= rmax_s; r += WT) {
            const double v = A.hist[r];
            if (v != 0.) atomicAdd(hist_out + (size_t)s * ND + r, v);
            A.hist[r] = 0.;
        }
        __syncthreads();  // the flush has read rmin_s / rmax_s before thread 0 resets them
    }
}

// ============================================================================ pass B
constexpr int BT = 256;  // pixels per tile == threads per block
constexpr int BQ = 13;   // float4 quads of a table row at most: E <= 52

// Table row stride in float4 units: ceil(E/4), made odd.
static int win_row_quads(int E) {
    int nq = (E + 3) / 4;
    return (nq & 1) ? nq : nq + 1;
}

struct WinLayout { size_t tab, stage, bar, total; };
static __host__ __device__ WinLayout win_layout(int E, int EQ) {
    WinLayout L;
    L.tab = 0;                                            // [ND + RW][EQ] float4 (RW zero guard rows)
    L.stage = (size_t)(ND + RW) * EQ * 16;                // per warp [32 * E + 8] floats
    L.bar = (L.stage + sizeof(float) * (size_t)(BT / 32) * (32 * E + 8) + 15) / 16 * 16;
    L.total = L.bar + 16;
    return L;
}

// One pixel's record as read by pass B: the main record, and for a window of more
// than REC_ROWS rows its extension.
struct PixRec { int meta; float4 wa, wb; };

__device__ __forceinline__ PixRec load_rec(const float4* rec, const float4* ext, size_t k, bool valid) {
    PixRec r;
    r.meta = 0;
    r.wa = make_float4(0.f, 0.f, 0.f, 0.f);
    r.wb = r.wa;
    if (valid) {
        const float4 m = __ldg(rec + k);
        r.meta = __float_as_int(m.w);
        r.wa = make_float4(m.x, m.y, m.z, 0.f);
        if (r.meta >= 0 && (r.meta >> 16) > REC_ROWS) {
            r.wa = __ldg(ext + 2 * k);
            r.wb = __ldg(ext + 2 * k + 1);
        }
    }
    return r;
}

// Warps run independently: each owns 32 pixels of the tile, a slice of the
// stage and its own TMA bulk store, so no block barrier is needed except when the
// block moves on to the next source's table.
// Pixels of a source in the write pass: the dense map (every source H * W pixels,
// records from s * npix, output from (s_base + s) * npix) or a cutout window
// (cut[s].nh * cut[s].nw pixels, records and output from cut[s].offset).
template <bool CUT>
struct SrcSpan {
    const xts_cutout* cut;
    int S, s_base, npix;
    __device__ __forceinline__ int pixels(int s) const {
        if (!CUT) return npix;
        return s < S ? cut[s].nh * cut[s].nw : 0;
    }
    __device__ __forceinline__ long long rec_base(int s) const { return CUT ? cut[s].offset : (long long)s * npix; }
    __device__ __forceinline__ long long out_base(int s) const {
        return CUT ? cut[s].offset : (long long)(s_base + s) * npix;
    }
    __device__ __forceinline__ int tiles(int s) const { return (pixels(s) + BT - 1) / BT; }
};

template <int NQ, bool CUT>
__global__ void __launch_bounds__(BT, 2)
k_srcmap_win(const float4* __restrict__ win, const float4* __restrict__ ext, const float2* __restrict__ sparse,
             const float* __restrict__ lut, const double* __restrict__ corners, const double* __restrict__ omega,
             const SrcInfo* __restrict__ info, const SepTab* __restrict__ septab, const xts_cutout* __restrict__ cut,
             const long long* __restrict__ tile_off,
             int S, int s_base, int H, int W, int E, int EQ, int* status, float* __restrict__ out) {
    extern __shared__ __align__(16) unsigned char smem[];
    const WinLayout L = win_layout(E, EQ);
    float4* tab = (float4*)(smem + L.tab);
    const unsigned bar = smem_u32(smem + L.bar);
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    float* stage = (float*)(smem + L.stage) + warp * (32 * E + 8);
    const int W1 = W + 1;
    const SrcSpan<CUT> sp_{cut, S, s_base, H * W};
    const long long T = CUT ? tile_off[S] : (long long)S * sp_.tiles(0);
    const long long f0 = T * blockIdx.x / gridDim.x, f1 = T * (blockIdx.x + 1) / gridDim.x;
    const unsigned tab_bytes = (unsigned)(ND * EQ * 16);

    for (int k = t; k < RW * EQ; k += BT) tab[ND * EQ + k] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (t == 0) mbar_init(bar, 1);
    __syncthreads();

    int cur = -1;
    unsigned phase = 0;
    // (source, tile) of f, advanced by counting: no 64-bit division per tile
    int s, tile;
    if (CUT) {  // the source whose items hold f0: the last s with tile_off[s] <= f0
        int a = 0, b = S;
        while (b - a > 1) {
            const int mid = (a + b) >> 1;
            if (tile_off[mid] <= f0) a = mid; else b = mid;
        }
        s = a;
        while (s < S && tile_off[s + 1] <= f0) ++s;  // skip sources without tiles
        tile = (int)(f0 - tile_off[s]);
    } else {
        s = (int)(f0 / sp_.tiles(0));
        tile = (int)(f0 - (long long)s * sp_.tiles(0));
    }
    int np_s = sp_.pixels(s), nt_s = sp_.tiles(s);
    const bool any = f0 < f1 && s < S;
    PixRec rec = load_rec(win, ext, any ? (size_t)(sp_.rec_base(s) + tile * BT + t) : 0, any && tile * BT + t < np_s);
    for (long long f = f0; f < f1; ++f) {
        int sn = s, tn = tile + 1;  // the next tile
        while (tn >= sp_.tiles(sn) && sn < S) { tn = 0; ++sn; }
        int s2 = sn, t2 = tn + 1;   // and the one after
        while (t2 >= sp_.tiles(s2) && s2 < S) { t2 = 0; ++s2; }
        const int px0 = tile * BT + warp * 32;  // this warp's first pixel
        const int npw = min(32, np_s - px0);                                // may be <= 0 in the last tile
        const long long g0 = (sp_.out_base(s) + px0) * E;                   // first flat output of the whole map
        const int m = (int)(g0 & 3);                                        // staging residue
        const int nflat = npw > 0 ? npw * E : 0;
        const int pix = px0 + lane;

        // the next tile's records, in flight while this tile is computed, and the
        // one after that on its way into L2
        PixRec nxt;
        {
            const int pn = tn * BT;
            const bool more = f + 1 < f1 && sn < S;
            nxt = load_rec(win, ext, more ? (size_t)(sp_.rec_base(sn) + pn + t) : 0,
                           more && pn + t < sp_.pixels(sn));
            const int p2 = t2 * BT;
            if (f + 2 < f1 && s2 < S && p2 + t < sp_.pixels(s2) && (t & 7) == 0) {  // one prefetch per 128-byte line
                const size_t k2 = (size_t)(sp_.rec_base(s2) + p2 + t);
                asm volatile("prefetch.global.L2 [%0];" :: "l"(win + k2));
            }
        }
        if (s != cur) {
            __syncthreads();  // every warp is done with the previous source's table
            if (t == 0) {
                fence_async_shared();
                bulk_load(tab, lut + (size_t)s * ND * EQ * 4, tab_bytes, bar);
            }
            cur = s;
            const bool ok = mbar_wait(bar, phase);
            phase ^= 1;
            if (!__syncthreads_and(ok)) {
                if (t == 0) {
                    atomicExch(status, 1);
                    mbar_wait(bar, phase ^ 1);  // bounded: let the copy land before the block exits
                }
                if (lane == 0) bulk_wait_all();
                return;
            }
        }
        // entries of this pixel: window rows rbase + j (j < nr), or a sparse record
        const int meta = rec.meta;
        const bool valid = lane < npw;
        const bool sp = valid && meta < 0 && meta != META_OVERFLOW;
        const bool slow = valid && meta == META_OVERFLOW;
        const int nent = sp ? NSP : (meta >= 0 ? (meta >> 16) : 0);
        const int rb = meta >= 0 ? (meta & 0xffff) : 0;
        const float2* se = sparse + (size_t)(sp ? -1 - meta : 0) * NSP;
        const int kmax = __reduce_max_sync(0xffffffffu, nent);
        const float w[RW] = {rec.wa.x, rec.wa.y, rec.wa.z, rec.wa.w, rec.wb.x, rec.wb.y, rec.wb.z, rec.wb.w};
        float4 acc[NQ];
#pragma unroll
        for (int q = 0; q < NQ; ++q) acc[q] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (kmax <= RW) {  // window records only (warp-uniform)
#pragma unroll
            for (int j = 0; j < RW; ++j) {
                if (j < kmax && j < nent) {  // rows past a pixel's own window carry weight 0: lanes
                    const float4* yr = tab + (rb + j) * EQ;  // past theirs issue no shared loads
                    const float wj = w[j];
#pragma unroll
                    for (int q = 0; q < NQ; ++q) {
                        const float4 y = yr[q];
                        acc[q].x = fmaf(wj, y.x, acc[q].x);
                        acc[q].y = fmaf(wj, y.y, acc[q].y);
                        acc[q].z = fmaf(wj, y.z, acc[q].z);
                        acc[q].w = fmaf(wj, y.w, acc[q].w);
                    }
                }
            }
        } else {  // some lanes hold sparse records (pixels next to the source)
#pragma unroll 1
            for (int j = 0; j < NSP; ++j) {
                float wj = 0.f;
                int row = rb;
#pragma unroll
                for (int i = 0; i < RW; ++i)
                    if (i == j) wj = w[i];
                if (j < RW) row = rb + j;
                if (sp) {
                    const float2 e = __ldg(se + j);
                    wj = e.x;
                    row = __float_as_int(e.y);
                }
                const float4* yr = tab + row * EQ;
#pragma unroll
                for (int q = 0; q < NQ; ++q) {
                    const float4 y = yr[q];
                    acc[q].x = fmaf(wj, y.x, acc[q].x);
                    acc[q].y = fmaf(wj, y.y, acc[q].y);
                    acc[q].z = fmaf(wj, y.z, acc[q].z);
                    acc[q].w = fmaf(wj, y.w, acc[q].w);
                }
            }
        }
        // the stage is reused only now: the previous bulk store's read-out overlapped the sums
        if (lane == 0) bulk_wait_read();
        __syncwarp();
        float* dst = stage + m + lane * E;
        if (valid && !slow) {
#pragma unroll
            for (int q = 0; q < NQ; ++q) {
                const int e = 4 * q;
                dst[e] = acc[q].x;
                if (q < NQ - 1 || e + 1 < E) dst[e + 1] = acc[q].y;
                if (q < NQ - 1 || e + 2 < E) dst[e + 2] = acc[q].z;
                if (q < NQ - 1 || e + 3 < E) dst[e + 3] = acc[q].w;
            }
        }
        if (slow) {  // sparse pool full: point by point from the shared table, compensated sum
            const SrcInfo si = info[s];
            int h, wc;
            if (CUT) {
                const xts_cutout cw = cut[s];
                h = cw.h0 + pix / cw.nw;
                wc = cw.w0 + pix % cw.nw;
            } else {
                h = pix / W;
                wc = pix - h * W;
            }
            const PixGeom g = pixel_geom(corners, W1, h, wc, si);
            const float om = omega ? (float)omega[(size_t)h * W + wc] : 1.f;
            const float* Y = (const float*)tab;
            const int ES = 4 * EQ;
            for (int e = 0; e < E; ++e) {
                float acc1 = 0.f, comp = 0.f;
                for (int p = 0; p < 12; ++p) {
                    float tt;
                    const int idx = point_row(point_q(g, p), septab->q, (const float4*)septab->coef, &tt);
                    const float wgt = (float)c_rule_uv[p][3];
                    const float* yl = Y + (idx - 1) * ES + e;
                    const float term = fmaf((1.f - tt) * wgt, yl[0], tt * wgt * yl[ES]);
                    const float s2 = acc1 + term;
                    comp += fabsf(acc1) >= fabsf(term) ? (acc1 - s2) + term : (term - s2) + acc1;
                    acc1 = s2;
                }
                dst[e] = (acc1 + comp) * om;
            }
        }
        fence_async_shared();
        __syncwarp();
        // TMA bulk store of the warp's 16-byte aligned body, lanes for the edges
        if (nflat > 0) {
            const long long ga = (g0 + 3) & ~3LL, gb = (g0 + nflat) & ~3LL;
            if (lane == 0 && gb > ga)
                bulk_store(out + ga, stage + m + (int)(ga - g0), (unsigned)((gb - ga) * 4));
            if (lane < 8) {
                const long long g = lane < 4 ? g0 + lane : gb + (lane - 4);
                const bool head = lane < 4 && g < ga && g < g0 + nflat;
                const bool tail = lane >= 4 && g >= gb && g >= ga && g < g0 + nflat;
                if (head || tail) out[g] = stage[m + (int)(g - g0)];
            }
        }
        rec = nxt;
        if (sn != s) {
            np_s = sp_.pixels(sn);
            nt_s = sp_.tiles(sn);
        }
        s = sn;
        tile = tn;
    }
    (void)nt_s;
    if (lane == 0) bulk_wait_all();
}

struct WriteArgs {
    const float4* win; const float4* ext; const float2* sparse; const float* lut;
    const double* corners; const double* omega; const SrcInfo* info; const SepTab* tab;
    const xts_cutout* cut; const long long* tile_off;  // cutouts (cut != NULL): tile_off [S + 1]
    int S, s_base, H, W, E, EQ;
    int* status; float* out;
};

template <int NQ>
static int launch_write_pass(unsigned G, size_t smem, cudaStream_t st, const WriteArgs& a, int* per_sm, bool query) {
    if (query) {
        int pd = 0, pc = 0;
        XTS_CUDA(cudaFuncSetAttribute(k_srcmap_win<NQ, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        XTS_CUDA(cudaFuncSetAttribute(k_srcmap_win<NQ, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        XTS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pd, k_srcmap_win<NQ, false>, BT, smem));
        XTS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pc, k_srcmap_win<NQ, true>, BT, smem));
        *per_sm = pd < pc ? pd : pc;
        return XTS_OK;
    }
    if (a.cut)
        XTS_LAUNCH("k_srcmap", st, k_srcmap_win<NQ, true><<<G, BT, smem, st>>>(
                                       a.win, a.ext, a.sparse, a.lut, a.corners, a.omega, a.info, a.tab, a.cut,
                                       a.tile_off, a.S, a.s_base, a.H, a.W, a.E, a.EQ, a.status, a.out));
    else
        XTS_LAUNCH("k_srcmap", st, k_srcmap_win<NQ, false><<<G, BT, smem, st>>>(
                                       a.win, a.ext, a.sparse, a.lut, a.corners, a.omega, a.info, a.tab, nullptr,
                                       nullptr, a.S, a.s_base, a.H, a.W, a.E, a.EQ, a.status, a.out));
    return XTS_OK;
}

typedef int (*WritePassFn)(unsigned, size_t, cudaStream_t, const WriteArgs&, int*, bool);
static const WritePassFn k_write_pass[BQ] = {
    launch_write_pass<1>, launch_write_pass<2>, launch_write_pass<3>, launch_write_pass<4>, launch_write_pass<5>,
    launch_write_pass<6>, launch_write_pass<7>, launch_write_pass<8>, launch_write_pass<9>, launch_write_pass<10>,
    launch_write_pass<11>, launch_write_pass<12>, launch_write_pass<13>};

// ============================================================================ host
bool srcmap_win_supported(int E) {
    return E >= 1 && E <= 4 * BQ && win_layout(E, win_row_quads(E)).total <= 227 * 1024;
}

// Parts per source group of the dense window pass (n sources of ntile tiles, G
// blocks): about 16 queue items per block (c2: 1.66 ms at 8, 1.57 at 16, 1.63 at 32),
// at most one part per tile.
static int window_parts(int n, int ntile, int G) {
    const long long ng = (n + NSG - 1) / NSG;
    long long P = (16LL * G + ng - 1) / ng;
    if (P > ntile) P = ntile;
    return P < 1 ? 1 : (int)P;
}

// Window records of one source chunk: a 16-byte main record and a 32-byte
// extension slot per (source, pixel); only windows of more than REC_ROWS rows
// write and read their extension.
static size_t win_bytes_per_source(int npix) { return (size_t)npix * 48; }

// When the sources come in several chunks (host-mode copy-out, or records above
// the buffer budget) and a geometry stream is given, the window pass of chunk k + 1
// (geometry stream) may run while chunk k is corrected and written (launching
// stream): window records, sparse records, row histograms and scaled tables are
// double-buffered and events order each buffer's reuse.  Splitting a device-mode
// job into chunks only for this overlap was measured slower (c1: 0.375 ms in 2
// chunks, 0.392 in 4, 0.320 in one), so a device-mode job is one chunk.

int launch_srcmap_win(const double* corners, const double* centers, const double* omega,
                      const SrcInfo* info, int S, int H, int W, int E,
                      const double* upsf, const double* partial, const double* exposure,
                      double* scale, double* inv_integ, double* correction, double* radius,
                      int* in_fov, int* status, float* out, int chunk_sources,
                      int (*on_chunk)(void*, int, int, cudaStream_t), void* on_chunk_ctx,
                      StreamJoin& geo, cudaStream_t st, bool means_only) {
    int rc = upload_rule_uv(st);
    if (rc) return rc;
    const SepTab* tab = nullptr;
    rc = build_septab(st, &tab);
    if (rc) return rc;
    const cudaStream_t gs = geo.from;
    const bool pipe = gs != st;
    const int npix = H * W;
    const int EQ = win_row_quads(E);
    const WinLayout L = win_layout(E, EQ);
    // sources per chunk: window records of at most ~1 GiB per buffer
    const size_t budget = (size_t)4 << 30;
    int Sc = (int)(budget / win_bytes_per_source(npix));
    if (chunk_sources > 0 && chunk_sources < Sc) Sc = chunk_sources;
    if (g_tuning.chunk_sources > 0 && g_tuning.chunk_sources < Sc) Sc = g_tuning.chunk_sources;
    Sc = Sc < 1 ? 1 : (Sc > S ? S : Sc);
    const size_t rec_n = (size_t)Sc * npix + 4, ext_n = (size_t)Sc * npix * 2 + 4;
    const size_t lut_n = (size_t)Sc * ND * EQ * 4 + 4;
    // sparse records for wide pixels: room for 1/8 of the chunk's pixels (at least 64k)
    long long cap = (long long)Sc * npix / 8;
    cap = cap < 65536 ? 65536 : cap;
    cap = cap > (long long)Sc * npix ? (long long)Sc * npix : cap;
    const size_t sp_n = (size_t)NSP * cap + 2;
    float4* rec0 = (float4*)workspace(W_WIN, sizeof(float4) * 2 * rec_n);
    float4* ext0 = (float4*)workspace(W_WMETA, sizeof(float4) * 2 * ext_n);
    float* lut0 = (float*)workspace(W_LUT, sizeof(float) * 2 * lut_n);
    float2* sparse0 = (float2*)workspace(W_SPARSE, sizeof(float2) * 2 * sp_n);
    int dev = 0, nsm = 148, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    // pass A: one block per work item, items sized for about 16 per block of the
    // resident set (at most window_blocks_per_sm blocks per SM)
    int resident = 0;
    XTS_CUDA(cudaFuncSetAttribute(k_pixel_windows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)WA_SMEM));
    XTS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, k_pixel_windows, WT, WA_SMEM));
    resident = resident < 1 ? 1 : resident;
    if (g_tuning.window_blocks_per_sm > 0 && g_tuning.window_blocks_per_sm < resident)
        resident = g_tuning.window_blocks_per_sm;
    const int nparts = window_parts(Sc, (npix + WT - 1) / WT, resident * nsm);
    const size_t hist_n = (size_t)Sc * ND + 1;
    double* hist0 = (double*)workspace(W_PARTSUM, sizeof(double) * 2 * hist_n);
    if (!rec0 || !ext0 || !lut0 || !sparse0 || !hist0) return XTS_ERR_OOM;
    const WritePassFn wp = k_write_pass[(E + 3) / 4 - 1];
    rc = wp(0, L.total, st, WriteArgs{}, &per_sm, true);
    if (rc) return rc;
    if (per_sm < 1) return set_error(XTS_ERR_ARG, "source-map write pass does not fit on an SM (E=%d)", E);
    cudaEvent_t evA[2], evB[2];  // window pass of a buffer done; write pass of a buffer done
    pipe_events(evA, evB);
    int k = 0;
    for (int s0 = 0; s0 < S; s0 += Sc, ++k) {
        const int n = S - s0 < Sc ? S - s0 : Sc, b = k & 1;
        const size_t oE = (size_t)s0 * E;
        float4* rec = rec0 + b * rec_n;
        float4* ext = ext0 + b * ext_n;
        float* lut = lut0 + b * lut_n;
        float2* sparse = sparse0 + b * sp_n;
        double* hist = hist0 + b * hist_n;
        int* sparse_count = status + 1 + b;
        // the window pass is geometry only: it runs on the geometry stream, once
        // the write pass that last read its buffers is done
        if (pipe && k >= 2) XTS_CUDA(cudaStreamWaitEvent(gs, evB[b], 0));
        const int n_items = (n + NSG - 1) / NSG * nparts;  // one block per item
        XTS_CUDA(cudaMemsetAsync(sparse_count, 0, sizeof(int), gs));
        XTS_CUDA(cudaMemsetAsync(hist, 0, sizeof(double) * (size_t)n * ND, gs));
        XTS_LAUNCH("k_pixel_windows", gs, k_pixel_windows<<<n_items, WT, WA_SMEM, gs>>>(
                                              corners, centers, means_only ? nullptr : omega, info + s0, tab, n, H, W,
                                              nparts,
                                              hist, rec, ext, sparse, (int)cap,
                                              sparse_count));
        if (pipe) {
            XTS_CUDA(cudaEventRecord(evA[b], gs));
            XTS_CUDA(cudaStreamWaitEvent(st, evA[b], 0));
        }
        if (means_only) {
            XTS_LAUNCH("k_lut_scaled", st, k_lut_scaled<<<lut_scaled_grid(n), 256, 0, st>>>(
                                               upsf + oE * ND, nullptr, n, E, EQ * 4, lut, nullptr, nullptr));
        } else {
            rc = launch_correction(hist, 1, info + s0, n, upsf + oE * ND, partial + oE * ND,
                                   exposure + oE, E, scale + oE, inv_integ ? inv_integ + oE : nullptr,
                                   correction ? correction + oE : nullptr, radius ? radius + s0 : nullptr,
                                   in_fov ? in_fov + s0 : nullptr, st, lut, EQ * 4);
            if (rc) return rc;
        }
        const long long T = (long long)n * ((npix + BT - 1) / BT);
        long long G = (long long)nsm * (g_tuning.write_blocks_per_sm > 0 && g_tuning.write_blocks_per_sm < per_sm
                                            ? g_tuning.write_blocks_per_sm : per_sm);
        if (G > T) G = T;
        WriteArgs wa{rec, ext, sparse, lut, corners, means_only ? nullptr : omega, info + s0, tab, nullptr, nullptr,
                     n, s0, H, W, E, EQ, status, out};
        rc = wp((unsigned)G, L.total, st, wa, nullptr, false);
        if (rc) return rc;
        if (on_chunk && (rc = on_chunk(on_chunk_ctx, s0, n, st))) return rc;
        if (pipe) XTS_CUDA(cudaEventRecord(evB[b], st));
    }
    return geo.join();
}

// ============================================================================ cutouts
// Items of the cutout work queue: tile_off[s] = the first (source, tile) item of
// source s (tiles of WT pixels of its window), tile_off[S] = the item count.  One
// block; the sources in runs of 1024 with a block scan.
__global__ void __launch_bounds__(1024) k_cut_tiles(const xts_cutout* __restrict__ cut, int S,
                                                    long long* __restrict__ tile_off) {
    __shared__ long long part[32];
    __shared__ long long carry_s;
    const int t = threadIdx.x, lane = t & 31, wp = t >> 5;
    if (t == 0) carry_s = 0;
    __syncthreads();
    for (int s0 = 0; s0 < S; s0 += 1024) {
        const int s = s0 + t;
        const long long n = s < S ? ((long long)cut[s].nh * cut[s].nw + WT - 1) / WT : 0;
        long long inc = n;
        for (int o = 1; o < 32; o <<= 1) {
            const long long v = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += v;
        }
        if (lane == 31) part[wp] = inc;
        __syncthreads();
        long long before = carry_s;
        for (int k = 0; k < wp; ++k) before += part[k];
        if (s < S) tile_off[s] = before + inc - n;
        __syncthreads();
        if (t == 1023) carry_s = before + inc;
        __syncthreads();
    }
    if (t == 0) tile_off[S] = carry_s;
}

// item_src[i] = the source of item i (one block per source).
__global__ void k_cut_item_src(const long long* __restrict__ tile_off, int* __restrict__ item_src) {
    const int s = blockIdx.x;
    for (long long i = tile_off[s] + threadIdx.x; i < tile_off[s + 1]; i += blockDim.x) item_src[i] = s;
}

int launch_srcmap_win_cut(const double* corners, const double* centers, const double* omega, const SrcInfo* info,
                          const xts_cutout* cut, int S, int H, int W, int E, const double* upsf,
                          const double* partial, const double* exposure, double* scale, double* inv_integ,
                          double* correction, double* radius, int* in_fov, int* status, float* out, cudaStream_t st) {
    int rc = upload_rule_uv(st);
    if (rc) return rc;
    const SepTab* tab = nullptr;
    if ((rc = build_septab(st, &tab))) return rc;
    const long long npix = (long long)H * W;
    const int EQ = win_row_quads(E);
    const WinLayout L = win_layout(E, EQ);
    // buffers sized for the largest windows (every window the whole map): nothing here
    // depends on the windows' sizes on the host, so the call needs no synchronisation
    const long long max_items = (long long)S * ((npix + WT - 1) / WT);
    const size_t rec_n = (size_t)S * npix + 4;
    float4* rec = (float4*)workspace(W_WIN, sizeof(float4) * rec_n);
    float4* ext = (float4*)workspace(W_WMETA, sizeof(float4) * 2 * rec_n);
    float* lut = (float*)workspace(W_LUT, sizeof(float) * ((size_t)S * ND * EQ * 4 + 4));
    long long cap = (long long)S * npix / 8;
    cap = cap < 65536 ? 65536 : cap;
    float2* sparse = (float2*)workspace(W_SPARSE, sizeof(float2) * ((size_t)NSP * cap + 2));
    double* hist = (double*)workspace(W_PARTSUM, sizeof(double) * ((size_t)S * ND + 1));
    char* items = (char*)workspace(W_CUT_ITEMS, align_up(sizeof(long long) * (S + 1), 256) +
                                                    align_up(sizeof(int) * (size_t)max_items, 256) + 256);
    if (!rec || !ext || !lut || !sparse || !hist || !items) return XTS_ERR_OOM;
    long long* tile_off = (long long*)items;
    int* item_src = (int*)(items + align_up(sizeof(long long) * (S + 1), 256));
    unsigned long long* queue = (unsigned long long*)(items + align_up(sizeof(long long) * (S + 1), 256) +
                                                      align_up(sizeof(int) * (size_t)max_items, 256));
    int* sparse_count = status + 1;
    XTS_CUDA(cudaMemsetAsync(hist, 0, sizeof(double) * (size_t)S * ND, st));
    XTS_CUDA(cudaMemsetAsync(queue, 0, sizeof(unsigned long long), st));
    XTS_CUDA(cudaMemsetAsync(sparse_count, 0, sizeof(int), st));
    XTS_LAUNCH("k_cut_tiles", st, k_cut_tiles<<<1, 1024, 0, st>>>(cut, S, tile_off));
    XTS_LAUNCH("k_cut_item_src", st, k_cut_item_src<<<S, 256, 0, st>>>(tile_off, item_src));
    int dev = 0, nsm = 148, resident = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    XTS_CUDA(cudaFuncSetAttribute(k_pixel_windows_cut, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)WA_SMEM));
    XTS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, k_pixel_windows_cut, WT, WA_SMEM));
    resident = resident < 1 ? 1 : resident;
    if (g_tuning.queue_blocks_per_sm > 0 && g_tuning.queue_blocks_per_sm < resident) resident = g_tuning.queue_blocks_per_sm;
    // pass A: one persistent wave pulling (source, tile) items from the queue
    XTS_LAUNCH("k_pixel_windows", st, k_pixel_windows_cut<<<(unsigned)(resident * nsm), WT, WA_SMEM, st>>>(
                                          corners, centers, omega, info, cut, item_src, tile_off, queue, tab, S, W,
                                          hist, rec, ext, sparse, (int)cap, sparse_count));
    rc = launch_correction(hist, 1, info, S, upsf, partial, exposure, E, scale, inv_integ, correction, radius, in_fov,
                           st, lut, EQ * 4);
    if (rc) return rc;
    const WritePassFn wp = k_write_pass[(E + 3) / 4 - 1];
    if ((rc = wp(0, L.total, st, WriteArgs{}, &per_sm, true))) return rc;
    if (per_sm < 1) return set_error(XTS_ERR_ARG, "source-map write pass does not fit on an SM (E=%d)", E);
    WriteArgs wa{rec, ext, sparse, lut, corners, omega, info, tab, cut, tile_off, S, 0, H, W, E, EQ, status, out};
    if (g_tuning.write_blocks_per_sm > 0 && g_tuning.write_blocks_per_sm < per_sm) per_sm = g_tuning.write_blocks_per_sm;
    // pass B: one persistent wave over the same items, split evenly between the blocks
    return wp((unsigned)(nsm * per_sm), L.total, st, wa, nullptr, false);
}

}  // namespace xts
