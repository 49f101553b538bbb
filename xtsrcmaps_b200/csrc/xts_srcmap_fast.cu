// xts_srcmap_fast.cu -- the FP32 source-map write pass (d1 + d2 + c8 + c10) on
// CUDA cores, and the FP64 map integral (c7) of the fast path.
//
// Phase 1 (one thread per pixel) builds the pixel's dense window of at most RW
// table rows: the points' weights (1-t) w and t w (xts_point.cuh) times the
// pixel's solid angle.  Pixels whose points leave the window (the few next to
// the source) are evaluated point by point.  Phase 2 walks the tile's output in
// flat (pixel, energy) order: each value is sum_j W[p][j] * Y'[rbase + j][e],
// Y' = uPsf * exposure * correction in FP32, read through L1.  Values are staged
// in shared memory and written with one TMA bulk store per tile.
#include "xts_point.cuh"

namespace xts {

constexpr int FT = 256;  // pixels per tile == threads per block

// Shared-memory layout (byte offsets, each 16-byte aligned).
constexpr size_t OFF_SQ = 0;
constexpr size_t OFF_COEF = (8 * (ND + 1) + 15) / 16 * 16;
constexpr size_t OFF_WIN = OFF_COEF + sizeof(float4) * 2 * ND;
constexpr size_t OFF_META = OFF_WIN + (sizeof(float) * FT * WST + 15) / 16 * 16;
constexpr size_t OFF_STAGE = OFF_META + sizeof(int) * FT;

size_t srcmap_fast_smem(int E) { return OFF_STAGE + sizeof(float) * ((size_t)FT * E + 8); }

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
    XTS_LAUNCH("k_lut_scaled", st, k_lut_scaled<<<lut_scaled_grid(S), 256, 0, st>>>(upsf, scale, S, E, Epad, lut, nullptr, nullptr));
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
