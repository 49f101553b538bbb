// xts_srcmap_tc.cu -- the FP32 source-map write pass (d1 + d2 + c8 + c10) with the
// interpolation contraction on the 5th-generation tensor cores (tcgen05).
//
// For a tile of TM = 128 pixels of one source, the map values are
//     out[p][e] = sum_r W[p][r] * Y'[r][e]
// where W[p][r] is pixel p's interpolation weight on table row r (its rule
// points' (1-t) w and t w times the pixel's solid angle, at most RW = 8
// consecutive rows per pixel, built on CUDA cores in FP64/FP32 by
// xts_point.cuh) and Y' = uPsf * exposure * correction (FP32).  The tile's rows
// [R0, R0 + 32 nk) are processed in chunks of KC = 32:
//   * A = W[:, chunk] (128 x 32, K-major, 128-byte swizzle) is written to shared
//     memory by the threads, split into TF32 hi and lo parts;
//   * B = Y'[chunk rows, 0..N) (N x 32, K-major, 128-byte swizzle) is loaded by
//     TMA from transposed hi and lo tables [s][e][row] (rows past 400 and
//     energies past E read as zeros; tf32 MMAs need B K-major);
//   * one thread issues tcgen05.mma.kind::tf32 (M = 128, N = 16 ceil(E/16), K = 8)
//     for A_hi B_hi + A_lo B_hi + A_hi B_lo into an FP32 accumulator in tensor
//     memory (3xTF32: ~2^-21 relative per product, FP32 accumulation);
//   * the four warps read the accumulator back with tcgen05.ld, stage the tile
//     in shared memory in the map's [pixel][energy] order, and one TMA bulk store
//     writes it out.
// Pixels whose rule points span more than RW rows (next to the source) are
// evaluated on CUDA cores by all threads of the CTA, point by point with a
// compensated sum.  Every wait on an mbarrier is bounded; on timeout the kernel
// records an error, stops issuing work, frees its tensor memory and returns.
#include <cuda.h>

#include "xts_point.cuh"

namespace xts {

constexpr int TM = 128;  // pixels per tile == MMA M == threads per block
constexpr int KC = 32;   // table rows per K chunk (128 bytes of TF32: one swizzle atom)

struct TcLayout {  // shared-memory byte offsets, all multiples of 16 (A, B: 1024)
    int na, N, E;
    size_t a_hi, a_lo, b_hi, b_lo, sq, coef, win, meta, wpts, wom, stage, bars, total;
};

XTS_HD inline TcLayout tc_layout(int E) {
    TcLayout L;
    L.E = E;
    L.N = (E + 15) / 16 * 16;
    L.na = (L.N + 31) / 32;
    size_t o = 0;
    L.a_hi = o; o += TM * KC * 4;
    L.a_lo = o; o += TM * KC * 4;
    L.b_hi = o; o += (size_t)L.N * 128;
    L.b_lo = o; o += (size_t)L.N * 128;
    L.sq = o; o += (8 * (ND + 1) + 15) / 16 * 16;
    L.coef = o; o += 16 * 2 * ND;
    L.win = o; o += (4 * TM * WST + 15) / 16 * 16;
    L.meta = o; o += 16 * TM;                     // rbase, nrows, wide slot, pad per pixel
    L.wpts = o; o += 8 * 12 * TM;                 // (row, t) of the 12 points of wide pixels
    L.wom = o; o += 8 * TM + 64;                  // omega and pixel of wide slots, counters
    L.stage = o; o += ((size_t)4 * TM * E + 32 + 15) / 16 * 16;
    L.bars = o; o += 64;
    L.total = o;
    return L;
}

// UMMA shared-memory descriptors (sm_100 format: start >> 4 in [0,14), LBO >> 4 in
// [16,30), SBO >> 4 in [32,46), version 1 at bit 46, layout type in [61,64); 2 = 128B swizzle).
__device__ __forceinline__ unsigned long long sw128_desc(unsigned addr, unsigned lbo, unsigned sbo) {
    return (unsigned long long)((addr >> 4) & 0x3FFF) | ((unsigned long long)((lbo >> 4) & 0x3FFF) << 16) |
           ((unsigned long long)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46) | (2ull << 61);
}

// Instruction descriptor: D f32, A/B tf32, both K-major, M = 128, N.
__host__ __device__ constexpr unsigned tf32_idesc(int N) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((unsigned)(N >> 3) << 17) | ((unsigned)(TM >> 4) << 24);
}

__device__ __forceinline__ unsigned tf32_round(float v) {
    unsigned r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(v));
    return r;
}

__global__ void __launch_bounds__(TM, 2)
k_srcmap_tc(const __grid_constant__ CUtensorMap tm_hi, const __grid_constant__ CUtensorMap tm_lo,
            const double* __restrict__ corners, const double* __restrict__ omega,
            const SrcInfo* __restrict__ info, const float* __restrict__ lut,
            const SepTab* __restrict__ septab, int H, int W, int E, int Epad, int nchunk,
            float* __restrict__ out, int* __restrict__ status) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // the dynamic buffer is re-aligned to 1024 bytes for the swizzled operands
    unsigned char* smem = smem_raw + ((1024 - (smem_u32(smem_raw) & 1023)) & 1023);
    const TcLayout L = tc_layout(E);
    double* sq = (double*)(smem + L.sq);
    float4* scoef = (float4*)(smem + L.coef);
    float* win = (float*)(smem + L.win);
    int4* meta = (int4*)(smem + L.meta);
    int2* wpts = (int2*)(smem + L.wpts);
    float* wom = (float*)(smem + L.wom);
    int* wpix = (int*)(smem + L.wom + 4 * TM);     // pixel (tile index) of each wide slot
    int* cnt = (int*)(smem + L.wom + 8 * TM);      // [0] wide count, [1] row min, [2] row max, [3] abort
    float* stage = (float*)(smem + L.stage);
    unsigned long long* bars = (unsigned long long*)(smem + L.bars);
    unsigned* tmem_slot = (unsigned*)(smem + L.bars + 32);
    const unsigned bar_tma = smem_u32(&bars[0]), bar_mma = smem_u32(&bars[1]);

    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int s = blockIdx.y;
    const int N = L.N;
    const unsigned ncols = N <= 32 ? 32u : (N <= 64 ? 64u : (N <= 128 ? 128u : 256u));
    const unsigned idesc = tf32_idesc(N);

    for (int k = t; k < ND + 1; k += TM) sq[k] = septab->q[k];
    for (int k = t; k < 2 * ND; k += TM) scoef[k] = ((const float4*)septab->coef)[k];
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(bar_tma));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(bar_mma));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        cnt[3] = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(tmem_slot)), "r"(ncols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const unsigned tmem = *tmem_slot;

    const SrcInfo si = info[s];
    const int npix = H * W, W1 = W + 1;
    const int ntiles = (npix + TM - 1) / TM;
    const float* Y = lut + (size_t)s * ND * Epad;
    float* wr = win + t * WST;
    unsigned ph_tma = 0, ph_mma = 0;
    bool ok = true;

    for (int tile = blockIdx.x; tile < ntiles && ok; tile += nchunk) {
        const int p0 = tile * TM;
        const int np = min(TM, npix - p0);
        const long long g0 = ((long long)s * npix + p0) * E;
        const int m0 = (int)(g0 & 3);
        const int nflat = np * E;
        if (t == 0) { cnt[0] = 0; cnt[1] = ND; cnt[2] = -1; }
        __syncthreads();

        // ---------------- phase 1: the pixel's row window (CUDA cores)
        int nrows = 0, rbase = 0, wslot = -1;
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
            bool wide = false;
            int pidx[12];
            float pt[12];
#pragma unroll
            for (int p = 0; p < 12; ++p) {
                float tt;
                const int idx = point_row(point_q(g, p), sq, scoef, &tt);
                pidx[p] = idx;
                pt[p] = tt;
                const int r = idx - 1 - rbase;
                if (r >= 0 && r < RW - 1) {
                    const float wgt = (float)c_rule_uv[p][3];
                    wr[r] = fmaf(1.f - tt, wgt, wr[r]);
                    wr[r + 1] = fmaf(tt, wgt, wr[r + 1]);
                    lo = min(lo, r);
                    hi = max(hi, r + 1);
                } else {
                    wide = true;
                }
            }
            const float om = (float)omega[pix];
            if (!wide) {
                nrows = hi - lo + 1;
                for (int j = 0; j < nrows; ++j) wr[j] = wr[j + lo] * om;
                rbase += lo;
                atomicMin(&cnt[1], rbase);
                atomicMax(&cnt[2], rbase + nrows - 1);
            } else {
                wslot = atomicAdd(&cnt[0], 1);
#pragma unroll
                for (int p = 0; p < 12; ++p) wpts[wslot * 12 + p] = make_int2(pidx[p], __float_as_int(pt[p]));
                wom[wslot] = om;
                wpix[wslot] = t;
            }
        }
        meta[t] = make_int4(rbase, nrows, wslot, pix);
        __syncthreads();
        const int R0 = cnt[1] & ~3, Rmax = cnt[2], nwide = cnt[0];  // TMA x coordinate: multiple of 4
        const int nk = Rmax >= R0 ? (Rmax - R0) / KC + 1 : 0;

        // ---------------- tensor cores: K chunks of 32 rows
        for (int c = 0; c < nk && ok; ++c) {
            const int rc = R0 + KC * c;
            if (t == 0) {
                if (c > 0) { ok = mbar_wait(bar_mma, ph_mma); ph_mma ^= 1; }  // previous chunk done with A, B
                if (ok) {
                    const unsigned bytes = (unsigned)(2 * N * 128);
                    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(bar_tma), "r"(bytes) : "memory");
                    asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
                                 :: "r"(smem_u32(smem + L.b_hi)), "l"((unsigned long long)&tm_hi),
                                    "r"(rc), "r"(0), "r"(s), "r"(bar_tma) : "memory");
                    asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
                                 :: "r"(smem_u32(smem + L.b_lo)), "l"((unsigned long long)&tm_lo),
                                    "r"(rc), "r"(0), "r"(s), "r"(bar_tma) : "memory");
                } else {
                    cnt[3] = 1;
                }
            }
            __syncthreads();
            if (cnt[3]) { ok = false; break; }
            // A row of pixel t for rows [rc, rc + KC): zero, then scatter its window
            {
                unsigned char* ahi = smem + L.a_hi + (t >> 3) * 1024 + (t & 7) * 128;
                unsigned char* alo = smem + L.a_lo + (t >> 3) * 1024 + (t & 7) * 128;
                const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    *(float4*)(ahi + (j << 4)) = z4;
                    *(float4*)(alo + (j << 4)) = z4;
                }
                for (int j = 0; j < nrows; ++j) {
                    const int k = rbase + j - rc;
                    if (k >= 0 && k < KC) {
                        const float v = wr[j];
                        const float vh = __uint_as_float(tf32_round(v));
                        const int off = ((((k >> 2) ^ (t & 7)) << 4)) + (k & 3) * 4;
                        *(float*)(ahi + off) = vh;
                        *(float*)(alo + off) = v - vh;
                    }
                }
            }
            fence_async_shared();
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncthreads();
            if (t == 0) {
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                ok = mbar_wait(bar_tma, ph_tma);
                ph_tma ^= 1;
                if (ok) {
                    const unsigned a_hi = smem_u32(smem + L.a_hi), a_lo = smem_u32(smem + L.a_lo);
                    const unsigned b_hi = smem_u32(smem + L.b_hi), b_lo = smem_u32(smem + L.b_lo);
#pragma unroll
                    for (int ks = 0; ks < KC / 8; ++ks) {
                        const unsigned long long dah = sw128_desc(a_hi + 32 * ks, 16, 1024);
                        const unsigned long long dal = sw128_desc(a_lo + 32 * ks, 16, 1024);
                        const unsigned long long dbh = sw128_desc(b_hi + 32 * ks, 16, 1024);
                        const unsigned long long dbl = sw128_desc(b_lo + 32 * ks, 16, 1024);
                        // small cross terms first, the full-size hi*hi term last, so that
                        // the accumulator's FP32 rounding acts once at full magnitude per step
                        const unsigned long long da[3] = {dal, dah, dah};
                        const unsigned long long db[3] = {dbh, dbl, dbh};
#pragma unroll
                        for (int term = 0; term < 3; ++term) {
                            const unsigned acc = (c > 0 || ks > 0 || term > 0) ? 1u : 0u;
                            asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                                         "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n"
                                         :: "r"(tmem), "l"(da[term]), "l"(db[term]), "r"(idesc), "r"(acc), "r"(0u));
                        }
                    }
                    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                                 :: "r"(bar_mma) : "memory");
                } else {
                    cnt[3] = 1;
                }
            }
            __syncthreads();
            if (cnt[3]) { ok = false; break; }
        }
        if (!ok) break;

        // ---------------- epilogue: accumulator -> stage (after the last MMA and the previous store)
        if (t == 0) {
            bulk_wait_read();
            if (nk > 0) {
                ok = mbar_wait(bar_mma, ph_mma);
                ph_mma ^= 1;
                if (!ok) cnt[3] = 1;
            }
        }
        __syncthreads();
        if (cnt[3]) { ok = false; break; }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (nk > 0) {
            const int m = warp * 32 + lane;  // this thread's accumulator row = pixel
            for (int c0 = 0; c0 < N; c0 += 16) {
                unsigned v[16];
                const unsigned taddr = tmem + ((unsigned)(warp * 32) << 16) + (unsigned)c0;
                asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                             : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                               "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                             : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                if (m < np && meta[m].y > 0) {
                    float* dst = stage + m0 + m * E + c0;
#pragma unroll
                    for (int j = 0; j < 16; ++j)
                        if (c0 + j < E) dst[j] = __uint_as_float(v[j]);
                }
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        // wide pixels: (pixel, energy) items shared by all threads
        for (int item = t; item < nwide * E; item += TM) {
            const int sl = item / E, e = item - sl * E;
            const int2* pp = wpts + sl * 12;
            float acc = 0.f, comp = 0.f;
#pragma unroll
            for (int p = 0; p < 12; ++p) {
                const int idx = pp[p].x;
                const float tt = __int_as_float(pp[p].y);
                const float wgt = (float)c_rule_uv[p][3];
                const float* yl = Y + (size_t)(idx - 1) * Epad + e;
                const float term = fmaf((1.f - tt) * wgt, __ldg(yl), tt * wgt * __ldg(yl + Epad));
                const float s2 = acc + term;
                comp += fabsf(acc) >= fabsf(term) ? (acc - s2) + term : (term - s2) + acc;
                acc = s2;
            }
            stage[m0 + wpix[sl] * E + e] = (acc + comp) * wom[sl];
        }
        fence_async_shared();
        __syncthreads();
        // ---------------- store: TMA bulk for the 16-byte aligned body, threads for the edges
        const long long ga = (g0 + 3) & ~3LL, gb = (g0 + nflat) & ~3LL;
        if (t == 0 && gb > ga) bulk_store(out + ga, stage + m0 + (int)(ga - g0), (unsigned)((gb - ga) * 4));
        if (t < 8) {
            const long long gg = t < 4 ? g0 + t : gb + (t - 4);
            const bool head = t < 4 && gg < ga && gg < g0 + nflat;
            const bool tail = t >= 4 && gg >= gb && gg >= ga && gg < g0 + nflat;
            if (head || tail) out[gg] = stage[m0 + (int)(gg - g0)];
        }
        __syncthreads();
    }
    if (t == 0) {
        bulk_wait_all();
        if (!ok) {
            // a wait gave up: record it and let in-flight copies and MMAs land
            // (again bounded) before the shared and tensor memory are released
            atomicExch(status, 1);
            mbar_wait(bar_tma, ph_tma);
            mbar_wait(bar_mma, ph_mma);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(ncols));
}

// ------------------------------------------------------------------ host side
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
        else
            cudaGetLastError();
    }
    return fn;
}

// 3-D map over a transposed [S][E][NDP] float table (rows contiguous), boxes of
// 32 rows x N energies; rows past 400 and energies past E read as zeros.
constexpr int NDP = 404;  // row stride of the transposed tables (16-byte multiple)

static int make_table_map(CUtensorMap* m, const float* base, int S, int E, int N) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return set_error(XTS_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
    cuuint64_t dims[3] = {(cuuint64_t)ND, (cuuint64_t)E, (cuuint64_t)S};
    cuuint64_t strides[2] = {(cuuint64_t)NDP * 4, (cuuint64_t)NDP * E * 4};
    cuuint32_t box[3] = {(cuuint32_t)KC, (cuuint32_t)N, 1};
    cuuint32_t es[3] = {1, 1, 1};
    CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void*)base, dims, strides, box, es,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_error(XTS_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return XTS_OK;
}

// Transposed 3xTF32 split of the scaled table: hi = tf32(Y'), lo = Y' - hi, [s][e][row].
__global__ void k_lut_split_t(const float* lut, int S, int E, int Epad, float* hi, float* lo) {
    size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    size_t n = (size_t)S * E * NDP;
    if (k >= n) return;
    int r = (int)(k % NDP);
    size_t se = k / NDP;
    int e = (int)(se % E), s = (int)(se / E);
    float v = r < ND ? lut[((size_t)s * ND + r) * Epad + e] : 0.f;
    float h = __uint_as_float(tf32_round(v));
    hi[k] = h;
    lo[k] = v - h;
}

size_t srcmap_tc_smem(int E) { return tc_layout(E).total + 1024; }

int launch_srcmap_tc(const double* corners, const double* omega, const SrcInfo* info,
                     const double* upsf, const double* scale, int S, int H, int W, int E, float* out,
                     int* status, cudaStream_t st) {
    int rc = upload_rule_uv(st);
    if (rc) return rc;
    const SepTab* tab = nullptr;
    rc = build_septab(st, &tab);
    if (rc) return rc;
    int Epad = (E + 3) & ~3;
    const int N = tc_layout(E).N;
    size_t n = (size_t)S * ND * Epad, nt = (size_t)S * E * NDP;
    float* lut = (float*)workspace(W_LUT, sizeof(float) * (n + 2 * nt) + 64);
    if (!lut) return XTS_ERR_OOM;
    float* hi = lut + ((n + 3) & ~(size_t)3);
    float* lo = hi + nt;
    XTS_LAUNCH("k_lut_scaled", st, k_lut_scaled<<<lut_scaled_grid(S), 256, 0, st>>>(upsf, scale, S, E, Epad, lut, nullptr, nullptr));
    XTS_LAUNCH("k_lut_split_t", st, k_lut_split_t<<<(unsigned)((nt + 255) / 256), 256, 0, st>>>(lut, S, E, Epad, hi, lo));
    CUtensorMap mhi, mlo;
    if ((rc = make_table_map(&mhi, hi, S, E, N))) return rc;
    if ((rc = make_table_map(&mlo, lo, S, E, N))) return rc;
    size_t smem = srcmap_tc_smem(E);
    XTS_CUDA(cudaFuncSetAttribute(k_srcmap_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    int per_sm = 0;
    XTS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_srcmap_tc, TM, smem));
    if (per_sm < 1) return set_error(XTS_ERR_ARG, "source-map tensor-core kernel does not fit (E=%d)", E);
    int npix = H * W, ntiles = (npix + TM - 1) / TM;
    int target = nsm * per_sm * 4;
    int nchunk = (target + S - 1) / S;
    nchunk = nchunk > ntiles ? ntiles : (nchunk < 1 ? 1 : nchunk);
    XTS_LAUNCH("k_srcmap", st, k_srcmap_tc<<<dim3(nchunk, S), TM, smem, st>>>(mhi, mlo, corners, omega, info, lut, tab, H, W, E, Epad, nchunk, out, status));
    return XTS_OK;
}

}  // namespace xts
