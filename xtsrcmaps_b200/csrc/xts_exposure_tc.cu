// xts_exposure_tc.cu -- the full-sky exposure contraction on tcgen05 tensor
// cores: for every HEALPix pixel p of the livetime cube,
//     expo[p][e] = L0[e] sum_c X[p][c] A[c][e] + L1[e] sum_c Wt[p][c] A[c][e]
// with X, Wt the livetime and weighted-livetime rows [12 nside^2, C], A the
// summed front and back effective area [C, E] (the back side uses the front
// livetime-efficiency factors, psf.psf_lookup_table_and_partial_integrals.cxx:151-156
// and exposure/exposure.cxx:159-263) and L0, L1 = front_LTF [2, E].  A source's
// exposure (Exposure::exposure) is the row of this map at the source's NESTED
// pixel (exposure/exposure.cxx:42-63).
//
// One GEMM: M = pixels, K = [X | Wt] (each half zero-padded from C to 64 by the
// TMA fill, four K chunks of 32), N = E rounded up to 16, B = [A L0 ; A L1]
// prepared once (K-major).  Per tile of 128 pixels and K chunk: TMA loads the
// raw FP32 livetime rows (128-byte swizzle) and the B chunk's TF32 hi and lo
// parts; the threads split the A tile in place into hi = tf32(x) and lo = x - hi
// (same byte positions, so the swizzle needs no handling); one thread issues
// tcgen05.mma.kind::tf32 for A_lo B_hi + A_hi B_lo + A_hi B_hi (3xTF32, small
// terms first) into an FP32 accumulator in tensor memory.  The epilogue reads it
// with tcgen05.ld, stages the tile and writes FP64 rows with coalesced stores.
// Every mbarrier wait is bounded; a timeout sets the status word, lets in-flight
// copies and MMAs land (bounded), frees tensor memory and returns.
#include <cuda.h>

#include "xts_point.cuh"

namespace xts {

constexpr int XM = 128;  // pixels per tile == MMA M == threads per block
constexpr int XK = 32;   // floats per K chunk (one 128-byte swizzle atom)
constexpr int XKP = 64;  // padded K of each half (livetime, weighted livetime)

struct XLayout { int N; size_t a_hi, a_lo, b_hi, b_lo, stage, bars, total; };

XTS_HD inline XLayout x_layout(int E) {
    XLayout L;
    L.N = (E + 15) / 16 * 16;
    size_t o = 0;
    L.a_hi = o; o += XM * XK * 4;
    L.a_lo = o; o += XM * XK * 4;
    L.b_hi = o; o += (size_t)L.N * 128;
    L.b_lo = o; o += (size_t)L.N * 128;
    L.stage = o; o += ((size_t)XM * E * 4 + 15) / 16 * 16;
    L.bars = o; o += 64;
    L.total = o;
    return L;
}

static __device__ __forceinline__ unsigned long long x_desc(unsigned addr) {
    // K-major, 128-byte swizzle: start >> 4, LBO 16 >> 4, SBO 1024 >> 4 (8-row groups), version 1
    return (unsigned long long)((addr >> 4) & 0x3FFF) | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}

// D f32, A/B tf32, both K-major, M = 128, N.
static __host__ __device__ constexpr unsigned x_idesc(int N) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((unsigned)(N >> 3) << 17) | ((unsigned)(XM >> 4) << 24);
}

static __device__ __forceinline__ float tf32_hi(float v) {
    unsigned r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(v));
    return __uint_as_float(r);
}

__global__ void __launch_bounds__(XM, 1)
k_exposure_map_tc(const __grid_constant__ CUtensorMap tm_x, const __grid_constant__ CUtensorMap tm_w,
                  const __grid_constant__ CUtensorMap tm_bhi, const __grid_constant__ CUtensorMap tm_blo,
                  int npix, int E, double* __restrict__ out, int* __restrict__ status) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* smem = smem_raw + ((1024 - (smem_u32(smem_raw) & 1023)) & 1023);
    const XLayout L = x_layout(E);
    float* stage = (float*)(smem + L.stage);
    unsigned long long* bars = (unsigned long long*)(smem + L.bars);
    unsigned* tmem_slot = (unsigned*)(smem + L.bars + 32);
    int* abort_flag = (int*)(smem + L.bars + 48);
    const unsigned bar_tma = smem_u32(&bars[0]), bar_mma = smem_u32(&bars[1]);
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int N = L.N;
    const unsigned ncols = N <= 32 ? 32u : (N <= 64 ? 64u : (N <= 128 ? 128u : 256u));
    const unsigned idesc = x_idesc(N);

    if (t == 0) {
        mbar_init(bar_tma, 1);
        mbar_init(bar_mma, 1);
        *abort_flag = 0;
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

    const int ntiles = (npix + XM - 1) / XM;
    unsigned ph_tma = 0, ph_mma = 0;
    bool ok = true;
    const unsigned bytes = (unsigned)(XM * XK * 4 + 2 * N * 128);
    for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const int p0 = tile * XM;
        for (int c = 0; c < 2 * XKP / XK && ok; ++c) {
            // chunk c: livetime (c < 2) or weighted livetime (c >= 2) columns [32 (c & 1), +32)
            if (t == 0) {
                if (c > 0) { ok = mbar_wait(bar_mma, ph_mma); ph_mma ^= 1; }  // the previous MMAs read A and B
                if (ok) {
                    const CUtensorMap* ta = c < 2 ? &tm_x : &tm_w;
                    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(bar_tma), "r"(bytes) : "memory");
                    asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
                                 :: "r"(smem_u32(smem + L.a_hi)), "l"((unsigned long long)ta), "r"(XK * (c & 1)), "r"(p0),
                                    "r"(bar_tma) : "memory");
                    asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
                                 :: "r"(smem_u32(smem + L.b_hi)), "l"((unsigned long long)&tm_bhi), "r"(XK * c), "r"(0),
                                    "r"(bar_tma) : "memory");
                    asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
                                 :: "r"(smem_u32(smem + L.b_lo)), "l"((unsigned long long)&tm_blo), "r"(XK * c), "r"(0),
                                    "r"(bar_tma) : "memory");
                }
                if (!ok) *abort_flag = 1;
            }
            __syncthreads();
            if (*abort_flag) { ok = false; break; }
            // every thread waits for the copies it is about to read (bounded)
            const bool got = mbar_wait(bar_tma, ph_tma);
            ph_tma ^= 1;
            if (!__syncthreads_and(got)) {
                if (t == 0) *abort_flag = 1;
                ok = false;
                break;
            }
            // split the A tile in place: row t (128 bytes) -> hi here, lo in a_lo
            {
                float4* ah = (float4*)(smem + L.a_hi + t * 128);
                float4* al = (float4*)(smem + L.a_lo + t * 128);
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const float4 v = ah[j];
                    const float4 h = make_float4(tf32_hi(v.x), tf32_hi(v.y), tf32_hi(v.z), tf32_hi(v.w));
                    ah[j] = h;
                    al[j] = make_float4(v.x - h.x, v.y - h.y, v.z - h.z, v.w - h.w);
                }
            }
            fence_async_shared();
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncthreads();
            if (t == 0) {
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const unsigned a_hi = smem_u32(smem + L.a_hi), a_lo = smem_u32(smem + L.a_lo);
                const unsigned b_hi = smem_u32(smem + L.b_hi), b_lo = smem_u32(smem + L.b_lo);
#pragma unroll
                for (int ks = 0; ks < XK / 8; ++ks) {
                    const unsigned long long da[3] = {x_desc(a_lo + 32 * ks), x_desc(a_hi + 32 * ks), x_desc(a_hi + 32 * ks)};
                    const unsigned long long db[3] = {x_desc(b_hi + 32 * ks), x_desc(b_lo + 32 * ks), x_desc(b_hi + 32 * ks)};
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
            }
        }
        if (!ok) break;
        // epilogue: wait for the tile's last MMAs, accumulator -> stage -> FP64 rows
        if (t == 0) {
            ok = mbar_wait(bar_mma, ph_mma);
            ph_mma ^= 1;
            if (!ok) *abort_flag = 1;
        }
        __syncthreads();
        if (*abort_flag) { ok = false; break; }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int m = warp * 32 + lane;
        for (int c0 = 0; c0 < N; c0 += 16) {
            unsigned v[16];
            const unsigned taddr = tmem + ((unsigned)(warp * 32) << 16) + (unsigned)c0;
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                         : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                           "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                         : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int j = 0; j < 16; ++j)
                if (c0 + j < E) stage[m * E + c0 + j] = __uint_as_float(v[j]);
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        const int np = min(XM, npix - p0);
        double* dst = out + (size_t)p0 * E;
        for (int k = t; k < np * E; k += XM) dst[k] = (double)stage[k];
        __syncthreads();
    }
    if (t == 0 && !ok) {
        atomicExch(status, 1);
        mbar_wait(bar_tma, ph_tma);  // bounded: let in-flight copies and MMAs land
        mbar_wait(bar_mma, ph_mma);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(ncols));
}

// B = [A L0 ; A L1] as TF32 hi and lo, [N][2 * XKP] (K contiguous); rows past E,
// and the padding columns of each half, are zero.
__global__ void k_exposure_b(const double* af, const double* ab, const double* ltf, int C, int E, int N,
                             float* bhi, float* blo) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= N * 2 * XKP) return;
    const int e = k / (2 * XKP), kk = k - e * (2 * XKP);
    const int half = kk / XKP, c = kk - half * XKP;
    double v = 0.;
    if (e < E && c < C) v = (af[(size_t)c * E + e] + ab[(size_t)c * E + e]) * ltf[(size_t)half * E + e];
    const float f = (float)v;
    const float h = tf32_hi(f);
    bhi[k] = h;
    blo[k] = f - h;
}

typedef CUresult (*XEncodeFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                              const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                              CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static XEncodeFn x_encode() {
    static XEncodeFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (XEncodeFn)p;
        else
            cudaGetLastError();
    }
    return fn;
}

// 2-D FP32 map [rows][cols], boxes of 32 columns x box_rows rows, 128-byte swizzle;
// columns past `cols` and rows past `rows` read as zeros.
static int x_map(CUtensorMap* m, const float* base, long long rows, int cols, int box_rows) {
    XEncodeFn fn = x_encode();
    if (!fn) return set_error(XTS_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)cols * 4};
    cuuint32_t box[2] = {(cuuint32_t)XK, (cuuint32_t)box_rows};
    cuuint32_t es[2] = {1, 1};
    CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void*)base, dims, strides, box, es,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_error(XTS_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return XTS_OK;
}

bool exposure_map_supported(int C, int E) { return C >= 1 && C <= XKP && (C * 4) % 16 == 0 && E >= 1 && E <= 256; }

int launch_exposure_map_tc(const float* cube, const float* wcube, long long npix, int C, const double* front_aeff,
                           const double* back_aeff, const double* ltf, int E, double* out, int* status,
                           cudaStream_t st) {
    if (!exposure_map_supported(C, E))
        return set_error(XTS_ERR_ARG, "exposure map: needs C <= 64 with 16-byte rows (C %% 4 == 0) and E <= 256");
    if (npix > 0x7fffffffLL) return set_error(XTS_ERR_ARG, "exposure map: too many pixels");
    const XLayout L = x_layout(E);
    const int N = L.N;
    float* b = (float*)workspace(W_MISC2, sizeof(float) * 2 * (size_t)N * 2 * XKP + 64);
    if (!b) return XTS_ERR_OOM;
    float* bhi = b;
    float* blo = b + (size_t)N * 2 * XKP;
    const int nb = N * 2 * XKP;
    XTS_LAUNCH("k_exposure_b", st, k_exposure_b<<<(nb + 255) / 256, 256, 0, st>>>(front_aeff, back_aeff, ltf, C, E, N,
                                                                                  bhi, blo));
    CUtensorMap mx, mw, mbh, mbl;
    int rc;
    if ((rc = x_map(&mx, cube, npix, C, XM))) return rc;
    if ((rc = x_map(&mw, wcube, npix, C, XM))) return rc;
    if ((rc = x_map(&mbh, bhi, N, 2 * XKP, N))) return rc;
    if ((rc = x_map(&mbl, blo, N, 2 * XKP, N))) return rc;
    const size_t smem = L.total + 1024;
    XTS_CUDA(cudaFuncSetAttribute(k_exposure_map_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    // as many blocks per SM as shared memory allows, within the 512 tensor-memory
    // columns of an SM (each block allocates its accumulator's columns): the blocks'
    // load -> split -> MMA -> epilogue chains overlap one another
    int per_sm = 1;
    XTS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_exposure_map_tc, XM, smem));
    const int ncols = N <= 32 ? 32 : (N <= 64 ? 64 : (N <= 128 ? 128 : 256));
    per_sm = per_sm < 1 ? 1 : per_sm;
    per_sm = per_sm > 512 / ncols ? 512 / ncols : per_sm;
    const long long ntiles = (npix + XM - 1) / XM;
    const int G = (int)(ntiles < (long long)per_sm * nsm ? ntiles : (long long)per_sm * nsm);
    XTS_LAUNCH("k_exposure_map_tc", st, k_exposure_map_tc<<<G, XM, smem, st>>>(mx, mw, mbh, mbl, (int)npix, E, out,
                                                                                status));
    return XTS_OK;
}

}  // namespace xts
