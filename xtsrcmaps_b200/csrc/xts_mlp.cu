// xts_mlp.cu -- the surrogate network of the pixel cubature: a 5 -> 128 -> 128 ->
// 128 -> 1 perceptron with tanh-form GELU (Hendrycks & Gimpel, "Gaussian Error
// Linear Units", 2016: gelu(z) = z/2 (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3)))),
// its forward pass, its gradient and an Adam update (Kingma & Ba, 2015).
//
// The two 128 x 128 layers run on tcgen05 tensor cores: BF16 operands in shared
// memory (K-major, 128-byte swizzle: a [128 rows][64] BF16 atom is 16 KB, rows
// of 128 bytes whose 16-byte chunks are permuted by row & 7, 8-row groups 1024
// bytes apart), one thread issuing tcgen05.mma.kind::f16 (M = N = 128, K = 16)
// into an FP32 accumulator of 128 tensor-memory columns, the four warps reading
// it back with tcgen05.ld (warp w owns lanes 32w..32w+31 = rows of the tile).
//
//   * k_mlp_forward: one tile of 128 rows per step of a persistent loop, two
//     blocks of two warpgroups per SM (each row's 128 columns split between two
//     threads).  Layer 1 (K = 5) and the GELUs on CUDA cores; each hidden layer's
//     BF16 activations are written by their row's threads straight into the
//     swizzled A operand of the next MMA; the output layer is a per-row dot
//     product.  For training it
//     also writes the pre-activations z1..z3 and the activations h1, h2,
//     transposed ([128][n], coalesced across the threads of a warp).
//   * k_gemm_bf16: C = A B^T for the backward pass (dW = dZ^T H, dH = dZ W), with
//     either operand given transposed (gathered into the swizzled layout by the
//     loading threads), a two-stage shared-memory ring and split-K whose partial
//     tiles are summed in a fixed order (k_sum_splits), so training is
//     reproducible.
//   * k_mlp_bwd_elem: dZ = dH * gelu'(Z) per layer in the [unit][row] layout, with
//     the bias (and output-layer and first-layer weight) gradients reduced per
//     block into partials that k_bwd_reduce sums in a fixed order.
//   * k_mlp_adam: the update of the FP32 master parameters and the BF16 copies.
//
// Every mbarrier wait is bounded (WAIT_LIMIT polls); a timeout sets the status
// word, stops issuing work, lets issued MMAs complete (bounded) and frees the
// tensor memory.
#include <cuda_bf16.h>

#include "xts_point.cuh"

namespace xts {

constexpr int MH = XTS_MLP_HID;  // hidden width == MMA N
constexpr int MI = XTS_MLP_IN;
constexpr int MT = 128;          // rows per tile == MMA M == threads per block
constexpr int ATOM = 16384;      // bytes of a [128][64] BF16 swizzled atom

static_assert(MH == 128 && MT == 128, "the MMA shapes below assume 128 x 128 tiles");

struct MlpNorm {
    float mu[MI], sd[MI], out_mu, out_sd;
};

static MlpNorm mlp_norm(const xts_mlp* net) {
    MlpNorm m;
    for (int k = 0; k < MI; ++k) { m.mu[k] = net->in_mu[k]; m.sd[k] = net->in_sd[k]; }
    m.out_mu = net->out_mu;
    m.out_sd = net->out_sd;
    return m;
}

__device__ __forceinline__ float tanh_fast(float x) {
    float r;
    asm("tanh.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
constexpr float GK0 = 0.7978845608028654f;  // sqrt(2 / pi)
constexpr float GK1 = 0.044715f;
__device__ __forceinline__ float gelu(float z) {
    return 0.5f * z * (1.f + tanh_fast(GK0 * fmaf(GK1 * z * z, z, z)));
}
// two GELUs with packed FP32 arithmetic (same formula as gelu, rounding order differs)
__device__ __forceinline__ float2 gelu2(float2 z) {
    const float2 t = __ffma2_rn(make_float2(GK1, GK1), __fmul2_rn(z, z), make_float2(1.f, 1.f));
    const float2 u = __fmul2_rn(__fmul2_rn(make_float2(GK0, GK0), z), t);
    const float2 hz = __fmul2_rn(make_float2(0.5f, 0.5f), z);
    return __ffma2_rn(hz, make_float2(tanh_fast(u.x), tanh_fast(u.y)), hz);
}
// 2 gelu(z) for two values: the same rounding as gelu2 scaled by 2 (exact), one
// multiply fewer; the inference kernel halves the next layer's weights to match
__device__ __forceinline__ float2 gelu2x(float2 z) {
    const float2 t = __ffma2_rn(make_float2(GK1, GK1), __fmul2_rn(z, z), make_float2(1.f, 1.f));
    const float2 u = __fmul2_rn(__fmul2_rn(make_float2(GK0, GK0), z), t);
    return __ffma2_rn(z, make_float2(tanh_fast(u.x), tanh_fast(u.y)), z);
}
__device__ __forceinline__ float gelu_grad(float z) {
    const float z2 = z * z, th = tanh_fast(GK0 * fmaf(GK1 * z2, z, z));
    return 0.5f * (1.f + th) + 0.5f * z * (1.f - th * th) * GK0 * fmaf(3.f * GK1, z2, 1.f);
}

// byte offset of element (r, k) of a [128][K] BF16 operand made of [128][64] atoms
__device__ __forceinline__ unsigned sw_off(int r, int k) {
    return (unsigned)((k >> 6) * ATOM + r * 128 + ((((k & 63) >> 3) ^ (r & 7)) << 4) + (k & 7) * 2);
}

static __device__ __forceinline__ unsigned long long m_desc(unsigned addr) {
    // K-major, 128-byte swizzle: start >> 4, LBO 16 >> 4, SBO 1024 >> 4 (8-row groups), version 1
    return (unsigned long long)((addr >> 4) & 0x3FFF) | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}

// D f32, A and B bf16, both K-major, M = 128, N = 128.
constexpr unsigned M_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(MH >> 3) << 17) |
                             ((unsigned)(MT >> 4) << 24);

// K = 16 * nk of one MMA chain; a, b: shared addresses of the operands (atoms
// 16 KB apart); acc0: accumulate onto D from the first step.
__device__ __forceinline__ void mma_chain(unsigned tmem, unsigned a, unsigned b, int nk, bool acc0) {
    for (int ks = 0; ks < nk; ++ks) {
        const unsigned off = (unsigned)((ks >> 2) * ATOM + (ks & 3) * 32);
        const unsigned long long da = m_desc(a + off), db = m_desc(b + off);
        const unsigned acc = (acc0 || ks > 0) ? 1u : 0u;
        asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                     "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n"
                     :: "r"(tmem), "l"(da), "l"(db), "r"(M_IDESC), "r"(acc), "r"(0u));
    }
}

__device__ __forceinline__ void mma_commit(unsigned bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" :: "r"(bar) : "memory");
}

// 16 accumulator columns c0..c0+15 of this thread's row
__device__ __forceinline__ void tmem_ld16(unsigned taddr, float* v) {
    unsigned r[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

__device__ __forceinline__ unsigned pack_bf16(float a, float b) {
    const __nv_bfloat162 p = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const unsigned*>(&p);
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ unsigned tmem_alloc(unsigned slot_addr, unsigned ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" :: "r"(slot_addr), "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    return 0;
}
__device__ __forceinline__ void tmem_free(unsigned tmem, unsigned ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(ncols));
}

// ====================================================================== forward
constexpr int FT = 2 * MT;  // forward threads: two warpgroups, each row's 128 columns split in halves

struct FwdLayout {
    static constexpr size_t w2 = 0, w3 = 2 * ATOM, act = 4 * ATOM;
    // W1 transposed [5][128] and b1 [128] (six rows of 128), then 2 rows of padding, b2, b3,
    // w4 [128], b4 (+3), partial y [128]
    static constexpr size_t f32 = 6 * ATOM;
    static constexpr size_t bars = f32 + 4 * (MH * 8 + 3 * MH + 4 + MT);
    static constexpr size_t total = bars + 64;
};
constexpr size_t FWD_SMEM = FwdLayout::total + 1024;

struct FwdSaves {  // training only; all NULL for inference
    float* z1; float* z2; float* z3;  // [128][n]
    __nv_bfloat16* h1; __nv_bfloat16* h2;  // [128][n]
    float* yn;  // [n] standardised output
};

// Thread t works on row r = t & 127 of the tile and hidden columns [64 hf, 64 hf + 64),
// hf = t >> 7: warp w reads tensor-memory lanes 32 (w & 3).. and, in the A operand,
// writes the [128][64] atom hf of its rows.
// SAVE: training (pre-activations, activations and the standardised output saved;
// y unused); else inference (y only).
template <bool SAVE>
__global__ void __launch_bounds__(FT, 2)
k_mlp_forward(const float* __restrict__ params, const __nv_bfloat16* __restrict__ wbf, MlpNorm nm,
              const float* __restrict__ X, long long n, const unsigned long long* __restrict__ n_dev,
              long long ldx, float* __restrict__ y, FwdSaves sv, int* __restrict__ status) {
    if (n_dev) n = min(n, (long long)*n_dev);  // rows counted on the device (at most n)
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* smem = smem_raw + ((1024 - (smem_u32(smem_raw) & 1023)) & 1023);
    const int t = threadIdx.x, warp = t >> 5, r = t & (MT - 1), hf = t >> 7, cb = 64 * hf;
    float* w1 = (float*)(smem + FwdLayout::f32);  // [6][128]: W1^T rows, then b1
    float* b2 = w1 + MH * 8;
    float* b3 = b2 + MH;
    float* w4 = b3 + MH;
    float* b4 = w4 + MH;
    float* ypart = b4 + 4;
    unsigned long long* bars = (unsigned long long*)(smem + FwdLayout::bars);
    unsigned* tmem_slot = (unsigned*)(smem + FwdLayout::bars + 32);
    const unsigned bar = smem_u32(&bars[0]);
    const unsigned s_w2 = smem_u32(smem + FwdLayout::w2), s_w3 = smem_u32(smem + FwdLayout::w3);
    const unsigned s_act = smem_u32(smem + FwdLayout::act);

    // weights: W2, W3 [out][in] BF16 -> swizzled B operands (row = out, K = in)
    for (int idx = t; idx < 2 * MH * (MH / 8); idx += FT) {
        const int l = idx / (MH * (MH / 8)), rem = idx - l * (MH * (MH / 8));
        const int row = rem >> 4, ch = rem & 15;
        const uint4 v = *reinterpret_cast<const uint4*>(wbf + (size_t)l * MH * MH + row * MH + ch * 8);
        *reinterpret_cast<uint4*>(smem + (l ? FwdLayout::w3 : FwdLayout::w2) + sw_off(row, ch * 8)) = v;
    }
    for (int k = t; k < MH * 8; k += FT) {
        const int q = k >> 7, j = k & (MH - 1);
        w1[k] = q < MI ? __bfloat162float(__float2bfloat16_rn(params[XTS_MLP_W1 + j * MI + q]))
                       : (q == MI ? params[XTS_MLP_B1 + j] : 0.f);
    }
    for (int k = t; k < MH; k += FT) {
        b2[k] = params[XTS_MLP_B2 + k];
        b3[k] = params[XTS_MLP_B3 + k];
        w4[k] = __bfloat162float(__float2bfloat16_rn(params[XTS_MLP_W4 + k]));
    }
    if (t == 0) {
        b4[0] = params[XTS_MLP_B4];
        mbar_init(bar, 1);
    }
    if (warp == 0) tmem_alloc(smem_u32(tmem_slot), 128);
    fence_async_shared();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const unsigned tmem = *tmem_slot;
    const unsigned trow = tmem + ((unsigned)((warp & 3) * 32) << 16) + (unsigned)cb;
    unsigned ph = 0;
    bool ok = true;
    const long long ntiles = (n + MT - 1) / MT;
    // layer 1 of tile tl on CUDA cores: this thread's 64 BF16 activations of its row
    auto layer1 = [&](long long tl, uint4* hq) {
        const long long rw = tl * MT + r;
        const bool lv = rw < n;
        float x[MI];
#pragma unroll
        for (int k = 0; k < MI; ++k)
            x[k] = lv ? (X[ldx ? k * ldx + rw : rw * MI + k] - nm.mu[k]) / nm.sd[k] : 0.f;
#pragma unroll
        for (int g = 0; g < 8; ++g) {
            const int j0 = cb + 8 * g;
            float h[8];
#pragma unroll
            for (int j = 0; j < 8; j += 2) {
                const float2* wp = reinterpret_cast<const float2*>(w1 + j0 + j);  // units j0 + j, j0 + j + 1
                float2 z = wp[MI * MH / 2];  // b1
#pragma unroll
                for (int k = 0; k < MI; ++k) z = __ffma2_rn(wp[k * MH / 2], make_float2(x[k], x[k]), z);
                const float2 g2 = gelu2(z);
                h[j] = g2.x;
                h[j + 1] = g2.y;
                if (SAVE && lv) {
                    sv.z1[(size_t)(j0 + j) * n + rw] = z.x;
                    sv.z1[(size_t)(j0 + j + 1) * n + rw] = z.y;
                }
            }
            hq[g] = make_uint4(pack_bf16(h[0], h[1]), pack_bf16(h[2], h[3]), pack_bf16(h[4], h[5]),
                               pack_bf16(h[6], h[7]));
            if (SAVE && lv) {
                const __nv_bfloat16* hb = reinterpret_cast<const __nv_bfloat16*>(&hq[g]);
#pragma unroll
                for (int j = 0; j < 8; ++j) sv.h1[(size_t)(j0 + j) * n + rw] = hb[j];
            }
        }
    };
    uint4 hq[8];
    if (!SAVE && (long long)blockIdx.x < ntiles) layer1(blockIdx.x, hq);
    for (long long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const long long row = tile * MT + r;
        const bool live = row < n;
        // the A operand of layer 2: this tile's layer 1 (for inference computed while the
        // previous tile's last MMA ran; the MMA that read the buffer has completed)
        if (SAVE) layer1(tile, hq);
#pragma unroll
        for (int g = 0; g < 8; ++g) *reinterpret_cast<uint4*>(smem + FwdLayout::act + sw_off(r, cb + 8 * g)) = hq[g];
        float yacc = 0.f;
        for (int layer = 2; layer <= 3 && ok; ++layer) {
            fence_async_shared();
            tc_fence_before();
            __syncthreads();
            if (t == 0) {
                tc_fence_after();
                mma_chain(tmem, s_act, layer == 2 ? s_w2 : s_w3, MH / 16, false);
                mma_commit(bar);
            }
            // inference: layer 1 of the next tile in registers while the last MMA of this one runs
            if (!SAVE && layer == 3 && tile + gridDim.x < ntiles) layer1(tile + gridDim.x, hq);
            const bool got = mbar_wait(bar, ph);
            if (!__syncthreads_and(got)) { ok = false; break; }  // ph stays: the exit path waits on it
            ph ^= 1;
            tc_fence_after();
            const float* bias = layer == 2 ? b2 : b3;
            float* zs = SAVE ? (layer == 2 ? sv.z2 : sv.z3) : nullptr;
            for (int c0 = 0; c0 < 64; c0 += 16) {
                float v[16], bv[16];
                tmem_ld16(trow + (unsigned)c0, v);
                const int cc = cb + c0;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float4 b = reinterpret_cast<const float4*>(bias + cc)[q];
                    bv[4 * q] = b.x; bv[4 * q + 1] = b.y; bv[4 * q + 2] = b.z; bv[4 * q + 3] = b.w;
                }
#pragma unroll
                for (int j = 0; j < 16; j += 2) {
                    const float2 z = __fadd2_rn(make_float2(v[j], v[j + 1]), make_float2(bv[j], bv[j + 1]));
                    if (SAVE && live) {
                        zs[(size_t)(cc + j) * n + row] = z.x;
                        zs[(size_t)(cc + j + 1) * n + row] = z.y;
                    }
                    const float2 g2 = gelu2(z);
                    v[j] = g2.x;
                    v[j + 1] = g2.y;
                }
                if (layer == 2) {
#pragma unroll
                    for (int q = 0; q < 2; ++q) {
                        const float* u = v + 8 * q;
                        uint4 pk = make_uint4(pack_bf16(u[0], u[1]), pack_bf16(u[2], u[3]), pack_bf16(u[4], u[5]),
                                              pack_bf16(u[6], u[7]));
                        if (SAVE && live) {
                            const __nv_bfloat16* hb = reinterpret_cast<const __nv_bfloat16*>(&pk);
#pragma unroll
                            for (int j = 0; j < 8; ++j) sv.h2[(size_t)(cc + 8 * q + j) * n + row] = hb[j];
                        }
                        *reinterpret_cast<uint4*>(smem + FwdLayout::act + sw_off(r, cc + 8 * q)) = pk;
                    }
                } else {
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const float4 wv = reinterpret_cast<const float4*>(w4 + cc)[q];
                        yacc = fmaf(v[4 * q], wv.x, fmaf(v[4 * q + 1], wv.y, fmaf(v[4 * q + 2], wv.z,
                                                                                   fmaf(v[4 * q + 3], wv.w, yacc))));
                    }
                }
            }
        }
        if (!ok) break;
        if (hf) ypart[r] = yacc;
        tc_fence_before();  // the next tile's MMA overwrites the accumulator read above
        __syncthreads();
        if (!hf && live) {
            const float yn = (yacc + ypart[r]) + b4[0];
            if (SAVE) sv.yn[row] = yn;
            else y[row] = fmaf(yn, nm.out_sd, nm.out_mu);
        }
    }
    if (!ok && t == 0) {
        atomicExch(status, 1);
        mbar_wait(bar, ph);  // bounded: let an issued MMA land
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) tmem_free(tmem, 128);
}

// ====================================================================== inference
// k_mlp_infer: the same forward arithmetic as k_mlp_forward<false>, with four tiles in
// flight per SM.  One block per SM of four warpgroups; warpgroup g owns tile slot g
// (its BF16 activation operand and accumulator columns [128 g, 128 g + 128) of tensor
// memory) and runs its own tiles, thread = row, all 128 columns per thread; the two
// weight operands are shared.  A warpgroup synchronises only with itself (named
// barrier 1 + g, its own mbarrier), so while one waits for its MMAs the other three
// run their GELUs: the tensor pipe, the FMA pipe and the tanh unit overlap across
// the four tiles.  The hidden activations are kept as 2 gelu(z) (gelu2x, one multiply
// fewer per value) and the weights that read them (W2, W3, w4) are halved on loading;
// both scalings are exact, so the outputs are those of k_mlp_forward bit for bit.
constexpr int IG = 4;                    // warpgroups (tile slots) per block
constexpr int IT = IG * MT;              // threads per block
struct InfLayout {
    static constexpr size_t w2 = 0, w3 = 2 * ATOM, act = 4 * ATOM;  // act: IG slots of 2 atoms
    static constexpr size_t f32 = act + (size_t)IG * 2 * ATOM;      // W1^T [5][128], b1, pad, b2, b3, w4, b4
    static constexpr size_t bars = f32 + 4 * (MH * 8 + 3 * MH + 4);
    static constexpr size_t total = bars + 64;
};
constexpr size_t INF_SMEM = InfLayout::total + 1024;

__device__ __forceinline__ void group_sync(int g) {
    asm volatile("bar.sync %0, %1;" :: "r"(1 + g), "r"(MT) : "memory");
}
__device__ __forceinline__ bool group_and(int g, bool v) {
    int r;
    asm volatile("{\n\t.reg .pred p, q;\n\tsetp.ne.s32 p, %1, 0;\n\tbar.red.and.pred q, %2, %3, p;\n\t"
                 "selp.s32 %0, 1, 0, q;\n\t}\n" : "=r"(r) : "r"((int)v), "r"(1 + g), "r"(MT) : "memory");
    return r != 0;
}

__global__ void __launch_bounds__(IT, 1)
k_mlp_infer(const float* __restrict__ params, const __nv_bfloat16* __restrict__ wbf, MlpNorm nm,
            const float* __restrict__ X, long long n, const unsigned long long* __restrict__ n_dev,
            long long ldx, float* __restrict__ y, int* __restrict__ status) {
    if (n_dev) n = min(n, (long long)*n_dev);  // rows counted on the device (at most n)
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* smem = smem_raw + ((1024 - (smem_u32(smem_raw) & 1023)) & 1023);
    const int t = threadIdx.x, warp = t >> 5, g = t >> 7, r = t & (MT - 1);
    float* w1 = (float*)(smem + InfLayout::f32);  // [6][128]: W1^T rows, then b1
    float* b2 = w1 + MH * 8;
    float* b3 = b2 + MH;
    float* w4 = b3 + MH;
    float* b4 = w4 + MH;
    unsigned long long* bars = (unsigned long long*)(smem + InfLayout::bars);
    unsigned* tmem_slot = (unsigned*)(smem + InfLayout::bars + 8 * IG);
    const unsigned bar = smem_u32(&bars[g]);
    const unsigned s_w2 = smem_u32(smem + InfLayout::w2), s_w3 = smem_u32(smem + InfLayout::w3);
    unsigned char* act = smem + InfLayout::act + (size_t)g * 2 * ATOM;
    const unsigned s_act = smem_u32(act);

    for (int idx = t; idx < 2 * MH * (MH / 8); idx += IT) {
        const int l = idx / (MH * (MH / 8)), rem = idx - l * (MH * (MH / 8));
        const int row = rem >> 4, ch = rem & 15;
        uint4 v = *reinterpret_cast<const uint4*>(wbf + (size_t)l * MH * MH + row * MH + ch * 8);
        __nv_bfloat162* h2 = reinterpret_cast<__nv_bfloat162*>(&v);
#pragma unroll
        for (int q = 0; q < 4; ++q) h2[q] = __hmul2(h2[q], __float2bfloat162_rn(0.5f));  // exact: a power of 2
        *reinterpret_cast<uint4*>(smem + (l ? InfLayout::w3 : InfLayout::w2) + sw_off(row, ch * 8)) = v;
    }
    for (int k = t; k < MH * 8; k += IT) {
        const int q = k >> 7, j = k & (MH - 1);
        w1[k] = q < MI ? __bfloat162float(__float2bfloat16_rn(params[XTS_MLP_W1 + j * MI + q]))
                       : (q == MI ? params[XTS_MLP_B1 + j] : 0.f);
    }
    for (int k = t; k < MH; k += IT) {
        b2[k] = params[XTS_MLP_B2 + k];
        b3[k] = params[XTS_MLP_B3 + k];
        w4[k] = 0.5f * __bfloat162float(__float2bfloat16_rn(params[XTS_MLP_W4 + k]));
    }
    if (t < IG) mbar_init(smem_u32(&bars[t]), 1);
    if (t == 0) b4[0] = params[XTS_MLP_B4];
    if (warp == 0) tmem_alloc(smem_u32(tmem_slot), 128 * IG);
    fence_async_shared();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const unsigned tmem = *tmem_slot + (unsigned)(MH * g);  // this slot's accumulator columns
    const unsigned trow = tmem + ((unsigned)((warp & 3) * 32) << 16);
    unsigned ph = 0;
    bool ok = true;
    const long long ntiles = (n + MT - 1) / MT;
    const long long stride = (long long)gridDim.x * IG;
    // the features of this slot's next row, loaded one tile ahead
    float xn[MI];
    auto load_x = [&](long long tl) {
        const long long rw = tl * MT + r;
#pragma unroll
        for (int k = 0; k < MI; ++k) xn[k] = tl < ntiles && rw < n ? X[ldx ? k * ldx + rw : rw * MI + k] : 0.f;
    };
    load_x((long long)blockIdx.x * IG + g);
    for (long long tile = (long long)blockIdx.x * IG + g; tile < ntiles && ok; tile += stride) {
        const long long row = tile * MT + r;
        const bool live = row < n;
        // layer 1 on CUDA cores, the row's 128 BF16 activations into the A operand
        {
            float x[MI];
#pragma unroll
            for (int k = 0; k < MI; ++k) x[k] = live ? (xn[k] - nm.mu[k]) / nm.sd[k] : 0.f;
            load_x(tile + stride);
#pragma unroll 2
            for (int g8 = 0; g8 < MH / 8; ++g8) {
                const int j0 = 8 * g8;
                float h[8];
#pragma unroll
                for (int j = 0; j < 8; j += 4) {
                    const float4* wp = reinterpret_cast<const float4*>(w1 + j0 + j);
                    const float4 bq = wp[MI * MH / 4];  // b1
                    float2 za = make_float2(bq.x, bq.y), zb = make_float2(bq.z, bq.w);
#pragma unroll
                    for (int k = 0; k < MI; ++k) {
                        const float4 wq = wp[k * MH / 4];
                        za = __ffma2_rn(make_float2(wq.x, wq.y), make_float2(x[k], x[k]), za);
                        zb = __ffma2_rn(make_float2(wq.z, wq.w), make_float2(x[k], x[k]), zb);
                    }
                    const float2 ga = gelu2x(za), gb = gelu2x(zb);
                    h[j] = ga.x; h[j + 1] = ga.y; h[j + 2] = gb.x; h[j + 3] = gb.y;
                }
                *reinterpret_cast<uint4*>(act + sw_off(r, j0)) =
                    make_uint4(pack_bf16(h[0], h[1]), pack_bf16(h[2], h[3]), pack_bf16(h[4], h[5]),
                               pack_bf16(h[6], h[7]));
            }
        }
        float ylo = 0.f, yhi = 0.f;  // the output layer over columns 0..63 and 64..127
        for (int layer = 2; layer <= 3 && ok; ++layer) {
            fence_async_shared();
            tc_fence_before();
            group_sync(g);
            if (r == 0) {
                tc_fence_after();
                mma_chain(tmem, s_act, layer == 2 ? s_w2 : s_w3, MH / 16, false);
                mma_commit(bar);
            }
            // one warp of the group polls the MMA's mbarrier; the other three sleep in the
            // group's barrier instead of spinning (their issue slots go to the other groups)
            bool got = true;
            if ((warp & 3) == 0) got = mbar_wait(bar, ph);
            if (!group_and(g, got)) { ok = false; break; }  // ph stays: the exit path waits on it
            ph ^= 1;
            tc_fence_after();
            const float* bias = layer == 2 ? b2 : b3;
#pragma unroll 1
            for (int c0 = 0; c0 < MH; c0 += 16) {
                float v[16], bv[16];
                tmem_ld16(trow + (unsigned)c0, v);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float4 b = reinterpret_cast<const float4*>(bias + c0)[q];
                    bv[4 * q] = b.x; bv[4 * q + 1] = b.y; bv[4 * q + 2] = b.z; bv[4 * q + 3] = b.w;
                }
#pragma unroll
                for (int j = 0; j < 16; j += 2) {
                    const float2 z = __fadd2_rn(make_float2(v[j], v[j + 1]), make_float2(bv[j], bv[j + 1]));
                    const float2 g2 = gelu2x(z);
                    v[j] = g2.x;
                    v[j + 1] = g2.y;
                }
                if (layer == 2) {
#pragma unroll
                    for (int q = 0; q < 2; ++q) {
                        const float* u = v + 8 * q;
                        *reinterpret_cast<uint4*>(act + sw_off(r, c0 + 8 * q)) =
                            make_uint4(pack_bf16(u[0], u[1]), pack_bf16(u[2], u[3]), pack_bf16(u[4], u[5]),
                                       pack_bf16(u[6], u[7]));
                    }
                } else {
                    float ya = c0 < 64 ? ylo : yhi;
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const float4 wv = reinterpret_cast<const float4*>(w4 + c0)[q];
                        ya = fmaf(v[4 * q], wv.x, fmaf(v[4 * q + 1], wv.y, fmaf(v[4 * q + 2], wv.z,
                                                                                fmaf(v[4 * q + 3], wv.w, ya))));
                    }
                    if (c0 < 64) ylo = ya; else yhi = ya;
                }
            }
            tc_fence_before();  // the next MMA overwrites the accumulator read above
        }
        if (!ok) break;
        if (live) y[row] = fmaf((ylo + yhi) + b4[0], nm.out_sd, nm.out_mu);
    }
    if (!ok && r == 0) {
        atomicExch(status, 1);
        mbar_wait(bar, ph);  // bounded: let this slot's issued MMA land
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) tmem_free(*tmem_slot, 128 * IG);
}

// ====================================================================== GEMM
constexpr size_t GEMM_SMEM = 4 * ATOM / 2 * 2 + 64 + 1024;  // two stages of A and B chunks ([128][64] each)

// Stage the [128 rows][64] chunk (rows r0.., K columns k0..) of an operand into
// one swizzled atom.  trans: the operand is stored [K][ld] (row index fastest).
__device__ __forceinline__ void load_chunk(unsigned char* dst, const __nv_bfloat16* src, int trans, long long ld,
                                           long long r0, long long k0, int t) {
    if (!trans) {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int idx = t + MT * i, r = idx >> 3, ch = idx & 7;
            const uint4 v = *reinterpret_cast<const uint4*>(src + (r0 + r) * ld + k0 + ch * 8);
            *reinterpret_cast<uint4*>(dst + sw_off(r, ch * 8)) = v;
        }
    } else {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int idx = t + MT * i, kk = idx >> 4, rg = idx & 15;
            const uint4 v = *reinterpret_cast<const uint4*>(src + (k0 + kk) * ld + r0 + rg * 8);
            const unsigned short* e = reinterpret_cast<const unsigned short*>(&v);
#pragma unroll
            for (int j = 0; j < 8; ++j) *reinterpret_cast<unsigned short*>(dst + sw_off(rg * 8 + j, kk)) = e[j];
        }
    }
}

__global__ void __launch_bounds__(MT, 1)
k_gemm_bf16(const __nv_bfloat16* __restrict__ A, int a_trans, const __nv_bfloat16* __restrict__ B, int b_trans,
            int M, int K, int cps, float* __restrict__ C, int c_trans, int atomic, int* __restrict__ status) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* smem = smem_raw + ((1024 - (smem_u32(smem_raw) & 1023)) & 1023);
    const int t = threadIdx.x, warp = t >> 5;
    const int nkc = K / 64;
    const int kc0 = blockIdx.y * cps, kc1 = min(kc0 + cps, nkc);
    if (kc0 >= kc1) return;  // uniform over the block, before any tensor memory is held
    const long long m0 = (long long)blockIdx.x * MT;
    unsigned long long* bars = (unsigned long long*)(smem + 4 * ATOM);
    unsigned* tmem_slot = (unsigned*)(smem + 4 * ATOM + 32);
    if (t == 0) {
        mbar_init(smem_u32(&bars[0]), 1);
        mbar_init(smem_u32(&bars[1]), 1);
    }
    if (warp == 0) tmem_alloc(smem_u32(tmem_slot), 128);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const unsigned tmem = *tmem_slot;
    unsigned ph[2] = {0, 0};
    int pending[2] = {0, 0};
    bool ok = true;
    for (int c = kc0; c < kc1; ++c) {
        const int st = (c - kc0) & 1;
        unsigned char* sa = smem + st * 2 * ATOM;
        unsigned char* sb = sa + ATOM;
        if (pending[st]) {  // the MMAs issued two chunks ago read this stage
            const bool got = mbar_wait(smem_u32(&bars[st]), ph[st]);
            if (!__syncthreads_and(got)) { ok = false; break; }  // still pending: the exit path waits
            ph[st] ^= 1;
            pending[st] = 0;
        }
        load_chunk(sa, A, a_trans, a_trans ? (long long)M : (long long)K, m0, (long long)c * 64, t);
        load_chunk(sb, B, b_trans, b_trans ? (long long)MH : (long long)K, 0, (long long)c * 64, t);
        fence_async_shared();
        tc_fence_before();
        __syncthreads();
        if (t == 0) {
            tc_fence_after();
            mma_chain(tmem, smem_u32(sa), smem_u32(sb), 4, c > kc0);
            mma_commit(smem_u32(&bars[st]));
        }
        pending[st] = 1;
    }
    // the last commit covers every MMA issued before it
    const int last = (kc1 - 1 - kc0) & 1;
    if (ok) {
        const bool got = mbar_wait(smem_u32(&bars[last]), ph[last]);
        ok = __syncthreads_and(got);
        if (ok) {
            ph[last] ^= 1;
            pending[last] = 0;
        }
    }
    if (ok) {
        tc_fence_after();
        const long long m = m0 + t;
        const unsigned trow = tmem + ((unsigned)(warp * 32) << 16);
        for (int c0 = 0; c0 < MH; c0 += 16) {
            float v[16];
            tmem_ld16(trow + (unsigned)c0, v);
            float* Cs = atomic ? C + (size_t)blockIdx.y * M * MH : C;  // split-K: this split's partial tile
#pragma unroll
            for (int j = 0; j < 16; ++j)
                *(c_trans ? Cs + (size_t)(c0 + j) * M + m : Cs + (size_t)m * MH + c0 + j) = v[j];
        }
    } else if (t == 0) {
        atomicExch(status, 1);
        for (int s = 0; s < 2; ++s)
            if (pending[s]) mbar_wait(smem_u32(&bars[s]), ph[s]);  // bounded
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) tmem_free(tmem, 128);
}

// ====================================================================== backward
// Per layer, in the [unit][row] layout: dz = dh * gelu'(z) (head: dh = dy * w4).
// Block (row range, unit j): bias gradient, and for the head the output-layer
// weight, for layer 1 the first-layer weights, reduced per block.
enum { BW_HEAD = 0, BW_HIDDEN = 1, BW_FIRST = 2 };
constexpr int BW_ROWS = 1024;  // rows per block (256 threads x 4)

__global__ void __launch_bounds__(256) k_mlp_bwd_elem(int mode, const float* __restrict__ params, MlpNorm nm,
                                                      const float* __restrict__ zT, const float* __restrict__ dhT,
                                                      const float* __restrict__ yn, const float* __restrict__ Y,
                                                      const float* __restrict__ X, long long n,
                                                      __nv_bfloat16* __restrict__ dzT,
                                                      float* __restrict__ part) {
    __shared__ float red[8][8];
    const int j = blockIdx.y, t = threadIdx.x, lane = t & 31, wp = t >> 5;
    const float w4 = __bfloat162float(__float2bfloat16_rn(params[XTS_MLP_W4 + j]));
    const float inv_n = 1.f / (float)n;
    // accumulators: 0 bias, 1 w4 (head) / dy (head, unit 0), 2 loss, 3..7 first-layer weights
    float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    const long long r0 = (long long)blockIdx.x * BW_ROWS;
    for (int i = 0; i < BW_ROWS / 256; ++i) {
        const long long r = r0 + t + 256 * i;
        if (r >= n) break;
        const size_t k = (size_t)j * n + r;
        const float z = zT[k];
        float dh;
        if (mode == BW_HEAD) {
            const float tgt = (Y[r] - nm.out_mu) / nm.out_sd;
            const float d = yn[r] - tgt;
            const float dy = 2.f * d * inv_n;
            dh = dy * w4;
            acc[1] = fmaf(dy, gelu(z), acc[1]);
            if (j == 0) { acc[2] = fmaf(d, d, acc[2]); acc[3] += dy; }
        } else {
            dh = dhT[k];
        }
        const float dz = dh * gelu_grad(z);
        acc[0] += dz;
        if (mode == BW_FIRST) {
#pragma unroll
            for (int q = 0; q < MI; ++q) acc[3 + q] = fmaf(dz, (X[r * MI + q] - nm.mu[q]) / nm.sd[q], acc[3 + q]);
        } else {
            dzT[k] = __float2bfloat16_rn(dz);
        }
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        float v = acc[q];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) red[wp][q] = v;
    }
    __syncthreads();
    if (t < 8) {
        float v = 0.f;
        for (int w = 0; w < 8; ++w) v += red[w][t];
        part[((size_t)blockIdx.x * MH + j) * 8 + t] = v;
    }
}

// The per-block partials of k_mlp_bwd_elem summed over the row blocks in order and
// added to the gradient (and the loss); one thread per (unit, quantity).
__global__ void k_bwd_reduce(int mode, const float* __restrict__ part, int nbx, float inv_n,
                             float* __restrict__ grads, float* __restrict__ loss) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= MH * 8) return;
    const int j = i >> 3, q = i & 7;
    float v = 0.f;
    for (int b = 0; b < nbx; ++b) v += part[((size_t)b * MH + j) * 8 + q];
    if (mode == BW_HEAD) {
        if (q == 0) grads[XTS_MLP_B3 + j] += v;
        if (q == 1) grads[XTS_MLP_W4 + j] += v;
        if (j == 0 && q == 2 && loss) *loss += v * inv_n;
        if (j == 0 && q == 3) grads[XTS_MLP_B4] += v;
    } else if (mode == BW_HIDDEN) {
        if (q == 0) grads[XTS_MLP_B2 + j] += v;
    } else {
        if (q == 0) grads[XTS_MLP_B1 + j] += v;
        if (q >= 3 && q < 3 + MI) grads[XTS_MLP_W1 + j * MI + (q - 3)] += v;
    }
}

// C[i] += sum over the splits s (in order) of part[s][i]
__global__ void k_sum_splits(const float* __restrict__ part, int nsplit, long long n, float* __restrict__ C) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float v = 0.f;
    for (int s = 0; s < nsplit; ++s) v += part[(size_t)s * n + i];
    C[i] += v;
}

// Adam on the FP32 master parameters; the BF16 copies of W2 and W3 follow.
__global__ void k_mlp_adam(float* __restrict__ p, float* __restrict__ g, float* __restrict__ m,
                           float* __restrict__ v, __nv_bfloat16* __restrict__ wbf, float lr, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= XTS_MLP_NPARAM) return;
    const float gi = g[i];
    const float mi = fmaf(0.9f, m[i], 0.1f * gi);
    const float vi = fmaf(0.999f, v[i], 0.001f * gi * gi);
    m[i] = mi;
    v[i] = vi;
    g[i] = 0.f;
    const float pi = p[i] - lr * (mi * c1) / (sqrtf(vi * c2) + 1e-8f);
    p[i] = pi;
    if (i >= XTS_MLP_W2 && i < XTS_MLP_B2) wbf[i - XTS_MLP_W2] = __float2bfloat16_rn(pi);
    if (i >= XTS_MLP_W3 && i < XTS_MLP_B3) wbf[MH * MH + (i - XTS_MLP_W3)] = __float2bfloat16_rn(pi);
}

// ====================================================================== launchers
static int sm_count() {
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    return nsm;
}

static int mlp_status(int* status, cudaStream_t st) {
    int v = 0;
    XTS_CUDA(cudaMemcpyAsync(&v, status, sizeof(int), cudaMemcpyDeviceToHost, st));
    XTS_CUDA(cudaStreamSynchronize(st));
    if (v) {
        cudaMemsetAsync(status, 0, sizeof(int), st);
        return set_error(XTS_ERR_TIMEOUT, "a bounded tensor-core wait gave up (surrogate network)");
    }
    return XTS_OK;
}

int launch_gemm_bf16(const void* A, int a_trans, const void* B, int b_trans, int M, int K, float* C, int c_trans,
                     int accumulate, int* status, cudaStream_t st) {
    if (M <= 0 || K <= 0 || M % MT || K % 64)
        return set_error(XTS_ERR_ARG, "gemm_bf16: M (%d) must be a multiple of 128 and K (%d) of 64", M, K);
    XTS_CUDA(cudaFuncSetAttribute(k_gemm_bf16, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GEMM_SMEM));
    const int mt = M / MT, nkc = K / 64;
    int nsplit = 1;
    if (accumulate) {  // spread the K chunks over about one wave of blocks
        nsplit = (sm_count() + mt - 1) / mt;
        nsplit = nsplit < 1 ? 1 : (nsplit > nkc ? nkc : nsplit);
    }
    const int cps = (nkc + nsplit - 1) / nsplit;
    nsplit = (nkc + cps - 1) / cps;
    if (!accumulate && nsplit != 1) return set_error(XTS_ERR_ARG, "gemm_bf16: internal split");
    float* dst = C;
    const long long nc = (long long)M * MH;
    if (accumulate) {  // partial tiles per split, summed in a fixed order below
        dst = (float*)workspace(W_MLP_PART, sizeof(float) * (size_t)nsplit * nc);
        if (!dst) return XTS_ERR_OOM;
    }
    XTS_LAUNCH("k_gemm_bf16", st, k_gemm_bf16<<<dim3(mt, nsplit), MT, GEMM_SMEM, st>>>(
                                      (const __nv_bfloat16*)A, a_trans, (const __nv_bfloat16*)B, b_trans, M, K, cps,
                                      dst, c_trans, accumulate, status));
    if (accumulate)
        XTS_LAUNCH("k_sum_splits", st, k_sum_splits<<<(unsigned)((nc + 255) / 256), 256, 0, st>>>(dst, nsplit, nc, C));
    return XTS_OK;
}

// X: row-major [n][5] (ldx 0) or feature-major [5][ldx] (ldx >= n)
static int forward(const xts_mlp* net, const float* X, long long n, const unsigned long long* n_dev, float* y,
                   FwdSaves sv, int* status, cudaStream_t st, long long ldx = 0) {
    // per call: the attribute belongs to the current device's context
    XTS_CUDA(cudaFuncSetAttribute(k_mlp_forward<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)FWD_SMEM));
    XTS_CUDA(cudaFuncSetAttribute(k_mlp_forward<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)FWD_SMEM));
    const bool save = sv.z1 != nullptr;
    if (save && !(sv.z2 && sv.z3 && sv.h1 && sv.h2 && sv.yn)) return set_error(XTS_ERR_ARG, "mlp forward: saves");
    if (!save && !y) return set_error(XTS_ERR_ARG, "mlp forward: output");
    const long long ntiles = (n + MT - 1) / MT;
    const int bps = g_tuning.mlp_blocks_per_sm > 0 ? g_tuning.mlp_blocks_per_sm : 2;  // blocks per SM (two fit)
    const long long g = ntiles < bps * sm_count() ? ntiles : bps * sm_count();
    if (save) {
        XTS_LAUNCH("k_mlp_forward", st, k_mlp_forward<true><<<(unsigned)g, FT, FWD_SMEM, st>>>(
                                            net->params, (const __nv_bfloat16*)net->wbf16, mlp_norm(net), X, n, n_dev,
                                            ldx, y, sv, status));
    } else if (g_tuning.mlp_blocks_per_sm == 0) {
        // inference: four tiles in flight per SM, one block per SM
        XTS_CUDA(cudaFuncSetAttribute(k_mlp_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)INF_SMEM));
        const long long gi = (ntiles + IG - 1) / IG < sm_count() ? (ntiles + IG - 1) / IG : sm_count();
        XTS_LAUNCH("k_mlp_infer", st, k_mlp_infer<<<(unsigned)gi, IT, INF_SMEM, st>>>(
                                            net->params, (const __nv_bfloat16*)net->wbf16, mlp_norm(net), X, n, n_dev,
                                            ldx, y, status));
    } else {
        XTS_LAUNCH("k_mlp_forward", st, k_mlp_forward<false><<<(unsigned)g, FT, FWD_SMEM, st>>>(
                                            net->params, (const __nv_bfloat16*)net->wbf16, mlp_norm(net), X, n, n_dev,
                                            ldx, y, sv, status));
    }
    return XTS_OK;
}

int launch_mlp_forward(const xts_mlp* net, const float* X, long long n, float* y, int* status, cudaStream_t st) {
    if (n <= 0) return XTS_OK;
    return forward(net, X, n, nullptr, y, FwdSaves{}, status, st);
}

int launch_mlp_forward_dev(const xts_mlp* net, const float* X, const unsigned long long* n_dev, long long n_max,
                           float* y, int* status, cudaStream_t st, long long ldx) {
    if (n_max <= 0) return XTS_OK;
    if (ldx && ldx < n_max) return set_error(XTS_ERR_ARG, "mlp forward: feature stride below the row count");
    return forward(net, X, n_max, n_dev, y, FwdSaves{}, status, st, ldx);
}

// forward with saves, then the gradient accumulated into grads (zero on entry)
static int mlp_backprop(const xts_mlp* net, const float* X, const float* Y, long long n, float* grads,
                        float* loss, int* status, cudaStream_t st) {
    if (n <= 0 || n % MT) return set_error(XTS_ERR_ARG, "surrogate training: n (%lld) must be a positive multiple of 128", n);
    if (n > (1ll << 24)) return set_error(XTS_ERR_ARG, "surrogate training: n (%lld) above 2^24 rows per batch", n);
    const size_t hn = (size_t)MH * n;
    float* z = (float*)workspace(W_MLP_Z, sizeof(float) * 3 * hn);
    __nv_bfloat16* h = (__nv_bfloat16*)workspace(W_MLP_H, sizeof(__nv_bfloat16) * 2 * hn);
    __nv_bfloat16* dz = (__nv_bfloat16*)workspace(W_MLP_DZ, sizeof(__nv_bfloat16) * hn);
    float* dh = (float*)workspace(W_MLP_DH, sizeof(float) * hn);
    float* yn = (float*)workspace(W_MLP_Y, sizeof(float) * n);
    if (!z || !h || !dz || !dh || !yn) return XTS_ERR_OOM;
    FwdSaves sv{z, z + hn, z + 2 * hn, h, h + hn, yn};
    int rc = forward(net, X, n, nullptr, nullptr, sv, status, st);
    if (rc) return rc;
    const MlpNorm nm = mlp_norm(net);
    const int nbx = (int)((n + BW_ROWS - 1) / BW_ROWS);
    const dim3 eg((unsigned)nbx, MH);
    const float inv_n = 1.f / (float)n;
    float* part = (float*)workspace(W_MLP_PART2, sizeof(float) * (size_t)nbx * MH * 8);
    if (!part) return XTS_ERR_OOM;
    const __nv_bfloat16* w2 = (const __nv_bfloat16*)net->wbf16;
    const __nv_bfloat16* w3 = w2 + MH * MH;
    // head: dz3 = dy w4 gelu'(z3); dW3 = dz3^T h2; dh2 = dz3 W3
    XTS_LAUNCH("k_mlp_bwd", st, k_mlp_bwd_elem<<<eg, 256, 0, st>>>(BW_HEAD, net->params, nm, sv.z3, nullptr, yn, Y,
                                                                     X, n, dz, part));
    XTS_LAUNCH("k_bwd_reduce", st, k_bwd_reduce<<<(MH * 8 + 255) / 256, 256, 0, st>>>(BW_HEAD, part, nbx, inv_n,
                                                                                      grads, loss));
    if ((rc = launch_gemm_bf16(dz, 0, sv.h2, 0, MH, (int)n, grads + XTS_MLP_W3, 0, 1, status, st))) return rc;
    if ((rc = launch_gemm_bf16(dz, 1, w3, 1, (int)n, MH, dh, 1, 0, status, st))) return rc;
    // layer 2: dz2 = dh2 gelu'(z2); dW2 = dz2^T h1; dh1 = dz2 W2
    XTS_LAUNCH("k_mlp_bwd", st, k_mlp_bwd_elem<<<eg, 256, 0, st>>>(BW_HIDDEN, net->params, nm, sv.z2, dh, yn, Y, X,
                                                                     n, dz, part));
    XTS_LAUNCH("k_bwd_reduce", st, k_bwd_reduce<<<(MH * 8 + 255) / 256, 256, 0, st>>>(BW_HIDDEN, part, nbx, inv_n,
                                                                                      grads, loss));
    if ((rc = launch_gemm_bf16(dz, 0, sv.h1, 0, MH, (int)n, grads + XTS_MLP_W2, 0, 1, status, st))) return rc;
    if ((rc = launch_gemm_bf16(dz, 1, w2, 1, (int)n, MH, dh, 1, 0, status, st))) return rc;
    // layer 1: dz1 = dh1 gelu'(z1); dW1 = dz1^T x
    XTS_LAUNCH("k_mlp_bwd", st, k_mlp_bwd_elem<<<eg, 256, 0, st>>>(BW_FIRST, net->params, nm, sv.z1, dh, yn, Y, X,
                                                                     n, dz, part));
    XTS_LAUNCH("k_bwd_reduce", st, k_bwd_reduce<<<(MH * 8 + 255) / 256, 256, 0, st>>>(BW_FIRST, part, nbx, inv_n,
                                                                                      grads, loss));
    return XTS_OK;
}

int launch_mlp_grads(const xts_mlp* net, const float* X, const float* Y, long long n, float* grads, float* loss,
                     int* status, cudaStream_t st) {
    XTS_CUDA(cudaMemsetAsync(grads, 0, sizeof(float) * XTS_MLP_NPARAM, st));
    if (loss) XTS_CUDA(cudaMemsetAsync(loss, 0, sizeof(float), st));
    int rc = mlp_backprop(net, X, Y, n, grads, loss, status, st);
    if (rc) return rc;
    return mlp_status(status, st);
}

int launch_mlp_train_step(const xts_mlp* net, const float* X, const float* Y, long long n, float* grads,
                          float* m, float* v, int step, float lr, float* loss, int* status, cudaStream_t st) {
    if (step < 1) return set_error(XTS_ERR_ARG, "surrogate training: step must be >= 1");
    int rc = mlp_backprop(net, X, Y, n, grads, loss, status, st);
    if (rc) return rc;
    const float c1 = (float)(1.0 / (1.0 - pow(0.9, step))), c2 = (float)(1.0 / (1.0 - pow(0.999, step)));
    XTS_LAUNCH("k_mlp_adam", st, k_mlp_adam<<<(XTS_MLP_NPARAM + 255) / 256, 256, 0, st>>>(
                                     net->params, grads, m, v, (__nv_bfloat16*)net->wbf16, lr, c1, c2));
    return XTS_OK;
}

int mlp_check_status(int* status, cudaStream_t st) { return mlp_status(status, st); }

}  // namespace xts
