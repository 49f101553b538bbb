// xts_mlp.cu -- the surrogate network of the pixel cubature: a 5 -> 128 -> 128 ->
// 128 -> 1 perceptron with tanh-form GELU (Hendrycks & Gimpel, "Gaussian Error
// Linear Units", 2016: gelu(z) = z/2 (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3)))),
// its forward pass, its gradient and an Adam update (Kingma & Ba, 2015).
//
// The three hidden layers run on tcgen05 tensor cores: BF16 operands in shared
// memory (K-major, 128-byte swizzle: a [128 rows][64] BF16 atom is 16 KB, rows
// of 128 bytes whose 16-byte chunks are permuted by row & 7, 8-row groups 1024
// bytes apart), one thread issuing tcgen05.mma.kind::f16 (M = N = 128, K = 16)
// into an FP32 accumulator of 128 tensor-memory columns, the four warps reading
// it back with tcgen05.ld (warp w owns lanes 32w..32w+31 = rows of the tile).
//
//   * k_mlp_forward: one tile of 128 rows per step of a persistent loop, two
//     blocks of two warpgroups per SM (each row's 128 columns split between two
//     threads).  Layer 1 (K = 5) is one K = 16 MMA over the features split into
//     three BF16 terms; the GELUs run on CUDA cores; each hidden layer's BF16
//     activations are written by their row's threads straight into the swizzled
//     A operand of the next MMA; the output layer is a per-row dot product.  For
//     training it
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
constexpr float GK0 = 0.7978845608028654f;   // sqrt(2 / pi)
constexpr float GK1 = 0.035677408136300125f; // sqrt(2 / pi) * 0.044715
// the tanh argument sqrt(2/pi) (z + 0.044715 z^3) as z (GK0 + GK1 z^2): two multiplies and
// one FMA
__device__ __forceinline__ float gelu_arg(float z) { return z * fmaf(z * z, GK1, GK0); }
__device__ __forceinline__ float gelu(float z) {
    return 0.5f * z * (1.f + tanh_fast(gelu_arg(z)));
}
__device__ __forceinline__ float2 gelu_arg2(float2 z) {
    return __fmul2_rn(z, __ffma2_rn(__fmul2_rn(z, z), make_float2(GK1, GK1), make_float2(GK0, GK0)));
}
// two GELUs with packed FP32 arithmetic (same formula as gelu, rounding order differs)
__device__ __forceinline__ float2 gelu2(float2 z) {
    const float2 u = gelu_arg2(z);
    const float2 hz = __fmul2_rn(make_float2(0.5f, 0.5f), z);
    return __ffma2_rn(hz, make_float2(tanh_fast(u.x), tanh_fast(u.y)), hz);
}
// 2 gelu(z) for two values: the same rounding as gelu2 scaled by 2 (exact), one
// multiply fewer; the inference kernel halves the next layer's weights to match
__device__ __forceinline__ float2 gelu2x(float2 z) {
    const float2 u = gelu_arg2(z);
    return __ffma2_rn(z, make_float2(tanh_fast(u.x), tanh_fast(u.y)), z);
}
__device__ __forceinline__ float gelu_grad(float z) {
    const float z2 = z * z, th = tanh_fast(z * fmaf(z2, GK1, GK0));
    return 0.5f * (1.f + th) + 0.5f * z * (1.f - th * th) * fmaf(3.f * GK1, z2, GK0);
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

// K-major without swizzle (layer 1's W1 operand, K = 16): core matrices of 8 rows x 16
// bytes, the two along K (leading byte offset) 128 bytes apart, 8-row groups (stride
// byte offset) 256 bytes apart; version 1, layout type 0
static __device__ __forceinline__ unsigned long long m_desc_ns(unsigned addr) {
    return (unsigned long long)((addr >> 4) & 0x3FFF) | ((unsigned long long)(128 >> 4) << 16) |
           ((unsigned long long)(256 >> 4) << 32) | (1ull << 46);
}
// byte offset of element (r, k) of that [128][16] BF16 operand
__device__ __forceinline__ unsigned ns_off(int r, int k) {
    return (unsigned)((r >> 3) * 256 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}
constexpr int W1OP = MH * 16 * 2;  // bytes of the W1 operand

// Layer 1 on the tensor cores.  A row of A holds the standardised features split into
// three BF16 terms, x = hi + mid + lo (each difference exact in FP32, so the sum
// equals x to 2^-27 relative), at K = 0..4, 5..9, 10..14; B holds W1 (already BF16)
// three times over, so one K = 16 MMA forms W1 x with every product exact.
__device__ __forceinline__ void fill_w1_operand(unsigned char* dst, const float* params, int t, int nt) {
    for (int e = t; e < MH * 16; e += nt) {
        const int j = e >> 4, k = e & 15;
        const __nv_bfloat16 w = k < 3 * MI ? __float2bfloat16_rn(params[XTS_MLP_W1 + j * MI + k % MI])
                                           : __float2bfloat16_rn(0.f);
        *reinterpret_cast<__nv_bfloat16*>(dst + ns_off(j, k)) = w;
    }
}
__device__ __forceinline__ void store_x_split(unsigned char* act, int r, const float* x) {
    unsigned short e[16];
#pragma unroll
    for (int k = 0; k < MI; ++k) {
        const __nv_bfloat16 hi = __float2bfloat16_rn(x[k]);
        const float r1 = x[k] - __bfloat162float(hi);
        const __nv_bfloat16 mid = __float2bfloat16_rn(r1);
        const __nv_bfloat16 lo = __float2bfloat16_rn(r1 - __bfloat162float(mid));
        e[k] = __bfloat16_as_ushort(hi);
        e[MI + k] = __bfloat16_as_ushort(mid);
        e[2 * MI + k] = __bfloat16_as_ushort(lo);
    }
    e[15] = 0;
    uint4 q[2];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        reinterpret_cast<unsigned*>(q)[i] = (unsigned)e[2 * i] | ((unsigned)e[2 * i + 1] << 16);
    }
    *reinterpret_cast<uint4*>(act + sw_off(r, 0)) = q[0];
    *reinterpret_cast<uint4*>(act + sw_off(r, 8)) = q[1];
}
// the layer-1 MMA: A = K columns 0..15 of the swizzled activation operand, B = W1
__device__ __forceinline__ void mma_layer1(unsigned tmem, unsigned a, unsigned w1op) {
    const unsigned long long da = m_desc(a), db = m_desc_ns(w1op);
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n"
                 :: "r"(tmem), "l"(da), "l"(db), "r"(M_IDESC), "r"(0u), "r"(0u));
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

// the same load without its wait, for a load kept in flight while other columns are
// worked on; tmem_ld_done waits for every load issued so far and ties r to that wait
__device__ __forceinline__ void tmem_ld16_issue(unsigned taddr, unsigned* r) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld_done(unsigned* r) {
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    // no use of r may be moved above the wait
    asm volatile("" : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                      "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15]));
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
    static constexpr size_t w2 = 0, w3 = 2 * ATOM, act = 4 * ATOM, w1 = 6 * ATOM;
    // b1, b2, b3, w4 [128 each], b4 (+3), partial y [128]
    static constexpr size_t f32 = w1 + W1OP;
    static constexpr size_t bars = f32 + 4 * (4 * MH + 4 + MT);
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
// writes the [128][64] atom hf of its rows.  All three layers run on the tensor cores
// (layer 1 as one K = 16 MMA over the split features); the GELUs on CUDA cores.
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
    float* b1 = (float*)(smem + FwdLayout::f32);
    float* b2 = b1 + MH;
    float* b3 = b2 + MH;
    float* w4 = b3 + MH;
    float* b4 = w4 + MH;
    float* ypart = b4 + 4;
    unsigned long long* bars = (unsigned long long*)(smem + FwdLayout::bars);
    unsigned* tmem_slot = (unsigned*)(smem + FwdLayout::bars + 32);
    const unsigned bar = smem_u32(&bars[0]);
    const unsigned s_w2 = smem_u32(smem + FwdLayout::w2), s_w3 = smem_u32(smem + FwdLayout::w3);
    const unsigned s_w1 = smem_u32(smem + FwdLayout::w1);
    const unsigned s_act = smem_u32(smem + FwdLayout::act);

    // weights: W2, W3 [out][in] BF16 -> swizzled B operands (row = out, K = in)
    for (int idx = t; idx < 2 * MH * (MH / 8); idx += FT) {
        const int l = idx / (MH * (MH / 8)), rem = idx - l * (MH * (MH / 8));
        const int row = rem >> 4, ch = rem & 15;
        const uint4 v = *reinterpret_cast<const uint4*>(wbf + (size_t)l * MH * MH + row * MH + ch * 8);
        *reinterpret_cast<uint4*>(smem + (l ? FwdLayout::w3 : FwdLayout::w2) + sw_off(row, ch * 8)) = v;
    }
    fill_w1_operand(smem + FwdLayout::w1, params, t, FT);
    for (int k = t; k < MH; k += FT) {
        b1[k] = params[XTS_MLP_B1 + k];
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
    for (long long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const long long row = tile * MT + r;
        const bool live = row < n;
        // layer 1's A operand (the accumulator's last reader, the previous tile's
        // epilogue, has finished: the barrier below orders it before the MMA)
        if (!hf) {
            float x[MI];
#pragma unroll
            for (int k = 0; k < MI; ++k)
                x[k] = live ? (X[ldx ? k * ldx + row : row * MI + k] - nm.mu[k]) / nm.sd[k] : 0.f;
            store_x_split(smem + FwdLayout::act, r, x);
        }
        float yacc = 0.f;
        for (int layer = 1; layer <= 3 && ok; ++layer) {
            fence_async_shared();
            tc_fence_before();
            __syncthreads();
            if (t == 0) {
                tc_fence_after();
                if (layer == 1) mma_layer1(tmem, s_act, s_w1);
                else mma_chain(tmem, s_act, layer == 2 ? s_w2 : s_w3, MH / 16, false);
                mma_commit(bar);
            }
            const bool got = mbar_wait(bar, ph);
            if (!__syncthreads_and(got)) { ok = false; break; }  // ph stays: the exit path waits on it
            ph ^= 1;
            tc_fence_after();
            const float* bias = layer == 1 ? b1 : layer == 2 ? b2 : b3;
            float* zs = SAVE ? (layer == 1 ? sv.z1 : layer == 2 ? sv.z2 : sv.z3) : nullptr;
            __nv_bfloat16* hs = SAVE ? (layer == 1 ? sv.h1 : sv.h2) : nullptr;
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
                if (layer < 3) {
#pragma unroll
                    for (int q = 0; q < 2; ++q) {
                        const float* u = v + 8 * q;
                        uint4 pk = make_uint4(pack_bf16(u[0], u[1]), pack_bf16(u[2], u[3]), pack_bf16(u[4], u[5]),
                                              pack_bf16(u[6], u[7]));
                        if (SAVE && live) {
                            const __nv_bfloat16* hb = reinterpret_cast<const __nv_bfloat16*>(&pk);
#pragma unroll
                            for (int j = 0; j < 8; ++j) hs[(size_t)(cc + 8 * q + j) * n + row] = hb[j];
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
// memory) and runs its own tiles, thread = row, all 128 columns per thread; the three
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
    static constexpr size_t w1 = act + (size_t)IG * 2 * ATOM;       // layer 1's B operand
    static constexpr size_t f32 = w1 + W1OP;                        // b1, b2, b3, w4, b4
    static constexpr size_t bars = f32 + 4 * (4 * MH + 4);
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
    float* b1 = (float*)(smem + InfLayout::f32);
    float* b2 = b1 + MH;
    float* b3 = b2 + MH;
    float* w4 = b3 + MH;
    float* b4 = w4 + MH;
    unsigned long long* bars = (unsigned long long*)(smem + InfLayout::bars);
    unsigned* tmem_slot = (unsigned*)(smem + InfLayout::bars + 8 * IG);
    const unsigned bar = smem_u32(&bars[g]);
    const unsigned s_w2 = smem_u32(smem + InfLayout::w2), s_w3 = smem_u32(smem + InfLayout::w3);
    const unsigned s_w1 = smem_u32(smem + InfLayout::w1);
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
    fill_w1_operand(smem + InfLayout::w1, params, t, IT);
    for (int k = t; k < MH; k += IT) {
        b1[k] = params[XTS_MLP_B1 + k];
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
        // layer 1's A operand: the row's split features (the slot's last MMA, which read
        // the operand, has completed)
        {
            float x[MI];
#pragma unroll
            for (int k = 0; k < MI; ++k) x[k] = live ? (xn[k] - nm.mu[k]) / nm.sd[k] : 0.f;
            load_x(tile + stride);
            store_x_split(act, r, x);
        }
        float ylo = 0.f, yhi = 0.f;  // the output layer over columns 0..63 and 64..127
        for (int layer = 1; layer <= 3 && ok; ++layer) {
            fence_async_shared();
            tc_fence_before();
            group_sync(g);
            if (r == 0) {
                tc_fence_after();
                if (layer == 1) mma_layer1(tmem, s_act, s_w1);
                else mma_chain(tmem, s_act, layer == 2 ? s_w2 : s_w3, MH / 16, false);
                mma_commit(bar);
            }
            // one warp of the group polls the MMA's mbarrier; the other three sleep in the
            // group's barrier instead of spinning (their issue slots go to the other groups)
            bool got = true;
            if ((warp & 3) == 0) got = mbar_wait(bar, ph);
            if (!group_and(g, got)) { ok = false; break; }  // ph stays: the exit path waits on it
            ph ^= 1;
            tc_fence_after();
            const float* bias = layer == 1 ? b1 : layer == 2 ? b2 : b3;
            // the accumulator read 16 columns at a time, the next 16 in flight while
            // these are worked on
            unsigned ra[16], rb[16];
            tmem_ld16_issue(trow, ra);
            tmem_ld_done(ra);
#pragma unroll
            for (int c0 = 0; c0 < MH; c0 += 16) {
                if (c0 + 16 < MH) tmem_ld16_issue(trow + (unsigned)(c0 + 16), rb);
                float v[16], bv[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(ra[j]);
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
                if (layer < 3) {
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
                if (c0 + 16 < MH) {
                    tmem_ld_done(rb);
#pragma unroll
                    for (int j = 0; j < 16; ++j) ra[j] = rb[j];
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
