// xts_fits.cu -- the source maps as a FITS file (Fermi::fits::write_src_model,
// xtsrcmaps/fits/fits.write_src_model.cxx:10-66; its call at main.cxx:40).
//
// File layout, as the reference writes it through cfitsio: a primary HDU with no
// data and HDUNAME = 'PRIMARY', then one IMAGE extension per source with
// EXTNAME = the source name, NAXIS = 3, the map reordered SHWE -> SEHW
// (reorder_tensor(model_map, {0, 3, 2, 1}), :43: img[s][e][w][h] = map[s][h][w][e],
// so h is the fastest axis of the data), and CHECKSUM / DATASUM (:63).  The
// reference declares NAXIS1 = Nw and NAXIS2 = Nh over data whose fastest axis
// is h; the two agree only for square maps (the only maps its cubature fills,
// points_weights.hpp:21), so here NAXIS1 = H, the fastest axis of the data.
//
// The device does the per-value work: k_fits_encode transposes a chunk of maps
// into FITS order, converts to the output type, byte-swaps to big-endian and
// forms each source's DATASUM (the 32-bit ones'-complement sum of the data, an
// integer sum, so the same in any order).  The host writes the headers and
// streams the encoded chunks to the file while the next chunk is encoded.
// CHECKSUM follows the FITS checksum convention (Seaman, Pence and Rots, "FITS
// Checksum Proposal", 2002; FITS standard 4.0 appendix J): the 16-character
// ASCII encoding of the complement of the HDU's ones'-complement sum, so that
// the whole HDU then sums to -0.
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>

#include "xts_internal.cuh"

namespace xts {

constexpr int FH = 32;  // h values per tile: one per lane
static_assert(FH == 32, "k_fits_encode maps lanes to h");
constexpr int FE = 64;  // energies per tile (E is looped over in chunks of FE)

__device__ __forceinline__ unsigned long long bswap64(unsigned long long b) {
    const unsigned lo = (unsigned)b, hi = (unsigned)(b >> 32);
    return ((unsigned long long)__byte_perm(lo, 0, 0x0123) << 32) | __byte_perm(hi, 0, 0x0123);
}

// Block (h tile, w, source of the chunk), 256 threads: the tile of 32 h x all E at
// one w, read along e (E contiguous values per h) and written along h (32
// contiguous values per e).
template <typename Tin, bool F64OUT>
__global__ void __launch_bounds__(256) k_fits_encode(const Tin* __restrict__ map, int H, int W, int E,
                                                     void* __restrict__ out,
                                                     unsigned long long* __restrict__ datasum) {
    __shared__ double tile[FH][FE + 1];
    __shared__ unsigned long long red[8];
    const int h0 = blockIdx.x * FH, w = blockIdx.y, s = blockIdx.z, t = threadIdx.x;  // FH == 32 lanes
    const int nh = min(FH, H - h0);
    const size_t per_src = (size_t)H * W * E;
    const Tin* src = map + per_src * s + ((size_t)h0 * W + w) * E;  // (h0, w, 0)
    const size_t hstride = (size_t)W * E;                              // next h
    const int lane = t & 31, warp = t >> 5;
    unsigned long long sum = 0;
    for (int e0 = 0; e0 < E; e0 += FE) {
        const int ne = min(FE, E - e0);
        if (e0) __syncthreads();
        for (int h = warp; h < nh; h += 8)  // warp per h row, lanes along e
            for (int e = lane; e < ne; e += 32) tile[h][e] = (double)src[(size_t)h * hstride + e0 + e];
        __syncthreads();
        for (int e = warp; e < ne; e += 8) {  // warp per energy plane, lanes along h
            const size_t o = per_src * s + ((size_t)(e0 + e) * W + w) * H + h0 + lane;
            if (lane < nh) {
                const double v = tile[lane][e];
                if (F64OUT) {
                    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
                    sum += (b >> 32) + (b & 0xffffffffull);
                    ((unsigned long long*)out)[o] = bswap64(b);
                } else {
                    const unsigned b = __float_as_uint((float)v);
                    sum += b;
                    ((unsigned*)out)[o] = __byte_perm(b, 0, 0x0123);
                }
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if ((t & 31) == 0) red[t >> 5] = sum;
    __syncthreads();
    if (t == 0) {
        unsigned long long b = 0;
        for (int k = 0; k < 8; ++k) b += red[k];
        atomicAdd(datasum + s, b);
    }
}

// ------------------------------------------------------------------ host side
static uint32_t ones_fold(uint64_t s) {
    while (s >> 32) s = (s & 0xffffffffull) + (s >> 32);
    return (uint32_t)s;
}

static uint64_t sum_be_words(const unsigned char* p, size_t n) {  // n % 4 == 0
    uint64_t s = 0;
    for (size_t i = 0; i < n; i += 4)
        s += ((uint32_t)p[i] << 24) | ((uint32_t)p[i + 1] << 16) | ((uint32_t)p[i + 2] << 8) | p[i + 3];
    return s;
}

// The checksum convention's ASCII encoding of a 32-bit value: each byte becomes
// four characters from '0' whose offsets sum to it, avoiding the punctuation
// between the digits and the letters; the 16 characters are then rotated right
// by one to line up with the 32-bit words of the card (the value starts at byte
// 11 of its card).
static void checksum_encode(uint32_t value, char out[16]) {
    static const int exclude[13] = {0x3a, 0x3b, 0x3c, 0x3d, 0x3e, 0x3f, 0x40,
                                    0x5b, 0x5c, 0x5d, 0x5e, 0x5f, 0x60};
    char asc[16];
    for (int i = 0; i < 4; ++i) {
        const int byte = (int)((value >> (24 - 8 * i)) & 0xff);
        const int quot = byte / 4 + 0x30, rem = byte % 4;
        int ch[4] = {quot + rem, quot, quot, quot};
        bool again = true;
        while (again) {
            again = false;
            for (int k = 0; k < 13; ++k)
                for (int j = 0; j < 4; j += 2)
                    if (ch[j] == exclude[k] || ch[j + 1] == exclude[k]) {
                        ++ch[j];
                        --ch[j + 1];
                        again = true;
                    }
        }
        for (int j = 0; j < 4; ++j) asc[4 * j + i] = (char)ch[j];
    }
    for (int i = 0; i < 16; ++i) out[i] = asc[(i + 15) % 16];
}

// One 80-character header card.
static void card(std::string& h, const char* key, const std::string& value, bool str) {
    char buf[81];
    if (str) {
        std::string q = "'";
        for (char c : value) q += (c == '\'') ? std::string("''") : std::string(1, c);
        while (q.size() < 9) q += ' ';  // at least 8 characters between the quotes
        q += "'";
        snprintf(buf, sizeof buf, "%-8.8s= %-70.70s", key, q.c_str());
    } else {
        snprintf(buf, sizeof buf, "%-8.8s= %20s%50s", key, value.c_str(), "");
    }
    h.append(buf, 80);
}
static void card_end(std::string& h) {
    char buf[81];
    snprintf(buf, sizeof buf, "%-80s", "END");
    h.append(buf, 80);
    while (h.size() % 2880) h += ' ';
}

static std::string primary_header(int bitpix) {
    std::string h;
    card(h, "SIMPLE", "T", false);
    card(h, "BITPIX", std::to_string(bitpix), false);
    card(h, "NAXIS", "0", false);
    card(h, "EXTEND", "T", false);
    card(h, "HDUNAME", "PRIMARY", true);
    card_end(h);
    return h;
}

// The extension header with DATASUM and CHECKSUM filled in.
static std::string image_header(int bitpix, int H, int W, int E, const std::string& name, uint32_t datasum) {
    std::string h;
    card(h, "XTENSION", "IMAGE", true);
    card(h, "BITPIX", std::to_string(bitpix), false);
    card(h, "NAXIS", "3", false);
    card(h, "NAXIS1", std::to_string(H), false);
    card(h, "NAXIS2", std::to_string(W), false);
    card(h, "NAXIS3", std::to_string(E), false);
    card(h, "PCOUNT", "0", false);
    card(h, "GCOUNT", "1", false);
    card(h, "EXTNAME", name, true);
    const size_t ck = h.size();
    card(h, "CHECKSUM", "0000000000000000", true);
    card(h, "DATASUM", std::to_string(datasum), true);
    card_end(h);
    const uint32_t total = ones_fold((uint64_t)ones_fold(sum_be_words((const unsigned char*)h.data(), h.size())) +
                                     datasum);
    char enc[16];
    checksum_encode(~total, enc);
    memcpy(&h[ck + 11], enc, 16);
    return h;
}

template <typename Tin>
static int launch_encode(const Tin* map, int n, int H, int W, int E, bool f64out, void* out,
                         unsigned long long* datasum, cudaStream_t st) {
    const dim3 g((unsigned)((H + FH - 1) / FH), (unsigned)W, (unsigned)n);
    if (f64out)
        XTS_LAUNCH("k_fits_encode", st, (k_fits_encode<Tin, true><<<g, 256, 0, st>>>(map, H, W, E, out, datasum)));
    else
        XTS_LAUNCH("k_fits_encode", st, (k_fits_encode<Tin, false><<<g, 256, 0, st>>>(map, H, W, E, out, datasum)));
    return XTS_OK;
}

struct HostBuf {
    void* p = nullptr;
    ~HostBuf() { if (p) cudaFreeHost(p); }
};

int write_src_model(const char* filename, const void* model_map, int S, int H, int W, int E,
                    const char* const* names, bool dev_ptrs, bool f64in, bool f64out, cudaStream_t st) {
    const int bitpix = f64out ? -64 : -32;
    const size_t in_bps = (size_t)H * W * E * (f64in ? 8 : 4);    // bytes per source in
    const size_t out_bps = (size_t)H * W * E * (f64out ? 8 : 4);  // bytes per source out
    // encoded bytes per chunk: 256 MiB, or XTS_FITS_CHUNK_MB (tests use small chunks)
    size_t budget = (size_t)256 << 20;
    if (const char* env = getenv("XTS_FITS_CHUNK_MB")) {
        const long mb = atol(env);
        if (mb > 0) budget = (size_t)mb << 20;
    }
    int nc = (int)(budget / (out_bps > in_bps ? out_bps : in_bps));
    nc = nc < 1 ? 1 : (nc > S ? (S > 0 ? S : 1) : nc);
    if (nc > 65535) nc = 65535;
    void* dout = workspace(W_FITS_OUT, out_bps * nc);
    unsigned long long* dsum = (unsigned long long*)workspace(W_FITS_SUM, sizeof(unsigned long long) * nc);
    void* din = dev_ptrs ? nullptr : workspace(W_FITS_IN, in_bps * nc);
    if (!dout || !dsum || (!dev_ptrs && !din)) return XTS_ERR_OOM;
    HostBuf hb[2], hs[2];
    for (int b = 0; b < 2 && S > 0; ++b) {
        XTS_CUDA(cudaMallocHost(&hb[b].p, out_bps * nc));
        XTS_CUDA(cudaMallocHost(&hs[b].p, sizeof(unsigned long long) * nc));
    }
    cudaEvent_t ev[2] = {};
    for (int b = 0; b < 2; ++b) XTS_CUDA(cudaEventCreateWithFlags(&ev[b], cudaEventDisableTiming));
    struct EvGuard { cudaEvent_t* e; ~EvGuard() { for (int b = 0; b < 2; ++b) if (e[b]) cudaEventDestroy(e[b]); } } eg{ev};
    FILE* f = fopen(filename, "wb");
    if (!f) return set_error(XTS_ERR_IO, "write_src_model: cannot open %s", filename);
    struct FileGuard { FILE*& f; ~FileGuard() { if (f) fclose(f); } } fg{f};
    const std::string ph = primary_header(bitpix);
    if (fwrite(ph.data(), 1, ph.size(), f) != ph.size()) return set_error(XTS_ERR_IO, "write_src_model: write failed");
    static const char zeros[2880] = {};
    const size_t pad = (2880 - out_bps % 2880) % 2880;
    auto emit = [&](int b, int s0, int n) -> int {
        XTS_CUDA(cudaEventSynchronize(ev[b]));
        const unsigned long long* sums = (const unsigned long long*)hs[b].p;
        for (int i = 0; i < n; ++i) {
            char dflt[32];
            snprintf(dflt, sizeof dflt, "SRC%05d", s0 + i);
            const std::string name = names && names[s0 + i] ? names[s0 + i] : dflt;
            size_t len = 0;
            for (char c : name) {
                if (c < 0x20 || c > 0x7e) return set_error(XTS_ERR_ARG, "write_src_model: source %d name is not printable ASCII", s0 + i);
                len += c == '\'' ? 2 : 1;
            }
            if (len > 68) return set_error(XTS_ERR_ARG, "write_src_model: source %d name longer than a FITS string card", s0 + i);
            const std::string hdr = image_header(bitpix, H, W, E, name, ones_fold(sums[i]));
            const char* data = (const char*)hb[b].p + (size_t)i * out_bps;
            if (fwrite(hdr.data(), 1, hdr.size(), f) != hdr.size() || fwrite(data, 1, out_bps, f) != out_bps ||
                fwrite(zeros, 1, pad, f) != pad)
                return set_error(XTS_ERR_IO, "write_src_model: write failed");
        }
        return XTS_OK;
    };
    int prev_s0 = -1, prev_n = 0;
    for (int s0 = 0, k = 0; s0 < S; s0 += nc, ++k) {
        const int n = S - s0 < nc ? S - s0 : nc, b = k & 1;
        const char* src = (const char*)model_map + (size_t)s0 * in_bps;
        if (!dev_ptrs) {
            XTS_CUDA(cudaMemcpyAsync(din, src, in_bps * n, cudaMemcpyHostToDevice, st));
            src = (const char*)din;
        }
        XTS_CUDA(cudaMemsetAsync(dsum, 0, sizeof(unsigned long long) * n, st));
        const int rc = f64in ? launch_encode((const double*)src, n, H, W, E, f64out, dout, dsum, st)
                             : launch_encode((const float*)src, n, H, W, E, f64out, dout, dsum, st);
        if (rc) return rc;
        XTS_CUDA(cudaMemcpyAsync(hb[b].p, dout, out_bps * n, cudaMemcpyDeviceToHost, st));
        XTS_CUDA(cudaMemcpyAsync(hs[b].p, dsum, sizeof(unsigned long long) * n, cudaMemcpyDeviceToHost, st));
        XTS_CUDA(cudaEventRecord(ev[b], st));
        if (prev_n) {  // the previous chunk goes to the file while this one is encoded
            const int rc2 = emit(b ^ 1, prev_s0, prev_n);
            if (rc2) return rc2;
        }
        prev_s0 = s0;
        prev_n = n;
    }
    if (prev_n) {
        const int rc2 = emit(((S - 1) / nc) & 1, prev_s0, prev_n);
        if (rc2) return rc2;
    }
    FILE* g = f;
    f = nullptr;
    if (fclose(g) != 0) return set_error(XTS_ERR_IO, "write_src_model: close failed");
    return XTS_OK;
}

}  // namespace xts
