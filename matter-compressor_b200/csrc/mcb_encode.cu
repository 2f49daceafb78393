// mcb_encode.cu -- sm_100a block encode and chunk-blob assembly.
//
// k_encode: one CTA (128 threads) per 16^3 block (src/mc_codec.c:629-736).
//   gather + sum/count -> dc, material nibble -> forward DCT-II along x, y, z
//   (each output a sequential single-precision sum over n of the even/odd
//   halves, src/mc_codec_float.h:83-95) -> fused dead-zone quantiser
//   (src/mc_codec.c:686-692) -> optional max-error pass: dequantise, inverse
//   transform, lrint + dc, list every voxel whose error exceeds tau
//   (:697-708) -> range coding of header bins, coefficients and corrections
//   by one thread (the coder is a serial chain; src/mc_codec.c:178-233).
// k_blob_layout / k_blob_fill / k_blob_hash: per-chunk blob assembly
//   (src/mc_codec.c:809-845, src/mc_archive.c:861-901): bitmap + u16 lengths
//   in block order, fraction map range-coded (src/mc_codec.c:600-611),
//   payloads concatenated in block order, xxh64 chain over
//   fmap | bitmap | lengths | payloads (src/mc_archive.c:76-88).
#include <cuda_runtime.h>
#include <stdint.h>

#include "mcb_devinfo.h"
#include "mcb_format.h"
#include "mcb_kernels.h"

namespace mcb {

__constant__ float c_cos[16][16];   // this translation unit's copy (no -rdc)

namespace {

__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }

// ------------------------------------------------------------ range encoder
struct Enc {
    uint8_t *out;
    uint32_t cap, len;
    uint64_t low;
    uint32_t range;
    uint32_t cache;
    uint32_t pending;   // bytes held back for carry propagation (cache + 0xFF run)
};

__device__ __forceinline__ void enc_emit(Enc &e, uint32_t b) {
    if (e.len < e.cap) e.out[e.len] = (uint8_t)b;
    e.len++;
}
// src/mc_codec.c:180-187
__device__ __forceinline__ void enc_shift(Enc &e) {
    uint32_t top = (uint32_t)(e.low >> 32);
    if (top != 0 || e.low < 0xFF000000ull) {
        enc_emit(e, (e.cache + top) & 0xFF);
        for (uint32_t i = 1; i < e.pending; ++i) enc_emit(e, (0xFF + top) & 0xFF);
        e.pending = 0;
        e.cache = (uint32_t)(e.low >> 24) & 0xFF;
    }
    e.pending++;
    e.low = (e.low << 8) & 0xFFFFFFFFull;
}
__device__ __forceinline__ void enc_norm(Enc &e) {
    while (e.range < (1u << 24)) { enc_shift(e); e.range <<= 8; }
}
__device__ __forceinline__ void enc_bit(Enc &e, uint16_t &p0, uint32_t bit) {
    uint32_t r0 = (e.range >> 12) * (uint32_t)p0;
    if (!bit) { e.range = r0; p0 = (uint16_t)(p0 + ((4096u - p0) >> 4)); }
    else { e.low += r0; e.range -= r0; p0 = (uint16_t)(p0 - (p0 >> 4)); }
    enc_norm(e);
}
__device__ __forceinline__ void enc_bypass(Enc &e, uint32_t bit) {
    e.range >>= 1;
    if (bit) e.low += e.range;
    enc_norm(e);
}
// k bits MSB-first, 16 at a time from the top (src/mc_codec.c:209-215)
__device__ void enc_bits(Enc &e, uint32_t v, int k) {
    int chunks = k > 16 ? (k - 1) / 16 : 0;    // leading 16-bit pieces
    for (int c = chunks; c > 0; --c) {
        int sh = k - 16;
        uint32_t piece = (sh >= 32 ? 0u : (v >> sh)) & 0xFFFFu;
        e.range >>= 16;
        e.low += (uint64_t)piece * e.range;
        enc_norm(e);
        k -= 16;
    }
    if (k == 0) return;
    e.range >>= k;
    e.low += (uint64_t)(v & ((1u << k) - 1u)) * e.range;
    enc_norm(e);
}
__device__ __forceinline__ int bitlen32(uint32_t v) { return v ? 32 - __clz(v) : 0; }
// order-0 Exp-Golomb (src/mc_codec.c:229-233)
__device__ void enc_eg(Enc &e, uint32_t v) {
    uint32_t t = v + 1u;
    int nb = t ? bitlen32(t) - 1 : 0;
    for (int i = 0; i < nb; ++i) enc_bypass(e, 1);
    enc_bypass(e, 0);
    if (nb) enc_bits(e, (v + 1u) & ((1u << nb) - 1u), nb);
}

// ------------------------------------------------------------ transforms
// forward DCT-II, outputs k in {j, j+4, j+8, j+12} of one line
__device__ __forceinline__ void fdct_quad(const float *in, int si, float *out, int so, int j) {
    float s[8], d[8];
#pragma unroll
    for (int n = 0; n < 8; ++n) {
        float a = in[n * si], b = in[(15 - n) * si];
        s[n] = fadd(a, b);
        d[n] = fsub(a, b);
    }
    const bool odd = j & 1;    // k = j + 4q keeps the parity of j
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        int k = j + 4 * q;
        float acc = 0.0f;
#pragma unroll
        for (int n = 0; n < 8; ++n) acc = fadd(acc, fmul(c_cos[k][n], odd ? d[n] : s[n]));
        out[k * so] = acc;
    }
}
// inverse DCT-III over all 16 k, outputs n and 15-n for n in {j, j+4}
__device__ __forceinline__ void idct_quad(const float *in, int si, float *out, int so, int j) {
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        int n = j + 4 * q;
        float ev = 0.0f, od = 0.0f;
#pragma unroll
        for (int k = 0; k < 16; k += 2) ev = fadd(ev, fmul(c_cos[k][n], in[k * si]));
#pragma unroll
        for (int k = 1; k < 16; k += 2) od = fadd(od, fmul(c_cos[k][n], in[k * si]));
        out[n * so] = fadd(ev, od);
        out[(15 - n) * so] = fsub(ev, od);
    }
}

// three passes x, y, z over a [z][y][x] cube, ping-ponging a <-> b;
// result in b. 128 threads, 256 lines x 4 quads per pass.
template <bool FWD>
__device__ void transform3(float *a, float *b) {
    const int tid = threadIdx.x;
    for (int t = tid; t < 1024; t += 128) {           // x lines: (z,y)
        int line = t >> 2, j = t & 3;
        if (FWD) fdct_quad(a + line * 16, 1, b + line * 16, 1, j);
        else idct_quad(a + line * 16, 1, b + line * 16, 1, j);
    }
    __syncthreads();
    for (int t = tid; t < 1024; t += 128) {           // y lines: (z,x)
        int j = t & 3, x = (t >> 2) & 15, z = t >> 6;
        if (FWD) fdct_quad(b + z * 256 + x, 16, a + z * 256 + x, 16, j);
        else idct_quad(b + z * 256 + x, 16, a + z * 256 + x, 16, j);
    }
    __syncthreads();
    for (int t = tid; t < 1024; t += 128) {           // z lines: (y,x)
        int j = t & 3, line = t >> 2;
        if (FWD) fdct_quad(a + line, 256, b + line, 256, j);
        else idct_quad(a + line, 256, b + line, 256, j);
    }
    __syncthreads();
}

// dead-zone reconstruction (src/mc_codec_float.h:185-190)
__device__ __forceinline__ float dequant(int lv, int f, const QTab &qt) {
    if (!lv) return 0.0f;
    float a = (float)(lv < 0 ? -lv : lv);
    float r = fadd(fadd(fmul(fsub(a, 1.0f), qt.step[f]), qt.dz8[f]), qt.dz4[f]);
    return lv < 0 ? -r : r;
}

struct EncSmem {
    float a[kN3];
    float b[kN3];
    int16_t lv[kN3];
    uint8_t vox[kN3];
    uint32_t mask[4][32];   // max-error pass: hit masks per warp and step
    uint32_t red[8];
    uint32_t ncorr;
    uint32_t eob;
};

}  // namespace

__global__ void __launch_bounds__(128) k_encode(EncParams P) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    EncSmem &S = *reinterpret_cast<EncSmem *>(smem_raw);
    const int tid = threadIdx.x;

    for (int item = blockIdx.x; item < P.n; item += gridDim.x) {
        const EncItem it = P.items[item];
        const QTab &qt = P.qtab[it.qslot];
        const uint8_t *src = reinterpret_cast<const uint8_t *>(it.src);
        // gather: thread per 16-voxel row
        uint32_t sum = 0, cnt = 0;
        for (int r = tid; r < 256; r += 128) {
            int z = r >> 4, y = r & 15;
            const uint8_t *row = src + z * it.sz + y * it.sy;
            uint4 w;
            if (((uintptr_t)row & 15) == 0) {
                w = *reinterpret_cast<const uint4 *>(row);
            } else {
                uint8_t b[16];
#pragma unroll
                for (int x = 0; x < 16; ++x) b[x] = row[x];
                memcpy(&w, b, 16);
            }
            *reinterpret_cast<uint4 *>(S.vox + r * 16) = w;
            const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
            for (int q = 0; q < 4; ++q) {
#pragma unroll
                for (int bb = 0; bb < 4; ++bb) {
                    uint32_t v = (ws[q] >> (8 * bb)) & 0xFF;
                    sum += v;
                    cnt += v != 0;
                }
            }
        }
        // block reduce sum, count
        for (int o = 16; o; o >>= 1) {
            sum += __shfl_xor_sync(0xFFFFFFFFu, sum, o);
            cnt += __shfl_xor_sync(0xFFFFFFFFu, cnt, o);
        }
        if ((tid & 31) == 0) { S.red[tid >> 5] = sum; S.red[4 + (tid >> 5)] = cnt; }
        if (tid == 0) { S.ncorr = 0; S.eob = 0; }
        __syncthreads();
        sum = S.red[0] + S.red[1] + S.red[2] + S.red[3];
        cnt = S.red[4] + S.red[5] + S.red[6] + S.red[7];
        if (tid == 0) {
            uint32_t f = (cnt * 15u + 2048u) / 4096u;    // material nibble (src/mc_codec.c:820-822)
            if (cnt && !f) f = 1;
            P.frac[item] = (uint8_t)f;
            if (!cnt) { P.len[item] = 0; P.sym[item] = make_uint2(0, 0); }
        }
        if (!cnt) { __syncthreads(); continue; }       // all air: not coded
        const int dc = (int)((sum + kN3 / 2) / kN3);
        for (int i = tid; i < kN3; i += 128) S.a[i] = (float)((int)S.vox[i] - dc);
        __syncthreads();
        transform3<true>(S.a, S.b);                     // coefficients in S.b
        // fused quantiser: t = |c|*rstep + (1-0.8), clamp [0,32767], truncate
        const float bias = 1.0f - 0.80f;
        uint32_t last = 0;
        for (int i = tid; i < kN3; i += 128) {
            float c = S.b[i];
            int f = (i >> 8) + ((i >> 4) & 15) + (i & 15);
            float t = fadd(fmul(fabsf(c), qt.rstep[f]), bias);
            if (!(t > 0.0f)) t = 0.0f;
            if (!(t < 32767.0f)) t = 32767.0f;
            int v = (int)t;
            S.lv[i] = (int16_t)(c < 0.0f ? -v : v);
        }
        __syncthreads();
        // eob = 1 + last scan position holding a nonzero level
        for (int p = tid; p < kN3; p += 128)
            if (S.lv[__ldg(P.scan + p) & 0xFFF]) last = max(last, (uint32_t)p + 1);
        for (int o = 16; o; o >>= 1) last = max(last, __shfl_xor_sync(0xFFFFFFFFu, last, o));
        if ((tid & 31) == 0) atomicMax(&S.eob, last);
        if (it.tau > 0) {
            // local reconstruction for the max-error pass
            for (int i = tid; i < kN3; i += 128) {
                int f = (i >> 8) + ((i >> 4) & 15) + (i & 15);
                S.a[i] = dequant(S.lv[i], f, qt);
            }
            __syncthreads();
            transform3<false>(S.a, S.b);                 // reconstruction in S.b
            // corrections in ascending voxel order, written straight to the
            // coder's scratch: warp w owns voxels [1024w, 1024w + 1024) in 32
            // steps of 32; a first pass counts its hits (the step masks kept
            // in shared memory), one barrier gives every warp its start, and a
            // second pass writes the entries
            const int lane = tid & 31, w = tid >> 5;
            auto hit_at = [&](int i, int &dl) {
                long long rr = __float2ll_rn(S.b[i]);
                int v = (int)(uint32_t)(unsigned long long)rr + dc;
                v = v < 0 ? 0 : v > 255 ? 255 : v;
                const int err = (int)S.vox[i] - v;
                const int ae = err < 0 ? -err : err;
                dl = err < 0 ? -(ae - (int)it.tau) : (ae - (int)it.tau);
                return ae > (int)it.tau;
            };
            uint32_t cnt_w = 0;
            for (int k = 0; k < 32; ++k) {
                int dl;
                const uint32_t m = __ballot_sync(0xFFFFFFFFu, hit_at(1024 * w + 32 * k + lane, dl));
                if (lane == 0) S.mask[w][k] = m;
                cnt_w += __popc(m);
            }
            if (lane == 0) S.red[w] = cnt_w;
            __syncthreads();
            uint32_t at = 0;
            for (int ww = 0; ww < w; ++ww) at += S.red[ww];
            uint32_t *cor = P.corr + (size_t)item * kN3;
            for (int k = 0; k < 32; ++k) {
                const uint32_t m = S.mask[w][k];
                if ((m >> lane) & 1) {
                    int dl;
                    const int i = 1024 * w + 32 * k + lane;
                    hit_at(i, dl);
                    cor[at + __popc(m & ((1u << lane) - 1u))] = (uint32_t)i | ((uint32_t)(uint16_t)(int16_t)dl << 16);
                }
                at += __popc(m);
            }
            if (tid == 0) S.ncorr = S.red[0] + S.red[1] + S.red[2] + S.red[3];
        }
        __syncthreads();   // eob (per-warp atomics) and ncorr complete
        // the block's symbols for k_encode_rc: levels in scan order up to the
        // EOB, the corrections, and (dc, eob, ncorr) with the coded flag
        const uint32_t eob = S.eob, ncorr = S.ncorr;
        int16_t *lvs = P.levels + (size_t)item * kN3;
        for (uint32_t p = tid; p < eob; p += 128) lvs[p] = S.lv[__ldg(P.scan + p) & 0xFFF];
        if (tid == 0) P.sym[item] = make_uint2(0x80000000u | (eob << 8) | (uint32_t)dc, ncorr);
        __syncthreads();
    }
}

// Range coding of every coded block, one lane per block (src/mc_codec.c:
// 330-350, 710-729): header bins, EOB, the coefficient loop and the
// corrections, in the order the reference writes them. The coder of a block is
// a serial chain; lanes in a warp code different blocks, with contexts in
// shared memory (one 16-bit word per context per lane).
__global__ void __launch_bounds__(128) k_encode_rc(EncParams P) {
    __shared__ uint16_t s_ctx[4][kNumCtx][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint16_t *ctx = &s_ctx[warp][0][lane];
    for (int item = blockIdx.x * blockDim.x + threadIdx.x; item < P.n; item += gridDim.x * blockDim.x) {
        const uint2 sy = P.sym[item];
        if (!(sy.x & 0x80000000u)) continue;   // all air: not coded
        const EncItem it = P.items[item];
        const QTab &qt = P.qtab[it.qslot];
        const uint32_t dc = sy.x & 0xFF, eob = (sy.x >> 8) & 0x1FFF, ncorr = sy.y;
        const int16_t *lvs = P.levels + (size_t)item * kN3;
        const uint32_t *cor = P.corr + (size_t)item * kN3;
        Enc e;
        e.out = reinterpret_cast<uint8_t *>(it.out);
        e.cap = kEncCap; e.len = 0; e.low = 0; e.range = 0xFFFFFFFFu; e.cache = 0; e.pending = 1;
        for (int j = 0; j < kNumCtx; ++j) ctx[j * 32] = qt.ctx[j];
        enc_bit(e, ctx[(kCtxFlag + 0) * 32], 0);                 // reserved
        enc_bit(e, ctx[(kCtxFlag + 1) * 32], ncorr > 0);
        for (int b = 0; b < 8; ++b) enc_bit(e, ctx[(kCtxDc + b) * 32], (dc >> (7 - b)) & 1);
        {   // EOB: bit length prefix then the bits below the MSB (src/mc_codec.c:314-320)
            int k = bitlen32(eob);
            for (int i = 0; i < k; ++i) enc_bit(e, ctx[(kCtxEob + i) * 32], 1);
            if (k < 13) enc_bit(e, ctx[(kCtxEob + k) * 32], 0);
            if (k > 1) enc_bits(e, eob & ((1u << (k - 1)) - 1u), k - 1);
        }
        uint32_t hist = 0;
        for (uint32_t p = 0; p < eob; ++p) {              // src/mc_codec.c:337-349
            const int v = lvs[p];
            if (p != eob - 1) {
                const uint32_t dens = min(__popc(hist & 0xFFFFu), 3);
                enc_bit(e, ctx[(kCtxSig + (__ldg(P.scan + p) >> 12) * 4 + dens) * 32], v != 0);
            }
            hist = (hist << 1) | (v != 0);
            if (!v) continue;
            uint32_t m = (uint32_t)(v < 0 ? -v : v), rest = m - 1;
            int k = 0;
            while (rest > 0 && k < 11) { enc_bit(e, ctx[(kCtxMag + k) * 32], 1); rest--; k++; }
            if (rest == 0) enc_bit(e, ctx[(kCtxMag + k) * 32], 0);
            else { enc_bit(e, ctx[(kCtxMag + 11) * 32], 1); enc_eg(e, rest); }
            enc_bypass(e, v < 0);
        }
        if (ncorr) {                                     // src/mc_codec.c:721-729
            enc_eg(e, ncorr - 1);
            uint32_t prev = 0;
            for (uint32_t c = 0; c < ncorr; ++c) {
                const uint32_t w = cor[c];
                const uint32_t pos = w & 0xFFFF;
                enc_eg(e, pos - prev);
                prev = pos;
                const int d = (int16_t)(w >> 16);
                enc_bypass(e, d < 0);
                enc_eg(e, (uint32_t)(d < 0 ? -d : d) - 1u);
            }
        }
        for (int i = 0; i < 5; ++i) enc_shift(e);
        if (e.len > e.cap) atomicAdd(P.status, 1u);
        P.len[item] = e.len > e.cap ? e.cap : e.len;
    }
}

// ------------------------------------------------------------ blob assembly
// Sizing pass, one CTA of 1024 threads per chunk: block-order exclusive scans
// of (present, bytes), the u16 length table and bitmap into side buffers, the
// fraction map range-coded by one thread (src/mc_codec.c:600-611), and the
// blob's total length (0 when every block is air).
__global__ void __launch_bounds__(1024) k_blob_layout(BlobParams P) {
    __shared__ uint32_t s_wnp[32], s_wby[32];
    const int c = blockIdx.x, tid = threadIdx.x;
    const int lane = tid & 31, w = tid >> 5;
    const uint32_t *len = P.len + (size_t)c * kGrid3;
    uint32_t *pref = P.scratch + (size_t)c * kGrid3;
    uint32_t l[4], np = 0, bytes = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) { l[i] = len[tid * 4 + i]; np += l[i] != 0; bytes += l[i]; }
    uint32_t snp = np, sby = bytes;
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t a = __shfl_up_sync(0xFFFFFFFFu, snp, o);
        uint32_t b = __shfl_up_sync(0xFFFFFFFFu, sby, o);
        if (lane >= o) { snp += a; sby += b; }
    }
    if (lane == 31) { s_wnp[w] = snp; s_wby[w] = sby; }
    __syncthreads();
    if (w == 0) {
        uint32_t a = s_wnp[lane], b = s_wby[lane];
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t x = __shfl_up_sync(0xFFFFFFFFu, a, o);
            uint32_t y = __shfl_up_sync(0xFFFFFFFFu, b, o);
            if (lane >= o) { a += x; b += y; }
        }
        s_wnp[lane] = a; s_wby[lane] = b;
    }
    __syncthreads();
    uint32_t slot = snp - np + (w ? s_wnp[w - 1] : 0);
    uint32_t off = sby - bytes + (w ? s_wby[w - 1] : 0);
    const uint32_t np_total = s_wnp[31], by_total = s_wby[31];
    uint16_t *lens16 = P.lens16 + (size_t)c * kGrid3;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        pref[tid * 4 + i] = off;
        if (l[i]) { lens16[slot] = (uint16_t)l[i]; slot++; off += l[i]; }
    }
    if (tid < kBitmapBytes) {
        uint32_t byte = 0;
        for (int b = 0; b < 8; ++b) byte |= (len[tid * 8 + b] != 0 ? 1u : 0u) << b;
        P.bitmap[(size_t)c * kBitmapBytes + tid] = (uint8_t)byte;
    }
    if (tid == 0) {
        Enc e;
        e.out = P.fmap + (size_t)c * kFmapCap;
        e.cap = kFmapCap; e.len = 0; e.low = 0; e.range = 0xFFFFFFFFu; e.cache = 0; e.pending = 1;
        uint16_t cx[3][4];
        for (int i = 0; i < 3; ++i) for (int j = 0; j < 4; ++j) cx[i][j] = 2048;
        const uint8_t *fr = P.frac + (size_t)c * kGrid3;
        int prev = 0;
        for (int i = 0; i < kGrid3; ++i) {
            int v = fr[i] & 15, b = prev == 0 ? 0 : prev == 15 ? 2 : 1;
            for (int bit = 3; bit >= 0; --bit) enc_bit(e, cx[b][bit], (v >> bit) & 1);
            prev = v;
        }
        for (int i = 0; i < 5; ++i) enc_shift(e);
        const uint32_t fml = e.len > (uint32_t)kFmapCap ? (uint32_t)kFmapCap : e.len;
        P.fml[c] = fml;
        P.np[c] = np_total;
        P.blob_len[c] = np_total ? (uint64_t)kBlobHdr + fml + kBitmapBytes + 2ull * np_total + by_total : 0;
    }
}

// Write pass: header (hash patched by k_blob_hash), fmap, bitmap, lengths and
// the payloads in block order. Grid (64, nchunks), a warp per block.
__global__ void __launch_bounds__(256) k_blob_fill(BlobParams P) {
    const int c = blockIdx.y;
    const uint64_t total = P.blob_len[c];
    if (!total) return;
    uint8_t *blob = P.blobs + P.blob_off[c];
    const uint32_t fml = P.fml[c], np = P.np[c];
    const int tid = threadIdx.x;
    if (blockIdx.x == 0) {
        if (tid == 0) {
            float q = P.header_q[c];
            memcpy(blob, &q, 4);
            for (int i = 4; i < 12; ++i) blob[i] = 0;
            blob[12] = (uint8_t)fml;
            blob[13] = (uint8_t)(fml >> 8);
        }
        const uint8_t *fm = P.fmap + (size_t)c * kFmapCap;
        for (uint32_t i = tid; i < fml; i += blockDim.x) blob[kBlobHdr + i] = fm[i];
        const uint8_t *bm = P.bitmap + (size_t)c * kBitmapBytes;
        for (int i = tid; i < kBitmapBytes; i += blockDim.x) blob[kBlobHdr + fml + i] = bm[i];
        const uint16_t *l16 = P.lens16 + (size_t)c * kGrid3;
        uint8_t *lens = blob + kBlobHdr + fml + kBitmapBytes;
        for (uint32_t i = tid; i < np; i += blockDim.x) {
            lens[2 * i] = (uint8_t)l16[i];
            lens[2 * i + 1] = (uint8_t)(l16[i] >> 8);
        }
    }
    uint8_t *pay = blob + kBlobHdr + fml + kBitmapBytes + 2ull * np;
    const int lane = tid & 31, w = tid >> 5;
    for (int b = blockIdx.x * 8 + w; b < kGrid3; b += gridDim.x * 8) {
        size_t item = (size_t)c * kGrid3 + b;
        uint32_t l = P.len[item];
        if (!l) continue;
        uint32_t off = P.scratch[item];
        const uint8_t *s = P.payload + item * (size_t)kEncCap;
        for (uint32_t i = lane; i < l; i += 32) pay[off + i] = s[i];
    }
}

// ------------------------------------------------------------ xxh64
namespace {
constexpr uint64_t XP1 = 0x9E3779B185EBCA87ull, XP2 = 0xC2B2AE3D27D4EB4Full,
                   XP3 = 0x165667B19E3779F9ull, XP4 = 0x85EBCA77C2B2AE63ull,
                   XP5 = 0x27D4EB2F165667C5ull;
__device__ __forceinline__ uint64_t rotl64(uint64_t x, int r) { return (x << r) | (x >> (64 - r)); }
__device__ __forceinline__ uint64_t xround(uint64_t acc, uint64_t in) { return rotl64(acc + in * XP2, 31) * XP1; }
__device__ __forceinline__ uint64_t ld64u(const uint8_t *p) {
    uint64_t v = 0;
    for (int i = 7; i >= 0; --i) v = (v << 8) | p[i];
    return v;
}

}  // namespace

// Device verify (src/mc_archive.c:1072-1111): the chained hash of every
// listed blob of an archive held in device memory, compared with the hash
// stored in the blob's header; bad[i] = 1 on a mismatch.
//
// One warp per blob. XXH64 keeps 4 serial accumulators, so 4 lanes hash; the
// whole warp first brings each 4 KiB tile of the blob into shared memory with
// coalesced 16-byte loads (many in flight at once), and the hashing lanes then
// read their stripes from shared memory: the serial round chain no longer
// waits on memory for every stripe.
namespace {
constexpr int kVerifyWarps = 4;
constexpr int kTileStripes = 128;
constexpr int kTileBytes = kTileStripes * 32;
constexpr int kTileBuf = kTileBytes + 64;   // a window plus its misaligned head and tail

// Bytes [start, start + n) of the archive into tile (n <= kTileBytes + 32),
// from the 16-byte boundary at or below start; bytes outside [base, limit)
// read 0. Returns that boundary. Every lane of the warp calls it.
__device__ const uint8_t *load_window(const uint8_t *base, const uint8_t *limit, const uint8_t *start, uint32_t n,
                                      uint8_t *tile) {
    const int lane = threadIdx.x & 31;
    const uint8_t *wb = reinterpret_cast<const uint8_t *>((uintptr_t)start & ~(uintptr_t)15);
    const uint32_t nvec = (uint32_t)((start + n - wb + 15) / 16);
    for (uint32_t i = lane; i < nvec; i += 32) {
        const uint8_t *q = wb + 16 * i;
        uint4 v;
        if (q >= base && q + 16 <= limit) {
            v = __ldg(reinterpret_cast<const uint4 *>(q));
        } else {
            uint8_t b[16];
            for (int k = 0; k < 16; ++k) b[k] = (q + k >= base && q + k < limit) ? q[k] : 0;
            memcpy(&v, b, 16);
        }
        reinterpret_cast<uint4 *>(tile)[i] = v;
    }
    __syncwarp();
    return wb;
}

// 8 little-endian bytes at tile offset o (any alignment)
__device__ __forceinline__ uint64_t tile64(const uint8_t *tile, uint32_t o) {
    const uint32_t a = o & 7;
    const uint64_t lo = *reinterpret_cast<const uint64_t *>(tile + (o - a));
    if (!a) return lo;
    const uint64_t hi = *reinterpret_cast<const uint64_t *>(tile + (o - a) + 8);
    return (lo >> (8 * a)) | (hi << (64 - 8 * a));
}

// XXH64 of [p, p + len) by a whole warp through tile; the hash in every lane.
__device__ uint64_t xxh64_warp(const uint8_t *base, const uint8_t *limit, const uint8_t *p, uint64_t len,
                               uint64_t seed, uint8_t *tile) {
    const int lane = threadIdx.x & 31;
    const uint64_t nstripes = len >= 32 ? len / 32 : 0;
    uint64_t acc = lane == 0 ? seed + XP1 + XP2 : lane == 1 ? seed + XP2 : lane == 2 ? seed : seed - XP1;
    for (uint64_t s0 = 0; s0 < nstripes; s0 += kTileStripes) {
        const uint32_t n = (uint32_t)min((uint64_t)kTileStripes, nstripes - s0);
        const uint8_t *start = p + 32 * s0;
        const uint8_t *wb = load_window(base, limit, start, 32 * n, tile);
        if (lane < 4) {
            const uint32_t o0 = (uint32_t)(start - wb) + 8 * lane;
#pragma unroll 8
            for (uint32_t s = 0; s < n; ++s) acc = xround(acc, tile64(tile, o0 + 32 * s));
        }
        __syncwarp();
    }
    const uint64_t a0 = __shfl_sync(0xFFFFFFFFu, acc, 0), a1 = __shfl_sync(0xFFFFFFFFu, acc, 1);
    const uint64_t a2 = __shfl_sync(0xFFFFFFFFu, acc, 2), a3 = __shfl_sync(0xFFFFFFFFu, acc, 3);
    uint64_t h;
    if (nstripes) {
        h = rotl64(a0, 1) + rotl64(a1, 7) + rotl64(a2, 12) + rotl64(a3, 18);
        h = (h ^ xround(0, a0)) * XP1 + XP4;
        h = (h ^ xround(0, a1)) * XP1 + XP4;
        h = (h ^ xround(0, a2)) * XP1 + XP4;
        h = (h ^ xround(0, a3)) * XP1 + XP4;
    } else {
        h = seed + XP5;
    }
    h += len;
    // the tail (< 32 bytes) by every lane alike, from one more window
    const uint8_t *t = p + nstripes * 32;
    const uint32_t rem = (uint32_t)(len - nstripes * 32);
    const uint8_t *wb = load_window(base, limit, t, rem, tile);
    uint32_t o = (uint32_t)(t - wb), end = o + rem;
    for (; end - o >= 8; o += 8) h = rotl64(h ^ xround(0, tile64(tile, o)), 27) * XP1 + XP4;
    if (end - o >= 4) {
        const uint64_t w = tile64(tile, o) & 0xFFFFFFFFull;
        h = rotl64(h ^ (w * XP1), 23) * XP2 + XP3;
        o += 4;
    }
    for (; o < end; ++o) h = rotl64(h ^ ((uint64_t)tile[o] * XP5), 11) * XP1;
    h ^= h >> 33; h *= XP2; h ^= h >> 29; h *= XP3; h ^= h >> 32;
    __syncwarp();   // the tile is reused by the next call
    return h;
}
}  // namespace

__global__ void __launch_bounds__(kVerifyWarps * 32) k_verify_hash(const uint8_t *arc, uint64_t arc_len,
                                                                   const VerifyItem *items, int n, uint32_t *bad) {
    __shared__ __align__(16) uint8_t s_tile[kVerifyWarps][kTileBuf];
    const int w = threadIdx.x >> 5;
    const int c = blockIdx.x * kVerifyWarps + w;
    if (c >= n) return;   // whole warps leave together
    uint8_t *tile = s_tile[w];
    const VerifyItem it = items[c];
    const uint8_t *blob = arc + it.co, *limit = arc + arc_len;
    const uint16_t fml = (uint16_t)(blob[12] | (blob[13] << 8));
    const uint8_t *fmap = blob + kBlobHdr, *bm = fmap + fml, *lens = bm + kBitmapBytes;
    const uint64_t pay = (uint64_t)kBlobHdr + fml + kBitmapBytes + 2ull * it.np;
    uint64_t h = xxh64_warp(arc, limit, fmap, fml, kHashSeed, tile);
    h ^= xxh64_warp(arc, limit, bm, kBitmapBytes, h, tile);
    h ^= xxh64_warp(arc, limit, lens, 2ull * it.np, h, tile);
    h ^= xxh64_warp(arc, limit, blob + pay, it.len - pay, h, tile);
    if ((threadIdx.x & 31) == 0) bad[c] = h != ld64u(blob + 4) ? 1u : 0u;
}

// Hash chain per chunk blob (src/mc_archive.c:76-88), one warp per blob
// through the same shared-memory tiles as the verify kernel; the hash goes
// into the blob header.
__global__ void __launch_bounds__(kVerifyWarps * 32) k_blob_hash(BlobParams P) {
    __shared__ __align__(16) uint8_t s_tile[kVerifyWarps][kTileBuf];
    const int w = threadIdx.x >> 5;
    const int c = blockIdx.x * kVerifyWarps + w;
    if (c >= P.nchunks) return;   // whole warps leave together
    const uint64_t total = P.blob_len[c];
    if (!total) return;
    uint8_t *tile = s_tile[w];
    uint8_t *blob = P.blobs + P.blob_off[c];
    const uint8_t *limit = blob + total;
    const uint16_t fml = (uint16_t)(blob[12] | (blob[13] << 8));
    const uint8_t *fmap = blob + kBlobHdr, *bm = fmap + fml, *lens = bm + kBitmapBytes;
    const uint32_t np = P.np[c];
    const uint64_t pay = (uint64_t)kBlobHdr + fml + kBitmapBytes + 2ull * np;
    uint64_t h = xxh64_warp(blob, limit, fmap, fml, kHashSeed, tile);
    h ^= xxh64_warp(blob, limit, bm, kBitmapBytes, h, tile);
    h ^= xxh64_warp(blob, limit, lens, 2ull * np, h, tile);
    h ^= xxh64_warp(blob, limit, blob + pay, total - pay, h, tile);
    if ((threadIdx.x & 31) == 0)
        for (int i = 0; i < 8; ++i) blob[4 + i] = (uint8_t)(h >> (8 * i));
}

cudaError_t launch_verify_hash(const uint8_t *d_arc, uint64_t arc_len, const VerifyItem *d_items, int n,
                               uint32_t *d_bad, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    k_verify_hash<<<(unsigned)((n + kVerifyWarps - 1) / kVerifyWarps), kVerifyWarps * 32, 0, s>>>(d_arc, arc_len,
                                                                                                d_items, n, d_bad);
    return cudaGetLastError();
}

cudaError_t upload_cos_encode(const float cmf[16][16], cudaStream_t s) {
    return cudaMemcpyToSymbolAsync(c_cos, cmf, sizeof(float) * 256, 0, cudaMemcpyHostToDevice, s);
}

cudaError_t launch_encode(const EncParams &p, cudaStream_t s) {
    if (p.n <= 0) return cudaSuccess;
    const int smem = (int)sizeof(EncSmem);
    // per device: the dynamic shared memory opt-in and the carveout (1), or
    // the error code of the attribute call that failed (negated)
    static std::atomic<int> attr[kMaxDevs];
    const int a = dev_once(attr, [smem] {
        cudaError_t e = cudaFuncSetAttribute(k_encode, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_encode, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     (int)cudaSharedmemCarveoutMaxShared);
        return e == cudaSuccess ? 1 : -(int)e;
    });
    if (a < 0) return (cudaError_t)(-a);
    const int sms = dev_sms();
    // one wave of CTAs: as many per SM as fit (45.6 KB of shared memory plus
    // the per-CTA reserve, in allocation units, leaves room for 4). CTAs walk
    // the blocks with a fixed stride, so CTAs beyond one wave would start
    // their whole share late.
    static std::atomic<int> occ_by_dev[kMaxDevs];
    const int occ = dev_once(occ_by_dev, [smem] {
        int o = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k_encode, 128, smem) != cudaSuccess || o < 1) o = 1;
        return o;
    });
    int blocks = p.n < sms * occ ? p.n : sms * occ;
    k_encode<<<blocks, 128, smem, s>>>(p);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const int rc_blocks = (p.n + 127) / 128;
    k_encode_rc<<<rc_blocks < sms * 16 ? rc_blocks : sms * 16, 128, 0, s>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_blob_layout(const BlobParams &p, cudaStream_t s) {
    if (p.nchunks <= 0) return cudaSuccess;
    k_blob_layout<<<p.nchunks, 1024, 0, s>>>(p);
    return cudaGetLastError();
}
cudaError_t launch_blob_fill(const BlobParams &p, cudaStream_t s) {
    if (p.nchunks <= 0) return cudaSuccess;
    k_blob_fill<<<dim3(64, p.nchunks), 256, 0, s>>>(p);
    return cudaGetLastError();
}
cudaError_t launch_blob_hash(const BlobParams &p, cudaStream_t s) {
    if (p.nchunks <= 0) return cudaSuccess;
    k_blob_hash<<<(p.nchunks + kVerifyWarps - 1) / kVerifyWarps, kVerifyWarps * 32, 0, s>>>(p);
    return cudaGetLastError();
}

}  // namespace mcb
