// mcb_decode.cu -- sm_100a block decode: entropy stage + reconstruction stage.
//
// Stage 1, k_entropy: one LANE per block. The adaptive binary range decoder
// is a serial dependency chain per block (src/mc_codec.c:197-226), so the
// parallelism is across blocks: every lane of a warp runs its own decoder and
// the loop body decodes exactly one bin per lane per iteration (a flat state
// machine), so lanes never wait on each other inside a block. The lane's 68
// adaptive contexts sit in shared memory (context j of lane l at word
// j*32+l: conflict-free), the scan table is staged once per CTA. Output per
// block: a small header (dc, flags, extents) and a list of nonzero levels plus
// corrections.
//
// Stage 2, k_reconstruct: one CTA (128 threads) per block. Dequantise into a
// dense coefficient box bounded by the block's extents, then the three
// separable DCT-III passes along x, y, z, each output accumulated over
// ascending k in single precision with explicit round-to-nearest adds and
// multiplies (no FMA), exactly the order of src/mc_codec_float.h:98-105.
// Coefficients outside the extent box are zero and the reference skips them;
// including zero terms inside the box adds +/-0 to an accumulator that can
// never be -0, so the dense box sum is bit-identical to the sparse one.
// Then lrint + dc, clamp to u8 (src/mc_codec.c:766-769), the sparse
// corrections in stream order (:770-782), and the clipped store.
#include <cuda_runtime.h>
#include <stdint.h>

#include "mcb_format.h"
#include "mcb_kernels.h"

namespace mcb {

__constant__ float c_cos[16][16];

// ---------------------------------------------------------------- stage 1
enum : uint32_t {
    S_FLAG = 0, S_DC, S_EOBP, S_SIG, S_MAG,   // context-coded bins
    S_EOBS, S_SIGN, S_EGP, S_EGS, S_CSIGN,    // bypass bins
    S_DONE, S_IDLE
};
enum : uint32_t { R_MAG = 0, R_CCOUNT, R_CGAP, R_CMAG };

struct LaneState {
    const uint8_t *src;
    uint32_t len, pos, code, range;
    uint32_t state, k, p, eob, hist;
    uint32_t dc, flags;
    int ez, ey, ex;
    uint32_t mag, nbits, rem, acc, ret;
    uint32_t nent, nnz, ncorr, ccount, cpos, cneg;
    uint64_t base;
    uint32_t cap, ovf, bad;
    int item;
};

__device__ __forceinline__ uint8_t fetch(LaneState &L) {
    uint8_t b = 0;
    if (L.pos < L.len) { b = __ldg(L.src + L.pos); L.pos++; }
    return b;
}

__device__ __forceinline__ void put_entry(LaneState &L, const EntParams &P, uint32_t v) {
    uint32_t j = L.nent;
    if (j < L.cap) {
        P.arena[L.base + j] = v;
    } else {
        if (L.ovf == 0xFFFFFFFFu) {
            uint32_t need = kEntryMax - L.cap;
            uint32_t off = atomicAdd(P.pool_used, need);
            if ((uint64_t)off + need > P.pool_cap) { L.bad = 1; L.state = S_DONE; return; }
            L.ovf = off;
        }
        P.pool[L.ovf + (j - L.cap)] = v;
    }
    L.nent = j + 1;
}

__device__ __forceinline__ void lane_begin(LaneState &L, const EntParams &P, uint32_t *ctx, int slot) {
    L.item = slot;
    const DecItem &it = P.items[slot];
    L.src = reinterpret_cast<const uint8_t *>(it.src);
    L.len = it.len;
    L.pos = 0;
    L.base = P.base[slot];
    L.cap = entry_cap(it.len);
    L.ovf = 0xFFFFFFFFu;
    L.bad = 0;
    L.nent = 0; L.nnz = 0; L.ncorr = 0; L.ccount = 0; L.cpos = 0; L.cneg = 0;
    L.ez = L.ey = L.ex = -1;
    L.dc = 0; L.flags = 0;
    L.k = 0; L.p = 0; L.eob = 0; L.hist = 0; L.mag = 0;
    L.nbits = 0; L.rem = 0; L.acc = 0; L.ret = 0;
    if (it.len == 0) { L.state = S_DONE; return; }   // absent block: zeros
    const QTab &qt = P.qtab[it.qslot];
    for (int j = 0; j < kNumCtx; ++j) ctx[j * 32] = qt.ctx[j];
    L.range = 0xFFFFFFFFu;
    L.code = 0;
    for (int i = 0; i < 5; ++i) L.code = (L.code << 8) | fetch(L);
    L.state = S_FLAG;
}

__device__ __forceinline__ void lane_finish(LaneState &L, const EntParams &P) {
    EntHdr h;
    h.dc = (uint8_t)L.dc;
    h.flags = (uint8_t)L.flags;
    h.bad = (uint8_t)L.bad;
    h.pad = 0;
    h.ez = (int8_t)L.ez; h.ey = (int8_t)L.ey; h.ex = (int8_t)L.ex; h.pad2 = 0;
    h.nnz = (uint16_t)L.nnz;
    h.ncorr = (uint16_t)L.ccount;
    h.ovf = L.ovf;
    P.hdr[L.item] = h;
    if (L.bad) atomicAdd(P.status, 1u);
}

// Position p of the coefficient scan becomes current: the last position is
// significant by definition and costs no bin (src/mc_codec.c:364).
__device__ __forceinline__ void goto_position(LaneState &L) {
    if (L.p >= L.eob) {
        if (L.flags & 2) { L.state = S_EGP; L.nbits = 0; L.ret = R_CCOUNT; }
        else L.state = S_DONE;
    } else if (L.p == L.eob - 1) {
        L.hist = (L.hist << 1) | 1u;
        L.state = S_MAG; L.k = 0;
    } else {
        L.state = S_SIG;
    }
}

__device__ __forceinline__ void eg_return(LaneState &L, const EntParams &P, const uint16_t *scan, uint32_t val) {
    switch (L.ret) {
    case R_MAG:
        L.mag = 12u + val;            // 11 unary rungs + Exp-Golomb tail + 1
        L.state = S_SIGN;
        break;
    case R_CCOUNT: {
        uint32_t n = val + 1u;
        if (n > (uint32_t)kN3) n = kN3;
        L.ncorr = n; L.ccount = 0; L.cpos = 0;
        if (n == 0) L.state = S_DONE;
        else { L.state = S_EGP; L.nbits = 0; L.ret = R_CGAP; }
        break;
    }
    case R_CGAP:
        L.cpos += val;
        L.state = S_CSIGN;
        break;
    default: {   // R_CMAG
        uint32_t m = val + 1u;
        if (L.cpos >= (uint32_t)kN3) { L.state = S_DONE; break; }
        put_entry(L, P, L.cpos);
        if (L.state == S_DONE) break;
        put_entry(L, P, L.cneg ? 0u - m : m);
        if (L.state == S_DONE) break;
        L.ccount++;
        if (L.ccount == L.ncorr) L.state = S_DONE;
        else { L.state = S_EGP; L.nbits = 0; L.ret = R_CGAP; }
        break;
    }
    }
}

template <int WARPS>
__global__ void __launch_bounds__(WARPS * 32) k_entropy(EntParams P) {
    __shared__ uint16_t s_scan[kN3];
    __shared__ uint32_t s_ctx[WARPS][kNumCtx][32];
    for (int i = threadIdx.x; i < kN3; i += blockDim.x) s_scan[i] = P.scan[i];
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t *ctx = &s_ctx[warp][0][lane];

    const int stride = gridDim.x * blockDim.x;
    int next = blockIdx.x * blockDim.x + threadIdx.x;
    LaneState L;
    L.state = S_IDLE;
    L.item = -1;
    auto claim = [&]() -> bool {
        while (next < P.n) {
            int slot = P.order ? (int)P.order[next] : next;
            next += stride;
            lane_begin(L, P, ctx, slot);
            if (L.state != S_DONE) return true;
            lane_finish(L, P);
        }
        L.state = S_IDLE;
        return false;
    };
    claim();

    // Every iteration decodes at most one bin per lane; a bounded number of
    // iterations per block follows from the Exp-Golomb cap and the finite
    // scan, so the loop always terminates.
    while (__any_sync(0xFFFFFFFFu, L.state != S_IDLE)) {
        if (L.state == S_IDLE) continue;
        const uint32_t st = L.state;
        uint32_t bit;
        if (st < S_EOBS) {
            // ---- context-coded bin (src/mc_codec.c:198-204)
            uint32_t cidx;
            if (st == S_SIG) {
                uint32_t sc = s_scan[L.p];
                uint32_t dens = min(__popc(L.hist & 0xFFFFu), 3);
                cidx = kCtxSig + (sc >> 12) * 4 + dens;
            } else {
                // FLAG 0, DC 2, EOB 10, MAG 56 (+k)
                const uint32_t base = st == S_FLAG ? kCtxFlag : st == S_DC ? kCtxDc : st == S_EOBP ? kCtxEob : kCtxMag;
                cidx = base + L.k;
            }
            uint32_t p0 = ctx[cidx * 32];
            uint32_t r0 = (L.range >> 12) * p0;
            if (L.code < r0) {
                L.range = r0; bit = 0; p0 += (4096u - p0) >> 4;
            } else {
                L.code -= r0; L.range -= r0; bit = 1; p0 -= p0 >> 4;
            }
            ctx[cidx * 32] = p0;
        } else {
            // ---- bypass bits, k at once (src/mc_codec.c:205,216-226)
            uint32_t nb = (st == S_EOBS) ? L.k : (st == S_EGS ? min(L.rem, 16u) : 1u);
            L.range >>= nb;
            uint32_t q;
            if (nb == 1) q = L.code >= L.range ? 1u : 0u;
            else { q = L.code / L.range; uint32_t mx = (1u << nb) - 1u; q = q > mx ? mx : q; }
            L.code -= q * L.range;
            bit = q;
        }
        while (L.range < (1u << 24)) { L.code = (L.code << 8) | fetch(L); L.range <<= 8; }

        switch (st) {
        case S_FLAG:
            L.flags |= bit << L.k;
            if (++L.k == 2) { L.state = S_DC; L.k = 0; }
            break;
        case S_DC:
            L.dc = (L.dc << 1) | bit;
            if (++L.k == 8) { L.state = S_EOBP; L.k = 0; }
            break;
        case S_EOBP:   // bit length of eob, 13 context bins at most (src/mc_codec.c:321-327)
            if (bit && ++L.k < 13) break;
            if (L.k == 0) { L.eob = 0; L.p = 0; goto_position(L); }
            else if (L.k == 1) { L.eob = 1; L.p = 0; L.hist = 0; goto_position(L); }
            else { L.state = S_EOBS; L.k = L.k - 1; }
            break;
        case S_EOBS:
            L.eob = (1u << L.k) | bit;
            if (L.eob > (uint32_t)kN3) L.eob = kN3;
            L.p = 0; L.hist = 0;
            goto_position(L);
            break;
        case S_SIG:
            L.hist = (L.hist << 1) | bit;
            if (bit) { L.state = S_MAG; L.k = 0; }
            else { L.p++; goto_position(L); }
            break;
        case S_MAG:    // 12 adaptive unary rungs (src/mc_codec.c:268-275)
            if (!bit) { L.mag = L.k + 1; L.state = S_SIGN; }
            else if (L.k < 11) L.k++;
            else { L.state = S_EGP; L.nbits = 0; L.ret = R_MAG; }
            break;
        case S_SIGN: {
            uint32_t sc = s_scan[L.p];
            uint32_t idx = sc & 0xFFFu;
            int32_t lv = bit ? -(int32_t)L.mag : (int32_t)L.mag;
            put_entry(L, P, idx | ((uint32_t)(uint16_t)(int16_t)lv << 16));
            if (L.state == S_DONE) break;
            L.nnz++;
            L.ez = max(L.ez, (int)(idx >> 8));
            L.ey = max(L.ey, (int)((idx >> 4) & 15));
            L.ex = max(L.ex, (int)(idx & 15));
            L.p++;
            goto_position(L);
            break;
        }
        case S_EGP:    // Exp-Golomb prefix: count one-bits (src/mc_codec.c:234-238)
            if (bit) {
                if (++L.nbits >= (uint32_t)kEgCap) { L.bad = 1; L.state = S_DONE; }
            } else if (L.nbits == 0) {
                eg_return(L, P, s_scan, 0);
            } else {
                L.state = S_EGS; L.rem = L.nbits; L.acc = 0;
            }
            break;
        case S_EGS: {
            uint32_t nb = min(L.rem, 16u);
            L.acc = (L.acc << nb) | bit;
            L.rem -= nb;
            if (L.rem == 0) eg_return(L, P, s_scan, ((1u << (L.nbits & 31)) | L.acc) - 1u);
            break;
        }
        case S_CSIGN:
            L.cneg = bit;
            L.state = S_EGP; L.nbits = 0; L.ret = R_CMAG;
            break;
        default:
            break;
        }
        if (L.state == S_DONE) {
            lane_finish(L, P);
            claim();
        }
    }
}

// ---------------------------------------------------------------- stage 2
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }

__device__ __forceinline__ uint32_t entry_at(const RecParams &P, uint64_t base, uint32_t cap, uint32_t ovf, uint32_t j) {
    if (j < cap) return P.arena[base + j];
    return ovf == 0xFFFFFFFFu ? 0u : P.pool[ovf + (j - cap)];
}

__device__ __forceinline__ uint8_t to_u8(float v, int dc) {
    long long r = __float2ll_rn(v);          // lrintf: round half to even
    int s = (int)(uint32_t)(unsigned long long)r + dc;
    return (uint8_t)(s < 0 ? 0 : s > 255 ? 255 : s);
}

// one transform line: e/o halves for outputs (m, m+1) over k < K,
// sequential in k (src/mc_codec_float.h:102-104)
__device__ __forceinline__ void line_pair(const float *in, int si, int K, int m,
                                          float &e0, float &e1, float &o0, float &o1) {
    e0 = e1 = o0 = o1 = 0.0f;
    for (int k = 0; k < K; k += 2) {
        float v = in[k * si];
        e0 = fadd(e0, fmul(c_cos[k][m], v));
        e1 = fadd(e1, fmul(c_cos[k][m + 1], v));
    }
    for (int k = 1; k < K; k += 2) {
        float v = in[k * si];
        o0 = fadd(o0, fmul(c_cos[k][m], v));
        o1 = fadd(o1, fmul(c_cos[k][m + 1], v));
    }
}

__global__ void __launch_bounds__(128) k_reconstruct(RecParams P) {
    __shared__ __align__(16) float sA[kN3];
    __shared__ __align__(16) float sB[kN3];
    uint8_t *stage = reinterpret_cast<uint8_t *>(sA);
    const int tid = threadIdx.x;

    for (int item = blockIdx.x; item < P.n; item += gridDim.x) {
        const DecItem it = P.items[item];
        const EntHdr h = P.hdr[item];
        const uint64_t base = P.base[item];
        const uint32_t cap = entry_cap(it.len);
        // the header comes from k_entropy; the guards keep every index below
        // inside shared memory whatever its contents
        const bool sane = h.ez <= 15 && h.ey <= 15 && h.ex <= 15 && h.nnz <= kN3 && h.ncorr <= kN3 &&
                          (h.nnz == 0 || (h.ez >= 0 && h.ey >= 0 && h.ex >= 0));
        const int dc = it.len && sane ? h.dc : 0;
        const int nnz = it.len && sane ? h.nnz : 0;
        const int ncorr = it.len && sane ? h.ncorr : 0;

        if (nnz == 0) {
            // constant block (src/mc_codec.c:757-759) or absent block (zeros)
            uint32_t w = (uint32_t)dc * 0x01010101u;
            uint4 v = make_uint4(w, w, w, w);
            for (int i = tid; i < kN3 / 16; i += 128) reinterpret_cast<uint4 *>(stage)[i] = v;
        } else {
            const int E = h.ez + 1, Y = h.ey + 1, X = h.ex + 1;
            const QTab &qt = P.qtab[it.qslot];
            for (int i = tid; i < E * Y * X; i += 128) sB[i] = 0.0f;
            __syncthreads();
            // dequantise (src/mc_codec_float.h:185-190) into box[cz][cy][cx]
            for (int j = tid; j < nnz; j += 128) {
                uint32_t e = entry_at(P, base, cap, h.ovf, j);
                int idx = e & 0xFFF;
                int lv = (int16_t)(e >> 16);
                if (!lv) continue;
                int cz = idx >> 8, cy = (idx >> 4) & 15, cx = idx & 15;
                if (cz >= E || cy >= Y || cx >= X) continue;
                int f = cz + cy + cx;
                float a = (float)(lv < 0 ? -lv : lv);
                float r = fadd(fadd(fmul(fsub(a, 1.0f), qt.step[f]), qt.dz8[f]), qt.dz4[f]);
                sB[(cz * Y + cy) * X + cx] = lv < 0 ? -r : r;
            }
            __syncthreads();
            // pass 1: lines along x, box -> A[cz][cy][x]
            for (int t = tid; t < E * Y * 4; t += 128) {
                int line = t >> 2, m = (t & 3) * 2;
                float e0, e1, o0, o1;
                line_pair(sB + line * X, 1, X, m, e0, e1, o0, o1);
                float *o = sA + line * 16;
                o[m] = fadd(e0, o0); o[m + 1] = fadd(e1, o1);
                o[15 - m] = fsub(e0, o0); o[14 - m] = fsub(e1, o1);
            }
            __syncthreads();
            // pass 2: lines along y, A[cz][k][x] -> B[cz][y][x]
            for (int t = tid; t < E * 64; t += 128) {
                int m = (t & 3) * 2, x = (t >> 2) & 15, cz = t >> 6;
                float e0, e1, o0, o1;
                line_pair(sA + cz * Y * 16 + x, 16, Y, m, e0, e1, o0, o1);
                float *o = sB + cz * 256 + x;
                o[m * 16] = fadd(e0, o0); o[(m + 1) * 16] = fadd(e1, o1);
                o[(15 - m) * 16] = fsub(e0, o0); o[(14 - m) * 16] = fsub(e1, o1);
            }
            __syncthreads();
            // pass 3: lines along z, B[k][y][x] -> voxels, lrint + dc, clamp
            for (int t = tid; t < 256 * 4; t += 128) {
                int m = (t & 3) * 2, line = t >> 2;
                float e0, e1, o0, o1;
                line_pair(sB + line, 256, E, m, e0, e1, o0, o1);
                stage[m * 256 + line] = to_u8(fadd(e0, o0), dc);
                stage[(m + 1) * 256 + line] = to_u8(fadd(e1, o1), dc);
                stage[(15 - m) * 256 + line] = to_u8(fsub(e0, o0), dc);
                stage[(14 - m) * 256 + line] = to_u8(fsub(e1, o1), dc);
            }
        }
        __syncthreads();
        if (ncorr && tid == 0) {
            // corrections in stream order: a position may repeat, each
            // application clamps (src/mc_codec.c:775-781)
            for (int c = 0; c < ncorr; ++c) {
                uint32_t pos = entry_at(P, base, cap, h.ovf, nnz + 2 * c);
                uint32_t d = entry_at(P, base, cap, h.ovf, nnz + 2 * c + 1);
                if (pos >= (uint32_t)kN3) break;
                int v = (int)((uint32_t)stage[pos] + d);
                stage[pos] = (uint8_t)(v < 0 ? 0 : v > 255 ? 255 : v);
            }
        }
        __syncthreads();
        // clipped store: one 16-voxel row per thread step
        const int z0 = it.clip_lo >> 8, y0 = (it.clip_lo >> 4) & 15, x0 = it.clip_lo & 15;
        const int z1 = it.clip_hi >> 8, y1 = (it.clip_hi >> 4) & 15, x1 = it.clip_hi & 15;
        const int ny = y1 - y0 + 1, nrows = (z1 - z0 + 1) * ny;
        uint8_t *dst = reinterpret_cast<uint8_t *>(it.dst);
        for (int r = tid; r < nrows; r += 128) {
            int z = z0 + r / ny, y = y0 + r % ny;
            uint8_t *row = dst + z * it.sz + y * it.sy;
            const uint8_t *srow = stage + z * 256 + y * 16;
            if (x0 == 0 && x1 == 15 && ((uintptr_t)row & 15) == 0) {
                *reinterpret_cast<uint4 *>(row) = *reinterpret_cast<const uint4 *>(srow);
            } else {
                for (int x = x0; x <= x1; ++x) row[x] = srow[x];
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- launchers
cudaError_t upload_cos(const float cmf[16][16], cudaStream_t s) {
    return cudaMemcpyToSymbolAsync(c_cos, cmf, sizeof(float) * 256, 0, cudaMemcpyHostToDevice, s);
}

static int g_num_sms = 0;
static int num_sms() {
    if (!g_num_sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
        if (g_num_sms <= 0) g_num_sms = 148;
    }
    return g_num_sms;
}

cudaError_t launch_entropy(const EntParams &p, const LaunchCfg &cfg, cudaStream_t s) {
    if (p.n <= 0) return cudaSuccess;
    constexpr int W = 4;
    int lanes = p.n;
    int blocks = (lanes + W * 32 - 1) / (W * 32);
    int cap = num_sms() * (cfg.ent_ctas_per_sm > 0 ? cfg.ent_ctas_per_sm : 8);
    if (blocks > cap) blocks = cap;
    k_entropy<W><<<blocks, W * 32, 0, s>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_reconstruct(const RecParams &p, const LaunchCfg &cfg, cudaStream_t s) {
    if (p.n <= 0) return cudaSuccess;
    int blocks = p.n;
    int cap = num_sms() * (cfg.rec_ctas_per_sm > 0 ? cfg.rec_ctas_per_sm : 6);
    if (blocks > cap) blocks = cap;
    k_reconstruct<<<blocks, 128, 0, s>>>(p);
    return cudaGetLastError();
}

}  // namespace mcb
