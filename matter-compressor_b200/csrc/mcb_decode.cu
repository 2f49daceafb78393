// mcb_decode.cu -- sm_100a block decode: entropy stage + reconstruction stage.
//
// Stage 1, k_entropy: one LANE per block. The adaptive binary range decoder
// is a serial dependency chain per block (src/mc_codec.c:197-226), so the
// parallelism is across blocks: every lane of a warp runs its own decoder and
// the loop body decodes exactly one bin per lane per iteration (a flat state
// machine), so lanes never wait on each other inside a block. The per-bin
// chain is kept short: the significance band is tracked by scan-position
// boundaries and the density by a running count, so the only shared-memory
// read on the chain is the context itself. The lane's adaptive contexts sit
// in shared memory as 32-bit words (context j of lane l at word j*32+l:
// conflict-free). Output per block: a small header (dc, flags) and a list of
// nonzero levels plus corrections.
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

#include "mcb_devinfo.h"
#include "mcb_format.h"
#include "mcb_kernels.h"
#include "mcb_rowstore.cuh"

namespace mcb {

__constant__ float c_cos[16][16];
// c_bend[b]: the first scan position past band b (b < 7), then kN3 and a
// sentinel; kernels copy it into shared memory at start
__constant__ uint16_t c_bend[9];

// ---------------------------------------------------------------- stage 1
// Lane states. The three fast states cover every bin of the coefficient loop
// and share one branch-free step that every lane of a warp runs together; the
// slow states occur a few times per block and are worked off by the lanes
// that hold them while the rest of the warp waits (see run_lanes). S_IDLE is
// a parked lane, a fixed point of the fast step (see park). The block header
// and EOB are decoded when a lane starts its block.
enum : uint32_t {
    F_SIG = 0,   // significance of scan position p: context sigb + min(popcount(last 16 flags), 3)
    F_MAG,       // unary magnitude rung k: context 56 + k
    F_BYP,       // a bypass bin: the sign of the coefficient at p (m != 0), an Exp-Golomb prefix
                 // bit (m == 0, rem == 0; k counts 12 + the one-bits) or a suffix bit (rem != 0)
    S_IDLE,      // no more blocks for this lane
    S_END,       // scan done: corrections, then the block is finished
    S_EGS,       // an Exp-Golomb suffix of more than 16 bits (only corrupt streams)
    S_DONE
};
// Context slots per lane: the 68 adaptive contexts plus one scratch slot that
// bypass bins read and write in place of a real context. The scratch slot
// directly follows the magnitude ladder, so "the next rung" of rung 11 is it.
constexpr int kCtxSlots = kNumCtx + 1;
constexpr uint32_t kScr = kNumCtx;
static_assert(kScr == kCtxMag + 12, "scratch slot follows the 12 magnitude rungs");
// Exp-Golomb prefixes count in k from this base (the magnitude ladder hands
// over at its 12th rung with k = 12).
constexpr uint32_t kEgBase = 12;
// Byte-permute selector that shifts code left one byte and brings in byte i
// of the window: result = {code.b2, code.b1, code.b0, w.b[i]}; i = sel - kSel0.
constexpr uint32_t kSel0 = 0x2104u;

struct LaneState {
    const uint8_t *abase;      // payload start rounded down to 4 bytes
    uint32_t *ent;             // the block's entries in the arena (first cap of them)
    uint32_t len, off0;        // payload length, payload start - abase
    uint32_t w, nxt, sel, jn;  // window word, next word (raw), byte selector, index of the next word
    uint32_t nmask;            // the next word's payload bytes (applied when it enters the window)
    uint32_t code, range;
    uint32_t st, p, eob, hist, sigb, band, bend, stop;   // hist: significance flags, newest in bit 0
    uint32_t k, m, rem, acc;   // rung / prefix count, magnitude of the pending sign, suffix bits left and read
    uint32_t cc, pc;           // context slot of the next bin and its probability
    uint32_t hdr;              // flag0, flag1, dc bits 7..0 (10 bits, first bin highest)
    uint32_t nent, cap, ovf, bad, ccount;
    int item;
};

// Payload word j (bytes 4j-off0 .. 4j-off0+3 of the payload), bytes past the
// payload read as zero (src/mc_codec.c:96). Loads are 4-byte aligned and never
// start past the word holding the payload's last byte. The raw load and the
// mask of its payload bytes are kept apart: the next word is loaded a refill
// ahead and masked only when it enters the window, so nothing waits on the
// load until then.
__device__ __forceinline__ uint32_t word_mask(const LaneState &L, uint32_t j) {
    const int avail = (int)L.len - ((int)(4 * j) - (int)L.off0);
    return avail >= 4 ? 0xFFFFFFFFu : (avail <= 0 ? 0u : (1u << (8 * avail)) - 1u);
}
__device__ __forceinline__ uint32_t word_raw(const LaneState &L, uint32_t j) {
    uint32_t v = 0;
    if ((int)(4 * j) - (int)L.off0 < (int)L.len) v = __ldg(reinterpret_cast<const uint32_t *>(L.abase) + j);
    return v;
}
__device__ __forceinline__ uint32_t load_word(const LaneState &L, uint32_t j) {
    return word_raw(L, j) & word_mask(L, j);
}

__device__ __forceinline__ void refill(LaneState &L) {
    L.w = L.nxt & L.nmask;
    L.sel = kSel0;
    ++L.jn;
    L.nmask = word_mask(L, L.jn);
    L.nxt = word_raw(L, L.jn);
}

// One payload byte (slow paths). The window always holds an unread byte:
// consuming the last one refills it at once.
__device__ __forceinline__ uint32_t next_byte(LaneState &L) {
    const uint32_t b = (L.w >> (8 * (L.sel - kSel0))) & 0xFFu;
    if (++L.sel == kSel0 + 4) refill(L);
    return b;
}

// Renormalise (src/mc_codec.c:202).
__device__ __forceinline__ void renorm(LaneState &L) {
    while (L.range < (1u << 24)) { L.code = (L.code << 8) | next_byte(L); L.range <<= 8; }
}

// One adaptive bin (src/mc_codec.c:198-204).
__device__ __forceinline__ uint32_t ctx_bin(LaneState &L, uint32_t *cp) {
    const uint32_t p0 = *cp;
    const uint32_t r0 = (L.range >> 12) * p0;
    const uint32_t bit = L.code >= r0 ? 1u : 0u;
    L.code -= bit ? r0 : 0u;
    L.range = bit ? L.range - r0 : r0;
    *cp = bit ? p0 - (p0 >> 4) : p0 + ((4096u - p0) >> 4);
    renorm(L);
    return bit;
}

// nb bypass bits read as one batch, 1 <= nb <= 16 (src/mc_codec.c:205,216-226).
__device__ __forceinline__ uint32_t bypass_bits(LaneState &L, uint32_t nb) {
    L.range >>= nb;
    uint32_t q;
    if (nb == 1) {
        q = L.code >= L.range ? 1u : 0u;
    } else {
        q = L.code / L.range;
        const uint32_t mx = (1u << nb) - 1u;
        q = q > mx ? mx : q;
    }
    L.code -= q * L.range;
    renorm(L);
    return q;
}

// Any number of bypass bits: pieces of 16, most significant first
// (src/mc_codec.c:219-220).
__device__ __forceinline__ uint32_t bypass_long(LaneState &L, uint32_t nb) {
    uint32_t v = 0;
    while (nb > 16) { v = (v << 16) | bypass_bits(L, 16); nb -= 16; }
    return nb ? (v << nb) | bypass_bits(L, nb) : v;
}

// Exp-Golomb value in bypass bins (src/mc_codec.c:234-238); a prefix of
// kEgCap one-bits marks the stream bad and yields 0.
__device__ __forceinline__ uint32_t eg_value(LaneState &L) {
    uint32_t nb = 0;
    while (bypass_bits(L, 1)) {
        if (++nb >= (uint32_t)kEgCap) { L.bad = 1; return 0; }
    }
    if (!nb) return 0;
    return ((1u << (nb & 31)) | bypass_long(L, nb)) - 1u;
}

// Appends one entry; false (stream cut short) when a corrupt stream also
// exhausts the shared overflow pool.
__device__ __forceinline__ bool put_entry(LaneState &L, const EntParams &P, uint32_t v) {
    const uint32_t j = L.nent;
    if (j < L.cap) {
        L.ent[j] = v;
    } else {   // only corrupt streams get here
        if (L.ovf == 0xFFFFFFFFu) {
            const uint32_t need = kEntryMax - L.cap;
            const uint32_t off = atomicAdd(P.pool_used, need);
            if ((uint64_t)off + need > P.pool_cap) { L.bad = 1; L.st = S_DONE; return false; }
            L.ovf = off;
        }
        P.pool[L.ovf + (j - L.cap)] = v;
    }
    L.nent = j + 1;
    return true;
}

// Context slot of the bin the lane's state asks for next and its current
// value; bypass bins use the scratch slot.
__device__ __forceinline__ void load_ctx(LaneState &L, const uint32_t *ctx) {
    L.cc = L.st == F_SIG ? L.sigb + min((uint32_t)__popc(L.hist & 0xFFFFu), 3u)
                         : (L.st == F_MAG ? (uint32_t)kCtxMag + L.k : kScr);
    L.pc = ctx[L.cc * 32];
}

// flags bit 1 (has corrections) is the second header bin
__device__ __forceinline__ bool has_corr(const LaneState &L) { return (L.hdr >> 8) & 1; }

// A lane with no more work: a fixed point of fast_step. With code 0, range
// 0xFFFFF000 and probability 4096 on the scratch slot, every step decodes a
// 0 that leaves range, probability and selector as they are, so the lane
// reads nothing, stores nothing and raises no event.
__device__ __forceinline__ void park(LaneState &L) {
    L.st = S_IDLE;
    L.item = -1;
    L.code = 0;
    L.range = 0xFFFFF000u;
    L.pc = 4096;
    L.cc = kScr;
    L.sel = kSel0;
    L.m = 0;
    L.rem = 0;
}

// Scan position L.p is current and L.p >= L.stop: a band change and/or the
// end of the scan. The last position before the EOB is significant by
// definition and costs no bin (src/mc_codec.c:364); past the EOB the
// coefficient loop ends.
__device__ __forceinline__ void position_event(LaneState &L, const uint32_t *ctx, const uint16_t *s_bend) {
    while (L.p >= L.bend) { L.band++; L.sigb += 4; L.bend = s_bend[L.band]; }
    if (L.p + 1 >= L.eob) {
        if (L.p + 1 == L.eob) {
            L.hist = (L.hist << 1) | 1u;
            L.st = F_MAG;
            L.k = 0;
        } else {
            L.st = S_END;
        }
    }
    L.stop = min(L.bend, L.eob - 1);   // eob >= 1 here (eob == 0 never enters the scan)
    load_ctx(L, ctx);
}

// Starts block `slot`: contexts from the quality table, range decoder,
// header bins, EOB (src/mc_codec.c:739-757, 321-327).
__device__ __forceinline__ void lane_begin(LaneState &L, const EntParams &P, uint32_t *ctx, const uint16_t *s_bend,
                                           int slot) {
    const DecItem &it = P.items[slot];
    L.item = slot;
    const uintptr_t src = (uintptr_t)it.src;
    L.abase = reinterpret_cast<const uint8_t *>(src & ~(uintptr_t)3);
    L.off0 = (uint32_t)(src & 3);
    L.len = it.len;
    L.ent = P.arena + P.base[slot];
    L.cap = entry_cap(L.len);
    L.ovf = 0xFFFFFFFFu;
    L.bad = 0;
    L.nent = 0;
    L.ccount = 0;
    L.hdr = 0;
    L.p = 0; L.eob = 0; L.hist = 0; L.k = 0; L.m = 0; L.rem = 0; L.acc = 0;
    L.band = 0; L.sigb = kCtxSig; L.bend = s_bend[0]; L.stop = 0;
    if (L.len == 0) { L.st = S_DONE; return; }   // absent block: zeros
    const uint4 *q = reinterpret_cast<const uint4 *>(P.qtab[it.qslot].ctx);
#pragma unroll
    for (int j = 0; j < 9; ++j) {               // 72 u16 initial contexts
        const uint4 v = __ldg(q + j);
        const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int h = 0; h < 4; ++h) {
            const int c = j * 8 + h * 2;
            if (c < kNumCtx) ctx[c * 32] = w[h] & 0xFFFFu;
            if (c + 1 < kNumCtx) ctx[(c + 1) * 32] = w[h] >> 16;
        }
    }
    L.w = load_word(L, 0);
    L.sel = kSel0 + L.off0;
    L.jn = 1;
    L.nmask = word_mask(L, 1);
    L.nxt = word_raw(L, 1);
    L.range = 0xFFFFFFFFu;
    L.code = 0;
    for (int i = 0; i < 5; ++i) L.code = (L.code << 8) | next_byte(L);
    for (int i = 0; i < 10; ++i) L.hdr = (L.hdr << 1) | ctx_bin(L, ctx + (kCtxFlag + i) * 32);
    uint32_t k = 0;
    while (k < 13 && ctx_bin(L, ctx + (kCtxEob + k) * 32)) k++;
    const uint32_t eob = k < 2 ? k : (1u << (k - 1)) | bypass_bits(L, k - 1);
    L.eob = eob > (uint32_t)kN3 ? (uint32_t)kN3 : eob;
    if (L.eob == 0) { L.st = S_END; return; }
    L.st = F_SIG;
    position_event(L, ctx, s_bend);
}

__device__ __forceinline__ void lane_finish(LaneState &L, const EntParams &P) {
    EntHdr h;
    h.dc = (uint8_t)(L.hdr & 0xFF);
    h.flags = (uint8_t)(((L.hdr >> 9) & 1) | (((L.hdr >> 8) & 1) << 1));
    h.bad = (uint8_t)L.bad;
    h.pad = 0;
    h.ez = h.ey = h.ex = -1;    // extents are taken from the entries by k_reconstruct
    h.pad2 = 0;
    h.nnz = (uint16_t)(L.nent - 2 * L.ccount);
    h.ncorr = (uint16_t)L.ccount;
    h.ovf = L.ovf;
    P.hdr[L.item] = h;
    if (L.bad) atomicAdd(P.status, 1u);
}

// The sparse max-error corrections after the scan (src/mc_codec.c:770-782):
// count, then per correction a position gap, a sign and a magnitude, each
// gap and magnitude an Exp-Golomb value. Recorded as entry pairs (position,
// wrapping delta) after the coefficients.
__device__ __forceinline__ void decode_corrections(LaneState &L, const EntParams &P) {
    uint32_t n = eg_value(L) + 1u;
    if (L.bad) return;
    if (n > (uint32_t)kN3) n = kN3;
    uint32_t pos = 0;
    for (uint32_t c = 0; c < n; ++c) {
        pos += eg_value(L);
        if (L.bad) return;
        const uint32_t neg = bypass_bits(L, 1);
        const uint32_t m = eg_value(L) + 1u;
        if (L.bad || pos >= (uint32_t)kN3) return;
        if (!put_entry(L, P, pos) || !put_entry(L, P, neg ? 0u - m : m)) return;
        L.ccount++;
    }
}

// The slow states of one lane, run while the rest of its warp waits.
__device__ __forceinline__ void slow_work(LaneState &L, const EntParams &P, const uint32_t *ctx,
                                          const uint16_t *s_bend) {
    if (L.st == S_EGS) {
        // a suffix of more than 16 bits: the batched division form in pieces
        // (src/mc_codec.c:219-224); magnitude 12 + x, x = (1 << nb | suffix) - 1
        const uint32_t nb = L.rem;
        const uint32_t m = 11u + ((1u << (nb & 31)) | bypass_long(L, nb));
        L.rem = 0;
        L.acc = 0;
        if (m != 0) {   // the sign follows as a fast bypass bin
            L.m = m;
            L.st = F_BYP;
            load_ctx(L, ctx);
            return;
        }
        // m wrapped to 0 (a corrupt stream only): a zero-level coefficient,
        // recorded here so that m == 0 keeps meaning "Exp-Golomb prefix"
        bypass_bits(L, 1);
        if (!put_entry(L, P, L.p)) return;
        L.p++;
        L.st = F_SIG;
        L.k = 0;
        if (L.p >= L.stop) position_event(L, ctx, s_bend);
        else load_ctx(L, ctx);
        return;
    }
    // S_END
    if (has_corr(L)) decode_corrections(L, P);
    L.st = S_DONE;
}

// Predicated global store (the compiler turns this into one predicated
// instruction, no branch).
__device__ __forceinline__ void stg_if(bool pred, uint32_t *p, uint32_t v) {
    if (pred) *p = v;
}

// The rare events of a fast step, in this order: a window refill, the rest of
// a renormalisation (none inside an Exp-Golomb suffix), an entry past the
// block's arena share, the end of an Exp-Golomb prefix (a suffix of nb bits
// follows: the range loses its low nb bits, which is the batched read's
// range >> nb, and the suffix bits then halve it, or nb = 0 and the sign
// follows), the end of a suffix (the magnitude is known; the sign follows),
// and a scan position at a band change or the end of the scan.
enum : uint32_t { EV_PFX = 1, EV_PFX_ONE = 2, EV_SFX = 4, EV_OVF = 8, EV_POS = 16 };
__device__ __forceinline__ void fast_event(LaneState &L, const EntParams &P, const uint32_t *ctx,
                                           const uint16_t *s_bend, uint32_t why, uint32_t v) {
    if (L.sel == kSel0 + 4) refill(L);
    if (!(L.st == F_BYP && L.rem != 0)) renorm(L);
    if ((why & EV_OVF) && !put_entry(L, P, v)) return;   // corrupt stream: pool exhausted, block ends
    if (why & EV_PFX) {
        if (why & EV_PFX_ONE) { L.bad = 1; L.st = S_DONE; return; }   // prefix cap reached (corrupt stream)
        const uint32_t nb = L.k - kEgBase;                            // one-bits of the prefix
        if (nb == 0) {
            L.m = 12;
        } else if (nb <= 16) {
            L.rem = nb;
            L.acc = 0;
            L.range &= ~((1u << nb) - 1u);
        } else {
            L.rem = nb;
            L.st = S_EGS;
        }
    }
    if (why & EV_SFX) L.m = 11u + ((1u << (L.k - kEgBase)) | L.acc);
    if (why & EV_POS) position_event(L, ctx, s_bend);
}

// One bin of every lane. The significance bin of position p uses context
// band*4 + min(popcount(last 16 significance flags), 3) (src/mc_codec.c:249-259
// and 353-375); magnitude rung k context 56+k (src/mc_codec.c:268-275); signs
// and Exp-Golomb bits are bypass bins (:205, 216-238) computed by the same
// instructions with r0 = range/2 and the scratch context slot. An Exp-Golomb
// suffix of nb <= 16 bits is the reference's batched read range >>= nb,
// q = min(code / range, 2^nb - 1), code -= q * range: with the range's low nb
// bits cleared first, nb halvings without renormalisation between them are
// that long division bit by bit, clamp included, and leave the same code and
// range; the renormalisation follows the last bit.
// The step is software-pipelined: the bin's context value (pc, slot cc) was
// fetched during the previous step, and this step fetches both candidate
// contexts of the next bin (one per value of this bin) before it decodes, so
// the shared-memory round trip overlaps the arithmetic; a next context equal
// to this bin's takes the freshly updated value instead. Every lane runs the
// same straight-line code of selects and predicated stores; a parked lane
// passes through unchanged, and lanes in slow states never get here. Rare
// events (see fast_event) share one branch.
__device__ __forceinline__ void fast_step(LaneState &L, const EntParams &P, uint32_t *ctx, const uint16_t *s_bend) {
    const uint32_t st = L.st, m0 = L.m, rem0 = L.rem, k0 = L.k, cc = L.cc, pc = L.pc;
    const bool is_sig = st == F_SIG, is_mag = st == F_MAG, is_byp = st == F_BYP;
    const bool is_sign = is_byp & (m0 != 0u);
    const bool is_sfx = is_byp & (rem0 != 0u);
    const bool is_pfx = is_byp & !is_sign & !is_sfx;
    // candidate contexts of the next bin: c0 if this bin is 0, c1 if it is 1.
    // After a significance bin of 0 the flag window drops its oldest flag.
    const uint32_t csig = L.sigb + min((uint32_t)__popc(L.hist & (is_sig ? 0x7FFFu : 0xFFFFu)), 3u);
    const uint32_t c0 = (is_sig | is_sign) ? csig : kScr;
    const uint32_t c1 = is_sig ? (uint32_t)kCtxMag : (is_mag ? min(cc + 1u, kScr) : c0);
    const uint32_t q0 = ctx[c0 * 32];
    const uint32_t q1 = ctx[c1 * 32];
    // this bin
    const uint32_t r0 = is_byp ? L.range >> 1 : (L.range >> 12) * pc;
    const bool bit = L.code >= r0;
    const uint32_t code = bit ? L.code - r0 : L.code;
    const uint32_t range = (bit & !is_byp) ? L.range - r0 : r0;
    const uint32_t np0 = (15u * pc + (bit ? 15u : 4096u)) >> 4;   // p - (p >> 4) or p + ((4096 - p) >> 4)
    ctx[cc * 32] = np0;   // bypass bins write the scratch slot
    // renormalisation, first byte (src/mc_codec.c:202); not between the bits
    // of a suffix
    const bool sup = is_sfx & (rem0 > 1u);
    const bool need = (range < (1u << 24)) & !sup;
    L.code = need ? __byte_perm(code, L.w, L.sel) : code;
    L.range = need ? range << 8 : range;
    L.sel += need ? 1u : 0u;
    // next bin's context
    const uint32_t ncc = bit ? c1 : c0;
    L.pc = ncc == cc ? np0 : (bit ? q1 : q0);
    L.cc = ncc;
    // state
    const bool esc = is_mag & bit & (k0 == 11u);   // 12th rung set: Exp-Golomb tail
    L.hist = is_sig ? (L.hist << 1) | (bit ? 1u : 0u) : L.hist;
    L.k = is_sig ? 0u : ((bit & !is_sfx) ? k0 + 1u : k0);
    L.m = (is_mag & !bit) ? k0 + 1u : (is_sign ? 0u : m0);
    L.acc = is_sfx ? (L.acc << 1) | (bit ? 1u : 0u) : L.acc;
    L.rem = is_sfx ? rem0 - 1u : rem0;
    L.st = is_sig ? (bit ? (uint32_t)F_MAG : (uint32_t)F_SIG)
                  : (is_mag ? ((bit & !esc) ? (uint32_t)F_MAG : (uint32_t)F_BYP) : (is_sign ? (uint32_t)F_SIG : st));
    // a sign completes the coefficient at scan position p: its entry
    const uint32_t p = L.p;
    const bool adv = (is_sig & !bit) | is_sign;
    const uint32_t np = p + (adv ? 1u : 0u);
    L.p = np;
    const uint32_t v = p | ((bit ? 0u - m0 : m0) << 16);
    const bool room = L.nent < L.cap;
    stg_if(is_sign & room, L.ent + L.nent, v);
    L.nent += (is_sign & room) ? 1u : 0u;
    const bool pfx_end = is_pfx & (!bit | (k0 + 1u >= kEgBase + (uint32_t)kEgCap));
    const bool pos = adv & (np >= L.stop);
    const bool ovf = is_sign & !room;
    const bool sfx_end = is_sfx & (rem0 == 1u);
    if ((L.sel == kSel0 + 4) | ((L.range < (1u << 24)) & !sup) | pfx_end | sfx_end | pos | ovf) {
        const uint32_t why = (pfx_end ? (uint32_t)EV_PFX : 0u) | ((pfx_end & bit) ? (uint32_t)EV_PFX_ONE : 0u) |
                             (sfx_end ? (uint32_t)EV_SFX : 0u) | (ovf ? (uint32_t)EV_OVF : 0u) |
                             (pos ? (uint32_t)EV_POS : 0u);
        fast_event(L, P, ctx, s_bend, why, v);
    }
}

// Work queue of a launch: the first ncoded entries of the processing order
// (longest payload first). Lane g starts with entry g; later entries are
// claimed from the launch's counter in runs of P.claim consecutive entries.
struct Claim {
    int next, end;
};
__device__ __forceinline__ int claim_next(Claim &c, const EntParams &P, int nlanes) {
    if (c.next >= c.end) {
        const uint32_t run = P.claim > 0 ? (uint32_t)P.claim : 1u;
        c.next = nlanes + (int)atomicAdd(P.counter, run);
        c.end = c.next + (int)run;
    }
    return c.next++;
}

// Every lane of the warp decodes blocks until the queue is empty. Lane gtid
// starts with entry gtid (none when gtid < 0), then claims from the counter. Fast steps
// run while every lane is in a fast state or parked; when a lane reaches a
// slow state the warp leaves the loop, that lane works its slow states off
// (finishing its block and starting the next one), and the loop resumes.
// Every block ends after a bounded number of bins (finite scan, capped
// Exp-Golomb prefixes, bounded correction count) and every lane claims at
// most ncoded blocks, so the loop ends. on_done(item) runs for every
// finished block.
template <class OnDone>
__device__ __forceinline__ void run_lanes(LaneState &L, const EntParams &P, uint32_t *ctx, const uint16_t *s_bend,
                                          int gtid, int nlanes, OnDone on_done) {
    memset(&L, 0, sizeof L);
    park(L);
    L.st = S_DONE;
    Claim c = gtid >= 0 ? Claim{gtid, gtid + 1} : Claim{0, 0};   // gtid < 0: queue claims only
    for (;;) {
        // two steps per loop turn (the loop-carried lane state then needs
        // no register shuffling between the two), the check after each
        for (;;) {
            if (__any_sync(0xFFFFFFFFu, L.st >= S_END)) break;
            fast_step(L, P, ctx, s_bend);
            if (__any_sync(0xFFFFFFFFu, L.st >= S_END)) break;
            fast_step(L, P, ctx, s_bend);
        }
        while (L.st >= S_END) {
            if (L.st != S_DONE) {
                slow_work(L, P, ctx, s_bend);
                continue;
            }
            if (L.item >= 0) {
                lane_finish(L, P);
                on_done(L.item);
            }
            const int nx = claim_next(c, P, nlanes);
            if (nx < P.ncoded) lane_begin(L, P, ctx, s_bend, P.order ? (int)P.order[nx] : nx);
            else park(L);
        }
        if (__all_sync(0xFFFFFFFFu, L.st == S_IDLE)) break;
    }
}

// The whole stream of one block on one thread, after lane_begin, written for
// the latency of one thread alone on its warp (no other lane shares its
// instructions). All contexts of the coefficient loop that the common bins
// use are held in registers: the four significance contexts of the current
// band (the one in use as a live probability, written back when the density
// changes) and the twelve magnitude rungs. A run of insignificant positions
// then costs per bin the range split, the compare, the probability update
// and one test for the rare events (a renormalisation, the flag that leaves
// the 16-position density window, the end of the band or the scan). A
// significant bin decodes its coefficient (magnitude, sign, entry) in place
// and the run goes on; the common steps of a coefficient use selects rather
// than branches, whose divergence bookkeeping costs more than their work.
// Band changes, Exp-Golomb tails and the corrections take the shared step
// functions (position_event, renorm, eg_value, put_entry, slow_work). Bands
// only advance, so a band's register contexts are never written back to
// shared memory, and the magnitude rungs are used by nothing else.
__device__ __forceinline__ uint32_t pick4(uint32_t c, uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3) {
    return c == 0 ? a0 : (c == 1 ? a1 : (c == 2 ? a2 : a3));
}
// p + ((4096 - p) >> 4) and p - (p >> 4) (src/mc_codec.c:198-204) as one
// multiply-add and a shift: equal for every p in 0..4096
__device__ __forceinline__ uint32_t prob_after0(uint32_t p) { return (15u * p + 4096u) >> 4; }
__device__ __forceinline__ uint32_t prob_after1(uint32_t p) { return (15u * p + 15u) >> 4; }
// One magnitude rung on a register context; after a 1 the range is
// renormalised here, after the closing 0 by the caller.
__device__ __forceinline__ bool rung(LaneState &L, uint32_t &g) {
    const uint32_t r = (L.range >> 12) * g;
    if (L.code < r) {
        L.range = r;
        g = prob_after0(g);
        return false;
    }
    L.code -= r;
    L.range -= r;
    g = prob_after1(g);
    if (L.range < (1u << 24)) renorm(L);
    return true;
}

// Renormalisation with the common case (one byte, the window not emptied)
// by selects; a second byte or a window refill takes the loop.
__device__ __forceinline__ void renorm_sel(LaneState &L) {
    const bool need = L.range < (1u << 24);
    L.code = need ? __byte_perm(L.code, L.w, L.sel) : L.code;
    L.range = need ? L.range << 8 : L.range;
    L.sel += need ? 1u : 0u;
    if ((L.sel == kSel0 + 4) | (L.range < (1u << 24))) {
        if (L.sel == kSel0 + 4) refill(L);
        renorm(L);
    }
}

__device__ __forceinline__ void solo_entropy(LaneState &L, const EntParams &P, uint32_t *ctx,
                                             const uint16_t *s_bend) {
    uint32_t sigb = L.sigb;
    uint32_t s0 = ctx[(sigb + 0) * 32], s1 = ctx[(sigb + 1) * 32];
    uint32_t s2 = ctx[(sigb + 2) * 32], s3 = ctx[(sigb + 3) * 32];
    uint32_t g0 = ctx[(kCtxMag + 0) * 32], g1 = ctx[(kCtxMag + 1) * 32], g2 = ctx[(kCtxMag + 2) * 32];
    uint32_t g3 = ctx[(kCtxMag + 3) * 32], g4 = ctx[(kCtxMag + 4) * 32], g5 = ctx[(kCtxMag + 5) * 32];
    uint32_t g6 = ctx[(kCtxMag + 6) * 32], g7 = ctx[(kCtxMag + 7) * 32], g8 = ctx[(kCtxMag + 8) * 32];
    uint32_t g9 = ctx[(kCtxMag + 9) * 32], g10 = ctx[(kCtxMag + 10) * 32], g11 = ctx[(kCtxMag + 11) * 32];
    uint32_t h = L.hist & 0xFFFFu;   // the last 16 significance flags, newest in bit 0
    uint32_t cnt = __popc(h);
    // a position event; the band's contexts come into registers when it changes
    auto event = [&]() {
        L.hist = h;
        position_event(L, ctx, s_bend);
        if (L.sigb != sigb) {
            sigb = L.sigb;
            s0 = ctx[(sigb + 0) * 32]; s1 = ctx[(sigb + 1) * 32];
            s2 = ctx[(sigb + 2) * 32]; s3 = ctx[(sigb + 3) * 32];
        }
        h = L.hist & 0xFFFFu;
        cnt = __popc(h);
    };
    // the coefficient at L.p, known significant: the unary magnitude
    // (src/mc_codec.c:268-275), the sign, the entry, the next position;
    // false when the block ends (an Exp-Golomb prefix at the cap or the
    // overflow pool exhausted: corrupt streams only)
    auto coef = [&]() -> bool {
        uint32_t m;
        const uint32_t r = (L.range >> 12) * g0;   // rung 0, by selects
        const bool b0 = L.code >= r;
        L.code = b0 ? L.code - r : L.code;
        L.range = b0 ? L.range - r : r;
        g0 = (15u * g0 + (b0 ? 15u : 4096u)) >> 4;
        renorm_sel(L);
        if (!b0) {
            m = 1;
        } else {
            if (!rung(L, g1)) m = 2;
            else if (!rung(L, g2)) m = 3;
            else if (!rung(L, g3)) m = 4;
            else if (!rung(L, g4)) m = 5;
            else if (!rung(L, g5)) m = 6;
            else if (!rung(L, g6)) m = 7;
            else if (!rung(L, g7)) m = 8;
            else if (!rung(L, g8)) m = 9;
            else if (!rung(L, g9)) m = 10;
            else if (!rung(L, g10)) m = 11;
            else if (!rung(L, g11)) m = 12;
            else m = 0;
            if (m == 0) {   // the twelfth rung set: 12 + an Exp-Golomb value
                m = 12u + eg_value(L);
                if (L.bad) { L.st = S_DONE; return false; }   // prefix cap
            }
            renorm(L);
        }
        L.range >>= 1;   // the sign, a bypass bin (src/mc_codec.c:205)
        const bool neg = L.code >= L.range;
        L.code = neg ? L.code - L.range : L.code;
        renorm_sel(L);
        const uint32_t v = L.p | ((neg ? 0u - m : m) << 16);
        if (L.nent < L.cap) {
            L.ent[L.nent++] = v;
        } else if (!put_entry(L, P, v)) {
            return false;   // S_DONE
        }
        ++L.p;
        L.st = F_SIG;
        if (L.p >= L.stop) event();
        return true;
    };
    for (;;) {
        if (L.st == F_MAG) {   // the implicit last position (lane_begin or an event)
            if (!coef()) break;
            continue;
        }
        if (L.st != F_SIG) break;
        // a run of significance bins at L.p < L.stop, the context in use as
        // the live probability pc
        uint32_t c = min(cnt, 3u);
        uint32_t pc = pick4(c, s0, s1, s2, s3);
        for (;;) {
            const uint32_t r0 = (L.range >> 12) * pc;
            if (L.code >= r0) {   // significant
                L.code -= r0;
                L.range -= r0;
                pc = prob_after1(pc);
                s0 = c == 0 ? pc : s0; s1 = c == 1 ? pc : s1;
                s2 = c == 2 ? pc : s2; s3 = c == 3 ? pc : s3;
                h = (h << 1) | 1u;
                cnt += 1u - (h >> 16);   // the flag that entered, the one that left
                h &= 0xFFFFu;
                renorm_sel(L);
                if (!coef()) break;
                if (L.st != F_SIG) break;
                c = min(cnt, 3u);
                pc = pick4(c, s0, s1, s2, s3);
                continue;
            }
            L.range = r0;
            pc = prob_after0(pc);
            h <<= 1;
            ++L.p;
            if ((L.range < (1u << 24)) | (L.p >= L.stop) | (h > 0xFFFFu)) {
                if (L.range < (1u << 24)) renorm(L);
                if ((L.p >= L.stop) | (h > 0xFFFFu)) {
                    s0 = c == 0 ? pc : s0; s1 = c == 1 ? pc : s1;
                    s2 = c == 2 ? pc : s2; s3 = c == 3 ? pc : s3;
                    cnt -= h >> 16;   // the flag that left the window
                    h &= 0xFFFFu;
                    if (L.p >= L.stop) {
                        event();
                        if (L.st != F_SIG) break;
                    }
                    c = min(cnt, 3u);
                    pc = pick4(c, s0, s1, s2, s3);
                }
            }
        }
    }
    while (L.st != S_DONE) slow_work(L, P, ctx, s_bend);
}

template <int WARPS>
__global__ void __launch_bounds__(WARPS * 32) k_entropy(EntParams P) {
    // s_bend[b]: first scan position past band b; then the lanes' contexts,
    // context j of lane l of warp w at word (w * kCtxSlots + j) * 32 + l
    extern __shared__ uint32_t s_ent[];
    uint16_t *s_bend = reinterpret_cast<uint16_t *>(s_ent);
    if (threadIdx.x < 9) s_bend[threadIdx.x] = c_bend[threadIdx.x];
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t *ctx = s_ent + 8 + warp * kCtxSlots * 32 + lane;
    LaneState L;
    // warps 0..nsolo-1 of the grid: order entry `warp` on the warp's first
    // thread alone, then the queue
    const int gwarp = blockIdx.x * WARPS + warp;
    if (gwarp < P.nsolo) {
        if (lane == 0) {
            memset(&L, 0, sizeof L);
            lane_begin(L, P, ctx, s_bend, (int)P.order[gwarp]);
            solo_entropy(L, P, ctx, s_bend);
            lane_finish(L, P);
        }
        __syncwarp();
    }
    EntParams F = P;   // the rest of the order, one lane per block
    F.order = P.order ? P.order + P.nsolo : nullptr;
    F.ncoded = P.ncoded - P.nsolo;
    const int gtid = (int)(blockIdx.x * blockDim.x + threadIdx.x) - 32 * P.nsolo;
    run_lanes(L, F, ctx, s_bend, gtid, (int)(gridDim.x * blockDim.x) - 32 * P.nsolo, [](int) {});
}
// dynamic shared memory of k_entropy<W>
constexpr size_t entropy_smem(int warps) { return 32 + sizeof(uint32_t) * kCtxSlots * 32 * (size_t)warps; }

// The entropy stage with every block on a single thread: each warp's first
// thread decodes blocks of the order one after another (entry `warp` first,
// then claims from the counter), the other 31 threads leave at once. A block
// then costs a few times fewer cycles per bin than as a lane of k_entropy, at
// several times the issue slots per bin, which pays where a batch is too
// small to fill the machine and its longest blocks set the stage's time. The
// threads' contexts share one 32-column region of shared memory (column =
// warp index), conflict-free like k_entropy's. Two CTAs of 16 warps per SM
// fit the register file at 64 registers a thread.
constexpr int kSoloWarps = 16;
__global__ void __launch_bounds__(kSoloWarps * 32, 2) k_entropy_solo(EntParams P) {
    __shared__ uint32_t s_ctx[kCtxSlots * 32];
    __shared__ uint16_t s_bend[9];
    if (threadIdx.x < 9) s_bend[threadIdx.x] = c_bend[threadIdx.x];
    __syncthreads();
    if (threadIdx.x & 31) return;
    const int warp = threadIdx.x >> 5;
    uint32_t *ctx = s_ctx + warp;
    const int nwarps = gridDim.x * kSoloWarps;
    for (int j = blockIdx.x * kSoloWarps + warp; j < P.ncoded; j = nwarps + (int)atomicAdd(P.counter, 1u)) {
        LaneState L;
        memset(&L, 0, sizeof L);
        lane_begin(L, P, ctx, s_bend, P.order ? (int)P.order[j] : j);
        solo_entropy(L, P, ctx, s_bend);
        lane_finish(L, P);
    }
}

// ---------------------------------------------------------------- stage 2
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }

// Packed pairs: sm_100 executes two IEEE single-precision round-to-nearest
// adds or multiplies per instruction (add/sub/mul.rn.f32x2), each lane of the
// pair rounding exactly like its scalar __fadd_rn / __fmul_rn. One caution,
// measured with ptxas 12.9 on sm_100a: a packed multiply whose result feeds a
// packed add is contracted into a single-rounding packed FMA despite the .rn
// qualifiers (even inside one asm statement, and also when the product is
// written as fma with a -0 addend). The multiply-accumulates below therefore
// pair a packed multiply with scalar __fadd_rn adds, a combination that keeps
// both roundings; packed adds are used only on sums.
__device__ __forceinline__ float2 add2(float2 a, float2 b) {
    float2 d;
    asm("{.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "add.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;}"
        : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
    float2 d;
    asm("{.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "sub.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;}"
        : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b) {
    float2 d;
    asm("{.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "mul.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;}"
        : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}
// acc + w*v per lane with two roundings (see above)
__device__ __forceinline__ float2 madd2(float2 acc, float2 w, float2 v) {
    const float2 p = mul2(w, v);
    return make_float2(__fadd_rn(acc.x, p.x), __fadd_rn(acc.y, p.y));
}
__device__ __forceinline__ float2 lo2(float4 v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(float4 v) { return make_float2(v.z, v.w); }

// 4 adjacent lines x 2 outputs (m, m+1): even-k and odd-k halves, each a
// sequential sum over ascending k (src/mc_codec_float.h:102-104). in[k*ks]
// holds the 4 lines' k-th inputs, W[k*16 + m/2] = {c[k][m], c[k][m], c[k][m+1], c[k][m+1]}.
struct Acc4 { float2 e0a, e0b, e1a, e1b, o0a, o0b, o1a, o1b; };
// From four terms on, each sum starts from its first product rather than
// from 0 plus it: equal, except that 0 + (-0) is +0 where the product alone
// keeps -0; a zero of either sign stays a zero through every later add and
// multiply and rounds to the same voxel, and every nonzero sum is unchanged.
// With fewer terms a half-sum could be a bare product, which the packed e +/- o
// below would take into one fused rounding (see madd2), so those start at 0.
__device__ __forceinline__ Acc4 lines4(const float4 *in, int ks, int K, const float4 *W, int mh) {
    Acc4 a;
    int k;
    if (K >= 4) {
        const float4 v = in[0], w = W[mh];
        const float2 w0 = lo2(w), w1 = hi2(w);
        a.e0a = mul2(w0, lo2(v)); a.e0b = mul2(w0, hi2(v));
        a.e1a = mul2(w1, lo2(v)); a.e1b = mul2(w1, hi2(v));
        const float4 u = in[ks], x = W[8 + mh];
        const float2 x0 = lo2(x), x1 = hi2(x);
        a.o0a = mul2(x0, lo2(u)); a.o0b = mul2(x0, hi2(u));
        a.o1a = mul2(x1, lo2(u)); a.o1b = mul2(x1, hi2(u));
        k = 2;
    } else {
        const float2 z = make_float2(0.f, 0.f);
        a.e0a = a.e0b = a.e1a = a.e1b = a.o0a = a.o0b = a.o1a = a.o1b = z;
        k = 0;
    }
    // (even, odd) pairs of k without a per-step guard, then the last even k
#pragma unroll 2
    for (; k + 1 < K; k += 2) {
        const float4 v = in[k * ks], w = W[k * 8 + mh];
        const float2 w0 = lo2(w), w1 = hi2(w);
        a.e0a = madd2(a.e0a, w0, lo2(v)); a.e0b = madd2(a.e0b, w0, hi2(v));
        a.e1a = madd2(a.e1a, w1, lo2(v)); a.e1b = madd2(a.e1b, w1, hi2(v));
        const float4 u = in[(k + 1) * ks], x = W[(k + 1) * 8 + mh];
        const float2 x0 = lo2(x), x1 = hi2(x);
        a.o0a = madd2(a.o0a, x0, lo2(u)); a.o0b = madd2(a.o0b, x0, hi2(u));
        a.o1a = madd2(a.o1a, x1, lo2(u)); a.o1b = madd2(a.o1b, x1, hi2(u));
    }
    if (k < K) {
        const float4 v = in[k * ks], w = W[k * 8 + mh];
        const float2 w0 = lo2(w), w1 = hi2(w);
        a.e0a = madd2(a.e0a, w0, lo2(v)); a.e0b = madd2(a.e0b, w0, hi2(v));
        a.e1a = madd2(a.e1a, w1, lo2(v)); a.e1b = madd2(a.e1b, w1, hi2(v));
    }
    return a;
}

// Entry j of a block. CG: read through L2 only (__ldcg), for entries that
// another SM may have written during this kernel (the fused decode): a line
// this SM cached earlier for a neighbouring block must not be reused.
template <bool CG>
__device__ __forceinline__ uint32_t entry_at(const RecParams &P, uint64_t base, uint32_t cap, uint32_t ovf, uint32_t j) {
    if (j < cap) return CG ? __ldcg(P.arena + base + j) : P.arena[base + j];
    if (ovf == 0xFFFFFFFFu) return 0u;
    return CG ? __ldcg(P.pool + ovf + (j - cap)) : P.pool[ovf + (j - cap)];
}
template <bool CG>
__device__ __forceinline__ EntHdr load_hdr(const EntHdr *h) {
    if (!CG) return *h;
    const uint4 v = __ldcg(reinterpret_cast<const uint4 *>(h));
    EntHdr r;
    memcpy(&r, &v, sizeof r);
    return r;
}

// (int)lrintf(v) + dc clamped to u8 (src/mc_codec.c:766-769). Adding 1.5*2^23
// rounds to an integer half-to-even for |v| < 2^22, which is exactly lrintf;
// larger values (only from corrupt streams) take the 64-bit conversion.
__device__ __forceinline__ uint32_t to_u8(float v, int dc) {
    int r;
    if (fabsf(v) < 4194304.0f) {
        r = __float_as_int(fadd(v, 12582912.0f)) - 0x4B400000;
    } else {
        r = (int)(uint32_t)(unsigned long long)__float2ll_rn(v);
    }
    const int s = r + dc;
    return (uint32_t)(s < 0 ? 0 : s > 255 ? 255 : s);
}
// four voxels (x, x+1 | x+2, x+3) -> little-endian u8x4
__device__ __forceinline__ uint32_t pack4(float2 a, float2 b, int dc) {
    return to_u8(a.x, dc) | (to_u8(a.y, dc) << 8) | (to_u8(b.x, dc) << 16) | (to_u8(b.y, dc) << 24);
}
// The same for a block whose voxels are all known to satisfy |v| < 2^21:
// round half to even by the magic add, + dc, and a saturating pack (four
// ints to u8, s0 in the low byte).
__device__ __forceinline__ int rint_dc(float v, int dc) {
    return __float_as_int(fadd(v, 12582912.0f)) - 0x4B400000 + dc;
}
__device__ __forceinline__ uint32_t pack4_fast(float2 a, float2 b, int dc) {
    uint32_t t, d;
    asm("cvt.pack.sat.u8.s32.b32 %0, %1, %2, 0;" : "=r"(t) : "r"(rint_dc(b.y, dc)), "r"(rint_dc(b.x, dc)));
    asm("cvt.pack.sat.u8.s32.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(rint_dc(a.y, dc)), "r"(rint_dc(a.x, dc)), "r"(t));
    return d;
}
// Every output voxel is a sum of at most 4096 terms coef * c[kz][z]c[ky][y]c[kx][x]
// with |c| <= sqrt(2/16), so |v| <= L1(coef) * 0.0442; below this L1 norm
// (with a factor-2 margin for rounding) every voxel takes the fast rounding.
constexpr float kFastL1 = 2097152.0f / 0.04419417f;

// Shared-memory layouts. A (pass-1 output) rows of 16 floats are padded to
// kRowF so that the lanes of a warp that write the four outputs
// (m, m+1, 15-m, 14-m) of a line hit different banks. B (pass-2 output) rows
// are not padded: float4 group g of row y (in every cz plane) sits at group
// g ^ bswz(y), so pass-3 loads (rows y, y+1 of one plane) are conflict-free
// and pass-2 stores at most 2-way, in 4 KB less shared memory per CTA.
constexpr int kRowF = 20;            // A rows of 16 floats
constexpr int kRowB = 16;            // B rows
constexpr int kPlaneB = 16 * kRowB;  // one cz plane of B
__device__ __forceinline__ int bswz(int y) { return (y >> 1) & 3; }
// The coefficient box in B: coefficient (cz, cy, cx) at cz*kBoxPlane + cx*16 + cy.
// For one (cz, cx) the 16 cy values are contiguous, so pass 1 reads the k-th
// inputs of 4 adjacent x-lines as one float4; planes are padded by 16 floats
// so that the two planes a warp reads sit in different banks. B holds kBoxB
// floats (the pass-2 output uses the first 16 * kPlaneB).
constexpr int kBoxPlane = 16 * 16 + 16;
constexpr int kBoxB = 16 * kBoxPlane;
constexpr int kStageZ = 272;         // stage: one z slice of 16 rows of 16 bytes
constexpr int kStageBytes = 16 * kStageZ;

// Per-CTA state of the block being reconstructed: extents and L1 norm. Both
// are zero when a block starts, like the coefficient box (rec_init, then
// every block puts them back).
__shared__ int s_rec_ext[3];
__shared__ float s_rec_l1;

// Before a CTA's first block: an all-zero coefficient box, zero extents and
// L1 norm. The caller synchronises before the first block.
__device__ __forceinline__ void rec_init(float *sB) {
    for (int i = threadIdx.x; i < kBoxB / 4; i += blockDim.x)
        reinterpret_cast<float4 *>(sB)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (threadIdx.x < 3) s_rec_ext[threadIdx.x] = 0;
    if (threadIdx.x == 3) s_rec_l1 = 0.0f;
}

// Reconstruct one block into a stage (z slices of kStageZ bytes). Thread t owns the
// output pair (m, m+1) = 2*(t&3) of every line it touches; its cosine weights
// come from the shared table W.
// On entry the coefficient box in sB, s_rec_ext and s_rec_l1 are zero; the
// block leaves them zero again.
// next: the item this CTA reconstructs after this one (-1: none). While this
// block's transform runs, the start of the next block's entry list is
// prefetched into L2, so that its loads do not wait on DRAM.
template <bool CG>
__device__ __forceinline__ void reconstruct_block(const RecParams &P, int item, float *sA, float *sB,
                                                  uint8_t *stage, const float4 *W, int next = -1) {
    const int tid = threadIdx.x;
    const int m = (tid & 3) * 2;
    // the next block's entry window, fetched early (used after the dequantisation)
    uint64_t nbase = 0;
    uint32_t nlines = 0;
    if (next >= 0 && tid < 32) {
        // the entries it reads: coefficients and correction pairs, at most 512
        nbase = __ldg(P.base + next);
        const uint4 hv = __ldg(reinterpret_cast<const uint4 *>(P.hdr + next));
        EntHdr hn;
        memcpy(&hn, &hv, sizeof hn);
        const uint32_t used = min((uint32_t)hn.nnz + 2u * hn.ncorr, entry_cap(__ldg(&P.items[next].len)));
        nlines = (min(used, 512u) + 31) / 32;   // 128-byte lines
    }
    const DecItem it = P.items[item];
    const EntHdr h = load_hdr<CG>(P.hdr + item);
    const uint64_t base = P.base[item];
    const uint32_t cap = entry_cap(it.len);
    // the header comes from k_entropy; the guards keep every index below
    // inside shared memory whatever its contents
    const bool sane = h.nnz <= kN3 && h.ncorr <= kN3;
    const int dc = it.len && sane ? h.dc : 0;
    const int nnz = it.len && sane ? h.nnz : 0;
    const int ncorr = it.len && sane ? h.ncorr : 0;
    int E = 0;   // cz planes of the box this block wrote

    if (nnz == 0) {
        // constant block (src/mc_codec.c:757-759) or absent block (zeros)
        const uint32_t w = (uint32_t)dc * 0x01010101u;
        const uint4 v = make_uint4(w, w, w, w);
        for (int i = tid; i < kStageBytes / 16; i += 128) reinterpret_cast<uint4 *>(stage)[i] = v;
    } else {
        // One pass over the entries: the extents of the coefficient box
        // (largest cz, cy, cx of any entry, src/mc_codec.c:371-372), the
        // dequantised coefficients (src/mc_codec_float.h:185-190) straight
        // into the zeroed box, and the L1 norm. Four entries per thread are
        // in flight at a time.
        const QTab &qt = P.qtab[it.qslot];
        int mz = 0, my = 0, mx = 0;
        float l1 = 0.0f;
        for (int j0 = tid; j0 < nnz; j0 += 512) {
            uint32_t e[4], ix[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) e[k] = j0 + 128 * k < nnz ? entry_at<CG>(P, base, cap, h.ovf, j0 + 128 * k) : 0u;
#pragma unroll
            for (int k = 0; k < 4; ++k) ix[k] = j0 + 128 * k < nnz ? __ldg(P.scan + (e[k] & 0xFFFu)) & 0xFFFu : 0u;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                if (j0 + 128 * k >= nnz) break;
                const int idx = (int)ix[k];
                const int cz = idx >> 8, cy = (idx >> 4) & 15, cx = idx & 15;
                mz = max(mz, cz);
                my = max(my, cy);
                mx = max(mx, cx);
                const int lv = (int16_t)(e[k] >> 16);
                if (lv) {
                    const int f = cz + cy + cx;
                    const float a = (float)(lv < 0 ? -lv : lv);
                    const float r = fadd(fadd(fmul(fsub(a, 1.0f), qt.step[f]), qt.dz8[f]), qt.dz4[f]);
                    sB[cz * kBoxPlane + cx * 16 + cy] = lv < 0 ? -r : r;
                    l1 = fadd(l1, r);
                }
            }
        }
        // one shared-memory atomic per warp and value; the L1 norm only
        // bounds the voxels, so any summation order will do
        mz = (int)__reduce_max_sync(0xFFFFFFFFu, (unsigned)mz);
        my = (int)__reduce_max_sync(0xFFFFFFFFu, (unsigned)my);
        mx = (int)__reduce_max_sync(0xFFFFFFFFu, (unsigned)mx);
        for (int o = 16; o > 0; o >>= 1) l1 += __shfl_xor_sync(0xFFFFFFFFu, l1, o);
        if ((tid & 31) == 0) {
            atomicMax(&s_rec_ext[0], mz);
            atomicMax(&s_rec_ext[1], my);
            atomicMax(&s_rec_ext[2], mx);
            atomicAdd(&s_rec_l1, l1);
        }
        __syncthreads();
        E = s_rec_ext[0] + 1;
        const int Y = s_rec_ext[1] + 1, X = s_rec_ext[2] + 1;
        const bool fast = s_rec_l1 < kFastL1;
        if ((uint32_t)tid < nlines)
            asm volatile("prefetch.global.L2 [%0];" ::"l"(P.arena + nbase + 32ull * tid));
        // pass 1: lines along x for 4 adjacent cy at once, box[cz][k][cy..cy+3]
        // -> A[cz*Y + cy][x]. Group g of plane cz holds lines cy = 4g..4g+3;
        // lines at cy >= Y are zero and not stored. gi < 64, so
        // gi * ceil(2^16 / G) >> 16 is exactly gi / G.
        const int mh = tid & 3;   // this thread's output pair (m, m+1) = (2mh, 2mh+1)
        const int G = (Y + 3) >> 2;
        const int invG = (65536 + G - 1) / G;
        for (int t = tid; t < E * G * 4; t += 128) {
            const int gi = t >> 2;
            const int cz = (gi * invG) >> 16;
            const int cy0 = (gi - cz * G) << 2;
            const Acc4 a = lines4(reinterpret_cast<const float4 *>(sB + cz * kBoxPlane + cy0), 4, X, W, mh);
            // line i of the group: outputs m, m+1 (e + o) and 15-m, 14-m (e - o)
            const float2 p0 = add2(a.e0a, a.o0a), p1 = add2(a.e0b, a.o0b);
            const float2 q0 = add2(a.e1a, a.o1a), q1 = add2(a.e1b, a.o1b);
            const float2 r0 = sub2(a.e0a, a.o0a), r1 = sub2(a.e0b, a.o0b);
            const float2 s0 = sub2(a.e1a, a.o1a), s1 = sub2(a.e1b, a.o1b);
            float *out = sA + (cz * Y + cy0) * kRowF;
            const int nl = min(Y - cy0, 4);
            *reinterpret_cast<float2 *>(out + m) = make_float2(p0.x, q0.x);
            *reinterpret_cast<float2 *>(out + 14 - m) = make_float2(s0.x, r0.x);
            if (nl > 1) {
                *reinterpret_cast<float2 *>(out + kRowF + m) = make_float2(p0.y, q0.y);
                *reinterpret_cast<float2 *>(out + kRowF + 14 - m) = make_float2(s0.y, r0.y);
            }
            if (nl > 2) {
                *reinterpret_cast<float2 *>(out + 2 * kRowF + m) = make_float2(p1.x, q1.x);
                *reinterpret_cast<float2 *>(out + 2 * kRowF + 14 - m) = make_float2(s1.x, r1.x);
            }
            if (nl > 3) {
                *reinterpret_cast<float2 *>(out + 3 * kRowF + m) = make_float2(p1.y, q1.y);
                *reinterpret_cast<float2 *>(out + 3 * kRowF + 14 - m) = make_float2(s1.y, r1.y);
            }
        }
        __syncthreads();
        // every thread has read the extents and the norm: zero for the next block
        if (tid < 3) s_rec_ext[tid] = 0;
        if (tid == 3) s_rec_l1 = 0.0f;
        // pass 2: lines along y for 4 adjacent x at once, A[cz][k][x..x+3] -> B[cz][y][x..x+3]
        for (int t = tid; t < E * 16; t += 128) {
            const int xg = (t >> 2) & 3, cz = t >> 4;
            const Acc4 a = lines4(reinterpret_cast<const float4 *>(sA + cz * Y * kRowF + xg * 4), kRowF / 4, Y,
                                  W, mh);
            // rows m, m+1 swizzle by bswz(m) = mh, rows 15-m, 14-m by 3 - mh
            float *ob = sB + cz * kPlaneB;
            const int ga = (xg ^ mh) << 2, gb = (xg ^ (3 - mh)) << 2;
            const float2 p0 = add2(a.e0a, a.o0a), p1 = add2(a.e0b, a.o0b);
            const float2 q0 = add2(a.e1a, a.o1a), q1 = add2(a.e1b, a.o1b);
            const float2 r0 = sub2(a.e0a, a.o0a), r1 = sub2(a.e0b, a.o0b);
            const float2 s0 = sub2(a.e1a, a.o1a), s1 = sub2(a.e1b, a.o1b);
            *reinterpret_cast<float4 *>(ob + m * kRowB + ga) = make_float4(p0.x, p0.y, p1.x, p1.y);
            *reinterpret_cast<float4 *>(ob + (m + 1) * kRowB + ga) = make_float4(q0.x, q0.y, q1.x, q1.y);
            *reinterpret_cast<float4 *>(ob + (15 - m) * kRowB + gb) = make_float4(r0.x, r0.y, r1.x, r1.y);
            *reinterpret_cast<float4 *>(ob + (14 - m) * kRowB + gb) = make_float4(s0.x, s0.y, s1.x, s1.y);
        }
        __syncthreads();
        // pass 3: lines along z for 4 adjacent x, B[k][y][x..x+3] -> voxels
        for (int t = tid; t < 256; t += 128) {
            const int xg = (t >> 2) & 3, y = t >> 4;
            const Acc4 a = lines4(reinterpret_cast<const float4 *>(sB + y * kRowB + ((xg ^ bswz(y)) << 2)), kPlaneB / 4,
                                  E, W, mh);
            uint32_t *row = reinterpret_cast<uint32_t *>(stage + y * 16 + xg * 4);
            constexpr int Z = kStageZ / 4;
            if (fast) {
                row[m * Z] = pack4_fast(add2(a.e0a, a.o0a), add2(a.e0b, a.o0b), dc);
                row[(m + 1) * Z] = pack4_fast(add2(a.e1a, a.o1a), add2(a.e1b, a.o1b), dc);
                row[(15 - m) * Z] = pack4_fast(sub2(a.e0a, a.o0a), sub2(a.e0b, a.o0b), dc);
                row[(14 - m) * Z] = pack4_fast(sub2(a.e1a, a.o1a), sub2(a.e1b, a.o1b), dc);
            } else {
                row[m * Z] = pack4(add2(a.e0a, a.o0a), add2(a.e0b, a.o0b), dc);
                row[(m + 1) * Z] = pack4(add2(a.e1a, a.o1a), add2(a.e1b, a.o1b), dc);
                row[(15 - m) * Z] = pack4(sub2(a.e0a, a.o0a), sub2(a.e0b, a.o0b), dc);
                row[(14 - m) * Z] = pack4(sub2(a.e1a, a.o1a), sub2(a.e1b, a.o1b), dc);
            }
        }
    }
    __syncthreads();
    // the box planes this block wrote (coefficients and pass-2 output) back to zero
    for (int i = tid; i < E * (kBoxPlane / 4); i += 128)
        reinterpret_cast<float4 *>(sB)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (ncorr && tid == 0) {
        // corrections in stream order: a position may repeat, each
        // application clamps (src/mc_codec.c:775-781)
        for (int c = 0; c < ncorr; ++c) {
            const uint32_t pos = entry_at<CG>(P, base, cap, h.ovf, nnz + 2 * c);
            const uint32_t d = entry_at<CG>(P, base, cap, h.ovf, nnz + 2 * c + 1);
            if (pos >= (uint32_t)kN3) break;
            uint8_t &vox = stage[(pos >> 8) * kStageZ + (pos & 255)];
            const int v = (int)((uint32_t)vox + d);
            vox = (uint8_t)(v < 0 ? 0 : v > 255 ? 255 : v);
        }
    }
    __syncthreads();
}

// Clipped store of one staged block: one 16-voxel row per thread step.
__device__ __forceinline__ void store_block(const DecItem &it, const uint8_t *stage) {
    const int z0 = it.clip_lo >> 8, y0 = (it.clip_lo >> 4) & 15, x0 = it.clip_lo & 15;
    const int z1 = it.clip_hi >> 8, y1 = (it.clip_hi >> 4) & 15, x1 = it.clip_hi & 15;
    const int ny = y1 - y0 + 1, nrows = (z1 - z0 + 1) * ny;
    uint8_t *dst = reinterpret_cast<uint8_t *>(it.dst);
    for (int r = threadIdx.x; r < nrows; r += blockDim.x) {
        const int z = z0 + r / ny, y = y0 + r % ny;
        uint8_t *row = dst + z * it.sz + y * it.sy;
        const uint8_t *srow = stage + z * kStageZ + y * 16;
        if (x0 == 0 && x1 == 15) {
            store_row16(row, *reinterpret_cast<const uint4 *>(srow));
        } else {
            for (int x = x0; x <= x1; ++x) row[x] = srow[x];
        }
    }
}

// Two blocks that sit side by side in x in the same output: one 32-byte
// row per step, so every DRAM sector is written whole (16-byte halves of a
// sector written apart cost a read-modify-write).
__device__ __forceinline__ bool pairable(const DecItem &a, const DecItem &b) {
    return a.clip_lo == kClipFullLo && a.clip_hi == kClipFullHi && b.clip_lo == kClipFullLo &&
           b.clip_hi == kClipFullHi && b.dst == a.dst + 16 && a.sz == b.sz && a.sy == b.sy && (a.dst & 31) == 0 &&
           (a.sy & 31) == 0 && (a.sz & 31) == 0;
}

__global__ void __launch_bounds__(128, 5) k_reconstruct(RecParams P) {
    // sA: pass-1 output, then the second block's stage; sB: coefficient box,
    // then pass-2 output; sStage0: the first block's stage
    __shared__ __align__(16) float sA[16 * 16 * kRowF];
    __shared__ __align__(16) float sB[kBoxB];
    __shared__ __align__(16) uint8_t sStage0[kStageBytes];
    __shared__ __align__(16) float4 sW[16 * 8];   // [k][m/2] = {c[k][m], c[k][m], c[k][m+1], c[k][m+1]}
    uint8_t *const sStage1 = reinterpret_cast<uint8_t *>(sA);
    for (int i = threadIdx.x; i < 16 * 8; i += blockDim.x) {
        const int k = i >> 3, mm = (i & 7) * 2;
        sW[i] = make_float4(c_cos[k][mm], c_cos[k][mm], c_cos[k][mm + 1], c_cos[k][mm + 1]);
    }
    rec_init(sB);
    __syncthreads();
    const int tid = threadIdx.x;
    const int npairs = (P.n + 1) / 2;
    for (int pr = blockIdx.x; pr < npairs; pr += gridDim.x) {
        const int j0 = 2 * pr, j1 = 2 * pr + 1;
        const int i0 = P.idx ? (int)P.idx[j0] : j0;
        const int i1 = j1 < P.n ? (P.idx ? (int)P.idx[j1] : j1) : -1;
        const int jn = 2 * (pr + gridDim.x);   // this CTA's next pair
        const int in = jn < P.n ? (P.idx ? (int)P.idx[jn] : jn) : -1;
        reconstruct_block<false>(P, i0, sA, sB, sStage0, sW, i1 >= 0 ? i1 : in);
        const DecItem a = P.items[i0];
        if (i1 >= 0) {
            reconstruct_block<false>(P, i1, sA, sB, sStage1, sW, in);
            const DecItem b = P.items[i1];
            if (pairable(a, b)) {
                uint8_t *dst = reinterpret_cast<uint8_t *>(a.dst);
                for (int r = tid; r < 256; r += 128) {
                    const int z = r >> 4, y = r & 15;
                    uint4 *row = reinterpret_cast<uint4 *>(dst + z * a.sz + y * a.sy);
                    row[0] = *reinterpret_cast<const uint4 *>(sStage0 + z * kStageZ + y * 16);
                    row[1] = *reinterpret_cast<const uint4 *>(sStage1 + z * kStageZ + y * 16);
                }
            } else {
                store_block(a, sStage0);
                store_block(b, sStage1);
            }
        } else {
            store_block(a, sStage0);
        }
        __syncthreads();
    }
}


// ---------------------------------------------------------------- fused decode
// One persistent kernel for both stages. Every CTA first runs entropy lanes
// (the k_entropy loop) until the shared block queue is drained. Blocks are
// reconstructed in the pairs k_reconstruct uses (items 2j, 2j+1, x-neighbours
// inside a chunk): the block that completes a pair -- an absent block at
// kernel start, a coded one when its lane finishes -- appends the pair to a
// completion list. A CTA whose lanes are all idle reconstructs pairs in list
// order, while CTAs that still hold long blocks finish their entropy decode:
// the tail of the entropy stage overlaps the reconstruction of everything
// else, and the entries of a finished block are read back while still in L2.
// A CTA that claims a list position not yet written polls with a bounded
// backoff; if the bound runs out it records the position and leaves, and
// k_fused_tail (launched after, stream-ordered) reconstructs whatever was
// recorded or never claimed. No wait is unbounded.
struct FusedSmem {
    union {
        struct {
            uint16_t bend[9];
            uint32_t ctx[4][kCtxSlots][32];
        } e;
        struct {
            float A[16 * 16 * kRowF];
            float B[kBoxB];
            uint8_t stage0[kStageBytes];
        } r;
    } u;
    float4 W[16 * 8];
    int pair;
};

// Item `item` is ready for reconstruction; the last of its pair appends the pair.
__device__ __forceinline__ void pair_ready(const FusedParams &F, int item) {
    const uint32_t j = (uint32_t)item >> 1;
    const uint32_t size = 2u * j + 1u < (uint32_t)F.r.n ? 2u : 1u;
    __threadfence();   // this block's header and entries before the pair's count
    if (atomicAdd(F.pair_cnt + j, 1u) + 1u == size) {
        const uint32_t pos = atomicAdd(F.ws + kFusedDone, 1u);
        __threadfence();   // the other block's results, seen through the count, before the list entry
        atomicExch(F.rlist + pos, j + 1u);
    }
}

// Pair at completion-list position p, or -1 if not written yet.
__device__ __forceinline__ int list_pair(const FusedParams &F, uint32_t p) {
    const uint32_t v = *reinterpret_cast<const volatile uint32_t *>(F.rlist + p);
    return (int)v - 1;
}

template <bool CG>
__device__ __forceinline__ void reconstruct_pair(const RecParams &P, int j, float *sA, float *sB, uint8_t *stage0,
                                                 const float4 *W) {
    const int tid = threadIdx.x;
    uint8_t *const stage1 = reinterpret_cast<uint8_t *>(sA);   // sA is free once a block is staged
    const int i0 = 2 * j, i1 = 2 * j + 1;
    reconstruct_block<CG>(P, i0, sA, sB, stage0, W);
    const DecItem a = P.items[i0];
    if (i1 < P.n) {
        reconstruct_block<CG>(P, i1, sA, sB, stage1, W);
        const DecItem b = P.items[i1];
        if (pairable(a, b)) {
            uint8_t *dst = reinterpret_cast<uint8_t *>(a.dst);
            for (int r = tid; r < 256; r += 128) {
                const int z = r >> 4, y = r & 15;
                uint4 *row = reinterpret_cast<uint4 *>(dst + z * a.sz + y * a.sy);
                row[0] = *reinterpret_cast<const uint4 *>(stage0 + z * kStageZ + y * 16);
                row[1] = *reinterpret_cast<const uint4 *>(stage1 + z * kStageZ + y * 16);
            }
        } else {
            store_block(a, stage0);
            store_block(b, stage1);
        }
    } else {
        store_block(a, stage0);
    }
}

__global__ void __launch_bounds__(128, 4) k_decode_fused(FusedParams F) {
    extern __shared__ __align__(16) uint8_t s_raw[];
    FusedSmem &S = *reinterpret_cast<FusedSmem *>(s_raw);
    const EntParams &P = F.e;
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int nlanes = gridDim.x * blockDim.x;
    // absent blocks are ready at once
    for (int q = P.ncoded + gtid; q < P.n; q += nlanes) pair_ready(F, (int)P.order[q]);
    if (threadIdx.x < 9) S.u.e.bend[threadIdx.x] = c_bend[threadIdx.x];
    for (int i = threadIdx.x; i < 16 * 8; i += blockDim.x) {
        const int k = i >> 3, mm = (i & 7) * 2;
        S.W[i] = make_float4(c_cos[k][mm], c_cos[k][mm], c_cos[k][mm + 1], c_cos[k][mm + 1]);
    }
    __syncthreads();

    // ---- entropy: the k_entropy loop, each finished block marked ready;
    // warps 0..nsolo-1 of the grid first decode order entry `warp` on their
    // first thread alone, as in k_entropy
    {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        uint32_t *ctx = &S.u.e.ctx[warp][0][lane];
        LaneState L;
        const int gwarp = (int)(blockIdx.x * blockDim.x + threadIdx.x) >> 5;
        if (gwarp < P.nsolo) {
            if (lane == 0) {
                memset(&L, 0, sizeof L);
                lane_begin(L, P, ctx, S.u.e.bend, (int)P.order[gwarp]);
                solo_entropy(L, P, ctx, S.u.e.bend);
                lane_finish(L, P);
                pair_ready(F, L.item);
            }
            __syncwarp();
        }
        EntParams E = P;   // the rest of the order, one lane per block
        E.order = P.order + P.nsolo;
        E.ncoded = P.ncoded - P.nsolo;
        run_lanes(L, E, ctx, S.u.e.bend, gtid - 32 * P.nsolo, nlanes - 32 * P.nsolo,
                  [&F](int item) { pair_ready(F, item); });
    }
    __syncthreads();   // the shared memory changes hands
    rec_init(S.u.r.B);
    __syncthreads();

    // ---- reconstruction over the completion list, one pair per claim
    const uint32_t npairs = ((uint32_t)F.r.n + 1u) >> 1;
    for (;;) {
        if (threadIdx.x == 0) {
            int j = -1;
            const uint32_t p = atomicAdd(F.ws + kFusedClaim, 1u);
            if (p < npairs) {
                j = list_pair(F, p);
                uint32_t ns = 32;
                for (uint32_t tries = 0; j < 0 && tries < F.spin_limit; ++tries) {
                    __nanosleep(ns);
                    if (ns < 1024) ns <<= 1;
                    j = list_pair(F, p);
                }
                if (j < 0) F.ws[kFusedSkip0 + atomicAdd(F.ws + kFusedNSkip, 1u)] = p;   // k_fused_tail takes it
                __threadfence();   // the pair's results after its list entry
            }
            S.pair = j;
        }
        __syncthreads();
        const int j = S.pair;
        if (j < 0) break;
        reconstruct_pair<true>(F.r, j, S.u.r.A, S.u.r.B, S.u.r.stage0, S.W);
        __syncthreads();
    }
}

// List positions that k_decode_fused recorded as given up or never claimed
// (normally none): one pair per CTA step. Runs after it, stream-ordered, so
// every pair is in the list.
__global__ void __launch_bounds__(128) k_fused_tail(FusedParams F) {
    __shared__ __align__(16) float sA[16 * 16 * kRowF];
    __shared__ __align__(16) float sB[kBoxB];
    __shared__ __align__(16) uint8_t sStage0[kStageBytes];
    __shared__ __align__(16) float4 sW[16 * 8];
    const uint32_t npairs = ((uint32_t)F.r.n + 1u) >> 1;
    const uint32_t claimed = min(F.ws[kFusedClaim], npairs);
    const uint32_t nsk = min(F.ws[kFusedNSkip], (uint32_t)kFusedMaxSkip);
    const uint32_t work = nsk + (npairs - claimed);
    if (blockIdx.x >= work) return;
    for (int i = threadIdx.x; i < 16 * 8; i += blockDim.x) {
        const int k = i >> 3, mm = (i & 7) * 2;
        sW[i] = make_float4(c_cos[k][mm], c_cos[k][mm], c_cos[k][mm + 1], c_cos[k][mm + 1]);
    }
    rec_init(sB);
    __syncthreads();
    for (uint32_t w = blockIdx.x; w < work; w += gridDim.x) {
        const uint32_t p = w < nsk ? F.ws[kFusedSkip0 + w] : claimed + (w - nsk);
        const int j = p < npairs ? list_pair(F, p) : -1;
        if (j < 0 || (uint32_t)j >= npairs) continue;   // every pair is listed by now
        reconstruct_pair<false>(F.r, j, sA, sB, sStage0, sW);
        __syncthreads();
    }
}

// ---------------------------------------------------------------- one block
// The single-block calls (mc_archive_decode_block, mc_dec_block): one CTA
// decodes one block end to end in one launch, with the work item as a kernel
// argument -- no batch layout, no host-to-device copies, no second launch.
// Thread 0 runs the entropy decode through the k_entropy step functions
// (fast_step, slow_work for the rare states), the CTA then reconstructs
// the block. A branchy scalar loop over the same states was measured slower
// per bin (p99 block latency 1.23 ms against 0.93): each bin's shared-memory
// context load and branch resolution then sit on the serial chain, which the
// warp step avoids by fetching both candidate contexts ahead, without
// branches.

static_assert(sizeof(DecItem) % 16 == 0, "SoloScratch::hdr must sit on a 16-byte boundary");

__global__ void __launch_bounds__(128) k_decode_one(DecItem it, SoloScratch *S, const QTab *qtab,
                                                    const uint16_t *scan, uint32_t *status) {
    // sA holds thread 0's entropy contexts (one column of 32-word rows, the
    // layout k_entropy uses) until the entropy decode is done, then the
    // pass-1 output
    __shared__ __align__(16) float sA[16 * 16 * kRowF];
    __shared__ __align__(16) float sB[kBoxB];
    __shared__ __align__(16) uint8_t sStage[kStageBytes];
    __shared__ __align__(16) float4 sW[16 * 8];
    __shared__ uint16_t s_bend[9];
    static_assert(sizeof(sA) >= sizeof(uint32_t) * kCtxSlots * 32, "contexts fit in sA");
    const int tid = threadIdx.x;
    if (tid < 9) s_bend[tid] = c_bend[tid];
    for (int i = tid; i < 16 * 8; i += blockDim.x) {
        const int k = i >> 3, mm = (i & 7) * 2;
        sW[i] = make_float4(c_cos[k][mm], c_cos[k][mm], c_cos[k][mm + 1], c_cos[k][mm + 1]);
    }
    rec_init(sB);
    const uint32_t cap = entry_cap(it.len);
    if (tid == 0) {
        S->item = it;
        S->base = 0;
        S->pool_used = 0;
        status[0] = 0;
    }
    __syncthreads();
    if (tid == 0) {
        EntParams P;
        P.items = &S->item;
        P.order = nullptr;
        P.n = 1;
        P.ncoded = 1;
        P.base = &S->base;
        P.arena = S->entries;
        P.hdr = &S->hdr;
        P.pool = S->entries + cap;       // the overflow continues the list
        P.pool_cap = kEntryMax - cap;    // what one block may ask of the pool
        P.pool_used = &S->pool_used;
        P.qtab = qtab;
        P.scan = scan;
        P.status = status;
        P.counter = nullptr;
        P.claim = 1;
        uint32_t *ctx = reinterpret_cast<uint32_t *>(sA);
        LaneState L;
        memset(&L, 0, sizeof L);
        lane_begin(L, P, ctx, s_bend, 0);
        solo_entropy(L, P, ctx, s_bend);
        lane_finish(L, P);
    }
    __syncthreads();   // thread 0's header and entries are visible to the CTA
    RecParams R;
    R.items = &S->item;
    R.idx = nullptr;
    R.n = 1;
    R.hdr = &S->hdr;
    R.base = &S->base;
    R.arena = S->entries;
    R.pool = S->entries + cap;
    R.qtab = qtab;
    R.scan = scan;
    reconstruct_block<true>(R, 0, sA, sB, sStage, sW);   // written in this kernel: read through L2
    store_block(it, sStage);
}

// ---------------------------------------------------------------- launchers
cudaError_t preload_decode_kernels() {
    // under lazy module loading a kernel's code is loaded at its first launch,
    // which would put a few milliseconds into the first call that uses it
    cudaFuncAttributes fa;
    const void *fns[] = {(const void *)k_entropy<2>, (const void *)k_entropy<4>, (const void *)k_entropy<8>,
                         (const void *)k_entropy_solo, (const void *)k_reconstruct, (const void *)k_decode_fused,
                         (const void *)k_fused_tail, (const void *)k_decode_one};
    for (const void *f : fns) {
        const cudaError_t e = cudaFuncGetAttributes(&fa, f);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t upload_decode_tables(const float cmf[16][16], const uint16_t scan[kN3], cudaStream_t s) {
    // pageable sources: the copies are staged before these calls return
    static uint16_t bend[9];
    for (int i = 1; i < kN3; ++i) {
        const uint32_t b = scan[i] >> 12;
        if ((uint32_t)(scan[i - 1] >> 12) != b) bend[b - 1] = (uint16_t)i;
    }
    bend[7] = kN3;
    bend[8] = 0xFFFF;
    const cudaError_t e = cudaMemcpyToSymbolAsync(c_cos, cmf, sizeof(float) * 256, 0, cudaMemcpyHostToDevice, s);
    return e != cudaSuccess ? e : cudaMemcpyToSymbolAsync(c_bend, bend, sizeof bend, 0, cudaMemcpyHostToDevice, s);
}

static int num_sms() { return dev_sms(); }

template <int W>
static cudaError_t launch_entropy_w(const EntParams &p, int ctas_per_sm, cudaStream_t s) {
    // per device: the dynamic shared memory opt-in of this instantiation
    static std::atomic<int> attr[kMaxDevs];
    const int a = dev_once(attr, [] {
        const cudaError_t e = cudaFuncSetAttribute(k_entropy<W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)entropy_smem(W));
        return e == cudaSuccess ? 1 : -(int)e;
    });
    if (a < 0) return (cudaError_t)(-a);
    // one warp per solo block, one lane per other block
    EntParams q = p;
    if (!q.order || q.nsolo < 0) q.nsolo = 0;
    if (q.nsolo > q.ncoded) q.nsolo = q.ncoded;
    int blocks = (q.nsolo + (q.ncoded - q.nsolo + 31) / 32 + W - 1) / W;
    const int cap = num_sms() * ctas_per_sm;
    if (blocks > cap) blocks = cap;
    if (q.nsolo > blocks * W / 2) q.nsolo = blocks * W / 2;   // at most half of the warps
    k_entropy<W><<<blocks, W * 32, entropy_smem(W), s>>>(q);
    return cudaGetLastError();
}

// The single-thread share when a launch configuration leaves it open, from
// the launch's coded blocks (q=6 batches on a B200): up to about 10 chunks'
// worth every block on a single thread (its time is the longest block's
// chain, a few times shorter there), up to about 30 chunks' worth the longest
// 1/64, beyond that none (a lane of 32 issues fewer instructions per bin).
constexpr int kSoloAllMax = 28 * 1024, kSoloShareMax = 90 * 1024;
static int auto_solo(int ncoded) { return ncoded <= kSoloAllMax ? 1 : (ncoded <= kSoloShareMax ? 64 : 0); }

cudaError_t launch_entropy(const EntParams &p, const LaunchCfg &cfg, cudaStream_t s) {
    if (p.ncoded <= 0) return cudaSuccess;
    const int solo = cfg.ent_solo >= 0 ? cfg.ent_solo : auto_solo(p.ncoded);
    if (solo == 1) {   // every block on a single thread
        int blocks = (p.ncoded + kSoloWarps - 1) / kSoloWarps;
        if (blocks > 2 * num_sms()) blocks = 2 * num_sms();
        k_entropy_solo<<<blocks, kSoloWarps * 32, 0, s>>>(p);
        return cudaGetLastError();
    }
    EntParams q = p;
    q.claim = cfg.ent_claim > 0 ? cfg.ent_claim : 1;
    q.nsolo = solo > 0 ? p.ncoded / solo : 0;
    const int per_sm = cfg.ent_ctas_per_sm > 0 ? cfg.ent_ctas_per_sm : 5;
    switch (cfg.ent_warps) {
    case 2: return launch_entropy_w<2>(q, per_sm, s);
    case 8: return launch_entropy_w<8>(q, per_sm, s);
    default: return launch_entropy_w<4>(q, per_sm, s);
    }
}

int fused_grid(const LaunchCfg &cfg) {
    static std::atomic<int> occ_by_dev[kMaxDevs];
    const int occ = dev_once(occ_by_dev, [] {
        // dynamic shared memory above 48 KiB: opt in once per device
        int o = 0;
        if (cudaFuncSetAttribute(k_decode_fused, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sizeof(FusedSmem)) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k_decode_fused, 128, sizeof(FusedSmem)) !=
                cudaSuccess || o < 1)
            o = -1;
        return o;
    });
    if (occ < 0) return 0;
    // every CTA resident at once: a CTA's waits are then on CTAs that run
    const int per_sm = std::min(cfg.fused_ctas_per_sm > 0 ? cfg.fused_ctas_per_sm : 4, occ);
    return std::min(num_sms() * per_sm, kFusedMaxSkip);
}

cudaError_t launch_fused(const FusedParams &f, const LaunchCfg &cfg, cudaStream_t s) {
    const int blocks = fused_grid(cfg);
    if (blocks <= 0) return cudaErrorInvalidConfiguration;
    // the single-thread share (all blocks is not a fused layout: at most half
    // of the warps, as in k_entropy)
    FusedParams g = f;
    const int solo = cfg.ent_solo >= 0 ? cfg.ent_solo : auto_solo(f.e.ncoded);
    g.e.nsolo = solo > 0 ? std::min(f.e.ncoded / solo, blocks * 4 / 2) : 0;
    k_decode_fused<<<blocks, 128, sizeof(FusedSmem), s>>>(g);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_fused_tail<<<num_sms(), 128, 0, s>>>(f);
    return cudaGetLastError();
}

cudaError_t launch_reconstruct(const RecParams &p, const LaunchCfg &cfg, cudaStream_t s) {
    if (p.n <= 0) return cudaSuccess;
    int blocks = (p.n + 1) / 2;   // one CTA step per pair of blocks
    int cap = num_sms() * (cfg.rec_ctas_per_sm > 0 ? cfg.rec_ctas_per_sm : 5);
    if (blocks > cap) blocks = cap;
    // per device: the largest shared-memory carveout, so that 5 CTAs per SM fit
    static std::atomic<int> carve_set[kMaxDevs];
    dev_once(carve_set, [] {
        cudaFuncSetAttribute(k_reconstruct, cudaFuncAttributePreferredSharedMemoryCarveout,
                             (int)cudaSharedmemCarveoutMaxShared);
        return 1;
    });
    k_reconstruct<<<blocks, 128, 0, s>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_decode_one(const DecItem &it, SoloScratch *scratch, const QTab *qtab, const uint16_t *scan,
                              uint32_t *status, cudaStream_t s) {
    k_decode_one<<<1, 128, 0, s>>>(it, scratch, qtab, scan, status);
    return cudaGetLastError();
}

}  // namespace mcb
