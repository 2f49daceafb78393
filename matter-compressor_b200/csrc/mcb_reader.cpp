// mcb_reader.cpp -- read-only archive readers (src/mc_stream.c): over bytes in
// memory (mc_open) or over a byte-range callback (mc_open_streaming), with the
// partial-fetch mode that reads only a chunk's bitmap and length table plus
// the payloads of the blocks asked for. Every block is decoded on the GPU.
//
// The single-block drop-in (mc_decode_block) decodes through mc_dec_block.
// The batched form (mc_b200_reader_decode_blocks) gathers the payloads of many
// blocks of one chunk -- in partial mode with one range read per run of
// adjacent payloads -- into one staging buffer, copies it to the device once
// and decodes all blocks in one batch into device memory.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "mcb_archive.h"
#include "mcb_host_codec.h"
#include "mcb_tables.h"

using namespace mcb;

namespace {

// header fields (src/mc_archive.h:73-94)
constexpr uint32_t kMagic = 0x0043434Du;
constexpr uint64_t HMAGIC = 0, HNX = 12, HNY = 16, HNZ = 20, HROOT = 24, HQUALITY = 120, HPRIOR = 128;
constexpr uint64_t kHdr = 256;
constexpr uint64_t kNodeBytes = (uint64_t)kGrid3 * 8;
constexpr uint32_t kPriorsMagic = 0x53524950u;
constexpr uint64_t kPriorsBytes = 8 + 2 * 8 * 32 * 2;
constexpr int kNodeCache = 512;   // node tables cached per streaming reader (src/mc_stream.c:28)

inline uint64_t rd64(const uint8_t *p) { uint64_t v; memcpy(&v, p, 8); return v; }
inline int nib(int c, int level) { return (c >> (4 * level)) & 15; }

// Total length of the blob at co if its structure lies inside [0, end), else 0
// (src/mc_archive.h:212-226).
uint64_t blob_struct_len(const uint8_t *arc, uint64_t co, uint64_t end) {
    if (co > end || end - co < (uint64_t)kBlobHdr) return 0;
    uint16_t fml;
    memcpy(&fml, arc + co + 12, 2);
    const uint64_t bm_off = co + kBlobHdr + fml;
    if (bm_off > end || end - bm_off < (uint64_t)kBitmapBytes) return 0;
    uint32_t np = 0;
    for (int i = 0; i < kBitmapBytes; ++i) np += (uint32_t)__builtin_popcount(arc[bm_off + i]);
    const uint64_t lens_off = bm_off + kBitmapBytes;
    if (end - lens_off < 2ull * np) return 0;
    uint64_t pay = 0;
    for (uint32_t s = 0; s < np; ++s) {
        uint16_t l;
        memcpy(&l, arc + lens_off + 2 * s, 2);
        pay += l;
    }
    const uint64_t total = lens_off + 2ull * np + pay - co;
    return co + total > end ? 0 : total;
}

// Quality of a chunk from its (untrusted) blob header: NaN, infinite or out of
// range reads as 1 (src/mc_stream.c:283-285, 312-315).
float clamp_q(float q) { return (!(q > 0.0f) || q > 1024.0f) ? 1.0f : q; }

}  // namespace

struct mc_reader {
    const uint8_t *arc = nullptr;   // flat: the archive bytes
    size_t len = 0;
    mc_read_fn read = nullptr;      // streaming: the byte source
    void *ud = nullptr;
    int nx = 0, ny = 0, nz = 0;
    float quality = 0.0f;
    uint64_t roots[8] = {0};
    bool has_priors = false;
    uint8_t priors[kPriorsBytes];
    mc_codec_ctx *codec = nullptr;
    bool partial = false;
    // streaming node tables (FIFO)
    std::vector<std::vector<uint8_t>> ntab;
    std::vector<uint64_t> ntab_off;
    int ntab_next = 0;
    // full-fetch: the last chunk blob
    std::vector<uint8_t> cbuf;
    uint64_t cbuf_off = ~0ull;
    // partial-fetch: the last chunk's header, bitmap and lengths, with
    // every present block's payload offset
    uint64_t hdr_off = ~0ull;
    float hdr_q = 0.0f;
    uint8_t bm[kBitmapBytes];
    std::vector<uint64_t> pay_off;   // per block (absolute), kGrid3 entries
    std::vector<uint16_t> pay_len;
    std::vector<uint8_t> pbuf;
};

namespace {

void load_header(mc_reader *r, const uint8_t *hdr) {
    uint32_t v;
    memcpy(&v, hdr + HNX, 4); r->nx = (int)v;
    memcpy(&v, hdr + HNY, 4); r->ny = (int)v;
    memcpy(&v, hdr + HNZ, 4); r->nz = (int)v;
    memcpy(&r->quality, hdr + HQUALITY, 4);
    for (int l = 0; l < 8; ++l) r->roots[l] = rd64(hdr + HROOT + 8 * l);
}

int sread(mc_reader *r, uint64_t off, uint32_t len, uint8_t *dst) { return r->read(r->ud, off, len, dst); }

const uint8_t *node_table(mc_reader *r, uint64_t off) {
    for (size_t i = 0; i < r->ntab_off.size(); ++i)
        if (r->ntab_off[i] == off && !r->ntab[i].empty()) return r->ntab[i].data();
    if (r->ntab.size() < (size_t)kNodeCache) {
        r->ntab.emplace_back();
        r->ntab_off.push_back(~0ull);
        r->ntab_next = (int)r->ntab.size() - 1;
    }
    const int slot = r->ntab_next;
    r->ntab_next = (slot + 1) % kNodeCache;
    std::vector<uint8_t> &t = r->ntab[slot];
    t.resize(kNodeBytes);
    if (sread(r, off, (uint32_t)kNodeBytes, t.data()) != 0) {
        t.clear();
        r->ntab_off[slot] = ~0ull;
        return nullptr;
    }
    r->ntab_off[slot] = off;
    return t.data();
}

// src/mc_archive.h:133-145 (flat, bounded) and src/mc_stream.c:379-392 (streaming)
uint64_t resolve(mc_reader *r, int lod, int cz, int cy, int cx, int *err) {
    uint64_t node = r->roots[lod];
    for (int level = 2; level >= 0; --level) {
        if (!node) return 0;
        const int idx = (nib(cz, level) * 16 + nib(cy, level)) * 16 + nib(cx, level);
        if (r->arc) {
            if (node > r->len || (uint64_t)idx * 8 + 8 > r->len - node) return 0;
            node = rd64(r->arc + node + (uint64_t)idx * 8);
        } else {
            const uint8_t *t = node_table(r, node);
            if (!t) { if (err) *err = 1; return 0; }
            node = rd64(t + (uint64_t)idx * 8);
        }
    }
    return node;
}

// Streaming: the whole blob at co in r->cbuf (src/mc_stream.c:234-256).
const uint8_t *fetch_blob(mc_reader *r, uint64_t co) {
    if (r->cbuf_off == co && !r->cbuf.empty()) return r->cbuf.data();
    uint8_t bh[kBlobHdr];
    if (sread(r, co, kBlobHdr, bh) != 0) return nullptr;
    uint16_t fml;
    memcpy(&fml, bh + 12, 2);
    const uint64_t bm_off = co + kBlobHdr + fml;
    uint8_t bm[kBitmapBytes];
    if (sread(r, bm_off, kBitmapBytes, bm) != 0) return nullptr;
    uint32_t np = 0;
    for (int i = 0; i < kBitmapBytes; ++i) np += (uint32_t)__builtin_popcount(bm[i]);
    std::vector<uint8_t> lens(2ull * np);
    if (np && sread(r, bm_off + kBitmapBytes, 2 * np, lens.data()) != 0) return nullptr;
    uint64_t pay = 0;
    for (uint32_t s = 0; s < np; ++s) pay += (uint16_t)(lens[2 * s] | (lens[2 * s + 1] << 8));
    const uint64_t total = bm_off + kBitmapBytes + 2ull * np + pay - co;
    r->cbuf.resize(total);
    r->cbuf_off = ~0ull;
    if (sread(r, co, (uint32_t)total, r->cbuf.data()) != 0) return nullptr;
    r->cbuf_off = co;
    return r->cbuf.data();
}

// Partial fetch: header, bitmap and lengths of the chunk at co, cached, with
// every present block's payload offset (src/mc_stream.c:257-272).
bool fetch_index(mc_reader *r, uint64_t co) {
    if (r->hdr_off == co) return true;
    uint8_t bh[kBlobHdr];
    if (sread(r, co, kBlobHdr, bh) != 0) return false;
    uint16_t fml;
    memcpy(&fml, bh + 12, 2);
    if (sread(r, co + kBlobHdr + fml, kBitmapBytes, r->bm) != 0) return false;
    uint32_t np = 0;
    for (int i = 0; i < kBitmapBytes; ++i) np += (uint32_t)__builtin_popcount(r->bm[i]);
    std::vector<uint8_t> lens(2ull * np);
    if (np && sread(r, co + kBlobHdr + fml + kBitmapBytes, 2 * np, lens.data()) != 0) return false;
    float q;
    memcpy(&q, bh, 4);
    r->hdr_q = clamp_q(q);
    r->pay_off.assign(kGrid3, 0);
    r->pay_len.assign(kGrid3, 0);
    uint64_t pay = co + kBlobHdr + fml + kBitmapBytes + 2ull * np;
    uint32_t slot = 0;
    for (int bi = 0; bi < kGrid3; ++bi) {
        if (!((r->bm[bi >> 3] >> (bi & 7)) & 1)) continue;
        const uint16_t l = (uint16_t)(lens[2 * slot] | (lens[2 * slot + 1] << 8));
        r->pay_off[bi] = pay;
        r->pay_len[bi] = l;
        pay += l;
        ++slot;
    }
    r->hdr_off = co;
    return true;
}

// Where the payload of block bi of the chunk at co is: a pointer into host
// bytes (flat or a fetched blob), or (partial) an absolute range to read.
// Returns false when the chunk cannot be read; *present = false for an
// absent block.
struct BlockSrc {
    const uint8_t *ptr;   // host bytes, or null in partial mode
    uint64_t off;         // partial mode: absolute payload offset
    uint32_t len;
    bool present;
};
bool chunk_blocks(mc_reader *r, uint64_t co, float *q, const uint8_t **base) {
    *base = nullptr;
    if (r->arc) {
        if (!blob_struct_len(r->arc, co, r->len)) return false;
        *base = r->arc;
    } else if (r->partial) {
        if (!fetch_index(r, co)) return false;
        *q = r->hdr_q;
        return true;
    } else {
        const uint8_t *b = fetch_blob(r, co);
        if (!b) return false;
        *base = b - co;   // absolute offsets index into the fetched window
    }
    float cq;
    memcpy(&cq, *base + co, 4);
    *q = clamp_q(cq);
    return true;
}
BlockSrc block_src(mc_reader *r, uint64_t co, const uint8_t *base, int bi) {
    if (!base) {
        return BlockSrc{nullptr, r->pay_off[bi], r->pay_len[bi], r->pay_off[bi] != 0};
    }
    // flat / fetched blob: walk the bitmap to the block's payload (src/mc_archive.h:175-206)
    const ChunkIndex &ix = chunk_index(base, co);
    return BlockSrc{ix.off[bi] ? base + ix.off[bi] : nullptr, ix.off[bi], ix.len[bi], ix.off[bi] != 0};
}

}  // namespace

extern "C" {

mc_reader *mc_open(const uint8_t *arc, size_t len) {
    if (!arc || len < kHdr) return nullptr;
    uint32_t magic;
    memcpy(&magic, arc + HMAGIC, 4);
    if (magic != kMagic) return nullptr;
    mc_reader *r = new mc_reader();
    r->arc = arc;
    r->len = len;
    r->codec = mc_codec_ctx_new();
    load_header(r, arc);
    const uint64_t poff = rd64(arc + HPRIOR);
    if (poff && poff <= len && len - poff >= kPriorsBytes) {
        uint32_t pm;
        memcpy(&pm, arc + poff, 4);
        if (pm == kPriorsMagic) {
            memcpy(r->priors, arc + poff, kPriorsBytes);
            r->has_priors = true;
            mc_codec_set_priors(reinterpret_cast<const uint16_t *>(arc + poff + 8),
                                reinterpret_cast<const uint16_t *>(arc + poff + 8 + 8 * 32 * 2));
        }
    }
    return r;
}

mc_reader *mc_open_streaming(mc_read_fn read, void *ud, uint64_t total_len) {
    if (!read) return nullptr;
    uint8_t hdr[kHdr];
    if (read(ud, 0, (uint32_t)kHdr, hdr) != 0) return nullptr;
    uint32_t magic;
    memcpy(&magic, hdr + HMAGIC, 4);
    if (magic != kMagic) return nullptr;
    mc_reader *r = new mc_reader();
    r->read = read;
    r->ud = ud;
    r->len = (size_t)total_len;
    r->codec = mc_codec_ctx_new();
    load_header(r, hdr);
    // the archive's priors through the callback, else the baked ones (src/mc_stream.c:104-119)
    const uint64_t poff = rd64(hdr + HPRIOR);
    uint8_t pb[kPriorsBytes];
    uint32_t pm = 0;
    if (poff && read(ud, poff, (uint32_t)kPriorsBytes, pb) == 0) memcpy(&pm, pb, 4);
    if (pm == kPriorsMagic) {
        memcpy(r->priors, pb, kPriorsBytes);
        r->has_priors = true;
        mc_codec_set_priors(reinterpret_cast<const uint16_t *>(pb + 8),
                            reinterpret_cast<const uint16_t *>(pb + 8 + 8 * 32 * 2));
    } else {
        mc_codec_set_priors(nullptr, nullptr);
    }
    return r;
}

void mc_close(mc_reader *r) {
    if (!r) return;
    if (r->codec) mc_codec_ctx_free(r->codec);
    delete r;
}

void mc_reader_set_quality(mc_reader *r, float q) {
    if (r && r->codec) mc_codec_ctx_set_quality(r->codec, q);
}

void mc_reader_set_partial_fetch(mc_reader *r, int on) {
    if (!r) return;
    r->partial = on != 0;
    r->hdr_off = ~0ull;
}

uint64_t mc_chunk_offset_chk(mc_reader *r, int lod, int cz, int cy, int cx, int *err) {
    if (err) *err = 0;
    if (!r || lod < 0 || lod > 7) return 0;
    return resolve(r, lod, cz, cy, cx, err);
}

uint64_t mc_chunk_offset(mc_reader *r, int lod, int cz, int cy, int cx) {
    return mc_chunk_offset_chk(r, lod, cz, cy, cx, nullptr);
}

// src/mc_stream.c:292-323
void mc_decode_block(mc_reader *r, uint64_t co, int bz, int by, int bx, mc_u8 *dst) {
    if (!dst) return;
    float q = 1.0f;
    const uint8_t *base;
    if (!r || co <= kSlotZero || bz < 0 || by < 0 || bx < 0 || bz > 15 || by > 15 || bx > 15 ||
        !chunk_blocks(r, co, &q, &base)) {
        memset(dst, 0, kN3);
        return;
    }
    const BlockSrc b = block_src(r, co, base, (bz * 16 + by) * 16 + bx);
    if (!b.present) { memset(dst, 0, kN3); return; }
    const uint8_t *p = b.ptr;
    if (!p) {   // partial: the block's own payload
        r->pbuf.resize(b.len ? b.len : 1);
        if (b.len && sread(r, b.off, b.len, r->pbuf.data()) != 0) { memset(dst, 0, kN3); return; }
        p = r->pbuf.data();
    }
    mc_codec_ctx_set_quality(r->codec, q);
    mc_dec_block(r->codec, p, b.len, dst);
}

uint64_t mc_reader_chunk_blob_len(mc_reader *r, uint64_t co) {
    if (!r || !co) return 0;
    if (r->arc) return blob_struct_len(r->arc, co, r->len);
    uint8_t bh[kBlobHdr];
    if (sread(r, co, kBlobHdr, bh) != 0) return 0;
    uint16_t fml;
    memcpy(&fml, bh + 12, 2);
    const uint64_t bm_off = co + kBlobHdr + fml;
    uint8_t bm[kBitmapBytes];
    if (sread(r, bm_off, kBitmapBytes, bm) != 0) return 0;
    uint32_t np = 0;
    for (int i = 0; i < kBitmapBytes; ++i) np += (uint32_t)__builtin_popcount(bm[i]);
    if (!np) return bm_off + kBitmapBytes - co;
    std::vector<uint8_t> lens(2ull * np);
    if (sread(r, bm_off + kBitmapBytes, 2 * np, lens.data()) != 0) return 0;
    uint64_t pay = 0;
    for (uint32_t s = 0; s < np; ++s) pay += (uint16_t)(lens[2 * s] | (lens[2 * s + 1] << 8));
    return bm_off + kBitmapBytes + 2ull * np + pay - co;
}

int mc_reader_read_blob(mc_reader *r, uint64_t co, size_t len, uint8_t *dst) {
    if (!r || !co || !len || !dst) return -1;
    if (r->arc) {
        if (co > r->len || len > r->len - co) return -1;
        memcpy(dst, r->arc + co, len);
        return 0;
    }
    for (size_t done = 0; done < len;) {
        const uint32_t n = len - done > 0x40000000u ? 0x40000000u : (uint32_t)(len - done);
        if (sread(r, co + done, n, dst + done) != 0) return -1;
        done += n;
    }
    return 0;
}

int mc_reader_priors(mc_reader *r, const uint16_t **plo, const uint16_t **phi) {
    if (!r || !r->has_priors) return 0;
    if (plo) *plo = reinterpret_cast<const uint16_t *>(r->priors + 8);
    if (phi) *phi = reinterpret_cast<const uint16_t *>(r->priors + 8 + 8 * 32 * 2);
    return 1;
}

void mc_reader_dims(mc_reader *r, int *nx, int *ny, int *nz) {
    if (nx) *nx = r ? r->nx : 0;
    if (ny) *ny = r ? r->ny : 0;
    if (nz) *nz = r ? r->nz : 0;
}

float mc_reader_quality(mc_reader *r) { return r ? r->quality : 0.0f; }

int mc_reader_nlods(mc_reader *r) {
    if (!r) return 0;
    int n = 0;
    for (int l = 0; l < 8; ++l)
        if (r->roots[l]) n = l + 1;
    return n;
}

// Batched: blocks (bz, by, bx) = coords[3i..3i+2] of the chunk at co into
// DEVICE memory d_out + 4096*i (16^3, z,y,x). Absent blocks, a missing chunk
// and unreadable bytes decode to zeros. In partial mode only the asked-for
// payloads are read, adjacent ones in one range read each.
int mc_b200_reader_decode_blocks(mc_reader *r, uint64_t co, const int *coords, int n, mc_u8 *d_out, void *stream) {
    if (!r || n < 0 || (n && (!coords || !d_out))) {
        set_error("reader_decode_blocks: bad arguments");
        return -1;
    }
    if (!n) return 0;
    Lane *L = lane();
    if (!L) return -1;
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : L->stream;
    float q = 1.0f;
    const uint8_t *base = nullptr;
    const bool readable = co > kSlotZero && chunk_blocks(r, co, &q, &base);
    mc_codec_ctx_set_quality(r->codec, q);   // the quality mc_decode_block decodes at
    const int slot = qslot(r->codec->quality);
    if (slot < 0) return -1;
    // payload source of every requested block, then the packed staging layout
    std::vector<BlockSrc> src((size_t)n);
    uint64_t total = 0;
    for (int i = 0; i < n; ++i) {
        const int bz = coords[3 * i], by = coords[3 * i + 1], bx = coords[3 * i + 2];
        const bool ok = readable && bz >= 0 && by >= 0 && bx >= 0 && bz < 16 && by < 16 && bx < 16;
        src[i] = ok ? block_src(r, co, base, (bz * 16 + by) * 16 + bx) : BlockSrc{nullptr, 0, 0, false};
        if (src[i].present) total += src[i].len;
    }
    if (!L->h_stage.ensure(total + 64) || !L->src.ensure(total + 64) || !cuda_ok(cudaStreamSynchronize(s), "sync"))
        return -1;
    uint8_t *hs = L->h_stage.as<uint8_t>();
    std::vector<uint64_t> at((size_t)n, 0);
    if (base) {   // host bytes: pack the payloads
        uint64_t pos = 0;
        for (int i = 0; i < n; ++i) {
            if (!src[i].present) continue;
            memcpy(hs + pos, src[i].ptr, src[i].len);
            at[i] = pos;
            pos += src[i].len;
        }
    } else if (readable) {   // partial: one range read per run of adjacent payloads
        std::vector<int> ord;
        for (int i = 0; i < n; ++i)
            if (src[i].present) ord.push_back(i);
        std::sort(ord.begin(), ord.end(), [&](int a, int b) { return src[a].off < src[b].off; });
        uint64_t pos = 0;
        for (size_t k = 0; k < ord.size();) {
            const uint64_t run0 = src[ord[k]].off;
            uint64_t run1 = run0 + src[ord[k]].len;
            size_t e = k + 1;
            while (e < ord.size() && src[ord[e]].off <= run1) {   // adjacent or repeated blocks
                run1 = std::max(run1, src[ord[e]].off + src[ord[e]].len);
                ++e;
            }
            if (run1 > run0 && sread(r, run0, (uint32_t)(run1 - run0), hs + pos) != 0) {
                for (size_t j = k; j < e; ++j) src[ord[j]].present = false;   // unreadable: zeros
            } else {
                for (size_t j = k; j < e; ++j) at[ord[j]] = pos + (src[ord[j]].off - run0);
                pos += run1 - run0;
            }
            k = e;
        }
        total = pos;
    }
    std::vector<DecItem> items((size_t)n);
    for (int i = 0; i < n; ++i) {
        DecItem &it = items[i];
        it = DecItem{};
        it.src = (uint64_t)(uintptr_t)(L->src.as<uint8_t>() + at[i]);
        it.dst = (uint64_t)(uintptr_t)(d_out + (size_t)kN3 * i);
        it.sz = 256;
        it.sy = 16;
        it.len = src[i].present ? src[i].len : 0;
        it.qslot = (uint16_t)slot;
        it.clip_lo = kClipFullLo;
        it.clip_hi = kClipFullHi;
    }
    if ((total && !cuda_ok(cudaMemcpyAsync(L->src.p, hs, total, cudaMemcpyHostToDevice, s), "H2D payloads")) ||
        !decode_items(*L, items.data(), n, s) || !cuda_ok(cudaStreamSynchronize(s), "sync"))
        return -1;
    return 0;
}

}  // extern "C"
