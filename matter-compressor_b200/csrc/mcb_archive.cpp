// mcb_archive.cpp -- the reference's appendable mmap archive and its C ABI,
// with the block work sent to the GPU.
//
// Host side (this file): the on-disk format and its write discipline
// (src/mc_archive.c:247-601): a [256 B header][128 KiB metadata] prefix, dense
// 4096-slot u64 node tables allocated 8-aligned at the append cursor and
// CAS-published, chunk blobs appended at EOF with the shard slot written last
// as the commit word. Every allocation happens in the reference's order, so a
// call sequence produces a byte-identical file.
//
// Device side: the archive's bytes are mirrored in HBM (synced lazily before a
// decode: new bytes past the synced mark plus the in-place index writes made
// since), block payloads are decoded straight from the mirror, and encoded
// blobs come back from the device for installation.
#include <errno.h>
#include <fcntl.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <memory>
#include <atomic>
#include <mutex>
#include <vector>

#include "mcb_archive.h"
#include "mcb_host_codec.h"
#include "mcb_kernels.h"
#include "mcb_tables.h"

using namespace mcb;

namespace {
// header field offsets (src/mc_archive.h:73-94)
constexpr uint32_t kMagic = 0x0043434Du, kVersion = 7;
constexpr uint64_t HMAGIC = 0, HVER = 4, HNX = 12, HNY = 16, HNZ = 20, HROOT = 24, HTOTLEN = 88,
                   HMETAOFF = 96, HMETACAP = 104, HMETALEN = 112, HQUALITY = 120, HCODEC = 124,
                   HPRIOR = 128;
constexpr uint64_t kHdr = 256, kMetaEnd = 128 * 1024, kMetaCap = kMetaEnd - kHdr;
constexpr uint64_t kNodeBytes = (uint64_t)kGrid3 * 8;
constexpr uint32_t kPriorsMagic = 0x53524950u;
constexpr uint64_t kPriorsBytes = 8 + 2 * 8 * 32 * 2;
constexpr uint64_t kGrowStep = 1ull << 30;
constexpr uint64_t kReserveMax = 10ull << 40;
}  // namespace

// ================================================================= helpers
namespace {

inline uint64_t rd64(const uint8_t *p) { uint64_t v; memcpy(&v, p, 8); return v; }
inline void wr64(uint8_t *p, uint64_t v) { memcpy(p, &v, 8); }
inline int nib(int c, int level) { return (c >> (4 * level)) & 15; }
inline std::atomic<uint64_t> *slot_at(mc_archive *a, uint64_t off) {
    return reinterpret_cast<std::atomic<uint64_t> *>(a->base + off);
}
// record an in-place write for the device mirror (caller holds write_mu)
inline void touch(mc_archive *a, uint64_t off, uint64_t len) {
    std::lock_guard<std::mutex> g(a->mir_mu);
    if (off < a->synced) a->dirty.emplace_back(off, len);
}

// src/mc_archive.c:494-503
uint64_t reserve_for_dims(int nx, int ny, int nz) {
    uint64_t need = 0, dz = nz, dy = ny, dx = nx;
    for (int l = 0; l < 8; ++l) {
        uint64_t pz = (dz + 255) / 256 * 256, py = (dy + 255) / 256 * 256, px = (dx + 255) / 256 * 256;
        need += pz * py * px;
        dz = (dz + 1) / 2; dy = (dy + 1) / 2; dx = (dx + 1) / 2;
    }
    uint64_t r = need + need / 2 + (1ull << 30);
    return r > kReserveMax ? kReserveMax : r;
}

// grow the file so [0, need) is backed (src/mc_archive.c:327-354)
int ensure_len(mc_archive *a, uint64_t need) {
    if (need <= a->file_len.load(std::memory_order_acquire)) return 0;
    std::lock_guard<std::mutex> g(a->grow_mu);
    uint64_t fl = a->file_len.load(std::memory_order_relaxed);
    if (need <= fl) return 0;
    uint64_t nf = fl;
    while (nf < need) nf += kGrowStep;
    if (nf > a->reserve) {
        fprintf(stderr, "mc_archive: grow beyond reservation (%llu > %llu)\n", (unsigned long long)nf,
                (unsigned long long)a->reserve);
        return -1;
    }
    int gr = fallocate(a->fd, 0, (off_t)fl, (off_t)(nf - fl));
    if (gr != 0 && (errno == EOPNOTSUPP || errno == ENOSYS)) gr = ftruncate(a->fd, (off_t)nf);
    if (gr != 0) return -1;
    a->file_len.store(nf, std::memory_order_release);
    return 0;
}
uint64_t alloc_at_eof(mc_archive *a, uint64_t n) {
    uint64_t off = a->cursor.fetch_add(n, std::memory_order_relaxed);
    if (ensure_len(a, off + n) != 0) return ~0ull;
    return off;
}
uint64_t alloc_aligned(mc_archive *a, uint64_t n, uint64_t align) {
    uint64_t cur = a->cursor.load(std::memory_order_relaxed);
    for (;;) {
        uint64_t off = (cur + (align - 1)) & ~(align - 1);
        if (a->cursor.compare_exchange_weak(cur, off + n, std::memory_order_relaxed)) {
            if (ensure_len(a, off + n) != 0) return ~0ull;
            return off;
        }
    }
}
// publish `want` into an empty slot; returns the slot's winner
uint64_t publish_child(mc_archive *a, uint64_t at, uint64_t want) {
    uint64_t exp = 0;
    if (slot_at(a, at)->compare_exchange_strong(exp, want, std::memory_order_release, std::memory_order_acquire)) {
        touch(a, at, 8);
        return want;
    }
    return exp;
}
// index path root -> inner -> shard for a chunk; returns the shard slot's file
// offset (src/mc_archive.c:408-442)
uint64_t ensure_shard_slot(mc_archive *a, int lod, int cz, int cy, int cx) {
    uint64_t root = slot_at(a, HROOT + (uint64_t)lod * 8)->load(std::memory_order_acquire);
    if (!root) {
        uint64_t no = alloc_aligned(a, kNodeBytes, 8);
        if (no == ~0ull) return ~0ull;
        memset(a->base + no, 0, kNodeBytes);
        root = publish_child(a, HROOT + (uint64_t)lod * 8, no);
    }
    uint64_t node = root;
    for (int level = 2; level >= 1; --level) {
        int idx = (nib(cz, level) * 16 + nib(cy, level)) * 16 + nib(cx, level);
        uint64_t child = slot_at(a, node + (uint64_t)idx * 8)->load(std::memory_order_acquire);
        if (!child) {
            uint64_t no = alloc_aligned(a, kNodeBytes, 8);
            if (no == ~0ull) return ~0ull;
            memset(a->base + no, 0, kNodeBytes);
            child = publish_child(a, node + (uint64_t)idx * 8, no);
        }
        node = child;
    }
    int n0 = (nib(cz, 0) * 16 + nib(cy, 0)) * 16 + nib(cx, 0);
    return node + (uint64_t)n0 * 8;
}
}  // namespace

namespace mcb {
// src/mc_archive.c:447-456
int mark_zero(mc_archive *a, int lod, int cz, int cy, int cx) {
    std::lock_guard<std::mutex> g(a->write_mu);
    uint64_t slot = ensure_shard_slot(a, lod, cz, cy, cx);
    if (slot == ~0ull) return -1;
    wr64(a->base + slot, kSlotZero);
    touch(a, slot, 8);
    a->gen.fetch_add(1, std::memory_order_release);
    return 0;
}
// Bytes into the file at off, seen through the shared mapping at once (one
// page cache): pwrite fills the pages without a fault per page of the
// mapping, which a memcpy into freshly allocated file pages takes.
static void write_file(mc_archive *a, uint64_t off, const uint8_t *src, size_t len) {
    size_t done = 0;
    while (done < len) {
        const ssize_t w = pwrite(a->fd, src + done, len - done, (off_t)(off + done));
        if (w < 0 && errno == EINTR) continue;
        if (w <= 0) break;
        done += (size_t)w;
    }
    if (done < len) memcpy(a->base + off + done, src + done, len - done);
}

// src/mc_archive.c:458-485
int install_blob(mc_archive *a, int lod, int cz, int cy, int cx, const uint8_t *blob, size_t len) {
    std::lock_guard<std::mutex> g(a->write_mu);
    uint64_t slot = ensure_shard_slot(a, lod, cz, cy, cx);
    if (slot == ~0ull) return -1;
    uint64_t off = alloc_at_eof(a, len);
    if (off == ~0ull) return -1;
    write_file(a, off, blob, len);
    slot_at(a, slot)->store(off, std::memory_order_release);
    touch(a, slot, 8);
    a->gen.fetch_add(1, std::memory_order_release);
    uint64_t cur = a->cursor.load(std::memory_order_relaxed);
    slot_at(a, HTOTLEN)->store(cur, std::memory_order_relaxed);
    touch(a, HTOTLEN, 8);
    return 0;
}

}  // namespace mcb

namespace {
// src/mc_archive.h:133-145: walk the 3 dense levels; out-of-range -> absent
uint64_t resolve_chunk(const uint8_t *arc, uint64_t root, int cz, int cy, int cx, uint64_t end) {
    uint64_t node = root;
    for (int level = 2; level >= 0; --level) {
        if (!node) return 0;
        int idx = (nib(cz, level) * 16 + nib(cy, level)) * 16 + nib(cx, level);
        if (node > end || (uint64_t)idx * 8 + 8 > end - node) return 0;
        node = rd64(arc + node + (uint64_t)idx * 8);
    }
    return node;
}

}  // namespace

namespace mcb {
// keyed by (archive base, chunk offset, stored hash): a reused offset with new
// content never serves a stale index. Each thread keeps the indexes of its 32
// most recent chunks (direct-mapped by offset), so block walks that alternate
// between neighbouring chunks (regions across chunk borders) reuse them.
const ChunkIndex &chunk_index(const uint8_t *arc, uint64_t co) {
    constexpr int kWays = 32;
    static thread_local std::unique_ptr<ChunkIndex[]> cache;
    if (!cache) cache.reset(new ChunkIndex[kWays]);
    ChunkIndex &ix = cache[(co * 0x9E3779B97F4A7C15ull) >> 59];
    uint64_t tag = rd64(arc + co + 4);
    if (ix.arc == arc && ix.chunk_off == co && ix.tag == tag) return ix;
    uint16_t fml;
    memcpy(&fml, arc + co + 12, 2);
    uint64_t bm_off = co + kBlobHdr + fml;
    const uint8_t *bm = arc + bm_off;
    uint32_t np = 0;
    for (int i = 0; i < kBitmapBytes; ++i) np += (uint32_t)__builtin_popcount(bm[i]);
    const uint8_t *lens = bm + kBitmapBytes;
    uint64_t pay = bm_off + kBitmapBytes + 2ull * np;
    uint32_t slot = 0;
    for (int bi = 0; bi < kGrid3; ++bi) {
        if ((bm[bi >> 3] >> (bi & 7)) & 1) {
            uint16_t l;
            memcpy(&l, lens + 2 * slot, 2);
            ix.off[bi] = pay;
            ix.len[bi] = l;
            pay += l;
            ++slot;
        } else {
            ix.off[bi] = 0;
            ix.len[bi] = 0;
        }
    }
    ix.arc = arc; ix.chunk_off = co; ix.tag = tag;
    return ix;
}

float chunk_q(const mc_archive *a, uint64_t co) {
    float q;
    memcpy(&q, a->base + co, 4);
    return q;
}
}  // namespace mcb

namespace {

// Load the archive's prior blob, if any, as the process-global priors
// (src/mc_archive.c:665-672).
void priors_load(const uint8_t *base) {
    uint64_t off = rd64(base + HPRIOR);
    if (!off) { priors_set(nullptr, nullptr); return; }
    uint32_t magic;
    memcpy(&magic, base + off, 4);
    if (magic != kPriorsMagic) { priors_set(nullptr, nullptr); return; }
    priors_set(reinterpret_cast<const uint16_t *>(base + off + 8),
               reinterpret_cast<const uint16_t *>(base + off + 8 + 8 * 32 * 2));
}

}  // namespace

// ================================================================= mirror
namespace mcb {
uint8_t *mirror_sync(mc_archive *a, Lane &L) {
    std::lock_guard<std::mutex> gw(a->write_mu);
    std::lock_guard<std::mutex> gm(a->mir_mu);
    const uint64_t cur = a->cursor.load(std::memory_order_acquire);
    if (!a->mir_ev && !cuda_ok(cudaEventCreateWithFlags(&a->mir_ev, cudaEventDisableTiming), "event")) return nullptr;
    if (cur > a->d_cap) {
        uint64_t cap = std::max<uint64_t>(cur + (cur >> 2) + (1 << 20), 1 << 24);
        uint8_t *nd = nullptr;
        if (!cuda_ok(cudaMalloc(&nd, cap + 64), "mirror alloc")) return nullptr;
        if (a->d_base) {
            cudaDeviceSynchronize();   // no decode may still read the old mirror
            cudaMemcpy(nd, a->d_base, a->synced, cudaMemcpyDeviceToDevice);
            cudaFree(a->d_base);
        }
        cudaMemset(nd + cap, 0, 64);
        a->d_base = nd;
        a->d_cap = cap;
    }
    bool copied = false;
    for (auto &d : a->dirty) {
        uint64_t end = std::min(d.first + d.second, a->synced);
        if (d.first < end) {
            if (!cuda_ok(cudaMemcpyAsync(a->d_base + d.first, a->base + d.first, end - d.first,
                                         cudaMemcpyHostToDevice, L.stream), "mirror sync"))
                return nullptr;
            copied = true;
        }
    }
    a->dirty.clear();
    if (cur > a->synced) {
        if (!copy_to_device(L, a->d_base + a->synced, a->base + a->synced, cur - a->synced)) return nullptr;
        a->synced = cur;
        copied = true;
    }
    if (copied && !cuda_ok(cudaEventRecord(a->mir_ev, L.stream), "event")) return nullptr;
    if (!cuda_ok(cudaStreamWaitEvent(L.stream, a->mir_ev, 0), "stream wait")) return nullptr;
    return a->d_base;
}
}  // namespace mcb

// ================================================================= codec ctx
namespace mcb {

// The node walk of src/mc_archive.c:1072-1111 with its bounds: every header-
// derived offset is checked against [kHdr, len) before it is read, and a
// blob's structure (header, fmap, bitmap, length table, payloads) must lie
// inside the archive (src/mc_archive.h:212-226). Node tables and blobs that
// fail count as bad; the blobs that pass are appended to `out` for hashing.
long verify_walk(const uint8_t *arc, size_t len, std::vector<VerifyBlob> &out, long *total) {
    *total = 0;
    if (!arc || len < kHdr) return -1;
    auto node_ok = [len](uint64_t off) { return off >= kHdr && off <= len && len - off >= kNodeBytes; };
    long bad = 0;
    for (int lod = 0; lod < 8; ++lod) {
        uint64_t root = rd64(arc + HROOT + (uint64_t)lod * 8);
        if (!root) continue;
        if (!node_ok(root)) { bad++; continue; }
        for (int n2 = 0; n2 < kGrid3; ++n2) {
            uint64_t inner = rd64(arc + root + (uint64_t)n2 * 8);
            if (!inner) continue;
            if (!node_ok(inner)) { bad++; continue; }
            for (int n1 = 0; n1 < kGrid3; ++n1) {
                uint64_t shard = rd64(arc + inner + (uint64_t)n1 * 8);
                if (!shard) continue;
                if (!node_ok(shard)) { bad++; continue; }
                for (int n0 = 0; n0 < kGrid3; ++n0) {
                    uint64_t co = rd64(arc + shard + (uint64_t)n0 * 8);
                    if (co <= kSlotZero) continue;
                    (*total)++;
                    if (co > len || len - co < (uint64_t)kBlobHdr) { bad++; continue; }
                    uint16_t fml;
                    memcpy(&fml, arc + co + 12, 2);
                    const uint64_t bm_off = co + kBlobHdr + fml;
                    if (bm_off > len || len - bm_off < (uint64_t)kBitmapBytes) { bad++; continue; }
                    uint32_t np = 0;
                    for (int i = 0; i < kBitmapBytes; ++i) np += (uint32_t)__builtin_popcount(arc[bm_off + i]);
                    const uint64_t lens_off = bm_off + kBitmapBytes;
                    if (len - lens_off < 2ull * np) { bad++; continue; }
                    uint64_t pay = 0;
                    for (uint32_t k = 0; k < np; ++k) {
                        uint16_t l;
                        memcpy(&l, arc + lens_off + 2 * k, 2);
                        pay += l;
                    }
                    const uint64_t bl = lens_off + 2ull * np + pay - co;
                    if (co + bl > len) { bad++; continue; }
                    out.push_back(VerifyBlob{co, bl, np, lod, n2, n1, n0});
                }
            }
        }
    }
    return bad;
}

}  // namespace mcb

extern "C" {

mc_codec_ctx *mc_codec_ctx_new(void) { return new (std::nothrow) mc_codec_ctx(); }
void mc_codec_ctx_free(mc_codec_ctx *C) { delete C; }
void mc_codec_ctx_set_quality(mc_codec_ctx *C, float q) {
    q = sanitize_q(q);
    if (C) C->quality = q;
}
float mc_codec_ctx_get_quality(mc_codec_ctx *C) { return C ? C->quality : 0.0f; }
void mc_codec_ctx_set_max_error(mc_codec_ctx *C, int tau) { if (C) C->max_err = tau < 0 ? 0 : tau; }
int mc_codec_ctx_get_max_error(mc_codec_ctx *C) { return C ? C->max_err : 0; }

// calibrated preset ladder (src/mc_codec.c:504-531)
static const struct { float q; int tau; const char *name; } kPresets[8] = {
    {0.5f, 1, "archival"}, {0.5f, 2, "master"}, {1.0f, 4, "high"}, {2.5f, 8, "balanced"},
    {6.0f, 16, "streaming"}, {16.0f, 32, "fast"}, {32.0f, 64, "ultrafast"}, {64.0f, 128, "preview"},
};
float mc_preset_quality(mc_preset p) {
    if ((unsigned)p >= MC_PRESET_COUNT) p = MC_PRESET_STREAMING;
    return kPresets[p].q;
}
int mc_preset_tau(mc_preset p) {
    if ((unsigned)p >= MC_PRESET_COUNT) p = MC_PRESET_STREAMING;
    return kPresets[p].tau;
}
const char *mc_preset_name(mc_preset p) {
    if ((unsigned)p >= MC_PRESET_COUNT) return "?";
    return kPresets[p].name;
}
float mc_apply_preset(mc_codec_ctx *C, mc_preset p) {
    if ((unsigned)p >= MC_PRESET_COUNT) p = MC_PRESET_STREAMING;
    mc_codec_ctx_set_quality(C, kPresets[p].q);
    mc_codec_ctx_set_max_error(C, kPresets[p].tau);
    return kPresets[p].q;
}
void mc_codec_init(void) { runtime(); }
void mc_codec_set_priors(const uint16_t *plo, const uint16_t *phi) { priors_set(plo, phi); }

void mc_buf_put(mc_buf *b, const void *s, size_t n) {
    if (b->len + n > b->cap) {
        size_t nc = b->cap ? b->cap * 2 : 1 << 16;
        while (nc < b->len + n) nc *= 2;
        void *t = realloc(b->p, nc);
        if (!t) return;
        b->p = static_cast<mc_u8 *>(t);
        b->cap = nc;
    }
    memcpy(b->p + b->len, s, n);
    b->len += n;
}

uint32_t mc_enc_fracmap(const mc_u8 *frac, mc_u8 *out, size_t cap) { return host_enc_fracmap(frac, out, cap); }
void mc_dec_fracmap(const mc_u8 *in, uint32_t len, mc_u8 *frac) { host_dec_fracmap(in, len, frac); }
uint64_t mc_xxh64(const void *data, size_t len, uint64_t seed) { return host_xxh64(data, len, seed); }
uint64_t mc_chunk_compute_hash(const uint8_t *blob, uint64_t blob_len) { return host_blob_hash(blob, blob_len); }

// ---------------------------------------------------------------- block codec
int mc_enc_block(mc_codec_ctx *C, const mc_u8 *vox, mc_buf *out, uint32_t *len_out) {
    *len_out = 0;
    Lane *L = lane();
    Runtime *R = runtime();
    if (!L || !R || !C) return 0;
    int slot = qslot(C->quality);
    if (slot < 0) return 0;
    if (!cuda_ok(cudaEventSynchronize(L->done), "sync") || !L->src.ensure(kN3) || !L->enc_pay.ensure(kEncCap) ||
        !L->enc_len.ensure(4) || !L->enc_frac.ensure(4) || !L->enc_items.ensure(sizeof(EncItem)) ||
        !L->status.ensure(16) || !L->h_stage.ensure(kEncCap + 64) || !L->enc_lv.ensure(2 * kN3) ||
        !L->enc_corr.ensure(4 * kN3) || !L->enc_sym.ensure(8))
        return 0;
    EncItem it{};
    it.src = (uint64_t)(uintptr_t)L->src.p;
    it.sz = 256;
    it.sy = 16;
    it.out = (uint64_t)(uintptr_t)L->enc_pay.p;
    it.qslot = (uint16_t)slot;
    it.tau = (uint16_t)std::min(C->max_err, 65535);
    uint8_t *hs = L->h_stage.as<uint8_t>();
    memcpy(hs, vox, kN3);
    memcpy(hs + kN3, &it, sizeof it);
    EncParams ep;
    ep.items = L->enc_items.as<EncItem>();
    ep.n = 1;
    ep.qtab = R->d_qtab;
    ep.scan = R->d_scan;
    ep.len = L->enc_len.as<uint32_t>();
    ep.frac = L->enc_frac.as<uint8_t>();
    ep.status = L->status.as<uint32_t>();
    ep.levels = L->enc_lv.as<int16_t>();
    ep.corr = L->enc_corr.as<uint32_t>();
    ep.sym = L->enc_sym.as<uint2>();
    uint32_t len = 0;
    if (!cuda_ok(cudaMemcpyAsync(L->src.p, hs, kN3, cudaMemcpyHostToDevice, L->stream), "H2D") ||
        !cuda_ok(cudaMemcpyAsync(L->enc_items.p, hs + kN3, sizeof it, cudaMemcpyHostToDevice, L->stream), "H2D") ||
        !cuda_ok(cudaMemsetAsync(L->status.p, 0, 16, L->stream), "memset") ||
        !cuda_ok(launch_encode(ep, L->stream), "encode launch") ||
        !cuda_ok(cudaMemcpyAsync(&len, L->enc_len.p, 4, cudaMemcpyDeviceToHost, L->stream), "D2H") ||
        !cuda_ok(cudaStreamSynchronize(L->stream), "sync"))
        return 0;
    if (!len) return 0;
    if (!cuda_ok(cudaMemcpy(hs, L->enc_pay.p, len, cudaMemcpyDeviceToHost), "D2H")) return 0;
    mc_buf_put(out, hs, len);
    *len_out = len;
    return 1;
}

void mc_dec_block(mc_codec_ctx *C, const mc_u8 *p, uint32_t plen, mc_u8 *dst) {
    Lane *L = lane();
    if (!L || !C) { memset(dst, 0, kN3); return; }
    int slot = qslot(C->quality);
    if (slot < 0 || !cuda_ok(cudaEventSynchronize(L->done), "sync") || !L->src.ensure(plen + 64) ||
        !L->h_stage.ensure(plen + 64)) {
        memset(dst, 0, kN3);
        return;
    }
    uint8_t *hs = L->h_stage.as<uint8_t>();
    if (plen) memcpy(hs, p, plen);
    DecItem it{};
    it.src = (uint64_t)(uintptr_t)L->src.p;
    it.len = plen;
    it.qslot = (uint16_t)slot;
    it.clip_lo = kClipFullLo;
    it.clip_hi = kClipFullHi;
    if ((plen && !cuda_ok(cudaMemcpyAsync(L->src.p, hs, plen, cudaMemcpyHostToDevice, L->stream), "H2D")) ||
        !decode_one_host(*L, it, dst))
        memset(dst, 0, kN3);
}

// ================================================================= archive
mc_archive *mc_archive_open(const char *path, int dim, float quality) {
    return mc_archive_open_dims(path, dim, dim, dim, quality);
}

mc_archive *mc_archive_open_dims(const char *path, int nx, int ny, int nz, float quality) {
    if (nx <= 0 || ny <= 0 || nz <= 0) { fprintf(stderr, "mc_archive_open: bad dims\n"); return nullptr; }
    int fd = open(path, O_RDWR | O_CREAT, 0644);
    if (fd < 0) { perror("mc_archive_open: open"); return nullptr; }
    struct stat sb;
    if (fstat(fd, &sb) != 0) { perror("fstat"); close(fd); return nullptr; }
    const bool fresh = sb.st_size == 0;
    const uint64_t reserve = reserve_for_dims(nx, ny, nz);
    uint64_t init_len;
    if (fresh) {
        init_len = kMetaEnd;
        if (ftruncate(fd, (off_t)init_len) != 0) { perror("ftruncate"); close(fd); return nullptr; }
    } else {
        init_len = (uint64_t)sb.st_size;
    }
    void *m = mmap(nullptr, reserve, PROT_READ | PROT_WRITE, MAP_SHARED | MAP_NORESERVE, fd, 0);
    if (m == MAP_FAILED) { perror("mmap"); close(fd); return nullptr; }
    uint8_t *base = static_cast<uint8_t *>(m);
    mc_archive *a = new mc_archive();
    a->fd = fd;
    a->base = base;
    a->quality = quality;
    a->reserve = reserve;
    a->file_len.store(init_len);
    if (fresh) {
        memset(base, 0, kHdr);
        uint32_t ux = nx, uy = ny, uz = nz;
        memcpy(base + HMAGIC, &kMagic, 4);
        memcpy(base + HVER, &kVersion, 4);
        memcpy(base + HNX, &ux, 4);
        memcpy(base + HNY, &uy, 4);
        memcpy(base + HNZ, &uz, 4);
        wr64(base + HMETAOFF, kHdr);
        wr64(base + HMETACAP, kMetaCap);
        wr64(base + HMETALEN, 0);
        wr64(base + HTOTLEN, kMetaEnd);
        memcpy(base + HQUALITY, &quality, 4);
        uint32_t bc = MC_BLOCKCODEC_CABAC;
        memcpy(base + HCODEC, &bc, 4);
        a->cursor.store(kMetaEnd);
    } else {
        uint32_t magic, ver, ux, uy, uz;
        memcpy(&magic, base + HMAGIC, 4);
        memcpy(&ver, base + HVER, 4);
        memcpy(&ux, base + HNX, 4);
        memcpy(&uy, base + HNY, 4);
        memcpy(&uz, base + HNZ, 4);
        if (magic != kMagic || ver != kVersion || (int)ux != nx || (int)uy != ny || (int)uz != nz) {
            fprintf(stderr, "mc_archive_open: %s is not a matching mc archive (magic/ver/dims)\n", path);
            munmap(base, reserve);
            close(fd);
            delete a;
            return nullptr;
        }
        uint64_t totlen = rd64(base + HTOTLEN);
        if (totlen < kMetaEnd) totlen = kMetaEnd;
        a->cursor.store(totlen);
        priors_load(base);
    }
    return a;
}

void mc_archive_close(mc_archive *a) {
    if (!a) return;
    uint64_t cur = a->cursor.load();
    wr64(a->base + HTOTLEN, cur);
    msync(a->base, cur, MS_SYNC);
    munmap(a->base, a->reserve);
    if (ftruncate(a->fd, (off_t)cur) != 0) perror("mc_archive_close: ftruncate");
    close(a->fd);
    if (a->d_base) {
        cudaDeviceSynchronize();
        cudaFree(a->d_base);
    }
    if (a->mir_ev) cudaEventDestroy(a->mir_ev);
    delete a;
}

int mc_archive_set_block_codec(mc_archive *a, uint32_t codec) {
    if (!a || codec != MC_BLOCKCODEC_CABAC) return -1;
    std::lock_guard<std::mutex> g(a->write_mu);
    a->block_codec = codec;
    memcpy(a->base + HCODEC, &codec, 4);
    touch(a, HCODEC, 4);
    return 0;
}
uint32_t mc_archive_block_codec(const mc_archive *a) { return a ? a->block_codec : MC_BLOCKCODEC_CABAC; }

int mc_archive_reserve_index(mc_archive *a, int lod, int cz, int cy, int cx) {
    if (!a || lod < 0 || lod > 7) return -1;
    std::lock_guard<std::mutex> g(a->write_mu);
    return ensure_shard_slot(a, lod, cz, cy, cx) == ~0ull ? -1 : 0;
}

int mc_archive_append_chunk_compressed(mc_archive *a, int lod, int cz, int cy, int cx, const uint8_t *blob,
                                       size_t len) {
    if (!a || lod < 0 || lod > 7 || !blob || !len) return -1;
    return install_blob(a, lod, cz, cy, cx, blob, len);
}

uint64_t mc_archive_data_len(mc_archive *a) { return a ? a->cursor.load(std::memory_order_relaxed) : 0; }

int mc_archive_set_metadata(mc_archive *a, const void *data, size_t len) {
    if (!a || (len && !data)) return -1;
    if (len > kMetaCap) return -1;
    std::lock_guard<std::mutex> g(a->write_mu);
    if (len) memcpy(a->base + kHdr, data, len);
    std::atomic_thread_fence(std::memory_order_release);
    wr64(a->base + HMETALEN, len);
    touch(a, kHdr, len);
    touch(a, HMETALEN, 8);
    return 0;
}

const char *mc_archive_metadata(mc_archive *a, size_t *out_len) {
    if (!a) { if (out_len) *out_len = 0; return nullptr; }
    uint64_t off = rd64(a->base + HMETAOFF), l = rd64(a->base + HMETALEN);
    if (off < kHdr || l > kMetaCap) { if (out_len) *out_len = 0; return nullptr; }
    if (out_len) *out_len = l;
    return reinterpret_cast<const char *>(a->base + off);
}

uint64_t mc_archive_chunk_offset(mc_archive *a, int lod, int cz, int cy, int cx) {
    if (!a || lod < 0 || lod > 7) return 0;
    uint64_t root = rd64(a->base + HROOT + (uint64_t)lod * 8);
    return resolve_chunk(a->base, root, cz, cy, cx, a->file_len.load(std::memory_order_relaxed));
}

mc_cover mc_archive_chunk_coverage(mc_archive *a, int lod, int cz, int cy, int cx) {
    if (!a || lod < 0 || lod > 7) return MC_ABSENT;
    uint64_t off = mc_archive_chunk_offset(a, lod, cz, cy, cx);
    if (!off) return MC_ABSENT;
    return off == kSlotZero ? MC_ZERO : MC_PRESENT;
}

int mc_archive_set_priors(mc_archive *a, const uint16_t plo[8][32], const uint16_t phi[8][32]) {
    if (!a || !plo || !phi) return -1;
    std::lock_guard<std::mutex> g(a->write_mu);
    uint64_t off = alloc_at_eof(a, kPriorsBytes);
    if (off == ~0ull) return -1;
    uint32_t magic = kPriorsMagic, ver = 1;
    memcpy(a->base + off, &magic, 4);
    memcpy(a->base + off + 4, &ver, 4);
    memcpy(a->base + off + 8, plo, 8 * 32 * 2);
    memcpy(a->base + off + 8 + 8 * 32 * 2, phi, 8 * 32 * 2);
    std::atomic_thread_fence(std::memory_order_release);
    wr64(a->base + HPRIOR, off);
    touch(a, HPRIOR, 8);
    priors_set(&plo[0][0], &phi[0][0]);
    return 0;
}

int mc_archive_block_blob(mc_archive *a, uint64_t co, int bz, int by, int bx, const uint8_t **ptr, uint32_t *len) {
    if (ptr) *ptr = nullptr;
    if (len) *len = 0;
    if (!a || co <= kSlotZero) return 0;
    const ChunkIndex &ix = chunk_index(a->base, co);
    int bi = (bz * 16 + by) * 16 + bx;
    if (!ix.off[bi]) return 0;
    if (ix.off[bi] + ix.len[bi] > a->cursor.load(std::memory_order_acquire)) return 0;
    if (ptr) *ptr = a->base + ix.off[bi];
    if (len) *len = ix.len[bi];
    return 1;
}

int mc_archive_block_present(mc_archive *a, int lod, int bz, int by, int bx) {
    if (!a || lod < 0 || lod > 7 || bz < 0 || by < 0 || bx < 0) return 0;
    uint64_t co = mc_archive_chunk_offset(a, lod, bz >> 4, by >> 4, bx >> 4);
    if (co <= kSlotZero) return 0;
    uint16_t fml;
    memcpy(&fml, a->base + co + 12, 2);
    const uint8_t *bm = a->base + co + kBlobHdr + fml;
    int bi = ((bz & 15) * 16 + (by & 15)) * 16 + (bx & 15);
    return (bm[bi >> 3] >> (bi & 7)) & 1;
}

float mc_archive_block_fraction(mc_archive *a, int lod, int bz, int by, int bx) {
    if (!a || lod < 0 || lod > 7 || bz < 0 || by < 0 || bx < 0) return 0.0f;
    uint64_t co = mc_archive_chunk_offset(a, lod, bz >> 4, by >> 4, bx >> 4);
    if (co <= kSlotZero) return 0.0f;
    uint16_t fml;
    memcpy(&fml, a->base + co + 12, 2);
    if (!fml) return 0.0f;
    uint8_t fr[kGrid3];
    host_dec_fracmap(a->base + co + kBlobHdr, fml, fr);
    return (float)fr[((bz & 15) * 16 + (by & 15)) * 16 + (bx & 15)] / 15.0f;
}

// xorshift64 sampler with fraction-map rejection (src/mc_archive.c:922-948)
int mc_archive_sample_boxes(mc_archive *a, int lod, uint64_t seed, int count, long dz, long dy, long dx,
                            float min_frac, mc_box *out) {
    if (!a || !out || count <= 0 || dz <= 0 || dy <= 0 || dx <= 0) return 0;
    uint32_t unx, uny, unz;
    memcpy(&unx, a->base + HNX, 4);
    memcpy(&uny, a->base + HNY, 4);
    memcpy(&unz, a->base + HNZ, 4);
    long NX = (long)unx >> lod, NY = (long)uny >> lod, NZ = (long)unz >> lod;
    if (NZ < dz || NY < dy || NX < dx) return 0;
    uint64_t s = seed ? seed : 0x9E3779B97F4A7C15ull;
    auto rng = [&s]() { uint64_t x = s; x ^= x << 13; x ^= x >> 7; x ^= x << 17; s = x; return x; };
    int got = 0;
    long attempts = 0, max_attempts = (long)count * 256;
    while (got < count && attempts++ < max_attempts) {
        long z0 = (long)(rng() % (uint64_t)(NZ - dz + 1));
        long y0 = (long)(rng() % (uint64_t)(NY - dy + 1));
        long x0 = (long)(rng() % (uint64_t)(NX - dx + 1));
        long bz0 = z0 >> 4, bz1 = (z0 + dz - 1) >> 4, by0 = y0 >> 4, by1 = (y0 + dy - 1) >> 4;
        long bx0 = x0 >> 4, bx1 = (x0 + dx - 1) >> 4;
        double fsum = 0;
        long nb = 0;
        for (long bz = bz0; bz <= bz1; ++bz)
            for (long by = by0; by <= by1; ++by)
                for (long bx = bx0; bx <= bx1; ++bx) {
                    fsum += mc_archive_block_fraction(a, lod, (int)bz, (int)by, (int)bx);
                    nb++;
                }
        if (nb && fsum / nb >= min_frac) { out[got].z0 = z0; out[got].y0 = y0; out[got].x0 = x0; got++; }
    }
    return got;
}

// mc_archive_sample_boxes with the scoring on the device. The fraction map of
// every chunk that a candidate can touch is decoded once into a block grid
// (0 where the chunk is absent, all air or has no map, as
// mc_archive_block_fraction reads it); candidates come from the same
// xorshift64 stream in the same order, scored a batch at a time; the first
// `count` accepted ones are the reference's boxes.
int mc_b200_sample_boxes(mc_archive *a, int lod, uint64_t seed, int count, long dz, long dy, long dx,
                         float min_frac, mc_box *out) {
    if (!a || !out || count <= 0 || dz <= 0 || dy <= 0 || dx <= 0 || lod < 0 || lod > 7) return 0;
    uint32_t unx, uny, unz;
    memcpy(&unx, a->base + HNX, 4);
    memcpy(&uny, a->base + HNY, 4);
    memcpy(&unz, a->base + HNZ, 4);
    const long NX = (long)unx >> lod, NY = (long)uny >> lod, NZ = (long)unz >> lod;
    if (NZ < dz || NY < dy || NX < dx) return 0;
    Lane *L = lane();
    if (!L) return 0;
    const long gz = (NZ + 15) >> 4, gy = (NY + 15) >> 4, gx = (NX + 15) >> 4;
    std::vector<uint8_t> grid((size_t)gz * gy * gx, 0);
    uint8_t fr[kGrid3];
    for (long cz = 0; cz * 16 < gz; ++cz)
        for (long cy = 0; cy * 16 < gy; ++cy)
            for (long cx = 0; cx * 16 < gx; ++cx) {
                const uint64_t co = mc_archive_chunk_offset(a, lod, (int)cz, (int)cy, (int)cx);
                if (co <= kSlotZero) continue;
                uint16_t fml;
                memcpy(&fml, a->base + co + 12, 2);
                if (!fml) continue;
                host_dec_fracmap(a->base + co + kBlobHdr, fml, fr);
                for (int b = 0; b < kGrid3; ++b) {
                    const long bz = cz * 16 + (b >> 8), by = cy * 16 + ((b >> 4) & 15), bx = cx * 16 + (b & 15);
                    if (bz < gz && by < gy && bx < gx) grid[(size_t)(bz * gy + by) * gx + bx] = fr[b];
                }
            }
    constexpr int B = 4096;   // candidates per scoring launch
    if (!L->smp_grid.ensure(grid.size()) || !L->smp_cand.ensure(sizeof(long) * 3 * B) || !L->smp_acc.ensure(B) ||
        !cuda_ok(cudaMemcpyAsync(L->smp_grid.p, grid.data(), grid.size(), cudaMemcpyHostToDevice, L->stream),
                 "H2D fraction grid"))
        return 0;
    uint64_t s = seed ? seed : 0x9E3779B97F4A7C15ull;
    auto rng = [&s]() { uint64_t x = s; x ^= x << 13; x ^= x >> 7; x ^= x << 17; s = x; return x; };
    int got = 0;
    long attempts = 0;
    const long max_attempts = (long)count * 256;
    std::vector<long> cand(3 * (size_t)B);
    std::vector<uint8_t> acc(B);
    while (got < count && attempts < max_attempts) {
        const int m = (int)std::min<long>(B, max_attempts - attempts);
        for (int i = 0; i < m; ++i) {
            cand[3 * i] = (long)(rng() % (uint64_t)(NZ - dz + 1));
            cand[3 * i + 1] = (long)(rng() % (uint64_t)(NY - dy + 1));
            cand[3 * i + 2] = (long)(rng() % (uint64_t)(NX - dx + 1));
        }
        attempts += m;
        if (!cuda_ok(cudaMemcpyAsync(L->smp_cand.p, cand.data(), sizeof(long) * 3 * m, cudaMemcpyHostToDevice,
                                     L->stream), "H2D candidates") ||
            !cuda_ok(launch_sample_score(L->smp_grid.as<uint8_t>(), gz, gy, gx, L->smp_cand.as<long>(), m, dz, dy, dx,
                                         min_frac, L->smp_acc.as<uint8_t>(), L->stream), "sample launch") ||
            !cuda_ok(cudaMemcpyAsync(acc.data(), L->smp_acc.p, m, cudaMemcpyDeviceToHost, L->stream), "D2H accept") ||
            !cuda_ok(cudaStreamSynchronize(L->stream), "sync"))
            return got;
        for (int i = 0; i < m && got < count; ++i)
            if (acc[i]) { out[got].z0 = cand[3 * i]; out[got].y0 = cand[3 * i + 1]; out[got].x0 = cand[3 * i + 2]; got++; }
    }
    return got;
}

// src/mc_archive.c:1072-1111: walk every chunk of every LOD, recompute its hash
long mc_verify_archive(const uint8_t *arc, size_t len, int verbose) {
    std::vector<VerifyBlob> blobs;
    long total = 0;
    long bad = verify_walk(arc, len, blobs, &total);
    if (bad < 0) return -1;
    for (const VerifyBlob &v : blobs) {
        if (rd64(arc + v.co + 4) != host_blob_hash(arc + v.co, v.len)) {
            bad++;
            if (verbose)
                fprintf(stderr, "mc_verify: lod %d node %d/%d/%d chunk@%llu CORRUPT\n", v.lod, v.n2, v.n1, v.n0,
                        (unsigned long long)v.co);
        }
    }
    if (verbose) fprintf(stderr, "mc_verify: %ld chunks checked, %ld corrupt\n", total, bad);
    return bad;
}

}  // extern "C"
