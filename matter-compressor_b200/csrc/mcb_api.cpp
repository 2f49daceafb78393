// mcb_api.cpp -- decode and append entry points of the C ABI.
//
// Decode: the host resolves chunks through the index and locates each block's
// payload (src/mc_archive.c:712-740, src/mc_archive.h:175-206); every block
// becomes one work item (payload address in the HBM mirror, output address,
// strides and clip box) and the whole request is decoded by the two kernel
// stages in one batch. Whole chunks, single blocks, regions and batches of
// regions are the same operation with different items.
//
// Append: chunks are encoded on the device, blobs come back to the host and
// are installed in call order, so the file is byte-identical to the
// reference's for the same call sequence (src/mc_archive.c:590-601,861-901).
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <vector>

#include "mcb_archive.h"
#include "mcb_tables.h"

using namespace mcb;

namespace {

constexpr size_t kChunkBytes = (size_t)256 * 256 * 256;

inline uint64_t dptr(const void *p) { return (uint64_t)(uintptr_t)p; }

// Items for every block of one present chunk (co > 1) into a 256^3 output.
void chunk_items(mc_archive *a, uint64_t co, const uint8_t *dbase, int slot, uint8_t *d_chunk_out, DecItem *items) {
    const ChunkIndex &ix = chunk_index(a->base, co);
    const uint64_t cur = a->cursor.load(std::memory_order_acquire);
    for (int bi = 0; bi < kGrid3; ++bi) {
        const int bz = bi >> 8, by = (bi >> 4) & 15, bx = bi & 15;
        DecItem &it = items[bi];
        memset(&it, 0, sizeof it);
        const uint64_t off = ix.off[bi];
        if (off && off + ix.len[bi] <= cur) {   // out-of-bounds payload decodes to zeros (src/mc_archive.c:737-738)
            it.src = dptr(dbase + off);
            it.len = ix.len[bi];
        }
        it.dst = dptr(d_chunk_out + (size_t)(bz * 16) * 65536 + (by * 16) * 256 + bx * 16);
        it.sz = 65536;
        it.sy = 256;
        it.qslot = (uint16_t)slot;
        it.clip_lo = kClipFullLo;
        it.clip_hi = kClipFullHi;
    }
}

// Items for every zero block of an absent chunk.
void zero_chunk_items(uint8_t *d_chunk_out, DecItem *items) {
    for (int bi = 0; bi < kGrid3; ++bi) {
        const int bz = bi >> 8, by = (bi >> 4) & 15, bx = bi & 15;
        DecItem &it = items[bi];
        memset(&it, 0, sizeof it);
        it.dst = dptr(d_chunk_out + (size_t)(bz * 16) * 65536 + (by * 16) * 256 + bx * 16);
        it.sz = 65536;
        it.sy = 256;
        it.clip_lo = kClipFullLo;
        it.clip_hi = kClipFullHi;
    }
}

// Items for one region of `lod` (src/mc_archive.c:984-1042): every touched
// block contributes its intersection with the region; voxel (z,y,x) of the
// region lands at d_origin + z*sz + y*sy + x. The blocks are walked chunk by
// chunk, so each touched chunk's block index is looked up once per region
// (a box crosses up to 8 chunks, whose indexes may share a slot of the
// per-thread index cache).
bool region_items(mc_archive *a, const uint8_t *dbase, int lod, long z0, long y0, long x0, long dz, long dy,
                  long dx, uint8_t *d_origin, int64_t sz, int64_t sy, std::vector<DecItem> &items) {
    const long bz0 = z0 >> 4, by0 = y0 >> 4, bx0 = x0 >> 4;
    const long bz1 = (z0 + dz + 15) >> 4, by1 = (y0 + dy + 15) >> 4, bx1 = (x0 + dx + 15) >> 4;   // exclusive
    if (bz1 <= bz0 || by1 <= by0 || bx1 <= bx0) return true;
    items.reserve(items.size() + (size_t)((bz1 - bz0) * (by1 - by0) * (bx1 - bx0)));
    const uint64_t cur = a->cursor.load(std::memory_order_acquire);
    for (long cz = bz0 >> 4; cz <= (bz1 - 1) >> 4; ++cz)
    for (long cy = by0 >> 4; cy <= (by1 - 1) >> 4; ++cy)
    for (long cx = bx0 >> 4; cx <= (bx1 - 1) >> 4; ++cx) {
        const uint64_t co = mc_archive_chunk_offset(a, lod, (int)cz, (int)cy, (int)cx);
        int slot = 0;
        const ChunkIndex *ix = nullptr;
        if (co > kSlotZero) {
            slot = qslot(sanitize_q(chunk_q(a, co)));
            if (slot < 0) return false;
            ix = &chunk_index(a->base, co);   // nothing below rebuilds another index
        }
        for (long bz = std::max(bz0, cz * 16); bz < std::min(bz1, cz * 16 + 16); ++bz)
        for (long by = std::max(by0, cy * 16); by < std::min(by1, cy * 16 + 16); ++by)
        for (long bx = std::max(bx0, cx * 16); bx < std::min(bx1, cx * 16 + 16); ++bx) {
            const long gz = bz * 16, gy = by * 16, gx = bx * 16;
            const long iz0 = std::max(gz, z0), iz1 = std::min(gz + 16, z0 + dz);
            const long iy0 = std::max(gy, y0), iy1 = std::min(gy + 16, y0 + dy);
            const long ix0 = std::max(gx, x0), ix1 = std::min(gx + 16, x0 + dx);
            if (iz0 >= iz1 || iy0 >= iy1 || ix0 >= ix1) continue;
            DecItem it;
            memset(&it, 0, sizeof it);
            if (ix) {
                const int bi = (int)(((bz & 15) * 16 + (by & 15)) * 16 + (bx & 15));
                const uint64_t off = ix->off[bi];
                if (off && off + ix->len[bi] <= cur) {
                    it.src = dptr(dbase + off);
                    it.len = ix->len[bi];
                }
            }
            it.dst = dptr(d_origin + (gz - z0) * sz + (gy - y0) * sy + (gx - x0));
            it.sz = sz;
            it.sy = sy;
            it.qslot = (uint16_t)slot;
            it.clip_lo = (uint16_t)(((iz0 - gz) << 8) | ((iy0 - gy) << 4) | (ix0 - gx));
            it.clip_hi = (uint16_t)(((iz1 - 1 - gz) << 8) | ((iy1 - 1 - gy) << 4) | (ix1 - 1 - gx));
            items.push_back(it);
        }
    }
    return true;
}

bool finish(Lane &L, cudaStream_t s) { return cuda_ok(cudaStreamSynchronize(s ? s : L.stream), "sync"); }

}  // namespace

// ============================================================ plans
struct mc_b200_plan {
    mc_archive *a = nullptr;
    const uint8_t *mirror = nullptr;
    DecodeBatch batch;
    LaunchCfg cfg;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int launches = 0;
    long blocks = 0;
    uint64_t payload = 0;
};

namespace {

std::mutex g_tune_mu;
std::map<uint64_t, LaunchCfg> g_tuned;   // per (quality bit pattern, batch size class)

// Pick the launch shape of each stage by timing the real batch (entropy
// alone, then reconstruction alone), then the stage layout; cached per
// quality and batch size class. Entropy: warps per CTA and CTAs per SM (how
// many lanes decode at once, and in how many CTAs), then the queue claim run
// (entries a lane takes per counter increment). Reconstruction: CTAs per SM.
LaunchCfg autotune(DecodeBatch &B, float q, int nblocks, cudaStream_t s) {
    uint32_t qb;
    memcpy(&qb, &q, 4);
    int size_class = 0;   // batches within a factor of two share a shape
    while (size_class < 31 && (1 << (size_class + 1)) <= nblocks) ++size_class;
    const uint64_t key = (uint64_t)qb << 8 | (uint64_t)size_class;
    {
        std::lock_guard<std::mutex> g(g_tune_mu);
        auto it = g_tuned.find(key);
        if (it != g_tuned.end()) return it->second;
    }
    LaunchCfg best;
    best.split = false;
    best.ent_solo = 0;   // explicit from here on: the knob below picks it
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    // Each trial starts from a cold L2 (a write larger than the L2 first), as a
    // batch of freshly mirrored payloads would, and times the stage alone; the
    // reconstruction trials rerun on the entropy output left by the entropy
    // trials.
    DevBuf flush;
    int l2 = 0, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev);
    const size_t fbytes = std::max<size_t>((size_t)l2 * 2, 64u << 20);
    const bool do_flush = flush.ensure(fbytes);
    auto time_cfg = [&](const LaunchCfg &c, int stage) {
        decode_enqueue_stage(B, c, stage, s);   // warm
        float total = 0.0f;
        for (int r = 0; r < 3; ++r) {
            if (do_flush) cudaMemsetAsync(flush.p, r, fbytes, s);
            cudaEventRecord(e0, s);
            decode_enqueue_stage(B, c, stage, s);
            cudaEventRecord(e1, s);
            cudaEventSynchronize(e1);
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            total += ms;
        }
        return total;
    };
    // two interleaved rounds over the candidates of each knob, best time of each counts
    auto pick = [&](int n, auto set, int stage) {
        std::vector<float> t(n, 1e30f);
        for (int round = 0; round < 2; ++round)
            for (int i = 0; i < n; ++i) {
                LaunchCfg c = best;
                set(c, i);
                t[i] = std::min(t[i], time_cfg(c, stage));
            }
        int b = 0;
        for (int i = 1; i < n; ++i) if (t[i] < t[b]) b = i;
        set(best, b);
    };
    // (warps per CTA, CTAs per SM): 16 to 24 resident warps per SM; 8.8 KB of
    // contexts per warp bound it at 25
    static const int ent_shape[][2] = {{4, 4}, {4, 5}, {4, 6}, {2, 8}, {2, 10}, {2, 12}, {8, 2}, {8, 3}};
    pick(8, [](LaunchCfg &c, int i) { c.ent_warps = ent_shape[i][0]; c.ent_ctas_per_sm = ent_shape[i][1]; }, 0);
    static const int ent_claim[] = {1, 2, 4};
    pick(3, [](LaunchCfg &c, int i) { c.ent_claim = ent_claim[i]; }, 0);
    // the longest 1/64 .. 1/8 of the blocks on single-thread warps, none, or
    // all of them (the single-thread kernel)
    static const int ent_solo[] = {0, 64, 32, 16, 8, 1};
    pick(6, [](LaunchCfg &c, int i) { c.ent_solo = ent_solo[i]; }, 0);
    static const int rec_opts[] = {3, 4, 5};
    pick(3, [](LaunchCfg &c, int i) { c.rec_ctas_per_sm = rec_opts[i]; }, 1);
    // the whole decode: separate kernels, the long blocks on a second
    // stream, or both stages in one persistent kernel (two rounds, best of each)
    {
        float t[3] = {1e30f, 1e30f, 1e30f};
        for (int round = 0; round < 2; ++round)
            for (int mode = 0; mode < 3; ++mode) {
                LaunchCfg c = best;
                c.split = mode == 1;
                c.fused = mode == 2;
                if (c.fused && fused_grid(c) <= 0) continue;
                t[mode] = std::min(t[mode], time_cfg(c, -1));
            }
        int bm = t[2] < t[0] && t[2] < t[1] ? 2 : (t[1] < t[0] ? 1 : 0);
        // MC_B200_STAGES=sequential|split|fused overrides the choice
        if (const char *f = getenv("MC_B200_STAGES")) {
            if (!strcmp(f, "sequential")) bm = 0;
            else if (!strcmp(f, "split")) bm = 1;
            else if (!strcmp(f, "fused") && t[2] < 1e30f) bm = 2;
        }
        best.split = bm == 1;
        best.fused = bm == 2;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    std::lock_guard<std::mutex> g(g_tune_mu);
    g_tuned[key] = best;
    return best;
}

// (Re)capture the plan's launches with its current configuration.
bool plan_capture(mc_b200_plan *p) {
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    p->exec = nullptr;
    p->graph = nullptr;
    cudaStream_t cs = nullptr;
    bool ok = cuda_ok(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), "stream") &&
              cuda_ok(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal), "begin capture") &&
              decode_enqueue(p->batch, p->cfg, cs);
    cudaGraph_t g = nullptr;
    if (cs) {
        cudaError_t ce = cudaStreamEndCapture(cs, &g);
        ok = ok && cuda_ok(ce, "end capture") && cuda_ok(cudaGraphInstantiate(&p->exec, g, 0), "instantiate");
        cudaStreamDestroy(cs);
    }
    p->graph = g;
    p->launches = 0;
    for (size_t si = 0; si < p->batch.subs.size(); ++si)   // two kernels a sub-batch, four when split
        p->launches += !p->cfg.fused && p->cfg.split && p->batch.split[si] ? 4 : 2;
    return ok;
}

// A plan over a finished work list: its batch laid out in HBM once, the launch
// shape autotuned (per quality and batch size), the launches captured.
mc_b200_plan *plan_build(mc_archive *a, const uint8_t *dbase, const std::vector<DecItem> &items, float q, Lane &L) {
    mc_b200_plan *p = new mc_b200_plan();
    p->a = a;
    p->mirror = dbase;
    for (const auto &it : items) {
        p->blocks++;
        p->payload += it.len;
    }
    if (!decode_prepare(p->batch, items.data(), (int)items.size(), L.stream)) { delete p; return nullptr; }
    p->cfg = autotune(p->batch, q, (int)items.size(), L.stream);
    if (!plan_capture(p)) { mc_b200_plan_free(p); return nullptr; }
    return p;
}

}  // namespace

extern "C" {

// ============================================================ runtime
int mc_b200_init(void) { return runtime() ? 0 : -1; }
int mc_b200_device(void) {
    Runtime *R = runtime();
    return R ? R->device : -1;
}
const char *mc_b200_last_error(void) { return last_error(); }
void mc_b200_clear_error(void) { clear_error(); }
int mc_b200_set_entropy_solo(int share) {
    if (share < -1) {
        set_error("set_entropy_solo: bad arguments");
        return -1;
    }
    Lane *L = lane();
    if (!L) return -1;
    L->cfg.ent_solo = share;
    return 0;
}
uint32_t mc_b200_last_bad_blocks(void) {
    Lane *L = lane();
    return L ? lane_bad_blocks(*L) : 0;
}

// ============================================================ archive decode
void mc_archive_decode_block(mc_archive *a, uint64_t co, int bz, int by, int bx, mc_u8 *dst) {
    if (!a || co <= kSlotZero || (unsigned)bz > 15 || (unsigned)by > 15 || (unsigned)bx > 15) {
        memset(dst, 0, kN3);
        return;
    }
    Lane *L = lane();
    if (!L) { memset(dst, 0, kN3); return; }
    const int slot = qslot(sanitize_q(chunk_q(a, co)));
    uint8_t *dbase = slot < 0 ? nullptr : mirror_sync(a, *L);
    if (!dbase) { memset(dst, 0, kN3); return; }
    const ChunkIndex &ix = chunk_index(a->base, co);
    const int bi = (bz * 16 + by) * 16 + bx;
    DecItem it;
    memset(&it, 0, sizeof it);
    if (ix.off[bi] && ix.off[bi] + ix.len[bi] <= a->cursor.load(std::memory_order_acquire)) {
        it.src = dptr(dbase + ix.off[bi]);
        it.len = ix.len[bi];
    }
    it.qslot = (uint16_t)slot;
    it.clip_lo = kClipFullLo;
    it.clip_hi = kClipFullHi;
    if (!decode_one_host(*L, it, dst)) memset(dst, 0, kN3);
}

void mc_archive_decode_chunk(mc_archive *a, uint64_t co, mc_u8 *out, int nthreads) {
    (void)nthreads;
    if (!a || !out) return;
    if (co <= kSlotZero) { memset(out, 0, kChunkBytes); return; }
    Lane *L = lane();
    if (!L) { memset(out, 0, kChunkBytes); return; }
    const int slot = qslot(sanitize_q(chunk_q(a, co)));
    uint8_t *dbase = slot < 0 ? nullptr : mirror_sync(a, *L);
    if (!dbase || !L->out.ensure(kChunkBytes)) { memset(out, 0, kChunkBytes); return; }
    std::vector<DecItem> items(kGrid3);
    chunk_items(a, co, dbase, slot, L->out.as<uint8_t>(), items.data());
    if (!decode_items(*L, items.data(), kGrid3) || !copy_to_host(*L, out, L->out.as<uint8_t>(), kChunkBytes))
        memset(out, 0, kChunkBytes);
}

void mc_archive_read_region(mc_archive *a, int lod, long z0, long y0, long x0, long dz, long dy, long dx,
                            mc_u8 *out, size_t sz, size_t sy, int nthreads) {
    (void)nthreads;
    if (!a || lod < 0 || lod > 7 || !out || dz <= 0 || dy <= 0 || dx <= 0) return;
    Lane *L = lane();
    if (!L) return;
    uint8_t *dbase = mirror_sync(a, *L);
    const size_t dense = (size_t)dz * dy * dx;
    if (!dbase || !L->out.ensure(dense)) return;
    std::vector<DecItem> items;
    if (!region_items(a, dbase, lod, z0, y0, x0, dz, dy, dx, L->out.as<uint8_t>(), (int64_t)dy * dx, dx, items))
        return;
    if (!decode_items(*L, items.data(), (int)items.size())) return;
    bool ok = true;
    if (sy == (size_t)dx && sz == (size_t)dy * dx) {
        copy_to_host(*L, out, L->out.as<uint8_t>(), dense);
        return;
    }
    for (long z = 0; z < dz && ok; ++z)
        ok = cuda_ok(cudaMemcpy2DAsync(out + z * sz, sy, L->out.as<uint8_t>() + (size_t)z * dy * dx, dx, dx, dy,
                                       cudaMemcpyDeviceToHost, L->stream),
                     "D2H");
    if (ok) finish(*L, nullptr);
}

void mc_archive_read_regions(mc_archive *a, int lod, const mc_box *boxes, int n, long dz, long dy, long dx,
                             mc_u8 *out, size_t batch_stride, int nthreads) {
    (void)nthreads;
    if (!a || !boxes || n <= 0 || !out) return;
    if (lod < 0 || lod > 7 || dz <= 0 || dy <= 0 || dx <= 0) return;   // each crop's read_region returns
    Lane *L = lane();
    if (!L) return;
    uint8_t *dbase = mirror_sync(a, *L);
    const size_t crop = (size_t)dz * dy * dx;
    if (!dbase || !L->out.ensure(crop * n)) return;
    std::vector<DecItem> items;
    for (int i = 0; i < n; ++i)
        if (!region_items(a, dbase, lod, boxes[i].z0, boxes[i].y0, boxes[i].x0, dz, dy, dx,
                          L->out.as<uint8_t>() + crop * i, (int64_t)dy * dx, dx, items))
            return;
    if (!decode_items(*L, items.data(), (int)items.size())) return;
    copy_to_host(*L, out, L->out.as<uint8_t>(), crop * n, crop, batch_stride);
}

// ============================================================ device-output decode
int mc_b200_archive_sync(mc_archive *a, const uint8_t **dev_base, uint64_t *len) {
    if (!a) return -1;
    Lane *L = lane();
    if (!L) return -1;
    uint8_t *d = mirror_sync(a, *L);
    if (!d || !finish(*L, nullptr)) return -1;
    if (dev_base) *dev_base = d;
    if (len) *len = a->synced;
    return 0;
}

int mc_b200_decode_chunks_dev(mc_archive *a, const uint64_t *offs, int n, mc_u8 *d_out, size_t stride, void *stream) {
    if (!a || !offs || n < 0 || !d_out) return -1;
    Lane *L = lane();
    if (!L) return -1;
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : L->stream;
    uint8_t *dbase = mirror_sync(a, *L);
    if (!dbase) return -1;
    if (s != L->stream && !cuda_ok(cudaStreamWaitEvent(s, a->mir_ev, 0), "stream wait")) return -1;
    std::vector<DecItem> items((size_t)n * kGrid3);
    for (int c = 0; c < n; ++c) {
        uint8_t *dst = d_out + (size_t)c * stride;
        if (offs[c] <= kSlotZero) { zero_chunk_items(dst, &items[(size_t)c * kGrid3]); continue; }
        int slot = qslot(sanitize_q(chunk_q(a, offs[c])));
        if (slot < 0) return -1;
        chunk_items(a, offs[c], dbase, slot, dst, &items[(size_t)c * kGrid3]);
    }
    if (!decode_items(*L, items.data(), (int)items.size(), s)) return -1;
    if (!stream && !finish(*L, nullptr)) return -1;
    return 0;
}

int mc_b200_read_regions_dev(mc_archive *a, int lod, const mc_box *boxes, int n, long dz, long dy, long dx,
                             mc_u8 *d_out, size_t batch_stride, void *stream) {
    if (!a || !boxes || n <= 0 || !d_out || lod < 0 || lod > 7 || dz <= 0 || dy <= 0 || dx <= 0) return -1;
    Lane *L = lane();
    if (!L) return -1;
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : L->stream;
    uint8_t *dbase = mirror_sync(a, *L);
    if (!dbase) return -1;
    if (s != L->stream && !cuda_ok(cudaStreamWaitEvent(s, a->mir_ev, 0), "stream wait")) return -1;
    std::vector<DecItem> items;
    // at most this many blocks per box (an unaligned box touches one more per axis)
    items.reserve((size_t)n * (size_t)((dz + 31) >> 4) * (size_t)((dy + 31) >> 4) * (size_t)((dx + 31) >> 4));
    for (int i = 0; i < n; ++i)
        if (!region_items(a, dbase, lod, boxes[i].z0, boxes[i].y0, boxes[i].x0, dz, dy, dx,
                          d_out + (size_t)i * batch_stride, (int64_t)dy * dx, dx, items))
            return -1;
    if (!decode_items(*L, items.data(), (int)items.size(), s)) return -1;
    if (!stream && !finish(*L, nullptr)) return -1;
    return 0;
}

// ============================================================ deblocking
// Gate and clamp from the quality, with the reference's float expressions
// (src/mc_codec.c:577-578), evaluated on the host.
static void deblock_params(float quality, int *beta, int *tc) {
    *beta = (int)(3.0f * quality + 6.0f);
    *tc = (int)(0.5f * quality + 1.0f);
}

int mc_b200_deblock_dev(mc_u8 *d_vol, int count, size_t vol_stride, int nz, int ny, int nx, float quality,
                        void *stream) {
    if (!d_vol || count <= 0 || nz <= 0 || ny <= 0 || nx <= 0) {
        set_error("deblock: bad arguments");
        return -1;
    }
    Lane *L = lane();
    if (!L) return -1;
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : L->stream;
    int beta, tc;
    deblock_params(quality, &beta, &tc);
    if (!cuda_ok(launch_deblock(d_vol, count, vol_stride, nz, ny, nx, beta, tc, s), "deblock launch")) return -1;
    if (!stream && !finish(*L, nullptr)) return -1;
    return 0;
}

void mc_deblock(mc_u8 *vol, int nz, int ny, int nx, float quality) {
    if (!vol || nz <= 0 || ny <= 0 || nx <= 0) return;
    Lane *L = lane();
    if (!L) return;   // no device: the volume stays as it was, the error says why
    const size_t n = (size_t)nz * ny * nx;
    if (!L->out.ensure(n)) return;
    int beta, tc;
    deblock_params(quality, &beta, &tc);
    cuda_ok(cudaMemcpyAsync(L->out.p, vol, n, cudaMemcpyHostToDevice, L->stream), "H2D") &&
        cuda_ok(launch_deblock(L->out.as<uint8_t>(), 1, n, nz, ny, nx, beta, tc, L->stream), "deblock launch") &&
        cuda_ok(cudaMemcpyAsync(vol, L->out.p, n, cudaMemcpyDeviceToHost, L->stream), "D2H") && finish(*L, nullptr);
}

// Blobs in host memory -> voxels in host memory, in groups of chunks.
// Work items of one host blob whose bytes sit at d_blob on the device: block
// payloads located through the blob's bitmap and length table
// (src/mc_archive.h:175-206), bounded by the blob; every block of a blob that
// is absent, short or malformed decodes to zeros. False only on a table error.
static bool blob_items(const uint8_t *b, uint64_t bl, const uint8_t *d_blob, DecItem *it) {
    if (!b || bl < (uint64_t)kBlobHdr) return true;
    uint16_t fml;
    memcpy(&fml, b + 12, 2);
    const uint64_t bm_off = kBlobHdr + (uint64_t)fml;
    if (bm_off + kBitmapBytes > bl) return true;
    const uint8_t *bm = b + bm_off;
    uint32_t np = 0;
    for (int i = 0; i < kBitmapBytes; ++i) np += (uint32_t)__builtin_popcount(bm[i]);
    const uint8_t *l16 = bm + kBitmapBytes;
    if (bm_off + kBitmapBytes + 2ull * np > bl) return true;
    float q;
    memcpy(&q, b, 4);
    const int slot = qslot(sanitize_q(q));
    if (slot < 0) return false;
    uint64_t pay = bm_off + kBitmapBytes + 2ull * np;
    uint32_t k = 0;
    for (int bi = 0; bi < kGrid3; ++bi) {
        it[bi].qslot = (uint16_t)slot;
        if (!((bm[bi >> 3] >> (bi & 7)) & 1)) continue;
        uint16_t l;
        memcpy(&l, l16 + 2 * k, 2);
        ++k;
        if (pay + l <= bl) {
            it[bi].src = dptr(d_blob + pay);
            it[bi].len = l;
        }
        pay += l;
    }
    return true;
}

// Host blobs in, host voxels out, as a pipeline of kBlobSlots slots over
// groups of kBlobGroup chunks: while one slot's voxels travel device->host,
// the next slots' blobs travel host->device and decode. A slot is reused once
// the event recorded after its previous group's copy-out has fired. A
// group's decode takes about its longest block's serial chain, 1.5-1.7 ms at
// q=6 whatever the group's size, so small groups with many in flight keep the
// link busy soonest: 2-chunk groups over 8 slots reached 50.5 GB/s for 64
// chunks where 8-chunk groups over 3 slots gave 49.1 (the plain device-to-host
// copy on that box: 57.2 GB/s).
int mc_b200_decode_chunk_blobs(const uint8_t *const *blobs, const uint64_t *lens, int n, mc_u8 *out,
                               size_t out_stride) {
    if (n < 0 || (n && (!blobs || !lens || !out))) return -1;
    Lane *L = lane();
    if (!L) return -1;
    // 2 chunks per group when their blobs are small: the link binds, and a
    // small first group starts it soonest (a q=6 pair is about 0.9 MB, q=3
    // about 2.0 MB). 8 when two chunks' blobs pass 4 MiB (a q=1 pair is about
    // 6.7 MB): the decode binds there and larger launches use the GPU better
    // (q=1, 64 chunks: 34.2 GB/s end to end against 28.2 with 2-chunk groups;
    // at q=3, 8-chunk groups gave 40.6 against 44.2)
    constexpr int kBlobGroupMax = 8, kBlobGroupSmall = 2;
    constexpr uint64_t kBigPairBytes = 4ull << 20;
    bool ok = true;
    for (int k = 0; k < kBlobSlots; ++k) ok = ok && blob_slot_ready(L->pipe[k]);
    uint32_t bad = 0;
    int used[kBlobSlots] = {};
    auto collect = [&](BlobSlot &S, int &u) {   // after S.done: count its cut-short blocks
        if (u && S.batch.h_status.p) bad += *S.batch.h_status.as<uint32_t>();
        u = 0;
    };
    for (int c0 = 0, gi = 0, g = 0; ok && c0 < n; c0 += g, ++gi) {
        BlobSlot &S = L->pipe[gi % kBlobSlots];
        uint64_t pair = 0;
        for (int j = c0; j < std::min(n, c0 + kBlobGroupSmall); ++j) pair += blobs[j] ? lens[j] : 0;
        g = std::min(pair > kBigPairBytes ? kBlobGroupMax : kBlobGroupSmall, n - c0);
        ok = cuda_ok(cudaEventSynchronize(S.done), "event sync");
        if (!ok) break;
        collect(S, used[gi % kBlobSlots]);
        uint64_t total = 0;
        uint64_t at[kBlobGroupMax];
        for (int j = 0; j < g; ++j) {
            at[j] = total;
            total += blobs[c0 + j] ? ((lens[c0 + j] + 15) & ~15ull) : 0;
        }
        DecodeBatch &B = S.batch;
        const size_t ni = (size_t)g * kGrid3;
        ok = S.src.ensure(total + 64) && S.out.ensure(kChunkBytes * g) && B.h_items.ensure(sizeof(DecItem) * ni) &&
             B.h_status.ensure(16);
        if (!ok) break;
        DecItem *items = B.h_items.as<DecItem>();
        for (int j = 0; j < g && ok; ++j) {
            const uint8_t *b = blobs[c0 + j];
            DecItem *it = items + (size_t)j * kGrid3;
            zero_chunk_items(S.out.as<uint8_t>() + kChunkBytes * j, it);
            if (b && lens[c0 + j] >= (uint64_t)kBlobHdr)
                ok = cuda_ok(cudaMemcpyAsync(S.src.as<uint8_t>() + at[j], b, lens[c0 + j], cudaMemcpyHostToDevice,
                                             S.stream), "H2D blob") &&
                     blob_items(b, lens[c0 + j], S.src.as<uint8_t>() + at[j], it);
        }
        // groups decode while others are in flight, so the lane-per-block
        // kernel's fewer instructions per bin count, not one group's chain
        // length: no single-thread share (measured on 64 chunks: 49.0 GB/s
        // against 45.5 with the share by block count, 43.7 with it for the
        // first group only, whose single-thread kernel holds every SM's
        // registers while the next group waits to start)
        LaunchCfg cfg = L->cfg;
        if (cfg.ent_solo < 0) cfg.ent_solo = 0;
        ok = ok && decode_prepare_staged(B, (int)ni, S.stream) && decode_enqueue(B, cfg, S.stream) &&
             cuda_ok(cudaMemcpyAsync(B.h_status.p, B.status.p, 4, cudaMemcpyDeviceToHost, S.stream), "D2H status");
        if (!ok) break;
        if (out_stride == kChunkBytes) {
            ok = cuda_ok(cudaMemcpyAsync(out + kChunkBytes * c0, S.out.p, kChunkBytes * g, cudaMemcpyDeviceToHost,
                                         S.stream), "D2H");
        } else {
            for (int j = 0; j < g && ok; ++j)
                ok = cuda_ok(cudaMemcpyAsync(out + out_stride * (c0 + j), S.out.as<uint8_t>() + kChunkBytes * j,
                                             kChunkBytes, cudaMemcpyDeviceToHost, S.stream), "D2H");
        }
        ok = ok && cuda_ok(cudaEventRecord(S.done, S.stream), "event record");
        used[gi % kBlobSlots] = 1;
    }
    for (int k = 0; k < kBlobSlots; ++k) {   // drain every slot, also after an error
        if (L->pipe[k].stream && cuda_ok(cudaStreamSynchronize(L->pipe[k].stream), "sync")) collect(L->pipe[k], used[k]);
        else ok = false;
    }
    // the lane's status word reports the cut-short blocks of this call (mc_b200_last_bad_blocks)
    if (ok && L->batch.status.ensure(16))
        ok = cuda_ok(cudaMemcpy(L->batch.status.p, &bad, 4, cudaMemcpyHostToDevice), "status");
    return ok ? 0 : -1;
}

// ============================================================ plans
mc_b200_plan *mc_b200_plan_decode_chunks(mc_archive *a, const uint64_t *offs, int n, mc_u8 *d_out, size_t stride) {
    if (!a || !offs || n <= 0 || !d_out) return nullptr;
    Lane *L = lane();
    if (!L) return nullptr;
    uint8_t *dbase = mirror_sync(a, *L);
    if (!dbase || !finish(*L, nullptr)) return nullptr;
    std::vector<DecItem> items((size_t)n * kGrid3);
    float q_major = 6.0f;
    for (int c = 0; c < n; ++c) {
        uint8_t *dst = d_out + (size_t)c * stride;
        if (offs[c] <= kSlotZero) { zero_chunk_items(dst, &items[(size_t)c * kGrid3]); continue; }
        float q = sanitize_q(chunk_q(a, offs[c]));
        q_major = q;
        int slot = qslot(q);
        if (slot < 0) return nullptr;
        chunk_items(a, offs[c], dbase, slot, dst, &items[(size_t)c * kGrid3]);
    }
    return plan_build(a, dbase, items, q_major, *L);
}

mc_b200_plan *mc_b200_plan_read_regions(mc_archive *a, int lod, const mc_box *boxes, int n, long dz, long dy,
                                        long dx, mc_u8 *d_out, size_t batch_stride) {
    if (!a || !boxes || n <= 0 || !d_out || lod < 0 || lod > 7 || dz <= 0 || dy <= 0 || dx <= 0) return nullptr;
    Lane *L = lane();
    if (!L) return nullptr;
    uint8_t *dbase = mirror_sync(a, *L);
    if (!dbase || !finish(*L, nullptr)) return nullptr;
    std::vector<DecItem> items;
    for (int i = 0; i < n; ++i)
        if (!region_items(a, dbase, lod, boxes[i].z0, boxes[i].y0, boxes[i].x0, dz, dy, dx,
                          d_out + (size_t)i * batch_stride, (int64_t)dy * dx, dx, items))
            return nullptr;
    if (items.empty()) return nullptr;
    // the quality the most blocks are coded at picks the tuned shape
    std::map<uint16_t, size_t> per_slot;
    for (const auto &it : items) per_slot[it.qslot] += it.len != 0;
    uint16_t major = items[0].qslot;
    for (const auto &kv : per_slot) if (kv.second > per_slot[major]) major = kv.first;
    return plan_build(a, dbase, items, slot_quality(major), *L);
}

int mc_b200_plan_launch(mc_b200_plan *p, void *stream) {
    if (!p || !p->exec) return -1;
    if (p->a->d_base != p->mirror) {
        set_error("decode plan is stale: the archive's device mirror moved since the plan was built");
        return -1;
    }
    return cuda_ok(cudaGraphLaunch(p->exec, static_cast<cudaStream_t>(stream)), "graph launch") ? 0 : -1;
}

int mc_b200_plan_launch_stage(mc_b200_plan *p, int stage, void *stream) {
    if (!p || stage < 0 || stage > 1) return -1;
    if (p->a->d_base != p->mirror) {
        set_error("decode plan is stale: the archive's device mirror moved since the plan was built");
        return -1;
    }
    return decode_enqueue_stage(p->batch, p->cfg, stage, static_cast<cudaStream_t>(stream)) ? 0 : -1;
}

void mc_b200_plan_info(const mc_b200_plan *p, int *launches, long *blocks, uint64_t *payload_bytes) {
    if (launches) *launches = p ? p->launches : 0;
    if (blocks) *blocks = p ? p->blocks : 0;
    if (payload_bytes) *payload_bytes = p ? p->payload : 0;
}

void mc_b200_plan_config(const mc_b200_plan *p, int out[3]) {
    if (!out) return;
    out[0] = p ? p->cfg.ent_ctas_per_sm : 0;
    out[1] = p ? p->cfg.rec_ctas_per_sm : 0;
    out[2] = p ? (p->cfg.fused ? 2 : (int)p->cfg.split) : 0;
}

int mc_b200_plan_set_config(mc_b200_plan *p, const int cfg[3]) {
    if (!p || !cfg || cfg[0] < 1 || cfg[0] > 16 || cfg[1] < 1 || cfg[1] > 16 || cfg[2] < 0 || cfg[2] > 2) {
        set_error("plan_set_config: bad arguments");
        return -1;
    }
    LaunchCfg c = p->cfg;
    c.ent_ctas_per_sm = cfg[0];
    c.rec_ctas_per_sm = cfg[1];
    c.split = cfg[2] == 1;
    c.fused = cfg[2] == 2;
    if (c.fused && fused_grid(c) <= 0) {
        set_error("plan_set_config: the fused kernel cannot launch on this device");
        return -1;
    }
    p->cfg = c;
    return plan_capture(p) ? 0 : -1;
}

void mc_b200_plan_tuning(const mc_b200_plan *p, int out[6]) {
    if (!out) return;
    out[0] = p ? p->cfg.ent_warps : 0;
    out[1] = p ? p->cfg.ent_ctas_per_sm : 0;
    out[2] = p ? p->cfg.ent_claim : 0;
    out[3] = p ? p->cfg.rec_ctas_per_sm : 0;
    out[4] = p ? (p->cfg.fused ? 2 : (int)p->cfg.split) : 0;
    out[5] = p ? p->cfg.ent_solo : 0;
}

int mc_b200_plan_set_tuning(mc_b200_plan *p, const int cfg[6]) {
    if (!p || !cfg || (cfg[0] != 2 && cfg[0] != 4 && cfg[0] != 8) || cfg[1] < 1 || cfg[0] * cfg[1] > 25 ||
        cfg[2] < 1 || cfg[2] > 64 || cfg[3] < 1 || cfg[3] > 16 || cfg[4] < 0 || cfg[4] > 2 || cfg[5] < 0) {
        set_error("plan_set_tuning: bad arguments");
        return -1;
    }
    LaunchCfg c = p->cfg;
    c.ent_warps = cfg[0];
    c.ent_ctas_per_sm = cfg[1];
    c.ent_claim = cfg[2];
    c.rec_ctas_per_sm = cfg[3];
    c.split = cfg[4] == 1;
    c.fused = cfg[4] == 2;
    c.ent_solo = cfg[5];
    if (c.fused && fused_grid(c) <= 0) {
        set_error("plan_set_tuning: the fused kernel cannot launch on this device");
        return -1;
    }
    p->cfg = c;
    return plan_capture(p) ? 0 : -1;
}

int mc_b200_plan_set_fused_wait(mc_b200_plan *p, uint32_t polls) {
    if (!p) return -1;
    p->cfg.fused_wait_polls = polls;
    return plan_capture(p) ? 0 : -1;
}

// ============================================================ device verify
long mc_b200_verify_archive_dev(const uint8_t *arc, const uint8_t *d_arc, size_t len, int verbose) {
    if (!arc || !d_arc) {
        set_error("verify: bad arguments");
        return -1;
    }
    std::vector<VerifyBlob> blobs;
    long total = 0;
    long bad = verify_walk(arc, len, blobs, &total);
    if (bad < 0) return -1;
    const int n = (int)blobs.size();
    if (n) {
        Lane *L = lane();
        if (!L) return -1;
        std::vector<VerifyItem> items((size_t)n);
        for (int i = 0; i < n; ++i) items[i] = VerifyItem{blobs[i].co, blobs[i].len, blobs[i].np, 0};
        std::vector<uint32_t> flags((size_t)n);
        if (!L->ver_items.ensure(sizeof(VerifyItem) * (size_t)n) || !L->ver_bad.ensure(sizeof(uint32_t) * (size_t)n) ||
            !cuda_ok(cudaMemcpyAsync(L->ver_items.p, items.data(), sizeof(VerifyItem) * (size_t)n,
                                     cudaMemcpyHostToDevice, L->stream), "H2D verify items") ||
            !cuda_ok(launch_verify_hash(d_arc, len, L->ver_items.as<VerifyItem>(), n, L->ver_bad.as<uint32_t>(),
                                        L->stream), "verify launch") ||
            !cuda_ok(cudaMemcpyAsync(flags.data(), L->ver_bad.p, sizeof(uint32_t) * (size_t)n, cudaMemcpyDeviceToHost,
                                     L->stream), "D2H verify flags") ||
            !finish(*L, nullptr))
            return -1;
        for (int i = 0; i < n; ++i) {
            if (!flags[i]) continue;
            bad++;
            if (verbose)
                fprintf(stderr, "mc_verify: lod %d node %d/%d/%d chunk@%llu CORRUPT\n", blobs[i].lod, blobs[i].n2,
                        blobs[i].n1, blobs[i].n0, (unsigned long long)blobs[i].co);
        }
    }
    if (verbose) fprintf(stderr, "mc_verify: %ld chunks checked, %ld corrupt\n", total, bad);
    return bad;
}

// ============================================================ LOD pyramid
int mc_b200_decimate_dev(const mc_u8 *d_src, int nz, int ny, int nx, mc_u8 *d_dst, void *stream) {
    if (!d_src || !d_dst || nz <= 0 || ny <= 0 || nx <= 0) {
        set_error("decimate: bad arguments");
        return -1;
    }
    Lane *L = lane();
    if (!L) return -1;
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : L->stream;
    if (!cuda_ok(launch_decimate(d_src, nz, ny, nx, d_dst, s), "decimate launch")) return -1;
    if (!stream && !finish(*L, nullptr)) return -1;
    return 0;
}

// The one-shot builder's pyramid (src/mc_archive.c:184-234) over a device
// volume: LOD 0 is the volume zero-padded to whole chunks; each next level is
// the 2x decimation of the previous one while any axis of the current padded
// extent is at least 256 (LOD 1 always follows LOD 0), at most 8 levels.
// Decimating the unpadded content gives the padded level's voxels, since a
// padding child is a zero child. Chunks are gathered 8 at a time; all-air
// chunks are left out, as the builder leaves them out; the rest are encoded
// and installed by the batched ctx append.
int mc_b200_append_pyramid(mc_archive *a, const mc_u8 *d_vol, int nz, int ny, int nx, float quality, int *nlods) {
    if (nlods) *nlods = 0;
    if (!a || !d_vol || nz <= 0 || ny <= 0 || nx <= 0) {
        set_error("append_pyramid: bad arguments");
        return -1;
    }
    Lane *L = lane();
    if (!L) return -1;
    constexpr int G = 8;
    auto pad = [](int n) { return (int)(((int64_t)n + 255) / 256 * 256); };
    int pd[3] = {pad(nz), pad(ny), pad(nx)};   // padded extent of the current level
    int cd[3] = {nz, ny, nx};                  // its non-padding content
    const size_t lod1 = (size_t)((nz + 1) / 2) * ((ny + 1) / 2) * ((nx + 1) / 2);
    const size_t lod2 = (size_t)((nz + 3) / 4) * ((ny + 3) / 4) * ((nx + 3) / 4);
    if (!L->pyr_stage.ensure(kChunkBytes * G) || !L->pyr_flag.ensure(sizeof(uint32_t) * G) ||
        !L->pyr_a.ensure(lod1) || !L->pyr_b.ensure(lod2 ? lod2 : 1))
        return -1;
    mc_codec_ctx *C = mc_codec_ctx_new();
    if (!C) {
        set_error("append_pyramid: out of memory");
        return -1;
    }
    mc_codec_ctx_set_quality(C, quality);
    const uint8_t *cur = d_vol;
    int done = 0, rc = 0;
    for (int lod = 0; lod < 8 && rc == 0; ++lod) {
        const int mn = std::min(pd[0], std::min(pd[1], pd[2])), mx = std::max(pd[0], std::max(pd[1], pd[2]));
        if (mn < 1 || !(mx >= 256 || lod == 0)) break;
        const int nc[3] = {(pd[0] + 255) / 256, (pd[1] + 255) / 256, (pd[2] + 255) / 256};
        const int total = nc[0] * nc[1] * nc[2];
        for (int c0 = 0; c0 < total && rc == 0; c0 += G) {
            const int g = std::min(G, total - c0);
            uint32_t flags[G] = {0};
            bool ok = cuda_ok(cudaMemsetAsync(L->pyr_flag.p, 0, sizeof(uint32_t) * G, L->stream), "memset");
            for (int j = 0; j < g && ok; ++j) {
                const int c = c0 + j, cz = c / (nc[1] * nc[2]), cy = (c / nc[2]) % nc[1], cx = c % nc[2];
                ok = cuda_ok(launch_gather_chunk(cur, cd[0], cd[1], cd[2], cz, cy, cx,
                                                 L->pyr_stage.as<uint8_t>() + kChunkBytes * j,
                                                 L->pyr_flag.as<uint32_t>() + j, L->stream),
                             "gather launch");
            }
            ok = ok && cuda_ok(cudaMemcpyAsync(flags, L->pyr_flag.p, sizeof(uint32_t) * G, cudaMemcpyDeviceToHost,
                                               L->stream), "D2H flags") &&
                 finish(*L, nullptr);
            if (!ok) { rc = -1; break; }
            std::vector<int> coords;
            std::vector<const mc_u8 *> ptrs;
            for (int j = 0; j < g; ++j) {
                if (!flags[j]) continue;   // all air: left out
                const int c = c0 + j;
                coords.insert(coords.end(), {c / (nc[1] * nc[2]), (c / nc[2]) % nc[1], c % nc[2]});
                ptrs.push_back(L->pyr_stage.as<uint8_t>() + kChunkBytes * j);
            }
            if (!ptrs.empty() &&
                mc_b200_append_chunks(a, C, lod, coords.data(), (int)ptrs.size(), ptrs.data(), 1, quality) != 0)
                rc = -1;
        }
        if (rc) break;
        done = lod + 1;
        if (mn / 2 < 1) break;
        if (mx / 2 < 256 && lod >= 1) break;
        uint8_t *next = (lod & 1) ? L->pyr_b.as<uint8_t>() : L->pyr_a.as<uint8_t>();
        if (!cuda_ok(launch_decimate(cur, cd[0], cd[1], cd[2], next, L->stream), "decimate launch")) {
            rc = -1;
            break;
        }
        cur = next;
        for (int k = 0; k < 3; ++k) {
            cd[k] = (cd[k] + 1) / 2;
            pd[k] = (pd[k] + 1) / 2;
        }
    }
    mc_codec_ctx_free(C);
    if (nlods) *nlods = done;
    return rc;
}

void mc_b200_plan_free(mc_b200_plan *p) {
    if (!p) return;
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    delete p;
}

// ============================================================ append
int mc_b200_append_chunks(mc_archive *a, mc_codec_ctx *C, int lod, const int *coords, int n,
                          const mc_u8 *const *vox, int vox_on_device, float q) {
    if (!a || lod < 0 || lod > 7 || n < 0 || (n && (!coords || !vox))) return -1;
    for (int i = 0; i < n; ++i)
        if (!vox[i]) return -1;
    Lane *L = lane();
    if (!L) return -1;
    const int G = 8;
    std::vector<float> hq(G), qq(G);
    std::vector<int> tau(G);
    std::vector<uint64_t> boff, blen;
    for (int c0 = 0; c0 < n; c0 += G) {
        const int g = std::min(G, n - c0);
        std::vector<const uint8_t *> dv(g);
        if (!vox_on_device && !L->src.ensure(kChunkBytes * g)) return -1;
        for (int j = 0; j < g; ++j) {
            if (vox_on_device) {
                dv[j] = vox[c0 + j];
            } else {
                dv[j] = L->src.as<uint8_t>() + kChunkBytes * j;
                if (!cuda_ok(cudaMemcpyAsync(const_cast<uint8_t *>(dv[j]), vox[c0 + j], kChunkBytes,
                                             cudaMemcpyHostToDevice, L->stream), "H2D voxels"))
                    return -1;
            }
            if (C) {   // caller's context: its quality and max error (src/mc_archive.c:590-601)
                hq[j] = qq[j] = C->quality;
                tau[j] = C->max_err;
            } else {   // parallel path: raw q in the header, no max error (src/mc_archive.c:864-866)
                float qv = q > 0 ? q : a->quality;
                hq[j] = qv;
                qq[j] = sanitize_q(qv);
                tau[j] = 0;
            }
        }
        if (!encode_chunks(*L, dv.data(), g, hq.data(), qq.data(), tau.data(), boff, blen)) return -1;
        uint64_t total = 0;
        for (int j = 0; j < g; ++j) total = std::max(total, boff[j] + blen[j]);
        if (!L->h_stage.ensure(total + 16)) return -1;
        if (total && !cuda_ok(cudaMemcpy(L->h_stage.p, L->blobs.p, total, cudaMemcpyDeviceToHost), "D2H blobs"))
            return -1;
        for (int j = 0; j < g; ++j) {
            const int *cc = coords + 3 * (c0 + j);
            int rc;
            if (blen[j]) rc = install_blob(a, lod, cc[0], cc[1], cc[2], L->h_stage.as<uint8_t>() + boff[j], blen[j]);
            else rc = C ? mark_zero(a, lod, cc[0], cc[1], cc[2]) : 0;   // all air
            if (rc) return rc;
        }
    }
    return 0;
}

int mc_archive_append_chunk_par(mc_archive *a, int lod, int cz, int cy, int cx, const mc_u8 vox[256 * 256 * 256],
                                float q, int nthreads) {
    (void)nthreads;
    if (!a || lod < 0 || lod > 7 || !vox) return -1;
    const int cc[3] = {cz, cy, cx};
    const mc_u8 *v = vox;
    return mc_b200_append_chunks(a, nullptr, lod, cc, 1, &v, 0, q);
}

int mc_archive_append_chunk_ctx(mc_archive *a, mc_codec_ctx *C, int lod, int cz, int cy, int cx,
                                const mc_u8 vox[256 * 256 * 256]) {
    if (!a || !C || lod < 0 || lod > 7 || !vox) return -1;
    const int cc[3] = {cz, cy, cx};
    const mc_u8 *v = vox;
    return mc_b200_append_chunks(a, C, lod, cc, 1, &v, 0, 0.0f);
}

int mc_archive_append_chunk_raw_q(mc_archive *a, int lod, int cz, int cy, int cx, const mc_u8 vox[256 * 256 * 256],
                                  float q) {
    if (!a || lod < 0 || lod > 7 || !vox) return -1;
    mc_codec_ctx C;
    mc_codec_ctx_set_quality(&C, q);   // throwaway ctx: quality only (src/mc_archive.c:602-611)
    return mc_archive_append_chunk_ctx(a, &C, lod, cz, cy, cx, vox);
}

int mc_archive_append_chunk_raw(mc_archive *a, int lod, int cz, int cy, int cx, const mc_u8 vox[256 * 256 * 256]) {
    return mc_archive_append_chunk_raw_q(a, lod, cz, cy, cx, vox, a ? a->quality : 8.0f);
}

}  // extern "C"
