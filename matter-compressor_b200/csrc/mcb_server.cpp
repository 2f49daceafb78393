// mcb_server.cpp -- the serving loop: block, region and chunk reads of one
// archive, batched continuously on the GPU behind a decoded-block cache in HBM.
//
// The reference serves reads through mc_cache (src/mc_cache.c): a 4 KiB slot
// arena of decoded blocks, a hash from block id to slot and S3-FIFO eviction,
// with misses decoded on the CPU one block at a time. Here the slot arena is a
// device buffer, the hash lives on the host beside the archive's node tables,
// eviction follows the same S3-FIFO rules over slots no batch in flight
// holds, and misses are decoded on the GPU in batches:
//
//   submit()  queues a request and returns a ticket;
//   worker    forms a batch from a queue head while the batch's output bytes
//             stay within the batch budget and its missing blocks find free
//             cache slots (admission by memory), decodes the batch's misses
//             straight into their cache slots (one entropy + one
//             reconstruction launch), gathers every request's blocks from the
//             cache into its output (one launch), and marks the tickets done
//             from a stream callback.
//
// Requests travel in two classes, each with its own queue, its own worker
// thread, its own CUDA stream and two batches in flight at most: small requests (a block, a small
// region) on a high-priority stream, large ones (regions over 256 KiB of
// output, chunks) on a normal one. A block request therefore never waits
// behind a chunk's decode in the same batch, and the GPU runs a small batch's
// work ahead of a large batch's queued kernels. The classes share the cache:
// a batch that reads a chunk whose misses a batch of the other class is still
// decoding waits on that batch's decode event first, so a block is never read
// before it is written; slots of chunks that any batch in flight holds are
// never evicted.
//
// Results equal the plain decode paths byte for byte: a cached block is the
// block decoded by the same kernels, and an absent or out-of-range block reads
// as zeros.
#include <stdio.h>
#include <string.h>
#include <time.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/matter_compressor_b200.h"
#include "mcb_archive.h"
#include "mcb_format.h"
#include "mcb_kernels.h"
#include "mcb_runtime.h"
#include "mcb_tables.h"

using namespace mcb;

namespace {

constexpr size_t kChunkBytes = (size_t)256 * 256 * 256;
// requests with at most this many output bytes go to the small class
constexpr size_t kSmallBytes = (size_t)256 << 10;
constexpr int kClasses = 2, kBatchesPerClass = 2;

uint64_t now_ns() {
    return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Ticket {
    int state = 0;                 // 0 pending, 1 done, -1 failed
    uint64_t t_submit = 0, t_done = 0;
};

// Cache bookkeeping of one chunk blob (keyed by its archive offset): the
// cache slot of each of its blocks, mirrored in a device table the gather
// reads. kEmptySlot: not resolved yet; kZeroSlot: an absent block.
struct SrvBatch;
struct ChunkRes {
    uint64_t co = 0;
    uint32_t table = 0;
    uint32_t resolved = 0, resident = 0, pins = 0;
    uint64_t pin_seq = 0, last_use = 0;
    int qslot = -1;
    SrvBatch *dec_batch = nullptr;   // the last batch that decoded misses of this chunk
    uint64_t dec_seq = 0;            // ... and its sequence number then
    uint32_t slot[kGrid3];
};

struct SrvBatch {
    DecodeBatch dec;                          // the batch's cache misses
    std::vector<DecItem> miss;                // blocks to decode into their cache slots
    std::vector<GatherItem> gather;           // every request's chunk pieces
    std::vector<uint2> upd;                   // slot-table writes
    uint32_t nblocks = 0;
    HostBuf h_gather, h_upd;
    DevBuf d_gather, d_upd, staging;          // staging: outputs of host-memory requests
    std::vector<long> tickets;
    std::vector<ChunkRes *> pins;             // chunks the batch reads
    struct D2H { void *dst; size_t off, bytes; };
    std::vector<D2H> d2h;
    size_t staged = 0;                        // staging bytes (host outputs)
    bool busy = false, gpu_done = false;
    uint64_t seq = 0;
    int cls = 0;                              // request class (stream) of the batch
    cudaEvent_t decoded = nullptr;            // recorded once the batch's misses are in the cache
    std::atomic<uint64_t> launched{0};        // seq of the last use whose launch has returned
    // other-class batches (and their seq) whose decodes this batch reads after
    std::vector<std::pair<SrvBatch *, uint64_t>> waits;
    struct mc_b200_server *srv = nullptr;
};

}  // namespace

struct mc_b200_server {
    mc_archive *a = nullptr;
    bool dev_out = true;
    size_t batch_bytes = 0;
    // decoded-block cache: slots of 4096 bytes under S3-FIFO (see take_slot)
    uint8_t *d_cache = nullptr;
    uint32_t nslots = 0, pinned_slots = 0;
    std::vector<ChunkRes *> slot_owner;
    std::vector<uint16_t> slot_block;
    std::vector<uint32_t> free_slots;            // never used yet
    std::vector<uint8_t> slot_freq;              // reads since the slot's block entered its queue, up to 3
    std::deque<uint32_t> q_small, q_main;        // every used slot sits in one of the two
    std::deque<uint64_t> ghost;                  // keys evicted from the small queue, oldest first
    std::unordered_map<uint64_t, uint32_t> ghost_n;   // how often each key is in `ghost`
    size_t ghost_cap = 0;
    // per-chunk slot tables (device) and their owners
    uint32_t *d_tables = nullptr;
    uint32_t ntables = 0;
    std::vector<ChunkRes *> table_owner;
    std::vector<uint32_t> free_tables;
    std::unordered_map<uint64_t, ChunkRes *> chunks;
    uint64_t use_clock = 0;
    std::vector<uint2> pending_upd;   // table writes of a formed batch that admitted nothing
    // requests
    std::mutex mu;
    std::condition_variable cv[kClasses];   // a class's worker: new requests, finished batches, close
    std::condition_variable cv_done;   // callers waiting for tickets
    std::deque<mc_b200_request> queue_req[kClasses];
    std::deque<long> queue_tk[kClasses];
    std::deque<Ticket> tickets;
    SrvBatch batch[kClasses][kBatchesPerClass];
    cudaStream_t stream[kClasses] = {nullptr, nullptr};
    cudaEvent_t mirror_ev[kClasses] = {nullptr, nullptr};   // each worker's last mirror sync on its lane stream
    uint64_t seq = 0;
    bool stop = false;
    bool waiting[kClasses] = {false, false};        // a worker sleeps on its cv
    bool head_blocked[kClasses] = {false, false};   // a queue head waits for cache slots held by a batch in flight
    std::thread worker[kClasses];
    // statistics
    uint64_t st_req = 0, st_batches = 0, st_blocks = 0, st_hits = 0, st_miss = 0, st_zero = 0, st_evict = 0,
             st_bytes = 0;
};

namespace {

size_t out_bytes(const mc_b200_request &r) {
    switch (r.kind) {
    case MC_B200_REQ_BLOCK: return kN3;
    case MC_B200_REQ_CHUNK: return kChunkBytes;
    default: return (size_t)r.dz * r.dy * r.dx;
    }
}

int class_of(const mc_b200_request &r) { return out_bytes(r) <= kSmallBytes ? 0 : 1; }

// One chunk's share of a request, before cache resolution.
struct Piece {
    long cz, cy, cx;
    int lo[3], hi[3];   // voxel clip, chunk-local, inclusive
    GatherItem g;
};

// The chunk pieces of one request, in output coordinates (the block walk of
// the region read, src/mc_archive.c:984-1042, grouped by chunk).
void pieces_of(const mc_b200_request &r, uint8_t *out, std::vector<Piece> &ps) {
    long z0, y0, x0, dz, dy, dx;
    int64_t sz, sy;
    if (r.kind == MC_B200_REQ_BLOCK) {
        z0 = r.z * 16; y0 = r.y * 16; x0 = r.x * 16; dz = dy = dx = 16; sz = 256; sy = 16;
    } else if (r.kind == MC_B200_REQ_CHUNK) {
        z0 = r.z * 256; y0 = r.y * 256; x0 = r.x * 256; dz = dy = dx = 256; sz = 65536; sy = 256;
    } else {
        z0 = r.z; y0 = r.y; x0 = r.x; dz = r.dz; dy = r.dy; dx = r.dx;
        sz = r.sz ? (int64_t)r.sz : (int64_t)(dy * dx);
        sy = r.sy ? (int64_t)r.sy : (int64_t)dx;
    }
    const long c0[3] = {z0 >> 8, y0 >> 8, x0 >> 8};
    const long c1[3] = {(z0 + dz - 1) >> 8, (y0 + dy - 1) >> 8, (x0 + dx - 1) >> 8};
    const long org[3] = {z0, y0, x0}, ext[3] = {dz, dy, dx};
    for (long cz = c0[0]; cz <= c1[0]; ++cz)
        for (long cy = c0[1]; cy <= c1[1]; ++cy)
            for (long cx = c0[2]; cx <= c1[2]; ++cx) {
                Piece p;
                memset(&p, 0, sizeof p);
                p.cz = cz; p.cy = cy; p.cx = cx;
                const long cc[3] = {cz, cy, cx};
                for (int a = 0; a < 3; ++a) {
                    p.lo[a] = (int)(std::max(org[a], cc[a] * 256) - cc[a] * 256);
                    p.hi[a] = (int)(std::min(org[a] + ext[a], cc[a] * 256 + 256) - 1 - cc[a] * 256);
                }
                p.g.dst = (uint64_t)(uintptr_t)(out + (cz * 256 - z0) * sz + (cy * 256 - y0) * sy + (cx * 256 - x0));
                p.g.sz = sz;
                p.g.sy = sy;
                p.g.table = kNoTable;
                p.g.box_lo = (uint16_t)((p.lo[0] >> 4) << 8 | (p.lo[1] >> 4) << 4 | (p.lo[2] >> 4));
                p.g.box_hi = (uint16_t)((p.hi[0] >> 4) << 8 | (p.hi[1] >> 4) << 4 | (p.hi[2] >> 4));
                for (int a = 0; a < 3; ++a) { p.g.lo[a] = (uint8_t)p.lo[a]; p.g.hi[a] = (uint8_t)p.hi[a]; }
                ps.push_back(p);
            }
}

uint32_t box_blocks(const GatherItem &g) {
    return (uint32_t)(((g.box_hi >> 8) - (g.box_lo >> 8) + 1) * (((g.box_hi >> 4) & 15) - ((g.box_lo >> 4) & 15) + 1) *
                      ((g.box_hi & 15) - (g.box_lo & 15) + 1));
}

void pin_chunk(mc_b200_server *S, SrvBatch &B, ChunkRes *c) {
    if (c->pin_seq == B.seq) return;
    c->pin_seq = B.seq;
    if (c->pins++ == 0) S->pinned_slots += c->resident;
    B.pins.push_back(c);
}

void unpin_chunk(mc_b200_server *S, ChunkRes *c) {
    if (--c->pins == 0) S->pinned_slots -= c->resident;
}

void release_slot(mc_b200_server *S, uint32_t s) {
    ChunkRes *o = S->slot_owner[s];
    if (!o) return;
    const uint32_t bi = S->slot_block[s];
    // the device table keeps the stale number: the gather reads an entry only
    // after the block was resolved again, which rewrites it
    o->slot[bi] = kEmptySlot;
    o->resolved--;
    o->resident--;
    S->slot_owner[s] = nullptr;
    S->st_evict++;
}

// A block's cache key: its chunk's blob offset and its index in the chunk.
uint64_t block_key(const ChunkRes *c, uint32_t bi) { return c->co * (uint64_t)kGrid3 + bi; }

void ghost_add(mc_b200_server *S, uint64_t key) {
    if (S->ghost.size() >= S->ghost_cap && !S->ghost.empty()) {
        auto it = S->ghost_n.find(S->ghost.front());
        if (it != S->ghost_n.end() && --it->second == 0) S->ghost_n.erase(it);
        S->ghost.pop_front();
    }
    S->ghost.push_back(key);
    S->ghost_n[key]++;
}

// A slot for a missing block, under S3-FIFO (the admission and eviction of
// src/mc_cache.c:300-383, after Yang et al., SOSP 2023): a never-used slot
// if any; else, while the small queue holds more than a tenth of the slots,
// its head leaves it -- to the main queue if it was read again or a batch in
// flight holds its chunk, otherwise evicted, its key remembered in the ghost
// queue -- and else the main queue's head: kept (its read count lowered) if
// read or held, otherwise evicted. A held slot is never evicted. Once every
// slot of the main queue has been kept in a row, the small queue is worked
// whatever its length, so slots held by the batches in flight cannot keep
// the loop in the main queue. The caller has checked that an unheld slot
// exists; every pass lowers a read count or shortens the small queue, so the
// loop ends. A slot whose chunk gave up its table is free at once.
uint32_t take_slot(mc_b200_server *S) {
    if (!S->free_slots.empty()) {
        const uint32_t s = S->free_slots.back();
        S->free_slots.pop_back();
        return s;
    }
    size_t main_kept = 0;   // main-queue heads kept in a row
    for (;;) {
        const bool small = !S->q_small.empty() && (S->q_small.size() > S->nslots / 10 || S->q_main.empty() ||
                                                   main_kept >= S->q_main.size());
        std::deque<uint32_t> &q = small ? S->q_small : S->q_main;
        const uint32_t s = q.front();
        q.pop_front();
        ChunkRes *o = S->slot_owner[s];
        if (!o) return s;
        if (S->slot_freq[s] > 0 || o->pins) {
            if (small) {
                S->slot_freq[s] = 0;
            } else {
                if (S->slot_freq[s] > 0) S->slot_freq[s]--;
                ++main_kept;
            }
            S->q_main.push_back(s);
            continue;
        }
        if (small) ghost_add(S, block_key(o, S->slot_block[s]));
        release_slot(S, s);
        return s;
    }
}

// A slot just given to block bi of chunk c joins the main queue if the
// block was evicted from the small queue not long ago, else the small queue.
void admit_slot(mc_b200_server *S, uint32_t s, const ChunkRes *c, uint32_t bi) {
    S->slot_freq[s] = 0;
    if (S->ghost_n.count(block_key(c, bi))) S->q_main.push_back(s);
    else S->q_small.push_back(s);
}

// A read of a cached block.
inline void touch_slot(mc_b200_server *S, uint32_t s) {
    if (s < kZeroSlot && S->slot_freq[s] < 3) S->slot_freq[s]++;
}

// The bookkeeping of chunk co, created on first use; when every slot table is
// taken, the least recently used chunk no batch holds gives up its table and
// its slots. Null if every table belongs to a held chunk.
ChunkRes *chunk_res(mc_b200_server *S, uint64_t co) {
    auto it = S->chunks.find(co);
    if (it != S->chunks.end()) return it->second;
    if (S->free_tables.empty()) {
        ChunkRes *victim = nullptr;
        for (auto &kv : S->chunks)
            if (!kv.second->pins && (!victim || kv.second->last_use < victim->last_use)) victim = kv.second;
        if (!victim) return nullptr;
        for (uint32_t bi = 0; bi < (uint32_t)kGrid3; ++bi) {
            const uint32_t s = victim->slot[bi];
            if (s < kZeroSlot) { S->slot_owner[s] = nullptr; S->st_evict++; }
        }
        S->chunks.erase(victim->co);
        S->table_owner[victim->table] = nullptr;
        S->free_tables.push_back(victim->table);
        delete victim;
    }
    ChunkRes *c = new ChunkRes();
    c->co = co;
    c->table = S->free_tables.back();
    S->free_tables.pop_back();
    // a reused table may hold another chunk's slots on the device; each entry is
    // rewritten when its block is resolved, before any gather reads it, and
    // every entry is written at most once per batch
    for (uint32_t bi = 0; bi < (uint32_t)kGrid3; ++bi) c->slot[bi] = kEmptySlot;
    S->table_owner[c->table] = c;
    S->chunks[co] = c;
    return c;
}

// Forms a batch from the queue head (caller holds the lock). Allocates nothing
// on the device: buffers grow in launch(), outside the lock that the completion
// callback takes.
void form(mc_b200_server *S, SrvBatch &B, const uint8_t *dbase) {
    const int cls = B.cls;
    std::deque<mc_b200_request> &qr = S->queue_req[cls];
    std::deque<long> &qt = S->queue_tk[cls];
    B.gather.clear();
    B.waits.clear();
    B.miss.clear();
    B.upd.swap(S->pending_upd);   // writes left over from an empty batch go first
    S->pending_upd.clear();
    B.tickets.clear();
    B.pins.clear();
    B.d2h.clear();
    B.nblocks = 0;
    B.seq = ++S->seq;
    mc_archive *a = S->a;
    const uint64_t cur = a->cursor.load(std::memory_order_acquire);
    std::vector<Piece> ps;
    std::vector<std::pair<ChunkRes *, uint32_t>> misses;   // (chunk, block) to decode
    size_t bytes = 0, staged = 0;
    while (!qr.empty()) {
        const mc_b200_request r = qr.front();
        const long t = qt.front();
        const size_t nb = out_bytes(r);
        if (!B.tickets.empty() && bytes + nb > S->batch_bytes) break;
        // host outputs land in the batch's staging buffer (offsets until launch)
        uint8_t *out = S->dev_out ? r.out : reinterpret_cast<uint8_t *>(staged);
        ps.clear();
        pieces_of(r, out, ps);
        // resolve each piece's chunk; count the blocks that need a cache slot
        misses.clear();
        bool fail = false, no_table = false;
        uint64_t zeros = 0;
        for (auto &p : ps) {
            const uint64_t co = mc_archive_chunk_offset(a, r.lod, (int)p.cz, (int)p.cy, (int)p.cx);
            if (co <= kSlotZero) { zeros += box_blocks(p.g); continue; }   // absent or all air: zeros
            ChunkRes *c = chunk_res(S, co);
            if (!c) { no_table = true; break; }
            if (c->qslot < 0) {
                c->qslot = qslot(sanitize_q(chunk_q(a, co)));
                if (c->qslot < 0) { fail = true; break; }
            }
            pin_chunk(S, B, c);   // keeps the chunk's table and slots while the batch forms
            c->last_use = ++S->use_clock;
            // misses of this chunk still being decoded by a batch of the other class
            SrvBatch *db = c->dec_batch;
            if (db && db->busy && db->cls != cls && db->seq == c->dec_seq &&
                std::find(B.waits.begin(), B.waits.end(), std::make_pair(db, db->seq)) == B.waits.end())
                B.waits.emplace_back(db, db->seq);
            p.g.table = c->table;
            if (c->resolved == (uint32_t)kGrid3) {   // every block resolved: count the reads
                for (int bz = p.lo[0] >> 4; bz <= p.hi[0] >> 4; ++bz)
                    for (int by = p.lo[1] >> 4; by <= p.hi[1] >> 4; ++by)
                        for (int bx = p.lo[2] >> 4; bx <= p.hi[2] >> 4; ++bx)
                            touch_slot(S, c->slot[bz << 8 | by << 4 | bx]);
                continue;
            }
            const ChunkIndex &ix = chunk_index(a->base, co);
            for (int bz = p.lo[0] >> 4; bz <= p.hi[0] >> 4; ++bz)
                for (int by = p.lo[1] >> 4; by <= p.hi[1] >> 4; ++by)
                    for (int bx = p.lo[2] >> 4; bx <= p.hi[2] >> 4; ++bx) {
                        const uint32_t bi = (uint32_t)(bz << 8 | by << 4 | bx);
                        if (c->slot[bi] != kEmptySlot) {
                            touch_slot(S, c->slot[bi]);
                            continue;
                        }
                        const uint64_t off = ix.off[bi];
                        if (!off || off + ix.len[bi] > cur) {   // absent block: zeros
                            c->slot[bi] = kZeroSlot;
                            c->resolved++;
                            zeros++;
                            B.upd.push_back(make_uint2(c->table * kGrid3 + bi, kZeroSlot));
                        } else {
                            misses.emplace_back(c, bi);
                        }
                    }
        }
        if (fail || misses.size() > S->nslots) {   // cannot be served
            S->tickets[t].state = -1;
            qr.pop_front();
            qt.pop_front();
            continue;
        }
        if (no_table || misses.size() > S->nslots - S->pinned_slots) {
            bool in_flight = false;
            for (auto &cb : S->batch)
                for (auto &b : cb) in_flight |= b.busy;
            if (B.tickets.empty() && !in_flight) {
                // only this request's own chunks hold the slots it lacks, and
                // no batch will retire to free any: refuse it rather than wait
                S->tickets[t].state = -1;
                qr.pop_front();
                qt.pop_front();
                // a later request of this batch that reads one of these chunks
                // pins it afresh
                for (ChunkRes *c : B.pins) {
                    unpin_chunk(S, c);
                    c->pin_seq = 0;
                }
                B.pins.clear();
                B.waits.clear();
                continue;
            }
            if (B.tickets.empty()) S->head_blocked[cls] = true;   // wait until a batch in flight retires
            break;
        }
        for (auto &m : misses) {
            ChunkRes *c = m.first;
            const uint32_t bi = m.second;
            if (c->slot[bi] != kEmptySlot) continue;   // the same block twice in one request
            const uint32_t s = take_slot(S);
            admit_slot(S, s, c, bi);
            c->slot[bi] = s;
            c->resolved++;
            c->resident++;
            S->pinned_slots++;   // c is pinned by this batch
            S->slot_owner[s] = c;
            S->slot_block[s] = (uint16_t)bi;
            c->dec_batch = &B;
            c->dec_seq = B.seq;
            B.upd.push_back(make_uint2(c->table * kGrid3 + bi, s));
            const ChunkIndex &ix = chunk_index(a->base, c->co);
            DecItem d;
            memset(&d, 0, sizeof d);
            d.src = (uint64_t)(uintptr_t)(dbase + ix.off[bi]);
            d.len = ix.len[bi];
            d.dst = (uint64_t)(uintptr_t)(S->d_cache + (size_t)s * kN3);
            d.sz = 256;
            d.sy = 16;
            d.qslot = (uint16_t)c->qslot;
            d.clip_lo = kClipFullLo;
            d.clip_hi = kClipFullHi;
            B.miss.push_back(d);
        }
        for (auto &p : ps) {
            p.g.first = B.nblocks;
            const uint32_t n = box_blocks(p.g);
            B.nblocks += n;
            S->st_blocks += n;
            B.gather.push_back(p.g);
        }
        uint64_t nblk = 0;
        for (auto &p : ps) nblk += box_blocks(p.g);
        S->st_miss += misses.size();
        S->st_zero += zeros;
        S->st_hits += nblk - zeros - misses.size();
        if (!S->dev_out) {
            B.d2h.push_back({r.out, staged, nb});
            staged += (nb + 255) & ~(size_t)255;
        }
        bytes += nb;
        B.tickets.push_back(t);
        qr.pop_front();
        qt.pop_front();
    }
    if (B.tickets.empty()) {   // nothing admitted: let go of the chunks pinned while trying
        for (ChunkRes *c : B.pins) unpin_chunk(S, c);
        B.pins.clear();
        B.waits.clear();
        S->pending_upd.swap(B.upd);   // the device tables still need these writes
        B.upd.clear();
    }
    B.staged = staged;
    if (!B.tickets.empty()) S->st_batches++;
    S->st_req += B.tickets.size();
    S->st_bytes += bytes;
}

void CUDART_CB on_done(void *p) {
    SrvBatch *B = static_cast<SrvBatch *>(p);
    const uint64_t t = now_ns();
    std::lock_guard<std::mutex> g(B->srv->mu);
    for (long k : B->tickets) B->srv->tickets[k].t_done = t;
    B->gpu_done = true;
    B->srv->cv[B->cls].notify_one();
}

// Enqueues a formed batch on the stream: misses into their slots, gather,
// host copies, completion callback.
bool launch(mc_b200_server *S, SrvBatch &B, Lane &L) {
    cudaStream_t s = S->stream[B.cls];
    // after the archive mirror's sync and the other class's decodes it reads;
    // the other class's worker may still be enqueueing such a batch: its
    // decode event exists once that launch has returned, which takes
    // microseconds, so wait for that first
    if (!cuda_ok(cudaStreamWaitEvent(s, S->mirror_ev[B.cls], 0), "stream wait")) return false;
    for (auto &w : B.waits) {
        while (w.first->launched.load(std::memory_order_acquire) < w.second) std::this_thread::yield();
        if (!cuda_ok(cudaStreamWaitEvent(s, w.first->decoded, 0), "stream wait")) return false;
    }
    const size_t nu = B.upd.size();
    if (nu) {
        if (!B.h_upd.ensure(sizeof(uint2) * nu) || !B.d_upd.ensure(sizeof(uint2) * nu)) return false;
        memcpy(B.h_upd.p, B.upd.data(), sizeof(uint2) * nu);
        if (!cuda_ok(cudaMemcpyAsync(B.d_upd.p, B.h_upd.p, sizeof(uint2) * nu, cudaMemcpyHostToDevice, s), "H2D") ||
            !cuda_ok(launch_table_update(B.d_upd.as<uint2>(), (int)nu, S->d_tables, s), "table update"))
            return false;
    }
    const int nmiss = (int)B.miss.size();
    if (nmiss) {
        if (!B.dec.h_items.ensure(sizeof(DecItem) * nmiss)) return false;
        memcpy(B.dec.h_items.p, B.miss.data(), sizeof(DecItem) * nmiss);
        if (!decode_prepare_staged(B.dec, nmiss, s) || !decode_enqueue(B.dec, L.cfg, s)) return false;
    }
    if (!cuda_ok(cudaEventRecord(B.decoded, s), "event record")) return false;
    if (!S->dev_out) {   // host outputs: destinations were offsets into the staging buffer
        if (!B.staging.ensure(std::max<size_t>(B.staged, 256))) return false;
        for (auto &g : B.gather) g.dst += (uint64_t)(uintptr_t)B.staging.p;
    }
    const size_t ng = B.gather.size();
    if (ng) {
        if (!B.h_gather.ensure(sizeof(GatherItem) * ng) || !B.d_gather.ensure(sizeof(GatherItem) * ng)) return false;
        memcpy(B.h_gather.p, B.gather.data(), sizeof(GatherItem) * ng);
        if (!cuda_ok(cudaMemcpyAsync(B.d_gather.p, B.h_gather.p, sizeof(GatherItem) * ng, cudaMemcpyHostToDevice, s),
                     "H2D gather") ||
            !cuda_ok(launch_gather_boxes(B.d_gather.as<GatherItem>(), (int)ng, B.nblocks, S->d_tables, S->d_cache, s),
                     "gather launch"))
            return false;
    }
    for (auto &c : B.d2h)
        if (!cuda_ok(cudaMemcpyAsync(c.dst, B.staging.as<uint8_t>() + c.off, c.bytes, cudaMemcpyDeviceToHost, s),
                     "D2H"))
            return false;
    B.srv = S;
    return cuda_ok(cudaLaunchHostFunc(s, on_done, &B), "host callback");
}

void retire(mc_b200_server *S, SrvBatch &B) {   // caller holds the lock
    for (ChunkRes *c : B.pins) unpin_chunk(S, c);
    for (long t : B.tickets)
        if (S->tickets[t].state == 0) S->tickets[t].state = 1;
    B.pins.clear();
    B.busy = false;
    B.gpu_done = false;
    // slots and tables this batch held are free again: either class may go on
    for (int c = 0; c < kClasses; ++c) {
        S->head_blocked[c] = false;
        S->cv[c].notify_one();
    }
    S->cv_done.notify_all();
}

void fail_queued(mc_b200_server *S, int c) {   // caller holds the lock
    while (!S->queue_tk[c].empty()) {
        S->tickets[S->queue_tk[c].front()].state = -1;
        S->queue_tk[c].pop_front();
        S->queue_req[c].pop_front();
    }
    S->cv_done.notify_all();
}

// The worker of request class c: forms its class's batches from its queue,
// launches them on its stream and retires them. The two workers share the
// cache bookkeeping under the server's lock; each launches without it.
void worker_main(mc_b200_server *S, int c) {
    Lane *L = lane();
    std::unique_lock<std::mutex> lk(S->mu);
    if (!L) {   // no usable device: refuse everything of this class
        S->stop = true;
        fail_queued(S, c);
        return;
    }
    auto free_batch = [&]() -> SrvBatch * {
        for (auto &b : S->batch[c])
            if (!b.busy) return &b;
        return nullptr;
    };
    for (;;) {
        S->waiting[c] = true;
        S->cv[c].wait(lk, [&] {
            bool any_busy = false;
            for (auto &b : S->batch[c]) {
                if (b.busy && b.gpu_done) return true;
                any_busy |= b.busy;
            }
            if (!S->queue_req[c].empty() && !S->head_blocked[c] && free_batch()) return true;
            return S->stop && S->queue_req[c].empty() && !any_busy;
        });
        S->waiting[c] = false;
        for (auto &b : S->batch[c])
            if (b.busy && b.gpu_done) retire(S, b);
        if (S->stop && S->queue_req[c].empty()) {   // closing: drain what is in flight, then leave
            bool busy = false;
            for (auto &b : S->batch[c]) busy |= b.busy;
            if (!busy) break;
            continue;
        }
        SrvBatch *fb = free_batch();
        if (!fb || S->queue_req[c].empty() || S->head_blocked[c]) continue;
        // the archive mirror up to date, ordered before this batch's work
        lk.unlock();
        const uint8_t *dbase = mirror_sync(S->a, *L);
        const bool synced = dbase && cuda_ok(cudaEventRecord(S->mirror_ev[c], L->stream), "event record");
        lk.lock();
        if (!synced) {
            fail_queued(S, c);
            continue;
        }
        form(S, *fb, dbase);
        if (fb->tickets.empty()) { S->cv_done.notify_all(); continue; }   // refused requests
        fb->busy = true;
        fb->gpu_done = false;
        lk.unlock();
        const bool ok = launch(S, *fb, *L);
        fb->launched.store(fb->seq, std::memory_order_release);   // its decode event is recorded (or it failed)
        lk.lock();
        if (!ok) {
            cudaStreamSynchronize(S->stream[c]);
            for (long t : fb->tickets) S->tickets[t].state = -1;
            fb->gpu_done = true;
            retire(S, *fb);
        }
    }
    fail_queued(S, c);   // whatever is still queued
}

}  // namespace

// Frees a server whose worker is not running (never started or joined).
static void server_free(mc_b200_server *S) {
    for (int c = 0; c < kClasses; ++c)
        if (S->stream[c]) cudaStreamSynchronize(S->stream[c]);
    if (S->d_cache) cudaFree(S->d_cache);
    if (S->d_tables) cudaFree(S->d_tables);
    for (int c = 0; c < kClasses; ++c) {
        for (auto &b : S->batch[c])
            if (b.decoded) cudaEventDestroy(b.decoded);
        if (S->stream[c]) cudaStreamDestroy(S->stream[c]);
    }
    for (int c = 0; c < kClasses; ++c)
        if (S->mirror_ev[c]) cudaEventDestroy(S->mirror_ev[c]);
    for (auto &kv : S->chunks) delete kv.second;
    delete S;
}

extern "C" {

mc_b200_server *mc_b200_server_open(mc_archive *a, size_t cache_bytes, size_t batch_bytes, int out_on_device) {
    if (!a || cache_bytes < (size_t)kN3) return nullptr;
    if (!runtime()) return nullptr;
    mc_b200_server *S = new (std::nothrow) mc_b200_server();
    if (!S) return nullptr;
    S->a = a;
    S->dev_out = out_on_device != 0;
    S->batch_bytes = batch_bytes ? batch_bytes : ((size_t)256 << 20);
    // at least one chunk's blocks: a request whose chunks' cached blocks fill
    // the cache could otherwise never be admitted
    S->nslots = (uint32_t)std::min<size_t>(std::max<size_t>(cache_bytes / kN3, kGrid3), 0xFFFFFFF0u);
    if (!cuda_ok(cudaMalloc(&S->d_cache, (size_t)S->nslots * kN3), "cache alloc")) { server_free(S); return nullptr; }
    S->slot_owner.assign(S->nslots, nullptr);
    S->slot_block.assign(S->nslots, 0);
    S->slot_freq.assign(S->nslots, 0);
    S->free_slots.reserve(S->nslots);
    for (uint32_t t = S->nslots; t-- > 0;) S->free_slots.push_back(t);
    S->ghost_cap = std::max<size_t>(S->nslots - S->nslots / 10, 1);   // as many keys as the main queue's share
    S->ghost_n.reserve(S->ghost_cap);
    // slot tables: room for every chunk the cache could hold a block of, within reason
    S->ntables = (uint32_t)std::min<size_t>(std::max<size_t>(S->nslots, 1024), 16384);
    if (!cuda_ok(cudaMalloc(&S->d_tables, (size_t)S->ntables * kGrid3 * 4), "table alloc")) {
        server_free(S);
        return nullptr;
    }
    S->table_owner.assign(S->ntables, nullptr);
    for (uint32_t t = S->ntables; t-- > 0;) S->free_tables.push_back(t);
    // the small class on the device's highest stream priority (numerically least)
    int prio_lo = 0, prio_hi = 0;
    cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
    bool ok = cuda_ok(cudaStreamCreateWithPriority(&S->stream[0], cudaStreamNonBlocking, prio_hi), "stream") &&
              cuda_ok(cudaStreamCreateWithPriority(&S->stream[1], cudaStreamNonBlocking, prio_lo), "stream");
    for (int c = 0; c < kClasses && ok; ++c)
        ok = cuda_ok(cudaEventCreateWithFlags(&S->mirror_ev[c], cudaEventDisableTiming), "event");
    for (int c = 0; c < kClasses && ok; ++c)
        for (auto &b : S->batch[c]) {
            b.cls = c;
            ok = ok && cuda_ok(cudaEventCreateWithFlags(&b.decoded, cudaEventDisableTiming), "event");
        }
    if (!ok) {
        server_free(S);
        return nullptr;
    }
    for (int c = 0; c < kClasses; ++c) S->worker[c] = std::thread(worker_main, S, c);
    return S;
}

long mc_b200_server_submit(mc_b200_server *S, const mc_b200_request *r) {
    if (!S || !r || !r->out || r->lod < 0 || r->lod > 7) return -1;
    if (r->kind == MC_B200_REQ_REGION) {
        if (r->dz <= 0 || r->dy <= 0 || r->dx <= 0) return -1;
        if (!S->dev_out && ((r->sz && r->sz != (size_t)(r->dy * r->dx)) || (r->sy && r->sy != (size_t)r->dx)))
            return -1;   // host outputs are dense
    } else if (r->kind != MC_B200_REQ_BLOCK && r->kind != MC_B200_REQ_CHUNK) {
        return -1;
    }
    std::lock_guard<std::mutex> g(S->mu);
    if (S->stop) return -1;
    const long t = (long)S->tickets.size();
    S->tickets.emplace_back();
    S->tickets.back().t_submit = now_ns();
    const int c = class_of(*r);
    S->queue_req[c].push_back(*r);
    S->queue_tk[c].push_back(t);
    if (S->waiting[c]) S->cv[c].notify_one();
    return t;
}

int mc_b200_server_poll(mc_b200_server *S, long t) {
    if (!S || t < 0) return -1;
    std::lock_guard<std::mutex> g(S->mu);
    if ((size_t)t >= S->tickets.size()) return -1;
    return S->tickets[t].state;
}

int mc_b200_server_wait(mc_b200_server *S, long t) {
    if (!S || t < 0) return -1;
    std::unique_lock<std::mutex> lk(S->mu);
    if ((size_t)t >= S->tickets.size()) return -1;
    S->cv_done.wait(lk, [&] { return S->tickets[t].state != 0; });
    return S->tickets[t].state == 1 ? 0 : -1;
}

int mc_b200_server_ticket_times(mc_b200_server *S, long t, uint64_t *submit_ns, uint64_t *done_ns) {
    if (!S || t < 0) return -1;
    std::lock_guard<std::mutex> g(S->mu);
    if ((size_t)t >= S->tickets.size()) return -1;
    if (submit_ns) *submit_ns = S->tickets[t].t_submit;
    if (done_ns) *done_ns = S->tickets[t].t_done;
    return S->tickets[t].state;
}

int mc_b200_server_replay(mc_b200_server *S, const mc_b200_request *reqs, const uint64_t *arrival_ns, int n,
                          uint64_t *latency_ns) {
    if (!S || n < 0 || (n && (!reqs || !arrival_ns))) return -1;
    std::vector<long> tk((size_t)n);
    const uint64_t t0 = now_ns();
    for (int i = 0; i < n; ++i) {
        const uint64_t due = t0 + arrival_ns[i];
        for (uint64_t t = now_ns(); t < due; t = now_ns()) {
            if (due - t > 200000) std::this_thread::sleep_for(std::chrono::microseconds(100));
        }
        tk[i] = mc_b200_server_submit(S, &reqs[i]);
    }
    int rc = 0;
    for (int i = 0; i < n; ++i) {
        if (tk[i] < 0 || mc_b200_server_wait(S, tk[i]) != 0) { rc = -1; if (latency_ns) latency_ns[i] = 0; continue; }
        if (latency_ns) {
            uint64_t done = 0;
            mc_b200_server_ticket_times(S, tk[i], nullptr, &done);
            latency_ns[i] = done - (t0 + arrival_ns[i]);
        }
    }
    return rc;
}

void mc_b200_server_stats(mc_b200_server *S, uint64_t out[8]) {
    if (!out) return;
    if (!S) { memset(out, 0, 8 * sizeof(uint64_t)); return; }
    std::lock_guard<std::mutex> g(S->mu);
    out[0] = S->st_req; out[1] = S->st_batches; out[2] = S->st_blocks; out[3] = S->st_hits;
    out[4] = S->st_miss; out[5] = S->st_zero; out[6] = S->st_evict; out[7] = S->st_bytes;
}

void mc_b200_server_close(mc_b200_server *S) {
    if (!S) return;
    {
        std::lock_guard<std::mutex> g(S->mu);
        S->stop = true;
        for (int c = 0; c < kClasses; ++c) S->cv[c].notify_one();
    }
    for (int c = 0; c < kClasses; ++c)
        if (S->worker[c].joinable()) S->worker[c].join();
    server_free(S);
}

}  // extern "C"
