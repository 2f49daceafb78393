// mcb_server.cpp -- the serving loop: block, region and chunk reads of one
// archive, batched continuously on the GPU behind a decoded-block cache in HBM.
//
// The reference serves reads through mc_cache (src/mc_cache.c): a 4 KiB slot
// arena of decoded blocks, a hash from block id to slot and S3-FIFO eviction,
// with misses decoded on the CPU one block at a time. Here the slot arena is a
// device buffer, the hash lives on the host beside the archive's node tables,
// eviction is FIFO over unpinned slots, and misses are decoded on the GPU in
// batches:
//
//   submit()  queues a request and returns a ticket;
//   worker    forms a batch from the queue head while the batch's output bytes
//             stay within the batch budget and its missing blocks find free
//             cache slots (admission by memory), decodes the batch's misses
//             straight into their cache slots (one entropy + one
//             reconstruction launch), gathers every request's blocks from the
//             cache into its output (one launch), and marks the tickets done
//             from a stream callback. Two batches are in flight at most: while
//             one runs on the GPU the next is formed from the requests that
//             arrived meanwhile.
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
constexpr uint32_t kNoSlot = 0xFFFFFFFFu;

uint64_t now_ns() {
    return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Ticket {
    int state = 0;                 // 0 pending, 1 done, -1 failed
    uint64_t t_submit = 0, t_done = 0;
};

struct SrvBatch {
    DecodeBatch dec;                          // the batch's cache misses
    std::vector<DecItem> gather;              // every requested block -> its output
    HostBuf h_gather;
    DevBuf d_gather, staging;                 // staging: outputs of host-memory requests
    std::vector<DecItem> miss;                // blocks to decode into their cache slots
    std::vector<long> tickets;
    std::vector<uint32_t> pins;               // cache slots the batch reads or fills
    struct D2H { void *dst; size_t off, bytes; };
    std::vector<D2H> d2h;
    size_t staged = 0;                        // staging bytes (host outputs)
    bool busy = false, gpu_done = false;
    uint64_t seq = 0;
    struct mc_b200_server *srv = nullptr;
};

}  // namespace

struct mc_b200_server {
    mc_archive *a = nullptr;
    bool dev_out = true;
    size_t batch_bytes = 0;
    // decoded-block cache
    uint8_t *d_cache = nullptr;
    uint32_t nslots = 0, hand = 0, npinned = 0;
    std::unordered_map<uint64_t, uint32_t> map;   // (chunk offset << 12 | block) -> slot
    std::vector<uint64_t> slot_key;
    std::vector<uint32_t> slot_pin;
    // requests
    std::mutex mu;
    std::condition_variable cv;
    std::deque<mc_b200_request> queue_req;
    std::deque<long> queue_tk;
    std::deque<Ticket> tickets;
    SrvBatch batch[2];
    uint64_t seq = 0;
    bool stop = false;
    bool head_blocked = false;   // the queue head waits for cache slots held by a batch in flight
    std::thread worker;
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

// One block of a request: where it comes from and where it goes.
struct Need {
    uint64_t key;         // 0: zeros (absent block, chunk or out of the volume)
    uint64_t pay_off;     // payload offset in the archive
    uint32_t len;
    uint16_t qslot;
    DecItem g;            // gather item (src filled in once the slot is known)
};

// The blocks of one request, in output coordinates (the same block walk as the
// region read, src/mc_archive.c:984-1042).
bool enumerate(mc_b200_server *S, const mc_b200_request &r, uint8_t *out, std::vector<Need> &need) {
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
    mc_archive *a = S->a;
    const uint64_t cur = a->cursor.load(std::memory_order_acquire);
    const long bz0 = z0 >> 4, by0 = y0 >> 4, bx0 = x0 >> 4;
    const long nbz = ((z0 + dz + 15) >> 4) - bz0, nby = ((y0 + dy + 15) >> 4) - by0, nbx = ((x0 + dx + 15) >> 4) - bx0;
    long last_cz = -1, last_cy = -1, last_cx = -1;
    uint64_t co = 0;
    int slot = 0;
    for (long w = 0; w < nbz * nby * nbx; ++w) {
        const long bz = bz0 + w / (nby * nbx), by = by0 + (w / nbx) % nby, bx = bx0 + w % nbx;
        const long gz = bz * 16, gy = by * 16, gx = bx * 16;
        const long iz0 = std::max(gz, z0), iz1 = std::min(gz + 16, z0 + dz);
        const long iy0 = std::max(gy, y0), iy1 = std::min(gy + 16, y0 + dy);
        const long ix0 = std::max(gx, x0), ix1 = std::min(gx + 16, x0 + dx);
        if (iz0 >= iz1 || iy0 >= iy1 || ix0 >= ix1) continue;
        const long cz = bz >> 4, cy = by >> 4, cx = bx >> 4;
        if (cz != last_cz || cy != last_cy || cx != last_cx) {
            co = mc_archive_chunk_offset(a, r.lod, (int)cz, (int)cy, (int)cx);
            last_cz = cz; last_cy = cy; last_cx = cx;
            if (co > kSlotZero) {
                slot = qslot(sanitize_q(chunk_q(a, co)));
                if (slot < 0) return false;
            }
        }
        Need n;
        memset(&n, 0, sizeof n);
        if (co > kSlotZero) {
            const ChunkIndex &ix = chunk_index(a->base, co);
            const int bi = (int)(((bz & 15) * 16 + (by & 15)) * 16 + (bx & 15));
            const uint64_t off = ix.off[bi];
            if (off && off + ix.len[bi] <= cur) {
                n.key = (co << 12) | (uint64_t)bi;
                n.pay_off = off;
                n.len = ix.len[bi];
                n.qslot = (uint16_t)slot;
            }
        }
        n.g.dst = (uint64_t)(uintptr_t)(out + (gz - z0) * sz + (gy - y0) * sy + (gx - x0));
        n.g.sz = sz;
        n.g.sy = sy;
        n.g.clip_lo = (uint16_t)(((iz0 - gz) << 8) | ((iy0 - gy) << 4) | (ix0 - gx));
        n.g.clip_hi = (uint16_t)(((iz1 - 1 - gz) << 8) | ((iy1 - 1 - gy) << 4) | (ix1 - 1 - gx));
        need.push_back(n);
    }
    return true;
}

// Next unpinned slot in FIFO order (the caller has checked that one exists);
// its old block, if any, leaves the cache.
uint32_t take_slot(mc_b200_server *S) {
    for (;;) {
        const uint32_t s = S->hand;
        S->hand = S->hand + 1 == S->nslots ? 0 : S->hand + 1;
        if (S->slot_pin[s]) continue;
        if (S->slot_key[s]) {
            S->map.erase(S->slot_key[s]);
            S->slot_key[s] = 0;
            S->st_evict++;
        }
        return s;
    }
}

void pin(mc_b200_server *S, SrvBatch &B, uint32_t s) {
    if (S->slot_pin[s]++ == 0) S->npinned++;
    B.pins.push_back(s);
}

// Forms a batch from the queue head (caller holds the lock). Device-side
// addresses of the archive mirror come from dbase.
// Allocates nothing on the device: buffers grow in launch(), outside the lock
// that the completion callback takes.
void form(mc_b200_server *S, SrvBatch &B, const uint8_t *dbase) {
    B.gather.clear();
    B.tickets.clear();
    B.pins.clear();
    B.d2h.clear();
    B.miss.clear();
    std::vector<DecItem> &miss = B.miss;
    std::vector<Need> need;
    size_t bytes = 0, staged = 0;
    while (!S->queue_req.empty()) {
        const mc_b200_request r = S->queue_req.front();
        const long t = S->queue_tk.front();
        const size_t nb = out_bytes(r);
        if (!B.tickets.empty() && bytes + nb > S->batch_bytes) break;
        // host outputs land in the batch's staging buffer first
        uint8_t *out = S->dev_out ? r.out : reinterpret_cast<uint8_t *>(staged);   // offset until the buffer exists
        need.clear();
        if (!enumerate(S, r, out, need)) {
            S->tickets[t].state = -1;
            S->queue_req.pop_front();
            S->queue_tk.pop_front();
            continue;
        }
        // admission: every missing block needs a free (unpinned) cache slot
        uint32_t misses = 0;
        for (auto &n : need)
            if (n.key && !S->map.count(n.key)) misses++;
        if (misses > S->nslots - S->npinned) {
            if (misses > S->nslots) {   // larger than the whole cache: refused
                S->tickets[t].state = -1;
                S->queue_req.pop_front();
                S->queue_tk.pop_front();
                continue;
            }
            if (B.tickets.empty()) S->head_blocked = true;   // wait until a batch in flight retires
            break;
        }
        for (auto &n : need) {
            S->st_blocks++;
            if (!n.key) {
                n.g.src = 0;
                S->st_zero++;
            } else {
                auto it = S->map.find(n.key);
                uint32_t s;
                if (it != S->map.end()) {
                    s = it->second;
                    S->st_hits++;
                } else {
                    s = take_slot(S);
                    S->map[n.key] = s;
                    S->slot_key[s] = n.key;
                    DecItem d;
                    memset(&d, 0, sizeof d);
                    d.src = (uint64_t)(uintptr_t)(dbase + n.pay_off);
                    d.len = n.len;
                    d.dst = (uint64_t)(uintptr_t)(S->d_cache + (size_t)s * kN3);
                    d.sz = 256;
                    d.sy = 16;
                    d.qslot = n.qslot;
                    d.clip_lo = kClipFullLo;
                    d.clip_hi = kClipFullHi;
                    miss.push_back(d);
                    S->st_miss++;
                }
                pin(S, B, s);
                n.g.src = (uint64_t)(uintptr_t)(S->d_cache + (size_t)s * kN3);
            }
            B.gather.push_back(n.g);
        }
        if (!S->dev_out) {
            B.d2h.push_back({r.out, staged, nb});
            staged += (nb + 255) & ~(size_t)255;
        }
        bytes += nb;
        B.tickets.push_back(t);
        S->queue_req.pop_front();
        S->queue_tk.pop_front();
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
    B->srv->cv.notify_all();
}

// Enqueues a formed batch on the stream: misses into their slots, gather,
// host copies, completion callback.
bool launch(mc_b200_server *S, SrvBatch &B, Lane &L) {
    cudaStream_t s = L.stream;
    const int nmiss = (int)B.miss.size();
    if (nmiss) {
        if (!B.dec.h_items.ensure(sizeof(DecItem) * nmiss)) return false;
        memcpy(B.dec.h_items.p, B.miss.data(), sizeof(DecItem) * nmiss);
        if (!decode_prepare_staged(B.dec, nmiss, s) || !decode_enqueue(B.dec, L.cfg, s)) return false;
    }
    if (!S->dev_out) {   // host outputs: destinations were offsets into the staging buffer
        if (!B.staging.ensure(std::max<size_t>(B.staged, 256))) return false;
        for (auto &g : B.gather) g.dst += (uint64_t)(uintptr_t)B.staging.p;
    }
    const size_t ng = B.gather.size();
    if (ng) {
        if (!B.h_gather.ensure(sizeof(DecItem) * ng) || !B.d_gather.ensure(sizeof(DecItem) * ng)) return false;
        memcpy(B.h_gather.p, B.gather.data(), sizeof(DecItem) * ng);
        if (!cuda_ok(cudaMemcpyAsync(B.d_gather.p, B.h_gather.p, sizeof(DecItem) * ng, cudaMemcpyHostToDevice, s),
                     "H2D gather") ||
            !cuda_ok(launch_gather(B.d_gather.as<DecItem>(), (int)ng, s), "gather launch"))
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
    for (uint32_t s : B.pins)
        if (--S->slot_pin[s] == 0) S->npinned--;
    for (long t : B.tickets)
        if (S->tickets[t].state == 0) S->tickets[t].state = 1;
    B.pins.clear();
    B.busy = false;
    B.gpu_done = false;
    S->head_blocked = false;
    S->cv.notify_all();
}

void worker_main(mc_b200_server *S) {
    Lane *L = lane();
    std::unique_lock<std::mutex> lk(S->mu);
    if (!L) {   // no usable device: refuse everything
        S->stop = true;
        while (!S->queue_tk.empty()) { S->tickets[S->queue_tk.front()].state = -1; S->queue_tk.pop_front(); S->queue_req.pop_front(); }
        S->cv.notify_all();
        return;
    }
    for (;;) {
        S->cv.wait(lk, [&] {
            bool any_busy = false, any_free = false;
            for (auto &b : S->batch) {
                if (b.busy && b.gpu_done) return true;
                any_busy |= b.busy;
                any_free |= !b.busy;
            }
            if (!S->queue_req.empty() && any_free && !S->head_blocked) return true;
            return S->stop && S->queue_req.empty() && !any_busy;
        });
        for (auto &b : S->batch)
            if (b.busy && b.gpu_done) retire(S, b);
        if (S->stop && S->queue_req.empty()) {   // closing: drain what is in flight, then leave
            bool busy = false;
            for (auto &b : S->batch) busy |= b.busy;
            if (!busy) break;
            continue;
        }
        SrvBatch *fb = nullptr;
        for (auto &b : S->batch)
            if (!b.busy) { fb = &b; break; }
        if (!fb || S->queue_req.empty()) continue;
        // the archive mirror up to date, ordered before this batch's work
        lk.unlock();
        const uint8_t *dbase = mirror_sync(S->a, *L);
        lk.lock();
        if (!dbase) {
            while (!S->queue_tk.empty()) { S->tickets[S->queue_tk.front()].state = -1; S->queue_tk.pop_front(); S->queue_req.pop_front(); }
            S->cv.notify_all();
            continue;
        }
        form(S, *fb, dbase);
        if (fb->tickets.empty()) { S->cv.notify_all(); continue; }
        fb->busy = true;
        fb->gpu_done = false;
        fb->seq = ++S->seq;
        lk.unlock();
        const bool ok = launch(S, *fb, *L);
        lk.lock();
        if (!ok) {
            cudaStreamSynchronize(L->stream);
            for (long t : fb->tickets) S->tickets[t].state = -1;
            fb->gpu_done = true;
            retire(S, *fb);
        }
    }
    // fail whatever is still queued
    while (!S->queue_tk.empty()) { S->tickets[S->queue_tk.front()].state = -1; S->queue_tk.pop_front(); S->queue_req.pop_front(); }
    S->cv.notify_all();
}

}  // namespace

extern "C" {

mc_b200_server *mc_b200_server_open(mc_archive *a, size_t cache_bytes, size_t batch_bytes, int out_on_device) {
    if (!a || cache_bytes < (size_t)kN3) return nullptr;
    if (!runtime()) return nullptr;
    mc_b200_server *S = new (std::nothrow) mc_b200_server();
    if (!S) return nullptr;
    S->a = a;
    S->dev_out = out_on_device != 0;
    S->batch_bytes = batch_bytes ? batch_bytes : ((size_t)256 << 20);
    S->nslots = (uint32_t)std::min<size_t>(cache_bytes / kN3, 0xFFFFFFF0u);
    if (!cuda_ok(cudaMalloc(&S->d_cache, (size_t)S->nslots * kN3), "cache alloc")) { delete S; return nullptr; }
    S->slot_key.assign(S->nslots, 0);
    S->slot_pin.assign(S->nslots, 0);
    S->map.reserve(std::min<size_t>(S->nslots, 1u << 22));
    S->worker = std::thread(worker_main, S);
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
    S->queue_req.push_back(*r);
    S->queue_tk.push_back(t);
    S->cv.notify_all();
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
    S->cv.wait(lk, [&] { return S->tickets[t].state != 0; });
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
        S->cv.notify_all();
    }
    if (S->worker.joinable()) S->worker.join();
    cudaDeviceSynchronize();
    if (S->d_cache) cudaFree(S->d_cache);
    delete S;
}

}  // extern "C"
