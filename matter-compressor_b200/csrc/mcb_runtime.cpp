// mcb_runtime.cpp -- device runtime (see mcb_runtime.h).
#include "mcb_runtime.h"

#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <thread>

#include "mcb_tables.h"

namespace mcb {

// ------------------------------------------------------------------ errors
static thread_local std::string t_err;

bool set_error(const std::string &msg) {
    t_err = msg;
    fprintf(stderr, "matter-compressor-b200: %s\n", msg.c_str());
    return false;
}
bool cuda_ok(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return true;
    return set_error(std::string(what) + ": " + cudaGetErrorString(e));
}
const char *last_error() { return t_err.empty() ? nullptr : t_err.c_str(); }
void clear_error() { t_err.clear(); }

// ------------------------------------------------------------------ buffers
bool DevBuf::ensure(size_t n) {
    if (n <= cap) return true;
    size_t want = std::max(n, cap + cap / 2);
    void *np = nullptr;
    if (!cuda_ok(cudaMalloc(&np, want), "cudaMalloc")) return false;
    if (p) {
        cudaDeviceSynchronize();   // no kernel may still read the old buffer
        cudaFree(p);
    }
    p = np;
    cap = want;
    return true;
}
void DevBuf::release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
}
bool HostBuf::ensure(size_t n) {
    if (n <= cap) return true;
    size_t want = std::max(n, cap + cap / 2);
    void *np = nullptr;
    if (!cuda_ok(cudaMallocHost(&np, want), "cudaMallocHost")) return false;
    if (p) cudaFreeHost(p);
    p = np;
    cap = want;
    return true;
}
void HostBuf::release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
}

// ------------------------------------------------------------------ runtime
static Runtime *g_rt = nullptr;
static std::once_flag g_rt_once;
static std::string g_rt_err;

static void runtime_init() {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        g_rt_err = std::string("no CUDA device available (") + cudaGetErrorString(e) + ")";
        return;
    }
    Runtime *R = new Runtime();
    cudaGetDevice(&R->device);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, R->device) == cudaSuccess) {
        R->sms = prop.multiProcessorCount;
        if (prop.major < 10) {
            g_rt_err = std::string("device ") + prop.name + " is not sm_100 (Blackwell); kernels are built for sm_100a only";
            delete R;
            return;
        }
    }
    table_scan(R->h_scan);
    table_cos(R->h_cos);
    if (cudaMalloc(&R->d_scan, sizeof R->h_scan) != cudaSuccess ||
        cudaMalloc(&R->d_qtab, sizeof(QTab) * kMaxQSlots) != cudaSuccess ||
        cudaMemcpy(R->d_scan, R->h_scan, sizeof R->h_scan, cudaMemcpyHostToDevice) != cudaSuccess ||
        upload_decode_tables(R->h_cos, R->h_scan, 0) != cudaSuccess || upload_cos_encode(R->h_cos, 0) != cudaSuccess ||
        preload_decode_kernels() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) {
        g_rt_err = std::string("device table upload failed: ") + cudaGetErrorString(cudaGetLastError());
        delete R;
        return;
    }
    g_rt = R;
}

Runtime *runtime() {
    std::call_once(g_rt_once, runtime_init);
    if (!g_rt) set_error(g_rt_err);
    return g_rt;
}

int qslot(float q) {
    Runtime *R = runtime();
    if (!R) return -1;
    uint32_t qb;
    memcpy(&qb, &q, 4);
    const uint64_t key = ((uint64_t)qb << 32) | priors_generation();
    std::lock_guard<std::mutex> g(R->qmu);
    for (size_t i = 0; i < R->qkeys.size(); ++i)
        if (R->qkeys[i] == key) return (int)i;
    if (R->qkeys.size() >= (size_t)kMaxQSlots) {
        // every slot taken: wait for in-flight work, then start over
        cudaDeviceSynchronize();
        R->qkeys.clear();
    }
    QTab t;
    table_qtab(q, &t);
    int slot = (int)R->qkeys.size();
    if (!cuda_ok(cudaMemcpy(R->d_qtab + slot, &t, sizeof t, cudaMemcpyHostToDevice), "qtab upload")) return -1;
    R->qkeys.push_back(key);
    return slot;
}

float slot_quality(int slot) {
    Runtime *R = runtime();
    if (!R) return 6.0f;
    std::lock_guard<std::mutex> g(R->qmu);
    if (slot < 0 || (size_t)slot >= R->qkeys.size()) return 6.0f;
    const uint32_t qb = (uint32_t)(R->qkeys[slot] >> 32);
    float q;
    memcpy(&q, &qb, 4);
    return q;
}

// ------------------------------------------------------------------ lanes
Lane::~Lane() {
    for (cudaEvent_t e : bounce_ev)
        if (e) cudaEventDestroy(e);
    if (done) cudaEventDestroy(done);
    if (stream) cudaStreamDestroy(stream);
}

// ------------------------------------------------------------- host copies
// A few host threads that split large memcpys into stripes; the calling
// thread takes stripes too. One job at a time (calls from several host
// threads queue on the pool's lock).
namespace {
struct CopyPool {
    std::mutex run_mu;                 // one job at a time
    std::mutex mu;                     // guards the job's fields, gen, active, stop
    std::condition_variable cv, done_cv;
    std::vector<std::thread> workers;
    uint8_t *dst = nullptr;
    const uint8_t *src = nullptr;
    size_t n = 0, stripe = 0;
    std::atomic<size_t> next{0}, left{0};
    uint64_t gen = 0;
    int active = 0;                    // workers inside a job's stripes
    bool stop = false;

    // Stripes of the current job until none is left; the fields were read
    // under mu by the caller of work().
    void work(uint8_t *d, const uint8_t *s_, size_t bytes, size_t st) {
        for (;;) {
            const size_t off = next.fetch_add(1) * st;
            if (off >= bytes) return;
            memcpy(d + off, s_ + off, std::min(st, bytes - off));
            if (left.fetch_sub(1) == 1) {
                std::lock_guard<std::mutex> g(mu);
                done_cv.notify_all();
            }
        }
    }
    void loop() {
        uint64_t seen = 0;
        for (;;) {
            uint8_t *d;
            const uint8_t *s_;
            size_t bytes, st;
            {
                std::unique_lock<std::mutex> g(mu);
                cv.wait(g, [&] { return stop || gen != seen; });
                if (stop) return;
                seen = gen;
                ++active;
                d = dst; s_ = src; bytes = n; st = stripe;
            }
            work(d, s_, bytes, st);
            {
                std::lock_guard<std::mutex> g(mu);
                --active;
            }
            done_cv.notify_all();
        }
    }
    CopyPool() {
        const unsigned hw = std::thread::hardware_concurrency();
        const unsigned t = std::min(7u, hw > 2 ? hw / 2 : 1u);
        for (unsigned i = 0; i < t; ++i) workers.emplace_back([this] { loop(); });
    }
    ~CopyPool() {
        {
            std::lock_guard<std::mutex> g(mu);
            stop = true;
        }
        cv.notify_all();
        for (auto &w : workers) w.join();
    }
    void copy(uint8_t *d, const uint8_t *s_, size_t bytes) {
        constexpr size_t kStripe = 256u << 10;   // a 2 MiB segment still spreads over 8 threads
        if (bytes < 2 * kStripe || workers.empty()) {
            memcpy(d, s_, bytes);
            return;
        }
        std::lock_guard<std::mutex> r(run_mu);
        {
            // no worker is still inside the previous job when its counters reset
            std::unique_lock<std::mutex> g(mu);
            done_cv.wait(g, [&] { return active == 0; });
            dst = d; src = s_; n = bytes; stripe = kStripe;
            left.store((bytes + kStripe - 1) / kStripe);
            next.store(0);
            ++gen;
        }
        cv.notify_all();
        work(d, s_, bytes, kStripe);
        std::unique_lock<std::mutex> g(mu);
        done_cv.wait(g, [&] { return left.load() == 0; });
    }
};
CopyPool &copy_pool() {
    static CopyPool pool;
    return pool;
}
}  // namespace

bool copy_to_host(Lane &L, uint8_t *dst, const uint8_t *d_src, size_t n, size_t seg, size_t dst_stride) {
    if (seg == 0 || seg > n) seg = n;
    if (dst_stride == 0) dst_stride = seg;
    if (n == 0) return cuda_ok(cudaStreamSynchronize(L.stream), "sync");
    cudaPointerAttributes pa;
    const bool pinned = cudaPointerGetAttributes(&pa, dst) == cudaSuccess && pa.type == cudaMemoryTypeHost;
    cudaGetLastError();   // a pageable pointer may leave an error behind on older drivers
    constexpr size_t kPiece = 8u << 20;
    if (pinned || n <= kPiece) {
        // pinned: the link's rate directly; small: one pageable copy per segment
        bool ok = true;
        for (size_t o = 0; o < n && ok; o += seg)
            ok = cuda_ok(cudaMemcpyAsync(dst + (o / seg) * dst_stride, d_src + o, std::min(seg, n - o),
                                         cudaMemcpyDeviceToHost, L.stream), "D2H");
        return cuda_ok(cudaStreamSynchronize(L.stream), "sync") && ok;
    }
    constexpr int K = 3;
    for (int k = 0; k < K; ++k)
        if (!L.h_bounce[k].ensure(kPiece) ||
            (!L.bounce_ev[k] && !cuda_ok(cudaEventCreateWithFlags(&L.bounce_ev[k], cudaEventDisableTiming), "event")))
            return false;
    const size_t pieces = (n + kPiece - 1) / kPiece;
    auto len_of = [&](size_t i) { return std::min(kPiece, n - i * kPiece); };
    auto enqueue = [&](size_t i) {
        return cuda_ok(cudaMemcpyAsync(L.h_bounce[i % K].p, d_src + i * kPiece, len_of(i), cudaMemcpyDeviceToHost,
                                       L.stream), "D2H") &&
               cuda_ok(cudaEventRecord(L.bounce_ev[i % K], L.stream), "event record");
    };
    bool ok = true;
    for (size_t i = 0; i < std::min<size_t>(K, pieces) && ok; ++i) ok = enqueue(i);
    for (size_t j = 0; j < pieces && ok; ++j) {
        ok = cuda_ok(cudaEventSynchronize(L.bounce_ev[j % K]), "event sync");
        if (!ok) break;
        // the piece's bytes [o, o + len) of the device range, split at segment ends
        const uint8_t *b = L.h_bounce[j % K].as<uint8_t>();
        const size_t o0 = j * kPiece, o1 = o0 + len_of(j);
        for (size_t o = o0; o < o1;) {
            const size_t e = std::min(o1, (o / seg + 1) * seg);
            copy_pool().copy(dst + (o / seg) * dst_stride + o % seg, b + (o - o0), e - o);
            o = e;
        }
        if (j + K < pieces) ok = enqueue(j + K);   // buffer j % K is free again
    }
    // nothing of this call may still be in flight when it returns
    return cuda_ok(cudaStreamSynchronize(L.stream), "sync") && ok;
}

bool copy_to_device(Lane &L, uint8_t *d_dst, const uint8_t *src, size_t n) {
    constexpr size_t kPiece = 8u << 20;
    if (n <= kPiece)
        return cuda_ok(cudaMemcpyAsync(d_dst, src, n, cudaMemcpyHostToDevice, L.stream), "H2D");
    constexpr int K = 3;
    for (int k = 0; k < K; ++k)
        if (!L.h_bounce[k].ensure(kPiece) ||
            (!L.bounce_ev[k] && !cuda_ok(cudaEventCreateWithFlags(&L.bounce_ev[k], cudaEventDisableTiming), "event")))
            return false;
    const size_t pieces = (n + kPiece - 1) / kPiece;
    bool ok = true;
    for (size_t i = 0; i < pieces && ok; ++i) {
        const int k = (int)(i % K);
        const size_t len = std::min(kPiece, n - i * kPiece);
        // the buffer's previous piece (of this call or an earlier one) has left
        // it; an event never recorded counts as done
        ok = cuda_ok(cudaEventSynchronize(L.bounce_ev[k]), "event sync");
        if (!ok) break;
        copy_pool().copy(L.h_bounce[k].as<uint8_t>(), src + i * kPiece, len);
        ok = cuda_ok(cudaMemcpyAsync(d_dst + i * kPiece, L.h_bounce[k].p, len, cudaMemcpyHostToDevice, L.stream),
                     "H2D") &&
             cuda_ok(cudaEventRecord(L.bounce_ev[k], L.stream), "event record");
    }
    return ok;
}

static thread_local Lane *t_lane = nullptr;
static thread_local struct LaneOwner { ~LaneOwner() { delete t_lane; t_lane = nullptr; } } t_lane_owner;

Lane *lane() {
    if (t_lane) return t_lane;
    if (!runtime()) return nullptr;
    Lane *L = new Lane();
    if (!cuda_ok(cudaStreamCreateWithFlags(&L->stream, cudaStreamNonBlocking), "stream") ||
        !cuda_ok(cudaEventCreateWithFlags(&L->done, cudaEventDisableTiming), "event")) {
        delete L;
        return nullptr;
    }
    (void)t_lane_owner;
    t_lane = L;
    return L;
}

// ------------------------------------------------------------------ decode
// 8 GiB of entries per sub-batch: the per-block bound is 8 entries per payload
// byte, so a 64-chunk batch at q = 1 (about 1 KB per block) needs 6 GiB; a
// split would run the entropy stage once per sub-batch, each run bounded by
// its longest block's serial chain.
static constexpr uint64_t kArenaMaxEntries = 2048ull << 20;
static constexpr uint32_t kPoolEntries = 4u << 20;           // overflow pool, 16 MiB

// Splits the items into sub-batches that fit the arena, writes each item's
// arena offset (hb) and the entropy-stage order, and returns the largest
// sub-batch's entry count. The order within a sub-batch is longest payload
// first (counting sort by length), so the lanes of a warp decode blocks of
// similar size and the per-lane totals balance (longest-processing-time-first).
// Sub-batches with at least this many coded blocks split off their longest
// sixteenth (see DecodeBatch::split).
static constexpr int kSplitMin = 16384;

static uint64_t batch_layout(DecodeBatch &B, const DecItem *h_items, int n, uint64_t *hb, uint32_t *order,
                             uint32_t *recidx) {
    B.n = n;
    B.subs.clear();
    B.coded.clear();
    B.split.clear();
    uint64_t max_acc = 1;
    int i0 = 0;
    while (i0 < n) {
        uint64_t acc = 0;
        int i1 = i0;
        while (i1 < n) {
            uint64_t c = entry_cap(h_items[i1].len);
            if (i1 > i0 && acc + c > kArenaMaxEntries) break;
            hb[i1] = acc;
            acc += c;
            ++i1;
        }
        max_acc = std::max(max_acc, acc);
        B.subs.emplace_back(i0, i1);
        i0 = i1;
    }
    static thread_local std::vector<uint32_t> cnt;
    cnt.resize(65536);
    for (auto &r : B.subs) {
        std::fill(cnt.begin(), cnt.end(), 0u);
        auto key = [&](int i) { return 65535u - std::min<uint32_t>(h_items[i].len, 65535u); };
        for (int i = r.first; i < r.second; ++i) cnt[key(i)]++;
        uint32_t acc = 0;
        for (auto &c : cnt) { uint32_t t = c; c = acc; acc += t; }
        int coded = 0;
        for (int i = r.first; i < r.second; ++i) {
            order[r.first + cnt[key(i)]++] = (uint32_t)(i - r.first);
            coded += h_items[i].len > 0;
        }
        B.coded.push_back(coded);   // absent blocks sort last: the first `coded` entries have payloads
        const int k = coded >= kSplitMin ? coded / 16 : 0;
        B.split.push_back(k);
        // reconstruction lists: the split-off blocks ascending, then the rest ascending
        const int m = r.second - r.first;
        static thread_local std::vector<uint8_t> head;
        head.assign((size_t)m, 0);
        for (int j = 0; j < k; ++j) head[order[r.first + j]] = 1;
        int a = 0, b = k;
        for (int i = 0; i < m; ++i) recidx[r.first + (head[i] ? a++ : b++)] = (uint32_t)i;
    }
    return max_acc;
}

static bool batch_buffers(DecodeBatch &B, int n, uint64_t max_acc) {
    return B.order.ensure(sizeof(uint32_t) * (size_t)n) && B.rec_idx.ensure(sizeof(uint32_t) * (size_t)n) &&
           B.items.ensure(sizeof(DecItem) * (size_t)n) &&
           B.base.ensure(sizeof(uint64_t) * (size_t)n) && B.hdr.ensure(sizeof(EntHdr) * (size_t)n) &&
           B.arena.ensure(sizeof(uint32_t) * max_acc) && B.pool.ensure(sizeof(uint32_t) * kPoolEntries) &&
           B.status.ensure(16) && B.fws.ensure(sizeof(uint32_t) * fused_ws_words(n));
}

static bool batch_upload(DecodeBatch &B, const DecItem *items, const uint32_t *order, const uint64_t *hb,
                         const uint32_t *recidx, int n, cudaStream_t s) {
    return cuda_ok(cudaMemcpyAsync(B.items.p, items, sizeof(DecItem) * (size_t)n, cudaMemcpyHostToDevice, s),
                   "H2D items") &&
           cuda_ok(cudaMemcpyAsync(B.rec_idx.p, recidx, sizeof(uint32_t) * (size_t)n, cudaMemcpyHostToDevice, s),
                   "H2D rec idx") &&
           cuda_ok(cudaMemcpyAsync(B.order.p, order, sizeof(uint32_t) * (size_t)n, cudaMemcpyHostToDevice, s),
                   "H2D order") &&
           cuda_ok(cudaMemcpyAsync(B.base.p, hb, sizeof(uint64_t) * (size_t)n, cudaMemcpyHostToDevice, s),
                   "H2D base");
}

bool decode_prepare(DecodeBatch &B, const DecItem *h_items, int n, cudaStream_t s) {
    B.n = n;
    B.subs.clear();
    if (n <= 0) return true;
    std::vector<uint64_t> hb((size_t)n);
    std::vector<uint32_t> order((size_t)n), recidx((size_t)n);
    const uint64_t max_acc = batch_layout(B, h_items, n, hb.data(), order.data(), recidx.data());
    // synchronous copies: the host arrays may be pageable and short-lived
    return batch_buffers(B, n, max_acc) && batch_upload(B, h_items, order.data(), hb.data(), recidx.data(), n, s) &&
           cuda_ok(cudaStreamSynchronize(s), "sync");
}

bool decode_prepare_staged(DecodeBatch &B, int n, cudaStream_t s) {
    B.n = n;
    B.subs.clear();
    if (n <= 0) return true;
    if (!B.h_order.ensure(sizeof(uint32_t) * (size_t)n) || !B.h_base.ensure(sizeof(uint64_t) * (size_t)n) ||
        !B.h_rec.ensure(sizeof(uint32_t) * (size_t)n))
        return false;
    const DecItem *items = B.h_items.as<DecItem>();
    const uint64_t max_acc =
        batch_layout(B, items, n, B.h_base.as<uint64_t>(), B.h_order.as<uint32_t>(), B.h_rec.as<uint32_t>());
    return batch_buffers(B, n, max_acc) &&
           batch_upload(B, items, B.h_order.as<uint32_t>(), B.h_base.as<uint64_t>(), B.h_rec.as<uint32_t>(), n, s);
}

BlobSlot::~BlobSlot() {
    if (done) cudaEventDestroy(done);
    if (stream) cudaStreamDestroy(stream);
}

bool blob_slot_ready(BlobSlot &S) {
    if (S.stream) return true;
    if (!cuda_ok(cudaStreamCreateWithFlags(&S.stream, cudaStreamNonBlocking), "stream")) return false;
    return cuda_ok(cudaEventCreateWithFlags(&S.done, cudaEventDisableTiming), "event");
}

bool decode_enqueue(DecodeBatch &B, const LaunchCfg &cfg, cudaStream_t s) {
    return decode_enqueue_stage(B, cfg, -1, s);
}

DecodeBatch::~DecodeBatch() {
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (side) cudaStreamDestroy(side);
}

static bool side_stream(DecodeBatch &B) {
    if (B.side) return true;
    int least = 0, greatest = 0;
    cudaDeviceGetStreamPriorityRange(&least, &greatest);
    return cuda_ok(cudaStreamCreateWithPriority(&B.side, cudaStreamNonBlocking, greatest), "stream") &&
           cuda_ok(cudaEventCreateWithFlags(&B.ev_fork, cudaEventDisableTiming), "event") &&
           cuda_ok(cudaEventCreateWithFlags(&B.ev_join, cudaEventDisableTiming), "event");
}

bool decode_enqueue_stage(DecodeBatch &B, const LaunchCfg &cfg, int stage, cudaStream_t s) {
    Runtime *R = runtime();
    if (!R) return false;
    const bool ent = stage != 1, rec = stage != 0;
    if (ent && !cuda_ok(cudaMemsetAsync(B.status.p, 0, 16, s), "memset")) return false;
    uint32_t *status = B.status.as<uint32_t>();
    for (size_t si = 0; si < B.subs.size(); ++si) {
        const int i0 = B.subs[si].first, m = B.subs[si].second - B.subs[si].first;
        const int k = cfg.split ? B.split[si] : 0;
        if (k && !side_stream(B)) return false;
        EntParams ep;
        ep.items = B.items.as<DecItem>() + i0;
        ep.order = B.order.as<uint32_t>() + i0;
        ep.n = m;
        ep.ncoded = B.coded[si];
        ep.base = B.base.as<uint64_t>() + i0;
        ep.arena = B.arena.as<uint32_t>();
        ep.hdr = B.hdr.as<EntHdr>() + i0;
        ep.pool = B.pool.as<uint32_t>();
        ep.pool_cap = kPoolEntries;
        ep.pool_used = status + 1;
        ep.qtab = R->d_qtab;
        ep.scan = R->d_scan;
        ep.status = status;
        ep.counter = status + 2;
        ep.claim = cfg.ent_claim > 0 ? cfg.ent_claim : 1;
        RecParams rp;
        rp.items = B.items.as<DecItem>() + i0;
        rp.idx = nullptr;
        rp.n = m;
        rp.hdr = B.hdr.as<EntHdr>() + i0;
        rp.base = B.base.as<uint64_t>() + i0;
        rp.arena = B.arena.as<uint32_t>();
        rp.pool = B.pool.as<uint32_t>();
        rp.qtab = R->d_qtab;
        rp.scan = R->d_scan;
        // each sub-batch's entropy launches start their work counters at zero
        if (ent && si > 0 && !cuda_ok(cudaMemsetAsync(status + 2, 0, 8, s), "memset")) return false;
        if (cfg.fused && ent && rec) {
            // both stages in one persistent kernel
            FusedParams fp;
            fp.e = ep;
            fp.r = rp;
            fp.ws = B.fws.as<uint32_t>();
            fp.pair_cnt = fp.ws + kFusedSkip0 + kFusedMaxSkip;
            fp.rlist = fp.pair_cnt + (m + 1) / 2;
            fp.spin_limit = cfg.fused_wait_polls;
            if (!cuda_ok(cudaMemsetAsync(fp.ws, 0, sizeof(uint32_t) * fused_ws_words(m), s), "memset") ||
                !cuda_ok(launch_fused(fp, cfg, s), "fused decode launch"))
                return false;
            continue;
        }
        if (!k) {
            if (ent && !cuda_ok(launch_entropy(ep, cfg, s), "entropy launch")) return false;
            if (rec && !cuda_ok(launch_reconstruct(rp, cfg, s), "reconstruct launch")) return false;
            continue;
        }
        // fork: the longest k blocks on the side stream, the rest here
        if (!cuda_ok(cudaEventRecord(B.ev_fork, s), "event record") ||
            !cuda_ok(cudaStreamWaitEvent(B.side, B.ev_fork, 0), "stream wait"))
            return false;
        EntParams ea = ep, eb = ep;
        ea.ncoded = k;
        ea.counter = status + 3;
        eb.order = ep.order + k;
        eb.ncoded = ep.ncoded - k;
        RecParams ra = rp, rb = rp;
        ra.idx = B.rec_idx.as<uint32_t>() + i0;
        ra.n = k;
        rb.idx = ra.idx + k;
        rb.n = m - k;
        if (ent && !cuda_ok(launch_entropy(ea, cfg, B.side), "entropy launch")) return false;
        if (rec && !cuda_ok(launch_reconstruct(ra, cfg, B.side), "reconstruct launch")) return false;
        if (ent && !cuda_ok(launch_entropy(eb, cfg, s), "entropy launch")) return false;
        if (rec && !cuda_ok(launch_reconstruct(rb, cfg, s), "reconstruct launch")) return false;
        if (!cuda_ok(cudaEventRecord(B.ev_join, B.side), "event record") ||
            !cuda_ok(cudaStreamWaitEvent(s, B.ev_join, 0), "stream wait"))
            return false;
    }
    return true;
}

bool decode_items(Lane &L, const DecItem *items, int n, cudaStream_t s) {
    if (n <= 0) return true;
    if (!s) s = L.stream;
    if (!cuda_ok(cudaEventSynchronize(L.done), "event sync")) return false;
    // the items go to the lane's pinned staging (the caller's array may be
    // pageable and short-lived), then every upload is asynchronous; the
    // staging is reused only after L.done, recorded behind this batch
    DecodeBatch &B = L.batch;
    if (!B.h_items.ensure(sizeof(DecItem) * (size_t)n)) return false;
    memcpy(B.h_items.p, items, sizeof(DecItem) * (size_t)n);
    if (!decode_prepare_staged(B, n, s) || !decode_enqueue(B, L.cfg, s)) return false;
    return cuda_ok(cudaEventRecord(L.done, s), "event record");
}

bool decode_one(Lane &L, const DecItem &it) {
    Runtime *R = runtime();
    if (!R) return false;
    // the previous batch may still use the lane's status word
    if (!cuda_ok(cudaEventSynchronize(L.done), "event sync") || !L.solo.ensure(sizeof(SoloScratch)) ||
        !L.batch.status.ensure(16))
        return false;
    return cuda_ok(launch_decode_one(it, L.solo.as<SoloScratch>(), R->d_qtab, R->d_scan, L.batch.status.as<uint32_t>(),
                                     L.stream),
                   "single-block decode launch") &&
           cuda_ok(cudaEventRecord(L.done, L.stream), "event record");
}

bool decode_one_host(Lane &L, DecItem it, uint8_t *dst) {
    if (!L.h_one.ensure(kN3)) return false;
    // pinned memory is mapped into the device's address space (unified
    // addressing); the kernel's row stores cross the bus as posted writes
    // when the device cannot address it, the block goes to device memory and
    // comes back by one copy
    void *d = nullptr;
    const bool mapped = cudaHostGetDevicePointer(&d, L.h_one.p, 0) == cudaSuccess;
    if (!mapped) {
        cudaGetLastError();
        if (!L.out.ensure(kN3)) return false;
        d = L.out.p;
    }
    it.dst = (uint64_t)(uintptr_t)d;
    it.sz = 256;
    it.sy = 16;
    if (!decode_one(L, it) ||
        (!mapped && !cuda_ok(cudaMemcpyAsync(L.h_one.p, L.out.p, kN3, cudaMemcpyDeviceToHost, L.stream), "D2H")) ||
        !cuda_ok(cudaStreamSynchronize(L.stream), "sync"))
        return false;
    memcpy(dst, L.h_one.p, kN3);
    return true;
}

uint32_t lane_bad_blocks(Lane &L) {
    uint32_t v = 0;
    if (L.batch.status.p) cudaMemcpy(&v, L.batch.status.p, 4, cudaMemcpyDeviceToHost);
    return v;
}

// ------------------------------------------------------------------ encode
bool encode_chunks(Lane &L, const uint8_t *const *d_vox, int nchunks, const float *header_q, const float *q,
                   const int *tau, std::vector<uint64_t> &blob_off, std::vector<uint64_t> &blob_len) {
    Runtime *R = runtime();
    if (!R) return false;
    blob_off.assign(nchunks, 0);
    blob_len.assign(nchunks, 0);
    if (nchunks <= 0) return true;
    if (!cuda_ok(cudaEventSynchronize(L.done), "event sync")) return false;
    const size_t n = (size_t)nchunks * kGrid3;
    if (!L.h_items.ensure(sizeof(EncItem) * n) || !L.enc_items.ensure(sizeof(EncItem) * n) ||
        !L.enc_len.ensure(4 * n) || !L.enc_frac.ensure(n) || !L.enc_pay.ensure((size_t)kEncCap * n) ||
        !L.status.ensure(16) || !L.b_scratch.ensure(4 * n) || !L.b_lens16.ensure(2 * n) ||
        !L.b_bitmap.ensure((size_t)kBitmapBytes * nchunks) || !L.b_fmap.ensure((size_t)kFmapCap * nchunks) ||
        !L.b_fml.ensure(4 * nchunks) || !L.b_np.ensure(4 * nchunks) || !L.b_len.ensure(8 * nchunks) ||
        !L.b_off.ensure(8 * nchunks) || !L.b_q.ensure(4 * nchunks) || !L.h_misc.ensure(16 * (size_t)nchunks) ||
        !L.enc_lv.ensure(2 * (size_t)kN3 * n) || !L.enc_corr.ensure(4 * (size_t)kN3 * n) || !L.enc_sym.ensure(8 * n))
        return false;
    EncItem *hi = L.h_items.as<EncItem>();
    for (int c = 0; c < nchunks; ++c) {
        int slot = qslot(q[c]);
        if (slot < 0) return false;
        for (int bi = 0; bi < kGrid3; ++bi) {
            int bz = bi >> 8, by = (bi >> 4) & 15, bx = bi & 15;
            EncItem &it = hi[(size_t)c * kGrid3 + bi];
            it.src = (uint64_t)(uintptr_t)(d_vox[c] + (size_t)(bz * 16) * 65536 + (by * 16) * 256 + bx * 16);
            it.sz = 65536;
            it.sy = 256;
            it.out = (uint64_t)(uintptr_t)(L.enc_pay.as<uint8_t>() + ((size_t)c * kGrid3 + bi) * kEncCap);
            it.qslot = (uint16_t)slot;
            it.tau = (uint16_t)std::min(std::max(tau[c], 0), 65535);
            it.pad = 0;
        }
    }
    float *hq = L.h_misc.as<float>();
    memcpy(hq, header_q, 4 * (size_t)nchunks);
    if (!cuda_ok(cudaMemcpyAsync(L.enc_items.p, hi, sizeof(EncItem) * n, cudaMemcpyHostToDevice, L.stream), "H2D") ||
        !cuda_ok(cudaMemcpyAsync(L.b_q.p, hq, 4 * (size_t)nchunks, cudaMemcpyHostToDevice, L.stream), "H2D") ||
        !cuda_ok(cudaMemsetAsync(L.status.p, 0, 16, L.stream), "memset"))
        return false;
    EncParams ep;
    ep.items = L.enc_items.as<EncItem>();
    ep.n = (int)n;
    ep.qtab = R->d_qtab;
    ep.scan = R->d_scan;
    ep.len = L.enc_len.as<uint32_t>();
    ep.frac = L.enc_frac.as<uint8_t>();
    ep.status = L.status.as<uint32_t>();
    ep.levels = L.enc_lv.as<int16_t>();
    ep.corr = L.enc_corr.as<uint32_t>();
    ep.sym = L.enc_sym.as<uint2>();
    if (!cuda_ok(launch_encode(ep, L.stream), "encode launch")) return false;
    BlobParams bp;
    bp.nchunks = nchunks;
    bp.payload = L.enc_pay.as<uint8_t>();
    bp.len = L.enc_len.as<uint32_t>();
    bp.frac = L.enc_frac.as<uint8_t>();
    bp.header_q = L.b_q.as<float>();
    bp.scratch = L.b_scratch.as<uint32_t>();
    bp.lens16 = L.b_lens16.as<uint16_t>();
    bp.bitmap = L.b_bitmap.as<uint8_t>();
    bp.fmap = L.b_fmap.as<uint8_t>();
    bp.fml = L.b_fml.as<uint32_t>();
    bp.np = L.b_np.as<uint32_t>();
    bp.blob_len = L.b_len.as<uint64_t>();
    bp.blob_off = L.b_off.as<uint64_t>();
    bp.blobs = nullptr;
    if (!cuda_ok(launch_blob_layout(bp, L.stream), "blob layout launch")) return false;
    uint64_t *hl = reinterpret_cast<uint64_t *>(L.h_misc.as<uint8_t>() + 8 * (size_t)nchunks);
    uint32_t status = 0;
    if (!cuda_ok(cudaMemcpyAsync(hl, L.b_len.p, 8 * (size_t)nchunks, cudaMemcpyDeviceToHost, L.stream), "D2H") ||
        !cuda_ok(cudaMemcpyAsync(&status, L.status.p, 4, cudaMemcpyDeviceToHost, L.stream), "D2H") ||
        !cuda_ok(cudaStreamSynchronize(L.stream), "encode sync"))
        return false;
    if (status) return set_error("block payload exceeded the encoder bound");
    uint64_t total = 0;
    for (int c = 0; c < nchunks; ++c) {
        blob_len[c] = hl[c];
        blob_off[c] = total;
        total += (hl[c] + 15) & ~15ull;
    }
    uint64_t *ho = hl;   // reuse the staging for offsets
    for (int c = 0; c < nchunks; ++c) ho[c] = blob_off[c];
    if (!L.blobs.ensure(std::max<uint64_t>(total, 16))) return false;
    bp.blobs = L.blobs.as<uint8_t>();
    if (!cuda_ok(cudaMemcpyAsync(L.b_off.p, ho, 8 * (size_t)nchunks, cudaMemcpyHostToDevice, L.stream), "H2D") ||
        !cuda_ok(launch_blob_fill(bp, L.stream), "blob fill launch") ||
        !cuda_ok(launch_blob_hash(bp, L.stream), "blob hash launch") ||
        !cuda_ok(cudaStreamSynchronize(L.stream), "blob sync"))
        return false;
    return true;
}

}  // namespace mcb
