// mcb_noalloc.cu -- block decode for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc at all: code that runs inside a
// framework's memory pool or allocator hook (allocating there re-enters the
// allocator), real-time paths that forbid allocation after start-up, and
// hosts that hand the library a fixed memory budget. The regular decode path
// grows its work lists and scratch on demand; this entry point instead keeps
// every piece of scratch in one file-scope device array of fixed size, so a
// call allocates nothing, on the device or the host.
//
// The kernels are the regular ones (k_entropy, k_reconstruct); only where
// their work list, headers, coefficient arena and tables live differs.
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <mutex>

#include "../../include/matter_compressor_b200.h"
#include "mcb_format.h"
#include "mcb_kernels.h"
#include "mcb_tables.h"

namespace mcb {
namespace {

// Limits of one call.
constexpr int kNaMaxBlocks = 4096;                 // one chunk's worth of blocks
constexpr uint64_t kNaArenaEntries = 4ull << 20;    // decoded-coefficient list entries (16 MiB)
constexpr uint32_t kNaPoolEntries = 256u << 10;     // overflow pool for corrupt streams (1 MiB)

// Scratch layout (byte offsets, each 256-aligned).
constexpr size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }
constexpr size_t kOffItems = 0;
constexpr size_t kOffBase = align256(kOffItems + sizeof(DecItem) * kNaMaxBlocks);
constexpr size_t kOffHdr = align256(kOffBase + 8 * kNaMaxBlocks);
constexpr size_t kOffScan = align256(kOffHdr + sizeof(EntHdr) * kNaMaxBlocks);
constexpr size_t kOffQtab = align256(kOffScan + 2 * kN3);
constexpr size_t kOffStatus = align256(kOffQtab + sizeof(QTab));
constexpr size_t kOffPool = align256(kOffStatus + 16);
constexpr size_t kOffArena = align256(kOffPool + 4 * (size_t)kNaPoolEntries);
constexpr size_t kScratchBytes = align256(kOffArena + 4 * kNaArenaEntries);   // 17.3 MiB

// The scratch: every GPU that loads the library holds it until the process
// exits. All calls share it, so calls whose work overlaps on the GPU race.
static __device__ __align__(256) uint8_t g_noalloc_scratch[kScratchBytes];

// Per-device set-up state: the scratch's device address and whether the
// constant tables are in place on that device.
struct DevSetup {
    uint8_t *scratch = nullptr;
    bool ready = false;
};
constexpr int kMaxDevices = 64;
DevSetup g_setup[kMaxDevices];
std::mutex g_mu;

// What a call passes to the GPU: the payload lengths and the quality table
// travel by value as the kernel's parameter (copied at launch), so no host
// buffer outlives the call and concurrent calls from several host threads
// share nothing on the host. 16.8 KB, within the 32,764-byte parameter limit.
struct NaCall {
    QTab qtab;
    uint64_t start;                 // h_offsets[0]
    int n;
    uint32_t len[kNaMaxBlocks];     // payload bytes of block i
};
static_assert(sizeof(NaCall) < 32764, "kernel parameter size limit");

// One CTA of 1024 threads: writes the quality table into the scratch, builds
// the work list from the payload lengths (payload offsets and arena offsets
// are exclusive prefix sums over the blocks, the latter of each block's entry
// bound) and clears the status words.
__global__ void __launch_bounds__(1024) k_noalloc_prepare(const NaCall c, uint8_t *scratch, const uint8_t *payloads,
                                                          uint8_t *out) {
    DecItem *items = reinterpret_cast<DecItem *>(scratch + kOffItems);
    uint64_t *base = reinterpret_cast<uint64_t *>(scratch + kOffBase);
    uint32_t *status = reinterpret_cast<uint32_t *>(scratch + kOffStatus);
    __shared__ uint64_t s_warp[32][2];
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, n = c.n;
    if (tid < 4) status[tid] = 0;   // bad blocks, pool use, work counter
    {
        const uint32_t *q = reinterpret_cast<const uint32_t *>(&c.qtab);
        uint32_t *d = reinterpret_cast<uint32_t *>(scratch + kOffQtab);
        for (int i = tid; i < (int)(sizeof(QTab) / 4); i += blockDim.x) d[i] = q[i];
    }
    uint32_t cap[4];
    uint64_t csum = 0, lsum = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int i = tid * 4 + j;
        const uint32_t len = i < n ? c.len[i] : 0u;
        cap[j] = i < n ? entry_cap(len) : 0u;
        csum += cap[j];
        lsum += len;
    }
    // inclusive scans of (entry bound, payload bytes) over the threads
    uint64_t ic = csum, il = lsum;
    for (int o = 1; o < 32; o <<= 1) {
        const uint64_t vc = __shfl_up_sync(0xFFFFFFFFu, ic, o), vl = __shfl_up_sync(0xFFFFFFFFu, il, o);
        if (lane >= o) { ic += vc; il += vl; }
    }
    if (lane == 31) { s_warp[w][0] = ic; s_warp[w][1] = il; }
    __syncthreads();
    if (w == 0) {
        uint64_t vc = s_warp[lane][0], vl = s_warp[lane][1];
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t tc = __shfl_up_sync(0xFFFFFFFFu, vc, o), tl = __shfl_up_sync(0xFFFFFFFFu, vl, o);
            if (lane >= o) { vc += tc; vl += tl; }
        }
        s_warp[lane][0] = vc;
        s_warp[lane][1] = vl;
    }
    __syncthreads();
    uint64_t acc = ic - csum + (w ? s_warp[w - 1][0] : 0);
    uint64_t pos = c.start + il - lsum + (w ? s_warp[w - 1][1] : 0);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int i = tid * 4 + j;
        if (i < n) {
            DecItem it;
            it.src = (uint64_t)(uintptr_t)(payloads + pos);
            it.dst = (uint64_t)(uintptr_t)(out + (size_t)i * kN3);
            it.sz = 256;
            it.sy = 16;
            it.len = c.len[i];
            it.qslot = 0;
            it.clip_lo = kClipFullLo;
            it.clip_hi = kClipFullHi;
            it.pad0 = 0;
            it.pad1 = 0;
            items[i] = it;
            base[i] = acc;
            pos += c.len[i];
        }
        acc += cap[j];
    }
}

int fail(int code, const char *msg) {
    fprintf(stderr, "mc_b200_decode_blocks_noalloc: %s\n", msg);
    return code;
}

// The scratch's device address on device `dev` (current), set up on the
// first call there: the address lookup (the array's name is only a host-side
// stand-in) and the constant tables, synchronously. 0 or -4.
int device_scratch(int dev, uint8_t **out) {
    std::lock_guard<std::mutex> g(g_mu);
    DevSetup &ds = g_setup[dev];
    if (!ds.ready) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return fail(-4, cudaGetErrorString(e));
        static uint16_t scan[kN3];
        static float cosm[16][16];
        table_scan(scan);
        table_cos(cosm);
        e = cudaMemcpy(static_cast<uint8_t *>(p) + kOffScan, scan, sizeof scan, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = upload_decode_tables(cosm, scan, nullptr);
        if (e == cudaSuccess) e = cudaStreamSynchronize(nullptr);
        if (e != cudaSuccess) return fail(-4, cudaGetErrorString(e));
        ds.scratch = static_cast<uint8_t *>(p);
        ds.ready = true;
    }
    *out = ds.scratch;
    return 0;
}

}  // namespace
}  // namespace mcb

using namespace mcb;

extern "C" int mc_b200_decode_blocks_noalloc(const uint8_t *d_payloads, const uint64_t *h_offsets, int n,
                                             float quality, uint8_t *d_out, void *stream) {
    if (n < 0 || (n > 0 && (!d_payloads || !h_offsets || !d_out))) return fail(-1, "invalid arguments");
    if (n > kNaMaxBlocks) return fail(-2, "more than 4096 blocks in one call; split the request");
    if (n == 0) return 0;
    if ((uintptr_t)d_payloads & 7) return fail(-1, "payload buffer must be 8-byte aligned");
    uint64_t entries = 0;
    for (int i = 0; i < n; ++i) {
        if (h_offsets[i + 1] < h_offsets[i] || h_offsets[i + 1] - h_offsets[i] > 0xFFFFFFFFull)
            return fail(-1, "payload offsets must be non-decreasing");
        entries += entry_cap((uint32_t)(h_offsets[i + 1] - h_offsets[i]));
    }
    if (entries > kNaArenaEntries)
        return fail(-3, "payloads too large for the fixed scratch (sum over blocks of min(12288, 8*len+64) "
                        "must stay within 4194304); split the request");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return fail(-4, "no current CUDA device");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    uint8_t *sc = nullptr;
    const int rc = device_scratch(dev, &sc);
    if (rc) return rc;
    NaCall c;   // on the host stack; the launch copies it
    table_qtab(sanitize_q(quality), &c.qtab);
    c.start = h_offsets[0];
    c.n = n;
    for (int i = 0; i < n; ++i) c.len[i] = (uint32_t)(h_offsets[i + 1] - h_offsets[i]);
    k_noalloc_prepare<<<1, 1024, 0, s>>>(c, sc, d_payloads, d_out);
    EntParams ep;
    ep.items = reinterpret_cast<const DecItem *>(sc + kOffItems);
    ep.order = nullptr;
    ep.n = n;
    ep.ncoded = n;
    ep.base = reinterpret_cast<const uint64_t *>(sc + kOffBase);
    ep.arena = reinterpret_cast<uint32_t *>(sc + kOffArena);
    ep.hdr = reinterpret_cast<EntHdr *>(sc + kOffHdr);
    ep.pool = reinterpret_cast<uint32_t *>(sc + kOffPool);
    ep.pool_cap = kNaPoolEntries;
    ep.pool_used = reinterpret_cast<uint32_t *>(sc + kOffStatus) + 1;
    ep.qtab = reinterpret_cast<const QTab *>(sc + kOffQtab);
    ep.scan = reinterpret_cast<const uint16_t *>(sc + kOffScan);
    ep.status = reinterpret_cast<uint32_t *>(sc + kOffStatus);
    ep.counter = ep.status + 2;
    ep.claim = 1;
    RecParams rp;
    rp.items = ep.items;
    rp.idx = nullptr;
    rp.n = n;
    rp.hdr = ep.hdr;
    rp.base = ep.base;
    rp.arena = ep.arena;
    rp.pool = ep.pool;
    rp.qtab = ep.qtab;
    rp.scan = ep.scan;
    LaunchCfg cfg;
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = launch_entropy(ep, cfg, s);
    if (e == cudaSuccess) e = launch_reconstruct(rp, cfg, s);
    if (e != cudaSuccess) return fail(-4, cudaGetErrorString(e));
    return 0;
}
