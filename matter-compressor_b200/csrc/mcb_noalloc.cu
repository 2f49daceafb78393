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
constexpr size_t kOffOffsets = 0;
constexpr size_t kOffItems = align256(kOffOffsets + 8 * (kNaMaxBlocks + 1));
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
// Host staging for the per-call uploads (static: no allocation).
uint64_t g_offsets[kNaMaxBlocks + 1];
QTab g_qtab;

// One CTA of 1024 threads: builds the work list from the payload offsets,
// the arena offsets (exclusive prefix sum of each block's entry bound) and
// clears the status words.
__global__ void __launch_bounds__(1024) k_noalloc_prepare(uint8_t *scratch, const uint8_t *payloads, int n,
                                                          uint8_t *out) {
    const uint64_t *off = reinterpret_cast<const uint64_t *>(scratch + kOffOffsets);
    DecItem *items = reinterpret_cast<DecItem *>(scratch + kOffItems);
    uint64_t *base = reinterpret_cast<uint64_t *>(scratch + kOffBase);
    uint32_t *status = reinterpret_cast<uint32_t *>(scratch + kOffStatus);
    __shared__ uint32_t s_warp[32];
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    if (tid < 4) status[tid] = 0;   // bad blocks, pool use, work counter
    uint32_t cap[4], sum = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int i = tid * 4 + j;
        cap[j] = 0;
        if (i < n) {
            const uint32_t len = (uint32_t)(off[i + 1] - off[i]);
            DecItem it;
            it.src = (uint64_t)(uintptr_t)(payloads + off[i]);
            it.dst = (uint64_t)(uintptr_t)(out + (size_t)i * kN3);
            it.sz = 256;
            it.sy = 16;
            it.len = len;
            it.qslot = 0;
            it.clip_lo = kClipFullLo;
            it.clip_hi = kClipFullHi;
            it.pad0 = 0;
            it.pad1 = 0;
            items[i] = it;
            cap[j] = entry_cap(len);
        }
        sum += cap[j];
    }
    uint32_t incl = sum;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) s_warp[w] = incl;
    __syncthreads();
    if (w == 0) {
        uint32_t v = s_warp[lane];
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, v, o);
            if (lane >= o) v += t;
        }
        s_warp[lane] = v;
    }
    __syncthreads();
    uint64_t acc = incl - sum + (w ? s_warp[w - 1] : 0);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int i = tid * 4 + j;
        if (i < n) base[i] = acc;
        acc += cap[j];
    }
}

int fail(int code, const char *msg) {
    fprintf(stderr, "mc_b200_decode_blocks_noalloc: %s\n", msg);
    return code;
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
    std::lock_guard<std::mutex> g(g_mu);
    DevSetup &ds = g_setup[dev];
    if (!ds.ready) {
        // once per device, with that device current: the scratch's device
        // address (the array's name is only a host-side stand-in) and the
        // constant tables
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return fail(-4, cudaGetErrorString(e));
        static uint16_t scan[kN3];
        static float cosm[16][16];
        table_scan(scan);
        table_cos(cosm);
        e = cudaMemcpy(static_cast<uint8_t *>(p) + kOffScan, scan, sizeof scan, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = upload_cos(cosm, nullptr);
        if (e == cudaSuccess) e = cudaStreamSynchronize(nullptr);
        if (e != cudaSuccess) return fail(-4, cudaGetErrorString(e));
        ds.scratch = static_cast<uint8_t *>(p);
        ds.ready = true;
    }
    uint8_t *sc = ds.scratch;
    memcpy(g_offsets, h_offsets, sizeof(uint64_t) * (size_t)(n + 1));
    table_qtab(sanitize_q(quality), &g_qtab);
    // pageable sources: both copies complete before cudaMemcpyAsync returns
    cudaError_t e = cudaMemcpyAsync(sc + kOffOffsets, g_offsets, sizeof(uint64_t) * (size_t)(n + 1),
                                    cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(sc + kOffQtab, &g_qtab, sizeof g_qtab, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return fail(-4, cudaGetErrorString(e));
    k_noalloc_prepare<<<1, 1024, 0, s>>>(sc, d_payloads, n, d_out);
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
    e = cudaGetLastError();
    if (e == cudaSuccess) e = launch_entropy(ep, cfg, s);
    if (e == cudaSuccess) e = launch_reconstruct(rp, cfg, s);
    if (e != cudaSuccess) return fail(-4, cudaGetErrorString(e));
    return 0;
}
