// mcb_runtime.h -- device runtime behind the C ABI: lazy CUDA initialisation,
// the per-quality table registry, per-thread streams and grow-only buffers, and
// the decode / encode pipelines that feed the kernels.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <mutex>
#include <string>
#include <vector>

#include "mcb_format.h"
#include "mcb_kernels.h"

namespace mcb {

// Records the last error of the calling thread; returns false for chaining.
bool set_error(const std::string &msg);
bool cuda_ok(cudaError_t e, const char *what);
const char *last_error();
void clear_error();

// Grow-only device buffer.
struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
    bool ensure(size_t n);
    void release();
    template <class T> T *as() const { return static_cast<T *>(p); }
    ~DevBuf() { release(); }
};
// Grow-only pinned host buffer.
struct HostBuf {
    void *p = nullptr;
    size_t cap = 0;
    bool ensure(size_t n);
    void release();
    template <class T> T *as() const { return static_cast<T *>(p); }
    ~HostBuf() { release(); }
};

struct Runtime {
    int device = -1;
    int sms = 148;
    uint16_t *d_scan = nullptr;   // scan position -> idx | band<<12
    QTab *d_qtab = nullptr;       // kMaxQSlots tables
    uint16_t h_scan[kN3];
    float h_cos[16][16];
    std::mutex qmu;
    std::vector<uint64_t> qkeys; // (q bits << 32 | prior generation) per slot
};

// The process-wide runtime, initialised on first use. Null (with the thread's
// error set) when no CUDA device is usable: the product has no CPU path.
Runtime *runtime();
// Device table slot for a (sanitised) quality under the active priors.
int qslot(float q);
// The quality a slot was made for (6 for a slot not in use).
float slot_quality(int slot);

// Device-side state of one batched decode: items, arena offsets, entropy
// headers, arena and overflow pool. decode_prepare sizes the buffers for the
// host item array and uploads items and offsets; decode_enqueue launches the
// two stages (capturable into a CUDA graph).
struct DecodeBatch {
    DevBuf items, order, base, hdr, arena, pool, status, rec_idx;
    DevBuf fws;   // work area of the fused decode kernel
    HostBuf h_items, h_order, h_base, h_status, h_rec;   // pinned staging of decode_prepare_staged
    int n = 0;
    std::vector<std::pair<int, int>> subs;   // [i0, i1) ranges that fit the arena
    std::vector<int> coded;                  // per sub-batch: items with a payload
    // Per sub-batch: the longest `split` coded blocks (the head of the
    // processing order) decode and reconstruct on a second, high-priority
    // stream, so that the long serial chains of their entropy decode overlap
    // the reconstruction of everything else. rec_idx lists, per sub-batch,
    // those blocks' items ascending, then the other items ascending.
    std::vector<int> split;
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    DecodeBatch() = default;
    DecodeBatch(const DecodeBatch &) = delete;
    DecodeBatch &operator=(const DecodeBatch &) = delete;
    ~DecodeBatch();
};
// One stage of the host-blob decode pipeline: its own stream, batch and
// device buffers, reused once the event of its previous group has fired.
struct BlobSlot {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    DecodeBatch batch;
    DevBuf src, out;
    ~BlobSlot();
};
// Per-thread execution resources: a stream and reusable buffers.
// Slots of the host-blob decode pipeline (mc_b200_decode_chunk_blobs).
constexpr int kBlobSlots = 8;

struct Lane {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    DevBuf status, out;
    DecodeBatch batch;
    DevBuf enc_items, enc_len, enc_frac, enc_pay, src;
    DevBuf enc_lv, enc_corr, enc_sym;   // encoder symbol scratch (levels, corrections, per-block info)
    DevBuf b_scratch, b_lens16, b_bitmap, b_fmap, b_fml, b_np, b_len, b_off, b_q, blobs;
    DevBuf pyr_stage, pyr_a, pyr_b, pyr_flag;   // LOD pyramid: chunk staging, level volumes, all-air flags
    DevBuf ver_items, ver_bad;                  // device verify: blob list, mismatch flags
    DevBuf smp_grid, smp_cand, smp_acc;         // box sampling: block-fraction grid, candidates, accept flags
    DevBuf solo;                                // single-block decode scratch (SoloScratch)
    HostBuf h_items, h_base, h_stage, h_misc;
    HostBuf h_one;                              // single-block output, written by the kernel over the bus
    HostBuf h_bounce[3];                        // device-to-host pieces bound for pageable memory
    cudaEvent_t bounce_ev[3] = {};
    LaunchCfg cfg;
    BlobSlot pipe[kBlobSlots];
    ~Lane();
};
Lane *lane();

bool decode_prepare(DecodeBatch &B, const DecItem *h_items, int n, cudaStream_t s);
// decode_prepare without any host synchronisation: the n items are already in
// B.h_items (pinned), order and offsets are built in B's pinned staging, and
// every upload is asynchronous on s. The caller guarantees that the batch's
// previous use has completed.
bool decode_prepare_staged(DecodeBatch &B, int n, cudaStream_t s);
// Creates the stream and event of a pipeline slot on first use.
bool blob_slot_ready(BlobSlot &S);
bool decode_enqueue(DecodeBatch &B, const LaunchCfg &cfg, cudaStream_t s);
// One stage only: 0 = status reset + entropy, 1 = reconstruction.
bool decode_enqueue_stage(DecodeBatch &B, const LaunchCfg &cfg, int stage, cudaStream_t s);

// Copies n bytes of device memory to host memory dst after the work already
// on the lane's stream, and returns when they are there. A dst in pageable
// memory takes pinned bounce buffers: 8 MiB pieces travel while earlier ones
// are copied out by host threads, so the copy runs near the link's rate
// instead of the driver's pageable path (about 3 GB/s here). False on a CUDA
// error. With seg > 0 the device range is n / seg segments of seg bytes,
// segment k bound for dst + k * dst_stride.
bool copy_to_host(Lane &L, uint8_t *dst, const uint8_t *d_src, size_t n, size_t seg = 0, size_t dst_stride = 0);
// The other direction, for large ranges of pageable host memory (a mapped
// archive file): host threads fill 8 MiB pinned pieces while earlier pieces
// cross the link. The copies are enqueued on the lane's stream; the call
// returns once the last piece has been handed to the stream, so later work
// on the stream sees the bytes. False on a CUDA error.
bool copy_to_device(Lane &L, uint8_t *d_dst, const uint8_t *src, size_t n);

// Decodes n items whose src/dst are device addresses (host-side item array),
// enqueued on stream s (null: the lane's stream); false on a launch error.
bool decode_items(Lane &L, const DecItem *items, int n, cudaStream_t s = nullptr);
// One block on the lane's stream through the single-block kernel (no
// batch layout, no copies): the output lands at it.dst; the lane's status
// word reports whether its stream was cut short.
bool decode_one(Lane &L, const DecItem &it);
// decode_one into host memory, synchronously: the kernel stores the 16^3
// voxels straight into the lane's pinned, device-mapped output buffer (no
// device-to-host copy is enqueued), then they are copied to dst. it.dst,
// it.sz and it.sy are set here.
bool decode_one_host(Lane &L, DecItem it, uint8_t *dst);

// Encodes chunks of 256^3 voxels resident on the device (chunk c at
// d_vox[c]) into assembled blobs. Synchronises; on return blob_len[c]
// (0 = all air) and the blob offsets inside L.blobs are filled.
bool encode_chunks(Lane &L, const uint8_t *const *d_vox, int nchunks, const float *header_q, const float *q,
                   const int *tau, std::vector<uint64_t> &blob_off, std::vector<uint64_t> &blob_len);

// Blocks whose corrupt streams were cut short during the last decode on the lane.
uint32_t lane_bad_blocks(Lane &L);

}  // namespace mcb
