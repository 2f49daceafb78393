// mcb_kernels.h -- launch interface of the sm_100a kernels (host side).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "mcb_format.h"

namespace mcb {

// Launch shape knobs, picked per quality by the autotuner.
struct LaunchCfg {
    int ent_warps = 4;         // entropy stage: warps per CTA (2, 4 or 8)
    int ent_claim = 1;         // entropy stage: queue entries a lane claims at a time (1, 2 or 4)
    int ent_ctas_per_sm = 5;   // entropy stage: CTAs per SM (8.8 KB of contexts per warp)
    int rec_ctas_per_sm = 4;   // reconstruction stage: CTAs of 128 threads per SM (<= 4: 47 KB smem)
    int ent_solo = -1;         // entropy stage: the longest ncoded / ent_solo blocks are decoded one per
                               // warp by a single thread (0: none; see EntParams::nsolo); 1: every
                               // block, by the single-thread kernel k_entropy_solo; -1: by the
                               // launch's coded-block count (see launch_entropy)
    bool split = false;        // long blocks on a second stream (batches large enough to split)
    bool fused = false;        // both stages in one persistent kernel (k_decode_fused)
    int fused_ctas_per_sm = 4;
    // fused layout: polls (of at most 1 us each) of an unwritten completion-list
    // position before a CTA gives the position to k_fused_tail and leaves
    uint32_t fused_wait_polls = 1u << 15;
};

struct EntParams {
    const DecItem *items;
    const uint32_t *order;     // optional processing order (by payload size), or null
    int n;
    int ncoded;                // blocks to decode: the first ncoded of the order (the
                               // rest are absent, len 0, and need no entropy stage)
    const uint64_t *base;      // per-item arena offset (entries)
    uint32_t *arena;
    EntHdr *hdr;
    uint32_t *pool;            // overflow pool for corrupt streams
    uint32_t pool_cap;
    uint32_t *pool_used;
    const QTab *qtab;
    const uint16_t *scan;      // scan position -> raster idx | band<<12
    uint32_t *status;          // [0]: blocks whose stream was cut short, [1]: pool entries used
    uint32_t *counter;         // work counter of this launch, zero at launch
    int claim;                 // queue entries claimed per counter increment (>= 1)
    // k_entropy: the first nsolo entries of the order (the longest payloads)
    // are decoded one per warp by the warp's first thread alone, which gives a
    // block's serial chain a few times the speed of a lane sharing its warp's
    // instructions with 31 others; warps 0..nsolo-1 of the grid do this
    // first, then join the other warps on the rest of the order. Needs an
    // order and at most half of the launch's warps (launch_entropy clamps it).
    int nsolo = 0;
};

struct RecParams {
    const DecItem *items;
    const uint32_t *idx;       // optional: the items to reconstruct (n of them), ascending; null = 0..n-1
    int n;
    const EntHdr *hdr;
    const uint64_t *base;
    const uint32_t *arena;
    const uint32_t *pool;
    const QTab *qtab;
    const uint16_t *scan;      // scan position -> raster idx | band<<12
};

// Both stages in one persistent kernel: entropy lanes mark finished blocks
// ready, the block completing a pair (2j, 2j+1) appends it to a completion
// list, and CTAs whose lanes are idle reconstruct pairs from that list
// (k_decode_fused); then a tail kernel for positions a CTA gave up waiting on.
// Work area F.ws, zeroed before each launch: kFusedDone, kFusedClaim and
// kFusedNSkip counters, kFusedMaxSkip skipped positions, then pair_cnt and
// rlist (fused_ws_words(n) words in all).
constexpr int kFusedDone = 0, kFusedClaim = 1, kFusedNSkip = 2, kFusedSkip0 = 4;
constexpr int kFusedMaxSkip = 4096;   // also the largest grid
inline size_t fused_ws_words(int n) { return (size_t)kFusedSkip0 + kFusedMaxSkip + 2 * (((size_t)n + 1) / 2); }
struct FusedParams {
    EntParams e;               // e.order holds the coded blocks first, then the absent ones
    RecParams r;               // r.n: items of the batch; r.idx unused
    uint32_t *ws;              // the work area
    uint32_t *pair_cnt;        // ws + kFusedSkip0 + kFusedMaxSkip: blocks of pair j ready
    uint32_t *rlist;           // pair_cnt + npairs: list position -> pair + 1, 0 until written
    uint32_t spin_limit;       // polls of an unwritten position before giving up
};
int fused_grid(const LaunchCfg &cfg);   // CTAs of k_decode_fused (0: cannot launch)
cudaError_t launch_fused(const FusedParams &f, const LaunchCfg &cfg, cudaStream_t s);
// The decode kernels' constant tables: the cosine basis and the band ends of
// the scan order (scan position -> raster idx | band << 12).
cudaError_t upload_decode_tables(const float cmf[16][16], const uint16_t scan[kN3], cudaStream_t s);
// Loads the decode kernels' code now (first-call latency under lazy loading).
cudaError_t preload_decode_kernels();
// Deblocking filter in place on `count` dense nz x ny x nx volumes vstride
// bytes apart (three stream-ordered kernels: x, y, z faces).
// LOD pyramid: 2x decimation of a dense dz x dy x dx volume into
// ((dz+1)/2, (dy+1)/2, (dx+1)/2), and the gather of chunk (cz, cy, cx) of a
// dense volume into a 256^3 buffer (zeros outside; *d_any |= 1 if non-zero).
cudaError_t launch_decimate(const uint8_t *d_src, int dz, int dy, int dx, uint8_t *d_dst, cudaStream_t s);
cudaError_t launch_gather_chunk(const uint8_t *d_src, int nz, int ny, int nx, int cz, int cy, int cx, uint8_t *d_dst,
                                uint32_t *d_any, cudaStream_t s);
// Rejection-sampling scores: accept[i] = 1 when candidate box i (z0, y0, x0
// at d_cand[3i..3i+2], extent dz x dy x dx) has a mean block fraction of at
// least min_frac over the gz x gy x gx block-fraction grid (nibbles 0..15).
cudaError_t launch_sample_score(const uint8_t *d_grid, long gz, long gy, long gx, const long *d_cand, int n,
                                long dz, long dy, long dx, float min_frac, uint8_t *d_accept, cudaStream_t s);
cudaError_t launch_deblock(uint8_t *d_vol, int count, size_t vstride, int nz, int ny, int nx, int beta, int tc,
                           cudaStream_t s);
// ---- serving ----
// One chunk's share of a request: a box of blocks, the request's voxel clip in
// chunk-local coordinates, and where chunk-local voxel (0,0,0) maps in the output.
constexpr uint32_t kNoTable = 0xFFFFFFFFu;    // chunk absent or all air: zeros
constexpr uint32_t kZeroSlot = 0xFFFFFFFEu;   // table entry of an absent block
constexpr uint32_t kEmptySlot = 0xFFFFFFFFu;  // table entry not resolved yet
struct GatherItem {
    uint64_t dst;              // output address of chunk-local voxel (0,0,0)
    int64_t sz, sy;            // output byte strides
    uint32_t table;            // slot table of the chunk, or kNoTable
    uint32_t first;            // flattened index of the item's first block
    uint16_t box_lo, box_hi;   // block box (z<<8|y<<4|x), inclusive
    uint8_t lo[3], hi[3];      // voxel clip (z, y, x), chunk-local, inclusive
    uint8_t pad[2];
};
static_assert(sizeof(GatherItem) == 48, "GatherItem layout");
// tables[u.x] = u.y for each update
cudaError_t launch_table_update(const uint2 *d_upd, int n, uint32_t *d_tables, cudaStream_t s);
// Copies every block of every item from the cache (slot s at cache + s*4096,
// dense z,y,x) into the outputs; nblocks = sum of the items' block counts.
cudaError_t launch_gather_boxes(const GatherItem *d_items, int nitems, uint32_t nblocks, const uint32_t *d_tables,
                                const uint8_t *d_cache, cudaStream_t s);
cudaError_t launch_entropy(const EntParams &p, const LaunchCfg &cfg, cudaStream_t s);
cudaError_t launch_reconstruct(const RecParams &p, const LaunchCfg &cfg, cudaStream_t s);

// Device scratch of the single-block decode (k_decode_one): the block's work
// item, its entropy header and its entry list.
struct SoloScratch {
    DecItem item;                  // offset 0 (16-byte aligned buffer)
    EntHdr hdr;                    // read back as one 16-byte load
    uint64_t base;                 // the block's entries start the list: 0
    uint32_t pool_used, pad;
    uint32_t entries[kEntryMax];   // the first entry_cap(len) are the arena, the rest the overflow pool
};
// One block end to end in one CTA: scalar entropy decode on one thread, then
// the CTA's reconstruction and clipped store. status[0] becomes the number of
// cut-short blocks (0 or 1).
cudaError_t launch_decode_one(const DecItem &it, SoloScratch *scratch, const QTab *qtab, const uint16_t *scan,
                              uint32_t *status, cudaStream_t s);

// ---- encode ----
// One 16^3 block to encode, gathered from a strided u8 source.
struct EncItem {
    uint64_t src;      // device address of source voxel (0,0,0) of the block
    int64_t sz, sy;    // source byte strides
    uint64_t out;      // device address of this block's payload slot (kEncCap bytes)
    uint16_t qslot;
    uint16_t tau;      // max-error bound, 0 = off
    uint32_t pad;
};
static_assert(sizeof(EncItem) == 40, "EncItem layout");

struct EncParams {
    const EncItem *items;
    int n;
    const QTab *qtab;
    const uint16_t *scan;
    uint32_t *len;       // per item: payload bytes (0 = all air, not coded)
    uint8_t *frac;       // per item: material nibble
    uint32_t *status;    // [0]: payloads that overflowed kEncCap
    // symbol scratch between the transform and the coder, per item: levels in
    // scan order (kN3 int16), corrections (kN3 u32: pos | delta << 16), and
    // (coded flag | eob << 8 | dc, ncorr)
    int16_t *levels;
    uint32_t *corr;
    uint2 *sym;
};
cudaError_t upload_cos_encode(const float cmf[16][16], cudaStream_t s);
cudaError_t launch_encode(const EncParams &p, cudaStream_t s);

// Chunk-blob assembly for chunks whose blocks were encoded by launch_encode
// with items in block order (chunk c owns items [4096c, 4096c+4096)).
struct BlobParams {
    int nchunks;
    const uint8_t *payload;   // item i's payload at payload + i*kEncCap
    const uint32_t *len;      // per item
    const uint8_t *frac;      // per item
    const float *header_q;    // per chunk: q written into the blob header
    // sizing-pass outputs (side buffers)
    uint32_t *scratch;        // per item: payload offset within the chunk's payloads
    uint16_t *lens16;         // per chunk: 4096 u16 length table
    uint8_t *bitmap;          // per chunk: 512 B
    uint8_t *fmap;            // per chunk: kFmapCap bytes
    uint32_t *fml, *np;       // per chunk
    uint64_t *blob_len;       // per chunk: total blob bytes, 0 = all air
    // write-pass inputs
    const uint64_t *blob_off; // per chunk: offset of the blob in `blobs`
    uint8_t *blobs;
};
cudaError_t launch_blob_layout(const BlobParams &p, cudaStream_t s);   // sizing pass
cudaError_t launch_blob_fill(const BlobParams &p, cudaStream_t s);     // write pass
cudaError_t launch_blob_hash(const BlobParams &p, cudaStream_t s);     // xxh64 chain
// Device verify: blob i at d_arc + co, `len` bytes, np present blocks; its
// chained xxh64 against the stored one, d_bad[i] = 1 on a mismatch.
struct VerifyItem {
    uint64_t co, len;
    uint32_t np, pad;
};
cudaError_t launch_verify_hash(const uint8_t *d_arc, uint64_t arc_len, const VerifyItem *d_items, int n,
                               uint32_t *d_bad, cudaStream_t s);

}  // namespace mcb
