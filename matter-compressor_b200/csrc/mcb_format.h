// mcb_format.h -- constants and plain-data records shared by the host runtime
// and the sm_100a kernels of the matter-compressor 16^3 block codec.
//
// On-disk formats follow the reference byte for byte:
//   chunk blob  = [f32 q][u64 xxh64][u16 fmaplen][fmap][512 B block bitmap]
//                 [u16 len per present block][payloads]      (src/mc_archive.h:147-151)
//   archive     = [256 B header][metadata to 128 KiB][node tables + blobs at EOF]
//                                                             (src/mc_archive.h:56-94)
#pragma once
#include <stddef.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define MCB_HD __host__ __device__
#else
#define MCB_HD
#endif

namespace mcb {

constexpr int kBlk = 16;            // block edge (voxels)
constexpr int kN3 = 4096;           // voxels per block
constexpr int kChunk = 256;         // chunk edge (voxels)
constexpr int kGrid3 = 4096;        // blocks per chunk, slots per index node
constexpr int kBitmapBytes = 512;   // chunk blob block bitmap
constexpr int kBlobHdr = 14;        // [f32 q][u64 hash][u16 fmaplen]
constexpr int kFmapCap = kGrid3 / 2 + 64;
constexpr uint64_t kSlotZero = 1;   // index slot sentinel: visited, all air
constexpr uint64_t kHashSeed = 0x6D636368756E6Bull;
constexpr int kEgCap = 64;          // Exp-Golomb prefix cap on corrupt streams
constexpr int kMaxQSlots = 256;     // distinct (quality, prior set) tables on device
constexpr int kEncCap = kN3 * 4 + 1024;   // per-block encoder output bound (src/mc_codec.c:442)

// Context layout of one block's adaptive bins (u16 p0 each).
constexpr int kCtxFlag = 0;    // 2 header bins
constexpr int kCtxDc = 2;      // 8 dc bins, MSB first
constexpr int kCtxEob = 10;    // 14 EOB-prefix bins (13 used)
constexpr int kCtxSig = 24;    // 32 significance bins: band*4 + density
constexpr int kCtxMag = 56;    // 12 magnitude rungs
constexpr int kNumCtx = 68;

// Per-quality tables. Dead-zone step depends on the coefficient only through
// its L1 frequency cz+cy+cx in [0,45], so one row per L1 value suffices.
struct QTab {
    float step[48];    // q * (1+L1)^0.65
    float dz8[48];     // 0.80f * step   (as the reference evaluates it)
    float dz4[48];     // 0.40f * step
    float rstep[48];   // 1.0f / step
    uint16_t ctx[72];  // initial p0 of the 68 contexts for this q
    float q;
    uint32_t pad[3];
};

// One block to decode. Output voxel (z,y,x) of the block, for z,y,x inside the
// clip box, lands at dst + z*sz + y*sy + x.
struct DecItem {
    uint64_t src;      // device address of the payload
    uint64_t dst;      // device address of block voxel (0,0,0); may lie outside
                       // the caller's buffer when the clip box excludes it
    int64_t sz;        // byte strides of the output
    int64_t sy;
    uint32_t len;      // payload bytes; 0 = absent block (zeros)
    uint16_t qslot;
    uint16_t clip_lo;  // z0<<8 | y0<<4 | x0
    uint16_t clip_hi;  // (z1-1)<<8 | (y1-1)<<4 | (x1-1)
    uint16_t pad0;
    uint32_t pad1;
};
static_assert(sizeof(DecItem) == 48, "DecItem layout");

constexpr uint16_t kClipFullLo = 0x000;
constexpr uint16_t kClipFullHi = 0xFFF;

// Entropy-stage result of one block.
struct EntHdr {
    uint8_t dc, flags, bad, pad;
    int8_t ez, ey, ex, pad2;   // largest coefficient coordinate per axis (-1: none)
    uint16_t nnz, ncorr;       // coefficients, corrections recorded
    uint32_t ovf;              // overflow-pool offset (entries), 0xFFFFFFFF: none
};
static_assert(sizeof(EntHdr) == 16, "EntHdr layout");

// Entry list of a block: nnz coefficient entries (scan position | level<<16) followed by
// ncorr correction pairs (pos, wrapping delta).  The first cap entries live in
// the arena at the block's base; later ones continue in the overflow pool.
MCB_HD inline uint32_t entry_cap(uint32_t len) {
    uint64_t c = 8ull * len + 64;
    return c > 12288 ? 12288u : (uint32_t)c;
}
constexpr uint32_t kEntryMax = 12288;

}  // namespace mcb
