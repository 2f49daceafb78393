// mcb_archive.h -- private: the archive handle and the helpers shared by the
// archive format code (mcb_archive.cpp) and the decode / append entry points
// (mcb_api.cpp).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <mutex>
#include <utility>
#include <vector>

#include "../../include/matter_compressor_b200.h"
#include "mcb_format.h"
#include "mcb_runtime.h"

struct mc_codec_ctx {
    float quality = 8.0f;   // default quality (src/mc_codec.c:480)
    int max_err = 0;
};

struct mc_archive {
    int fd = -1;
    uint8_t *base = nullptr;
    std::atomic<uint64_t> cursor{0}, file_len{0};
    float quality = 0;
    uint32_t block_codec = MC_BLOCKCODEC_CABAC;
    uint64_t reserve = 0;
    std::mutex grow_mu, write_mu;
    std::atomic<uint64_t> gen{0};
    // device mirror of [0, synced)
    std::mutex mir_mu;
    uint8_t *d_base = nullptr;
    uint64_t d_cap = 0, synced = 0;
    std::vector<std::pair<uint64_t, uint64_t>> dirty;   // in-place writes below `synced`
    cudaEvent_t mir_ev = nullptr;
};

namespace mcb {

// Per-thread index of one chunk blob: payload offset (0 = absent) and length
// of each block (src/mc_archive.h:175-206).
struct ChunkIndex {
    const uint8_t *arc = nullptr;
    uint64_t chunk_off = ~0ull, tag = 0;
    uint64_t off[kGrid3];
    uint16_t len[kGrid3];
};
const ChunkIndex &chunk_index(const uint8_t *arc, uint64_t chunk_off);
float chunk_q(const mc_archive *a, uint64_t chunk_off);
int install_blob(mc_archive *a, int lod, int cz, int cy, int cx, const uint8_t *blob, size_t len);
int mark_zero(mc_archive *a, int lod, int cz, int cy, int cx);
// Bring the HBM mirror up to date and order the lane's stream after it.
uint8_t *mirror_sync(mc_archive *a, Lane &L);
// A chunk blob that passed the structural checks of the verify walk.
struct VerifyBlob {
    uint64_t co, len;       // blob offset and length in the archive
    uint32_t np;            // present blocks (bitmap popcount)
    int lod, n2, n1, n0;    // where the walk found it
};
// The mc_verify_archive node walk: -1 if the header is unusable, else the
// number of node tables and blobs that fail their bounds; the rest go to out.
long verify_walk(const uint8_t *arc, size_t len, std::vector<VerifyBlob> &out, long *total);

}  // namespace mcb
