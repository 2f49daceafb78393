// mcb_host_codec.cpp -- host-side codec utilities for archive METADATA paths:
// XXH64 for mc_verify_archive / mc_chunk_compute_hash and the fraction-map
// range coder for mc_archive_block_fraction / mc_archive_sample_boxes. Block
// payloads are never coded here: block encode and decode run on the GPU only.
#include <stdint.h>
#include <string.h>

#include "mcb_format.h"
#include "mcb_host_codec.h"

namespace mcb {

namespace {
constexpr uint64_t P1 = 0x9E3779B185EBCA87ull, P2 = 0xC2B2AE3D27D4EB4Full, P3 = 0x165667B19E3779F9ull,
                   P4 = 0x85EBCA77C2B2AE63ull, P5 = 0x27D4EB2F165667C5ull;
inline uint64_t rotl(uint64_t x, int r) { return (x << r) | (x >> (64 - r)); }
inline uint64_t mix(uint64_t acc, uint64_t in) { return rotl(acc + in * P2, 31) * P1; }
inline uint64_t rd64(const uint8_t *p) { uint64_t v; memcpy(&v, p, 8); return v; }
inline uint32_t rd32(const uint8_t *p) { uint32_t v; memcpy(&v, p, 4); return v; }
}  // namespace

// Published XXH64 (as used by src/mc_codec.c:393-414).
uint64_t host_xxh64(const void *data, size_t len, uint64_t seed) {
    const uint8_t *p = static_cast<const uint8_t *>(data), *end = p + len;
    uint64_t h;
    if (len >= 32) {
        uint64_t v[4] = {seed + P1 + P2, seed + P2, seed, seed - P1};
        for (; end - p >= 32; p += 32)
            for (int i = 0; i < 4; ++i) v[i] = mix(v[i], rd64(p + 8 * i));
        h = rotl(v[0], 1) + rotl(v[1], 7) + rotl(v[2], 12) + rotl(v[3], 18);
        for (int i = 0; i < 4; ++i) h = (h ^ mix(0, v[i])) * P1 + P4;
    } else {
        h = seed + P5;
    }
    h += (uint64_t)len;
    for (; end - p >= 8; p += 8) h = rotl(h ^ mix(0, rd64(p)), 27) * P1 + P4;
    if (end - p >= 4) { h = rotl(h ^ ((uint64_t)rd32(p) * P1), 23) * P2 + P3; p += 4; }
    for (; p < end; ++p) h = rotl(h ^ ((uint64_t)*p * P5), 11) * P1;
    h ^= h >> 33; h *= P2; h ^= h >> 29; h *= P3; h ^= h >> 32;
    return h;
}

// Chained blob hash over fmap | bitmap | lengths | payloads (src/mc_archive.c:76-88).
uint64_t host_blob_hash(const uint8_t *blob, uint64_t blob_len) {
    uint16_t fml;
    memcpy(&fml, blob + 12, 2);
    const uint8_t *fmap = blob + kBlobHdr, *bm = fmap + fml, *lens = bm + kBitmapBytes;
    uint32_t np = 0;
    for (int i = 0; i < kBitmapBytes; ++i) np += (uint32_t)__builtin_popcount(bm[i]);
    const uint64_t pay = (uint64_t)kBlobHdr + fml + kBitmapBytes + 2ull * np;
    uint64_t h = host_xxh64(fmap, fml, kHashSeed);
    h ^= host_xxh64(bm, kBitmapBytes, h);
    h ^= host_xxh64(lens, 2ull * np, h);
    h ^= host_xxh64(blob + pay, blob_len - pay, h);
    return h;
}

// Fraction-map coder: 4096 nibbles, 4 adaptive bins each (initial p0 2048),
// context = bucket of the previous nibble (src/mc_codec.c:597-621), coded
// with the reference's LZMA-style binary range coder (src/mc_codec.c:178-205).
namespace {
struct HostEnc {
    uint8_t *out; size_t cap, len; uint64_t low; uint32_t range; uint8_t cache; uint64_t pending;
    void shift() {
        uint32_t top = (uint32_t)(low >> 32);
        if (top != 0 || low < 0xFF000000ull) {
            emit((uint8_t)(cache + top));
            for (uint64_t i = 1; i < pending; ++i) emit((uint8_t)(0xFF + top));
            pending = 0;
            cache = (uint8_t)(low >> 24);
        }
        pending++;
        low = (low << 8) & 0xFFFFFFFFull;
    }
    void emit(uint8_t b) { if (len < cap) out[len] = b; len++; }
    void bit(uint16_t &p0, int b) {
        uint32_t r0 = (range >> 12) * p0;
        if (!b) { range = r0; p0 = (uint16_t)(p0 + ((4096 - p0) >> 4)); }
        else { low += r0; range -= r0; p0 = (uint16_t)(p0 - (p0 >> 4)); }
        while (range < (1u << 24)) { shift(); range <<= 8; }
    }
};
struct HostDec {
    const uint8_t *buf; size_t len, pos; uint32_t code, range;
    uint8_t byte() { return pos < len ? buf[pos++] : 0; }
    int bit(uint16_t &p0) {
        uint32_t r0 = (range >> 12) * p0;
        int b;
        if (code < r0) { range = r0; b = 0; p0 = (uint16_t)(p0 + ((4096 - p0) >> 4)); }
        else { code -= r0; range -= r0; b = 1; p0 = (uint16_t)(p0 - (p0 >> 4)); }
        while (range < (1u << 24)) { code = (code << 8) | byte(); range <<= 8; }
        return b;
    }
};
inline int bucket(int prev) { return prev == 0 ? 0 : prev == 15 ? 2 : 1; }
}  // namespace

uint32_t host_enc_fracmap(const uint8_t *frac, uint8_t *out, size_t cap) {
    HostEnc e{out, cap, 0, 0, 0xFFFFFFFFu, 0, 1};
    uint16_t c[3][4];
    for (auto &r : c) for (auto &v : r) v = 2048;
    int prev = 0;
    for (int i = 0; i < kGrid3; ++i) {
        int v = frac[i] & 15, b = bucket(prev);
        for (int k = 3; k >= 0; --k) e.bit(c[b][k], (v >> k) & 1);
        prev = v;
    }
    for (int i = 0; i < 5; ++i) e.shift();
    return (uint32_t)e.len;
}

void host_dec_fracmap(const uint8_t *in, uint32_t len, uint8_t *frac) {
    HostDec d{in, len, 0, 0, 0xFFFFFFFFu};
    for (int i = 0; i < 5; ++i) d.code = (d.code << 8) | d.byte();
    uint16_t c[3][4];
    for (auto &r : c) for (auto &v : r) v = 2048;
    int prev = 0;
    for (int i = 0; i < kGrid3; ++i) {
        int v = 0, b = bucket(prev);
        for (int k = 3; k >= 0; --k) v |= d.bit(c[b][k]) << k;
        frac[i] = (uint8_t)v;
        prev = v;
    }
}

}  // namespace mcb
