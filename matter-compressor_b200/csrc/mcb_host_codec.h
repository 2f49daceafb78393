// mcb_host_codec.h -- host-side metadata utilities (see mcb_host_codec.cpp).
#pragma once
#include <stddef.h>
#include <stdint.h>

namespace mcb {
uint64_t host_xxh64(const void *data, size_t len, uint64_t seed);
uint64_t host_blob_hash(const uint8_t *blob, uint64_t blob_len);
uint32_t host_enc_fracmap(const uint8_t *frac, uint8_t *out, size_t cap);
void host_dec_fracmap(const uint8_t *in, uint32_t len, uint8_t *frac);
}  // namespace mcb
