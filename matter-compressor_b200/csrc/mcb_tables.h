// mcb_tables.h -- host-side construction of the codec's fixed tables.
//
// Everything that the reference computes with libm (cos, powf, log) is
// computed here on the host with the same expressions and uploaded, so the
// device never evaluates a transcendental and the tables are bit-identical
// to the reference's.
#pragma once
#include <stdint.h>

#include "mcb_format.h"

namespace mcb {

// cmf[k][n] = ck*cos(pi*(2n+1)*k/32), orthonormal DCT-II (src/mc_codec_float.h:70-78).
void table_cos(float cmf[16][16]);
// scan position -> raster index | band<<12, ascending L1 frequency with ties in
// raster order (src/mc_codec.c:280-308).
void table_scan(uint16_t scan[kN3]);
// Prior state: process-global override of the trained tables
// (src/mc_codec.c:141-154). Returns the generation after the change.
uint32_t priors_set(const uint16_t *plo, const uint16_t *phi);
uint32_t priors_generation();
// Copies the active endpoint tables (u16[8][32] each).
void priors_active(uint16_t lo[8][32], uint16_t hi[8][32]);
// Per-quality table: dead-zone steps and the initial contexts for q
// (src/mc_codec.c:156-167, 542-552). q must already be sanitised.
void table_qtab(float q, QTab *out);
// mc_codec_ctx_set_quality's guard (src/mc_codec.c:493-498).
inline float sanitize_q(float q) { return (!(q > 0.0f) || q > 1024.0f) ? 8.0f : q; }

}  // namespace mcb
