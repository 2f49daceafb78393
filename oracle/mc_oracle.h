/*
 * mc_oracle.h -- CPU restatement of matter-compressor's 16^3 block codec.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker that the CUDA product
 * path is compared against; it is loaded by tests/, by __graft_entry__.smoke()
 * and by bench.py's cpu_baseline leg, and nothing in the product links it.
 *
 * Parity is pinned two ways: (1) tests/golden/ holds vectors produced by the
 * reference's own sources compiled in strict-IEEE mode (oracle/Makefile ->
 * oracle/_ref/libmcref.so), and the tests require this restatement to
 * reproduce them byte-for-byte; (2) where oracle/_ref/libmcref.so is present
 * the tests also compare against it directly.
 *
 * Every function cites the reference file:line whose behaviour it restates
 * (paths relative to the reference checkout).
 */
#ifndef MC_ORACLE_H
#define MC_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Process-global trained-prior override (src/mc_codec.c:144-154).
 * plo/phi are u16[8][32]; NULL,NULL restores the baked tables. */
void or_set_priors(const uint16_t *plo, const uint16_t *phi);
/* Interpolated per-q prior table u16[8][32] (src/mc_codec.c:156-167). */
void or_priors_for_q(float q, uint16_t out[256]);
/* Quality sanitiser of mc_codec_ctx_set_quality (src/mc_codec.c:493-498). */
float or_sanitize_q(float q);
/* Dead-zone step table for a quality (src/mc_codec.c:542-552). */
void or_step_table(float q, float step[4096], float rstep[4096]);
/* Ascending-L1 scan order (src/mc_codec.c:280-304). */
void or_scan_table(uint16_t scan[4096]);

/* Block codec (src/mc_codec.c:629-783). q is sanitised like the ctx does.
 * Returns the payload length, 0 for an all-air block. cap >= 17408 is safe. */
uint32_t or_enc_block(const uint8_t vox[4096], float q, int tau,
                      uint8_t *out, uint32_t cap);
void     or_dec_block(const uint8_t *payload, uint32_t plen, float q,
                      uint8_t dst[4096]);
/* Decode that also reports the entropy-stage results: levels (raster),
 * extents, dc, flags, correction count.  Used to localise mismatches. */
void     or_dec_block_levels(const uint8_t *payload, uint32_t plen, float q,
                             int16_t levels[4096], int info[8]);

/* Fraction map (src/mc_codec.c:597-621). */
uint32_t or_enc_fracmap(const uint8_t frac[4096], uint8_t *out, uint32_t cap);
void     or_dec_fracmap(const uint8_t *in, uint32_t len, uint8_t frac[4096]);
/* Per-block material nibble (src/mc_codec.c:820-822). */
uint8_t  or_frac_nibble(const uint8_t vox[4096]);

/* XXH64 (src/mc_codec.c:378-414) and the chunk-blob hash chain
 * (src/mc_archive.c:76-88). */
uint64_t or_xxh64(const void *data, size_t len, uint64_t seed);
uint64_t or_blob_hash(const uint8_t *blob, uint64_t blob_len);

/* Whole-chunk blob encode (src/mc_codec.c:809-845, src/mc_archive.c:861-901).
 * header_q is written into the blob, q drives the codec (the parallel path
 * stores the caller's raw q while coding with the sanitised one). Returns the
 * blob length, 0 when the chunk is all air. */
size_t or_encode_chunk(const uint8_t *vox256, float header_q, float q, int tau,
                       uint8_t *out, size_t cap);
/* Decode every block of a chunk blob into a 256^3 z,y,x buffer
 * (src/mc_archive.c:787-820 with src/mc_archive.h:175-206). */
void   or_decode_chunk(const uint8_t *blob, uint64_t blob_len, uint8_t *out256);
/* Decode one block of a chunk blob (src/mc_archive.c:728-740). */
void   or_decode_chunk_block(const uint8_t *blob, uint64_t blob_len,
                             int bz, int by, int bx, uint8_t dst[4096]);

/* Decode-side deblocking filter, in place on a dense nz x ny x nx volume
 * (src/mc_codec.c:561-595, declared at src/matter_compressor.h:106). The
 * faces between 16-aligned blocks are filtered axis by axis: x, then y, then
 * z. Neighbours are addressed linearly, as the reference does (a face in the
 * last voxel of a row reads the next row's first voxel); a read past the end
 * of the volume, undefined in the reference, reads 0 here. */
void   or_deblock(uint8_t *vol, int nz, int ny, int nx, float quality);

/* 2x LOD decimation (src/mc_archive.c:63-72): output voxel (z,y,x) of a
 * ((DZ+1)/2, (DY+1)/2, (DX+1)/2) volume is the rounded mean of the NON-ZERO
 * voxels among its up to 8 children (children past an odd edge do not
 * exist), or 0 when all children are 0. */
void   or_decimate(const uint8_t *src, int DZ, int DY, int DX, uint8_t *dst);

/* A voxel source over a dense buffer for the reference's one-shot builder
 * (mc_voxel_fn, src/matter_compressor.h:134): ud points to an
 * or_volume_src; voxels outside the buffer read 0. */
typedef struct { const uint8_t *v; int nz, ny, nx; } or_volume_src;
uint8_t or_voxel_source(void *ud, int x, int y, int z);

#ifdef __cplusplus
}
#endif
#endif
