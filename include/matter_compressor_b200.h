/*
 * matter_compressor_b200.h -- C ABI of the B200 (sm_100a) implementation of
 * matter-compressor's 16^3 block codec and its archive read/append paths.
 *
 * Part 1 re-declares, with identical names, signatures and semantics, the
 * entry points of the reference's public header that this library replaces;
 * each cites the reference declaration (src/matter_compressor.h:<line>). A
 * program built against the reference links against libmc_b200.so unchanged
 * for these calls. Decoding and encoding run on the GPU; there is no CPU
 * fallback: without a usable sm_100 device the calls report an error through
 * mc_b200_last_error() (decode calls also zero their output, append calls
 * return -1).
 *
 * Part 2 adds what the reference has no counterpart for: device-resident
 * (HBM) archives, batched decodes into device buffers, graph-captured decode
 * plans and batched encode. Pointers documented as "device" are CUDA device
 * addresses; `stream` is a cudaStream_t passed as void* (NULL: the library's
 * per-thread stream, synchronised before return).
 */
#ifndef MATTER_COMPRESSOR_B200_H
#define MATTER_COMPRESSOR_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef uint8_t mc_u8;

/* ======================================================== part 1: drop-in */

/* ---- codec context and presets ---- */
typedef struct mc_codec_ctx mc_codec_ctx;
mc_codec_ctx *mc_codec_ctx_new(void);                            /* src/matter_compressor.h:42 */
void  mc_codec_ctx_free(mc_codec_ctx *ctx);                      /* :43 */
void  mc_codec_ctx_set_quality(mc_codec_ctx *ctx, float quality);/* :44 */
float mc_codec_ctx_get_quality(mc_codec_ctx *ctx);               /* :45 */
void  mc_codec_ctx_set_max_error(mc_codec_ctx *ctx, int tau);    /* :58 */
int   mc_codec_ctx_get_max_error(mc_codec_ctx *ctx);             /* :59 */

typedef enum {
    MC_PRESET_ARCHIVAL = 0, MC_PRESET_MASTER = 1, MC_PRESET_HIGH = 2, MC_PRESET_BALANCED = 3,
    MC_PRESET_STREAMING = 4, MC_PRESET_FAST = 5, MC_PRESET_ULTRAFAST = 6, MC_PRESET_PREVIEW = 7,
    MC_PRESET_COUNT = 8
} mc_preset;                                                      /* :74-84 */
float       mc_apply_preset(mc_codec_ctx *ctx, mc_preset level); /* :88 */
float       mc_preset_quality(mc_preset level);                  /* :89 */
int         mc_preset_tau(mc_preset level);                      /* :90 */
const char *mc_preset_name(mc_preset level);                     /* :91 */
void  mc_codec_init(void);                                        /* :92 */
void  mc_codec_set_priors(const uint16_t *plo, const uint16_t *phi); /* :96 */

typedef struct { mc_u8 *p; size_t len, cap; } mc_buf;            /* :99 */
void  mc_buf_put(mc_buf *b, const void *s, size_t n);             /* :100 */

/* ---- block codec (GPU) ---- */
int   mc_enc_block(mc_codec_ctx *ctx, const mc_u8 *vox, mc_buf *out, uint32_t *len_out); /* :111 */
void  mc_dec_block(mc_codec_ctx *ctx, const mc_u8 *payload, uint32_t plen, mc_u8 *dst); /* :114 */
uint32_t mc_enc_fracmap(const mc_u8 *frac, mc_u8 *out, size_t cap);                    /* :117 */
void     mc_dec_fracmap(const mc_u8 *in, uint32_t len, mc_u8 *frac);                   /* :118 */

/* ---- archive ---- */
typedef struct mc_archive mc_archive;
typedef enum { MC_ABSENT = 0, MC_PRESENT = 1, MC_ZERO = 2 } mc_cover;                   /* :173 */
#define MC_BLOCKCODEC_CABAC 0u
mc_archive *mc_archive_open(const char *path, int dim, float quality);                  /* :177 */
mc_archive *mc_archive_open_dims(const char *path, int nx, int ny, int nz, float quality); /* :180 */
int      mc_archive_set_block_codec(mc_archive *a, uint32_t codec);                     /* :188 */
uint32_t mc_archive_block_codec(const mc_archive *a);                                  /* :189 */
int mc_archive_block_blob(mc_archive *a, uint64_t chunk_off, int bz, int by, int bx,
                          const uint8_t **ptr, uint32_t *len);                         /* :194 */
int mc_archive_append_chunk_raw(mc_archive *a, int lod, int cz, int cy, int cx,
                                const mc_u8 vox[256 * 256 * 256]);                     /* :201 */
int mc_archive_append_chunk_raw_q(mc_archive *a, int lod, int cz, int cy, int cx,
                                  const mc_u8 vox[256 * 256 * 256], float q);          /* :206 */
int mc_archive_append_chunk_ctx(mc_archive *a, mc_codec_ctx *C, int lod, int cz, int cy, int cx,
                                const mc_u8 vox[256 * 256 * 256]);                     /* :212 */
int mc_archive_append_chunk_compressed(mc_archive *a, int lod, int cz, int cy, int cx,
                                       const uint8_t *blob, size_t len);               /* :227 */
int mc_archive_reserve_index(mc_archive *a, int lod, int cz, int cy, int cx);          /* :235 */
mc_cover mc_archive_chunk_coverage(mc_archive *a, int lod, int cz, int cy, int cx);    /* :238 */
uint64_t mc_archive_data_len(mc_archive *a);                                           /* :243 */
int mc_archive_set_metadata(mc_archive *a, const void *data, size_t len);              /* :250 */
const char *mc_archive_metadata(mc_archive *a, size_t *out_len);                       /* :251 */
uint64_t mc_archive_chunk_offset(mc_archive *a, int lod, int cz, int cy, int cx);      /* :255 */
void mc_archive_decode_block(mc_archive *a, uint64_t chunk_off, int bz, int by, int bx,
                             mc_u8 *dst);                                              /* :260 */
void mc_archive_decode_chunk(mc_archive *a, uint64_t chunk_off, mc_u8 *out, int nthreads); /* :265 */
int mc_archive_append_chunk_par(mc_archive *a, int lod, int cz, int cy, int cx,
                                const mc_u8 vox[256 * 256 * 256], float q, int nthreads); /* :269 */
void mc_archive_read_region(mc_archive *a, int lod, long z0, long y0, long x0,
                            long dz, long dy, long dx, mc_u8 *out, size_t sz, size_t sy,
                            int nthreads);                                             /* :279 */
int mc_archive_block_present(mc_archive *a, int lod, int bz, int by, int bx);          /* :287 */
float mc_archive_block_fraction(mc_archive *a, int lod, int bz, int by, int bx);       /* :292 */
typedef struct { long z0, y0, x0; } mc_box;                                            /* :299 */
int mc_archive_sample_boxes(mc_archive *a, int lod, uint64_t seed, int count,
                            long dz, long dy, long dx, float min_frac, mc_box *out);  /* :300 */
void mc_archive_read_regions(mc_archive *a, int lod, const mc_box *boxes, int n,
                             long dz, long dy, long dx, mc_u8 *out, size_t batch_stride,
                             int nthreads);                                            /* :307 */
void mc_archive_close(mc_archive *a);                                                  /* :312 */
uint64_t mc_chunk_compute_hash(const uint8_t *blob, uint64_t blob_len);                /* :369 */
long mc_verify_archive(const uint8_t *arc, size_t len, int verbose);                   /* :370 */
int mc_archive_set_priors(mc_archive *a, const uint16_t plo[8][32], const uint16_t phi[8][32]); /* :377 */
uint64_t mc_xxh64(const void *data, size_t len, uint64_t seed);            /* src/mc_codec.h:17 */
/* Decode-side deblocking, in place on a dense HOST volume (staged through the
 * device). A read past the volume's end, undefined in the reference, reads 0. */
void mc_deblock(mc_u8 *vol, int nz, int ny, int nx, float quality);      /* src/matter_compressor.h:106 */

/* ---- read-only readers (blocks decoded on the GPU) ---- */
typedef struct mc_reader mc_reader;
typedef int (*mc_read_fn)(void *ud, uint64_t off, uint32_t len, uint8_t *dst);        /* :329 */
mc_reader *mc_open(const uint8_t *arc, size_t len);                                     /* :316 */
void       mc_close(mc_reader *r);                                                      /* :317 */
void       mc_reader_set_quality(mc_reader *r, float q);                                /* :318 */
uint64_t   mc_chunk_offset(mc_reader *r, int lod, int cz, int cy, int cx);              /* :319 */
uint64_t   mc_chunk_offset_chk(mc_reader *r, int lod, int cz, int cy, int cx, int *err); /* :323 */
void       mc_decode_block(mc_reader *r, uint64_t chunk_off, int bz, int by, int bx, mc_u8 *dst); /* :324 */
mc_reader *mc_open_streaming(mc_read_fn read, void *ud, uint64_t total_len);           /* :334 */
void       mc_reader_set_partial_fetch(mc_reader *r, int on);                           /* :341 */
uint64_t   mc_reader_chunk_blob_len(mc_reader *r, uint64_t chunk_off);                  /* :346 */
int        mc_reader_read_blob(mc_reader *r, uint64_t chunk_off, size_t len, uint8_t *dst); /* :352 */
int        mc_reader_priors(mc_reader *r, const uint16_t **plo, const uint16_t **phi);  /* :356 */
void       mc_reader_dims(mc_reader *r, int *nx, int *ny, int *nz);                     /* :359 */
float      mc_reader_quality(mc_reader *r);                                             /* :360 */
int        mc_reader_nlods(mc_reader *r);                                               /* :361 */

/* ====================================================== part 2: additions */

/* Runtime. mc_b200_init returns 0 when an sm_100 device is usable, -1 (with
 * the reason in mc_b200_last_error) otherwise. The last error is per thread. */
int  mc_b200_init(void);
/* The CUDA device ordinal the library's runtime is bound to (the calling
 * thread's current device at the library's first use; one device per
 * process), or -1 without a usable device. No reference counterpart. */
int  mc_b200_device(void);
const char *mc_b200_last_error(void);
void mc_b200_clear_error(void);
/* Blocks of the calling thread's last decode whose corrupt stream was cut
 * short (Exp-Golomb prefix cap or overflow-pool exhaustion). */
uint32_t mc_b200_last_bad_blocks(void);
/* How the calling thread's decodes without a plan (per-call chunk, block and
 * region reads, the host-blob pipeline) split the entropy stage between its
 * two kernels. A lane of a warp decodes a block at about 5 issue slots per
 * bin but about 450 cycles per bin; one thread alone takes about 25 slots but
 * about 120 cycles. share > 1: the longest coded/share blocks on single
 * threads, the rest one per lane; 1: every block on a single thread; 0: every
 * block on a lane; -1 (the default): by the launch's coded-block count (every
 * block on single threads up to 28 K blocks, the longest 1/64 up to 90 K), and
 * lanes only in the host-blob pipeline, whose groups overlap. Decoded voxels
 * are the same in every case. Returns 0; -1 (with the last error set) for
 * share < -1 or without a usable device. No reference counterpart. */
int  mc_b200_set_entropy_solo(int share);

/* Decode n whole chunk blobs held in HOST memory (blob i: blobs[i], blob_lens[i]
 * bytes, as stored in an archive) into HOST memory, chunk i at
 * out + i*out_stride (256^3 z,y,x). A NULL blob decodes to zeros. Payload
 * bytes go host->device, voxels device->host, inside the call. Returns 0. */
int mc_b200_decode_chunk_blobs(const uint8_t *const *blobs, const uint64_t *blob_lens, int n,
                               mc_u8 *out, size_t out_stride);

/* HBM-resident archive: mirror the archive's bytes in device memory (kept in
 * sync lazily on later calls). Returns 0; dev_base and len (if non-NULL) receive
 * the device mirror's address and synced length. */
int mc_b200_archive_sync(mc_archive *a, const uint8_t **dev_base, uint64_t *len);

/* Decode n chunks of the archive (offsets from mc_archive_chunk_offset) into
 * DEVICE memory, chunk i at d_out + i*out_stride. */
int mc_b200_decode_chunks_dev(mc_archive *a, const uint64_t *chunk_offs, int n,
                              mc_u8 *d_out, size_t out_stride, void *stream);

/* mc_archive_read_regions into DEVICE memory: crop i at d_out + i*batch_stride,
 * dense z,y,x; decode and crop fused. */
int mc_b200_read_regions_dev(mc_archive *a, int lod, const mc_box *boxes, int n,
                             long dz, long dy, long dx, mc_u8 *d_out, size_t batch_stride,
                             void *stream);

/* Decode plan: the work list, scratch and a CUDA graph of the whole batched
 * decode of n chunks into DEVICE memory, built once and replayed. */
typedef struct mc_b200_plan mc_b200_plan;
mc_b200_plan *mc_b200_plan_decode_chunks(mc_archive *a, const uint64_t *chunk_offs, int n,
                                         mc_u8 *d_out, size_t out_stride);
/* The same for a batch of regions (mc_archive_read_regions' arguments, DEVICE
 * output: crop i at d_out + i*batch_stride, dense z,y,x): the boxes' blocks,
 * clipped, decoded and cropped by every replay. */
mc_b200_plan *mc_b200_plan_read_regions(mc_archive *a, int lod, const mc_box *boxes, int n, long dz, long dy,
                                        long dx, mc_u8 *d_out, size_t batch_stride);
/* Replays the plan on `stream` and returns at once. Unlike the other calls,
 * a NULL stream here is the legacy default stream (the graph launch's own
 * meaning of NULL), not the library's per-thread stream. */
int  mc_b200_plan_launch(mc_b200_plan *p, void *stream);
/* Launch one stage of the plan outside its graph (stage 0: entropy decode,
 * 1: reconstruction; stage 1 consumes stage 0's output), e.g. to time the
 * kernels one by one. Asynchronous on `stream`, NULL = legacy default stream,
 * as for mc_b200_plan_launch. */
int  mc_b200_plan_launch_stage(mc_b200_plan *p, int stage, void *stream);
/* Kernel launches per replay, blocks decoded, and total payload bytes. */
void mc_b200_plan_info(const mc_b200_plan *p, int *launches, long *blocks, uint64_t *payload_bytes);
/* The launch shape the plan's autotuner chose: entropy CTAs per SM,
 * reconstruction CTAs per SM, and the stage layout: 0 two kernels in sequence,
 * 1 the longest blocks on a second stream, 2 both stages in one persistent
 * kernel. */
void mc_b200_plan_config(const mc_b200_plan *p, int out[3]);
/* Deblocking filter (mc_deblock's arithmetic) in place on `count` dense DEVICE
 * volumes of nz x ny x nx voxels, vol_stride bytes apart. 0 on success, -1 on
 * bad arguments (count <= 65535 and each per-axis face count of one volume
 * below 2^32) or a CUDA error. */
int mc_b200_deblock_dev(mc_u8 *d_vol, int count, size_t vol_stride, int nz, int ny, int nx, float quality,
                        void *stream);

/* Replace the autotuner's choice (same layout as mc_b200_plan_config) and
 * recapture the plan. 0 on success, -1 on bad arguments or a CUDA error. */
int  mc_b200_plan_set_config(mc_b200_plan *p, const int cfg[3]);
/* The whole launch shape the autotuner chose, which it times on the plan's
 * own batch (cached per quality and batch size): out[0] entropy warps per CTA
 * (2, 4, 8), out[1] entropy CTAs per SM, out[2] entropy queue claim run
 * (entries a lane takes per claim), out[3] reconstruction CTAs per SM,
 * out[4] the stage layout as in mc_b200_plan_config, out[5] the single-thread
 * share: the longest coded/out[5] blocks of a launch are entropy-decoded one
 * per warp by one thread, at a few times a shared lane's speed per bin
 * (0: none; at most half of the launch's warps). */
void mc_b200_plan_tuning(const mc_b200_plan *p, int out[6]);
/* Replace it (same layout; warps x CTAs per SM at most 25) and recapture the
 * plan. 0 on success, -1 on bad arguments or a CUDA error. */
int  mc_b200_plan_set_tuning(mc_b200_plan *p, const int cfg[6]);
/* Fused layout only: how many times (each a sleep of at most 1 us) a CTA
 * polls a completion-list position that no block pair has filled yet before
 * it hands the position to the tail kernel and leaves (default 32768). Any
 * value gives the same voxels; 0 makes every such wait give up at once, which
 * moves the waiting pairs to the tail kernel. Recaptures the plan. 0 on
 * success, -1 on a CUDA error. */
int  mc_b200_plan_set_fused_wait(mc_b200_plan *p, uint32_t polls);
void mc_b200_plan_free(mc_b200_plan *p);

/* Batched append: encode n chunks (chunk i's 256^3 voxels at HOST vox[i], or
 * DEVICE memory when vox_on_device) in one batch and install them in order,
 * byte-identical to n calls of mc_archive_append_chunk_par (C == NULL, q) or
 * mc_archive_append_chunk_ctx (C != NULL). coords holds n (cz,cy,cx) triples. */
int mc_b200_append_chunks(mc_archive *a, mc_codec_ctx *C, int lod, const int *coords, int n,
                          const mc_u8 *const *vox, int vox_on_device, float q);

/* mc_verify_archive with the hashing on the device: the archive's bytes in
 * HOST memory (arc, for the walk over its node tables) and the same bytes in
 * DEVICE memory (d_arc, e.g. the mirror from mc_b200_archive_sync), len bytes
 * each. Every chunk blob's chained XXH64 is recomputed on the GPU and
 * compared with the stored one. Returns the number of corrupt node tables and
 * blobs, like mc_verify_archive (src/matter_compressor.h:370), or -1. */
long mc_b200_verify_archive_dev(const uint8_t *arc, const uint8_t *d_arc, size_t len, int verbose);

/* mc_archive_sample_boxes with the scoring on the device: the same boxes, in
 * the same order, from the same seed (src/matter_compressor.h:300). Each
 * chunk's fraction map is decoded once into a block-fraction grid in device
 * memory and candidates are scored in batches. Returns the number of boxes
 * written to out (0 also for a lod outside 0..7 or on a CUDA error). */
int mc_b200_sample_boxes(mc_archive *a, int lod, uint64_t seed, int count, long dz, long dy, long dx,
                         float min_frac, mc_box *out);

/* Reader batch decode: n blocks (bz, by, bx) = coords[3i..3i+2] of the chunk
 * at chunk_off into DEVICE memory, block i at d_out + 4096*i (16^3, z,y,x),
 * decoded on the GPU in one batch, the same voxels mc_decode_block gives.
 * Flat and full-fetch readers copy the payloads from the chunk blob; a
 * partial-fetch streaming reader reads only the asked-for payloads, one range
 * read per run of adjacent ones. Absent blocks, a missing chunk and unreadable
 * bytes decode to zeros. Returns 0 (after the decode ends), -1 on bad
 * arguments or a CUDA error. */
int mc_b200_reader_decode_blocks(mc_reader *r, uint64_t chunk_off, const int *coords, int n, mc_u8 *d_out,
                                 void *stream);

/* LOD pyramid on the device. mc_b200_decimate_dev: 2x box decimation of a
 * dense DEVICE volume nz x ny x nx into d_dst ((nz+1)/2 x (ny+1)/2 x
 * (nx+1)/2): each output voxel is the rounded mean of its non-zero children,
 * 0 when all are 0 (src/mc_archive.c:63-72). 0 on success, -1 on bad
 * arguments or a CUDA error.
 * mc_b200_append_pyramid: the one-shot builder's pyramid (mc_build,
 * src/mc_archive.c:184-234) appended to an archive from a dense DEVICE volume:
 * LOD 0 (the volume zero-padded to whole chunks) and each decimated LOD while
 * any axis of the current level is at least 256 voxels (LOD 1 always), at
 * most 8. Chunks are encoded at `quality` (max error 0) with chunk blobs
 * byte-identical to mc_build's; all-air chunks are left out. *nlods (if
 * non-NULL) receives the number of levels appended. 0 on success, -1 on an
 * error (levels appended before it stay in the archive). */
int mc_b200_decimate_dev(const mc_u8 *d_src, int nz, int ny, int nx, mc_u8 *d_dst, void *stream);
int mc_b200_append_pyramid(mc_archive *a, const mc_u8 *d_vol, int nz, int ny, int nx, float quality, int *nlods);

/* Serving: block, region and chunk reads of one archive, batched continuously
 * on the GPU behind a decoded-block cache in HBM -- the device-side analogue
 * of the reference's mc_cache read path (src/mc_cache.h). Requests queue on
 * submit; a worker thread admits them into a batch while the batch's output
 * bytes stay within batch_bytes and their missing blocks find free cache
 * slots, decodes the misses into the cache, gathers every request's blocks
 * into its output and completes the tickets. Small requests (up to 256 KiB
 * of output: blocks, small regions) and large ones queue and batch apart, on
 * a high-priority and a normal CUDA stream, so a block never waits for a
 * chunk decode in its own batch. Eviction follows the reference's S3-FIFO
 * (small and main FIFOs, a ghost queue of evicted keys) over slots no batch
 * in flight is using. Results are byte-identical to
 * mc_archive_decode_block / read_region / decode_chunk.
 *
 * out_on_device: request outputs are DEVICE pointers (any strides for
 * regions); otherwise HOST pointers (dense outputs only), copied back inside
 * the batch. The archive must not be appended to while the server is open.
 * cache_bytes is raised to at least one chunk's blocks (16 MiB). A batch in
 * flight holds every cached block of the chunks it reads; a request whose
 * chunks' cached blocks leave too few slots for its misses, with no batch in
 * flight that could free any, is refused (its wait returns -1) rather than
 * left waiting. */
typedef struct mc_b200_server mc_b200_server;
enum { MC_B200_REQ_BLOCK = 0, MC_B200_REQ_REGION = 1, MC_B200_REQ_CHUNK = 2 };
typedef struct {
    int kind;              /* MC_B200_REQ_* */
    int lod;
    long z, y, x;          /* block: block coordinates; chunk: chunk coordinates; region: voxel origin */
    long dz, dy, dx;       /* region extent in voxels (ignored otherwise) */
    mc_u8 *out;            /* block: 4096 bytes z,y,x; chunk: 256^3 z,y,x; region: crop at out + z*sz + y*sy + x */
    size_t sz, sy;         /* region output byte strides; 0 = dense (dy*dx, dx) */
} mc_b200_request;
mc_b200_server *mc_b200_server_open(mc_archive *a, size_t cache_bytes, size_t batch_bytes, int out_on_device);
/* Returns a ticket (>= 0) or -1 for an invalid request. */
long mc_b200_server_submit(mc_b200_server *s, const mc_b200_request *r);
/* 1 done, 0 pending, -1 failed or unknown ticket. */
int  mc_b200_server_poll(mc_b200_server *s, long ticket);
/* Blocks until the ticket completes: 0 done, -1 failed. */
int  mc_b200_server_wait(mc_b200_server *s, long ticket);
/* Steady-clock submit and completion times of a ticket (ns); returns its state. */
int  mc_b200_server_ticket_times(mc_b200_server *s, long ticket, uint64_t *submit_ns, uint64_t *done_ns);
/* Trace replay: submits reqs[i] at arrival_ns[i] after the call starts (i in
 * order), waits for all, and stores each completion time minus its arrival
 * time in latency_ns (may be NULL). Returns 0, or -1 if any request failed. */
int  mc_b200_server_replay(mc_b200_server *s, const mc_b200_request *reqs, const uint64_t *arrival_ns, int n,
                           uint64_t *latency_ns);
/* requests, batches, blocks, cache hits, misses (decoded), zero blocks,
 * evictions, output bytes. */
void mc_b200_server_stats(mc_b200_server *s, uint64_t out[8]);
/* Completes every queued request, then frees the server. */
void mc_b200_server_close(mc_b200_server *s);

/* Allocation-free block decode. This entry point has no counterpart in the
 * reference; it is for callers that must not allocate memory: code running
 * inside a memory pool's or allocator's own hooks (an allocation there would
 * re-enter the allocator), and real-time loops that forbid allocation once
 * started. It allocates nothing, on the device or the host: its work list,
 * coefficient lists and tables live in one fixed 17.3 MiB array in device
 * memory that the library declares statically.
 *
 * Decodes n payloads (as mc_dec_block takes them) already in DEVICE memory:
 * payload i is d_payloads[h_offsets[i] .. h_offsets[i+1]) (h_offsets: n+1
 * HOST values; an empty payload decodes to zeros), all at the one quality q
 * of the payloads' context. Block i lands at d_out + i*4096 (z,y,x raster).
 * Work is enqueued on `stream` (a cudaStream_t, NULL = legacy default
 * stream); the call returns before it ends.
 *
 * Limits: n <= 4096, and the sum over blocks of min(12288, 8*len_i + 64)
 * <= 4194304 (the per-block coefficient bound; a block of 1500 bytes or more
 * counts 12288); larger requests return -2 / -3 and must be split. d_payloads
 * must be 8-byte aligned with 16 readable bytes after the last payload;
 * d_out must hold n*4096 bytes. The payload lengths and the quality table
 * travel to the GPU inside the kernel launch itself, so the call keeps no
 * host buffer once it returns. Corrupt payloads decode as the reference decodes
 * them, except that their spill past the fixed 1 MiB overflow area is cut
 * short; no bad-block count is kept.
 * Returns 0, or -1 (bad arguments), -2, -3 (limits), -4 (CUDA error); each
 * failure prints one line to stderr.
 *
 * The first call on each device looks up the array's device address and
 * uploads the constant tables, synchronously, with that device current. All
 * calls share the one array, so two calls
 * whose work overlaps on the GPU (other streams, other host threads) race:
 * order them on one stream or with events. */
int mc_b200_decode_blocks_noalloc(const uint8_t *d_payloads, const uint64_t *h_offsets, int n,
                                  float q, mc_u8 *d_out, void *stream);

#ifdef __cplusplus
}
#endif
#endif
