/* mc_cache_trace.c -- BENCHMARK INFRASTRUCTURE: drives the reference's own
 * decoded-block cache (src/mc_cache.c, reached through its public API in
 * src/matter_compressor.h:412-530) over a serving trace, one request at a
 * time, and times each request on the host. It is linked against the
 * reference build in oracle/_ref/ and is never part of the product.
 *
 * A request is served the way a client of mc_cache does it: a single block
 * is one mc_cache_get_copy (decoded on a miss); a region or a chunk first
 * brings its blocks in with mc_cache_update (the reference's worker pool,
 * src/mc_cache.c:499-526), then copies each block's part of the request out
 * of the cache with mc_cache_get_copy into a dense z,y,x output. */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "matter_compressor.h"

enum { REQ_BLOCK = 0, REQ_REGION = 1, REQ_CHUNK = 2 };

static double now_ms(void) {
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return t.tv_sec * 1e3 + t.tv_nsec * 1e-6;
}

/* req: n rows of 8 int64 (kind, lod, z, y, x, dz, dy, dx): block and chunk
 * requests give block / chunk coordinates, regions voxel origin and extent.
 * out: at least 256^3 bytes (every request's output lands here in turn).
 * lat_ms: n latencies. Returns 0, or -1 when the archive or cache cannot be
 * opened. */
int mcct_run(const char *path, int nx, int ny, int nz, float q, size_t cache_bytes, int nthreads, int n,
             const int64_t *req, uint8_t *out, double *lat_ms) {
    mc_archive *a = mc_archive_open_dims(path, nx, ny, nz, q);
    if (!a) return -1;
    mc_cache *c = mc_cache_new_archive(cache_bytes, a);
    if (!c) { mc_archive_close(a); return -1; }
    mc_block_id *ids = malloc(sizeof(mc_block_id) * 4096 * 8);
    uint8_t blk[4096];
    for (int i = 0; i < n; ++i) {
        const int64_t *r = req + 8 * (size_t)i;
        const int kind = (int)r[0], lod = (int)r[1];
        const double t0 = now_ms();
        if (kind == REQ_BLOCK) {
            mc_cache_get_copy(c, lod, (int)r[2], (int)r[3], (int)r[4], out);
        } else {
            long z0, y0, x0, dz, dy, dx;
            if (kind == REQ_CHUNK) {
                z0 = r[2] * 256; y0 = r[3] * 256; x0 = r[4] * 256; dz = dy = dx = 256;
            } else {
                z0 = r[2]; y0 = r[3]; x0 = r[4]; dz = r[5]; dy = r[6]; dx = r[7];
            }
            const long b0[3] = {z0 >> 4, y0 >> 4, x0 >> 4};
            const long b1[3] = {(z0 + dz - 1) >> 4, (y0 + dy - 1) >> 4, (x0 + dx - 1) >> 4};
            size_t m = 0;
            for (long bz = b0[0]; bz <= b1[0]; ++bz)
                for (long by = b0[1]; by <= b1[1]; ++by)
                    for (long bx = b0[2]; bx <= b1[2]; ++bx)
                        if (m < 4096 * 8) ids[m++] = (mc_block_id){lod, (int)bz, (int)by, (int)bx};
            mc_cache_update(c, ids, m, nthreads);
            for (size_t k = 0; k < m; ++k) {
                const long bz = ids[k].bz, by = ids[k].by, bx = ids[k].bx;
                mc_cache_get_copy(c, lod, (int)bz, (int)by, (int)bx, blk);
                const long zs = bz * 16 > z0 ? bz * 16 : z0, ze = bz * 16 + 16 < z0 + dz ? bz * 16 + 16 : z0 + dz;
                const long ys = by * 16 > y0 ? by * 16 : y0, ye = by * 16 + 16 < y0 + dy ? by * 16 + 16 : y0 + dy;
                const long xs = bx * 16 > x0 ? bx * 16 : x0, xe = bx * 16 + 16 < x0 + dx ? bx * 16 + 16 : x0 + dx;
                for (long z = zs; z < ze; ++z)
                    for (long y = ys; y < ye; ++y)
                        memcpy(out + ((z - z0) * dy + (y - y0)) * dx + (xs - x0),
                               blk + ((z - bz * 16) * 16 + (y - by * 16)) * 16 + (xs - bx * 16), (size_t)(xe - xs));
            }
        }
        lat_ms[i] = now_ms() - t0;
    }
    free(ids);
    mc_cache_free(c);
    mc_archive_close(a);
    return 0;
}
