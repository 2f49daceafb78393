// mcb_gather.cu -- the serving loop's device side: slot-table updates and the
// gather of cached blocks into request outputs.
//
// A request is described by one GatherItem per chunk it touches: a box of
// blocks inside the chunk, the voxel clip of the request in chunk-local
// coordinates, and the output address of chunk-local voxel (0,0,0). Every
// resident chunk owns a table of 4096 cache-slot numbers in device memory;
// kZeroSlot marks an absent (all-air) block. The gather flattens all items'
// blocks into one index space and copies one block per warp.
#include <cuda_runtime.h>
#include <stdint.h>

#include "mcb_devinfo.h"
#include "mcb_format.h"
#include "mcb_kernels.h"
#include "mcb_rowstore.cuh"

namespace mcb {

__global__ void __launch_bounds__(256) k_table_update(const uint2 *upd, int n, uint32_t *tables) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint2 u = upd[i];
        tables[u.x] = u.y;
    }
}

__global__ void __launch_bounds__(128) k_gather_boxes(const GatherItem *items, int nitems, uint32_t nblocks,
                                                      const uint32_t *tables, const uint8_t *cache) {
    const int lane = threadIdx.x & 31;
    const uint32_t nwarps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t g = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); g < nblocks; g += nwarps) {
        // the item holding flattened block g: the last one whose first <= g
        int lo = 0, hi = nitems - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (items[mid].first <= g) lo = mid;
            else hi = mid - 1;
        }
        const GatherItem it = items[lo];
        const uint32_t local = g - it.first;
        const int bz0 = it.box_lo >> 8, by0 = (it.box_lo >> 4) & 15, bx0 = it.box_lo & 15;
        const int nby = ((it.box_hi >> 4) & 15) - by0 + 1, nbx = (it.box_hi & 15) - bx0 + 1;
        const int bz = bz0 + (int)(local / (uint32_t)(nby * nbx));
        const int by = by0 + (int)((local / (uint32_t)nbx) % (uint32_t)nby);
        const int bx = bx0 + (int)(local % (uint32_t)nbx);
        const uint32_t slot = it.table == kNoTable ? kZeroSlot : tables[(size_t)it.table * kGrid3 + (bz << 8 | by << 4 | bx)];
        const uint8_t *src = slot >= kZeroSlot ? nullptr : cache + (size_t)slot * kN3;
        // the block's voxels inside the clip, chunk-local
        const int z0 = max(bz * 16, (int)it.lo[0]), z1 = min(bz * 16 + 15, (int)it.hi[0]);
        const int y0 = max(by * 16, (int)it.lo[1]), y1 = min(by * 16 + 15, (int)it.hi[1]);
        const int x0 = max(bx * 16, (int)it.lo[2]), x1 = min(bx * 16 + 15, (int)it.hi[2]);
        if (z0 > z1 || y0 > y1 || x0 > x1) continue;
        const int ny = y1 - y0 + 1, nrows = (z1 - z0 + 1) * ny;
        const bool full_x = x0 == bx * 16 && x1 == bx * 16 + 15;
        uint8_t *dst = reinterpret_cast<uint8_t *>(it.dst);
        for (int r = lane; r < nrows; r += 32) {
            const int z = z0 + r / ny, y = y0 + r % ny;
            uint8_t *row = dst + z * it.sz + y * it.sy;
            const uint8_t *srow = src ? src + (z - bz * 16) * 256 + (y - by * 16) * 16 - bx * 16 : nullptr;
            if (full_x) {   // a whole 16-byte block row: one aligned load from the cache slot
                store_row16(row + x0, srow ? *reinterpret_cast<const uint4 *>(srow + x0) : make_uint4(0, 0, 0, 0));
            } else {
                for (int x = x0; x <= x1; ++x) row[x] = srow ? srow[x] : 0;
            }
        }
    }
}

static int sm_count() { return dev_sms(); }

cudaError_t launch_table_update(const uint2 *d_upd, int n, uint32_t *d_tables, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    int blocks = (n + 255) / 256;
    if (blocks > sm_count() * 4) blocks = sm_count() * 4;
    k_table_update<<<blocks, 256, 0, s>>>(d_upd, n, d_tables);
    return cudaGetLastError();
}

cudaError_t launch_gather_boxes(const GatherItem *d_items, int nitems, uint32_t nblocks, const uint32_t *d_tables,
                                const uint8_t *d_cache, cudaStream_t s) {
    if (nitems <= 0 || nblocks == 0) return cudaSuccess;
    uint32_t blocks = (nblocks + 3) / 4;   // a block per warp, at most 8 CTAs per SM
    const uint32_t cap = (uint32_t)sm_count() * 8;
    if (blocks > cap) blocks = cap;
    k_gather_boxes<<<blocks, 128, 0, s>>>(d_items, nitems, nblocks, d_tables, d_cache);
    return cudaGetLastError();
}

}  // namespace mcb
