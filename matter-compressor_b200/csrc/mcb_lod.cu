// mcb_lod.cu -- LOD pyramid on the device: 2x box decimation
// (src/mc_archive.c:63-72) and the gather of 256^3 chunks out of a volume
// for the batched encoder (src/mc_archive.c:110-115).
//
// Decimation: one thread per output voxel; its up to 8 children are two
// adjacent bytes in each of 4 rows, so a warp's loads cover 64 contiguous
// bytes per row. Output voxel = rounded mean of the non-zero children, 0
// when all are 0; children past an odd edge do not exist. HBM-bound: the
// source is read once, an eighth of it is written.
//
// Gather: one thread per 16-byte row segment of the chunk; voxels outside
// the source volume read 0 (the zero padding to whole chunks). A per-chunk
// flag records whether any voxel is non-zero, so all-air chunks can be left
// out as the reference's builder leaves them out.
#include <cuda_runtime.h>
#include <stdint.h>

#include "mcb_devinfo.h"
#include "mcb_kernels.h"

namespace mcb {

__global__ void __launch_bounds__(256) k_decimate2(const uint8_t *__restrict__ src, uint32_t dz, uint32_t dy,
                                                   uint32_t dx, uint8_t *__restrict__ dst, uint32_t hy,
                                                   uint32_t hx, uint64_t nout) {
    for (uint64_t o = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; o < nout;
         o += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t x = (uint32_t)(o % hx);
        const uint64_t t = o / hx;
        const uint32_t y = (uint32_t)(t % hy), z = (uint32_t)(t / hy);
        uint32_t sum = 0, n = 0;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const uint32_t sz = 2 * z + (c >> 2), sy = 2 * y + ((c >> 1) & 1), sx = 2 * x + (c & 1);
            if (sz >= dz || sy >= dy || sx >= dx) continue;
            const uint32_t v = __ldg(src + ((uint64_t)sz * dy + sy) * dx + sx);
            sum += v;
            n += v != 0;
        }
        dst[o] = n ? (uint8_t)((sum + n / 2) / n) : 0;
    }
}

// Chunk (cz, cy, cx) of a dense nz x ny x nx volume into a dense 256^3
// buffer; *any |= 1 if a voxel is non-zero.
__global__ void __launch_bounds__(256) k_gather_chunk(const uint8_t *__restrict__ src, uint32_t nz, uint32_t ny,
                                                      uint32_t nx, uint32_t cz, uint32_t cy, uint32_t cx,
                                                      uint8_t *__restrict__ dst, uint32_t *any) {
    bool nonzero = false;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < 256u * 256u * 16u; s += gridDim.x * blockDim.x) {
        const uint32_t z = s >> 12, y = (s >> 4) & 255u, xs = (s & 15u) * 16u;
        const uint64_t gz = (uint64_t)cz * 256 + z, gy = (uint64_t)cy * 256 + y, gx = (uint64_t)cx * 256 + xs;
        uint4 v = make_uint4(0, 0, 0, 0);
        if (gz < nz && gy < ny && gx < nx) {
            const uint8_t *row = src + (gz * ny + gy) * nx;
            if (gx + 16 <= nx && ((uintptr_t)(row + gx) & 15) == 0) {
                v = __ldg(reinterpret_cast<const uint4 *>(row + gx));
            } else {
                uint8_t b[16];
#pragma unroll
                for (int i = 0; i < 16; ++i) b[i] = gx + i < nx ? __ldg(row + gx + i) : 0;
                memcpy(&v, b, 16);
            }
        }
        nonzero |= (v.x | v.y | v.z | v.w) != 0;
        reinterpret_cast<uint4 *>(dst)[s] = v;
    }
    if (__any_sync(0xFFFFFFFFu, nonzero) && (threadIdx.x & 31) == 0) atomicOr(any, 1u);
}

static int lod_sms() { return dev_sms(); }

cudaError_t launch_decimate(const uint8_t *d_src, int dz, int dy, int dx, uint8_t *d_dst, cudaStream_t s) {
    if (dz <= 0 || dy <= 0 || dx <= 0) return cudaErrorInvalidValue;
    const uint32_t hz = (uint32_t)(dz + 1) / 2, hy = (uint32_t)(dy + 1) / 2, hx = (uint32_t)(dx + 1) / 2;
    const uint64_t nout = (uint64_t)hz * hy * hx;
    uint64_t blocks = (nout + 255) / 256;
    const uint64_t cap = (uint64_t)lod_sms() * 16;
    if (blocks > cap) blocks = cap;
    k_decimate2<<<(unsigned)blocks, 256, 0, s>>>(d_src, (uint32_t)dz, (uint32_t)dy, (uint32_t)dx, d_dst, hy, hx, nout);
    return cudaGetLastError();
}

cudaError_t launch_gather_chunk(const uint8_t *d_src, int nz, int ny, int nx, int cz, int cy, int cx, uint8_t *d_dst,
                                uint32_t *d_any, cudaStream_t s) {
    k_gather_chunk<<<(unsigned)lod_sms() * 4, 256, 0, s>>>(d_src, (uint32_t)nz, (uint32_t)ny, (uint32_t)nx,
                                                           (uint32_t)cz, (uint32_t)cy, (uint32_t)cx, d_dst, d_any);
    return cudaGetLastError();
}

}  // namespace mcb
