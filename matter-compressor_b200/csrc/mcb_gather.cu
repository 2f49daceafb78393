// mcb_gather.cu -- copies decoded 16^3 blocks (dense z,y,x, 4096 bytes) from
// the serving cache into request outputs: whole chunks, single blocks and
// clipped region crops. One warp per block; a null source writes zeros (an
// absent or all-air block).
#include <cuda_runtime.h>
#include <stdint.h>

#include "mcb_format.h"
#include "mcb_kernels.h"

namespace mcb {

__global__ void __launch_bounds__(128) k_gather(const DecItem *items, int n) {
    const int lane = threadIdx.x & 31;
    const int nwarps = gridDim.x * (blockDim.x >> 5);
    for (int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += nwarps) {
        const DecItem it = items[i];
        const int z0 = it.clip_lo >> 8, y0 = (it.clip_lo >> 4) & 15, x0 = it.clip_lo & 15;
        const int z1 = it.clip_hi >> 8, y1 = (it.clip_hi >> 4) & 15, x1 = it.clip_hi & 15;
        const int ny = y1 - y0 + 1, nrows = (z1 - z0 + 1) * ny;
        const uint8_t *src = reinterpret_cast<const uint8_t *>(it.src);
        uint8_t *dst = reinterpret_cast<uint8_t *>(it.dst);
        const bool full_x = x0 == 0 && x1 == 15;
        for (int r = lane; r < nrows; r += 32) {
            const int z = z0 + r / ny, y = y0 + r % ny;
            uint8_t *row = dst + z * it.sz + y * it.sy;
            if (full_x && ((uintptr_t)row & 15) == 0) {
                *reinterpret_cast<uint4 *>(row) =
                    src ? *reinterpret_cast<const uint4 *>(src + z * 256 + y * 16) : make_uint4(0, 0, 0, 0);
            } else {
                for (int x = x0; x <= x1; ++x) row[x] = src ? src[z * 256 + y * 16 + x] : 0;
            }
        }
    }
}

cudaError_t launch_gather(const DecItem *d_items, int n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int blocks = (n + 3) / 4;
    if (blocks > sms * 8) blocks = sms * 8;
    k_gather<<<blocks, 128, 0, s>>>(d_items, n);
    return cudaGetLastError();
}

}  // namespace mcb
