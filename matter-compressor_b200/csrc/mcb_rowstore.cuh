// mcb_rowstore.cuh -- storing one 16-byte voxel row of a block to an output
// row at any byte address (region crops and strided batches start anywhere).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace mcb {

// Writes the 16 bytes of v (byte i of the row = byte i of v, little endian) to
// d..d+15 with the widest aligned stores the address allows: one 16-byte
// store, four 4-byte stores, or, off a 4-byte boundary by s, the head's 4 - s
// bytes, three 4-byte words of funnel-shifted bytes and the tail's s bytes.
__device__ __forceinline__ void store_row16(uint8_t *d, const uint4 v) {
    const uint32_t mis = (uint32_t)(uintptr_t)d & 15;
    if (mis == 0) {
        *reinterpret_cast<uint4 *>(d) = v;
    } else if ((mis & 3) == 0) {
        uint32_t *dw = reinterpret_cast<uint32_t *>(d);
        dw[0] = v.x; dw[1] = v.y; dw[2] = v.z; dw[3] = v.w;
    } else {
        const uint32_t sft = mis & 3, w[4] = {v.x, v.y, v.z, v.w};
        for (uint32_t i = 0; i < 4 - sft; ++i) d[i] = (uint8_t)(w[0] >> (8 * i));
        uint32_t *dw = reinterpret_cast<uint32_t *>(d + 4 - sft);
#pragma unroll
        for (int j = 1; j < 4; ++j) dw[j - 1] = __funnelshift_r(w[j - 1], w[j], 8 * (4 - sft));
        for (uint32_t i = 0; i < sft; ++i) d[16 - sft + i] = (uint8_t)(w[3] >> (8 * (4 - sft + i)));
    }
}

}  // namespace mcb
