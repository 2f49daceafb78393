// mcb_sample.cu -- fraction-map rejection sampling of training boxes on the
// device (src/mc_archive.c:911-948): the score of a candidate box is the
// mean, over the 16^3 blocks it touches, of each block's material fraction
// (its fraction-map nibble / 15). The host generates the candidates in the
// reference's order from its xorshift64 stream and keeps the first `count`
// accepted; this kernel scores a batch of candidates at once, one thread per
// candidate, from a block-fraction grid in device memory. The sum runs in
// double over z, then y, then x blocks, adding each block's float fraction,
// as the reference does, so every accept decision is the reference's.
#include <cuda_runtime.h>
#include <stdint.h>

#include "mcb_kernels.h"

namespace mcb {

__global__ void __launch_bounds__(128) k_sample_score(const uint8_t *__restrict__ grid, long gz, long gy, long gx,
                                                      const long *__restrict__ cand, int n, long dz, long dy,
                                                      long dx, float min_frac, uint8_t *__restrict__ accept) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long z0 = cand[3 * i], y0 = cand[3 * i + 1], x0 = cand[3 * i + 2];
    const long bz0 = z0 >> 4, bz1 = (z0 + dz - 1) >> 4, by0 = y0 >> 4, by1 = (y0 + dy - 1) >> 4;
    const long bx0 = x0 >> 4, bx1 = (x0 + dx - 1) >> 4;
    double fsum = 0;
    long nb = 0;
    for (long bz = bz0; bz <= bz1; ++bz)
        for (long by = by0; by <= by1; ++by)
            for (long bx = bx0; bx <= bx1; ++bx) {
                const bool in = bz < gz && by < gy && bx < gx;
                const float f = in ? (float)__ldg(grid + (bz * gy + by) * gx + bx) / 15.0f : 0.0f;
                fsum = __dadd_rn(fsum, (double)f);
                nb++;
            }
    accept[i] = nb && fsum / (double)nb >= (double)min_frac;
}

cudaError_t launch_sample_score(const uint8_t *d_grid, long gz, long gy, long gx, const long *d_cand, int n,
                                long dz, long dy, long dx, float min_frac, uint8_t *d_accept, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    k_sample_score<<<(n + 127) / 128, 128, 0, s>>>(d_grid, gz, gy, gx, d_cand, n, dz, dy, dx, min_frac, d_accept);
    return cudaGetLastError();
}

}  // namespace mcb
