// mcb_deblock.cu -- the decode-side deblocking filter on the device
// (src/mc_codec.c:561-595, declared at src/matter_compressor.h:106).
//
// The filter works in place, axis by axis: every x face, then every y face,
// then every z face between 16-aligned blocks. A face at coordinate f of its
// axis reads the voxels at f-2, f-1, f, f+1 along the axis and writes f-1 and
// f; faces of one axis sit 16 apart, so no two of them touch a common voxel
// and all faces of an axis run in parallel. One kernel per axis, in stream
// order, gives the reference's result: each axis sees the previous axes'
// output. Volumes of a batch are independent (grid.y).
//
// Neighbours are addressed linearly, like the reference's pointer arithmetic:
// a face in the last voxel of a row (or plane) reads the next row's (plane's)
// first voxel, which no face of the same axis writes. A read past the end of
// the volume -- undefined in the reference -- reads 0.
//
// Memory: the x pass touches every 32-byte sector of the volume (faces every
// 16 bytes), the y and z passes a quarter of the rows and planes, so one call
// moves about 2.75x the volume's bytes. Where rows are 16-byte aligned the y
// and z passes take 16 faces per thread as 16-byte row vectors (four
// independent loads in flight per thread instead of four single bytes).
#include <cuda_runtime.h>
#include <stdint.h>

#include "mcb_devinfo.h"
#include "mcb_kernels.h"

namespace mcb {

struct DbParams {
    uint8_t *vol;
    size_t vstride;      // bytes between the volumes of a batch
    size_t total;        // voxels of one volume
    uint32_t nx, ny, nz;
    uint32_t sz;         // ny * nx
    uint32_t nf;         // faces of this pass's axis: (n - 1) / 16 for n > 16, else 0
    uint32_t work;       // face positions of this pass in one volume
    int beta, tc;
};

// One face: p1 p0 | q0 q1, q0 at index i, neighbours `step` apart
// (src/mc_codec.c:563-574).
__device__ __forceinline__ void db_face(uint8_t *v, size_t total, size_t i, size_t step, int beta, int tc) {
    const int p0 = v[i - step], q0 = v[i];
    if (p0 == 0 || q0 == 0) return;          // air is never touched
    const int d = q0 - p0;
    if (abs(d) >= beta) return;              // a real edge is kept
    const int p1 = v[i - 2 * step];
    const int q1 = i + step < total ? v[i + step] : 0;
    const int pn = p1 ? p1 : p0, qn = q1 ? q1 : q0;
    int delta = (4 * d + (pn - qn) + 4) >> 3;
    delta = delta > tc ? tc : delta;
    delta = delta < -tc ? -tc : delta;
    v[i - step] = (uint8_t)min(max(p0 + delta, 1), 255);
    v[i] = (uint8_t)min(max(q0 - delta, 1), 255);
}

// x faces: work = rows (nz*ny) x nf, the face index fastest.
__global__ void __launch_bounds__(256) k_deblock_x(DbParams P) {
    uint8_t *v = P.vol + (size_t)blockIdx.y * P.vstride;
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < P.work; g += gridDim.x * blockDim.x) {
        const uint32_t row = g / P.nf, j = g - row * P.nf;
        db_face(v, P.total, (size_t)row * P.nx + 16u * (j + 1u), 1, P.beta, P.tc);
    }
}

// y faces: work = nz x nf x nx, x fastest (coalesced).
__global__ void __launch_bounds__(256) k_deblock_y(DbParams P) {
    uint8_t *v = P.vol + (size_t)blockIdx.y * P.vstride;
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < P.work; g += gridDim.x * blockDim.x) {
        const uint32_t t = g / P.nx, x = g - t * P.nx;
        const uint32_t z = t / P.nf, k = t - z * P.nf;
        db_face(v, P.total, (size_t)z * P.sz + (size_t)(16u * (k + 1u)) * P.nx + x, P.nx, P.beta, P.tc);
    }
}

// z faces: work = nf x (ny*nx), the in-plane index fastest.
__global__ void __launch_bounds__(256) k_deblock_z(DbParams P) {
    uint8_t *v = P.vol + (size_t)blockIdx.y * P.vstride;
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < P.work; g += gridDim.x * blockDim.x) {
        const uint32_t k = g / P.sz, r = g - k * P.sz;
        db_face(v, P.total, (size_t)(16u * (k + 1u)) * P.sz + r, P.sz, P.beta, P.tc);
    }
}

// The same filter on 16 faces side by side in x: rows p1, p0, q0, q1 as
// 16-byte vectors; p0 and q0 come back. Used when rows are 16-byte aligned.
__device__ __forceinline__ void db_face16(uint8_t *v, size_t total, size_t i, size_t step, int beta, int tc) {
    const uint4 P1 = *reinterpret_cast<const uint4 *>(v + i - 2 * step);
    uint4 P0 = *reinterpret_cast<const uint4 *>(v + i - step);
    uint4 Q0 = *reinterpret_cast<const uint4 *>(v + i);
    const uint4 Q1 = i + step < total ? *reinterpret_cast<const uint4 *>(v + i + step) : make_uint4(0, 0, 0, 0);
    const uint8_t *p1 = reinterpret_cast<const uint8_t *>(&P1), *q1 = reinterpret_cast<const uint8_t *>(&Q1);
    uint8_t *p0 = reinterpret_cast<uint8_t *>(&P0), *q0 = reinterpret_cast<uint8_t *>(&Q0);
#pragma unroll
    for (int b = 0; b < 16; ++b) {
        const int a = p0[b], c = q0[b];
        if (a == 0 || c == 0) continue;
        const int d = c - a;
        if (abs(d) >= beta) continue;
        const int pn = p1[b] ? p1[b] : a, qn = q1[b] ? q1[b] : c;
        int delta = (4 * d + (pn - qn) + 4) >> 3;
        delta = delta > tc ? tc : delta;
        delta = delta < -tc ? -tc : delta;
        p0[b] = (uint8_t)min(max(a + delta, 1), 255);
        q0[b] = (uint8_t)min(max(c - delta, 1), 255);
    }
    *reinterpret_cast<uint4 *>(v + i - step) = P0;
    *reinterpret_cast<uint4 *>(v + i) = Q0;
}

// y faces, 16 x at a time: work = nz x nf x (nx/16).
__global__ void __launch_bounds__(256) k_deblock_y16(DbParams P) {
    uint8_t *v = P.vol + (size_t)blockIdx.y * P.vstride;
    const uint32_t nxs = P.nx >> 4;
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < P.work; g += gridDim.x * blockDim.x) {
        const uint32_t t = g / nxs, xs = g - t * nxs;
        const uint32_t z = t / P.nf, k = t - z * P.nf;
        db_face16(v, P.total, (size_t)z * P.sz + (size_t)(16u * (k + 1u)) * P.nx + 16u * xs, P.nx, P.beta, P.tc);
    }
}

// z faces, 16 x at a time: work = nf x (ny*nx/16).
__global__ void __launch_bounds__(256) k_deblock_z16(DbParams P) {
    uint8_t *v = P.vol + (size_t)blockIdx.y * P.vstride;
    const uint32_t s16 = P.sz >> 4;
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < P.work; g += gridDim.x * blockDim.x) {
        const uint32_t k = g / s16, r = g - k * s16;
        db_face16(v, P.total, (size_t)(16u * (k + 1u)) * P.sz + 16u * r, P.sz, P.beta, P.tc);
    }
}

static int db_sms() { return dev_sms(); }

static uint32_t faces(uint32_t n) { return n > 16 ? (n - 1) / 16 : 0; }

cudaError_t launch_deblock(uint8_t *d_vol, int count, size_t vstride, int nz, int ny, int nx, int beta, int tc,
                           cudaStream_t s) {
    if (count <= 0 || nz <= 0 || ny <= 0 || nx <= 0) return cudaSuccess;
    if (count > 65535) return cudaErrorInvalidValue;
    const uint64_t sz = (uint64_t)ny * (uint64_t)nx;
    const uint64_t rows = (uint64_t)nz * (uint64_t)ny;
    // every per-pass index of one volume in 32 bits
    if (sz >= (1ull << 32) || rows >= (1ull << 32) || rows * faces((uint32_t)nx) >= (1ull << 32) ||
        (uint64_t)nz * faces((uint32_t)ny) * (uint64_t)nx >= (1ull << 32) ||
        (uint64_t)faces((uint32_t)nz) * sz >= (1ull << 32))
        return cudaErrorInvalidValue;
    DbParams P;
    P.vol = d_vol;
    P.vstride = vstride;
    P.total = (size_t)rows * (size_t)nx;
    P.nx = (uint32_t)nx;
    P.ny = (uint32_t)ny;
    P.nz = (uint32_t)nz;
    P.sz = (uint32_t)sz;
    P.beta = beta;
    P.tc = tc;
    const uint32_t cap = (uint32_t)db_sms() * 8u;
    auto grid = [&](uint32_t work) {
        uint32_t b = (work + 255u) / 256u;
        return dim3(b < cap ? b : cap, (unsigned)count);
    };
    P.nf = faces(P.nx);
    P.work = (uint32_t)(rows * P.nf);
    if (P.work) k_deblock_x<<<grid(P.work), 256, 0, s>>>(P);
    // rows of 16-byte vectors when every row of every volume starts on a 16-byte boundary
    const bool vec = nx % 16 == 0 && ((uintptr_t)d_vol & 15) == 0 && (count == 1 || vstride % 16 == 0);
    P.nf = faces(P.ny);
    P.work = P.nz * P.nf * (vec ? P.nx / 16 : P.nx);
    if (P.work) {
        if (vec) k_deblock_y16<<<grid(P.work), 256, 0, s>>>(P);
        else k_deblock_y<<<grid(P.work), 256, 0, s>>>(P);
    }
    P.nf = faces(P.nz);
    P.work = P.nf * (vec ? P.sz / 16 : P.sz);
    if (P.work) {
        if (vec) k_deblock_z16<<<grid(P.work), 256, 0, s>>>(P);
        else k_deblock_z<<<grid(P.work), 256, 0, s>>>(P);
    }
    return cudaGetLastError();
}

}  // namespace mcb
