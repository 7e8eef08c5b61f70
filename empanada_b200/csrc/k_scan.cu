// k_scan.cu -- single-pass exclusive scan of u32 counts (decoupled look-back).
//
// Used for the newline counts of FASTQ tiles, the kept-read flags and the
// per-suffix edge counts (the roles the reference gives to
// thrust::exclusive_scan / transform_exclusive_scan, preprocess.cu:31,140 and
// overlap.cu:564).  A tile is 256 threads x 4 chunks x uint4 (4096 values);
// chunk c of thread t covers values [c*1024 + t*4, +4), so every load is a
// fully coalesced 16-byte vector load.
#include "kernels.h"

namespace emp {

template <typename OutT>
__global__ void __launch_bounds__(256) scan_kernel(const uint32_t *__restrict__ in, OutT *out, uint64_t n,
                                                   uint64_t *status, uint32_t *tile_ctr, uint64_t *total,
                                                   uint32_t *err) {
    __shared__ uint32_t s_tile;
    __shared__ uint64_t s_warp[8];
    __shared__ uint64_t s_base;
    if (threadIdx.x == 0) s_tile = atomicAdd(tile_ctr, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint64_t base = (uint64_t)tile * kScanTile;
    uint32_t v[4][4];
    uint64_t texcl[4];
    uint64_t running = 0;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const uint64_t i0 = base + (uint64_t)c * 1024 + threadIdx.x * 4;
        if (i0 + 4 <= n && ((reinterpret_cast<uintptr_t>(in + i0) & 15) == 0)) {
            uint4 w = *reinterpret_cast<const uint4 *>(in + i0);
            v[c][0] = w.x; v[c][1] = w.y; v[c][2] = w.z; v[c][3] = w.w;
        } else {
#pragma unroll
            for (int j = 0; j < 4; ++j) v[c][j] = (i0 + j < n) ? in[i0 + j] : 0u;
        }
        uint64_t sum = (uint64_t)v[c][0] + v[c][1] + v[c][2] + v[c][3];
        uint64_t tot;
        texcl[c] = running + block_exclusive_scan<256, uint64_t>(sum, s_warp, &tot);
        running += tot;
    }
    if (threadIdx.x == 0) s_base = lookback_exclusive(status, tile, running, err);
    __syncthreads();
    const uint64_t tb = s_base;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const uint64_t i0 = base + (uint64_t)c * 1024 + threadIdx.x * 4;
        uint64_t x = tb + texcl[c];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (i0 + j < n) out[i0 + j] = (OutT)x;
            x += v[c][j];
        }
    }
    if (threadIdx.x == 0 && (uint64_t)tile == scan_tiles(n) - 1) *total = tb + running;
}

void launch_scan_u32_u64(const uint32_t *in, uint64_t *out, uint64_t n, uint64_t *status, uint32_t *tile_ctr,
                         uint64_t *total, uint32_t *err, cudaStream_t s) {
    if (n == 0) {
        cudaMemsetAsync(total, 0, sizeof(uint64_t), s);
        return;
    }
    count_launch();
    scan_kernel<uint64_t><<<(unsigned)scan_tiles(n), 256, 0, s>>>(in, out, n, status, tile_ctr, total, err);
}

void launch_scan_u32_u32(const uint32_t *in, uint32_t *out, uint64_t n, uint64_t *status, uint32_t *tile_ctr,
                         uint64_t *total, uint32_t *err, cudaStream_t s) {
    if (n == 0) {
        cudaMemsetAsync(total, 0, sizeof(uint64_t), s);
        return;
    }
    count_launch();
    scan_kernel<uint32_t><<<(unsigned)scan_tiles(n), 256, 0, s>>>(in, out, n, status, tile_ctr, total, err);
}

}  // namespace emp
