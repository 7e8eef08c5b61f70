// k_sort.cu -- stable onesweep LSD radix sort of (u64 fingerprint, u32 value)
// pairs by the 59-bit sort key  fp1:29 | fp2:29 | table:1  (common.cuh).
//
// Replaces the reference's thrust::sort_by_key calls on fingerprints
// (cqutils.cuh:163,195,213; in-core case of cq_sort_by_key 180-202), which
// are stable (CUB radix sort), so equal keys keep their input order.
//
// Structure (Adinets & Merrill, "Onesweep", 2022):
//   prepare  new epoch for the look-back words, tile tickets reset
//   hist     one read of the keys builds the histograms of all 8 digits
//   small    up to 4096 pairs: one CTA runs all 8 passes in shared memory
//   pass p   (more than 4096 pairs) one kernel per 8-bit digit.  A CTA turns
//            the digit histogram into bucket bases, then repeatedly takes
//            the next tile (atomic ticket, so every predecessor is already
//            running) and runs onesweep_tile on it (sort_block.cuh): stable
//            warp match-any ranking, per-digit decoupled look-back over
//            epoch-tagged words with bounded waits, reorder in shared
//            memory, one contiguous run per digit.
// The element count is read from device memory and no step needs the host,
// so a sort is a fixed sequence of launches (it can be captured in a graph).
#include <atomic>

#include "sort_block.cuh"

namespace emp {

static_assert(kSmallSort == kSortTile, "the small sort handles exactly one tile");

size_t sort_scratch_bytes(uint64_t n) {
    return sizeof(SortScratch) + (size_t)sort_tiles(n < 1 ? 1 : n) * kSortRadix * sizeof(uint64_t);
}

__global__ void __launch_bounds__(256) sort_prepare_kernel(SortScratch *sc, int zero_hist) {
    if (zero_hist)
        for (int i = threadIdx.x; i < kSortPasses * kSortRadix; i += blockDim.x) (&sc->hist[0][0])[i] = 0;
    if (threadIdx.x < kSortPasses) sc->tile_ctr[threadIdx.x] = 0;
    if (threadIdx.x == 0) sc->epoch = (sc->epoch + 1) & 0x1ffffu;
}

__global__ void __launch_bounds__(256) sort_hist_kernel(const uint64_t *__restrict__ keys,
                                                        const uint32_t *__restrict__ vals,
                                                        const uint64_t *__restrict__ n_dev, SortScratch *sc) {
    __shared__ uint32_t s_hist[kSortPasses][kSortRadix];
    const uint64_t n = *n_dev;
    if (n <= 1) return;
    for (int i = threadIdx.x; i < kSortPasses * kSortRadix; i += blockDim.x) (&s_hist[0][0])[i] = 0;
    __syncthreads();
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t sk = sort_key(keys[i], vals[i]);
#pragma unroll
        for (int p = 0; p < kSortPasses; ++p) atomicAdd(&s_hist[p][(sk >> (p * kSortBits)) & (kSortRadix - 1)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kSortPasses * kSortRadix; i += blockDim.x) {
        const uint32_t c = (&s_hist[0][0])[i];
        if (c) atomicAdd(&sc->hist[0][0] + i, c);
    }
}

// One CTA sorts up to kSmallSort pairs in place, all passes in shared memory.
__global__ void __launch_bounds__(kBlkThreads) small_sort_kernel(uint64_t *keys, uint32_t *vals,
                                                                 const uint64_t *__restrict__ n_dev) {
    extern __shared__ __align__(16) uint8_t smem[];
    const uint64_t n = *n_dev;
    if (n <= 1 || n > kSmallSort) return;
    block_sort(keys, vals, keys, vals, (uint32_t)n, 0, kSortPasses, smem);
}

__global__ void __launch_bounds__(kBlkThreads, 2) onesweep_kernel(
    const uint64_t *__restrict__ kin, const uint32_t *__restrict__ vin, uint64_t *__restrict__ kout,
    uint32_t *__restrict__ vout, const uint64_t *__restrict__ n_dev, int pass, SortScratch *sc,
    uint32_t *__restrict__ err) {
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ uint32_t s_bucket[kSortRadix];
    __shared__ uint32_t s_scan[32];
    __shared__ uint32_t s_tile;
    const uint64_t n = *n_dev;
    if (n <= kSmallSort) return;  // small_sort_kernel handled it
    const int tid = threadIdx.x;
    const uint64_t ntiles = sort_tiles(n);
    const int shift = pass * kSortBits;
    const uint32_t epoch = ((*(volatile uint32_t *)&sc->epoch) * kSortPasses + pass) & 0xfffffu;
    uint64_t *lookback = reinterpret_cast<uint64_t *>(sc + 1);
    {  // bucket bases of this digit from the histogram
        uint32_t tot;
        const uint32_t c = tid < kSortRadix ? sc->hist[pass][tid] : 0u;
        const uint32_t ex = block_exclusive_scan<kBlkThreads, uint32_t>(c, s_scan, &tot);
        if (tid < kSortRadix) s_bucket[tid] = ex;
    }
    for (;;) {
        if (tid == 0) s_tile = atomicAdd(&sc->tile_ctr[pass], 1u);
        __syncthreads();
        const uint32_t tile = s_tile;
        __syncthreads();
        if (tile >= ntiles) break;
        onesweep_tile(kin, vin, kout, vout, n, tile, shift, s_bucket, lookback, epoch, err, smem);
    }
}

// Persistent onesweep grid of a device: SMs x resident CTAs per SM.  Found
// once per device (the first call sets the kernels' shared-memory
// attributes) and kept in a per-device atomic, so host threads driving
// different devices neither race nor see each other's grid.
static unsigned sort_grid_find(int dev) {
    cudaFuncSetAttribute(onesweep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kOnesweepSmem);
    cudaFuncSetAttribute(small_sort_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBlockSortSmem);
    int sms = 148, occ = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, onesweep_kernel, kBlkThreads, kOnesweepSmem) !=
            cudaSuccess || occ < 1)
        occ = 1;
    cudaGetLastError();
    return (unsigned)(sms > 0 ? sms : 148) * (unsigned)occ;
}

static unsigned sort_setup() {
    constexpr int kDevs = 64;
    static std::atomic<unsigned> grid[kDevs] = {};  // 0: not found yet
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kDevs) {
        cudaGetLastError();
        return sort_grid_find(dev < 0 ? 0 : dev);
    }
    unsigned g = grid[dev].load(std::memory_order_acquire);
    if (g == 0) {
        g = sort_grid_find(dev);
        grid[dev].store(g, std::memory_order_release);
    }
    return g;
}

void launch_sort_prepare(SortScratch *sc, bool zero_hist, cudaStream_t s) {
    count_launch();
    sort_prepare_kernel<<<1, 256, 0, s>>>(sc, zero_hist ? 1 : 0);
}

static void launch_sort_body(uint64_t *k0, uint32_t *v0, uint64_t *k1, uint32_t *v1, const uint64_t *n_dev,
                             uint64_t n_max, SortScratch *sc, uint32_t *err, cudaStream_t s, cudaEvent_t *ev) {
    const uint64_t cap = sort_setup();
    const uint64_t tiles = sort_tiles(n_max < 1 ? 1 : n_max);
    const uint64_t hb = (n_max + 255) / 256;
    const unsigned hblocks = (unsigned)(hb < 1 ? 1 : (hb < 148 * 4 ? hb : 148 * 4));
    const unsigned grid = (unsigned)(tiles < cap ? tiles : cap);
    count_launch(2 + kSortPasses);
    sort_hist_kernel<<<hblocks, 256, 0, s>>>(k0, v0, n_dev, sc);
    small_sort_kernel<<<1, kBlkThreads, kBlockSortSmem, s>>>(k0, v0, n_dev);
    uint64_t *kb[2] = {k0, k1};
    uint32_t *vb[2] = {v0, v1};
    for (int p = 0; p < kSortPasses; ++p) {
        if (ev) cudaEventRecord(ev[2 * p], s);
        onesweep_kernel<<<grid, kBlkThreads, kOnesweepSmem, s>>>(kb[p & 1], vb[p & 1], kb[(p & 1) ^ 1],
                                                                 vb[(p & 1) ^ 1], n_dev, p, sc, err);
        if (ev) cudaEventRecord(ev[2 * p + 1], s);
    }
}

void sort_pairs_prepared(uint64_t *k0, uint32_t *v0, uint64_t *k1, uint32_t *v1, const uint64_t *n_dev,
                         uint64_t n_max, SortScratch *sc, uint32_t *err, cudaStream_t s) {
    launch_sort_body(k0, v0, k1, v1, n_dev, n_max, sc, err, s, nullptr);
}

int sort_pairs_dev(uint64_t *k0, uint32_t *v0, uint64_t *k1, uint32_t *v1, const uint64_t *n_dev, uint64_t n_max,
                   void *scratch, uint32_t *err, cudaStream_t s, cudaEvent_t *pass_events) {
    SortScratch *sc = reinterpret_cast<SortScratch *>(scratch);
    launch_sort_prepare(sc, true, s);
    launch_sort_body(k0, v0, k1, v1, n_dev, n_max, sc, err, s, pass_events);
    return 0;  // kSortPasses is even: the result is back in (k0, v0)
}

int sort_pairs(uint64_t *k0, uint32_t *v0, uint64_t *k1, uint32_t *v1, uint64_t n, void *scratch, uint64_t *n_dev,
               uint32_t *err, cudaStream_t s, cudaEvent_t *pass_events) {
    cudaMemcpyAsync(n_dev, &n, sizeof(uint64_t), cudaMemcpyHostToDevice, s);
    return sort_pairs_dev(k0, v0, k1, v1, n_dev, n, scratch, err, s, pass_events);
}

}  // namespace emp
