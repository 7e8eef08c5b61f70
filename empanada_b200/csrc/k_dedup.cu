// k_dedup.cu -- duplicate removal of the read-end fingerprints when they fit
// one chunk of the reference's sort (2n <= M).
//
// The reference sorts all (fingerprint, rid) pairs stably and keeps the first
// pair of every equal-key run (cq_sort_by_key + cq_unique_by_key,
// overlap.cu:212-225, cqutils.cuh:180-202,272-306): with the rids in
// increasing order before the stable sort, the survivor of a run is its
// smallest rid.  Only that survivor set matters here (the list is rebuilt in
// id order afterwards), so no sort is needed:
//
//   hist     per-CTA shared-memory histogram of the key buckets (the top
//            bits of fp1 scaled to nb buckets), added into global counts
//   (scan)   bucket starts, copied to the bucket cursors
//   scatter  each (key, rid) to its bucket: a CTA ranks a tile of keys per
//            bucket in shared memory and reserves each bucket's run with one
//            atomic (up to 2048 buckets), or one atomic per run of equal
//            buckets within a warp (more buckets, cursors rarely shared)
//   mark     one CTA per bucket: a shared-memory hash set of the bucket's
//            distinct keys holding the smallest rid of each (atomicMin),
//            then alive[rid] = (rid is its key's smallest)
//
// About 45 bytes move per read-end (a sort moves over 200).  A bucket whose
// distinct keys do not fit the hash set raises kErrDedupFull; the engine then
// falls back to the sort.
#include <atomic>

#include "sort_block.cuh"

namespace emp {
namespace {

constexpr int kDT = 256;                // threads per CTA
constexpr uint32_t kDedupSlots = 8192;  // hash slots of the mark kernel (power of two)
constexpr uint32_t kDedupFull = 7680;   // distinct keys of one bucket at most
constexpr uint64_t kDedupEmpty = ~0ull; // never a key: fp1, fp2 < 2^29

__device__ __forceinline__ uint32_t dedup_bucket(uint64_t key, uint32_t nb) {
    return (uint32_t)(((key >> 32) * (uint64_t)nb) >> 29);  // fp1 < 2^29
}

__global__ void __launch_bounds__(kDT) dedup_hist_kernel(const uint64_t *__restrict__ keys, uint64_t n,
                                                         uint32_t nb, uint32_t *__restrict__ counts) {
    extern __shared__ uint32_t s_hist[];  // nb
    for (uint32_t i = threadIdx.x; i < nb; i += kDT) s_hist[i] = 0;
    __syncthreads();
    for (uint64_t e = (uint64_t)blockIdx.x * kDT + threadIdx.x; e < n; e += (uint64_t)gridDim.x * kDT)
        atomicAdd(&s_hist[dedup_bucket(__ldg(keys + e), nb)], 1u);
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < nb; i += kDT)
        if (s_hist[i]) atomicAdd(counts + i, s_hist[i]);
}

// cursor[b] = start[b] (the exclusive scan of the counts)
__global__ void __launch_bounds__(kDT) dedup_cursor_kernel(const uint64_t *__restrict__ start, uint32_t nb,
                                                           uint32_t *__restrict__ cursor) {
    for (uint32_t b = blockIdx.x * kDT + threadIdx.x; b < nb; b += gridDim.x * kDT) cursor[b] = (uint32_t)start[b];
}

__global__ void __launch_bounds__(kDT) dedup_scatter_kernel(const uint64_t *__restrict__ keys, uint64_t n,
                                                            uint32_t nb, uint32_t *__restrict__ cursor,
                                                            uint64_t *__restrict__ pk, uint32_t *__restrict__ pr) {
    const uint64_t stride = (uint64_t)gridDim.x * kDT;
    for (uint64_t e0 = (uint64_t)blockIdx.x * kDT; e0 < n; e0 += stride) {  // uniform per warp
        const uint64_t e = e0 + threadIdx.x;
        const bool act = e < n;
        const uint64_t k = act ? __ldg(keys + e) : 0;
        const uint32_t b = act ? dedup_bucket(k, nb) : 0u;
        const uint32_t m = __ballot_sync(0xffffffffu, act);
        if (!act) continue;
        const uint32_t peers = __match_any_sync(m, b);
        const uint32_t lane = threadIdx.x & 31, leader = __ffs(peers) - 1;
        uint32_t pos = 0;
        if (lane == leader) pos = atomicAdd(cursor + b, (uint32_t)__popc(peers));
        pos = __shfl_sync(peers, pos, leader) + __popc(peers & lanemask_lt_u32());
        pk[pos] = k;
        pr[pos] = (uint32_t)e;
    }
}

// The same for few buckets (nb <= kTiledBuckets), where the bucket cursors
// would be hot: a CTA ranks a tile of kScatterTile keys per bucket in shared
// memory and reserves each bucket's run with one atomic.
constexpr uint32_t kTiledBuckets = 2048;
constexpr int kScatterPer = 16;
constexpr uint32_t kScatterTile = kDT * kScatterPer;

__global__ void __launch_bounds__(kDT) dedup_scatter_tiled_kernel(const uint64_t *__restrict__ keys, uint64_t n,
                                                                  uint32_t nb, uint32_t *__restrict__ cursor,
                                                                  uint64_t *__restrict__ pk,
                                                                  uint32_t *__restrict__ pr) {
    __shared__ uint32_t s_cnt[kTiledBuckets];
    for (uint64_t t0 = (uint64_t)blockIdx.x * kScatterTile; t0 < n; t0 += (uint64_t)gridDim.x * kScatterTile) {
        for (uint32_t b = threadIdx.x; b < nb; b += kDT) s_cnt[b] = 0;
        __syncthreads();
        uint64_t k[kScatterPer];
        uint32_t bk[kScatterPer], rk[kScatterPer];
#pragma unroll
        for (int q = 0; q < kScatterPer; ++q) {
            const uint64_t e = t0 + (uint64_t)q * kDT + threadIdx.x;
            k[q] = e < n ? __ldg(keys + e) : 0;
            bk[q] = e < n ? dedup_bucket(k[q], nb) : 0u;
            rk[q] = e < n ? atomicAdd(&s_cnt[bk[q]], 1u) : 0u;
        }
        __syncthreads();
        for (uint32_t b = threadIdx.x; b < nb; b += kDT) {
            const uint32_t c = s_cnt[b];
            s_cnt[b] = c ? atomicAdd(cursor + b, c) : 0u;  // the run's global start
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < kScatterPer; ++q) {
            const uint64_t e = t0 + (uint64_t)q * kDT + threadIdx.x;
            if (e >= n) continue;
            const uint32_t pos = s_cnt[bk[q]] + rk[q];
            pk[pos] = k[q];
            pr[pos] = (uint32_t)e;
        }
        __syncthreads();
    }
}

__device__ __forceinline__ uint32_t dedup_slot(uint64_t key) {
    return (uint32_t)((key * 0x9E3779B97F4A7C15ull) >> 40) & (kDedupSlots - 1);
}

constexpr size_t kMarkSmem = kDedupSlots * (8 + 4);

__global__ void __launch_bounds__(kDT) dedup_mark_hash_kernel(const uint64_t *__restrict__ pk,
                                                              const uint32_t *__restrict__ pr,
                                                              const uint64_t *__restrict__ start, uint32_t nb,
                                                              uint64_t n, uint8_t *__restrict__ alive,
                                                              uint32_t *err) {
    extern __shared__ __align__(16) uint8_t smem[];
    uint64_t *s_key = reinterpret_cast<uint64_t *>(smem);
    uint32_t *s_min = reinterpret_cast<uint32_t *>(s_key + kDedupSlots);
    __shared__ uint32_t s_used;
    for (uint32_t b = blockIdx.x; b < nb; b += gridDim.x) {
        for (uint32_t i = threadIdx.x; i < kDedupSlots; i += kDT) {
            s_key[i] = kDedupEmpty;
            s_min[i] = 0xffffffffu;
        }
        if (threadIdx.x == 0) s_used = 0;
        __syncthreads();
        const uint64_t lo = start[b], hi = b + 1 < nb ? start[b + 1] : n;
        bool full = false;
        for (uint64_t x = lo + threadIdx.x; x < hi; x += kDT) {  // smallest rid of every key
            const uint64_t k = pk[x];
            const uint32_t r = pr[x];
            uint32_t s = dedup_slot(k);
            for (uint32_t probes = 0; probes < kDedupSlots; ++probes) {
                const uint64_t old = atomicCAS(reinterpret_cast<unsigned long long *>(s_key + s),
                                               (unsigned long long)kDedupEmpty, (unsigned long long)k);
                if (old == kDedupEmpty && atomicAdd(&s_used, 1u) >= kDedupFull) full = true;
                if (old == kDedupEmpty || old == k) {
                    atomicMin(s_min + s, r);
                    break;
                }
                s = (s + 1) & (kDedupSlots - 1);
            }
        }
        if (__syncthreads_or(full)) {  // too many distinct keys: the engine sorts instead
            if (threadIdx.x == 0) atomicOr(err, kErrDedupFull);
            return;
        }
        for (uint64_t x = lo + threadIdx.x; x < hi; x += kDT) {  // survivors
            const uint64_t k = pk[x];
            const uint32_t r = pr[x];
            uint32_t s = dedup_slot(k);
            while (s_key[s] != k) s = (s + 1) & (kDedupSlots - 1);  // present: inserted above
            alive[r] = s_min[s] == r ? 1 : 0;
        }
        __syncthreads();
    }
}

}  // namespace

uint32_t dedup_buckets(uint64_t n) {
    if (n == 0 || n > kDedupMaxEnds) return 0;
    uint64_t nb = (n + kDedupMean - 1) / kDedupMean;
    return (uint32_t)(nb > kDedupMaxBuckets ? kDedupMaxBuckets : nb);
}

size_t dedup_scratch_bytes(uint32_t nb) { return (size_t)nb * (4 + 8 + 4) + 64; }

// Shared-memory attributes of the kernels, set once per device.
static bool dedup_setup(int &sms) {
    constexpr int kDevs = 64;
    static std::atomic<int> done[kDevs] = {};  // SM count, 0: not set up yet
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kDevs) {
        cudaGetLastError();
        return false;
    }
    sms = done[dev].load(std::memory_order_acquire);
    if (sms) return true;
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (cudaFuncSetAttribute(dedup_hist_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(kDedupMaxBuckets * 4)) != cudaSuccess ||
        cudaFuncSetAttribute(dedup_mark_hash_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMarkSmem) !=
            cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    sms = n > 0 ? n : 148;
    done[dev].store(sms, std::memory_order_release);
    return true;
}

bool launch_dedup_hash(const uint64_t *keys, uint64_t n, uint32_t nb, void *scratch, uint64_t *pk, uint32_t *pr,
                       uint8_t *alive, uint64_t *status, uint32_t *tile_ctr, uint64_t *total, uint32_t *err,
                       cudaStream_t s) {
    int sms = 0;
    if (!n || !nb || !dedup_setup(sms)) return false;
    uint32_t *counts = reinterpret_cast<uint32_t *>(scratch);
    uint64_t *start = reinterpret_cast<uint64_t *>(counts + ((nb + 1) & ~1u));
    uint32_t *cursor = reinterpret_cast<uint32_t *>(start + nb);
    cudaMemsetAsync(counts, 0, (size_t)nb * 4, s);
    const uint64_t per = (n + kDT - 1) / kDT;
    const unsigned g_hist = (unsigned)(per < (uint64_t)sms * 4 ? per : (uint64_t)sms * 4);
    count_launch(4);
    dedup_hist_kernel<<<g_hist, kDT, nb * 4, s>>>(keys, n, nb, counts);
    launch_scan_u32_u64(counts, start, nb, status, tile_ctr, total, err, s);
    dedup_cursor_kernel<<<(nb + kDT - 1) / kDT, kDT, 0, s>>>(start, nb, cursor);
    if (nb <= kTiledBuckets) {
        const uint64_t tiles = (n + kScatterTile - 1) / kScatterTile;
        const unsigned g_t = (unsigned)(tiles < (uint64_t)sms * 8 ? tiles : (uint64_t)sms * 8);
        dedup_scatter_tiled_kernel<<<g_t, kDT, 0, s>>>(keys, n, nb, cursor, pk, pr);
    } else {
        const unsigned g_sc = (unsigned)(per < (uint64_t)sms * 8 ? per : (uint64_t)sms * 8);
        dedup_scatter_kernel<<<g_sc, kDT, 0, s>>>(keys, n, nb, cursor, pk, pr);
    }
    const unsigned g_mark = nb < (uint32_t)sms * 2 ? nb : (uint32_t)sms * 2;
    dedup_mark_hash_kernel<<<g_mark, kDT, kMarkSmem, s>>>(pk, pr, start, nb, n, alive, err);
    return true;
}

}  // namespace emp
