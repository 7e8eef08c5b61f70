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
//            running), ranks its 4096 pairs with warp match-any (stable
//            order: warp, item, lane), publishes its per-digit counts,
//            resolves the per-digit prefix of all earlier tiles by decoupled
//            look-back over epoch-tagged words (bounded waits), reorders the
//            tile in shared memory and writes each digit's run contiguously.
// The element count is read from device memory and no step needs the host,
// so a sort is a fixed sequence of launches (it can be captured in a graph).
#include "kernels.h"

namespace emp {

constexpr int kSortThreads = 512;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kItems = kSortTile / kSortThreads;  // 8
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

EMP_DEV uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Stable rank of the 8 items of each thread within its warp (order: item j,
// lane) for digit `shift`; wh = this warp's 256 digit counters (zeroed).
EMP_DEV void warp_rank(const uint64_t (&k)[kItems], const uint32_t (&v)[kItems], const bool (&ok)[kItems], int shift,
                       uint32_t *wh, uint32_t (&rank)[kItems]) {
    const uint32_t ltmask = lanemask_lt();
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const uint32_t d = ok[j] ? (uint32_t)(sort_key(k[j], v[j]) >> shift) & (kSortRadix - 1) : kSortRadix;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const uint32_t before = __popc(peers & ltmask);
        const uint32_t prior = d < kSortRadix ? wh[d] : 0u;
        __syncwarp();
        if (d < kSortRadix && before == 0) wh[d] = prior + __popc(peers);
        __syncwarp();
        rank[j] = prior + before;
    }
}

// One CTA sorts up to kSmallSort pairs in place, all passes in shared memory.
__global__ void __launch_bounds__(kSortThreads) small_sort_kernel(uint64_t *__restrict__ keys,
                                                                  uint32_t *__restrict__ vals,
                                                                  const uint64_t *__restrict__ n_dev) {
    extern __shared__ __align__(16) uint8_t smem[];
    const uint64_t n64 = *n_dev;
    if (n64 <= 1 || n64 > kSmallSort) return;
    const uint32_t n = (uint32_t)n64;
    uint64_t *ak = reinterpret_cast<uint64_t *>(smem);
    uint64_t *bk = ak + kSmallSort;
    uint32_t *av = reinterpret_cast<uint32_t *>(bk + kSmallSort);
    uint32_t *bv = av + kSmallSort;
    uint32_t *s_whist = bv + kSmallSort;
    uint32_t *s_dex = s_whist + kSortWarps * kSortRadix;
    uint32_t *s_scan = s_dex + kSortRadix;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (uint32_t i = tid; i < n; i += kSortThreads) {
        ak[i] = keys[i];
        av[i] = vals[i];
    }
    for (int pass = 0; pass < kSortPasses; ++pass) {
        const int shift = pass * kSortBits;
        for (int i = tid; i < kSortWarps * kSortRadix; i += kSortThreads) s_whist[i] = 0;
        __syncthreads();
        uint64_t k[kItems];
        uint32_t v[kItems], rank[kItems];
        bool ok[kItems];
#pragma unroll
        for (int j = 0; j < kItems; ++j) {
            const uint32_t e = warp * (kItems * 32) + j * 32 + lane;
            ok[j] = e < n;
            k[j] = ok[j] ? ak[e] : 0;
            v[j] = ok[j] ? av[e] : 0;
        }
        warp_rank(k, v, ok, shift, s_whist + warp * kSortRadix, rank);
        __syncthreads();
        uint32_t cnt = 0;
        if (tid < kSortRadix) {
#pragma unroll
            for (int w = 0; w < kSortWarps; ++w) {
                const uint32_t c = s_whist[w * kSortRadix + tid];
                s_whist[w * kSortRadix + tid] = cnt;
                cnt += c;
            }
        }
        uint32_t tot;
        const uint32_t dex = block_exclusive_scan<kSortThreads, uint32_t>(tid < kSortRadix ? cnt : 0u, s_scan, &tot);
        if (tid < kSortRadix) s_dex[tid] = dex;
        __syncthreads();
#pragma unroll
        for (int j = 0; j < kItems; ++j) {
            if (ok[j]) {
                const uint32_t d = (uint32_t)(sort_key(k[j], v[j]) >> shift) & (kSortRadix - 1);
                const uint32_t pos = s_dex[d] + s_whist[warp * kSortRadix + d] + rank[j];
                bk[pos] = k[j];
                bv[pos] = v[j];
            }
        }
        __syncthreads();
        uint64_t *tk = ak; ak = bk; bk = tk;
        uint32_t *tv = av; av = bv; bv = tv;
    }
    for (uint32_t i = tid; i < n; i += kSortThreads) {
        keys[i] = ak[i];
        vals[i] = av[i];
    }
}

__global__ void __launch_bounds__(kSortThreads, 2) onesweep_kernel(
    const uint64_t *__restrict__ kin, const uint32_t *__restrict__ vin, uint64_t *__restrict__ kout,
    uint32_t *__restrict__ vout, const uint64_t *__restrict__ n_dev, int pass, SortScratch *sc,
    uint32_t *__restrict__ err) {
    extern __shared__ __align__(16) uint8_t smem[];
    uint64_t *s_keys = reinterpret_cast<uint64_t *>(smem);
    uint32_t *s_vals = reinterpret_cast<uint32_t *>(s_keys + kSortTile);
    uint32_t *s_whist = s_vals + kSortTile;          // [warp][digit]
    uint32_t *s_texcl = s_whist + kSortWarps * kSortRadix;
    uint32_t *s_glob = s_texcl + kSortRadix;
    uint32_t *s_bucket = s_glob + kSortRadix;         // global bucket base of each digit
    uint32_t *s_misc = s_bucket + kSortRadix;         // [0] tile, [16..31] scan scratch

    const uint64_t n = *n_dev;
    if (n <= kSmallSort) return;  // small_sort_kernel handled it
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint64_t ntiles = sort_tiles(n);
    const int shift = pass * kSortBits;
    const uint32_t epoch = ((*(volatile uint32_t *)&sc->epoch) * kSortPasses + pass) & 0xfffffu;
    uint64_t *lookback = reinterpret_cast<uint64_t *>(sc + 1);
    {  // bucket bases of this digit from the histogram
        uint32_t tot;
        const uint32_t c = tid < kSortRadix ? sc->hist[pass][tid] : 0u;
        const uint32_t ex = block_exclusive_scan<kSortThreads, uint32_t>(c, s_misc + 16, &tot);
        if (tid < kSortRadix) s_bucket[tid] = ex;
    }

    for (;;) {
        if (tid == 0) s_misc[0] = atomicAdd(&sc->tile_ctr[pass], 1u);
        for (int i = tid; i < kSortWarps * kSortRadix; i += kSortThreads) s_whist[i] = 0;
        __syncthreads();
        const uint32_t tile = s_misc[0];
        if (tile >= ntiles) break;
        const uint64_t base = (uint64_t)tile * kSortTile;

        uint64_t k[kItems];
        uint32_t v[kItems], rank[kItems];
        bool ok[kItems];
#pragma unroll
        for (int j = 0; j < kItems; ++j) {
            const uint64_t idx = base + warp * (kItems * 32) + j * 32 + lane;
            ok[j] = idx < n;
            k[j] = ok[j] ? kin[idx] : 0;
            v[j] = ok[j] ? vin[idx] : 0;
        }
        warp_rank(k, v, ok, shift, s_whist + warp * kSortRadix, rank);
        __syncthreads();
        // per digit (threads 0..255): warp-exclusive offsets, tile count, publish
        uint32_t cnt = 0;
        if (tid < kSortRadix) {
#pragma unroll
            for (int w = 0; w < kSortWarps; ++w) {
                const uint32_t c = s_whist[w * kSortRadix + tid];
                s_whist[w * kSortRadix + tid] = cnt;
                cnt += c;
            }
            st_status(lookback + (uint64_t)tile * kSortRadix + tid,
                      ep_word(epoch, tile == 0 ? kEpInc : kEpAgg, cnt));
        }
        uint32_t tot;
        const uint32_t dex = block_exclusive_scan<kSortThreads, uint32_t>(tid < kSortRadix ? cnt : 0u, s_misc + 16,
                                                                          &tot);
        if (tid < kSortRadix) {
            s_texcl[tid] = dex;
            uint64_t excl = 0;
            if (tile > 0) {
                int64_t t = (int64_t)tile - 1;
                bool done = false;
                while (t >= 0 && !done) {
                    const int kk = t >= 3 ? 4 : (int)t + 1;
                    uint64_t w[4];
#pragma unroll
                    for (int i = 0; i < 4; ++i)
                        if (i < kk) w[i] = ld_status(lookback + (uint64_t)(t - i) * kSortRadix + tid);
                    for (int i = 0; i < kk && !done; ++i) {
                        uint32_t f, spins = 0;
                        while ((f = ep_flag(w[i], epoch)) == 0) {
                            if (++spins > kSpinLimit) {
                                atomicOr(err, kErrSpin);
                                done = true;
                                break;
                            }
                            if (spins > 32) __nanosleep(32);
                            w[i] = ld_status(lookback + (uint64_t)(t - i) * kSortRadix + tid);
                        }
                        if (done) break;
                        excl += w[i] & kEpVal;
                        done = f == 2;
                    }
                    t -= kk;
                }
                st_status(lookback + (uint64_t)tile * kSortRadix + tid, ep_word(epoch, kEpInc, excl + cnt));
            }
            s_glob[tid] = s_bucket[tid] + (uint32_t)excl;
        }
        __syncthreads();
        // reorder the tile in shared memory by digit (stable)
#pragma unroll
        for (int j = 0; j < kItems; ++j) {
            if (ok[j]) {
                const uint32_t d = (uint32_t)(sort_key(k[j], v[j]) >> shift) & (kSortRadix - 1);
                const uint32_t pos = s_texcl[d] + s_whist[warp * kSortRadix + d] + rank[j];
                s_keys[pos] = k[j];
                s_vals[pos] = v[j];
            }
        }
        __syncthreads();
        const uint32_t valid = n - base < kSortTile ? (uint32_t)(n - base) : kSortTile;
        for (uint32_t i = tid; i < valid; i += kSortThreads) {
            const uint64_t kk = s_keys[i];
            const uint32_t vv = s_vals[i];
            const uint32_t d = (uint32_t)(sort_key(kk, vv) >> shift) & (kSortRadix - 1);
            const uint64_t o = (uint64_t)s_glob[d] + (i - s_texcl[d]);
            kout[o] = kk;
            vout[o] = vv;
        }
        __syncthreads();
    }
}

static size_t onesweep_smem() {
    return kSortTile * (sizeof(uint64_t) + sizeof(uint32_t)) + (kSortWarps + 3) * kSortRadix * sizeof(uint32_t) +
           32 * sizeof(uint32_t);
}
static size_t small_sort_smem() {
    return 2 * kSmallSort * (sizeof(uint64_t) + sizeof(uint32_t)) + (kSortWarps + 1) * kSortRadix * sizeof(uint32_t) +
           32 * sizeof(uint32_t);
}

static int g_setup_device = -1;
static int g_sm_count = 148;
static int onesweep_ctas_per_sm = 2;

static void sort_setup() {
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev == g_setup_device) return;
    cudaFuncSetAttribute(onesweep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)onesweep_smem());
    cudaFuncSetAttribute(small_sort_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)small_sort_smem());
    cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, dev);
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, onesweep_kernel, kSortThreads, onesweep_smem()) ==
            cudaSuccess && occ > 0)
        onesweep_ctas_per_sm = occ;
    cudaGetLastError();
    g_setup_device = dev;
}

void launch_sort_prepare(SortScratch *sc, bool zero_hist, cudaStream_t s) {
    count_launch();
    sort_prepare_kernel<<<1, 256, 0, s>>>(sc, zero_hist ? 1 : 0);
}

void sort_pairs_prepared(uint64_t *k0, uint32_t *v0, uint64_t *k1, uint32_t *v1, const uint64_t *n_dev,
                         uint64_t n_max, SortScratch *sc, uint32_t *err, cudaStream_t s) {
    sort_setup();
    const uint64_t tiles = sort_tiles(n_max < 1 ? 1 : n_max);
    const uint64_t hb = (n_max + 255) / 256;
    const unsigned hblocks = (unsigned)(hb < 1 ? 1 : (hb < 148 * 4 ? hb : 148 * 4));
    const uint64_t cap = (uint64_t)g_sm_count * onesweep_ctas_per_sm;
    const unsigned grid = (unsigned)(tiles < cap ? tiles : cap);
    count_launch(2 + kSortPasses);
    sort_hist_kernel<<<hblocks, 256, 0, s>>>(k0, v0, n_dev, sc);
    small_sort_kernel<<<1, kSortThreads, small_sort_smem(), s>>>(k0, v0, n_dev);
    uint64_t *kb[2] = {k0, k1};
    uint32_t *vb[2] = {v0, v1};
    for (int p = 0; p < kSortPasses; ++p)
        onesweep_kernel<<<grid, kSortThreads, onesweep_smem(), s>>>(kb[p & 1], vb[p & 1], kb[(p & 1) ^ 1],
                                                                    vb[(p & 1) ^ 1], n_dev, p, sc, err);
}

int sort_pairs_dev(uint64_t *k0, uint32_t *v0, uint64_t *k1, uint32_t *v1, const uint64_t *n_dev, uint64_t n_max,
                   void *scratch, uint32_t *err, cudaStream_t s, cudaEvent_t *pass_events) {
    sort_setup();
    SortScratch *sc = reinterpret_cast<SortScratch *>(scratch);
    launch_sort_prepare(sc, true, s);
    if (!pass_events) {
        sort_pairs_prepared(k0, v0, k1, v1, n_dev, n_max, sc, err, s);
        return 0;
    }
    // the same launches, with events bracketing each digit pass
    const uint64_t tiles = sort_tiles(n_max < 1 ? 1 : n_max);
    const uint64_t hb = (n_max + 255) / 256;
    const unsigned hblocks = (unsigned)(hb < 1 ? 1 : (hb < 148 * 4 ? hb : 148 * 4));
    const uint64_t cap = (uint64_t)g_sm_count * onesweep_ctas_per_sm;
    const unsigned grid = (unsigned)(tiles < cap ? tiles : cap);
    count_launch(2 + kSortPasses);
    sort_hist_kernel<<<hblocks, 256, 0, s>>>(k0, v0, n_dev, sc);
    small_sort_kernel<<<1, kSortThreads, small_sort_smem(), s>>>(k0, v0, n_dev);
    uint64_t *kb[2] = {k0, k1};
    uint32_t *vb[2] = {v0, v1};
    for (int p = 0; p < kSortPasses; ++p) {
        cudaEventRecord(pass_events[2 * p], s);
        onesweep_kernel<<<grid, kSortThreads, onesweep_smem(), s>>>(kb[p & 1], vb[p & 1], kb[(p & 1) ^ 1],
                                                                    vb[(p & 1) ^ 1], n_dev, p, sc, err);
        cudaEventRecord(pass_events[2 * p + 1], s);
    }
    return 0;  // kSortPasses is even: the result is back in (k0, v0)
}

int sort_pairs(uint64_t *k0, uint32_t *v0, uint64_t *k1, uint32_t *v1, uint64_t n, void *scratch, uint64_t *n_dev,
               uint32_t *err, cudaStream_t s, cudaEvent_t *pass_events) {
    cudaMemcpyAsync(n_dev, &n, sizeof(uint64_t), cudaMemcpyHostToDevice, s);
    return sort_pairs_dev(k0, v0, k1, v1, n_dev, n, scratch, err, s, pass_events);
}

}  // namespace emp
