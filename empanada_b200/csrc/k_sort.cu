// k_sort.cu -- stable onesweep LSD radix sort of (u64 fingerprint, u32 value)
// pairs by the 59-bit sort key  fp1:29 | fp2:29 | table:1  (common.cuh).
//
// Replaces the reference's thrust::sort_by_key calls on fingerprints
// (cqutils.cuh:163,195,213; in-core case of cq_sort_by_key 180-202), which
// are stable (CUB radix sort), so equal keys keep their input order.
//
// Structure (Adinets & Merrill, "Onesweep", 2022):
//   hist     one read of the keys builds the histograms of all 8 digits
//   scan     exclusive prefix of each digit histogram (global bucket bases)
//   pass p   one kernel per 8-bit digit: a CTA takes the next tile (atomic
//            ticket, so predecessors are always running), ranks its 4096
//            pairs with warp match-any (stable), publishes its per-digit
//            counts, resolves the per-digit prefix of all earlier tiles by
//            decoupled look-back (bounded waits), reorders the tile in
//            shared memory and writes each digit's run contiguously.
#include "kernels.h"

namespace emp {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kItems = kSortTile / kSortThreads;  // 16
constexpr uint32_t kLbAgg = 1u << 30, kLbInc = 2u << 30, kLbVal = (1u << 30) - 1;

struct SortScratch {
    uint32_t hist[kSortPasses][kSortRadix];     // histogram, then exclusive bases
    uint32_t tile_ctr[kSortPasses];
    uint32_t pad[8];
    // followed by kSortPasses * tiles * kSortRadix look-back words
};

size_t sort_scratch_bytes(uint64_t n) {
    return sizeof(SortScratch) + (size_t)kSortPasses * sort_tiles(n) * kSortRadix * sizeof(uint32_t);
}

__global__ void __launch_bounds__(256) sort_hist_kernel(const uint64_t *__restrict__ keys,
                                                        const uint32_t *__restrict__ vals, uint64_t n,
                                                        uint32_t *__restrict__ hist) {
    __shared__ uint32_t s_hist[kSortPasses][kSortRadix];
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
        if (c) atomicAdd(hist + i, c);
    }
}

// one CTA per pass: histogram -> exclusive bases (in place)
__global__ void __launch_bounds__(256) sort_hist_scan_kernel(uint32_t *hist) {
    __shared__ uint32_t s_warp[8];
    uint32_t *h = hist + blockIdx.x * kSortRadix;
    const uint32_t v = h[threadIdx.x];
    uint32_t tot;
    const uint32_t ex = block_exclusive_scan<256, uint32_t>(v, s_warp, &tot);
    h[threadIdx.x] = ex;
}

EMP_DEV uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__global__ void __launch_bounds__(kSortThreads, 2) onesweep_kernel(
    const uint64_t *__restrict__ kin, const uint32_t *__restrict__ vin, uint64_t *__restrict__ kout,
    uint32_t *__restrict__ vout, uint64_t n, int shift, const uint32_t *__restrict__ bases,
    uint32_t *__restrict__ lookback, uint32_t *__restrict__ tile_ctr, uint32_t *__restrict__ err) {
    extern __shared__ __align__(16) uint8_t smem[];
    uint64_t *s_keys = reinterpret_cast<uint64_t *>(smem);
    uint32_t *s_vals = reinterpret_cast<uint32_t *>(s_keys + kSortTile);
    uint32_t *s_whist = s_vals + kSortTile;          // [warp][digit]
    uint32_t *s_texcl = s_whist + kSortWarps * kSortRadix;
    uint32_t *s_glob = s_texcl + kSortRadix;
    uint32_t *s_misc = s_glob + kSortRadix;           // [0] tile, [8..15] scan scratch

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_misc[0] = atomicAdd(tile_ctr, 1u);
    for (int i = tid; i < kSortWarps * kSortRadix; i += kSortThreads) s_whist[i] = 0;
    __syncthreads();
    const uint32_t tile = s_misc[0];
    const uint64_t base = (uint64_t)tile * kSortTile;

    uint64_t k[kItems];
    uint32_t v[kItems];
    uint32_t rank[kItems];
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const uint64_t idx = base + warp * (kItems * 32) + j * 32 + lane;
        if (idx < n) {
            k[j] = kin[idx];
            v[j] = vin[idx];
        } else {
            k[j] = 0;
            v[j] = 0;
        }
    }
    // stable warp-level ranking: element order (warp, j, lane)
    uint32_t *wh = s_whist + warp * kSortRadix;
    const uint32_t ltmask = lanemask_lt();
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const uint64_t idx = base + warp * (kItems * 32) + j * 32 + lane;
        const uint32_t d = idx < n ? (uint32_t)(sort_key(k[j], v[j]) >> shift) & (kSortRadix - 1) : kSortRadix;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const uint32_t before = __popc(peers & ltmask);
        const uint32_t prior = d < kSortRadix ? wh[d] : 0u;
        __syncwarp();
        if (d < kSortRadix && before == 0) wh[d] = prior + __popc(peers);
        __syncwarp();
        rank[j] = prior + before;
    }
    __syncthreads();
    // per digit (thread = digit): warp-exclusive offsets and tile count
    uint32_t cnt = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) {
        const uint32_t c = s_whist[w * kSortRadix + tid];
        s_whist[w * kSortRadix + tid] = cnt;
        cnt += c;
    }
    uint32_t *lb = lookback + (uint64_t)tile * kSortRadix + tid;
    *(volatile uint32_t *)lb = (tile == 0 ? kLbInc : kLbAgg) | cnt;
    uint32_t tot;
    const uint32_t dex = block_exclusive_scan<256, uint32_t>(cnt, s_misc + 8, &tot);
    s_texcl[tid] = dex;
    uint32_t excl = 0;
    if (tile > 0) {
        int64_t t = (int64_t)tile - 1;
        bool failed = false;
        while (t >= 0) {
            const volatile uint32_t *p = lookback + (uint64_t)t * kSortRadix + tid;
            uint32_t s;
            uint32_t spins = 0;
            while (((s = *p) >> 30) == 0) {
                if (++spins > kSpinLimit) {
                    failed = true;
                    break;
                }
                __nanosleep(32);
            }
            if (failed) {
                atomicOr(err, kErrSpin);
                break;
            }
            excl += s & kLbVal;
            if ((s >> 30) == 2) break;
            --t;
        }
        *(volatile uint32_t *)lb = kLbInc | (excl + cnt);
    }
    s_glob[tid] = bases[tid] + excl;
    __syncthreads();
    // reorder the tile in shared memory by digit (stable)
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const uint64_t idx = base + warp * (kItems * 32) + j * 32 + lane;
        if (idx < n) {
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
}

static size_t onesweep_smem() {
    return kSortTile * (sizeof(uint64_t) + sizeof(uint32_t)) + (kSortWarps + 2) * kSortRadix * sizeof(uint32_t) +
           16 * sizeof(uint32_t);
}

int sort_pairs(uint64_t *k0, uint32_t *v0, uint64_t *k1, uint32_t *v1, uint64_t n, void *scratch,
               uint32_t *hist_host, uint32_t *err, cudaStream_t s, cudaEvent_t *pass_events, uint32_t *passes_run) {
    cudaFuncSetAttribute(onesweep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)onesweep_smem());
    if (passes_run) *passes_run = 0;
    if (n < 2) return 0;
    SortScratch *sc = reinterpret_cast<SortScratch *>(scratch);
    uint32_t *lookback = reinterpret_cast<uint32_t *>(sc + 1);
    const uint64_t tiles = sort_tiles(n);
    cudaMemsetAsync(scratch, 0, sort_scratch_bytes(n), s);
    const uint64_t hb = (n + 255) / 256;
    const unsigned hblocks = (unsigned)(hb < 148 * 4 ? hb : 148 * 4);
    count_launch(2);
    sort_hist_kernel<<<hblocks, 256, 0, s>>>(k0, v0, n, &sc->hist[0][0]);
    bool skip[kSortPasses] = {false};
    if (hist_host) {
        cudaMemcpyAsync(hist_host, &sc->hist[0][0], sizeof(sc->hist), cudaMemcpyDeviceToHost, s);
        cudaStreamSynchronize(s);
        for (int p = 0; p < kSortPasses; ++p)
            for (int d = 0; d < kSortRadix; ++d)
                if (hist_host[p * kSortRadix + d] == n) skip[p] = true;
    }
    sort_hist_scan_kernel<<<kSortPasses, 256, 0, s>>>(&sc->hist[0][0]);
    int cur = 0;
    uint64_t *kb[2] = {k0, k1};
    uint32_t *vb[2] = {v0, v1};
    for (int p = 0; p < kSortPasses; ++p) {
        if (skip[p]) continue;
        count_launch();
        if (pass_events) cudaEventRecord(pass_events[2 * p], s);
        onesweep_kernel<<<(unsigned)tiles, kSortThreads, onesweep_smem(), s>>>(
            kb[cur], vb[cur], kb[cur ^ 1], vb[cur ^ 1], n, p * kSortBits, sc->hist[p],
            lookback + (uint64_t)p * tiles * kSortRadix, sc->tile_ctr + p, err);
        if (pass_events) cudaEventRecord(pass_events[2 * p + 1], s);
        if (passes_run) *passes_run |= 1u << p;
        cur ^= 1;
    }
    return cur;
}

}  // namespace emp
