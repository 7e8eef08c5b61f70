// sort_block.cuh -- block-level pieces of the stable LSD radix sort (k_sort.cu)
// and the shared helpers of the cooperative round kernel (k_bucket.cu).
// 512 threads per CTA, 8 pairs per thread, 4096-pair tiles.
#pragma once

#include "kernels.h"

namespace emp {

constexpr int kBlkThreads = 512;
constexpr int kBlkWarps = kBlkThreads / 32;
constexpr int kBlkItems = kSortTile / kBlkThreads;  // 8

EMP_DEV uint32_t lanemask_lt_u32() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

EMP_DEV uint32_t digit_of(uint64_t k, uint32_t v, int shift) {
    return (uint32_t)(sort_key(k, v) >> shift) & (kSortRadix - 1);
}

// Stable rank of each thread's 8 items within its warp (order: item j, lane);
// wh = this warp's 256 zeroed digit counters, left holding the warp's counts.
EMP_DEV void warp_rank8(const uint64_t (&k)[kBlkItems], const uint32_t (&v)[kBlkItems], const bool (&ok)[kBlkItems],
                        int shift, uint32_t *wh, uint32_t (&rank)[kBlkItems]) {
    const uint32_t ltmask = lanemask_lt_u32();
#pragma unroll
    for (int j = 0; j < kBlkItems; ++j) {
        const uint32_t d = ok[j] ? digit_of(k[j], v[j], shift) : kSortRadix;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const uint32_t before = __popc(peers & ltmask);
        const uint32_t prior = d < kSortRadix ? wh[d] : 0u;
        __syncwarp();
        if (d < kSortRadix && before == 0) wh[d] = prior + __popc(peers);
        __syncwarp();
        rank[j] = prior + before;
    }
}

// Shared memory of block_sort: two 4096-pair buffers, warp counters, scan room.
constexpr size_t kBlockSortSmem =
    2 * kSortTile * (sizeof(uint64_t) + sizeof(uint32_t)) + (kBlkWarps + 1) * kSortRadix * sizeof(uint32_t) +
    32 * sizeof(uint32_t);

// One CTA stably sorts n <= 4096 pairs (kin/vin -> kout/vout, which may alias)
// by the digits at shift0, shift0+8, ... (npasses of them).
EMP_DEV void block_sort(const uint64_t *kin, const uint32_t *vin, uint64_t *kout, uint32_t *vout, uint32_t n,
                        int shift0, int npasses, uint8_t *smem) {
    uint64_t *ak = reinterpret_cast<uint64_t *>(smem);
    uint64_t *bk = ak + kSortTile;
    uint32_t *av = reinterpret_cast<uint32_t *>(bk + kSortTile);
    uint32_t *bv = av + kSortTile;
    uint32_t *s_whist = bv + kSortTile;
    uint32_t *s_dex = s_whist + kBlkWarps * kSortRadix;
    uint32_t *s_scan = s_dex + kSortRadix;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (uint32_t i = tid; i < n; i += kBlkThreads) {
        ak[i] = __ldcg(kin + i);  // L2 only: the producer may be another SM of the same launch
        av[i] = __ldcg(vin + i);
    }
    for (int pass = 0; pass < npasses; ++pass) {
        const int shift = shift0 + pass * kSortBits;
        for (int i = tid; i < kBlkWarps * kSortRadix; i += kBlkThreads) s_whist[i] = 0;
        __syncthreads();
        uint64_t k[kBlkItems];
        uint32_t v[kBlkItems], rank[kBlkItems];
        bool ok[kBlkItems];
#pragma unroll
        for (int j = 0; j < kBlkItems; ++j) {
            const uint32_t e = warp * (kBlkItems * 32) + j * 32 + lane;
            ok[j] = e < n;
            k[j] = ok[j] ? ak[e] : 0;
            v[j] = ok[j] ? av[e] : 0;
        }
        warp_rank8(k, v, ok, shift, s_whist + warp * kSortRadix, rank);
        __syncthreads();
        uint32_t cnt = 0;
        if (tid < kSortRadix) {
#pragma unroll
            for (int w = 0; w < kBlkWarps; ++w) {
                const uint32_t c = s_whist[w * kSortRadix + tid];
                s_whist[w * kSortRadix + tid] = cnt;
                cnt += c;
            }
        }
        uint32_t tot;
        const uint32_t dex = block_exclusive_scan<kBlkThreads, uint32_t>(tid < kSortRadix ? cnt : 0u, s_scan, &tot);
        if (tid < kSortRadix) s_dex[tid] = dex;
        __syncthreads();
#pragma unroll
        for (int j = 0; j < kBlkItems; ++j) {
            if (ok[j]) {
                const uint32_t d = digit_of(k[j], v[j], shift);
                const uint32_t pos = s_dex[d] + s_whist[warp * kSortRadix + d] + rank[j];
                bk[pos] = k[j];
                bv[pos] = v[j];
            }
        }
        __syncthreads();
        uint64_t *tk = ak; ak = bk; bk = tk;
        uint32_t *tv = av; av = bv; bv = tv;
    }
    for (uint32_t i = tid; i < n; i += kBlkThreads) {
        kout[i] = ak[i];
        vout[i] = av[i];
    }
    __syncthreads();
}

constexpr uint32_t kRankSortMax = kBlkThreads;  // rank_sort handles up to one pair per thread
constexpr size_t kRankSortSmem = kRankSortMax * (2 * sizeof(uint64_t) + sizeof(uint32_t));

// One CTA stably sorts n <= 512 pairs by their full sort key: thread i counts
// the keys that precede its own (smaller, or equal and earlier) and writes its
// pair to that rank.  kout/vout may alias kin/vin.
EMP_DEV void rank_sort(const uint64_t *kin, const uint32_t *vin, uint64_t *kout, uint32_t *vout, uint32_t n,
                       uint8_t *smem) {
    uint64_t *sk = reinterpret_cast<uint64_t *>(smem);
    uint64_t *kk = sk + kRankSortMax;
    uint32_t *vv = reinterpret_cast<uint32_t *>(kk + kRankSortMax);
    const uint32_t tid = threadIdx.x;
    if (tid < n) {
        kk[tid] = __ldcg(kin + tid);
        vv[tid] = __ldcg(vin + tid);
        sk[tid] = sort_key(kk[tid], vv[tid]);
    }
    __syncthreads();
    if (tid < n) {
        const uint64_t my = sk[tid];
        uint32_t r = 0;
        for (uint32_t j = 0; j < n; ++j) {
            const uint64_t x = sk[j];
            r += (x < my) || (x == my && j < tid);
        }
        kout[r] = kk[tid];
        vout[r] = vv[tid];
    }
    __syncthreads();
}

// Shared memory of onesweep_tile: one 4096-pair tile, warp counters, digit
// offsets, and scan room.  `bucket` (256 words, caller-owned) holds the
// global bucket bases of the pass's digit.
constexpr size_t kOnesweepSmem = kSortTile * (sizeof(uint64_t) + sizeof(uint32_t)) +
                                 (kBlkWarps + 2) * kSortRadix * sizeof(uint32_t) + 32 * sizeof(uint32_t);

// One tile of one stable digit pass: rank, publish per-digit counts, resolve
// the prefix of earlier tiles by decoupled look-back (epoch-tagged words,
// bounded waits), reorder in shared memory, write each digit's run.
EMP_DEV void onesweep_tile(const uint64_t *__restrict__ kin, const uint32_t *__restrict__ vin,
                           uint64_t *__restrict__ kout, uint32_t *__restrict__ vout, uint64_t n, uint32_t tile,
                           int shift, const uint32_t *bucket, uint64_t *lookback, uint32_t epoch, uint32_t *err,
                           uint8_t *smem) {
    uint64_t *s_keys = reinterpret_cast<uint64_t *>(smem);
    uint32_t *s_vals = reinterpret_cast<uint32_t *>(s_keys + kSortTile);
    uint32_t *s_whist = s_vals + kSortTile;
    uint32_t *s_texcl = s_whist + kBlkWarps * kSortRadix;
    uint32_t *s_glob = s_texcl + kSortRadix;
    uint32_t *s_scan = s_glob + kSortRadix;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint64_t base = (uint64_t)tile * kSortTile;
    for (int i = tid; i < kBlkWarps * kSortRadix; i += kBlkThreads) s_whist[i] = 0;
    __syncthreads();
    uint64_t k[kBlkItems];
    uint32_t v[kBlkItems], rank[kBlkItems];
    bool ok[kBlkItems];
#pragma unroll
    for (int j = 0; j < kBlkItems; ++j) {
        const uint64_t idx = base + warp * (kBlkItems * 32) + j * 32 + lane;
        ok[j] = idx < n;
        k[j] = ok[j] ? __ldcg(kin + idx) : 0;  // L2 only (see block_sort)
        v[j] = ok[j] ? __ldcg(vin + idx) : 0;
    }
    warp_rank8(k, v, ok, shift, s_whist + warp * kSortRadix, rank);
    __syncthreads();
    uint32_t cnt = 0;
    if (tid < kSortRadix) {
#pragma unroll
        for (int w = 0; w < kBlkWarps; ++w) {
            const uint32_t c = s_whist[w * kSortRadix + tid];
            s_whist[w * kSortRadix + tid] = cnt;
            cnt += c;
        }
        st_status(lookback + (uint64_t)tile * kSortRadix + tid, ep_word(epoch, tile == 0 ? kEpInc : kEpAgg, cnt));
    }
    uint32_t tot;
    const uint32_t dex = block_exclusive_scan<kBlkThreads, uint32_t>(tid < kSortRadix ? cnt : 0u, s_scan, &tot);
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
        s_glob[tid] = bucket[tid] + (uint32_t)excl;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kBlkItems; ++j) {
        if (ok[j]) {
            const uint32_t d = digit_of(k[j], v[j], shift);
            const uint32_t pos = s_texcl[d] + s_whist[warp * kSortRadix + d] + rank[j];
            s_keys[pos] = k[j];
            s_vals[pos] = v[j];
        }
    }
    __syncthreads();
    const uint32_t valid = n - base < kSortTile ? (uint32_t)(n - base) : kSortTile;
    for (uint32_t i = tid; i < valid; i += kBlkThreads) {
        const uint64_t kk = s_keys[i];
        const uint32_t vv = s_vals[i];
        const uint32_t d = digit_of(kk, vv, shift);
        const uint64_t o = (uint64_t)s_glob[d] + (i - s_texcl[d]);
        kout[o] = kk;
        vout[o] = vv;
    }
    __syncthreads();
}

}  // namespace emp
