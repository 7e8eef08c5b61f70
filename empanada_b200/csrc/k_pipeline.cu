// k_pipeline.cu -- the overlap rounds as a device-resident pipeline.
//
// One round (overlap.cu:258-290) is a fixed sequence of launches that read
// every size from a RoundCtl word block in device memory, so the host issues
// all rounds without waiting (and can replay one round as a CUDA graph):
//
//   update_filter  drop ids used in the previous round (remove_used,
//                  overlap.cu:694-710), apply NextSfx / PrevPfx with the
//                  2-bit column store (regenerate_fingerprints + filter_bases,
//                  overlap.cu:605-692), compact the id-ordered list, and set
//                  two Bloom bits per surviving key in its table's filter
//   candidates     keep, in list order, the entries whose key may occur in
//                  the other table (both Bloom bits set there)
//   sort           onesweep radix sort of the candidates only (k_sort.cu)
//   join_count / scan / join_write
//                  equal-key runs of the sorted candidates -> edges at the
//                  running edge offset, used-id marks
//   round_end      bookkeeping: per-round record (S, P, E), loop exit when
//                  the suffix table is empty or all L-o rounds ran
//
// Only candidates are sorted.  An entry that is not a candidate has no equal
// key in the other table and takes part in no edge; the sort is stable and
// sees the candidates in list order, so the relative order of every matching
// entry -- and hence the edge order of get_edges (overlap.cu:557-603) -- is
// exactly that of the reference's full sort.
#include "kernels.h"

namespace emp {

constexpr int kChunks = kUpdTile / 256;  // 8

EMP_DEV uint32_t pl_column_code(const uint32_t *__restrict__ cols, uint64_t wpc, int col, uint32_t i) {
    return (__ldg(cols + (uint64_t)col * wpc + (i >> 4)) >> ((i & 15u) * 2u)) & 3u;
}

// two Bloom-filter bit positions from one multiplicative hash of the key
EMP_DEV void bloom_bits(uint64_t key, int bits, uint32_t &h1, uint32_t &h2) {
    const uint64_t x = key * 0x9E3779B97F4A7C15ull;
    h1 = (uint32_t)(x >> (64 - bits));
    h2 = (uint32_t)((x >> (64 - 2 * bits)) & ((1ull << bits) - 1));
}

EMP_DEV bool bloom_test(const uint32_t *__restrict__ bm, uint64_t key, int bits) {
    uint32_t h1, h2;
    bloom_bits(key, bits, h1, h2);
    return ((__ldcg(bm + (h1 >> 5)) >> (h1 & 31)) & 1u) && ((__ldcg(bm + (h2 >> 5)) >> (h2 & 31)) & 1u);
}

__global__ void __launch_bounds__(256) pl_update_filter_kernel(PipeArgs a) {
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_warp[8];
    __shared__ uint64_t s_base;
    __shared__ uint32_t s_sfx;
    RoundCtl *ctl = a.ctl;
    if (*(volatile uint32_t *)&ctl->done) return;
    const uint64_t n_in = ctl->n;
    const uint32_t cur = ctl->cur;
    const int L = a.L, r = (int)ctl->round;
    const int bits = (int)ctl->bloom_bits;
    const uint32_t epoch = (uint32_t)(r + 1) * 4u + 0u;
    const uint64_t *kin = cur ? a.lk1 : a.lk0;
    const uint32_t *vin = cur ? a.lv1 : a.lv0;
    uint64_t *kout = cur ? a.lk0 : a.lk1;
    uint32_t *vout = cur ? a.lv0 : a.lv1;
    const int cf = r, cb = L - 1 - r;
    const uint32_t pw1 = a.tables->pow1[L - r - 1], pw2 = a.tables->pow2[L - r - 1];
    const uint32_t inv1 = a.tables->inv1, inv2 = a.tables->inv2;
    const uint64_t ntiles = upd_tiles(n_in);
    for (;;) {
        if (threadIdx.x == 0) {
            s_tile = atomicAdd(&ctl->tile_ctr[0], 1u);
            s_sfx = 0;
        }
        __syncthreads();
        const uint32_t tile = s_tile;
        if (tile >= ntiles) break;
        const uint64_t base = (uint64_t)tile * kUpdTile;
        uint64_t key[kChunks];
        uint32_t val[kChunks], ex[kChunks];
        bool keep[kChunks];
        uint32_t running = 0, sfx_kept = 0;
#pragma unroll
        for (int c = 0; c < kChunks; ++c) {
            const uint64_t e = base + c * 256 + threadIdx.x;
            keep[c] = false;
            key[c] = 0;
            val[c] = 0;
            if (e < n_in) {
                uint64_t k = kin[e];
                const uint32_t v = vin[e];
                const uint32_t rid = v & 0x7fffffffu, t = v >> 31, s = rid & 1u, i = rid >> 1;
                const bool used = t ? a.used_p[rid] : a.used_s[rid];
                if (!used) {
                    const int col = t == 0 ? (s ? cb : cf) : (s ? cf : cb);
                    const uint32_t b = pl_column_code(a.cols, a.wpc, col, i) ^ (s << 1);
                    k = t == 0 ? next_sfx(k, b, pw1, pw2) : prev_pfx(k, b, inv1, inv2);
                    keep[c] = true;
                    sfx_kept += t == 0;
                    uint32_t h1, h2;
                    bloom_bits(k, bits, h1, h2);
                    uint32_t *bm = t ? a.bloom_p : a.bloom_s;
                    atomicOr(bm + (h1 >> 5), 1u << (h1 & 31));
                    atomicOr(bm + (h2 >> 5), 1u << (h2 & 31));
                }
                key[c] = k;
                val[c] = v;
            }
            uint32_t tot;
            ex[c] = running + block_exclusive_scan<256, uint32_t>(keep[c] ? 1u : 0u, s_warp, &tot);
            running += tot;
        }
        if (sfx_kept) atomicAdd(&s_sfx, sfx_kept);
        if (threadIdx.x < 32) {
            const uint64_t b = lookback_epoch_warp(a.st_upd, tile, running, epoch, a.err);
            if (threadIdx.x == 0) s_base = b;
        }
        __syncthreads();
#pragma unroll
        for (int c = 0; c < kChunks; ++c) {
            if (keep[c]) {
                const uint64_t o = s_base + ex[c];
                kout[o] = key[c];
                vout[o] = val[c];
            }
        }
        if (threadIdx.x == 0) {
            if (s_sfx) atomicAdd(reinterpret_cast<unsigned long long *>(&ctl->s_next), (unsigned long long)s_sfx);
            if ((uint64_t)tile == ntiles - 1) ctl->n_next = s_base + running;
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256) pl_candidates_kernel(PipeArgs a) {
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_warp[8];
    __shared__ uint64_t s_base;
    RoundCtl *ctl = a.ctl;
    if (*(volatile uint32_t *)&ctl->done) return;
    const uint64_t n = ctl->n_next;
    if (ctl->s_next == 0 || ctl->s_next == n) return;  // one table empty: no edge this round
    const int bits = (int)ctl->bloom_bits;
    const uint32_t cur = ctl->cur;
    const uint64_t *kin = cur ? a.lk0 : a.lk1;  // the list update_filter just wrote
    const uint32_t *vin = cur ? a.lv0 : a.lv1;
    const uint32_t epoch = (ctl->round + 1) * 4u + 1u;
    const uint64_t ntiles = upd_tiles(n);
    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(&ctl->tile_ctr[1], 1u);
        __syncthreads();
        const uint32_t tile = s_tile;
        if (tile >= ntiles) break;
        const uint64_t base = (uint64_t)tile * kUpdTile;
        uint64_t key[kChunks];
        uint32_t val[kChunks], ex[kChunks];
        bool cand[kChunks];
        uint32_t running = 0;
#pragma unroll
        for (int c = 0; c < kChunks; ++c) {
            const uint64_t e = base + c * 256 + threadIdx.x;
            cand[c] = false;
            key[c] = 0;
            val[c] = 0;
            if (e < n) {
                key[c] = kin[e];
                val[c] = vin[e];
                cand[c] = bloom_test((val[c] >> 31) ? a.bloom_s : a.bloom_p, key[c], bits);
            }
            uint32_t tot;
            ex[c] = running + block_exclusive_scan<256, uint32_t>(cand[c] ? 1u : 0u, s_warp, &tot);
            running += tot;
        }
        if (threadIdx.x < 32) {
            const uint64_t b = lookback_epoch_warp(a.st_cand, tile, running, epoch, a.err);
            if (threadIdx.x == 0) s_base = b;
        }
        __syncthreads();
#pragma unroll
        for (int c = 0; c < kChunks; ++c) {
            if (cand[c]) {
                const uint64_t o = s_base + ex[c];
                a.ck[o] = key[c];
                a.cv[o] = val[c];
            }
        }
        if (threadIdx.x == 0 && (uint64_t)tile == ntiles - 1) ctl->c = s_base + running;
        __syncthreads();
    }
}

// Also clears this round's Bloom filters (the candidates kernel was their last
// reader) so that the next round starts from empty filters.
__global__ void pl_join_count_kernel(PipeArgs a) {
    if (!*(volatile uint32_t *)&a.ctl->done) {
        const uint64_t words = (1ull << a.ctl->bloom_bits) >> 5;
        for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < words;
             i += (uint64_t)gridDim.x * blockDim.x) {
            a.bloom_s[i] = 0;
            a.bloom_p[i] = 0;
        }
    }
    const uint64_t n = a.ctl->c;
    const uint64_t *k = a.ck;
    const uint32_t *v = a.cv;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t vi = v[i];
        uint32_t c = 0;
        if ((vi >> 31) == 0) {
            const uint64_t ki = k[i];
            const uint32_t ri = (vi & 0x7fffffffu) >> 1;
            for (uint64_t j = i + 1; j < n && k[j] == ki; ++j) {
                const uint32_t vj = v[j];
                if ((vj >> 31) && ((vj & 0x7fffffffu) >> 1) != ri) ++c;
            }
        }
        a.cnt[i] = c;
    }
}

// exclusive scan of cnt[0..c) into offs; c and the round's edge count live in ctl
__global__ void __launch_bounds__(256) pl_scan_kernel(PipeArgs a) {
    __shared__ uint32_t s_tile;
    __shared__ uint64_t s_warp[8];
    __shared__ uint64_t s_base;
    RoundCtl *ctl = a.ctl;
    const uint64_t n = ctl->c;
    if (n == 0) return;
    const uint32_t epoch = (ctl->round + 1) * 4u + 2u;
    const uint64_t ntiles = scan_tiles(n);
    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(&ctl->tile_ctr[2], 1u);
        __syncthreads();
        const uint32_t tile = s_tile;
        if (tile >= ntiles) break;
        const uint64_t base = (uint64_t)tile * kScanTile;
        uint32_t v[4][4];
        uint64_t texcl[4];
        uint64_t running = 0;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const uint64_t i0 = base + (uint64_t)c * 1024 + threadIdx.x * 4;
#pragma unroll
            for (int j = 0; j < 4; ++j) v[c][j] = (i0 + j < n) ? a.cnt[i0 + j] : 0u;
            const uint64_t sum = (uint64_t)v[c][0] + v[c][1] + v[c][2] + v[c][3];
            uint64_t tot;
            texcl[c] = running + block_exclusive_scan<256, uint64_t>(sum, s_warp, &tot);
            running += tot;
        }
        if (threadIdx.x < 32) {
            const uint64_t b = lookback_epoch_warp(a.st_scan, tile, running, epoch, a.err);
            if (threadIdx.x == 0) s_base = b;
        }
        __syncthreads();
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const uint64_t i0 = base + (uint64_t)c * 1024 + threadIdx.x * 4;
            uint64_t x = s_base + texcl[c];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (i0 + j < n) a.offs[i0 + j] = x;
                x += v[c][j];
            }
        }
        if (threadIdx.x == 0 && (uint64_t)tile == ntiles - 1) ctl->e_round = s_base + running;
        __syncthreads();
    }
}

__global__ void pl_join_write_kernel(PipeArgs a) {
    RoundCtl *ctl = a.ctl;
    const uint64_t n = ctl->c;
    const uint64_t ebase = ctl->e_total;
    if (ebase + ctl->e_round > a.ecap) {
        if (blockIdx.x == 0 && threadIdx.x == 0) ctl->overflow = 1;
    }
    const uint64_t *k = a.ck;
    const uint32_t *v = a.cv;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        if (!a.cnt[i]) continue;
        const uint64_t ki = k[i];
        const uint32_t si = v[i] & 0x7fffffffu, ri = si >> 1;
        uint64_t o = ebase + a.offs[i];
        for (uint64_t j = i + 1; j < n && k[j] == ki; ++j) {
            const uint32_t vj = v[j];
            const uint32_t pj = vj & 0x7fffffffu;
            if ((vj >> 31) && (pj >> 1) != ri) {
                if (o < a.ecap) {
                    a.efrom[o] = si;
                    a.eto[o] = pj;
                }
                a.used_p[pj] = 1;
                ++o;
            }
        }
        a.used_s[si] = 1;
    }
}

// log2 of the Bloom filter size for a round over n entries (32 bits per
// entry of the larger table, which holds at most n entries), capped.
EMP_DEV uint32_t bloom_bits_for_n(uint64_t n, int max_bits) {
    uint32_t b = 16;
    while ((int)b < max_bits && (1ull << b) < 16 * n) ++b;
    return b;
}

// Round bookkeeping, then the next round's preparation: Bloom filter size,
// candidate-sort scratch (histogram, tickets, look-back epoch).
__global__ void __launch_bounds__(256) pl_round_end_kernel(PipeArgs a) {
    RoundCtl *ctl = a.ctl;
    if (threadIdx.x == 0 && !ctl->done) {
        const uint64_t S = ctl->s_next, P = ctl->n_next - ctl->s_next;
        const uint32_t r = ctl->round;
        if (S == 0) {
            ctl->done = 1;  // build_graph's loop condition: no suffix left
        } else {
            const uint64_t E = P ? ctl->e_round : 0;
            RoundRecord &rec = a.records[r];
            rec.S = S;
            rec.P = P;
            rec.E = E;
            rec.e0 = ctl->e_total;
            ctl->e_total += E;
            ctl->n = ctl->n_next;
            ctl->s = S;
            ctl->cur ^= 1u;
            ctl->round = r + 1;
            ctl->bloom_bits = bloom_bits_for_n(ctl->n_next, a.bloom_bits_max);
            if (r + 1 >= ctl->rounds) ctl->done = 1;
        }
        ctl->n_next = 0;
        ctl->s_next = 0;
        ctl->c = 0;
        ctl->e_round = 0;
    }
    for (int i = threadIdx.x; i < kSortPasses * kSortRadix; i += blockDim.x) (&a.sort->hist[0][0])[i] = 0;
    if (threadIdx.x < kSortPasses) a.sort->tile_ctr[threadIdx.x] = 0;
    if (threadIdx.x == 0) a.sort->epoch = (a.sort->epoch + 1) & 0x1ffffu;
    if (threadIdx.x < 8) ctl->tile_ctr[threadIdx.x] = 0;
}

static unsigned persistent_grid(uint64_t tiles, unsigned cap) {
    return (unsigned)(tiles < 1 ? 1 : (tiles < cap ? tiles : cap));
}

void launch_pipeline_round(const PipeArgs &a, uint64_t n_max, uint64_t cand_max, cudaStream_t s,
                           cudaEvent_t *upd_events) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const unsigned gu = persistent_grid(upd_tiles(n_max), (unsigned)sms * 8);
    count_launch(6);
    // External: inside a stream capture these become event-record nodes (timestamps)
    if (upd_events) cudaEventRecordWithFlags(upd_events[0], s, cudaEventRecordExternal);
    pl_update_filter_kernel<<<gu, 256, 0, s>>>(a);
    if (upd_events) cudaEventRecordWithFlags(upd_events[1], s, cudaEventRecordExternal);
    pl_candidates_kernel<<<gu, 256, 0, s>>>(a);
    sort_pairs_prepared(a.ck, a.cv, a.ck2, a.cv2, &a.ctl->c, cand_max, a.sort, a.err, s);
    const unsigned gj = (unsigned)sms * 8;
    pl_join_count_kernel<<<gj, 256, 0, s>>>(a);
    pl_scan_kernel<<<persistent_grid(scan_tiles(cand_max), (unsigned)sms * 8), 256, 0, s>>>(a);
    pl_join_write_kernel<<<gj, 256, 0, s>>>(a);
    pl_round_end_kernel<<<1, 256, 0, s>>>(a);
}

}  // namespace emp
