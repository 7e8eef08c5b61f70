// k_coop.cu -- every overlap round of one or many read sets in ONE cooperative
// launch (one CTA of 512 threads per SM, all co-resident).
//
// Each iteration runs one round (overlap.cu:258-290) of every unfinished job.
// Phases are separated by a grid barrier with a bounded wait; inside a phase
// the CTAs take tiles of all active jobs from one atomic ticket, so small and
// large jobs share the GPU:
//   1 update      drop used ids, NextSfx / PrevPfx with the 2-bit column
//                 store, order-preserving compaction (decoupled look-back),
//                 two Bloom bits per key in its table's filter
//                 (remove_used + regenerate_fingerprints, overlap.cu:605-710)
//   2 candidates  entries whose key may occur in the other table, in list
//                 order, with the digit histograms of their sort keys; the
//                 CTA that finishes a job's last tile picks its sort path
//   3 sort        <= 512 candidates: one CTA ranks them; <= 4096: one CTA runs
//                 all passes in shared memory; otherwise if every bucket of the
//                 top 8 key bits holds <= 4096: one MSD scatter pass, then one
//                 CTA per bucket sorts the low 51 bits in shared memory;
//                 otherwise the 8 LSD passes (stable in every path, i.e. the
//                 order of the reference's thrust::sort_by_key)
//   4 join        equal-key runs -> edges at the job's running offset, used
//                 marks (get_edges + remove_used, overlap.cu:557-603,694-710);
//                 Bloom filters and histograms cleared; the CTA that finishes
//                 a job's join records its round (S, P, E) and advances it,
//                 ending the job when its suffix table is empty or all L-o
//                 rounds ran (overlap.cu:258)
// Only candidates are sorted; non-candidates take part in no edge and the
// sort is stable, so every edge comes out in the reference's order.
//
// Streaming tiles (phases 1 and 2) adapt to the job size: up to 4 x 4096
// entries, sized so that one wave of CTAs covers the job when it can.  A tile
// compacts its survivors into shared memory, resolves its output offset with
// one look-back and copies them out contiguously.
#include "coop_common.cuh"

namespace emp {

constexpr uint32_t kSub = kCoopTile;    // 4096
constexpr size_t kStageBytes = (size_t)kCoopMaxSubs * kSub * (sizeof(uint64_t) + sizeof(uint32_t));
constexpr size_t kCoopDynSmem = kStageBytes > kBlockSortSmem ? kStageBytes : kBlockSortSmem;

struct CoopShared {
    uint32_t pref[kCoopMaxJobs + 1];  // tile prefix over jobs for the current phase
    uint32_t bucket[kSortRadix];
    uint32_t hist[9 * kSortRadix];    // candidate digit counts of the current tile
    uint32_t scan32[32];
    uint64_t scan64[32];
    uint32_t cnt32[kC * kBlkWarps + 1];  // per (chunk, warp) counts of a tile scan
    uint64_t cnt64[kC * kBlkWarps + 1];
    uint64_t base;
    uint32_t tile, flag, sfx, last;
    uint32_t gen;  // grid barriers passed
};


// 4096-entry chunks per streaming tile: enough that the job's tiles form one
// wave of CTAs when they can (at most kCoopMaxSubs)
EMP_DEV uint32_t subs_per_tile(uint64_t n) {
    const uint64_t per_cta = (n + gridDim.x - 1) / gridDim.x;
    const uint64_t s = (per_cta + kSub - 1) / kSub;
    return (uint32_t)(s < 1 ? 1 : (s > kCoopMaxSubs ? kCoopMaxSubs : s));
}
EMP_DEV uint32_t stream_tiles(uint64_t n) {
    const uint64_t te = (uint64_t)subs_per_tile(n) * kSub;
    return (uint32_t)((n + te - 1) / te);
}

EMP_DEV void bloom_pos(uint64_t key, int bits, uint32_t &h1, uint32_t &h2) {
    const uint64_t x = key * 0x9E3779B97F4A7C15ull;
    h1 = (uint32_t)(x >> (64 - bits));
    h2 = (uint32_t)((x >> (64 - 2 * bits)) & ((1ull << bits) - 1));
}

// ---------------------------------------------------------------- phase 1
EMP_DEV void update_tile(CoopJob &J, uint32_t lt, uint32_t iter, CoopShared &sh, const CoopCtl *ctl, uint32_t *err,
                         uint8_t *stage) {
    probe(ctl, iter, 2);
    const uint64_t n_in = vld(J.n);
    const uint32_t cur = vld(J.cur);
    const int L = J.L, r = (int)vld(J.round), bits = (int)vld(J.bloom_bits[iter & 1]);
    const uint64_t *kin = J.lk[cur];
    const uint32_t *vin = J.lv[cur];
    uint64_t *kout = J.lk[cur ^ 1];
    uint32_t *vout = J.lv[cur ^ 1];
    const int cf = r, cb = L - 1 - r;
    const uint32_t pw1 = J.tables->pow1[L - r - 1], pw2 = J.tables->pow2[L - r - 1];
    const uint32_t inv1 = J.tables->inv1, inv2 = J.tables->inv2;
    const uint32_t subs = subs_per_tile(n_in);
    const uint64_t base = (uint64_t)lt * subs * kSub;
    uint64_t *sk = reinterpret_cast<uint64_t *>(stage);
    uint32_t *sv = reinterpret_cast<uint32_t *>(sk + kCoopMaxSubs * kSub);
    if (threadIdx.x == 0) sh.sfx = 0;
    uint32_t local = 0, sfx_kept = 0;
    for (uint32_t sub = 0; sub < subs; ++sub) {
        const uint64_t sbase = base + (uint64_t)sub * kSub;
        // staged so that each stage's loads of all 8 chunks are in flight together
        uint64_t key[kC];
        uint32_t val[kC], ex[kC], word[kC];
        bool in[kC], keep[kC];
#pragma unroll
        for (int c = 0; c < kC; ++c) {  // 1: the entries
            const uint64_t e = sbase + c * kT + threadIdx.x;
            in[c] = e < n_in;
            key[c] = in[c] ? __ldcg(kin + e) : 0;
            val[c] = in[c] ? __ldcg(vin + e) : 0;
        }
#pragma unroll
        for (int c = 0; c < kC; ++c) {  // 2: used marks and the 2-bit base words
            const uint32_t v = val[c], rid = v & 0x7fffffffu, t = v >> 31, s = rid & 1u, i = rid >> 1;
            keep[c] = in[c] && __ldcg(t ? J.used_p + rid : J.used_s + rid) == 0;
            const int col = t == 0 ? (s ? cb : cf) : (s ? cf : cb);
            word[c] = in[c] ? __ldg(J.cols + (uint64_t)col * J.wpc + (i >> 4)) : 0u;
        }
#pragma unroll
        for (int c = 0; c < kC; ++c) {  // 3: hash step, Bloom bits
            if (!keep[c]) continue;
            const uint32_t v = val[c], rid = v & 0x7fffffffu, t = v >> 31, s = rid & 1u, i = rid >> 1;
            const uint32_t b = ((word[c] >> ((i & 15u) * 2u)) & 3u) ^ (s << 1);
            const uint64_t k = t == 0 ? next_sfx(key[c], b, pw1, pw2) : prev_pfx(key[c], b, inv1, inv2);
            key[c] = k;
            sfx_kept += t == 0;
            uint32_t h1, h2;
            bloom_pos(k, bits, h1, h2);
            uint32_t *bm = t ? J.bloom_p : J.bloom_s;
            atomicOr(bm + (h1 >> 5), 1u << (h1 & 31));
            atomicOr(bm + (h2 >> 5), 1u << (h2 & 31));
        }
        const uint32_t total = tile_flag_scan(keep, ex, sh.cnt32);
#pragma unroll
        for (int c = 0; c < kC; ++c) {
            if (keep[c]) {
                sk[local + ex[c]] = key[c];
                sv[local + ex[c]] = val[c];
            }
        }
        local += total;
    }
    probe(ctl, iter, 3);
    if (sfx_kept) atomicAdd(&sh.sfx, sfx_kept);
    if (threadIdx.x < 32) {
        const uint64_t b = lookback_epoch_warp(J.st_upd, lt, local, iter * 4u + 1u, err);
        if (threadIdx.x == 0) sh.base = b;
    }
    __syncthreads();
    probe(ctl, iter, 4);
    const uint64_t o = sh.base;
    for (uint32_t x = threadIdx.x; x < local; x += kT) {
        kout[o + x] = sk[x];
        vout[o + x] = sv[x];
    }
    if (threadIdx.x == 0) {
        if (sh.sfx) atomicAdd(reinterpret_cast<unsigned long long *>(&J.s_next), (unsigned long long)sh.sfx);
        if (lt == stream_tiles(n_in) - 1) J.n_next = o + local;
    }
    __syncthreads();
    probe(ctl, iter, 5);
}

// ---------------------------------------------------------------- phase 2
EMP_DEV void cand_tile(CoopJob &J, uint32_t lt, uint32_t iter, CoopShared &sh, CoopCtl *ctl, uint32_t *err,
                       uint8_t *stage) {
    probe(ctl, iter, 10);
    const uint64_t n = vld(J.n_next);
    const int bits = (int)vld(J.bloom_bits[iter & 1]);
    const uint32_t cur = vld(J.cur);
    const uint64_t *kin = J.lk[cur ^ 1];  // the list phase 1 wrote
    const uint32_t *vin = J.lv[cur ^ 1];
    const uint32_t subs = subs_per_tile(n);
    const uint64_t base = (uint64_t)lt * subs * kSub;
    uint64_t *sk = reinterpret_cast<uint64_t *>(stage);
    uint32_t *sv = reinterpret_cast<uint32_t *>(sk + kCoopMaxSubs * kSub);
    for (int i = threadIdx.x; i < 9 * kSortRadix; i += kT) sh.hist[i] = 0;
    __syncthreads();
    uint32_t local = 0;
    for (uint32_t sub = 0; sub < subs; ++sub) {
        const uint64_t sbase = base + (uint64_t)sub * kSub;
        uint64_t key[kC];
        uint32_t val[kC], ex[kC], w1[kC], w2[kC], h1[kC], h2[kC];
        bool in[kC], cand[kC];
#pragma unroll
        for (int c = 0; c < kC; ++c) {  // 1: the entries
            const uint64_t e = sbase + c * kT + threadIdx.x;
            in[c] = e < n;
            key[c] = in[c] ? __ldcg(kin + e) : 0;
            val[c] = in[c] ? __ldcg(vin + e) : 0;
        }
#pragma unroll
        for (int c = 0; c < kC; ++c) {  // 2: both Bloom words of the other table
            const uint32_t *bm = (val[c] >> 31) ? J.bloom_s : J.bloom_p;
            bloom_pos(key[c], bits, h1[c], h2[c]);
            w1[c] = in[c] ? __ldcg(bm + (h1[c] >> 5)) : 0u;
            w2[c] = in[c] ? __ldcg(bm + (h2[c] >> 5)) : 0u;
        }
#pragma unroll
        for (int c = 0; c < kC; ++c) {  // 3: candidates and their sort-key digits
            cand[c] = in[c] && ((w1[c] >> (h1[c] & 31)) & 1u) && ((w2[c] >> (h2[c] & 31)) & 1u);
            if (cand[c]) {
                const uint64_t sk8 = sort_key(key[c], val[c]);
#pragma unroll
                for (int p = 0; p < kSortPasses; ++p)
                    atomicAdd(&sh.hist[p * kSortRadix + ((sk8 >> (8 * p)) & 255)], 1u);
                atomicAdd(&sh.hist[8 * kSortRadix + ((sk8 >> 51) & 255)], 1u);
            }
        }
        const uint32_t total = tile_flag_scan(cand, ex, sh.cnt32);
#pragma unroll
        for (int c = 0; c < kC; ++c) {
            if (cand[c]) {
                sk[local + ex[c]] = key[c];
                sv[local + ex[c]] = val[c];
            }
        }
        local += total;
    }
    probe(ctl, iter, 11);
    if (threadIdx.x < 32) {
        const uint64_t b = lookback_epoch_warp(J.st_cand, lt, local, iter * 4u + 2u, err);
        if (threadIdx.x == 0) sh.base = b;
    }
    __syncthreads();
    probe(ctl, iter, 12);
    const uint64_t o = sh.base;
    for (uint32_t x = threadIdx.x; x < local; x += kT) {
        J.ck[o + x] = sk[x];
        J.cv[o + x] = sv[x];
    }
    for (int i = threadIdx.x; i < 9 * kSortRadix; i += kT) {
        const uint32_t h = sh.hist[i];
        if (h) atomicAdd(&J.hist[0][0] + i, h);
    }
    const uint32_t ntiles = stream_tiles(n);
    if (threadIdx.x == 0 && lt == ntiles - 1) J.c = o + local;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) sh.last = atomicAdd(&J.cand_done, 1u) == ntiles - 1;
    __syncthreads();
    if (sh.last && threadIdx.x < 32) {  // every tile of the job is in: choose the sort path
        __threadfence();
        const int lane = threadIdx.x;
        uint32_t c = 0, mx = 0;
        for (int b = lane; b < kSortRadix; b += 32) {
            c += vld(J.hist[0][b]);
            mx = max(mx, vld(J.hist[8][b]));
        }
#pragma unroll
        for (int off = 16; off; off >>= 1) {
            c += __shfl_xor_sync(0xffffffffu, c, off);
            mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, off));
        }
        if (lane == 0) {
            const uint32_t mode = c <= 1                ? kSortNone
                                  : c <= kRankSortMax   ? kSortRank
                                  : c <= kSmallSort     ? kSortSmall
                                  : mx <= kSmallSort    ? kSortMsd
                                                        : kSortLsd;
            J.mode = mode;
            if (mode == kSortLsd) atomicOr(&ctl->any_lsd, 1u);
        }
    }
    __syncthreads();
    probe(ctl, iter, 13);
}

// bucket bases of digit row `row` of the job's histogram
EMP_DEV void bucket_bases(const CoopJob &J, int row, CoopShared &sh) {
    uint32_t tot;
    const uint32_t c = threadIdx.x < kSortRadix ? vld(J.hist[row][threadIdx.x]) : 0u;
    const uint32_t ex = block_exclusive_scan<kT, uint32_t>(c, sh.scan32, &tot);
    if (threadIdx.x < kSortRadix) sh.bucket[threadIdx.x] = ex;
    __syncthreads();
}

// ---------------------------------------------------------------- phase 4
// The tile and a halo of the following candidates are staged in shared memory
// so the equal-key run scans read shared memory (global only past the halo).
constexpr uint32_t kJoinHalo = 1024;

EMP_DEV void join_tile(CoopJob &J, uint32_t lt, uint32_t iter, CoopShared &sh, const CoopCtl *ctl, uint32_t *err,
                       uint8_t *smem) {
    probe(ctl, iter, 20);
    const uint64_t n = vld(J.c);
    const uint64_t *k = J.ck;
    const uint32_t *v = J.cv;
    const uint64_t base = (uint64_t)lt * kCoopTile;
    const uint64_t span = (n - base < kCoopTile + kJoinHalo) ? n - base : kCoopTile + kJoinHalo;
    uint64_t *sk = reinterpret_cast<uint64_t *>(smem);
    uint32_t *sv = reinterpret_cast<uint32_t *>(sk + kCoopTile + kJoinHalo);
    for (uint32_t x = threadIdx.x; x < span; x += kT) {
        sk[x] = __ldcg(k + base + x);
        sv[x] = __ldcg(v + base + x);
    }
    __syncthreads();
    auto K = [&](uint64_t g) -> uint64_t { return g - base < span ? sk[g - base] : __ldcg(k + g); };
    auto V = [&](uint64_t g) -> uint32_t { return g - base < span ? sv[g - base] : __ldcg(v + g); };
    uint32_t cnt[kC];
    uint64_t ex[kC];
#pragma unroll
    for (int c = 0; c < kC; ++c) {
        const uint64_t i = base + c * kT + threadIdx.x;
        uint32_t cc = 0;
        if (i < n) {
            const uint32_t vi = V(i);
            if ((vi >> 31) == 0) {
                const uint64_t ki = K(i);
                const uint32_t ri = (vi & 0x7fffffffu) >> 1;
                for (uint64_t jx = i + 1; jx < n && K(jx) == ki; ++jx) {
                    const uint32_t vj = V(jx);
                    if ((vj >> 31) && ((vj & 0x7fffffffu) >> 1) != ri) ++cc;
                }
            }
        }
        cnt[c] = cc;
    }
    const uint64_t running = tile_value_scan(cnt, ex, sh.cnt64);
    probe(ctl, iter, 21);
    if (threadIdx.x < 32) {
        const uint64_t b = lookback_epoch_warp(J.st_join, lt, running, iter * 4u + 3u, err);
        if (threadIdx.x == 0) sh.base = b;
    }
    __syncthreads();
    probe(ctl, iter, 22);
    const uint64_t ebase = vld(J.e_total) + sh.base;
#pragma unroll
    for (int c = 0; c < kC; ++c) {
        if (!cnt[c]) continue;
        const uint64_t i = base + c * kT + threadIdx.x;
        const uint64_t ki = K(i);
        const uint32_t si = V(i) & 0x7fffffffu, ri = si >> 1;
        uint64_t o = ebase + ex[c];
        for (uint64_t jx = i + 1; jx < n && K(jx) == ki; ++jx) {
            const uint32_t vj = V(jx);
            const uint32_t pj = vj & 0x7fffffffu;
            if ((vj >> 31) && (pj >> 1) != ri) {
                if (o < J.ecap) {
                    J.efrom[o] = si;
                    J.eto[o] = pj;
                } else {
                    J.overflow = 1;
                }
                J.used_p[pj] = 1;
                ++o;
            }
        }
        J.used_s[si] = 1;
    }
    if (threadIdx.x == 0 && (uint64_t)lt == coop_tiles(n) - 1) J.e_round = sh.base + running;
    __syncthreads();
    probe(ctl, iter, 23);
}

EMP_DEV uint32_t bloom_bits_next(uint64_t n, int max_bits) {
    uint32_t b = 16;
    while ((int)b < max_bits && (1ull << b) < 16 * n) ++b;
    return b;
}

// Record round `round` of the job and advance it (one thread; called once the
// job's join is complete).  Next round's Bloom size goes to the other parity.
// It does not clear `c`: other CTAs may still be counting the join phase's
// tiles from it.  `c` is cleared at the start of the next iteration.
EMP_DEV void round_end(CoopJob &x, CoopCtl *ctl, uint32_t iter) {
    const uint64_t S = vld(x.s_next), nn = vld(x.n_next), P = nn - S;
    const uint32_t r = vld(x.round);
    if (S == 0) {
        x.done = 1;  // build_graph's loop condition: no suffix left
        atomicSub(&ctl->active, 1u);
        return;
    }
    const uint64_t E = P ? vld(x.e_round) : 0;
    const uint64_t e0 = vld(x.e_total);
    RoundRecord &rec = x.records[r];
    rec.S = S;
    rec.P = P;
    rec.E = E;
    rec.e0 = e0;
    rec.C = vld(x.c);
    x.e_total = e0 + E;
    x.n = nn;
    x.cur = vld(x.cur) ^ 1u;
    x.round = r + 1;
    x.bloom_bits[(iter + 1) & 1] = bloom_bits_next(nn, x.bloom_bits_max);
    x.n_next = 0;
    x.s_next = 0;
    x.e_round = 0;
    x.mode = kSortNone;
    x.cand_done = 0;
    x.join_done = 0;
    if ((int)(r + 1) >= x.rounds) {
        x.done = 1;
        atomicSub(&ctl->active, 1u);
    }
    __threadfence();
}

__global__ void __launch_bounds__(kT, 1) coop_rounds_kernel(CoopJob *jobs, CoopCtl *ctl, uint32_t *err) {
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ CoopShared sh;
    const int J = (int)ctl->njobs;
    if (threadIdx.x == 0) sh.gen = 0;
    __syncthreads();
    for (uint32_t iter = 0;; ++iter) {
        if (vld(ctl->active) == 0) break;
        if (blockIdx.x == 0 && threadIdx.x == 0) ctl->ticket[13] = 0;  // join ticket of the last iteration
        // candidate counts of the last round (also of jobs that ended in it);
        // cand_tile sets them again in phase 2
        for (int j = blockIdx.x * kT + threadIdx.x; j < J; j += gridDim.x * kT) jobs[j].c = 0;
        probe(ctl, iter, 0);
        // ---- 1: update
        uint32_t total = build_prefix(sh, J, [&](int j) -> uint32_t {
            return vld(jobs[j].done) ? 0u : stream_tiles(vld(jobs[j].n));
        });
        probe(ctl, iter, 1);
        tile_loop(sh, &ctl->ticket[0], J, total,
                  [&](int j, uint32_t lt) { update_tile(jobs[j], lt, iter, sh, ctl, err, smem); });
        probe(ctl, iter, 6);
        if (!grid_barrier(ctl, &sh.flag, &sh.gen, iter, 0)) return;
        probe(ctl, iter, 7);
        // ---- 2: candidates
        total = build_prefix(sh, J, [&](int j) -> uint32_t {
            const CoopJob &x = jobs[j];
            const uint64_t s = vld(x.s_next), nn = vld(x.n_next);
            return (vld(x.done) || s == 0 || s == nn) ? 0u : stream_tiles(nn);
        });
        probe(ctl, iter, 8);
        tile_loop(sh, &ctl->ticket[1], J, total,
                  [&](int j, uint32_t lt) { cand_tile(jobs[j], lt, iter, sh, ctl, err, smem); });
        probe(ctl, iter, 9);
        if (!grid_barrier(ctl, &sh.flag, &sh.gen, iter, 1)) return;
        probe(ctl, iter, 14);
        // ---- 3a: single-CTA sorts and the MSD scatter pass
        total = build_prefix(sh, J, [&](int j) -> uint32_t {
            const uint32_t m = vld(jobs[j].mode);
            return (m == kSortSmall || m == kSortRank) ? 1u : 0u;
        });
        tile_loop(sh, &ctl->ticket[2], J, total, [&](int j, uint32_t) {
            CoopJob &x = jobs[j];
            const uint32_t c = (uint32_t)vld(x.c);
            if (vld(x.mode) == kSortRank) rank_sort(x.ck, x.cv, x.ck, x.cv, c, smem);
            else block_sort(x.ck, x.cv, x.ck, x.cv, c, 0, kSortPasses, smem);
        });
        total = build_prefix(sh, J, [&](int j) -> uint32_t {
            return vld(jobs[j].mode) == kSortMsd ? (uint32_t)sort_tiles(vld(jobs[j].c)) : 0u;
        });
        tile_loop(sh, &ctl->ticket[3], J, total, [&](int j, uint32_t lt) {
            CoopJob &x = jobs[j];
            bucket_bases(x, 8, sh);
            onesweep_tile(x.ck, x.cv, x.ck2, x.cv2, vld(x.c), lt, 51, sh.bucket, x.st_sort,
                          (iter * 9u + 8u) & 0xfffffu, err, smem);
        });
        probe(ctl, iter, 15);
        if (!grid_barrier(ctl, &sh.flag, &sh.gen, iter, 2)) return;
        probe(ctl, iter, 16);
        // ---- 3b: per-bucket sorts of the MSD jobs, first LSD pass
        total = build_prefix(sh, J, [&](int j) -> uint32_t {
            return vld(jobs[j].mode) == kSortMsd ? (uint32_t)kSortRadix : 0u;
        });
        tile_loop(sh, &ctl->ticket[4], J, total, [&](int j, uint32_t b) {
            CoopJob &x = jobs[j];
            bucket_bases(x, 8, sh);
            const uint32_t lo = sh.bucket[b], cnt = vld(x.hist[8][b]);
            if (cnt == 1) {
                if (threadIdx.x == 0) {
                    x.ck[lo] = __ldcg(x.ck2 + lo);
                    x.cv[lo] = __ldcg(x.cv2 + lo);
                }
            } else if (cnt <= kRankSortMax) {
                if (cnt > 1) rank_sort(x.ck2 + lo, x.cv2 + lo, x.ck + lo, x.cv + lo, cnt, smem);
            } else {
                block_sort(x.ck2 + lo, x.cv2 + lo, x.ck + lo, x.cv + lo, cnt, 0, 7, smem);
            }
            __syncthreads();
        });
        const bool lsd = vld(ctl->any_lsd) != 0;
        for (int p = 0; lsd && p < kSortPasses; ++p) {
            total = build_prefix(sh, J, [&](int j) -> uint32_t {
                return vld(jobs[j].mode) == kSortLsd ? (uint32_t)sort_tiles(vld(jobs[j].c)) : 0u;
            });
            tile_loop(sh, &ctl->ticket[5 + p], J, total, [&](int j, uint32_t lt) {
                CoopJob &x = jobs[j];
                bucket_bases(x, p, sh);
                const bool even = (p & 1) == 0;
                onesweep_tile(even ? x.ck : x.ck2, even ? x.cv : x.cv2, even ? x.ck2 : x.ck, even ? x.cv2 : x.cv,
                              vld(x.c), lt, 8 * p, sh.bucket, x.st_sort, (iter * 9u + (uint32_t)p) & 0xfffffu, err,
                              smem);
            });
            if (p < kSortPasses - 1 && !grid_barrier(ctl, &sh.flag, &sh.gen, iter, 6)) return;
        }
        probe(ctl, iter, 17);
        if (!grid_barrier(ctl, &sh.flag, &sh.gen, iter, 3)) return;
        probe(ctl, iter, 18);
        // ---- 4: join, clears, round end
        if (blockIdx.x == 0 && threadIdx.x < 13) ctl->ticket[threadIdx.x] = 0;  // phases 1-3 are over
        if (blockIdx.x == 0 && threadIdx.x == 0) ctl->any_lsd = 0;
        // join tiles from `c` alone: round_end (below, by whichever CTA
        // finishes a job's join) changes `done` while other CTAs still build
        // this prefix, but never `c`; jobs that ended earlier have c == 0
        total = build_prefix(sh, J, [&](int j) -> uint32_t {
            const uint64_t c = vld(jobs[j].c);
            return c == 0 ? 0u : (uint32_t)coop_tiles(c);
        });
        for (int j = 0; j < J; ++j) {  // Bloom filters and histograms, grid-wide, before any round end
            CoopJob &x = jobs[j];
            if (vld(x.done)) continue;
            const uint64_t words = (1ull << vld(x.bloom_bits[iter & 1])) >> 5;
            for (uint64_t i = (uint64_t)blockIdx.x * kT + threadIdx.x; i < words; i += (uint64_t)gridDim.x * kT) {
                x.bloom_s[i] = 0;
                x.bloom_p[i] = 0;
            }
            for (uint32_t i = blockIdx.x * kT + threadIdx.x; i < 9u * kSortRadix; i += gridDim.x * kT)
                (&x.hist[0][0])[i] = 0;
        }
        probe(ctl, iter, 19);
        tile_loop(sh, &ctl->ticket[13], J, total, [&](int j, uint32_t lt) {
            CoopJob &x = jobs[j];
            join_tile(x, lt, iter, sh, ctl, err, smem);
            __threadfence();
            __syncthreads();
            if (threadIdx.x == 0) {
                const uint32_t nt = sh.pref[j + 1] - sh.pref[j];
                if (atomicAdd(&x.join_done, 1u) == nt - 1) {  // the job's join is complete
                    __threadfence();
                    round_end(x, ctl, iter);
                }
            }
            __syncthreads();
        });
        // active jobs without a join this round: round end by CTA (j mod grid)
        for (int j = blockIdx.x; j < J; j += gridDim.x) {
            if (threadIdx.x == 0 && sh.pref[j + 1] == sh.pref[j] && !vld(jobs[j].done)) round_end(jobs[j], ctl, iter);
        }
        probe(ctl, iter, 24);
        if (!grid_barrier(ctl, &sh.flag, &sh.gen, iter, 4)) return;
        probe(ctl, iter, 25);
    }
}

size_t coop_smem_bytes() { return kCoopDynSmem; }

// Found once per device (the first call on it sets the kernel's shared
// memory attribute) and kept: the engine asks for every job.
static int coop_grid_size_find(int dev) {
    int sms = 0, coop = 0, occ = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    if (!coop) return 0;
    if (cudaFuncSetAttribute(coop_rounds_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCoopDynSmem) !=
        cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, coop_rounds_kernel, kT, kCoopDynSmem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return occ >= 1 ? sms : 0;  // one CTA per SM
}

int coop_grid_size() {
    constexpr int kDevs = 64;
    static std::atomic<int> grid[kDevs] = {};  // grid + 1; 0: not found yet
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kDevs) {
        cudaGetLastError();
        return coop_grid_size_find(dev);
    }
    int g = grid[dev].load(std::memory_order_relaxed);
    if (g == 0) {
        g = coop_grid_size_find(dev) + 1;
        grid[dev].store(g, std::memory_order_relaxed);
    }
    return g - 1;
}

cudaError_t launch_coop_rounds(CoopJob *jobs, CoopCtl *ctl, uint32_t *err, cudaStream_t s) {
    const int grid = coop_grid_size();
    if (grid <= 0) return cudaErrorNotSupported;
    void *args[] = {&jobs, &ctl, &err};
    count_launch();
    return cudaLaunchCooperativeKernel((const void *)coop_rounds_kernel, dim3(grid), dim3(kT), args, kCoopDynSmem, s);
}

}  // namespace emp
