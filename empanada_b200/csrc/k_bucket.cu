// k_bucket.cu -- every overlap round of one or many read sets in ONE
// cooperative launch, with two grid barriers per round and no global random
// access on the streaming side.
//
// Round r of a job (overlap.cu:258-290):
//   A  stream the live entries in 4096-entry tiles: drop entries used in the
//      previous round (tombstones written by B, or the used marks of rounds
//      run before the launch: remove_used, overlap.cu:694-710), apply the
//      hash step NextSfx / PrevPfx (overlap.cu:57-91) with the base taken from
//      a 16-base word cached in the entry (one read-major load per 16 rounds:
//      regenerate_fingerprints + filter_bases, overlap.cu:605-692), and
//      partition the tile in shared memory by the top bb bits of the entry's
//      sort key.  The tile's output position comes from a decoupled look-back;
//      its bucket starts go to offs[tile][0..2^bb].
//   B  one CTA per bucket (buckets in key order): gather the bucket's piece of
//      every A tile, insert the suffix keys into a hash set, probe the prefix
//      keys, keep the entries whose key is in both tables, sort them by the
//      sort key with the tie order of the reference's stable sort (table,
//      then rid parity, then read index: the regenerated tables' order), and
//      join equal-key runs (get_edges, overlap.cu:557-603).  Edge offsets come
//      from a look-back over the buckets, so the round's edges are in the
//      reference's order; used entries get a tombstone in the list.  The CTA
//      finishing a job's last bucket records the round and advances the job.
// Keys equal across tables share a bucket, so every match is found inside one
// bucket, and bucket order is sort-key order.
//
// Buckets hold 3072 entries on average (2^bb buckets, bb from the list size);
// one that does not fit shared memory (6144 entries, or 3072 matched
// entries) uses the job's global scratch region instead, at the bucket's
// position in the round's bucket order.
#include "coop_common.cuh"

namespace emp {

namespace {

constexpr uint32_t kBStage = 6144;  // entries of a bucket staged in shared memory
constexpr uint32_t kBHash = 8192;   // hash slots in shared memory (power of two)
constexpr uint32_t kBCand = 3072;   // matched entries sorted in shared memory
constexpr uint64_t kEmptySlot = ~0ull;  // never a key: fp1, fp2 < 2^29

// shared-memory layout of phase B (bytes)
constexpr size_t kOffKey = 0;
constexpr size_t kOffVal = kOffKey + kBStage * 8;
constexpr size_t kOffPos = kOffVal + kBStage * 4;
constexpr size_t kOffFlag = kOffPos + kBStage * 4;
constexpr size_t kOffHash = kOffFlag + kBStage;
constexpr size_t kOffMatch = kOffHash + kBHash * 8;
constexpr size_t kBSmem = kOffMatch + kBHash;
// after the matched entries are compacted, the hash region holds the sort
// keys, tie keys, chunk order and edge counts of up to kBCand of them
static_assert(kBCand * (8 + 4 + 4 + 8) <= kBHash * 9, "sort arrays fit the hash region");
static_assert(kOffHash % 16 == 0, "aligned hash region");
// phase A: 2^kBktMaxBits bucket counters, then the staged tile
constexpr size_t kASmem = (1u << kBktMaxBits) * 4 + kBktTile * sizeof(BktEntry);
constexpr size_t kBktSmem = kBSmem > kASmem ? kBSmem : kASmem;

struct BShared {
    uint32_t pref[kCoopMaxJobs + 1];
    uint32_t scan32[32];
    uint64_t scan64[32];
    uint64_t seg_start[kT];
    uint32_t seg_pos[kT + 1];
    uint64_t base, tot, gpre;
    uint32_t tile, flag, sfx, last, c;
};

// global scratch arrays of a job (n_max entries each, hash arrays 2 n_max)
struct BScratch {
    uint64_t *key;
    uint32_t *val, *pos;
    uint8_t *flag;
    uint64_t *hslot;
    uint8_t *hmatch;
    uint64_t *sk;
    uint32_t *tb, *idx;
    uint64_t *cnt;
    uint64_t *skey;
    uint32_t *sval, *spos;
};

__host__ __device__ inline size_t al256(size_t x) { return (x + 255) / 256 * 256; }

__host__ __device__ inline size_t scratch_layout(uint8_t *base, uint64_t N, BScratch *s) {
    size_t o = 0;
    auto take = [&](size_t bytes) -> uint8_t * {
        uint8_t *p = base ? base + o : nullptr;
        o = al256(o + bytes);
        return p;
    };
    BScratch t;
    t.key = reinterpret_cast<uint64_t *>(take(N * 8));
    t.val = reinterpret_cast<uint32_t *>(take(N * 4));
    t.pos = reinterpret_cast<uint32_t *>(take(N * 4));
    t.flag = take(N);
    t.hslot = reinterpret_cast<uint64_t *>(take(2 * N * 8));
    t.hmatch = take(2 * N);
    t.sk = reinterpret_cast<uint64_t *>(take(N * 8));
    t.tb = reinterpret_cast<uint32_t *>(take(N * 4));
    t.idx = reinterpret_cast<uint32_t *>(take(N * 4));
    t.cnt = reinterpret_cast<uint64_t *>(take(N * 8));
    t.skey = reinterpret_cast<uint64_t *>(take(N * 8));
    t.sval = reinterpret_cast<uint32_t *>(take(N * 4));
    t.spos = reinterpret_cast<uint32_t *>(take(N * 4));
    if (s) *s = t;
    return o;
}

// Loads from a view that may be shared memory or global scratch written by
// this CTA (read around L1: an earlier user of the same lines was another SM).
template <class T>
EMP_DEV T ldv(const T *p) {
    return __isShared(p) ? *p : __ldcg(p);
}

struct BView {
    uint64_t *key;
    uint32_t *val, *pos;
    uint8_t *flag;
    uint64_t *hslot;
    uint8_t *hmatch;
    uint32_t hcap;
    bool hpow2;
    uint64_t *sk;
    uint32_t *tb, *idx;
    uint64_t *cnt;
    uint64_t *skey;
    uint32_t *sval, *spos;
};

EMP_DEV uint32_t slot_of(uint64_t key, const BView &v) {
    const uint32_t h = (uint32_t)((key * 0x9E3779B97F4A7C15ull) >> 32);
    return v.hpow2 ? (h & (v.hcap - 1)) : (h % v.hcap);
}
EMP_DEV uint32_t slot_next(uint32_t s, const BView &v) { return s + 1 == v.hcap ? 0 : s + 1; }

// tie order of equal sort keys in the reference's stable sort: rid parity,
// then read index (the regenerated tables list even rids, then odd rids)
EMP_DEV uint32_t tie_of(uint32_t val) {
    const uint32_t rid = val & 0x7fffffffu;
    return ((rid & 1u) << 31) | (rid >> 1);
}
EMP_DEV bool before(uint64_t ska, uint32_t tba, uint64_t skb, uint32_t tbb) {
    return ska < skb || (ska == skb && tba < tbb);
}

// ---------------------------------------------------------------- phase A
EMP_DEV void a_tile(BktJob &J, uint32_t k, uint32_t iter, BShared &sh, const CoopCtl *ctl, uint32_t *err,
                    uint8_t *smem) {
    probe(ctl, iter, 2);
    const uint32_t p = iter & 1;
    const uint64_t n_in = vld(J.it[p].n_in);
    const uint32_t bb = vld(J.it[p].bb), NB = 1u << bb, stride = NB + 1;
    const int L = J.L, r = (int)vld(J.round);
    const uint32_t pw1 = J.tables->pow1[L - r - 1], pw2 = J.tables->pow2[L - r - 1];
    const uint32_t inv1 = J.tables->inv1, inv2 = J.tables->inv2;
    const bool first = iter == 0;
    const BktEntry *lin = J.lst[p];
    BktEntry *lout = J.lst[p ^ 1];
    uint32_t *hist = reinterpret_cast<uint32_t *>(smem);
    uint4 *stage = reinterpret_cast<uint4 *>(smem + (1u << kBktMaxBits) * 4);
    for (uint32_t i = threadIdx.x; i < NB; i += kT) hist[i] = 0;
    if (threadIdx.x == 0) sh.sfx = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)k * kBktTile;
    uint64_t key[kC];
    uint32_t val[kC], word[kC], rank[kC], bkt[kC];
    bool keep[kC], refill[kC];
#pragma unroll
    for (int c = 0; c < kC; ++c) {  // 1: the entries
        const uint64_t e = base + c * kT + threadIdx.x;
        keep[c] = e < n_in;
        key[c] = 0;
        val[c] = 0;
        word[c] = 0;
        if (keep[c]) {
            if (first) {
                key[c] = __ldcg(J.lk_in + e);
                val[c] = __ldcg(J.lv_in + e);
            } else {
                const uint4 q = __ldcg(reinterpret_cast<const uint4 *>(lin + e));
                key[c] = (uint64_t)q.x | ((uint64_t)q.y << 32);
                val[c] = q.z;
                word[c] = q.w;
            }
        }
    }
#pragma unroll
    for (int c = 0; c < kC; ++c) {  // 2: used entries; bases not in the cached word
        refill[c] = false;
        if (!keep[c]) continue;
        const uint32_t v = val[c];
        if (v == kBktTomb) {
            keep[c] = false;
            continue;
        }
        const uint32_t rid = v & 0x7fffffffu, t = v >> 31, s = rid & 1u, i = rid >> 1;
        if (first) keep[c] = (t ? J.used_p[rid] : J.used_s[rid]) == 0;
        const bool inc = t == s;  // fwd suffix / RC prefix walk the read forwards
        const int col = inc ? r : L - 1 - r;
        refill[c] = keep[c] && (first || (col & 15) == (inc ? 0 : 15));
        if (refill[c]) word[c] = __ldg(J.seq2 + (uint64_t)i * J.wpr + (col >> 4));
    }
    uint32_t sfx = 0;
#pragma unroll
    for (int c = 0; c < kC; ++c) {  // 3: hash step, bucket, rank within the tile's bucket
        if (!keep[c]) continue;
        const uint32_t v = val[c], rid = v & 0x7fffffffu, t = v >> 31, s = rid & 1u;
        const bool inc = t == s;
        const int col = inc ? r : L - 1 - r;
        const uint32_t b = ((word[c] >> ((col & 15) * 2)) & 3u) ^ (s << 1);
        key[c] = t == 0 ? next_sfx(key[c], b, pw1, pw2) : prev_pfx(key[c], b, inv1, inv2);
        bkt[c] = (uint32_t)(sort_key(key[c], v) >> (59 - bb));
        rank[c] = atomicAdd(&hist[bkt[c]], 1u);
        sfx += t == 0;
    }
    if (sfx) atomicAdd(&sh.sfx, sfx);
    __syncthreads();
    probe(ctl, iter, 3);
    // bucket starts: exclusive scan of the NB counters, each thread a run of them
    const uint32_t per = (NB + kT - 1) / kT;
    const uint32_t b0 = threadIdx.x * per < NB ? threadIdx.x * per : NB;
    const uint32_t b1 = b0 + per < NB ? b0 + per : NB;
    uint32_t run = 0;
    for (uint32_t b = b0; b < b1; ++b) run += hist[b];
    uint32_t kept;
    uint32_t ex = block_exclusive_scan<kT, uint32_t>(run, sh.scan32, &kept);
    uint32_t *orow = J.offs + (uint64_t)k * stride;
    for (uint32_t b = b0; b < b1; ++b) {
        const uint32_t h = hist[b];
        hist[b] = ex;
        orow[b] = ex;
        ex += h;
    }
    if (threadIdx.x == 0) orow[NB] = kept;
    if (threadIdx.x < 32) {
        const uint64_t tb = lookback_epoch_warp(J.st_a, k, kept, iter * 2u + 1u, err);
        if (threadIdx.x == 0) {
            sh.base = tb;
            J.tile_base[k] = tb;
        }
    }
    __syncthreads();
    probe(ctl, iter, 4);
#pragma unroll
    for (int c = 0; c < kC; ++c) {
        if (!keep[c]) continue;
        stage[hist[bkt[c]] + rank[c]] =
            make_uint4((uint32_t)key[c], (uint32_t)(key[c] >> 32), val[c], word[c]);
    }
    __syncthreads();
    const uint64_t ob = sh.base;
    uint4 *dst = reinterpret_cast<uint4 *>(lout + ob);
    for (uint32_t x = threadIdx.x; x < kept; x += kT) dst[x] = stage[x];
    if (threadIdx.x == 0) {
        if (sh.sfx) atomicAdd(reinterpret_cast<unsigned long long *>(&J.it[p].s_out), (unsigned long long)sh.sfx);
        if ((uint64_t)k == bkt_tiles(n_in) - 1) J.it[p].n_out = ob + kept;
    }
    __syncthreads();
    probe(ctl, iter, 5);
}

// ---------------------------------------------------------------- phase B
// exclusive scan of cnt[0..c) in place (u64), returns the total
EMP_DEV uint64_t scan_counts(uint64_t *cnt, uint32_t c, BShared &sh) {
    uint64_t run = 0;
    for (uint32_t x0 = 0; x0 < c; x0 += kT) {
        const uint32_t x = x0 + threadIdx.x;
        const uint64_t v = x < c ? ldv(cnt + x) : 0;
        uint64_t tot;
        const uint64_t ex = block_exclusive_scan<kT, uint64_t>(v, sh.scan64, &tot);
        if (x < c) cnt[x] = run + ex;
        run += tot;
        __syncthreads();
    }
    return run;
}

EMP_DEV void b_tile(BktJob &J, uint32_t b, uint32_t iter, BShared &sh, const CoopCtl *ctl, uint32_t *err,
                    uint8_t *smem) {
    probe(ctl, iter, 11);
    const uint32_t p = iter & 1;
    const uint64_t n_in = vld(J.it[p].n_in);
    const uint32_t bb = vld(J.it[p].bb), NB = 1u << bb, stride = NB + 1;
    const uint32_t K = (uint32_t)bkt_tiles(n_in);
    BktEntry *lst = J.lst[p ^ 1];
    const uint32_t *offs = J.offs;
    // ---- pass 1: the bucket's size and its position in bucket order
    {
        uint64_t tot = 0, gpre = 0;
        for (uint32_t k = threadIdx.x; k < K; k += kT) {
            const uint32_t lo = __ldcg(offs + (uint64_t)k * stride + b), hi = __ldcg(offs + (uint64_t)k * stride + b + 1);
            tot += hi - lo;
            gpre += lo;
        }
        uint64_t t1, t2;
        block_exclusive_scan<kT, uint64_t>(tot, sh.scan64, &t1);
        block_exclusive_scan<kT, uint64_t>(gpre, sh.scan64, &t2);
        if (threadIdx.x == 0) {
            sh.tot = t1;
            sh.gpre = t2;
        }
        __syncthreads();
    }
    const uint32_t total = (uint32_t)sh.tot;
    const uint64_t G = sh.gpre;
    probe(ctl, iter, 12);
    BScratch gs;
    scratch_layout(J.scratch, J.n_max, &gs);
    BView v;
    const bool in_smem = total <= kBStage;
    if (in_smem) {
        v.key = reinterpret_cast<uint64_t *>(smem + kOffKey);
        v.val = reinterpret_cast<uint32_t *>(smem + kOffVal);
        v.pos = reinterpret_cast<uint32_t *>(smem + kOffPos);
        v.flag = smem + kOffFlag;
        v.hslot = reinterpret_cast<uint64_t *>(smem + kOffHash);
        v.hmatch = smem + kOffMatch;
        v.hcap = kBHash;
        v.hpow2 = true;
    } else {
        v.key = gs.key + G;
        v.val = gs.val + G;
        v.pos = gs.pos + G;
        v.flag = gs.flag + G;
        v.hslot = gs.hslot + 2 * G;
        v.hmatch = gs.hmatch + 2 * G;
        v.hcap = 2 * total;
        v.hpow2 = false;
    }
    // ---- pass 2: gather the bucket's pieces (512 tiles at a time)
    uint32_t gathered = 0;
    for (uint32_t k0 = 0; k0 < K && total; k0 += kT) {
        const uint32_t k = k0 + threadIdx.x;
        uint32_t cnt = 0;
        uint64_t start = 0;
        if (k < K) {
            const uint32_t lo = __ldcg(offs + (uint64_t)k * stride + b), hi = __ldcg(offs + (uint64_t)k * stride + b + 1);
            cnt = hi - lo;
            start = __ldcg(J.tile_base + k) + lo;
        }
        uint32_t ctot;
        const uint32_t ex = block_exclusive_scan<kT, uint32_t>(cnt, sh.scan32, &ctot);
        sh.seg_start[threadIdx.x] = start;
        sh.seg_pos[threadIdx.x] = ex;
        if (threadIdx.x == 0) sh.seg_pos[kT] = ctot;
        __syncthreads();
        for (uint32_t x = threadIdx.x; x < ctot; x += kT) {
            uint32_t lo = 0, hi = kT;  // last segment with seg_pos <= x
            while (hi - lo > 1) {
                const uint32_t m = (lo + hi) >> 1;
                if (sh.seg_pos[m] <= x) lo = m;
                else hi = m;
            }
            const uint64_t src = sh.seg_start[lo] + (x - sh.seg_pos[lo]);
            const uint4 q = __ldcg(reinterpret_cast<const uint4 *>(lst + src));
            const uint32_t d = gathered + x;
            v.key[d] = (uint64_t)q.x | ((uint64_t)q.y << 32);
            v.val[d] = q.z;
            v.pos[d] = (uint32_t)src;
        }
        gathered += ctot;
        __syncthreads();
    }
    probe(ctl, iter, 13);
    // ---- matches: suffix keys into the hash set, prefix keys probe it
    uint32_t c = 0;
    if (total) {
        for (uint32_t s = threadIdx.x; s < v.hcap; s += kT) {
            v.hslot[s] = kEmptySlot;
            v.hmatch[s] = 0;
        }
        __syncthreads();
        for (uint32_t x = threadIdx.x; x < total; x += kT) {
            if (ldv(v.val + x) >> 31) continue;
            const uint64_t key = ldv(v.key + x);
            uint32_t s = slot_of(key, v);
            for (uint32_t probes = 0; probes < v.hcap; ++probes) {
                const uint64_t prev = atomicCAS(reinterpret_cast<unsigned long long *>(v.hslot + s),
                                                (unsigned long long)kEmptySlot, (unsigned long long)key);
                if (prev == kEmptySlot || prev == key) break;
                s = slot_next(s, v);
            }
        }
        __syncthreads();
        for (uint32_t x = threadIdx.x; x < total; x += kT) {  // prefixes
            if (!(ldv(v.val + x) >> 31)) continue;
            const uint64_t key = ldv(v.key + x);
            uint32_t s = slot_of(key, v);
            uint8_t f = 0;
            for (uint32_t probes = 0; probes < v.hcap; ++probes) {
                const uint64_t h = ldv(v.hslot + s);
                if (h == kEmptySlot) break;
                if (h == key) {
                    f = 1;
                    v.hmatch[s] = 1;
                    break;
                }
                s = slot_next(s, v);
            }
            v.flag[x] = f;
        }
        __syncthreads();
        for (uint32_t x = threadIdx.x; x < total; x += kT) {  // suffixes
            if (ldv(v.val + x) >> 31) continue;
            const uint64_t key = ldv(v.key + x);
            uint32_t s = slot_of(key, v);
            uint8_t f = 0;
            for (uint32_t probes = 0; probes < v.hcap; ++probes) {
                const uint64_t h = ldv(v.hslot + s);
                if (h == key) {
                    f = ldv(v.hmatch + s);
                    break;
                }
                if (h == kEmptySlot) break;
                s = slot_next(s, v);
            }
            v.flag[x] = f;
        }
        __syncthreads();
        probe(ctl, iter, 14);
        // compact the matched entries to the front, in place, chunk by chunk
        for (uint32_t x0 = 0; x0 < total; x0 += kT) {
            const uint32_t x = x0 + threadIdx.x;
            const bool f = x < total && ldv(v.flag + x);
            uint64_t key = 0;
            uint32_t val = 0, pos = 0;
            if (f) {
                key = ldv(v.key + x);
                val = ldv(v.val + x);
                pos = ldv(v.pos + x);
            }
            uint32_t ctot;
            const uint32_t ex = block_exclusive_scan<kT, uint32_t>(f ? 1u : 0u, sh.scan32, &ctot);
            if (f) {
                v.key[c + ex] = key;
                v.val[c + ex] = val;
                v.pos[c + ex] = pos;
            }
            c += ctot;
            __syncthreads();
        }
    }
    probe(ctl, iter, 15);
    if (threadIdx.x == 0 && c) atomicAdd(reinterpret_cast<unsigned long long *>(&J.it[p].cands), (unsigned long long)c);
    uint64_t E = 0;
    if (c) {
        // ---- sort the matched entries by (sort key, tie)
        if (in_smem && c <= kBCand) {
            uint8_t *h = smem + kOffHash;
            v.sk = reinterpret_cast<uint64_t *>(h);
            v.tb = reinterpret_cast<uint32_t *>(h + kBCand * 8);
            v.idx = v.tb + kBCand;
            v.cnt = reinterpret_cast<uint64_t *>(h + kBCand * 16);
            v.skey = v.key + kBCand;
            v.sval = v.val + kBCand;
            v.spos = v.pos + kBCand;
        } else {
            v.sk = gs.sk + G;
            v.tb = gs.tb + G;
            v.idx = gs.idx + G;
            v.cnt = gs.cnt + G;
            v.skey = gs.skey + G;
            v.sval = gs.sval + G;
            v.spos = gs.spos + G;
        }
        for (uint32_t x = threadIdx.x; x < c; x += kT) {
            const uint32_t val = ldv(v.val + x);
            v.sk[x] = sort_key(ldv(v.key + x), val);
            v.tb[x] = tie_of(val);
        }
        __syncthreads();
        const uint32_t nch = (c + kT - 1) / kT;
        for (uint32_t q = 0; q < nch; ++q) {  // order within each 512-entry chunk
            const uint32_t lo = q * kT, m = c - lo < kT ? c - lo : kT;
            if (threadIdx.x < m) {
                const uint32_t x = lo + threadIdx.x;
                const uint64_t skx = ldv(v.sk + x);
                const uint32_t tbx = ldv(v.tb + x);
                uint32_t rk = 0;
                for (uint32_t u = 0; u < m; ++u) rk += before(ldv(v.sk + lo + u), ldv(v.tb + lo + u), skx, tbx);
                v.idx[lo + rk] = x;
                v.cnt[x] = rk;
            }
        }
        __syncthreads();
        for (uint32_t x = threadIdx.x; x < c; x += kT) {  // rank among all chunks
            const uint64_t skx = ldv(v.sk + x);
            const uint32_t tbx = ldv(v.tb + x);
            const uint32_t qx = x / kT;
            uint32_t rk = (uint32_t)ldv(v.cnt + x);
            for (uint32_t q = 0; q < nch; ++q) {
                if (q == qx) continue;
                const uint32_t lo = q * kT, m = c - lo < kT ? c - lo : kT;
                uint32_t a = 0, z = m;  // entries of chunk q before x
                while (a < z) {
                    const uint32_t mid = (a + z) >> 1;
                    const uint32_t y = ldv(v.idx + lo + mid);
                    if (before(ldv(v.sk + y), ldv(v.tb + y), skx, tbx)) a = mid + 1;
                    else z = mid;
                }
                rk += a;
            }
            v.skey[rk] = ldv(v.key + x);
            v.sval[rk] = ldv(v.val + x);
            v.spos[rk] = ldv(v.pos + x);
        }
        __syncthreads();
        probe(ctl, iter, 16);
        // ---- join: per suffix, the prefixes of its equal-key run from other reads
        for (uint32_t i = threadIdx.x; i < c; i += kT) {
            uint64_t cc = 0;
            const uint32_t vi = ldv(v.sval + i);
            if (!(vi >> 31)) {
                const uint64_t ki = ldv(v.skey + i);
                const uint32_t ri = (vi & 0x7fffffffu) >> 1;
                for (uint32_t j = i + 1; j < c && ldv(v.skey + j) == ki; ++j) {
                    const uint32_t vj = ldv(v.sval + j);
                    cc += (vj >> 31) && ((vj & 0x7fffffffu) >> 1) != ri;
                }
            }
            v.cnt[i] = cc;
        }
        __syncthreads();
        E = scan_counts(v.cnt, c, sh);
    }
    probe(ctl, iter, 17);
    if (threadIdx.x < 32) {
        const uint64_t eb = lookback_epoch_warp(J.st_b, b, E, iter * 2u + 2u, err);
        if (threadIdx.x == 0) sh.base = eb;
    }
    __syncthreads();
    probe(ctl, iter, 18);
    if (E) {
        const uint64_t ebase = vld(J.e_total) + sh.base;
        for (uint32_t i = threadIdx.x; i < c; i += kT) {
            const uint32_t vi = ldv(v.sval + i);
            if (vi >> 31) continue;
            const uint64_t ki = ldv(v.skey + i);
            const uint32_t si = vi & 0x7fffffffu, ri = si >> 1;
            const uint64_t o0 = ebase + ldv(v.cnt + i);
            uint64_t o = o0;
            for (uint32_t j = i + 1; j < c && ldv(v.skey + j) == ki; ++j) {
                const uint32_t vj = ldv(v.sval + j);
                const uint32_t pj = vj & 0x7fffffffu;
                if ((vj >> 31) && (pj >> 1) != ri) {
                    if (o < J.ecap) {
                        J.efrom[o] = si;
                        J.eto[o] = pj;
                    } else {
                        J.overflow = 1;
                    }
                    lst[ldv(v.spos + j)].val = kBktTomb;
                    ++o;
                }
            }
            if (o != o0) lst[ldv(v.spos + i)].val = kBktTomb;
        }
        if (threadIdx.x == 0) atomicAdd(reinterpret_cast<unsigned long long *>(&J.it[p].edges), (unsigned long long)E);
    }
    __syncthreads();
    probe(ctl, iter, 19);
}

// Record the round and advance the job (one thread, once every bucket of the
// round is done).  Writes only the other parity's iteration state.
EMP_DEV void round_end(BktJob &x, CoopCtl *ctl, uint32_t iter) {
    const uint32_t p = iter & 1, q = p ^ 1;
    const uint64_t N = vld(x.it[p].n_out), S = vld(x.it[p].s_out), P = N - S;
    const uint32_t r = vld(x.round);
    if (S == 0) {  // build_graph's loop condition: no suffix left
        x.end_iter = iter;
        atomicSub(&ctl->active, 1u);
        __threadfence();
        return;
    }
    const uint64_t E = P ? vld(x.it[p].edges) : 0;
    const uint64_t e0 = vld(x.e_total);
    RoundRecord &rec = x.records[r];
    rec.S = S;
    rec.P = P;
    rec.E = E;
    rec.e0 = e0;
    rec.C = vld(x.it[p].cands);
    x.e_total = e0 + E;
    x.round = r + 1;
    BktIter &nx = x.it[q];
    nx.n_in = N;
    nx.n_out = 0;
    nx.s_out = 0;
    nx.cands = 0;
    nx.edges = 0;
    nx.bb = bkt_bits(N);
    nx.b_done = 0;
    if ((int)(r + 1) >= x.rounds) {
        x.end_iter = iter;
        atomicSub(&ctl->active, 1u);
    }
    __threadfence();
}

__global__ void __launch_bounds__(kT, 1) bucket_rounds_kernel(BktJob *jobs, CoopCtl *ctl, uint32_t *err) {
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ BShared sh;
    const int J = (int)ctl->njobs;
    for (uint32_t iter = 0;; ++iter) {
        if (vld(ctl->active) == 0) break;
        const uint32_t p = iter & 1;
        if (blockIdx.x == 0 && threadIdx.x == 0) ctl->ticket[1] = 0;  // bucket ticket of the last iteration
        probe(ctl, iter, 0);
        // ---- A: stream, hash step, partition
        uint32_t total = build_prefix(sh, J, [&](int j) -> uint32_t {
            const BktJob &x = jobs[j];
            return vld(x.end_iter) >= iter ? (uint32_t)bkt_tiles(vld(x.it[p].n_in)) : 0u;
        });
        probe(ctl, iter, 1);
        tile_loop(sh, &ctl->ticket[0], J, total,
                  [&](int j, uint32_t k) { a_tile(jobs[j], k, iter, sh, ctl, err, smem); });
        probe(ctl, iter, 6);
        if (!grid_barrier(ctl, &sh.flag, iter, 0)) return;
        probe(ctl, iter, 7);
        if (blockIdx.x == 0 && threadIdx.x == 0) ctl->ticket[0] = 0;
        // ---- B: buckets; the last bucket of a job ends its round.  The
        // prefix reads only state round_end leaves alone (it writes the other
        // parity and end_iter, which stays >= iter for this iteration).
        total = build_prefix(sh, J, [&](int j) -> uint32_t {
            const BktJob &x = jobs[j];
            if (vld(x.end_iter) < iter) return 0u;
            const uint64_t S = vld(x.it[p].s_out), N = vld(x.it[p].n_out);
            return (S > 0 && S < N) ? (1u << vld(x.it[p].bb)) : 0u;
        });
        probe(ctl, iter, 10);
        tile_loop(sh, &ctl->ticket[1], J, total, [&](int j, uint32_t b) {
            BktJob &x = jobs[j];
            b_tile(x, b, iter, sh, ctl, err, smem);
            __threadfence();
            __syncthreads();
            if (threadIdx.x == 0) {
                const uint32_t nb = sh.pref[j + 1] - sh.pref[j];
                if (atomicAdd(&x.it[p].b_done, 1u) == nb - 1) {
                    __threadfence();
                    round_end(x, ctl, iter);
                }
            }
            __syncthreads();
        });
        // running jobs without buckets this round: round end by CTA (j mod grid)
        for (int j = blockIdx.x; j < J; j += gridDim.x)
            if (threadIdx.x == 0 && sh.pref[j + 1] == sh.pref[j] && vld(jobs[j].end_iter) >= iter)
                round_end(jobs[j], ctl, iter);
        probe(ctl, iter, 20);
        if (!grid_barrier(ctl, &sh.flag, iter, 1)) return;
        probe(ctl, iter, 21);
    }
}

}  // namespace

size_t bkt_scratch_bytes(uint64_t n_max) { return scratch_layout(nullptr, n_max < 1 ? 1 : n_max, nullptr); }

size_t bkt_offs_words(uint64_t n_max) {
    return (size_t)bkt_tiles(n_max < 1 ? 1 : n_max) * ((1u << bkt_bits(n_max)) + 1);
}

int bucket_grid_size() {
    int dev = 0, sms = 0, coop = 0, occ = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    if (!coop) return 0;
    if (cudaFuncSetAttribute(bucket_rounds_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBktSmem) !=
        cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, bucket_rounds_kernel, kT, kBktSmem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return occ >= 1 ? sms : 0;  // one CTA per SM
}

cudaError_t launch_bucket_rounds(BktJob *jobs, CoopCtl *ctl, uint32_t *err, cudaStream_t s) {
    const int grid = bucket_grid_size();
    if (grid <= 0) return cudaErrorNotSupported;
    void *args[] = {&jobs, &ctl, &err};
    count_launch();
    return cudaLaunchCooperativeKernel((const void *)bucket_rounds_kernel, dim3(grid), dim3(kT), args, kBktSmem, s);
}

}  // namespace emp
