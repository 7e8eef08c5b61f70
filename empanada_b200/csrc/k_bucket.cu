// k_bucket.cu -- every overlap round of one or many read sets in ONE
// cooperative launch: two grid barriers per round, no CTA waiting on another
// inside a phase, no global random access on the streaming side.
//
// Round r of a job (overlap.cu:258-290):
//   A  stream the live entries in 4096-entry tiles: drop entries used in the
//      previous round (tombstones written by B, or the used marks of rounds
//      run before the launch: remove_used, overlap.cu:694-710), apply the
//      hash step NextSfx / PrevPfx (overlap.cu:57-91) with the base taken from
//      a 16-base word cached in the entry (one read-major load per 16 rounds:
//      regenerate_fingerprints + filter_bases, overlap.cu:605-692), and
//      partition the tile in shared memory into the round's key buckets.  The
//      tile's output space comes from one atomic add; its bucket starts go to
//      offs[tile][0..nb].  List order is irrelevant from here on: B orders
//      everything it uses by a total order.
//   B  one CTA per bucket: gather the bucket's piece of every A tile, insert
//      the suffix keys into a hash set, probe the prefix keys, keep the
//      entries whose key is in both tables, sort them by the sort key with
//      the tie order of the reference's stable sort (table, then rid parity,
//      then read index: the regenerated tables' order), and join equal-key
//      runs (get_edges, overlap.cu:557-603).  The bucket's edges go to a
//      staging buffer at an atomically reserved offset, recorded per
//      (round, bucket); used entries get a tombstone in the list.  The CTA
//      finishing a job's last bucket records the round and advances the job.
//   end  after the last round, each round's output.bin record is written
//      (write_edges_binary, overlap.cu:148-161), its edges copied from the
//      staging buffer in bucket order, which is sort-key order: the
//      reference's order.
// Keys equal across tables share a bucket (the bucket is a function of the
// key's top bits), so every match is found inside one bucket.
//
// A bucket that does not fit shared memory (8192 entries, or 3072 matched
// entries) uses the job's global scratch region instead, at the bucket's
// position in the round's bucket order.
#include "coop_common.cuh"

namespace emp {

namespace {

constexpr uint32_t kBStage = 8192;  // entries of a bucket staged in shared memory
constexpr uint32_t kBHash = 16384;  // hash slots in shared memory (power of two)
constexpr uint32_t kBCand = 3072;   // matched entries sorted in shared memory
constexpr uint64_t kEmptySlot = ~0ull;  // never a key: fp1, fp2 < 2^29
constexpr uint32_t kFlag = 0x80000000u; // "matched" mark in a staged entry's position word

// shared-memory layout of phase B (bytes): the staged bucket (key, val,
// list position), then a region that holds in turn the gather's owner table
// (u16 per staged entry), the hash set (u32 slots + the u16 slot of each
// suffix), and the compacted matched entries; once those are compacted the
// stage region holds their sort arrays
constexpr size_t kOffKey = 0;
constexpr size_t kOffVal = kOffKey + kBStage * 8;
constexpr size_t kOffPos = kOffVal + kBStage * 4;
constexpr size_t kOffHash = kOffPos + kBStage * 4;
constexpr size_t kHashRegion = kBHash * 4 + kBStage * 2;
constexpr size_t kBSmem = kOffHash + kHashRegion;
static_assert(kBStage * 2 <= kHashRegion, "owner table fits the hash region");
static_assert(kBCand * (8 + 4 + 4) <= kHashRegion, "compacted matches fit the hash region");
static_assert(kOffHash % 16 == 0, "aligned hash region");
// phase A: 2 kBktMaxBuckets bin counters, then the staged tile
constexpr size_t kASmem = kBktMaxBuckets * 8 + kBktTile * sizeof(BktEntry);
// end phase: one round's bucket destinations, the record offsets of a job
constexpr size_t kESmem = (kBktMaxBuckets + 1 + kT) * 8;
constexpr size_t kBktSmem = kBSmem > kASmem ? (kBSmem > kESmem ? kBSmem : kESmem) : kASmem;

struct BShared {
    uint32_t pref[kCoopMaxJobs + 1];
    uint32_t scan32[32];
    uint64_t scan64[32];
    uint64_t seg_start[kT];
    uint32_t seg_pos[kT + 1];
    uint64_t base, tot, gpre;
    uint32_t tile, flag, sfx;
};

// global scratch arrays of a job (n_max entries each, hash arrays 2 n_max)
struct BScratch {
    uint64_t *key;
    uint32_t *val, *pos;
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
EMP_DEV void a_tile(BktJob &J, uint32_t k, uint32_t iter, BShared &sh, const CoopCtl *ctl, uint8_t *smem) {
    probe(ctl, iter, 2);
    const uint32_t p = iter & 1;
    const uint64_t n_in = vld(J.it[p].n_in);
    // bins: (bucket, table), so a tile's piece of a bucket is its suffixes
    // followed by its prefixes
    const uint32_t nb = vld(J.it[p].nb), nbin = 2 * nb, stride = nbin + 1;
    const int L = J.L, r = (int)vld(J.round);
    const uint32_t pw1 = J.tables->pow1[L - r - 1], pw2 = J.tables->pow2[L - r - 1];
    const uint32_t inv1 = J.tables->inv1, inv2 = J.tables->inv2;
    const bool first = iter == 0;
    const BktEntry *lin = J.lst[p];
    BktEntry *lout = J.lst[p ^ 1];
    uint32_t *hist = reinterpret_cast<uint32_t *>(smem);
    uint4 *stage = reinterpret_cast<uint4 *>(smem + kBktMaxBuckets * 8);
    for (uint32_t i = threadIdx.x; i < nbin; i += kT) hist[i] = 0;
    if (threadIdx.x == 0) sh.sfx = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)k * kBktTile;
    uint64_t key[kC];
    uint32_t val[kC], word[kC], rank[kC], bkt[kC];
    bool keep[kC];
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
        if (keep[c] && (first || (col & 15) == (inc ? 0 : 15)))
            word[c] = __ldg(J.seq2 + (uint64_t)i * J.wpr + (col >> 4));
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
        bkt[c] = 2 * bkt_of(sort_key(key[c], v), nb) + t;
        rank[c] = atomicAdd(&hist[bkt[c]], 1u);
        sfx += t == 0;
    }
    if (sfx) atomicAdd(&sh.sfx, sfx);
    __syncthreads();
    probe(ctl, iter, 3);
    // bin starts: exclusive scan of the nbin counters, each thread a run of them
    const uint32_t per = (nbin + kT - 1) / kT;
    const uint32_t b0 = threadIdx.x * per < nbin ? threadIdx.x * per : nbin;
    const uint32_t b1 = b0 + per < nbin ? b0 + per : nbin;
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
    if (threadIdx.x == 0) {
        orow[nbin] = kept;
        const uint64_t ob = atomicAdd(reinterpret_cast<unsigned long long *>(&J.it[p].n_out),
                                      (unsigned long long)kept);
        sh.base = ob;
        J.tile_base[k] = ob;
        if (sh.sfx) atomicAdd(reinterpret_cast<unsigned long long *>(&J.it[p].s_out), (unsigned long long)sh.sfx);
    }
    __syncthreads();
    probe(ctl, iter, 4);
#pragma unroll
    for (int c = 0; c < kC; ++c) {
        if (!keep[c]) continue;
        stage[hist[bkt[c]] + rank[c]] = make_uint4((uint32_t)key[c], (uint32_t)(key[c] >> 32), val[c], word[c]);
    }
    __syncthreads();
    uint4 *dst = reinterpret_cast<uint4 *>(lout + sh.base);
    for (uint32_t x = threadIdx.x; x < kept; x += kT) dst[x] = stage[x];
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

EMP_DEV void set_stage(BView &v, uint8_t *smem) {
    v.key = reinterpret_cast<uint64_t *>(smem + kOffKey);
    v.val = reinterpret_cast<uint32_t *>(smem + kOffVal);
    v.pos = reinterpret_cast<uint32_t *>(smem + kOffPos);
    v.hslot = nullptr;  // a staged bucket uses match_smem's own hash set
    v.hmatch = nullptr;
    v.hcap = 0;
    v.hpow2 = true;
}
EMP_DEV void set_stage(BView &v, const BScratch &gs, uint64_t G, uint32_t total) {
    v.key = gs.key + G;
    v.val = gs.val + G;
    v.pos = gs.pos + G;
    v.hslot = gs.hslot + 2 * G;
    v.hmatch = gs.hmatch + 2 * G;
    v.hcap = 2 * total;
    v.hpow2 = false;
}

EMP_DEV void put_entry(const BView &v, uint32_t d, const BktEntry *lst, uint64_t src) {
    const uint4 q = __ldcg(reinterpret_cast<const uint4 *>(lst + src));
    v.key[d] = (uint64_t)q.x | ((uint64_t)q.y << 32);
    v.val[d] = q.z;
    v.pos[d] = (uint32_t)src;
}

// Gather bucket b: returns its size and sets up v (shared memory, or the
// global scratch region at the bucket's place in bucket order).
EMP_DEV uint32_t gather(const BktJob &J, uint32_t b, uint32_t nb, uint32_t K, const BktEntry *lst, BShared &sh,
                        uint8_t *smem, BView &v, uint64_t &G, uint32_t &S) {
    // segments q = 0 .. 2K-1: the suffix piece of tile q, then (q >= K) the
    // prefix piece of tile q - K, so the bucket is staged suffixes first
    const uint32_t *offs = J.offs;
    const uint32_t stride = 2 * nb + 1, Q = 2 * K;
    auto seg = [&](uint32_t q, uint32_t &lo, uint32_t &cnt) -> uint64_t {  // returns the tile's base
        const uint32_t k = q < K ? q : q - K, bin = 2 * b + (q < K ? 0u : 1u);
        lo = __ldcg(offs + (uint64_t)k * stride + bin);
        cnt = __ldcg(offs + (uint64_t)k * stride + bin + 1) - lo;
        return k;
    };
    if (Q <= (uint32_t)kT) {
        // fast path: one segment per thread; an owner table maps staged
        // entries to segments
        const uint32_t q = threadIdx.x;
        uint32_t lo = 0, cnt = 0;
        uint64_t start = 0;
        if (q < Q) {
            const uint64_t k = seg(q, lo, cnt);
            start = __ldcg(J.tile_base + k) + lo;
        }
        uint32_t total;
        const uint32_t ex = block_exclusive_scan<kT, uint32_t>(cnt, sh.scan32, &total);
        if (q == K) sh.tile = ex;  // suffixes: the segments before the first prefix piece
        if (total <= kBStage) {
            G = 0;
            set_stage(v, smem);
            uint16_t *owner = reinterpret_cast<uint16_t *>(smem + kOffHash);
            sh.seg_start[threadIdx.x] = start;
            sh.seg_pos[threadIdx.x] = ex;
            for (uint32_t x = ex; x < ex + cnt; ++x) owner[x] = (uint16_t)q;
            __syncthreads();
            S = K ? sh.tile : 0u;
            constexpr int U = 4;
            for (uint32_t x0 = 0; x0 < total; x0 += U * kT) {
                uint4 e[U];
                uint64_t src[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const uint32_t x = x0 + u * kT + threadIdx.x;
                    if (x < total) {
                        const uint32_t o = owner[x];
                        src[u] = sh.seg_start[o] + (x - sh.seg_pos[o]);
                        e[u] = __ldcg(reinterpret_cast<const uint4 *>(lst + src[u]));
                    }
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const uint32_t x = x0 + u * kT + threadIdx.x;
                    if (x < total) {
                        v.key[x] = (uint64_t)e[u].x | ((uint64_t)e[u].y << 32);
                        v.val[x] = e[u].z;
                        v.pos[x] = (uint32_t)src[u];
                    }
                }
            }
            __syncthreads();
            return total;
        }
    }
    // general path: many tiles, or a bucket too big for shared memory
    uint64_t tot = 0, tsfx = 0, gpre = 0;
    for (uint32_t q = threadIdx.x; q < Q; q += kT) {
        uint32_t lo, cnt;
        seg(q, lo, cnt);
        tot += cnt;
        if (q < K) {
            tsfx += cnt;
            gpre += lo;  // entries of lower buckets in tile q
        }
    }
    uint64_t t1, t2, t3;
    block_exclusive_scan<kT, uint64_t>(tot, sh.scan64, &t1);
    block_exclusive_scan<kT, uint64_t>(tsfx, sh.scan64, &t2);
    block_exclusive_scan<kT, uint64_t>(gpre, sh.scan64, &t3);
    const uint32_t total = (uint32_t)t1;
    S = (uint32_t)t2;
    G = t3;
    if (total <= kBStage) {
        G = 0;
        set_stage(v, smem);
    } else {
        BScratch gs;
        scratch_layout(J.scratch, J.n_max, &gs);
        set_stage(v, gs, G, total);
    }
    uint32_t gathered = 0;
    for (uint32_t q0 = 0; q0 < Q && total; q0 += kT) {
        const uint32_t q = q0 + threadIdx.x;
        uint32_t lo = 0, cnt = 0;
        uint64_t start = 0;
        if (q < Q) {
            const uint64_t k = seg(q, lo, cnt);
            start = __ldcg(J.tile_base + k) + lo;
        }
        uint32_t ctot;
        const uint32_t ex = block_exclusive_scan<kT, uint32_t>(cnt, sh.scan32, &ctot);
        sh.seg_start[threadIdx.x] = start;
        sh.seg_pos[threadIdx.x] = ex;
        __syncthreads();
        for (uint32_t x = threadIdx.x; x < ctot; x += kT) {
            uint32_t lo2 = 0, hi = kT;  // last segment with seg_pos <= x
            while (hi - lo2 > 1) {
                const uint32_t m = (lo2 + hi) >> 1;
                if (sh.seg_pos[m] <= x) lo2 = m;
                else hi = m;
            }
            put_entry(v, gathered + x, lst, sh.seg_start[lo2] + (x - sh.seg_pos[lo2]));
        }
        gathered += ctot;
        __syncthreads();
    }
    return total;
}

// ---- shared-memory fast path of a bucket (the common case)
// Hash slots are u32: bit 31 matched, bits 13-30 an 18-bit tag of the key,
// bits 0-12 the staged index of a suffix with that key (keys compared in full
// through it).  A tag of all ones is never used, so kSlotEmpty is no slot.
constexpr uint32_t kSlotEmpty = 0xffffffffu;
constexpr uint32_t kSlotMatched = 0x80000000u;
static_assert(kBStage <= 8192 && kBHash == 16384, "13-bit staged indices, 14-bit slot numbers");

EMP_DEV void hash_tag(uint64_t key, uint32_t &slot, uint32_t &tag) {
    const uint32_t h = (uint32_t)((key * 0x9E3779B97F4A7C15ull) >> 32);
    slot = h & (kBHash - 1);
    tag = (h >> 14) & 0x3ffffu;
    if (tag == 0x3ffffu) tag = 0x3fffeu;
}
EMP_DEV bool slot_holds(uint32_t w, uint32_t tag, uint64_t k, const uint64_t *key) {
    return ((w >> 13) & 0x3ffffu) == tag && key[w & 8191u] == k;
}

// Mark (kFlag in pos) every staged entry whose key occurs in both tables.
// The bucket is staged suffixes first: [0, S) suffixes, [S, total) prefixes.
// Each thread works on kU entries at once so their shared-memory round trips
// overlap; a collision falls back to a probe loop.
EMP_DEV void match_smem(uint32_t total, uint32_t S, uint8_t *smem) {
    constexpr int kU = 4;
    const uint64_t *key = reinterpret_cast<const uint64_t *>(smem + kOffKey);
    uint32_t *pos = reinterpret_cast<uint32_t *>(smem + kOffPos);
    uint32_t *slot = reinterpret_cast<uint32_t *>(smem + kOffHash);
    uint16_t *sslot = reinterpret_cast<uint16_t *>(smem + kOffHash + kBHash * 4);
    for (uint32_t s = threadIdx.x; s < kBHash; s += kT) slot[s] = kSlotEmpty;
    __syncthreads();
    for (uint32_t x0 = 0; x0 < S; x0 += kU * kT) {  // suffixes: insert
        uint64_t k[kU];
        uint32_t s[kU], tag[kU], old[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const uint32_t x = x0 + u * kT + threadIdx.x;
            if (x < S) {
                k[u] = key[x];
                hash_tag(k[u], s[u], tag[u]);
                old[u] = atomicCAS(slot + s[u], kSlotEmpty, (tag[u] << 13) | x);
            }
        }
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const uint32_t x = x0 + u * kT + threadIdx.x;
            if (x >= S) continue;
            uint32_t sl = s[u], w = old[u];
            for (uint32_t probes = 1; w != kSlotEmpty && !slot_holds(w, tag[u], k[u], key) && probes < kBHash;
                 ++probes) {
                sl = (sl + 1) & (kBHash - 1);
                w = atomicCAS(slot + sl, kSlotEmpty, (tag[u] << 13) | x);
            }
            sslot[x] = (uint16_t)sl;
        }
    }
    __syncthreads();
    for (uint32_t x0 = S; x0 < total; x0 += kU * kT) {  // prefixes: probe
        uint64_t k[kU];
        uint32_t s[kU], tag[kU], w[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const uint32_t x = x0 + u * kT + threadIdx.x;
            if (x < total) {
                k[u] = key[x];
                hash_tag(k[u], s[u], tag[u]);
                w[u] = slot[s[u]];
            }
        }
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const uint32_t x = x0 + u * kT + threadIdx.x;
            if (x >= total) continue;
            uint32_t sl = s[u], ww = w[u];
            for (uint32_t probes = 1; ww != kSlotEmpty && probes < kBHash; ++probes) {
                if (slot_holds(ww, tag[u], k[u], key)) {
                    if (!(ww & kSlotMatched)) atomicOr(slot + sl, kSlotMatched);
                    pos[x] |= kFlag;
                    break;
                }
                sl = (sl + 1) & (kBHash - 1);
                ww = slot[sl];
            }
        }
    }
    __syncthreads();
    for (uint32_t x = threadIdx.x; x < S; x += kT)  // suffixes: matched?
        if (slot[sslot[x]] & kSlotMatched) pos[x] |= kFlag;
    __syncthreads();
}

// The generic matcher (global scratch, or any view): same marks.
EMP_DEV void match_view(const BView &v, uint32_t total) {
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
        for (uint32_t probes = 0; probes < v.hcap; ++probes) {
            const uint64_t h = ldv(v.hslot + s);
            if (h == kEmptySlot) break;
            if (h == key) {
                v.hmatch[s] = 1;
                v.pos[x] = ldv(v.pos + x) | kFlag;
                break;
            }
            s = slot_next(s, v);
        }
    }
    __syncthreads();
    for (uint32_t x = threadIdx.x; x < total; x += kT) {  // suffixes
        if (ldv(v.val + x) >> 31) continue;
        const uint64_t key = ldv(v.key + x);
        uint32_t s = slot_of(key, v);
        for (uint32_t probes = 0; probes < v.hcap; ++probes) {
            const uint64_t h = ldv(v.hslot + s);
            if (h == key) {
                if (ldv(v.hmatch + s)) v.pos[x] = ldv(v.pos + x) | kFlag;
                break;
            }
            if (h == kEmptySlot) break;
            s = slot_next(s, v);
        }
    }
    __syncthreads();
}

// Arrays of the matched entries: compacted (key, val, list position), their
// sort and tie keys, chunk order, edge counts, and the sorted copy.
struct CandView {
    uint64_t *ck;
    uint32_t *cv, *cp;
    uint64_t *sk;
    uint32_t *tb, *idx;
    uint64_t *cnt;
    uint64_t *skey;
    uint32_t *sval, *spos;
};

// Sort the c matched entries by (sort key, tie) and count each suffix's edges;
// returns the bucket's edge count (cnt then holds exclusive edge offsets).
EMP_DEV uint64_t sort_and_count(const CandView &w, uint32_t c, BShared &sh) {
    for (uint32_t x = threadIdx.x; x < c; x += kT) {
        const uint32_t val = ldv(w.cv + x);
        w.sk[x] = sort_key(ldv(w.ck + x), val);
        w.tb[x] = tie_of(val);
    }
    __syncthreads();
    const uint32_t nch = (c + kT - 1) / kT;
    for (uint32_t q = 0; q < nch; ++q) {  // order within each 512-entry chunk
        const uint32_t lo = q * kT, m = c - lo < kT ? c - lo : kT;
        if (threadIdx.x < m) {
            const uint32_t x = lo + threadIdx.x;
            const uint64_t skx = ldv(w.sk + x);
            const uint32_t tbx = ldv(w.tb + x);
            uint32_t rk = 0;
            for (uint32_t u = 0; u < m; ++u) rk += before(ldv(w.sk + lo + u), ldv(w.tb + lo + u), skx, tbx);
            w.idx[lo + rk] = x;
            w.cnt[x] = rk;
        }
    }
    __syncthreads();
    for (uint32_t x = threadIdx.x; x < c; x += kT) {  // rank among all chunks
        const uint64_t skx = ldv(w.sk + x);
        const uint32_t tbx = ldv(w.tb + x);
        const uint32_t qx = x / kT;
        uint32_t rk = (uint32_t)ldv(w.cnt + x);
        for (uint32_t q = 0; q < nch; ++q) {
            if (q == qx) continue;
            const uint32_t lo = q * kT, m = c - lo < kT ? c - lo : kT;
            uint32_t a = 0, z = m;  // entries of chunk q before x
            while (a < z) {
                const uint32_t mid = (a + z) >> 1;
                const uint32_t y = ldv(w.idx + lo + mid);
                if (before(ldv(w.sk + y), ldv(w.tb + y), skx, tbx)) a = mid + 1;
                else z = mid;
            }
            rk += a;
        }
        w.skey[rk] = ldv(w.ck + x);
        w.sval[rk] = ldv(w.cv + x);
        w.spos[rk] = ldv(w.cp + x);
    }
    __syncthreads();
    // join: per suffix, the prefixes of its equal-key run from other reads
    for (uint32_t i = threadIdx.x; i < c; i += kT) {
        uint64_t cc = 0;
        const uint32_t vi = ldv(w.sval + i);
        if (!(vi >> 31)) {
            const uint64_t ki = ldv(w.skey + i);
            const uint32_t ri = (vi & 0x7fffffffu) >> 1;
            for (uint32_t j = i + 1; j < c && ldv(w.skey + j) == ki; ++j) {
                const uint32_t vj = ldv(w.sval + j);
                cc += (vj >> 31) && ((vj & 0x7fffffffu) >> 1) != ri;
            }
        }
        w.cnt[i] = cc;
    }
    __syncthreads();
    return scan_counts(w.cnt, c, sh);
}

EMP_DEV void b_tile(BktJob &J, uint32_t b, uint32_t iter, BShared &sh, const CoopCtl *ctl, uint8_t *smem) {
    probe(ctl, iter, 11);
    const uint32_t p = iter & 1;
    const uint64_t n_in = vld(J.it[p].n_in);
    const uint32_t nb = vld(J.it[p].nb);
    const uint32_t K = (uint32_t)bkt_tiles(n_in);
    BktEntry *lst = J.lst[p ^ 1];
    BView v;
    uint64_t G = 0;
    uint32_t S = 0;
    const uint32_t total = gather(J, b, nb, K, lst, sh, smem, v, G, S);
    const bool in_smem = total <= kBStage;
    probe(ctl, iter, 13);
    // ---- matches: entries whose key is in both tables get kFlag in pos
    if (total) {
        if (in_smem) match_smem(total, S, smem);
        else match_view(v, total);
    }
    probe(ctl, iter, 14);
    uint32_t c = 0;
    for (uint32_t x0 = 0; x0 < total; x0 += kT) {
        const uint32_t x = x0 + threadIdx.x;
        c += __syncthreads_count(x < total && (ldv(v.pos + x) & kFlag));
    }
    if (threadIdx.x == 0 && c) atomicAdd(reinterpret_cast<unsigned long long *>(&J.it[p].cands), (unsigned long long)c);
    uint64_t E = 0;
    CandView w;
    if (c) {
        if (in_smem && c <= kBCand) {
            // compact (any order: the sort below fixes it) into the hash
            // region; the sort arrays then take the stage region
            uint8_t *h = smem + kOffHash;
            w.ck = reinterpret_cast<uint64_t *>(h);
            w.cv = reinterpret_cast<uint32_t *>(h + kBCand * 8);
            w.cp = w.cv + kBCand;
            if (threadIdx.x == 0) sh.tile = 0;  // compaction counter
            __syncthreads();
            const uint32_t lane = threadIdx.x & 31;
            for (uint32_t x0 = 0; x0 < total; x0 += kT) {
                const uint32_t x = x0 + threadIdx.x;
                const uint32_t ps = x < total ? v.pos[x] : 0u;
                const bool f = (ps & kFlag) != 0;
                const uint32_t m = __ballot_sync(0xffffffffu, f);
                if (!m) continue;
                const uint32_t leader = __ffs(m) - 1;
                uint32_t base = 0;
                if (lane == leader) base = atomicAdd(&sh.tile, (uint32_t)__popc(m));
                base = __shfl_sync(0xffffffffu, base, leader);
                if (f) {
                    const uint32_t d = base + __popc(m & lanemask_lt_u32());
                    w.ck[d] = v.key[x];
                    w.cv[d] = v.val[x];
                    w.cp[d] = ps & ~kFlag;
                }
            }
            __syncthreads();
            uint8_t *s = smem;  // stage region, free now
            w.sk = reinterpret_cast<uint64_t *>(s);
            w.tb = reinterpret_cast<uint32_t *>(s + kBCand * 8);
            w.idx = w.tb + kBCand;
            w.cnt = reinterpret_cast<uint64_t *>(s + kBCand * 16);
            w.skey = reinterpret_cast<uint64_t *>(s + kBCand * 24);
            w.sval = reinterpret_cast<uint32_t *>(s + kBCand * 32);
            w.spos = w.sval + kBCand;
            static_assert(kBCand * 40 <= kOffHash, "sort arrays fit the stage region");
        } else {
            // in place, in order, then the global scratch region of the bucket
            uint32_t cc = 0;
            for (uint32_t x0 = 0; x0 < total; x0 += kT) {
                const uint32_t x = x0 + threadIdx.x;
                const uint32_t ps = x < total ? ldv(v.pos + x) : 0u;
                const bool f = (ps & kFlag) != 0;
                uint64_t key = 0;
                uint32_t val = 0;
                if (f) {
                    key = ldv(v.key + x);
                    val = ldv(v.val + x);
                }
                uint32_t ctot;
                const uint32_t ex = block_exclusive_scan<kT, uint32_t>(f ? 1u : 0u, sh.scan32, &ctot);
                if (f) {
                    v.key[cc + ex] = key;
                    v.val[cc + ex] = val;
                    v.pos[cc + ex] = ps & ~kFlag;
                }
                cc += ctot;
                __syncthreads();
            }
            if (in_smem) {  // the bucket's place in bucket order picks its scratch region
                uint64_t gpre = 0;
                const uint32_t stride = 2 * nb + 1;
                for (uint32_t k = threadIdx.x; k < K; k += kT) gpre += __ldcg(J.offs + (uint64_t)k * stride + 2 * b);
                block_exclusive_scan<kT, uint64_t>(gpre, sh.scan64, &G);
            }
            BScratch gs;
            scratch_layout(J.scratch, J.n_max, &gs);
            w.ck = v.key;
            w.cv = v.val;
            w.cp = v.pos;
            w.sk = gs.sk + G;
            w.tb = gs.tb + G;
            w.idx = gs.idx + G;
            w.cnt = gs.cnt + G;
            w.skey = gs.skey + G;
            w.sval = gs.sval + G;
            w.spos = gs.spos + G;
        }
        probe(ctl, iter, 15);
        E = sort_and_count(w, c, sh);
    }
    probe(ctl, iter, 17);
    if (threadIdx.x == 0) {
        uint64_t off = 0;
        if (E) {
            off = atomicAdd(reinterpret_cast<unsigned long long *>(&J.e_stage), (unsigned long long)E);
            if (off + E > J.ecap) J.overflow = 1;
            atomicAdd(reinterpret_cast<unsigned long long *>(&J.it[p].edges), (unsigned long long)E);
        }
        sh.base = off;
        BktSpan &sp = J.spans[(uint64_t)(vld(J.round) - J.r0) * J.nb_max + b];
        sp.off = off;
        sp.cnt = E;
    }
    __syncthreads();
    probe(ctl, iter, 18);
    if (E && sh.base + E <= J.ecap) {
        const uint64_t ebase = sh.base;
        for (uint32_t i = threadIdx.x; i < c; i += kT) {
            const uint32_t vi = ldv(w.sval + i);
            if (vi >> 31) continue;
            const uint64_t ki = ldv(w.skey + i);
            const uint32_t si = vi & 0x7fffffffu, ri = si >> 1;
            const uint64_t o0 = ebase + ldv(w.cnt + i);
            uint64_t o = o0;
            for (uint32_t j = i + 1; j < c && ldv(w.skey + j) == ki; ++j) {
                const uint32_t vj = ldv(w.sval + j);
                const uint32_t pj = vj & 0x7fffffffu;
                if ((vj >> 31) && (pj >> 1) != ri) {
                    J.sfrom[o] = si;
                    J.sto[o] = pj;
                    lst[ldv(w.spos + j)].val = kBktTomb;
                    ++o;
                }
            }
            if (o != o0) lst[ldv(w.spos + i)].val = kBktTomb;
        }
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
    rec.nb = vld(x.it[p].nb);
    x.e_total = e0 + E;
    x.round = r + 1;
    BktIter &nx = x.it[q];
    nx.n_in = N;
    nx.n_out = 0;
    nx.s_out = 0;
    nx.cands = 0;
    nx.edges = 0;
    nx.nb = bkt_count(N, gridDim.x);
    nx.b_done = 0;
    if ((int)(r + 1) >= x.rounds) {
        x.end_iter = iter;
        atomicSub(&ctl->active, 1u);
    }
    __threadfence();
}

// After the last round: each round's edges from the staging buffer to the
// edge list in bucket order (rounds spread over the CTAs, no grid barrier).
EMP_DEV void place_edges(BktJob *jobs, int J, BShared &sh, uint8_t *smem) {
    uint64_t *dest = reinterpret_cast<uint64_t *>(smem);  // nb + 1 bucket starts
    uint64_t *roff = dest + kBktMaxBuckets + 1;          // byte offset of each round's record
    uint32_t g = 0;
    for (int j = 0; j < J; ++j) {
        BktJob &x = jobs[j];
        if (vld(x.overflow)) continue;
        const uint32_t r0 = (uint32_t)x.r0, r1 = vld(x.round);
        {  // records: one per round with a non-empty prefix table, 12 + 8 E bytes
            const uint32_t r = r0 + threadIdx.x;
            uint64_t sz = 0;
            if (r < r1 && __ldcg(&x.records[r].P)) sz = 12 + 8 * __ldcg(&x.records[r].E);
            uint64_t tot;
            const uint64_t ex = block_exclusive_scan<kT, uint64_t>(sz, sh.scan64, &tot);
            if (r < r1) roff[threadIdx.x] = ex;
            __syncthreads();
        }
        for (uint32_t r = r0; r < r1; ++r, ++g) {
            if (g % gridDim.x != blockIdx.x) continue;
            const RoundRecord &rec = x.records[r];
            if (!__ldcg(&rec.P)) continue;
            const uint64_t E = __ldcg(&rec.E);
            uint8_t *o = x.out + roff[r - r0];
            uint32_t *from = reinterpret_cast<uint32_t *>(o + 12), *to = from + E;
            if (threadIdx.x == 0) {  // u64 n, i32 ovlp_len (write_edges_binary, overlap.cu:148-161)
                uint32_t *h = reinterpret_cast<uint32_t *>(o);
                h[0] = (uint32_t)E;
                h[1] = (uint32_t)(E >> 32);
                h[2] = (uint32_t)(x.L - 1 - (int)r);
            }
            if (!E) continue;
            const uint32_t nb = (uint32_t)__ldcg(&rec.nb);
            const BktSpan *sp = x.spans + (uint64_t)(r - r0) * x.nb_max;
            uint64_t run = 0;
            for (uint32_t b0 = 0; b0 < nb; b0 += kT) {
                const uint32_t b = b0 + threadIdx.x;
                const uint64_t c = b < nb ? __ldcg(&sp[b].cnt) : 0;
                uint64_t tot;
                const uint64_t ex = block_exclusive_scan<kT, uint64_t>(c, sh.scan64, &tot);
                if (b < nb) dest[b] = run + ex;
                run += tot;
            }
            if (threadIdx.x == 0) dest[nb] = run;
            __syncthreads();
            for (uint64_t e = threadIdx.x; e < E; e += kT) {
                uint32_t lo = 0, hi = nb;  // last bucket with dest <= e
                while (hi - lo > 1) {
                    const uint32_t m = (lo + hi) >> 1;
                    if (dest[m] <= e) lo = m;
                    else hi = m;
                }
                const uint64_t src = __ldcg(&sp[lo].off) + (e - dest[lo]);
                from[e] = __ldcg(x.sfrom + src);
                to[e] = __ldcg(x.sto + src);
            }
            __syncthreads();
        }
    }
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
        tile_loop(sh, &ctl->ticket[0], J, total, [&](int j, uint32_t k) { a_tile(jobs[j], k, iter, sh, ctl, smem); });
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
            return (S > 0 && S < N) ? vld(x.it[p].nb) : 0u;
        });
        probe(ctl, iter, 10);
        tile_loop(sh, &ctl->ticket[1], J, total, [&](int j, uint32_t b) {
            BktJob &x = jobs[j];
            b_tile(x, b, iter, sh, ctl, smem);
            __threadfence();
            __syncthreads();
            if (threadIdx.x == 0) {
                const uint32_t nbj = sh.pref[j + 1] - sh.pref[j];
                if (atomicAdd(&x.it[p].b_done, 1u) == nbj - 1) {
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
    place_edges(jobs, J, sh, smem);
}

}  // namespace

size_t bkt_scratch_bytes(uint64_t n_max) { return scratch_layout(nullptr, n_max < 1 ? 1 : n_max, nullptr); }

size_t bkt_offs_words(uint64_t n_max, uint32_t G) {
    return (size_t)bkt_tiles(n_max < 1 ? 1 : n_max) * (2 * bkt_count(n_max, G) + 1);
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
