// k_bucket.cu -- every overlap round of one or many read sets in ONE
// cooperative launch, one grid barrier per round.
//
// A round's list holds 16-byte entries (key, rid | table, a cached 16-base
// word of the read), kept as one region of `cap` entries per (key bucket,
// table) bin; entries past a region's capacity go to a spill area tagged
// with their bin.  The bucket of an entry is the top 24 bits of its sort key
// scaled to the round's bucket count, so keys equal across tables share a
// bucket and bucket order is key order.
//
//   prologue  the launch's input list (id order; the keys of round r0 - 1)
//      is streamed in 4096-entry tiles: entries used in the rounds run
//      before the launch are dropped (remove_used, overlap.cu:694-710), the
//      hash step NextSfx / PrevPfx (overlap.cu:57-91) gives round r0's keys,
//      and each entry goes into its bin of round r0's list.
//   round r   one CTA per bucket: stage the bucket's suffix region, then its
//      prefix region (two contiguous runs, cp.async), flag the keys present
//      in both tables (a two-level filter, a tagged hash set as fallback),
//      rank the flagged entries by (sort key, rid parity, read index) -- the
//      order of the reference's stable sort over its regenerated tables
//      (regenerate_fingerprints, overlap.cu:605-692) -- and join equal-key
//      runs (get_edges, overlap.cu:557-603).  The bucket's edges go to a
//      staging buffer at an atomically reserved offset.  Then the same CTA
//      drops the bucket's used entries, applies round r+1's hash step to the
//      rest (the base from the cached word; one read-major load per 16
//      rounds) and writes them into round r+1's bins: positions reserved per
//      bin from a shared-memory histogram (up to kBktMaxBuckets buckets), or
//      one atomic per run of equal bins in a warp (more buckets).
//   end  every round's output.bin record (write_edges_binary,
//      overlap.cu:148-161) is written with its edges in bucket order, which
//      is sort-key order: the reference's order.
//
// A bucket that does not fit shared memory (7168 entries, or 2816 matched
// entries) uses the job's global scratch region at the bucket's position in
// bucket order instead.
#include "coop_common.cuh"

// Steps that run once per launch or only for oversized buckets are kept out
// of line, so their registers do not weigh on the per-bucket path.
#define EMP_COLD __device__ __noinline__

namespace emp {

namespace {

constexpr uint32_t kBStage = 3200;  // entries of a bucket staged in shared memory
constexpr uint32_t kBHash = 8192;   // hash slots in shared memory (power of two)
constexpr uint64_t kEmptySlot = ~0ull;  // never a key: fp1, fp2 < 2^29
constexpr uint8_t kMatched = 1, kUsed = 2;

// Shared memory of a round tile: the staged bucket, then a region used in
// turn by the gather (piece table + owner of each staged entry), the hash set
// (u32 slots + the slot of each suffix), the matched entries and their sort
// arrays, and the next round's partition (bin counters + permutation).
constexpr size_t kOffKey = 0;
constexpr size_t kOffVal = kOffKey + kBStage * 8;
constexpr size_t kOffWord = kOffVal + kBStage * 4;
constexpr size_t kOffFlag = kOffWord + kBStage * 4;
constexpr size_t kOffReg = kOffFlag + kBStage;
constexpr size_t kRegion = kBHash * 4 + kBStage * 2;
constexpr size_t kRSmem = kOffReg + kRegion;
static_assert(kOffReg % 16 == 0, "aligned region");
// hash set
constexpr size_t kHSlot = 0;                 // u32 [kBHash]
constexpr size_t kHSuffixSlot = kBHash * 4;  // u16 [kBStage]
// next round's partition
constexpr size_t kPHist = 0;                                // u32 [2 kBktMaxBuckets]
constexpr size_t kPInv = kPHist + 2 * kBktMaxBuckets * 4;   // u16 [kBStage]
constexpr size_t kPRank = kPInv + kBStage * 2;              // u16 [kBStage]
constexpr size_t kPBin = kPRank + kBStage * 2;              // u16 [kBStage]
static_assert(kPBin + kBStage * 2 <= kRegion, "partition tables fit the region");
static_assert(2 * kBktMaxBuckets <= 65536, "bins fit u16");
// prologue tile: bin counters, then the staged tile
constexpr size_t kASmem = 2 * kBktMaxBuckets * 4 + kBktTile * sizeof(BktEntry) + kBktTile * 2;
// end phase: one round's bucket destinations, the record offsets of a job
constexpr int kMaxJobRounds = 512;  // rounds of one job at most (L - o < kMaxReadLen)
constexpr size_t kESmem = (kBktMaxBuckets + 1 + 3 * kMaxJobRounds) * 8;
constexpr size_t kBktSmem = kRSmem > kASmem ? (kRSmem > kESmem ? kRSmem : kESmem) : kASmem;

struct BShared {
    uint32_t pref[kCoopMaxJobs + 1];
    uint32_t scan32[32];
    uint64_t scan64[32];
    uint64_t base;
    uint32_t tile, flag, sfx, cnt, kept;
    uint32_t gen;  // grid barriers passed
    const CoopCtl *pctl;  // profiling stamps from inside the steps of a tile
    uint32_t piter;
    HashTables tab;       // powers and inverses (every job of a launch shares them)
    uint32_t shp_nb[kCoopMaxJobs], shp_nbn[kCoopMaxJobs];  // this iteration's bucket counts
};
EMP_DEV void sprobe(const BShared &sh, int p) { probe(sh.pctl, sh.piter, p); }

// A job's global scratch (N = n_max entries per array, 2N hash slots): a
// bucket that does not fit shared memory uses the region of its position in
// bucket order.
struct BScratch {
    uint64_t *key;
    uint32_t *val, *word;
    uint8_t *flag;
    uint64_t *hslot;
    uint8_t *hmatch;
    uint32_t *sslot;
    uint64_t *ck;
    uint32_t *cv, *cx;
    uint64_t *sk;
    uint32_t *tb, *ord;
    uint64_t *cnt;
    uint64_t *skey;
    uint32_t *sval, *sidx;
    uint32_t *rank;
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
    t.word = reinterpret_cast<uint32_t *>(take(N * 4));
    t.flag = take(N);
    t.hslot = reinterpret_cast<uint64_t *>(take(2 * N * 8));
    t.hmatch = take(2 * N);
    t.sslot = reinterpret_cast<uint32_t *>(take(N * 4));
    t.ck = reinterpret_cast<uint64_t *>(take(N * 8));
    t.cv = reinterpret_cast<uint32_t *>(take(N * 4));
    t.cx = reinterpret_cast<uint32_t *>(take(N * 4));
    t.sk = reinterpret_cast<uint64_t *>(take(N * 8));
    t.tb = reinterpret_cast<uint32_t *>(take(N * 4));
    t.ord = reinterpret_cast<uint32_t *>(take(N * 4));
    t.cnt = reinterpret_cast<uint64_t *>(take(N * 8));
    t.skey = reinterpret_cast<uint64_t *>(take(N * 8));
    t.sval = reinterpret_cast<uint32_t *>(take(N * 4));
    t.sidx = reinterpret_cast<uint32_t *>(take(N * 4));
    t.rank = reinterpret_cast<uint32_t *>(take(N * 4));
    if (s) *s = t;
    return o;
}

// Loads from a view that may be shared memory or global scratch written by
// this CTA (read around L1: an earlier user of the same lines was another SM).
template <class T>
EMP_DEV T ldv(const T *p) {
    return __isShared(p) ? *p : __ldcg(p);
}

struct Stage {  // the staged bucket
    uint64_t *key;
    uint32_t *val, *word;
    uint8_t *flag;
};
struct Cands {  // the matched entries
    uint64_t *ck;
    uint32_t *cv, *cx;
    uint64_t *sk;
    uint32_t *tb, *ord;
    uint64_t *cnt;
    uint64_t *skey;
    uint32_t *sval, *sidx;
};

// tie order of equal sort keys in the reference's stable sort: rid parity,
// then read index (the regenerated tables list even rids, then odd rids)
EMP_DEV uint32_t tie_of(uint32_t val) {
    const uint32_t rid = val & 0x7fffffffu;
    return ((rid & 1u) << 31) | (rid >> 1);
}
EMP_DEV bool before(uint64_t ska, uint32_t tba, uint64_t skb, uint32_t tbb) {
    return ska < skb || (ska == skb && tba < tbb);
}

// Hash step of round r for one entry: key and cached word updated in place.
struct StepArgs {
    int L, r;
    uint32_t pw1, pw2, inv1, inv2;
    bool refill_all;  // the cached words are not valid (the launch's input list)
    const uint32_t *seq2;
    int wpr;
};
EMP_DEV StepArgs step_args(const BktJob &J, const HashTables &tab, int r, bool refill_all) {
    StepArgs a;
    a.L = J.L;
    a.r = r;
    a.pw1 = tab.pow1[J.L - r - 1];
    a.pw2 = tab.pow2[J.L - r - 1];
    a.inv1 = tab.inv1;
    a.inv2 = tab.inv2;
    a.refill_all = refill_all;
    a.seq2 = J.seq2;
    a.wpr = J.wpr;
    return a;
}
// column of the read's base that round r removes from the entry's key: a
// forward suffix or an RC prefix walks the read forwards (column r), the
// others backwards (column L-1-r)
EMP_DEV int step_col(const StepArgs &a, uint32_t val, bool &inc) {
    const uint32_t t = val >> 31, s = val & 1u;
    inc = t == s;
    return inc ? a.r : a.L - 1 - a.r;
}
EMP_DEV bool needs_refill(const StepArgs &a, uint32_t val) {
    bool inc;
    const int col = step_col(a, val, inc);
    return a.refill_all || (col & 15) == (inc ? 0 : 15);
}
EMP_DEV uint32_t refill_word(const StepArgs &a, uint32_t val) {
    bool inc;
    const int col = step_col(a, val, inc);
    return __ldg(a.seq2 + (uint64_t)((val & 0x7fffffffu) >> 1) * a.wpr + (col >> 4));
}
EMP_DEV uint64_t step_key(const StepArgs &a, uint64_t key, uint32_t val, uint32_t word) {
    bool inc;
    const int col = step_col(a, val, inc);
    const uint32_t t = val >> 31, s = val & 1u;
    const uint32_t b = ((word >> ((col & 15) * 2)) & 3u) ^ (s << 1);
    return t == 0 ? next_sfx(key, b, a.pw1, a.pw2) : prev_pfx(key, b, a.inv1, a.inv2);
}

// ---------------------------------------------------------------- lists
// The list of iteration g as read (round r0 + g) and as written.
struct ListIn {
    const uint4 *lst;      // regions, bin-major
    uint32_t cap;          // entries per region
    const uint4 *spill;    // entries past a region's capacity ...
    const uint32_t *stag;  // ... and their bins
    const uint32_t *spill_n;
    const uint32_t *cnt;   // entries of each bin
};
struct ListOut {
    uint4 *lst;
    uint32_t cap;
    uint4 *spill;
    uint32_t *stag;
    uint32_t *spill_n;
    uint32_t *cnt;
};
EMP_DEV ListIn list_in(const BktJob &J, uint32_t g) {
    ListIn l;
    l.lst = reinterpret_cast<const uint4 *>(J.lst[g & 1]);
    l.cap = J.cap;
    l.spill = reinterpret_cast<const uint4 *>(J.spill[g & 1]);
    l.stag = J.spill_tag[g & 1];
    l.spill_n = J.spill_n + g;
    l.cnt = J.cnt + (uint64_t)g * 2 * J.nb_max;
    return l;
}
EMP_DEV ListOut list_out(const BktJob &J, uint32_t g) {
    ListOut l;
    l.lst = reinterpret_cast<uint4 *>(J.lst[g & 1]);
    l.cap = J.cap;
    l.spill = reinterpret_cast<uint4 *>(J.spill[g & 1]);
    l.stag = J.spill_tag[g & 1];
    l.spill_n = J.spill_n + g;
    l.cnt = J.cnt + (uint64_t)g * 2 * J.nb_max;
    return l;
}
// entry e at position pos of bin `bin`: in the bin's region, or spilled
EMP_DEV void put_list(const ListOut &o, uint32_t bin, uint32_t pos, const uint4 &e) {
    if (pos < o.cap) {
        o.lst[(uint64_t)bin * o.cap + pos] = e;
    } else {
        const uint32_t q = atomicAdd(o.spill_n, 1u);
        o.spill[q] = e;
        o.stag[q] = bin;
    }
}

// Lists of more than kBktMaxBuckets buckets, whose bins do not fit a
// shared-memory histogram: an entry takes its position from the bin counter
// directly, one atomic per run of equal bins within the warp.  Every lane of
// the warp calls it; lanes with act = false only vote.
EMP_DEV void put_direct(const ListOut &o, bool act, uint32_t bin, const uint4 &e) {
    const uint32_t m = __ballot_sync(0xffffffffu, act);
    if (!act) return;
    const uint32_t peers = __match_any_sync(m, bin);
    const uint32_t lane = threadIdx.x & 31, leader = __ffs(peers) - 1;
    uint32_t pos = 0;
    if (lane == leader) pos = atomicAdd(o.cnt + bin, (uint32_t)__popc(peers));
    pos = __shfl_sync(peers, pos, leader);
    put_list(o, bin, pos + __popc(peers & lanemask_lt_u32()), e);
}

// put_direct in two halves, so that several reservations can be in flight:
// reserve_direct returns the leader's run start (in the leader's lane) and
// the lanes sharing the bin; position_direct gives each lane its position.
// Equal keys are common (overlapping reads), so runs of one bin in a warp
// take one atomic.
EMP_DEV uint32_t reserve_direct(const ListOut &o, bool act, uint32_t bin, uint32_t &peers) {
    const uint32_t m = __ballot_sync(0xffffffffu, act);
    peers = act ? __match_any_sync(m, bin) : 0u;
    if (act && (threadIdx.x & 31) == (uint32_t)(__ffs(peers) - 1)) return atomicAdd(o.cnt + bin, (uint32_t)__popc(peers));
    return 0u;
}
EMP_DEV uint32_t position_direct(uint32_t peers, uint32_t run) {
    return __shfl_sync(peers, run, __ffs(peers) - 1) + __popc(peers & lanemask_lt_u32());
}

// Add this CTA's kept entries and suffixes to a round's counts (sh.kept and
// sh.sfx zeroed, then a __syncthreads, before the per-thread counts came in).
EMP_DEV void add_counts(BktRound &nx, uint32_t kept, uint32_t sfx, BShared &sh) {
    if (kept) atomicAdd(&sh.kept, kept);
    if (sfx) atomicAdd(&sh.sfx, sfx);
    __syncthreads();
    if (threadIdx.x == 0) {
        if (sh.kept) atomicAdd(reinterpret_cast<unsigned long long *>(&nx.n), (unsigned long long)sh.kept);
        if (sh.sfx) atomicAdd(reinterpret_cast<unsigned long long *>(&nx.s), (unsigned long long)sh.sfx);
    }
    __syncthreads();
}

// hist[b] (this tile's count of bin b) -> its local start; returns the
// tile's entry count.
EMP_DEV uint32_t bin_starts(uint32_t *hist, uint32_t nbin, BShared &sh) {
    const uint32_t per = (nbin + kT - 1) / kT;
    const uint32_t b0 = threadIdx.x * per < nbin ? threadIdx.x * per : nbin;
    const uint32_t b1 = b0 + per < nbin ? b0 + per : nbin;
    uint32_t run = 0;
    for (uint32_t b = b0; b < b1; ++b) run += hist[b];
    uint32_t kept;
    uint32_t ex = block_exclusive_scan<kT, uint32_t>(run, sh.scan32, &kept);
    for (uint32_t b = b0; b < b1; ++b) {
        const uint32_t h = hist[b];
        hist[b] = ex;
        ex += h;
    }
    __syncthreads();
    return kept;
}

// Reserve this tile's entries of every bin in the list's bin counters
// (hist[b] = the bin's local start on entry).  Afterwards hist[b] = the
// bin's global position minus its local start (mod 2^32), or the global
// position itself when `base` is set.
EMP_DEV void reserve_bins(uint32_t *hist, uint32_t nbin, uint32_t kept, uint32_t *cnt, bool base) {
    constexpr int kMaxPer = 2 * kBktMaxBuckets / kT;
    const uint32_t per = (nbin + kT - 1) / kT;
    const uint32_t b0 = threadIdx.x * per < nbin ? threadIdx.x * per : nbin;
    const uint32_t b1 = b0 + per < nbin ? b0 + per : nbin;
    uint32_t v[kMaxPer];
#pragma unroll
    for (int i = 0; i < kMaxPer; ++i) {
        const uint32_t b = b0 + i;
        v[i] = 0;
        if (b < b1) {
            const uint32_t lo = hist[b], hi = b + 1 < nbin ? hist[b + 1] : kept;
            const uint32_t g = hi > lo ? atomicAdd(cnt + b, hi - lo) : 0u;
            v[i] = base ? g : g - lo;
        }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kMaxPer; ++i)
        if (b0 + i < b1) hist[b0 + i] = v[i];
    __syncthreads();
}

// ---------------------------------------------------------------- prologue
// Tile k of the launch's input list -> round r0's list (iteration 0's bins).
EMP_COLD void prologue_tile(BktJob &J, uint32_t k, BShared &sh, uint8_t *smem) {
    BktRound &I = J.meta[J.r0];
    const uint64_t n_in = J.n_in;
    const uint32_t nb = bkt_count(n_in, J.wave, J.mean), nbin = 2 * nb;
    const StepArgs a = step_args(J, sh.tab, J.r0, true);
    const ListOut lo = list_out(J, 0);
    uint32_t *hist = reinterpret_cast<uint32_t *>(smem);
    uint4 *stage = reinterpret_cast<uint4 *>(smem + 2 * kBktMaxBuckets * 4);
    uint16_t *sbin = reinterpret_cast<uint16_t *>(stage + kBktTile);
    const bool direct = nb > kBktMaxBuckets;
    if (!direct)
        for (uint32_t i = threadIdx.x; i < nbin; i += kT) hist[i] = 0;
    if (threadIdx.x == 0) {
        sh.sfx = 0;
        sh.kept = 0;
    }
    __syncthreads();
    const uint64_t base = (uint64_t)k * kBktTile;
    sprobe(sh, 23);
    uint64_t key[kC];
    uint32_t val[kC], word[kC], rank[kC], bin[kC];
    bool keep[kC];
#pragma unroll
    for (int c = 0; c < kC; ++c) {  // the entries
        const uint64_t e = base + c * kT + threadIdx.x;
        keep[c] = e < n_in;
        key[c] = keep[c] ? __ldcg(J.lk_in + e) : 0;
        val[c] = keep[c] ? __ldcg(J.lv_in + e) : 0;
    }
    const bool some_used = J.r0 > 0;  // host-synchronised rounds ran before the launch
#pragma unroll
    for (int c = 0; c < kC; ++c) {  // used before the launch; the base words
        word[c] = 0;
        if (!keep[c]) continue;
        const uint32_t rid = val[c] & 0x7fffffffu;
        if (some_used) keep[c] = ((val[c] >> 31) ? J.used_p[rid] : J.used_s[rid]) == 0;
        if (keep[c]) word[c] = refill_word(a, val[c]);
    }
    if (direct) {  // hash step, bin, position straight from the bin counter
        sprobe(sh, 24);
        uint32_t kept = 0, sfx = 0;
#pragma unroll
        for (int c = 0; c < kC; ++c) {
            uint32_t bn = 0;
            if (keep[c]) {
                key[c] = step_key(a, key[c], val[c], word[c]);
                bn = 2 * bkt_of(sort_key(key[c], val[c]), nb) + (val[c] >> 31);
                ++kept;
                sfx += (val[c] >> 31) == 0;
            }
            put_direct(lo, keep[c], bn, make_uint4((uint32_t)key[c], (uint32_t)(key[c] >> 32), val[c], word[c]));
        }
        sprobe(sh, 25);
        add_counts(I, kept, sfx, sh);
        sprobe(sh, 26);
        return;
    }
    uint32_t sfx = 0;
#pragma unroll
    for (int c = 0; c < kC; ++c) {  // hash step, bin, rank within the tile's bin
        if (!keep[c]) continue;
        key[c] = step_key(a, key[c], val[c], word[c]);
        bin[c] = 2 * bkt_of(sort_key(key[c], val[c]), nb) + (val[c] >> 31);
        rank[c] = atomicAdd(&hist[bin[c]], 1u);
        sfx += (val[c] >> 31) == 0;
    }
    if (sfx) atomicAdd(&sh.sfx, sfx);
    __syncthreads();
    const uint32_t kept = bin_starts(hist, nbin, sh);
    if (threadIdx.x == 0) {
        if (kept) atomicAdd(reinterpret_cast<unsigned long long *>(&I.n), (unsigned long long)kept);
        if (sh.sfx) atomicAdd(reinterpret_cast<unsigned long long *>(&I.s), (unsigned long long)sh.sfx);
    }
#pragma unroll
    for (int c = 0; c < kC; ++c) {  // the tile in bin order
        if (!keep[c]) continue;
        const uint32_t d = hist[bin[c]] + rank[c];
        stage[d] = make_uint4((uint32_t)key[c], (uint32_t)(key[c] >> 32), val[c], word[c]);
        sbin[d] = (uint16_t)bin[c];
    }
    __syncthreads();
    reserve_bins(hist, nbin, kept, lo.cnt, false);
    for (uint32_t x = threadIdx.x; x < kept; x += kT) put_list(lo, sbin[x], x + hist[sbin[x]], stage[x]);
    __syncthreads();
}

// ---------------------------------------------------------------- gather
// global -> shared copy of 4 or 8 bytes that completes asynchronously
// (cp.async; cp.async.wait_all waits for this thread's copies)
EMP_DEV void cp_async(void *dst_smem, const void *src, int bytes) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst_smem);
    if (bytes == 8) asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
    else asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}

EMP_DEV void put_entry(const Stage &v, uint32_t d, const uint4 *src) {
    const uint4 q = __ldcg(src);
    v.key[d] = (uint64_t)q.x | ((uint64_t)q.y << 32);
    v.val[d] = q.z;
    v.word[d] = q.w;
    v.flag[d] = 0;
}

// Entries of the list's bins below bin `bin` (the bucket's position in
// bucket order: its region of the global scratch).
EMP_DEV uint64_t bins_below(const uint32_t *cnt, uint32_t bin, BShared &sh) {
    uint64_t pre = 0;
    for (uint32_t q = threadIdx.x; q < bin; q += kT) pre += __ldcg(cnt + q);
    uint64_t tot;
    block_exclusive_scan<kT, uint64_t>(pre, sh.scan64, &tot);
    return tot;
}

// Bucket b with spilled entries or too big for shared memory: the region
// parts, then the bins' spilled entries found in the list's spill area;
// staged in shared memory when it fits, else in the scratch region G.
EMP_COLD uint32_t gather_general(const BktJob &J, const ListIn li, uint32_t b, uint32_t cS, uint32_t cP, BShared &sh,
                                 uint8_t *smem, Stage &v, uint64_t &G) {
    const uint32_t total = cS + cP;
    G = bins_below(li.cnt, 2 * b, sh);
    if (total <= kBStage) {
        v.key = reinterpret_cast<uint64_t *>(smem + kOffKey);
        v.val = reinterpret_cast<uint32_t *>(smem + kOffVal);
        v.word = reinterpret_cast<uint32_t *>(smem + kOffWord);
        v.flag = smem + kOffFlag;
    } else {
        BScratch gs;
        scratch_layout(J.scratch, J.n_max, &gs);
        v.key = gs.key + G;
        v.val = gs.val + G;
        v.word = gs.word + G;
        v.flag = gs.flag + G;
    }
    const uint32_t rS = cS < li.cap ? cS : li.cap, rP = cP < li.cap ? cP : li.cap;
    const uint4 *rs = li.lst + (uint64_t)(2 * b) * li.cap, *rp = li.lst + (uint64_t)(2 * b + 1) * li.cap;
    for (uint32_t x = threadIdx.x; x < rS; x += kT) put_entry(v, x, rs + x);
    for (uint32_t x = threadIdx.x; x < rP; x += kT) put_entry(v, cS + x, rp + x);
    if (cS > li.cap || cP > li.cap) {
        if (threadIdx.x == 0) {
            sh.cnt = 0;
            sh.tile = 0;
        }
        __syncthreads();
        const uint32_t ns = __ldcg(li.spill_n);
        for (uint32_t q = threadIdx.x; q < ns; q += kT) {
            const uint32_t t = __ldcg(li.stag + q);
            if (t == 2 * b) put_entry(v, rS + atomicAdd(&sh.cnt, 1u), li.spill + q);
            else if (t == 2 * b + 1) put_entry(v, cS + rP + atomicAdd(&sh.tile, 1u), li.spill + q);
        }
    }
    __syncthreads();
    return total;
}

// Gather bucket b of the list: its suffix region, then its prefix region
// (two contiguous runs), so the bucket is staged suffixes first.  Returns the
// bucket's size; S = its suffixes, G = its position in bucket order (for the
// global scratch), v = shared memory or the scratch region.
EMP_COLD uint32_t gather(const BktJob &J, const ListIn li, uint32_t b, BShared &sh, uint8_t *smem, Stage &v,
                         uint32_t &S, uint64_t &G) {
    if (threadIdx.x == 0) {
        sh.cnt = __ldcg(li.cnt + 2 * b);
        sh.tile = __ldcg(li.cnt + 2 * b + 1);
    }
    __syncthreads();
    const uint32_t cS = sh.cnt, cP = sh.tile, total = cS + cP;
    S = cS;
    sprobe(sh, 11);
    if (total <= kBStage && cS <= li.cap && cP <= li.cap) {
        G = 0;
        v.key = reinterpret_cast<uint64_t *>(smem + kOffKey);
        v.val = reinterpret_cast<uint32_t *>(smem + kOffVal);
        v.word = reinterpret_cast<uint32_t *>(smem + kOffWord);
        v.flag = smem + kOffFlag;
        const uint64_t rs = (uint64_t)(2 * b) * li.cap, rp = (uint64_t)(2 * b + 1) * li.cap;
        sprobe(sh, 12);
        // asynchronous copies straight into the staged arrays (every entry's
        // copies in flight at once, no registers): key 8 bytes, value 4, word 4
        for (uint32_t x = threadIdx.x; x < total; x += kT) {
            const uint4 *e = li.lst + (x < cS ? rs + x : rp + (x - cS));
            cp_async(v.key + x, e, 8);
            cp_async(v.val + x, reinterpret_cast<const uint8_t *>(e) + 8, 4);
            cp_async(v.word + x, reinterpret_cast<const uint8_t *>(e) + 12, 4);
            v.flag[x] = 0;
        }
        asm volatile("cp.async.wait_all;\n" ::: "memory");
        __syncthreads();
        return total;
    }
    return gather_general(J, li, b, cS, cP, sh, smem, v, G);
}

// ---------------------------------------------------------------- matching
// Hash slots are u32: bit 31 matched, bits 13-30 an 18-bit tag of the key,
// bits 0-12 the staged index of a suffix with that key (keys compared in full
// through it).  A tag of all ones is never used, so kSlotEmpty is no slot.
constexpr uint32_t kSlotEmpty = 0xffffffffu;
constexpr uint32_t kSlotMatched = 0x80000000u;
static_assert(kBStage <= 8192 && kBHash <= 16384, "13-bit staged indices, slot bits below the tag's");

EMP_DEV void hash_tag(uint64_t key, uint32_t &slot, uint32_t &tag) {
    const uint32_t h = (uint32_t)((key * 0x9E3779B97F4A7C15ull) >> 32);
    slot = h & (kBHash - 1);
    tag = (h >> 14) & 0x3ffffu;
    if (tag == 0x3ffffu) tag = 0x3fffeu;
}
EMP_DEV bool slot_holds(uint32_t w, uint32_t tag, uint64_t k, const uint64_t *key) {
    return ((w >> 13) & 0x3ffffu) == tag && key[w & 8191u] == k;
}

// Flag kMatched on every staged entry whose key occurs in both tables; the
// bucket is staged in shared memory, suffixes [0, S), prefixes [S, total).
// Each thread works on kU entries at once so that their shared-memory round
// trips overlap; a collision falls back to a probe loop.
EMP_COLD void match_smem(uint32_t total, uint32_t S, uint8_t *smem) {
    constexpr int kU = 4;
    const uint64_t *key = reinterpret_cast<const uint64_t *>(smem + kOffKey);
    uint8_t *flag = smem + kOffFlag;
    uint32_t *slot = reinterpret_cast<uint32_t *>(smem + kOffReg + kHSlot);
    uint16_t *sslot = reinterpret_cast<uint16_t *>(smem + kOffReg + kHSuffixSlot);
    for (uint32_t s = threadIdx.x; s < kBHash / 4; s += kT)
        reinterpret_cast<uint4 *>(slot)[s] = make_uint4(kSlotEmpty, kSlotEmpty, kSlotEmpty, kSlotEmpty);
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
                    flag[x] = kMatched;
                    break;
                }
                sl = (sl + 1) & (kBHash - 1);
                ww = slot[sl];
            }
        }
    }
    __syncthreads();
    for (uint32_t x = threadIdx.x; x < S; x += kT)  // suffixes: matched?
        if (slot[sslot[x]] & kSlotMatched) flag[x] = kMatched;
    __syncthreads();
}

// Cheaper matcher for the usual bucket, where at most a third of the entries
// match: a 2-bit Bloom filter of the suffix keys (128K bits) passes the
// prefixes that may match; a second filter of those prefixes' keys passes
// the suffixes that may match; the two short lists are then matched through
// a small hash set of the suffix list's keys.  No entry that matches is
// filtered out, so the flags equal match_smem's.  Returns false (flags
// untouched) when a list would be longer than kListMax; the caller then uses
// match_smem.
constexpr uint32_t kFilterWords = 2048;  // 64K bits per filter
constexpr uint32_t kListMax = 1024;
constexpr uint32_t kListHash = 4096;     // slots of the short lists' hash set (power of two)
constexpr size_t kFBm1 = 0, kFBm2 = kFilterWords * 4, kFPl = 2 * kFilterWords * 4, kFSl = kFPl + kListMax * 2;
constexpr size_t kFHash = kFSl + kListMax * 2;      // u32 [kListHash]: suffix-list index, bit 31 matched
constexpr size_t kFSlotOf = kFHash + kListHash * 4; // u16 [kListMax]: the slot of each suffix-list entry
static_assert(kFSlotOf + kListMax * 2 <= kRegion, "filters, lists and their hash set fit the region");
static_assert(kListMax < kListHash && kListMax <= 65536, "the hash set never fills; u16 list indices");

EMP_DEV void filter_bits(uint64_t key, uint32_t &b1, uint32_t &b2) {
    const uint32_t h = (uint32_t)((key * 0x9E3779B97F4A7C15ull) >> 32);
    b1 = h & (kFilterWords * 32 - 1);
    b2 = (h >> 16) & (kFilterWords * 32 - 1);
}
EMP_DEV bool filter_has(const uint32_t *bm, uint32_t b1, uint32_t b2) {
    return ((bm[b1 >> 5] >> (b1 & 31)) & (bm[b2 >> 5] >> (b2 & 31)) & 1u) != 0;
}
// warp-aggregated append of x to list (count in *n); false once it is full
EMP_DEV void list_push(bool f, uint32_t x, uint16_t *list, uint32_t *n) {
    const uint32_t m = __ballot_sync(0xffffffffu, f);
    if (!m) return;
    const uint32_t lane = threadIdx.x & 31, leader = __ffs(m) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(n, (uint32_t)__popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    const uint32_t d = base + __popc(m & lanemask_lt_u32());
    if (f && d < kListMax) list[d] = (uint16_t)x;
}

EMP_DEV bool match_filter(uint32_t total, uint32_t S, uint8_t *smem, BShared &sh) {
    const uint64_t *key = reinterpret_cast<const uint64_t *>(smem + kOffKey);
    uint8_t *flag = smem + kOffFlag;
    uint8_t *reg = smem + kOffReg;
    uint32_t *bm1 = reinterpret_cast<uint32_t *>(reg + kFBm1);
    uint32_t *bm2 = reinterpret_cast<uint32_t *>(reg + kFBm2);
    uint16_t *pl = reinterpret_cast<uint16_t *>(reg + kFPl);
    uint16_t *sl = reinterpret_cast<uint16_t *>(reg + kFSl);
    uint32_t *hs = reinterpret_cast<uint32_t *>(reg + kFHash);
    for (uint32_t i = threadIdx.x; i < 2 * kFilterWords / 4; i += kT)
        reinterpret_cast<uint4 *>(bm1)[i] = make_uint4(0, 0, 0, 0);  // bm1 and bm2
    for (uint32_t i = threadIdx.x; i < kListHash / 4; i += kT)  // the short lists' hash set, for later
        reinterpret_cast<uint4 *>(hs)[i] = make_uint4(kSlotEmpty, kSlotEmpty, kSlotEmpty, kSlotEmpty);
    if (threadIdx.x == 0) {
        sh.cnt = 0;
        sh.tile = 0;
    }
    __syncthreads();
    for (uint32_t x = threadIdx.x; x < S; x += kT) {  // suffix keys into filter 1
        uint32_t b1, b2;
        filter_bits(key[x], b1, b2);
        atomicOr(bm1 + (b1 >> 5), 1u << (b1 & 31));
        atomicOr(bm1 + (b2 >> 5), 1u << (b2 & 31));
    }
    __syncthreads();
    for (uint32_t x0 = S; x0 < total; x0 += kT) {  // prefixes through filter 1, their keys into filter 2
        const uint32_t x = x0 + threadIdx.x;
        bool f = false;
        if (x < total) {
            uint32_t b1, b2;
            filter_bits(key[x], b1, b2);
            f = filter_has(bm1, b1, b2);
            if (f) {
                atomicOr(bm2 + (b1 >> 5), 1u << (b1 & 31));
                atomicOr(bm2 + (b2 >> 5), 1u << (b2 & 31));
            }
        }
        list_push(f, x, pl, &sh.cnt);
    }
    __syncthreads();
    const uint32_t np = sh.cnt;
    if (np > kListMax) return false;
    for (uint32_t x0 = 0; x0 < S; x0 += kT) {  // suffixes through filter 2
        const uint32_t x = x0 + threadIdx.x;
        bool f = false;
        if (x < S) {
            uint32_t b1, b2;
            filter_bits(key[x], b1, b2);
            f = filter_has(bm2, b1, b2);
        }
        list_push(f, x, sl, &sh.tile);
    }
    __syncthreads();
    const uint32_t ns = sh.tile;
    if (ns > kListMax) return false;
    // the two lists: suffix-list keys into a hash set (equal keys share the
    // slot of the first one in), prefixes probe it, then every suffix of a
    // slot that a prefix hit is flagged
    uint16_t *slot_of = reinterpret_cast<uint16_t *>(reg + kFSlotOf);
    for (uint32_t j = threadIdx.x; j < ns; j += kT) {
        const uint64_t k = key[sl[j]];
        uint32_t sl0 = (uint32_t)((k * 0x9E3779B97F4A7C15ull) >> 32) & (kListHash - 1);
        for (uint32_t probes = 0; probes < kListHash; ++probes) {
            const uint32_t old = atomicCAS(hs + sl0, kSlotEmpty, j);
            if (old == kSlotEmpty || key[sl[old & 0xffffu]] == k) break;
            sl0 = (sl0 + 1) & (kListHash - 1);
        }
        slot_of[j] = (uint16_t)sl0;
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < np; i += kT) {
        const uint32_t xp = pl[i];
        const uint64_t k = key[xp];
        uint32_t sl0 = (uint32_t)((k * 0x9E3779B97F4A7C15ull) >> 32) & (kListHash - 1);
        for (uint32_t probes = 0; probes < kListHash; ++probes) {
            const uint32_t w = hs[sl0];
            if (w == kSlotEmpty) break;
            if (key[sl[w & 0xffffu]] == k) {
                flag[xp] = kMatched;
                if (!(w & kSlotMatched)) atomicOr(hs + sl0, kSlotMatched);
                break;
            }
            sl0 = (sl0 + 1) & (kListHash - 1);
        }
    }
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < ns; j += kT)
        if (hs[slot_of[j]] & kSlotMatched) flag[sl[j]] = kMatched;
    __syncthreads();
    return true;
}

// The same for a bucket staged in global scratch: open addressing on the full
// keys, 2 x total slots, in the bucket's scratch region.
EMP_COLD void match_global(const Stage &v, uint32_t total, uint32_t S, const BScratch &gs, uint64_t G) {
    uint64_t *hslot = gs.hslot + 2 * G;
    uint8_t *hmatch = gs.hmatch + 2 * G;
    uint32_t *sslot = gs.sslot + G;
    const uint32_t hcap = 2 * total;
    auto slot_of = [&](uint64_t key) -> uint32_t {
        return (uint32_t)((key * 0x9E3779B97F4A7C15ull) >> 32) % hcap;
    };
    for (uint32_t s = threadIdx.x; s < hcap; s += kT) {
        hslot[s] = kEmptySlot;
        hmatch[s] = 0;
    }
    __syncthreads();
    for (uint32_t x = threadIdx.x; x < S; x += kT) {
        const uint64_t key = ldv(v.key + x);
        uint32_t s = slot_of(key);
        for (uint32_t probes = 0; probes < hcap; ++probes) {
            const uint64_t prev = atomicCAS(reinterpret_cast<unsigned long long *>(hslot + s),
                                            (unsigned long long)kEmptySlot, (unsigned long long)key);
            if (prev == kEmptySlot || prev == key) break;
            s = s + 1 == hcap ? 0 : s + 1;
        }
        sslot[x] = s;
    }
    __syncthreads();
    for (uint32_t x = S + threadIdx.x; x < total; x += kT) {
        const uint64_t key = ldv(v.key + x);
        uint32_t s = slot_of(key);
        for (uint32_t probes = 0; probes < hcap; ++probes) {
            const uint64_t h = ldv(hslot + s);
            if (h == kEmptySlot) break;
            if (h == key) {
                hmatch[s] = 1;
                v.flag[x] = kMatched;
                break;
            }
            s = s + 1 == hcap ? 0 : s + 1;
        }
    }
    __syncthreads();
    for (uint32_t x = threadIdx.x; x < S; x += kT)
        if (ldv(hmatch + ldv(sslot + x))) v.flag[x] = kMatched;
    __syncthreads();
}

// ---------------------------------------------------------------- sort + join
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

// Rank the c matched entries by (sort key, tie) into skey/sval/sidx and count
// each suffix's edges; returns the bucket's edge count (cnt then holds
// exclusive edge offsets).  Chunks of 512 are ranked by comparing all pairs,
// then each entry adds, per other chunk, the entries before it (binary
// search), so any c works.
EMP_DEV uint64_t join_count(const Cands &w, uint32_t c, BShared &sh);

EMP_COLD uint64_t sort_and_count(const Cands &w, uint32_t c, BShared &sh) {
    for (uint32_t x = threadIdx.x; x < c; x += kT) {
        const uint32_t val = ldv(w.cv + x);
        w.sk[x] = sort_key(ldv(w.ck + x), val);
        w.tb[x] = tie_of(val);
    }
    __syncthreads();
    const uint32_t nch = (c + kT - 1) / kT;
    for (uint32_t q = 0; q < nch; ++q) {
        const uint32_t lo = q * kT, m = c - lo < kT ? c - lo : kT;
        if (threadIdx.x < m) {
            const uint32_t x = lo + threadIdx.x;
            const uint64_t skx = ldv(w.sk + x);
            const uint32_t tbx = ldv(w.tb + x);
            uint32_t rk = 0;
            for (uint32_t u = 0; u < m; ++u) rk += before(ldv(w.sk + lo + u), ldv(w.tb + lo + u), skx, tbx);
            w.ord[lo + rk] = x;
            w.cnt[x] = rk;
        }
    }
    __syncthreads();
    for (uint32_t x = threadIdx.x; x < c; x += kT) {
        const uint64_t skx = ldv(w.sk + x);
        const uint32_t tbx = ldv(w.tb + x);
        const uint32_t qx = x / kT;
        uint32_t rk = (uint32_t)ldv(w.cnt + x);
        for (uint32_t q = 0; q < nch; ++q) {
            if (q == qx) continue;
            const uint32_t lo = q * kT, m = c - lo < kT ? c - lo : kT;
            uint32_t a = 0, z = m;
            while (a < z) {
                const uint32_t mid = (a + z) >> 1;
                const uint32_t y = ldv(w.ord + lo + mid);
                if (before(ldv(w.sk + y), ldv(w.tb + y), skx, tbx)) a = mid + 1;
                else z = mid;
            }
            rk += a;
        }
        w.skey[rk] = ldv(w.ck + x);
        w.sval[rk] = ldv(w.cv + x);
        w.sidx[rk] = ldv(w.cx + x);
    }
    __syncthreads();
    return join_count(w, c, sh);
}

// Per suffix of the sorted matched entries: the prefixes of its equal-key run
// from other reads.  Returns the bucket's edge count; cnt then holds each
// suffix's exclusive edge offset.
EMP_DEV uint64_t join_count(const Cands &w, uint32_t c, BShared &sh) {
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

// ---------------------------------------------------------------- matched entries in shared memory
// Up to kBCand matched entries of a bucket staged in shared memory are ranked
// there, 26 bytes each in the region; their keys and values are read from the
// stage through their staged index.
constexpr uint32_t kBCand = 1408;
constexpr uint32_t kFine = 512;     // fine bins of the ranking
constexpr uint32_t kSmallRank = 96; // up to this many: all pairs compared
constexpr size_t kSCx = 0;                                  // u16 staged index, compaction order
constexpr size_t kSSk = (kSCx + kBCand * 2 + 7) / 8 * 8;    // u64 sort key
constexpr size_t kSTb = kSSk + kBCand * 8;                  // u32 tie key
constexpr size_t kSOrd = kSTb + kBCand * 4;                 // u32 fine bin << 16 | rank within the bin
constexpr size_t kSTmp = kSOrd + kBCand * 4;                // u16 compaction index, grouped by fine bin
constexpr size_t kSIdx = kSTmp + kBCand * 2;                // u16 staged index in (sort key, tie) order
constexpr size_t kSCnt = (kSIdx + kBCand * 2 + 3) / 4 * 4;  // u32 edges of each suffix, then their offsets
constexpr size_t kSHist = kSCnt + kBCand * 4;               // u32 [kFine + 1] fine-bin starts
static_assert(kSHist + (kFine + 1) * 4 <= kRegion, "matched entries fit the region");
static_assert(kBStage <= 65535 && kFine == 2 * kT, "u16 staged indices; two fine bins per thread");

struct CandS {
    uint16_t *cx, *tmp, *sidx;
    uint64_t *sk;
    uint32_t *tb, *ord, *cnt, *hist;
};
EMP_DEV CandS cand_s(uint8_t *smem) {
    uint8_t *reg = smem + kOffReg;
    CandS w;
    w.cx = reinterpret_cast<uint16_t *>(reg + kSCx);
    w.sk = reinterpret_cast<uint64_t *>(reg + kSSk);
    w.tb = reinterpret_cast<uint32_t *>(reg + kSTb);
    w.ord = reinterpret_cast<uint32_t *>(reg + kSOrd);
    w.tmp = reinterpret_cast<uint16_t *>(reg + kSTmp);
    w.sidx = reinterpret_cast<uint16_t *>(reg + kSIdx);
    w.cnt = reinterpret_cast<uint32_t *>(reg + kSCnt);
    w.hist = reinterpret_cast<uint32_t *>(reg + kSHist);
    return w;
}

// The staged indices of the matched entries into w.cx (any order: the
// ranking fixes it), at most kBCand of them; returns how many there are.
EMP_DEV uint32_t compact_s(const uint8_t *flag, uint32_t total, const CandS &w, BShared &sh) {
    if (threadIdx.x == 0) sh.tile = 0;
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31;
    for (uint32_t x0 = 0; x0 < total; x0 += kT) {
        const uint32_t x = x0 + threadIdx.x;
        const bool f = x < total && (flag[x] & kMatched);
        const uint32_t m = __ballot_sync(0xffffffffu, f);
        if (!m) continue;
        const uint32_t leader = __ffs(m) - 1;
        uint32_t base = 0;
        if (lane == leader) base = atomicAdd(&sh.tile, (uint32_t)__popc(m));
        base = __shfl_sync(0xffffffffu, base, leader);
        const uint32_t d = base + __popc(m & lanemask_lt_u32());
        if (f && d < kBCand) w.cx[d] = (uint16_t)x;
    }
    __syncthreads();
    return sh.tile;
}

// Rank the c <= kBCand matched entries of bucket b (nb buckets) by (sort key,
// tie): w.sidx[rank] = staged index.  Up to kSmallRank entries compare all
// pairs; more are counted into kFine finer bins (the same top-24-bit field of
// the sort key scaled to nb * kFine bins, so bin order is key order) and
// ranked among the members of their bin.
EMP_DEV void rank_s(const CandS &w, uint32_t c, uint32_t b, uint32_t nb, const uint64_t *key, const uint32_t *val,
                    BShared &sh) {
    for (uint32_t x = threadIdx.x; x < c; x += kT) {
        const uint32_t sx = w.cx[x], v = val[sx];
        w.sk[x] = sort_key(key[sx], v);
        w.tb[x] = tie_of(v);
    }
    __syncthreads();
    if (c <= kSmallRank) {
        if (threadIdx.x < c) {
            const uint32_t x = threadIdx.x;
            const uint64_t skx = w.sk[x];
            const uint32_t tbx = w.tb[x];
            uint32_t r = 0;
            for (uint32_t y = 0; y < c; ++y) r += before(w.sk[y], w.tb[y], skx, tbx);
            w.sidx[r] = w.cx[x];
        }
        __syncthreads();
        return;
    }
    uint32_t *hist = w.hist;
    const uint64_t scale = (uint64_t)nb * kFine, lo_bin = (uint64_t)b * kFine;
    for (uint32_t i = threadIdx.x; i <= kFine; i += kT) hist[i] = 0;
    __syncthreads();
    for (uint32_t x = threadIdx.x; x < c; x += kT) {
        const uint32_t f = (uint32_t)((((w.sk[x] >> 35) * scale) >> 24) - lo_bin);
        w.ord[x] = (f << 16) | atomicAdd(&hist[f], 1u);
    }
    __syncthreads();
    {  // bin starts: two bins per thread
        const uint32_t f0 = 2 * threadIdx.x;
        const uint32_t a0 = hist[f0], a1 = hist[f0 + 1];
        uint32_t tot;
        const uint32_t ex = block_exclusive_scan<kT, uint32_t>(a0 + a1, sh.scan32, &tot);
        hist[f0] = ex;
        hist[f0 + 1] = ex + a0;
        if (threadIdx.x == 0) hist[kFine] = tot;
    }
    __syncthreads();
    for (uint32_t x = threadIdx.x; x < c; x += kT) w.tmp[hist[w.ord[x] >> 16] + (w.ord[x] & 0xffffu)] = (uint16_t)x;
    __syncthreads();
    for (uint32_t q = threadIdx.x; q < c; q += kT) {
        const uint32_t x = w.tmp[q], f = w.ord[x] >> 16;
        const uint32_t lo = hist[f], hi = hist[f + 1];
        const uint64_t skx = w.sk[x];
        const uint32_t tbx = w.tb[x];
        uint32_t r = lo;
        for (uint32_t y = lo; y < hi; ++y) {
            const uint32_t z = w.tmp[y];
            r += before(w.sk[z], w.tb[z], skx, tbx);
        }
        w.sidx[r] = w.cx[x];
    }
    __syncthreads();
}

// Per suffix of the ranked entries: the prefixes of its equal-key run from
// other reads (get_edges, overlap.cu:557-603).  w.cnt then holds each one's
// exclusive edge offset; returns the bucket's edge count.
EMP_DEV uint64_t join_count_s(const CandS &w, uint32_t c, const uint64_t *key, const uint32_t *val, BShared &sh) {
    for (uint32_t i = threadIdx.x; i < c; i += kT) {
        uint32_t cc = 0;
        const uint32_t si = w.sidx[i], vi = val[si];
        if (!(vi >> 31)) {
            const uint64_t ki = key[si];
            const uint32_t ri = (vi & 0x7fffffffu) >> 1;
            for (uint32_t j = i + 1; j < c; ++j) {
                const uint32_t sj = w.sidx[j];
                if (key[sj] != ki) break;
                const uint32_t vj = val[sj];
                cc += (vj >> 31) && ((vj & 0x7fffffffu) >> 1) != ri;
            }
        }
        w.cnt[i] = cc;
    }
    __syncthreads();
    uint32_t run = 0;
    for (uint32_t x0 = 0; x0 < c; x0 += kT) {
        const uint32_t x = x0 + threadIdx.x;
        const uint32_t v = x < c ? w.cnt[x] : 0u;
        uint32_t tot;
        const uint32_t ex = block_exclusive_scan<kT, uint32_t>(v, sh.scan32, &tot);
        if (x < c) w.cnt[x] = run + ex;
        run += tot;
        __syncthreads();
    }
    return run;
}

// The bucket's edges at ebase (only when they fit) and the used marks: a
// suffix with an edge, a prefix that got one.
EMP_DEV void write_edges_s(BktJob &J, const CandS &w, uint32_t c, uint64_t ebase, bool room, const uint64_t *key,
                           const uint32_t *val, uint8_t *flag) {
    for (uint32_t i = threadIdx.x; i < c; i += kT) {
        const uint32_t si = w.sidx[i], vi = val[si];
        if (vi >> 31) continue;
        const uint64_t ki = key[si];
        const uint32_t rs = vi & 0x7fffffffu, ri = rs >> 1;
        const uint64_t o0 = ebase + w.cnt[i];
        uint64_t o = o0;
        for (uint32_t j = i + 1; j < c; ++j) {
            const uint32_t sj = w.sidx[j];
            if (key[sj] != ki) break;
            const uint32_t vj = val[sj], pj = vj & 0x7fffffffu;
            if ((vj >> 31) && (pj >> 1) != ri) {
                if (room) {
                    J.sfrom[o] = rs;
                    J.sto[o] = pj;
                }
                flag[sj] = kMatched | kUsed;
                ++o;
            }
        }
        if (o != o0) flag[si] = kMatched | kUsed;
    }
    __syncthreads();
}

// ---------------------------------------------------------------- next round
// The next list has more than kBktMaxBuckets buckets: drop the used entries,
// apply round a.r's hash step to the rest and put each one straight at a
// position taken from its bin's counter (the stage may be shared memory or
// global scratch).
EMP_COLD void write_next_direct(const Stage &v, uint32_t total, const StepArgs a, uint32_t nb, const ListOut lo,
                                BktRound &nx, BShared &sh) {
    if (threadIdx.x == 0) {
        sh.sfx = 0;
        sh.kept = 0;
    }
    __syncthreads();
    uint32_t kept = 0, sfx = 0;
    constexpr int kU = 4;  // entries per thread in flight
    for (uint32_t x0 = 0; x0 < total; x0 += kU * kT) {
        bool act[kU];
        uint32_t vl[kU], wd[kU];
        uint64_t ky[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const uint32_t x = x0 + u * kT + threadIdx.x;
            act[u] = x < total && !(ldv(v.flag + x) & kUsed);
            vl[u] = wd[u] = 0;
            ky[u] = 0;
            if (act[u]) {
                vl[u] = ldv(v.val + x);
                wd[u] = ldv(v.word + x);
                ky[u] = ldv(v.key + x);
            }
        }
#pragma unroll
        for (int u = 0; u < kU; ++u)
            if (act[u] && needs_refill(a, vl[u])) wd[u] = refill_word(a, vl[u]);
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            uint32_t bn = 0;
            if (act[u]) {
                ky[u] = step_key(a, ky[u], vl[u], wd[u]);
                bn = 2 * bkt_of(sort_key(ky[u], vl[u]), nb) + (vl[u] >> 31);
                ++kept;
                sfx += (vl[u] >> 31) == 0;
            }
            put_direct(lo, act[u], bn, make_uint4((uint32_t)ky[u], (uint32_t)(ky[u] >> 32), vl[u], wd[u]));
        }
    }
    add_counts(nx, kept, sfx, sh);
}

// The same for a bucket staged in shared memory, in passes so that the
// global atomics are not a chain: (1) the hash step of every kept entry in
// place and its next bin, (2) kU positions per thread reserved back to back,
// then the stores.
EMP_COLD void write_next_direct_smem(uint32_t total, const StepArgs a, uint32_t nb, const ListOut lo, BktRound &nx,
                                     BShared &sh, uint8_t *smem) {
    uint64_t *key = reinterpret_cast<uint64_t *>(smem + kOffKey);
    const uint32_t *val = reinterpret_cast<const uint32_t *>(smem + kOffVal);
    uint32_t *word = reinterpret_cast<uint32_t *>(smem + kOffWord);
    const uint8_t *flag = smem + kOffFlag;
    uint32_t *bin = reinterpret_cast<uint32_t *>(smem + kOffReg);  // next bin, or ~0: used
    if (threadIdx.x == 0) {
        sh.sfx = 0;
        sh.kept = 0;
    }
    __syncthreads();  // the region's previous users are done
    uint32_t kept = 0, sfx = 0;
    constexpr int kA = 4;
    for (uint32_t x0 = 0; x0 < total; x0 += kA * kT) {
        uint32_t vl[kA], wd[kA];
        bool act[kA];
#pragma unroll
        for (int u = 0; u < kA; ++u) {
            const uint32_t x = x0 + u * kT + threadIdx.x;
            act[u] = x < total && !(flag[x] & kUsed);
            vl[u] = act[u] ? val[x] : 0u;
            wd[u] = act[u] ? word[x] : 0u;
        }
#pragma unroll
        for (int u = 0; u < kA; ++u)
            if (act[u] && needs_refill(a, vl[u])) wd[u] = refill_word(a, vl[u]);
#pragma unroll
        for (int u = 0; u < kA; ++u) {
            const uint32_t x = x0 + u * kT + threadIdx.x;
            if (x >= total) continue;
            uint32_t bn = ~0u;
            if (act[u]) {
                const uint64_t ky = step_key(a, key[x], vl[u], wd[u]);
                bn = 2 * bkt_of(sort_key(ky, vl[u]), nb) + (vl[u] >> 31);
                key[x] = ky;
                word[x] = wd[u];
                ++kept;
                sfx += (vl[u] >> 31) == 0;
            }
            bin[x] = bn;
        }
    }
    __syncthreads();
    sprobe(sh, 13);
    constexpr int kU = 8;
    for (uint32_t x0 = 0; x0 < total; x0 += kU * kT) {
        uint32_t bn[kU], pos[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const uint32_t x = x0 + u * kT + threadIdx.x;
            bn[u] = x < total ? bin[x] : ~0u;
        }
        uint32_t peers[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u)  // reservations, independent of one another
            pos[u] = reserve_direct(lo, bn[u] != ~0u, bn[u], peers[u]);
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            if (bn[u] == ~0u) continue;
            const uint32_t x = x0 + u * kT + threadIdx.x;
            const uint64_t ky = key[x];
            put_list(lo, bn[u], position_direct(peers[u], pos[u]),
                     make_uint4((uint32_t)ky, (uint32_t)(ky >> 32), val[x], word[x]));
        }
    }
    sprobe(sh, 15);
    add_counts(nx, kept, sfx, sh);
}

// Drop the used entries of the staged bucket, apply round a.r's hash step to
// the rest and write them into the next list's bins (nb buckets).  Counts go
// to the next round's BktRound.
EMP_COLD void write_next_smem(uint32_t total, const StepArgs a, uint32_t nb, const ListOut lo, BktRound &nx,
                              BShared &sh, uint8_t *smem) {
    uint64_t *key = reinterpret_cast<uint64_t *>(smem + kOffKey);
    uint32_t *val = reinterpret_cast<uint32_t *>(smem + kOffVal);
    uint32_t *word = reinterpret_cast<uint32_t *>(smem + kOffWord);
    const uint8_t *flag = smem + kOffFlag;
    uint8_t *reg = smem + kOffReg;
    uint32_t *hist = reinterpret_cast<uint32_t *>(reg + kPHist);
    uint16_t *rank16 = reinterpret_cast<uint16_t *>(reg + kPRank);
    uint16_t *bin16 = reinterpret_cast<uint16_t *>(reg + kPBin);
    const uint32_t nbin = 2 * nb;
    for (uint32_t i = threadIdx.x; i < nbin; i += kT) hist[i] = 0;
    if (threadIdx.x == 0) sh.sfx = 0;
    __syncthreads();
    uint32_t sfx = 0;
    constexpr int kU = 4;  // entries per thread in flight
    for (uint32_t x0 = 0; x0 < total; x0 += kU * kT) {
        bool act[kU];
        uint32_t vl[kU], wd[kU];
        uint64_t ky[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const uint32_t x = x0 + u * kT + threadIdx.x;
            act[u] = x < total && !(flag[x] & kUsed);
            if (act[u]) {
                vl[u] = val[x];
                wd[u] = word[x];
                ky[u] = key[x];
            }
        }
#pragma unroll
        for (int u = 0; u < kU; ++u)
            if (act[u] && needs_refill(a, vl[u])) wd[u] = refill_word(a, vl[u]);
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            if (!act[u]) continue;
            const uint32_t x = x0 + u * kT + threadIdx.x;
            ky[u] = step_key(a, ky[u], vl[u], wd[u]);
            key[x] = ky[u];
            word[x] = wd[u];
            const uint32_t bn = 2 * bkt_of(sort_key(ky[u], vl[u]), nb) + (vl[u] >> 31);
            rank16[x] = (uint16_t)atomicAdd(&hist[bn], 1u);
            bin16[x] = (uint16_t)bn;
            sfx += (vl[u] >> 31) == 0;
        }
    }
    if (sfx) atomicAdd(&sh.sfx, sfx);
    __syncthreads();
    sprobe(sh, 13);
    const uint32_t kept = bin_starts(hist, nbin, sh);
    if (threadIdx.x == 0) {
        if (kept) atomicAdd(reinterpret_cast<unsigned long long *>(&nx.n), (unsigned long long)kept);
        if (sh.sfx) atomicAdd(reinterpret_cast<unsigned long long *>(&nx.s), (unsigned long long)sh.sfx);
    }
    sprobe(sh, 14);
    reserve_bins(hist, nbin, kept, lo.cnt, true);  // hist[bin] = the bin's global position
    sprobe(sh, 15);
    for (uint32_t x = threadIdx.x; x < total; x += kT) {  // each entry at its bin's position + its rank
        if (flag[x] & kUsed) continue;
        const uint32_t bin = bin16[x];
        const uint64_t k = key[x];
        put_list(lo, bin, hist[bin] + rank16[x], make_uint4((uint32_t)k, (uint32_t)(k >> 32), val[x], word[x]));
    }
    __syncthreads();
}

EMP_COLD void write_next(BktJob &J, const Stage &v, uint32_t total, bool in_smem, const StepArgs &a, uint32_t nb,
                         const ListOut lo, BktRound &nx, BShared &sh, uint8_t *smem, const BScratch &gs, uint64_t G) {
    uint8_t *reg = smem + kOffReg;
    uint32_t *hist = reinterpret_cast<uint32_t *>(reg + kPHist);
    uint16_t *inv = reinterpret_cast<uint16_t *>(reg + kPInv);
    uint16_t *rank16 = reinterpret_cast<uint16_t *>(reg + kPRank);
    uint16_t *bin16 = reinterpret_cast<uint16_t *>(reg + kPBin);
    uint32_t *rank32 = gs.rank + G;
    const uint32_t nbin = 2 * nb;
    for (uint32_t i = threadIdx.x; i < nbin; i += kT) hist[i] = 0;
    if (threadIdx.x == 0) sh.sfx = 0;
    __syncthreads();
    uint32_t sfx = 0;
    constexpr int kU = 4;  // entries per thread in flight
    for (uint32_t x0 = 0; x0 < total; x0 += kU * kT) {
        bool act[kU];
        uint32_t val[kU], word[kU];
        uint64_t key[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const uint32_t x = x0 + u * kT + threadIdx.x;
            act[u] = x < total && !(ldv(v.flag + x) & kUsed);
            if (act[u]) {
                val[u] = ldv(v.val + x);
                word[u] = ldv(v.word + x);
                key[u] = ldv(v.key + x);
            }
        }
#pragma unroll
        for (int u = 0; u < kU; ++u)
            if (act[u] && needs_refill(a, val[u])) word[u] = refill_word(a, val[u]);
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            if (!act[u]) continue;
            const uint32_t x = x0 + u * kT + threadIdx.x;
            key[u] = step_key(a, key[u], val[u], word[u]);
            v.key[x] = key[u];
            v.word[x] = word[u];
            const uint32_t bn = 2 * bkt_of(sort_key(key[u], val[u]), nb) + (val[u] >> 31);
            const uint32_t rk = atomicAdd(&hist[bn], 1u);
            if (in_smem) {
                rank16[x] = (uint16_t)rk;
                bin16[x] = (uint16_t)bn;
            } else {
                rank32[x] = rk;
            }
            sfx += (val[u] >> 31) == 0;
        }
    }
    if (sfx) atomicAdd(&sh.sfx, sfx);
    __syncthreads();
    sprobe(sh, 13);
    const uint32_t kept = bin_starts(hist, nbin, sh);
    if (threadIdx.x == 0) {
        if (kept) atomicAdd(reinterpret_cast<unsigned long long *>(&nx.n), (unsigned long long)kept);
        if (sh.sfx) atomicAdd(reinterpret_cast<unsigned long long *>(&nx.s), (unsigned long long)sh.sfx);
    }
    sprobe(sh, 14);
    if (in_smem) {  // permute in shared memory, then write each bin as a run
        for (uint32_t x = threadIdx.x; x < total; x += kT)
            if (!(v.flag[x] & kUsed)) inv[hist[bin16[x]] + rank16[x]] = (uint16_t)x;
        __syncthreads();
        reserve_bins(hist, nbin, kept, lo.cnt, false);
        sprobe(sh, 15);
        for (uint32_t d = threadIdx.x; d < kept; d += kT) {
            const uint32_t x = inv[d], bin = bin16[x];
            const uint64_t key = v.key[x];
            put_list(lo, bin, d + hist[bin], make_uint4((uint32_t)key, (uint32_t)(key >> 32), v.val[x], v.word[x]));
        }
    } else {
        reserve_bins(hist, nbin, kept, lo.cnt, true);  // hist[bin] = the bin's global position
        for (uint32_t x = threadIdx.x; x < total; x += kT) {
            if (ldv(v.flag + x) & kUsed) continue;
            const uint64_t key = ldv(v.key + x);
            const uint32_t val = ldv(v.val + x);
            const uint32_t bn = 2 * bkt_of(sort_key(key, val), nb) + (val >> 31);
            put_list(lo, bn, hist[bn] + ldv(rank32 + x), make_uint4((uint32_t)key, (uint32_t)(key >> 32), val, ldv(v.word + x)));
        }
    }
    __syncthreads();
}

// ---------------------------------------------------------------- a round tile
EMP_DEV Cands cands_global(const BktJob &J, uint64_t G) {
    BScratch gs;
    scratch_layout(J.scratch, J.n_max, &gs);
    Cands w;
    w.ck = gs.ck + G;
    w.cv = gs.cv + G;
    w.cx = gs.cx + G;
    w.sk = gs.sk + G;
    w.tb = gs.tb + G;
    w.ord = gs.ord + G;
    w.cnt = gs.cnt + G;
    w.skey = gs.skey + G;
    w.sval = gs.sval + G;
    w.sidx = gs.sidx + G;
    return w;
}

// Compact the matched staged entries into w (any order: the ranking fixes
// it), writing at most cap of them; returns how many there are.
EMP_DEV uint32_t compact(const Stage &v, uint32_t total, const Cands &w, uint32_t cap, BShared &sh) {
    if (threadIdx.x == 0) sh.tile = 0;
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31;
    for (uint32_t x0 = 0; x0 < total; x0 += kT) {
        const uint32_t x = x0 + threadIdx.x;
        const bool f = x < total && (ldv(v.flag + x) & kMatched);
        const uint32_t m = __ballot_sync(0xffffffffu, f);
        if (!m) continue;
        const uint32_t leader = __ffs(m) - 1;
        uint32_t base = 0;
        if (lane == leader) base = atomicAdd(&sh.tile, (uint32_t)__popc(m));
        base = __shfl_sync(0xffffffffu, base, leader);
        const uint32_t d = base + __popc(m & lanemask_lt_u32());
        if (f && d < cap) {
            w.ck[d] = ldv(v.key + x);
            w.cv[d] = ldv(v.val + x);
            w.cx[d] = x;
        }
    }
    __syncthreads();
    return sh.tile;
}

// More than kBCand matched entries, or a bucket staged in scratch: the
// matched entries go to the bucket's scratch region and are ranked there.
EMP_COLD uint64_t big_count(const BktJob &J, const Stage &v, uint32_t total, bool in_smem, uint64_t &G, uint32_t b,
                            const uint32_t *cnt, BShared &sh, uint32_t &c) {
    if (in_smem) G = bins_below(cnt, 2 * b, sh);  // the bucket's position in bucket order picks its scratch region
    const Cands w = cands_global(J, G);
    c = compact(v, total, w, total, sh);
    return c ? sort_and_count(w, c, sh) : 0;
}

// Edges of the ranked matched entries at ebase (only when they fit), and
// the used marks: a suffix with an edge, a prefix that got one.
EMP_DEV void write_edges(BktJob &J, const Cands &w, uint32_t c, uint64_t ebase, bool room, const Stage &v) {
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
                if (room) {
                    J.sfrom[o] = si;
                    J.sto[o] = pj;
                }
                v.flag[ldv(w.sidx + j)] = kMatched | kUsed;
                ++o;
            }
        }
        if (o != o0) v.flag[ldv(w.sidx + i)] = kMatched | kUsed;
    }
    __syncthreads();
}

// Shape of round r0 + iter of a job, the same in every CTA: counts of earlier
// rounds are final once the grid barrier before the iteration has passed.
struct RoundShape {
    bool active;       // the round runs: r < rounds and a suffix left (overlap.cu:258)
    int r;
    uint32_t K;        // tiles of the round's list
    uint32_t nb;       // its key buckets
    uint32_t nb_next;  // key buckets of the next round's list
};
EMP_DEV RoundShape round_shape(const BktJob &J, uint32_t iter) {
    RoundShape z;
    z.r = J.r0 + (int)iter;
    z.K = z.nb = z.nb_next = 0;
    z.active = false;
    if (z.r >= J.rounds) return z;
    // the four counts in one round trip (meta has rounds + 1 entries)
    const uint64_t s = __ldcg(&J.meta[z.r].s), n = __ldcg(&J.meta[z.r].n);
    const uint64_t n1 = iter >= 1 ? __ldcg(&J.meta[z.r - 1].n) : J.n_in;
    const uint64_t n2 = iter >= 2 ? __ldcg(&J.meta[z.r - 2].n) : J.n_in;
    z.active = s > 0;
    if (!z.active) return z;
    z.nb = bkt_count(n1, J.wave, J.mean);
    z.K = iter == 0 ? (uint32_t)bkt_tiles(J.n_in) : bkt_count(n2, J.wave, J.mean);
    z.nb_next = bkt_count(n, J.wave, J.mean);
    return z;
}

// The next tile this CTA runs (job, bucket, iteration), whose two regions
// are pulled into L2 while this one is worked on; job = nullptr: none.
struct NextTile {
    const BktJob *job;
    uint32_t b, iter;
};

EMP_DEV void round_tile(BktJob &J, uint32_t b, uint32_t iter, const RoundShape &z, BShared &sh, const CoopCtl *ctl,
                        uint8_t *smem, const NextTile &nt) {
    probe(ctl, iter, 2);
    if (threadIdx.x == 0) {
        sh.pctl = ctl;
        sh.piter = iter;
    }
    uint32_t ncS = 0, ncP = 0;  // the next tile's region sizes, loaded now and used after the staging
    ListIn nli;
    if (threadIdx.x == 0 && nt.job) {
        nli = list_in(*nt.job, nt.iter);
        ncS = __ldcg(nli.cnt + 2 * nt.b);
        ncP = __ldcg(nli.cnt + 2 * nt.b + 1);
    }
    __syncthreads();
    BktRound &I = J.meta[z.r];
    const uint32_t nb = z.nb;
    const ListIn li = list_in(J, iter);
    Stage v;
    uint32_t S = 0;
    uint64_t G = 0;
    const uint32_t total = gather(J, li, b, sh, smem, v, S, G);
    const bool in_smem = total <= kBStage;
    if (threadIdx.x == 0 && nt.job) {
        const uint32_t s1 = min(ncS, nli.cap), p1 = min(ncP, nli.cap);
        if (s1) prefetch_l2(nli.lst + (uint64_t)(2 * nt.b) * nli.cap, s1 * 16u);
        if (p1) prefetch_l2(nli.lst + (uint64_t)(2 * nt.b + 1) * nli.cap, p1 * 16u);
    }
    probe(ctl, iter, 3);
    // ---- entries whose key is in both tables: flagged, compacted, ranked, joined
    uint32_t c = 0;
    uint64_t E = 0;
    bool small = false;
    if (S && S < total) {
        if (in_smem) {
            if (!match_filter(total, S, smem, sh)) match_smem(total, S, smem);
            probe(ctl, iter, 4);
            c = compact_s(smem + kOffFlag, total, cand_s(smem), sh);
            small = c <= kBCand;
        } else {
            BScratch gs;
            scratch_layout(J.scratch, J.n_max, &gs);
            match_global(v, total, S, gs, G);
        }
        probe(ctl, iter, 5);
        if (small) {
            if (c) {
                const uint64_t *skey = reinterpret_cast<const uint64_t *>(smem + kOffKey);
                const uint32_t *sval = reinterpret_cast<const uint32_t *>(smem + kOffVal);
                rank_s(cand_s(smem), c, b, nb, skey, sval, sh);
                E = join_count_s(cand_s(smem), c, skey, sval, sh);
            }
        } else {
            E = big_count(J, v, total, in_smem, G, b, li.cnt, sh, c);
        }
        if (threadIdx.x == 0 && c)
            atomicAdd(reinterpret_cast<unsigned long long *>(&I.cands), (unsigned long long)c);
    }
    probe(ctl, iter, 6);
    if (threadIdx.x == 0) {
        uint64_t off = 0;
        if (E) {
            off = atomicAdd(reinterpret_cast<unsigned long long *>(&J.e_stage), (unsigned long long)E);
            if (off + E > J.ecap) J.overflow = 1;
            atomicAdd(reinterpret_cast<unsigned long long *>(&I.edges), (unsigned long long)E);
        }
        sh.base = off;
        BktSpan &sp = J.spans[(uint64_t)(z.r - J.r0) * J.nb_max + b];
        sp.off = off;
        sp.cnt = E;
    }
    __syncthreads();
    if (E) {
        const bool room = sh.base + E <= J.ecap;
        if (small)
            write_edges_s(J, cand_s(smem), c, sh.base, room, reinterpret_cast<const uint64_t *>(smem + kOffKey),
                          reinterpret_cast<const uint32_t *>(smem + kOffVal), smem + kOffFlag);
        else
            write_edges(J, cands_global(J, G), c, sh.base, room, v);
    }
    probe(ctl, iter, 7);
    // ---- round r+1's tile b
    if (z.r + 1 < J.rounds) {
        BktRound &N = J.meta[z.r + 1];
        const uint32_t nb_next = z.nb_next;
        const StepArgs a = step_args(J, sh.tab, z.r + 1, false);
        const ListOut lo = list_out(J, iter + 1);
        if (nb_next > kBktMaxBuckets && in_smem) {
            write_next_direct_smem(total, a, nb_next, lo, N, sh, smem);
        } else if (nb_next > kBktMaxBuckets) {
            write_next_direct(v, total, a, nb_next, lo, N, sh);
        } else if (in_smem) {
            write_next_smem(total, a, nb_next, lo, N, sh, smem);
        } else {
            BScratch gs;
            scratch_layout(J.scratch, J.n_max, &gs);
            write_next(J, v, total, false, a, nb_next, lo, N, sh, smem, gs, G);
        }
    }
    probe(ctl, iter, 8);
}

// After the launch's last iteration (its run), for every job with no round left:
// each round's record, edges from the staging buffer in bucket order (rounds
// spread over the CTAs, no grid barrier).  Jobs that still have rounds are
// left as they are for the next launch.
constexpr uint32_t kPlaceChunk = kT;  // buckets per edge-placing work item (one per thread)
EMP_COLD void place_edges(BktJob *jobs, int J, uint32_t its, BShared &sh, uint8_t *smem) {
    uint64_t *dest = reinterpret_cast<uint64_t *>(smem);  // nb + 1 bucket starts
    uint64_t *roff = dest + kBktMaxBuckets + 1;          // per round of the job: record offset,
    uint64_t *rE = roff + kMaxJobRounds;                 // edge count,
    uint64_t *rnb = rE + kMaxJobRounds;                  // bucket count
    constexpr int kRPT = kMaxJobRounds / kT;             // rounds per thread
    uint32_t g = 0;
    for (int j = 0; j < J; ++j) {
        BktJob &x = jobs[j];
        const uint32_t ran = x.iter_share && x.iter_share < its ? x.iter_share : its;
        if (round_shape(x, x.iter0 + ran).active) continue;  // resumes in the next launch
        if (blockIdx.x == 0 && threadIdx.x == 0) x.done = 1;
        const uint32_t r0 = (uint32_t)x.r0;
        // the rounds that ran: round r ran iff r < rounds and it had a suffix
        // (build_graph's loop condition, overlap.cu:258); they form a prefix
        uint32_t nran = 0;
#pragma unroll
        for (int q = 0; q < kRPT; ++q) {
            const uint32_t r = r0 + kRPT * threadIdx.x + q;
            nran += (int)r < x.rounds && __ldcg(&x.meta[r].s) > 0;
        }
        uint32_t ran_all;
        block_exclusive_scan<kT, uint32_t>(nran, sh.scan32, &ran_all);
        const uint32_t r1 = r0 + ran_all;
        uint64_t P[kRPT], E[kRPT], e_my = 0, b_my = 0;
#pragma unroll
        for (int q = 0; q < kRPT; ++q) {
            const uint32_t r = r0 + kRPT * threadIdx.x + q;
            P[q] = E[q] = 0;
            if (r < r1) {
                const BktRound &m = x.meta[r];
                P[q] = __ldcg(&m.n) - __ldcg(&m.s);
                E[q] = P[q] ? __ldcg(&m.edges) : 0;
            }
            e_my += E[q];
            b_my += P[q] ? 12 + 8 * E[q] : 0;
        }
        uint64_t e_all, bytes;
        uint64_t e0 = block_exclusive_scan<kT, uint64_t>(e_my, sh.scan64, &e_all);
        uint64_t off = block_exclusive_scan<kT, uint64_t>(b_my, sh.scan64, &bytes);
#pragma unroll
        for (int q = 0; q < kRPT; ++q) {
            const uint32_t r = r0 + kRPT * threadIdx.x + q;
            if (r < r1) {
                const BktRound &m = x.meta[r];
                const uint64_t nb = r == r0 ? bkt_count(x.n_in, x.wave, x.mean)
                                            : bkt_count(__ldcg(&x.meta[r - 1].n), x.wave, x.mean);
                roff[r - r0] = off;
                rE[r - r0] = E[q];
                rnb[r - r0] = nb;
                if (blockIdx.x == 0) {
                    RoundRecord &rec = x.records[r];
                    rec.S = __ldcg(&m.s);
                    rec.P = P[q];
                    rec.E = E[q];
                    rec.e0 = e0;
                    rec.C = __ldcg(&m.cands);
                    rec.nb = nb;
                }
            }
            e0 += E[q];
            off += P[q] ? 12 + 8 * E[q] : 0;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            x.round = r1;
            x.e_total = e_all;
        }
        __syncthreads();
        if (vld(x.overflow)) continue;
        // one work item per (round, chunk of kPlaceChunk buckets), spread over
        // the CTAs: a large round's edges are placed by many CTAs at once
        for (uint32_t q = r0; q < r1; ++q) {
            const bool rec_q = __ldcg(&x.meta[q].n) != __ldcg(&x.meta[q].s);  // no prefix: no record
            const uint64_t Eq = rE[q - r0];
            const uint32_t nbq = (uint32_t)rnb[q - r0];
            const uint32_t items = rec_q ? (Eq ? (nbq + kPlaceChunk - 1) / kPlaceChunk : 1u) : 0u;
            uint8_t *o = x.out + roff[q - r0];
            uint32_t *from = reinterpret_cast<uint32_t *>(o + 12), *to = from + Eq;
            const BktSpan *sp = x.spans + (uint64_t)(q - r0) * x.nb_max;
            for (uint32_t k = 0; k < items; ++k, ++g) {
                if (g % gridDim.x != blockIdx.x) continue;
                if (k == 0 && threadIdx.x == 0) {  // u64 n, i32 ovlp_len (write_edges_binary, overlap.cu:148-161)
                    uint32_t *h = reinterpret_cast<uint32_t *>(o);
                    h[0] = (uint32_t)Eq;
                    h[1] = (uint32_t)(Eq >> 32);
                    h[2] = (uint32_t)(x.L - 1 - (int)q);
                }
                if (!Eq) continue;
                const uint32_t c0 = k * kPlaceChunk;
                const uint32_t cn = nbq - c0 < kPlaceChunk ? nbq - c0 : kPlaceChunk;
                uint64_t pre = 0;  // edges of the buckets before the chunk
                for (uint32_t b = threadIdx.x; b < c0; b += kT) pre += __ldcg(&sp[b].cnt);
                uint64_t base;
                block_exclusive_scan<kT, uint64_t>(pre, sh.scan64, &base);
                const uint32_t b = threadIdx.x;
                const uint64_t c = b < cn ? __ldcg(&sp[c0 + b].cnt) : 0;
                uint64_t tot;
                const uint64_t ex = block_exclusive_scan<kT, uint64_t>(c, sh.scan64, &tot);
                if (b < cn) dest[b] = base + ex;
                if (threadIdx.x == 0) dest[cn] = base + tot;
                __syncthreads();
                for (uint64_t e = base + threadIdx.x; e < base + tot; e += kT) {
                    uint32_t lo = 0, hi = cn;  // last bucket of the chunk with dest <= e
                    while (hi - lo > 1) {
                        const uint32_t m = (lo + hi) >> 1;
                        if (dest[m] <= e) lo = m;
                        else hi = m;
                    }
                    const uint64_t src = __ldcg(&sp[c0 + lo].off) + (e - dest[lo]);
                    from[e] = __ldcg(x.sfrom + src);
                    to[e] = __ldcg(x.sto + src);
                }
                __syncthreads();
            }
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kT, 2) bucket_rounds_kernel(BktJob *jobs, CoopCtl *ctl, uint32_t *) {
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ BShared sh;
    const int J = (int)ctl->njobs;
    for (uint32_t i = threadIdx.x; i < sizeof(HashTables) / 4; i += kT)
        reinterpret_cast<uint32_t *>(&sh.tab)[i] = reinterpret_cast<const uint32_t *>(jobs[0].tables)[i];
    if (threadIdx.x == 0) {
        sh.gen = 0;
        sh.pctl = ctl;
        sh.piter = 0;
    }
    __syncthreads();
    probe(ctl, 0, 20);  // the launch's phases, stamped with iteration 0's points
    // ---- prologue: the input lists of the jobs this launch starts -> their round r0 lists
    uint32_t total = build_prefix(sh, J, [&](int j) -> uint32_t {
        return jobs[j].iter0 == 0 && !jobs[j].pre_done ? (uint32_t)bkt_tiles(jobs[j].n_in) : 0u;
    });
    tile_loop(sh, &ctl->ticket[0], J, total, [&](int j, uint32_t k) { prologue_tile(jobs[j], k, sh, smem); });
    if (!grid_barrier(ctl, &sh.flag, &sh.gen, 0, 7)) return;
    // ---- rounds: iteration iter0 + it of every job (round r0 + iter0 + it)
    // that still runs, for at most iter_cap iterations; a job resumes in a
    // later launch from the lists and counts the last iteration left behind
    const uint32_t cap = ctl->iter_cap ? ctl->iter_cap : 0xffffffffu;
    uint32_t it = 0;
    for (; it < cap; ++it) {
        uint32_t *ticket = &ctl->ticket[1 + (it & 1)];
        if (blockIdx.x == 0 && threadIdx.x == 0) ctl->ticket[1 + ((it + 1) & 1)] = 0;  // last iteration's
        probe(ctl, it, 0);
        total = build_prefix(sh, J, [&](int j) -> uint32_t {
            const uint32_t share = jobs[j].iter_share;
            if (share && it >= share) return 0u;  // its share of this launch is used up
            const RoundShape z = round_shape(jobs[j], jobs[j].iter0 + it);
            sh.shp_nb[j] = z.nb;
            sh.shp_nbn[j] = z.nb_next;
            return z.active ? z.nb : 0u;
        });
        if (total == 0) break;  // no job has a round left
        probe(ctl, it, 1);
        tile_loop_ahead(sh, ticket, J, total, [&](int j, uint32_t b, uint32_t next) {
            const uint32_t g = jobs[j].iter0 + it;
            RoundShape z;
            z.active = true;
            z.r = jobs[j].r0 + (int)g;
            z.nb = sh.shp_nb[j];
            z.nb_next = sh.shp_nbn[j];
            NextTile nt{nullptr, 0u, 0u};
            if (next != ~0u) {
                int lo = 0, hi = J;
                while (hi - lo > 1) {
                    const int m = (lo + hi) >> 1;
                    if (sh.pref[m] <= next) lo = m;
                    else hi = m;
                }
                nt = NextTile{&jobs[lo], next - sh.pref[lo], jobs[lo].iter0 + it};
            }
            round_tile(jobs[j], b, g, z, sh, ctl, smem, nt);
        });
        probe(ctl, it, 9);
        if (!grid_barrier(ctl, &sh.flag, &sh.gen, it, 0)) return;
        probe(ctl, it, 10);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) ctl->iters = it;
    probe(ctl, 0, 21);
    place_edges(jobs, J, it, sh, smem);
    probe(ctl, 0, 22);
}

// The prologue of a job whose first list is binned directly, as its own
// launch: no shared memory and a few entries per thread, so that many more
// warps per SM than the round kernel's hide the latency of the list loads,
// the base-word loads and the bin counters.  Same entries, same bins.
constexpr int kPreT = 256, kPreU = 4;
__global__ void __launch_bounds__(kPreT) bucket_prologue_kernel(const BktJob *job) {
    const BktJob &J = *job;
    const uint64_t n_in = J.n_in;
    const uint32_t nb = bkt_count(n_in, J.wave, J.mean);
    const StepArgs a = step_args(J, *J.tables, J.r0, true);
    const ListOut lo = list_out(J, 0);
    const uint64_t *lk = J.lk_in;
    const uint32_t *lv = J.lv_in;
    const uint8_t *used_s = J.used_s, *used_p = J.used_p;
    const bool some_used = J.r0 > 0;  // host-synchronised rounds ran before the launch
    uint32_t kept = 0, sfx = 0;
    const uint64_t stride = (uint64_t)gridDim.x * kPreT * kPreU;
    for (uint64_t e0 = (uint64_t)blockIdx.x * kPreT * kPreU; e0 < n_in; e0 += stride) {  // uniform per block
        uint64_t key[kPreU];
        uint32_t val[kPreU], word[kPreU];
        bool keep[kPreU];
#pragma unroll
        for (int u = 0; u < kPreU; ++u) {
            const uint64_t e = e0 + u * kPreT + threadIdx.x;
            keep[u] = e < n_in;
            key[u] = keep[u] ? __ldcs(lk + e) : 0;
            val[u] = keep[u] ? __ldcs(lv + e) : 0;
        }
#pragma unroll
        for (int u = 0; u < kPreU; ++u) {
            word[u] = 0;
            if (!keep[u]) continue;
            const uint32_t rid = val[u] & 0x7fffffffu;
            if (some_used) keep[u] = ((val[u] >> 31) ? used_p[rid] : used_s[rid]) == 0;
            if (keep[u]) word[u] = refill_word(a, val[u]);
        }
#pragma unroll
        for (int u = 0; u < kPreU; ++u) {
            uint32_t bn = 0;
            if (keep[u]) {
                key[u] = step_key(a, key[u], val[u], word[u]);
                bn = 2 * bkt_of(sort_key(key[u], val[u]), nb) + (val[u] >> 31);
                ++kept;
                sfx += (val[u] >> 31) == 0;
            }
            put_direct(lo, keep[u], bn, make_uint4((uint32_t)key[u], (uint32_t)(key[u] >> 32), val[u], word[u]));
        }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        kept += __shfl_xor_sync(0xffffffffu, kept, o);
        sfx += __shfl_xor_sync(0xffffffffu, sfx, o);
    }
    if ((threadIdx.x & 31) == 0) {
        BktRound &I = job->meta[J.r0];
        if (kept) atomicAdd(reinterpret_cast<unsigned long long *>(&I.n), (unsigned long long)kept);
        if (sfx) atomicAdd(reinterpret_cast<unsigned long long *>(&I.s), (unsigned long long)sfx);
    }
}

}  // namespace

bool bucket_prologue_apart(const BktJob &hj) {
    return hj.iter0 == 0 && hj.n_in > 0 && bkt_count(hj.n_in, hj.wave, hj.mean) > kBktMaxBuckets;
}

cudaError_t launch_bucket_prologue(BktJob *job, cudaStream_t s) {
    constexpr int kDevs = 64;
    static std::atomic<int> grid[kDevs] = {};  // SMs x resident CTAs, per device
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kDevs) {
        cudaGetLastError();
        dev = 0;
    }
    int g = grid[dev].load(std::memory_order_acquire);
    if (!g) {
        int sms = 148, occ = 1;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, bucket_prologue_kernel, kPreT, 0) != cudaSuccess ||
            occ < 1)
            occ = 1;
        cudaGetLastError();
        g = sms * occ;
        grid[dev].store(g, std::memory_order_release);
    }
    count_launch();
    bucket_prologue_kernel<<<g, kPreT, 0, s>>>(job);
    return cudaGetLastError();
}

size_t bkt_scratch_bytes(uint64_t n_max) { return scratch_layout(nullptr, n_max < 1 ? 1 : n_max, nullptr); }



// Found once per device (the first call on it sets the kernel's shared
// memory attribute) and kept: the engine asks for every job.
static int bucket_grid_size_find(int dev) {
    int sms = 0, coop = 0, occ = 0;
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
    return occ >= 2 ? 2 * sms : (occ >= 1 ? sms : 0);  // two CTAs per SM
}

int bucket_grid_size() {
    constexpr int kDevs = 64;
    static std::atomic<int> grid[kDevs] = {};  // grid + 1; 0: not found yet
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kDevs) {
        cudaGetLastError();
        return bucket_grid_size_find(dev);
    }
    int g = grid[dev].load(std::memory_order_relaxed);
    if (g == 0) {
        g = bucket_grid_size_find(dev) + 1;
        grid[dev].store(g, std::memory_order_relaxed);
    }
    return g - 1;
}

cudaError_t launch_bucket_rounds(BktJob *jobs, CoopCtl *ctl, uint32_t *err, cudaStream_t s) {
    const int grid = bucket_grid_size();
    if (grid <= 0) return cudaErrorNotSupported;
    void *args[] = {&jobs, &ctl, &err};
    count_launch();
    return cudaLaunchCooperativeKernel((const void *)bucket_rounds_kernel, dim3(grid), dim3(kT), args, kBktSmem, s);
}

}  // namespace emp
