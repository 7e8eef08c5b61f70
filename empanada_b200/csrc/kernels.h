// kernels.h -- host-side launchers of the overlap-path kernels (internal).
#pragma once

#include <atomic>
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "common.cuh"

namespace emp {

// Kernels launched by this library since load (every launcher adds its count).
extern std::atomic<uint64_t> g_launches;
inline void count_launch(uint64_t k = 1) { g_launches.fetch_add(k, std::memory_order_relaxed); }

// ---- generic single-pass exclusive scan (k_scan.cu) ----------------------
constexpr uint32_t kScanTile = 4096;  // u32 inputs per tile
__host__ __device__ inline uint64_t scan_tiles(uint64_t n) { return (n + kScanTile - 1) / kScanTile; }
// out[i] = sum(in[0..i)); *total = sum(in).  status: scan_tiles(n) u64,
// tile_ctr: one u32; both must be zero.  out may alias in.
void launch_scan_u32_u64(const uint32_t *in, uint64_t *out, uint64_t n, uint64_t *status, uint32_t *tile_ctr,
                         uint64_t *total, uint32_t *err, cudaStream_t s);
void launch_scan_u32_u32(const uint32_t *in, uint32_t *out, uint64_t n, uint64_t *status, uint32_t *tile_ctr,
                         uint64_t *total, uint32_t *err, cudaStream_t s);

// ---- map phase (k_map.cu) -------------------------------------------------
constexpr uint64_t kParseTile = 16384;  // FASTQ bytes per tile
__host__ __device__ inline uint64_t parse_tiles(uint64_t F) { return (F + kParseTile - 1) / kParseTile; }
// tile_counts[t] = newlines in FASTQ tile t; *len0 = length of the first
// record's sequence line when tile 0 holds its two newlines, else 0
void launch_nl_count(const uint8_t *fq, uint64_t F, uint32_t *tile_counts, uint64_t *len0, cudaStream_t s);
// Records k of the FASTQ (tile_excl: newlines before each parse tile):
// keep[k] = 1 iff the record's sequence line holds no N-class byte and is not
// empty; keys[2k] / keys[2k+1] = fingerprint of its read / of the reverse
// complement, seq2[k * wpr + w] = its bases 16w .. 16w+15 (2 bits each, zero
// past the read); *n_kept += the kept count (start it at 0), the kept reads'
// length extremes in len_minmax, kErrBadBase in *err.  Reads longer than
// kMaxReadLen are classified but not hashed.
void launch_read_pass(const uint8_t *fq, uint64_t F, const uint64_t *tile_excl, const HashTables *tables,
                      const ChunkWeights *weights, uint64_t *keys, uint32_t *seq2, int wpr, uint32_t *keep,
                      uint64_t *n_kept, uint32_t *len_minmax, uint32_t *err, cudaStream_t s);
// The kept records' keys and words to indices 0 .. n_kept-1 in file order;
// pos = exclusive scan of keep.
void launch_compact_reads(const uint32_t *pos, uint64_t n_rec, uint64_t n_kept, const uint64_t *keys,
                          const uint32_t *seq2, int wpr, uint64_t *keys_out, uint32_t *seq2_out, cudaStream_t s);
// cols[c * wpc + i/16] holds base c of read i at bits 2*(i%16)
void launch_columns(const uint32_t *seq2, uint64_t n, int L, int wpr, uint32_t *cols, uint64_t wpc, cudaStream_t s);

// ---- duplicate removal without a sort (k_dedup.cu) -------------------------
// alive[e] = 1 iff read-end e has the smallest rid of its fingerprint (the
// survivor of the reference's in-core sort + unique).  nb key buckets from
// dedup_buckets(n) (0: use the sort); scratch: dedup_scratch_bytes(nb);
// pk/pr: n pairs of room; status: scan_tiles(nb) zeroed look-back words,
// *tile_ctr zeroed.  kErrDedupFull in *err: a bucket overflowed, use the sort.
// Returns false when the kernels cannot run on this device.
constexpr uint32_t kDedupMean = 4096;
constexpr uint32_t kDedupMaxBuckets = 16384;
constexpr uint64_t kDedupMaxEnds = (uint64_t)kDedupMaxBuckets * 6000;
uint32_t dedup_buckets(uint64_t n);
size_t dedup_scratch_bytes(uint32_t nb);
bool launch_dedup_hash(const uint64_t *keys, uint64_t n, uint32_t nb, void *scratch, uint64_t *pk, uint32_t *pr,
                       uint8_t *alive, uint64_t *status, uint32_t *tile_ctr, uint64_t *total, uint32_t *err,
                       cudaStream_t s);

// ---- unitigs of the overlap graph (k_graph.cu) ----------------------------
// Device arrays of graph_build: per edge from/to (E), per node (nodes = 2n)
// the degrees, succ/pred, two hop/dist and mn/nx buffers, unitig sizes (at
// the heads), their starts (u64) and the nodes in unitig order; scan status
// words (scan_tiles(nodes), zeroed), a tile counter and a total (zeroed),
// the error word and a cycle counter (zeroed).
struct GraphBufs {
    uint32_t *from, *to;
    uint32_t *dout, *din, *succ, *pred, *hop[2], *dist[2], *mn[2], *nx[2], *size, *order;
    uint64_t *start;
    uint64_t *status;
    uint32_t *tile_ctr;
    uint64_t *total;
    uint32_t *err, *cycles;
};
// out: output.bin on the device; rec_off[k] its record k's byte offset,
// rec_e0[k] the record's first edge (rec_e0[nrec] = E).
void graph_build(const uint8_t *out, const uint64_t *rec_off, const uint64_t *rec_e0, uint32_t nrec, uint64_t E,
                 uint32_t nodes, const GraphBufs &b, cudaStream_t s);

// ---- radix sort (k_sort.cu) ---------------------------------------------
constexpr int kSortBits = 8;
constexpr int kSortRadix = 1 << kSortBits;
constexpr int kSortPasses = 8;           // 59-bit sort keys
constexpr uint32_t kSortTile = 4096;
__host__ __device__ inline uint64_t sort_tiles(uint64_t n) { return (n + kSortTile - 1) / kSortTile; }
constexpr uint32_t kSmallSort = 4096;    // up to this many pairs: one CTA sorts in shared memory
struct SortScratch {
    uint32_t hist[kSortPasses][kSortRadix];  // digit counts of the pairs being sorted
    uint32_t tile_ctr[kSortPasses];          // per-pass tile tickets
    uint32_t epoch;                          // look-back epoch of the current sort
    uint32_t pad[7];
    // followed by sort_tiles(n_max) * kSortRadix epoch-tagged look-back words
};
// Start a new sort on this scratch: advance the epoch, reset the tickets and
// (zero_hist) the histogram.  One CTA.
void launch_sort_prepare(SortScratch *sc, bool zero_hist, cudaStream_t s);
// Bytes of scratch a sort of up to n pairs needs (histograms, tile tickets,
// epoch, look-back words).  Zero it once after allocation; it resets itself
// between sorts (re-zero after 100000 sorts, before the epoch can wrap).
size_t sort_scratch_bytes(uint64_t n);
// Stable sort of (keys, vals) by sort_key(key, val), count *n_dev (device)
// with n_max >= *n_dev sizing the grid.  Ping-pongs between (k0,v0) and
// (k1,v1); kSortPasses is even, so the result ends in (k0,v0) (returns 0).
// pass_events (optional, 2*kSortPasses events) bracket each digit pass.
int sort_pairs_dev(uint64_t *k0, uint32_t *v0, uint64_t *k1, uint32_t *v1, const uint64_t *n_dev, uint64_t n_max,
                   void *scratch, uint32_t *err, cudaStream_t s, cudaEvent_t *pass_events = nullptr);
// The same without the prepare step: the caller has already prepared the
// scratch (pipeline rounds prepare the next sort in their round_end kernel).
void sort_pairs_prepared(uint64_t *k0, uint32_t *v0, uint64_t *k1, uint32_t *v1, const uint64_t *n_dev,
                         uint64_t n_max, SortScratch *sc, uint32_t *err, cudaStream_t s);
// Same with a host count (copied into the device word n_dev first).
int sort_pairs(uint64_t *k0, uint32_t *v0, uint64_t *k1, uint32_t *v1, uint64_t n, void *scratch, uint64_t *n_dev,
               uint32_t *err, cudaStream_t s, cudaEvent_t *pass_events = nullptr);

// ---- sort of a table larger than M (k_chunked.cu) --------------------------
struct ChunkPart {  // one merge partition: A entries [a0, a0+pa), B entries [b0, b0+pb)
    uint64_t a0, pa, b0, pb;
};
// Chunk of each entry of (v)[0..n) as a sort key ((rank / M) << 32) with its
// index: rank = read-end id when lst is null (the table holds ids 0..n-1 in
// order), else the entry's rank among the ids of lst (the table in list
// order: even ids ascending, then odd ids ascending).
void launch_chunk_keys(const uint32_t *v, uint64_t n, const uint32_t *lst, uint64_t M, uint64_t *ck, uint32_t *ci,
                       cudaStream_t s);
// (rk, rv)[i] = (k, v)[idx[i]], i < n
void launch_ring_gather(const uint64_t *k, const uint32_t *v, const uint32_t *idx, uint64_t n, uint64_t *rk,
                        uint32_t *rv, cudaStream_t s);
// (k, v)[i] = ring entry start + i (ring of C entries), i < n
void launch_ring_copy(const uint64_t *rk, const uint32_t *rv, uint64_t C, uint64_t start, uint64_t n, uint64_t *k,
                      uint32_t *v, cudaStream_t s);
// Merge ring tables A (start sa, nA entries) and B into the one at so, along
// the reference's merge partitions of windows h; parts: room for cap.
void launch_merge(uint64_t *rk, uint32_t *rv, uint64_t C, uint64_t sa, uint64_t nA, uint64_t sb, uint64_t nB,
                  uint64_t so, uint64_t h, ChunkPart *parts, uint64_t cap, uint64_t *count, uint32_t *err,
                  cudaStream_t s);
// kErrHang when the reference's duplicate-removal partition walk over the
// sorted keys k[0..n) stops advancing.
void launch_unique_walk(const uint64_t *k, uint64_t n, uint64_t M, uint32_t *err, cudaStream_t s);

// ---- rounds (k_round.cu) --------------------------------------------------
void launch_dedup_mark(const uint64_t *skeys, const uint32_t *svals, uint64_t n2, uint8_t *alive, cudaStream_t s);
// rid order (evens ascending, then odds ascending) of the alive read-ends
void launch_init_list(const uint64_t *keys0, const uint8_t *alive, uint64_t n, uint64_t *lkeys, uint32_t *lvals,
                      uint64_t *status, uint32_t *tile_ctr, uint64_t *count, uint32_t *err, cudaStream_t s);
void launch_dup_prefix_half(uint64_t *lkeys, uint32_t *lvals, uint64_t u, cudaStream_t s);
void launch_iota(uint32_t *v, uint64_t n, cudaStream_t s);
constexpr uint32_t kUpdTile = 2048;
__host__ __device__ inline uint64_t upd_tiles(uint64_t n) { return (n + kUpdTile - 1) / kUpdTile; }
struct RoundArgs {
    const uint64_t *kin;
    const uint32_t *vin;
    uint64_t n_in;
    uint64_t *kout;
    uint32_t *vout;
    const uint8_t *used_s;
    const uint8_t *used_p;
    const uint32_t *cols;
    uint64_t wpc;
    const HashTables *tables;
    int L;
    int round;
    uint64_t *status;
    uint32_t *tile_ctr;
    uint64_t *n_out;   // total survivors
    uint64_t *s_out;   // survivors of the suffix table (must be zero)
    uint32_t *err;
};
void launch_update_compact(const RoundArgs &a, cudaStream_t s);
// Record splitting (cq_get_search_partitions, cqutils.cuh:108-137).
// split_tables: sorted merged list -> sorted suffix keys (+ their merged
// positions) and sorted prefix keys.
void launch_split_tables(const uint64_t *skeys, const uint32_t *svals, uint64_t n, uint64_t *akeys, uint32_t *apos,
                         uint64_t *bkeys, uint64_t *status, uint32_t *tile_ctr, uint32_t *err, cudaStream_t s);
struct SearchPart {
    uint64_t pa, pb;  // suffixes / prefixes in the partition
    uint64_t e0, e1;  // its edges in the round's edge list
};
// One thread walks the reference's partition loop with windows of h = M/2.
void launch_search_partitions(const uint64_t *akeys, uint64_t S, const uint64_t *bkeys, uint64_t P, uint64_t h,
                              const uint32_t *apos, const uint64_t *offs, uint64_t E, SearchPart *parts,
                              uint64_t cap, uint64_t *count, uint32_t *err, cudaStream_t s);
// ---- per-round counts of the all-rounds kernel --------------------------
struct RoundRecord {
    uint64_t S, P, E, e0;  // table sizes, edges, first edge of the round
    uint64_t C;            // entries found in both tables (ranked and joined)
    uint64_t nb;           // key buckets of the round (bucket kernel only)
};
// ---- cooperative multi-job launches (k_bucket.cu) --------------------------
constexpr int kCoopMaxJobs = 1024;
constexpr uint64_t kBarrierTimeoutNs = 20ull * 1000 * 1000 * 1000;  // default limit of a grid-barrier wait
struct CoopCtl {
    uint32_t njobs;
    uint32_t active;    // jobs not finished (the host sets njobs)
    uint32_t all_done;
    uint32_t any_lsd;
    uint32_t bar_count;  // grid-barrier arrivals since the launch
    uint32_t bar_gen;    // unused
    uint32_t err;
    uint32_t pad;
    uint32_t ticket[16];
    uint64_t *trace;  // optional: kCoopTracePhases globaltimer stamps per iteration
    uint32_t trace_cap;  // iterations the trace holds
    uint32_t probe_iter;  // iteration whose per-CTA stamps go to `probe`
    uint64_t *probe;      // optional: kCoopProbePoints stamps per CTA (profiling)
    uint32_t iter_cap;    // bucket kernel: iterations this launch runs at most (0: until every job is done)
    uint32_t iters;       // bucket kernel: iterations it ran
    uint64_t wait_ns;     // limit of each grid-barrier wait (0: kBarrierTimeoutNs)
    uint32_t bar_extra;   // testing: added to every barrier's target, so that no arrival completes one
    uint32_t pad2;
};
constexpr int kCoopTracePhases = 8;
constexpr int kCoopProbePoints = 32;
// ---- bucket rounds (k_bucket.cu) ------------------------------------------
// A round's list of 16-byte entries is kept as one region per (key bucket,
// table) bin.  A prologue bins the launch's input list; then each round gives
// each key bucket to one CTA, which stages the bucket's two regions, finds
// the keys present in both tables, ranks and joins those entries, drops the
// used ones, applies the next round's hash step to the rest and writes them
// into the next round's bins (positions reserved from per-bin counters).  One
// grid barrier per round; the edges are put in bucket order once all rounds
// are done.
struct BktEntry {
    uint64_t key;   // fp1 << 32 | fp2
    uint32_t val;   // rid | table << 31
    uint32_t word;  // cached 16 bases (one seq2 word) of the entry's read
};
constexpr int kBktThreads = 256;                  // threads of a bucket-kernel CTA (two CTAs per SM)
constexpr uint32_t kBktTile = 2048;               // entries per prologue tile (8 per thread)
constexpr uint32_t kBktMean = 2900;               // entries per bucket aimed at (mean; 5.5 sigma below the staging limit)
constexpr uint32_t kBktMeanMin = 512;             // tuning range of the mean
constexpr uint32_t kBktMeanMax = 3000;
constexpr uint32_t kBktMaxBuckets = 2048;         // up to this many buckets a CTA bins its entries in shared memory
constexpr uint32_t kBktHugeBuckets = 1u << 20;    // above kBktMaxBuckets: one global atomic per run of equal bins
constexpr uint64_t kBktMaxEntries = 320ull << 20; // larger lists run host-synchronised rounds until they fit
__host__ __device__ inline uint64_t bkt_tiles(uint64_t n) { return (n + kBktTile - 1) / kBktTile; }
// Buckets of a round with n entries on a grid of G CTAs: whole waves of G,
// at most `mean` entries each on average.  Bucket of a sort key sk: its top
// 24 bits scaled to [0, nb), so bucket order is key order.
__host__ __device__ inline uint32_t bkt_count(uint64_t n, uint32_t G, uint32_t mean) {
    uint64_t waves = (n + (uint64_t)G * mean - 1) / ((uint64_t)G * mean);
    if (waves < 1) waves = 1;
    uint64_t nb = waves * G;
    return (uint32_t)(nb > kBktHugeBuckets ? kBktHugeBuckets : nb);
}
__host__ __device__ inline uint32_t bkt_of(uint64_t sk, uint32_t nb) {
    return (uint32_t)(((sk >> 35) * (uint64_t)nb) >> 24);
}
struct BktRound {        // counts of one round (atomic while the round, or its list, is written)
    uint64_t n;          // entries of the round's list
    uint64_t s;          // of which suffixes
    uint64_t cands;      // entries found in both tables
    uint64_t edges;      // edges of the round
};
struct BktSpan {         // one bucket's edges in the staging buffer
    uint64_t off, cnt;
};
struct BktJob {
    const uint64_t *lk_in;   // the list at launch (id order, suffixes then prefixes)
    const uint32_t *lv_in;
    const uint8_t *used_s, *used_p;  // marks of rounds run before the launch
    uint64_t n_in;           // entries of that list
    // The current and the next round's list: one region of `cap` entries per
    // (bucket, table) bin, bin = 2 bucket + table, filled through the round's
    // bin counters; entries past a region's capacity go to the list's spill
    // area with their bin as tag.
    BktEntry *lst[2];        // nb_max * 2 * cap entries each
    uint32_t *cnt;           // [iteration][2 nb_max]: entries reserved in each bin (zeroed at the start)
    BktEntry *spill[2];      // n_max entries each
    uint32_t *spill_tag[2];  // their bins
    uint32_t *spill_n;       // [iteration]: spilled entries (zeroed at the start)
    uint32_t cap;            // region capacity (entries)
    const uint32_t *seq2;    // read-major 2-bit bases, wpr words per read
    int32_t wpr, L, rounds, r0;
    const HashTables *tables;
    BktSpan *spans;          // [round - r0][bucket]: edges in the staging buffer
    uint32_t *sfrom, *sto;   // staging buffer (bucket order within a round is restored at the end)
    uint8_t *out;            // output.bin records of the launch's rounds (12 * rounds + 8 * ecap bytes)
    uint64_t ecap;
    RoundRecord *records;
    uint8_t *scratch;        // bkt_scratch_bytes(n_max): buckets too big for shared memory
    uint64_t n_max;
    uint32_t nb_max;         // row length of spans
    uint32_t round;          // rounds run (set at the end of the launch)
    uint32_t wave;           // bucket counts are multiples of this (the grid for a job alone)
    uint32_t mean;           // entries per bucket aimed at (bkt_count)
    uint32_t overflow;       // the edge buffer was too small
    uint32_t iter0;          // iterations run by earlier launches (0: the launch starts the job)
    uint32_t pre_done;       // the prologue ran in its own launch (launch_bucket_prologue)
    uint32_t iter_share;     // iterations this launch runs for the job at most (0: no limit)
    uint32_t done;           // set at the end of a launch after which the job has no round left
    uint64_t e_total;        // edges of the finished rounds of this launch
    uint64_t e_stage;        // staging buffer fill
    BktRound *meta;          // [rounds + 1], zeroed; round r at meta[r]
};
size_t bkt_scratch_bytes(uint64_t n_max);
constexpr uint32_t kBktRegionCap = 2048;  // entries per (bucket, table) region: 15 sigma above the mean of 1450
int bucket_grid_size();                             // 0: no cooperative launch on this device
cudaError_t launch_bucket_rounds(BktJob *jobs, CoopCtl *ctl, uint32_t *err, cudaStream_t s);
// Whether a job the round kernel starts (iter0 = 0) bins its first list
// directly (more than kBktMaxBuckets buckets); such a job's prologue runs
// faster as its own launch before the round kernel, with pre_done set.
bool bucket_prologue_apart(const BktJob &host_job);
// The current device's L2 read bandwidth (GB/s) on a buffer of `bytes`
// (smaller than L2), read 20 times with 16-byte loads (k_probe.cu).
cudaError_t measure_l2_read(uint64_t bytes, double *gbs);
cudaError_t launch_bucket_prologue(BktJob *job, cudaStream_t s);

void launch_join_count(const uint64_t *skeys, const uint32_t *svals, uint64_t n, uint32_t *cnt, cudaStream_t s);
void launch_join_write(const uint64_t *skeys, const uint32_t *svals, uint64_t n, const uint32_t *cnt,
                       const uint64_t *offs, uint32_t *from, uint32_t *to, uint8_t *used_s, uint8_t *used_p,
                       cudaStream_t s);

}  // namespace emp
