// engine.cu -- job orchestration and the C ABI (include/empanada.h).
//
// One job runs the reference program's two phases on the device:
//   map     main.cu:42-58  -> nl_count + scan, read_pass (and compact_reads
//                             when a read is dropped) (k_map.cu)
//   reduce  overlap.cu:206-293 -> duplicate removal by key buckets
//                             (k_dedup.cu; the sort when 2n > M) +
//                             init_list, then every round in the bucket
//                             kernel (k_bucket.cu), or host-synchronised
//                             rounds while a round's tables reach M/2
//                             (k_round.cu, k_sort.cu, k_chunked.cu)
// All tables stay in HBM; the host traffic is the FASTQ in and output.bin
// out.  output.bin records (write_edges_binary, overlap.cu:148-161) are
// written on the device by the bucket kernel, on the host for
// host-synchronised rounds.  Files come in through ingest.cpp.
#include <algorithm>
#include <cerrno>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <vector>

#include <sys/stat.h>

#include "../../include/empanada.h"
#include "ingest.h"
#include "kernels.h"

namespace emp {
std::atomic<uint64_t> g_launches{0};
}

using namespace emp;

namespace {

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    cudaStream_t pool_stream = nullptr;  // set: from the context's pool, freed in this stream's order
    bool pooled = false;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) {
            if (pooled) cudaFreeAsync(p, pool_stream);
            else cudaFree(p);
        }
        p = nullptr;
        bytes = 0;
        pooled = false;
    }
    template <class T>
    T *as() const { return reinterpret_cast<T *>(p); }
};

// exchange two buffers (both from the same pool)
void swap_buf(DevBuf &a, DevBuf &b) {
    std::swap(a.p, b.p);
    std::swap(a.bytes, b.bytes);
    std::swap(a.pool_stream, b.pool_stream);
    std::swap(a.pooled, b.pooled);
}

struct PinnedBuf {
    void *p = nullptr;
    size_t bytes = 0;
    bool owned = true;  // false: a piece of the context's host slab
    PinnedBuf() = default;
    PinnedBuf(const PinnedBuf &) = delete;
    PinnedBuf &operator=(const PinnedBuf &) = delete;
    ~PinnedBuf() { drop(); }
    void drop() {
        if (p && owned) cudaFreeHost(p);
        p = nullptr;
        bytes = 0;
        owned = true;
    }
    void bind(void *q, size_t b) {
        drop();
        p = q;
        bytes = b;
        owned = false;
    }
    bool ensure(size_t b) {
        if (b <= bytes) return true;
        drop();
        size_t nb = b < 4096 ? 4096 : b + b / 2;
        if (cudaHostAlloc(&p, nb, cudaHostAllocDefault) != cudaSuccess) { p = nullptr; return false; }
        bytes = nb;
        return true;
    }
    template <class T>
    T *as() const { return reinterpret_cast<T *>(p); }
};

// Pinned host slots for the small per-job host words (counts, histograms,
// launch descriptors, round records), carved from 4 MiB chunks: page-locking
// a small buffer costs about a millisecond, so a job takes a slot instead.
constexpr size_t kSlotBytes = 64 << 10;
constexpr size_t kSlotChunk = 4 << 20;
constexpr size_t kSlotMisc = 0, kSlotHist = 4 << 10, kSlotCoop = 12 << 10, kSlotCtl = 24 << 10,
                 kSlotRecords = 28 << 10;
struct HostSlab {
    std::mutex mu;
    std::vector<void *> chunks, free_slots;
    ~HostSlab() {
        for (void *c : chunks) cudaFreeHost(c);
    }
    void *take() {
        std::lock_guard<std::mutex> g(mu);
        if (free_slots.empty()) {
            void *c = nullptr;
            if (cudaHostAlloc(&c, kSlotChunk, cudaHostAllocDefault) != cudaSuccess) return nullptr;
            chunks.push_back(c);
            for (size_t o = 0; o + kSlotBytes <= kSlotChunk; o += kSlotBytes)
                free_slots.push_back(static_cast<uint8_t *>(c) + o);
        }
        void *q = free_slots.back();
        free_slots.pop_back();
        return q;
    }
    void give(void *q) {
        std::lock_guard<std::mutex> g(mu);
        free_slots.push_back(q);
    }
};

}  // namespace

constexpr int kMapStreams = 32;     // streams of a batch's map phase at most
constexpr int kMapStreamsDefault = 8;

struct emp_ctx {
    int device = 0;
    uint64_t budget = 0;
    uint64_t in_use = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t copy_stream = nullptr;  // asynchronous FASTQ feeds
    // device memory of the jobs' work buffers: a stream-ordered pool that keeps
    // what is freed, so that a job's buffers come and go without cudaMalloc
    cudaMemPool_t pool = nullptr;
    DevBuf tables;  // HashTables, then ChunkWeights
    // emp_sort_pairs working set, kept for the next call
    DevBuf sort_k1, sort_v1, sort_scr, sort_err;
    uint64_t sort_cap = 0;
    uint64_t sort_calls = 0;
    HostSlab slab;
    // emp_batch_run: the BktJob array and control block of one launch, their
    // host copies, and the launch's events
    DevBuf batch_jobs, batch_ctl;
    PinnedBuf h_batch;
    cudaEvent_t batch_ev[2] = {};
    // the map phase of a batch of jobs: jobs on kMapStreams streams, so that
    // the small kernels of small read sets run side by side
    cudaStream_t map_streams[kMapStreams] = {};
    cudaEvent_t map_ev[kMapStreams + 1] = {};
    emp_tuning tune{};  // engine choices (zero fields: defaults)
    // profiling aids, read from the environment when the context is made:
    // EMP_COOP_TRACE=<file> (per-round durations of the bucket kernel),
    // EMP_COOP_PROBE=<file>[:iteration] (per-CTA stamps of one iteration)
    std::string trace_path, probe_spec;
};

struct JobPrep {
    uint64_t n = 0, n_rec = 0, U = 0, M = 0, wpc = 0, ecap = 0, launches0 = 0;
    int L = 0, wpr = 0, rounds = 0;
    bool done = false;  // nothing more to run (empty input, no reads)
};

struct emp_job {
    emp_ctx *ctx = nullptr;
    emp_params p{};
    // input
    DevBuf fq;
    uint64_t F = 0;
    bool fed_last = false;
    double ms_h2d = 0.0;
    // work buffers
    DevBuf tile_counts, tile_excl, status, misc, keys0, cols, seq2, dedup_scr, keep, keys_tmp, seq2_tmp;
    DevBuf sk0, sv0, sk1, sv1, alive, lk0, lv0, lk1, lv1, used_s, used_p, cnt, offs, efrom, eto, sort_scratch;
    DevBuf akeys, apos, bkeys, parts;  // record splitting
    DevBuf xk0, xv0, xk1, xv1, ring_k, ring_v, cparts;  // sort of a table larger than M
    PinnedBuf h_parts;
    DevBuf records;  // round records
    PinnedBuf h_records;
    uint64_t ecap_hint = 0;
    uint64_t sorts_since_clear = 0;
    DevBuf coop_ctl, coop_trace, coop_probe;  // bucket kernel: control block, profiling stamps
    DevBuf dout;                 // output.bin records written on the device (after those in `out`)
    uint64_t dout_bytes = 0;
    PinnedBuf h_out;
    DevBuf bk_lst0, bk_lst1, bk_cnt, bk_spill, bk_spans, bk_sfrom, bk_sto, bk_scratch, bk_job, bk_meta;  // bucket kernel
    PinnedBuf h_coop;
    cudaEvent_t sort_ev[2 * kSortPasses] = {};
    cudaEvent_t upd_ev[2 * EMP_MAX_ROUNDS] = {};
    uint64_t sort_n = 0;
    bool sort_timed = false;
    PinnedBuf h_misc, h_hist, h_from, h_to;
    uint64_t n_ends = 0;
    // map-phase state (map_begin .. map_list) and its events
    JobPrep prep;
    cudaEvent_t map_ev[5] = {};
    // asynchronous feeds: copies on the context's copy stream, bracketed by
    // these events; the next run waits for feed_ev[1]
    cudaEvent_t feed_ev[2] = {};
    bool feed_pending = false;
    // served: the job's bucket-kernel descriptor between launches, its
    // admission estimate, and whether a server holds it
    BktJob bk{};
    uint64_t admit_est = 0;
    emp_server *server = nullptr;
    emp_status last_rc = EMP_E_STATE;  // status of the last run (EMP_E_STATE: none yet)
    void *slot = nullptr;              // the job's slot of the context's host slab
    cudaStream_t stream = nullptr;     // stream of the current run
    // results
    std::vector<uint8_t> out;
    emp_stats st{};
    bool have_result = false;
};

namespace {

// misc device words (u64 slots)
enum MiscSlot { kMiscErr = 0, kMiscTotal = 1, kMiscLen = 2, kMiscN = 3, kMiscU = 4, kMiscNout = 5, kMiscSout = 6,
                kMiscE = 7, kMiscCtr = 8, kMiscParts = 9, kMiscSortN = 10, kMiscLen0 = 11, kMiscKept = 12,
                kMiscSlots = 16 };

// internal: the pipeline's edge buffer was too small (never returned by the ABI)
constexpr emp_status kNeedEdgeRoom = -1000;

emp_status cuda_status(cudaError_t e) { return e == cudaSuccess ? EMP_OK : (e == cudaErrorMemoryAllocation ? EMP_E_NOMEM : EMP_E_CUDA); }

// Grow b to at least `bytes` from the context's pool, in the order of stream
// s (the old contents are not kept).
emp_status ctx_ensure(emp_ctx *c, DevBuf &b, size_t bytes, cudaStream_t s) {
    if (bytes <= b.bytes) return EMP_OK;
    const size_t old = b.bytes;
    if (c->budget && c->in_use - old + bytes > c->budget) return EMP_E_NOMEM;
    if (b.p && b.pooled) {
        cudaFreeAsync(b.p, s);
        b.p = nullptr;
        b.bytes = 0;
        b.pooled = false;
    }
    b.release();
    c->in_use -= old;
    void *p = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&p, bytes ? bytes : 16, c->pool, s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return EMP_E_NOMEM;
    }
    b.p = p;
    b.bytes = bytes;
    b.pooled = true;
    b.pool_stream = c->stream;
    c->in_use += bytes;
    return EMP_OK;
}

// a job's buffers grow in the order of the stream its current run uses
emp_status ensure(emp_job *j, DevBuf &b, size_t bytes) {
    return ctx_ensure(j->ctx, b, bytes, j->stream ? j->stream : j->ctx->stream);
}

void free_buf(emp_job *j, DevBuf &b) {
    j->ctx->in_use -= b.bytes;
    b.release();
}

uint32_t host_modpow(uint64_t a, uint32_t e, uint32_t p) {
    uint64_t r = 1;
    while (e) {
        if (e & 1) r = (r * a) % p;
        a = (a * a) % p;
        e >>= 1;
    }
    return (uint32_t)r;
}

void host_tables(HashTables &t, ChunkWeights &cw) {
    t.pow1[0] = t.pow2[0] = 1;
    for (int i = 1; i <= kMaxReadLen; ++i) {
        t.pow1[i] = (uint32_t)(((uint64_t)t.pow1[i - 1] * kR1) % kP1);
        t.pow2[i] = (uint32_t)(((uint64_t)t.pow2[i - 1] * kR2) % kP2);
    }
    t.inv1 = host_modpow(kR1, kP1 - 2, kP1);
    t.inv2 = host_modpow(kR2, kP2 - 2, kP2);
    for (int c = 0; c < kMaxReadLen / 16; ++c) {
        const uint64_t t0 = 16ull * c;
        cw.w[c][0] = host_modpow(t.inv1, (uint32_t)(t0 + 7), kP1);
        cw.w[c][1] = host_modpow(t.inv1, (uint32_t)(t0 + 15), kP1);
        cw.w[c][2] = host_modpow(t.inv2, (uint32_t)(t0 + 7), kP2);
        cw.w[c][3] = host_modpow(t.inv2, (uint32_t)(t0 + 15), kP2);
        cw.w[c][4] = t.pow1[t0];
        cw.w[c][5] = t.pow1[t0 + 8];
        cw.w[c][6] = t.pow2[t0];
        cw.w[c][7] = t.pow2[t0 + 8];
    }
}

#define EMP_TRY(x)                         \
    do {                                   \
        emp_status _s = (x);               \
        if (_s != EMP_OK) return _s;       \
    } while (0)
#define EMP_CUDA(x) EMP_TRY(cuda_status(x))

struct Events {
    cudaEvent_t e[5] = {};
    Events() { for (auto &x : e) cudaEventCreate(&x); }
    ~Events() { for (auto &x : e) cudaEventDestroy(x); }
};

float ms_between(cudaEvent_t a, cudaEvent_t b);
// time between two events that may not have completed yet: 0 until they have
float ms_between_later(cudaEvent_t a, cudaEvent_t b) {
    if (cudaEventQuery(b) != cudaSuccess) {
        cudaGetLastError();
        return 0.f;
    }
    return ms_between(a, b);
}

float ms_between(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) { cudaGetLastError(); return 0.f; }
    return ms;
}

emp_status sync_and_check(emp_job *j, cudaStream_t s) {
    EMP_CUDA(cudaMemcpyAsync(j->h_misc.p, j->misc.p, kMiscSlots * sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
    EMP_CUDA(cudaStreamSynchronize(s));
    const uint64_t err = j->h_misc.as<uint64_t>()[kMiscErr];
    if (err & kErrSpin) return EMP_E_TIMEOUT;
    return EMP_OK;
}

// fold the per-pass event times of the last sort into the stats (after a sync)
void account_sort(emp_job *j) {
    if (!j->sort_timed) return;
    for (int p = 0; p < kSortPasses; ++p) {
        j->st.ms_sort_passes += ms_between(j->sort_ev[2 * p], j->sort_ev[2 * p + 1]);
        j->st.sort_passes += 1;
        j->st.sort_pass_elems += j->sort_n;
    }
    j->sort_timed = false;
}

void append_bytes(std::vector<uint8_t> &o, const void *p, size_t n) {
    const uint8_t *b = reinterpret_cast<const uint8_t *>(p);
    o.insert(o.end(), b, b + n);
}

// reset look-back status words + tile counter for a chained scan over `tiles`
emp_status reset_chain(emp_job *j, uint64_t tiles, cudaStream_t s) {
    EMP_TRY(ensure(j, j->status, tiles * sizeof(uint64_t) + 64));
    EMP_CUDA(cudaMemsetAsync(j->status.p, 0, tiles * sizeof(uint64_t), s));
    EMP_CUDA(cudaMemsetAsync(j->misc.as<uint64_t>() + kMiscCtr, 0, sizeof(uint64_t), s));
    return EMP_OK;
}
uint32_t *chain_ctr(emp_job *j) { return reinterpret_cast<uint32_t *>(j->misc.as<uint64_t>() + kMiscCtr); }
uint32_t *err_word(emp_job *j) { return reinterpret_cast<uint32_t *>(j->misc.as<uint64_t>() + kMiscErr); }

// the sort scratch must start zeroed and be re-zeroed before its epoch wraps
emp_status ensure_sort_scratch(emp_job *j, uint64_t n_max, cudaStream_t s) {
    const size_t need = sort_scratch_bytes(n_max);
    if (need > j->sort_scratch.bytes || j->sorts_since_clear > 100000) {
        EMP_TRY(ensure(j, j->sort_scratch, need));
        EMP_CUDA(cudaMemsetAsync(j->sort_scratch.p, 0, j->sort_scratch.bytes, s));
        j->sorts_since_clear = 0;
    }
    return EMP_OK;
}

// stable sort of (sk0, sv0)[0..n) in place (ping-pong through sk1/sv1);
// per-pass events for the stats
void timed_sort(emp_job *j, uint64_t n, cudaStream_t s) {
    j->sort_n = n;
    j->sort_timed = true;
    ++j->sorts_since_clear;
    sort_pairs(j->sk0.as<uint64_t>(), j->sv0.as<uint32_t>(), j->sk1.as<uint64_t>(), j->sv1.as<uint32_t>(), n,
               j->sort_scratch.p, j->misc.as<uint64_t>() + kMiscSortN, err_word(j), s, j->sort_ev);
}

// stable sort of (k, v)[0..n) in place through (k1, v1), on the job's sort scratch
void seg_sort(emp_job *j, uint64_t *k, uint32_t *v, uint64_t *k1, uint32_t *v1, uint64_t n, cudaStream_t s) {
    ++j->sorts_since_clear;
    sort_pairs(k, v, k1, v1, n, j->sort_scratch.p, j->misc.as<uint64_t>() + kMiscSortN, err_word(j), s);
}

// The reference's fingerprint sort of a table of n > M entries
// (cq_sort_by_key, cqutils.cuh:180-247; kernels in k_chunked.cu), in place
// on (k, v)[0..n), which hold the table in list order; (k1, v1): n entries
// of scratch.  lst: the table's list values for the read-end ranks that cut
// the chunks, null for the initial table (ids 0..n-1 in order).
emp_status chunked_sort(emp_job *j, uint64_t *k, uint32_t *v, uint64_t *k1, uint32_t *v1, uint64_t n, uint64_t M,
                        const uint32_t *lst, cudaStream_t s) {
    const uint64_t C = 2 * n, h = M / 2;
    EMP_TRY(ensure(j, j->xk0, n * 8));
    EMP_TRY(ensure(j, j->xv0, n * 4));
    EMP_TRY(ensure(j, j->xk1, n * 8));
    EMP_TRY(ensure(j, j->xv1, n * 4));
    EMP_TRY(ensure(j, j->ring_k, C * 8));
    EMP_TRY(ensure(j, j->ring_v, C * 4));
    const uint64_t pcap = n / (h ? h : 1) + 8;  // partitions of one merge of at most n entries
    EMP_TRY(ensure(j, j->cparts, pcap * sizeof(ChunkPart)));
    // sorted by key, then (stably) by chunk: each chunk sorted on its own
    seg_sort(j, k, v, k1, v1, n, s);
    launch_chunk_keys(v, n, lst, M, j->xk0.as<uint64_t>(), j->xv0.as<uint32_t>(), s);
    seg_sort(j, j->xk0.as<uint64_t>(), j->xv0.as<uint32_t>(), j->xk1.as<uint64_t>(), j->xv1.as<uint32_t>(), n, s);
    uint64_t *rk = j->ring_k.as<uint64_t>();
    uint32_t *rv = j->ring_v.as<uint32_t>();
    launch_ring_gather(k, v, j->xv0.as<uint32_t>(), n, rk, rv, s);
    // the FIFO of sorted tables (ring start, entries), oldest first
    std::deque<std::pair<uint64_t, uint64_t>> q;
    for (uint64_t off = 0; off < n; off += M) q.emplace_back(off, n - off < M ? n - off : M);
    uint64_t tail = n;  // ring position after the newest table
    uint64_t *count = j->misc.as<uint64_t>() + kMiscParts;
    while (q.size() > 1) {
        const auto a = q.front();
        q.pop_front();
        const auto b = q.front();
        q.pop_front();
        const uint64_t no = a.second + b.second;
        launch_merge(rk, rv, C, a.first, a.second, b.first, b.second, tail, h, j->cparts.as<ChunkPart>(), pcap,
                     count, err_word(j), s);
        q.emplace_back(tail, no);
        tail = (tail + no) % C;
    }
    launch_ring_copy(rk, rv, C, q.front().first, n, k, v, s);
    return EMP_OK;
}

// Record `ne` edges from the host edge arrays into output.bin (overlap.cu:148-161).
void emit_record(emp_job *j, int32_t ovlp, uint64_t e0, uint64_t e1) {
    const uint64_t ne = e1 - e0;
    append_bytes(j->out, &ne, 8);
    append_bytes(j->out, &ovlp, 4);
    if (ne) {
        append_bytes(j->out, j->h_from.as<uint32_t>() + e0, ne * 4);
        append_bytes(j->out, j->h_to.as<uint32_t>() + e0, ne * 4);
    }
    j->st.n_records += 1;
}

struct RoundEnv {
    int L;
    int rounds;
    uint64_t M;
    uint64_t wpc;
    const HashTables *tables;
    const uint32_t *seq2;  // read-major 2-bit bases, wpr words per read
    int wpr;
};

// One round with host synchronisation: used while the tables are large enough
// for the reference to split a round into several search partitions
// (cq_get_search_partitions, cqutils.cuh:108-137).  Full sort of both tables.
emp_status sync_round(emp_job *j, cudaStream_t s, const RoundEnv &env, int r, int &cur, uint64_t &n_in,
                      uint64_t &S_out, uint64_t &P_out, bool &stop) {
    emp_stats &st = j->st;
    uint64_t *hm = j->h_misc.as<uint64_t>();
    uint64_t *dm = j->misc.as<uint64_t>();
    uint64_t *lk[2] = {j->lk0.as<uint64_t>(), j->lk1.as<uint64_t>()};
    uint32_t *lv[2] = {j->lv0.as<uint32_t>(), j->lv1.as<uint32_t>()};
    const uint64_t M = env.M;
    EMP_TRY(reset_chain(j, upd_tiles(n_in), s));
    EMP_CUDA(cudaMemsetAsync(dm + kMiscNout, 0, 2 * sizeof(uint64_t), s));
    RoundArgs a{};
    a.kin = lk[cur];
    a.vin = lv[cur];
    a.n_in = n_in;
    a.kout = lk[cur ^ 1];
    a.vout = lv[cur ^ 1];
    a.used_s = j->used_s.as<uint8_t>();
    a.used_p = j->used_p.as<uint8_t>();
    a.cols = j->cols.as<uint32_t>();
    a.wpc = env.wpc;
    a.tables = env.tables;
    a.L = env.L;
    a.round = r;
    a.status = j->status.as<uint64_t>();
    a.tile_ctr = chain_ctr(j);
    a.n_out = dm + kMiscNout;
    a.s_out = dm + kMiscSout;
    a.err = err_word(j);
    launch_update_compact(a, s);
    EMP_TRY(sync_and_check(j, s));
    const uint64_t N = hm[kMiscNout], S = hm[kMiscSout], P = N - S;
    S_out = S;
    P_out = P;
    if (S == 0) {  // loop condition of build_graph (overlap.cu:258)
        stop = true;
        return EMP_OK;
    }
    cur ^= 1;
    n_in = N;
    if (r < EMP_MAX_ROUNDS) {
        st.sfx_live[r] = S;
        st.pfx_live[r] = P;
    }
    st.n_rounds = r + 1;
    if (P == 0) return EMP_OK;  // one-sided search partition: no record
    const bool split = S >= M / 2 || P >= M / 2;
    // sort a copy of the merged list (the list itself carries over); a table
    // larger than M first takes the order of the reference's chunked sort,
    // which the stable sort of both tables then keeps among equal keys
    EMP_CUDA(cudaMemcpyAsync(j->sk0.p, lk[cur], N * 8, cudaMemcpyDeviceToDevice, s));
    EMP_CUDA(cudaMemcpyAsync(j->sv0.p, lv[cur], N * 4, cudaMemcpyDeviceToDevice, s));
    if (S > M)
        EMP_TRY(chunked_sort(j, j->sk0.as<uint64_t>(), j->sv0.as<uint32_t>(), j->sk1.as<uint64_t>(),
                             j->sv1.as<uint32_t>(), S, M, lv[cur], s));
    if (P > M)
        EMP_TRY(chunked_sort(j, j->sk0.as<uint64_t>() + S, j->sv0.as<uint32_t>() + S, j->sk1.as<uint64_t>() + S,
                             j->sv1.as<uint32_t>() + S, P, M, lv[cur] + S, s));
    timed_sort(j, N, s);
    const uint64_t *sk = j->sk0.as<uint64_t>();
    const uint32_t *sv = j->sv0.as<uint32_t>();
    EMP_TRY(ensure(j, j->cnt, N * 4));
    EMP_TRY(ensure(j, j->offs, N * 8));
    launch_join_count(sk, sv, N, j->cnt.as<uint32_t>(), s);
    EMP_TRY(reset_chain(j, scan_tiles(N), s));
    launch_scan_u32_u64(j->cnt.as<uint32_t>(), j->offs.as<uint64_t>(), N, j->status.as<uint64_t>(), chain_ctr(j),
                        dm + kMiscE, err_word(j), s);
    EMP_TRY(sync_and_check(j, s));
    account_sort(j);
    const uint64_t E = hm[kMiscE];
    if (E) {
        EMP_TRY(ensure(j, j->efrom, E * 4));
        EMP_TRY(ensure(j, j->eto, E * 4));
        if (!j->h_from.ensure(E * 4) || !j->h_to.ensure(E * 4)) return EMP_E_NOMEM;
        launch_join_write(sk, sv, N, j->cnt.as<uint32_t>(), j->offs.as<uint64_t>(), j->efrom.as<uint32_t>(),
                          j->eto.as<uint32_t>(), j->used_s.as<uint8_t>(), j->used_p.as<uint8_t>(), s);
        EMP_CUDA(cudaMemcpyAsync(j->h_from.p, j->efrom.p, E * 4, cudaMemcpyDeviceToHost, s));
        EMP_CUDA(cudaMemcpyAsync(j->h_to.p, j->eto.p, E * 4, cudaMemcpyDeviceToHost, s));
        EMP_CUDA(cudaStreamSynchronize(s));
    }
    const int32_t ovlp = env.L - 1 - r;
    if (!split) {
        emit_record(j, ovlp, 0, E);
    } else {
        // search partitions of windows M/2; each two-sided one is a record
        EMP_TRY(ensure(j, j->akeys, S * 8));
        EMP_TRY(ensure(j, j->apos, S * 4));
        EMP_TRY(ensure(j, j->bkeys, P * 8));
        const uint64_t pcap = 4 * (N / (M / 2) + 1) + 1024;
        EMP_TRY(ensure(j, j->parts, pcap * sizeof(SearchPart)));
        EMP_TRY(reset_chain(j, upd_tiles(N), s));
        launch_split_tables(sk, sv, N, j->akeys.as<uint64_t>(), j->apos.as<uint32_t>(), j->bkeys.as<uint64_t>(),
                            j->status.as<uint64_t>(), chain_ctr(j), err_word(j), s);
        launch_search_partitions(j->akeys.as<uint64_t>(), S, j->bkeys.as<uint64_t>(), P, M / 2,
                                 j->apos.as<uint32_t>(), j->offs.as<uint64_t>(), E, j->parts.as<SearchPart>(), pcap,
                                 dm + kMiscParts, err_word(j), s);
        EMP_TRY(sync_and_check(j, s));
        if (hm[kMiscErr] & kErrHang) return EMP_E_HANG;
        if (hm[kMiscErr] & kErrCapacity) return EMP_E_UNSUPPORTED;
        const uint64_t np = hm[kMiscParts];
        if (!j->h_parts.ensure(np * sizeof(SearchPart) + 16)) return EMP_E_NOMEM;
        EMP_CUDA(cudaMemcpyAsync(j->h_parts.p, j->parts.p, np * sizeof(SearchPart), cudaMemcpyDeviceToHost, s));
        EMP_CUDA(cudaStreamSynchronize(s));
        const SearchPart *ps = j->h_parts.as<SearchPart>();
        for (uint64_t q = 0; q < np; ++q)
            if (ps[q].pa && ps[q].pb) emit_record(j, ovlp, ps[q].e0, ps[q].e1);
    }
    st.n_edges += E;
    if (r < EMP_MAX_ROUNDS) st.edges[r] = E;
    return EMP_OK;
}

// Profiling aid: per-round phase durations (us) of a cooperative round kernel
// whose barriers stamp phases 0 .. nph-1 of every iteration.
void write_coop_trace(emp_job *j, const char *path, int rounds, int r0, const RoundRecord *rec, cudaStream_t s,
                      int nph, const char *phase_cols) {
    std::vector<uint64_t> t((size_t)rounds * kCoopTracePhases);
    if (cudaMemcpyAsync(t.data(), j->coop_trace.p, t.size() * 8, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return;
    FILE *f = std::fopen(path, "w");
    if (!f) return;
    std::fprintf(f, "round,%s,S,P,C,E\n", phase_cols);
    for (int i = 0; i + r0 < rounds; ++i) {
        const uint64_t *p = &t[(size_t)i * kCoopTracePhases];
        if (!p[nph - 1]) break;
        uint64_t prev = i ? t[(size_t)(i - 1) * kCoopTracePhases + nph - 1] : p[0];
        std::fprintf(f, "%d", i + r0);
        for (int q = 0; q < nph; ++q) {
            std::fprintf(f, ",%.2f", (p[q] - prev) / 1e3);
            prev = p[q];
        }
        const RoundRecord &x = rec[i + r0];
        std::fprintf(f, ",%llu,%llu,%llu,%llu\n", (unsigned long long)x.S, (unsigned long long)x.P,
                     (unsigned long long)x.C, (unsigned long long)x.E);
    }
    std::fclose(f);
}

// Profiling aid: per-CTA stamps (ns after the earliest stamp) of one iteration.
void write_coop_probe(emp_job *j, const char *path, int grid, cudaStream_t s) {
    std::vector<uint64_t> t((size_t)grid * kCoopProbePoints);
    if (cudaMemcpyAsync(t.data(), j->coop_probe.p, t.size() * 8, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return;
    uint64_t t0 = ~0ull;
    for (uint64_t x : t)
        if (x && x < t0) t0 = x;
    FILE *f = std::fopen(path, "w");
    if (!f) return;
    std::fprintf(f, "cta");
    for (int p = 0; p < kCoopProbePoints; ++p) std::fprintf(f, ",p%d", p);
    std::fprintf(f, "\n");
    for (int c = 0; c < grid; ++c) {
        std::fprintf(f, "%d", c);
        for (int p = 0; p < kCoopProbePoints; ++p) {
            const uint64_t x = t[(size_t)c * kCoopProbePoints + p];
            std::fprintf(f, ",%lld", x ? (long long)(x - t0) : -1ll);
        }
        std::fprintf(f, "\n");
    }
    std::fclose(f);
}

// Whether rounds may run in the bucket kernel on this context (cooperative
// launch available, not turned off by the tuning).
bool bucket_rounds_usable(const emp_ctx *c) { return c->tune.round_driver == 0 && bucket_grid_size() > 0; }

// The control block of a bucket-kernel launch: the context's grid-barrier
// limit, and the testing barrier that no arrival completes (used once).
void coop_ctl_init(emp_ctx *c, CoopCtl *hc, uint32_t njobs) {
    std::memset(hc, 0, sizeof(CoopCtl));
    hc->njobs = njobs;
    hc->active = njobs;
    hc->wait_ns = c->tune.wait_limit_ns;
    if (c->tune.block_next_wait) {
        hc->bar_extra = 1;
        c->tune.block_next_wait = 0;
    }
}

// Buffers and launch description (host copy *hj) of rounds r0 .. of one job
// in the bucket kernel (k_bucket.cu).  `wave`: bucket counts are multiples
// of it (the grid when the job has the GPU alone, 1 in a batch).
emp_status bucket_prepare(emp_job *j, cudaStream_t s, const RoundEnv &env, int r0, int cur, uint64_t n_in,
                          uint64_t ecap, uint32_t wave, BktJob *hj) {
    const uint64_t nmax = n_in;
    const emp_tuning &tu = j->ctx->tune;
    const uint32_t mean = tu.bucket_mean ? tu.bucket_mean : kBktMean;
    const uint32_t nb_max = bkt_count(nmax, wave, mean);
    const uint32_t cap = tu.region_cap ? tu.region_cap : kBktRegionCap;
    const uint64_t list_entries = (uint64_t)nb_max * 2 * cap;
    const uint64_t iters = (uint64_t)(env.rounds - r0) + 1;  // lists of iterations 0 .. rounds - r0
    const size_t cnt_bytes = iters * 2 * nb_max * 4;
    EMP_TRY(ensure(j, j->bk_lst0, list_entries * sizeof(BktEntry)));
    EMP_TRY(ensure(j, j->bk_lst1, list_entries * sizeof(BktEntry)));
    EMP_TRY(ensure(j, j->bk_cnt, cnt_bytes + iters * 4));
    EMP_TRY(ensure(j, j->bk_spill, 2 * nmax * (sizeof(BktEntry) + 4)));
    EMP_CUDA(cudaMemsetAsync(j->bk_cnt.p, 0, cnt_bytes + iters * 4, s));
    EMP_TRY(ensure(j, j->bk_spans, (size_t)env.rounds * nb_max * sizeof(BktSpan)));
    EMP_TRY(ensure(j, j->bk_sfrom, ecap * 4));
    EMP_TRY(ensure(j, j->bk_sto, ecap * 4));
    EMP_TRY(ensure(j, j->bk_scratch, bkt_scratch_bytes(nmax)));
    EMP_TRY(ensure(j, j->bk_meta, ((size_t)env.rounds + 1) * sizeof(BktRound)));
    EMP_CUDA(cudaMemsetAsync(j->bk_meta.p, 0, ((size_t)env.rounds + 1) * sizeof(BktRound), s));
    EMP_TRY(ensure(j, j->dout, (size_t)env.rounds * 12 + ecap * 8));
    EMP_TRY(ensure(j, j->records, (size_t)env.rounds * sizeof(RoundRecord)));
    if (!j->h_records.ensure((size_t)env.rounds * sizeof(RoundRecord))) return EMP_E_NOMEM;
    std::memset(hj, 0, sizeof(BktJob));
    hj->lk_in = cur ? j->lk1.as<uint64_t>() : j->lk0.as<uint64_t>();
    hj->lv_in = cur ? j->lv1.as<uint32_t>() : j->lv0.as<uint32_t>();
    hj->used_s = j->used_s.as<uint8_t>();
    hj->used_p = j->used_p.as<uint8_t>();
    hj->lst[0] = j->bk_lst0.as<BktEntry>();
    hj->lst[1] = j->bk_lst1.as<BktEntry>();
    hj->seq2 = env.seq2;
    hj->wpr = env.wpr;
    hj->L = env.L;
    hj->rounds = env.rounds;
    hj->tables = env.tables;
    hj->n_in = n_in;
    hj->cnt = j->bk_cnt.as<uint32_t>();
    hj->spill_n = hj->cnt + iters * 2 * nb_max;
    hj->spill[0] = j->bk_spill.as<BktEntry>();
    hj->spill[1] = hj->spill[0] + nmax;
    hj->spill_tag[0] = reinterpret_cast<uint32_t *>(hj->spill[1] + nmax);
    hj->spill_tag[1] = hj->spill_tag[0] + nmax;
    hj->cap = cap;
    hj->spans = j->bk_spans.as<BktSpan>();
    hj->sfrom = j->bk_sfrom.as<uint32_t>();
    hj->sto = j->bk_sto.as<uint32_t>();
    hj->out = j->dout.as<uint8_t>();
    hj->ecap = ecap;
    hj->records = j->records.as<RoundRecord>();
    hj->scratch = j->bk_scratch.as<uint8_t>();
    hj->n_max = nmax;
    hj->nb_max = nb_max;
    hj->wave = wave;
    hj->mean = mean;
    hj->r0 = r0;
    hj->meta = j->bk_meta.as<BktRound>();
    return EMP_OK;
}

// Queue the copy of the job's round records to the host.
emp_status bucket_fetch(emp_job *j, const RoundEnv &env, cudaStream_t s) {
    EMP_CUDA(cudaMemcpyAsync(j->h_records.p, j->records.p, (size_t)env.rounds * sizeof(RoundRecord),
                             cudaMemcpyDeviceToHost, s));
    return EMP_OK;
}

// After the launch and a synchronisation: the job's counts and output size
// from its launch description (copied back) and records.  kNeedEdgeRoom with
// *needed set when its edge buffer was too small.
emp_status bucket_collect(emp_job *j, int r0, uint64_t n_in, const BktJob &hj, uint64_t *needed) {
    emp_stats &st = j->st;
    if (hj.overflow) {
        *needed = hj.e_total;
        return kNeedEdgeRoom;
    }
    const RoundRecord *rec = j->h_records.as<RoundRecord>();
    const int r_end = (int)hj.round;  // rounds run with a non-empty suffix table
    uint64_t prev_n = n_in;
    for (int q = r0; q < r_end; ++q) {
        const RoundRecord &x = rec[q];
        const uint64_t n_out = x.S + x.P;
        // each round gathers its entries and writes the kept ones for the next
        st.round_kernel_bytes += 16 * prev_n + 16 * n_out + 8 * x.E;
        if (q < EMP_MAX_ROUNDS) {
            st.sfx_live[q] = x.S;
            st.pfx_live[q] = x.P;
            st.edges[q] = x.E;
        }
        if (x.P) {  // the kernel wrote the record into dout
            j->dout_bytes += 12 + 8 * x.E;
            st.n_records += 1;
        }
        st.n_edges += x.E;
        prev_n = n_out;
    }
    st.n_rounds = r_end;
    return EMP_OK;
}

// Rounds r0 .. of one job alone in the bucket kernel: one cooperative launch,
// one grid barrier per round.
emp_status run_rounds_bucket(emp_job *j, cudaStream_t s, const RoundEnv &env, int r0, int cur, uint64_t n_in,
                             uint64_t ecap, uint64_t *needed) {
    emp_stats &st = j->st;
    const int grid = bucket_grid_size();
    EMP_TRY(ensure(j, j->bk_job, sizeof(BktJob)));
    EMP_TRY(ensure(j, j->coop_ctl, sizeof(CoopCtl)));
    if (!j->h_coop.ensure(sizeof(BktJob) + sizeof(CoopCtl))) return EMP_E_NOMEM;
    BktJob *hj = j->h_coop.as<BktJob>();
    CoopCtl *hc = reinterpret_cast<CoopCtl *>(hj + 1);
    EMP_TRY(bucket_prepare(j, s, env, r0, cur, n_in, ecap, (uint32_t)grid, hj));
    coop_ctl_init(j->ctx, hc, 1);
    const char *trace_path = j->ctx->trace_path.empty() ? nullptr : j->ctx->trace_path.c_str();
    if (trace_path) {
        EMP_TRY(ensure(j, j->coop_trace, (size_t)env.rounds * kCoopTracePhases * 8));
        EMP_CUDA(cudaMemsetAsync(j->coop_trace.p, 0, j->coop_trace.bytes, s));
        hc->trace = j->coop_trace.as<uint64_t>();
        hc->trace_cap = (uint32_t)env.rounds;
    }
    const char *probe_env = j->ctx->probe_spec.empty() ? nullptr : j->ctx->probe_spec.c_str();
    std::string probe_path;
    if (probe_env) {
        const char *colon = std::strrchr(probe_env, ':');
        probe_path.assign(probe_env, colon ? (size_t)(colon - probe_env) : std::strlen(probe_env));
        hc->probe_iter = colon ? (uint32_t)std::atoi(colon + 1) : 0u;
        EMP_TRY(ensure(j, j->coop_probe, (size_t)grid * kCoopProbePoints * 8));
        EMP_CUDA(cudaMemsetAsync(j->coop_probe.p, 0, j->coop_probe.bytes, s));
        hc->probe = j->coop_probe.as<uint64_t>();
    }
    hj->pre_done = bucket_prologue_apart(*hj) ? 1u : 0u;
    EMP_CUDA(cudaMemcpyAsync(j->bk_job.p, hj, sizeof(BktJob), cudaMemcpyHostToDevice, s));
    EMP_CUDA(cudaMemcpyAsync(j->coop_ctl.p, hc, sizeof(CoopCtl), cudaMemcpyHostToDevice, s));
    cudaEvent_t e0 = j->upd_ev[0], e1 = j->upd_ev[1];
    EMP_CUDA(cudaEventRecord(e0, s));
    if (hj->pre_done) EMP_CUDA(launch_bucket_prologue(j->bk_job.as<BktJob>(), s));
    EMP_CUDA(launch_bucket_rounds(j->bk_job.as<BktJob>(), j->coop_ctl.as<CoopCtl>(), err_word(j), s));
    EMP_CUDA(cudaEventRecord(e1, s));
    EMP_CUDA(cudaMemcpyAsync(hj, j->bk_job.p, sizeof(BktJob), cudaMemcpyDeviceToHost, s));
    EMP_CUDA(cudaMemcpyAsync(hc, j->coop_ctl.p, sizeof(CoopCtl), cudaMemcpyDeviceToHost, s));
    EMP_TRY(bucket_fetch(j, env, s));
    EMP_TRY(sync_and_check(j, s));
    if (hc->err & kErrSpin) return EMP_E_TIMEOUT;
    st.ms_round_kernel += ms_between(e0, e1);
    if (trace_path) write_coop_trace(j, trace_path, env.rounds, r0, j->h_records.as<RoundRecord>(), s, 1, "round_us");
    if (probe_env) write_coop_probe(j, probe_path.c_str(), grid, s);
    return bucket_collect(j, r0, n_in, *hj, needed);
}

// Round counters, output and used marks of a job, before its rounds.
emp_status rounds_prelude(emp_job *j, cudaStream_t s) {
    emp_stats &st = j->st;
    st.n_rounds = 0;
    st.n_edges = 0;
    st.n_records = 0;
    std::memset(st.sfx_live, 0, sizeof st.sfx_live);
    std::memset(st.pfx_live, 0, sizeof st.pfx_live);
    std::memset(st.edges, 0, sizeof st.edges);
    j->out.clear();
    j->dout_bytes = 0;
    EMP_CUDA(cudaMemsetAsync(j->used_s.p, 0, j->used_s.bytes, s));
    EMP_CUDA(cudaMemsetAsync(j->used_p.p, 0, j->used_p.bytes, s));
    return EMP_OK;
}

// All rounds: synchronous ones while a round could split into several search
// partitions (sizes only shrink), then the device-resident pipeline for the
// rest with a single synchronisation at the end.  Returns kNeedEdgeRoom with
// *needed set when the pipeline's edge buffer (ecap edges) was too small.
emp_status run_rounds(emp_job *j, cudaStream_t s, const RoundEnv &env, uint64_t U, uint64_t ecap, uint64_t *needed) {
    if (!j->upd_ev[0]) {  // per-round events, made when a job first runs rounds on its own
        for (auto &e : j->upd_ev) EMP_CUDA(cudaEventCreate(&e));
    }
    EMP_TRY(rounds_prelude(j, s));
    int cur = 0, r = 0;
    uint64_t n_in = 2 * U, S = U, P = U;
    const uint64_t M = env.M;
    const bool bucket = bucket_rounds_usable(j->ctx);
    // host-synchronised rounds (one full sort each) while a round may split
    // into several search partitions, and while the list is too large for the
    // bucket kernel
    while (r < env.rounds && (!bucket || S >= M / 2 || P >= M / 2 || n_in > kBktMaxEntries)) {
        bool stop = false;
        EMP_TRY(sync_round(j, s, env, r, cur, n_in, S, P, stop));
        if (stop) return EMP_OK;
        ++r;
    }
    if (r >= env.rounds) return EMP_OK;
    return run_rounds_bucket(j, s, env, r, cur, n_in, ecap, needed);
}

// The map phase of a job, in stages that each end where the host must read
// a count before sizing the next step (one stream synchronisation between
// stages; a batch of jobs shares it).  A stage returns EMP_OK with j->prep.done
// set once the job has nothing more to run.
emp_status map_begin(emp_job *j, cudaStream_t s) {
    emp_stats &st = j->st;
    j->stream = s;
    if (j->feed_pending) {  // the FASTQ is still being copied in
        EMP_CUDA(cudaStreamWaitEvent(s, j->feed_ev[1], 0));
        j->feed_pending = false;
        j->ms_h2d += ms_between_later(j->feed_ev[0], j->feed_ev[1]);
    }
    std::memset(&st, 0, sizeof st);
    j->out.clear();
    j->dout_bytes = 0;
    j->have_result = false;
    j->n_ends = 0;
    j->prep = JobPrep{};
    st.fastq_bytes = j->F;
    st.ms_h2d = j->ms_h2d;
    j->prep.launches0 = g_launches.load();
    j->prep.M = j->p.reduce_mem / 16;
    if (j->prep.M < 2) return EMP_E_INVAL;
    cudaEventRecord(j->map_ev[0], s);
    EMP_TRY(ensure(j, j->misc, kMiscSlots * sizeof(uint64_t)));
    if (!j->h_misc.ensure(kMiscSlots * sizeof(uint64_t)) || !j->h_hist.ensure(kSortPasses * kSortRadix * 4))
        return EMP_E_NOMEM;
    EMP_CUDA(cudaMemsetAsync(j->misc.p, 0, kMiscSlots * sizeof(uint64_t), s));
    const uint64_t F = j->F;
    if (!F) return EMP_OK;
    // ---- K1: newline index
    const uint64_t T = parse_tiles(F);
    EMP_TRY(ensure(j, j->tile_counts, T * 4));
    EMP_TRY(ensure(j, j->tile_excl, T * 8));
    launch_nl_count(j->fq.as<uint8_t>(), F, j->tile_counts.as<uint32_t>(), j->misc.as<uint64_t>() + kMiscLen0, s);
    EMP_TRY(reset_chain(j, scan_tiles(T), s));
    launch_scan_u32_u64(j->tile_counts.as<uint32_t>(), j->tile_excl.as<uint64_t>(), T, j->status.as<uint64_t>(),
                        chain_ctr(j), j->misc.as<uint64_t>() + kMiscTotal, err_word(j), s);
    return EMP_OK;
}

// queue the copy of the job's device words that the next stage reads
emp_status map_fetch(emp_job *j, cudaStream_t s) {
    EMP_CUDA(cudaMemcpyAsync(j->h_misc.p, j->misc.p, kMiscSlots * sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
    return EMP_OK;
}
emp_status map_check(emp_job *j) {
    return (j->h_misc.as<uint64_t>()[kMiscErr] & kErrSpin) ? EMP_E_TIMEOUT : EMP_OK;
}

// nothing (more) to run: close the job's timings
void map_finish_empty(emp_job *j, cudaStream_t s) {
    cudaEventRecord(j->map_ev[4], s);
    j->prep.done = true;
}

emp_status launch_reads(emp_job *j, cudaStream_t s, int wpr);
emp_status dedup_by_sort(emp_job *j, cudaStream_t s);

emp_status map_records(emp_job *j, cudaStream_t s) {
    EMP_TRY(map_check(j));
    uint64_t *hm = j->h_misc.as<uint64_t>();
    uint64_t *dm = j->misc.as<uint64_t>();
    const uint64_t F = j->F;
    const uint64_t total_nl = F ? hm[kMiscTotal] : 0;
    const uint64_t n_rec = total_nl ? (total_nl + 3) / 4 : 0;
    j->prep.n_rec = n_rec;
    if (!n_rec) {
        map_finish_empty(j, s);
        return EMP_OK;
    }
    // the map kernels load the FASTQ as aligned 16-byte blocks
    if (reinterpret_cast<uintptr_t>(j->fq.p) & 15u) return EMP_E_CUDA;
    // ---- K2: every record in one pass: N filter, length, fingerprints of
    // both read-ends, read-major 2-bit words; kept reads numbered in order.
    // The words are laid out for the first record's length (the usual case:
    // every read has it); map_keys runs the pass again when the kept reads'
    // length needs another layout.
    const uint64_t len0 = hm[kMiscLen0];
    const int wpr = len0 >= 1 && len0 <= (uint64_t)kMaxReadLen ? (int)((len0 + 15) / 16) : kMaxReadLen / 16;
    return launch_reads(j, s, wpr);
}

// The read pass (K2) with `wpr` read-major words per read.
emp_status launch_reads(emp_job *j, cudaStream_t s, int wpr) {
    uint64_t *hm = j->h_misc.as<uint64_t>();
    uint64_t *dm = j->misc.as<uint64_t>();
    const uint64_t n_rec = j->prep.n_rec;
    j->prep.wpr = wpr;
    EMP_TRY(ensure(j, j->keys0, n_rec * 16));
    EMP_TRY(ensure(j, j->seq2, n_rec * (uint64_t)wpr * 4));
    EMP_TRY(ensure(j, j->keep, n_rec * 4));
    const uint32_t mm[4] = {0xffffffffu, 0u, 0u, 0u};  // length extremes, then the kept count
    std::memcpy(hm + kMiscLen, mm, 16);
    EMP_CUDA(cudaMemcpyAsync(dm + kMiscLen, hm + kMiscLen, 16, cudaMemcpyHostToDevice, s));
    launch_read_pass(j->fq.as<uint8_t>(), j->F, j->tile_excl.as<uint64_t>(), j->ctx->tables.as<HashTables>(),
                     reinterpret_cast<const ChunkWeights *>(j->ctx->tables.as<uint8_t>() + sizeof(HashTables)),
                     j->keys0.as<uint64_t>(), j->seq2.as<uint32_t>(), wpr, j->keep.as<uint32_t>(), dm + kMiscN,
                     reinterpret_cast<uint32_t *>(dm + kMiscLen), err_word(j), s);
    cudaEventRecord(j->map_ev[1], s);
    return EMP_OK;
}

// Whether a round of a job of n reads may run outside the bucket kernel (the
// host-synchronised rounds, the pipeline and the per-round cooperative
// kernel read bases from the column store; the bucket kernel from seq2).
// Each table holds at most 2n entries and the list at most 4n, so with
// 2n < M/2 and 4n within the bucket kernel's list limit every round runs
// there.
bool columns_needed(const emp_ctx *c, uint64_t n, uint64_t M) {
    return !bucket_rounds_usable(c) || 2 * n >= M / 2 || 4 * n > kBktMaxEntries;
}

emp_status map_keys(emp_job *j, cudaStream_t s) {
    EMP_TRY(map_check(j));
    JobPrep &q = j->prep;
    uint64_t *hm = j->h_misc.as<uint64_t>();
    uint64_t *dm = j->misc.as<uint64_t>();
    emp_stats &st = j->st;
    if (hm[kMiscErr] & kErrBadBase) return EMP_E_FORMAT;
    const uint64_t n = hm[kMiscN];
    uint32_t mm2[2];
    std::memcpy(mm2, hm + kMiscLen, 8);
    int L = 0;
    if (n) {
        if (mm2[0] != mm2[1]) return EMP_E_FORMAT;
        L = (int)mm2[0];
        if (mm2[0] > (uint32_t)kMaxReadLen) return EMP_E_UNSUPPORTED;
    }
    q.n = n;
    q.L = L;
    st.n_reads = n;
    st.read_len = L;
    if (n == 0) {
        map_finish_empty(j, s);
        return EMP_OK;
    }
    if (j->p.min_ovlp < 0) return EMP_E_INVAL;
    const uint64_t n2 = 2 * n;
    if (n2 >= (1ull << 31)) return EMP_E_UNSUPPORTED;
    if (q.wpr != (L + 15) / 16) {  // the kept reads are not as long as the first record: lay the words out again
        EMP_TRY(launch_reads(j, s, (L + 15) / 16));
        EMP_TRY(sync_and_check(j, s));
        if (hm[kMiscErr] & kErrBadBase) return EMP_E_FORMAT;
    }
    if (n < q.n_rec) {  // the N filter or an empty line dropped a record: the kept ones to indices 0 .. n-1
        EMP_TRY(ensure(j, j->keys_tmp, n * 16));
        EMP_TRY(ensure(j, j->seq2_tmp, n * (uint64_t)q.wpr * 4));
        EMP_TRY(reset_chain(j, scan_tiles(q.n_rec), s));
        launch_scan_u32_u32(j->keep.as<uint32_t>(), j->keep.as<uint32_t>(), q.n_rec, j->status.as<uint64_t>(),
                            chain_ctr(j), dm + kMiscKept, err_word(j), s);
        launch_compact_reads(j->keep.as<uint32_t>(), q.n_rec, n, j->keys0.as<uint64_t>(), j->seq2.as<uint32_t>(),
                             q.wpr, j->keys_tmp.as<uint64_t>(), j->seq2_tmp.as<uint32_t>(), s);
        swap_buf(j->keys0, j->keys_tmp);
        swap_buf(j->seq2, j->seq2_tmp);
    }
    // ---- column-major 2-bit store, for rounds that run outside the bucket kernel
    q.wpc = (n + 15) / 16;
    if (columns_needed(j->ctx, n, q.M)) {
        EMP_TRY(ensure(j, j->cols, (uint64_t)L * q.wpc * 4));
        launch_columns(j->seq2.as<uint32_t>(), n, L, q.wpr, j->cols.as<uint32_t>(), q.wpc, s);
    }
    j->n_ends = n2;
    // ---- fingerprint sort + duplicate removal (overlap.cu:212-225)
    const uint64_t cap = 2 * n2;  // both tables, each at most n2 entries
    EMP_TRY(ensure(j, j->sk0, cap * 8));
    EMP_TRY(ensure(j, j->sk1, cap * 8));
    EMP_TRY(ensure(j, j->sv0, cap * 4));
    EMP_TRY(ensure(j, j->sv1, cap * 4));
    EMP_TRY(ensure(j, j->lk0, cap * 8));
    EMP_TRY(ensure(j, j->lk1, cap * 8));
    EMP_TRY(ensure(j, j->lv0, cap * 4));
    EMP_TRY(ensure(j, j->lv1, cap * 4));
    EMP_TRY(ensure(j, j->alive, n2));
    EMP_TRY(ensure(j, j->used_s, n2));
    EMP_TRY(ensure(j, j->used_p, n2));
    EMP_TRY(ensure_sort_scratch(j, cap, s));
    const uint32_t nbd = n2 <= q.M && j->ctx->tune.dedup_driver == 0 ? dedup_buckets(n2) : 0u;
    bool hashed = false;
    if (nbd) {  // in core: the smallest rid of every fingerprint survives, no sort needed
        EMP_TRY(ensure(j, j->dedup_scr, dedup_scratch_bytes(nbd)));
        EMP_TRY(reset_chain(j, scan_tiles(nbd), s));
        hashed = launch_dedup_hash(j->keys0.as<uint64_t>(), n2, nbd, j->dedup_scr.p, j->sk0.as<uint64_t>(),
                                   j->sv0.as<uint32_t>(), j->alive.as<uint8_t>(), j->status.as<uint64_t>(),
                                   chain_ctr(j), dm + kMiscSortN, err_word(j), s);
    }
    if (!hashed) EMP_TRY(dedup_by_sort(j, s));
    EMP_TRY(reset_chain(j, upd_tiles(n2), s));
    launch_init_list(j->keys0.as<uint64_t>(), j->alive.as<uint8_t>(), n, j->lk0.as<uint64_t>(), j->lv0.as<uint32_t>(),
                     j->status.as<uint64_t>(), chain_ctr(j), dm + kMiscU, err_word(j), s);
    return EMP_OK;
}

// Duplicate removal through the sort of all (fingerprint, rid) pairs: the
// reference's chunked sort when 2n > M (its merge tree picks the survivors),
// else one stable radix sort; the first of every equal-key run survives.
emp_status dedup_by_sort(emp_job *j, cudaStream_t s) {
    const JobPrep &q = j->prep;
    const uint64_t n2 = 2 * q.n;
    EMP_CUDA(cudaMemcpyAsync(j->sk0.p, j->keys0.p, n2 * 8, cudaMemcpyDeviceToDevice, s));
    launch_iota(j->sv0.as<uint32_t>(), n2, s);
    if (n2 > q.M) {  // chunked sort and its duplicate-removal walk (2n > M)
        EMP_TRY(chunked_sort(j, j->sk0.as<uint64_t>(), j->sv0.as<uint32_t>(), j->sk1.as<uint64_t>(),
                             j->sv1.as<uint32_t>(), n2, q.M, nullptr, s));
        launch_unique_walk(j->sk0.as<uint64_t>(), n2, q.M, err_word(j), s);
    } else {
        timed_sort(j, n2, s);
    }
    launch_dedup_mark(j->sk0.as<uint64_t>(), j->sv0.as<uint32_t>(), n2, j->alive.as<uint8_t>(), s);
    return EMP_OK;
}

// The initial list (suffixes then prefixes) is ready; the rounds environment
// follows.
emp_status map_list(emp_job *j, cudaStream_t s) {
    EMP_TRY(map_check(j));
    JobPrep &q = j->prep;
    if (j->h_misc.as<uint64_t>()[kMiscErr] & kErrDedupFull) {  // a dedup bucket overflowed: sort instead
        uint64_t *dm = j->misc.as<uint64_t>();
        const uint32_t clear = (uint32_t)(j->h_misc.as<uint64_t>()[kMiscErr] & ~(uint64_t)kErrDedupFull);
        EMP_CUDA(cudaMemcpyAsync(dm + kMiscErr, &clear, 4, cudaMemcpyHostToDevice, s));
        EMP_TRY(dedup_by_sort(j, s));
        EMP_TRY(reset_chain(j, upd_tiles(2 * q.n), s));
        launch_init_list(j->keys0.as<uint64_t>(), j->alive.as<uint8_t>(), q.n, j->lk0.as<uint64_t>(),
                         j->lv0.as<uint32_t>(), j->status.as<uint64_t>(), chain_ctr(j), dm + kMiscU, err_word(j), s);
        EMP_TRY(sync_and_check(j, s));
    }
    if (j->h_misc.as<uint64_t>()[kMiscErr] & kErrHang) return EMP_E_HANG;
    if (j->h_misc.as<uint64_t>()[kMiscErr] & kErrCapacity) return EMP_E_UNSUPPORTED;
    account_sort(j);
    const uint64_t U = j->h_misc.as<uint64_t>()[kMiscU];
    q.U = U;
    j->st.n_unique = U;
    launch_dup_prefix_half(j->lk0.as<uint64_t>(), j->lv0.as<uint32_t>(), U, s);
    cudaEventRecord(j->map_ev[2], s);
    q.rounds = q.L - j->p.min_ovlp;
    if (q.rounds <= 0) return EMP_OK;
    const uint64_t ecap0 = j->ctx->tune.edge_cap ? j->ctx->tune.edge_cap : (4 * U > (1u << 20) ? 4 * U : (1u << 20));
    q.ecap = j->ecap_hint ? j->ecap_hint : ecap0;
    return EMP_OK;
}

RoundEnv job_env(emp_job *j) {
    const JobPrep &q = j->prep;
    return RoundEnv{q.L, q.rounds, q.M, q.wpc, j->ctx->tables.as<HashTables>(), j->seq2.as<uint32_t>(), q.wpr};
}

// All rounds of one job, restarting with a larger edge buffer when needed.
emp_status job_rounds(emp_job *j, cudaStream_t s) {
    JobPrep &q = j->prep;
    if (q.rounds <= 0) return EMP_OK;
    const RoundEnv env = job_env(j);
    for (int attempt = 0;; ++attempt) {
        uint64_t needed = 0;
        emp_status rc = run_rounds(j, s, env, q.U, q.ecap, &needed);
        if (rc == EMP_OK) return EMP_OK;
        if (rc != kNeedEdgeRoom || attempt >= 2) return rc == kNeedEdgeRoom ? EMP_E_NOMEM : rc;
        q.ecap = needed + needed / 4 + 1024;
        j->ecap_hint = q.ecap;
        // the round drivers overwrite the list buffers: build the initial list again
        // from the fingerprints and survivor marks, which the rounds leave intact
        EMP_TRY(reset_chain(j, upd_tiles(2 * q.n), s));
        launch_init_list(j->keys0.as<uint64_t>(), j->alive.as<uint8_t>(), q.n, j->lk0.as<uint64_t>(),
                         j->lv0.as<uint32_t>(), j->status.as<uint64_t>(), chain_ctr(j),
                         j->misc.as<uint64_t>() + kMiscU, err_word(j), s);
        launch_dup_prefix_half(j->lk0.as<uint64_t>(), j->lv0.as<uint32_t>(), q.U, s);
    }
}

// Timings and counts of a finished job (after its stream is synchronised).
void job_finish(emp_job *j) {
    emp_stats &st = j->st;
    if (!j->prep.done) {
        st.ms_map = ms_between(j->map_ev[0], j->map_ev[1]);
        st.ms_dedup = ms_between(j->map_ev[1], j->map_ev[2]);
        st.ms_rounds = ms_between(j->map_ev[2], j->map_ev[3]);
    }
    st.ms_total = ms_between(j->map_ev[0], j->map_ev[4]);
    st.output_bytes = j->out.size() + j->dout_bytes;
    st.gpu_launches = g_launches.load() - j->prep.launches0;
    j->have_result = true;
}

emp_status run_job(emp_job *j, cudaStream_t s) {
    EMP_TRY(map_begin(j, s));
    EMP_TRY(map_fetch(j, s));
    EMP_CUDA(cudaStreamSynchronize(s));
    EMP_TRY(map_records(j, s));
    if (!j->prep.done) {
        EMP_TRY(sync_and_check(j, s));
        EMP_TRY(map_keys(j, s));
    }
    if (!j->prep.done) {
        EMP_TRY(sync_and_check(j, s));
        EMP_TRY(map_list(j, s));
        EMP_TRY(job_rounds(j, s));
        cudaEventRecord(j->map_ev[3], s);
        cudaEventRecord(j->map_ev[4], s);
    }
    EMP_TRY(sync_and_check(j, s));
    EMP_CUDA(cudaGetLastError());
    job_finish(j);
    return EMP_OK;
}

// ---- batches -------------------------------------------------------------

// A job's rounds can join a batched bucket launch when all of them fit the
// bucket kernel from round 0: no round could split into several search
// partitions (S, P < M/2) and the list fits the kernel.
bool batch_eligible(const emp_job *j) {
    const JobPrep &q = j->prep;
    return q.rounds > 0 && q.U < q.M / 2 && 2 * q.U <= kBktMaxEntries && bucket_rounds_usable(j->ctx);
}

// The rounds of jobs[idx[..]] (all eligible, lists ready) in one launch of
// the bucket kernel; per-job status in rc.  A job whose edge buffer was too
// small runs its rounds again alone with a larger one.
emp_status batch_rounds(emp_ctx *ctx, emp_job **jobs, const std::vector<int> &idx, std::vector<emp_status> &rc,
                        cudaStream_t s) {
    const size_t nb = idx.size();
    EMP_TRY(ctx_ensure(ctx, ctx->batch_jobs, nb * sizeof(BktJob), s));
    EMP_TRY(ctx_ensure(ctx, ctx->batch_ctl, sizeof(CoopCtl), s));
    if (!ctx->h_batch.ensure(nb * sizeof(BktJob) + sizeof(CoopCtl))) return EMP_E_NOMEM;
    if (!ctx->batch_ev[0]) {
        for (auto &e : ctx->batch_ev) EMP_CUDA(cudaEventCreate(&e));
    }
    BktJob *hj = ctx->h_batch.as<BktJob>();
    CoopCtl *hc = reinterpret_cast<CoopCtl *>(hj + nb);
    for (size_t k = 0; k < nb; ++k) {
        emp_job *j = jobs[idx[k]];
        const JobPrep &q = j->prep;
        EMP_TRY(rounds_prelude(j, s));
        EMP_TRY(bucket_prepare(j, s, job_env(j), 0, 0, 2 * q.U, q.ecap, 1u, &hj[k]));
    }
    coop_ctl_init(ctx, hc, (uint32_t)nb);
    EMP_CUDA(cudaMemcpyAsync(ctx->batch_jobs.p, hj, nb * sizeof(BktJob), cudaMemcpyHostToDevice, s));
    EMP_CUDA(cudaMemcpyAsync(ctx->batch_ctl.p, hc, sizeof(CoopCtl), cudaMemcpyHostToDevice, s));
    EMP_CUDA(cudaEventRecord(ctx->batch_ev[0], s));
    EMP_CUDA(launch_bucket_rounds(ctx->batch_jobs.as<BktJob>(), ctx->batch_ctl.as<CoopCtl>(),
                                  err_word(jobs[idx[0]]), s));
    EMP_CUDA(cudaEventRecord(ctx->batch_ev[1], s));
    EMP_CUDA(cudaMemcpyAsync(hj, ctx->batch_jobs.p, nb * sizeof(BktJob), cudaMemcpyDeviceToHost, s));
    EMP_CUDA(cudaMemcpyAsync(hc, ctx->batch_ctl.p, sizeof(CoopCtl), cudaMemcpyDeviceToHost, s));
    for (size_t k = 0; k < nb; ++k) EMP_TRY(bucket_fetch(jobs[idx[k]], job_env(jobs[idx[k]]), s));
    EMP_CUDA(cudaStreamSynchronize(s));
    if (hc->err & kErrSpin) return EMP_E_TIMEOUT;
    const float ms = ms_between(ctx->batch_ev[0], ctx->batch_ev[1]);
    for (size_t k = 0; k < nb; ++k) {
        emp_job *j = jobs[idx[k]];
        JobPrep &q = j->prep;
        j->st.ms_round_kernel += ms;  // the whole batch's launch
        uint64_t needed = 0;
        emp_status r = bucket_collect(j, 0, 2 * q.U, hj[k], &needed);
        if (r == kNeedEdgeRoom) {  // alone again, with room for every edge
            q.ecap = needed + needed / 4 + 1024;
            j->ecap_hint = q.ecap;
            r = job_rounds(j, s);
        }
        rc[idx[k]] = r;
    }
    return EMP_OK;
}

// The map phase of jobs[0..n) with one stream synchronisation per stage for
// all of them; a job that fails gets its status in rc.  Jobs left with rc
// EMP_OK and prep.done unset have their lists ready for the rounds.
emp_status map_batch(emp_job **jobs, int n, std::vector<emp_status> &rc, cudaStream_t s) {
    auto live = [&](int i) { return rc[i] == EMP_OK && !jobs[i]->prep.done; };
    auto fail = [&](int i, emp_status e) {
        if (rc[i] == EMP_OK) rc[i] = e;
    };
    // job i on stream i mod K (K = 1: s itself), every stream after s's work so far
    emp_ctx *ctx = n ? jobs[0]->ctx : nullptr;
    const int want = ctx && ctx->tune.map_streams ? (int)ctx->tune.map_streams : kMapStreamsDefault;
    const int K = n > 1 ? std::min(n, want) : 1;
    std::vector<cudaStream_t> st((size_t)K, s);
    if (K > 1) {
        for (int k = 0; k <= kMapStreams; ++k)
            if (!ctx->map_ev[k]) EMP_CUDA(cudaEventCreateWithFlags(&ctx->map_ev[k], cudaEventDisableTiming));
        EMP_CUDA(cudaEventRecord(ctx->map_ev[kMapStreams], s));  // the last event: the start of the phase
        for (int k = 0; k < K; ++k) {
            if (!ctx->map_streams[k]) EMP_CUDA(cudaStreamCreateWithFlags(&ctx->map_streams[k], cudaStreamNonBlocking));
            st[k] = ctx->map_streams[k];
            EMP_CUDA(cudaStreamWaitEvent(st[k], ctx->map_ev[kMapStreams], 0));
        }
    }
    auto sync_all = [&]() -> emp_status {
        for (cudaStream_t q : st) EMP_CUDA(cudaStreamSynchronize(q));
        return EMP_OK;
    };
    // largest jobs first, each to the stream with the fewest FASTQ bytes so
    // far (so that no stream ends a stage long after the others)
    std::vector<int> order((size_t)n), sid((size_t)n, 0);
    for (int i = 0; i < n; ++i) order[(size_t)i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return jobs[a]->F > jobs[b]->F; });
    {
        std::vector<uint64_t> load((size_t)K, 0);
        for (int i : order) {
            const int k = (int)(std::min_element(load.begin(), load.end()) - load.begin());
            sid[(size_t)i] = k;
            load[(size_t)k] += jobs[i]->F + 4096;
        }
    }
    auto stages = [&]() -> emp_status {
        for (int i : order) {
            fail(i, map_begin(jobs[i], st[sid[i]]));
            if (rc[i] == EMP_OK) fail(i, map_fetch(jobs[i], st[sid[i]]));
        }
        EMP_TRY(sync_all());
        for (int i : order) {
            if (!live(i)) continue;
            fail(i, map_records(jobs[i], st[sid[i]]));
            if (live(i)) fail(i, map_fetch(jobs[i], st[sid[i]]));
        }
        EMP_TRY(sync_all());
        for (int i : order) {
            if (!live(i)) continue;
            fail(i, map_keys(jobs[i], st[sid[i]]));
            if (live(i)) fail(i, map_fetch(jobs[i], st[sid[i]]));
        }
        EMP_TRY(sync_all());
        for (int i : order)
            if (live(i)) fail(i, map_list(jobs[i], st[sid[i]]));
        return EMP_OK;
    };
    const emp_status e = stages();
    if (K > 1) {  // the rest of the jobs' work (and any error path) is on s, after all of this
        for (int k = 0; k < K; ++k) {
            cudaEventRecord(ctx->map_ev[k], st[k]);
            cudaStreamWaitEvent(s, ctx->map_ev[k], 0);
        }
        for (int i = 0; i < n; ++i) jobs[i]->stream = s;
    }
    return e;
}

// Close jobs[0..n) whose work is all queued: their last events, one
// synchronisation, then results (rc[i] == EMP_OK) or none.  Sets each job's
// last_rc; returns the first failure.
emp_status close_jobs(emp_job **jobs, int n, std::vector<emp_status> &rc, cudaStream_t s) {
    for (int i = 0; i < n; ++i) {
        if (rc[i] != EMP_OK) continue;
        if (!jobs[i]->prep.done) {
            cudaEventRecord(jobs[i]->map_ev[3], s);
            cudaEventRecord(jobs[i]->map_ev[4], s);
        }
        rc[i] = map_fetch(jobs[i], s);
    }
    EMP_CUDA(cudaStreamSynchronize(s));
    EMP_CUDA(cudaGetLastError());
    emp_status first = EMP_OK;
    for (int i = 0; i < n; ++i) {
        if (rc[i] == EMP_OK) rc[i] = map_check(jobs[i]);
        if (rc[i] == EMP_OK) {
            job_finish(jobs[i]);
        } else {
            jobs[i]->have_result = false;
            if (first == EMP_OK) first = rc[i];
        }
        jobs[i]->last_rc = rc[i];
    }
    return first;
}

// Every job of a batch through the map phase, the rounds of the eligible
// ones in one bucket-kernel launch, the others' rounds one job after another.
emp_status run_batch(emp_ctx *ctx, emp_job **jobs, int n, cudaStream_t s) {
    std::vector<emp_status> rc((size_t)n, EMP_OK);
    EMP_TRY(map_batch(jobs, n, rc, s));
    std::vector<int> batch, alone;
    for (int i = 0; i < n; ++i) {
        if (rc[i] != EMP_OK || jobs[i]->prep.done) continue;
        if (batch_eligible(jobs[i])) batch.push_back(i);
        else alone.push_back(i);
    }
    if (!batch.empty()) {
        const emp_status e = batch_rounds(ctx, jobs, batch, rc, s);
        if (e != EMP_OK)
            for (int i : batch)
                if (rc[i] == EMP_OK) rc[i] = e;
    }
    for (int i : alone) rc[i] = job_rounds(jobs[i], s);
    return close_jobs(jobs, n, rc, s);
}

// ---- served jobs -----------------------------------------------------------

// Device footprint assumed for a queued job before its reads are known
// (admission): the FASTQ, about 400 B of tables and lists per read at
// 100+ bases per read (so 3 B per FASTQ byte), and the fixed minimum of the
// edge and output buffers.
uint64_t served_footprint(uint64_t F) { return 4 * F + (64ull << 20); }

}  // namespace

struct emp_server {
    emp_ctx *ctx = nullptr;
    emp_server_params p{};
    std::deque<emp_job *> queue;     // submitted, not yet admitted
    std::vector<emp_job *> live;     // in the bucket-kernel batch
    std::vector<emp_job *> finished; // completed, not yet handed out
    uint64_t admitted = 0;           // footprint estimates of the admitted jobs
    DevBuf d_jobs, d_ctl;
    PinnedBuf h_jobs;
    cudaEvent_t ev[2] = {};
    emp_server_stats st{};
};

namespace {

// a finished job waits in `finished` (still held by the server) until a step hands it out
void server_complete(emp_server *srv, emp_job *j) {
    srv->admitted -= j->admit_est;
    j->admit_est = 0;
    srv->finished.push_back(j);
}

// One step: the launch of at most rounds_per_launch rounds of every job in
// the batch goes first, so that the FASTQ copies of newly admitted jobs run
// beside it; then the admitted jobs' map phase (queued behind the launch),
// the eligible ones joining the batch for the next step and the others run
// alone; then the launch's results: jobs with no round left complete.
emp_status server_step(emp_server *srv, cudaStream_t s) {
    emp_ctx *ctx = srv->ctx;
    emp_server_stats &ss = srv->st;
    ss.steps += 1;
    const auto ts = std::chrono::steady_clock::now();
    const uint64_t budget = srv->p.hbm_budget_bytes ? srv->p.hbm_budget_bytes : ctx->budget;
    std::vector<emp_job *> adm;
    while (!srv->queue.empty() && (int)(srv->live.size() + adm.size()) < srv->p.max_jobs) {
        emp_job *j = srv->queue.front();
        const uint64_t est = served_footprint(j->F);
        if (budget && srv->admitted + est > budget && !(srv->live.empty() && adm.empty())) break;
        srv->queue.pop_front();
        srv->admitted += est;
        j->admit_est = est;
        adm.push_back(j);
    }
    // ---- the launch (not waited for yet)
    const size_t nb = srv->live.size();
    BktJob *hj = nullptr;
    CoopCtl *hc = nullptr;
    if (nb) {
        EMP_TRY(ctx_ensure(ctx, srv->d_jobs, nb * sizeof(BktJob), s));
        EMP_TRY(ctx_ensure(ctx, srv->d_ctl, sizeof(CoopCtl), s));
        if (!srv->h_jobs.ensure(nb * sizeof(BktJob) + sizeof(CoopCtl))) return EMP_E_NOMEM;
        if (!srv->ev[0]) {
            for (auto &e : srv->ev) EMP_CUDA(cudaEventCreate(&e));
        }
        hj = srv->h_jobs.as<BktJob>();
        hc = reinterpret_cast<CoopCtl *>(hj + nb);
        // Per-job shares of the launch's iterations: a large job runs a few
        // rounds (short launches while jobs wait to join, long ones when none
        // does); a small one all its rounds, which after the large jobs' share
        // cost a few microseconds each, so it leaves in the launch it joins.
        const uint32_t share = (uint32_t)(srv->queue.empty() && adm.empty() ? srv->p.rounds_per_launch_idle
                                                                             : srv->p.rounds_per_launch);
        bool any_unlimited = false;
        for (size_t k = 0; k < nb; ++k) {
            hj[k] = srv->live[k]->bk;
            const bool large = !srv->p.share_min_entries || 2 * srv->live[k]->prep.U >= srv->p.share_min_entries;
            hj[k].iter_share = large ? share : 0u;
            any_unlimited |= !large;
        }
        coop_ctl_init(ctx, hc, (uint32_t)nb);
        hc->iter_cap = any_unlimited ? 0u : share;
        EMP_CUDA(cudaMemcpyAsync(srv->d_jobs.p, hj, nb * sizeof(BktJob), cudaMemcpyHostToDevice, s));
        EMP_CUDA(cudaMemcpyAsync(srv->d_ctl.p, hc, sizeof(CoopCtl), cudaMemcpyHostToDevice, s));
        EMP_CUDA(cudaEventRecord(srv->ev[0], s));
        EMP_CUDA(launch_bucket_rounds(srv->d_jobs.as<BktJob>(), srv->d_ctl.as<CoopCtl>(), err_word(srv->live[0]), s));
        EMP_CUDA(cudaEventRecord(srv->ev[1], s));
        EMP_CUDA(cudaMemcpyAsync(hj, srv->d_jobs.p, nb * sizeof(BktJob), cudaMemcpyDeviceToHost, s));
        EMP_CUDA(cudaMemcpyAsync(hc, srv->d_ctl.p, sizeof(CoopCtl), cudaMemcpyDeviceToHost, s));
    }
    ss.ms_launch += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - ts).count();
    // ---- the admitted jobs' map phase
    std::vector<emp_job *> joining;
    if (!adm.empty()) {
        const auto t0 = std::chrono::steady_clock::now();
        const int n = (int)adm.size();
        std::vector<emp_status> rc((size_t)n, EMP_OK);
        EMP_TRY(map_batch(adm.data(), n, rc, s));
        const auto t1 = std::chrono::steady_clock::now();
        ss.ms_map += std::chrono::duration<double, std::milli>(t1 - t0).count();
        std::vector<emp_job *> close;
        std::vector<emp_status> crc;
        // a lone job in an idle server (nothing in flight, nothing queued)
        // runs alone, as emp_job_run runs it: one launch for all its rounds
        const bool solo = nb == 0 && n == 1 && srv->queue.empty();
        for (int i = 0; i < n; ++i) {
            emp_job *j = adm[i];
            JobPrep &q = j->prep;
            const bool fits = !srv->p.batch_max_entries || 2 * q.U <= srv->p.batch_max_entries;
            if (rc[i] == EMP_OK && !q.done && batch_eligible(j) && fits && !solo) {
                rc[i] = rounds_prelude(j, s);
                if (rc[i] == EMP_OK) rc[i] = bucket_prepare(j, s, job_env(j), 0, 0, 2 * q.U, q.ecap, 1u, &j->bk);
                if (rc[i] == EMP_OK) {
                    joining.push_back(j);
                    continue;
                }
            } else if (rc[i] == EMP_OK && !q.done) {
                const auto ta = std::chrono::steady_clock::now();
                rc[i] = job_rounds(j, s);  // too large for the batch, rounds that split, or solo: alone
                ss.alone += 1;
                ss.ms_alone += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - ta).count();
            }
            close.push_back(j);
            crc.push_back(rc[i]);
        }
        if (!close.empty()) {
            close_jobs(close.data(), (int)close.size(), crc, s);
            for (emp_job *j : close) server_complete(srv, j);
        }
        ss.admitted += (uint64_t)n;
        ss.ms_admit += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    if (!nb) {
        srv->live.swap(joining);
        return EMP_OK;
    }
    // ---- the launch's results
    const auto tw = std::chrono::steady_clock::now();
    EMP_CUDA(cudaStreamSynchronize(s));
    const auto tr = std::chrono::steady_clock::now();
    ss.ms_wait += std::chrono::duration<double, std::milli>(tr - tw).count();
    struct ResultClock {
        double &acc;
        std::chrono::steady_clock::time_point t;
        ~ResultClock() { acc += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t).count(); }
    } result_clock{ss.ms_results, tr};
    const bool timed_out = (hc->err & kErrSpin) != 0;
    const float ms = ms_between(srv->ev[0], srv->ev[1]);
    ss.launches += 1;
    ss.rounds += hc->iters;
    ss.batch_jobs += nb;
    ss.ms_kernel += ms;
    std::vector<emp_job *> still, done;
    for (size_t k = 0; k < nb; ++k) {
        emp_job *j = srv->live[k];
        j->bk = hj[k];
        j->st.ms_round_kernel += ms;  // every launch the job took part in
        if (timed_out || j->bk.done) {
            done.push_back(j);
            if (!timed_out) EMP_TRY(bucket_fetch(j, job_env(j), s));
        } else {
            const uint32_t sh = j->bk.iter_share;
            j->bk.iter0 += sh && sh < hc->iters ? sh : hc->iters;  // the iterations it ran
            still.push_back(j);
        }
    }
    still.insert(still.end(), joining.begin(), joining.end());
    srv->live.swap(still);
    if (done.empty()) return EMP_OK;
    EMP_CUDA(cudaStreamSynchronize(s));
    std::vector<emp_status> rc(done.size(), timed_out ? EMP_E_TIMEOUT : EMP_OK);
    for (size_t k = 0; k < done.size() && !timed_out; ++k) {
        emp_job *j = done[k];
        JobPrep &q = j->prep;
        uint64_t needed = 0;
        rc[k] = bucket_collect(j, 0, 2 * q.U, j->bk, &needed);
        if (rc[k] == kNeedEdgeRoom) {  // alone again, with room for every edge
            q.ecap = needed + needed / 4 + 1024;
            j->ecap_hint = q.ecap;
            rc[k] = job_rounds(j, s);
        }
    }
    close_jobs(done.data(), (int)done.size(), rc, s);
    for (emp_job *j : done) server_complete(srv, j);
    return timed_out ? EMP_E_TIMEOUT : EMP_OK;
}

}  // namespace

// =========================================================================
// C ABI
// =========================================================================
extern "C" {

const char *emp_status_string(emp_status st) {
    switch (st) {
    case EMP_OK: return "ok";
    case EMP_E_INVAL: return "invalid argument";
    case EMP_E_NOMEM: return "out of memory or over the HBM budget";
    case EMP_E_CUDA: return "CUDA error";
    case EMP_E_TIMEOUT: return "bounded device wait timed out";
    case EMP_E_FORMAT: return "reads of unequal length or a base outside ACGTacgt";
    case EMP_E_STATE: return "call out of order";
    case EMP_E_IO: return "file could not be read or written";
    case EMP_E_UNSUPPORTED: return "unsupported input";
    case EMP_E_HANG: return "input on which the reference never terminates";
    default: return "unknown status";
    }
}

int emp_abi_version(void) { return EMP_ABI_VERSION; }

emp_status emp_params_default(emp_params *p) {
    if (!p) return EMP_E_INVAL;
    p->min_ovlp = 31;
    p->map_mem = 1ull << 30;
    p->reduce_mem = 1ull << 30;
    p->base_blocksz = 32ull << 20;
    p->kv_chunksz = 64ull << 20;
    return EMP_OK;
}

emp_status emp_parse_size(const char *s, uint64_t *bytes) {
    if (!s || !bytes || !*s) return EMP_E_INVAL;
    std::string h(s);
    const char unit = h.back();
    int shift = 0;
    emp_status st = EMP_OK;
    if (!(unit >= '0' && unit <= '9')) {
        h.pop_back();
        switch (unit) {
        case 'k': case 'K': shift = 10; break;
        case 'm': case 'M': shift = 20; break;
        case 'g': case 'G': shift = 30; break;
        default: st = EMP_E_INVAL; break;  // reference: LOG_ERR, value without the suffix
        }
    }
    if (h.empty() || !(h[0] >= '0' && h[0] <= '9') ) {
        // std::stoul accepts leading blanks and a sign; anything else throws
        size_t k = 0;
        while (k < h.size() && (h[k] == ' ' || h[k] == '\t')) ++k;
        if (k >= h.size() || !((h[k] >= '0' && h[k] <= '9') || h[k] == '+' || h[k] == '-')) return EMP_E_INVAL;
    }
    errno = 0;
    char *end = nullptr;
    unsigned long long v = std::strtoull(h.c_str(), &end, 10);
    if (end == h.c_str() || errno == ERANGE) return EMP_E_INVAL;
    *bytes = (uint64_t)v << shift;
    return st;
}

emp_status emp_tuning_default(emp_tuning *t) {
    if (!t) return EMP_E_INVAL;
    std::memset(t, 0, sizeof *t);
    t->bucket_mean = kBktMean;
    t->region_cap = kBktRegionCap;
    t->map_streams = kMapStreamsDefault;
    t->wait_limit_ns = kBarrierTimeoutNs;
    return EMP_OK;
}

emp_status emp_ctx_set_tuning(emp_ctx *ctx, const emp_tuning *t) {
    if (!ctx || !t) return EMP_E_INVAL;
    if (t->round_driver < 0 || t->round_driver > 1 || t->dedup_driver < 0 || t->dedup_driver > 1) return EMP_E_INVAL;
    if (t->bucket_mean && (t->bucket_mean < kBktMeanMin || t->bucket_mean > kBktMeanMax)) return EMP_E_INVAL;
    if (t->region_cap > kBktRegionCap || t->map_streams > (uint32_t)kMapStreams) return EMP_E_INVAL;
    ctx->tune = *t;
    return EMP_OK;
}

emp_status emp_ctx_get_tuning(emp_ctx *ctx, emp_tuning *t) {
    if (!ctx || !t) return EMP_E_INVAL;
    emp_tuning_default(t);
    const emp_tuning &c = ctx->tune;
    t->round_driver = c.round_driver;
    t->dedup_driver = c.dedup_driver;
    if (c.bucket_mean) t->bucket_mean = c.bucket_mean;
    if (c.region_cap) t->region_cap = c.region_cap;
    if (c.map_streams) t->map_streams = c.map_streams;
    t->edge_cap = c.edge_cap;
    if (c.wait_limit_ns) t->wait_limit_ns = c.wait_limit_ns;
    t->block_next_wait = c.block_next_wait;
    return EMP_OK;
}

emp_status emp_ctx_create(int device, uint64_t hbm_budget_bytes, emp_ctx **out) {
    if (!out) return EMP_E_INVAL;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return EMP_E_CUDA;
    }
    if (device < 0) {
        if (cudaGetDevice(&device) != cudaSuccess) return EMP_E_CUDA;
    }
    if (device >= ndev) return EMP_E_INVAL;
    if (cudaSetDevice(device) != cudaSuccess) return EMP_E_CUDA;
    emp_ctx *c = new (std::nothrow) emp_ctx();
    if (!c) return EMP_E_NOMEM;
    c->device = device;
    c->budget = hbm_budget_bytes;
    if (const char *t = std::getenv("EMP_COOP_TRACE")) c->trace_path = t;
    if (const char *t = std::getenv("EMP_COOP_PROBE")) c->probe_spec = t;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return EMP_E_CUDA;
    }
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    if (cudaMemPoolCreate(&c->pool, &props) != cudaSuccess) {
        cudaGetLastError();
        cudaStreamDestroy(c->stream);
        delete c;
        return EMP_E_CUDA;
    }
    uint64_t keep = ~0ull;  // keep freed memory in the pool
    cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    if (cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaStreamDestroy(c->stream);
        cudaMemPoolDestroy(c->pool);
        delete c;
        return EMP_E_CUDA;
    }
    void *p = nullptr;
    struct {  // HashTables, then the read pass's ChunkWeights
        HashTables h;
        ChunkWeights w;
    } tabs;
    static_assert(sizeof(HashTables) % 16 == 0, "the weights start 16-byte aligned");
    if (cudaMalloc(&p, sizeof tabs) != cudaSuccess) {
        cudaStreamDestroy(c->stream);
        cudaMemPoolDestroy(c->pool);
        delete c;
        return EMP_E_NOMEM;
    }
    c->tables.p = p;
    c->tables.bytes = sizeof tabs;
    host_tables(tabs.h, tabs.w);
    if (cudaMemcpy(p, &tabs, sizeof tabs, cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaStreamDestroy(c->stream);
        cudaMemPoolDestroy(c->pool);
        delete c;
        return EMP_E_CUDA;
    }
    *out = c;
    return EMP_OK;
}

emp_status emp_ctx_destroy(emp_ctx *ctx) {
    if (!ctx) return EMP_E_INVAL;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (auto &e : ctx->batch_ev)
        if (e) cudaEventDestroy(e);
    ctx->in_use -= ctx->batch_jobs.bytes + ctx->batch_ctl.bytes;
    ctx->batch_jobs.release();
    ctx->batch_ctl.release();
    for (int k = 0; k < kMapStreams; ++k) {
        if (ctx->map_streams[k]) {
            cudaStreamSynchronize(ctx->map_streams[k]);
            cudaStreamDestroy(ctx->map_streams[k]);
        }
    }
    for (auto &e : ctx->map_ev)
        if (e) cudaEventDestroy(e);
    cudaStreamSynchronize(ctx->stream);
    cudaStreamDestroy(ctx->stream);
    cudaStreamSynchronize(ctx->copy_stream);
    cudaStreamDestroy(ctx->copy_stream);
    if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
    delete ctx;
    return EMP_OK;
}

emp_status emp_job_create(emp_ctx *ctx, const emp_params *p, emp_job **out) {
    if (!ctx || !out) return EMP_E_INVAL;
    emp_job *j = new (std::nothrow) emp_job();
    if (!j) return EMP_E_NOMEM;
    j->ctx = ctx;
    if (p) j->p = *p;
    else emp_params_default(&j->p);
    cudaSetDevice(ctx->device);
    for (auto &e : j->sort_ev) {
        if (cudaEventCreate(&e) != cudaSuccess) {
            emp_job_destroy(j);
            return EMP_E_CUDA;
        }
    }
    for (auto &e : j->map_ev) {
        if (cudaEventCreate(&e) != cudaSuccess) {
            emp_job_destroy(j);
            return EMP_E_CUDA;
        }
    }
    static_assert(kSlotHist >= kMiscSlots * sizeof(uint64_t) && kSlotCoop - kSlotHist >= kSortPasses * kSortRadix * 4,
                  "slab layout");
    static_assert(kSlotCtl - kSlotCoop >= sizeof(BktJob) + sizeof(CoopCtl),
                  "slab layout");
    static_assert(kSlotBytes - kSlotRecords >= EMP_MAX_ROUNDS * sizeof(RoundRecord),
                  "slab layout");
    j->slot = ctx->slab.take();
    if (!j->slot) {
        emp_job_destroy(j);
        return EMP_E_NOMEM;
    }
    uint8_t *sl = static_cast<uint8_t *>(j->slot);
    j->h_misc.bind(sl + kSlotMisc, kSlotHist - kSlotMisc);
    j->h_hist.bind(sl + kSlotHist, kSlotCoop - kSlotHist);
    j->h_coop.bind(sl + kSlotCoop, kSlotCtl - kSlotCoop);
    j->h_records.bind(sl + kSlotRecords, kSlotBytes - kSlotRecords);
    *out = j;
    return EMP_OK;
}

static void release_buffers(emp_job *job);

emp_status emp_job_trim(emp_job *job) {
    if (!job) return EMP_E_INVAL;
    if (job->server) return EMP_E_STATE;
    cudaSetDevice(job->ctx->device);
    cudaStreamSynchronize(job->ctx->stream);
    if (job->feed_pending) cudaEventSynchronize(job->feed_ev[1]);
    job->feed_pending = false;
    release_buffers(job);
    job->F = 0;
    job->fed_last = false;
    job->ms_h2d = 0.0;
    job->have_result = false;
    job->out.clear();
    job->dout_bytes = 0;
    job->n_ends = 0;
    job->last_rc = EMP_E_STATE;
    return EMP_OK;
}

emp_status emp_job_destroy(emp_job *job) {
    if (!job) return EMP_E_INVAL;
    if (job->server) return EMP_E_STATE;
    cudaSetDevice(job->ctx->device);
    cudaStreamSynchronize(job->ctx->stream);
    if (job->feed_pending) cudaEventSynchronize(job->feed_ev[1]);
    for (auto &e : job->feed_ev)
        if (e) cudaEventDestroy(e);
    release_buffers(job);
    for (auto &e : job->sort_ev)
        if (e) cudaEventDestroy(e);
    for (auto &e : job->upd_ev)
        if (e) cudaEventDestroy(e);
    for (auto &e : job->map_ev)
        if (e) cudaEventDestroy(e);
    if (job->slot) {
        job->h_misc.drop();
        job->h_hist.drop();
        job->h_coop.drop();
        job->h_records.drop();
        job->ctx->slab.give(job->slot);
    }
    delete job;
    return EMP_OK;
}

// every device buffer of the job back to the context (its pool)
static void release_buffers(emp_job *job) {
    DevBuf *bufs[] = {&job->fq, &job->tile_counts, &job->tile_excl, &job->status, &job->misc, &job->keys0,
                      &job->keep, &job->keys_tmp, &job->seq2_tmp, &job->dedup_scr, &job->cols, &job->seq2, &job->sk0, &job->sv0, &job->sk1, &job->sv1, &job->alive, &job->lk0, &job->lv0, &job->lk1, &job->lv1,
                      &job->used_s, &job->used_p, &job->cnt, &job->offs, &job->efrom, &job->eto,
                      &job->sort_scratch, &job->akeys, &job->apos, &job->bkeys, &job->parts, &job->records, &job->coop_ctl, &job->coop_trace,
                      &job->coop_probe, &job->bk_lst0, &job->bk_lst1, &job->bk_cnt, &job->bk_spill, &job->bk_spans,
                      &job->bk_sfrom, &job->bk_sto, &job->bk_scratch, &job->bk_job, &job->dout,
                      &job->bk_meta, &job->xk0, &job->xv0, &job->xk1, &job->xv1, &job->ring_k, &job->ring_v,
                      &job->cparts};
    for (DevBuf *b : bufs) free_buf(job, *b);
    job->sorts_since_clear = 0;
}

emp_status emp_job_reserve(emp_job *job, uint64_t bytes) {
    if (!job) return EMP_E_INVAL;
    if (job->server) return EMP_E_STATE;
    if (bytes <= job->fq.bytes) return EMP_OK;
    cudaSetDevice(job->ctx->device);
    if (job->feed_pending && cudaEventSynchronize(job->feed_ev[1]) != cudaSuccess) return EMP_E_CUDA;
    DevBuf nb;
    emp_ctx *c = job->ctx;
    if (c->budget && c->in_use + bytes > c->budget) return EMP_E_NOMEM;
    if (cudaMallocFromPoolAsync(&nb.p, bytes + 16, c->pool, c->stream) != cudaSuccess) {
        cudaGetLastError();
        return EMP_E_NOMEM;
    }
    nb.bytes = bytes + 16;
    nb.pooled = true;
    nb.pool_stream = c->stream;
    c->in_use += nb.bytes;
    if (job->F && cudaMemcpyAsync(nb.p, job->fq.p, job->F, cudaMemcpyDeviceToDevice, c->stream) != cudaSuccess)
        return EMP_E_CUDA;
    free_buf(job, job->fq);
    job->fq.p = nb.p;
    job->fq.bytes = nb.bytes;
    job->fq.pooled = true;
    job->fq.pool_stream = c->stream;
    nb.p = nullptr;
    nb.bytes = 0;
    nb.pooled = false;
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return EMP_E_CUDA;
    return EMP_OK;
}

emp_status emp_job_reset(emp_job *job) {
    if (!job) return EMP_E_INVAL;
    if (job->server) return EMP_E_STATE;
    cudaSetDevice(job->ctx->device);
    cudaStreamSynchronize(job->ctx->stream);
    if (job->feed_pending) cudaEventSynchronize(job->feed_ev[1]);
    job->feed_pending = false;
    job->F = 0;
    job->fed_last = false;
    job->ms_h2d = 0.0;
    job->out.clear();
    job->dout_bytes = 0;
    job->have_result = false;
    job->n_ends = 0;
    return EMP_OK;
}

static emp_status feed(emp_job *job, const void *src, uint64_t n, int last, cudaMemcpyKind kind) {
    if (!job || (n && !src)) return EMP_E_INVAL;
    if (job->server) return EMP_E_STATE;
    if (job->fed_last) return EMP_E_STATE;
    cudaSetDevice(job->ctx->device);
    if (job->feed_pending) {
        if (cudaEventSynchronize(job->feed_ev[1]) != cudaSuccess) return EMP_E_CUDA;
        job->ms_h2d += ms_between(job->feed_ev[0], job->feed_ev[1]);
        job->feed_pending = false;
    }
    if (job->F + n > job->fq.bytes) {
        uint64_t want = job->F + n;
        if (!last) want += want / 2;
        EMP_TRY(emp_job_reserve(job, want));
    }
    if (n) {
        cudaEvent_t a = nullptr, b = nullptr;
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        cudaEventRecord(a, job->ctx->stream);
        cudaError_t e = cudaMemcpyAsync(job->fq.as<uint8_t>() + job->F, src, n, kind, job->ctx->stream);
        cudaEventRecord(b, job->ctx->stream);
        cudaError_t e2 = cudaStreamSynchronize(job->ctx->stream);
        if (kind == cudaMemcpyHostToDevice) job->ms_h2d += ms_between(a, b);
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        if (e != cudaSuccess || e2 != cudaSuccess) return EMP_E_CUDA;
        job->F += n;
    }
    if (last) job->fed_last = true;
    return EMP_OK;
}

emp_status emp_job_feed_fastq(emp_job *job, const char *bytes, uint64_t n, int last) {
    return feed(job, bytes, n, last, cudaMemcpyHostToDevice);
}

emp_status emp_job_feed_fastq_async(emp_job *job, const char *bytes, uint64_t n, int last) {
    if (!job || (n && !bytes)) return EMP_E_INVAL;
    if (job->server) return EMP_E_STATE;
    if (job->fed_last) return EMP_E_STATE;
    cudaSetDevice(job->ctx->device);
    emp_ctx *c = job->ctx;
    cudaStream_t cs = c->copy_stream;
    if (!job->feed_ev[0]) {
        for (auto &e : job->feed_ev) EMP_CUDA(cudaEventCreate(&e));
    }
    if (!job->feed_pending) EMP_CUDA(cudaEventRecord(job->feed_ev[0], cs));
    if (job->F + n > job->fq.bytes) {  // grow in the copy stream's order
        uint64_t want = job->F + n;
        if (!last) want += want / 2;
        if (c->budget && c->in_use - job->fq.bytes + want + 16 > c->budget) return EMP_E_NOMEM;
        void *p = nullptr;
        if (cudaMallocFromPoolAsync(&p, want + 16, c->pool, cs) != cudaSuccess) {
            cudaGetLastError();
            return EMP_E_NOMEM;
        }
        if (job->F) EMP_CUDA(cudaMemcpyAsync(p, job->fq.p, job->F, cudaMemcpyDeviceToDevice, cs));
        if (job->fq.p) {
            if (job->fq.pooled) cudaFreeAsync(job->fq.p, cs);
            else {
                cudaStreamSynchronize(cs);
                cudaFree(job->fq.p);
            }
        }
        c->in_use += want + 16 - job->fq.bytes;
        job->fq.p = p;
        job->fq.bytes = want + 16;
        job->fq.pooled = true;
        job->fq.pool_stream = c->stream;
    }
    if (n) EMP_CUDA(cudaMemcpyAsync(job->fq.as<uint8_t>() + job->F, bytes, n, cudaMemcpyHostToDevice, cs));
    EMP_CUDA(cudaEventRecord(job->feed_ev[1], cs));
    job->feed_pending = true;
    job->F += n;
    if (last) job->fed_last = true;
    return EMP_OK;
}

emp_status emp_job_feed_fastq_device(emp_job *job, const void *dev_bytes, uint64_t n, int last) {
    return feed(job, dev_bytes, n, last, cudaMemcpyDeviceToDevice);
}

emp_status emp_job_run(emp_job *job, void *stream) {
    if (!job) return EMP_E_INVAL;
    if (cudaSetDevice(job->ctx->device) != cudaSuccess) return EMP_E_CUDA;
    if (job->server) return EMP_E_STATE;
    cudaStream_t s = stream ? reinterpret_cast<cudaStream_t>(stream) : job->ctx->stream;
    emp_status st = run_job(job, s);
    if (st != EMP_OK) {
        cudaStreamSynchronize(s);
        cudaGetLastError();
        job->have_result = false;
    }
    job->last_rc = st;
    return st;
}

emp_status emp_batch_run(emp_ctx *ctx, emp_job **jobs, int njobs, void *stream) {
    if (!ctx || njobs < 0 || (njobs && !jobs) || njobs > kCoopMaxJobs) return EMP_E_INVAL;
    for (int i = 0; i < njobs; ++i) {
        if (!jobs[i] || jobs[i]->ctx != ctx || jobs[i]->server) return EMP_E_INVAL;
        for (int k = 0; k < i; ++k)
            if (jobs[k] == jobs[i]) return EMP_E_INVAL;
    }
    if (!njobs) return EMP_OK;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return EMP_E_CUDA;
    cudaStream_t s = stream ? reinterpret_cast<cudaStream_t>(stream) : ctx->stream;
    emp_status st = run_batch(ctx, jobs, njobs, s);
    if (st != EMP_OK) {
        cudaStreamSynchronize(s);
        cudaGetLastError();
    }
    return st;
}

emp_status emp_job_status(emp_job *job) { return job ? job->last_rc : EMP_E_INVAL; }

emp_status emp_server_params_default(emp_server_params *p) {
    if (!p) return EMP_E_INVAL;
    p->rounds_per_launch = 16;
    p->max_jobs = 256;
    p->hbm_budget_bytes = 0;
    p->rounds_per_launch_idle = 64;
    p->batch_max_entries = 0;
    p->share_min_entries = 8000000;
    return EMP_OK;
}

emp_status emp_server_create(emp_ctx *ctx, const emp_server_params *p, emp_server **out) {
    if (!ctx || !out) return EMP_E_INVAL;
    *out = nullptr;
    emp_server_params q;
    if (p) q = *p;
    else emp_server_params_default(&q);
    if (q.rounds_per_launch < 1 || q.rounds_per_launch_idle < 1 || q.max_jobs < 1 || q.max_jobs > kCoopMaxJobs)
        return EMP_E_INVAL;
    emp_server *srv = new (std::nothrow) emp_server();
    if (!srv) return EMP_E_NOMEM;
    srv->ctx = ctx;
    srv->p = q;
    // launch descriptors for max_jobs up front: growing them later would free
    // pinned memory, which waits for the device, in the middle of a step
    cudaSetDevice(ctx->device);
    const size_t desc = (size_t)q.max_jobs * sizeof(BktJob);
    emp_status st = srv->h_jobs.ensure(desc + sizeof(CoopCtl)) ? EMP_OK : EMP_E_NOMEM;
    if (st == EMP_OK) st = ctx_ensure(ctx, srv->d_jobs, desc, ctx->stream);
    if (st == EMP_OK) st = ctx_ensure(ctx, srv->d_ctl, sizeof(CoopCtl), ctx->stream);
    if (st != EMP_OK) {
        ctx->in_use -= srv->d_jobs.bytes + srv->d_ctl.bytes;
        delete srv;
        return st;
    }
    *out = srv;
    return EMP_OK;
}

emp_status emp_server_destroy(emp_server *srv) {
    if (!srv) return EMP_E_INVAL;
    cudaSetDevice(srv->ctx->device);
    cudaStreamSynchronize(srv->ctx->stream);
    auto drop = [](emp_job *j) {
        j->server = nullptr;
        j->admit_est = 0;
        j->have_result = false;
        j->last_rc = EMP_E_STATE;
    };
    for (emp_job *j : srv->queue) drop(j);
    for (emp_job *j : srv->live) drop(j);
    for (emp_job *j : srv->finished) j->server = nullptr;
    for (auto &e : srv->ev)
        if (e) cudaEventDestroy(e);
    srv->ctx->in_use -= srv->d_jobs.bytes + srv->d_ctl.bytes;
    delete srv;
    return EMP_OK;
}

emp_status emp_server_submit(emp_server *srv, emp_job *job) {
    if (!srv || !job || job->ctx != srv->ctx) return EMP_E_INVAL;
    if (job->server) return EMP_E_STATE;
    if ((int)(srv->queue.size() + srv->live.size() + srv->finished.size()) >= (1 << 20)) return EMP_E_NOMEM;
    job->server = srv;
    job->have_result = false;
    job->last_rc = EMP_E_STATE;
    srv->queue.push_back(job);
    return EMP_OK;
}

emp_status emp_server_step(emp_server *srv, emp_job **done, int cap, int *n_done) {
    if (!srv || cap < 0 || (cap && !done)) return EMP_E_INVAL;
    if (n_done) *n_done = 0;
    if (cudaSetDevice(srv->ctx->device) != cudaSuccess) return EMP_E_CUDA;
    cudaStream_t s = srv->ctx->stream;
    emp_status st = server_step(srv, s);
    if (st != EMP_OK) {
        cudaStreamSynchronize(s);
        cudaGetLastError();
    }
    const int k = (int)std::min<size_t>((size_t)cap, srv->finished.size());
    for (int i = 0; i < k; ++i) {
        done[i] = srv->finished[i];
        done[i]->server = nullptr;
    }
    srv->finished.erase(srv->finished.begin(), srv->finished.begin() + k);
    if (n_done) *n_done = k;
    return st;
}

emp_status emp_server_get_stats(emp_server *srv, emp_server_stats *st) {
    if (!srv || !st) return EMP_E_INVAL;
    *st = srv->st;
    return EMP_OK;
}

emp_status emp_server_counts(emp_server *srv, int *queued, int *in_flight, int *finished) {
    if (!srv) return EMP_E_INVAL;
    if (queued) *queued = (int)srv->queue.size();
    if (in_flight) *in_flight = (int)srv->live.size();
    if (finished) *finished = (int)srv->finished.size();
    return EMP_OK;
}

emp_status emp_job_output_size(emp_job *job, uint64_t *bytes) {
    if (!job || !bytes) return EMP_E_INVAL;
    if (!job->have_result) return EMP_E_STATE;
    *bytes = job->out.size() + job->dout_bytes;
    return EMP_OK;
}

emp_status emp_job_output_copy(emp_job *job, void *dst, uint64_t cap) {
    if (!job) return EMP_E_INVAL;
    const uint64_t host = job->out.size(), total = host + job->dout_bytes;
    if (!dst && total) return EMP_E_INVAL;
    if (!job->have_result) return EMP_E_STATE;
    if (cap < total) return EMP_E_INVAL;
    if (host) std::memcpy(dst, job->out.data(), host);
    if (job->dout_bytes) {  // records of the device-resident rounds follow those of the host-driven ones
        cudaSetDevice(job->ctx->device);
        if (cudaMemcpy(static_cast<uint8_t *>(dst) + host, job->dout.p, job->dout_bytes, cudaMemcpyDeviceToHost) !=
            cudaSuccess) {
            cudaGetLastError();
            return EMP_E_CUDA;
        }
    }
    return EMP_OK;
}

emp_status emp_job_edges(emp_job *job, emp_edge_sink cb, void *user) {
    if (!job || !cb) return EMP_E_INVAL;
    if (!job->have_result) return EMP_E_STATE;
    const uint64_t total = job->out.size() + job->dout_bytes;
    std::vector<uint8_t> buf;
    const uint8_t *p = job->out.data();
    if (job->dout_bytes) {  // one host copy of the whole output
        try {
            buf.resize(total);
        } catch (...) {
            return EMP_E_NOMEM;
        }
        EMP_TRY(emp_job_output_copy(job, buf.data(), total));
        p = buf.data();
    }
    std::vector<uint32_t> from, to;  // aligned copies of one record's arrays
    for (uint64_t o = 0; o + 12 <= total;) {
        uint64_t n;
        int32_t ovlp;
        std::memcpy(&n, p + o, 8);
        std::memcpy(&ovlp, p + o + 8, 4);
        o += 12;
        if (n > (total - o) / 8) return EMP_E_STATE;  // a malformed record cannot come from a run
        try {
            from.resize(n);
            to.resize(n);
        } catch (...) {
            return EMP_E_NOMEM;
        }
        if (n) {
            std::memcpy(from.data(), p + o, 4 * n);
            std::memcpy(to.data(), p + o + 4 * n, 4 * n);
        }
        o += 8 * n;
        if (cb(user, ovlp, n, from.data(), to.data())) break;
    }
    return EMP_OK;
}

emp_status emp_job_stats(emp_job *job, emp_stats *st) {
    if (!job || !st) return EMP_E_INVAL;
    if (!job->have_result) return EMP_E_STATE;
    *st = job->st;
    return EMP_OK;
}

emp_status emp_job_fingerprints(emp_job *job, uint64_t *keys, uint64_t cap, uint64_t *n_ends) {
    if (!job || !n_ends) return EMP_E_INVAL;
    if (!job->have_result) return EMP_E_STATE;
    *n_ends = job->n_ends;
    if (!job->n_ends || (!keys && cap == 0)) return EMP_OK;  // size query
    if (!keys || cap < job->n_ends) return EMP_E_INVAL;
    cudaSetDevice(job->ctx->device);
    if (cudaMemcpy(keys, job->keys0.p, job->n_ends * 8, cudaMemcpyDeviceToHost) != cudaSuccess) return EMP_E_CUDA;
    return EMP_OK;
}

emp_status emp_job_feed_files(emp_job *job, const char *const *paths, int n_paths) {
    if (!job) return EMP_E_INVAL;
    if (job->server) return EMP_E_STATE;
    if (job->fed_last) return EMP_E_STATE;
    FastqReader rd;
    EMP_TRY(rd.open(paths, n_paths));
    emp_ctx *ctx = job->ctx;
    cudaSetDevice(ctx->device);
    if (rd.size_hint()) EMP_TRY(emp_job_reserve(job, job->F + rd.size_hint()));
    // Two pinned buffers in turn: piece k+1 is read (or inflated) while
    // piece k copies to the device on the copy stream.
    const size_t chunk = 128ull << 20;
    PinnedBuf hb[2];
    cudaEvent_t copied[2] = {nullptr, nullptr};
    emp_status st = EMP_OK;
    if (cudaEventCreateWithFlags(&copied[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&copied[1], cudaEventDisableTiming) != cudaSuccess)
        st = EMP_E_CUDA;
    for (int k = 0; st == EMP_OK; ++k) {
        const int b = k & 1;
        if (k >= 2 && cudaEventSynchronize(copied[b]) != cudaSuccess) {  // the copy that used this buffer
            st = EMP_E_CUDA;
            break;
        }
        if (!hb[b].ensure(chunk)) {
            st = EMP_E_NOMEM;
            break;
        }
        size_t got = 0;
        st = rd.read(hb[b].p, chunk, &got);
        if (st != EMP_OK || got == 0) break;
        st = emp_job_feed_fastq_async(job, hb[b].as<char>(), got, 0);
        if (st == EMP_OK && cudaEventRecord(copied[b], ctx->copy_stream) != cudaSuccess) st = EMP_E_CUDA;
    }
    if (st == EMP_OK) st = emp_job_feed_fastq_async(job, nullptr, 0, 1);
    // the pinned buffers are released below: their copies must be done
    if (cudaStreamSynchronize(ctx->copy_stream) != cudaSuccess && st == EMP_OK) st = EMP_E_CUDA;
    for (cudaEvent_t e : copied)
        if (e) cudaEventDestroy(e);
    return st;
}

emp_status emp_fastq_load(const char *const *paths, int n_paths, void **data, uint64_t *bytes) {
    if (!data || !bytes) return EMP_E_INVAL;
    *data = nullptr;
    *bytes = 0;
    FastqReader rd;
    EMP_TRY(rd.open(paths, n_paths));
    size_t cap = (size_t)rd.size_hint() + FastqReader::kMinChunk;  // the last, empty read fits too
    uint8_t *buf = static_cast<uint8_t *>(std::malloc(cap));
    if (!buf) return EMP_E_NOMEM;
    size_t n = 0;
    for (;;) {
        if (cap - n < FastqReader::kMinChunk) {  // room for one more piece
            const size_t nc = std::max(cap + cap / 2, n + FastqReader::kMinChunk);
            uint8_t *q = static_cast<uint8_t *>(std::realloc(buf, nc));
            if (!q) {
                std::free(buf);
                return EMP_E_NOMEM;
            }
            buf = q;
            cap = nc;
        }
        size_t got = 0;
        const emp_status st = rd.read(buf + n, cap - n, &got);
        if (st != EMP_OK) {
            std::free(buf);
            return st;
        }
        if (got == 0) break;
        n += got;
    }
    if (n == 0) {
        std::free(buf);
        return EMP_OK;
    }
    *data = buf;
    *bytes = n;
    return EMP_OK;
}

void emp_free(void *p) { std::free(p); }

emp_status emp_measure_l2_read(int device, uint64_t bytes, double *gbs) {
    if (!gbs || bytes < 16) return EMP_E_INVAL;
    if (device >= 0 && cudaSetDevice(device) != cudaSuccess) return EMP_E_CUDA;
    return cuda_status(measure_l2_read(bytes, gbs));
}

emp_status emp_run_files(const char *const *input_paths, int n_inputs, const char *output_path, const emp_params *p,
                         int device, emp_stats *stats) {
    if (!output_path || n_inputs < 0 || (n_inputs && !input_paths)) return EMP_E_INVAL;
    for (int i = 0; i < n_inputs; ++i)
        if (!input_paths[i]) return EMP_E_INVAL;
    emp_ctx *ctx = nullptr;
    EMP_TRY(emp_ctx_create(device, 0, &ctx));
    emp_job *job = nullptr;
    emp_status st = emp_job_create(ctx, p, &job);
    if (st != EMP_OK) {
        emp_ctx_destroy(ctx);
        return st;
    }
    st = emp_job_feed_files(job, input_paths, n_inputs);
    if (st == EMP_OK) st = emp_job_run(job, nullptr);  // waits for the last copy
    if (st == EMP_OK) {
        FILE *g = std::fopen(output_path, "wb");
        if (!g) st = EMP_E_IO;
        else {
            if (!job->out.empty() && std::fwrite(job->out.data(), 1, job->out.size(), g) != job->out.size())
                st = EMP_E_IO;
            if (st == EMP_OK && job->dout_bytes) {
                if (!job->h_out.ensure(job->dout_bytes) ||
                    cudaMemcpy(job->h_out.p, job->dout.p, job->dout_bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
                    st = EMP_E_CUDA;
                else if (std::fwrite(job->h_out.p, 1, job->dout_bytes, g) != job->dout_bytes)
                    st = EMP_E_IO;
            }
            if (std::fclose(g) != 0) st = EMP_E_IO;
        }
        if (stats) *stats = job->st;
    }
    emp_job_destroy(job);
    emp_ctx_destroy(ctx);
    return st;
}

emp_status emp_run_file(const char *input_path, const char *output_path, const emp_params *p, int device,
                        emp_stats *stats) {
    if (!input_path) return EMP_E_INVAL;
    return emp_run_files(&input_path, 1, output_path, p, device, stats);
}

}  // extern "C"

// ---- unitigs of an output.bin ------------------------------------------------
struct emp_graph {
    emp_ctx *ctx = nullptr;
    std::vector<uint8_t> bin;         // the output.bin bytes (the L lines come from them)
    std::vector<uint64_t> rec_off;    // byte offset of every record
    uint64_t nodes = 0, edges = 0;
    std::vector<uint32_t> order;      // read-ends in unitig order
    std::vector<uint64_t> starts;     // first position of every unitig, then `nodes`
    emp_graph_stats st{};
};

extern "C" {

emp_status emp_graph_build(emp_ctx *ctx, const void *output_bin, uint64_t bytes, uint64_t n_reads, emp_graph **out) {
    if (!ctx || !out || (bytes && !output_bin)) return EMP_E_INVAL;
    *out = nullptr;
    if (n_reads == 0 || 2 * n_reads >= (1ull << 31)) return n_reads ? EMP_E_UNSUPPORTED : EMP_E_INVAL;
    const uint8_t *b = static_cast<const uint8_t *>(output_bin);
    emp_graph *g = new (std::nothrow) emp_graph();
    if (!g) return EMP_E_NOMEM;
    g->ctx = ctx;
    g->nodes = 2 * n_reads;
    // the records: u64 n | i32 ovlp_len | u32 from[n] | u32 to[n]
    std::vector<uint64_t> e0{0};
    for (uint64_t o = 0; o < bytes;) {
        uint64_t n = 0;
        if (o + 12 > bytes) { delete g; return EMP_E_FORMAT; }
        std::memcpy(&n, b + o, 8);
        if (n > (bytes - o - 12) / 8) { delete g; return EMP_E_FORMAT; }
        g->rec_off.push_back(o);
        e0.push_back(e0.back() + n);
        o += 12 + 8 * n;
    }
    g->edges = e0.back();
    g->bin.assign(b, b + bytes);
    cudaSetDevice(ctx->device);
    const uint32_t V = (uint32_t)g->nodes;
    const uint64_t E = g->edges, nrec = g->rec_off.size();
    // one device allocation for everything, in the context's pool
    const uint64_t scan_t = scan_tiles(V);
    size_t off = 0;
    auto take = [&](size_t bytes_) { const size_t o = off; off = (off + bytes_ + 255) / 256 * 256; return o; };
    const size_t o_bin = take(bytes + 16), o_roff = take(nrec * 8 + 8), o_e0 = take((nrec + 1) * 8);
    const size_t o_from = take(E * 4 + 4), o_to = take(E * 4 + 4);
    size_t o_node[15];
    for (auto &x : o_node) x = take((size_t)V * 4);
    const size_t o_start = take((size_t)V * 8), o_status = take(scan_t * 8 + 64), o_small = take(64);
    cudaStream_t s = ctx->stream;
    void *dev = nullptr;
    if (cudaMallocFromPoolAsync(&dev, off, ctx->pool, s) != cudaSuccess) {
        cudaGetLastError();
        delete g;
        return EMP_E_NOMEM;
    }
    uint8_t *d = static_cast<uint8_t *>(dev);
    GraphBufs gb{};
    gb.from = reinterpret_cast<uint32_t *>(d + o_from);
    gb.to = reinterpret_cast<uint32_t *>(d + o_to);
    uint32_t **node_arrays[15] = {&gb.dout, &gb.din, &gb.succ, &gb.pred, &gb.hop[0], &gb.hop[1], &gb.dist[0],
                                  &gb.dist[1], &gb.mn[0], &gb.mn[1], &gb.nx[0], &gb.nx[1], &gb.size, &gb.order,
                                  nullptr};
    for (int k = 0; k < 14; ++k) *node_arrays[k] = reinterpret_cast<uint32_t *>(d + o_node[k]);
    gb.start = reinterpret_cast<uint64_t *>(d + o_start);
    gb.status = reinterpret_cast<uint64_t *>(d + o_status);
    uint64_t *small = reinterpret_cast<uint64_t *>(d + o_small);  // tile counter, total, error, cycles
    gb.tile_ctr = reinterpret_cast<uint32_t *>(small);
    gb.total = small + 1;
    gb.err = reinterpret_cast<uint32_t *>(small + 2);
    gb.cycles = reinterpret_cast<uint32_t *>(small + 3);
    emp_status rc = EMP_OK;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    PinnedBuf hs;
    if (!hs.ensure(64)) rc = EMP_E_NOMEM;
    if (rc == EMP_OK && (cudaEventCreate(&ev[0]) != cudaSuccess || cudaEventCreate(&ev[1]) != cudaSuccess))
        rc = EMP_E_CUDA;
    if (rc == EMP_OK) {
        cudaEventRecord(ev[0], s);
        if (bytes) cudaMemcpyAsync(d + o_bin, b, bytes, cudaMemcpyHostToDevice, s);
        if (nrec) cudaMemcpyAsync(d + o_roff, g->rec_off.data(), nrec * 8, cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(d + o_e0, e0.data(), (nrec + 1) * 8, cudaMemcpyHostToDevice, s);
        cudaMemsetAsync(gb.status, 0, scan_t * 8 + 64, s);
        cudaMemsetAsync(small, 0, 64, s);
        graph_build(d + o_bin, reinterpret_cast<uint64_t *>(d + o_roff), reinterpret_cast<uint64_t *>(d + o_e0),
                    (uint32_t)nrec, E, V, gb, s);
        cudaEventRecord(ev[1], s);
        g->order.resize(V);
        std::vector<uint32_t> size(V);
        cudaMemcpyAsync(g->order.data(), gb.order, (size_t)V * 4, cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(size.data(), gb.size, (size_t)V * 4, cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(hs.p, small, 32, cudaMemcpyDeviceToHost, s);
        if (cudaStreamSynchronize(s) != cudaSuccess || cudaGetLastError() != cudaSuccess) rc = EMP_E_CUDA;
        const uint64_t *hw = hs.as<uint64_t>();
        if (rc == EMP_OK && (hw[2] & kErrSpin)) rc = EMP_E_TIMEOUT;
        if (rc == EMP_OK && (hw[2] & kErrCapacity)) rc = EMP_E_FORMAT;  // an edge beyond the read-ends given
        if (rc == EMP_OK) {
            uint64_t pos = 0;
            for (uint32_t u = 0; u < V; ++u)
                if (size[u]) {
                    g->starts.push_back(pos);
                    pos += size[u];
                    g->st.long_unitigs += size[u] >= 2;
                }
            g->starts.push_back(pos);
            g->st.nodes = V;
            g->st.edges = E;
            g->st.unitigs = g->starts.size() - 1;
            g->st.cycles = (uint32_t)hw[3];
            g->st.ms_build = ms_between(ev[0], ev[1]);
            if (pos != V) rc = EMP_E_CUDA;
        }
    }
    for (cudaEvent_t e : ev)
        if (e) cudaEventDestroy(e);
    cudaFreeAsync(dev, s);
    if (rc != EMP_OK) {
        cudaStreamSynchronize(s);
        delete g;
        return rc;
    }
    *out = g;
    return EMP_OK;
}

emp_status emp_graph_get_stats(emp_graph *g, emp_graph_stats *st) {
    if (!g || !st) return EMP_E_INVAL;
    *st = g->st;
    return EMP_OK;
}

emp_status emp_graph_unitigs(emp_graph *g, uint32_t *order, uint64_t order_cap, uint64_t *starts, uint64_t starts_cap) {
    if (!g) return EMP_E_INVAL;
    if (order) {
        if (order_cap < g->order.size()) return EMP_E_INVAL;
        std::memcpy(order, g->order.data(), g->order.size() * 4);
    }
    if (starts) {
        if (starts_cap < g->starts.size()) return EMP_E_INVAL;
        std::memcpy(starts, g->starts.data(), g->starts.size() * 8);
    }
    return EMP_OK;
}

namespace {
// decimal digits of v at p; returns the end
char *put_u64(char *p, uint64_t v) {
    char t[24];
    int k = 0;
    do {
        t[k++] = (char)('0' + v % 10);
        v /= 10;
    } while (v);
    while (k) *p++ = t[--k];
    return p;
}
}  // namespace

emp_status emp_graph_write_gfa(emp_graph *g, const char *path, int32_t read_len) {
    if (!g || !path || read_len < 0) return EMP_E_INVAL;
    FILE *f = std::fopen(path, "wb");
    if (!f) return EMP_E_IO;
    std::vector<char> buf(1 << 22);
    size_t used = 0;
    bool ok = true;
    auto flush = [&](size_t room) {
        if (used + room > buf.size()) {
            ok = ok && std::fwrite(buf.data(), 1, used, f) == used;
            used = 0;
        }
    };
    auto put = [&](const char *str) {
        const size_t l = std::strlen(str);
        flush(l);
        std::memcpy(buf.data() + used, str, l);
        used += l;
    };
    put("H\tVN:Z:1.0\n");
    const uint64_t n_reads = g->nodes / 2;
    for (uint64_t i = 0; i < n_reads; ++i) {  // S <id> * LN:i:<L>
        flush(64);
        char *p = buf.data() + used;
        *p++ = 'S';
        *p++ = '\t';
        p = put_u64(p, i);
        std::memcpy(p, "\t*\tLN:i:", 8);
        p = put_u64(p + 8, (uint64_t)read_len);
        *p++ = '\n';
        used = (size_t)(p - buf.data());
    }
    const uint8_t *b = g->bin.data();
    for (uint64_t o : g->rec_off) {  // L <u> <+|-> <v> <+|-> <len>M, edges in output.bin order
        uint64_t n = 0;
        int32_t ovlp = 0;
        std::memcpy(&n, b + o, 8);
        std::memcpy(&ovlp, b + o + 8, 4);
        const uint8_t *fr = b + o + 12, *to = fr + 4 * n;
        for (uint64_t k = 0; k < n; ++k) {
            uint32_t u, v;
            std::memcpy(&u, fr + 4 * k, 4);
            std::memcpy(&v, to + 4 * k, 4);
            flush(80);
            char *p = buf.data() + used;
            *p++ = 'L';
            *p++ = '\t';
            p = put_u64(p, u >> 1);
            *p++ = '\t';
            *p++ = (u & 1) ? '-' : '+';
            *p++ = '\t';
            p = put_u64(p, v >> 1);
            *p++ = '\t';
            *p++ = (v & 1) ? '-' : '+';
            *p++ = '\t';
            p = put_u64(p, (uint64_t)(ovlp < 0 ? 0 : ovlp));
            *p++ = 'M';
            *p++ = '\n';
            used = (size_t)(p - buf.data());
        }
    }
    uint64_t k = 0;
    for (size_t q = 0; q + 1 < g->starts.size(); ++q) {  // P utg<k> <id><+|->,... *
        const uint64_t a = g->starts[q], z = g->starts[q + 1];
        if (z - a < 2) continue;
        flush(32);
        char *p = buf.data() + used;
        std::memcpy(p, "P\tutg", 5);
        p = put_u64(p + 5, k++);
        *p++ = '\t';
        used = (size_t)(p - buf.data());
        for (uint64_t x = a; x < z; ++x) {
            flush(32);
            p = buf.data() + used;
            if (x != a) *p++ = ',';
            const uint32_t u = g->order[x];
            p = put_u64(p, u >> 1);
            *p++ = (u & 1) ? '-' : '+';
            used = (size_t)(p - buf.data());
        }
        put("\t*\n");
    }
    flush(buf.size());
    ok = ok && std::fwrite(buf.data(), 1, used, f) == used;
    if (std::fclose(f) != 0) ok = false;
    return ok ? EMP_OK : EMP_E_IO;
}

emp_status emp_graph_destroy(emp_graph *g) {
    if (!g) return EMP_E_INVAL;
    delete g;
    return EMP_OK;
}

emp_status emp_sort_pairs(emp_ctx *ctx, uint64_t *d_keys, uint32_t *d_vals, uint64_t n, void *stream) {
    if (!ctx || (n && (!d_keys || !d_vals))) return EMP_E_INVAL;
    if (n < 2) return EMP_OK;
    if (n >= (1ull << 30)) return EMP_E_UNSUPPORTED;
    cudaSetDevice(ctx->device);
    cudaStream_t s = stream ? reinterpret_cast<cudaStream_t>(stream) : ctx->stream;
    auto grow = [&](DevBuf &b, size_t bytes) -> bool {
        if (b.bytes >= bytes) return true;
        b.release();
        if (cudaMalloc(&b.p, bytes) != cudaSuccess) {
            cudaGetLastError();
            b.p = nullptr;
            return false;
        }
        b.bytes = bytes;
        return true;
    };
    // the working set is kept in the context for the next call
    if (n > ctx->sort_cap || ctx->sort_calls > 100000) {
        if (!grow(ctx->sort_k1, n * 8) || !grow(ctx->sort_v1, n * 4) || !grow(ctx->sort_scr, sort_scratch_bytes(n)) ||
            !grow(ctx->sort_err, 16))
            return EMP_E_NOMEM;
        if (cudaMemsetAsync(ctx->sort_scr.p, 0, ctx->sort_scr.bytes, s) != cudaSuccess) return EMP_E_CUDA;
        ctx->sort_cap = n;
        ctx->sort_calls = 0;
    }
    ++ctx->sort_calls;
    // sort_err: the error word, then (8 bytes in) the device copy of n
    uint64_t *err = ctx->sort_err.as<uint64_t>();
    cudaMemsetAsync(err, 0, 8, s);
    sort_pairs(d_keys, d_vals, ctx->sort_k1.as<uint64_t>(), ctx->sort_v1.as<uint32_t>(), n, ctx->sort_scr.p, err + 1,
               reinterpret_cast<uint32_t *>(err), s);
    uint32_t herr = 0;
    cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return EMP_E_CUDA;
    if (herr & kErrSpin) return EMP_E_TIMEOUT;
    return EMP_OK;
}

}  // extern "C"
