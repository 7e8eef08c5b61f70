/*
 * empanada.h -- C ABI of the B200 read-overlap engine (libempanada_b200.so).
 *
 * Drop-in for empanada's read-overlap path: FASTQ -> 2-bit bases ->
 * Rabin-Karp fingerprints of every read-end -> sort -> per-round
 * suffix/prefix join -> output.bin.  The reference has no FFI; its seams are
 * the process CLI (config.h:120-140, main.cu:9-77), the output.bin format
 * (overlap.cu:148-161) and the internal C++ functions of assembly.cuh:67-82.
 * Each entry point below names the reference code it replaces.
 *
 * Conventions: plain pointers and sizes, no exceptions and no exit() across
 * the ABI; every call returns an emp_status (0 = OK, < 0 = error).  A context
 * or job is driven by one host thread at a time; distinct jobs may be driven
 * from distinct threads.  Every device wait inside the engine is bounded and
 * reports EMP_E_TIMEOUT instead of hanging.
 *
 * output.bin: a sequence of records, little-endian, no header:
 *     u64 n | i32 ovlp_len | u32 from[n] | u32 to[n]
 * one record per (round, search partition) that has both suffixes and
 * prefixes, ovlp_len = L-1-round, ids rid = 2i (read i) / 2i+1 (its reverse
 * complement), i counting reads without N in file order.
 */
#ifndef EMPANADA_H
#define EMPANADA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EMP_ABI_VERSION 6

typedef int emp_status;
#define EMP_OK 0
#define EMP_E_INVAL (-1)       /* bad argument (reference: usage / LOG_ERR) */
#define EMP_E_NOMEM (-2)       /* device or host allocation failed, or over the HBM budget */
#define EMP_E_CUDA (-3)        /* CUDA runtime error (reference: CUDA_SAFE -> exit(1)) */
#define EMP_E_TIMEOUT (-4)     /* a bounded device wait ran out */
#define EMP_E_FORMAT (-5)      /* kept reads of unequal length, or a base outside ACGTacgt */
#define EMP_E_STATE (-6)       /* call out of order (e.g. feed after run) */
#define EMP_E_IO (-7)          /* file could not be read or written */
#define EMP_E_UNSUPPORTED (-8) /* read length above 512 (the reference stops at 255; above it its result is undefined) */
#define EMP_E_HANG (-9)        /* input on which the reference never terminates */

typedef struct emp_ctx emp_ctx;
typedef struct emp_job emp_job;
typedef struct emp_server emp_server;

/* The reference's command-line options (config.h:120-140). */
typedef struct emp_params {
    int32_t min_ovlp;      /* -o, minimum overlap length (default 31) */
    uint64_t map_mem;      /* -m, bytes (default 1g); FASTQ block = map_mem/16 (main.cu:16) */
    uint64_t reduce_mem;   /* -r, bytes (default 1g); M = reduce_mem/16 pairs (main.cu:69) */
    uint64_t base_blocksz; /* -b, bytes (default 32m) */
    uint64_t kv_chunksz;   /* -c, count (default 64m) */
} emp_params;

#define EMP_MAX_ROUNDS 512

typedef struct emp_stats {
    uint64_t n_reads;      /* reads kept after the N filter */
    int32_t read_len;      /* L */
    int32_t n_rounds;      /* rounds executed */
    uint64_t n_unique;     /* read-ends after duplicate removal */
    uint64_t n_edges;      /* edges written */
    uint64_t n_records;    /* output.bin records */
    uint64_t fastq_bytes;  /* input size */
    uint64_t output_bytes; /* output.bin size */
    uint64_t gpu_launches; /* engine kernels launched by the last run */
    double ms_h2d;         /* FASTQ host->device copy (0 for device input) */
    double ms_map;         /* parse + fingerprint + column store (device time) */
    double ms_dedup;       /* fingerprint sort + duplicate removal (device time) */
    double ms_rounds;      /* overlap rounds (device time, incl. edge copies) */
    double ms_total;       /* whole run (device time) */
    double ms_sort_passes; /* device time of all radix-sort digit passes (CUDA events per launch) */
    uint64_t sort_passes;  /* digit-pass launches */
    uint64_t sort_pass_elems; /* sum over those launches of the pairs each one moved */
    double ms_update;      /* device time of the per-round table update kernel (CUDA events per launch) */
    uint64_t update_launches; /* its launches that processed entries */
    uint64_t update_bytes;    /* their algorithmic bytes (13 B read + 1/4 B of bases per entry in, 12 B per entry out) */
    double ms_round_kernel;   /* device time of the cooperative all-rounds kernel (CUDA events), 0 if not used */
    uint64_t round_kernel_bytes; /* its algorithmic bytes: update + candidates + candidate sort + join, per round */
    uint64_t sfx_live[EMP_MAX_ROUNDS]; /* suffix-table size in round r */
    uint64_t pfx_live[EMP_MAX_ROUNDS]; /* prefix-table size in round r */
    uint64_t edges[EMP_MAX_ROUNDS];    /* edges written in round r */
} emp_stats;

/* Human-readable name of a status code. */
const char *emp_status_string(emp_status st);
int emp_abi_version(void);

/* Defaults of config.h:124-128 (o=31, m=1g, r=1g, b=32m, c=64m). */
emp_status emp_params_default(emp_params *p);

/* hmsize2bytes (config.h:75-100): digits with an optional k/K/m/M/g/G
 * binary suffix.  An unknown suffix is reported and ignored, like the
 * reference (value returned without the suffix, status EMP_E_INVAL). */
emp_status emp_parse_size(const char *s, uint64_t *bytes);

/* A context owns one device (cudaSetDevice), its stream and hash tables.
 * hbm_budget_bytes = 0: no budget.  Replaces the process-wide singletons and
 * precomputeModulos/init_match (fingerprint.cu:26-34, overlap.cu:117-127). */
emp_status emp_ctx_create(int device, uint64_t hbm_budget_bytes, emp_ctx **out);
emp_status emp_ctx_destroy(emp_ctx *ctx);

/* Engine choices of a context; they have no counterpart in the reference.
 * Every choice gives the same output.bin: they trade speed and memory (the
 * autotuner, empanada_b200.tune, picks them by timing) or serve tests.  A
 * zero field means its default.  Set them while no job of the context runs. */
typedef struct emp_tuning {
    int32_t round_driver;     /* 0: the bucket kernel for every round that cannot split into
                                 several search partitions; 1: host-synchronised rounds only */
    uint32_t bucket_mean;     /* bucket kernel: entries per key bucket aimed at, 512..3000 (default 2900) */
    uint32_t region_cap;      /* bucket kernel: entries per (bucket, table) region, 1..2048 (default 2048);
                                 a region's overflow goes to a spill area */
    int32_t dedup_driver;     /* 0: duplicate removal by key buckets and hash sets where 2n <= M (the
                                 reference's in-core survivor, the smallest rid of each fingerprint);
                                 1: always by sorting all fingerprints */
    uint64_t edge_cap;        /* first edge-buffer size in edges (default: 4 per read-end, at least 2^20);
                                 a run that needs more reruns its rounds with a larger one */
    uint64_t wait_limit_ns;   /* time limit of every grid-barrier wait of the bucket kernel (default 20 s) */
    int32_t block_next_wait;  /* testing: the context's next bucket-kernel launch meets a grid barrier
                                 that no arrival completes, so its waits run out after wait_limit_ns and
                                 the run returns EMP_E_TIMEOUT; that launch clears the flag */
    uint32_t map_streams;     /* streams that the map phase of a batch (or a server step) spreads its
                                 jobs over, 1..32 (default 8) */
} emp_tuning;
emp_status emp_tuning_default(emp_tuning *t);
/* EMP_E_INVAL for a value outside its range (the context keeps its choices). */
emp_status emp_ctx_set_tuning(emp_ctx *ctx, const emp_tuning *t);
emp_status emp_ctx_get_tuning(emp_ctx *ctx, emp_tuning *t);

/* One job = one read set with the reference's options. */
emp_status emp_job_create(emp_ctx *ctx, const emp_params *p, emp_job **out);
emp_status emp_job_destroy(emp_job *job);

/* Append FASTQ bytes (host memory, any split, records may straddle calls);
 * replaces read_block's file reads (preprocess.cu:195-237).  `last` marks
 * the final piece. */
emp_status emp_job_feed_fastq(emp_job *job, const char *bytes, uint64_t n, int last);
/* emp_job_feed_fastq without waiting for the copy: it runs on the
 * context's copy stream (concurrently with other jobs' kernels) and the
 * job's next run waits for it.  `bytes` must stay valid and unchanged until
 * then; page-locked memory makes the copy truly asynchronous. */
emp_status emp_job_feed_fastq_async(emp_job *job, const char *bytes, uint64_t n, int last);
/* Same for bytes already in device memory on the context's device. */
emp_status emp_job_feed_fastq_device(emp_job *job, const void *dev_bytes, uint64_t n, int last);
/* Append the FASTQ of files, in order, and mark the end of the input: each
 * file plain, gzip (one or more members) or BGZF (blocked gzip, its blocks
 * inflated in parallel on the host cores); a newline is added after a file
 * that does not end with one when another non-empty file follows.  A
 * missing file reads as empty (as the reference's read of its one plain
 * file, preprocess.cu:195-237); a path that exists but is not a readable
 * regular file is EMP_E_IO, a damaged gzip stream or BGZF block
 * EMP_E_FORMAT.  The files are read into two page-locked buffers in turn:
 * one piece is inflated or read while the previous one copies to the
 * device (no counterpart in the reference). */
emp_status emp_job_feed_files(emp_job *job, const char *const *paths, int n_paths);
/* Reserve device room for `bytes` of FASTQ (optional; avoids regrowth). */
emp_status emp_job_reserve(emp_job *job, uint64_t bytes);
/* Forget the fed input and the last result but keep every device buffer, so
 * the job can take the next read set without new allocations. */
emp_status emp_job_reset(emp_job *job);
/* Forget the fed input and the last result and give every device buffer
 * back to the context's memory pool (stream-ordered, no device-wide
 * synchronisation), so that idle jobs hold no device memory; the next run
 * takes its buffers from the pool again. */
emp_status emp_job_trim(emp_job *job);

/* Map + reduce phases: main.cu:42-71 (read_block, transpose_reads,
 * get_reverse_complements, generate_fingerprint_read_pairs) and build_graph
 * (overlap.cu:206-293).  stream: a cudaStream_t, or NULL for the context's. */
emp_status emp_job_run(emp_job *job, void *stream);

/* emp_job_run of njobs independent jobs of one context (at most 1024, each
 * once) as one batch: the map phase of every job with one stream
 * synchronisation per stage for the whole batch, and the rounds of all jobs
 * whose lists fit the bucket kernel in a single launch of it.  Replaces one
 * run of the reference's whole program (main.cu:42-71, then build_graph,
 * overlap.cu:206-293) per read set; each job's output is byte-identical to
 * emp_job_run's.  Returns the first failing job's status (jobs that failed
 * have no result; the others do), EMP_OK when all succeeded. */
emp_status emp_batch_run(emp_ctx *ctx, emp_job **jobs, int njobs, void *stream);

/* Status of the job's last run (emp_job_run, a batch or a server):
 * EMP_E_STATE while it has none. */
emp_status emp_job_status(emp_job *job);

/* Served jobs (no counterpart in the reference, which is one process per
 * read set): a request loop with continuous batching.  Fed jobs are
 * submitted; each step admits queued jobs (first come, first served, while
 * the footprint estimates of the jobs in flight stay within the budget: 4 B
 * per FASTQ byte + 64 MiB per job), runs their map phase, adds them to the
 * batch, and runs one bucket-kernel launch of at most rounds_per_launch
 * rounds of every job in the batch; jobs join and leave the batch between
 * launches.  A job too large for the batch, or whose rounds split into
 * several search partitions, runs alone within the step, and so does a job
 * admitted alone into an idle server (no job in flight or queued), as
 * emp_job_run runs it.  Every job's output
 * equals its emp_job_run output.  A job held by a server (submitted, not yet
 * handed out by a step) accepts no other call. */
typedef struct emp_server_params {
    int32_t rounds_per_launch; /* bucket-kernel rounds per launch (default 16) */
    int32_t max_jobs;          /* jobs in the batch at most, <= 1024 (default 256) */
    uint64_t hbm_budget_bytes; /* admission budget (0: the context's, or none) */
    int32_t rounds_per_launch_idle; /* the same while no job waits to join (default 64) */
    uint64_t batch_max_entries; /* a job whose first round list is longer runs alone (0: the bucket kernel's 16M) */
    uint64_t share_min_entries; /* a job whose first round list is at least this long runs rounds_per_launch
                                   (rounds_per_launch_idle while no job waits) rounds of a launch; a shorter
                                   one runs all its rounds in the launch it joins (default 8M; 0: every job
                                   the launch's rounds) */
} emp_server_params;
emp_status emp_server_params_default(emp_server_params *p);
emp_status emp_server_create(emp_ctx *ctx, const emp_server_params *p, emp_server **out);
/* Jobs still queued or in the batch are released without a result. */
emp_status emp_server_destroy(emp_server *srv);
emp_status emp_server_submit(emp_server *srv, emp_job *job);
/* One step; up to cap finished jobs are handed out in done[0..*n_done)
 * (each with emp_job_status set), the rest wait for the next step. */
emp_status emp_server_step(emp_server *srv, emp_job **done, int cap, int *n_done);
emp_status emp_server_counts(emp_server *srv, int *queued, int *in_flight, int *finished);
typedef struct emp_server_stats {
    uint64_t steps;      /* emp_server_step calls */
    uint64_t admitted;   /* jobs admitted */
    uint64_t launches;   /* bucket-kernel launches */
    uint64_t rounds;     /* launch iterations (each runs one round of every job in the batch) */
    uint64_t batch_jobs; /* sum over launches of the jobs in the batch */
    double ms_kernel;    /* device time of those launches */
    double ms_admit;     /* host wall time of admission + map phase + jobs run alone */
    double ms_map;       /* of which the map phase */
    double ms_alone;     /* of which jobs run alone */
    uint64_t alone;      /* jobs run alone */
    double ms_wait;      /* host wall time waiting for the launch once admission is done */
    double ms_results;   /* host wall time of launch results: copies back, completed jobs closed */
    double ms_launch;    /* host wall time from the step's start to the launch queued */
} emp_server_stats;
emp_status emp_server_get_stats(emp_server *srv, emp_server_stats *st);

/* output.bin bytes of the last run (write_edges_binary, overlap.cu:148-161). */
emp_status emp_job_output_size(emp_job *job, uint64_t *bytes);
emp_status emp_job_output_copy(emp_job *job, void *dst, uint64_t cap);
emp_status emp_job_stats(emp_job *job, emp_stats *st);
/* The last run's records in output.bin order, one call per record:
 * overlap length, edge count n, and the n (from, to) read-end ids (arrays
 * valid during the call).  A nonzero return stops the walk.  The records
 * write_edges_binary would write (overlap.cu:148-161), without the file. */
typedef int (*emp_edge_sink)(void *user, int32_t ovlp_len, uint64_t n, const uint32_t *from, const uint32_t *to);
emp_status emp_job_edges(emp_job *job, emp_edge_sink cb, void *user);

/* Full-length fingerprints of every read-end of the last run, indexed by
 * read-end id (generate_fingerprint_read_pairs, fingerprint.cu:75-115).
 * keys = NULL with cap = 0 only reports *n_ends. */
emp_status emp_job_fingerprints(emp_job *job, uint64_t *keys, uint64_t cap, uint64_t *n_ends);

/* The whole reference program (main.cu:9-77): read input_path, write
 * output_path.  A missing input file gives an empty output.bin, as in the
 * reference.  device < 0: current device.  The input may also be gzip or
 * BGZF compressed (emp_job_feed_files). */
emp_status emp_run_file(const char *input_path, const char *output_path, const emp_params *p, int device,
                        emp_stats *st);
/* emp_run_file over the FASTQ of several files in order (emp_job_feed_files). */
emp_status emp_run_files(const char *const *input_paths, int n_inputs, const char *output_path, const emp_params *p,
                         int device, emp_stats *st);
/* The FASTQ of files as emp_job_feed_files reads them, into host memory
 * (malloc'd, freed by emp_free): *data = NULL when it is empty.  No device
 * is used. */
emp_status emp_fastq_load(const char *const *paths, int n_paths, void **data, uint64_t *bytes);
void emp_free(void *p);

/* Measurement aid (no counterpart in the reference): the device's L2 read
 * bandwidth in GB/s, a buffer of `bytes` (keep it well below the L2's size)
 * read again and again with 16-byte loads once it is in L2.  The round
 * kernel's lists stay in L2 on smaller workloads; this is the denominator of
 * its L2 roofline.  device < 0: current device. */
emp_status emp_measure_l2_read(int device, uint64_t bytes, double *gbs);

/* Unitigs of the overlap graph in an output.bin: the downstream consumer
 * that the reference leaves out (its GFA writers, overlap.cu:129-190, are dead
 * code).  Nodes are read-ends (rid 2i = read i, 2i+1 = its reverse
 * complement, i < n_reads), edges the records' (from, to) pairs.  Under the
 * reference's remove_used rule every suffix keeps only its longest overlaps,
 * so no edge is transitive.  A unitig is a maximal path of edges u -> v with
 * out-degree(u) = in-degree(v) = 1 (a cycle of them is cut before its
 * smallest read-end); every read-end is in exactly one unitig.  Built on the
 * context's device; output_bin is host memory. */
typedef struct emp_graph emp_graph;
typedef struct emp_graph_stats {
    uint64_t nodes;        /* read-ends, 2 n_reads */
    uint64_t edges;        /* edges of output.bin */
    uint64_t unitigs;      /* unitigs, singletons included */
    uint64_t long_unitigs; /* unitigs of two or more read-ends */
    uint64_t cycles;       /* cycles cut */
    double ms_build;       /* device time of the build */
} emp_graph_stats;
emp_status emp_graph_build(emp_ctx *ctx, const void *output_bin, uint64_t bytes, uint64_t n_reads, emp_graph **out);
emp_status emp_graph_get_stats(emp_graph *g, emp_graph_stats *st);
/* The read-ends in unitig order (order[nodes]) and each unitig's first
 * position (starts[unitigs + 1]); unitigs are ordered by their first
 * read-end's id.  Either array may be NULL. */
emp_status emp_graph_unitigs(emp_graph *g, uint32_t *order, uint64_t order_cap, uint64_t *starts, uint64_t starts_cap);
/* GFA 1.0: a header, one S line per read (length read_len), one L line per
 * edge in output.bin order (orientation + for rid 2i, - for 2i+1; overlap as
 * <len>M), one P line per unitig of two or more read-ends. */
emp_status emp_graph_write_gfa(emp_graph *g, const char *path, int32_t read_len);
emp_status emp_graph_destroy(emp_graph *g);

/* Stable sort of n (key, value) pairs in device memory by
 * (fp1, fp2, value>>31) -- the key order of thrust::sort_by_key on the
 * reference's fingerprints (cqutils.cuh:195).  Allocates its scratch.
 * stream: a cudaStream_t or NULL. */
emp_status emp_sort_pairs(emp_ctx *ctx, uint64_t *d_keys, uint32_t *d_vals, uint64_t n, void *stream);

/* emp_sort_pairs without any allocation; it has no counterpart in the
 * reference.  For callers that must not allocate device memory: a host
 * program that owns the whole device through an arena or allocator of its
 * own (an extra cudaMalloc would bypass its accounting, or fail once the
 * arena holds the memory), and latency-bound loops in which cudaMalloc or
 * cudaFree would synchronise the device.  The working set -- alternate
 * key/value buffers, histograms, look-back words, error word -- lives in one
 * statically sized device array of this library (about 12.6 MB, held on
 * every device that loads the library until the process exits), so n is
 * limited to EMP_SORT_STATIC_MAX_PAIRS; a larger n returns EMP_E_INVAL.
 * Runs on the current device; the first call on a device looks up the
 * array's device address (make that first call before any stream capture).
 * Returns after the sort has finished on `stream`.  All calls on one device
 * share the array: calls whose GPU work overlaps (other streams, other host
 * threads) race on it and give wrong results. */
#define EMP_SORT_STATIC_MAX_PAIRS (1u << 20)
emp_status emp_sort_pairs_static(uint64_t *d_keys, uint32_t *d_vals, uint64_t n, void *stream);

#ifdef __cplusplus
}
#endif
#endif
