/*
 * empanada_oracle.h -- CPU restatement of empanada's read-overlap path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the parity tests, the
 * package's smoke check and the benchmark's CPU-baseline leg compare the
 * CUDA path against; the product never links, loads or calls it.
 *
 * Parity is pinned: tests/test_oracle.py compares this restatement
 * byte-for-byte with the reference's own sources built as a CPU program
 * (oracle/Makefile target ref-cpu) on seeded inputs, and against the golden
 * output.bin fixtures in tests/golden/ that the reference build produced.
 */
#ifndef EMPANADA_ORACLE_H
#define EMPANADA_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes: the same values as the product's include/empanada.h */
#define EMP_ORACLE_OK 0
#define EMP_ORACLE_E_INVAL (-1)
#define EMP_ORACLE_E_NOMEM (-2)
#define EMP_ORACLE_E_FORMAT (-5)      /* unequal read lengths / unsupported base */
#define EMP_ORACLE_E_UNSUPPORTED (-8) /* read length above 512 */
#define EMP_ORACLE_E_HANG (-9)        /* input on which the reference never terminates */

#define EMP_ORACLE_MAX_ROUNDS 512

typedef struct emp_oracle_stats {
    uint64_t n_reads;        /* reads kept after the N filter */
    int32_t read_len;        /* L */
    int32_t n_rounds;        /* rounds executed */
    uint64_t n_unique;       /* read-ends left after duplicate removal */
    uint64_t n_edges;        /* total edges written */
    uint64_t n_records;      /* output.bin records written */
    uint64_t sfx_live[EMP_ORACLE_MAX_ROUNDS]; /* |suffix table| entering round r */
    uint64_t pfx_live[EMP_ORACLE_MAX_ROUNDS]; /* |prefix table| entering round r */
    uint64_t edges[EMP_ORACLE_MAX_ROUNDS];    /* edges emitted in round r */
} emp_oracle_stats;

/* Whole pipeline: FASTQ bytes -> output.bin bytes (malloc'd, free with
 * emp_oracle_free).  reduce_mem is the reference's -r value in bytes
 * (M = reduce_mem / 16 key-value pairs). */
int emp_oracle_run(const char *fastq, size_t fastq_len, int32_t min_ovlp, uint64_t reduce_mem,
                   uint8_t **out, size_t *out_len, emp_oracle_stats *stats);

/* Variable-length extension of emp_oracle_run (the reference requires equal
 * read lengths, fingerprint.cu:134-135).  Overlap lengths ell run from the
 * longest read's L-1 down to min_ovlp; a read-end of length len joins the
 * suffix and prefix tables at ell = len-1, so the tables at ell hold the
 * read-ends longer than ell that have not left them, and each round is the
 * reference's round on those tables (same tie order, partitions, records and
 * removal).  Duplicates are removed by full-length key, as in the reference.
 * Equals emp_oracle_run when every kept read has the same length;
 * stats->read_len is the longest length. */
int emp_oracle_run_var(const char *fastq, size_t fastq_len, int32_t min_ovlp, uint64_t reduce_mem,
                       uint8_t **out, size_t *out_len, emp_oracle_stats *stats);

/* FASTQ -> kept reads (n x L ASCII bases, malloc'd) */
int emp_oracle_parse(const char *fastq, size_t fastq_len, char **reads, uint64_t *n_reads, int32_t *read_len);

/* Full-length fingerprints of every read-end: keys[2i] = read i, keys[2i+1] = its reverse complement. */
int emp_oracle_fingerprints(const char *fastq, size_t fastq_len, uint64_t *keys, uint64_t cap,
                            uint64_t *n_reads, int32_t *read_len);

/* Single-step functions (known-answer tests). */
uint64_t emp_oracle_hash(const char *s, int32_t len);
uint64_t emp_oracle_next_sfx(uint64_t key, char base, int32_t len);
uint64_t emp_oracle_prev_pfx(uint64_t key, char base);
uint32_t emp_oracle_radix_inv(int which); /* 1 -> RADIX1^-1 mod PRIME1, 2 -> RADIX2^-1 mod PRIME2 */

void emp_oracle_free(void *p);

#ifdef __cplusplus
}
#endif
#endif
