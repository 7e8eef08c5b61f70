/*
 * synth_reads.c -- seeded synthetic FASTQ generator for the read-overlap
 * workloads (test and benchmark input; not part of the overlap path).
 *
 * Contract (every step is a pure function of the seed):
 *   genome    G bases, i.i.d. uniform over ACGT;
 *   repeats   optional: families of length U[rep_min_len, rep_max_len] with
 *             U{rep_min_copies..rep_max_copies} copies, each copy written at
 *             a uniform genome position with rep_divergence substitutions,
 *             until repeat_frac * G bases are covered;
 *   reads     start uniform in [0, G-L]; each base substituted with
 *             probability sub_rate by one of the other three bases
 *             (uniform); the read is reverse-complemented with
 *             probability rc_prob;
 *   record    "@r<i>\n<seq>\n+\n<'I' x L>\n".
 * Reads are generated in chunks of EMP_SYNTH_CHUNK reads, each chunk with its
 * own PRNG stream derived from (seed, chunk), so the output is identical for
 * any thread count.
 *
 * PRNG: xoshiro256** seeded through splitmix64 (Blackman & Vigna, public
 * domain algorithms restated here).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define EMP_SYNTH_CHUNK 65536u

typedef struct emp_synth_params {
    uint64_t seed;
    uint64_t genome_len;
    uint64_t n_reads;
    int32_t read_len;
    int32_t n_threads;       /* <= 0: all available */
    double sub_rate;
    double rc_prob;
    double repeat_frac;      /* 0: no repeat families */
    int32_t rep_min_len, rep_max_len;
    int32_t rep_min_copies, rep_max_copies;
    double rep_divergence;
} emp_synth_params;

typedef struct { uint64_t s[4]; } rng_t;

static uint64_t splitmix64(uint64_t *x) {
    uint64_t z = (*x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static void rng_seed(rng_t *r, uint64_t seed, uint64_t stream) {
    uint64_t x = seed ^ (0xD1B54A32D192ED03ull * (stream + 1));
    for (int i = 0; i < 4; ++i) r->s[i] = splitmix64(&x);
}

static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

static inline uint64_t rng_next(rng_t *r) {
    uint64_t *s = r->s;
    uint64_t result = rotl(s[1] * 5, 7) * 9;
    uint64_t t = s[1] << 17;
    s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
    s[2] ^= t; s[3] = rotl(s[3], 45);
    return result;
}

/* uniform integer in [0, m) (multiply-high; bias < m / 2^64) */
static inline uint64_t rng_below(rng_t *r, uint64_t m) {
    return (uint64_t)(((unsigned __int128)rng_next(r) * m) >> 64);
}

/* uniform double in [0, 1) with 53 random bits */
static inline double rng_unit(rng_t *r) { return (double)(rng_next(r) >> 11) * (1.0 / 9007199254740992.0); }

static const char BASES[4] = {'A', 'C', 'G', 'T'};

static inline char complement(char c) {
    switch (c) { case 'A': return 'T'; case 'C': return 'G'; case 'G': return 'C'; default: return 'A'; }
}

static inline char substitute(rng_t *r, char c) {
    /* one of the other three bases, uniformly */
    int idx = (c == 'A') ? 0 : (c == 'C') ? 1 : (c == 'G') ? 2 : 3;
    int k = (int)rng_below(r, 3);
    return BASES[(idx + 1 + k) & 3];
}

static int digits10(uint64_t v) { int d = 1; while (v >= 10) { v /= 10; ++d; } return d; }

/* Exact FASTQ size for n reads of length L. */
uint64_t emp_synth_fastq_size(uint64_t n_reads, int32_t read_len) {
    uint64_t total = n_reads * (uint64_t)(2 * read_len + 7);
    uint64_t lo = 0, p = 10; int d = 1;
    while (lo < n_reads) {
        uint64_t hi = p < n_reads ? p : n_reads;
        total += (hi - lo) * (uint64_t)d;
        lo = hi; p *= 10; ++d;
    }
    return total;
}

static uint64_t record_offset(uint64_t i, int32_t L) { return emp_synth_fastq_size(i, L); }

/* Fill genome[0..G) (ASCII ACGT) including repeat families.  Returns 0 on success. */
int emp_synth_genome(const emp_synth_params *p, char *genome) {
    uint64_t G = p->genome_len;
    rng_t r; rng_seed(&r, p->seed, 0xFFFFFFFFull);
    uint64_t i = 0;
    while (i < G) {
        uint64_t w = rng_next(&r);
        for (int k = 0; k < 32 && i < G; ++k, ++i, w >>= 2) genome[i] = BASES[w & 3];
    }
    if (p->repeat_frac > 0.0 && p->rep_max_len > 0 && (uint64_t)p->rep_max_len < G) {
        uint64_t target = (uint64_t)(p->repeat_frac * (double)G), covered = 0;
        char *fam = (char *)malloc((size_t)p->rep_max_len);
        if (!fam) return -1;
        rng_t rr; rng_seed(&rr, p->seed, 0xFFFFFFFEull);
        while (covered < target) {
            int32_t len = p->rep_min_len + (int32_t)rng_below(&rr, (uint64_t)(p->rep_max_len - p->rep_min_len + 1));
            int32_t copies = p->rep_min_copies + (int32_t)rng_below(&rr, (uint64_t)(p->rep_max_copies - p->rep_min_copies + 1));
            for (int32_t j = 0; j < len; ++j) fam[j] = BASES[rng_below(&rr, 4)];
            for (int32_t c = 0; c < copies && covered < target; ++c) {
                uint64_t pos = rng_below(&rr, G - (uint64_t)len + 1);
                for (int32_t j = 0; j < len; ++j) {
                    char b = fam[j];
                    if (rng_unit(&rr) < p->rep_divergence) b = substitute(&rr, b);
                    genome[pos + (uint64_t)j] = b;
                }
                covered += (uint64_t)len;
            }
        }
        free(fam);
    }
    return 0;
}

/* Write the FASTQ for p into out (cap bytes).  Returns bytes written, or 0 on error. */
uint64_t emp_synth_fastq(const emp_synth_params *p, char *out, uint64_t cap) {
    const int32_t L = p->read_len;
    const uint64_t G = p->genome_len, n = p->n_reads;
    if (L <= 0 || G < (uint64_t)L) return 0;
    uint64_t need = emp_synth_fastq_size(n, L);
    if (cap < need) return 0;
    char *genome = (char *)malloc((size_t)G);
    if (!genome) return 0;
    if (emp_synth_genome(p, genome) != 0) { free(genome); return 0; }
    const uint64_t nchunks = (n + EMP_SYNTH_CHUNK - 1) / EMP_SYNTH_CHUNK;
#ifdef _OPENMP
    int nt = p->n_threads > 0 ? p->n_threads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
#endif
    for (long long c = 0; c < (long long)nchunks; ++c) {
        rng_t r; rng_seed(&r, p->seed, (uint64_t)c);
        char *seq = (char *)malloc((size_t)L);
        uint64_t i0 = (uint64_t)c * EMP_SYNTH_CHUNK;
        uint64_t i1 = i0 + EMP_SYNTH_CHUNK < n ? i0 + EMP_SYNTH_CHUNK : n;
        char *o = out + record_offset(i0, L);
        for (uint64_t i = i0; i < i1; ++i) {
            uint64_t start = rng_below(&r, G - (uint64_t)L + 1);
            memcpy(seq, genome + start, (size_t)L);
            if (p->sub_rate > 0.0)
                for (int32_t j = 0; j < L; ++j)
                    if (rng_unit(&r) < p->sub_rate) seq[j] = substitute(&r, seq[j]);
            if (rng_unit(&r) < p->rc_prob) {
                for (int32_t j = 0, k = L - 1; j < k; ++j, --k) {
                    char a = seq[j]; seq[j] = complement(seq[k]); seq[k] = complement(a);
                }
                if (L & 1) seq[L / 2] = complement(seq[L / 2]);
            }
            *o++ = '@'; *o++ = 'r';
            int d = digits10(i);
            uint64_t v = i;
            for (int k = d - 1; k >= 0; --k) { o[k] = (char)('0' + v % 10); v /= 10; }
            o += d;
            *o++ = '\n';
            memcpy(o, seq, (size_t)L); o += L;
            *o++ = '\n'; *o++ = '+'; *o++ = '\n';
            memset(o, 'I', (size_t)L); o += L;
            *o++ = '\n';
        }
        free(seq);
    }
    free(genome);
    return need;
}
