/*
 * empanada_oracle.c -- CPU restatement of empanada's read-overlap path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path (see
 * empanada_oracle.h).  Plain C, single thread, no dependence on the product.
 *
 * Each function restates one piece of the reference (file:line into the
 * reference project):
 *   parse            preprocess.cu:26-237 (parseLines, resizeBuffer,
 *                    extractReads, removeLQReads, read_block) on the whole
 *                    file; the reference's -m blocking is transparent for
 *                    well-formed FASTQ, so it is not modelled.
 *   hash             fingerprint.cu:26-115 (precomputeModulos, FingerprintMul,
 *                    EncodeBases, generate_fingerprint_read_pairs) and
 *                    assembly.cuh:29-34,50-52 (primes, radices, ENCODING, APPEND64)
 *   next_sfx         overlap.cu:57-75 (NextSfx)
 *   prev_pfx         overlap.cu:77-91 (PrevPfx), overlap.cu:30-39,121-122 (inverses)
 *   fp_sort          cqutils.cuh:180-247 (cq_sort_by_key) with
 *                    cqutils.cuh:140-177 (cq_merge_by_key) and
 *                    cqutils.cuh:37-84 (cq_get_merge_partitions)
 *   dedup            cqutils.cuh:272-306 (cq_unique_by_key), 87-105 (cq_get_partitions)
 *   regen            overlap.cu:605-692 (regenerate_fingerprints, filter_bases)
 *   emit             overlap.cu:361-456 (emit_edges), 557-603 (get_edges),
 *                    694-710 (remove_used), cqutils.cuh:108-137
 *                    (cq_get_search_partitions), overlap.cu:148-161
 *                    (write_edges_binary)
 *   run              overlap.cu:206-293 (build_graph), main.cu:9-77
 *
 * Inputs on which the reference loops forever (a run of >= M equal keys in
 * cq_get_partitions, or a (0,0) search partition) return EMP_ORACLE_E_HANG.
 * Inputs on which the reference's result is undefined (unequal read lengths,
 * bases outside ACGTacgt that survive the N filter) return EMP_ORACLE_E_FORMAT;
 * reads longer than 512 return EMP_ORACLE_E_UNSUPPORTED (lengths 256-512 are
 * the reference's undefined range, extended with the same exact hash).
 * emp_oracle_run_var is the variable-length extension of the same run (the
 * reference requires equal lengths, fingerprint.cu:134-135): it defines the
 * result for reads of unequal length and equals emp_oracle_run when every
 * read has the same length.
 */
#include "empanada_oracle.h"

#include <limits.h>
#include <stdlib.h>
#include <string.h>

#define PRIME1 536870909u
#define PRIME2 536870879u
#define RADIX1 5u
#define RADIX2 7u
/* The reference's MAX_RD_LEN (assembly.cuh:17) is 255; beyond it its u8
 * lengths and 256-entry power tables overflow and its result is undefined.
 * This restatement carries the same exact hash on to 512 bases (the CUDA
 * path's limit), so reads of 256-512 bases are checked against it alone. */
#define MAX_RD_LEN 512

static uint32_t MOD1[MAX_RD_LEN + 1], MOD2[MAX_RD_LEN + 1];
static uint32_t INV1, INV2;
static int tables_ready;

/* R^(e) mod p by square-and-multiply in 64-bit (overlap.cu:30-39) */
static uint32_t mod_pow(uint64_t a, uint32_t e, uint32_t p) {
    uint64_t r = 1;
    while (e) {
        if (e & 1) r = (r * a) % p;
        a = (a * a) % p;
        e >>= 1;
    }
    return (uint32_t)r;
}

static void init_tables(void) {
    if (tables_ready) return;
    MOD1[0] = MOD2[0] = 1;
    for (int i = 1; i <= MAX_RD_LEN; ++i) {
        MOD1[i] = (uint32_t)(((uint64_t)MOD1[i - 1] * RADIX1) % PRIME1);
        MOD2[i] = (uint32_t)(((uint64_t)MOD2[i - 1] * RADIX2) % PRIME2);
    }
    INV1 = mod_pow(RADIX1, PRIME1 - 2, PRIME1);
    INV2 = mod_pow(RADIX2, PRIME2 - 2, PRIME2);
    tables_ready = 1;
}

/* ENCODING(c) = ((c >> 1) & 3) + 1: A1 C2 T3 G4 (assembly.cuh:34) */
static inline uint32_t enc(char c) { return ((((unsigned char)c) >> 1) & 3u) + 1u; }

/* Watson-Crick complement as the reference's revc table (preprocess.cu:18) */
static inline char comp(char c) {
    static const char revc[8] = {0, 'T', 0, 'G', 'A', 0, 0, 'C'};
    return revc[((unsigned char)c) & 7];
}

static inline int is_acgt(char c) {
    switch (c) {
    case 'A': case 'C': case 'G': case 'T': case 'a': case 'c': case 'g': case 't': return 1;
    default: return 0;
    }
}

uint32_t emp_oracle_radix_inv(int which) {
    init_tables();
    return which == 1 ? INV1 : INV2;
}

/* Horner form of the associative FingerprintMul scan (fingerprint.cu:36-57,90) */
uint64_t emp_oracle_hash(const char *s, int32_t len) {
    uint64_t h1 = 0, h2 = 0;
    for (int32_t j = 0; j < len; ++j) {
        h1 = (h1 * RADIX1 + enc(s[j])) % PRIME1;
        h2 = (h2 * RADIX2 + enc(s[j])) % PRIME2;
    }
    return (h1 << 32) | h2;
}

/* NextSfx (overlap.cu:57-75): drop the first base of a length-len suffix.
 * The product enc * R^(len-1) is a 32-bit unsigned product (< 2^31). */
uint64_t emp_oracle_next_sfx(uint64_t key, char base, int32_t len) {
    init_tables();
    uint64_t fp1 = key >> 32, fp2 = key & 0xffffffffu;
    uint32_t e = enc(base);
    fp1 = (fp1 + PRIME1 - (uint32_t)(e * MOD1[len - 1]) % PRIME1) % PRIME1;
    fp2 = (fp2 + PRIME2 - (uint32_t)(e * MOD2[len - 1]) % PRIME2) % PRIME2;
    return (fp1 << 32) | fp2;
}

/* PrevPfx (overlap.cu:77-91): drop the last base.  The subtraction and the
 * product are wrapping 64-bit arithmetic, exactly as in the reference
 * (fp < enc wraps and is then reduced mod p). */
uint64_t emp_oracle_prev_pfx(uint64_t key, char base) {
    init_tables();
    uint64_t fp1 = key >> 32, fp2 = key & 0xffffffffu;
    uint64_t e = enc(base);
    fp1 = ((uint64_t)INV1 * (fp1 - e)) % PRIME1;
    fp2 = ((uint64_t)INV2 * (fp2 - e)) % PRIME2;
    return (fp1 << 32) | fp2;
}

void emp_oracle_free(void *p) { free(p); }

/* ------------------------------------------------------------------ parse */

/* preprocess.cu:26-237 on the whole file.  Line g is the g-th '\n'-terminated
 * line (the last may be unterminated); record k's sequence is line 4k+1
 * (extractReads :70-87).  markNs (:119-121) marks each byte; a sequence whose
 * maximum mark is 9 (an N-class byte) is dropped, and '\n' bytes are removed
 * (:146-155); an empty sequence vanishes (:164-167).
 *
 * allow_var keeps reads of unequal length (the variable-length extension);
 * offs_out then receives n + 1 offsets into the concatenated reads (read i is
 * reads[offs[i], offs[i+1])) and L_out the longest length. */
static int parse_core(const char *fq, size_t len, int allow_var, char **reads_out, uint64_t **offs_out,
                      uint64_t *n_out, int32_t *L_out) {
    size_t cap = 1 << 20, used = 0, ocap = 1024;
    char *reads = (char *)malloc(cap);
    uint64_t *offs = allow_var ? (uint64_t *)malloc(ocap * sizeof(uint64_t)) : NULL;
    if (!reads || (allow_var && !offs)) { free(reads); free(offs); return EMP_ORACLE_E_NOMEM; }
    int32_t L = -1;
    uint64_t n = 0, line = 0;
    size_t pos = 0;
    int st = EMP_ORACLE_OK;
    while (pos < len) {
        const char *nl = (const char *)memchr(fq + pos, '\n', len - pos);
        size_t e = nl ? (size_t)(nl - fq) : len;
        if (line % 4 == 1) {
            int maxv = INT_MIN;
            for (size_t j = pos; j < e; ++j) {
                int c = (signed char)fq[j];
                int v = (c >> 6) * (1 + (c & 8));
                if (v > maxv) maxv = v;
            }
            if (e < len && maxv < 0) maxv = 0; /* the terminating '\n' marks 0 */
            size_t sl = e - pos;
            if (maxv != 9 && sl > 0) {
                for (size_t j = pos; j < e; ++j)
                    if (!is_acgt(fq[j])) { st = EMP_ORACLE_E_FORMAT; goto fail; }
                const int32_t sl32 = (int32_t)(sl > (size_t)INT32_MAX ? INT32_MAX : sl);
                if (L < 0) L = sl32;
                if ((size_t)L != sl) {
                    if (!allow_var) { st = EMP_ORACLE_E_FORMAT; goto fail; }
                    if (sl32 > L) L = sl32;
                }
                if (used + sl > cap) {
                    while (used + sl > cap) cap *= 2;
                    char *nr = (char *)realloc(reads, cap);
                    if (!nr) { st = EMP_ORACLE_E_NOMEM; goto fail; }
                    reads = nr;
                }
                if (allow_var) {
                    if (n + 2 > ocap) {
                        ocap *= 2;
                        uint64_t *no = (uint64_t *)realloc(offs, ocap * sizeof(uint64_t));
                        if (!no) { st = EMP_ORACLE_E_NOMEM; goto fail; }
                        offs = no;
                    }
                    offs[n] = used;
                }
                memcpy(reads + used, fq + pos, sl);
                used += sl;
                ++n;
            }
        }
        ++line;
        pos = e + 1;
    }
    /* format errors anywhere in the file take precedence over the length limit */
    if (n && L > MAX_RD_LEN) { st = EMP_ORACLE_E_UNSUPPORTED; goto fail; }
    if (allow_var) {
        offs[n] = used;
        *offs_out = offs;
    }
    *reads_out = reads;
    *n_out = n;
    *L_out = n ? L : 0;
    return EMP_ORACLE_OK;
fail:
    free(reads);
    free(offs);
    return st;
}

int emp_oracle_parse(const char *fq, size_t len, char **reads_out, uint64_t *n_out, int32_t *L_out) {
    return parse_core(fq, len, 0, reads_out, NULL, n_out, L_out);
}

/* The kept reads: n reads of L bases back to back, or (off != NULL) read i at
 * base + off[i] with off[i+1] - off[i] bases. */
typedef struct {
    const char *base;
    const uint64_t *off;
    int32_t L;
} readset_t;

static inline const char *rs_read(const readset_t *rs, uint64_t i) {
    return rs->off ? rs->base + rs->off[i] : rs->base + i * (uint64_t)rs->L;
}
static inline int32_t rs_len(const readset_t *rs, uint64_t i) {
    return rs->off ? (int32_t)(rs->off[i + 1] - rs->off[i]) : rs->L;
}

/* hash of read i (rid 2i) and of its reverse complement (rid 2i+1);
 * fingerprint.cu:75-115 interleaves forward and RC line ids, so rid = 2i+s. */
static void fingerprints_of(const readset_t *rs, uint64_t n, uint64_t *keys) {
    char rc[MAX_RD_LEN + 1];
    for (uint64_t i = 0; i < n; ++i) {
        const char *s = rs_read(rs, i);
        const int32_t L = rs_len(rs, i);
        for (int32_t j = 0; j < L; ++j) rc[j] = comp(s[L - 1 - j]);
        keys[2 * i] = emp_oracle_hash(s, L);
        keys[2 * i + 1] = emp_oracle_hash(rc, L);
    }
}

int emp_oracle_fingerprints(const char *fq, size_t len, uint64_t *keys, uint64_t cap, uint64_t *n_out,
                            int32_t *L_out) {
    char *reads = NULL;
    uint64_t n = 0;
    int32_t L = 0;
    int st = emp_oracle_parse(fq, len, &reads, &n, &L);
    if (st) return st;
    *n_out = n;
    *L_out = L;
    if (2 * n > cap) { free(reads); return EMP_ORACLE_E_INVAL; }
    const readset_t rs = {reads, NULL, L};
    fingerprints_of(&rs, n, keys);
    free(reads);
    return EMP_ORACLE_OK;
}

/* ------------------------------------------------------------- tables */

typedef struct { uint64_t *k; uint32_t *v; size_t n, cap; } table_t;

static int tab_reserve(table_t *t, size_t cap) {
    if (cap <= t->cap) return 0;
    uint64_t *k = (uint64_t *)realloc(t->k, (cap ? cap : 1) * sizeof(uint64_t));
    if (!k) return -1;
    t->k = k;
    uint32_t *v = (uint32_t *)realloc(t->v, (cap ? cap : 1) * sizeof(uint32_t));
    if (!v) return -1;
    t->v = v;
    t->cap = cap;
    return 0;
}
static void tab_free(table_t *t) { free(t->k); free(t->v); t->k = NULL; t->v = NULL; t->n = t->cap = 0; }
static int tab_append(table_t *t, const uint64_t *k, const uint32_t *v, size_t n) {
    if (tab_reserve(t, t->n + n)) return -1;
    memcpy(t->k + t->n, k, n * sizeof(uint64_t));
    memcpy(t->v + t->n, v, n * sizeof(uint32_t));
    t->n += n;
    return 0;
}

/* Stable LSD radix sort of (key, value) pairs by key (11-bit digits; passes
 * whose digit is constant are skipped).  by_value sorts by the value instead
 * (used for the read-id sorts). */
static uint64_t *g_tk;
static uint32_t *g_tv;
static size_t g_tcap;
static int scratch_reserve(size_t n) {
    if (n <= g_tcap) return 0;
    uint64_t *k = (uint64_t *)realloc(g_tk, n * sizeof(uint64_t));
    if (!k) return -1;
    g_tk = k;
    uint32_t *v = (uint32_t *)realloc(g_tv, n * sizeof(uint32_t));
    if (!v) return -1;
    g_tv = v;
    g_tcap = n;
    return 0;
}

static int radix_sort(uint64_t *k, uint32_t *v, size_t n, int by_value) {
    if (n < 2) return 0;
    if (scratch_reserve(n)) return -1;
    static size_t cnt[2048];
    uint64_t *sk = k, *dk = g_tk;
    uint32_t *sv = v, *dv = g_tv;
    int bits = by_value ? 32 : 64;
    for (int shift = 0; shift < bits; shift += 11) {
        memset(cnt, 0, sizeof cnt);
        for (size_t i = 0; i < n; ++i) {
            uint64_t x = by_value ? sv[i] : sk[i];
            cnt[(x >> shift) & 2047]++;
        }
        int constant = 0;
        for (int d = 0; d < 2048; ++d)
            if (cnt[d] == n) { constant = 1; break; }
        if (constant) continue;
        size_t s = 0;
        for (int d = 0; d < 2048; ++d) { size_t c = cnt[d]; cnt[d] = s; s += c; }
        for (size_t i = 0; i < n; ++i) {
            uint64_t x = by_value ? sv[i] : sk[i];
            size_t o = cnt[(x >> shift) & 2047]++;
            dk[o] = sk[i];
            dv[o] = sv[i];
        }
        uint64_t *tk = sk; sk = dk; dk = tk;
        uint32_t *tv = sv; sv = dv; dv = tv;
    }
    if (sk != k) {
        memcpy(k, sk, n * sizeof(uint64_t));
        memcpy(v, sv, n * sizeof(uint32_t));
    }
    return 0;
}

static size_t lower_bound(const uint64_t *a, size_t lo, size_t hi, uint64_t key) {
    while (lo < hi) {
        size_t m = lo + (hi - lo) / 2;
        if (a[m] < key) lo = m + 1; else hi = m;
    }
    return lo;
}
static size_t upper_bound(const uint64_t *a, size_t lo, size_t hi, uint64_t key) {
    while (lo < hi) {
        size_t m = lo + (hi - lo) / 2;
        if (key < a[m]) hi = m; else lo = m + 1;
    }
    return lo;
}

typedef struct { size_t a, b; } part_t;
typedef struct { part_t *p; size_t n, cap; } parts_t;
static int parts_push(parts_t *ps, size_t a, size_t b) {
    if (ps->n == ps->cap) {
        size_t c = ps->cap ? 2 * ps->cap : 16;
        part_t *p = (part_t *)realloc(ps->p, c * sizeof(part_t));
        if (!p) return -1;
        ps->p = p;
        ps->cap = c;
    }
    ps->p[ps->n].a = a;
    ps->p[ps->n].b = b;
    ps->n++;
    return 0;
}

/* cq_get_merge_partitions (cqutils.cuh:37-84) */
static int merge_partitions(const table_t *A, const table_t *B, size_t M, parts_t *ps) {
    const size_t nA = A->n, nB = B->n, h = M / 2;
    size_t offA = 0, offB = 0;
    while (offA < nA && offB < nB) {
        size_t pa = nA - offA < h ? nA - offA : h, pb = nB - offB < h ? nB - offB : h;
        if (pa < h && pb < h) {
            if (parts_push(ps, pa, pb)) return -1;
            offA += pa; offB += pb;
            break;
        }
        if (A->k[offA + pa - 1] <= B->k[offB]) {
            if (parts_push(ps, pa, 0)) return -1;
            offA += pa;
        } else if (B->k[offB + pb - 1] <= A->k[offA]) {
            if (parts_push(ps, 0, pb)) return -1;
            offB += pb;
        } else {
            uint64_t la = A->k[offA + pa - 1], lb = B->k[offB + pb - 1];
            if (la < lb) pb = upper_bound(B->k, offB, offB + pb, la) - offB;
            else if (lb < la) pa = upper_bound(A->k, offA, offA + pa, lb) - offA;
            if (parts_push(ps, pa, pb)) return -1;
            offA += pa; offB += pb;
        }
    }
    if (offA == nA && offB < nB) { if (parts_push(ps, 0, nB - offB)) return -1; }
    else if (offB == nB && offA < nA) { if (parts_push(ps, nA - offA, 0)) return -1; }
    return 0;
}

/* cq_merge_by_key (cqutils.cuh:140-177): each two-sided partition is the
 * stable sort of [A part, B part]; one-sided partitions pass through. */
static int merge_tables(table_t *A, table_t *B, size_t M, table_t *C) {
    parts_t ps = {0};
    if (merge_partitions(A, B, M, &ps)) return -1;
    size_t offA = 0, offB = 0;
    if (tab_reserve(C, A->n + B->n)) { free(ps.p); return -1; }
    for (size_t i = 0; i < ps.n; ++i) {
        size_t pa = ps.p[i].a, pb = ps.p[i].b, start = C->n;
        if (tab_append(C, A->k + offA, A->v + offA, pa) || tab_append(C, B->k + offB, B->v + offB, pb)) {
            free(ps.p);
            return -1;
        }
        if (pa && pb && radix_sort(C->k + start, C->v + start, pa + pb, 0)) { free(ps.p); return -1; }
        offA += pa; offB += pb;
    }
    free(ps.p);
    return 0;
}

/* cq_sort_by_key by fingerprint (cqutils.cuh:180-247): one stable sort when
 * N <= M; otherwise stable M-chunk sorts merged pairwise through a FIFO. */
static int fp_sort(table_t *T, size_t M) {
    const size_t N = T->n;
    if (N <= M) return radix_sort(T->k, T->v, N, 0);
    size_t nchunks = (N + M - 1) / M, qcap = 2 * nchunks + 2, head = 0, tail = 0;
    table_t *q = (table_t *)calloc(qcap, sizeof(table_t));
    if (!q) return -1;
    for (size_t off = 0; off < N; off += M) {
        size_t np = N - off < M ? N - off : M;
        table_t c = {0};
        if (tab_append(&c, T->k + off, T->v + off, np) || radix_sort(c.k, c.v, np, 0)) { free(q); return -1; }
        q[tail++] = c;
    }
    while (tail - head > 1) {
        table_t l = q[head++], r = q[head++], o = {0};
        if (merge_tables(&l, &r, M, &o)) { free(q); return -1; }
        tab_free(&l);
        tab_free(&r);
        q[tail++] = o;
    }
    table_t res = q[head];
    free(q);
    tab_free(T);
    *T = res;
    return 0;
}

/* cq_unique_by_key (cqutils.cuh:272-306) with cq_get_partitions (87-105):
 * partitions never split an equal-key run, so the result is "first of each
 * run"; a run of >= M equal keys makes the reference loop forever. */
static int dedup(table_t *T, size_t M) {
    size_t off = 0, n = T->n;
    while (off < n) {
        if (n - off <= M) break;
        size_t np = M;
        np = lower_bound(T->k, off, off + np, T->k[off + np - 1]) - off;
        if (np == 0) return EMP_ORACLE_E_HANG;
        off += np;
    }
    size_t w = 0;
    for (size_t i = 0; i < n; ++i) {
        if (i > 0 && T->k[i] == T->k[i - 1]) continue;
        T->k[w] = T->k[i];
        T->v[w] = T->v[i];
        ++w;
    }
    T->n = w;
    return 0;
}

/* regenerate_fingerprints + filter_bases (overlap.cu:605-692).  Sorted by
 * read-end id, then per M-chunk: even ids (forward read-ends) ascending,
 * then odd ids (reverse complements) ascending.  Going from overlap length
 * ell + 1 to ell, a suffix drops the first base of its read-end (a forward
 * read-end of length len: base len-1-ell of the read; a reverse complement:
 * the complement of base ell) and a prefix its last base (forward: base ell;
 * reverse complement: the complement of base len-1-ell).  With every read of
 * length L and ell = L-1-round these are the reference's columns: suffix
 * round, L-1-round; prefix L-1-round, round. */
static int regen(table_t *T, const readset_t *rs, int32_t ell, size_t M, int sfx) {
    const size_t N = T->n;
    if (radix_sort(T->k, T->v, N, 1)) return -1;
    if (scratch_reserve(N)) return -1;
    for (size_t off = 0; off < N; off += M) {
        size_t np = N - off < M ? N - off : M, w = 0;
        for (int parity = 0; parity < 2; ++parity) {
            for (size_t i = off; i < off + np; ++i) {
                uint32_t rid = T->v[i];
                if ((int)(rid & 1) != parity) continue;
                const char *rd = rs_read(rs, rid / 2);
                const int32_t len = rs_len(rs, rid / 2);
                const int32_t fcol = sfx ? len - 1 - ell : ell, rcol = sfx ? ell : len - 1 - ell;
                char base = parity ? comp(rd[rcol]) : rd[fcol];
                g_tk[w] = sfx ? emp_oracle_next_sfx(T->k[i], base, ell + 1) : emp_oracle_prev_pfx(T->k[i], base);
                g_tv[w] = rid;
                ++w;
            }
        }
        memcpy(T->k + off, g_tk, np * sizeof(uint64_t));
        memcpy(T->v + off, g_tv, np * sizeof(uint32_t));
    }
    return 0;
}

/* cq_get_search_partitions (cqutils.cuh:108-137) */
static int search_partitions(const table_t *A, const table_t *B, size_t M, parts_t *ps) {
    const size_t nA = A->n, nB = B->n, h = M / 2;
    size_t offA = 0, offB = 0;
    while (offA < nA && offB < nB) {
        size_t pa = nA - offA < h ? nA - offA : h, pb = nB - offB < h ? nB - offB : h;
        if (pa < h && pb < h) {
            if (parts_push(ps, pa, pb)) return -1;
            offA += pa; offB += pb;
            break;
        }
        uint64_t la = A->k[offA + pa - 1], lb = B->k[offB + pb - 1];
        uint64_t m = la < lb ? la : lb;
        pa = lower_bound(A->k, offA, offA + pa, m) - offA;
        pb = lower_bound(B->k, offB, offB + pb, m) - offB;
        if (pa == 0 && pb == 0) return EMP_ORACLE_E_HANG;
        if (parts_push(ps, pa, pb)) return -1;
        offA += pa; offB += pb;
    }
    if (offA == nA && offB < nB) { if (parts_push(ps, 0, nB - offB)) return -1; }
    else if (offB == nB && offA < nA) { if (parts_push(ps, nA - offA, 0)) return -1; }
    return 0;
}

typedef struct { uint8_t *p; size_t n, cap; } bytes_t;
static int bytes_put(bytes_t *b, const void *src, size_t n) {
    if (b->n + n > b->cap) {
        size_t c = b->cap ? b->cap : 4096;
        while (c < b->n + n) c *= 2;
        uint8_t *p = (uint8_t *)realloc(b->p, c);
        if (!p) return -1;
        b->p = p;
        b->cap = c;
    }
    memcpy(b->p + b->n, src, n);
    b->n += n;
    return 0;
}

/* emit_edges + get_edges + remove_used + write_edges_binary.  For each
 * two-sided partition: every suffix i (sorted order) pairs with every prefix
 * j of equal key (sorted order); pairs of the same read (from/2 == to/2) are
 * dropped; one record "u64 n, i32 ovlp_len, u32 from[n], u32 to[n]" is
 * written (also when n == 0); suffixes that emitted and prefixes that
 * received an edge leave their tables. */
static int emit(table_t *A, table_t *B, size_t M, int32_t ovlp_len, uint8_t *mark, bytes_t *out,
                uint64_t *n_edges, uint64_t *n_records) {
    parts_t ps = {0};
    int st = search_partitions(A, B, M, &ps);
    if (st) { free(ps.p); return st; }
    table_t nA = {0}, nB = {0};
    uint32_t *from = NULL, *to = NULL;
    size_t ecap = 0;
    size_t offA = 0, offB = 0;
    int rc = 0;
    for (size_t p = 0; p < ps.n && !rc; ++p) {
        size_t pa = ps.p[p].a, pb = ps.p[p].b;
        if (pa && pb) {
            size_t ne = 0;
            for (size_t i = offA; i < offA + pa; ++i) {
                size_t lb = lower_bound(B->k, offB, offB + pb, A->k[i]);
                size_t ub = upper_bound(B->k, offB, offB + pb, A->k[i]);
                for (size_t j = lb; j < ub; ++j) {
                    if (A->v[i] / 2 == B->v[j] / 2) continue;
                    if (ne == ecap) {
                        ecap = ecap ? 2 * ecap : 1024;
                        uint32_t *f2 = (uint32_t *)realloc(from, ecap * 4), *t2;
                        if (!f2) { rc = -1; break; }
                        from = f2;
                        t2 = (uint32_t *)realloc(to, ecap * 4);
                        if (!t2) { rc = -1; break; }
                        to = t2;
                    }
                    from[ne] = A->v[i];
                    to[ne] = B->v[j];
                    ++ne;
                }
                if (rc) break;
            }
            if (rc) break;
            uint64_t n64 = ne;
            if (bytes_put(out, &n64, 8) || bytes_put(out, &ovlp_len, 4) || bytes_put(out, from, ne * 4) ||
                bytes_put(out, to, ne * 4)) { rc = -1; break; }
            *n_edges += ne;
            *n_records += 1;
            for (size_t e = 0; e < ne; ++e) mark[from[e]] |= 1;
            for (size_t e = 0; e < ne; ++e) mark[to[e]] |= 2;
            for (size_t i = offA; i < offA + pa && !rc; ++i)
                if (!(mark[A->v[i]] & 1)) rc = tab_append(&nA, A->k + i, A->v + i, 1);
            for (size_t j = offB; j < offB + pb && !rc; ++j)
                if (!(mark[B->v[j]] & 2)) rc = tab_append(&nB, B->k + j, B->v + j, 1);
            for (size_t e = 0; e < ne; ++e) { mark[from[e]] = 0; mark[to[e]] = 0; }
        } else if (pa) {
            rc = tab_append(&nA, A->k + offA, A->v + offA, pa);
        } else {
            rc = tab_append(&nB, B->k + offB, B->v + offB, pb);
        }
        offA += pa; offB += pb;
    }
    free(from);
    free(to);
    free(ps.p);
    tab_free(A);
    tab_free(B);
    *A = nA;
    *B = nB;
    return rc;
}

/* build_graph (overlap.cu:206-293) after the map phase (main.cu:42-67).
 *
 * allow_var runs the variable-length extension (the reference asserts equal
 * lengths, fingerprint.cu:134-135): the overlap length ell goes from the
 * longest read's L-1 down to min_ovlp, and a read-end of length len joins both
 * tables at ell = len-1 (its first proper suffix and prefix), so a table at
 * ell holds the read-ends longer than ell that have not left it.  Duplicate
 * removal works on the full-length keys of all read-ends, as in the
 * reference.  With every read of one length all read-ends join at ell = L-1
 * and the run is the reference's. */
static int run_core(const char *fq, size_t len, int32_t min_ovlp, uint64_t reduce_mem, int allow_var, uint8_t **out,
                    size_t *out_len, emp_oracle_stats *stats) {
    init_tables();
    emp_oracle_stats local;
    if (!stats) stats = &local;
    memset(stats, 0, sizeof *stats);
    const size_t M = (size_t)(reduce_mem / 16);
    if (M < 2) return EMP_ORACLE_E_INVAL;
    char *reads = NULL;
    uint64_t *offs = NULL;
    uint64_t n = 0;
    int32_t L = 0;
    int st = parse_core(fq, len, allow_var, &reads, &offs, &n, &L);
    if (st) return st;
    stats->n_reads = n;
    stats->read_len = L;
    if (L > 0 && min_ovlp < 0) { free(reads); free(offs); return EMP_ORACLE_E_INVAL; }
    const readset_t rs = {reads, offs, L};

    table_t S = {0}, P = {0}, J = {0};
    bytes_t o = {0};
    uint8_t *mark = NULL;
    int rc = 0;
    size_t next = 0;
    if (tab_reserve(&J, 2 * n)) { rc = EMP_ORACLE_E_NOMEM; goto done; }
    fingerprints_of(&rs, n, J.k);
    for (uint64_t r = 0; r < 2 * n; ++r) J.v[r] = (uint32_t)r;
    J.n = 2 * n;
    /* cq_sort_by_key by read id (overlap.cu:212) leaves the rid order as is */
    if (fp_sort(&J, M)) { rc = EMP_ORACLE_E_NOMEM; goto done; }          /* overlap.cu:213 */
    if ((rc = dedup(&J, M)) != 0) goto done;                             /* overlap.cu:222 */
    stats->n_unique = J.n;
    if (allow_var) { /* joining order: longest read-ends first (a counting sort by length) */
        static size_t at[MAX_RD_LEN + 2];
        memset(at, 0, sizeof at);
        for (size_t i = 0; i < J.n; ++i) at[MAX_RD_LEN - rs_len(&rs, J.v[i] / 2) + 1]++;
        for (int c = 1; c <= MAX_RD_LEN + 1; ++c) at[c] += at[c - 1];
        table_t K = {0};
        if (tab_reserve(&K, J.n)) { tab_free(&K); rc = EMP_ORACLE_E_NOMEM; goto done; }
        for (size_t i = 0; i < J.n; ++i) {
            const size_t d = at[MAX_RD_LEN - rs_len(&rs, J.v[i] / 2)]++;
            K.k[d] = J.k[i];
            K.v[d] = J.v[i];
        }
        K.n = J.n;
        tab_free(&J);
        J = K;
    }
    mark = (uint8_t *)calloc(2 * n + 1, 1);
    if (!mark) { rc = EMP_ORACLE_E_NOMEM; goto done; }
    for (int32_t ell = L - 1, round = 0; ell >= min_ovlp; --ell, ++round) {
        /* read-ends of length ell+1 join (all of them at ell = L-1 when lengths are equal; :241-242) */
        size_t end = next;
        while (end < J.n && (!allow_var || rs_len(&rs, J.v[end] / 2) == ell + 1)) ++end;
        if (end > next && (tab_append(&S, J.k + next, J.v + next, end - next) ||
                           tab_append(&P, J.k + next, J.v + next, end - next))) { rc = EMP_ORACLE_E_NOMEM; goto done; }
        next = end;
        int more = 0; /* read-ends still to join at some ell' >= min_ovlp */
        if (next < J.n) more = rs_len(&rs, J.v[next] / 2) - 1 >= min_ovlp;
        if (S.n == 0 && !more) break;
        if (round < EMP_ORACLE_MAX_ROUNDS) {
            stats->sfx_live[round] = S.n;
            stats->pfx_live[round] = P.n;
        }
        uint64_t e0 = stats->n_edges;
        if (regen(&S, &rs, ell, M, 1) || regen(&P, &rs, ell, M, 0)) { rc = EMP_ORACLE_E_NOMEM; goto done; }
        if (fp_sort(&S, M) || fp_sort(&P, M)) { rc = EMP_ORACLE_E_NOMEM; goto done; }
        rc = emit(&S, &P, M, ell, mark, &o, &stats->n_edges, &stats->n_records);
        if (rc) { if (rc < 0 && rc != EMP_ORACLE_E_HANG) rc = EMP_ORACLE_E_NOMEM; goto done; }
        if (round < EMP_ORACLE_MAX_ROUNDS) stats->edges[round] = stats->n_edges - e0;
        stats->n_rounds = round + 1;
    }
done:
    free(reads);
    free(offs);
    free(mark);
    tab_free(&S);
    tab_free(&P);
    tab_free(&J);
    if (rc) { free(o.p); return rc; }
    *out = o.p;
    *out_len = o.n;
    return EMP_ORACLE_OK;
}

int emp_oracle_run(const char *fq, size_t len, int32_t min_ovlp, uint64_t reduce_mem, uint8_t **out, size_t *out_len,
                   emp_oracle_stats *stats) {
    return run_core(fq, len, min_ovlp, reduce_mem, 0, out, out_len, stats);
}

int emp_oracle_run_var(const char *fq, size_t len, int32_t min_ovlp, uint64_t reduce_mem, uint8_t **out,
                       size_t *out_len, emp_oracle_stats *stats) {
    return run_core(fq, len, min_ovlp, reduce_mem, 1, out, out_len, stats);
}
