/*
 * graph_oracle.c -- CPU restatement of the unitig layer over output.bin
 * (test infrastructure: the checker of emp_graph_* in the CUDA library).
 *
 * Read-ends 0 .. 2n-1 are the nodes and the records' (from, to) pairs the
 * edges of the overlap graph that output.bin describes (records as written
 * by write_edges_binary, overlap.cu:148-161).  A unitig is a maximal path of
 * edges u -> v with out-degree(u) = in-degree(v) = 1; a cycle of such edges
 * is cut before its smallest read-end; every read-end is in exactly one
 * unitig.  The GFA text follows the layout the reference's dead writers
 * sketch (overlap.cu:129-190) with the read index rid / 2 and the
 * orientation of rid's low bit: a header, S per read, L per edge in file
 * order, P per unitig of two or more read-ends ordered by their first
 * read-end.  Walked serially, node by node.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define NONE 0xffffffffu

typedef struct {
    char *p;
    size_t n, cap;
} sbuf;

static int sb_put(sbuf *b, const char *s, size_t l) {
    if (b->n + l + 1 > b->cap) {
        size_t c = b->cap ? b->cap : 4096;
        while (c < b->n + l + 1) c *= 2;
        char *q = realloc(b->p, c);
        if (!q) return -1;
        b->p = q;
        b->cap = c;
    }
    memcpy(b->p + b->n, s, l);
    b->n += l;
    return 0;
}

static int sb_fmt(sbuf *b, const char *fmt, unsigned long long x, unsigned long long y) {
    char t[96];
    int l = snprintf(t, sizeof t, fmt, x, y);
    return sb_put(b, t, (size_t)l);
}

/* Unitigs of the graph: order[] read-ends in unitig order, starts[] the
 * first position of each unitig (count + 1 entries), ordered by first
 * read-end.  Returns 0, or -1 on a bad record / an edge beyond 2n. */
int emp_oracle_unitigs(const uint8_t *bin, size_t bytes, uint64_t n_reads, uint32_t *order, uint64_t *starts,
                       uint64_t *n_unitigs) {
    const uint64_t V = 2 * n_reads;
    uint32_t *dout = calloc(V ? V : 1, 4), *din = calloc(V ? V : 1, 4);
    uint32_t *succ = malloc((V ? V : 1) * 4), *pred = malloc((V ? V : 1) * 4);
    uint8_t *seen = calloc(V ? V : 1, 1);
    int rc = 0;
    if (!dout || !din || !succ || !pred || !seen) rc = -1;
    for (uint64_t u = 0; rc == 0 && u < V; ++u) succ[u] = pred[u] = NONE;
    for (int pass = 0; rc == 0 && pass < 2; ++pass) {  /* degrees, then the unitig edges */
        for (size_t o = 0; o < bytes;) {
            uint64_t n;
            if (o + 12 > bytes) { rc = -1; break; }
            memcpy(&n, bin + o, 8);
            if (n > (bytes - o - 12) / 8) { rc = -1; break; }
            for (uint64_t k = 0; k < n; ++k) {
                uint32_t u, v;
                memcpy(&u, bin + o + 12 + 4 * k, 4);
                memcpy(&v, bin + o + 12 + 4 * (n + k), 4);
                if (u >= V || v >= V) { rc = -1; break; }
                if (pass == 0) {
                    dout[u]++;
                    din[v]++;
                } else if (dout[u] == 1 && din[v] == 1) {
                    succ[u] = v;
                    pred[v] = u;
                }
            }
            o += 12 + 8 * n;
        }
    }
    /* heads: read-ends without a predecessor, and the smallest read-end of
       every cycle (a cycle's read-ends all have one) */
    uint8_t *head = calloc(V ? V : 1, 1);
    if (!head) rc = -1;
    for (uint64_t u = 0; rc == 0 && u < V; ++u)
        if (pred[u] == NONE) {
            head[u] = 1;
            for (uint32_t x = (uint32_t)u; x != NONE; x = succ[x]) seen[x] = 1;
        }
    for (uint64_t u = 0; rc == 0 && u < V; ++u)
        if (!seen[u]) {  /* on a cycle: u is its smallest unseen read-end, as u ascends */
            head[u] = 1;
            uint32_t x = (uint32_t)u;
            do {
                seen[x] = 1;
                x = succ[x];
            } while (x != (uint32_t)u);
        }
    uint64_t pos = 0, cnt = 0;
    for (uint64_t u = 0; rc == 0 && u < V; ++u) {
        if (!head[u]) continue;
        starts[cnt++] = pos;
        uint32_t x = (uint32_t)u;
        do {
            order[pos++] = x;
            x = succ[x];
        } while (x != NONE && x != (uint32_t)u);
    }
    if (rc == 0) {
        starts[cnt] = pos;
        *n_unitigs = cnt;
        if (pos != V) rc = -1;
    }
    free(dout);
    free(din);
    free(succ);
    free(pred);
    free(seen);
    free(head);
    return rc;
}

/* The GFA text (malloc'd, *len bytes); 0 or -1. */
int emp_oracle_gfa(const uint8_t *bin, size_t bytes, uint64_t n_reads, int32_t read_len, char **text, size_t *len) {
    const uint64_t V = 2 * n_reads;
    uint32_t *order = malloc((V ? V : 1) * 4);
    uint64_t *starts = malloc((V + 1) * 8), nu = 0;
    sbuf b = {0, 0, 0};
    int rc = (order && starts) ? emp_oracle_unitigs(bin, bytes, n_reads, order, starts, &nu) : -1;
    if (rc == 0) rc = sb_put(&b, "H\tVN:Z:1.0\n", 11);
    for (uint64_t i = 0; rc == 0 && i < n_reads; ++i) rc = sb_fmt(&b, "S\t%llu\t*\tLN:i:%llu\n", i, (unsigned long long)read_len);
    for (size_t o = 0; rc == 0 && o < bytes;) {
        uint64_t n;
        int32_t ovlp;
        memcpy(&n, bin + o, 8);
        memcpy(&ovlp, bin + o + 8, 4);
        for (uint64_t k = 0; rc == 0 && k < n; ++k) {
            uint32_t u, v;
            char t[96];
            memcpy(&u, bin + o + 12 + 4 * k, 4);
            memcpy(&v, bin + o + 12 + 4 * (n + k), 4);
            int l = snprintf(t, sizeof t, "L\t%u\t%c\t%u\t%c\t%dM\n", u >> 1, (u & 1) ? '-' : '+', v >> 1,
                             (v & 1) ? '-' : '+', ovlp < 0 ? 0 : ovlp);
            rc = sb_put(&b, t, (size_t)l);
        }
        o += 12 + 8 * n;
    }
    uint64_t k = 0;
    for (uint64_t q = 0; rc == 0 && q < nu; ++q) {
        if (starts[q + 1] - starts[q] < 2) continue;
        rc = sb_fmt(&b, "P\tutg%llu\t", k++, 0);
        for (uint64_t x = starts[q]; rc == 0 && x < starts[q + 1]; ++x) {
            char t[32];
            int l = snprintf(t, sizeof t, "%s%u%c", x == starts[q] ? "" : ",", order[x] >> 1, (order[x] & 1) ? '-' : '+');
            rc = sb_put(&b, t, (size_t)l);
        }
        if (rc == 0) rc = sb_put(&b, "\t*\n", 3);
    }
    free(order);
    free(starts);
    if (rc != 0) {
        free(b.p);
        return -1;
    }
    *text = b.p ? b.p : calloc(1, 1);
    *len = b.n;
    return 0;
}
