/*
 * oracle_main.c -- command-line front end of the CPU restatement (test
 * infrastructure).  Same positional arguments and short options as the
 * reference (config.h:120-140); -m/-b/-c are accepted and ignored because
 * they never change output.bin.
 *
 *   empanada_oracle input.fastq output.bin [-o N] [-m SIZE] [-r SIZE] [-b SIZE] [-c SIZE]
 */
#include "empanada_oracle.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static uint64_t parse_size(const char *s) {
    char *end = NULL;
    uint64_t v = strtoull(s, &end, 10);
    switch (*end) {
    case 'k': case 'K': v <<= 10; break;
    case 'm': case 'M': v <<= 20; break;
    case 'g': case 'G': v <<= 30; break;
    default: break;
    }
    return v;
}

int main(int argc, char **argv) {
    const char *pos[2] = {NULL, NULL};
    int npos = 0;
    int32_t o = 31;
    uint64_t r = 1ull << 30;
    for (int i = 1; i < argc; ++i) {
        if (argv[i][0] == '-' && argv[i][1] && i + 1 < argc) {
            char f = argv[i][1];
            const char *v = argv[++i];
            if (f == 'o') o = (int32_t)parse_size(v);
            else if (f == 'r') r = parse_size(v);
            continue;
        }
        if (npos < 2) pos[npos++] = argv[i];
    }
    if (npos < 2) {
        fprintf(stderr, "usage: empanada_oracle input.fastq output.bin [-o N] [-r SIZE]\n");
        return 2;
    }
    FILE *f = fopen(pos[0], "rb");
    char *buf = NULL;
    size_t len = 0;
    if (f) {
        fseek(f, 0, SEEK_END);
        long sz = ftell(f);
        fseek(f, 0, SEEK_SET);
        buf = (char *)malloc(sz > 0 ? (size_t)sz : 1);
        len = fread(buf, 1, (size_t)(sz > 0 ? sz : 0), f);
        fclose(f);
    } else {
        buf = (char *)malloc(1);
    }
    uint8_t *out = NULL;
    size_t out_len = 0;
    emp_oracle_stats st;
    int rc = emp_oracle_run(buf, len, o, r, &out, &out_len, &st);
    free(buf);
    if (rc) {
        fprintf(stderr, "empanada_oracle: error %d\n", rc);
        return 1;
    }
    FILE *g = fopen(pos[1], "wb");
    if (!g) {
        fprintf(stderr, "empanada_oracle: cannot open %s\n", pos[1]);
        return 1;
    }
    if (out_len) fwrite(out, 1, out_len, g);
    fclose(g);
    printf("reads=%llu L=%d unique=%llu rounds=%d edges=%llu records=%llu\n", (unsigned long long)st.n_reads,
           st.read_len, (unsigned long long)st.n_unique, st.n_rounds, (unsigned long long)st.n_edges,
           (unsigned long long)st.n_records);
    emp_oracle_free(out);
    return 0;
}
