/*
 * cof_oracle_cli.c -- command-line front of the CPU restatement.
 *
 * TEST INFRASTRUCTURE ONLY.  Reads a cas-offinder input file like
 * cas-offinder-cli/src/cli_utils.rs:37-148 and writes the 8-column output of
 * cas-offinder-cli/src/main.rs:130-242 (header + rows, rows in batch order).
 *
 *   cof_oracle {input|-} {C|G|A} {output|-}
 *
 * C uses the CPU batch size (64 chunks, search.rs:21), G/A the GPU batch size
 * (16384 chunks, search.rs:22); the arithmetic is the CPU path's in both.
 */
#define _GNU_SOURCE
#include "cof_oracle.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static int is_mixed(char c) {
    static const char *ok = "ACGTRYSWKMBDHVNacgtryswkmbdhvn";
    return c && strchr(ok, c) != NULL;
}
static int is_mixed_str(const char *s) {
    for (; *s; s++) if (!is_mixed(*s)) return 0;
    return 1;
}

static void die(const char *msg) {
    fprintf(stderr, "error: %s\n", msg);
    exit(1);
}

/* split_ascii_whitespace into at most 8 parts */
static int split_ws(char *line, char **parts, int maxp) {
    int n = 0;
    char *p = line;
    while (*p) {
        while (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r' || *p == '\f') p++;
        if (!*p) break;
        if (n < maxp) parts[n] = p;
        n++;
        while (*p && !(*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r' || *p == '\f')) p++;
        if (*p) *p++ = 0;
    }
    return n;
}

static int parse_u32(const char *s, uint32_t *v) {
    if (!*s) return -1;
    unsigned long long x = 0;
    for (const char *q = s; *q; q++) {
        if (*q < '0' || *q > '9') return -1;
        x = x * 10 + (unsigned)(*q - '0');
        if (x > 0xFFFFFFFFull) return -1;
    }
    *v = (uint32_t)x;
    return 0;
}

int main(int argc, char **argv) {
    if (argc < 4) die("Too few arguments, expected 3 arguments");
    FILE *in = strcmp(argv[1], "-") ? fopen(argv[1], "rb") : stdin;
    if (!in) die("cannot open input file");
    if (strlen(argv[2]) != 1 || !strchr("CGA", argv[2][0]))
        die("2nd argument must be one of {C|G|A}");
    char *line = NULL;
    size_t cap = 0;
    ssize_t got;
    char *genome = NULL, *filter = NULL;
    uint32_t db = 0, rb = 0, mm = 0;
    int have_mm = 0, use_info = -1;
    char **pats = NULL;
    size_t np = 0;
    int lineno = 0;
    while ((got = getline(&line, &cap, in)) >= 0) {
        size_t len = (size_t)got;
        if (len && line[len - 1] == '\n') {
            line[--len] = 0;
            if (len && line[len - 1] == '\r') line[--len] = 0;
        }
        lineno++;
        if (lineno == 1) { genome = strdup(line); continue; }
        char *parts[8];
        int n = split_ws(line, parts, 8);
        if (lineno == 2) {
            if (n == 1) { filter = strdup(parts[0]); }
            else if (n == 3) {
                filter = strdup(parts[0]);
                if (parse_u32(parts[1], &db)) die("bulge_dna must be a non-negative integer");
                if (parse_u32(parts[2], &rb)) die("bulge_rna must be a non-negative integer");
            } else die("2nd line must be: <search_filter> [<bulge_dna> <bulge_rna>]");
            if (!is_mixed_str(filter)) die("Pattern in input file needs to be a mixed base string");
            continue;
        }
        if (n != 2 && n != 3)
            die("Pattern line must have following elements: <patterns> <mismatches> [<label>]");
        if (!is_mixed_str(parts[0])) die("Pattern in input file needs to be a mixed base string");
        uint32_t cur;
        if (parse_u32(parts[1], &cur))
            die("2nd element of each pattern in mismatches must be an unsigned integer");
        if (!have_mm) { mm = cur; have_mm = 1; }
        if (use_info < 0) use_info = n == 3;
        if (mm != cur)
            die("In this version of cas-offinder, all mismatches on every line of input file must be the same");
        if (use_info && n < 3)
            die("Pattern lines in input file must be consistently have either 2 or 3 elements, no mixing and matching allowed");
        if (strlen(parts[0]) != strlen(filter)) die("All patters in input file must be same length");
        pats = (char **)realloc(pats, (np + 1) * sizeof(char *));
        pats[np++] = strdup(parts[0]);
    }
    if (lineno < 2) die("Input file must contain at least 3 lines");
    if (!have_mm) die("Input file must contain at least 1 pattern line");
    char err[512] = {0};
    orc_genome *g = orc_genome_load(genome, err, sizeof err);
    if (!g) die(err);
    orc_request r;
    memset(&r, 0, sizeof r);
    r.filter = filter;
    r.patterns = (const char *const *)pats;
    r.n_patterns = np;
    r.max_mismatches = mm;
    r.max_dna_bulges = db;
    r.max_rna_bulges = rb;
    r.chunks_per_search = argv[2][0] == 'C' ? 64 : 16384;
    char *rows = NULL;
    size_t rl = 0;
    uint64_t nr = 0;
    if (orc_search(g, &r, &rows, &rl, &nr, err, sizeof err)) die(err);
    FILE *out = strcmp(argv[3], "-") ? fopen(argv[3], "wb") : stdout;
    if (!out) die("cannot open output file");
    fputs("#Bulge type\tcrRNA\tDNA\tChromosome\tPosition\tDirection\tMismatches\tBulge Size\n", out);
    fwrite(rows, 1, rl, out);
    if (out != stdout) fclose(out);
    orc_free(rows);
    orc_genome_free(g);
    return 0;
}
