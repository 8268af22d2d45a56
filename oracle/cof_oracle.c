/*
 * cof_oracle.c -- CPU restatement of cas-offinder-rust's off-target search.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA product (parity tests,
 * smoke check, bench.py CPU baseline).  Never called by the product path.
 *
 * Every function names the reference file:line it restates (paths relative
 * to the reference project root).  The arithmetic is the reference's own:
 * the popcount scan keeps the u64-block / 16-shift / 4-blocks-per-exec loop
 * of search.rs:378-463 so that the timed CPU baseline is the reference
 * algorithm, and the Myers path keeps the per-end-position PAM check, Myers
 * sweep and exhaustive traceback enumeration of search.rs:779-897 and
 * traceback.rs:181-381.
 */
#define _GNU_SOURCE
#include "cof_oracle.h"

#include <dirent.h>
#include <errno.h>
#include <pthread.h>
#include <stdarg.h>
#include <stdatomic.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <unistd.h>

#define CHUNK_SIZE 65536u            /* chrom_chunk.rs:1 */
#define CHUNK_BYTES (CHUNK_SIZE / 2) /* chrom_chunk.rs:2 */
#define DEFAULT_CPS 16384u           /* search.rs:22 (GPU batch, 1 Gnt) */

/* ------------------------------------------------------------------------ */
/* bit4 tables: bit4ops.rs:1-121                                            */
/* ------------------------------------------------------------------------ */

static uint8_t STR2B4[2][256]; /* [mixed_base][char] */
static uint8_t B4STR[16];      /* BIT4_TO_STR restricted to nibbles */
static pthread_once_t tables_once = PTHREAD_ONCE_INIT;

static void init_tables(void) {
    /* makebit4map + apply_lower (bit4ops.rs:17-47) */
    for (int mixed = 0; mixed < 2; mixed++) {
        uint8_t up[256];
        memset(up, 0, sizeof up);
        up['G'] = 8; up['C'] = 2; up['A'] = 4; up['T'] = 1;
        if (mixed) {
            up['R'] = 4 | 8; up['Y'] = 2 | 1; up['S'] = 8 | 2; up['W'] = 4 | 1;
            up['K'] = 8 | 1; up['M'] = 4 | 2; up['B'] = 2 | 8 | 1;
            up['D'] = 4 | 8 | 1; up['H'] = 4 | 2 | 1; up['V'] = 4 | 2 | 8;
            up['N'] = 15;
        }
        memset(STR2B4[mixed], 0, 256);
        for (int i = 1; i <= 26; i++) {
            STR2B4[mixed][i + 96] = up[i + 64];
            STR2B4[mixed][i + 64] = up[i + 64];
        }
    }
    /* invert_chrmap (bit4ops.rs:48-59): the lowest char code wins. */
    memset(B4STR, 0, sizeof B4STR);
    for (int c = 255; c >= 0; c--) {
        uint8_t v = STR2B4[1][c];
        if (v != 0) B4STR[v] = (uint8_t)c;
    }
}
static void tables(void) { pthread_once(&tables_once, init_tables); }

static inline uint8_t get_bit4(const uint8_t *d, uint64_t i) { /* bit4ops.rs:281-288 */
    uint8_t b = d[i >> 1];
    return (i & 1) ? (uint8_t)(b >> 4) : (uint8_t)(b & 0xF);
}

/* compliment_char (bit4ops.rs:207-221) */
static uint8_t compliment_char(uint8_t c) {
    uint8_t b4 = STR2B4[1][c];
    uint8_t rev = (uint8_t)(((b4 << 2) | (b4 >> 2)) & 0xF);
    uint8_t out = b4 ? B4STR[rev] : c;
    return (uint8_t)(out | (c & 0x20));
}
/* reverse_compliment_char_i (bit4ops.rs:222-227) */
static void revcomp_inplace(uint8_t *s, size_t n) {
    for (size_t i = 0; i < n; i++) s[i] = compliment_char(s[i]);
    for (size_t i = 0; i < n / 2; i++) {
        uint8_t t = s[i];
        s[i] = s[n - 1 - i];
        s[n - 1 - i] = t;
    }
}
/* cmp_chars (bit4ops.rs:233-237) */
static inline int cmp_chars(uint8_t dna, uint8_t rna) {
    return (STR2B4[0][dna] & STR2B4[1][rna]) != 0;
}
static inline int is_n_char(uint8_t c) { return c == 'N' || c == 'n'; }

/* ------------------------------------------------------------------------ */
/* small growable buffers                                                   */
/* ------------------------------------------------------------------------ */

typedef struct { char *p; size_t n, cap; } sbuf;
static void sb_reserve(sbuf *b, size_t extra) {
    if (b->n + extra <= b->cap) return;
    size_t nc = b->cap ? b->cap * 2 : 4096;
    while (nc < b->n + extra) nc *= 2;
    char *q = (char *)realloc(b->p, nc);
    if (!q) { fprintf(stderr, "cof_oracle: out of memory\n"); abort(); }
    b->p = q; b->cap = nc;
}
static void sb_put(sbuf *b, const void *s, size_t n) {
    sb_reserve(b, n);
    memcpy(b->p + b->n, s, n);
    b->n += n;
}
static void sb_putc(sbuf *b, char c) { sb_put(b, &c, 1); }
static void sb_putu(sbuf *b, uint64_t v) {
    char tmp[24];
    int k = 0;
    do { tmp[k++] = (char)('0' + v % 10); v /= 10; } while (v);
    sb_reserve(b, (size_t)k);
    while (k) b->p[b->n++] = tmp[--k];
}

static void set_err(char *err, size_t errlen, const char *fmt, ...) {
    if (!err || !errlen) return;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(err, errlen, fmt, ap);
    va_end(ap);
}

/* ------------------------------------------------------------------------ */
/* genome: the ChromChunkInfo stream, tight-packed                          */
/* ------------------------------------------------------------------------ */

struct orc_genome {
    size_t n, cap;
    uint32_t *name_idx; /* per chunk: index into names */
    uint64_t *start, *end;
    uint64_t *boff;     /* byte offset of each chunk in data; boff[n] = size */
    char **names;
    size_t n_names, names_cap;
    uint8_t *data;
    size_t data_n, data_cap;
    uint8_t chunk[CHUNK_BYTES]; /* the chunk being filled by a loader */
};

static int add_name(orc_genome *g, const char *s, size_t n) {
    if (g->n_names == g->names_cap) {
        size_t nc = g->names_cap ? g->names_cap * 2 : 64;
        char **q = (char **)realloc(g->names, nc * sizeof(char *));
        if (!q) return -1;
        g->names = q; g->names_cap = nc;
    }
    char *c = (char *)malloc(n + 1);
    if (!c) return -1;
    memcpy(c, s, n);
    c[n] = 0;
    g->names[g->n_names++] = c;
    return (int)(g->n_names - 1);
}

/* The channel send of a ChromChunkInfo: append the chunk's valid bytes. */
static int push_chunk(orc_genome *g, uint32_t name, uint64_t cstart, uint64_t cend,
                      const uint8_t *bytes) {
    if (g->n + 1 >= g->cap) {
        size_t nc = g->cap ? g->cap * 2 : 256;
        g->name_idx = (uint32_t *)realloc(g->name_idx, nc * sizeof(uint32_t));
        g->start = (uint64_t *)realloc(g->start, nc * sizeof(uint64_t));
        g->end = (uint64_t *)realloc(g->end, nc * sizeof(uint64_t));
        g->boff = (uint64_t *)realloc(g->boff, (nc + 1) * sizeof(uint64_t));
        if (!g->name_idx || !g->start || !g->end || !g->boff) return -1;
        g->cap = nc;
    }
    size_t nb = (size_t)((cend - cstart + 1) / 2);
    if (g->data_n + nb > g->data_cap) {
        size_t nc = g->data_cap ? g->data_cap * 2 : (1u << 20);
        while (nc < g->data_n + nb) nc *= 2;
        uint8_t *q = (uint8_t *)realloc(g->data, nc);
        if (!q) return -1;
        g->data = q; g->data_cap = nc;
    }
    memcpy(g->data + g->data_n, bytes, nb);
    g->name_idx[g->n] = name;
    g->start[g->n] = cstart;
    g->end[g->n] = cend;
    g->boff[g->n] = g->data_n;
    g->data_n += nb;
    g->n++;
    g->boff[g->n] = g->data_n;
    return 0;
}

/* string_to_bit4 (bit4ops.rs:145-165), mixed_base selectable. */
static void string_to_bit4(uint8_t *out, const uint8_t *s, size_t n, size_t write_offset,
                           int mixed) {
    for (size_t i = 0; i < n; i++) {
        size_t o = write_offset + i;
        uint8_t v = STR2B4[mixed][s[i]];
        out[o >> 1] |= (o & 1) ? (uint8_t)(v << 4) : v;
    }
}

/* read_fasta (read_fasta.rs:9-71).  Lines are split on '\n' with one
 * trailing '\r' removed, like BufRead::lines(). */
static int read_fasta(orc_genome *g, const char *path, char *err, size_t errlen) {
    FILE *f = fopen(path, "rb");
    if (!f) { set_err(err, errlen, "cannot open %s: %s", path, strerror(errno)); return -1; }
    char *line = NULL;
    size_t lcap = 0;
    ssize_t got;
    int started = 0;
    int cur_name = -1; /* -1: empty name */
    int have_name = 0;
    uint64_t cs = 0, ce = 0;
    memset(g->chunk, 0, CHUNK_BYTES);
    int rc = 0;
    while ((got = getline(&line, &lcap, f)) >= 0) {
        size_t len = (size_t)got;
        if (len && line[len - 1] == '\n') {
            len--;
            if (len && line[len - 1] == '\r') len--;
        }
        if (len >= 1 && line[0] == '>') {
            if (ce != cs) {
                if (push_chunk(g, (uint32_t)cur_name, cs, ce, g->chunk)) { rc = -2; break; }
            }
            cur_name = add_name(g, line + 1, len - 1);
            if (cur_name < 0) { rc = -2; break; }
            have_name = (len - 1) > 0;
            cs = ce = 0;
            memset(g->chunk, 0, CHUNK_BYTES);
            started = 1;
        } else {
            if (!started) {
                set_err(err, errlen, "fasta file needs to start with >");
                rc = -1; break;
            }
            if (!have_name) {
                set_err(err, errlen, "> must be followed by chromosome name");
                rc = -1; break;
            }
            if (len + (size_t)(ce - cs) > CHUNK_SIZE) {
                if (push_chunk(g, (uint32_t)cur_name, cs, ce, g->chunk)) { rc = -2; break; }
                cs = ce;
                memset(g->chunk, 0, CHUNK_BYTES);
            }
            if (len > CHUNK_SIZE) {
                set_err(err, errlen, "line in fasta too long");
                rc = -1; break;
            }
            string_to_bit4(g->chunk, (const uint8_t *)line, len, (size_t)(ce - cs), 1);
            ce += len;
        }
    }
    if (rc == 0 && ce > cs) {
        if (push_chunk(g, (uint32_t)cur_name, cs, ce, g->chunk)) rc = -2;
    }
    if (rc == -2) set_err(err, errlen, "out of memory");
    free(line);
    fclose(f);
    return rc;
}

/* memsetbit4 (bit4ops.rs:184-200) */
static void memsetbit4(uint8_t *d, uint8_t v, size_t start, size_t end) {
    for (size_t i = start; i < end; i++) {
        if (i & 1) d[i >> 1] = (uint8_t)((d[i >> 1] & 0x0F) | (v << 4));
        else d[i >> 1] = (uint8_t)((d[i >> 1] & 0xF0) | v);
    }
}

static int rd(FILE *f, void *p, size_t n) { return fread(p, 1, n, f) == n ? 0 : -1; }
static int rd_u32(FILE *f, uint32_t *v) { return rd(f, v, 4); }

typedef struct { uint32_t s, z; } nblock;
static int cmp_nblock(const void *a, const void *b) {
    uint32_t x = ((const nblock *)a)->s, y = ((const nblock *)b)->s;
    return x < y ? -1 : x > y;
}

/* read_2bit (read_2bit.rs:33-118).  Sequences are read in index order,
 * straight after each other, like the reference (the per-sequence offsets are
 * skipped).  2-bit codes T=0 C=1 A=2 G=3, first base in the high bits
 * (bit4ops.rs:60-75).  N blocks become 0xF, soft masks are ignored. */
static int read_2bit(orc_genome *g, const char *path, char *err, size_t errlen) {
    FILE *f = fopen(path, "rb");
    if (!f) { set_err(err, errlen, "cannot open %s: %s", path, strerror(errno)); return -1; }
    int rc = -1;
    uint32_t magic, version, cnt, reserved;
    uint32_t *names = NULL;
    nblock *nb = NULL;
    uint8_t *raw = NULL;
    if (rd_u32(f, &magic) || magic != 0x1A412743u) {
        set_err(err, errlen, ".2bit file badly formatted header"); goto out;
    }
    if (rd_u32(f, &version) || version != 0) {
        set_err(err, errlen, "only supports version 0 of .2bit format"); goto out;
    }
    if (rd_u32(f, &cnt) || rd_u32(f, &reserved)) { set_err(err, errlen, "truncated .2bit"); goto out; }
    names = (uint32_t *)calloc(cnt ? cnt : 1, sizeof(uint32_t));
    for (uint32_t i = 0; i < cnt; i++) {
        uint8_t nl;
        char nm[256];
        uint32_t off;
        if (rd(f, &nl, 1) || rd(f, nm, nl) || rd_u32(f, &off)) {
            set_err(err, errlen, "truncated .2bit index"); goto out;
        }
        int ni = add_name(g, nm, nl);
        if (ni < 0) { set_err(err, errlen, "out of memory"); goto out; }
        names[i] = (uint32_t)ni;
    }
    raw = (uint8_t *)malloc(CHUNK_SIZE / 4);
    for (uint32_t s = 0; s < cnt; s++) {
        uint32_t chrlen, nbc, mbc;
        if (rd_u32(f, &chrlen) || rd_u32(f, &nbc)) { set_err(err, errlen, "truncated .2bit"); goto out; }
        free(nb);
        nb = (nblock *)calloc(nbc ? nbc : 1, sizeof(nblock));
        for (uint32_t i = 0; i < nbc; i++)
            if (rd_u32(f, &nb[i].s)) { set_err(err, errlen, "truncated .2bit"); goto out; }
        for (uint32_t i = 0; i < nbc; i++)
            if (rd_u32(f, &nb[i].z)) { set_err(err, errlen, "truncated .2bit"); goto out; }
        qsort(nb, nbc, sizeof(nblock), cmp_nblock);
        if (rd_u32(f, &mbc)) { set_err(err, errlen, "truncated .2bit"); goto out; }
        if (fseek(f, (long)((uint32_t)(mbc * 8u + 4u)), SEEK_CUR)) {
            set_err(err, errlen, "truncated .2bit"); goto out;
        }
        size_t read_pos = 0;
        int64_t bmi = 0;
        while (read_pos < chrlen) {
            size_t read_size = chrlen - read_pos < CHUNK_SIZE ? chrlen - read_pos : CHUNK_SIZE;
            size_t nbytes = (read_size + 3) / 4;
            if (rd(f, raw, nbytes)) { set_err(err, errlen, "truncated .2bit"); goto out; }
            memset(g->chunk, 0, CHUNK_BYTES);
            /* bit2_to_bit4 (bit4ops.rs:166-183) */
            for (size_t i = 0; i < nbytes; i++) {
                uint16_t v = 0;
                for (int j = 0; j < 4; j++) {
                    int b2 = (raw[i] >> ((4 - j - 1) * 2)) & 3;
                    v |= (uint16_t)((1u << b2) << (j * 4));
                }
                g->chunk[2 * i] = (uint8_t)(v & 0xFF);
                g->chunk[2 * i + 1] = (uint8_t)(v >> 8);
            }
            if (read_size % 4) memsetbit4(g->chunk, 0, read_size, nbytes * 4);
            bmi = bmi - 1 > 0 ? bmi - 1 : 0;
            while (bmi < (int64_t)nbc) {
                int64_t bcs = (int64_t)nb[bmi].s - (int64_t)read_pos;
                int64_t bce = (int64_t)(uint32_t)(nb[bmi].s + nb[bmi].z) - (int64_t)read_pos;
                if (bcs > (int64_t)read_size) break;
                int64_t a = bcs > 0 ? bcs : 0;
                int64_t e = bce > 0 ? bce : 0;
                if (e > (int64_t)read_size) e = (int64_t)read_size;
                if (a < e) memsetbit4(g->chunk, 0xF, (size_t)a, (size_t)e);
                bmi++;
            }
            if (push_chunk(g, names[s], read_pos, read_pos + read_size, g->chunk)) {
                set_err(err, errlen, "out of memory"); goto out;
            }
            read_pos += read_size;
        }
    }
    rc = 0;
out:
    free(names);
    free(nb);
    free(raw);
    fclose(f);
    return rc;
}

/* read_fasta_folder (read_fasta_folder.rs:8-23): every regular file whose
 * path ends in ".fa", in readdir order. */
static int read_fasta_folder(orc_genome *g, const char *dir, char *err, size_t errlen) {
    DIR *d = opendir(dir);
    if (!d) { set_err(err, errlen, "cannot open folder %s", dir); return -1; }
    struct dirent *e;
    int rc = 0;
    while ((e = readdir(d)) != NULL) {
        if (!strcmp(e->d_name, ".") || !strcmp(e->d_name, "..")) continue;
        char path[4096];
        size_t dl = strlen(dir);
        snprintf(path, sizeof path, "%s%s%s", dir, (dl && dir[dl - 1] == '/') ? "" : "/", e->d_name);
        struct stat st;
        if (stat(path, &st) || !S_ISREG(st.st_mode)) continue;
        size_t pl = strlen(path);
        if (pl >= 3 && !strcmp(path + pl - 3, ".fa")) {
            rc = read_fasta(g, path, err, errlen);
            if (rc) break;
        }
    }
    closedir(d);
    return rc;
}

orc_genome *orc_genome_load(const char *path, char *err, size_t errlen) {
    tables();
    orc_genome *g = (orc_genome *)calloc(1, sizeof(orc_genome));
    if (!g) return NULL;
    g->boff = (uint64_t *)calloc(1, sizeof(uint64_t));
    struct stat st;
    int rc;
    if (stat(path, &st)) {
        set_err(err, errlen, "cannot stat %s", path);
        rc = -1;
    } else if (S_ISDIR(st.st_mode)) {
        rc = read_fasta_folder(g, path, err, errlen);
    } else {
        FILE *f = fopen(path, "rb");
        int c = f ? fgetc(f) : EOF;
        if (f) fclose(f);
        if (c == EOF) { set_err(err, errlen, "cannot read %s", path); rc = -1; }
        else if (c == '>') rc = read_fasta(g, path, err, errlen);
        else rc = read_2bit(g, path, err, errlen);
    }
    if (rc) { orc_genome_free(g); return NULL; }
    return g;
}

orc_genome *orc_genome_new(void) {
    tables();
    orc_genome *g = (orc_genome *)calloc(1, sizeof(orc_genome));
    if (g) g->boff = (uint64_t *)calloc(1, sizeof(uint64_t));
    return g;
}

int orc_genome_add_chunk(orc_genome *g, const char *name, const uint8_t *bit4,
                         uint64_t chunk_start, uint64_t chunk_end) {
    if (chunk_end <= chunk_start) return 0;
    if (chunk_end - chunk_start > CHUNK_SIZE) return -1;
    int ni;
    if (chunk_start != 0 && g->n && !strcmp(g->names[g->name_idx[g->n - 1]], name))
        ni = (int)g->name_idx[g->n - 1];
    else
        ni = add_name(g, name, strlen(name));
    if (ni < 0) return -1;
    return push_chunk(g, (uint32_t)ni, chunk_start, chunk_end, bit4);
}

void orc_genome_free(orc_genome *g) {
    if (!g) return;
    for (size_t i = 0; i < g->n_names; i++) free(g->names[i]);
    free(g->names);
    free(g->name_idx);
    free(g->start);
    free(g->end);
    free(g->boff);
    free(g->data);
    free(g);
}

size_t orc_genome_n_chunks(const orc_genome *g) { return g->n; }
uint64_t orc_genome_n_nucl(const orc_genome *g) {
    uint64_t s = 0;
    for (size_t k = 0; k < g->n; k++) s += g->end[k] - g->start[k];
    return s;
}
const char *orc_chunk_name(const orc_genome *g, size_t k) { return g->names[g->name_idx[k]]; }
uint64_t orc_chunk_start(const orc_genome *g, size_t k) { return g->start[k]; }
uint64_t orc_chunk_end(const orc_genome *g, size_t k) { return g->end[k]; }
const uint8_t *orc_chunk_data(const orc_genome *g, size_t k) { return g->data + g->boff[k]; }

char *orc_genome_decode(const orc_genome *g, size_t *len) {
    tables();
    uint64_t tot = orc_genome_n_nucl(g);
    char *s = (char *)malloc((size_t)tot + 1);
    size_t o = 0;
    for (size_t k = 0; k < g->n; k++) {
        uint64_t n = g->end[k] - g->start[k];
        const uint8_t *d = g->data + g->boff[k];
        for (uint64_t i = 0; i < n; i++) s[o++] = (char)B4STR[get_bit4(d, i)];
    }
    s[o] = 0;
    if (len) *len = o;
    return s;
}

void orc_free(void *p) { free(p); }

/* ------------------------------------------------------------------------ */
/* batcher: send thread of search.rs:1531-1572 + chunks_to_searchchunk      */
/* ------------------------------------------------------------------------ */

typedef struct { size_t first, last; int has_head; } batch;

static size_t make_batches(const orc_genome *g, uint32_t cps, batch **out) {
    size_t cap = 16, n = 0;
    batch *b = (batch *)malloc(cap * sizeof(batch));
    size_t buf_first = 0, buf_len = 0;
    int has_head = 0;
    for (size_t k = 0; k < g->n; k++) {
        if (buf_len == 0) buf_first = k;
        buf_len++;
        if (buf_len == cps) {
            if (n == cap) { cap *= 2; b = (batch *)realloc(b, cap * sizeof(batch)); }
            b[n].first = buf_first; b[n].last = k; b[n].has_head = has_head; n++;
            buf_first = k; buf_len = 1; has_head = 1;
        }
    }
    if (buf_len && !(has_head && buf_len == 1)) {
        if (n == cap) { cap *= 2; b = (batch *)realloc(b, cap * sizeof(batch)); }
        b[n].first = buf_first; b[n].last = buf_first + buf_len - 1; b[n].has_head = has_head; n++;
    }
    *out = b;
    return n;
}

size_t orc_n_batches(const orc_genome *g, uint32_t cps) {
    batch *b;
    size_t n = make_batches(g, cps ? cps : DEFAULT_CPS, &b);
    free(b);
    return n;
}

/* Batch-local view of SearchChunkMeta (search.rs:57-79). */
typedef struct {
    const orc_genome *g;
    size_t first, nch;   /* chunks [first, first+nch) */
    uint64_t base;       /* global byte offset of the batch */
    uint64_t valid;      /* valid bytes of the batch */
    int has_head;
} bview;

static void bview_init(bview *v, const orc_genome *g, const batch *b) {
    v->g = g;
    v->first = b->first;
    v->nch = b->last - b->first + 1;
    v->base = g->boff[b->first];
    v->valid = g->boff[b->last + 1] - v->base;
    v->has_head = b->has_head;
}
static inline uint64_t bv_off(const bview *v, size_t i) { /* chunk_byte_offsets[i] */
    return v->g->boff[v->first + i] - v->base;
}
/* partition_point(|off| off <= byte_pos).saturating_sub(1) over the byte
 * offsets including the sentinel (search.rs:1441-1445). */
static size_t bv_find(const bview *v, uint64_t byte_pos) {
    size_t lo = 0, hi = v->nch + 1;
    while (lo < hi) {
        size_t mid = (lo + hi) / 2;
        if (bv_off(v, mid) <= byte_pos) lo = mid + 1; else hi = mid;
    }
    return lo ? lo - 1 : 0;
}

/* ------------------------------------------------------------------------ */
/* request compile: main.rs:253-259 + search.rs:1516-1523                    */
/* ------------------------------------------------------------------------ */

typedef struct {
    size_t L, n_user, n_pat;
    uint8_t **pat_ascii;   /* fwd then rc, as main.rs builds all_patterns */
    uint8_t **pat_bit4;    /* string_to_bit4(mixed) packed, ceil(L/2) bytes */
    const char *filter;
    uint32_t mm, db, rb;
    uint64_t pam_len;      /* main.rs:80-91 */
    int raw;               /* emit raw Match lines */
} creq;

static void creq_free(creq *c) {
    for (size_t i = 0; i < c->n_pat; i++) { free(c->pat_ascii[i]); free(c->pat_bit4[i]); }
    free(c->pat_ascii);
    free(c->pat_bit4);
}

static int creq_init(creq *c, const orc_request *r, char *err, size_t errlen) {
    memset(c, 0, sizeof *c);
    if (!r->filter || r->n_patterns == 0) { set_err(err, errlen, "no patterns"); return -1; }
    c->L = strlen(r->filter);
    c->n_user = r->n_patterns;
    c->n_pat = 2 * r->n_patterns;
    c->filter = r->filter;
    c->mm = r->max_mismatches; c->db = r->max_dna_bulges; c->rb = r->max_rna_bulges;
    c->raw = r->raw_matches;
    if (c->L == 0) { set_err(err, errlen, "empty filter"); return -1; }
    for (size_t i = 0; i < r->n_patterns; i++) {
        if (strlen(r->patterns[i]) != c->L) {
            set_err(err, errlen, "All patterns must have same length"); return -1;
        }
    }
    int use_myers = c->db > 0 || c->rb > 0;
    if (use_myers && c->L > 64) { set_err(err, errlen, "Myers requires pattern length <= 64"); return -1; }
    if (c->L > 1000 || c->db > 64 || c->rb > 64) {
        set_err(err, errlen, "pattern length or bulge limit out of range"); return -1;
    }
    if (!use_myers && c->mm >= c->L) {
        /* search.rs:1441-1448 indexes past chunk_starts when a window that lies
         * wholly in the zero tail of the batch buffer passes the threshold. */
        set_err(err, errlen, "max_mismatches must be below the pattern length"); return -1;
    }
    c->pat_ascii = (uint8_t **)calloc(c->n_pat, sizeof(uint8_t *));
    c->pat_bit4 = (uint8_t **)calloc(c->n_pat, sizeof(uint8_t *));
    for (size_t i = 0; i < c->n_pat; i++) {
        c->pat_ascii[i] = (uint8_t *)malloc(c->L + 1);
        const char *src = r->patterns[i % c->n_user];
        memcpy(c->pat_ascii[i], src, c->L);
        c->pat_ascii[i][c->L] = 0;
        if (i >= c->n_user) revcomp_inplace(c->pat_ascii[i], c->L);
        c->pat_bit4[i] = (uint8_t *)calloc((c->L + 1) / 2 + 1, 1);
        string_to_bit4(c->pat_bit4[i], c->pat_ascii[i], c->L, 0, 1);
    }
    uint64_t pl = 0;
    for (size_t i = c->L; i > 0; i--) {
        if (is_n_char((uint8_t)r->patterns[0][i - 1])) pl++; else break;
    }
    c->pam_len = pl;
    return 0;
}

/* writer row tail: chromosome, position, direction, mismatches, bulge size
 * (main.rs:226-242). */
static void put_row_tail(sbuf *o, const char *chr, uint64_t chrom_idx, int fwd, uint32_t db,
                         uint32_t mm, uint32_t bulge_size, uint64_t pam_len) {
    uint64_t pos = chrom_idx;
    if (!fwd) {
        uint64_t a = pam_len ? pam_len - 1 : 0;
        a = a > db ? a - db : 0;
        pos += a;
    }
    sb_putc(o, '\t');
    sb_put(o, chr, strlen(chr));
    sb_putc(o, '\t');
    sb_putu(o, pos);
    sb_putc(o, '\t');
    sb_putc(o, fwd ? '+' : '-');
    sb_putc(o, '\t');
    sb_putu(o, mm);
    sb_putc(o, '\t');
    sb_putu(o, bulge_size);
    sb_putc(o, '\n');
}

/* ------------------------------------------------------------------------ */
/* popcount path                                                            */
/* ------------------------------------------------------------------------ */

typedef struct { uint32_t start, pattern; int32_t mm; } rawhit;
typedef struct { rawhit *p; size_t n, cap; } hitvec;
static void hv_push(hitvec *h, uint32_t s, uint32_t p, int32_t mm) {
    if (h->n == h->cap) {
        h->cap = h->cap ? 2 * h->cap : 1024;
        h->p = (rawhit *)realloc(h->p, h->cap * sizeof(rawhit));
    }
    h->p[h->n].start = s; h->p[h->n].pattern = p; h->p[h->n].mm = mm;
    h->n++;
}

/* search_chunk_cpu (search.rs:378-463): u64 blocks of 16 nucleotides, four
 * blocks per exec, sixteen 4-bit shifts, popcount of genome & pattern.
 * Emits (start, pattern, max(mm, 0)) for mm <= max_mm (signed) and
 * start >= match_start_min_nucl.  genome_blocks must be a multiple of 4;
 * buf must hold genome_blocks + pattern_blocks + 5 zero-padded blocks. */
static void search_chunk_cpu(uint32_t max_mm, size_t L, const uint64_t *pat, size_t n_pat,
                             const uint64_t *gen, size_t genome_blocks, uint32_t msmin,
                             hitvec *out) {
    const size_t pb = (L + 15) / 16;
    const size_t pps = (pb + 1) / 2 * 2;
    uint64_t sd[64 + 8];
    for (size_t gbi = 0; gbi < genome_blocks / 4; gbi++) {
        size_t gi = gbi * 4;
        size_t ncopy = 4 + pb + 1;
        if (ncopy > genome_blocks - gi) ncopy = genome_blocks - gi;
        memset(sd, 0, sizeof(uint64_t) * (4 + pb + 1));
        memcpy(sd, gen + gi, ncopy * sizeof(uint64_t));
        for (size_t l = 0; l < 16; l++) {
            for (size_t j = 0; j < n_pat; j++) {
                uint32_t nm[4] = {0, 0, 0, 0};
                const uint64_t *pj = pat + j * pps;
                for (size_t k = 0; k < pb; k++)
                    for (size_t o = 0; o < 4; o++)
                        nm[o] += (uint32_t)__builtin_popcountll(sd[k + o] & pj[k]);
                for (size_t o = 0; o < 4; o++) {
                    int32_t mmi = (int32_t)L - (int32_t)nm[o];
                    if (mmi <= (int32_t)max_mm) {
                        uint32_t s = (uint32_t)((gi + o) * 16 + l);
                        if (s < msmin) continue;
                        hv_push(out, s, (uint32_t)j, mmi > 0 ? mmi : 0);
                    }
                }
            }
            for (size_t k = 0; k < pb + 3; k++) sd[k] = (sd[k] >> 4) | (sd[k + 1] << 60);
            sd[pb + 3] >>= 4;
        }
    }
}

/* mask_genome_n_to_zero_inplace (search.rs:512-531) */
static void mask_n(uint8_t *d, size_t n) {
    for (size_t i = 0; i < n; i++) {
        uint8_t lo = d[i] & 0xF, hi = d[i] >> 4;
        if (lo == 0xF) lo = 0;
        if (hi == 0xF) hi = 0;
        d[i] = (uint8_t)(lo | (hi << 4));
    }
}

/* pack_patterns (search.rs:465-477) as u64 blocks. */
static uint64_t *pack_patterns(const creq *c, size_t *pps_out) {
    size_t pb = (c->L + 15) / 16;
    size_t pps = (pb + 1) / 2 * 2;
    uint64_t *p = (uint64_t *)calloc(c->n_pat * pps, sizeof(uint64_t));
    size_t nb = (c->L + 1) / 2;
    for (size_t j = 0; j < c->n_pat; j++) memcpy((uint8_t *)(p + j * pps), c->pat_bit4[j], nb);
    *pps_out = pps;
    return p;
}

/* Builds the batch buffer (chunks_to_searchchunk: tight-packed, zero tail),
 * masked for the popcount path.  Returns the number of u64 blocks to scan. */
static uint64_t *batch_buffer(const bview *v, size_t L, int mask, size_t *genome_blocks) {
    size_t scan_bytes = (size_t)((v->valid + 31) / 32 * 32);
    size_t pad = ((L + 15) / 16 + 8) * 8;
    uint64_t *buf = (uint64_t *)calloc((scan_bytes + pad) / 8 + 1, sizeof(uint64_t));
    memcpy(buf, v->g->data + v->base, (size_t)v->valid);
    if (mask) mask_n((uint8_t *)buf, (size_t)v->valid);
    *genome_blocks = scan_bytes / 8;
    return buf;
}

/* legacy_match_start_min_nucl (search.rs:540-546) */
static uint32_t msmin_of(const bview *v, size_t L) {
    if (!v->has_head) return 0;
    uint64_t c1 = bv_off(v, 1) * 2;
    return c1 > L - 1 ? (uint32_t)(c1 - (L - 1)) : 0;
}

/* convert_matches (search.rs:1428-1488) + the popcount branch of the writer
 * (main.rs:159-242). */
static void convert_and_write_popcount(const bview *v, const creq *c, const uint8_t *buf,
                                       const hitvec *h, sbuf *out, uint64_t *n_rows) {
    const size_t L = c->L;
    uint8_t *dna = (uint8_t *)malloc(L), *rna = (uint8_t *)malloc(L);
    for (size_t q = 0; q < h->n; q++) {
        const rawhit *m = &h->p[q];
        size_t idx = bv_find(v, m->start / 2);
        if (idx >= v->nch) continue; /* unreachable for mm < L */
        uint64_t off = m->start - bv_off(v, idx) * 2;
        size_t k = v->first + idx;
        uint64_t pos = v->g->start[k] + off;
        int is_end_chrom = idx == v->nch - 1 || v->g->start[k + 1] == 0;
        int is_past_end = pos + L > v->g->end[k];
        if (is_end_chrom && is_past_end) continue;
        int fwd = m->pattern < c->n_pat / 2;
        for (size_t i = 0; i < L; i++) {
            dna[i] = B4STR[get_bit4(buf, (uint64_t)m->start + i)];
            rna[i] = B4STR[get_bit4(c->pat_bit4[m->pattern], i)];
        }
        if (!fwd) { revcomp_inplace(dna, L); revcomp_inplace(rna, L); }
        if (c->raw) {
            sb_put(out, v->g->names[v->g->name_idx[k]], strlen(v->g->names[v->g->name_idx[k]]));
            sb_putc(out, '\t');
            sb_putu(out, pos);
            sb_putc(out, '\t');
            sb_putu(out, m->pattern);
            sb_putc(out, '\t');
            sb_putc(out, fwd ? '+' : '-');
            sb_putc(out, '\t');
            sb_putu(out, (uint64_t)m->mm);
            sb_put(out, "\t0\t0\t", 5);
            sb_put(out, rna, L);
            sb_putc(out, '\t');
            sb_put(out, dna, L);
            sb_putc(out, '\n');
            (*n_rows)++;
            continue;
        }
        /* writer post-filter, main.rs:172-197 */
        int pam_ok = 1;
        uint32_t actual = 0;
        for (size_t i = 0; i < L; i++) {
            uint8_t fc = (uint8_t)c->filter[i];
            if (!is_n_char(fc) && !cmp_chars(dna[i], fc)) { pam_ok = 0; break; }
            if (!is_n_char(rna[i]) && !cmp_chars(dna[i], rna[i])) actual++;
        }
        if (!pam_ok || actual > c->mm) continue;
        /* lowercase marking, main.rs:198-217 */
        for (size_t i = 0; i < L; i++) {
            int rn = is_n_char(rna[i]);
            int dn = is_n_char(dna[i]);
            if (dna[i] == 0) dna[i] = rn ? 'N' : 'n';
            else if (rn) {}
            else if (dn) dna[i] = 'n';
            else if (!cmp_chars(dna[i], rna[i])) dna[i] |= 0x20;
        }
        sb_put(out, "X\t", 2);
        sb_put(out, rna, L);
        sb_putc(out, '\t');
        sb_put(out, dna, L);
        put_row_tail(out, v->g->names[v->g->name_idx[k]], pos, fwd, 0, actual, 0, c->pam_len);
        (*n_rows)++;
    }
    free(dna);
    free(rna);
}

/* ------------------------------------------------------------------------ */
/* Myers path                                                               */
/* ------------------------------------------------------------------------ */

typedef struct {
    uint64_t peq[4], peq_n;     /* myers.rs:12-16 */
    uint8_t *b4;                /* char_to_bit4 per cell */
    uint8_t *is_n;              /* pattern char is N/n */
    uint8_t *eff;               /* effective filter bit4 per cell */
    size_t pam_off;             /* precompute_pam_precheck */
    uint8_t *pam_f;
    size_t pam_n;
} mpat;

/* build_peq (myers.rs:32-50) */
static void build_peq(mpat *m, const uint8_t *p, size_t L) {
    memset(m->peq, 0, sizeof m->peq);
    m->peq_n = 0;
    for (size_t i = 0; i < L; i++) {
        uint8_t u = (uint8_t)((p[i] >= 'a' && p[i] <= 'z') ? p[i] - 32 : p[i]);
        int idx = u == 'A' ? 0 : u == 'C' ? 1 : u == 'G' ? 2 : u == 'T' ? 3 : 4;
        if (idx < 4) m->peq[idx] |= 1ull << i;
        else {
            for (int k = 0; k < 4; k++) m->peq[k] |= 1ull << i;
            m->peq_n |= 1ull << i;
        }
    }
}

/* check_pam_quick (search.rs:703-755) */
static int check_pam_quick(const uint8_t *g, uint64_t total, uint64_t end_pos, size_t L,
                           const mpat *m, uint32_t db, uint32_t rb) {
    int64_t dr = m->pam_off == 0 ? (int64_t)db + 1 : 1;
    int64_t rr = m->pam_off == 0 ? (int64_t)rb + 1 : 1;
    for (int64_t bd = 0; bd < dr; bd++) {
        for (int64_t br = 0; br < rr; br++) {
            int64_t span = (int64_t)L + bd - br;
            if (span <= 0 || span > (int64_t)end_pos + 1) continue;
            uint64_t as = end_pos + 1 - (uint64_t)span;
            int ok = 1;
            for (size_t k = 0; k < m->pam_n; k++) {
                uint64_t gp = as + m->pam_off + k;
                if (gp >= total) { ok = 0; break; }
                uint8_t gv = get_bit4(g, gp), f = m->pam_f[k];
                int pos_ok = f == 0xF ? gv != 0 : (gv == 0 || gv == 0xF) ? 0 : (gv & f) != 0;
                if (!pos_ok) { ok = 0; break; }
            }
            if (ok) return 1;
        }
    }
    return 0;
}

/* cmp_loose_bit4 (traceback.rs:41-46) */
static inline int cmp_loose_bit4(uint8_t p, uint8_t t) {
    if (t == 0) return 0;
    if (p == 0xF) return 1;
    if (t == 0xF) return 0;
    return (p & t) != 0;
}

enum { OP_M = 0, OP_S = 1, OP_D = 2, OP_R = 3 }; /* Match, Substitution, DnaBulge, RnaBulge */

typedef struct {
    /* per candidate */
    const uint8_t *pb4;  /* pattern bit4 cells */
    const uint8_t *is_n;
    const uint8_t *text; /* text window bit4 cells */
    size_t m, n;
    uint64_t *dp;        /* (m+1)*(n+1) */
    uint32_t max_edits, max_db, max_rb, max_mm;
    uint8_t ops[160];
    size_t nops;
    /* emission */
    void (*emit)(void *ctx, const uint8_t *ops_rev, size_t nops, size_t j, uint32_t mm,
                 uint32_t db, uint32_t rb);
    void *ctx;
} tbs;

#define DP(t, i, j) ((t)->dp[(i) * ((t)->n + 1) + (j)])

/* enumerate (traceback.rs:242-381) */
static void enumerate(tbs *t, size_t i, size_t j, uint64_t cost, uint32_t mm, uint32_t db,
                      uint32_t rb) {
    if (cost + DP(t, i, j) > t->max_edits) return;
    if (mm > t->max_mm || db > t->max_db || rb > t->max_rb) return;
    if (i == 0) {
        t->emit(t->ctx, t->ops, t->nops, j, mm, db, rb);
        return;
    }
    if (j > 0) {
        uint32_t mc = cmp_loose_bit4(t->pb4[i - 1], t->text[j - 1]) ? 0 : 1;
        int touches_n = mc == 1 && t->is_n[i - 1];
        if (!touches_n) {
            t->ops[t->nops++] = mc ? OP_S : OP_M;
            enumerate(t, i - 1, j - 1, cost + mc, mm + mc, db, rb);
            t->nops--;
        }
    }
    if (rb < t->max_rb && t->max_rb > 0) {
        int pn = t->is_n[i - 1];
        int next_pam = i < t->m && t->is_n[i];
        int prev_pam = i >= 2 && t->is_n[i - 2];
        if (!pn && !next_pam && !prev_pam) {
            t->ops[t->nops++] = OP_R;
            enumerate(t, i - 1, j, cost + 1, mm, db, rb + 1);
            t->nops--;
        }
    }
    if (db < t->max_db && t->max_db > 0 && j > 0 && i < t->m) {
        int prev_n = i > 0 && t->is_n[i - 1];
        int next_n = t->is_n[i];
        if (!(prev_n && next_n)) {
            t->ops[t->nops++] = OP_D;
            enumerate(t, i, j - 1, cost + 1, mm, db + 1, rb);
            t->nops--;
        }
    }
}

/* traceback_all (traceback.rs:181-239) */
static void traceback_all(tbs *t) {
    const uint64_t INF = 0x7FFFFFFFull; /* u32::MAX / 2 */
    uint64_t dna_cost = t->max_db == 0 ? INF : 1;
    uint64_t rna_cost = t->max_rb == 0 ? INF : 1;
    for (size_t i = 0; i <= t->m; i++) {
        uint64_t v = (uint64_t)i * rna_cost;
        DP(t, i, 0) = v < INF ? v : INF;
    }
    for (size_t j = 1; j <= t->n; j++) DP(t, 0, j) = 0;
    for (size_t i = 1; i <= t->m; i++) {
        for (size_t j = 1; j <= t->n; j++) {
            if (t->text[j - 1] == 0) { DP(t, i, j) = INF; continue; }
            uint64_t mc = cmp_loose_bit4(t->pb4[i - 1], t->text[j - 1]) ? 0 : 1;
            uint64_t a = DP(t, i - 1, j - 1) + mc;
            uint64_t b = DP(t, i - 1, j) + rna_cost;
            uint64_t c = DP(t, i, j - 1) + dna_cost;
            uint64_t v = a < b ? a : b;
            DP(t, i, j) = v < c ? v : c;
        }
    }
    if (DP(t, t->m, t->n) > t->max_edits) return;
    t->nops = 0;
    enumerate(t, t->m, t->n, 0, 0, 0, 0);
}

typedef struct {
    const bview *v;
    const creq *c;
    const mpat *mp;
    size_t p;
    uint64_t end_pos;      /* batch-local */
    uint64_t text_start;   /* batch-local */
    const uint8_t *text;
    size_t text_len;
    sbuf *out;
    uint64_t *n_rows;
    uint8_t *pa, *ta;      /* scratch strings */
} mctx;

/* classify_myers_candidate's per-alignment tail (search.rs:634-686) fused
 * with convert_matches_myers (search.rs:1316-1374) and the Myers branch of
 * the writer (main.rs:145-157, 224-242). */
static void emit_alignment(void *vctx, const uint8_t *ops_rev, size_t nops, size_t j,
                           uint32_t mm, uint32_t db, uint32_t rb) {
    mctx *x = (mctx *)vctx;
    const mpat *mp = &x->mp[x->p];
    const size_t L = x->c->L;
    /* forward ops, strings (traceback.rs:267-298) */
    size_t pi = 0, ti = j, na = 0;
    for (size_t q = nops; q > 0; q--) {
        uint8_t op = ops_rev[q - 1];
        if (op == OP_M || op == OP_S) {
            x->pa[na] = B4STR[mp->b4[pi]];
            x->ta[na] = B4STR[x->text[ti] & 0xF];
            pi++; ti++;
        } else if (op == OP_R) {
            x->pa[na] = B4STR[mp->b4[pi]];
            x->ta[na] = '-';
            pi++;
        } else {
            x->pa[na] = '-';
            x->ta[na] = B4STR[x->text[ti] & 0xF];
            ti++;
        }
        na++;
    }
    size_t span = 0;
    for (size_t q = 0; q < na; q++) span += x->ta[q] != '-';
    /* PAM check at every Match/Substitution cell (search.rs:638-670) */
    size_t off = x->text_len - span, pp = 0, go = off;
    for (size_t q = nops; q > 0; q--) {
        uint8_t op = ops_rev[q - 1];
        if (op == OP_M || op == OP_S) {
            uint8_t gv = x->text[go], f = mp->eff[pp];
            int ok = f == 0xF ? gv != 0 : (gv == 0 || gv == 0xF) ? 0 : (gv & f) != 0;
            if (!ok) return;
            pp++; go++;
        } else if (op == OP_D) go++;
        else pp++;
    }
    uint64_t start = x->end_pos + 1 - span;
    /* convert_matches_myers */
    const bview *v = x->v;
    size_t idx = bv_find(v, start / 2);
    if (idx >= v->nch) return;
    uint64_t coff = start - bv_off(v, idx) * 2;
    size_t k = v->first + idx;
    uint64_t pos = v->g->start[k] + coff;
    int is_end_chrom = idx == v->nch - 1 || v->g->start[k + 1] == 0;
    uint64_t extent = (uint64_t)L + db - rb;
    int past = pos + extent > v->g->end[k];
    if (is_end_chrom && past) return;
    int fwd = x->p < x->c->n_pat / 2;
    if (!fwd) { revcomp_inplace(x->ta, na); revcomp_inplace(x->pa, na); }
    sbuf *o = x->out;
    if (x->c->raw) {
        const char *nm = v->g->names[v->g->name_idx[k]];
        sb_put(o, nm, strlen(nm));
        sb_putc(o, '\t');
        sb_putu(o, pos);
        sb_putc(o, '\t');
        sb_putu(o, x->p);
        sb_putc(o, '\t');
        sb_putc(o, fwd ? '+' : '-');
        sb_putc(o, '\t');
        sb_putu(o, mm);
        sb_putc(o, '\t');
        sb_putu(o, db);
        sb_putc(o, '\t');
        sb_putu(o, rb);
        sb_putc(o, '\t');
        sb_put(o, x->pa, na);
        sb_putc(o, '\t');
        sb_put(o, x->ta, na);
        sb_putc(o, '\n');
        (*x->n_rows)++;
        return;
    }
    uint32_t tot = db + rb;
    if (tot == 0) sb_put(o, "X\t", 2);
    else if (db > 0) sb_put(o, "DNA\t", 4);
    else sb_put(o, "RNA\t", 4);
    sb_put(o, x->pa, na);
    sb_putc(o, '\t');
    sb_put(o, x->ta, na);
    put_row_tail(o, v->g->names[v->g->name_idx[k]], pos, fwd, db, mm, tot, x->c->pam_len);
    (*x->n_rows)++;
}

static void mpat_init(mpat *mp, const creq *c, size_t p) {
    const size_t L = c->L;
    build_peq(mp, c->pat_ascii[p], L);
    mp->b4 = (uint8_t *)malloc(L);
    mp->is_n = (uint8_t *)malloc(L);
    mp->eff = (uint8_t *)malloc(L);
    mp->pam_f = (uint8_t *)malloc(L);
    uint8_t *f = (uint8_t *)malloc(L);
    memcpy(f, c->filter, L);
    if (p >= c->n_user) revcomp_inplace(f, L); /* search.rs:971-983 */
    for (size_t i = 0; i < L; i++) {
        mp->b4[i] = STR2B4[1][c->pat_ascii[p][i]];
        mp->is_n[i] = is_n_char(c->pat_ascii[p][i]);
        mp->eff[i] = STR2B4[1][f[i]];
    }
    free(f);
    /* precompute_pam_precheck (search.rs:761-777) */
    size_t ps = L;
    for (size_t i = 0; i < L; i++) if (mp->is_n[i]) { ps = i; break; }
    mp->pam_off = ps;
    mp->pam_n = 0;
    for (size_t i = ps; i < L; i++) if (mp->is_n[i]) mp->pam_f[mp->pam_n++] = mp->eff[i];
}
static void mpat_free(mpat *mp) { free(mp->b4); free(mp->is_n); free(mp->eff); free(mp->pam_f); }

/* search_chunk_myers (search.rs:779-897) over one batch. */
static void search_batch_myers(const bview *v, const creq *c, const mpat *mps, sbuf *out,
                               uint64_t *n_rows) {
    const size_t L = c->L;
    const uint8_t *gd = v->g->data + v->base; /* batch buffer = global slice */
    uint64_t active_start = v->has_head ? bv_off(v, 1) * 2 : 0;
    uint64_t total = v->valid * 2; /* chunk_byte_offsets[n_chunks] * 2 */
    size_t W = L + c->db;
    uint32_t max_edits = c->mm + c->db + c->rb;
    uint64_t mask = L < 64 ? (1ull << L) - 1 : ~0ull;
    uint64_t last = 1ull << (L - 1);
    uint8_t *text = (uint8_t *)malloc(W + 1);
    tbs t;
    memset(&t, 0, sizeof t);
    t.dp = (uint64_t *)malloc((L + 1) * (W + 1) * sizeof(uint64_t));
    t.max_edits = max_edits; t.max_db = c->db; t.max_rb = c->rb; t.max_mm = c->mm;
    t.emit = emit_alignment;
    mctx x;
    x.v = v; x.c = c; x.mp = mps; x.out = out; x.n_rows = n_rows;
    x.pa = (uint8_t *)malloc(L + W + 8);
    x.ta = (uint8_t *)malloc(L + W + 8);
    t.ctx = &x;
    for (size_t p = 0; p < c->n_pat; p++) {
        const mpat *mp = &mps[p];
        for (uint64_t tp = active_start; tp < total; tp++) {
            if (tp + 1 < L) continue;
            if (!check_pam_quick(gd, total, tp, L, mp, c->db, c->rb)) continue;
            uint64_t ts = tp + 1 > W ? tp + 1 - W : 0;
            uint64_t vp = mask, vn = 0;
            int32_t score = (int32_t)L;
            for (uint64_t q = ts; q <= tp; q++) {
                uint8_t b4 = get_bit4(gd, q);
                uint64_t eq;
                if (b4 == 0) eq = 0;
                else if (b4 == 0xF) eq = mp->peq_n;
                else {
                    eq = 0;
                    if (b4 & 4) eq |= mp->peq[0];
                    if (b4 & 2) eq |= mp->peq[1];
                    if (b4 & 8) eq |= mp->peq[2];
                    if (b4 & 1) eq |= mp->peq[3];
                }
                uint64_t xx = eq | vn;
                uint64_t d0 = (((xx & vp) + vp) ^ vp) | xx;
                uint64_t hn = vp & d0;
                uint64_t hp = vn | ~(vp | d0);
                uint64_t xs = hp << 1;
                vn = xs & d0;
                vp = (hn << 1) | ~(xs | d0);
                vp &= mask;
                vn &= mask;
                if (hp & last) score++;
                if (hn & last) score--;
            }
            if (score < 0 || (uint32_t)score > max_edits) continue;
            /* classify_myers_candidate (search.rs:597-631) */
            size_t tl = (size_t)(tp + 1 - ts);
            for (size_t q = 0; q < tl; q++) text[q] = get_bit4(gd, ts + q);
            t.pb4 = mp->b4; t.is_n = mp->is_n; t.text = text; t.m = L; t.n = tl;
            x.p = p; x.end_pos = tp; x.text_start = ts; x.text = text; x.text_len = tl;
            traceback_all(&t);
        }
    }
    free(text);
    free(t.dp);
    free(x.pa);
    free(x.ta);
}

/* ------------------------------------------------------------------------ */
/* driver: one worker per hardware thread pulling batches                   */
/* ------------------------------------------------------------------------ */

typedef struct {
    const orc_genome *g;
    const creq *c;
    const batch *batches;
    size_t nb;
    atomic_size_t next;
    sbuf *outs;
    uint64_t *rows;
    const uint64_t *pat;
    size_t pps;
    const mpat *mps;
    int use_myers;
    int scan_only;
    uint64_t *raw_counts;
} work;

static void *worker(void *arg) {
    work *w = (work *)arg;
    for (;;) {
        size_t b = atomic_fetch_add(&w->next, 1);
        if (b >= w->nb) break;
        bview v;
        bview_init(&v, w->g, &w->batches[b]);
        if (w->use_myers) {
            search_batch_myers(&v, w->c, w->mps, &w->outs[b], &w->rows[b]);
            continue;
        }
        size_t gb;
        uint64_t *buf = batch_buffer(&v, w->c->L, 1, &gb);
        hitvec h = {0, 0, 0};
        search_chunk_cpu(w->c->mm, w->c->L, w->pat, w->c->n_pat, buf, gb, msmin_of(&v, w->c->L), &h);
        if (w->scan_only) w->raw_counts[b] = h.n;
        else convert_and_write_popcount(&v, w->c, (const uint8_t *)buf, &h, &w->outs[b], &w->rows[b]);
        free(h.p);
        free(buf);
    }
    return NULL;
}

static int run(const orc_genome *g, const orc_request *req, size_t bbeg, size_t bend,
               int scan_only, char **rows, size_t *rows_len, uint64_t *n_rows,
               uint64_t *n_raw, char *err, size_t errlen) {
    tables();
    creq c;
    if (creq_init(&c, req, err, errlen)) { creq_free(&c); return -1; }
    uint32_t cps = req->chunks_per_search ? req->chunks_per_search : DEFAULT_CPS;
    if (cps < 2) { set_err(err, errlen, "chunks_per_search must be >= 2"); creq_free(&c); return -1; }
    batch *bs;
    size_t nb = make_batches(g, cps, &bs);
    if (bend > nb) bend = nb;
    if (bbeg > bend) bbeg = bend;
    work w;
    memset(&w, 0, sizeof w);
    w.g = g; w.c = &c; w.batches = bs + bbeg; w.nb = bend - bbeg;
    atomic_init(&w.next, 0);
    w.outs = (sbuf *)calloc(w.nb + 1, sizeof(sbuf));
    w.rows = (uint64_t *)calloc(w.nb + 1, sizeof(uint64_t));
    w.raw_counts = (uint64_t *)calloc(w.nb + 1, sizeof(uint64_t));
    w.scan_only = scan_only;
    w.use_myers = c.db > 0 || c.rb > 0;
    mpat *mps = NULL;
    if (w.use_myers) {
        mps = (mpat *)calloc(c.n_pat, sizeof(mpat));
        for (size_t p = 0; p < c.n_pat; p++) mpat_init(&mps[p], &c, p);
        w.mps = mps;
    } else {
        w.pat = pack_patterns(&c, &w.pps);
    }
    int nt = req->n_threads > 0 ? req->n_threads : (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (nt < 1) nt = 1;
    if ((size_t)nt > w.nb && w.nb > 0) nt = (int)w.nb;
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)nt);
    for (int i = 0; i < nt; i++) pthread_create(&th[i], NULL, worker, &w);
    for (int i = 0; i < nt; i++) pthread_join(th[i], NULL);
    free(th);
    sbuf all = {0, 0, 0};
    uint64_t nr = 0, raw = 0;
    for (size_t b = 0; b < w.nb; b++) {
        if (w.outs[b].n) sb_put(&all, w.outs[b].p, w.outs[b].n);
        free(w.outs[b].p);
        nr += w.rows[b];
        raw += w.raw_counts[b];
    }
    sb_reserve(&all, 1);
    all.p[all.n] = 0;
    if (rows) *rows = all.p; else free(all.p);
    if (rows_len) *rows_len = all.n;
    if (n_rows) *n_rows = nr;
    if (n_raw) *n_raw = raw;
    free(w.outs);
    free(w.rows);
    free(w.raw_counts);
    free((void *)w.pat);
    if (mps) {
        for (size_t p = 0; p < c.n_pat; p++) mpat_free(&mps[p]);
        free(mps);
    }
    free(bs);
    creq_free(&c);
    return 0;
}

int orc_search(const orc_genome *g, const orc_request *req, char **rows, size_t *rows_len,
               uint64_t *n_rows, char *err, size_t errlen) {
    return run(g, req, 0, (size_t)-1, 0, rows, rows_len, n_rows, NULL, err, errlen);
}

int orc_popcount_scan_only(const orc_genome *g, const orc_request *req, size_t batch_begin,
                           size_t batch_end, uint64_t *n_raw_hits, char *err, size_t errlen) {
    if (req->max_dna_bulges || req->max_rna_bulges) {
        set_err(err, errlen, "scan-only is the popcount path");
        return -1;
    }
    return run(g, req, batch_begin, batch_end, 1, NULL, NULL, NULL, n_raw_hits, err, errlen);
}
