/*
 * cof_oracle.h -- CPU restatement of cas-offinder-rust's off-target search.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA
 * product in cas-offinder-rust-old_b200/: the parity tests, the smoke check
 * and the CPU-baseline leg of bench.py link it.  Nothing in the product path
 * calls it.
 *
 * What it restates (paths relative to the reference project root):
 *   cas-offinder-lib/src/bit4ops.rs        bit4 tables, revcomp, cmp_chars
 *   cas-offinder-lib/src/read_fasta.rs     FASTA -> 64 Knt chunks
 *   cas-offinder-lib/src/read_2bit.rs      .2bit -> 64 Knt chunks
 *   cas-offinder-lib/src/read_fasta_folder.rs
 *   cas-offinder-lib/src/search.rs         batcher (1376-1427, 1531-1572),
 *                                          popcount CPU scan (378-463),
 *                                          N masking (512-531), head overlap
 *                                          (540-546), convert (1428-1488),
 *                                          Myers CPU path (597-1031),
 *                                          convert_matches_myers (1316-1374)
 *   cas-offinder-lib/src/myers.rs          build_peq (32-50)
 *   cas-offinder-lib/src/traceback.rs      traceback_all / enumerate (181-381)
 *   cas-offinder-cli/src/main.rs           fwd+rc patterns (253-259), writer
 *                                          post-filter and row format
 *                                          (80-91, 130-245)
 *   cas-offinder-cli/src/cli_utils.rs      input-file parser (37-125)
 *
 * Parity pins: the reader golden (cas-offinder-lib/tests/file_test.rs with
 * tests/test_data/expected.txt) and the 117-row popcount count pin
 * (cas-offinder-lib/tests/integration_bulge.rs:156-176); see tests/.
 */
#ifndef COF_ORACLE_H
#define COF_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_genome orc_genome;

/* Loads a genome the way cas-offinder-cli/src/main.rs:106-121 dispatches:
 * a directory -> every *.fa file in readdir order, a file whose first byte is
 * '>' -> FASTA, anything else -> .2bit.  Returns NULL and fills err on error. */
orc_genome *orc_genome_load(const char *path, char *err, size_t errlen);
void orc_genome_free(orc_genome *g);

/* Builds a genome from chunks sent one by one, like the ChromChunkInfo
 * channel (chrom_chunk.rs:4-16): name, bit4 bytes (ceil(n/2)), start, end.
 * A chunk with start == 0 opens a new record name. */
orc_genome *orc_genome_new(void);
int orc_genome_add_chunk(orc_genome *g, const char *name, const uint8_t *bit4,
                         uint64_t chunk_start, uint64_t chunk_end);

/* Number of 64 Knt chunks, total valid nucleotides. */
size_t orc_genome_n_chunks(const orc_genome *g);
uint64_t orc_genome_n_nucl(const orc_genome *g);

/* Chunk accessors (name, chunk_start, chunk_end, bit4 bytes). */
const char *orc_chunk_name(const orc_genome *g, size_t k);
uint64_t orc_chunk_start(const orc_genome *g, size_t k);
uint64_t orc_chunk_end(const orc_genome *g, size_t k);
const uint8_t *orc_chunk_data(const orc_genome *g, size_t k);

/* Concatenation of bit4_to_string over every chunk, the string the reader
 * tests compare with expected.txt (file_test.rs:17-25).  Caller frees with
 * orc_free. */
char *orc_genome_decode(const orc_genome *g, size_t *len);

/* One search request, as main.rs hands it to search(): the user patterns
 * (the oracle appends their reverse complements, main.rs:253-259), the
 * filter, the thresholds.  cps = chunks per search batch (16384 for a GPU
 * device, 64 for the CPU device; search.rs:21-50).  n_threads = worker
 * threads (0 = all hardware threads, like search.rs:556).
 *
 * On success *rows is a malloc'd buffer of output rows (one per line, the
 * 8-column format of main.rs:237-242, header not included) in unspecified
 * order and *rows_len its length; *n_rows the row count.  Returns 0, or a
 * negative status with a message in err. */
typedef struct {
    const char *filter;          /* search filter, length = pattern_len */
    const char *const *patterns; /* user patterns */
    size_t n_patterns;
    uint32_t max_mismatches;
    uint32_t max_dna_bulges;
    uint32_t max_rna_bulges;
    uint32_t chunks_per_search;  /* 0 -> 16384 */
    int n_threads;               /* 0 -> hardware threads */
    int raw_matches;             /* 1: emit search()'s Match stream instead of
                                    the writer's rows (see below) */
} orc_request;

/* Raw Match lines (raw_matches = 1), one per element of the Vec<Match>
 * batches search() sends (chrom_chunk.rs:19-29; built at search.rs:1474-1484
 * and :1361-1371):
 *   chr_name \t chrom_idx \t pattern_idx \t +|- \t mismatches \t
 *   dna_bulge_size \t rna_bulge_size \t rna_seq \t dna_seq \n
 * The popcount path's dna_seq may contain NUL bytes (N and padding decode to
 * 0 on the masked batch buffer); its mismatches are max(kernel count, 0). */

int orc_search(const orc_genome *g, const orc_request *req, char **rows,
               size_t *rows_len, uint64_t *n_rows, char *err, size_t errlen);

/* Popcount-path raw stage only (search_chunk_cpu over every batch, no
 * convert / writer), used to time the CPU baseline over a bounded slice of
 * the genome: scans batches [batch_begin, batch_end) and returns the number
 * of raw kernel hits.  Patterns are the full fwd+rc list, pre-encoded. */
int orc_popcount_scan_only(const orc_genome *g, const orc_request *req,
                           size_t batch_begin, size_t batch_end,
                           uint64_t *n_raw_hits, char *err, size_t errlen);

/* Number of search batches for cps chunks per batch. */
size_t orc_n_batches(const orc_genome *g, uint32_t cps);

void orc_free(void *p);

#ifdef __cplusplus
}
#endif
#endif
