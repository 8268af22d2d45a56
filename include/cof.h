/*
 * cof.h -- C ABI of the B200 off-target search engine (libcof.so).
 *
 * This is the drop-in boundary for cas-offinder-rust's search path.  The
 * Rust entry point it replaces is
 *
 *   pub fn search(devices: OclRunConfig, max_mismatches: u32,
 *                 max_dna_bulges: u32, max_rna_bulges: u32,
 *                 search_filter_ascii: &[u8], pattern_len: usize,
 *                 patterns_ascii: &Vec<Vec<u8>>,
 *                 recv: mpsc::Receiver<ChromChunkInfo>,
 *                 dest: mpsc::SyncSender<Vec<Match>>)
 *   (cas-offinder-lib/src/search.rs:1490-1500)
 *
 * together with the writer thread that turns its Match stream into the
 * cas-offinder 2.5 / cas-offinder-bulge 8-column rows
 * (cas-offinder-cli/src/main.rs:122-247).  The ChromChunkInfo channel becomes
 * a genome handle that is filled once (chunk by chunk, or from a FASTA/.2bit
 * path) and then stays resident in HBM across searches.
 *
 * Every function returns COF_OK (0) or a negative status; the message of the
 * last failure on the calling thread is available from cof_last_error().  No
 * call aborts the process.  One genome handle drives one GPU; calls on the
 * same handle are serialised internally.
 */
#ifndef COF_H
#define COF_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define COF_API __attribute__((visibility("default")))
#else
#define COF_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The reference panics on these conditions
 * (search.rs:1502-1507 asserts, :1617 and :1655 CUDA errors, loader
 * CliError unwraps in main.rs:106-121). */
#define COF_OK 0
#define COF_E_BADINPUT (-1)    /* invalid request, pattern or genome file  */
#define COF_E_OOM (-2)         /* device or host allocation failed         */
#define COF_E_CUDA (-3)        /* CUDA runtime error                       */
#define COF_E_IO (-4)          /* genome file could not be read            */
#define COF_E_UNSUPPORTED (-5) /* valid input outside the library's limits */
#define COF_E_STATE (-6)       /* call order (e.g. add_chunk after upload) */
#define COF_E_TIMEOUT (-7)     /* a bounded device wait gave up            */
#define COF_E_CANCELLED (-8)   /* a result sink stopped the search         */

/* Request flags. */
#define COF_F_ADD_REVCOMP 1u   /* patterns are user patterns; append their
                                  reverse complements as main.rs:253-259 does */
#define COF_F_RAW_MATCHES 2u   /* return search()'s raw Match stream instead of
                                  the writer's rows: one line per Match
                                  (chrom_chunk.rs:19-29),
                                  name \t chrom_idx \t pattern_idx \t +|- \t
                                  mismatches \t dna_bulge_size \t
                                  rna_bulge_size \t rna_seq \t dna_seq \n;
                                  the popcount path's raw stream has no PAM
                                  filter (the writer applies it), its
                                  mismatches are max(kernel count, 0) and its
                                  dna_seq keeps NUL bytes for N and padding */

typedef struct cof_genome cof_genome;

/* Creates an empty genome bound to CUDA device `device`.
 * Replaces the Receiver<ChromChunkInfo> side of search.rs:1498. */
COF_API int cof_genome_create(int device, cof_genome **out);

/* Appends one chunk, in stream order.  Fields of ChromChunkInfo
 * (cas-offinder-lib/src/chrom_chunk.rs:4-16): the record name, the bit4
 * one-hot data (two nucleotides per byte, even index in the low nibble,
 * ceil((chunk_end - chunk_start) / 2) bytes), and the nucleotide range
 * [chunk_start, chunk_end) within the record; chunk_start == 0 starts a new
 * record.  At most 65536 nucleotides per chunk. */
COF_API int cof_genome_add_chunk(cof_genome *g, const char *chr_name,
                                 const uint8_t *bit4, uint64_t chunk_start,
                                 uint64_t chunk_end);

/* Loads a genome path the way cas-offinder-cli/src/main.rs:106-121 does:
 * a directory -> read_fasta_folder, first byte '>' -> read_fasta, otherwise
 * read_2bit (cas-offinder-lib/src/read_fasta.rs:9-71, read_2bit.rs:33-118,
 * read_fasta_folder.rs:8-23).  May be mixed with cof_genome_add_chunk.
 * A single FASTA or .2bit file loaded into an empty genome is only indexed
 * here (chunk table, names, N ranges); its bases are read from the file
 * again and converted on the device by cof_genome_upload (or the first
 * search), so the file must not change in between -- a changed size or line
 * count fails the upload with COF_E_IO.  Adding chunks or files to such a
 * genome converts its bases on the host first. */
COF_API int cof_genome_load(cof_genome *g, const char *path);

/* Packs the chunk stream into HBM (bit4 stream + 2-bit/N-mask planes).
 * Called implicitly by the first search; after it no chunk may be added. */
COF_API int cof_genome_upload(cof_genome *g);

COF_API uint64_t cof_genome_n_nucl(const cof_genome *g);
COF_API uint64_t cof_genome_n_chunks(const cof_genome *g);
COF_API void cof_genome_free(cof_genome *g);

/* One search, with the arguments of search() (search.rs:1490-1500).
 * patterns: patterns_ascii, all of length pattern_len; the first half are
 * the forward patterns and the second half the reverse strand (as main.rs
 * builds them), unless COF_F_ADD_REVCOMP is set, in which case they are the
 * user patterns and the library appends the reverse complements.
 * max_dna_bulges or max_rna_bulges > 0 selects the bulge (Myers) path
 * exactly as search.rs:1513 does.
 * chunks_per_search: 64 Knt chunks per search batch; 0 selects 16384, the
 * batch search() uses with a GPU device (search.rs:22, :44-50).
 * pattern_len: at most 64 on every path (the bulge path's Myers filter is
 * one u64 word in the reference, myers.rs:3), and pattern_len +
 * max_dna_bulges at most 72; longer requests fail with COF_E_UNSUPPORTED. */
typedef struct {
    const char *search_filter;
    size_t pattern_len;
    const char *const *patterns;
    size_t n_patterns;
    uint32_t max_mismatches;
    uint32_t max_dna_bulges;
    uint32_t max_rna_bulges;
    uint32_t flags;
    uint32_t chunks_per_search;
} cof_request;

/* Output of one request: the writer's rows (main.rs:130-245) without the
 * header line, '\n'-terminated.  Popcount rows are ordered by genome
 * position, then by pattern (the order of cof_request.patterns, then their
 * reverse complements); bulge rows by pattern, then position, within each
 * candidate chunk (a large result is walked in several chunks).  The
 * reference's order is unspecified; compare sorted. */
typedef struct {
    char *text;
    size_t text_len;
    uint64_t n_rows;
    double device_ms;      /* device time of this call's kernels + copies */
} cof_result;

/* The header line main.rs:131-135 writes before the rows. */
#define COF_HEADER \
    "#Bulge type\tcrRNA\tDNA\tChromosome\tPosition\tDirection\tMismatches\tBulge Size\n"

/* search() followed by main.rs's writer, for one request. */
COF_API int cof_search(cof_genome *g, const cof_request *req, cof_result *out);

/* Many requests over one genome pass: guide sets of different lengths,
 * PAMs and thresholds are scanned by one persistent launch per kernel
 * stage.  outs[i] receives exactly what cof_search(reqs[i]) would return.
 * No reference counterpart (the reference takes one filter per run,
 * cli_utils.rs:97-108). */
COF_API int cof_search_batch(cof_genome *g, const cof_request *reqs, size_t n_reqs,
                             cof_result *outs);

COF_API void cof_result_free(cof_result *r);

/* Streamed results: search()'s `dest: SyncSender<Vec<Match>>` channel
 * (search.rs:1490-1500), through which the reference hands batches of
 * matches to the writer thread while the search runs (the Myers host emits
 * them per sub-range, search.rs:1106-1168).  Instead of one whole-result
 * buffer per request, the rows reach a callback piece by piece -- a
 * popcount genome slice, a bulge candidate chunk, or one request's rows of
 * a pass -- while the GPU works on the next piece, so a result may be far
 * larger than host memory.  Host memory in use stays at a few pieces. */

/* One Match (cas-offinder-lib/src/chrom_chunk.rs:19-29) as plain data,
 * 32 bytes.  The dna and rna strings of the Match are the fields of its
 * line in the piece's text: columns 2 and 3 of a row, 8 and 9 of a raw
 * Match line. */
typedef struct {
    uint64_t chrom_idx;      /* Match.chrom_idx: position of the site's first
                                cell in its record (the writer prints
                                chrom_idx + pam_len - 1 - db for '-' rows,
                                main.rs:229-236) */
    uint64_t text_offset;    /* byte offset of this match's line in the
                                piece's text */
    uint32_t record;         /* record index (cof_genome_record_name) */
    uint32_t pattern_idx;    /* Match.pattern_idx: index into the request's
                                full pattern list (forward, then reverse) */
    uint8_t mismatches;      /* Match.mismatches (the writer's recount) */
    uint8_t dna_bulge_size;  /* Match.dna_bulge_size */
    uint8_t rna_bulge_size;  /* Match.rna_bulge_size */
    uint8_t is_forward;      /* Match.is_forward */
    uint32_t pad;
} cof_match;

/* A piece of one request's output, in the order of that request's
 * cof_search text: concatenating a request's pieces gives its cof_search
 * text (for the bulge path, whose row order depends on candidate order,
 * the same rows).  text and matches are valid only during the callback. */
typedef struct {
    size_t request;             /* index into the call's request array */
    const char *text;           /* rows (or raw Match lines), each ending '\n' */
    size_t text_len;
    uint64_t n_rows;
    const cof_match *matches;   /* n_rows records in text order with
                                   COF_STREAM_MATCHES, else NULL (always NULL
                                   for the popcount path's raw stream) */
} cof_piece;

/* Receives each piece on the calling thread; a nonzero return stops the
 * search, which then returns COF_E_CANCELLED. */
typedef int (*cof_sink)(void *user, const cof_piece *piece);

#define COF_STREAM_MATCHES 1u  /* pieces carry cof_match records */

/* cof_search_batch with results streamed to `sink`.  n_rows (nullable, n_reqs
 * entries) receives each request's row count. */
COF_API int cof_search_stream(cof_genome *g, const cof_request *reqs, size_t n_reqs,
                              uint32_t stream_flags, cof_sink sink, void *user,
                              uint64_t *n_rows);

/* Name of record `record` (cof_match.record): the FASTA header line after
 * '>' or the .2bit sequence name (Match.chr_name); NULL if out of range.
 * Valid while the genome lives. */
COF_API const char *cof_genome_record_name(const cof_genome *g, uint32_t record);
COF_API uint32_t cof_genome_n_records(const cof_genome *g);

/* Continuous-batching request server over a resident genome.  No reference
 * counterpart.  A worker thread walks the genome as a ring of ring_slices
 * slices, one slice per step: every step searches one slice for all active
 * requests in one batched pass (cof_search_batch restricted to the slice's
 * pattern starts, or alignment ends with bulges).  Before each step it
 * admits queued requests in arrival order while their estimated device
 * memory for candidate and row buffers fits memory_budget_bytes (0 = half
 * of the device memory free after the genome upload) and, if
 * max_requests_per_pass > 0, while the active requests number at most that
 * many.  So a request that arrives while others are on the GPU joins them
 * at the next slice boundary, and completes after one full turn of the
 * ring, its slices' rows joined in genome order: the text cof_search gives
 * (byte for byte on the popcount path; the same rows on the bulge path).
 * ring_slices 0 picks about one slice per 512 Mnt (at most 16); 1 runs
 * whole-genome passes.  max_requests_per_pass = 1 gives the plain
 * one-request-per-pass loop (whole-genome passes).  Direct searches on the
 * same genome are serialised with the server's steps. */
typedef struct cof_server cof_server;
typedef struct {
    uint32_t max_requests_per_pass;
    uint64_t memory_budget_bytes;
    uint32_t ring_slices;
} cof_server_config;

COF_API int cof_server_create(cof_genome *g, const cof_server_config *cfg, cof_server **out);
/* Queues a copy of *req; *ticket identifies it for cof_server_wait. */
COF_API int cof_server_submit(cof_server *s, const cof_request *req, uint64_t *ticket);
/* Waits up to timeout_ms (< 0: forever) for a ticket; COF_E_TIMEOUT if it is
 * still pending.  On completion fills *out (free with cof_result_free) and
 * *latency_ms (submit to completion, host clock) and forgets the ticket. */
COF_API int cof_server_wait(cof_server *s, uint64_t ticket, int64_t timeout_ms, cof_result *out,
                            double *latency_ms);
/* stats4 = {steps (slice searches; whole-genome passes when the ring has
 * one slice), completed requests, queued requests, most requests active in
 * one step}. */
COF_API int cof_server_stats(cof_server *s, uint64_t *stats4);
/* Finishes the queued requests, stops the worker and frees the server. */
COF_API void cof_server_free(cof_server *s);

/* Device timings and counters of the last search on `g`: ms5 = {scan,
 * verify, format, device->host copy, total} milliseconds (CUDA events);
 * counts5 = {PAM-passing windows, window x pattern comparisons, scan
 * candidates, rows, kernel launches}.  Instrumentation for benchmarks; no
 * reference counterpart. */
COF_API int cof_genome_last_stats(const cof_genome *g, double *ms5, uint64_t *counts5);

/* Popcount search over one sequence that already sits in device memory,
 * without allocating any memory.  No counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc: an application whose own pool
 * allocator owns the device memory and only hands out pointers into it (an
 * allocation from this library would bypass or exceed that pool), or a
 * serving loop that must not allocate while requests are in flight because
 * allocation can synchronise the whole device.  The caller passes the input
 * and the output as device pointers; counters, pattern tables and the
 * candidate list live in one fixed device array of 8 MiB that every GPU which
 * loads libcof.so keeps until the process exits.
 *
 * d_bit4: one record of n_nucl nucleotides in the reference's bit4 one-hot
 * encoding (two per byte, even index in the low nibble), 16-byte aligned,
 * n_nucl < 2^31.  patterns: the full fwd + reverse list as search() takes
 * it (the forward patterns, then as many reverse complements: an odd count
 * is rejected with COF_E_BADINPUT), 2..512 patterns of the filter's length
 * (<= 32).  Rows are the writer's
 * rows of cof_search for a genome made of this one record: every window start
 * s with s + L <= n_nucl that passes the PAM filter and the mismatch
 * recount.  Each row is three uint32 in d_rows: s (0-based, the scan
 * orientation start), pattern index, mismatches; order unspecified.
 * *n_rows receives the number of rows found; if it exceeds rows_cap, rows_cap
 * of them (in no particular order) are written and COF_E_UNSUPPORTED is
 * returned.  Requests
 * beyond the stated maximums are rejected with COF_E_UNSUPPORTED and a
 * message in cof_last_error(), and so is a call whose row count would not
 * fit 32 bits (*n_rows is then 0xFFFFFFFF).  stream: a cudaStream_t
 * (NULL = default) of the current device; a stream of another device is
 * rejected with COF_E_BADINPUT.
 *
 * The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) with that device current; make it before any
 * stream capture.  The address is kept until the process exits, so a
 * cudaDeviceReset of that device ends the use of this entry point there.
 * All calls share the array and leave their data in it;
 * each call clears its counters first.  Calls are serialised inside the
 * library and wait for their stream before returning; work from two calls
 * that overlapped on the GPU would race on the shared array. */
COF_API int cof_search_seq_noalloc(const uint8_t *d_bit4, uint64_t n_nucl,
                                   const char *search_filter, const char *const *patterns,
                                   size_t n_patterns, uint32_t max_mismatches,
                                   uint32_t *d_rows, uint32_t rows_cap, uint32_t *n_rows,
                                   void *stream);

/* Autotuner state as JSON: {"last": tile shape of the last scan, "variant":
 * its index, "cache": {request-shape key: variant index}}.  The scan's tile
 * shape is chosen per request shape by timing the candidate shapes on a
 * sample of the genome at the first search of that shape (COF_AUTOTUNE=0
 * turns this off; COF_TUNE_CACHE=<file> persists the choices).  No reference
 * counterpart. */
COF_API int cof_genome_tuning(cof_genome *g, char *buf, size_t len);

/* Message of the last failed call on this thread ("" if none). */
COF_API const char *cof_last_error(void);

/* ABI version of this header. */
#define COF_ABI_VERSION 2
COF_API int cof_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif
