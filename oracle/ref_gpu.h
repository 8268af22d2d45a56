/* Launcher for the reference's own CUDA kernels (test and measurement
 * infrastructure, not product code).
 *
 * The reference ships two device kernels, kernel.cu `find_matches` and
 * kernel_myers.cu `find_matches_myers`, which it JIT-compiles with NVRTC and
 * launches from Rust (search.rs:249-320 and :1054-1187).  Rust cannot be
 * built here, so this library restates those two host loops in C++ and
 * launches the unmodified kernels, compiled from the reference sources with
 * nvcc for sm_100a into oracle/_ref/ (recipe: oracle/Makefile, target
 * `ref`).  Uses: a second, independent check of the product's raw match
 * stream, and the speed of the reference's GPU path on the same B200.
 *
 * Deviations from search.rs, all outside the kernels:
 *  - the popcount output buffer is sized to the true match count of each
 *    batch instead of 1<<22 slots: find_matches appends without a bounds
 *    check (kernel.cu:104-112), so the count is taken first by sub-range
 *    launches of the same kernel whose worst case fits the buffer;
 *  - the device genome buffer has 256 bytes of zero padding after the
 *    batch budget, because a completely full batch makes the last threads
 *    read up to BLOCKS_PER_PATTERN words past it (kernel.cu:72-75);
 *  - a Myers request whose pattern N cells are not one contiguous run is
 *    refused, because the kernel would index past its PAM filter table
 *    (kernel_myers.cu:297-298).
 */
#ifndef REF_GPU_H
#define REF_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* kernel.cu s_match (kernel.cu:36-42), 16 bytes */
typedef struct {
    uint32_t loc;
    uint32_t pattern_idx;
    uint32_t mismatches;
    uint16_t dna_bulge_size;
    uint16_t rna_bulge_size;
} refgpu_pmatch;

/* kernel_myers.cu s_match / search.rs GpuEnumMatch, 32 bytes */
typedef struct {
    uint32_t chunk_idx;
    uint32_t pattern_idx;
    uint64_t ops_packed;
    uint32_t mismatches;
    uint16_t dna_bulge_size;
    uint16_t rna_bulge_size;
    uint32_t ops_count;
    uint32_t pad;
} refgpu_mmatch;

typedef struct {
    double kernel_ms;   /* sum of kernel durations (CUDA events) */
    double h2d_ms;      /* batch and counter uploads (synchronous, pageable) */
    double d2h_ms;      /* count and match read-back */
    double host_ms;     /* tight packing and N masking of the batch buffers */
    double wall_ms;     /* whole device loop */
    uint64_t launches;
    uint64_t n_batches;
    uint64_t matches;   /* matches read back over all batches */
} refgpu_times;

typedef struct refgpu_ctx refgpu_ctx;

/* Chunks as the reference's reader yields them (bit4, ceil(len/2) bytes),
 * batched like search.rs:1531-1572 with `chunks_per_search` chunks per batch
 * (0 = 16384, the GPU batch of init_search_chunk_nucl_from_devices).  The
 * chunk bytes are borrowed and must outlive the context. */
refgpu_ctx *refgpu_open(const uint8_t *const *chunk_data, const uint64_t *chunk_start,
                        const uint64_t *chunk_end, size_t n_chunks, uint32_t chunks_per_search,
                        int device, char *err, size_t errlen);
size_t refgpu_n_batches(const refgpu_ctx *c);
/* first chunk index, chunk count and head flag of batch b */
void refgpu_batch(const refgpu_ctx *c, size_t b, size_t *first, size_t *n, int *head);
void refgpu_close(refgpu_ctx *c);

/* Exact number of matches find_matches appends in every batch, taken with
 * sub-range launches of at most count_cap / (32 * n_patterns) threads per
 * pattern row, so no launch can write past its count_cap-slot buffer. */
int refgpu_popcount_count(refgpu_ctx *c, const char *cubin, const char *const *patterns,
                          size_t n_patterns, uint32_t max_mismatches, uint64_t count_cap,
                          uint64_t *batch_counts, char *err, size_t errlen);

/* search_device_cuda (search.rs:249-320): one launch per batch into a buffer
 * of `capacity` slots, which must be >= every batch count (from
 * refgpu_popcount_count; checked).  Matches are copied into `out` (nullable)
 * batch after batch; batch_offsets[b] (nullable, n_batches + 1 entries) gets
 * each batch's first index. */
int refgpu_popcount_run(refgpu_ctx *c, const char *cubin, const char *const *patterns,
                        size_t n_patterns, uint32_t max_mismatches, uint64_t capacity,
                        const uint64_t *batch_counts, refgpu_pmatch *out, uint64_t out_cap,
                        uint64_t *batch_offsets, refgpu_times *t, char *err, size_t errlen);

/* search_device_cuda_myers (search.rs:1054-1187) with the tables of
 * search_chunk_cuda_myers (:1189-1262): bisected sub-range launches into a
 * buffer of out_buf_size slots (the OUT_BUF_SIZE the cubin was built with). */
int refgpu_myers_run(refgpu_ctx *c, const char *cubin, const char *search_filter,
                     const char *const *patterns, size_t n_patterns, size_t n_fwd_patterns,
                     uint32_t out_buf_size, refgpu_mmatch *out, uint64_t out_cap,
                     uint64_t *batch_offsets, refgpu_times *t, char *err, size_t errlen);

/* search()'s raw Match lines of the Myers records `recs` (from
 * refgpu_myers_run, batch_offsets as it filled them): decode_gpu_enum_match
 * (search.rs:152-206) and convert_matches_myers (search.rs:1316-1374), the
 * line format of the product's COF_F_RAW_MATCHES.  chunk_names: the record
 * name of every chunk.  Returns a malloc'd NUL-terminated text (free with
 * refgpu_free), or NULL when out of memory. */
char *refgpu_myers_lines(refgpu_ctx *c, const char *const *chunk_names,
                         const char *const *patterns, size_t n_patterns, size_t n_fwd_patterns,
                         const refgpu_mmatch *recs, const uint64_t *batch_offsets,
                         uint64_t *text_len, uint64_t *n_lines);
void refgpu_free(void *p);

#ifdef __cplusplus
}
#endif

#endif
