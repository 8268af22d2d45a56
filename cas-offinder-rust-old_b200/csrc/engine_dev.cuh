// engine_dev.cuh -- device-side definitions shared by the popcount path
// (engine.cu) and the bulge path (bulge.cu): the resident genome, search
// batches, small device helpers and scratch buffers.
#pragma once

#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "cof_engine.h"

namespace cof {

#define CU(call)                                                                     \
    do {                                                                             \
        cudaError_t e_ = (call);                                                     \
        if (e_ != cudaSuccess) {                                                     \
            err = {e_ == cudaErrorMemoryAllocation ? kOom : kCuda,                   \
                   std::string(#call) + ": " + cudaGetErrorString(e_)};              \
            return err.code;                                                         \
        }                                                                            \
    } while (0)

// One search batch of the reference (SearchChunkInfo, search.rs:57-90): the
// chunks [first, first + nch) of the stream, starting at nucleotide `base`.
struct BatchDev {
    uint64_t base;         // global nucleotide index of the batch start
    uint32_t valid;        // valid nucleotides (2 x tight-packed bytes)
    uint32_t pad0;
    uint32_t first;        // first chunk
    uint32_t nch;          // chunks in the batch
    uint32_t active_start; // Myers active start (search.rs:1087-1091)
    uint32_t pad;
};

// BIT4_TO_STR of bit4ops.rs:118 for one nibble: 0 -> NUL, T C Y A W M H G
// K S B R D V N for 1..15 (one byte per nibble value, little endian).
__device__ __forceinline__ char b4char(uint32_t v) {
    constexpr unsigned long long lo = 0x484D574159435400ull;  // 7..0: H M W A Y C T NUL
    constexpr unsigned long long hi = 0x4E56445242534B47ull;  // 15..8: N V D R B S K G
    return (char)(((v & 8) ? hi : lo) >> ((v & 7) * 8));
}

// Popcount path records.
struct Hit {
    uint32_t s_local, pattern, batch, pad;
};

struct Row {
    uint64_t s_global;   // window start
    uint64_t clip;       // batch end (exclusive); cells at or past it read 0
    uint64_t pos;        // chrom_idx (record coordinate)
    uint32_t chunk;
    uint32_t pattern;
    uint32_t mm;
    uint32_t pad;
};

struct Counters {
    uint32_t hits;
    uint32_t rows;
    uint32_t overflow;
    uint32_t pad;
    unsigned long long candidates;
    unsigned long long pairs;
    unsigned long long next_item;  // work-item counter of the persistent scan
};

// Bulge path records.
// A Myers/PAM candidate: end position t (batch-local) of pattern p.
struct MyersCand {
    uint32_t t_local, batch, pattern, pad;
};
// One enumerated alignment that survived classify and convert.
struct MyersRow {
    uint64_t start;      // global nucleotide index of the alignment start
    uint64_t pos;        // chrom_idx (record coordinate)
    uint64_t ops[2];     // 2 bits per op, forward order: 0 M, 1 S, 2 DNA bulge, 3 RNA bulge
    uint32_t chunk, pattern;
    uint8_t n_ops, mm, db, rb;
    uint32_t ops_hi;     // ops 64..79 (patterns of 33..64 cells with DNA bulges)
};

// op k (forward order) of an alignment row
__device__ __forceinline__ uint32_t mrow_op(const MyersRow &w, uint32_t k) {
    const uint64_t x = k < 32 ? w.ops[0] >> (2 * k)
                     : k < 64 ? w.ops[1] >> (2 * (k - 32))
                              : (uint64_t)(w.ops_hi >> (2 * (k - 64)));
    return (uint32_t)(x & 3);
}

__device__ __forceinline__ uint8_t nib(const uint8_t *__restrict__ g, uint64_t i) {
    uint8_t b = __ldg(g + (i >> 1));
    return (i & 1) ? (uint8_t)(b >> 4) : (uint8_t)(b & 0xF);
}
__device__ __forceinline__ uint8_t dcomp4(uint8_t v) {
    return (uint8_t)(((v << 2) | (v >> 2)) & 0xF);
}
__device__ __forceinline__ bool single_base(uint8_t v) { return v && !(v & (v - 1)); }

struct GenomeDev {
    const uint8_t *bit4;
    const uint64_t *boff, *start, *end;
    const uint32_t *name_idx;
    const char *names;
    const uint32_t *name_off;
    uint64_t n_chunks;
    // bulge row sort keys: pattern << key_shift | global start, with
    // 2^key_shift above every start, so the sort covers only the bits in use
    uint32_t key_shift;
};

__device__ __forceinline__ uint32_t ndigits(uint64_t v) {
    uint32_t d = 1;
    while (v >= 10) { v /= 10; ++d; }
    return d;
}
__device__ __forceinline__ char *put_u64(char *o, uint64_t v) {
    char t[20];
    int k = 0;
    do { t[k++] = (char)('0' + v % 10); v /= 10; } while (v);
    while (k) *o++ = t[--k];
    return o;
}

// A slot in an append-only list: the lanes that append together take
// consecutive slots with one atomic on the list's counter.
__device__ __forceinline__ uint32_t append_slot(uint32_t *counter) {
    namespace cg = cooperative_groups;
    const cg::coalesced_group g = cg::coalesced_threads();
    uint32_t base = 0;
    if (g.thread_rank() == 0) base = atomicAdd(counter, g.size());
    return g.shfl(base, 0) + g.thread_rank();
}

// Starting entries of a candidate list (scan hits, Myers candidates); a
// search that overflows it grows it and runs again.  COF_CAND_CAP lowers the
// start (tests of the overflow path).
inline size_t first_cand_cap() {
    size_t cap = size_t(1) << 22;
    if (const char *e = std::getenv("COF_CAND_CAP")) {
        const long v = std::atol(e);
        if (v > 0) cap = std::min(cap, (size_t)v);
    }
    return cap;
}

template <class T>
struct DevBuf {
    T *p = nullptr;
    size_t cap = 0;
    // Grows to at least n elements; contents are not kept.  The new buffer
    // is allocated before the old one is freed, so it never reuses the old
    // address: a pointer still held to the old buffer cannot pass for the
    // new one (the overflow tests depend on that).
    int ensure(size_t n, Error &err) {
        if (n <= cap) return kOk;
        const size_t want = std::max<size_t>(n, 64);
        T *q = nullptr;
        const cudaError_t e = cudaMalloc((void **)&q, want * sizeof(T));
        if (e != cudaSuccess) {  // retry with the old buffer released first
            cudaGetLastError();
            if (p) cudaFree(p);
            p = nullptr;
            cap = 0;
            CU(cudaMalloc((void **)&q, want * sizeof(T)));
        } else if (p) {
            cudaFree(p);
        }
        p = q;
        cap = want;
        return kOk;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
};

// Copies file bytes [begin, begin + n) to device memory dst through
// page-locked staging buffers on several host threads (twobit.cu); fails if
// the file's size is no longer file_bytes.  Returns when the copy is done.
int copy_file_to_device(const std::string &path, uint64_t file_bytes, uint64_t begin,
                        uint64_t n, uint8_t *dst, int device, Error &err);
// Copies a planned .2bit file's packed bases to the device and decodes them
// into bit4 (twobit.cu); returns after the decode has finished on s.
int upload_2bit(const TwoBitPlan &plan, uint8_t *bit4, int device, cudaStream_t s, Error &err);
// Copies a planned FASTA file to the device and converts its chunks' lines
// into bit4 (fasta_dev.cu); returns after the conversion has finished on s.
int upload_fasta(const FastaPlan &plan, uint8_t *bit4, uint64_t bit4_bytes, int device,
                 cudaStream_t s, Error &err);

class DeviceGenome {
  public:
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t copy_stream = nullptr;  // result text to the host, beside the next slice's scan
    cudaEvent_t ev[10] = {};
    cudaEvent_t fmt_done = nullptr, copy_done = nullptr;  // a slice's text written / copied
    int n_sm = 0;
    DevBuf<uint8_t> bit4;
    DevBuf<uint32_t> planes;
    uint64_t n_words = 0;
    DevBuf<uint64_t> boff, start, end;
    DevBuf<uint32_t> name_idx, name_off;
    DevBuf<char> names;
    uint64_t n_chunks = 0;
    // per-search scratch
    DevBuf<unsigned char> tables;
    DevBuf<Hit> hits;
    DevBuf<Row> rows;
    DevBuf<uint64_t> keys, keys2, offs;
    DevBuf<uint32_t> vals, vals2, lens, req_rows;
    DevBuf<Counters> ctr;
    DevBuf<char> text;
    DevBuf<unsigned char> cub_tmp;
    DevBuf<MyersCand> mcand, mcand2;
    DevBuf<MyersRow> mrows;
    DevBuf<unsigned char> tb_items;  // two queues of handed-on traceback subtrees
    DevBuf<MatchRec> recs;           // match records of a streamed piece
    DevBuf<uint32_t> req_first;      // first sorted row of each request in a piece
    DevBuf<uint64_t> bandtbl;        // band tables of a bulge chunk's survivors

    ~DeviceGenome() {
        bit4.release(); planes.release(); boff.release(); start.release(); end.release();
        name_idx.release(); name_off.release(); names.release(); tables.release();
        hits.release(); rows.release(); keys.release(); keys2.release(); offs.release();
        vals.release(); vals2.release(); lens.release(); req_rows.release(); ctr.release();
        text.release(); cub_tmp.release(); mcand.release(); mcand2.release(); mrows.release();
        tb_items.release(); recs.release(); req_first.release(); bandtbl.release();
        for (auto &e : ev)
            if (e) cudaEventDestroy(e);
        if (fmt_done) cudaEventDestroy(fmt_done);
        if (copy_done) cudaEventDestroy(copy_done);
        if (copy_stream) cudaStreamDestroy(copy_stream);
        if (stream) cudaStreamDestroy(stream);
    }
    // bits of the largest global nucleotide index (the plane words cover
    // every start)
    uint32_t key_shift() const {
        uint32_t b = 1;
        while (b < 63 && (1ull << b) <= n_words * 32) ++b;
        return b;
    }
    GenomeDev view() const {
        return GenomeDev{bit4.p, boff.p,   start.p,  end.p,       name_idx.p,
                         names.p, name_off.p, n_chunks, key_shift()};
    }
};

struct HostBatch {
    size_t first, last;
    bool has_head;
};

// Send thread of search.rs:1531-1572.
inline std::vector<HostBatch> make_batches(size_t n_chunks, uint32_t cps) {
    std::vector<HostBatch> out;
    size_t bfirst = 0, blen = 0;
    bool head = false;
    for (size_t k = 0; k < n_chunks; ++k) {
        if (blen == 0) bfirst = k;
        ++blen;
        if (blen == cps) {
            out.push_back({bfirst, k, head});
            bfirst = k;
            blen = 1;
            head = true;
        }
    }
    if (blen && !(head && blen == 1)) out.push_back({bfirst, bfirst + blen - 1, head});
    return out;
}

// Packs plain-old-data tables into one upload buffer.
struct TablePack {
    std::vector<unsigned char> buf;
    template <class T>
    size_t add(const std::vector<T> &v) {
        size_t o = (buf.size() + 255) & ~size_t(255);
        buf.resize(o + std::max<size_t>(v.size(), 1) * sizeof(T));
        if (!v.empty()) std::memcpy(buf.data() + o, v.data(), v.size() * sizeof(T));
        return o;
    }
};

inline uint32_t code2(uint8_t b4) {  // single base one-hot -> 2-bit code A0 C1 G2 T3
    switch (b4) {
        case 4: return 0;
        case 2: return 1;
        case 8: return 2;
        default: return 3;
    }
}

// Row text through shared memory: a warp formats its 32 consecutive rows
// (one per lane) into `stage`, whose bytes line up with the output modulo 4,
// then stores the warp's contiguous output range with aligned, coalesced
// 4-byte stores (single bytes at the two ragged ends).  Without the stage
// every byte store of a warp would touch 32 scattered lines.  A range longer
// than `cap` bytes (very long record names) is written directly.
// `row(i, dst)` formats row i at dst; `off` holds each row's output offset
// (n + 1 entries).
template <class RowFn>
__device__ __forceinline__ void warp_rows_staged(uint32_t i0, uint32_t n,
                                                 const uint64_t *__restrict__ off,
                                                 char *__restrict__ text, char *stage,
                                                 uint32_t cap, RowFn row) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t i = i0 + lane;
    const uint64_t start = off[i0], end = off[min(i0 + 32, n)];
    // stage byte k <-> output byte start - mis + k, so that 4-byte-aligned
    // stage words land on 4-byte-aligned output addresses (text itself may
    // start anywhere)
    const uintptr_t tb = reinterpret_cast<uintptr_t>(text);
    const uint32_t mis = (uint32_t)((tb + start) & 3u);
    if (end - start + mis > cap) {
        if (i < n) row(i, text + off[i]);
        return;
    }
    if (i < n) row(i, stage + (off[i] - start + mis));
    __syncwarp();
    const uint64_t a0 = start + ((4u - mis) & 3u);           // first aligned output byte
    const uint64_t a1 = end - (uint64_t)((tb + end) & 3u);  // end of the last aligned word
    auto sb = [&](uint64_t g) { return stage[g - start + mis]; };
    if (a0 >= a1) {  // no whole aligned word: bytes only
        for (uint64_t g = start + lane; g < end; g += 32) text[g] = sb(g);
    } else {
        if (start + lane < a0) text[start + lane] = sb(start + lane);
        if (a1 + lane < end) text[a1 + lane] = sb(a1 + lane);
        const uint32_t *sw = reinterpret_cast<const uint32_t *>(stage + (a0 - start + mis));
        uint32_t *gw = reinterpret_cast<uint32_t *>(text + a0);
        for (uint64_t w = lane; w < (a1 - a0) / 4; w += 32) gw[w] = sw[w];
    }
    __syncwarp();
}

}  // namespace cof
