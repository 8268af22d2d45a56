// engine.cu -- device side of the B200 off-target search (sm_100a).
//
// Data layout in HBM (resident per genome):
//   bit4   : the reference's tight-packed chunk stream (two nucleotides per
//            byte, one-hot T=1 C=2 A=4 G=8, N=0xF, IUPAC = union, 0 = pad),
//            i.e. the concatenation of every search batch buffer
//            (search.rs:1376-1427).  Used for exact verification, Myers/DP
//            and site strings.
//   planes : three bit planes per 32-nucleotide word, bit k = nucleotide
//            32w+k: H and L (2-bit code A=00 C=01 G=10 T=11) and S (set when
//            the nibble is not a single base: pad, N or IUPAC).  12 bytes per
//            32 nt (0.375 B/nt).  Used by the PAM prefilter and the scan.
//   chunk metadata (byte offset, record start/end, record name index) and
//   the record names.
//
// Popcount path pipeline (db == rb == 0), one launch per stage:
//   scan   : PAM prefilter on 32 window starts per lane from the planes,
//            warp-ballot compaction of PAM-passing starts into a per-warp
//            shared-memory queue, then every queued window x every pattern of
//            the group: popc(((H^pH)|(L^pL)|S) & care) <= max_mm.  This is a
//            superset of the reference's rows (see verify).
//   verify : per candidate, the reference's exact decision: kernel popcount
//            count with N masked to 0 (search.rs:378-463, :512-531), batch
//            ownership and record-end drops (search.rs:540-546, :1428-1488),
//            writer PAM filter and mismatch recount (main.rs:159-197).
//   format : site strings with lowercase mismatches and the 8-column row text
//            (main.rs:198-242), laid out by an exclusive scan of row lengths.
#include <unistd.h>

#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "cof_engine.h"
#include "engine_dev.cuh"
#include "textout.h"

namespace cof {

// ---------------------------------------------------------------------------
// error plumbing
// ---------------------------------------------------------------------------

// ---------------------------------------------------------------------------
// device structures
// ---------------------------------------------------------------------------

// PAM cell of a scan group: window cell index and allowed 2-bit codes as
// full-word masks (all ones if the code is allowed).
struct PamCell {
    uint32_t cell, fa, fc, fg, ft;
};

constexpr int kMaxPamCells = 32;
constexpr int kMaxCareClasses = 8;

// Patterns of a group that compare the same window cells (single-base cells
// of the pattern) from the same place in the window: windows are masked
// once per class.  Pattern indices are relative to the group; `off` is where
// the patterns' first cell sits in the 32-cell window (32 - L for groups
// anchored at the PAM's end, 0 for groups anchored at the window start).
struct CareClass {
    uint32_t care, pat_begin, pat_end, off;
};

// One strand of every request whose filter has the same non-N cells at the
// same place relative to its anchor (the PAM: e.g. every NRG request, of any
// guide length): the windows whose non-N filter cells all hold a single base
// of the filter's set are scanned against the patterns [pat_begin, pat_end).
struct ScanGroup {
    uint32_t n_pam;
    uint32_t pat_begin, pat_end;
    uint32_t seg_begin, seg_end;  // scan segments of this group
    uint32_t n_class;
    uint32_t pad[2];
    PamCell pam[kMaxPamCells];
    CareClass cls[kMaxCareClasses];
};

// A contiguous range of window starts inside one batch.  Window starts are
// global nucleotide indices + 32 (the planes begin with one padding word),
// so that windows anchored at a PAM near position 0 can start before it.
struct ScanSeg {
    uint64_t lo, hi;        // range [lo, hi) of shifted window starts
    uint64_t base;          // batch base + 32: window start - base = start in the batch
    uint64_t w0;            // first plane word (lo / 32)
    uint64_t tile_begin;    // prefix count of 1024-start tiles
    uint32_t batch;
    uint32_t pad;
};

// Scan-form pattern (window cells in bit positions 0..L-1), code bits
// already masked by the pattern's care cells.
struct FastPattern {
    uint32_t h, l, care;
    int32_t k;  // max mismatches
};

// Exact-form pattern for verify / format.
struct ExactPattern {
    uint32_t request, strand, L, max_mm;
    uint8_t b4[kMaxPatternLen];  // bit4 cells in scan orientation
};

struct RequestDev {
    uint32_t L, max_mm, pam_len, first_pattern;
    uint8_t fset[2][kMaxPatternLen];  // filter bit4 per strand, scan orientation
    uint8_t fisn[2][kMaxPatternLen];  // filter char is N/n
};

// ---------------------------------------------------------------------------
// pack: bit4 stream -> H / L / S planes (one thread per 32 nt word)
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint32_t gather_nibble_bit0(uint32_t v) {
    // bits 0,4,...,28 -> bits 0..7
    v &= 0x11111111u;
    v = (v | (v >> 3)) & 0x03030303u;
    v = (v | (v >> 6)) & 0x000F000Fu;
    v = (v | (v >> 12)) & 0xFFu;
    return v;
}

__global__ void pack_planes_kernel(const uint4 *__restrict__ bit4, uint64_t n_words,
                                   uint32_t *__restrict__ H, uint32_t *__restrict__ L,
                                   uint32_t *__restrict__ S) {
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < n_words;
         w += (uint64_t)gridDim.x * blockDim.x) {
        uint4 q = bit4[w];
        uint32_t x[4] = {q.x, q.y, q.z, q.w};
        uint32_t h = 0, l = 0, s = 0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            uint32_t v = x[j];
            uint32_t hb = (v >> 3) | v;                     // G or T
            uint32_t lb = (v >> 1) | v;                     // C or T
            uint32_t pc = v - ((v >> 1) & 0x55555555u);     // per-nibble popcount
            pc = (pc & 0x33333333u) + ((pc >> 2) & 0x33333333u);
            uint32_t t = pc ^ 0x11111111u;                  // zero nibble iff single base
            uint32_t sb = t | (t >> 1) | (t >> 2);
            h |= gather_nibble_bit0(hb) << (8 * j);
            l |= gather_nibble_bit0(lb) << (8 * j);
            s |= gather_nibble_bit0(sb) << (8 * j);
        }
        H[w] = h;
        L[w] = l;
        S[w] = s;
    }
}

// ---------------------------------------------------------------------------
// scan: PAM prefilter + warp-queue compaction + popcount compare
// ---------------------------------------------------------------------------

// Tile shape of the scan (chosen per request shape by the autotuner):
//   CPT   queued windows per lane in a flush (the queue flushes at 32 x CPT)
//   WARPS warps per CTA
//   MINB  CTAs per SM the register allocation is bounded for
constexpr int kSmemPatterns = 2048;    // patterns staged in shared memory
constexpr int kMaxSegs = 64;


// The two strand groups of one filter (or one group alone) scanned by one
// work item: their windows come from the same plane words, so each tile's
// words are loaded and its place resolved once for both.  g[1] = ~0u for a
// group scanned alone.
struct ScanPair {
    uint32_t g[2];
    uint32_t seg_begin, seg_end;  // PairSeg range
};

// One batch of a pair: each group's range of shifted window starts, and the
// tiles of their union.
struct PairSeg {
    uint64_t lo[2], hi[2];
    uint64_t base;        // batch base + 32 (the same for both groups)
    uint64_t w0;          // first plane word of the union
    uint64_t tile_begin;  // prefix count of 1024-start tiles within the pair
    uint32_t batch, pad;
};

struct ScanParams {
    const uint32_t *H, *L, *S;
    const ScanGroup *groups;
    const ScanSeg *segs;
    const FastPattern *pats;
    const uint64_t *item_begin;  // per group (pair): first work item; [n] = total
    uint32_t n_groups;
    uint32_t span_tiles;         // 1024-start tiles per work item
    uint32_t n_pats;             // patterns of all groups (the table at pats)
    Hit *hits;
    uint32_t hit_cap;
    Counters *ctr;
    const ScanPair *pairs;       // scan_pair_kernel: work items over pairs
    const PairSeg *psegs;
    uint32_t n_pairs;
};

// Compares the first n <= 32 x CPT queued windows with every pattern of the
// group, CPT windows per lane.  Per care class the windows are masked once;
// per pattern the lane keeps the minimum mismatch count over its windows and
// only a pattern whose minimum passes takes the (rare) emitting branch.
// One pattern from shared memory (ld.shared.v4: the caller knows the
// table is staged there; a generic load would have to resolve the window).
__device__ __forceinline__ FastPattern lds_pattern(uint32_t saddr) {
    FastPattern f;
    uint32_t k;
    asm("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];"
        : "=r"(f.h), "=r"(f.l), "=r"(f.care), "=r"(k)
        : "r"(saddr));
    f.k = (int32_t)k;
    return f;
}

// Compares the queued windows (32 * kCpt at most, kCpt per lane) with every
// pattern of the group and appends the hits.  kSmem: the pattern table is in
// shared memory (all but the largest groups).  kPair selects how a lane
// reduces its kCpt mismatch counts per pattern: 1 one minimum chain, 4
// three-input minima (__vimin3_s32).
template <int kCpt, int kPair, bool kSmem>
__device__ __forceinline__ void flush_body(const uint4 *q, int n, const FastPattern *pt,
                                           const ScanGroup &G, uint32_t batch,
                                           const ScanParams &P, int lane) {
    const uint32_t pt_s = kSmem ? (uint32_t)__cvta_generic_to_shared(pt) : 0u;
    auto load = [&](uint32_t p) -> FastPattern {
        return kSmem ? lds_pattern(pt_s + p * (uint32_t)sizeof(FastPattern)) : pt[p];
    };
    for (uint32_t c = 0; c < G.n_class; ++c) {
        const CareClass K = G.cls[c];
        uint32_t mh[kCpt], ml[kCpt], ms[kCpt];
#pragma unroll
        for (int j = 0; j < kCpt; ++j) {
            const int idx = lane + 32 * j;
            const uint4 e = idx < n ? q[idx] : make_uint4(0, 0, 0, 0xFFFFFFFFu);
            mh[j] = e.y & K.care;
            ml[j] = e.z & K.care;
            ms[j] = e.w & K.care;
        }
        auto emit = [&](uint32_t p, const FastPattern &fp) {
#pragma unroll
            for (int j = 0; j < kCpt; ++j) {
                const int idx = lane + 32 * j;
                if (idx < n && (int)__popc((mh[j] ^ fp.h) | (ml[j] ^ fp.l) | ms[j]) <= fp.k) {
                    const uint32_t i = atomicAdd(&P.ctr->hits, 1u);
                    if (i < P.hit_cap) P.hits[i] = Hit{q[idx].x + K.off, G.pat_begin + p, batch, 0};
                    else P.ctr->overflow = 1;
                }
            }
        };
        uint32_t p = K.pat_begin;
        if (kPair == 4) {  // minimum of three per instruction, depth log3(kCpt)
            for (; p < K.pat_end; ++p) {
                const FastPattern f0 = load(p);
                int c[kCpt];
#pragma unroll
                for (int j = 0; j < kCpt; ++j)
                    c[j] = (int)__popc((mh[j] ^ f0.h) | (ml[j] ^ f0.l) | ms[j]);
#pragma unroll
                for (int w = 1; w < kCpt; w *= 3)
#pragma unroll
                    for (int j = 0; j < kCpt; j += 3 * w)
                        c[j] = j + 2 * w < kCpt ? __vimin3_s32(c[j], c[j + w], c[j + 2 * w])
                               : j + w < kCpt   ? min(c[j], c[j + w])
                                                : c[j];
                if (c[0] <= f0.k) emit(p, f0);
            }
        }
        for (; p < K.pat_end; ++p) {
            const FastPattern f0 = load(p);
            int m0 = 64;
#pragma unroll
            for (int j = 0; j < kCpt; ++j)
                m0 = min(m0, (int)__popc((mh[j] ^ f0.h) | (ml[j] ^ f0.l) | ms[j]));
            if (m0 <= f0.k) emit(p, f0);
        }
    }
}

// One call target for both table locations keeps the caller's register
// use around the (rare) call as low as with a single variant.
template <int kCpt, int kPair>
__device__ __noinline__ void flush_queue(const uint4 *q, int n, const FastPattern *pt,
                                            bool smem, const ScanGroup &G, uint32_t batch,
                                            const ScanParams &P, int lane) {
    if (smem) flush_body<kCpt, kPair, true>(q, n, pt, G, batch, P, lane);
    else flush_body<kCpt, kPair, false>(q, n, pt, G, batch, P, lane);
}

template <int kCpt, int kPair>
__device__ __forceinline__ void flush(const uint4 *q, int n, const FastPattern *pt,
                                      const FastPattern *spat, const ScanGroup &G,
                                      uint32_t batch, const ScanParams &P, int lane) {
    flush_queue<kCpt, kPair>(q, n, pt, pt == spat, G, batch, P, lane);
}

// One 1024-start tile of a scan segment for one warp: PAM prefilter of the
// lane's 32 starts, then the passing starts are drained into the warp's
// queue, which is compared with the group's patterns whenever it fills (or
// the batch changes: hits carry their batch).
template <int kCpt, int kPair>
__device__ __forceinline__ void scan_tile(const ScanParams &P, const ScanGroup &G,
                                          const ScanSeg &sgm, uint64_t tile, uint4 *q, int &qn,
                                          uint32_t &qbatch, const FastPattern *pt, bool smem,
                                          uint32_t npat, unsigned long long &ncand,
                                          unsigned long long &npairs, int lane) {
    constexpr int kQCap = 32 * kCpt;
    const uint32_t lt_mask = (1u << lane) - 1u;
    if (sgm.batch != qbatch) {
        if (qn) {
            __syncwarp();
            flush_queue<kCpt, kPair>(q, qn, pt, smem, G, qbatch, P, lane);
            __syncwarp();
            qn = 0;
        }
        qbatch = sgm.batch;
    }
    const uint64_t w = sgm.w0 + (tile - sgm.tile_begin) * 32 + lane;
    const uint32_t h0 = __ldg(P.H + w), h1 = __ldg(P.H + w + 1);
    const uint32_t l0 = __ldg(P.L + w), l1 = __ldg(P.L + w + 1);
    const uint32_t s0 = __ldg(P.S + w), s1 = __ldg(P.S + w + 1);
    // window starts 32w + k in [lo, hi)
    const uint64_t p0 = w * 32;
    uint32_t m = 0xFFFFFFFFu;
    if (p0 < sgm.lo) m = (sgm.lo - p0 >= 32) ? 0u : (m << (uint32_t)(sgm.lo - p0));
    if (p0 + 32 > sgm.hi) m = (sgm.hi <= p0) ? 0u : (m & (0xFFFFFFFFu >> (uint32_t)(32 - (sgm.hi - p0))));
    for (uint32_t c = 0; c < G.n_pam && m; ++c) {
        const PamCell pc = G.pam[c];
        const uint32_t h = __funnelshift_r(h0, h1, pc.cell);
        const uint32_t l = __funnelshift_r(l0, l1, pc.cell);
        const uint32_t s = __funnelshift_r(s0, s1, pc.cell);
        const uint32_t t0 = (l & pc.fc) | (~l & pc.fa);
        const uint32_t t1 = (l & pc.ft) | (~l & pc.fg);
        m &= ((h & t1) | (~h & t0)) & ~s;
    }
    const uint32_t nm = __popc(m);
    ncand += nm;
    npairs += (unsigned long long)nm * npat;
    // drain PAM-passing starts into the warp queue, one per lane per step
    while (__any_sync(0xFFFFFFFFu, m)) {
        const bool has = m != 0;
        const uint32_t bal = __ballot_sync(0xFFFFFFFFu, has);
        if (has) {
            const uint32_t k = __ffs(m) - 1;
            m &= m - 1;
            const int slot = qn + __popc(bal & lt_mask);
            q[slot] = make_uint4((uint32_t)(p0 + k - sgm.base), __funnelshift_r(h0, h1, k),
                                 __funnelshift_r(l0, l1, k), __funnelshift_r(s0, s1, k));
        }
        qn += __popc(bal);
        if (qn >= kQCap) {
            // full pass over kQCap windows; the (< 32) windows beyond it
            // move to the front of the queue
            __syncwarp();
            flush_queue<kCpt, kPair>(q, kQCap, pt, smem, G, qbatch, P, lane);
            const int rest = qn - kQCap;
            uint4 e = make_uint4(0, 0, 0, 0);
            if (lane < rest) e = q[kQCap + lane];
            __syncwarp();
            if (lane < rest) q[lane] = e;
            __syncwarp();
            qn = rest;
        }
    }
}

// scan_tile with the segment's fields held in registers and one ballot per
// drain step: fewer instructions per tile, which pays with few patterns per
// group (2-6 %), while with hundreds of patterns the longer live ranges
// around the flush call cost a few percent; the autotuner picks per shape.
template <int kCpt, int kPair>
__device__ __forceinline__ void scan_tile_lean(const ScanParams &P, const ScanGroup &G,
                                          const ScanSeg &sgm, uint64_t tile, uint4 *q, int &qn,
                                          uint32_t &qbatch, const FastPattern *pt, bool smem,
                                          uint32_t npat, unsigned long long &ncand,
                                          unsigned long long &npairs, int lane) {
    constexpr int kQCap = 32 * kCpt;
    const uint32_t lt_mask = (1u << lane) - 1u;
    // the segment's fields once, in registers: the queue stores below go
    // through a generic pointer and would otherwise force reloads
    const uint64_t seg_lo = sgm.lo, seg_hi = sgm.hi, seg_w0 = sgm.w0, seg_t0 = sgm.tile_begin;
    const uint64_t seg_base = sgm.base;
    const uint32_t seg_batch = sgm.batch;
    if (seg_batch != qbatch) {
        if (qn) {
            __syncwarp();
            flush_queue<kCpt, kPair>(q, qn, pt, smem, G, qbatch, P, lane);
            __syncwarp();
            qn = 0;
        }
        qbatch = seg_batch;
    }
    const uint64_t w = seg_w0 + (tile - seg_t0) * 32 + lane;
    const uint32_t h0 = __ldg(P.H + w), h1 = __ldg(P.H + w + 1);
    const uint32_t l0 = __ldg(P.L + w), l1 = __ldg(P.L + w + 1);
    const uint32_t s0 = __ldg(P.S + w), s1 = __ldg(P.S + w + 1);
    // window starts 32w + k in [lo, hi)
    const uint64_t p0 = w * 32;
    uint32_t m = 0xFFFFFFFFu;
    if (p0 < seg_lo) m = (seg_lo - p0 >= 32) ? 0u : (m << (uint32_t)(seg_lo - p0));
    if (p0 + 32 > seg_hi) m = (seg_hi <= p0) ? 0u : (m & (0xFFFFFFFFu >> (uint32_t)(32 - (seg_hi - p0))));
    for (uint32_t c = 0; c < G.n_pam && m; ++c) {
        const PamCell pc = G.pam[c];
        const uint32_t h = __funnelshift_r(h0, h1, pc.cell);
        const uint32_t l = __funnelshift_r(l0, l1, pc.cell);
        const uint32_t s = __funnelshift_r(s0, s1, pc.cell);
        const uint32_t t0 = (l & pc.fc) | (~l & pc.fa);
        const uint32_t t1 = (l & pc.ft) | (~l & pc.fg);
        m &= ((h & t1) | (~h & t0)) & ~s;
    }
    const uint32_t nm = __popc(m);
    ncand += nm;
    npairs += (unsigned long long)nm * npat;
    // drain PAM-passing starts into the warp queue, one per lane per step
    const uint32_t off0 = (uint32_t)(p0 - seg_base);  // batch-local start of bit 0
    for (;;) {
        const bool has = m != 0;
        const uint32_t bal = __ballot_sync(0xFFFFFFFFu, has);
        if (!bal) break;
        if (has) {
            const uint32_t k = __ffs(m) - 1;
            m &= m - 1;
            const int slot = qn + __popc(bal & lt_mask);
            q[slot] = make_uint4(off0 + k, __funnelshift_r(h0, h1, k), __funnelshift_r(l0, l1, k),
                                 __funnelshift_r(s0, s1, k));
        }
        qn += __popc(bal);
        if (qn >= kQCap) {
            // full pass over kQCap windows; the (< 32) windows beyond it
            // move to the front of the queue
            __syncwarp();
            flush_queue<kCpt, kPair>(q, kQCap, pt, smem, G, qbatch, P, lane);
            const int rest = qn - kQCap;
            uint4 e = make_uint4(0, 0, 0, 0);
            if (lane < rest) e = q[kQCap + lane];
            __syncwarp();
            if (lane < rest) q[lane] = e;
            __syncwarp();
            qn = rest;
        }
    }
}

// Persistent scan: CTAs pull work items -- a span of kSpanTiles tiles of one
// scan group -- from a global counter, so groups of very different sizes
// (few or many patterns, sparse or dense PAMs) share the GPU evenly.  A CTA
// stages a group's patterns in shared memory when it switches groups; each
// warp takes every kScanWarps-th tile of the span.
template <int kCpt, int kScanWarps, int kMinBlocks, int kPair>
__global__ void __launch_bounds__(kScanWarps * 32, kMinBlocks)
scan_kernel(ScanParams P) {
    constexpr int kQCap = 32 * kCpt;     // flush threshold per warp queue
    constexpr int kQSlots = kQCap + 32;  // one drain step adds at most 32
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint4 *queues = reinterpret_cast<uint4 *>(smem_raw);
    FastPattern *spat = reinterpret_cast<FastPattern *>(queues + kScanWarps * kQSlots);
    __shared__ ScanGroup sg;
    __shared__ ScanSeg ssegs[kMaxSegs];
    __shared__ unsigned long long s_item;
    __shared__ uint32_t s_group;

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint4 *q = queues + warp * kQSlots;
    int qn = 0;
    uint32_t qbatch = 0xFFFFFFFFu;
    unsigned long long ncand = 0, npairs = 0;
    uint32_t cur_g = 0xFFFFFFFFu, nseg = 0, npat = 0;
    uint64_t g_tiles = 0;
    const FastPattern *pt = spat;
    const uint64_t total_items = P.item_begin[P.n_groups];

    while (true) {
        if (threadIdx.x == 0) {
            const unsigned long long it = atomicAdd(&P.ctr->next_item, 1ull);
            uint32_t lo = 0, hi = P.n_groups;
            if (it < total_items) {
                while (hi - lo > 1) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (P.item_begin[mid] <= it) lo = mid; else hi = mid;
                }
            }
            s_item = it;
            s_group = lo;
        }
        __syncthreads();
        const uint64_t item = s_item;
        const uint32_t g = s_group;
        if (item >= total_items) break;
        if (g != cur_g) {
            if (qn) {  // the queue belongs to the previous group's patterns
                __syncwarp();
                flush<kCpt, kPair>(q, qn, pt, spat, sg, qbatch, P, lane);
                __syncwarp();
                qn = 0;
            }
            __syncthreads();
            if (threadIdx.x == 0) sg = P.groups[g];
            __syncthreads();
            nseg = sg.seg_end - sg.seg_begin;
            for (uint32_t i = threadIdx.x; i < nseg; i += blockDim.x) ssegs[i] = P.segs[sg.seg_begin + i];
            npat = sg.pat_end - sg.pat_begin;
            pt = P.pats + sg.pat_begin;
            if (npat <= (uint32_t)kSmemPatterns) {
                for (uint32_t i = threadIdx.x; i < npat; i += blockDim.x) spat[i] = pt[i];
                pt = spat;
            }
            __syncthreads();
            g_tiles = ssegs[nseg - 1].tile_begin +
                      ((ssegs[nseg - 1].hi - ssegs[nseg - 1].w0 * 32 + 1023) >> 10);
            cur_g = g;
            qbatch = 0xFFFFFFFFu;
        }
        const uint64_t t_begin = (item - P.item_begin[g]) * P.span_tiles;
        const uint64_t t_end = min(t_begin + P.span_tiles, g_tiles);
        uint32_t sidx = 0;
        for (uint64_t tile = t_begin + warp; tile < t_end; tile += kScanWarps) {
            while (sidx + 1 < nseg && tile >= ssegs[sidx + 1].tile_begin) ++sidx;
            scan_tile<kCpt, kPair>(P, sg, ssegs[sidx], tile, q, qn, qbatch, pt, pt == spat, npat,
                                   ncand, npairs, lane);
        }
        __syncthreads();  // s_item / s_group are rewritten by the next fetch
    }
    if (qn) {
        __syncwarp();
        flush<kCpt, kPair>(q, qn, pt, spat, sg, qbatch, P, lane);
    }
    // candidate and pair counts (the roofline's algorithmic work)
    for (int o = 16; o; o >>= 1) {
        ncand += __shfl_down_sync(0xFFFFFFFFu, ncand, o);
        npairs += __shfl_down_sync(0xFFFFFFFFu, npairs, o);
    }
    if (lane == 0 && ncand) {
        atomicAdd(&P.ctr->candidates, ncand);
        atomicAdd(&P.ctr->pairs, npairs);
    }
}

// Persistent scan with per-warp work items: each warp pulls its own span of
// kSpanTiles tiles from the global counter, so a warp never waits at a CTA
// barrier while another warp of its CTA compares a full queue.  The pattern
// table of all groups is staged in shared memory once, up to kSmemPatterns
// patterns; a group whose patterns lie beyond that prefix reads them from
// global memory.  Group and segment descriptors are read through L1.
template <int kCpt, int kScanWarps, int kMinBlocks, int kPair, int kPatCap, int kLean>
__global__ void __launch_bounds__(kScanWarps * 32, kMinBlocks)
scan_warp_kernel(ScanParams P) {
    constexpr int kQSlots = 32 * kCpt + 32;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint4 *queues = reinterpret_cast<uint4 *>(smem_raw);
    FastPattern *spat = reinterpret_cast<FastPattern *>(queues + kScanWarps * kQSlots);
    const uint32_t n_staged = min(P.n_pats, (uint32_t)kPatCap);
    for (uint32_t i = threadIdx.x; i < n_staged; i += blockDim.x) spat[i] = P.pats[i];
    __syncthreads();

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint4 *q = queues + warp * kQSlots;
    int qn = 0;
    uint32_t qbatch = 0xFFFFFFFFu;
    unsigned long long ncand = 0, npairs = 0;
    uint32_t cur_g = 0xFFFFFFFFu, nseg = 0, npat = 0;
    uint64_t g_tiles = 0;
    const ScanGroup *G = P.groups;
    const ScanSeg *segs = P.segs;
    const FastPattern *pt = spat;
    bool smem = true;
    const uint64_t total_items = P.item_begin[P.n_groups];

    while (true) {
        unsigned long long it = 0;
        if (lane == 0) it = atomicAdd(&P.ctr->next_item, 1ull);
        it = __shfl_sync(0xFFFFFFFFu, it, 0);
        if (it >= total_items) break;
        uint32_t lo = 0, hi = P.n_groups;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (__ldg(P.item_begin + mid) <= it) lo = mid; else hi = mid;
        }
        if (lo != cur_g) {
            if (qn) {  // the queue belongs to the previous group's patterns
                __syncwarp();
                flush_queue<kCpt, kPair>(q, qn, pt, smem, *G, qbatch, P, lane);
                __syncwarp();
                qn = 0;
            }
            cur_g = lo;
            G = P.groups + lo;
            segs = P.segs + G->seg_begin;
            nseg = G->seg_end - G->seg_begin;
            npat = G->pat_end - G->pat_begin;
            smem = G->pat_end <= n_staged;
            pt = (smem ? spat : P.pats) + G->pat_begin;
            const ScanSeg &last = segs[nseg - 1];
            g_tiles = last.tile_begin + ((last.hi - last.w0 * 32 + 1023) >> 10);
            qbatch = 0xFFFFFFFFu;
        }
        const uint64_t t_begin = (it - P.item_begin[lo]) * P.span_tiles;
        const uint64_t t_end = min(t_begin + P.span_tiles, g_tiles);
        uint32_t sidx = 0;
        for (uint64_t tile = t_begin; tile < t_end; ++tile) {
            while (sidx + 1 < nseg && tile >= segs[sidx + 1].tile_begin) ++sidx;
            if (kLean)
                scan_tile_lean<kCpt, kPair>(P, *G, segs[sidx], tile, q, qn, qbatch, pt, smem, npat,
                                            ncand, npairs, lane);
            else
                scan_tile<kCpt, kPair>(P, *G, segs[sidx], tile, q, qn, qbatch, pt, smem, npat,
                                       ncand, npairs, lane);
        }
    }
    if (qn) {
        __syncwarp();
        flush_queue<kCpt, kPair>(q, qn, pt, smem, *G, qbatch, P, lane);
    }
    for (int o = 16; o; o >>= 1) {
        ncand += __shfl_down_sync(0xFFFFFFFFu, ncand, o);
        npairs += __shfl_down_sync(0xFFFFFFFFu, npairs, o);
    }
    if (lane == 0 && ncand) {
        atomicAdd(&P.ctr->candidates, ncand);
        atomicAdd(&P.ctr->pairs, npairs);
    }
}

// ---------------------------------------------------------------------------
// direct scan of strand pairs (few patterns per group)
// ---------------------------------------------------------------------------

// The patterns of one group (at most kNP), in registers: scan form, the
// window cell of each pattern's first cell (its care class offset) and its
// index in the pattern table.  Unused slots never match (k = -1).
template <int kNP>
struct RegPats {
    uint32_t h[kNP], l[kNP], care[kNP], off[kNP], idx[kNP];
    int32_t k[kNP];
};

template <int kNP>
__device__ __forceinline__ void load_reg_pats(const ScanGroup *G, const FastPattern *pats,
                                              RegPats<kNP> &R) {
    const uint32_t n = G ? G->pat_end - G->pat_begin : 0;
#pragma unroll
    for (int j = 0; j < kNP; ++j) {
        R.h[j] = R.l[j] = R.care[j] = R.off[j] = R.idx[j] = 0;
        R.k[j] = -1;
        if ((uint32_t)j < n) {
            const uint32_t p = G->pat_begin + j;
            const FastPattern f = pats[p];
            R.h[j] = f.h;
            R.l[j] = f.l;
            R.care[j] = f.care;
            R.k[j] = f.k;
            R.idx[j] = p;
            for (uint32_t c = 0; c < G->n_class; ++c)
                if ((uint32_t)j >= G->cls[c].pat_begin && (uint32_t)j < G->cls[c].pat_end)
                    R.off[j] = G->cls[c].off;
        }
    }
}

// Every PAM-passing start of a lane's word (mask m) against the group's
// patterns, straight from the lane's plane words: no queue, no loads.  The
// warp steps together (a vote per step), one start per lane per step: left
// to diverge, lanes with different start counts ran their loops apart, with
// about 6 of 32 lanes active per instruction.
template <int kNP>
__device__ __forceinline__ void compare_direct(uint32_t m, const RegPats<kNP> &R, uint32_t h0,
                                               uint32_t h1, uint32_t l0, uint32_t l1,
                                               uint32_t s0, uint32_t s1, uint32_t off0,
                                               uint32_t batch, const ScanParams &P) {
    while (__any_sync(0xFFFFFFFFu, m)) {
        if (!m) continue;
        const uint32_t k = __ffs(m) - 1;
        m &= m - 1;
        const uint32_t wh = __funnelshift_r(h0, h1, k), wl = __funnelshift_r(l0, l1, k),
                       ws = __funnelshift_r(s0, s1, k);
#pragma unroll
        for (int j = 0; j < kNP; ++j) {
            if ((int)__popc(((wh ^ R.h[j]) | (wl ^ R.l[j]) | ws) & R.care[j]) <= R.k[j]) {
                const uint32_t i = atomicAdd(&P.ctr->hits, 1u);
                if (i < P.hit_cap) P.hits[i] = Hit{off0 + k + R.off[j], R.idx[j], batch, 0};
                else P.ctr->overflow = 1;
            }
        }
    }
}

// Persistent scan over strand pairs with per-warp work items (a span of
// tiles of one pair), for groups of at most kNP patterns.  Per 1024-start
// tile a lane loads its plane words once, runs both groups' PAM prefilters
// on them, and compares each PAM-passing start with the group's patterns in
// registers.  With few patterns the queue of scan_warp_kernel costs more
// than the comparisons it batches: a queued window is stored, reloaded and
// masked per care class, while here it costs three funnel shifts.
constexpr uint32_t kDirectPamCells = 8;  // PAM cells per group a direct scan stages

// The PAM prefilter of a group whose cells a warp staged in shared memory
// (code masks fa fc fg ft, and window cells).
__device__ __forceinline__ uint32_t pam_mask_staged(const uint4 *cm, const uint32_t *ci,
                                                    uint32_t n, uint32_t m, uint32_t h0,
                                                    uint32_t h1, uint32_t l0, uint32_t l1,
                                                    uint32_t s0, uint32_t s1) {
    for (uint32_t c = 0; c < n; ++c) {
        const uint4 f = cm[c];  // fa, fc, fg, ft
        const uint32_t cell = ci[c];
        const uint32_t h = __funnelshift_r(h0, h1, cell);
        const uint32_t l = __funnelshift_r(l0, l1, cell);
        const uint32_t sv = __funnelshift_r(s0, s1, cell);
        const uint32_t t0 = (l & f.y) | (~l & f.x);
        const uint32_t t1 = (l & f.w) | (~l & f.z);
        m &= ((h & t1) | (~h & t0)) & ~sv;
    }
    return m;
}

// Starts 0..31 of a lane whose first start is p (relative to its segment's
// first plane word) that lie in [lo, hi).
__device__ __forceinline__ uint32_t range_mask32(uint32_t p, uint32_t lo, uint32_t hi) {
    uint32_t m = 0xFFFFFFFFu;
    if (p < lo) m = (lo - p >= 32) ? 0u : (m << (lo - p));
    if (p + 32 > hi) m = (hi <= p) ? 0u : (m & (0xFFFFFFFFu >> (32 - (hi - p))));
    return m;
}

template <int kNP, int kScanWarps, int kMinBlocks>
__global__ void __launch_bounds__(kScanWarps * 32, kMinBlocks)
scan_direct_kernel(ScanParams P) {
    __shared__ uint4 s_cm[kScanWarps][2][kDirectPamCells];
    __shared__ uint32_t s_ci[kScanWarps][2][kDirectPamCells];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long ncand = 0, npairs = 0;
    uint32_t cur = 0xFFFFFFFFu, nseg = 0, npat0 = 0, npat1 = 0, npam0 = 0, npam1 = 0;
    uint64_t p_tiles = 0;
    bool two = false;
    const PairSeg *segs = P.psegs;
    RegPats<kNP> R0, R1;
    const uint64_t total_items = P.item_begin[P.n_pairs];

    while (true) {
        unsigned long long it = 0;
        if (lane == 0) it = atomicAdd(&P.ctr->next_item, 1ull);
        it = __shfl_sync(0xFFFFFFFFu, it, 0);
        if (it >= total_items) break;
        uint32_t lo = 0, hi = P.n_pairs;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (__ldg(P.item_begin + mid) <= it) lo = mid; else hi = mid;
        }
        if (lo != cur) {
            cur = lo;
            const ScanPair pr = P.pairs[lo];
            const ScanGroup *G0 = P.groups + pr.g[0];
            const ScanGroup *G1 = pr.g[1] == 0xFFFFFFFFu ? nullptr : P.groups + pr.g[1];
            two = G1 != nullptr;
            npat0 = G0->pat_end - G0->pat_begin;
            npat1 = two ? G1->pat_end - G1->pat_begin : 0;
            npam0 = G0->n_pam;
            npam1 = two ? G1->n_pam : 0;
            load_reg_pats<kNP>(G0, P.pats, R0);
            load_reg_pats<kNP>(G1, P.pats, R1);
            __syncwarp();
            if ((uint32_t)lane < npam0) {
                const PamCell c = G0->pam[lane];
                s_cm[warp][0][lane] = make_uint4(c.fa, c.fc, c.fg, c.ft);
                s_ci[warp][0][lane] = c.cell;
            }
            if ((uint32_t)lane < npam1) {
                const PamCell c = G1->pam[lane];
                s_cm[warp][1][lane] = make_uint4(c.fa, c.fc, c.fg, c.ft);
                s_ci[warp][1][lane] = c.cell;
            }
            __syncwarp();
            segs = P.psegs + pr.seg_begin;
            nseg = pr.seg_end - pr.seg_begin;
            const PairSeg &last = segs[nseg - 1];
            const uint64_t hi_u = max(last.hi[0], last.hi[1]);
            p_tiles = last.tile_begin + ((hi_u - last.w0 * 32 + 1023) >> 10);
        }
        const uint64_t t_begin = (it - P.item_begin[lo]) * P.span_tiles;
        const uint64_t t_end = min(t_begin + P.span_tiles, p_tiles);
        // the current segment, as offsets from its first plane word's
        // first start (32-bit: a segment spans one batch)
        uint32_t sidx = 0;
        while (sidx + 1 < nseg && t_begin >= segs[sidx + 1].tile_begin) ++sidx;
        uint64_t seg_w0 = 0, seg_t0 = 0, next_t = 0;
        uint32_t lo0 = 0, hi0 = 0, lo1 = 0, hi1 = 0, offb = 0, batch = 0;
        bool fresh = true;
        uint32_t c_cand = 0, c_pairs = 0;
        for (uint64_t tile = t_begin; tile < t_end; ++tile) {
            if (fresh || tile >= next_t) {
                if (!fresh) ++sidx;
                fresh = false;
                const PairSeg &sg = segs[sidx];
                seg_w0 = sg.w0;
                seg_t0 = sg.tile_begin;
                next_t = sidx + 1 < nseg ? segs[sidx + 1].tile_begin : ~0ull;
                const uint64_t p0s = sg.w0 * 32;
                lo0 = (uint32_t)(sg.lo[0] - p0s);
                hi0 = (uint32_t)(sg.hi[0] - p0s);
                lo1 = two ? (uint32_t)(sg.lo[1] - p0s) : 0u;
                hi1 = two ? (uint32_t)(sg.hi[1] - p0s) : 0u;
                offb = (uint32_t)(p0s - sg.base);
                batch = sg.batch;
            }
            const uint32_t trel = (uint32_t)(tile - seg_t0);
            const uint64_t w = seg_w0 + (uint64_t)trel * 32 + lane;
            const uint32_t h0 = __ldg(P.H + w), h1 = __ldg(P.H + w + 1);
            const uint32_t l0 = __ldg(P.L + w), l1 = __ldg(P.L + w + 1);
            const uint32_t s0 = __ldg(P.S + w), s1 = __ldg(P.S + w + 1);
            const uint32_t t0 = trel * 1024u;  // the tile's first start
            const uint32_t pl = t0 + (uint32_t)lane * 32u;
            // a tile inside both ranges (nearly all) skips the range masks
            const uint32_t r0 = t0 >= lo0 && t0 + 1024u <= hi0 ? 0xFFFFFFFFu : range_mask32(pl, lo0, hi0);
            const uint32_t m0 = pam_mask_staged(s_cm[warp][0], s_ci[warp][0], npam0, r0, h0, h1,
                                                l0, l1, s0, s1);
            uint32_t m1 = 0;
            if (two) {
                const uint32_t r1 = t0 >= lo1 && t0 + 1024u <= hi1 ? 0xFFFFFFFFu : range_mask32(pl, lo1, hi1);
                m1 = pam_mask_staged(s_cm[warp][1], s_ci[warp][1], npam1, r1, h0, h1, l0, l1, s0,
                                     s1);
            }
            const uint32_t n0 = __popc(m0), n1 = __popc(m1);
            c_cand += n0 + n1;
            c_pairs += n0 * npat0 + n1 * npat1;
            // batch-local start of bit 0 (a window may begin before its
            // batch; the class offset brings every hit's start back into it)
            const uint32_t off0 = offb + pl;
            compare_direct<kNP>(m0, R0, h0, h1, l0, l1, s0, s1, off0, batch, P);
            compare_direct<kNP>(m1, R1, h0, h1, l0, l1, s0, s1, off0, batch, P);
        }
        ncand += c_cand;
        npairs += c_pairs;
    }
    for (int o = 16; o; o >>= 1) {
        ncand += __shfl_down_sync(0xFFFFFFFFu, ncand, o);
        npairs += __shfl_down_sync(0xFFFFFFFFu, npairs, o);
    }
    if (lane == 0 && ncand) {
        atomicAdd(&P.ctr->candidates, ncand);
        atomicAdd(&P.ctr->pairs, npairs);
    }
}

struct ScanVariant {
    int cpt, warps, min_blocks, pair;
    uint32_t span_tiles;
    void (*kernel)(ScanParams);
    bool per_warp;
    uint32_t pat_cap;  // patterns staged in shared memory
    bool lean;         // scan_tile_lean
    bool paired;       // scan_direct_kernel: work items over strand pairs
    uint32_t max_pats; // patterns per group the kernel holds (0: any)
    size_t smem() const {
        if (paired) return 0;
        return (size_t)warps * (32 * cpt + 32) * sizeof(uint4) + pat_cap * sizeof(FastPattern);
    }
};

template <int C, int W, int B, int Q = 1>
constexpr ScanVariant variant(uint32_t span) {
    return ScanVariant{C, W, B, Q, span, scan_kernel<C, W, B, Q>, false, kSmemPatterns, false,
                       false, 0};
}
// NP: patterns per group held in registers
template <int NP, int W, int B>
constexpr ScanVariant direct_variant(uint32_t span) {
    return ScanVariant{0, W, B, 0, span, scan_direct_kernel<NP, W, B>, true, 0, false, true,
                       (uint32_t)NP};
}
// span: tiles per warp work item; K: patterns staged in shared memory;
// N: scan_tile_lean (1) or scan_tile (0)
template <int C, int W, int B, int Q = 1, int K = kSmemPatterns, int N = 0>
constexpr ScanVariant warp_variant(uint32_t span) {
    return ScanVariant{C, W, B, Q, span, scan_warp_kernel<C, W, B, Q, K, N>, true, (uint32_t)K,
                       N != 0, false, 0};
}

// Candidate tile shapes (windows per lane x warps x min blocks per SM, and
// how a lane reduces its mismatch counts); the autotuner times them on a
// sample of the genome.  Four CTAs per SM leave 64 registers per thread.
const ScanVariant kScanVariants[] = {
    // per-warp work items: four CTAs per SM (1024 staged patterns), then three
    warp_variant<8, 8, 4, 4, 1024, 1>(8), warp_variant<8, 8, 4, 1, 1024>(8),
    warp_variant<4, 8, 4, 4, 1024>(8), warp_variant<8, 8, 3, 4>(8), warp_variant<8, 8, 3>(8),
    // CTA work items
    variant<8, 8, 3>(64), variant<4, 8, 4>(64), variant<4, 16, 2>(128),
    // the default shape without the lean tile (more patterns per group)
    warp_variant<8, 8, 4, 4, 1024>(8),
    // strand pairs compared directly, the default for up to 2 patterns per
    // group.  Scan at 3.1 Gbp: 1 guide 1.60 ms at six CTAs per SM (1.66 at
    // five, 1.86 at four) against 2.80 ms for the lean tile; 2 guides 2.25
    // (2.31, 2.45) against 2.92.  With 4 patterns in registers 3.23 against
    // 3.17 ms, so none is compiled.
    direct_variant<1, 8, 6>(8), direct_variant<2, 8, 6>(8),
    direct_variant<1, 8, 5>(8), direct_variant<2, 8, 5>(8),
};
constexpr int kFirstPairVariant = 9;      // the first usable one from here is the default
constexpr uint32_t kPairMaxPatterns = 2;  // patterns per group up to which they are the default
constexpr int kNumScanVariants = sizeof(kScanVariants) / sizeof(kScanVariants[0]);
static_assert(kNumScanVariants <= 16, "Engine::scan_occ_ holds 16 shapes");

// ---------------------------------------------------------------------------
// verify: the reference's exact decision per candidate hit
// ---------------------------------------------------------------------------

__global__ void verify_kernel(GenomeDev G, const BatchDev *__restrict__ batches,
                              const ExactPattern *__restrict__ pats,
                              const uint32_t *__restrict__ fast2exact,
                              const RequestDev *__restrict__ reqs, const Hit *__restrict__ hits,
                              const Counters *__restrict__ scan_ctr, uint32_t hit_cap,
                              uint32_t sg_bits, uint32_t e_bits, uint64_t range_lo,
                              uint64_t range_hi, Row *__restrict__ rows,
                              uint64_t *__restrict__ keys, uint32_t *__restrict__ vals,
                              Counters *ctr, uint32_t *__restrict__ req_rows) {
    // row sort key: request, then genome position, then the pattern's index
    // within its request (sg < 2^sg_bits, index < 2^e_bits)
    // the block steps through the hits together, so every lane of a warp
    // reaches the row emission below; rows get their slots and requests
    // their counts with one atomic per warp (per request), not per row
    const uint32_t lane = threadIdx.x & 31, lt_mask = (1u << lane) - 1u;
    // the scan's hit count (read on the device: no host round trip between
    // the two kernels); an overflowed list is verified up to its capacity
    // and the whole pass is rerun
    const uint32_t n_hits = min(*(volatile const uint32_t *)&scan_ctr->hits, hit_cap);
    for (uint32_t base = blockIdx.x * blockDim.x; base < n_hits; base += gridDim.x * blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        bool emit = false;
        Row row{};
        uint64_t key = 0;
        uint32_t req = 0xFFFFFFFFu;
        do {
            if (i >= n_hits) break;
            const Hit h = hits[i];
            const BatchDev B = batches[h.batch];
            const uint32_t pe = fast2exact[h.pattern];
            const ExactPattern &P = pats[pe];
            const RequestDev &R = reqs[P.request];
            const uint32_t L = P.L;
            // a scan group's windows cover the starts of all its pattern
            // lengths: keep this length's own range
            // (legacy_match_start_min_nucl, search.rs:540-546, up to the
            // batch's valid cells)
            const uint32_t msmin = B.active_start > L - 1 ? B.active_start - (L - 1) : 0;
            if (h.s_local < msmin || h.s_local >= B.valid) break;
            const uint64_t sg = B.base + h.s_local;
            // a scan group's window range is the union over its lengths:
            // keep this pattern's starts inside the searched range
            if (sg < range_lo || sg >= range_hi) break;
            // search_chunk_cpu count on the N-masked batch buffer (zero past
            // the batch's valid bytes)
            uint8_t g[kMaxPatternLen];
            int matches = 0;
            for (uint32_t c = 0; c < L; ++c) {
                uint8_t v = (h.s_local + c < B.valid) ? nib(G.bit4, sg + c) : 0;
                if (v == 0xF) v = 0;
                g[c] = v;
                matches += __popc(v & P.b4[c]);
            }
            if ((int)L - matches > (int)R.max_mm) break;
            // convert_matches: owning chunk, record position, record-end drop
            const uint64_t gbyte = sg >> 1;
            uint32_t lo = B.first, hi = B.first + B.nch;  // boff[lo] <= gbyte < boff[hi]
            while (hi - lo > 1) {
                uint32_t mid = (lo + hi) >> 1;
                if (G.boff[mid] <= gbyte) lo = mid; else hi = mid;
            }
            const uint32_t k = lo;
            const uint64_t pos = G.start[k] + (sg - 2 * G.boff[k]);
            const bool end_chrom = (k == B.first + B.nch - 1) || G.start[k + 1] == 0;
            if (end_chrom && pos + L > G.end[k]) break;
            // writer: PAM filter and mismatch recount
            const uint32_t st = P.strand;
            uint32_t actual = 0;
            bool pam_ok = true;
            for (uint32_t c = 0; c < L; ++c) {
                const bool sb = single_base(g[c]);
                if (!R.fisn[st][c] && !(sb && (g[c] & R.fset[st][c]))) { pam_ok = false; break; }
                if (P.b4[c] != 0xF && !(sb && (g[c] & P.b4[c]))) ++actual;
            }
            if (!pam_ok || actual > R.max_mm) break;
            emit = true;
            row = Row{sg, B.base + B.valid, pos, k, pe, actual, 0};
            key = ((uint64_t)P.request << (sg_bits + e_bits)) | (sg << e_bits) |
                  (pe - R.first_pattern);
            req = P.request;
        } while (false);
        const uint32_t em = __ballot_sync(0xFFFFFFFFu, emit);
        if (!em) continue;
        const int leader = __ffs(em) - 1;
        uint32_t r0 = 0;
        if ((int)lane == leader) r0 = atomicAdd(&ctr->rows, (uint32_t)__popc(em));
        r0 = __shfl_sync(0xFFFFFFFFu, r0, leader);
        const uint32_t peers = __match_any_sync(0xFFFFFFFFu, req);
        if (emit) {
            const uint32_t r = r0 + __popc(em & lt_mask);
            rows[r] = row;
            keys[r] = key;
            vals[r] = r;
            if ((int)lane == __ffs(peers) - 1) atomicAdd(&req_rows[req], (uint32_t)__popc(peers));
        }
    }
}

// ---------------------------------------------------------------------------
// format: row lengths, then row text (main.rs:198-242)
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint64_t pos_out(const Row &w, const RequestDev &R, uint32_t strand) {
    uint64_t a = R.pam_len ? R.pam_len - 1 : 0;  // db == 0 on this path
    return strand ? w.pos + a : w.pos;
}

__global__ void row_len_kernel(GenomeDev G, const Row *__restrict__ rows,
                               const uint32_t *__restrict__ order, uint32_t n,
                               const ExactPattern *__restrict__ pats,
                               const RequestDev *__restrict__ reqs, uint32_t *__restrict__ len) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const Row w = rows[order[i]];
        const ExactPattern &P = pats[w.pattern];
        const RequestDev &R = reqs[P.request];
        const uint32_t ni = G.name_idx[w.chunk];
        const uint32_t name_len = G.name_off[ni + 1] - G.name_off[ni];
        // "X\t" rna "\t" dna "\t" name "\t" pos "\t" dir "\t" mm "\t0\n"
        len[i] = 2 + P.L + 1 + P.L + 1 + name_len + 1 + ndigits(pos_out(w, R, P.strand)) + 3 +
                 ndigits(w.mm) + 3;
    }
}

constexpr uint32_t kRowStage = 4096;  // staged text bytes per warp

__global__ void __launch_bounds__(256)
row_write_kernel(GenomeDev G, const Row *__restrict__ rows, const uint32_t *__restrict__ order,
                 uint32_t n, const ExactPattern *__restrict__ pats,
                 const RequestDev *__restrict__ reqs, const uint64_t *__restrict__ off,
                 char *__restrict__ text) {
    __shared__ __align__(16) char stage_all[8][kRowStage];
    char *stage = stage_all[threadIdx.x >> 5];
    const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i0 = gw * 32; i0 < n; i0 += nw * 32) {
        warp_rows_staged((uint32_t)i0, n, off, text, stage, kRowStage, [&](uint32_t i, char *o) {
            const Row w = rows[order[i]];
            const ExactPattern &P = pats[w.pattern];
            const RequestDev &R = reqs[P.request];
            const uint32_t L = P.L;
            const bool fwd = P.strand == 0;
            *o++ = 'X';
            *o++ = '\t';
            char *rna = o;
            char *dna = o + L + 1;
            for (uint32_t c = 0; c < L; ++c) {
                // output orientation: reverse strand strings are reverse complemented
                const uint32_t sc = fwd ? c : L - 1 - c;
                const uint64_t gi = w.s_global + sc;
                uint8_t g = gi < w.clip ? nib(G.bit4, gi) : 0;
                if (g == 0xF) g = 0;
                uint8_t p = P.b4[sc];
                if (!fwd) { g = dcomp4(g); p = dcomp4(p); }
                rna[c] = b4char(p);
                char d = b4char(g);
                if (g == 0) d = (p == 0xF) ? 'N' : 'n';
                else if (p == 0xF) {}
                else if (!(single_base(g) && (g & p))) d = (char)(d | 0x20);
                dna[c] = d;
            }
            o += L;
            *o++ = '\t';
            o += L;
            *o++ = '\t';
            const uint32_t ni = G.name_idx[w.chunk];
            for (uint32_t c = G.name_off[ni]; c < G.name_off[ni + 1]; ++c) *o++ = G.names[c];
            *o++ = '\t';
            o = put_u64(o, pos_out(w, R, P.strand));
            *o++ = '\t';
            *o++ = fwd ? '+' : '-';
            *o++ = '\t';
            o = put_u64(o, w.mm);
            *o++ = '\t';
            *o++ = '0';
            *o++ = '\n';

        });
    }
}

// Match records of formatted rows, in text order (row i of the sorted
// order): the fields of search()'s Match (chrom_chunk.rs:19-29) and the
// offset of the row's line in its piece, which holds the rows of one request
// from row req_first[request] on.
__global__ void row_rec_kernel(GenomeDev G, const Row *__restrict__ rows,
                               const uint32_t *__restrict__ order, uint32_t n,
                               const ExactPattern *__restrict__ pats,
                               const RequestDev *__restrict__ reqs,
                               const uint64_t *__restrict__ off,
                               const uint32_t *__restrict__ req_first, MatchRec *__restrict__ recs) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const Row w = rows[order[i]];
        const ExactPattern &P = pats[w.pattern];
        const RequestDev &R = reqs[P.request];
        MatchRec m{};
        m.chrom_idx = w.pos;
        m.text_offset = off[i] - off[req_first[P.request]];
        m.record = G.name_idx[w.chunk];
        m.pattern_idx = w.pattern - R.first_pattern;
        m.mismatches = (uint8_t)w.mm;
        m.is_forward = P.strand == 0;
        recs[i] = m;
    }
}

// ---------------------------------------------------------------------------
// device genome + scratch
// ---------------------------------------------------------------------------

namespace {
void *warm_context(void *arg) {
    const int device = (int)(intptr_t)arg;
    if (cudaSetDevice(device) == cudaSuccess) cudaFree(nullptr);
    return nullptr;
}
}  // namespace

Engine::Engine(int device) : device_(device) {
    // context creation costs a few hundred ms on a large GPU; it overlaps
    // the file read that precedes every upload
    warm_pid_ = (int)::getpid();
    warm_live_ = pthread_create(&warm_, nullptr, warm_context, (void *)(intptr_t)device) == 0;
}

void Engine::join_warm() {
    if (warm_live_ && (int)::getpid() == warm_pid_) pthread_join(warm_, nullptr);
    warm_live_ = false;
}

Engine::~Engine() {
    join_warm();
    if (dev_) {
        cudaSetDevice(device_);
        delete dev_;
    }
}

int Engine::upload(Error &err) {
    if (dev_) return kOk;
    join_warm();
    CU(cudaSetDevice(device_));
    std::unique_ptr<DeviceGenome> d(new DeviceGenome());
    d->device = device_;
    CU(cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking));
    CU(cudaStreamCreateWithFlags(&d->copy_stream, cudaStreamNonBlocking));
    for (auto &e : d->ev) CU(cudaEventCreate(&e));
    CU(cudaEventCreate(&d->fmt_done));
    CU(cudaEventCreate(&d->copy_done));
    CU(cudaDeviceGetAttribute(&d->n_sm, cudaDevAttrMultiProcessorCount, device_));
    const HostGenome &h = host_;
    const uint64_t n_bytes = h.n_bytes();
    const uint64_t n_nucl = 2 * n_bytes;
    // 64 pad words (all non-single) so that a scan tile's last lanes and the
    // funnel-shift neighbour word stay inside the planes
    d->n_words = (n_nucl + 31) / 32 + 64;
    if (d->bit4.ensure(d->n_words * 16 + 64, err)) return err.code;
    CU(cudaMemsetAsync(d->bit4.p, 0, d->n_words * 16 + 64, d->stream));
    if (h.deferred) {  // a .2bit file: the packed bases are decoded here
        if (upload_2bit(*h.deferred, d->bit4.p, device_, d->stream, err)) return err.code;
    } else if (h.deferred_fa) {  // a FASTA file: its lines are converted here
        if (upload_fasta(*h.deferred_fa, d->bit4.p, d->n_words * 16 + 64, device_, d->stream, err))
            return err.code;
    } else if (n_bytes) {
        CU(cudaMemcpyAsync(d->bit4.p, h.data.data(), n_bytes, cudaMemcpyHostToDevice, d->stream));
    }
    // each plane starts with one padding word (32 non-single cells before
    // position 0) for windows anchored at a PAM near the genome start
    const uint64_t pw = d->n_words + 1;
    if (d->planes.ensure(3 * pw, err)) return err.code;
    CU(cudaMemsetAsync(d->planes.p, 0, 4, d->stream));
    CU(cudaMemsetAsync(d->planes.p + pw, 0, 4, d->stream));
    CU(cudaMemsetAsync(d->planes.p + 2 * pw, 0xFF, 4, d->stream));
    {
        int threads = 256;
        uint64_t blocks = std::min<uint64_t>((d->n_words + threads - 1) / threads, 65535ull * 16);
        pack_planes_kernel<<<(unsigned)std::max<uint64_t>(blocks, 1), threads, 0, d->stream>>>(
            reinterpret_cast<const uint4 *>(d->bit4.p), d->n_words, d->planes.p + 1,
            d->planes.p + pw + 1, d->planes.p + 2 * pw + 1);
        CU(cudaGetLastError());
    }
    const size_t nc = h.n_chunks();
    d->n_chunks = nc;
    if (d->boff.ensure(nc + 1, err) || d->start.ensure(nc + 1, err) ||
        d->end.ensure(nc + 1, err) || d->name_idx.ensure(nc + 1, err))
        return err.code;
    std::vector<uint64_t> st(h.start), en(h.end);
    st.push_back(0);  // sentinel: a record start after the last chunk
    en.push_back(0);
    std::vector<uint32_t> ni(h.name_idx);
    ni.push_back(0);
    CU(cudaMemcpyAsync(d->boff.p, h.boff.data(), (nc + 1) * 8, cudaMemcpyHostToDevice, d->stream));
    CU(cudaMemcpyAsync(d->start.p, st.data(), (nc + 1) * 8, cudaMemcpyHostToDevice, d->stream));
    CU(cudaMemcpyAsync(d->end.p, en.data(), (nc + 1) * 8, cudaMemcpyHostToDevice, d->stream));
    CU(cudaMemcpyAsync(d->name_idx.p, ni.data(), (nc + 1) * 4, cudaMemcpyHostToDevice, d->stream));
    std::vector<uint32_t> noff{0};
    std::string all;
    for (const auto &s : h.names) {
        all += s;
        noff.push_back((uint32_t)all.size());
    }
    if (d->names.ensure(all.size() + 1, err) || d->name_off.ensure(noff.size(), err)) return err.code;
    if (!all.empty())
        CU(cudaMemcpyAsync(d->names.p, all.data(), all.size(), cudaMemcpyHostToDevice, d->stream));
    CU(cudaMemcpyAsync(d->name_off.p, noff.data(), noff.size() * 4, cudaMemcpyHostToDevice, d->stream));
    CU(cudaStreamSynchronize(d->stream));
    dev_ = d.release();
    return kOk;
}

// ---------------------------------------------------------------------------
// host orchestration
// ---------------------------------------------------------------------------

int Engine::free_device_bytes(uint64_t *free_bytes, Error &err) {
    CU(cudaSetDevice(device_));
    size_t f = 0, total = 0;
    CU(cudaMemGetInfo(&f, &total));
    *free_bytes = f;
    return kOk;
}

int Engine::search(const std::vector<Request> &reqs, std::vector<Result> &out, Error &err,
                   const Sink *sink, const SearchRange *range) {
    times_ = StageTimes();
    const SearchRange whole;
    const SearchRange &rg = range ? *range : whole;
    out.clear();
    out.resize(reqs.size());
    if (reqs.empty()) return kOk;
    for (const Request &r : reqs) {
        if (r.cps != reqs[0].cps) {
            err = {kBadInput, "batched requests must share chunks_per_search"};
            return err.code;
        }
    }
    if (upload(err)) return err.code;
    CU(cudaSetDevice(device_));
    DeviceGenome &d = *dev_;
    CU(cudaEventRecord(d.ev[8], d.stream));
    // search.rs:1513: any bulge selects the Myers path for that request
    std::vector<size_t> pi, bi;
    std::vector<Request> pr, br;
    for (size_t i = 0; i < reqs.size(); ++i) {
        if (reqs[i].raw && !reqs[i].max_db && !reqs[i].max_rb) {
            // search()'s raw stream: every window, no PAM prefilter
            if (run_raw(reqs[i], out[i], err, rg)) return err.code;
            if (out[i].text) out[i].text = out[i].owned.data();
            if (sink) {  // one piece, without match records
                Piece pc;
                pc.request = i;
                pc.text = out[i].text ? out[i].text : "";
                pc.text_len = out[i].text_len;
                pc.n_rows = out[i].n_rows;
                if (sink->fn(pc)) {
                    err = {kCancelled, "the result sink stopped the search"};
                    return err.code;
                }
                out[i].owned.clear();
                out[i].owned.shrink_to_fit();
                out[i].text = nullptr;
                out[i].text_len = 0;
            }
            continue;
        }
        if (reqs[i].max_db || reqs[i].max_rb) {
            bi.push_back(i);
            br.push_back(reqs[i]);
        } else {
            pi.push_back(i);
            pr.push_back(reqs[i]);
        }
    }
    // a path sees its own requests; the sink hears the caller's indices
    auto sub_sink = [&](const std::vector<size_t> &idx, Sink &sub) -> const Sink * {
        if (!sink) return nullptr;
        sub.records = sink->records;
        sub.fn = [sink, &idx](const Piece &p) {
            Piece q = p;
            q.request = idx[p.request];
            return sink->fn(q);
        };
        return &sub;
    };
    if (!pr.empty()) {
        std::vector<Result> po;
        Sink sub;
        if (run_popcount(pr, po, err, sub_sink(pi, sub), rg)) return err.code;
        for (size_t k = 0; k < pi.size(); ++k) out[pi[k]] = std::move(po[k]);
    }
    if (!br.empty()) {
        std::vector<Result> bo;
        Sink sub;
        if (run_bulge(br, bo, err, sub_sink(bi, sub), rg)) return err.code;
        for (size_t k = 0; k < bi.size(); ++k) out[bi[k]] = std::move(bo[k]);
    }
    CU(cudaEventRecord(d.ev[9], d.stream));
    CU(cudaEventSynchronize(d.ev[9]));
    float ms = 0;
    cudaEventElapsedTime(&ms, d.ev[8], d.ev[9]);
    times_.total_ms = ms;
    for (auto &r : out) r.device_ms = ms;
    return kOk;
}

int Engine::run_popcount(const std::vector<Request> &reqs, std::vector<Result> &out, Error &err,
                         const Sink *sink, const SearchRange &range) {
    out.clear();
    out.resize(reqs.size());
    DeviceGenome &d = *dev_;
    const HostGenome &h = host_;
    const Bit4Tables &t = bit4();

    // batches
    const auto hb = make_batches(h.n_chunks(), reqs[0].cps);
    std::vector<BatchDev> batches;
    for (const HostBatch &b : hb) {
        BatchDev x{};
        x.base = 2 * h.boff[b.first];
        x.valid = (uint32_t)(2 * (h.boff[b.last + 1] - h.boff[b.first]));
        x.first = (uint32_t)b.first;
        x.nch = (uint32_t)(b.last - b.first + 1);
        const uint64_t c1 = b.has_head ? 2 * (h.boff[b.first + 1] - h.boff[b.first]) : 0;
        x.active_start = (uint32_t)c1;
        batches.push_back(x);
    }

    // requests -> groups, patterns, segments
    std::vector<RequestDev> rdev;
    std::vector<FastPattern> fpats;
    std::vector<ExactPattern> epats;
    std::vector<ScanGroup> groups;
    std::vector<ScanSeg> segs;
    std::vector<uint32_t> req_first_pat;
    // Exact patterns are laid out request-major (the row sort key).  Scan
    // groups gather, per strand, the patterns of every request whose filter
    // has the same non-N cells at the same place relative to its anchor --
    // the window end when the PAM ends the pattern (3' PAMs), else the
    // window start -- so that one PAM sweep serves requests of different
    // guide lengths and mismatch limits.
    std::vector<uint32_t> fast2exact;
    // per scan group: shifted window start - pattern start, when all of its
    // patterns have one length (always so within one request); else ~0u
    std::vector<uint32_t> group_shift;
    std::map<std::string, std::vector<uint32_t>> by_key;
    std::vector<std::string> key_order;
    std::vector<uint32_t> ep_off;  // window offset of each exact pattern's first cell
    for (size_t ri = 0; ri < reqs.size(); ++ri) {
        const Request &r = reqs[ri];
        const uint32_t L = (uint32_t)r.filter.size();
        RequestDev rd{};
        rd.L = L;
        rd.max_mm = r.max_mm;
        rd.pam_len = (uint32_t)r.pam_len;
        rd.first_pattern = (uint32_t)epats.size();
        for (uint32_t c = 0; c < L; ++c) {
            const char f = r.filter[c];
            rd.fset[0][c] = t.str2b4[1][(uint8_t)f];
            rd.fisn[0][c] = (f == 'N' || f == 'n');
            const char fr = r.filter[L - 1 - c];
            rd.fset[1][c] = comp4(t.str2b4[1][(uint8_t)fr]);
            rd.fisn[1][c] = (fr == 'N' || fr == 'n');
        }
        rdev.push_back(rd);
        req_first_pat.push_back((uint32_t)epats.size());
        std::string key[2];
        uint32_t off[2];
        for (uint32_t st = 0; st < 2; ++st) {
            int first = -1, last = -1;
            for (uint32_t c = 0; c < L; ++c) {
                if (rd.fisn[st][c]) continue;
                if (first < 0) first = (int)c;
                last = (int)c;
            }
            const bool end_anchor = last == (int)L - 1 && first > 0;
            // window cell of pattern cell 0: the 32-cell window ends at the
            // pattern end (END anchor) or starts at its start; a pattern
            // longer than the window has cells outside it (negative offset,
            // kept as a wrapped uint32) that only verify compares
            off[st] = end_anchor ? kScanWindow - L : 0;
            key[st] = std::string(end_anchor ? "E" : "S") + (st ? "-" : "+");
            for (uint32_t c = 0; c < L; ++c)
                if (!rd.fisn[st][c])
                    key[st] += std::to_string((int)c + (int)off[st]) + ":" +
                               std::to_string(rd.fset[st][c]) + ",";
        }
        const size_t np = r.patterns.size(), nfwd = np / 2;
        for (size_t p = 0; p < np; ++p) {
            const uint32_t strand = p >= nfwd;
            ExactPattern ep{};
            ep.request = (uint32_t)ri;
            ep.strand = strand;
            ep.L = L;
            ep.max_mm = r.max_mm;
            for (uint32_t c = 0; c < L; ++c) ep.b4[c] = t.str2b4[1][(uint8_t)r.patterns[p][c]];
            if (!by_key.count(key[strand])) key_order.push_back(key[strand]);
            by_key[key[strand]].push_back((uint32_t)epats.size());
            epats.push_back(ep);
            ep_off.push_back(off[strand]);
        }
    }
    // row sort key (verify_kernel): request | genome position | pattern
    // index within the request, each field as wide as this pass needs
    auto width = [](uint64_t v) {  // bits of v's binary form
        uint32_t b = 0;
        while (b < 64 && (v >> b) != 0) ++b;
        return b;
    };
    size_t max_np = 1;
    for (const Request &r : reqs) max_np = std::max(max_np, r.patterns.size());
    const uint32_t sg_bits = width(2 * h.boff.back()), e_bits = width(max_np - 1),
                   key_bits = width(reqs.size() - 1) + sg_bits + e_bits;
    if (key_bits > 64) {
        err = {kUnsupported, "too many requests x patterns in one pass for the row sort key"};
        return err.code;
    }
    for (const auto &key : key_order) {
        const std::vector<uint32_t> &members = by_key[key];
        const ExactPattern &e0 = epats[members[0]];
        const uint32_t strand = e0.strand;
        const RequestDev &rd = rdev[e0.request];
        const uint32_t off0 = ep_off[members[0]];
        ScanGroup proto{};
        for (uint32_t c = 0; c < rd.L; ++c) {  // the same cells for every member
            if (rd.fisn[strand][c]) continue;
            if (proto.n_pam == kMaxPamCells) break;
            const int wc = (int)c + (int)off0;  // window cell
            if (wc < 0 || wc >= (int)kScanWindow) continue;  // verify tests it
            const uint8_t fs = rd.fset[strand][c];
            PamCell pc{(uint32_t)wc, (fs & 4) ? ~0u : 0u, (fs & 2) ? ~0u : 0u, (fs & 8) ? ~0u : 0u,
                       (fs & 1) ? ~0u : 0u};
            proto.pam[proto.n_pam++] = pc;
        }
        // the members' pattern lengths (with their window offsets)
        std::vector<std::pair<uint32_t, uint32_t>> lens;
        for (uint32_t e : members) lens.push_back({epats[e].L, ep_off[e]});
        std::sort(lens.begin(), lens.end());
        lens.erase(std::unique(lens.begin(), lens.end()), lens.end());
        const uint32_t key_shift = lens.size() == 1 ? kScanWindow - lens[0].second : ~0u;
        // scan segments: one per batch, the union of the members' window
        // ranges; verify re-applies each length's own head-overlap threshold
        std::vector<ScanSeg> kseg;
        uint64_t tiles = 0;
        for (size_t bi = 0; bi < batches.size(); ++bi) {
            const BatchDev &b = batches[bi];
            // legacy_match_start_min_nucl (search.rs:540-546): starts in the
            // head chunk that the previous batch already emitted
            const uint64_t c1 = hb[bi].has_head ? b.active_start : 0;
            uint64_t lo = ~0ull, hi = 0;
            for (const auto &lo_ : lens) {
                const uint32_t L = lo_.first, o = lo_.second;
                const uint64_t msmin = c1 > L - 1 ? c1 - (L - 1) : 0;
                // this length's pattern starts in the batch and the range
                const uint64_t s_lo = std::max(b.base + msmin, range.lo);
                const uint64_t s_hi = std::min<uint64_t>(b.base + b.valid, range.hi);
                if (s_hi <= s_lo) continue;
                // shifted window start of pattern start s: s + kScanWindow - o
                // (a 32-bit difference: L for an END anchor of any length)
                const uint32_t shift = kScanWindow - o;
                lo = std::min<uint64_t>(lo, s_lo + shift);
                hi = std::max<uint64_t>(hi, s_hi + shift);
            }
            if (hi <= lo) continue;
            ScanSeg sgm{};
            sgm.lo = lo;
            sgm.hi = hi;
            sgm.base = b.base + kScanWindow;
            sgm.w0 = sgm.lo / 32;
            sgm.tile_begin = tiles;
            sgm.batch = (uint32_t)bi;
            tiles += (sgm.hi - sgm.w0 * 32 + 1023) / 1024;
            kseg.push_back(sgm);
        }
        if (kseg.empty()) continue;
        // scan form of the members (window cells from their offset), ordered
        // by care mask and offset
        struct Comp {
            FastPattern fp;
            uint32_t off, exact;
        };
        std::vector<Comp> comp;
        for (uint32_t e : members) {
            const ExactPattern &ep = epats[e];
            const uint32_t o = ep_off[e];
            FastPattern fp{0, 0, 0, (int32_t)ep.max_mm};
            for (uint32_t c = 0; c < ep.L; ++c) {
                const uint8_t v = ep.b4[c];
                const int wc = (int)c + (int)o;  // window cell; outside: verify only
                if (wc >= 0 && wc < (int)kScanWindow && v && !(v & (v - 1))) {
                    const uint32_t cd = code2(v);
                    fp.care |= 1u << wc;
                    fp.h |= ((cd >> 1) & 1u) << wc;
                    fp.l |= (cd & 1u) << wc;
                }
            }
            comp.push_back({fp, o, e});
        }
        std::stable_sort(comp.begin(), comp.end(), [](const Comp &x, const Comp &y) {
            return x.fp.care != y.fp.care ? x.fp.care < y.fp.care : x.off < y.off;
        });
        // a scan group stages at most kMaxSegs batch segments in shared
        // memory: longer batch lists (small chunks_per_search on a large
        // genome) split into groups with the same patterns, tiles counted
        // from each group's first segment
        for (size_t s0 = 0; s0 < kseg.size(); s0 += kMaxSegs) {
            const size_t s1 = std::min(kseg.size(), s0 + (size_t)kMaxSegs);
            proto.seg_begin = (uint32_t)segs.size();
            for (size_t k = s0; k < s1; ++k) {
                ScanSeg sgm = kseg[k];
                sgm.tile_begin -= kseg[s0].tile_begin;
                segs.push_back(sgm);
            }
            proto.seg_end = (uint32_t)segs.size();
            // groups of at most kMaxCareClasses classes
            ScanGroup g = proto;
            g.pat_begin = (uint32_t)fpats.size();
            g.n_class = 0;
            for (size_t i = 0; i < comp.size(); ++i) {
                const uint32_t care = comp[i].fp.care, o = comp[i].off;
                const bool new_class = g.n_class == 0 || g.cls[g.n_class - 1].care != care ||
                                       g.cls[g.n_class - 1].off != o;
                if (new_class && g.n_class == (uint32_t)kMaxCareClasses) {
                    g.pat_end = (uint32_t)fpats.size();
                    groups.push_back(g);
                    group_shift.push_back(key_shift);
                    g = proto;
                    g.pat_begin = (uint32_t)fpats.size();
                    g.n_class = 0;
                }
                const uint32_t rel = (uint32_t)fpats.size() - g.pat_begin;
                if (g.n_class == 0 || g.cls[g.n_class - 1].care != care || g.cls[g.n_class - 1].off != o)
                    g.cls[g.n_class++] = CareClass{care, rel, rel, o};
                g.cls[g.n_class - 1].pat_end = rel + 1;
                fpats.push_back(comp[i].fp);
                fast2exact.push_back(comp[i].exact);
            }
            g.pat_end = (uint32_t)fpats.size();
            groups.push_back(g);
            group_shift.push_back(key_shift);
        }
    }

    TablePack tp;
    // work items: spans of span_tiles tiles per group (a table per span in
    // use).  The autotuner's sample is the first tune_tiles tiles of every
    // group, sized so that the sample alone fills every SM.
    uint64_t full_tiles = 0;
    for (const ScanGroup &g : groups) {
        const ScanSeg &last = segs[g.seg_end - 1];
        full_tiles += last.tile_begin + (last.hi - last.w0 * 32 + 1023) / 1024;
    }
    // ~16 work items of 64 tiles per resident CTA, so that the sample runs in
    // steady state rather than in its tail
    const uint64_t tune_tiles =
        std::max<uint64_t>(256, (uint64_t)16 * 64 * 3 * d.n_sm / std::max<size_t>(groups.size(), 1));
    auto make_items = [&](uint32_t span, uint64_t cap_tiles) {
        std::vector<uint64_t> ib{0};
        for (const ScanGroup &g : groups) {
            const ScanSeg &last = segs[g.seg_end - 1];
            const uint64_t tiles = std::min<uint64_t>(
                last.tile_begin + (last.hi - last.w0 * 32 + 1023) / 1024, cap_tiles);
            ib.push_back(ib.back() + (tiles + span - 1) / span);
        }
        return ib;
    };
    std::map<uint32_t, size_t> o_items, o_sample;
    std::map<uint32_t, uint64_t> n_items, n_sample;
    const size_t o_batch = tp.add(batches), o_rdev = tp.add(rdev), o_fp = tp.add(fpats),
                 o_ep = tp.add(epats), o_grp = tp.add(groups), o_seg = tp.add(segs),
                 o_f2e = tp.add(fast2exact);
    for (const ScanVariant &v : kScanVariants) {
        if (v.paired || o_items.count(v.span_tiles)) continue;
        auto full = make_items(v.span_tiles, ~0ull);
        auto samp = make_items(v.span_tiles, tune_tiles);
        n_items[v.span_tiles] = full.back();
        n_sample[v.span_tiles] = samp.back();
        o_items[v.span_tiles] = tp.add(full);
        o_sample[v.span_tiles] = tp.add(samp);
    }

    // Strand pairs for scan_direct_kernel: a group and the next one whose
    // segments cover the same batches (the two strands of a filter) become
    // one work unit over the union of their window ranges; a group without
    // such a partner is scanned alone.
    const bool pairs_ok = !groups.empty();
    auto make_pairs = [&](const std::vector<ScanGroup> &G, const std::vector<ScanSeg> &S,
                          std::vector<ScanPair> &pairs, std::vector<PairSeg> &ps) {
        std::vector<char> used(G.size(), 0);
        for (size_t i = 0; i < G.size(); ++i) {
            if (used[i]) continue;
            used[i] = 1;
            const uint32_t ni = G[i].seg_end - G[i].seg_begin;
            size_t j = G.size();
            for (size_t k = i + 1; k < G.size() && j == G.size(); ++k) {
                if (used[k] || G[k].seg_end - G[k].seg_begin != ni) continue;
                bool same = true;
                for (uint32_t t = 0; t < ni && same; ++t) {
                    const ScanSeg &a = S[G[i].seg_begin + t], &b = S[G[k].seg_begin + t];
                    same = a.batch == b.batch && a.base == b.base;
                }
                if (same) j = k;
            }
            const bool two = j < G.size();
            if (two) used[j] = 1;
            ScanPair pr{{(uint32_t)i, two ? (uint32_t)j : 0xFFFFFFFFu}, (uint32_t)ps.size(), 0};
            uint64_t tiles = 0;
            for (uint32_t t = 0; t < ni; ++t) {
                const ScanSeg &a = S[G[i].seg_begin + t];
                PairSeg x{};
                x.lo[0] = a.lo;
                x.hi[0] = a.hi;
                uint64_t lo = a.lo, hi = a.hi;
                if (two) {
                    const ScanSeg &b = S[G[j].seg_begin + t];
                    x.lo[1] = b.lo;
                    x.hi[1] = b.hi;
                    lo = std::min(lo, b.lo);
                    hi = std::max(hi, b.hi);
                }
                x.base = a.base;
                x.w0 = lo / 32;
                x.tile_begin = tiles;
                x.batch = a.batch;
                tiles += (hi - x.w0 * 32 + 1023) / 1024;
                ps.push_back(x);
            }
            pr.seg_end = (uint32_t)ps.size();
            pairs.push_back(pr);
        }
    };
    // work-item tables of pairs: spans of `span` tiles of each pair's union
    auto pair_items = [](const std::vector<ScanPair> &pairs, const std::vector<PairSeg> &ps,
                         uint32_t span, uint64_t cap_tiles) {
        std::vector<uint64_t> ib{0};
        for (const ScanPair &pr : pairs) {
            const PairSeg &last = ps[pr.seg_end - 1];
            const uint64_t hi = std::max(last.hi[0], last.hi[1]);
            const uint64_t tiles =
                std::min<uint64_t>(last.tile_begin + (hi - last.w0 * 32 + 1023) / 1024, cap_tiles);
            ib.push_back(ib.back() + (tiles + span - 1) / span);
        }
        return ib;
    };
    std::vector<ScanPair> pairs;
    std::vector<PairSeg> psegs;
    std::map<uint32_t, size_t> o_pitems, o_psample;
    std::map<uint32_t, uint64_t> n_pitems, n_psample;
    size_t o_pairs = 0, o_psegs = 0;
    if (pairs_ok) {
        make_pairs(groups, segs, pairs, psegs);
        o_pairs = tp.add(pairs);
        o_psegs = tp.add(psegs);
        for (const ScanVariant &v : kScanVariants) {
            if (!v.paired || o_pitems.count(v.span_tiles)) continue;
            auto full = pair_items(pairs, psegs, v.span_tiles, ~0ull);
            auto samp = pair_items(pairs, psegs, v.span_tiles, tune_tiles);
            n_pitems[v.span_tiles] = full.back();
            n_psample[v.span_tiles] = samp.back();
            o_pitems[v.span_tiles] = tp.add(full);
            o_psample[v.span_tiles] = tp.add(samp);
        }
    }

    // Slices: one request on a large genome is scanned in slices of pattern
    // start positions, [cut_j, cut_j+1) of the global start coordinate.  A
    // slice's rows are verified, sorted and written while the previous
    // slice's text is still crossing to the host, so the copy runs beside
    // the scan.  Rows sort by position first, so the slices' texts follow
    // each other in the order of one unsliced pass.  A scan group's segment
    // holds shifted window starts (start + the group's shift), clipped here
    // to the slice.
    struct SliceTab {
        size_t o_grp = 0, o_seg = 0;
        uint32_t n_groups = 0;
        std::map<uint32_t, size_t> o_items;
        std::map<uint32_t, uint64_t> n_items;
        size_t o_pairs = 0, o_psegs = 0;  // strand pairs of the slice (pairs_ok)
        uint32_t n_pairs = 0;
        std::map<uint32_t, size_t> o_pitems;
        std::map<uint32_t, uint64_t> n_pitems;
    };
    std::vector<SliceTab> slices;
    {
        // 768 Mnt: 4 slices of a 3.1 Gbp genome (3, 4 and 6 slices measured
        // 18.99, 18.83 and 19.40 ms per 100-guide search; one pass 20.02)
        uint64_t slice_nt = uint64_t(768) << 20;
        const char *force = std::getenv("COF_SLICE_NT");  // tests: slice small genomes too
        if (force) slice_nt = std::max<uint64_t>(1024, std::strtoull(force, nullptr, 10));
        const uint64_t total_nt = 2 * h.boff.back();
        const bool whole = range.lo == 0 && range.hi == ~0ull;
        bool ok = whole && reqs.size() == 1 && !groups.empty() && total_nt >= 2 * slice_nt;
        if (ok && !force) {
            // slice only when the text is expected to be large enough for
            // its copy to outweigh the slices' own cost (about 0.2 ms each).
            // For i.i.d. uniform bases, rows per pattern ~ starts x P(the
            // filter cells under the pattern's N cells match) x P(<= mm of
            // the pattern's other cells mismatch); a reverse-strand pattern
            // meets the filter reversed
            const Request &r = reqs[0];
            const uint32_t L = (uint32_t)r.filter.size();
            const size_t nfwd = r.patterns.size() / 2;
            double rows = 0;
            for (size_t pi = 0; pi < r.patterns.size(); ++pi) {
                const std::string &pat = r.patterns[pi];
                double p_pam = 1;
                std::vector<double> q;  // match probability of each care cell
                for (uint32_t c = 0; c < L; ++c) {
                    const uint8_t pb = t.str2b4[1][(uint8_t)pat[c]];
                    const uint8_t fb = t.str2b4[1][(uint8_t)r.filter[pi < nfwd ? c : L - 1 - c]];
                    if (pb == 0xF) p_pam *= __builtin_popcount(fb) / 4.0;
                    else q.push_back(__builtin_popcount(pb) / 4.0);
                }
                // P(at most max_mm of the care cells mismatch), by DP
                std::vector<double> dp(r.max_mm + 2, 0.0);
                dp[0] = 1;
                for (double m : q)
                    for (int k = (int)r.max_mm + 1; k >= 0; --k)
                        dp[k] = dp[k] * m + (k ? dp[k - 1] * (1 - m) : 0);
                double p_mm = 0;
                for (uint32_t k = 0; k <= r.max_mm; ++k) p_mm += dp[k];
                rows += (double)total_nt * p_pam * p_mm;
            }
            ok = rows * (2.0 * L + 30) >= 32.0 * (1 << 20);
        }
        for (uint32_t sh : group_shift) ok = ok && sh != ~0u;
        const uint64_t n_slices = ok ? (total_nt + slice_nt - 1) / slice_nt : 0;
        for (uint64_t j = 0; j < n_slices; ++j) {
            const uint64_t c0 = total_nt * j / n_slices;
            const uint64_t c1 = j + 1 == n_slices ? ~0ull : total_nt * (j + 1) / n_slices;
            std::vector<ScanGroup> gj;
            std::vector<ScanSeg> sj;
            for (size_t gi = 0; gi < groups.size(); ++gi) {
                ScanGroup ng = groups[gi];
                const uint64_t sh = group_shift[gi];
                const uint64_t lo_cut = c0 + sh, hi_cut = c1 == ~0ull ? ~0ull : c1 + sh;
                ng.seg_begin = (uint32_t)sj.size();
                uint64_t tiles = 0;
                for (uint32_t k = groups[gi].seg_begin; k < groups[gi].seg_end; ++k) {
                    ScanSeg x = segs[k];
                    const uint64_t lo = std::max(x.lo, lo_cut), hi = std::min(x.hi, hi_cut);
                    if (hi <= lo) continue;
                    x.lo = lo;
                    x.hi = hi;
                    x.w0 = lo / 32;
                    x.tile_begin = tiles;
                    tiles += (hi - x.w0 * 32 + 1023) / 1024;
                    sj.push_back(x);
                }
                ng.seg_end = (uint32_t)sj.size();
                if (ng.seg_end > ng.seg_begin) gj.push_back(ng);
            }
            if (gj.empty()) continue;
            SliceTab st;
            st.n_groups = (uint32_t)gj.size();
            st.o_grp = tp.add(gj);
            st.o_seg = tp.add(sj);
            if (pairs_ok) {
                std::vector<ScanPair> pj;
                std::vector<PairSeg> psj;
                make_pairs(gj, sj, pj, psj);
                st.n_pairs = (uint32_t)pj.size();
                st.o_pairs = tp.add(pj);
                st.o_psegs = tp.add(psj);
                for (const ScanVariant &v : kScanVariants) {
                    if (!v.paired || st.o_pitems.count(v.span_tiles)) continue;
                    auto ib = pair_items(pj, psj, v.span_tiles, ~0ull);
                    st.n_pitems[v.span_tiles] = ib.back();
                    st.o_pitems[v.span_tiles] = tp.add(ib);
                }
            }
            for (const ScanVariant &v : kScanVariants) {
                if (v.paired || st.o_items.count(v.span_tiles)) continue;
                std::vector<uint64_t> ib{0};
                for (const ScanGroup &g : gj) {
                    const ScanSeg &last = sj[g.seg_end - 1];
                    const uint64_t t = last.tile_begin + (last.hi - last.w0 * 32 + 1023) / 1024;
                    ib.push_back(ib.back() + (t + v.span_tiles - 1) / v.span_tiles);
                }
                st.n_items[v.span_tiles] = ib.back();
                st.o_items[v.span_tiles] = tp.add(ib);
            }
            slices.push_back(std::move(st));
        }
    }
    if (d.tables.ensure(tp.buf.size(), err)) return err.code;
    cudaStream_t s = d.stream;
    CU(cudaEventRecord(d.ev[0], s));
    CU(cudaMemcpyAsync(d.tables.p, tp.buf.data(), tp.buf.size(), cudaMemcpyHostToDevice, s));
    auto tab = [&](size_t o) { return (const void *)(d.tables.p + o); };
    if (d.ctr.ensure(1, err) || d.req_rows.ensure(reqs.size(), err)) return err.code;
    if (d.hits.cap == 0 && d.hits.ensure(first_cand_cap(), err)) return err.code;

    ScanParams sp{};
    sp.H = d.planes.p;  // word w holds shifted window starts [32 w, 32 w + 32)
    sp.L = d.planes.p + (d.n_words + 1);
    sp.S = d.planes.p + 2 * (d.n_words + 1);
    sp.groups = (const ScanGroup *)tab(o_grp);
    sp.segs = (const ScanSeg *)tab(o_seg);
    sp.pats = (const FastPattern *)tab(o_fp);
    sp.n_groups = (uint32_t)groups.size();
    sp.n_pats = (uint32_t)fpats.size();
    sp.hits = d.hits.p;
    sp.ctr = d.ctr.p;
    // launches variant v over the full work list, over the tuning sample or
    // over one slice's work list
    auto launch = [&](const ScanVariant &v, bool sample, const SliceTab *sl = nullptr) -> int {
        const size_t smem = v.smem();
        // the shape's shared-memory opt-in and occupancy, once per engine
        int &occ = scan_occ_[&v - kScanVariants];
        if (occ == 0) {
            CU(cudaFuncSetAttribute(v.kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, v.kernel, v.warps * 32, smem));
            occ = std::max(occ, 1);
        }
        sp.span_tiles = v.span_tiles;
        sp.groups = (const ScanGroup *)tab(sl ? sl->o_grp : o_grp);
        sp.segs = (const ScanSeg *)tab(sl ? sl->o_seg : o_seg);
        sp.n_groups = sl ? sl->n_groups : (uint32_t)groups.size();
        uint64_t items = 0;
        if (v.paired) {
            sp.pairs = (const ScanPair *)tab(sl ? sl->o_pairs : o_pairs);
            sp.psegs = (const PairSeg *)tab(sl ? sl->o_psegs : o_psegs);
            sp.n_pairs = sl ? sl->n_pairs : (uint32_t)pairs.size();
            sp.item_begin = (const uint64_t *)tab(sl ? sl->o_pitems.at(v.span_tiles)
                                                  : sample ? o_psample[v.span_tiles]
                                                           : o_pitems[v.span_tiles]);
            items = sl ? sl->n_pitems.at(v.span_tiles)
                       : sample ? n_psample[v.span_tiles] : n_pitems[v.span_tiles];
        } else {
            sp.item_begin = (const uint64_t *)tab(sl ? sl->o_items.at(v.span_tiles)
                                                  : sample ? o_sample[v.span_tiles]
                                                           : o_items[v.span_tiles]);
            items = sl ? sl->n_items.at(v.span_tiles)
                       : sample ? n_sample[v.span_tiles] : n_items[v.span_tiles];
        }
        sp.hits = d.hits.p;  // the list may have grown (and moved) since the last launch
        sp.hit_cap = (uint32_t)std::min<size_t>(d.hits.cap, 0xFFFFFFF0u);
        const unsigned gx = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(items, (uint64_t)d.n_sm * occ));
        CU(cudaMemsetAsync(d.ctr.p, 0, sizeof(Counters), s));
        v.kernel<<<gx, v.warps * 32, smem, s>>>(sp);
        CU(cudaGetLastError());
        ++times_.kernel_launches;
        return kOk;
    };

    // the scan over one work list (the full one, or a slice's) and the
    // verify of its hits, with one host wait; rerun once with a larger
    // candidate list if the scan overflowed.  n_rows and the rows per
    // request come back.
    Counters hc{};
    // runs while a scan is on the device, just before the host waits for it
    // (a streamed search hands the previous slice's rows to its sink here)
    std::function<int()> before_wait;
    auto scan_verify = [&](const ScanVariant *v, const SliceTab *sl, uint32_t &n_rows,
                           std::vector<uint32_t> &req_rows) -> int {
        for (int attempt = 0; attempt < 2; ++attempt) {
            CU(cudaEventRecord(d.ev[1], s));
            if (v) {
                if (launch(*v, false, sl)) return err.code;
            } else {
                CU(cudaMemsetAsync(d.ctr.p, 0, sizeof(Counters), s));
            }
            CU(cudaEventRecord(d.ev[2], s));
            const size_t cap = std::max<size_t>(d.hits.cap, 1);
            if (d.rows.ensure(cap + 1, err) || d.keys.ensure(cap + 1, err) ||
                d.keys2.ensure(cap + 1, err) || d.vals.ensure(cap + 1, err) ||
                d.vals2.ensure(cap + 1, err))
                return err.code;
            CU(cudaMemsetAsync(d.req_rows.p, 0, reqs.size() * 4, s));
            if (v) {
                verify_kernel<<<d.n_sm * 8, 256, 0, s>>>(
                    d.view(), (const BatchDev *)tab(o_batch), (const ExactPattern *)tab(o_ep),
                    (const uint32_t *)tab(o_f2e), (const RequestDev *)tab(o_rdev), d.hits.p, d.ctr.p,
                    (uint32_t)std::min<size_t>(d.hits.cap, 0xFFFFFFF0u), sg_bits, e_bits, range.lo,
                    range.hi, d.rows.p, d.keys.p, d.vals.p, d.ctr.p, d.req_rows.p);
                CU(cudaGetLastError());
                ++times_.kernel_launches;
            }
            CU(cudaEventRecord(d.ev[3], s));
            CU(cudaMemcpyAsync(&hc, d.ctr.p, sizeof(Counters), cudaMemcpyDeviceToHost, s));
            req_rows.assign(reqs.size(), 0);
            CU(cudaMemcpyAsync(req_rows.data(), d.req_rows.p, reqs.size() * 4,
                               cudaMemcpyDeviceToHost, s));
            if (before_wait && before_wait()) return err.code;
            CU(cudaStreamSynchronize(s));
            if (!hc.overflow && hc.hits <= d.hits.cap) break;
            if (attempt == 1) {
                err = {kOom, "candidate buffer overflow after resize"};
                return err.code;
            }
            if (d.hits.ensure((size_t)hc.hits + hc.hits / 4 + 1024, err)) return err.code;
        }
        float ms = 0;
        cudaEventElapsedTime(&ms, d.ev[1], d.ev[2]);
        times_.scan_ms += ms;
        cudaEventElapsedTime(&ms, d.ev[2], d.ev[3]);
        times_.verify_ms += ms;
        times_.raw_hits += hc.hits;
        times_.candidates += hc.candidates;
        times_.pairs += hc.pairs;
        n_rows = hc.rows;
        times_.rows += n_rows;
        return kOk;
    };
    // sort the verified rows by (request, position, pattern) and write their
    // text into d.text; the text bytes come back.  before_write runs just
    // before the text is written (the sliced path waits there for the
    // previous copy).
    auto format_rows = [&](uint32_t n_rows, uint64_t &text_bytes, auto &&before_write) -> int {
        CU(cudaEventRecord(d.ev[6], s));  // format interval: ev[6] -> ev[4]
        text_bytes = 0;
        if (!n_rows) return kOk;
        size_t tmp = 0;
        CU(cub::DeviceRadixSort::SortPairs(nullptr, tmp, d.keys.p, d.keys2.p, d.vals.p, d.vals2.p,
                                           (int)n_rows, 0, (int)key_bits, s));
        size_t tmp2 = 0;
        CU(cub::DeviceScan::ExclusiveSum(nullptr, tmp2, d.lens.p, d.offs.p, (int)n_rows + 1, s));
        if (d.cub_tmp.ensure(std::max(tmp, tmp2), err)) return err.code;
        tmp = d.cub_tmp.cap;
        CU(cub::DeviceRadixSort::SortPairs(d.cub_tmp.p, tmp, d.keys.p, d.keys2.p, d.vals.p,
                                           d.vals2.p, (int)n_rows, 0, (int)key_bits, s));
        const uint32_t *order = d.vals2.p;
        if (d.lens.ensure(n_rows + 1, err) || d.offs.ensure(n_rows + 1, err)) return err.code;
        unsigned fb = (unsigned)std::min<uint64_t>((n_rows + 255) / 256, (uint64_t)d.n_sm * 8);
        row_len_kernel<<<fb, 256, 0, s>>>(d.view(), d.rows.p, order, n_rows,
                                          (const ExactPattern *)tab(o_ep),
                                          (const RequestDev *)tab(o_rdev), d.lens.p);
        CU(cudaGetLastError());
        CU(cudaMemsetAsync(d.lens.p + n_rows, 0, 4, s));
        // widen lengths to 64-bit offsets
        tmp2 = d.cub_tmp.cap;
        CU(cub::DeviceScan::ExclusiveSum(d.cub_tmp.p, tmp2, d.lens.p, d.offs.p, (int)n_rows + 1, s));
        CU(cudaMemcpyAsync(&text_bytes, d.offs.p + n_rows, 8, cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        if (before_write(text_bytes)) return err.code;
        if (d.text.ensure(text_bytes + 1, err)) return err.code;
        row_write_kernel<<<fb, 256, 0, s>>>(d.view(), d.rows.p, order, n_rows,
                                            (const ExactPattern *)tab(o_ep),
                                            (const RequestDev *)tab(o_rdev), d.offs.p, d.text.p);
        CU(cudaGetLastError());
        times_.kernel_launches += 4;
        return kOk;
    };

    // match records of the n_rows formatted rows (streamed searches that ask
    // for them); first[r]: the first sorted row of request r in this piece
    auto write_records = [&](uint32_t n_rows, const std::vector<uint32_t> &first) -> int {
        if (!n_rows) return kOk;
        if (d.recs.ensure(n_rows, err) || d.req_first.ensure(first.size(), err)) return err.code;
        CU(cudaMemcpyAsync(d.req_first.p, first.data(), first.size() * 4, cudaMemcpyHostToDevice,
                           s));
        const unsigned fb = (unsigned)std::min<uint64_t>((n_rows + 255) / 256, (uint64_t)d.n_sm * 8);
        row_rec_kernel<<<fb, 256, 0, s>>>(d.view(), d.rows.p, d.vals2.p, n_rows,
                                          (const ExactPattern *)tab(o_ep),
                                          (const RequestDev *)tab(o_rdev), d.offs.p,
                                          d.req_first.p, d.recs.p);
        CU(cudaGetLastError());
        ++times_.kernel_launches;
        return kOk;
    };

    const ScanVariant *vsel = nullptr;
    if (!groups.empty()) {
        // autotuner: the fastest tile shape for this request shape, timed on
        // the first kTuneTiles tiles of every group; cached per shape
        uint32_t tot_pat = 0, max_l = 0, n_pam = 0, max_mm = 0;
        for (const ScanGroup &g : groups) {
            tot_pat += g.pat_end - g.pat_begin;
            n_pam += g.n_pam;
        }
        for (const RequestDev &r : rdev) {
            max_l = std::max(max_l, r.L);
            max_mm = std::max(max_mm, r.max_mm);
        }
        // shape key: patterns per group (power-of-4 bucket), groups (bucket),
        // PAM cells per group, longest pattern, largest threshold
        const uint32_t per_group = tot_pat / (uint32_t)groups.size();
        uint32_t bucket = 1;
        while (bucket < per_group) bucket <<= 2;
        const uint32_t gbucket = groups.size() <= 2 ? (uint32_t)groups.size()
                                 : groups.size() <= 8 ? 8u : 64u;
        const std::string key = "pat" + std::to_string(bucket) + "-grp" + std::to_string(gbucket) +
                                "-pam" + std::to_string(n_pam / groups.size()) + "-L" +
                                std::to_string(max_l) + "-mm" + std::to_string(max_mm);
        // tuning pays off only when the search is much larger than its sample
        const bool worth = full_tiles >= 8 * tune_tiles * groups.size();
        // the default: strand pairs compared directly for few patterns per
        // group (the fixed work per tile dominates there), else the per-warp
        // lean tile.  A direct shape holds a fixed number of patterns per
        // group and cannot run larger groups.
        uint32_t max_group_pats = 0;
        for (const ScanGroup &g : groups) max_group_pats = std::max(max_group_pats, g.pat_end - g.pat_begin);
        uint32_t max_group_pam = 0;
        for (const ScanGroup &g : groups) max_group_pam = std::max(max_group_pam, g.n_pam);
        auto usable = [&](int k) {
            const ScanVariant &x = kScanVariants[k];
            return !x.paired || (pairs_ok && max_group_pats <= x.max_pats &&
                                 max_group_pam <= kDirectPamCells);
        };
        int v_default = 0;
        if (max_group_pats <= kPairMaxPatterns)
            for (int k = kFirstPairVariant; k < kNumScanVariants && !v_default; ++k)
                if (usable(k)) v_default = k;
        int vi = v_default;
        const char *force = std::getenv("COF_SCAN_VARIANT");  // testing: pin a shape
        if (force && *force) {
            vi = std::max(0, std::min(kNumScanVariants - 1, std::atoi(force)));
            if (!usable(vi)) vi = 0;
        } else if (!tuner_.lookup(key, vi) && tuner_.enabled() && worth) {
            if (launch(kScanVariants[vi], true)) return err.code;  // warm-up
            float t[kNumScanVariants];
            for (int k = 0; k < kNumScanVariants; ++k) t[k] = 1e30f;
            for (int rep = 0; rep < 2; ++rep) {  // interleaved repeats, best of two
                for (int k = 0; k < kNumScanVariants; ++k) {
                    if (!usable(k)) continue;
                    CU(cudaEventRecord(d.ev[1], s));
                    if (launch(kScanVariants[k], true)) return err.code;
                    CU(cudaEventRecord(d.ev[2], s));
                    CU(cudaEventSynchronize(d.ev[2]));
                    float ms = 0;
                    cudaEventElapsedTime(&ms, d.ev[1], d.ev[2]);
                    t[k] = std::min(t[k], ms);
                }
            }
            // the default shape wins unless another is clearly faster
            for (int k = 0; k < kNumScanVariants; ++k)
                if (k != v_default && t[k] < 0.97f * t[vi]) vi = k;
            tuner_.store(key, vi);
        }
        if (!usable(vi)) vi = v_default;  // a cached choice for larger groups
        const ScanVariant &v = kScanVariants[vi];
        times_.scan_variant = vi;
        static const char *const kMinName[] = {"", "", "", "", "min3-"};
        if (v.paired)
            times_.scan_shape = "pair-direct-np" + std::to_string(v.max_pats) + "-warps" +
                                std::to_string(v.warps) + "-minb" + std::to_string(v.min_blocks) +
                                "-span" + std::to_string(v.span_tiles);
        else
            times_.scan_shape = std::string(v.per_warp ? "warp-" : "") + (v.lean ? "lean-" : "") +
                                kMinName[v.pair] + "cpt" + std::to_string(v.cpt) + "-warps" +
                                std::to_string(v.warps) + "-minb" + std::to_string(v.min_blocks) +
                                "-span" + std::to_string(v.span_tiles);
        vsel = &v;
    }
    if (!slices.empty()) {
        // one request, scanned slice by slice (slices need scan groups, so a
        // tile shape was chosen above); each slice's text is copied into the
        // page-locked result on the copy stream while the next slice scans
        PooledText hbuf;  // the result text, released on every early return
        // destroyed before hbuf: no copy may still write into it then
        struct CopyDrain {
            cudaStream_t cs;
            ~CopyDrain() { cudaStreamSynchronize(cs); }
        } drain{d.copy_stream};
        size_t hcap = 0;
        uint64_t host_off = 0, rows_total = 0;
        bool copy_pending = false;
        float ms = 0;
        // grows the result buffer to `need` bytes, keeping the text copied so far
        auto reserve = [&](size_t need) -> int {
            if (need <= hcap) return kOk;
            CU(cudaStreamSynchronize(d.copy_stream));
            PooledText nb;
            nb.p = PinnedPool::get().acquire(need);
            if (!nb.p) {
                err = {kOom, "out of page-locked host memory for result text"};
                return err.code;
            }
            if (hbuf.p) std::memcpy(nb.p, hbuf.p, host_off);
            hbuf = std::move(nb);
            hcap = need;
            return kOk;
        };
        times_.slices = (int)slices.size();
        // a streamed search: each slice's rows are one piece, handed to the
        // sink while the next slice scans
        std::unique_ptr<TextOut> tout;
        if (sink) {
            tout.reset(new TextOut(d.copy_stream, sink, out));
            before_wait = [&]() { return tout->drain(err); };
        }
        for (size_t j = 0; j < slices.size(); ++j) {
            uint32_t nr = 0;
            std::vector<uint32_t> rq;
            if (scan_verify(vsel, &slices[j], nr, rq)) return err.code;  // ends with a stream sync
            if (j > 0) {  // the previous slice's text write has finished
                cudaEventElapsedTime(&ms, d.ev[6], d.ev[4]);
                times_.format_ms += ms;
            }
            auto before_write = [&](uint64_t bytes) -> int {
                // d.text still feeds the previous slice's copy
                if (tout) return tout->drain(err);
                if (copy_pending) CU(cudaEventSynchronize(d.copy_done));
                size_t need = host_off + bytes + 1;
                if (need > hcap)  // room for the rest at this slice's rate (+20 %)
                    need = std::max<size_t>({need, (size_t)slice_text_hint_,
                                             (size_t)((double)(host_off + bytes) * slices.size() /
                                                      (double)(j + 1) * 1.2) + (1u << 20)});
                return reserve(need);
            };
            uint64_t tb = 0;
            if (format_rows(nr, tb, before_write)) return err.code;
            if (tout && tout->records() && write_records(nr, {0u})) return err.code;
            CU(cudaEventRecord(d.ev[4], s));
            rows_total += nr;
            if (tout) {
                CU(cudaEventRecord(d.fmt_done, s));
                if (tout->put(0, d.text.p, tb, nr, d.recs.p, d.fmt_done, err)) return err.code;
                copy_pending = tb != 0;
                continue;
            }
            if (tb) {
                CU(cudaEventRecord(d.fmt_done, s));
                CU(cudaStreamWaitEvent(d.copy_stream, d.fmt_done, 0));
                CU(cudaMemcpyAsync(hbuf.p + host_off, d.text.p, tb, cudaMemcpyDeviceToHost,
                                   d.copy_stream));
                CU(cudaEventRecord(d.copy_done, d.copy_stream));
                copy_pending = true;
                host_off += tb;
            }
        }
        before_wait = nullptr;
        CU(cudaEventRecord(d.ev[5], d.copy_stream));
        CU(cudaStreamSynchronize(d.copy_stream));
        CU(cudaStreamSynchronize(s));
        cudaEventElapsedTime(&ms, d.ev[6], d.ev[4]);
        times_.format_ms += ms;
        if (copy_pending) {  // the copy time left after the last slice's text
            cudaEventElapsedTime(&ms, d.ev[4], d.ev[5]);
            times_.d2h_ms += std::max(0.0f, ms);
        }
        if (tout) return tout->finish(err);
        if (reserve(host_off + 1)) return err.code;
        hbuf.p[host_off] = 0;
        out[0].text = hbuf.p;
        out[0].pooled = std::move(hbuf);
        out[0].text_len = host_off;
        out[0].n_rows = rows_total;
        slice_text_hint_ = host_off + host_off / 50 + 1;
        return kOk;
    }

    uint32_t n_rows = 0;
    uint64_t text_bytes = 0;
    std::vector<uint32_t> req_rows;
    if (scan_verify(vsel, nullptr, n_rows, req_rows) ||
        format_rows(n_rows, text_bytes, [](uint64_t) { return 0; }))
        return err.code;
    // each request's rows (sorted request-major) go straight from the
    // device into its own page-locked result buffer
    CU(cudaEventRecord(d.ev[4], s));
    // text offset where each request's rows end: one small asynchronous copy
    // per request into a page-locked array, then a single wait
    std::vector<uint64_t> tend(reqs.size(), text_bytes);
    if (reqs.size() > 1) {
        PooledText bnd;
        bnd.p = PinnedPool::get().acquire(8 * reqs.size());
        if (!bnd.p) {
            err = {kOom, "out of page-locked host memory for result text"};
            return err.code;
        }
        uint64_t *hb = reinterpret_cast<uint64_t *>(bnd.p);
        uint64_t r1 = 0;
        for (size_t ri = 0; ri < reqs.size(); ++ri) {
            r1 += req_rows[ri];
            hb[ri] = text_bytes;
            if (r1 < n_rows)
                CU(cudaMemcpyAsync(hb + ri, d.offs.p + r1, 8, cudaMemcpyDeviceToHost, s));
        }
        CU(cudaStreamSynchronize(s));
        for (size_t ri = 0; ri < reqs.size(); ++ri) tend[ri] = hb[ri];
    }
    if (sink) {
        // a streamed search: each request's rows are one piece
        TextOut tout(d.copy_stream, sink, out);
        std::vector<uint32_t> first(reqs.size());
        for (size_t ri = 0, r = 0; ri < reqs.size(); r += req_rows[ri], ++ri)
            first[ri] = (uint32_t)r;
        if (tout.records() && write_records(n_rows, first)) return err.code;
        CU(cudaEventRecord(d.fmt_done, s));
        uint64_t t0 = 0;
        for (size_t ri = 0; ri < reqs.size(); ++ri) {
            if (tout.put(ri, d.text.p + t0, tend[ri] - t0, req_rows[ri], d.recs.p + first[ri],
                         d.fmt_done, err))
                return err.code;
            t0 = tend[ri];
        }
        CU(cudaEventRecord(d.ev[5], d.copy_stream));
        if (tout.finish(err)) return err.code;
        float ms;
        cudaEventElapsedTime(&ms, d.ev[6], d.ev[4]);
        times_.format_ms += ms;
        cudaEventElapsedTime(&ms, d.ev[4], d.ev[5]);
        times_.d2h_ms += std::max(0.0f, ms);
        return kOk;
    }
    uint64_t r0 = 0, t0 = 0;
    for (size_t ri = 0; ri < reqs.size(); ++ri) {
        const uint64_t r1 = r0 + req_rows[ri];
        const uint64_t t1 = tend[ri];
        char *buf = PinnedPool::get().acquire(t1 - t0 + 1);
        if (!buf) {
            err = {kOom, "out of page-locked host memory for result text"};
            return err.code;
        }
        out[ri].pooled.p = buf;
        if (t1 > t0) CU(cudaMemcpyAsync(buf, d.text.p + t0, t1 - t0, cudaMemcpyDeviceToHost, s));
        out[ri].n_rows = req_rows[ri];
        out[ri].text = buf;
        out[ri].text_len = t1 - t0;
        r0 = r1;
        t0 = t1;
    }
    CU(cudaEventRecord(d.ev[5], s));
    CU(cudaStreamSynchronize(s));
    for (Result &r : out) r.pooled.p[r.text_len] = 0;
    float ms;
    cudaEventElapsedTime(&ms, d.ev[6], d.ev[4]);
    times_.format_ms += ms;
    cudaEventElapsedTime(&ms, d.ev[4], d.ev[5]);
    times_.d2h_ms += ms;
    return kOk;
}

}  // namespace cof
