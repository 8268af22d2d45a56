// bulge.cu -- the DNA/RNA-bulge search path (max_dna_bulges or
// max_rna_bulges > 0, search.rs:1513) on sm_100a.
//
// Reference semantics (the CPU path, search.rs:779-897 + traceback.rs:181-381
// + search.rs:1316-1374 + main.rs:145-157): for every end position t of a
// batch's active range and every pattern, check_pam_quick, a windowed Myers
// edit distance <= mm + db + rb, then the full DP over the text window
// [t + 1 - (L + db), t] and a depth-first enumeration of EVERY traceback
// within the caps, each one a row after the PAM check at its match cells and
// the record-end drop.
//
// Kernels:
//   myers_filter_kernel  one thread per (1024-position tile, pattern): a
//       streaming Myers sweep (Myers 1999, semi-global; 32-bit words for
//       patterns of at most 32 cells, 64-bit words up to 64 cells, the
//       single-u64 limit of myers.rs:3) started >= W - 1 positions before
//       the tile (W = L + max_db, the reference's text window).  Its score at t bounds the windowed
//       score from below (more start positions), which bounds the DP cost from
//       below (the DP forbids padding cells and may forbid bulges), so
//       "score <= max_edits" keeps every position the reference can emit.
//       Positions that also pass the exact check_pam_quick become candidates.
//   traceback_kernel  one thread per candidate: the reference's DP and its
//       enumeration in the same transition order (diagonal, RNA bulge, DNA
//       bulge) with the same pruning, then classify's PAM check and
//       convert_matches_myers; survivors are written as alignment records.
//   mrow_len_kernel / mrow_write_kernel  the 8-column rows with '-' gaps,
//       reverse-complemented for reverse-strand patterns.
#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "cof_engine.h"
#include "engine_dev.cuh"
#include "textout.h"

namespace cof {

namespace {

constexpr int kMaxCells = 72;          // L <= 64, L + max_db <= 72
constexpr uint32_t kBulgeChunkMax = 1u << 21;  // candidates per chunk at most
constexpr uint32_t kBulgeProbe = 1u << 18;     // probe chunk of a very large set
constexpr uint32_t kTile = 1024;       // end positions per filter work item
constexpr uint32_t kWarmMin = 48;      // Myers warm-up before a tile (>= W - 1)
constexpr int kSmemMyers = 512;        // patterns whose eq tables fit in smem

// Myers warm-up for windows of at most wmax cells: W - 1, in whole 16-cell
// words, and never below the 48 cells every window of <= 40 cells uses
inline uint32_t myers_warm(uint32_t wmax) {
    const uint32_t need = wmax > 0 ? ((wmax - 1 + 15) & ~15u) : 0;
    return need > kWarmMin ? need : kWarmMin;
}

struct MyersPattern {
    uint32_t request, strand, L, E;    // E = max edits = mm + db + rb
    uint32_t W, pam_off, pam_n, pad;
    uint32_t eq_lo[16], eq_hi[16];     // Myers Eq per genome nibble value, cells 0..31 / 32..63
    uint8_t b4[kMaxCells];             // pattern bit4 cells
    uint8_t isn[kMaxCells];            // pattern char is N/n (pam_is_n)
    uint8_t eff[kMaxCells];            // effective filter bit4 per cell
    uint8_t pamf[kMaxCells];           // PAM precheck filter list
};

struct MyersReqDev {
    uint32_t L, mm, db, rb, E, W, pam_len, raw;  // raw: Match lines, not rows
    uint32_t first_pattern, T, nbits, pad;       // T = mm + 1 thresholds per budget
    // bit sets of the budget DP cells (bit b * T + v: "F[b] <= v"):
    uint64_t m_valid[2];  // the (db + 1)(rb + 1) * T bits in use
    uint64_t m_sub[2];    // valid bits with v >= 1 (targets of a +1 shift)
    uint64_t m_rna[2];    // budgets with br >= 1 (targets of an RNA step)
    uint64_t m_dna[2];    // budgets with bd >= 1 (targets of a DNA step)
    uint64_t m_full[2];   // the full budget (db, rb)
};

struct MyersTile {
    uint64_t t0, t1;                   // global end positions [t0, t1)
    uint32_t batch, pad0;
    uint64_t pad1;
};

// check_pam_quick (search.rs:703-755) in batch-local coordinates.
__device__ bool pam_quick(const uint8_t *bit4, const BatchDev &B, uint32_t end_pos,
                          const MyersPattern &P, uint32_t db, uint32_t rb) {
    const int dr = P.pam_off == 0 ? (int)db + 1 : 1;
    const int rr = P.pam_off == 0 ? (int)rb + 1 : 1;
    for (int bd = 0; bd < dr; ++bd) {
        for (int br = 0; br < rr; ++br) {
            const int span = (int)P.L + bd - br;
            if (span <= 0 || (uint32_t)span > end_pos + 1) continue;
            const uint32_t as = end_pos + 1 - (uint32_t)span;
            bool ok = true;
            for (uint32_t k = 0; k < P.pam_n; ++k) {
                const uint32_t gp = as + P.pam_off + k;
                if (gp >= B.valid) { ok = false; break; }
                const uint8_t g = nib(bit4, B.base + gp), f = P.pamf[k];
                const bool good = f == 0xF ? g != 0 : (g != 0 && g != 0xF && (g & f));
                if (!good) { ok = false; break; }
            }
            if (ok) return true;
        }
    }
    return false;
}

// one column of the streaming Myers sweep (Myers 1999, the step of
// myers.rs:56-90) over a Word-wide pattern bit vector; returns the score change
template <typename Word>
__device__ __forceinline__ int myers_step(Word eq, Word &vp, Word &vn, Word mask, uint32_t sh) {
    const Word x = eq | vn;
    const Word d0 = (((x & vp) + vp) ^ vp) | x;
    const Word hn = vp & d0;
    const Word hp = vn | ~(vp | d0);
    const Word xs = hp << 1;
    vn = xs & d0;
    vp = ((hn << 1) | ~(xs | d0)) & mask;
    vn &= mask;
    return (int)((hp >> sh) & 1u) - (int)((hn >> sh) & 1u);
}

// myers_step without the pattern mask: bits above the pattern's last cell
// hold garbage that never reaches the score bit sh (the step only carries
// toward higher bits)
template <typename Word>
__device__ __forceinline__ int myers_step_unmasked(Word eq, Word &vp, Word &vn, uint32_t sh) {
    const Word x = eq | vn;
    const Word d0 = (((x & vp) + vp) ^ vp) | x;
    const Word hn = vp & d0;
    const Word hp = vn | ~(vp | d0);
    const Word xs = hp << 1;
    vn = xs & d0;
    vp = (hn << 1) | ~(xs | d0);
    return (int)((hp >> sh) & 1u) - (int)((hn >> sh) & 1u);
}

// the Word-wide Eq vector of genome nibble b
template <typename Word>
__device__ __forceinline__ Word eq_word(const MyersPattern &P, uint32_t b) {
    if constexpr (sizeof(Word) == 4) return P.eq_lo[b];
    else return ((uint64_t)P.eq_hi[b] << 32) | P.eq_lo[b];
}

template <typename Word>
__device__ __forceinline__ Word myers_mask(uint32_t L) {
    return L >= 8 * sizeof(Word) ? ~(Word)0 : (((Word)1 << L) - 1);
}

template <typename Word>
__global__ void myers_filter_kernel(const uint8_t *__restrict__ bit4,
                                    const BatchDev *__restrict__ batches,
                                    const MyersTile *__restrict__ tiles, uint64_t n_tiles,
                                    const MyersPattern *__restrict__ pats, uint32_t n_pat,
                                    const MyersReqDev *__restrict__ reqs, uint32_t warm,
                                    MyersCand *cand, uint32_t cap, Counters *ctr) {
    constexpr uint32_t kStaged = kSmemMyers * 4 / sizeof(Word);  // 32 KB of eq tables
    __shared__ Word seq[kStaged * 16];
    const bool staged = n_pat <= kStaged;
    if (staged)
        for (uint32_t i = threadIdx.x; i < n_pat * 16; i += blockDim.x) seq[i] = eq_word<Word>(pats[i / 16], i % 16);
    __syncthreads();
    const uint64_t n_items = n_tiles * n_pat;
    for (uint64_t item = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; item < n_items;
         item += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t ti = item / n_pat;
        const uint32_t p = (uint32_t)(item % n_pat);
        const MyersTile T = tiles[ti];
        const BatchDev B = batches[T.batch];
        const MyersPattern &P = pats[p];
        const MyersReqDev R = reqs[P.request];
        const uint32_t L = P.L;
        const Word mask = myers_mask<Word>(L);
        const uint32_t sh = L - 1;
        Word vp = mask, vn = 0;
        int score = (int)L;
        const uint64_t ws = T.t0 >= warm ? ((T.t0 - warm) & ~15ull) : 0;
        unsigned long long word = 0;
        for (uint64_t q = ws; q < T.t1; ++q) {
            if ((q & 15) == 0 || q == ws)
                word = __ldg(reinterpret_cast<const unsigned long long *>(bit4 + ((q >> 1) & ~7ull)));
            const uint32_t b = (uint32_t)(word >> ((q & 15) * 4)) & 0xF;
            score += myers_step<Word>(staged ? seq[16 * p + b] : eq_word<Word>(P, b), vp, vn, mask, sh);
            if (q >= T.t0 && score <= (int)P.E) {
                const uint32_t tl = (uint32_t)(q - B.base);
                if (tl + 1 >= L && pam_quick(bit4, B, tl, P, R.db, R.rb)) {
                    const uint32_t i = append_slot(&ctr->hits);
                    if (i < cap) cand[i] = MyersCand{tl, T.batch, p, 0};
                    else ctr->overflow = 1;
                }
            }
        }
    }
}

// ---- Myers filter with the PAM test precomputed per tile --------------------
//
// check_pam_quick depends on the pattern only through its PAM form: the
// filter bit4 of its N cells from the first N cell on (pam_off) and the
// alignment spans it tries (L + bd - br for every bd <= db, br <= rb when the
// PAM leads the pattern, L otherwise).  All patterns of one request strand
// share a form.  A block takes a few consecutive tiles and first computes,
// for every form, Q(y) = "the PAM cells starting at batch cell y are all
// good" and from it pam_ok(t) = OR over spans of Q(t + 1 - span + pam_off)
// for the tile's end positions t, into shared memory.  Then every
// (tile, pattern) thread runs the streaming Myers sweep a 16-cell genome
// word at a time and meets each word's "score <= E" bits with 16 pam_ok
// bits, instead of the reference's per-position cell loads; a round's
// candidates are staged in shared memory and appended with one atomic.
constexpr uint32_t kMfThreads = 256;
constexpr uint32_t kMfMaxTiles = 32;           // tiles per block
constexpr uint32_t kMfMaxForms = 8;            // PAM forms per launch
constexpr uint32_t kMfQWords = kTile / 32 + 2; // Q bits: 1024 ends + <= 16 span shifts
constexpr uint32_t kMfStage = 3072;            // candidates staged per block and round

struct PamForm {
    uint32_t pam_off, pam_n, span_lo, span_hi;  // spans span_lo..span_hi
    uint8_t f[kMaxCells];                        // filter bit4 of the PAM cells
};

template <typename Word>
__global__ void __launch_bounds__(kMfThreads)
myers_tile_kernel(const uint8_t *__restrict__ bit4, const BatchDev *__restrict__ batches,
                  const MyersTile *__restrict__ tiles, uint64_t n_tiles,
                  const MyersPattern *__restrict__ pats, uint32_t n_pat,
                  const PamForm *__restrict__ forms, uint32_t n_forms, uint32_t tpb,
                  uint32_t warm, MyersCand *cand, uint32_t cap, Counters *ctr,
                  uint32_t stage_cap) {
    extern __shared__ __align__(16) uint32_t mf_smem[];
    uint32_t *q_bits = mf_smem;                            // [tpb][n_forms][kMfQWords]
    uint32_t *ok_bits = q_bits + tpb * n_forms * kMfQWords; // [tpb][n_forms][32]
    // [16][n_pat] when staged (lanes of one tile read one nibble's row:
    // no bank conflicts); 8-byte aligned (kMfQWords and 32 words are even)
    Word *seq = reinterpret_cast<Word *>(ok_bits + tpb * n_forms * 32);
    const bool staged = n_pat <= (uint32_t)kSmemMyers;
    // a round's candidates (tile-local end, tile << 24 | pattern), then
    // the stage's fill count and the round's base in the candidate list
    uint2 *stage = reinterpret_cast<uint2 *>(seq + (staged ? n_pat * 16 : 0));
    uint32_t *stage_n = reinterpret_cast<uint32_t *>(stage + kMfStage);
    uint32_t *stage_base = stage_n + 1;
    if (staged)
        for (uint32_t i = threadIdx.x; i < n_pat * 16; i += blockDim.x) seq[i] = eq_word<Word>(pats[i % n_pat], i / n_pat);
    for (uint64_t tb = blockIdx.x; tb * tpb < n_tiles; tb += gridDim.x) {
        const uint64_t tile0 = tb * tpb;
        const uint32_t nt = (uint32_t)(n_tiles - tile0 < tpb ? n_tiles - tile0 : tpb);
        __syncthreads();  // the previous tile block's readers are done
        // Q words: bit i of word w is Q(y0 + 32 w + i), y0 = t0 + 1 - span_hi + pam_off
        for (uint32_t i = threadIdx.x; i < nt * n_forms * kMfQWords; i += blockDim.x) {
            const uint32_t tl = i / (n_forms * kMfQWords), fi = (i / kMfQWords) % n_forms,
                           w = i % kMfQWords;
            const MyersTile T = tiles[tile0 + tl];
            const BatchDev B = batches[T.batch];
            const PamForm &F = forms[fi];
            const int64_t y0 = (int64_t)(T.t0 - B.base) + 1 - (int64_t)F.span_hi + F.pam_off;
            uint32_t bits = 0;
            for (uint32_t b = 0; b < 32; ++b) {
                const int64_t y = y0 + 32 * (int64_t)w + b;
                if (y < (int64_t)F.pam_off) continue;  // alignment start before the batch
                bool ok = true;
                for (uint32_t k = 0; k < F.pam_n && ok; ++k) {
                    const uint64_t gp = (uint64_t)y + k;
                    if (gp >= B.valid) { ok = false; break; }
                    const uint8_t g = nib(bit4, B.base + gp), f = F.f[k];
                    ok = f == 0xF ? g != 0 : (g != 0 && g != 0xF && (g & f));
                }
                bits |= (uint32_t)ok << b;
            }
            q_bits[i] = bits;
        }
        __syncthreads();
        // pam_ok words: end position t0 + 32 w + j, OR over the span shifts
        for (uint32_t i = threadIdx.x; i < nt * n_forms * 32; i += blockDim.x) {
            const uint32_t tf = i / 32, w = i % 32;
            const PamForm &F = forms[tf % n_forms];
            const uint32_t *Q = q_bits + tf * kMfQWords;
            uint32_t v = 0;
            for (uint32_t d = 0; d <= F.span_hi - F.span_lo; ++d) {
                // bits 32 w + j + (span_hi - span) of Q, span = span_hi - d
                const uint32_t s = 32 * w + d;
                v |= __funnelshift_r(Q[s >> 5], Q[(s >> 5) + 1], s & 31);
            }
            ok_bits[i] = v;
        }
        __syncthreads();
        // streaming Myers per (tile, pattern), in rounds of one item per
        // thread.  A round's candidates are staged in shared memory and
        // appended with one global atomic: one counter shared by every SM,
        // taken once per candidate, serialised the whole sweep.
        for (uint32_t round0 = 0; round0 < nt * n_pat; round0 += blockDim.x) {
            if (threadIdx.x == 0) *stage_n = 0;
            __syncthreads();
            const uint32_t i = round0 + threadIdx.x;
            if (i < nt * n_pat) {
                const uint32_t tl = i / n_pat, p = i % n_pat;
                const MyersTile T = tiles[tile0 + tl];
                const BatchDev B = batches[T.batch];
                const MyersPattern &P = pats[p];
                const uint32_t *okw = ok_bits + (tl * n_forms + P.pad) * 32;
                const uint32_t L = P.L;
                const uint32_t sh = L - 1;
                const int E = (int)P.E;
                // The Eq lookup reads the staged table ([16][n_pat]: the lanes of
                // one tile read one row, without bank conflicts) straight from
                // shared memory; a pointer that could point to either table
                // would make every lookup a generic load, which waits like a
                // global one.
                // No mask on vp / vn: every operation of the step (bitwise
                // logic, the add, left shifts) carries information only toward
                // higher bits, so the bits above L - 1 never reach bit L - 1,
                // the only one the score reads.
                Word vp = ~(Word)0, vn = 0;
                int score = (int)L;
                const uint64_t t0 = T.t0, t1 = T.t1;
                // whole 16-cell genome words from ws (a multiple of 16) on:
                // the warm-up words before t0 run the sweep alone, the others
                // also collect a bit per cell whose score is within E.  Each
                // word is loaded one word ahead, under the 16 steps before.
                const uint64_t ws = t0 >= warm ? ((t0 - warm) & ~15ull) : 0;
                const unsigned long long *gw = reinterpret_cast<const unsigned long long *>(bit4);
                unsigned long long ahead = __ldg(gw + (ws >> 4));
                for (uint64_t qw = ws; qw < t1; qw += 16) {
                    const unsigned long long word = ahead;
                    if (qw + 16 < t1) ahead = __ldg(gw + ((qw + 16) >> 4));
                    uint32_t within = 0;
                    if (qw + 16 <= t0) {
#pragma unroll
                        for (uint32_t k = 0; k < 16; ++k) {
                            const uint32_t b = (uint32_t)(word >> (4 * k)) & 0xF;
                            const Word e = staged ? seq[b * n_pat + p] : eq_word<Word>(P, b);
                            score += myers_step_unmasked<Word>(e, vp, vn, sh);
                        }
                        continue;
                    }
#pragma unroll
                    for (uint32_t k = 0; k < 16; ++k) {
                        const uint32_t b = (uint32_t)(word >> (4 * k)) & 0xF;
                        const Word e = staged ? seq[b * n_pat + p] : eq_word<Word>(P, b);
                        score += myers_step_unmasked<Word>(e, vp, vn, sh);
                        within |= ((uint32_t)(score - E - 1) >> 31) << k;  // score <= E
                    }
                    // cells of the tile only: [t0, t1)
                    if (qw < t0) within &= ~0u << (uint32_t)(t0 - qw);
                    if (qw + 16 > t1) within &= (1u << (uint32_t)(t1 - qw)) - 1u;
                    if (!within) continue;
                    // pam_ok bits of cells qw .. qw + 15 (tile offsets r0 .. r0 + 15)
                    const int r0 = (int)(qw - t0);
                    uint32_t okb;
                    if (r0 >= 0) {
                        const uint32_t wi = (uint32_t)r0 >> 5;
                        const uint32_t hi = wi + 1 < 32 ? okw[wi + 1] : 0u;
                        okb = __funnelshift_r(okw[wi], hi, (uint32_t)r0 & 31);
                    } else {
                        okb = okw[0] << (uint32_t)(-r0);
                    }
                    uint32_t hits = within & okb & 0xFFFFu;
                    while (hits) {
                        const uint32_t k = __ffs(hits) - 1;
                        hits &= hits - 1;
                        const uint32_t tlc = (uint32_t)(qw + k - B.base);
                        if (tlc + 1 >= L) {
                            const uint32_t slot = atomicAdd(stage_n, 1u);
                            if (slot < stage_cap) {
                                stage[slot] = make_uint2(tlc, (tl << 24) | p);
                            } else {  // stage full: straight to the list
                                const uint32_t c = atomicAdd(&ctr->hits, 1u);
                                if (c < cap) cand[c] = MyersCand{tlc, T.batch, p, 0};
                                else ctr->overflow = 1;
                            }
                        }
                    }
                }
            }
            __syncthreads();
            const uint32_t ns = min(*stage_n, stage_cap);
            if (threadIdx.x == 0) *stage_base = ns ? atomicAdd(&ctr->hits, ns) : 0u;
            __syncthreads();
            const uint32_t gb = *stage_base;
            for (uint32_t k = threadIdx.x; k < ns; k += blockDim.x) {
                const uint2 e = stage[k];
                const uint64_t c = (uint64_t)gb + k;
                if (c < cap) cand[c] = MyersCand{e.x, tiles[tile0 + (e.y >> 24)].batch, e.y & 0xFFFFFFu, 0};
                else ctr->overflow = 1;
            }
            __syncthreads();  // the stage is read before the next round resets it
        }
    }
}

__device__ __forceinline__ bool loose(uint8_t p, uint8_t t) {  // cmp_loose_bit4
    if (t == 0) return false;
    if (p == 0xF) return true;
    if (t == 0xF) return false;
    return (p & t) != 0;
}

constexpr uint8_t kInf = 100;  // DP values are capped here (max_edits <= 30)

struct Frame {
    uint8_t i, j, st, cost, mm, db, rb, pad;
};

__global__ void __launch_bounds__(128)
traceback_kernel(GenomeDev G, const BatchDev *__restrict__ batches,
                 const MyersPattern *__restrict__ pats, const MyersReqDev *__restrict__ reqs,
                 const MyersCand *__restrict__ cand, uint32_t n_cand, MyersRow *rows,
                 uint32_t row_cap, uint64_t *keys, uint32_t *vals, Counters *ctr,
                 uint32_t *req_rows) {
    for (uint32_t ci = blockIdx.x * blockDim.x + threadIdx.x; ci < n_cand;
         ci += gridDim.x * blockDim.x) {
        const MyersCand c = cand[ci];
        const BatchDev B = batches[c.batch];
        const MyersPattern &P = pats[c.pattern];
        const MyersReqDev R = reqs[P.request];
        const uint32_t L = P.L, W = P.W, t = c.t_local;
        const uint32_t ts = t + 1 > W ? t + 1 - W : 0;
        const uint32_t n = t + 1 - ts;
        uint8_t text[kMaxCells];
        for (uint32_t k = 0; k < n; ++k) text[k] = nib(G.bit4, B.base + ts + k);
        uint8_t pb[kMaxCells], isn[kMaxCells];
        for (uint32_t k = 0; k < L; ++k) {
            pb[k] = P.b4[k];
            isn[k] = P.isn[k];
        }
        // DP (traceback.rs:194-225), row stride kMaxCells + 1
        uint8_t dp[(kMaxCells + 1) * (kMaxCells + 1)];
        const uint32_t dc = R.db == 0 ? kInf : 1, rc = R.rb == 0 ? kInf : 1;
#define DPA(i, j) dp[(i) * (kMaxCells + 1) + (j)]
        for (uint32_t i = 0; i <= L; ++i) DPA(i, 0) = (uint8_t)min(i * rc, (uint32_t)kInf);
        for (uint32_t j = 1; j <= n; ++j) DPA(0, j) = 0;
        for (uint32_t i = 1; i <= L; ++i) {
            for (uint32_t j = 1; j <= n; ++j) {
                if (text[j - 1] == 0) { DPA(i, j) = kInf; continue; }
                const uint32_t mc = loose(pb[i - 1], text[j - 1]) ? 0 : 1;
                uint32_t v = min(DPA(i - 1, j - 1) + mc, DPA(i - 1, j) + rc);
                v = min(v, DPA(i, j - 1) + dc);
                DPA(i, j) = (uint8_t)min(v, (uint32_t)kInf);
            }
        }
        if (DPA(L, n) > P.E) continue;
        // enumerate (traceback.rs:242-381), iterative, same transition order
        Frame stk[kMaxCells + 2];
        uint8_t ops[kMaxCells + 2];
        int sp = 0;
        stk[sp++] = Frame{(uint8_t)L, (uint8_t)n, 0, 0, 0, 0, 0, 0};
        while (sp > 0) {
            Frame &f = stk[sp - 1];
            if (f.st == 0) {
                f.st = 1;
                if ((uint32_t)f.cost + DPA(f.i, f.j) > P.E || f.mm > R.mm || f.db > R.db ||
                    f.rb > R.rb) {
                    --sp;
                    continue;
                }
                if (f.i == 0) {
                    // a complete alignment: ops[0 .. sp-2] in walk-back order
                    const int n_ops = sp - 1;
                    uint32_t span = 0;
                    for (int k = 0; k < n_ops; ++k) span += ops[k] != 3;
                    // classify: filter at every match / substitution cell
                    bool ok = true;
                    uint32_t pi = 0, gi = f.j;
                    uint64_t o0 = 0, o1 = 0;
                    uint32_t o2 = 0;
                    for (int k = 0; k < n_ops; ++k) {
                        const uint8_t op = ops[n_ops - 1 - k];
                        if (k < 32) o0 |= (uint64_t)op << (2 * k);
                        else if (k < 64) o1 |= (uint64_t)op << (2 * (k - 32));
                        else o2 |= (uint32_t)op << (2 * (k - 64));
                        if (op <= 1) {
                            const uint8_t g = text[gi], fl = P.eff[pi];
                            const bool good = fl == 0xF ? g != 0 : (g != 0 && g != 0xF && (g & fl));
                            if (!good) ok = false;
                            ++pi;
                            ++gi;
                        } else if (op == 2) {
                            ++gi;
                        } else {
                            ++pi;
                        }
                    }
                    if (ok) {
                        // convert_matches_myers: owning chunk, record-end drop
                        const uint64_t start = B.base + t + 1 - span;
                        const uint64_t gbyte = start >> 1;
                        uint32_t lo = B.first, hi = B.first + B.nch;
                        while (hi - lo > 1) {
                            const uint32_t mid = (lo + hi) >> 1;
                            if (G.boff[mid] <= gbyte) lo = mid; else hi = mid;
                        }
                        const uint32_t k = lo;
                        const uint64_t pos = G.start[k] + (start - 2 * G.boff[k]);
                        const bool end_chrom = (k == B.first + B.nch - 1) || G.start[k + 1] == 0;
                        const uint64_t extent = (uint64_t)L + f.db - f.rb;
                        if (!(end_chrom && pos + extent > G.end[k])) {
                            const uint32_t r = atomicAdd(&ctr->rows, 1u);
                            if (r < row_cap) {
                                MyersRow w;
                                w.start = start;
                                w.pos = pos;
                                w.ops[0] = o0;
                                w.ops[1] = o1;
                                w.chunk = k;
                                w.pattern = c.pattern;
                                w.n_ops = (uint8_t)n_ops;
                                w.mm = f.mm;
                                w.db = f.db;
                                w.rb = f.rb;
                                w.ops_hi = o2;
                                rows[r] = w;
                                keys[r] = ((uint64_t)c.pattern << G.key_shift) | start;
                                vals[r] = r;
                                atomicAdd(&req_rows[P.request], 1u);
                            } else {
                                ctr->overflow = 1;
                            }
                        }
                    }
                    --sp;
                    continue;
                }
            }
            const uint32_t i = f.i, j = f.j;
            if (f.st == 1) {  // diagonal: match / substitution
                f.st = 2;
                if (j > 0) {
                    const uint8_t mc = loose(pb[i - 1], text[j - 1]) ? 0 : 1;
                    if (!(mc && isn[i - 1])) {
                        ops[sp - 1] = mc;
                        stk[sp] = Frame{(uint8_t)(i - 1), (uint8_t)(j - 1), 0,
                                        (uint8_t)(f.cost + mc), (uint8_t)(f.mm + mc), f.db, f.rb, 0};
                        ++sp;
                        continue;
                    }
                }
            }
            if (f.st == 2) {  // RNA bulge: pattern cell skipped
                f.st = 3;
                if (f.rb < R.rb && R.rb > 0) {
                    const bool next_pam = i < L && isn[i];
                    const bool prev_pam = i >= 2 && isn[i - 2];
                    if (!isn[i - 1] && !next_pam && !prev_pam) {
                        ops[sp - 1] = 3;
                        stk[sp] = Frame{(uint8_t)(i - 1), (uint8_t)j, 0, (uint8_t)(f.cost + 1),
                                        f.mm, f.db, (uint8_t)(f.rb + 1), 0};
                        ++sp;
                        continue;
                    }
                }
            }
            if (f.st == 3) {  // DNA bulge: text cell skipped
                f.st = 4;
                if (f.db < R.db && R.db > 0 && j > 0 && i < L) {
                    const bool prev_n = i > 0 && isn[i - 1];
                    if (!(prev_n && isn[i])) {
                        ops[sp - 1] = 2;
                        stk[sp] = Frame{(uint8_t)i, (uint8_t)(j - 1), 0, (uint8_t)(f.cost + 1),
                                        f.mm, (uint8_t)(f.db + 1), f.rb, 0};
                        ++sp;
                        continue;
                    }
                }
            }
            --sp;
        }
#undef DPA
    }
}

// ---- warp-per-candidate traceback ------------------------------------------
//
// Same rows as traceback_kernel, with the work laid out for a GPU.
//
// Budget DP.  F[bd][br](i, j) = fewest mismatches on any alignment of
// pattern cells [0, i) ending at text cell j that uses at most bd DNA and
// br RNA bulges.  It obeys exactly the move rules of the enumeration: a
// diagonal step is barred under a pattern N on a mismatch and where
// classify's filter test fails; the bulge steps have their N-neighbour
// rules; a node over a padding cell is dead.  Only "F <= v" for
// v = 0..mm matters, so a cell is stored as a bit set over (budget, v):
// bit b * T + v (T = mm + 1, b = bd * (rb + 1) + br) is set iff
// F[b] <= v.  Then min is OR, a mismatch (+1) is a shift by one bit within
// each budget group, a bulge step (smaller budget) is a shift by whole
// groups, and values above mm are simply absent.  One or two 64-bit words
// per cell (NW) hold (db + 1)(rb + 1)(mm + 1) <= 128 bits.
//
// traceback_warp_kernel: one warp takes one candidate (or a handed-on
// subtree) from a dynamic queue, computes the table as a wavefront (lane =
// pattern row i, step s = i + j, the upper row arrives by shuffle) into
// shared memory, then enumerates with exact pruning: a node (i, j) with m
// mismatches and d, r bulges so far is kept iff bit
// ((db - d)(rb + 1) + rb - r) * T + mm - m of its cell is set, so every
// kept node lies on at least one emitted alignment (the reference's cost
// bound and caps are both implied, nothing else is cut).  The warp pops up
// to 32 nodes of a shared-memory stack, expands them in parallel and pushes
// the children; leaves (i = 0) are written as rows after the record-end
// drop (classify's filter test is already part of the moves).  A warp that
// spends kTbBudget iterations on one tree hands its remaining stack to a
// global queue, which the next pass spreads over all warps, so a candidate
// with thousands of alignments cannot serialise the launch.
//
// Patterns of more than 32 cells: the wavefront runs in passes of 32 rows,
// lane 0 of a later pass reading its upper row from the table.
constexpr int kTbWarps = 4;                  // warps per block (fewer for large tables)
constexpr uint32_t kTbSpare = 80;            // stack slots beyond the walk margin
constexpr uint32_t kTbMaxBits = 128;         // budget bits per cell (NW <= 2)
constexpr uint32_t kTbBudget = 128;          // iterations on one tree before handing it on
constexpr uint32_t kTbQueue = 1u << 21;      // subtrees per hand-on queue
constexpr int kTbMaxPasses = 24;             // the last pass finishes every tree
constexpr uint32_t kTbText = 80;             // staged window text bytes (>= kMaxCells)
constexpr uint32_t kTbPat = 64;              // staged bytes per pattern array (>= L)

// Stack slots a one-node-at-a-time walk can add to a warp's stack: at most
// two per level (three children, one popped), levels <= W; never below the
// 80 of a 40-cell window.
inline uint32_t tb_margin(uint32_t wmax) { return 2 * std::max(wmax, 40u); }

// A node of the enumeration.  NO 64-bit words and ops_hi hold its walk-back
// ops, 2 bits per op: depths 0..32 NO - 1 in ops, the next 16 in ops_hi
// (NO = 1: windows of <= 48 cells, NO = 2: <= 80).  Its depth is L - i + d
// (each step consumes a pattern cell, or a text cell for a DNA bulge).
template <int NO>
struct TbNode {
    uint64_t ops[NO];
    uint32_t ops_hi;
    uint32_t st;      // i | j << 7 | m << 14 | d << 20 | r << 24
};

// one unit of enumeration work: a candidate's root, or a subtree handed on
// by a warp that spent its iteration budget (cand == ~0u: an empty slot)
template <int NO>
struct TbItem {
    uint32_t cand, pad;
    TbNode<NO> node;
};

// the 32 two-bit groups of x in reverse order
__device__ __forceinline__ uint64_t rev2(uint64_t x) {
    const uint64_t k5 = 0x5555555555555555ull;
    x = __brevll(x);
    return ((x >> 1) & k5) | ((x & k5) << 1);
}

// walk-back ops (2 bits per step: steps 0..31 in a0, 32..63 in a1, 64..79
// in a2) into alignment order: reverse the 96 two-bit groups of
// (a2:a1:a0), which puts step g at group 95 - g, then shift right by
// 2 (96 - n_ops) so that op k = step n_ops - 1 - k lands at group k
__device__ __forceinline__ void ops_forward(uint64_t a0, uint64_t a1, uint32_t a2,
                                            uint32_t n_ops, uint64_t &o0, uint64_t &o1,
                                            uint32_t &o2) {
    const uint64_t r[3] = {rev2((uint64_t)a2), rev2(a1), rev2(a0)};
    const uint32_t sh = 2 * (96 - n_ops), w = sh >> 6, b = sh & 63;  // sh in 48..190
    auto word = [&](uint32_t k) -> uint64_t { return k == 0 ? r[0] : k == 1 ? r[1] : k == 2 ? r[2] : 0; };
    auto out = [&](uint32_t q) -> uint64_t {
        const uint64_t lo = word(w + q), hi = word(w + q + 1);
        return b ? (lo >> b) | (hi << (64 - b)) : lo;
    };
    o0 = out(0);
    o1 = out(1);
    o2 = (uint32_t)out(2);
}

__device__ __forceinline__ uint32_t tb_st(uint32_t i, uint32_t j, uint32_t m, uint32_t d,
                                          uint32_t r) {
    return i | (j << 7) | (m << 14) | (d << 20) | (r << 24);
}

// classify's filter test of a match / substitution cell
__device__ __forceinline__ bool filt_ok(uint8_t fl, uint8_t g) {
    return fl == 0xF ? g != 0 : (g != 0 && g != 0xF && (g & fl));
}

// NW-word bit set shifted toward higher bits by s (1..127), zeros in
template <int NW>
__device__ __forceinline__ void bshl(const uint64_t (&a)[NW], uint32_t s, uint64_t (&o)[NW]) {
    if (NW == 1) {
        o[0] = s < 64 ? a[0] << s : 0;
    } else if (s >= 64) {
        o[NW - 1] = a[0] << (s - 64);
        o[0] = 0;
    } else {
        o[NW - 1] = (a[NW - 1] << s) | (a[0] >> (64 - s));
        o[0] = a[0] << s;
    }
}

// one cell of the budget DP from its three neighbours: diagonal (i-1, j-1),
// up (i-1, j) and left (i, j-1)
template <int NW>
__device__ __forceinline__ void budget_cell(const uint64_t (&dg)[NW], const uint64_t (&up)[NW],
                                            const uint64_t (&lf)[NW], bool diag_ok, uint32_t mc,
                                            bool rna_ok, bool dna_ok, uint32_t T, uint32_t dsh,
                                            const MyersReqDev &R, uint64_t (&v)[NW]) {
#pragma unroll
    for (int w = 0; w < NW; ++w) v[w] = 0;
    if (diag_ok) {
        if (mc) {
            uint64_t x[NW];
            bshl<NW>(dg, 1, x);
#pragma unroll
            for (int w = 0; w < NW; ++w) v[w] = x[w] & R.m_sub[w];
        } else {
#pragma unroll
            for (int w = 0; w < NW; ++w) v[w] = dg[w];
        }
    }
    if (rna_ok) {
        uint64_t x[NW];
        bshl<NW>(up, T, x);
#pragma unroll
        for (int w = 0; w < NW; ++w) v[w] |= x[w] & R.m_rna[w];
    }
    if (dna_ok) {
        uint64_t x[NW];
        bshl<NW>(lf, dsh, x);
#pragma unroll
        for (int w = 0; w < NW; ++w) v[w] |= x[w] & R.m_dna[w];
    }
}

// shared-memory bytes one warp needs: a stack of cap nodes, tables of
// tbl_words 64-bit words, the window text and three pattern arrays
template <int NO>
__host__ __device__ constexpr size_t tb_warp_bytes(uint32_t tbl_words, uint32_t cap) {
    return ((size_t)cap * sizeof(TbNode<NO>) + (size_t)tbl_words * 8 + kTbText + 3 * kTbPat + 15) &
           ~(size_t)15;
}

// kBand: the budget DP comes from the candidate's band table in band_tbl
// (budget_band_kernel<.., true>: band_stride words per candidate of the
// chunk) instead of the wavefront below; a handed-on subtree reloads it.
template <int NW, int NO, bool kBand>
__global__ void __launch_bounds__(kTbWarps * 32, 8)
traceback_warp_kernel(GenomeDev G, const BatchDev *__restrict__ batches,
                      const MyersPattern *__restrict__ pats, const MyersReqDev *__restrict__ reqs,
                      const MyersCand *__restrict__ cand, uint32_t n_cand,
                      const TbItem<NO> *__restrict__ items, uint32_t n_items, TbItem<NO> *spill,
                      uint32_t spill_cap, uint32_t iter_budget, uint32_t tbl_words,
                      uint32_t stk_cap, uint32_t margin, MyersRow *rows, uint32_t row_cap,
                      uint64_t *keys, uint32_t *vals, Counters *ctr, uint32_t *req_rows,
                      const uint64_t *__restrict__ band_tbl, uint32_t band_stride) {
    using Node = TbNode<NO>;
    extern __shared__ __align__(16) unsigned char tb_smem[];
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char *wbase = tb_smem + warp * tb_warp_bytes<NO>(tbl_words, stk_cap);
    Node *stk = reinterpret_cast<Node *>(wbase);
    uint64_t *tbl = reinterpret_cast<uint64_t *>(wbase + stk_cap * sizeof(Node));
    uint8_t *stext = wbase + stk_cap * sizeof(Node) + (size_t)tbl_words * 8;
    uint8_t *spb = stext + kTbText, *sisn = spb + kTbPat, *seff = sisn + kTbPat;
    const unsigned full = 0xFFFFFFFFu;

    const uint32_t n_work = items ? n_items : n_cand;
    for (;;) {
        uint32_t wi = 0;
        if (lane == 0) wi = (uint32_t)min(atomicAdd(&ctr->next_item, 1ull), (unsigned long long)n_work);
        wi = __shfl_sync(full, wi, 0);
        if (wi >= n_work) break;
        __syncwarp();  // the previous item's readers are done
        uint32_t ci = wi;
        Node start_node{};
        if (items) {
            const TbItem<NO> it = items[wi];
            if (it.cand == ~0u) continue;
            ci = it.cand;
            start_node = it.node;
        }
        const MyersCand c = cand[ci];
        const BatchDev B = batches[c.batch];
        const MyersPattern &P = pats[c.pattern];
        const MyersReqDev &R = reqs[P.request];
        const uint32_t L = P.L, t = c.t_local, mm = R.mm, T = R.T;
        const uint32_t n = min(R.W, t + 1);  // text cells of the window
        const uint32_t cols = n + 1;
        const uint32_t rb1 = R.rb + 1, dsh = T * rb1;
        for (uint32_t k = lane; k < n; k += 32) stext[k] = nib(G.bit4, B.base + t + 1 - n + k);
        for (uint32_t k = lane; k < L; k += 32) {
            spb[k] = P.b4[k];
            sisn[k] = P.isn[k];
            seff[k] = P.eff[k];
        }
        const uint32_t bw = R.db + R.rb + 1;               // band cells per row
        const int blo = (int)n - (int)L - (int)R.db;        // j - i of band cell 0
        uint64_t valid[NW];
#pragma unroll
        for (int w = 0; w < NW; ++w) valid[w] = R.m_valid[w];
        if (kBand) {
            const uint64_t *src = band_tbl + (uint64_t)ci * band_stride;
            const uint32_t words = (L + 1) * bw * NW;
            for (uint32_t k = lane; k < words; k += 32) tbl[k] = src[k];
            __syncwarp();
        } else {
            for (uint32_t k = lane; k < cols; k += 32) {  // row 0: F = 0 for every budget
#pragma unroll
                for (int w = 0; w < NW; ++w) tbl[k * NW + w] = valid[w];
            }
            __syncwarp();
        }

        // -- 1. budget DP wavefront, 32 pattern rows per pass
        for (uint32_t r0 = 0; !kBand && r0 < L; r0 += 32) {
            const uint32_t i = r0 + lane + 1;
            const bool row_on = i <= L;
            uint8_t pbi = 0, effi = 0;
            bool isn1 = false, rna_ok = false, dna_ok = false;
            if (row_on) {
                pbi = spb[i - 1];
                effi = seff[i - 1];
                isn1 = sisn[i - 1];
                const bool isn0 = i < L && sisn[i];
                const bool isn2 = i >= 2 && sisn[i - 2];
                rna_ok = R.rb > 0 && !isn1 && !isn0 && !isn2;
                dna_ok = R.db > 0 && i < L && !(isn1 && isn0);
            }
            uint64_t left[NW], upc[NW], upp[NW];
#pragma unroll
            for (int w = 0; w < NW; ++w) left[w] = upc[w] = upp[w] = 0;
            const uint32_t n_rows = min(32u, L - r0);
            for (uint32_t s = 0; s < n_rows + n; ++s) {
#pragma unroll
                for (int w = 0; w < NW; ++w) {
                    uint64_t u = __shfl_up_sync(full, left[w], 1);
                    if (lane == 0)  // row r0, column s: row 0, or the previous pass
                        u = r0 == 0 ? valid[w] : (s <= n ? tbl[(r0 * cols + s) * NW + w] : 0);
                    upp[w] = upc[w];
                    upc[w] = u;
                }
                const int j = (int)s - (int)lane;
                if (row_on && j >= 0 && j <= (int)n) {
                    uint64_t v[NW];
                    const uint8_t tx = j ? stext[j - 1] : 0;
                    if (j == 0) {
                        budget_cell<NW>(upp, upc, left, false, 0, rna_ok, false, T, dsh, R, v);
                    } else if (tx == 0) {  // a node over a padding cell is dead
#pragma unroll
                        for (int w = 0; w < NW; ++w) v[w] = 0;
                    } else {
                        const uint32_t mc = loose(pbi, tx) ? 0u : 1u;
                        const bool dok = !(mc && isn1) && filt_ok(effi, tx);
                        budget_cell<NW>(upp, upc, left, dok, mc, rna_ok, dna_ok, T, dsh, R, v);
                    }
                    uint64_t *cell = tbl + (i * cols + (uint32_t)j) * NW;
#pragma unroll
                    for (int w = 0; w < NW; ++w) {
                        left[w] = v[w];
                        cell[w] = v[w];
                    }
                }
            }
            __syncwarp();
        }
        // F[b](ii, jj) <= mm - m ?
        auto feas = [&](uint32_t ii, uint32_t jj, uint32_t b, uint32_t m) -> bool {
            const uint32_t bit = b * T + (mm - m);
            uint32_t cell = ii * cols + jj;
            if (kBand) {  // a cell off the band lies on no path within the caps
                const int kk = (int)jj - (int)ii - blo;
                if (kk < 0 || kk >= (int)bw) return false;
                cell = ii * bw + (uint32_t)kk;
            }
            return (tbl[cell * NW + (bit >> 6)] >> (bit & 63)) & 1u;
        };
        if (!items) {
            if (!feas(L, n, R.db * rb1 + R.rb, 0)) continue;  // no alignment within the caps
            start_node = Node{};
            start_node.st = tb_st(L, n, 0, 0, 0);
        }
        // every leaf starts in [t + 1 - n, t + 1]: one chunk lookup serves
        // them all unless that range crosses a chunk boundary
        auto chunk_of = [&](uint64_t start) {
            const uint64_t gbyte = start >> 1;
            uint32_t lo = B.first, hi = B.first + B.nch;
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (G.boff[mid] <= gbyte) lo = mid; else hi = mid;
            }
            return lo;
        };
        const uint32_t k_lo = chunk_of(B.base + t + 1 - n), k_hi = chunk_of(B.base + t + 1);

        // -- 2. enumeration
        uint32_t size = 1;
        if (lane == 0) stk[0] = start_node;
        __syncwarp();
        uint32_t iters = 0;
        bool may_spill = iter_budget != 0 && spill != nullptr;
        while (size > 0) {
            if (may_spill && iters >= iter_budget) {
                // hand the rest of this tree to other warps
                uint32_t sb = 0;
                if (lane == 0) sb = atomicAdd(&ctr->hits, size);
                sb = __shfl_sync(full, sb, 0);
                if ((uint64_t)sb + size <= spill_cap) {
                    for (uint32_t q = lane; q < size; q += 32) spill[sb + q] = TbItem<NO>{ci, 0, stk[q]};
                    __syncwarp();
                    break;
                }
                for (uint32_t q = sb + lane; q < spill_cap && q < sb + size; q += 32) spill[q].cand = ~0u;
                may_spill = false;  // queue full: finish the tree here
            }
            ++iters;
            // pop k nodes; with size + 2k <= cap - margin the stack cannot
            // overflow, and below that a one-node walk adds <= margin slots
            const int room = (int)stk_cap - (int)margin - (int)size;
            const uint32_t k = room >= 2 ? min(min(32u, size), (uint32_t)room / 2) : 1u;
            const bool have = lane < k;
            Node nd{};
            if (have) nd = stk[size - 1 - lane];
            size -= k;
            __syncwarp();
            // up to three children (diagonal, RNA, DNA) and two leaves
            // (diagonal or RNA step into row 0), in named slots
            struct Kid { uint32_t st, op; bool on; };
            struct Leaf { uint64_t start, pos; uint32_t chunk, m, d, r, op; bool on; };
            Kid ka{0, 0, false}, kb{0, 0, false}, kc{0, 0, false};
            Leaf la{0, 0, 0, 0, 0, 0, 0, false}, lb{0, 0, 0, 0, 0, 0, 0, false};
            uint32_t dep = 0;
            if (have) {
                const uint32_t st = nd.st;
                const uint32_t ni = st & 127, nj = (st >> 7) & 127, m = (st >> 14) & 63;
                const uint32_t d = (st >> 20) & 15, r = (st >> 24) & 15;
                dep = L - ni + d;
                // convert_matches_myers: owning chunk and record-end drop
                auto leaf = [&](Leaf &o, uint32_t jf, uint32_t lm, uint32_t ld, uint32_t lr,
                                uint32_t op) {
                    const uint64_t start = B.base + t + 1 - (n - jf);
                    const uint32_t lo = k_lo == k_hi ? k_lo : chunk_of(start);
                    const uint64_t pos = G.start[lo] + (start - 2 * G.boff[lo]);
                    const bool end_chrom = (lo == B.first + B.nch - 1) || G.start[lo + 1] == 0;
                    if (end_chrom && pos + (uint64_t)L + ld - lr > G.end[lo]) return;
                    o = Leaf{start, pos, lo, lm, ld, lr, op, true};
                };
                // diagonal: match / substitution
                if (nj >= 1) {
                    const uint8_t tx = stext[nj - 1];
                    const uint32_t mc = loose(spb[ni - 1], tx) ? 0u : 1u;
                    if (!(mc && sisn[ni - 1]) && filt_ok(seff[ni - 1], tx) && m + mc <= mm) {
                        if (ni == 1)
                            leaf(la, nj - 1, m + mc, d, r, mc);
                        else if (feas(ni - 1, nj - 1, (R.db - d) * rb1 + (R.rb - r), m + mc))
                            ka = Kid{tb_st(ni - 1, nj - 1, m + mc, d, r), mc, true};
                    }
                }
                // RNA bulge: pattern cell skipped
                if (r < R.rb) {
                    const bool isn0 = ni < L && sisn[ni], isn2 = ni >= 2 && sisn[ni - 2];
                    if (!sisn[ni - 1] && !isn0 && !isn2) {
                        if (ni == 1)
                            leaf(lb, nj, m, d, r + 1, 3);
                        else if (feas(ni - 1, nj, (R.db - d) * rb1 + (R.rb - r - 1), m))
                            kb = Kid{tb_st(ni - 1, nj, m, d, r + 1), 3, true};
                    }
                }
                // DNA bulge: text cell skipped
                if (d < R.db && nj >= 1 && ni < L && !(sisn[ni - 1] && sisn[ni])) {
                    if (feas(ni, nj - 1, (R.db - d - 1) * rb1 + (R.rb - r), m))
                        kc = Kid{tb_st(ni, nj - 1, m, d + 1, r), 2, true};
                }
            }
            // nd's ops with op at depth dep
            auto ops_with = [&](uint32_t op, Node &o) {
#pragma unroll
                for (int q = 0; q < NO; ++q) o.ops[q] = nd.ops[q];
                o.ops_hi = nd.ops_hi;
                if (dep < 32) o.ops[0] |= (uint64_t)op << (2 * dep);
                else if (NO == 2 && dep < 64) o.ops[NO - 1] |= (uint64_t)op << (2 * (dep - 32));
                else o.ops_hi |= op << (2 * (dep - 32 * NO));
            };
            const uint32_t nc = (uint32_t)ka.on + kb.on + kc.on;
            const uint32_t ne = (uint32_t)la.on + lb.on;
            // push the children
            uint32_t incl = nc;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(full, incl, o);
                if ((int)lane >= o) incl += y;
            }
            const uint32_t tot = __shfl_sync(full, incl, 31);
            uint32_t at = size + incl - nc;
            auto push = [&](const Kid &k2) {
                if (!k2.on) return;
                Node o;
                ops_with(k2.op, o);
                o.st = k2.st;
                stk[at++] = o;
            };
            push(ka);
            push(kb);
            push(kc);
            size += tot;
            // write the rows, one counter update per warp
            uint32_t einc = ne;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(full, einc, o);
                if ((int)lane >= o) einc += y;
            }
            const uint32_t etot = __shfl_sync(full, einc, 31);
            if (etot) {
                uint32_t base = 0;
                if (lane == 0) {
                    base = atomicAdd(&ctr->rows, etot);
                    atomicAdd(&req_rows[P.request], etot);
                }
                base = __shfl_sync(full, base, 0);
                uint32_t rr = base + einc - ne;
                auto put = [&](const Leaf &l2) {
                    if (!l2.on) return;
                    if (rr < row_cap) {
                        Node o;
                        ops_with(l2.op, o);
                        const uint32_t n_ops = dep + 1;
                        MyersRow w;
                        w.start = l2.start;
                        w.pos = l2.pos;
                        // steps 0..31, 32..63, 64..79 of the walk-back ops
                        const uint64_t a1 = NO == 1 ? (uint64_t)o.ops_hi : o.ops[NO - 1];
                        const uint32_t a2 = NO == 1 ? 0u : o.ops_hi;
                        ops_forward(o.ops[0], a1, a2, n_ops, w.ops[0], w.ops[1], w.ops_hi);
                        w.chunk = l2.chunk;
                        w.pattern = c.pattern;
                        w.n_ops = (uint8_t)n_ops;
                        w.mm = (uint8_t)l2.m;
                        w.db = (uint8_t)l2.d;
                        w.rb = (uint8_t)l2.r;
                        rows[rr] = w;
                        keys[rr] = ((uint64_t)c.pattern << G.key_shift) | l2.start;
                        vals[rr] = rr;
                    } else {
                        ctr->overflow = 1;
                    }
                    ++rr;
                };
                put(la);
                put(lb);
            }
            __syncwarp();
        }
    }
}

// traceback_slots_kernel: the band-table traceback with several candidates
// resident in one warp.  traceback_warp_kernel pops up to 32 nodes of one
// tree per step, but a tree's frontier is seldom that wide (every walk
// starts from a single root, and most candidates have a few alignments),
// so about half of its lanes idle.  Here a warp keeps up to n_slots
// candidates loaded -- window text, pattern cells, a context record and
// (unless kGT) the band table per slot, in shared memory -- and their nodes
// share one stack, each node's st carrying its slot in bits 28-31.  A step pops up
// to 32 nodes of any of the trees.  Whenever the stack holds fewer than
// refill_below nodes, free slots take the next candidates (or handed-on
// subtrees) of the work queue (refill_below + n_slots <= kTbSlotSpare keeps
// the roots within the stack's spare slots); a slot is free again once no
// node of its tree is left (a live-node count per slot).  A slot loaded
// iter_budget steps ago hands its remaining nodes to the hand-on queue, as
// traceback_warp_kernel does with its one tree; the other slots' nodes
// stay.  Nodes are expanded, pruned and written as rows exactly as in
// traceback_warp_kernel<.., true>; only the warp step that expands a node
// differs, and the rows are sorted afterwards.
constexpr uint32_t kTbSlotsMax = 8;     // most candidates resident per warp
// the defaults.  Tables copied into the slots: 3 (10 Mbp bulge set, device
// total: 2: 10.38, 3: 9.99, 4: 10.14 with the earlier Myers filter; 3: 8.66
// with the current one).  Band tables read from global memory (through L1
// and L2): 6 (3: 8.75, 4: 8.58, 6: 8.34, 8: 8.55), but a chunk of a large
// set holds gigabytes of tables, far past L2, and the 500 Mbp set's
// traceback took 846 ms against 614 with copied tables.
constexpr uint32_t kTbSlotsGlobal = 6;
constexpr uint32_t kTbSlotsShared = 3;
constexpr uint32_t kTbSlotSpare = 128;  // stack slots beyond the walk margin
constexpr uint32_t kTbRefill = 32;      // refill free slots below this many stacked nodes
constexpr uint32_t kTbSlotBits = 28;    // st bits below the slot index

// one slot's context: the values of its candidate that a node's expansion
// reads (window, pattern and request limits, chunks for the leaf rule)
struct __align__(16) TbSlot {
    uint64_t wstart;           // global nucleotide index of window text cell 0
    uint32_t ci;               // candidate index (hand-on items)
    uint32_t pattern, request;
    uint32_t k_lo, k_hi;       // owning chunks of the window's first and last cell
    uint32_t b_first, b_last;  // the batch's first and last chunk
    uint32_t it0;              // the warp step the slot was loaded at
    uint16_t L, n;             // pattern cells, window text cells
    int16_t blo;               // j - i of band cell 0
    uint8_t mm, T, db, rb, bw, pad;
};

__host__ __device__ constexpr size_t tb_al16(size_t x) { return (x + 15) & ~(size_t)15; }

// byte offsets inside one warp's shared memory: the node stack, the slot
// records, the band tables, the live-node counts, the window texts and the
// pattern arrays (b4, isn, eff: kTbPat bytes each per slot)
struct TbSlotLayout {
    size_t stk, rec, tbl, live, text, pat, total;
};
__host__ __device__ inline TbSlotLayout tb_slot_layout(size_t node_bytes, uint32_t tbl_words,
                                                       uint32_t cap, uint32_t slots) {
    TbSlotLayout o{};
    o.stk = 0;
    o.rec = tb_al16((size_t)cap * node_bytes);
    o.tbl = o.rec + tb_al16((size_t)slots * sizeof(TbSlot));
    o.live = o.tbl + tb_al16((size_t)slots * tbl_words * 8);
    o.text = o.live + tb_al16((size_t)slots * 4);
    o.pat = o.text + tb_al16((size_t)slots * kTbText);
    o.total = o.pat + tb_al16((size_t)slots * 3 * kTbPat);
    return o;
}

// the chunk of batch chunks [first, last] that holds global nucleotide start
__device__ __forceinline__ uint32_t tb_chunk_of(const GenomeDev &G, uint32_t first, uint32_t last,
                                                uint64_t start) {
    const uint64_t gbyte = start >> 1;
    uint32_t lo = first, hi = last + 1;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (G.boff[mid] <= gbyte) lo = mid; else hi = mid;
    }
    return lo;
}

// kGT: the band tables are read where budget_band_kernel<.., true> wrote
// them, in global memory (through L1), instead of being copied into the
// slot; a slot then needs a few hundred bytes, so more slots fit.
template <int NW, int NO, bool kGT>
__global__ void __launch_bounds__(kTbWarps * 32, 6)
traceback_slots_kernel(GenomeDev G, const BatchDev *__restrict__ batches,
                       const MyersPattern *__restrict__ pats, const MyersReqDev *__restrict__ reqs,
                       const MyersCand *__restrict__ cand, uint32_t n_cand,
                       const TbItem<NO> *__restrict__ items, uint32_t n_items, TbItem<NO> *spill,
                       uint32_t spill_cap, uint32_t iter_budget, uint32_t tbl_words,
                       uint32_t stk_cap, uint32_t margin, uint32_t n_slots,
                       uint32_t refill_below, MyersRow *rows,
                       uint32_t row_cap, uint64_t *keys, uint32_t *vals, Counters *ctr,
                       uint32_t *req_rows, const uint64_t *__restrict__ band_tbl,
                       uint32_t band_stride) {
    using Node = TbNode<NO>;
    extern __shared__ __align__(16) unsigned char tb_smem[];
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const TbSlotLayout lay = tb_slot_layout(sizeof(Node), kGT ? 0u : tbl_words, stk_cap, n_slots);
    unsigned char *wbase = tb_smem + warp * lay.total;
    Node *stk = reinterpret_cast<Node *>(wbase + lay.stk);
    TbSlot *srec = reinterpret_cast<TbSlot *>(wbase + lay.rec);
    uint64_t *stbl = reinterpret_cast<uint64_t *>(wbase + lay.tbl);
    int *live = reinterpret_cast<int *>(wbase + lay.live);
    uint8_t *stext = wbase + lay.text;
    uint8_t *spat = wbase + lay.pat;
    const unsigned full = 0xFFFFFFFFu;
    const uint32_t all_slots = (1u << n_slots) - 1u;
    const uint32_t lanes_below = (1u << lane) - 1u;
    const uint32_t n_work = items ? n_items : n_cand;

    // warp-uniform state: nodes on the stack, occupied slots, steps taken
    uint32_t size = 0, used = 0, iters = 0;
    bool drained = false;  // the work queue is exhausted
    bool may_spill = iter_budget != 0 && spill != nullptr;

    // loads work item wi into free slot s and pushes its root; false for
    // an empty hand-on entry or a root with no alignment within the caps
    auto load = [&](uint32_t s, uint32_t wi) -> bool {
        uint32_t ci = wi;
        Node root{};
        if (items) {
            const TbItem<NO> it = items[wi];
            if (it.cand == ~0u) return false;
            ci = it.cand;
            root = it.node;
        }
        const MyersCand c = cand[ci];
        const BatchDev B = batches[c.batch];
        const MyersPattern &P = pats[c.pattern];
        const uint32_t req = P.request;
        const MyersReqDev &R = reqs[req];
        const uint32_t L = P.L, t = c.t_local;
        const uint32_t n = min(R.W, t + 1);
        const uint32_t bw = R.db + R.rb + 1;
        const uint64_t wstart = B.base + t + 1 - n;
        uint8_t *tx = stext + s * kTbText;
        for (uint32_t k = lane; k < n; k += 32) tx[k] = nib(G.bit4, wstart + k);
        uint8_t *pp = spat + s * (3 * kTbPat);
        for (uint32_t k = lane; k < L; k += 32) {
            pp[k] = P.b4[k];
            pp[kTbPat + k] = P.isn[k];
            pp[2 * kTbPat + k] = P.eff[k];
        }
        const uint64_t *src = band_tbl + (uint64_t)ci * band_stride;
        if (!kGT) {
            uint64_t *tbl = stbl + (size_t)s * tbl_words;
            const uint32_t words = (L + 1) * bw * NW;
            for (uint32_t k = lane; k < words; k += 32) tbl[k] = src[k];
        }
        if (lane == 0) {
            TbSlot o;
            o.wstart = wstart;
            o.ci = ci;
            o.pattern = c.pattern;
            o.request = req;
            o.b_first = B.first;
            o.b_last = B.first + B.nch - 1;
            o.k_lo = tb_chunk_of(G, o.b_first, o.b_last, wstart);
            o.k_hi = tb_chunk_of(G, o.b_first, o.b_last, B.base + t + 1);
            o.it0 = iters;
            o.L = (uint16_t)L;
            o.n = (uint16_t)n;
            o.blo = (int16_t)((int)n - (int)L - (int)R.db);
            o.mm = (uint8_t)R.mm;
            o.T = (uint8_t)R.T;
            o.db = (uint8_t)R.db;
            o.rb = (uint8_t)R.rb;
            o.bw = (uint8_t)bw;
            o.pad = 0;
            srec[s] = o;
        }
        __syncwarp();
        if (!items) {
            // the root cell (L, n): full budget at mm; n - L - blo = db
            // is its band cell
            const uint32_t bit = (R.db * (R.rb + 1) + R.rb) * R.T + R.mm;
            const uint32_t at = (L * bw + R.db) * NW + (bit >> 6);
            const uint64_t w = kGT ? src[at] : stbl[(size_t)s * tbl_words + at];
            if (!((w >> (bit & 63)) & 1u)) return false;
            root = Node{};
            root.st = tb_st(L, n, 0, 0, 0);
        }
        if (lane == 0) {
            root.st = (root.st & ((1u << kTbSlotBits) - 1u)) | (s << kTbSlotBits);
            stk[size] = root;
            live[s] = 1;
        }
        ++size;
        return true;
    };

    for (;;) {
        // -- refill: free slots take work while the stack is thin
        if (!drained && size < refill_below && used != all_slots) {
            const uint32_t want = n_slots - __popc(used);
            uint32_t w0 = 0;
            if (lane == 0)
                w0 = (uint32_t)min(atomicAdd(&ctr->next_item, (unsigned long long)want),
                                   (unsigned long long)n_work);
            w0 = __shfl_sync(full, w0, 0);
            const uint32_t got = min(want, n_work - w0);
            if (got < want) drained = true;
            for (uint32_t q = 0; q < got; ++q) {
                const uint32_t s = __ffs(~used & all_slots) - 1;
                if (load(s, w0 + q)) used |= 1u << s;
            }
            __syncwarp();
        }
        if (size == 0) {
            if (drained) break;
            continue;
        }

        // -- one step: pop k nodes (as traceback_warp_kernel: with
        // size + 2k <= cap - margin the stack cannot overflow, and below
        // that a one-node walk adds <= margin slots), expand them
        ++iters;
        const int room = (int)stk_cap - (int)margin - (int)size;
        const uint32_t k = room >= 2 ? min(min(32u, size), (uint32_t)room / 2) : 1u;
        const bool have = lane < k;
        Node nd{};
        if (have) nd = stk[size - 1 - lane];
        size -= k;
        __syncwarp();
        struct Kid { uint32_t st, op; bool on; };
        struct Leaf { uint64_t start, pos; uint32_t chunk, m, d, r, op; bool on; };
        Kid ka{0, 0, false}, kb{0, 0, false}, kc{0, 0, false};
        Leaf la{0, 0, 0, 0, 0, 0, 0, false}, lb{0, 0, 0, 0, 0, 0, 0, false};
        uint32_t dep = 0, s = 0, pattern = 0, req = 0;
        if (have) {
            const uint32_t st = nd.st;
            s = st >> kTbSlotBits;
            const TbSlot &S = srec[s];
            const uint32_t L = S.L, mm = S.mm, T = S.T, db = S.db, rb = S.rb;
            const uint32_t bw = S.bw, rb1 = rb + 1;
            const int blo = S.blo;
            pattern = S.pattern;
            req = S.request;
            const uint8_t *tx = stext + s * kTbText;
            const uint8_t *pb4 = spat + s * (3 * kTbPat), *pisn = pb4 + kTbPat, *peff = pisn + kTbPat;
            const uint64_t *tbl = kGT ? band_tbl + (uint64_t)S.ci * band_stride
                                      : stbl + (size_t)s * tbl_words;
            const uint32_t sbits = s << kTbSlotBits;
            // F[b](ii, jj) <= mm - m ?  (a cell off the band lies on no
            // path within the caps)
            auto feas = [&](uint32_t ii, uint32_t jj, uint32_t b, uint32_t m) -> bool {
                const int kk = (int)jj - (int)ii - blo;
                if (kk < 0 || kk >= (int)bw) return false;
                const uint32_t bit = b * T + (mm - m);
                return (tbl[(ii * bw + (uint32_t)kk) * NW + (bit >> 6)] >> (bit & 63)) & 1u;
            };
            const uint32_t ni = st & 127, nj = (st >> 7) & 127, m = (st >> 14) & 63;
            const uint32_t d = (st >> 20) & 15, r = (st >> 24) & 15;
            dep = L - ni + d;
            // convert_matches_myers: owning chunk and record-end drop
            auto leaf = [&](Leaf &o, uint32_t jf, uint32_t lm, uint32_t ld, uint32_t lr,
                            uint32_t op) {
                const uint64_t start = S.wstart + jf;
                const uint32_t k_lo = S.k_lo, k_hi = S.k_hi;
                const uint32_t lo = k_lo == k_hi ? k_lo : tb_chunk_of(G, S.b_first, S.b_last, start);
                const uint64_t pos = G.start[lo] + (start - 2 * G.boff[lo]);
                const bool end_chrom = (lo == S.b_last) || G.start[lo + 1] == 0;
                if (end_chrom && pos + (uint64_t)L + ld - lr > G.end[lo]) return;
                o = Leaf{start, pos, lo, lm, ld, lr, op, true};
            };
            // diagonal: match / substitution
            if (nj >= 1) {
                const uint8_t t1 = tx[nj - 1];
                const uint32_t mc = loose(pb4[ni - 1], t1) ? 0u : 1u;
                if (!(mc && pisn[ni - 1]) && filt_ok(peff[ni - 1], t1) && m + mc <= mm) {
                    if (ni == 1)
                        leaf(la, nj - 1, m + mc, d, r, mc);
                    else if (feas(ni - 1, nj - 1, (db - d) * rb1 + (rb - r), m + mc))
                        ka = Kid{tb_st(ni - 1, nj - 1, m + mc, d, r) | sbits, mc, true};
                }
            }
            // RNA bulge: pattern cell skipped
            if (r < rb) {
                const bool isn0 = ni < L && pisn[ni], isn2 = ni >= 2 && pisn[ni - 2];
                if (!pisn[ni - 1] && !isn0 && !isn2) {
                    if (ni == 1)
                        leaf(lb, nj, m, d, r + 1, 3);
                    else if (feas(ni - 1, nj, (db - d) * rb1 + (rb - r - 1), m))
                        kb = Kid{tb_st(ni - 1, nj, m, d, r + 1) | sbits, 3, true};
                }
            }
            // DNA bulge: text cell skipped
            if (d < db && nj >= 1 && ni < L && !(pisn[ni - 1] && pisn[ni])) {
                if (feas(ni, nj - 1, (db - d - 1) * rb1 + (rb - r), m))
                    kc = Kid{tb_st(ni, nj - 1, m, d + 1, r) | sbits, 2, true};
            }
        }
        // nd's ops with op at depth dep
        auto ops_with = [&](uint32_t op, Node &o) {
#pragma unroll
            for (int q = 0; q < NO; ++q) o.ops[q] = nd.ops[q];
            o.ops_hi = nd.ops_hi;
            if (dep < 32) o.ops[0] |= (uint64_t)op << (2 * dep);
            else if (NO == 2 && dep < 64) o.ops[NO - 1] |= (uint64_t)op << (2 * (dep - 32));
            else o.ops_hi |= op << (2 * (dep - 32 * NO));
        };
        const uint32_t nc = (uint32_t)ka.on + kb.on + kc.on;
        const uint32_t ne = (uint32_t)la.on + lb.on;
        // push the children
        uint32_t incl = nc;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(full, incl, o);
            if ((int)lane >= o) incl += y;
        }
        const uint32_t tot = __shfl_sync(full, incl, 31);
        uint32_t at = size + incl - nc;
        auto push = [&](const Kid &k2) {
            if (!k2.on) return;
            Node o;
            ops_with(k2.op, o);
            o.st = k2.st;
            stk[at++] = o;
        };
        push(ka);
        push(kb);
        push(kc);
        size += tot;
        if (have) atomicAdd(&live[s], (int)nc - 1);
        // write the rows: one row-counter update per warp, one request
        // count per warp when every writing lane has the same request
        uint32_t einc = ne;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(full, einc, o);
            if ((int)lane >= o) einc += y;
        }
        const uint32_t etot = __shfl_sync(full, einc, 31);
        if (etot) {
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(&ctr->rows, etot);
            base = __shfl_sync(full, base, 0);
            const uint32_t writers = __ballot_sync(full, ne != 0);
            const uint32_t req0 = __shfl_sync(full, req, __ffs(writers) - 1);
            if (__all_sync(full, ne == 0 || req == req0)) {
                if (lane == 0) atomicAdd(&req_rows[req0], etot);
            } else if (ne) {
                atomicAdd(&req_rows[req], ne);
            }
            uint32_t rr = base + einc - ne;
            auto put = [&](const Leaf &l2) {
                if (!l2.on) return;
                if (rr < row_cap) {
                    Node o;
                    ops_with(l2.op, o);
                    const uint32_t n_ops = dep + 1;
                    MyersRow w;
                    w.start = l2.start;
                    w.pos = l2.pos;
                    // steps 0..31, 32..63, 64..79 of the walk-back ops
                    const uint64_t a1 = NO == 1 ? (uint64_t)o.ops_hi : o.ops[NO - 1];
                    const uint32_t a2 = NO == 1 ? 0u : o.ops_hi;
                    ops_forward(o.ops[0], a1, a2, n_ops, w.ops[0], w.ops[1], w.ops_hi);
                    w.chunk = l2.chunk;
                    w.pattern = pattern;
                    w.n_ops = (uint8_t)n_ops;
                    w.mm = (uint8_t)l2.m;
                    w.db = (uint8_t)l2.d;
                    w.rb = (uint8_t)l2.r;
                    rows[rr] = w;
                    keys[rr] = ((uint64_t)pattern << G.key_shift) | l2.start;
                    vals[rr] = rr;
                } else {
                    ctr->overflow = 1;
                }
                ++rr;
            };
            put(la);
            put(lb);
        }
        __syncwarp();

        // -- slots whose trees are done are free again
        const bool mine = lane < n_slots && ((used >> lane) & 1u);
        const uint32_t done = __ballot_sync(full, mine && live[lane] == 0);
        used &= ~done;
        if (!may_spill) continue;
        // -- slots loaded iter_budget steps ago hand their nodes on
        const uint32_t over = __ballot_sync(
            full, mine && !((done >> lane) & 1u) && iters - srec[lane].it0 >= iter_budget);
        if (!over) continue;
        const uint32_t cnt = __reduce_add_sync(full, ((over >> lane) & 1u) ? (uint32_t)live[lane] : 0u);
        uint32_t sb = 0;
        if (lane == 0) sb = atomicAdd(&ctr->hits, cnt);
        sb = __shfl_sync(full, sb, 0);
        if ((uint64_t)sb + cnt <= spill_cap) {
            // compact the stack in place: the handed-on nodes go to the
            // queue, the others keep their order (a chunk is read before
            // any of it is overwritten, and writes land at or below it)
            uint32_t kept = 0, sent = 0;
            for (uint32_t b0 = 0; b0 < size; b0 += 32) {
                const uint32_t idx = b0 + lane;
                const bool in = idx < size;
                Node x{};
                if (in) x = stk[idx];
                const bool go = in && ((over >> (x.st >> kTbSlotBits)) & 1u);
                const bool keep = in && !go;
                const uint32_t gm = __ballot_sync(full, go), km = __ballot_sync(full, keep);
                __syncwarp();
                // (the live counts make exactly cnt such nodes; the bound
                // keeps the writes inside the reserved entries regardless)
                const uint32_t q = sent + __popc(gm & lanes_below);
                if (go && q < cnt) {
                    TbItem<NO> it;
                    it.cand = srec[x.st >> kTbSlotBits].ci;
                    it.pad = 0;
                    it.node = x;
                    it.node.st &= (1u << kTbSlotBits) - 1u;
                    spill[sb + q] = it;
                }
                if (keep) stk[kept + __popc(km & lanes_below)] = x;
                sent += __popc(gm);
                kept += __popc(km);
                __syncwarp();
            }
            size = kept;
            used &= ~over;
            if ((over >> lane) & 1u) live[lane] = 0;
        } else {
            for (uint32_t q = sb + lane; q < spill_cap && q < sb + cnt; q += 32) spill[q].cand = ~0u;
            may_spill = false;  // queue full: this warp finishes its trees
        }
        __syncwarp();
    }
}

// Exact pre-test of the warp traceback, one thread per candidate: the
// budget DP row by row (pattern cell i) with the previous row kept in
// shared memory, interleaved by thread so that a warp's accesses hit
// different banks, and only the root cell's full-budget bit at mm tested.
// Every alignment path crosses every row, and a smaller budget never needs
// fewer mismatches, so the root can only be feasible if some cell of every
// row has a full-budget bit at mm: a row without one ends the test early.
// Most candidates the Myers bound lets through fail here; only the others
// are passed on.
constexpr int kBfThreads = 128;

// TW: 64-bit words of window text, 16 cells each (3: windows of <= 48
// cells, 5: <= 80)
template <int NW, int TW>
__global__ void __launch_bounds__(kBfThreads)
budget_filter_kernel(GenomeDev G, const BatchDev *__restrict__ batches,
                     const MyersPattern *__restrict__ pats, const MyersReqDev *__restrict__ reqs,
                     const MyersCand *__restrict__ cand, uint32_t n_cand,
                     MyersCand *__restrict__ out, uint32_t *n_out) {
    extern __shared__ uint64_t bf_row[];  // [cell * NW + w][thread], cells 0..n
    const uint32_t tid = threadIdx.x;
    auto Rw = [&](uint32_t j, int w) -> uint64_t & {
        return bf_row[(j * NW + w) * kBfThreads + tid];
    };
    for (uint32_t base = blockIdx.x * kBfThreads; base < n_cand; base += gridDim.x * kBfThreads) {
        const uint32_t ci = base + tid;
        bool keep = false;
        MyersCand c{0, 0, 0, 0};
        if (ci < n_cand) {
            c = cand[ci];
            const BatchDev B = batches[c.batch];
            const MyersPattern &P = pats[c.pattern];
            const MyersReqDev &R = reqs[P.request];
            const uint32_t L = P.L, t = c.t_local, T = R.T;
            const uint32_t n = min(R.W, t + 1);
            const uint32_t dsh = T * (R.rb + 1);
            const uint32_t top = ((R.db + 1) * (R.rb + 1) - 1) * T + R.mm;  // root bit
            uint64_t fullg[NW], valid[NW];
#pragma unroll
            for (int w = 0; w < NW; ++w) {
                fullg[w] = R.m_full[w];
                valid[w] = R.m_valid[w];
            }
            // the window's n text cells, cell k in bits 4 (k % 16) of word k / 16
            // of (tw4:tw3:tw2:tw1:tw0)
            const uint64_t tbase = B.base + t + 1 - n;
            uint64_t tw0 = 0, tw1 = 0, tw2 = 0, tw3 = 0, tw4 = 0;
            for (uint32_t k = 0; k < n; ++k) {
                const uint64_t x = (uint64_t)nib(G.bit4, tbase + k) << (4 * (k & 15));
                if (k < 16) tw0 |= x;
                else if (k < 32) tw1 |= x;
                else if (TW == 3 || k < 48) tw2 |= x;
                else if (k < 64) tw3 |= x;
                else tw4 |= x;
            }
            for (uint32_t j = 0; j <= n; ++j) {
#pragma unroll
                for (int w = 0; w < NW; ++w) Rw(j, w) = valid[w];  // row 0
            }
            keep = true;
            for (uint32_t i = 1; i <= L && keep; ++i) {
                const uint8_t pb = P.b4[i - 1], ef = P.eff[i - 1];
                const bool isn1 = P.isn[i - 1], isn0 = i < L && P.isn[i],
                           isn2 = i >= 2 && P.isn[i - 2];
                const bool rna_ok = R.rb > 0 && !isn1 && !isn0 && !isn2;
                const bool dna_ok = R.db > 0 && i < L && !(isn1 && isn0);
                uint64_t dsrc[NW], left[NW], v[NW], up[NW];
                // column 0: only an RNA bulge from the cell above
#pragma unroll
                for (int w = 0; w < NW; ++w) dsrc[w] = Rw(0, w);
                budget_cell<NW>(dsrc, dsrc, dsrc, false, 0, rna_ok, false, T, dsh, R, left);
                uint64_t row_or = 0;
#pragma unroll
                for (int w = 0; w < NW; ++w) {
                    Rw(0, w) = left[w];
                    row_or |= left[w] & fullg[w];
                }
                uint64_t a0 = tw0, a1 = tw1, a2 = tw2, a3 = tw3, a4 = tw4;  // text shift register
                for (uint32_t j = 1; j <= n; ++j) {
                    const uint8_t tx = (uint8_t)(a0 & 0xF);
                    a0 = (a0 >> 4) | (a1 << 60);
                    a1 = (a1 >> 4) | (a2 << 60);
                    if (TW == 3) {
                        a2 >>= 4;
                    } else {
                        a2 = (a2 >> 4) | (a3 << 60);
                        a3 = (a3 >> 4) | (a4 << 60);
                        a4 >>= 4;
                    }
#pragma unroll
                    for (int w = 0; w < NW; ++w) up[w] = Rw(j, w);
                    if (tx == 0) {  // a node over a padding cell is dead
#pragma unroll
                        for (int w = 0; w < NW; ++w) v[w] = 0;
                    } else {
                        const uint32_t mc = loose(pb, tx) ? 0u : 1u;
                        const bool dok = !(mc && isn1) && filt_ok(ef, tx);
                        budget_cell<NW>(dsrc, up, left, dok, mc, rna_ok, dna_ok, T, dsh, R, v);
                    }
#pragma unroll
                    for (int w = 0; w < NW; ++w) {
                        Rw(j, w) = v[w];
                        dsrc[w] = up[w];
                        left[w] = v[w];
                        row_or |= v[w] & fullg[w];
                    }
                }
                if (!row_or) keep = false;
            }
            if (keep) keep = (Rw(n, (int)(top >> 6)) >> (top & 63)) & 1u;
        }
        // warp-aggregated compaction of the survivors
        const unsigned full = 0xFFFFFFFFu;
        const unsigned m = __ballot_sync(full, keep);
        const uint32_t lane = tid & 31;
        uint32_t o = 0;
        if (lane == 0 && m) o = atomicAdd(n_out, (uint32_t)__popc(m));
        o = __shfl_sync(full, o, 0);
        if (keep) out[o + __popc(m & ((1u << lane) - 1u))] = c;
    }
}

// The budget pre-test on the band of the DP that alignments within the caps
// can touch.  A path from the root (L, n) back to row 0 changes its
// diagonal j - i by +1 per RNA bulge and -1 per DNA bulge, so every cell of
// an alignment with at most db DNA and rb RNA bulges has
// n - L - db <= j - i <= n - L + rb: db + rb + 1 cells per row (5 of the
// 26 at L = 23, db = rb = 2).  Cells outside the band lie on no such path;
// taking them as dead changes no value that a path within the caps reads,
// so the test is exact and does a fifth of the work.  kBandMax: widest
// band (db + rb + 1) this kernel takes.
constexpr uint32_t kBandMax = 16;

//
// kTable: the same band DP for candidates known to pass (the traceback's
// survivors), without the early exit, writing every row's band cells to the
// candidate's table in tbl (tbl_stride words per candidate:
// [(i * band + k) * NW + w]); the traceback then reads the table instead of
// computing the DP again.
template <int NW, int TW, bool kTable>
__global__ void __launch_bounds__(kBfThreads)
budget_band_kernel(GenomeDev G, const BatchDev *__restrict__ batches,
                   const MyersPattern *__restrict__ pats, const MyersReqDev *__restrict__ reqs,
                   const MyersCand *__restrict__ cand, uint32_t n_cand,
                   MyersCand *__restrict__ out, uint32_t *n_out, uint64_t *__restrict__ tbl,
                   uint32_t tbl_stride) {
    extern __shared__ uint64_t bb_row[];  // [band cell * NW + w][thread]
    const uint32_t tid = threadIdx.x;
    auto Rw = [&](uint32_t k, int w) -> uint64_t & {
        return bb_row[(k * NW + w) * kBfThreads + tid];
    };
    for (uint32_t base = blockIdx.x * kBfThreads; base < n_cand; base += gridDim.x * kBfThreads) {
        const uint32_t ci = base + tid;
        bool keep = false;
        MyersCand c{0, 0, 0, 0};
        if (ci < n_cand) {
            c = cand[ci];
            const BatchDev B = batches[c.batch];
            const MyersPattern &P = pats[c.pattern];
            const MyersReqDev &R = reqs[P.request];
            const uint32_t L = P.L, t = c.t_local, T = R.T;
            const uint32_t n = min(R.W, t + 1);
            const uint32_t dsh = T * (R.rb + 1);
            const uint32_t top = ((R.db + 1) * (R.rb + 1) - 1) * T + R.mm;  // root bit
            const uint32_t bw = R.db + R.rb + 1;                         // band width
            const int lo = (int)n - (int)L - (int)R.db;                  // j - i of band cell 0
            uint64_t fullg[NW], valid[NW];
#pragma unroll
            for (int w = 0; w < NW; ++w) {
                fullg[w] = R.m_full[w];
                valid[w] = R.m_valid[w];
            }
            // the window's n text cells, cell k in bits 4 (k % 16) of word
            // k / 16 (cells from n on 0), from aligned 16-cell genome words
            // (the buffer is padded past the last cell by more than a word)
            const uint64_t tbase = B.base + t + 1 - n;
            const unsigned long long *gwp = reinterpret_cast<const unsigned long long *>(G.bit4);
            const uint64_t q0 = tbase >> 4;
            const uint32_t sh = 4 * (uint32_t)(tbase & 15);
            uint64_t tw[TW];
            {
                uint64_t a = __ldg(gwp + q0);
#pragma unroll
                for (int q = 0; q < TW; ++q) {
                    uint64_t x = 0;
                    if (16u * q < n) {
                        const uint64_t b = __ldg(gwp + q0 + q + 1);
                        x = sh ? (a >> sh) | (b << (64 - sh)) : a;
                        a = b;
                        if (16u * (q + 1) > n) x &= (1ull << (4 * (n - 16u * q))) - 1ull;
                    }
                    tw[q] = x;
                }
            }
            const uint64_t tw0 = tw[0], tw1 = tw[1], tw2 = tw[2];
            const uint64_t tw3 = TW == 5 ? tw[TW == 5 ? 3 : 0] : 0ull;
            const uint64_t tw4 = TW == 5 ? tw[TW == 5 ? 4 : 0] : 0ull;
            auto word = [&](int q) -> uint64_t {
                return q == 0 ? tw0 : q == 1 ? tw1 : q == 2 ? tw2
                     : (TW == 5 && q == 3) ? tw3 : (TW == 5 && q == 4) ? tw4 : 0ull;
            };
            // 16 text cells from cell cs on (cells below 0 read 0)
            auto text16 = [&](int cs) -> uint64_t {
                if (cs < 0) return cs <= -16 ? 0ull : tw0 << (4 * -cs);
                const int q = cs >> 4, b = 4 * (cs & 15);
                const uint64_t a = word(q), h = word(q + 1);
                return b ? (a >> b) | (h << (64 - b)) : a;
            };
            uint64_t *tb = kTable ? tbl + (uint64_t)ci * tbl_stride : nullptr;
            for (uint32_t k = 0; k < bw; ++k) {  // row 0: F = 0 for every budget
                const int j = lo + (int)k;
#pragma unroll
                for (int w = 0; w < NW; ++w) {
                    Rw(k, w) = (j >= 0 && j <= (int)n) ? valid[w] : 0;
                    if (kTable) tb[k * NW + w] = Rw(k, w);
                }
            }
            keep = true;
            for (uint32_t i = 1; i <= L && (kTable || keep); ++i) {
                const uint8_t pb = P.b4[i - 1], ef = P.eff[i - 1];
                const bool isn1 = P.isn[i - 1], isn0 = i < L && P.isn[i],
                           isn2 = i >= 2 && P.isn[i - 2];
                const bool rna_ok = R.rb > 0 && !isn1 && !isn0 && !isn2;
                const bool dna_ok = R.db > 0 && i < L && !(isn1 && isn0);
                const int j0 = (int)i + lo;                   // column of band cell 0
                const uint64_t tx16 = text16(j0 - 1);          // text cells j - 1
                uint64_t left[NW], row_or = 0;
#pragma unroll
                for (int w = 0; w < NW; ++w) left[w] = 0;
                for (uint32_t k = 0; k < bw; ++k) {
                    const int j = j0 + (int)k;
                    uint64_t dg[NW], up[NW], v[NW];
#pragma unroll
                    for (int w = 0; w < NW; ++w) {
                        dg[w] = Rw(k, w);                          // (i - 1, j - 1)
                        up[w] = k + 1 < bw ? Rw(k + 1, w) : 0ull;  // (i - 1, j)
                        v[w] = 0;
                    }
                    if (j == 0) {  // column 0: only an RNA bulge from the cell above
                        budget_cell<NW>(up, up, up, false, 0, rna_ok, false, T, dsh, R, v);
                    } else if (j > 0 && j <= (int)n) {
                        const uint8_t tx = (uint8_t)((tx16 >> (4 * k)) & 0xF);
                        if (tx != 0) {  // a node over a padding cell is dead
                            const uint32_t mc = loose(pb, tx) ? 0u : 1u;
                            const bool dok = !(mc && isn1) && filt_ok(ef, tx);
                            budget_cell<NW>(dg, up, left, dok, mc, rna_ok, dna_ok, T, dsh, R, v);
                        }
                    }
#pragma unroll
                    for (int w = 0; w < NW; ++w) {
                        Rw(k, w) = v[w];
                        left[w] = v[w];
                        row_or |= v[w] & fullg[w];
                        if (kTable) tb[(i * bw + k) * NW + w] = v[w];
                    }
                }
                if (!row_or) keep = false;
            }
            // the root (L, n) is band cell db
            if (keep) keep = (Rw(R.db, (int)(top >> 6)) >> (top & 63)) & 1u;
        }
        if (kTable) continue;
        const unsigned full = 0xFFFFFFFFu;
        const unsigned m = __ballot_sync(full, keep);
        const uint32_t lane = tid & 31;
        uint32_t o = 0;
        if (lane == 0 && m) o = atomicAdd(n_out, (uint32_t)__popc(m));
        o = __shfl_sync(full, o, 0);
        if (keep) out[o + __popc(m & ((1u << lane) - 1u))] = c;
    }
}

__device__ __forceinline__ uint64_t mpos_out(const MyersRow &w, const MyersReqDev &R,
                                             uint32_t strand) {
    if (!strand) return w.pos;
    const uint64_t a = R.pam_len ? R.pam_len - 1 : 0;
    return w.pos + (a > w.db ? a - w.db : 0);
}

__global__ void mrow_len_kernel(GenomeDev G, const MyersRow *__restrict__ rows,
                                const uint32_t *__restrict__ order, uint32_t n,
                                const MyersPattern *__restrict__ pats,
                                const MyersReqDev *__restrict__ reqs, uint32_t *__restrict__ len) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const MyersRow w = rows[order[i]];
        const MyersPattern &P = pats[w.pattern];
        const MyersReqDev R = reqs[P.request];
        const uint32_t ni = G.name_idx[w.chunk];
        const uint32_t name_len = G.name_off[ni + 1] - G.name_off[ni];
        const uint32_t size = w.db + w.rb;
        if (R.raw) {  // name pos pidx dir mm db rb rna dna
            len[i] = name_len + 1 + ndigits(w.pos) + 1 + ndigits(w.pattern - R.first_pattern) + 3 +
                     ndigits(w.mm) + 1 + ndigits(w.db) + 1 + ndigits(w.rb) + 1 + w.n_ops + 1 +
                     w.n_ops + 1;
            continue;
        }
        const uint32_t tlen = size == 0 ? 1 : 3;
        len[i] = tlen + 1 + w.n_ops + 1 + w.n_ops + 1 + name_len + 1 +
                 ndigits(mpos_out(w, R, P.strand)) + 3 + ndigits(w.mm) + 1 + ndigits(size) + 1;
    }
}

constexpr uint32_t kRowStage = 4096;  // staged text bytes per warp

__global__ void __launch_bounds__(256)
mrow_write_kernel(GenomeDev G, const MyersRow *__restrict__ rows,
                  const uint32_t *__restrict__ order, uint32_t n,
                  const MyersPattern *__restrict__ pats, const MyersReqDev *__restrict__ reqs,
                  const uint64_t *__restrict__ off, char *__restrict__ text) {
    __shared__ __align__(16) char stage_all[8][kRowStage];
    char *stage = stage_all[threadIdx.x >> 5];
    const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i0 = gw * 32; i0 < n; i0 += nw * 32) {
        warp_rows_staged((uint32_t)i0, n, off, text, stage, kRowStage, [&](uint32_t i, char *o) {
            const MyersRow w = rows[order[i]];
            const MyersPattern &P = pats[w.pattern];
            const MyersReqDev R = reqs[P.request];
            const bool fwd = P.strand == 0;
            const uint32_t size = w.db + w.rb;
            const uint32_t ni = G.name_idx[w.chunk];
            if (R.raw) {  // search()'s Match: name, chrom_idx, pattern, strand, mm, db, rb
                for (uint32_t c = G.name_off[ni]; c < G.name_off[ni + 1]; ++c) *o++ = G.names[c];
                *o++ = '\t';
                o = put_u64(o, w.pos);
                *o++ = '\t';
                o = put_u64(o, w.pattern - R.first_pattern);
                *o++ = '\t';
                *o++ = fwd ? '+' : '-';
                *o++ = '\t';
                o = put_u64(o, w.mm);
                *o++ = '\t';
                o = put_u64(o, w.db);
                *o++ = '\t';
                o = put_u64(o, w.rb);
                *o++ = '\t';
            } else if (size == 0) {
                *o++ = 'X';
            } else if (w.db > 0) {
                *o++ = 'D'; *o++ = 'N'; *o++ = 'A';
            } else {
                *o++ = 'R'; *o++ = 'N'; *o++ = 'A';
            }
            if (!R.raw) *o++ = '\t';
            const uint32_t no = w.n_ops;
            char *rna = o;
            char *dna = o + no + 1;
            // aligned strings in alignment order (traceback.rs:267-298), then
            // reverse-complemented for reverse-strand patterns
            uint32_t pi = 0;
            // genome cells from w.start on, through a 16-cell word cursor
            // (the buffer is padded past the last cell by more than a word)
            const unsigned long long *gwords = reinterpret_cast<const unsigned long long *>(G.bit4);
            uint64_t gi = w.start;
            unsigned long long gword = __ldg(gwords + (gi >> 4));
            auto gnext = [&]() -> uint8_t {
                const uint8_t v = (uint8_t)((gword >> (4 * (gi & 15))) & 0xF);
                if ((++gi & 15) == 0) gword = __ldg(gwords + (gi >> 4));
                return v;
            };
            for (uint32_t k = 0; k < no; ++k) {
                const uint32_t op = mrow_op(w, k);
                uint8_t pv = 0, gv = 0;
                bool pgap = false, ggap = false;
                if (op <= 1) {
                    pv = P.b4[pi++];
                    gv = gnext();
                } else if (op == 2) {
                    pgap = true;
                    gv = gnext();
                } else {
                    pv = P.b4[pi++];
                    ggap = true;
                }
                const uint32_t at = fwd ? k : no - 1 - k;
                if (!fwd) {
                    pv = dcomp4(pv);
                    gv = dcomp4(gv);
                }
                rna[at] = pgap ? '-' : b4char(pv);
                dna[at] = ggap ? '-' : b4char(gv);
            }
            o += no;
            *o++ = '\t';
            o += no;
            if (R.raw) {
                *o++ = '\n';
                return;
            }
            *o++ = '\t';
            for (uint32_t c = G.name_off[ni]; c < G.name_off[ni + 1]; ++c) *o++ = G.names[c];
            *o++ = '\t';
            o = put_u64(o, mpos_out(w, R, P.strand));
            *o++ = '\t';
            *o++ = fwd ? '+' : '-';
            *o++ = '\t';
            o = put_u64(o, w.mm);
            *o++ = '\t';
            o = put_u64(o, size);
            *o++ = '\n';

        });
    }
}

// One launch of the warp traceback; the work queues are untyped here
// because the node width is a template parameter.
// Match records of formatted alignment rows, in text order: the fields of
// search()'s Match (chrom_chunk.rs:19-29) and the offset of the row's line
// in its piece, which holds one request's rows from row req_first[request].
__global__ void mrow_rec_kernel(GenomeDev G, const MyersRow *__restrict__ rows,
                                const uint32_t *__restrict__ order, uint32_t n,
                                const MyersPattern *__restrict__ pats,
                                const MyersReqDev *__restrict__ reqs,
                                const uint64_t *__restrict__ off,
                                const uint32_t *__restrict__ req_first,
                                MatchRec *__restrict__ recs) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const MyersRow w = rows[order[i]];
        const MyersPattern &P = pats[w.pattern];
        MatchRec m{};
        m.chrom_idx = w.pos;
        m.text_offset = off[i] - off[req_first[P.request]];
        m.record = G.name_idx[w.chunk];
        m.pattern_idx = w.pattern - reqs[P.request].first_pattern;
        m.mismatches = w.mm;
        m.dna_bulge_size = w.db;
        m.rna_bulge_size = w.rb;
        m.is_forward = P.strand == 0;
        recs[i] = m;
    }
}

struct TbLaunch {
    unsigned grid, threads;
    size_t smem;
    cudaStream_t s;
    GenomeDev G;
    const BatchDev *batches;
    const MyersPattern *pats;
    const MyersReqDev *reqs;
    const MyersCand *cand;
    uint32_t n_cand;
    const char *items;
    uint32_t n_items;
    char *spill;
    uint32_t spill_cap, iter_budget, tbl_words, stk_cap, margin;
    MyersRow *rows;
    uint32_t row_cap;
    uint64_t *keys;
    uint32_t *vals;
    Counters *ctr;
    uint32_t *req_rows;
    const uint64_t *band_tbl;  // the chunk's band tables (kBand)
    uint32_t band_stride;
    uint32_t n_slots;          // candidates resident per warp (0: one tree per warp)
    uint32_t refill_below;     // free slots take work while the stack holds fewer nodes
};

template <int NW, int NO, bool kBand>
void launch_tb(const TbLaunch &a) {
    traceback_warp_kernel<NW, NO, kBand><<<a.grid, a.threads, a.smem, a.s>>>(
        a.G, a.batches, a.pats, a.reqs, a.cand, a.n_cand,
        reinterpret_cast<const TbItem<NO> *>(a.items), a.n_items,
        reinterpret_cast<TbItem<NO> *>(a.spill), a.spill_cap, a.iter_budget, a.tbl_words,
        a.stk_cap, a.margin, a.rows, a.row_cap, a.keys, a.vals, a.ctr, a.req_rows, a.band_tbl,
        a.band_stride);
}

template <int NW, int NO, bool kGT>
void launch_tb_slots(const TbLaunch &a) {
    traceback_slots_kernel<NW, NO, kGT><<<a.grid, a.threads, a.smem, a.s>>>(
        a.G, a.batches, a.pats, a.reqs, a.cand, a.n_cand,
        reinterpret_cast<const TbItem<NO> *>(a.items), a.n_items,
        reinterpret_cast<TbItem<NO> *>(a.spill), a.spill_cap, a.iter_budget, a.tbl_words,
        a.stk_cap, a.margin, a.n_slots, a.refill_below, a.rows, a.row_cap, a.keys, a.vals, a.ctr,
        a.req_rows,
        a.band_tbl, a.band_stride);
}

// Myers Eq table of one pattern (build_peq, myers.rs:32-50, and the eq rule
// of search.rs:846-858): nibble 0 -> 0, 0xF -> peq_n, else OR of the peqs of
// its set bits (A=4, C=2, G=8, T=1).
// Patterns of up to 64 cells: the low 32 bits go to eq_lo, the rest to eq_hi.
void build_eq16(const std::string &p, uint32_t eq_lo[16], uint32_t eq_hi[16]) {
    uint64_t peq[4] = {0, 0, 0, 0}, peq_n = 0;
    for (size_t i = 0; i < p.size(); ++i) {
        const char u = (char)((p[i] >= 'a' && p[i] <= 'z') ? p[i] - 32 : p[i]);
        const int idx = u == 'A' ? 0 : u == 'C' ? 1 : u == 'G' ? 2 : u == 'T' ? 3 : 4;
        if (idx < 4) {
            peq[idx] |= 1ull << i;
        } else {
            for (int k = 0; k < 4; ++k) peq[k] |= 1ull << i;
            peq_n |= 1ull << i;
        }
    }
    for (int b = 0; b < 16; ++b) {
        uint64_t e = 0;
        if (b == 15) e = peq_n;
        else {
            if (b & 4) e |= peq[0];
            if (b & 2) e |= peq[1];
            if (b & 8) e |= peq[2];
            if (b & 1) e |= peq[3];
        }
        eq_lo[b] = (uint32_t)e;
        eq_hi[b] = (uint32_t)(e >> 32);
    }
}

}  // namespace

int Engine::run_bulge(const std::vector<Request> &reqs, std::vector<Result> &out, Error &err,
                      const Sink *sink, const SearchRange &range) {
    DeviceGenome &d = *dev_;
    const HostGenome &h = host_;
    const Bit4Tables &t = bit4();
    cudaStream_t s = d.stream;
    out.clear();
    out.resize(reqs.size());

    const auto hb = make_batches(h.n_chunks(), reqs[0].cps);
    std::vector<BatchDev> batches;
    std::vector<MyersTile> tiles;
    for (size_t bi = 0; bi < hb.size(); ++bi) {
        const HostBatch &b = hb[bi];
        BatchDev x{};
        x.base = 2 * h.boff[b.first];
        x.valid = (uint32_t)(2 * (h.boff[b.last + 1] - h.boff[b.first]));
        x.first = (uint32_t)b.first;
        x.nch = (uint32_t)(b.last - b.first + 1);
        x.active_start = b.has_head ? (uint32_t)(2 * (h.boff[b.first + 1] - h.boff[b.first])) : 0;
        batches.push_back(x);
        // active end positions (search.rs:913-927, :1087-1092) inside the
        // searched range
        const uint64_t e_lo = std::max(x.base + x.active_start, range.lo);
        const uint64_t e_hi = std::min<uint64_t>(x.base + x.valid, range.hi);
        for (uint64_t a = e_lo; a < e_hi; a += kTile)
            tiles.push_back(MyersTile{a, std::min<uint64_t>(a + kTile, e_hi), (uint32_t)bi, 0, 0});
    }
    std::vector<MyersReqDev> rdev;
    std::vector<MyersPattern> pats;
    std::vector<PamForm> forms;
    for (size_t ri = 0; ri < reqs.size(); ++ri) {
        const Request &r = reqs[ri];
        const uint32_t L = (uint32_t)r.filter.size();
        MyersReqDev rd;
        std::memset(&rd, 0, sizeof rd);
        rd.L = L;
        rd.mm = r.max_mm;
        rd.db = r.max_db;
        rd.rb = r.max_rb;
        rd.E = r.max_mm + r.max_db + r.max_rb;
        rd.W = L + r.max_db;
        rd.pam_len = (uint32_t)r.pam_len;
        rd.raw = r.raw ? 1u : 0u;
        rd.first_pattern = (uint32_t)pats.size();
        // budget DP bit sets: bit b * T + v, b = bd * (rb + 1) + br
        rd.T = rd.mm + 1;
        const uint32_t nbud = (rd.db + 1) * (rd.rb + 1);
        rd.nbits = nbud * rd.T;
        auto setb = [](uint64_t(&m)[2], uint32_t bit) {
            if (bit < 128) m[bit >> 6] |= 1ull << (bit & 63);
        };
        for (uint32_t b = 0; b < nbud; ++b) {
            for (uint32_t v = 0; v < rd.T; ++v) {
                const uint32_t bit = b * rd.T + v;
                setb(rd.m_valid, bit);
                if (v >= 1) setb(rd.m_sub, bit);
                if (b % (rd.rb + 1) >= 1) setb(rd.m_rna, bit);
                if (b / (rd.rb + 1) >= 1) setb(rd.m_dna, bit);
                if (b == nbud - 1) setb(rd.m_full, bit);
            }
        }
        if (rd.L > 64 || rd.W > (uint32_t)kMaxCells) {
            err = {kUnsupported, "bulge search needs pattern length <= 64 and length + max_dna_bulges <= 72"};
            return err.code;
        }
        rdev.push_back(rd);
        std::string rf = r.filter;  // reverse_compliment_char of the filter
        for (char &c : rf) c = complement_char(c);
        std::reverse(rf.begin(), rf.end());
        const size_t np = r.patterns.size(), nfwd = np / 2;
        for (size_t p = 0; p < np; ++p) {
            MyersPattern mp;
            std::memset(&mp, 0, sizeof mp);
            mp.request = (uint32_t)ri;
            mp.strand = p >= nfwd;
            mp.L = L;
            mp.E = rd.E;
            mp.W = rd.W;
            const std::string &pa = r.patterns[p];
            const std::string &fa = p < nfwd ? r.filter : rf;
            build_eq16(pa, mp.eq_lo, mp.eq_hi);
            for (uint32_t c = 0; c < L; ++c) {
                mp.b4[c] = t.str2b4[1][(uint8_t)pa[c]];
                mp.isn[c] = pa[c] == 'N' || pa[c] == 'n';
                mp.eff[c] = t.str2b4[1][(uint8_t)fa[c]];
            }
            // precompute_pam_precheck (search.rs:761-777)
            uint32_t ps = L;
            for (uint32_t c = 0; c < L; ++c)
                if (mp.isn[c]) { ps = c; break; }
            mp.pam_off = ps;
            for (uint32_t c = ps; c < L; ++c)
                if (mp.isn[c]) mp.pamf[mp.pam_n++] = mp.eff[c];
            // its PAM form: cells, and the spans check_pam_quick tries
            // (search.rs:703-755; L + bd - br, or L alone when the PAM
            // does not lead the pattern)
            PamForm pf;
            std::memset(&pf, 0, sizeof pf);
            pf.pam_off = ps;
            pf.pam_n = mp.pam_n;
            std::memcpy(pf.f, mp.pamf, sizeof pf.f);
            pf.span_lo = ps == 0 ? (uint32_t)std::max<int>(1, (int)L - (int)r.max_rb) : L;
            pf.span_hi = ps == 0 ? L + r.max_db : L;
            uint32_t fi = 0;
            while (fi < forms.size() && std::memcmp(&forms[fi], &pf, sizeof pf) != 0) ++fi;
            if (fi == forms.size()) forms.push_back(pf);
            mp.pad = fi;
            pats.push_back(mp);
        }
    }
    if (tiles.empty() || pats.empty()) return kOk;
    // longest pattern and window: 64-bit Myers words above 32 cells, and
    // the warm-up every window needs
    uint32_t lmax = 0, wmax = 0;
    for (const MyersReqDev &rd : rdev) {
        lmax = std::max(lmax, rd.L);
        wmax = std::max(wmax, rd.W);
    }
    const bool wide = lmax > 32;
    const uint32_t warm = myers_warm(wmax);

    TablePack tp;
    const size_t o_b = tp.add(batches), o_t = tp.add(tiles), o_p = tp.add(pats),
                 o_r = tp.add(rdev), o_f = tp.add(forms);
    if (d.tables.ensure(tp.buf.size(), err)) return err.code;
    CU(cudaEventRecord(d.ev[0], s));
    CU(cudaMemcpyAsync(d.tables.p, tp.buf.data(), tp.buf.size(), cudaMemcpyHostToDevice, s));
    auto tab = [&](size_t o) { return (const void *)(d.tables.p + o); };
    const BatchDev *dB = (const BatchDev *)tab(o_b);
    const MyersPattern *dP = (const MyersPattern *)tab(o_p);
    const MyersReqDev *dR = (const MyersReqDev *)tab(o_r);
    if (d.ctr.ensure(1, err) || d.req_rows.ensure(reqs.size(), err)) return err.code;
    if (d.mcand.cap == 0 && d.mcand.ensure(first_cand_cap(), err)) return err.code;

    // stage 1: streaming Myers + PAM -> candidates
    Counters hc{};
    const uint32_t n_pat = (uint32_t)pats.size();
    if (n_pat >= (1u << 24)) {  // staged candidates keep the pattern in 24 bits
        err = {kUnsupported, "more than 16 M bulge patterns in one pass"};
        return err.code;
    }
    for (int attempt = 0; attempt < 2; ++attempt) {
        CU(cudaMemsetAsync(d.ctr.p, 0, sizeof(Counters), s));
        CU(cudaEventRecord(d.ev[1], s));
        const uint32_t cap = (uint32_t)std::min<size_t>(d.mcand.cap, 0xFFFFFFF0u);
        if (forms.size() <= kMfMaxForms) {
            // PAM test per tile in shared memory.  Tiles per block: a block
            // walks its tpb x n_pat (tile, pattern) items in rounds of
            // kMfThreads, and the grid walks the tile blocks in waves of
            // n_sm x (blocks per SM); take the tpb with the fewest
            // waves x rounds (ties: more tiles per block)
            auto mf_fn = wide ? myers_tile_kernel<uint64_t> : myers_tile_kernel<uint32_t>;
            // candidates staged per block round (COF_MYERS_STAGE lowers it:
            // tests of the overflow to direct appends)
            uint32_t stage_cap = kMfStage;
            if (const char *e = std::getenv("COF_MYERS_STAGE"))
                stage_cap = (uint32_t)std::min<long>(kMfStage, std::max(0L, std::atol(e)));
            const size_t eq_bytes = wide ? 8 : 4;
            auto smem_of = [&](uint32_t t) {
                return (size_t)t * forms.size() * (kMfQWords + 32) * 4 +
                       (n_pat <= (uint32_t)kSmemMyers ? (size_t)n_pat * 16 * eq_bytes : 0) +
                       (size_t)kMfStage * 8 + 8;
            };
            uint32_t tpb = 1;
            uint64_t best = ~0ull;
            int per_sm = 1;
            for (uint32_t t = 1; t <= kMfMaxTiles; ++t) {
                const size_t sm = smem_of(t);
                CU(cudaFuncSetAttribute(mf_fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
                int occ = 1;
                CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, mf_fn, kMfThreads, sm));
                occ = std::max(occ, 1);
                const uint64_t rounds = ((uint64_t)t * n_pat + kMfThreads - 1) / kMfThreads;
                const uint64_t tblk = (tiles.size() + t - 1) / t;
                const uint64_t slots = (uint64_t)d.n_sm * occ;
                const uint64_t cost = ((tblk + slots - 1) / slots) * rounds;
                if (cost <= best) {
                    best = cost;
                    tpb = t;
                    per_sm = occ;
                }
            }
            const size_t smem = smem_of(tpb);
            CU(cudaFuncSetAttribute(mf_fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            const uint64_t tblocks = (tiles.size() + tpb - 1) / tpb;
            const unsigned blocks = (unsigned)std::max<uint64_t>(
                1, std::min<uint64_t>(tblocks, (uint64_t)d.n_sm * std::max(1, per_sm)));
            mf_fn<<<blocks, kMfThreads, smem, s>>>(
                d.bit4.p, dB, (const MyersTile *)tab(o_t), tiles.size(), dP, n_pat,
                (const PamForm *)tab(o_f), (uint32_t)forms.size(), tpb, warm, d.mcand.p, cap,
                d.ctr.p, stage_cap);
        } else {
            const uint64_t items = (uint64_t)tiles.size() * n_pat;
            const unsigned blocks = (unsigned)std::max<uint64_t>(
                1, std::min<uint64_t>((items + 127) / 128, (uint64_t)d.n_sm * 16));
            auto ff = wide ? myers_filter_kernel<uint64_t> : myers_filter_kernel<uint32_t>;
            ff<<<blocks, 128, 0, s>>>(d.bit4.p, dB, (const MyersTile *)tab(o_t), tiles.size(), dP,
                                      n_pat, dR, warm, d.mcand.p, cap, d.ctr.p);
        }
        CU(cudaGetLastError());
        CU(cudaEventRecord(d.ev[2], s));
        ++times_.kernel_launches;
        CU(cudaMemcpyAsync(&hc, d.ctr.p, sizeof(Counters), cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        if (!hc.overflow && hc.hits <= d.mcand.cap) break;
        if (attempt == 1) {
            err = {kOom, "bulge candidate buffer overflow after resize"};
            return err.code;
        }
        if (d.mcand.ensure((size_t)hc.hits + hc.hits / 4 + 1024, err)) return err.code;
    }
    float ms = 0;
    cudaEventElapsedTime(&ms, d.ev[1], d.ev[2]);
    times_.scan_ms += ms;
    times_.candidates += hc.hits;
    const uint32_t n_cand = hc.hits;

    // stage 2: traceback over candidate chunks; each chunk's rows are sorted
    // (pattern, start), formatted, and copied to the host on the copy
    // stream while the next chunk's traceback runs: appended to each
    // request's result, or handed to the sink of a streamed search
    TextOut tout(d.copy_stream, sink, out);
    bool text_out = false;  // a chunk's text has been put
    // rows one chunk may produce; a chunk that produces more is halved and
    // walked again (COF_BULGE_ROW_CAP lowers the cap: tests of that path)
    size_t row_cap = 1u << 24;
    if (const char *e = std::getenv("COF_BULGE_ROW_CAP"))
        row_cap = std::min(row_cap, (size_t)std::max(64L, std::atol(e)));
    if (d.mrows.ensure(row_cap, err) || d.keys.ensure(row_cap, err) ||
        d.keys2.ensure(row_cap, err) || d.vals.ensure(row_cap, err) ||
        d.vals2.ensure(row_cap, err) || d.lens.ensure(row_cap + 1, err) ||
        d.offs.ensure(row_cap + 1, err))
        return err.code;
    // warp-per-candidate traceback when every request's budget bit set
    // fits 128 bits ((db + 1)(rb + 1)(mm + 1)); COF_BULGE_WARP=0 selects the
    // thread-per-candidate kernel
    bool warp_tb = true;
    uint32_t nw = 1;
    for (const MyersReqDev &rd : rdev) {
        if (rd.nbits > kTbMaxBits) warp_tb = false;
        nw = std::max(nw, (rd.nbits + 63) / 64);
    }
    if (const char *e = std::getenv("COF_BULGE_WARP"))
        if (e[0] == '0') warp_tb = false;
    // the band of the budget DP that alignments within the caps can touch
    // (db + rb + 1 cells per row): the pre-test computes only the band, and
    // the warp traceback reads each survivor's band table from a kernel
    // that writes them per chunk (COF_BULGE_BAND=0: whole tables)
    uint32_t band = 0;
    for (const MyersReqDev &rd : rdev) band = std::max(band, rd.db + rd.rb + 1);
    bool banded = band <= kBandMax;
    if (const char *e = std::getenv("COF_BULGE_BAND"))
        if (e[0] == '0') banded = false;
    uint32_t tbl_words = 0;  // 64-bit words of one warp's table
    for (const MyersReqDev &rd : rdev)
        tbl_words = std::max(tbl_words, (rd.L + 1) * (banded ? rd.db + rd.rb + 1 : rd.W + 1) * nw);
    // nodes with two op words for windows of more than 48 cells
    const bool wide_nodes = wmax > 48;
    const size_t item_bytes = wide_nodes ? sizeof(TbItem<2>) : sizeof(TbItem<1>);
    const uint32_t tb_mrg = tb_margin(wmax);
    // with band tables, several candidates are resident per warp
    // (traceback_slots_kernel), their tables copied into the slots
    // (COF_TB_GLOBAL=1: read from global memory); COF_TB_SLOTS sets
    // 1..kTbSlotsMax, or 0 for one tree per warp (traceback_warp_kernel)
    bool tb_global = false;
    if (const char *e = std::getenv("COF_TB_GLOBAL")) tb_global = e[0] == '1';
    uint32_t tb_slots = banded ? (tb_global ? kTbSlotsGlobal : kTbSlotsShared) : 0;
    if (const char *e = std::getenv("COF_TB_SLOTS"))
        if (banded) tb_slots = (uint32_t)std::min<long>(kTbSlotsMax, std::max(0L, std::atol(e)));
    if (!tb_slots) tb_global = false;
    // free slots take work while the stack holds fewer than tb_refill
    // nodes (COF_TB_REFILL)
    uint32_t tb_refill = kTbRefill;
    if (const char *e = std::getenv("COF_TB_REFILL"))
        tb_refill = (uint32_t)std::min<int>(kTbSlotSpare - kTbSlotsMax, std::max(1, std::atoi(e)));
    // a stack of the walk margin plus the spare slots
    const uint32_t stk_cap = tb_mrg + (tb_slots ? kTbSlotSpare : kTbSpare);
    if (warp_tb && d.tb_items.ensure(2 * (size_t)kTbQueue * item_bytes, err)) return err.code;
    uint32_t tb_budget = kTbBudget;  // COF_TB_BUDGET: iterations before a tree is handed on
    if (const char *e = std::getenv("COF_TB_BUDGET")) tb_budget = (uint32_t)std::max(1, std::atoi(e));
    int smem_optin = 0;
    CU(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, d.device));
    const size_t node_bytes = wide_nodes ? sizeof(TbNode<2>) : sizeof(TbNode<1>);
    auto warp_bytes_for = [&](uint32_t slots) -> size_t {
        if (slots) return tb_slot_layout(node_bytes, tb_global ? 0u : tbl_words, stk_cap, slots).total;
        return wide_nodes ? tb_warp_bytes<2>(tbl_words, stk_cap) : tb_warp_bytes<1>(tbl_words, stk_cap);
    };
    // fewer slots while kTbWarps warps of them exceed a block's shared memory
    while (tb_slots > 1 && warp_bytes_for(tb_slots) * kTbWarps > (size_t)smem_optin) --tb_slots;
    const size_t warp_bytes = warp_bytes_for(tb_slots);
    // warps per block: kTbWarps, fewer when their tables exceed a block's
    // shared memory (patterns of more than 32 cells with two-word cells)
    const uint32_t tb_wpb = (uint32_t)std::max<size_t>(
        1, std::min<size_t>(kTbWarps, (size_t)smem_optin / warp_bytes));
    if (warp_tb && warp_bytes > (size_t)smem_optin) warp_tb = false;
    const size_t tb_smem = (size_t)tb_wpb * warp_bytes;
    const void *tb_fn =
        tb_slots ? (tb_global
                        ? (wide_nodes ? (nw == 1 ? (const void *)traceback_slots_kernel<1, 2, true>
                                                 : (const void *)traceback_slots_kernel<2, 2, true>)
                                      : (nw == 1 ? (const void *)traceback_slots_kernel<1, 1, true>
                                                 : (const void *)traceback_slots_kernel<2, 1, true>))
                        : (wide_nodes ? (nw == 1 ? (const void *)traceback_slots_kernel<1, 2, false>
                                                 : (const void *)traceback_slots_kernel<2, 2, false>)
                                      : (nw == 1 ? (const void *)traceback_slots_kernel<1, 1, false>
                                                 : (const void *)traceback_slots_kernel<2, 1, false>)))
        : banded ? (wide_nodes ? (nw == 1 ? (const void *)traceback_warp_kernel<1, 2, true>
                                          : (const void *)traceback_warp_kernel<2, 2, true>)
                               : (nw == 1 ? (const void *)traceback_warp_kernel<1, 1, true>
                                          : (const void *)traceback_warp_kernel<2, 1, true>))
                 : (wide_nodes ? (nw == 1 ? (const void *)traceback_warp_kernel<1, 2, false>
                                          : (const void *)traceback_warp_kernel<2, 2, false>)
                               : (nw == 1 ? (const void *)traceback_warp_kernel<1, 1, false>
                                          : (const void *)traceback_warp_kernel<2, 1, false>));
    void (*tb_launch)(const TbLaunch &) =
        tb_slots ? (tb_global
                        ? (wide_nodes ? (nw == 1 ? launch_tb_slots<1, 2, true> : launch_tb_slots<2, 2, true>)
                                      : (nw == 1 ? launch_tb_slots<1, 1, true> : launch_tb_slots<2, 1, true>))
                        : (wide_nodes ? (nw == 1 ? launch_tb_slots<1, 2, false> : launch_tb_slots<2, 2, false>)
                                      : (nw == 1 ? launch_tb_slots<1, 1, false> : launch_tb_slots<2, 1, false>)))
        : banded ? (wide_nodes ? (nw == 1 ? launch_tb<1, 2, true> : launch_tb<2, 2, true>)
                               : (nw == 1 ? launch_tb<1, 1, true> : launch_tb<2, 1, true>))
                 : (wide_nodes ? (nw == 1 ? launch_tb<1, 2, false> : launch_tb<2, 2, false>)
                               : (nw == 1 ? launch_tb<1, 1, false> : launch_tb<2, 1, false>));
    int tb_blocks_per_sm = 1;
    if (warp_tb) {
        CU(cudaFuncSetAttribute(tb_fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tb_smem));
        CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&tb_blocks_per_sm, tb_fn, tb_wpb * 32,
                                                         tb_smem));
        tb_blocks_per_sm = std::max(1, tb_blocks_per_sm);
    }
    // exact pre-test: only candidates with an alignment within the caps go
    // on to the warp traceback
    const MyersCand *cands = d.mcand.p;
    uint32_t n_work = n_cand;
    if (warp_tb && n_cand) {
        if (d.mcand2.ensure(n_cand, err)) return err.code;
        const size_t bf_smem = (size_t)(banded ? band : wmax + 1) * nw * kBfThreads * 8;
        const void *fn = banded ? (wmax > 48 ? (nw == 1 ? (const void *)budget_band_kernel<1, 5, false>
                                                        : (const void *)budget_band_kernel<2, 5, false>)
                                             : (nw == 1 ? (const void *)budget_band_kernel<1, 3, false>
                                                        : (const void *)budget_band_kernel<2, 3, false>))
                                : (wmax > 48 ? (nw == 1 ? (const void *)budget_filter_kernel<1, 5>
                                                        : (const void *)budget_filter_kernel<2, 5>)
                                             : (nw == 1 ? (const void *)budget_filter_kernel<1, 3>
                                                        : (const void *)budget_filter_kernel<2, 3>));
        CU(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bf_smem));
        int bf_per_sm = 1;
        CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bf_per_sm, fn, kBfThreads, bf_smem));
        CU(cudaMemsetAsync(&d.ctr.p->rows, 0, 4, s));
        CU(cudaEventRecord(d.ev[3], s));
        const unsigned bg = (unsigned)std::max<uint64_t>(
            1, std::min<uint64_t>((n_cand + kBfThreads - 1) / kBfThreads,
                                  (uint64_t)d.n_sm * std::max(1, bf_per_sm)));
        const GenomeDev gv = d.view();
        const MyersCand *cin = d.mcand.p;
        MyersCand *cout = d.mcand2.p;
        uint32_t *nout = &d.ctr.p->rows;
        uint64_t *no_tbl = nullptr;
        uint32_t no_stride = 0;
        void *args[] = {(void *)&gv,  (void *)&dB,   (void *)&dP,     (void *)&dR,
                        (void *)&cin, (void *)&n_cand, (void *)&cout, (void *)&nout,
                        (void *)&no_tbl, (void *)&no_stride};
        CU(cudaLaunchKernel(fn, dim3(bg), dim3(kBfThreads), args, bf_smem, s));
        CU(cudaGetLastError());
        CU(cudaEventRecord(d.ev[4], s));
        ++times_.kernel_launches;
        CU(cudaMemcpyAsync(&n_work, &d.ctr.p->rows, 4, cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        cudaEventElapsedTime(&ms, d.ev[3], d.ev[4]);
        times_.verify_ms += ms;
        cands = d.mcand2.p;
    }
    // candidates per chunk; a chunk's rows cross to the host while the next
    // chunk's traceback runs.  COF_BULGE_CHUNK lowers it (tests: many
    // chunks).  Every chunk ends in a tail of a few long trees, so a set
    // that fits one chunk is walked whole (splitting the 10 Mbp benchmark
    // into four chunks to hide its copy made the traceback 9 ms slower
    // than the copy it hid).  A very large set (hundreds of millions of
    // rows) first walks a probe chunk; the later chunks are sized from its
    // rows per candidate to fill most of the row buffer, and a chunk that
    // overflows it is cut in proportion to its row count and walked again.
    // with band tables, a chunk's tables (tbl_words words per candidate)
    // stay within 4 GiB of device memory
    const uint32_t chunk_max = (warp_tb && banded)
        ? (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(kBulgeChunkMax,
                                                           (uint64_t(4) << 30) / (tbl_words * 8ull)))
        : kBulgeChunkMax;
    uint32_t chunk = std::max<uint32_t>(1, std::min<uint32_t>(n_work, chunk_max));
    bool probe = n_work > 4 * kBulgeProbe;
    if (probe) chunk = std::min(chunk, kBulgeProbe);
    if (const char *e = std::getenv("COF_BULGE_CHUNK")) {
        chunk = std::max<uint32_t>(1, std::min<uint32_t>(chunk, (uint32_t)std::max(1, std::atoi(e))));
        probe = false;
    }
    const double row_fill = 0.85 * (double)row_cap;  // rows a sized chunk aims at
    uint32_t c0 = 0;
    while (c0 < n_work) {
        const uint32_t cn = std::min(chunk, n_work - c0);
        CU(cudaMemsetAsync(d.ctr.p, 0, sizeof(Counters), s));
        CU(cudaMemsetAsync(d.req_rows.p, 0, reqs.size() * 4, s));
        CU(cudaEventRecord(d.ev[3], s));
        if (warp_tb && banded) {
            // the chunk's band tables, one thread per surviving candidate
            // at least 8 MiB, so that a stream of small requests of varying
            // size does not reallocate it (an allocation waits for the device)
            if (d.bandtbl.ensure(std::max<size_t>((size_t)cn * tbl_words, size_t(1) << 20), err))
                return err.code;
            auto tfn = wmax > 48 ? (nw == 1 ? budget_band_kernel<1, 5, true> : budget_band_kernel<2, 5, true>)
                                 : (nw == 1 ? budget_band_kernel<1, 3, true> : budget_band_kernel<2, 3, true>);
            const size_t tsm = (size_t)band * nw * kBfThreads * 8;
            CU(cudaFuncSetAttribute(tfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tsm));
            const unsigned tg = (unsigned)std::max<uint64_t>(
                1, std::min<uint64_t>((cn + kBfThreads - 1) / kBfThreads, (uint64_t)d.n_sm * 16));
            tfn<<<tg, kBfThreads, tsm, s>>>(d.view(), dB, dP, dR, cands + c0, cn, nullptr, nullptr,
                                            d.bandtbl.p, tbl_words);
            CU(cudaGetLastError());
            ++times_.kernel_launches;
        }
        if (warp_tb) {
            // pass 0 walks every candidate; a warp that spends kTbBudget
            // iterations on one tree hands its remaining stack on, and the
            // next pass spreads those subtrees over all warps
            const unsigned grid = (unsigned)((uint64_t)d.n_sm * tb_blocks_per_sm);
            char *tq = reinterpret_cast<char *>(d.tb_items.p);
            char *q[2] = {tq, tq + kTbQueue * item_bytes};
            const char *in = nullptr;
            uint32_t n_in = 0;
            for (int pass = 0;; ++pass) {
                const bool last = pass >= kTbMaxPasses;
                CU(cudaMemsetAsync(&d.ctr.p->next_item, 0, sizeof(unsigned long long), s));
                CU(cudaMemsetAsync(&d.ctr.p->hits, 0, sizeof(uint32_t), s));
                const uint64_t work = in ? n_in : cn;
                const unsigned tb = (unsigned)std::max<uint64_t>(
                    1, std::min<uint64_t>((work + tb_wpb - 1) / tb_wpb, grid));
                char *out_q = q[pass & 1];
                TbLaunch a{tb, tb_wpb * 32, tb_smem, s, d.view(), dB, dP, dR, cands + c0, cn,
                           in, n_in, last ? nullptr : out_q, kTbQueue, tb_budget, tbl_words,
                           stk_cap, tb_mrg, d.mrows.p, (uint32_t)row_cap, d.keys.p, d.vals.p,
                           d.ctr.p, d.req_rows.p, banded ? d.bandtbl.p : nullptr, tbl_words,
                           tb_slots, tb_refill};
                tb_launch(a);
                CU(cudaGetLastError());
                ++times_.kernel_launches;
                // pieces whose copies are done go to the sink beside this pass
                if (tout.poll(err)) return err.code;
                if (last) break;
                uint32_t n_spill = 0;
                CU(cudaMemcpyAsync(&n_spill, &d.ctr.p->hits, 4, cudaMemcpyDeviceToHost, s));
                CU(cudaStreamSynchronize(s));
                if (n_spill == 0) break;
                in = out_q;
                n_in = std::min<uint32_t>(n_spill, kTbQueue);
            }
            --times_.kernel_launches;  // counted once more below
        } else {
            const unsigned tb = (unsigned)std::min<uint64_t>((cn + 127) / 128, (uint64_t)d.n_sm * 32);
            traceback_kernel<<<tb, 128, 0, s>>>(d.view(), dB, dP, dR, cands + c0, cn, d.mrows.p,
                                                (uint32_t)row_cap, d.keys.p, d.vals.p, d.ctr.p,
                                                d.req_rows.p);
        }
        CU(cudaGetLastError());
        CU(cudaEventRecord(d.ev[4], s));
        ++times_.kernel_launches;
        CU(cudaMemcpyAsync(&hc, d.ctr.p, sizeof(Counters), cudaMemcpyDeviceToHost, s));
        std::vector<uint32_t> rq(reqs.size());
        CU(cudaMemcpyAsync(rq.data(), d.req_rows.p, reqs.size() * 4, cudaMemcpyDeviceToHost, s));
        if (tout.poll(err)) return err.code;  // beside this traceback
        CU(cudaStreamSynchronize(s));
        cudaEventElapsedTime(&ms, d.ev[3], d.ev[4]);
        times_.verify_ms += ms;
        if (hc.overflow || hc.rows > row_cap) {
            if (cn == 1) {
                err = {kUnsupported, "one bulge candidate has more alignments than the row buffer"};
                return err.code;
            }
            // hc.rows counts every alignment of the chunk (the walk goes on
            // past the buffer): cut the chunk in proportion
            const uint64_t fit = (uint64_t)((double)cn * row_fill / std::max<double>(hc.rows, row_cap + 1.0));
            chunk = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(fit, cn / 2));
            probe = false;
            continue;
        }
        const uint32_t nr = hc.rows;
        if (probe) {  // size the remaining chunks from the probe's rows per candidate
            const double per = std::max(1.0, (double)nr) / (double)cn;
            chunk = (uint32_t)std::max(1.0, std::min((double)chunk_max, row_fill / per));
            probe = false;
        }
        times_.rows += nr;
        if (nr) {
            CU(cudaEventRecord(d.ev[5], s));
            size_t tmp = 0, tmp2 = 0;
            // key bits in use: the start's, then the pattern index's
            int key_bits = (int)d.key_shift();
            for (size_t np = pats.size(); np > 1; np = (np + 1) / 2) ++key_bits;
            key_bits = std::min(key_bits, 64);
            CU(cub::DeviceRadixSort::SortPairs(nullptr, tmp, d.keys.p, d.keys2.p, d.vals.p,
                                               d.vals2.p, (int)nr, 0, key_bits, s));
            CU(cub::DeviceScan::ExclusiveSum(nullptr, tmp2, d.lens.p, d.offs.p, (int)nr + 1, s));
            if (d.cub_tmp.ensure(std::max(tmp, tmp2), err)) return err.code;
            tmp = d.cub_tmp.cap;
            CU(cub::DeviceRadixSort::SortPairs(d.cub_tmp.p, tmp, d.keys.p, d.keys2.p, d.vals.p,
                                               d.vals2.p, (int)nr, 0, key_bits, s));
            const unsigned fb = (unsigned)std::min<uint64_t>((nr + 255) / 256, (uint64_t)d.n_sm * 8);
            mrow_len_kernel<<<fb, 256, 0, s>>>(d.view(), d.mrows.p, d.vals2.p, nr, dP, dR, d.lens.p);
            CU(cudaGetLastError());
            CU(cudaMemsetAsync(d.lens.p + nr, 0, 4, s));
            tmp2 = d.cub_tmp.cap;
            CU(cub::DeviceScan::ExclusiveSum(d.cub_tmp.p, tmp2, d.lens.p, d.offs.p, (int)nr + 1, s));
            uint64_t bytes = 0;
            CU(cudaMemcpyAsync(&bytes, d.offs.p + nr, 8, cudaMemcpyDeviceToHost, s));
            CU(cudaStreamSynchronize(s));
            // d.text is rewritten below: the previous chunk's copy has run
            // beside this chunk's traceback and is waited for here
            if (tout.drain(err)) return err.code;
            if (d.text.ensure(bytes + 1, err)) return err.code;
            mrow_write_kernel<<<fb, 256, 0, s>>>(d.view(), d.mrows.p, d.vals2.p, nr, dP, dR,
                                                 d.offs.p, d.text.p);
            CU(cudaGetLastError());
            times_.kernel_launches += 4;
            // each request's first row inside this chunk's sorted rows
            std::vector<uint32_t> first(reqs.size());
            for (size_t ri = 0, r0 = 0; ri < reqs.size(); r0 += rq[ri], ++ri)
                first[ri] = (uint32_t)r0;
            if (tout.records()) {
                if (d.recs.ensure(nr, err) || d.req_first.ensure(reqs.size(), err)) return err.code;
                CU(cudaMemcpyAsync(d.req_first.p, first.data(), reqs.size() * 4,
                                   cudaMemcpyHostToDevice, s));
                mrow_rec_kernel<<<fb, 256, 0, s>>>(d.view(), d.mrows.p, d.vals2.p, nr, dP, dR,
                                                   d.offs.p, d.req_first.p, d.recs.p);
                CU(cudaGetLastError());
                ++times_.kernel_launches;
            }
            CU(cudaEventRecord(d.ev[6], s));
            CU(cudaEventRecord(d.fmt_done, s));
            // request boundaries (text bytes) inside this chunk
            std::vector<uint64_t> bound(reqs.size() + 1, bytes);
            for (size_t ri = 0; ri < reqs.size(); ++ri) {
                bound[ri] = bytes;
                if (first[ri] < nr)
                    CU(cudaMemcpyAsync(&bound[ri], d.offs.p + first[ri], 8, cudaMemcpyDeviceToHost, s));
            }
            CU(cudaStreamSynchronize(s));
            cudaEventElapsedTime(&ms, d.ev[5], d.ev[6]);
            times_.format_ms += ms;
            const uint64_t done = (uint64_t)c0 + cn;
            for (size_t ri = 0; ri < reqs.size(); ++ri) {
                const uint64_t b = bound[ri + 1] - bound[ri];
                if (!rq[ri]) continue;
                if (!text_out) {  // result size from the first chunk's share of the work
                    const double f = done >= n_work ? 1.0 : 1.15 * (double)n_work / (double)done;
                    if (tout.reserve(ri, (size_t)(b * f) + (done >= n_work ? 0 : 65536), err))
                        return err.code;
                }
                if (tout.put(ri, d.text.p + bound[ri], b, rq[ri], d.recs.p + first[ri],
                             d.fmt_done, err))
                    return err.code;
            }
            text_out = true;
        }
        c0 += cn;
    }
    // the copy time left after the last chunk's text
    CU(cudaEventRecord(d.ev[7], d.copy_stream));
    if (tout.finish(err)) return err.code;
    if (text_out) {
        cudaEventElapsedTime(&ms, d.ev[6], d.ev[7]);
        times_.d2h_ms += std::max(0.0f, ms);
    }
    return kOk;
}

}  // namespace cof
