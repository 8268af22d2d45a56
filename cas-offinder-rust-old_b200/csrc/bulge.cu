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
//       streaming Myers sweep (Myers 1999, semi-global, 32-bit words) started
//       >= 48 positions before the tile.  Its score at t bounds the windowed
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
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "cof_engine.h"
#include "engine_dev.cuh"

namespace cof {

namespace {

constexpr int kMaxCells = 40;          // L <= 32, L + max_db <= 40
constexpr uint32_t kTile = 1024;       // end positions per filter work item
constexpr uint32_t kWarm = 48;         // Myers warm-up before a tile (>= W - 1)
constexpr int kSmemMyers = 512;        // patterns whose eq tables fit in smem

struct MyersPattern {
    uint32_t request, strand, L, E;    // E = max edits = mm + db + rb
    uint32_t W, pam_off, pam_n, pad;
    uint32_t eq16[16];                 // Myers Eq per genome nibble value
    uint8_t b4[kMaxCells];             // pattern bit4 cells
    uint8_t isn[kMaxCells];            // pattern char is N/n (pam_is_n)
    uint8_t eff[kMaxCells];            // effective filter bit4 per cell
    uint8_t pamf[kMaxCells];           // PAM precheck filter list
};

struct MyersReqDev {
    uint32_t L, mm, db, rb, E, W, pam_len, raw;  // raw: Match lines, not rows
    uint32_t first_pattern, pad[3];
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

__global__ void myers_filter_kernel(const uint8_t *__restrict__ bit4,
                                    const BatchDev *__restrict__ batches,
                                    const MyersTile *__restrict__ tiles, uint64_t n_tiles,
                                    const MyersPattern *__restrict__ pats, uint32_t n_pat,
                                    const MyersReqDev *__restrict__ reqs, MyersCand *cand,
                                    uint32_t cap, Counters *ctr) {
    __shared__ uint32_t seq[kSmemMyers * 16];
    const bool staged = n_pat <= (uint32_t)kSmemMyers;
    if (staged)
        for (uint32_t i = threadIdx.x; i < n_pat * 16; i += blockDim.x) seq[i] = pats[i / 16].eq16[i % 16];
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
        const uint32_t *eq = staged ? seq + 16 * p : P.eq16;
        const uint32_t L = P.L;
        const uint32_t mask = L == 32 ? 0xFFFFFFFFu : ((1u << L) - 1u);
        const uint32_t sh = L - 1;
        uint32_t vp = mask, vn = 0;
        int score = (int)L;
        const uint64_t ws = T.t0 >= kWarm ? ((T.t0 - kWarm) & ~15ull) : 0;
        unsigned long long word = 0;
        for (uint64_t q = ws; q < T.t1; ++q) {
            if ((q & 15) == 0 || q == ws)
                word = __ldg(reinterpret_cast<const unsigned long long *>(bit4 + ((q >> 1) & ~7ull)));
            const uint32_t b = (uint32_t)(word >> ((q & 15) * 4)) & 0xF;
            const uint32_t x = eq[b] | vn;
            const uint32_t d0 = (((x & vp) + vp) ^ vp) | x;
            const uint32_t hn = vp & d0;
            const uint32_t hp = vn | ~(vp | d0);
            const uint32_t xs = hp << 1;
            vn = xs & d0;
            vp = ((hn << 1) | ~(xs | d0)) & mask;
            vn &= mask;
            score += (int)((hp >> sh) & 1u) - (int)((hn >> sh) & 1u);
            if (q >= T.t0 && score <= (int)P.E) {
                const uint32_t tl = (uint32_t)(q - B.base);
                if (tl + 1 >= L && pam_quick(bit4, B, tl, P, R.db, R.rb)) {
                    const uint32_t i = atomicAdd(&ctr->hits, 1u);
                    if (i < cap) cand[i] = MyersCand{tl, T.batch, p, 0};
                    else ctr->overflow = 1;
                }
            }
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
                    for (int k = 0; k < n_ops; ++k) {
                        const uint8_t op = ops[n_ops - 1 - k];
                        if (k < 32) o0 |= (uint64_t)op << (2 * k);
                        else o1 |= (uint64_t)op << (2 * (k - 32));
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
                                w.pad = 0;
                                rows[r] = w;
                                keys[r] = ((uint64_t)c.pattern << 34) | start;
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

__global__ void mrow_write_kernel(GenomeDev G, const MyersRow *__restrict__ rows,
                                  const uint32_t *__restrict__ order, uint32_t n,
                                  const MyersPattern *__restrict__ pats,
                                  const MyersReqDev *__restrict__ reqs,
                                  const uint64_t *__restrict__ off, char *__restrict__ text) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const MyersRow w = rows[order[i]];
        const MyersPattern &P = pats[w.pattern];
        const MyersReqDev R = reqs[P.request];
        const bool fwd = P.strand == 0;
        char *o = text + off[i];
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
        uint64_t gi = w.start;
        for (uint32_t k = 0; k < no; ++k) {
            const uint32_t op = (uint32_t)((k < 32 ? w.ops[0] >> (2 * k) : w.ops[1] >> (2 * (k - 32))) & 3);
            uint8_t pv = 0, gv = 0;
            bool pgap = false, ggap = false;
            if (op <= 1) {
                pv = P.b4[pi++];
                gv = nib(G.bit4, gi++);
            } else if (op == 2) {
                pgap = true;
                gv = nib(G.bit4, gi++);
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
            continue;
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
    }
}

// Myers Eq table of one pattern (build_peq, myers.rs:32-50, and the eq rule
// of search.rs:846-858): nibble 0 -> 0, 0xF -> peq_n, else OR of the peqs of
// its set bits (A=4, C=2, G=8, T=1).
void build_eq16(const std::string &p, uint32_t eq16[16]) {
    uint32_t peq[4] = {0, 0, 0, 0}, peq_n = 0;
    for (size_t i = 0; i < p.size(); ++i) {
        const char u = (char)((p[i] >= 'a' && p[i] <= 'z') ? p[i] - 32 : p[i]);
        const int idx = u == 'A' ? 0 : u == 'C' ? 1 : u == 'G' ? 2 : u == 'T' ? 3 : 4;
        if (idx < 4) {
            peq[idx] |= 1u << i;
        } else {
            for (int k = 0; k < 4; ++k) peq[k] |= 1u << i;
            peq_n |= 1u << i;
        }
    }
    for (int b = 0; b < 16; ++b) {
        uint32_t e = 0;
        if (b == 15) e = peq_n;
        else {
            if (b & 4) e |= peq[0];
            if (b & 2) e |= peq[1];
            if (b & 8) e |= peq[2];
            if (b & 1) e |= peq[3];
        }
        eq16[b] = e;
    }
}

}  // namespace

int Engine::run_bulge(const std::vector<Request> &reqs, std::vector<Result> &out, Error &err) {
    DeviceGenome &d = *dev_;
    const HostGenome &h = host_;
    const Bit4Tables &t = bit4();
    cudaStream_t s = d.stream;
    out.assign(reqs.size(), Result());

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
        // active end positions (search.rs:913-927, :1087-1092)
        for (uint64_t a = x.base + x.active_start; a < x.base + x.valid; a += kTile)
            tiles.push_back(MyersTile{a, std::min<uint64_t>(a + kTile, x.base + x.valid),
                                      (uint32_t)bi, 0, 0});
    }
    std::vector<MyersReqDev> rdev;
    std::vector<MyersPattern> pats;
    for (size_t ri = 0; ri < reqs.size(); ++ri) {
        const Request &r = reqs[ri];
        const uint32_t L = (uint32_t)r.filter.size();
        MyersReqDev rd{L, r.max_mm, r.max_db, r.max_rb, r.max_mm + r.max_db + r.max_rb,
                       L + r.max_db, (uint32_t)r.pam_len, r.raw ? 1u : 0u,
                       (uint32_t)pats.size(), {0, 0, 0}};
        if (rd.W > (uint32_t)kMaxCells) {
            err = {kUnsupported, "pattern length + max_dna_bulges above 40"};
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
            build_eq16(pa, mp.eq16);
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
            pats.push_back(mp);
        }
    }
    if (tiles.empty() || pats.empty()) return kOk;

    TablePack tp;
    const size_t o_b = tp.add(batches), o_t = tp.add(tiles), o_p = tp.add(pats),
                 o_r = tp.add(rdev);
    if (d.tables.ensure(tp.buf.size(), err)) return err.code;
    CU(cudaEventRecord(d.ev[0], s));
    CU(cudaMemcpyAsync(d.tables.p, tp.buf.data(), tp.buf.size(), cudaMemcpyHostToDevice, s));
    auto tab = [&](size_t o) { return (const void *)(d.tables.p + o); };
    const BatchDev *dB = (const BatchDev *)tab(o_b);
    const MyersPattern *dP = (const MyersPattern *)tab(o_p);
    const MyersReqDev *dR = (const MyersReqDev *)tab(o_r);
    if (d.ctr.ensure(1, err) || d.req_rows.ensure(reqs.size(), err)) return err.code;
    if (d.mcand.cap == 0 && d.mcand.ensure(1u << 22, err)) return err.code;

    // stage 1: streaming Myers + PAM -> candidates
    Counters hc{};
    const uint32_t n_pat = (uint32_t)pats.size();
    for (int attempt = 0; attempt < 2; ++attempt) {
        CU(cudaMemsetAsync(d.ctr.p, 0, sizeof(Counters), s));
        CU(cudaEventRecord(d.ev[1], s));
        const uint64_t items = (uint64_t)tiles.size() * n_pat;
        const unsigned blocks =
            (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((items + 127) / 128, (uint64_t)d.n_sm * 16));
        myers_filter_kernel<<<blocks, 128, 0, s>>>(d.bit4.p, dB, (const MyersTile *)tab(o_t),
                                                   tiles.size(), dP, n_pat, dR, d.mcand.p,
                                                   (uint32_t)std::min<size_t>(d.mcand.cap, 0xFFFFFFF0u),
                                                   d.ctr.p);
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
    // (pattern, start), formatted and appended to the requests' texts
    std::vector<std::string> texts(reqs.size());
    std::vector<uint64_t> nrows(reqs.size(), 0);
    const size_t row_cap = 1u << 24;
    if (d.mrows.ensure(row_cap, err) || d.keys.ensure(row_cap, err) ||
        d.keys2.ensure(row_cap, err) || d.vals.ensure(row_cap, err) ||
        d.vals2.ensure(row_cap, err) || d.lens.ensure(row_cap + 1, err) ||
        d.offs.ensure(row_cap + 1, err))
        return err.code;
    uint32_t chunk = std::max<uint32_t>(1, std::min<uint32_t>(n_cand, 1u << 21));
    uint32_t c0 = 0;
    while (c0 < n_cand) {
        const uint32_t cn = std::min(chunk, n_cand - c0);
        CU(cudaMemsetAsync(d.ctr.p, 0, sizeof(Counters), s));
        CU(cudaMemsetAsync(d.req_rows.p, 0, reqs.size() * 4, s));
        CU(cudaEventRecord(d.ev[3], s));
        const unsigned tb = (unsigned)std::min<uint64_t>((cn + 127) / 128, (uint64_t)d.n_sm * 32);
        traceback_kernel<<<tb, 128, 0, s>>>(d.view(), dB, dP, dR, d.mcand.p + c0, cn, d.mrows.p,
                                            (uint32_t)row_cap, d.keys.p, d.vals.p, d.ctr.p,
                                            d.req_rows.p);
        CU(cudaGetLastError());
        CU(cudaEventRecord(d.ev[4], s));
        ++times_.kernel_launches;
        CU(cudaMemcpyAsync(&hc, d.ctr.p, sizeof(Counters), cudaMemcpyDeviceToHost, s));
        std::vector<uint32_t> rq(reqs.size());
        CU(cudaMemcpyAsync(rq.data(), d.req_rows.p, reqs.size() * 4, cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        cudaEventElapsedTime(&ms, d.ev[3], d.ev[4]);
        times_.verify_ms += ms;
        if (hc.overflow || hc.rows > row_cap) {
            if (cn == 1) {
                err = {kUnsupported, "one bulge candidate has more alignments than the row buffer"};
                return err.code;
            }
            chunk = std::max<uint32_t>(1, cn / 2);
            continue;
        }
        const uint32_t nr = hc.rows;
        times_.rows += nr;
        if (nr) {
            CU(cudaEventRecord(d.ev[5], s));
            size_t tmp = 0, tmp2 = 0;
            CU(cub::DeviceRadixSort::SortPairs(nullptr, tmp, d.keys.p, d.keys2.p, d.vals.p,
                                               d.vals2.p, (int)nr, 0, 64, s));
            CU(cub::DeviceScan::ExclusiveSum(nullptr, tmp2, d.lens.p, d.offs.p, (int)nr + 1, s));
            if (d.cub_tmp.ensure(std::max(tmp, tmp2), err)) return err.code;
            tmp = d.cub_tmp.cap;
            CU(cub::DeviceRadixSort::SortPairs(d.cub_tmp.p, tmp, d.keys.p, d.keys2.p, d.vals.p,
                                               d.vals2.p, (int)nr, 0, 64, s));
            const unsigned fb = (unsigned)std::min<uint64_t>((nr + 255) / 256, (uint64_t)d.n_sm * 8);
            mrow_len_kernel<<<fb, 256, 0, s>>>(d.view(), d.mrows.p, d.vals2.p, nr, dP, dR, d.lens.p);
            CU(cudaGetLastError());
            CU(cudaMemsetAsync(d.lens.p + nr, 0, 4, s));
            tmp2 = d.cub_tmp.cap;
            CU(cub::DeviceScan::ExclusiveSum(d.cub_tmp.p, tmp2, d.lens.p, d.offs.p, (int)nr + 1, s));
            uint64_t bytes = 0;
            CU(cudaMemcpyAsync(&bytes, d.offs.p + nr, 8, cudaMemcpyDeviceToHost, s));
            CU(cudaStreamSynchronize(s));
            if (d.text.ensure(bytes + 1, err)) return err.code;
            mrow_write_kernel<<<fb, 256, 0, s>>>(d.view(), d.mrows.p, d.vals2.p, nr, dP, dR,
                                                 d.offs.p, d.text.p);
            CU(cudaGetLastError());
            times_.kernel_launches += 4;
            if (bytes > d.h_text_cap) {
                if (d.h_text) cudaFreeHost(d.h_text);
                d.h_text = nullptr;
                d.h_text_cap = 0;
                CU(cudaMallocHost((void **)&d.h_text, bytes));
                d.h_text_cap = bytes;
            }
            CU(cudaEventRecord(d.ev[6], s));
            CU(cudaMemcpyAsync(d.h_text, d.text.p, bytes, cudaMemcpyDeviceToHost, s));
            CU(cudaEventRecord(d.ev[7], s));
            // request boundaries inside this chunk's sorted rows
            std::vector<uint64_t> bound(reqs.size() + 1, bytes);
            uint64_t r0 = 0;
            for (size_t ri = 0; ri < reqs.size(); ++ri) {
                bound[ri] = 0;
                if (r0 < nr) CU(cudaMemcpyAsync(&bound[ri], d.offs.p + r0, 8, cudaMemcpyDeviceToHost, s));
                else bound[ri] = bytes;
                r0 += rq[ri];
            }
            CU(cudaStreamSynchronize(s));
            cudaEventElapsedTime(&ms, d.ev[5], d.ev[6]);
            times_.format_ms += ms;
            cudaEventElapsedTime(&ms, d.ev[6], d.ev[7]);
            times_.d2h_ms += ms;
            for (size_t ri = 0; ri < reqs.size(); ++ri) {
                texts[ri].append(d.h_text + bound[ri], d.h_text + bound[ri + 1]);
                nrows[ri] += rq[ri];
            }
        }
        c0 += cn;
    }
    for (size_t ri = 0; ri < reqs.size(); ++ri) {
        out[ri].owned = std::move(texts[ri]);
        out[ri].text = out[ri].owned.data();
        out[ri].text_len = out[ri].owned.size();
        out[ri].n_rows = nrows[ri];
    }
    return kOk;
}

}  // namespace cof
