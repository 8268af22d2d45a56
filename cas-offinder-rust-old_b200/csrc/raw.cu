// raw.cu -- search()'s raw Match stream for the popcount path
// (COF_F_RAW_MATCHES): every window whose masked popcount count passes the
// threshold, as search_chunk_cpu emits it (search.rs:378-463), kept by
// convert_matches (search.rs:1428-1488), before the CLI writer's PAM filter
// and mismatch recount.  There is no PAM prefilter on this stream, so every
// window start is compared with every pattern.
//
//   raw_scan_kernel   one thread per (32 window starts, pattern): the bit4
//                     window words (N masked to 0, zero past the batch end)
//                     funnel-shifted to each start, popcount against the
//                     pattern's bit4 words; emits starts with count <= max_mm
//   raw_verify_kernel convert_matches' ownership and record-end rules
//   raw_len/raw_write Match lines: name, chrom_idx, pattern index, strand,
//                     max(count, 0), 0, 0, rna_seq, dna_seq (NUL bytes kept)
#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "cof_engine.h"
#include "engine_dev.cuh"

namespace cof {

namespace {

struct RawSeg {
    uint64_t lo, hi;       // global window starts [lo, hi)
    uint64_t base, clip;   // batch base and end
    uint64_t blk_begin;    // prefix of 32-start blocks
    uint32_t batch, pad;
};

struct RawPattern {
    uint32_t w[8];         // bit4 cells, 8 per word, zero past L (L <= 64)
    uint32_t strand, pad[3];
};

// 32-bit word of masked, clipped bit4 nibbles of nucleotides [8j, 8j + 8).
__device__ __forceinline__ uint32_t masked_word(const uint8_t *bit4, uint64_t j, uint64_t clip) {
    const uint64_t n0 = 8 * j;
    if (n0 >= clip) return 0;
    uint32_t x = __ldg(reinterpret_cast<const uint32_t *>(bit4) + j);
    if (n0 + 8 > clip) x &= (1u << (4 * (clip - n0))) - 1u;
    // genome N (0xF) -> 0 (mask_genome_n_to_zero_inplace, search.rs:512-531)
    const uint32_t t = x & (x >> 1) & (x >> 2) & (x >> 3) & 0x11111111u;
    return x & ~(t * 0xFu);
}

// NWD: pattern words compared (4: patterns of <= 32 cells, 8: <= 64)
template <int NWD>
__global__ void raw_scan_kernel(const uint8_t *__restrict__ bit4, const RawSeg *__restrict__ segs,
                                uint32_t nseg, uint64_t n_blocks, const RawPattern *__restrict__ pats,
                                uint32_t npat, uint32_t L, int max_mm, Hit *hits, uint32_t cap,
                                Counters *ctr) {
    const uint32_t nw = (L + 7) / 8;
    const uint64_t items = n_blocks * npat;
    for (uint64_t it = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; it < items;
         it += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t blk = it / npat;
        const uint32_t p = (uint32_t)(it % npat);
        uint32_t si = 0;
        while (si + 1 < nseg && blk >= segs[si + 1].blk_begin) ++si;
        const RawSeg S = segs[si];
        const uint64_t p0 = (S.lo & ~31ull) + 32 * (blk - S.blk_begin);  // 32-aligned
        uint32_t W[NWD + 5];
#pragma unroll
        for (int k = 0; k < NWD + 5; ++k) W[k] = masked_word(bit4, p0 / 8 + k, S.clip);
        const RawPattern P = pats[p];
#pragma unroll
        for (int o = 0; o < 32; ++o) {
            const uint64_t st = p0 + o;
            const int sh = 4 * (o & 7);
            int matches = 0;
#pragma unroll
            for (int j = 0; j < NWD; ++j) {
                if (j < (int)nw) {
                    const uint32_t w = __funnelshift_r(W[(o >> 3) + j], W[(o >> 3) + j + 1], sh);
                    matches += __popc(w & P.w[j]);
                }
            }
            if ((int)L - matches <= max_mm && st >= S.lo && st < S.hi) {
                const uint32_t i = atomicAdd(&ctr->hits, 1u);
                if (i < cap) hits[i] = Hit{(uint32_t)(st - S.base), p, S.batch, (uint32_t)((int)L - matches)};
                else ctr->overflow = 1;
            }
        }
    }
}

__global__ void raw_verify_kernel(GenomeDev G, const BatchDev *__restrict__ batches,
                                  const Hit *__restrict__ hits, uint32_t n_hits, uint32_t L,
                                  Row *rows, uint64_t *keys, uint32_t *vals, Counters *ctr) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_hits; i += gridDim.x * blockDim.x) {
        const Hit h = hits[i];
        const BatchDev B = batches[h.batch];
        const uint64_t sg = B.base + h.s_local;
        const uint64_t gbyte = sg >> 1;
        uint32_t lo = B.first, hi = B.first + B.nch;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (G.boff[mid] <= gbyte) lo = mid; else hi = mid;
        }
        const uint32_t k = lo;
        const uint64_t pos = G.start[k] + (sg - 2 * G.boff[k]);
        const bool end_chrom = (k == B.first + B.nch - 1) || G.start[k + 1] == 0;
        if (end_chrom && pos + L > G.end[k]) continue;
        const int kmm = (int)h.pad;
        const uint32_t r = atomicAdd(&ctr->rows, 1u);
        rows[r] = Row{sg, B.base + B.valid, pos, k, h.pattern, (uint32_t)(kmm > 0 ? kmm : 0), 0};
        keys[r] = ((uint64_t)h.pattern << 34) | sg;
        vals[r] = r;
    }
}

__global__ void raw_len_kernel(GenomeDev G, const Row *__restrict__ rows, const uint32_t *order,
                               uint32_t n, uint32_t L, uint32_t *len) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const Row w = rows[order[i]];
        const uint32_t ni = G.name_idx[w.chunk];
        len[i] = (G.name_off[ni + 1] - G.name_off[ni]) + 1 + ndigits(w.pos) + 1 +
                 ndigits(w.pattern) + 3 + ndigits(w.mm) + 5 + L + 1 + L + 1;
    }
}

__global__ void raw_write_kernel(GenomeDev G, const Row *__restrict__ rows, const uint32_t *order,
                                 uint32_t n, uint32_t L, const RawPattern *__restrict__ pats,
                                 const uint64_t *off, char *text) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const Row w = rows[order[i]];
        const RawPattern &P = pats[w.pattern];
        const bool fwd = P.strand == 0;
        char *o = text + off[i];
        const uint32_t ni = G.name_idx[w.chunk];
        for (uint32_t c = G.name_off[ni]; c < G.name_off[ni + 1]; ++c) *o++ = G.names[c];
        *o++ = '\t';
        o = put_u64(o, w.pos);
        *o++ = '\t';
        o = put_u64(o, w.pattern);
        *o++ = '\t';
        *o++ = fwd ? '+' : '-';
        *o++ = '\t';
        o = put_u64(o, w.mm);
        *o++ = '\t';
        *o++ = '0';
        *o++ = '\t';
        *o++ = '0';
        *o++ = '\t';
        char *rna = o, *dna = o + L + 1;
        for (uint32_t c = 0; c < L; ++c) {
            const uint32_t sc = fwd ? c : L - 1 - c;
            const uint64_t gi = w.s_global + sc;
            uint8_t g = gi < w.clip ? nib(G.bit4, gi) : 0;
            if (g == 0xF) g = 0;
            uint8_t p = (uint8_t)((P.w[sc >> 3] >> (4 * (sc & 7))) & 0xF);
            if (!fwd) {
                g = dcomp4(g);
                p = dcomp4(p);
            }
            rna[c] = b4char(p);
            dna[c] = b4char(g);  // NUL for N and padding, as in the reference
        }
        o += L;
        *o++ = '\t';
        o += L;
        *o++ = '\n';
    }
}

}  // namespace

int Engine::run_raw(const Request &r, Result &out, Error &err, const SearchRange &range) {
    DeviceGenome &d = *dev_;
    const HostGenome &h = host_;
    const Bit4Tables &t = bit4();
    cudaStream_t s = d.stream;
    const uint32_t L = (uint32_t)r.filter.size();
    const auto hb = make_batches(h.n_chunks(), r.cps);
    std::vector<BatchDev> batches;
    std::vector<RawSeg> segs;
    uint64_t blocks = 0;
    for (size_t bi = 0; bi < hb.size(); ++bi) {
        const HostBatch &b = hb[bi];
        BatchDev x{};
        x.base = 2 * h.boff[b.first];
        x.valid = (uint32_t)(2 * (h.boff[b.last + 1] - h.boff[b.first]));
        x.first = (uint32_t)b.first;
        x.nch = (uint32_t)(b.last - b.first + 1);
        batches.push_back(x);
        const uint64_t c1 = b.has_head ? 2 * (h.boff[b.first + 1] - h.boff[b.first]) : 0;
        const uint64_t msmin = c1 > L - 1 ? c1 - (L - 1) : 0;  // search.rs:540-546
        RawSeg sg{};
        sg.lo = std::max(x.base + msmin, range.lo);
        sg.hi = std::min<uint64_t>(x.base + x.valid, range.hi);
        if (sg.hi <= sg.lo) continue;
        sg.base = x.base;
        sg.clip = x.base + x.valid;
        sg.blk_begin = blocks;
        sg.batch = (uint32_t)bi;
        blocks += (sg.hi - (sg.lo & ~31ull) + 31) / 32;
        segs.push_back(sg);
    }
    std::vector<RawPattern> pats;
    const size_t np = r.patterns.size(), nfwd = np / 2;
    for (size_t p = 0; p < np; ++p) {
        RawPattern rp{};
        rp.strand = p >= nfwd;
        for (uint32_t c = 0; c < L; ++c)
            rp.w[c / 8] |= (uint32_t)t.str2b4[1][(uint8_t)r.patterns[p][c]] << (4 * (c % 8));
        pats.push_back(rp);
    }
    out = Result();
    if (segs.empty()) return kOk;
    TablePack tp;
    const size_t o_b = tp.add(batches), o_s = tp.add(segs), o_p = tp.add(pats);
    if (d.tables.ensure(tp.buf.size(), err)) return err.code;
    CU(cudaMemcpyAsync(d.tables.p, tp.buf.data(), tp.buf.size(), cudaMemcpyHostToDevice, s));
    auto tab = [&](size_t o) { return (const void *)(d.tables.p + o); };
    if (d.ctr.ensure(1, err)) return err.code;
    if (d.hits.cap == 0 && d.hits.ensure(1u << 22, err)) return err.code;
    Counters hc{};
    for (int attempt = 0; attempt < 2; ++attempt) {
        CU(cudaMemsetAsync(d.ctr.p, 0, sizeof(Counters), s));
        CU(cudaEventRecord(d.ev[1], s));
        const uint64_t items = blocks * np;
        const unsigned gb = (unsigned)std::max<uint64_t>(
            1, std::min<uint64_t>((items + 255) / 256, (uint64_t)d.n_sm * 16));
        auto scan_fn = L > 32 ? raw_scan_kernel<8> : raw_scan_kernel<4>;
        scan_fn<<<gb, 256, 0, s>>>(d.bit4.p, (const RawSeg *)tab(o_s), (uint32_t)segs.size(), blocks,
                                   (const RawPattern *)tab(o_p), (uint32_t)np, L, (int)r.max_mm,
                                   d.hits.p, (uint32_t)std::min<size_t>(d.hits.cap, 0xFFFFFFF0u),
                                   d.ctr.p);
        CU(cudaGetLastError());
        CU(cudaEventRecord(d.ev[2], s));
        ++times_.kernel_launches;
        CU(cudaMemcpyAsync(&hc, d.ctr.p, sizeof(Counters), cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        if (!hc.overflow && hc.hits <= d.hits.cap) break;
        if (attempt == 1) {
            err = {kOom, "raw match buffer overflow after resize"};
            return err.code;
        }
        if (d.hits.ensure((size_t)hc.hits + hc.hits / 4 + 1024, err)) return err.code;
    }
    float ms = 0;
    cudaEventElapsedTime(&ms, d.ev[1], d.ev[2]);
    times_.scan_ms += ms;
    times_.raw_hits += hc.hits;
    const uint32_t n_hits = hc.hits;
    if (d.rows.ensure(n_hits + 1, err) || d.keys.ensure(n_hits + 1, err) ||
        d.keys2.ensure(n_hits + 1, err) || d.vals.ensure(n_hits + 1, err) ||
        d.vals2.ensure(n_hits + 1, err) || d.lens.ensure(n_hits + 1, err) ||
        d.offs.ensure(n_hits + 1, err))
        return err.code;
    if (n_hits) {
        const unsigned vb = (unsigned)std::min<uint64_t>((n_hits + 255) / 256, (uint64_t)d.n_sm * 8);
        raw_verify_kernel<<<vb, 256, 0, s>>>(d.view(), (const BatchDev *)tab(o_b), d.hits.p, n_hits,
                                             L, d.rows.p, d.keys.p, d.vals.p, d.ctr.p);
        CU(cudaGetLastError());
        ++times_.kernel_launches;
    }
    CU(cudaMemcpyAsync(&hc, d.ctr.p, sizeof(Counters), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    const uint32_t nr = hc.rows;
    times_.rows += nr;
    if (!nr) return kOk;
    size_t tmp = 0, tmp2 = 0;
    CU(cub::DeviceRadixSort::SortPairs(nullptr, tmp, d.keys.p, d.keys2.p, d.vals.p, d.vals2.p,
                                       (int)nr, 0, 64, s));
    CU(cub::DeviceScan::ExclusiveSum(nullptr, tmp2, d.lens.p, d.offs.p, (int)nr + 1, s));
    if (d.cub_tmp.ensure(std::max(tmp, tmp2), err)) return err.code;
    tmp = d.cub_tmp.cap;
    CU(cub::DeviceRadixSort::SortPairs(d.cub_tmp.p, tmp, d.keys.p, d.keys2.p, d.vals.p, d.vals2.p,
                                       (int)nr, 0, 64, s));
    const unsigned fb = (unsigned)std::min<uint64_t>((nr + 255) / 256, (uint64_t)d.n_sm * 8);
    raw_len_kernel<<<fb, 256, 0, s>>>(d.view(), d.rows.p, d.vals2.p, nr, L, d.lens.p);
    CU(cudaGetLastError());
    CU(cudaMemsetAsync(d.lens.p + nr, 0, 4, s));
    tmp2 = d.cub_tmp.cap;
    CU(cub::DeviceScan::ExclusiveSum(d.cub_tmp.p, tmp2, d.lens.p, d.offs.p, (int)nr + 1, s));
    uint64_t bytes = 0;
    CU(cudaMemcpyAsync(&bytes, d.offs.p + nr, 8, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    if (d.text.ensure(bytes + 1, err)) return err.code;
    raw_write_kernel<<<fb, 256, 0, s>>>(d.view(), d.rows.p, d.vals2.p, nr, L,
                                        (const RawPattern *)tab(o_p), d.offs.p, d.text.p);
    CU(cudaGetLastError());
    times_.kernel_launches += 4;
    out.owned.resize(bytes);
    CU(cudaMemcpyAsync(&out.owned[0], d.text.p, bytes, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    out.text = out.owned.data();
    out.text_len = bytes;
    out.n_rows = nr;
    return kOk;
}

}  // namespace cof
