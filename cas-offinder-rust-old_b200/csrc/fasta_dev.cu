// fasta_dev.cu -- the bases of a FASTA genome converted on the device at
// upload (read_fasta.rs:9-71, the per-chunk conversion; genome characters
// through the mixed-base map of bit4ops.rs:17-47).
//
// The host has already decided the chunks (loader.cpp, index_fasta): each
// chunk is a range of the file's lines with a bit4 byte offset.  Here the
// whole file is copied to the device, and
//   1. nl_count_kernel / nl_write_kernel list the positions of every '\n'
//      (per-block counts, an exclusive scan, then positions in order);
//   2. line_kernel gives every line its length (one '\r' before its '\n'
//      dropped), finds the chunk that holds it (headers count as length 0)
//      and an exclusive scan by chunk gives each line's nucleotide offset in
//      its chunk;
//   3. convert_kernel writes each line's nibbles into the zeroed bit4 stream
//      with 32-bit atomicOr (two lines may share a byte when a line has an
//      odd length).
// A line that would end past its chunk's size (the file changed after it was
// read) is not written; the upload then fails with an error.
#include <cub/cub.cuh>

#include <algorithm>

#include "cof_engine.h"
#include "engine_dev.cuh"

namespace cof {

namespace {

constexpr uint32_t kBlockBytes = 65536;  // file bytes per newline-scan block
constexpr int kScanThreads = 256;        // 256 bytes per thread

__device__ __forceinline__ uint32_t count_nl(uint4 q) {
    const uint32_t nl = 0x0A0A0A0Au;
    return (__popc(__vcmpeq4(q.x, nl)) + __popc(__vcmpeq4(q.y, nl)) + __popc(__vcmpeq4(q.z, nl)) +
            __popc(__vcmpeq4(q.w, nl))) >> 3;
}

// Bytes past the file end are zero (padding), so every thread reads whole
// 256-byte ranges.
__global__ void __launch_bounds__(kScanThreads)
nl_count_kernel(const uint8_t *__restrict__ R, unsigned long long *__restrict__ cnt) {
    const uint4 *q = reinterpret_cast<const uint4 *>(R + (uint64_t)blockIdx.x * kBlockBytes) +
                     threadIdx.x * 16;
    uint32_t c = 0;
#pragma unroll 4
    for (int k = 0; k < 16; ++k) c += count_nl(q[k]);
    using BR = cub::BlockReduce<uint32_t, kScanThreads>;
    __shared__ typename BR::TempStorage tmp;
    const uint32_t tot = BR(tmp).Sum(c);
    if (threadIdx.x == 0) cnt[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(kScanThreads)
nl_write_kernel(const uint8_t *__restrict__ R, const unsigned long long *__restrict__ boff,
                uint64_t *__restrict__ nlpos) {
    const uint64_t base = (uint64_t)blockIdx.x * kBlockBytes + threadIdx.x * 256u;
    const uint4 *q = reinterpret_cast<const uint4 *>(R + base);
    uint32_t c = 0;
#pragma unroll 4
    for (int k = 0; k < 16; ++k) c += count_nl(q[k]);
    using BS = cub::BlockScan<uint32_t, kScanThreads>;
    __shared__ typename BS::TempStorage tmp;
    uint32_t o = 0;
    BS(tmp).ExclusiveSum(c, o);
    if (!c) return;
    uint64_t w = boff[blockIdx.x] + o;
    for (int k = 0; k < 16; ++k) {
        const uint4 v = q[k];
        const uint32_t x[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            uint32_t m = __vcmpeq4(x[j], 0x0A0A0A0Au) & 0x01010101u;
            while (m) {
                const int b = (__ffs(m) - 1) >> 3;
                nlpos[w++] = base + 16u * k + 4u * j + b;
                m &= m - 1;
            }
        }
    }
}

struct LineArgs {
    const uint8_t *R;
    uint64_t n;
    const uint64_t *nlpos;
    uint64_t n_nl, n_lines;
    const uint64_t *first_line, *last_line;
    uint32_t n_chunks;
};

__device__ __forceinline__ void line_span(const LineArgs &A, uint64_t i, uint64_t &start,
                                          uint32_t &len, bool &hdr) {
    start = i ? A.nlpos[i - 1] + 1 : 0;
    const bool has_nl = i < A.n_nl;
    const uint64_t end = has_nl ? A.nlpos[i] : A.n;
    uint64_t l = end - start;
    if (has_nl && l && A.R[end - 1] == '\r') --l;
    hdr = l >= 1 && A.R[start] == '>';
    len = l > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)l;
}

// per line: the chunk that holds it (key) and its length in that chunk
__global__ void line_kernel(LineArgs A, uint32_t *__restrict__ key, uint32_t *__restrict__ val) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < A.n_lines;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t start;
        uint32_t len;
        bool hdr;
        line_span(A, i, start, len, hdr);
        // last chunk whose first line is <= i
        uint32_t lo = 0, hi = A.n_chunks;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (A.first_line[mid] <= i) lo = mid + 1; else hi = mid;
        }
        const bool in = lo > 0 && i < A.last_line[lo - 1] && !hdr;
        key[i] = lo == 0 ? 0xFFFFFFFFu : lo - 1;
        val[i] = in ? len : 0u;
    }
}

__global__ void convert_kernel(LineArgs A, const uint32_t *__restrict__ key,
                               const uint32_t *__restrict__ val, const uint32_t *__restrict__ off,
                               const uint64_t *__restrict__ out, const uint32_t *__restrict__ chunk_nt,
                               const uint8_t *__restrict__ map, uint32_t *__restrict__ words,
                               uint32_t *__restrict__ bad) {
    __shared__ uint8_t m[256];
    for (int k = threadIdx.x; k < 256; k += blockDim.x) m[k] = map[k];
    __syncthreads();
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < A.n_lines;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t len = val[i];
        if (!len) continue;
        const uint32_t c = key[i];
        if (c >= A.n_chunks || (uint64_t)off[i] + len > chunk_nt[c]) {
            atomicOr(bad, 1u);
            continue;
        }
        const uint64_t start = i ? A.nlpos[i - 1] + 1 : 0;
        const uint64_t p0 = 2 * out[c] + off[i];  // nibble index of the first base
        uint32_t acc = 0;
        for (uint32_t j = 0; j < len; ++j) {
            const uint64_t p = p0 + j;
            acc |= (uint32_t)m[A.R[start + j]] << (4 * (p & 7));
            if ((p & 7) == 7 || j + 1 == len) {
                if (acc) atomicOr(words + (p >> 3), acc);
                acc = 0;
            }
        }
    }
}

struct FaScratch {
    DevBuf<uint8_t> raw;
    DevBuf<unsigned long long> cnt, boff;
    DevBuf<uint64_t> nlpos, first, last, out;
    DevBuf<uint32_t> key, val, off, chunk_nt, bad;
    DevBuf<uint8_t> map, tmp;
    ~FaScratch() {
        raw.release();
        cnt.release();
        boff.release();
        nlpos.release();
        first.release();
        last.release();
        out.release();
        key.release();
        val.release();
        off.release();
        chunk_nt.release();
        bad.release();
        map.release();
        tmp.release();
    }
};

}  // namespace

int upload_fasta(const FastaPlan &plan, uint8_t *dst, uint64_t dst_bytes, int device,
                 cudaStream_t s, Error &err) {
    const uint32_t n_chunks = (uint32_t)plan.first_line.size();
    if (n_chunks == 0) return kOk;
    const uint64_t n = plan.file_bytes;
    const uint64_t n_blocks = (n + kBlockBytes - 1) / kBlockBytes;
    FaScratch sc;
    if (sc.raw.ensure(n_blocks * kBlockBytes, err) || sc.cnt.ensure(n_blocks + 1, err) ||
        sc.boff.ensure(n_blocks + 1, err))
        return err.code;
    CU(cudaMemsetAsync(sc.raw.p + n, 0, n_blocks * kBlockBytes - n, s));
    CU(cudaStreamSynchronize(s));
    if (copy_file_to_device(plan.path, n, 0, n, sc.raw.p, device, err)) return err.code;

    // 1. newline positions
    nl_count_kernel<<<(unsigned)n_blocks, kScanThreads, 0, s>>>(sc.raw.p, sc.cnt.p);
    CU(cudaGetLastError());
    CU(cudaMemsetAsync(sc.cnt.p + n_blocks, 0, sizeof(unsigned long long), s));
    size_t tb = 0;
    CU(cub::DeviceScan::ExclusiveSum(nullptr, tb, sc.cnt.p, sc.boff.p, (int)(n_blocks + 1), s));
    if (sc.tmp.ensure(tb, err)) return err.code;
    tb = sc.tmp.cap;
    CU(cub::DeviceScan::ExclusiveSum(sc.tmp.p, tb, sc.cnt.p, sc.boff.p, (int)(n_blocks + 1), s));
    unsigned long long n_nl = 0;
    uint8_t last = 0;
    CU(cudaMemcpyAsync(&n_nl, sc.boff.p + n_blocks, 8, cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(&last, sc.raw.p + n - 1, 1, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    const uint64_t n_lines = n_nl + (last != '\n' ? 1 : 0);
    if (n_lines != plan.n_lines) {
        err = {kIo, plan.path + " changed since it was loaded"};
        return err.code;
    }
    if (sc.nlpos.ensure(std::max<uint64_t>(n_nl, 1), err)) return err.code;
    nl_write_kernel<<<(unsigned)n_blocks, kScanThreads, 0, s>>>(sc.raw.p, sc.boff.p, sc.nlpos.p);
    CU(cudaGetLastError());

    // 2. chunk and offset of every line
    if (sc.first.ensure(n_chunks, err) || sc.last.ensure(n_chunks, err) ||
        sc.out.ensure(n_chunks, err) || sc.chunk_nt.ensure(n_chunks, err) ||
        sc.key.ensure(n_lines, err) || sc.val.ensure(n_lines, err) ||
        sc.off.ensure(n_lines, err) || sc.bad.ensure(1, err) || sc.map.ensure(256, err))
        return err.code;
    CU(cudaMemcpyAsync(sc.first.p, plan.first_line.data(), n_chunks * 8, cudaMemcpyHostToDevice, s));
    CU(cudaMemcpyAsync(sc.last.p, plan.last_line.data(), n_chunks * 8, cudaMemcpyHostToDevice, s));
    CU(cudaMemcpyAsync(sc.out.p, plan.out.data(), n_chunks * 8, cudaMemcpyHostToDevice, s));
    CU(cudaMemcpyAsync(sc.chunk_nt.p, plan.nt.data(), n_chunks * 4, cudaMemcpyHostToDevice, s));
    CU(cudaMemcpyAsync(sc.map.p, bit4().str2b4[1], 256, cudaMemcpyHostToDevice, s));
    CU(cudaMemsetAsync(sc.bad.p, 0, 4, s));
    LineArgs A{sc.raw.p, n, sc.nlpos.p, n_nl, n_lines, sc.first.p, sc.last.p, n_chunks};
    const unsigned lb = (unsigned)std::min<uint64_t>((n_lines + 255) / 256, 1u << 20);
    line_kernel<<<lb, 256, 0, s>>>(A, sc.key.p, sc.val.p);
    CU(cudaGetLastError());
    tb = 0;
    CU(cub::DeviceScan::ExclusiveSumByKey(nullptr, tb, sc.key.p, sc.val.p, sc.off.p,
                                          (int64_t)n_lines, cub::Equality(), s));
    if (sc.tmp.ensure(tb, err)) return err.code;
    tb = sc.tmp.cap;
    CU(cub::DeviceScan::ExclusiveSumByKey(sc.tmp.p, tb, sc.key.p, sc.val.p, sc.off.p,
                                          (int64_t)n_lines, cub::Equality(), s));

    // 3. nibbles into the zeroed bit4 stream
    if (plan.out.back() + (plan.nt.back() + 1) / 2 > dst_bytes) {
        err = {kBadInput, "bit4 buffer smaller than the planned chunks"};
        return err.code;
    }
    convert_kernel<<<lb, 256, 0, s>>>(A, sc.key.p, sc.val.p, sc.off.p, sc.out.p, sc.chunk_nt.p,
                                      sc.map.p, reinterpret_cast<uint32_t *>(dst), sc.bad.p);
    CU(cudaGetLastError());
    uint32_t bad = 0;
    CU(cudaMemcpyAsync(&bad, sc.bad.p, 4, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));  // the scratch buffers are freed on return
    if (bad) {
        err = {kIo, plan.path + " changed since it was loaded"};
        return err.code;
    }
    return kOk;
}

}  // namespace cof
