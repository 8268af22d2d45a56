// Launcher for the reference's own CUDA kernels -- test and measurement
// infrastructure only (interface and deviations: ref_gpu.h).  Host code
// only: the kernels are the reference's kernel.cu / kernel_myers.cu, built
// unmodified into cubins by `make -C oracle ref` and loaded at run time, the
// way search.rs loads its NVRTC PTX (search.rs:260-261, :1069-1070).
#include "ref_gpu.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace {

constexpr uint64_t kChunkNucl = 65536;         // read_fasta.rs CHUNK_SIZE
constexpr uint32_t kGpuCps = 16384;            // 1 Gnt batch (search.rs:22, :44-50)
constexpr uint32_t kBlockX = 128;              // launch_cfg_2d (search.rs:240-247)
constexpr size_t kDevicePad = 256;             // see ref_gpu.h

double now_ms() {
    return std::chrono::duration<double, std::milli>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

void set_err(char *err, size_t n, const std::string &s) {
    if (err && n) {
        std::snprintf(err, n, "%s", s.c_str());
    }
}

struct CudaFail {
    std::string what;
};

void ck(cudaError_t e, const char *what) {
    if (e != cudaSuccess) {
        throw CudaFail{std::string(what) + ": " + cudaGetErrorString(e)};
    }
}

// STR_2_BIT4[mixed_base = true] of bit4ops.rs: one-hot T=1 C=2 A=4 G=8,
// IUPAC letters the union of their bases, N = 0xF, anything else 0.
struct Bit4 {
    uint8_t v[256];
    Bit4() {
        std::memset(v, 0, sizeof v);
        const char *keys = "TCAGRYSWKMBDHVN";
        const uint8_t vals[] = {1, 2, 4, 8, 12, 3, 10, 5, 9, 6, 11, 13, 7, 14, 15};
        for (int i = 0; keys[i]; i++) {
            v[(uint8_t)keys[i]] = vals[i];
            v[(uint8_t)(keys[i] + 32)] = vals[i];
        }
    }
};
const Bit4 kB4;

// compliment_char (bit4ops.rs): swap A/T, C/G and the IUPAC pairs, keep case
char comp_char(char c) {
    static const char *from = "ACGTRYKMBVDHSWNacgtrykmbvdhswn";
    static const char *to = "TGCAYRMKVBHDSWNtgcayrmkvbhdswn";
    const char *p = std::strchr(from, c);
    return (p && c) ? to[p - from] : c;
}

// string_to_bit4(.., mixed_base = true): character i in byte i/2, even
// characters in the low nibble.
void to_bit4(uint8_t *out, const char *s, size_t n) {
    for (size_t i = 0; i < n; i++) {
        out[i / 2] |= (uint8_t)(kB4.v[(uint8_t)s[i]] << ((i & 1) * 4));
    }
}

struct Batch {
    size_t first, n;
    bool head;
};

struct Launch {
    cudaKernel_t fn = nullptr;
    cudaLibrary_t lib = nullptr;
    Launch(const char *cubin, const char *name) {
        ck(cudaLibraryLoadFromFile(&lib, cubin, nullptr, nullptr, 0, nullptr, nullptr, 0),
           "load cubin");
        ck(cudaLibraryGetKernel(&fn, lib, name), "find kernel");
    }
    ~Launch() {
        if (lib) {
            cudaLibraryUnload(lib);
        }
    }
};

}  // namespace

struct refgpu_ctx {
    const uint8_t *const *data;
    const uint64_t *start, *end;
    size_t n_chunks;
    uint32_t cps;
    size_t max_bytes;           // search_chunk_bytes()
    std::vector<Batch> batches;
    std::vector<uint8_t> host;  // the batch's tight-packed buffer
    std::vector<uint32_t> offs; // chunk_byte_offsets of the current batch
    uint8_t *d_genome = nullptr;
    // the legacy default stream: every kernel is ordered after the
    // synchronous pageable copies before it
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;

    // chunks_to_searchchunk (search.rs:1376-1427): tight-pack the batch's
    // chunks, ceil(len/2) bytes each, with a byte-offset sentinel.
    double pack(const Batch &b, bool mask_n) {
        double t0 = now_ms();
        offs.clear();
        size_t cur = 0;
        for (size_t k = b.first; k < b.first + b.n; k++) {
            size_t bytes = (size_t)((end[k] - start[k] + 1) / 2);
            offs.push_back((uint32_t)cur);
            std::memcpy(host.data() + cur, data[k], bytes);
            cur += bytes;
        }
        offs.push_back((uint32_t)cur);
        if (mask_n) {
            // mask_genome_n_to_zero_inplace (search.rs:512-531): nibbles equal
            // to 0xF become 0; the buffer past `cur` is not copied.
            for (size_t i = 0; i < cur; i++) {
                uint8_t x = host[i];
                if ((x & 0x0F) == 0x0F) x &= 0xF0;
                if ((x & 0xF0) == 0xF0) x &= 0x0F;
                host[i] = x;
            }
        }
        return now_ms() - t0;
    }

    void upload(refgpu_times *t) {
        double t0 = now_ms();
        ck(cudaMemcpy(d_genome, host.data(), offs.back(), cudaMemcpyHostToDevice), "batch H2D");
        t->h2d_ms += now_ms() - t0;
    }

    double timed_launch(const void *fn, dim3 grid, void **args) {
        ck(cudaEventRecord(ev0, stream), "event");
        ck(cudaLaunchKernel(fn, grid, dim3(kBlockX), args, 0, stream), "launch");
        ck(cudaEventRecord(ev1, stream), "event");
        ck(cudaEventSynchronize(ev1), "kernel");
        float ms = 0;
        ck(cudaEventElapsedTime(&ms, ev0, ev1), "elapsed");
        return ms;
    }
};

extern "C" {

refgpu_ctx *refgpu_open(const uint8_t *const *chunk_data, const uint64_t *chunk_start,
                        const uint64_t *chunk_end, size_t n_chunks, uint32_t chunks_per_search,
                        int device, char *err, size_t errlen) {
    auto *c = new refgpu_ctx();
    c->data = chunk_data;
    c->start = chunk_start;
    c->end = chunk_end;
    c->n_chunks = n_chunks;
    c->cps = chunks_per_search ? chunks_per_search : kGpuCps;
    c->max_bytes = (size_t)c->cps * kChunkNucl / 2;
    for (size_t k = 0; k < n_chunks; k++) {
        if (chunk_end[k] < chunk_start[k] || chunk_end[k] - chunk_start[k] > kChunkNucl) {
            set_err(err, errlen, "chunk longer than 65536 nt");
            delete c;
            return nullptr;
        }
    }
    // batcher (search.rs:1531-1572): cps chunks per batch; every later batch
    // starts with the previous batch's last chunk as head overlap, and a
    // lone head chunk at the end is not re-emitted.
    size_t first = 0, len = 0;
    bool head = false;
    for (size_t k = 0; k < n_chunks; k++) {
        if (len == 0) first = k;
        len++;
        if (len == c->cps) {
            c->batches.push_back({first, len, head});
            first = k;
            len = 1;
            head = true;
        }
    }
    if (len && !(head && len == 1)) {
        c->batches.push_back({first, len, head});
    }
    try {
        ck(cudaSetDevice(device), "set device");
        c->host.assign(c->max_bytes, 0);
        ck(cudaMalloc(&c->d_genome, c->max_bytes + kDevicePad), "genome buffer");
        ck(cudaMemset(c->d_genome, 0, c->max_bytes + kDevicePad), "genome zero");
        ck(cudaEventCreate(&c->ev0), "event");
        ck(cudaEventCreate(&c->ev1), "event");
        ck(cudaDeviceSynchronize(), "sync");
    } catch (const CudaFail &f) {
        set_err(err, errlen, f.what);
        refgpu_close(c);
        return nullptr;
    }
    return c;
}

size_t refgpu_n_batches(const refgpu_ctx *c) { return c->batches.size(); }

void refgpu_batch(const refgpu_ctx *c, size_t b, size_t *first, size_t *n, int *head) {
    *first = c->batches[b].first;
    *n = c->batches[b].n;
    *head = c->batches[b].head ? 1 : 0;
}

void refgpu_close(refgpu_ctx *c) {
    if (!c) return;
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->d_genome) cudaFree(c->d_genome);
    delete c;
}

}  // extern "C"

namespace {

// Popcount pattern table: string_to_bit4 per pattern (search.rs:1516-1523)
// then pack_patterns (search.rs:465-477): each pattern's ceil(L/2) bytes
// padded with zeros to a multiple of PATTERN_CHUNK_SIZE = 16 bytes.
std::vector<uint8_t> popcount_patterns(const char *const *pats, size_t n, size_t L) {
    size_t stride = (L + 1) / 2;
    stride = (stride + 15) / 16 * 16;
    std::vector<uint8_t> out(n * stride, 0);
    for (size_t p = 0; p < n; p++) {
        to_bit4(out.data() + p * stride, pats[p], L);
    }
    return out;
}

struct PopArgs {
    const uint32_t *genome;
    const uint32_t *patterns;
    uint32_t max_mm, msmin, n_execs, n_pat;
    refgpu_pmatch *out;
    int *count;
    void *v[8];
    void bind() {
        v[0] = &genome; v[1] = &patterns; v[2] = &max_mm; v[3] = &msmin;
        v[4] = &n_execs; v[5] = &n_pat; v[6] = &out; v[7] = &count;
    }
};

// legacy_match_start_min_nucl (search.rs:540-546)
uint32_t start_min(const refgpu_ctx *c, const Batch &b, size_t L) {
    if (!b.head) return 0;
    uint64_t s1 = (uint64_t)c->offs[1] * 2;
    return (uint32_t)(s1 > L - 1 ? s1 - (L - 1) : 0);
}

int check_patterns(const char *const *pats, size_t n, size_t &L, char *err, size_t errlen) {
    if (n == 0) {
        set_err(err, errlen, "no patterns");
        return -1;
    }
    L = std::strlen(pats[0]);
    for (size_t p = 0; p < n; p++) {
        if (std::strlen(pats[p]) != L) {
            set_err(err, errlen, "All patterns must have same length");
            return -1;
        }
    }
    if (L == 0 || L > 32) {
        set_err(err, errlen, "pattern length must be 1..32 for these cubins");
        return -1;
    }
    return 0;
}

}  // namespace

extern "C" {

int refgpu_popcount_count(refgpu_ctx *c, const char *cubin, const char *const *patterns,
                          size_t n_patterns, uint32_t max_mismatches, uint64_t count_cap,
                          uint64_t *batch_counts, char *err, size_t errlen) {
    size_t L;
    if (check_patterns(patterns, n_patterns, L, err, errlen)) return -1;
    uint64_t per_exec = 32ull * n_patterns;  // 4 blocks x 8 shifts per thread and pattern
    uint64_t sub_max = count_cap / per_exec;
    if (sub_max == 0) {
        set_err(err, errlen, "count_cap below one thread column of matches");
        return -1;
    }
    uint32_t *d_pat = nullptr;
    refgpu_pmatch *d_out = nullptr;
    int *d_count = nullptr;
    int rc = 0;
    try {
        Launch k(cubin, "find_matches");
        std::vector<uint8_t> pat = popcount_patterns(patterns, n_patterns, L);
        ck(cudaMalloc(&d_pat, pat.size()), "patterns");
        ck(cudaMemcpy(d_pat, pat.data(), pat.size(), cudaMemcpyHostToDevice), "patterns H2D");
        // every launch below has at most sub_max * per_exec <= count_cap
        // possible appends, so the buffer cannot overflow
        ck(cudaMalloc(&d_out, count_cap * sizeof(refgpu_pmatch)), "match buffer");
        ck(cudaMalloc(&d_count, sizeof(int)), "counter");
        refgpu_times scratch{};
        for (size_t bi = 0; bi < c->batches.size(); bi++) {
            const Batch &b = c->batches[bi];
            c->pack(b, true);
            c->upload(&scratch);
            uint32_t n_execs = c->offs.back() / 4 / 4;
            uint32_t msmin = start_min(c, b, L);
            uint64_t total = 0;
            for (uint64_t e0 = 0; e0 < n_execs; e0 += sub_max) {
                PopArgs a;
                a.genome = reinterpret_cast<const uint32_t *>(c->d_genome) + e0 * 4;
                a.patterns = d_pat;
                a.max_mm = max_mismatches;
                a.msmin = msmin > e0 * 32 ? (uint32_t)(msmin - e0 * 32) : 0;
                a.n_execs = (uint32_t)std::min<uint64_t>(sub_max, n_execs - e0);
                a.n_pat = (uint32_t)n_patterns;
                a.out = d_out;
                a.count = d_count;
                a.bind();
                ck(cudaMemsetAsync(d_count, 0, sizeof(int), c->stream), "counter zero");
                dim3 grid((a.n_execs + kBlockX - 1) / kBlockX, (uint32_t)n_patterns);
                c->timed_launch((const void *)k.fn, grid, a.v);
                int cnt = 0;
                ck(cudaMemcpy(&cnt, d_count, sizeof(int), cudaMemcpyDeviceToHost), "count D2H");
                total += (uint64_t)std::max(cnt, 0);
            }
            batch_counts[bi] = total;
        }
    } catch (const CudaFail &f) {
        set_err(err, errlen, f.what);
        rc = -1;
    }
    cudaFree(d_pat);
    cudaFree(d_out);
    cudaFree(d_count);
    return rc;
}

int refgpu_popcount_run(refgpu_ctx *c, const char *cubin, const char *const *patterns,
                        size_t n_patterns, uint32_t max_mismatches, uint64_t capacity,
                        const uint64_t *batch_counts, refgpu_pmatch *out, uint64_t out_cap,
                        uint64_t *batch_offsets, refgpu_times *t, char *err, size_t errlen) {
    size_t L;
    if (check_patterns(patterns, n_patterns, L, err, errlen)) return -1;
    for (size_t bi = 0; bi < c->batches.size(); bi++) {
        if (batch_counts[bi] > capacity) {
            set_err(err, errlen, "capacity below a batch's match count");
            return -1;
        }
    }
    *t = refgpu_times{};
    uint32_t *d_pat = nullptr;
    refgpu_pmatch *d_out = nullptr;
    int *d_count = nullptr;
    int rc = 0;
    try {
        Launch k(cubin, "find_matches");
        std::vector<uint8_t> pat = popcount_patterns(patterns, n_patterns, L);
        ck(cudaMalloc(&d_pat, pat.size()), "patterns");
        ck(cudaMemcpy(d_pat, pat.data(), pat.size(), cudaMemcpyHostToDevice), "patterns H2D");
        ck(cudaMalloc(&d_out, std::max<uint64_t>(capacity, 1) * sizeof(refgpu_pmatch)),
           "match buffer");
        ck(cudaMalloc(&d_count, sizeof(int)), "counter");
        std::vector<refgpu_pmatch> host_out;
        uint64_t n_out = 0;
        double w0 = now_ms();
        for (size_t bi = 0; bi < c->batches.size(); bi++) {
            const Batch &b = c->batches[bi];
            if (batch_offsets) batch_offsets[bi] = n_out;
            t->host_ms += c->pack(b, true);
            c->upload(t);
            double h0 = now_ms();
            int zero = 0;
            ck(cudaMemcpy(d_count, &zero, sizeof(int), cudaMemcpyHostToDevice), "counter H2D");
            t->h2d_ms += now_ms() - h0;
            PopArgs a;
            a.genome = reinterpret_cast<const uint32_t *>(c->d_genome);
            a.patterns = d_pat;
            a.max_mm = max_mismatches;
            a.msmin = start_min(c, b, L);
            a.n_execs = c->offs.back() / 4 / 4;  // search.rs:280-284
            a.n_pat = (uint32_t)n_patterns;
            a.out = d_out;
            a.count = d_count;
            a.bind();
            if (a.n_execs == 0) continue;  // an empty grid is not a valid launch
            dim3 grid((a.n_execs + kBlockX - 1) / kBlockX, (uint32_t)n_patterns);
            t->kernel_ms += c->timed_launch((const void *)k.fn, grid, a.v);
            t->launches++;
            double d0 = now_ms();
            int cnt = 0;
            ck(cudaMemcpy(&cnt, d_count, sizeof(int), cudaMemcpyDeviceToHost), "count D2H");
            uint64_t n = (uint64_t)std::max(cnt, 0);
            if (n != batch_counts[bi]) {
                throw CudaFail{"batch match count differs from the counting pass"};
            }
            if (n) {
                host_out.resize(n);
                ck(cudaMemcpy(host_out.data(), d_out, n * sizeof(refgpu_pmatch),
                              cudaMemcpyDeviceToHost),
                   "matches D2H");
            }
            t->d2h_ms += now_ms() - d0;
            if (out) {
                if (n_out + n > out_cap) throw CudaFail{"out_cap too small"};
                std::memcpy(out + n_out, host_out.data(), n * sizeof(refgpu_pmatch));
            }
            n_out += n;
        }
        if (batch_offsets) batch_offsets[c->batches.size()] = n_out;
        t->wall_ms = now_ms() - w0;
        t->n_batches = c->batches.size();
        t->matches = n_out;
    } catch (const CudaFail &f) {
        set_err(err, errlen, f.what);
        rc = -1;
    }
    cudaFree(d_pat);
    cudaFree(d_out);
    cudaFree(d_count);
    return rc;
}

int refgpu_myers_run(refgpu_ctx *c, const char *cubin, const char *search_filter,
                     const char *const *patterns, size_t n_patterns, size_t n_fwd_patterns,
                     uint32_t out_buf_size, refgpu_mmatch *out, uint64_t out_cap,
                     uint64_t *batch_offsets, refgpu_times *t, char *err, size_t errlen) {
    size_t L;
    if (check_patterns(patterns, n_patterns, L, err, errlen)) return -1;
    if (std::strlen(search_filter) != L) {
        set_err(err, errlen, "filter length differs from the patterns");
        return -1;
    }
    *t = refgpu_times{};
    // search_chunk_cuda_myers (search.rs:1189-1262): Peq tables (myers.rs
    // build_peq: A C G T N words, non-ACGT cells match every base and set
    // the N word), PAM precheck offsets and filters (precompute_pam_precheck,
    // search.rs:761-777, filters padded with 0xFF to the longest), bit4
    // patterns of ceil(L/2) bytes.
    std::vector<uint64_t> peq(n_patterns * 5, 0);
    std::vector<uint8_t> pam_off(n_patterns);
    std::vector<std::vector<uint8_t>> pam_f(n_patterns);
    std::string rfilt(search_filter);
    std::reverse(rfilt.begin(), rfilt.end());
    for (char &ch : rfilt) ch = comp_char(ch);
    size_t pam_len = 0;
    size_t pbytes = (L + 1) / 2;
    std::vector<uint8_t> pat_b4(n_patterns * pbytes, 0);
    for (size_t p = 0; p < n_patterns; p++) {
        const char *s = patterns[p];
        const char *eff = p < n_fwd_patterns ? search_filter : rfilt.c_str();
        size_t first_n = L;
        for (size_t i = 0; i < L; i++) {
            char u = (char)(s[i] & ~32);
            int idx = u == 'A' ? 0 : u == 'C' ? 1 : u == 'G' ? 2 : u == 'T' ? 3 : 4;
            if (idx < 4) {
                peq[p * 5 + idx] |= 1ull << i;
            } else {
                for (int q = 0; q < 4; q++) peq[p * 5 + q] |= 1ull << i;
                peq[p * 5 + 4] |= 1ull << i;
            }
            bool is_n = s[i] == 'N' || s[i] == 'n';
            if (is_n && first_n == L) first_n = i;
            if (is_n) pam_f[p].push_back(kB4.v[(uint8_t)eff[i]]);
        }
        // the kernel indexes the filter table by (cell - first N cell)
        // (kernel_myers.cu:297-298), which stays inside the table only when a
        // pattern's N cells are contiguous
        if (first_n + pam_f[p].size() > L ||
            std::any_of(s + first_n, s + first_n + pam_f[p].size(),
                        [](char ch) { return ch != 'N' && ch != 'n'; })) {
            set_err(err, errlen, "pattern N cells must be one contiguous run");
            return -1;
        }
        pam_off[p] = (uint8_t)first_n;
        pam_len = std::max(pam_len, pam_f[p].size());
        to_bit4(pat_b4.data() + p * pbytes, s, L);
    }
    std::vector<uint8_t> pam_flat;
    for (size_t p = 0; p < n_patterns; p++) {
        pam_flat.insert(pam_flat.end(), pam_f[p].begin(), pam_f[p].end());
        pam_flat.resize(pam_flat.size() + (pam_len - pam_f[p].size()), 0xFF);
    }
    if (pam_flat.empty()) pam_flat.push_back(0xFF);

    uint64_t *d_peq = nullptr;
    uint8_t *d_pat = nullptr, *d_off = nullptr, *d_filt = nullptr;
    refgpu_mmatch *d_out = nullptr;
    uint32_t *d_count = nullptr;
    int rc = 0;
    try {
        Launch k(cubin, "find_matches_myers");
        ck(cudaMalloc(&d_peq, peq.size() * 8), "peq");
        ck(cudaMalloc(&d_pat, pat_b4.size()), "patterns");
        ck(cudaMalloc(&d_off, pam_off.size()), "pam offsets");
        ck(cudaMalloc(&d_filt, pam_flat.size()), "pam filters");
        ck(cudaMemcpy(d_peq, peq.data(), peq.size() * 8, cudaMemcpyHostToDevice), "H2D");
        ck(cudaMemcpy(d_pat, pat_b4.data(), pat_b4.size(), cudaMemcpyHostToDevice), "H2D");
        ck(cudaMemcpy(d_off, pam_off.data(), pam_off.size(), cudaMemcpyHostToDevice), "H2D");
        ck(cudaMemcpy(d_filt, pam_flat.data(), pam_flat.size(), cudaMemcpyHostToDevice), "H2D");
        ck(cudaMalloc(&d_out, (size_t)out_buf_size * sizeof(refgpu_mmatch)), "match buffer");
        ck(cudaMalloc(&d_count, sizeof(uint32_t)), "counter");
        std::vector<refgpu_mmatch> host_out;
        uint64_t n_out = 0;
        uint32_t n_pat = (uint32_t)n_patterns, n_fwd = (uint32_t)n_fwd_patterns;
        double w0 = now_ms();
        for (size_t bi = 0; bi < c->batches.size(); bi++) {
            const Batch &b = c->batches[bi];
            if (batch_offsets) batch_offsets[bi] = n_out;
            t->host_ms += c->pack(b, false);
            c->upload(t);
            size_t nch = b.n;
            uint32_t active_start = b.head ? c->offs[1] * 2 : 0;
            uint32_t n_active = c->offs[nch] * 2;
            // sub-range bisection (search.rs:1097-1156)
            std::vector<std::pair<uint32_t, uint32_t>> pending{{active_start, n_active}};
            while (!pending.empty()) {
                auto [s, e] = pending.back();
                pending.pop_back();
                if (s >= e) continue;
                double h0 = now_ms();
                uint32_t zero = 0;
                ck(cudaMemcpy(d_count, &zero, 4, cudaMemcpyHostToDevice), "counter H2D");
                t->h2d_ms += now_ms() - h0;
                const uint8_t *g = c->d_genome;
                void *v[13] = {&g,     &d_peq,    &d_pat, &d_off, &d_filt,
                               &n_pat, &n_fwd,    &s,     &e,     &active_start,
                               &n_active, &d_out, &d_count};
                dim3 grid((e - s + kBlockX - 1) / kBlockX, n_pat);
                t->kernel_ms += c->timed_launch((const void *)k.fn, grid, v);
                t->launches++;
                double d0 = now_ms();
                uint32_t cnt = 0;
                ck(cudaMemcpy(&cnt, d_count, 4, cudaMemcpyDeviceToHost), "count D2H");
                t->d2h_ms += now_ms() - d0;
                if (cnt > out_buf_size) {
                    uint32_t mid = s + (e - s) / 2;
                    if (mid == s || mid == e) {
                        throw CudaFail{"match buffer overflow on a minimal sub-range"};
                    }
                    pending.push_back({mid, e});
                    pending.push_back({s, mid});
                    continue;
                }
                if (cnt == 0) continue;
                d0 = now_ms();
                host_out.resize(cnt);
                ck(cudaMemcpy(host_out.data(), d_out, (size_t)cnt * sizeof(refgpu_mmatch),
                              cudaMemcpyDeviceToHost),
                   "matches D2H");
                t->d2h_ms += now_ms() - d0;
                if (out) {
                    if (n_out + cnt > out_cap) throw CudaFail{"out_cap too small"};
                    std::memcpy(out + n_out, host_out.data(), (size_t)cnt * sizeof(refgpu_mmatch));
                }
                n_out += cnt;
            }
        }
        if (batch_offsets) batch_offsets[c->batches.size()] = n_out;
        t->wall_ms = now_ms() - w0;
        t->n_batches = c->batches.size();
        t->matches = n_out;
    } catch (const CudaFail &f) {
        set_err(err, errlen, f.what);
        rc = -1;
    }
    cudaFree(d_peq);
    cudaFree(d_pat);
    cudaFree(d_off);
    cudaFree(d_filt);
    cudaFree(d_out);
    cudaFree(d_count);
    return rc;
}

char *refgpu_myers_lines(refgpu_ctx *c, const char *const *chunk_names,
                         const char *const *patterns, size_t n_patterns, size_t n_fwd_patterns,
                         const refgpu_mmatch *recs, const uint64_t *batch_offsets,
                         uint64_t *text_len, uint64_t *n_lines) {
    static const char kDec[16] = {0,   'T', 'C', 'Y', 'A', 'W', 'M', 'H',
                                  'G', 'K', 'S', 'B', 'R', 'D', 'V', 'N'};
    const size_t L = n_patterns ? std::strlen(patterns[0]) : 0;
    std::string out;
    uint64_t lines = 0;
    std::string rna, dna;
    char num[64];
    for (size_t bi = 0; bi < c->batches.size(); bi++) {
        const Batch &b = c->batches[bi];
        c->pack(b, false);  // the batch buffer and its chunk byte offsets
        const uint8_t *buf = c->host.data();
        const uint64_t nbytes = c->offs.back();
        auto nib = [&](uint64_t i) -> uint8_t {
            if (i / 2 >= nbytes) return 0;
            const uint8_t x = buf[i / 2];
            return (i & 1) ? (uint8_t)(x >> 4) : (uint8_t)(x & 0xF);
        };
        for (uint64_t r = batch_offsets[bi]; r < batch_offsets[bi + 1]; r++) {
            const refgpu_mmatch &m = recs[r];
            const char *pat = patterns[m.pattern_idx];
            // decode_gpu_enum_match (search.rs:152-206): ops last to first;
            // an M / S / D op over a zero nibble drops the record
            rna.clear();
            dna.clear();
            uint64_t gi = m.chunk_idx;
            size_t pi = 0;
            bool ok = true;
            for (int k = (int)m.ops_count - 1; k >= 0; k--) {
                const unsigned op = (unsigned)(m.ops_packed >> (2 * k)) & 3u;
                if (op != 3) {
                    const uint8_t v = nib(gi);
                    if (!v) {
                        ok = false;
                        break;
                    }
                    dna.push_back(kDec[v]);
                    rna.push_back(op != 2 ? pat[pi] : '-');
                    pi += op != 2;
                    gi++;
                } else {
                    rna.push_back(pat[pi]);
                    dna.push_back('-');
                    pi++;
                }
            }
            if (!ok) continue;
            // convert_matches_myers (search.rs:1316-1374): owning chunk and
            // the record-end drop with extent L + db - rb
            const uint64_t start = m.chunk_idx;
            size_t idx = (size_t)(std::upper_bound(c->offs.begin(), c->offs.end(),
                                                   (uint32_t)(start / 2)) -
                                  c->offs.begin()) - 1;
            idx = std::min(idx, b.n - 1);
            const size_t k = b.first + idx;
            const uint64_t pos = c->start[k] + (start - (uint64_t)c->offs[idx] * 2);
            const bool end_chrom = idx == b.n - 1 || c->start[k + 1] == 0;
            const uint64_t extent = L + m.dna_bulge_size - m.rna_bulge_size;
            if (end_chrom && pos + extent > c->end[k]) continue;
            const bool fwd = m.pattern_idx < n_fwd_patterns;
            if (!fwd) {
                std::reverse(rna.begin(), rna.end());
                std::reverse(dna.begin(), dna.end());
                for (char &ch : rna) ch = ch == '-' ? ch : comp_char(ch);
                for (char &ch : dna) ch = ch == '-' ? ch : comp_char(ch);
            }
            out += chunk_names[k];
            std::snprintf(num, sizeof num, "\t%llu\t%u\t%c\t%u\t%u\t%u\t",
                          (unsigned long long)pos, m.pattern_idx, fwd ? '+' : '-', m.mismatches,
                          (unsigned)m.dna_bulge_size, (unsigned)m.rna_bulge_size);
            out += num;
            out += rna;
            out += '\t';
            out += dna;
            out += '\n';
            lines++;
        }
    }
    char *p = static_cast<char *>(std::malloc(out.size() + 1));
    if (!p) return nullptr;
    std::memcpy(p, out.data(), out.size());
    p[out.size()] = 0;
    *text_len = out.size();
    *n_lines = lines;
    return p;
}

void refgpu_free(void *p) { std::free(p); }

}  // extern "C"
