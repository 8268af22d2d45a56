// noalloc.cu -- popcount search over one caller-resident sequence that
// allocates no memory (cof_search_seq_noalloc, declared in include/cof.h).
//
// Some callers cannot call cudaMalloc: a host application that owns the whole
// device memory through its own pool allocator and only hands out pointers
// into it (an allocation from this library would bypass its accounting or
// fail once the pool holds the memory), or a serving process that must not
// allocate on its request path because an allocation can synchronise the
// device and stall unrelated work.  This entry point takes the caller's device
// buffers for its input (the bit4 sequence) and its output (the rows), and keeps
// everything else -- counters, pattern tables, the candidate list -- in one
// fixed file-scope device array, `g_noalloc_scratch`, that exists on every GPU
// that loads libcof.so until the process exits.
//
// It is a variant of the genome scan of engine.cu (same PAM prefilter and
// popcount lower bound, same exact decision of the reference writer,
// search.rs:378-463 + main.rs:159-222) restricted to a single record: every
// window start s with s + L <= n_nucl, the record-end drop of
// convert_matches (search.rs:1449-1454).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/cof.h"
#include "cof_engine.h"

namespace {

constexpr uint32_t kNaMaxPatterns = 512;                 // fwd + reverse patterns
constexpr size_t kNaScratchBytes = 8u << 20;              // 8 MiB per GPU
constexpr size_t kNaCounterBytes = 256;
constexpr size_t kNaTableBytes = 32u << 10;
constexpr size_t kNaCandOffset = kNaCounterBytes + kNaTableBytes;
constexpr uint32_t kNaMaxCandidates =
    (uint32_t)((kNaScratchBytes - kNaCandOffset) / sizeof(uint2));  // 1,044,448
// rows a call may count before its 32-bit row counter could wrap
constexpr uint32_t kNaRowCountLimit = 0xFFFFFFF0u;

struct NaPam {
    uint32_t cell, fa, fc, fg, ft;
};
struct NaFast {
    uint32_t h, l, care;
    int32_t k;
};
struct NaTables {
    uint32_t L, n_fwd, n_pat, max_mm;
    uint32_t n_pam[2];
    uint32_t pad[2];
    NaPam pam[2][32];
    uint8_t fset[2][32];
    uint8_t fisn[2][32];
    NaFast fast[kNaMaxPatterns];
    uint8_t b4[kNaMaxPatterns][32];
};
static_assert(sizeof(NaTables) <= kNaTableBytes, "pattern tables exceed their scratch slot");

// counters: [0] candidates, [1] candidate overflow, [2] rows, [3] row-count
// overflow (the 32-bit row counter came within 16 of wrapping)
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaScratchBytes];

__device__ __forceinline__ uint32_t na_gather(uint32_t v) {
    v &= 0x11111111u;
    v = (v | (v >> 3)) & 0x03030303u;
    v = (v | (v >> 6)) & 0x000F000Fu;
    return (v | (v >> 12)) & 0xFFu;
}

// H / L / S plane words of nucleotides [32w, 32w + 32); bytes past n_bytes
// read as padding (S set).
__device__ void na_planes(const uint8_t *bit4, uint64_t n_bytes, uint64_t w, uint32_t &h,
                          uint32_t &l, uint32_t &s) {
    uint32_t x[4] = {0, 0, 0, 0};
    const uint64_t b0 = 16 * w;
    if (b0 + 16 <= n_bytes) {
        const uint4 q = *reinterpret_cast<const uint4 *>(bit4 + b0);
        x[0] = q.x; x[1] = q.y; x[2] = q.z; x[3] = q.w;
    } else {
        for (int i = 0; i < 16; ++i)
            if (b0 + i < n_bytes) x[i >> 2] |= (uint32_t)bit4[b0 + i] << (8 * (i & 3));
    }
    h = l = s = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const uint32_t v = x[j];
        uint32_t pc = v - ((v >> 1) & 0x55555555u);
        pc = (pc & 0x33333333u) + ((pc >> 2) & 0x33333333u);
        const uint32_t t = pc ^ 0x11111111u;
        h |= na_gather((v >> 3) | v) << (8 * j);
        l |= na_gather((v >> 1) | v) << (8 * j);
        s |= na_gather(t | (t >> 1) | (t >> 2)) << (8 * j);
    }
}

__global__ void na_scan_kernel(const uint8_t *__restrict__ bit4, uint64_t n_bytes, uint32_t lo,
                               uint32_t hi, unsigned char *scratch) {
    const NaTables &T = *reinterpret_cast<const NaTables *>(scratch + kNaCounterBytes);
    uint32_t *ctr = reinterpret_cast<uint32_t *>(scratch);
    uint2 *cand = reinterpret_cast<uint2 *>(scratch + kNaCandOffset);
    const uint64_t w_lo = lo / 32, w_hi = ((uint64_t)hi + 31) / 32;
    for (uint64_t w = w_lo + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < w_hi;
         w += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t h0, l0, s0, h1, l1, s1;
        na_planes(bit4, n_bytes, w, h0, l0, s0);
        na_planes(bit4, n_bytes, w + 1, h1, l1, s1);
        const uint64_t p0 = 32 * w;
        uint32_t range = 0xFFFFFFFFu;
        if (p0 < lo) range = (lo - p0 >= 32) ? 0u : (range << (uint32_t)(lo - p0));
        if (p0 + 32 > hi) range = (hi <= p0) ? 0u : (range & (0xFFFFFFFFu >> (uint32_t)(32 - (hi - p0))));
        for (uint32_t st = 0; st < 2; ++st) {
            uint32_t m = range;
            for (uint32_t c = 0; c < T.n_pam[st] && m; ++c) {
                const NaPam pc = T.pam[st][c];
                const uint32_t h = __funnelshift_r(h0, h1, pc.cell);
                const uint32_t l = __funnelshift_r(l0, l1, pc.cell);
                const uint32_t s = __funnelshift_r(s0, s1, pc.cell);
                const uint32_t t0 = (l & pc.fc) | (~l & pc.fa);
                const uint32_t t1 = (l & pc.ft) | (~l & pc.fg);
                m &= ((h & t1) | (~h & t0)) & ~s;
            }
            const uint32_t pb = st ? T.n_fwd : 0, pe = st ? T.n_pat : T.n_fwd;
            while (m) {
                const uint32_t k = __ffs(m) - 1;
                m &= m - 1;
                const uint32_t wh = __funnelshift_r(h0, h1, k), wl = __funnelshift_r(l0, l1, k),
                               ws = __funnelshift_r(s0, s1, k);
                for (uint32_t p = pb; p < pe; ++p) {
                    const NaFast f = T.fast[p];
                    if ((int)__popc(((wh ^ f.h) | (wl ^ f.l) | ws) & f.care) <= f.k) {
                        const uint32_t i = atomicAdd(&ctr[0], 1u);
                        if (i < kNaMaxCandidates) cand[i] = make_uint2((uint32_t)(p0 + k), p);
                        else ctr[1] = 1;
                    }
                }
            }
        }
    }
}

__device__ __forceinline__ uint8_t na_nib(const uint8_t *g, uint64_t i) {
    const uint8_t b = g[i >> 1];
    return (i & 1) ? (uint8_t)(b >> 4) : (uint8_t)(b & 0xF);
}

__global__ void na_verify_kernel(const uint8_t *__restrict__ bit4, uint64_t n_nucl,
                                 uint32_t n_cand, unsigned char *scratch, uint32_t *rows,
                                 uint32_t rows_cap) {
    const NaTables &T = *reinterpret_cast<const NaTables *>(scratch + kNaCounterBytes);
    uint32_t *ctr = reinterpret_cast<uint32_t *>(scratch);
    const uint2 *cand = reinterpret_cast<const uint2 *>(scratch + kNaCandOffset);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_cand;
         i += gridDim.x * blockDim.x) {
        const uint32_t s = cand[i].x, p = cand[i].y, L = T.L;
        if ((uint64_t)s + L > n_nucl) continue;  // record-end drop
        const uint32_t st = p >= T.n_fwd;
        int matches = 0;
        uint32_t actual = 0;
        bool pam_ok = true;
        for (uint32_t c = 0; c < L; ++c) {
            uint8_t g = na_nib(bit4, (uint64_t)s + c);
            if (g == 0xF) g = 0;  // N masked for the popcount count
            const uint8_t pb = T.b4[p][c];
            matches += __popc(g & pb);
            const bool single = g && !(g & (g - 1));
            if (!T.fisn[st][c] && !(single && (g & T.fset[st][c]))) pam_ok = false;
            if (pb != 0xF && !(single && (g & pb))) ++actual;
        }
        if ((int)L - matches > (int)T.max_mm || !pam_ok || actual > T.max_mm) continue;
        const uint32_t r = atomicAdd(&ctr[2], 1u);
        if (r >= kNaRowCountLimit) ctr[3] = 1;  // every value is returned once: none is missed
        if (r < rows_cap) {
            const uint64_t o = 3ull * r;  // rows_cap may exceed 2^32 / 3
            rows[o] = s;
            rows[o + 1] = p;
            rows[o + 2] = actual;
        }
    }
}

std::mutex g_na_mu;
void *g_na_ptr[64] = {};  // device address of g_noalloc_scratch, per device

int na_fail(int code, const std::string &m) { return cof::set_last_error(code, m); }

uint32_t na_code(uint8_t b4) { return b4 == 4 ? 0 : b4 == 2 ? 1 : b4 == 8 ? 2 : 3; }

}  // namespace

// See include/cof.h.
extern "C" COF_API int cof_search_seq_noalloc(const uint8_t *d_bit4, uint64_t n_nucl,
                                              const char *search_filter,
                                              const char *const *patterns, size_t n_patterns,
                                              uint32_t max_mismatches, uint32_t *d_rows,
                                              uint32_t rows_cap, uint32_t *n_rows,
                                              void *stream) {
    if (!d_bit4 || !search_filter || !patterns || !n_rows || (!d_rows && rows_cap))
        return na_fail(COF_E_BADINPUT, "null argument");
    if (reinterpret_cast<uintptr_t>(d_bit4) % 16)
        return na_fail(COF_E_BADINPUT, "d_bit4 must be 16-byte aligned");
    const size_t L = std::strlen(search_filter);
    if (L == 0 || L > 32)
        return na_fail(COF_E_UNSUPPORTED, "pattern length must be 1..32");
    if (n_patterns == 0 || n_patterns > kNaMaxPatterns)
        return na_fail(COF_E_UNSUPPORTED,
                       "n_patterns must be 1.." + std::to_string(kNaMaxPatterns) +
                           " (fwd + reverse) for the fixed scratch tables");
    if (n_patterns % 2)
        return na_fail(COF_E_BADINPUT,
                       "n_patterns must be even: the forward patterns, then their reverse "
                       "complements (search.rs:1455 takes index < n / 2 as '+')");
    if (n_nucl >= (1ull << 31))
        return na_fail(COF_E_UNSUPPORTED, "sequence longer than 2^31 - 1 nucleotides");
    if (max_mismatches >= L)
        return na_fail(COF_E_BADINPUT, "max_mismatches must be below the pattern length");
    const cof::Bit4Tables &t = cof::bit4();
    NaTables T;
    std::memset(&T, 0, sizeof T);
    T.L = (uint32_t)L;
    T.n_pat = (uint32_t)n_patterns;
    T.n_fwd = (uint32_t)(n_patterns / 2);
    T.max_mm = max_mismatches;
    for (size_t c = 0; c < L; ++c) {
        const char f = search_filter[c], fr = search_filter[L - 1 - c];
        if (!cof::is_mixed_base(f))
            return na_fail(COF_E_BADINPUT, "search filter must be a mixed base string");
        T.fset[0][c] = t.str2b4[1][(uint8_t)f];
        T.fisn[0][c] = f == 'N' || f == 'n';
        T.fset[1][c] = cof::comp4(t.str2b4[1][(uint8_t)fr]);
        T.fisn[1][c] = fr == 'N' || fr == 'n';
        for (int st = 0; st < 2; ++st) {
            if (T.fisn[st][c]) continue;
            const uint8_t fs = T.fset[st][c];
            T.pam[st][T.n_pam[st]++] = NaPam{(uint32_t)c, (fs & 4) ? ~0u : 0u, (fs & 2) ? ~0u : 0u,
                                              (fs & 8) ? ~0u : 0u, (fs & 1) ? ~0u : 0u};
        }
    }
    for (size_t p = 0; p < n_patterns; ++p) {
        if (!patterns[p] || std::strlen(patterns[p]) != L)
            return na_fail(COF_E_BADINPUT, "All patterns must have same length");
        NaFast f{0, 0, 0, (int32_t)max_mismatches};
        for (size_t c = 0; c < L; ++c) {
            const char ch = patterns[p][c];
            if (!cof::is_mixed_base(ch))
                return na_fail(COF_E_BADINPUT, "pattern must be a mixed base string");
            const uint8_t v = t.str2b4[1][(uint8_t)ch];
            T.b4[p][c] = v;
            if (!(v & (v - 1))) {
                const uint32_t cd = na_code(v);
                f.care |= 1u << c;
                f.h |= ((cd >> 1) & 1u) << c;
                f.l |= (cd & 1u) << c;
            }
        }
        T.fast[p] = f;
    }

    std::lock_guard<std::mutex> lk(g_na_mu);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
        return na_fail(COF_E_CUDA, "no usable CUDA device");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (s) {
        // the scratch address below belongs to the current device: a stream
        // of another device would run the kernels against the wrong array
        int sdev = -1;
        const cudaError_t e = cudaStreamGetDevice(s, &sdev);
        if (e != cudaSuccess)
            return na_fail(COF_E_BADINPUT, std::string("stream: ") + cudaGetErrorString(e));
        if (sdev != dev)
            return na_fail(COF_E_BADINPUT, "stream belongs to device " + std::to_string(sdev) +
                                                ", the current device is " + std::to_string(dev));
    }
    if (!g_na_ptr[dev]) {
        // once per device, with that device current: the array's name is only
        // a host-side stand-in, the kernels need its device address.  The
        // address is kept for the process; a cudaDeviceReset of this device
        // by the caller invalidates it (and the array itself)
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return na_fail(COF_E_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_na_ptr[dev] = p;
    }
    unsigned char *scratch = static_cast<unsigned char *>(g_na_ptr[dev]);
    auto cu = [&](cudaError_t e, const char *what) {
        if (e == cudaSuccess) return 0;
        na_fail(COF_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
        return 1;
    };
    if (cu(cudaMemcpyAsync(scratch + kNaCounterBytes, &T, sizeof T, cudaMemcpyHostToDevice, s),
           "table upload") ||
        cu(cudaMemsetAsync(scratch, 0, kNaCounterBytes, s), "counter reset"))
        return COF_E_CUDA;
    const uint64_t n_bytes = (n_nucl + 1) / 2;
    // ranges still to scan; bisection keeps the stack below 2 x 31 + 1
    uint32_t pend_a[80], pend_b[80];
    int np = 0;
    if (n_nucl >= L) {
        pend_a[0] = 0;
        pend_b[0] = (uint32_t)(n_nucl - L + 1);
        np = 1;
    }
    while (np > 0) {
        --np;
        const uint32_t a = pend_a[np], b = pend_b[np];
        if (cu(cudaMemsetAsync(scratch, 0, 8, s), "counter reset")) return COF_E_CUDA;
        const uint64_t words = ((uint64_t)b + 31) / 32 - a / 32;
        const unsigned blocks = (unsigned)std::min<uint64_t>((words + 255) / 256, 4096);
        na_scan_kernel<<<blocks, 256, 0, s>>>(d_bit4, n_bytes, a, b, scratch);
        uint32_t c2[2] = {0, 0};
        if (cu(cudaGetLastError(), "scan launch") ||
            cu(cudaMemcpyAsync(c2, scratch, 8, cudaMemcpyDeviceToHost, s), "count readback") ||
            cu(cudaStreamSynchronize(s), "scan"))
            return COF_E_CUDA;
        if (c2[1] || c2[0] > kNaMaxCandidates) {
            // more candidates than the fixed list holds: split the range
            // (the reference bisects its Myers ranges the same way,
            // search.rs:1106-1153)
            if (b - a <= 64)
                return na_fail(COF_E_UNSUPPORTED, "candidate list overflow on a minimal range");
            const uint32_t mid = a + (b - a) / 2;
            pend_a[np] = mid;
            pend_b[np] = b;
            pend_a[np + 1] = a;
            pend_b[np + 1] = mid;
            np += 2;
            continue;
        }
        if (c2[0]) {
            const unsigned vb = (unsigned)std::min<uint32_t>((c2[0] + 255) / 256, 4096);
            na_verify_kernel<<<vb, 256, 0, s>>>(d_bit4, n_nucl, c2[0], scratch, d_rows, rows_cap);
            if (cu(cudaGetLastError(), "verify launch")) return COF_E_CUDA;
        }
    }
    uint32_t c23[2] = {0, 0};  // rows, row-count overflow
    if (cu(cudaMemcpyAsync(c23, scratch + 8, 8, cudaMemcpyDeviceToHost, s), "row count") ||
        cu(cudaStreamSynchronize(s), "verify"))
        return COF_E_CUDA;
    if (c23[1]) {
        *n_rows = 0xFFFFFFFFu;
        return na_fail(COF_E_UNSUPPORTED,
                       "more than 2^32 - 16 rows: the row count does not fit its 32-bit counter");
    }
    const uint32_t nr = c23[0];
    *n_rows = nr;
    if (nr > rows_cap)
        return na_fail(COF_E_UNSUPPORTED, "rows_cap too small: " + std::to_string(nr) +
                                              " rows found, the first rows_cap were written");
    return COF_OK;
}
