// intpeak.cu -- integer-pipe peaks of this GPU, the roofline denominators of
// the popcount scan (libcof_peak.so, used by bench.py; not part of libcof).
//
//   popc : __popc results per second (8 independent chains per thread)
//   lop3 : 3-input logic results per second (8 independent chains)
//   pair : window x pattern comparisons per second of the scan's inner loop
//          (popc((H^pH)|(L^pL)|S) folded into a per-pattern minimum over 8
//          windows, one threshold test per pattern) on register-resident,
//          care-masked windows and shared-memory patterns, i.e. the scan with
//          no memory traffic and no hits.
#include <cuda_runtime.h>

#include <cstdint>

namespace {

__global__ void popc_kernel(uint32_t seed, int iters, uint32_t *out) {
    uint32_t x[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) x[j] = seed * (threadIdx.x + 1 + j * 977) + blockIdx.x;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < 8; ++j) x[j] = __popc(x[j]) ^ (x[j] << 5);
    }
    uint32_t a = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) a ^= x[j];
    if (a == 0x12345678u) out[0] = a;
}

__global__ void lop3_kernel(uint32_t seed, int iters, uint32_t *out) {
    uint32_t x[8], y = seed ^ threadIdx.x, z = seed + blockIdx.x;
#pragma unroll
    for (int j = 0; j < 8; ++j) x[j] = seed * (threadIdx.x + 1 + j * 977);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < 8; ++j) x[j] = (x[j] ^ y) | (x[j] & z);
        y += 1;
    }
    uint32_t a = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) a ^= x[j];
    if (a == 0x12345678u) out[0] = a;
}

constexpr int kPats = 256;

__global__ void pair_kernel(uint32_t seed, int iters, uint32_t *out) {
    __shared__ uint4 pat[kPats];
    for (int i = threadIdx.x; i < kPats; i += blockDim.x)
        pat[i] = make_uint4(seed * (i + 3), seed ^ (i * 7919), 0x007FFFFFu, 0xFFFFFFFFu);
    __syncthreads();
    uint32_t h[8], l[8], s[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        h[j] = seed * (threadIdx.x + 11 + j);
        l[j] = seed ^ (threadIdx.x * 31 + j);
        s[j] = 0;
    }
    uint32_t hits = 0;
    for (int it = 0; it < iters; ++it) {
        for (int p = 0; p < kPats; ++p) {
            const uint4 q = pat[p];
            int mn = 64;
#pragma unroll
            for (int j = 0; j < 8; ++j) mn = min(mn, (int)__popc((h[j] ^ q.x) | (l[j] ^ q.y) | s[j]));
            if (mn <= (int)q.w) hits += mn + 1;  // q.w = -1: never
        }
    }
    if (hits) out[0] = hits;
}

template <class K>
double time_kernel(K kernel, int blocks, int threads, int iters, uint32_t *d_out, double per) {
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    kernel<<<blocks, threads>>>(0x9E3779B1u, iters / 8 + 1, d_out);  // warm-up
    cudaEventRecord(a);
    kernel<<<blocks, threads>>>(0x9E3779B1u, iters, d_out);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return (double)blocks * threads * (double)iters * per / (ms * 1e-3);
}

}  // namespace

// out[0] = popc/s, out[1] = lop3/s, out[2] = scan pairs/s, out[3] = SM clock
// (kHz) reported by the driver.  Returns 0 or a CUDA error code.
extern "C" __attribute__((visibility("default"))) int cof_peak_measure(int device, double *out) {
    if (cudaSetDevice(device) != cudaSuccess) return -1;
    int n_sm = 0, clk = 0;
    cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, device);
    cudaDeviceGetAttribute(&clk, cudaDevAttrClockRate, device);
    uint32_t *d_out = nullptr;
    if (cudaMalloc(&d_out, 16) != cudaSuccess) return -2;
    const int blocks = n_sm * 8, threads = 256;
    out[0] = time_kernel(popc_kernel, blocks, threads, 4096, d_out, 8.0);
    out[1] = time_kernel(lop3_kernel, blocks, threads, 4096, d_out, 8.0);
    out[2] = time_kernel(pair_kernel, n_sm * 4, threads, 64, d_out, 8.0 * kPats);
    out[3] = clk;
    cudaError_t e = cudaDeviceSynchronize();
    cudaFree(d_out);
    return e == cudaSuccess ? 0 : (int)e;
}
