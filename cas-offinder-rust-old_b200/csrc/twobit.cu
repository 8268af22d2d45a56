// twobit.cu -- the bases of a .2bit genome decoded on the device at upload
// (read_2bit.rs:33-118, the per-chunk conversion; BIT2_TO_BIT4 and
// memsetbit4, bit4ops.rs:60-75 and :145-200).
//
// The host has already read the file's index and N blocks into a TwoBitPlan
// (loader.cpp): per chunk the file offset of its packed bases, its byte
// offset in the bit4 stream, its length and its N ranges.  Here host threads
// read the packed bytes (a quarter of the bit4 size) into page-locked
// staging buffers and copy them to the device on their own streams, and one
// CTA per chunk writes the chunk's bit4 bytes: 2-bit codes T=0 C=1 A=2 G=3,
// first base in the high bits, become one-hot nibbles, the nibbles after the
// last base stay zero, and the N ranges become 0xF.
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "cof_engine.h"
#include "engine_dev.cuh"

namespace cof {

namespace {

__global__ void __launch_bounds__(256)
decode_2bit_kernel(const uint8_t *__restrict__ raw, uint64_t raw_begin,
                   const TwoBitPlan::Piece *__restrict__ pieces, const uint32_t *__restrict__ nr,
                   uint8_t *__restrict__ bit4) {
    const TwoBitPlan::Piece pc = pieces[blockIdx.x];
    const uint32_t r_end = pieces[blockIdx.x + 1].nr;
    const uint32_t rs = pc.rs;
    const uint32_t n_in = (rs + 3) >> 2, n_out = (rs + 1) >> 1;
    const uint8_t *src = raw + (pc.raw - raw_begin);
    uint8_t *dst = bit4 + pc.out;
    for (uint32_t j = threadIdx.x; j < n_in; j += blockDim.x) {
        const uint32_t v = src[j];
        uint32_t nib = 0;  // nucleotide 4j + k in bits [4k, 4k + 4)
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (4 * j + k < rs) nib |= (1u << ((v >> (6 - 2 * k)) & 3u)) << (4 * k);
        for (uint32_t r = pc.nr; r < r_end; ++r) {
            const uint32_t lo = nr[2 * r], hi = nr[2 * r + 1];
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (4 * j + k >= lo && 4 * j + k < hi) nib |= 0xFu << (4 * k);
        }
        dst[2 * j] = (uint8_t)nib;
        if (2 * j + 1 < n_out) dst[2 * j + 1] = (uint8_t)(nib >> 8);
    }
}

// Device buffers of one upload, freed on every return path.
struct Scratch {
    DevBuf<uint8_t> raw;
    DevBuf<TwoBitPlan::Piece> pieces;
    DevBuf<uint32_t> nr;
    ~Scratch() {
        raw.release();
        pieces.release();
        nr.release();
    }
};

// Reads file bytes [off, off + n) into dst; false on a short read.
bool read_fully(int fd, char *dst, size_t n, uint64_t off) {
    while (n) {
        const ssize_t r = ::pread(fd, dst, n, (off_t)off);
        if (r < 0 && errno == EINTR) continue;
        if (r <= 0) return false;
        dst += r;
        n -= (size_t)r;
        off += (uint64_t)r;
    }
    return true;
}

}  // namespace

int copy_file_to_device(const std::string &path, uint64_t file_bytes, uint64_t begin,
                        uint64_t n, uint8_t *dst, int device, Error &err) {
    if (n == 0) return kOk;
    const int fd = ::open(path.c_str(), O_RDONLY);
    if (fd < 0) {
        err = {kIo, "cannot open " + path + ": " + std::strerror(errno)};
        return err.code;
    }
    struct stat st;
    if (::fstat(fd, &st) || (uint64_t)st.st_size != file_bytes) {
        ::close(fd);
        err = {kIo, path + " changed since it was loaded"};
        return err.code;
    }
    // slices of kSlice bytes, every nt-th slice on one host thread, each
    // thread with two page-locked buffers and its own stream
    constexpr size_t kSlice = size_t(4) << 20;
    const size_t n_slices = (size_t)((n + kSlice - 1) / kSlice);
    const unsigned nt = (unsigned)std::max<size_t>(
        1, std::min<size_t>(n_slices, std::min(8u, std::max(1u, std::thread::hardware_concurrency()))));
    std::atomic<bool> failed{false};
    std::mutex mu;
    std::string msg;
    auto fail = [&](const std::string &m) {
        std::lock_guard<std::mutex> lk(mu);
        if (!failed.exchange(true)) msg = m;
    };
    auto worker = [&](unsigned t) {
        if (cudaSetDevice(device) != cudaSuccess) return fail("cudaSetDevice failed");
        cudaStream_t ts = nullptr;
        cudaEvent_t ev[2] = {nullptr, nullptr};
        PooledText buf[2];
        if (cudaStreamCreateWithFlags(&ts, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming) != cudaSuccess) {
            fail("cannot create a copy stream");
        } else {
            buf[0].p = PinnedPool::get().acquire(kSlice - 1);
            buf[1].p = PinnedPool::get().acquire(kSlice - 1);
            if (!buf[0].p || !buf[1].p) fail("out of page-locked host memory for the genome copy");
        }
        size_t it = 0;
        for (size_t i = t; i < n_slices && !failed.load(); i += nt, ++it) {
            const int b = (int)(it & 1);
            if (it >= 2 && cudaEventSynchronize(ev[b]) != cudaSuccess) {
                fail("genome copy failed");
                break;
            }
            const uint64_t off = (uint64_t)i * kSlice;
            const size_t len = (size_t)std::min<uint64_t>(kSlice, n - off);
            if (!read_fully(fd, buf[b].p, len, begin + off)) {
                fail("short read on " + path);
                break;
            }
            if (cudaMemcpyAsync(dst + off, buf[b].p, len, cudaMemcpyHostToDevice, ts) != cudaSuccess ||
                cudaEventRecord(ev[b], ts) != cudaSuccess) {
                fail("genome copy failed");
                break;
            }
        }
        if (ts) {
            if (cudaStreamSynchronize(ts) != cudaSuccess) fail("genome copy failed");
            cudaStreamDestroy(ts);
        }
        for (cudaEvent_t e : ev)
            if (e) cudaEventDestroy(e);
    };
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; ++t) th.emplace_back(worker, t);
    for (auto &x : th) x.join();
    ::close(fd);
    if (failed) {
        cudaGetLastError();
        err = {kIo, msg};
        return err.code;
    }
    return kOk;
}

int upload_2bit(const TwoBitPlan &plan, uint8_t *bit4, int device, cudaStream_t s, Error &err) {
    const size_t n_pieces = plan.pieces.size() - 1;
    if (n_pieces == 0) return kOk;
    const uint64_t raw_n = plan.raw_end - plan.raw_begin;
    Scratch sc;
    if (sc.raw.ensure(raw_n, err) || sc.pieces.ensure(plan.pieces.size(), err) ||
        sc.nr.ensure(std::max<size_t>(plan.nr.size(), 1), err))
        return err.code;
    if (copy_file_to_device(plan.path, plan.file_bytes, plan.raw_begin, raw_n, sc.raw.p, device,
                            err))
        return err.code;
    CU(cudaMemcpyAsync(sc.pieces.p, plan.pieces.data(), plan.pieces.size() * sizeof(TwoBitPlan::Piece),
                       cudaMemcpyHostToDevice, s));
    if (!plan.nr.empty())
        CU(cudaMemcpyAsync(sc.nr.p, plan.nr.data(), plan.nr.size() * 4, cudaMemcpyHostToDevice, s));
    decode_2bit_kernel<<<(unsigned)n_pieces, 256, 0, s>>>(sc.raw.p, plan.raw_begin, sc.pieces.p,
                                                         sc.nr.p, bit4);
    CU(cudaGetLastError());
    CU(cudaStreamSynchronize(s));  // the scratch buffers are freed on return
    return kOk;
}

}  // namespace cof
