// hostpool.cpp -- the page-locked result-buffer pool (PinnedPool in
// cof_engine.h).  Buffers are portable pinned allocations, usable from every
// device's stream.  Small results are blocks of size classes cut from shared
// slabs; larger ones are allocations of their own, rounded up to 2 MiB so
// that nearby sizes reuse each other.
#include <cuda_runtime.h>

#include "cof_engine.h"

namespace cof {

PinnedPool &PinnedPool::get() {
    static PinnedPool pool;  // process lifetime; buffers are released at exit
    return pool;
}

char *PinnedPool::alloc_large(size_t want) {
    char *p = nullptr;
    if (cudaHostAlloc((void **)&p, want, cudaHostAllocPortable) != cudaSuccess) {
        cudaGetLastError();  // clear the recorded error of the failed call
        // drop what is kept and try once more
        for (auto &kv : free_) cudaFreeHost(kv.second);
        free_.clear();
        free_bytes_ = 0;
        if (cudaHostAlloc((void **)&p, want, cudaHostAllocPortable) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
    }
    return p;
}

char *PinnedPool::acquire(size_t bytes) {
    const size_t need = bytes + 1;
    std::lock_guard<std::mutex> lk(mu_);
    if (need <= kSmallMax) {
        int c = 0;
        while ((kMinBlock << c) < need) ++c;
        const size_t block = kMinBlock << c;
        auto &fl = small_free_[c];
        if (fl.empty()) {
            const size_t slab = std::max(kSlabBytes, 16 * block);
            char *s = nullptr;
            if (slab_bytes_ + slab <= kSmallCap &&
                cudaHostAlloc((void **)&s, slab, cudaHostAllocPortable) == cudaSuccess) {
                slab_bytes_ += slab;
                for (size_t o = slab; o >= block; o -= block) fl.push_back(s + o - block);
            } else {
                cudaGetLastError();
            }
        }
        if (!fl.empty()) {
            char *p = fl.back();
            fl.pop_back();
            live_[p] = {block, c};
            return p;
        }
    }
    const size_t want = (need + (size_t(2) << 20) - 1) & ~((size_t(2) << 20) - 1);
    // best fit among the kept buffers, at most twice the size asked for
    auto it = free_.lower_bound(want);
    if (it != free_.end() && it->first <= 2 * want) {
        char *p = it->second;
        const size_t n = it->first;
        free_.erase(it);
        free_bytes_ -= n;
        live_[p] = {n, -1};
        return p;
    }
    char *p = alloc_large(want);
    if (p) live_[p] = {want, -1};
    return p;
}

bool PinnedPool::release(char *p) {
    if (!p) return false;
    std::lock_guard<std::mutex> lk(mu_);
    auto it = live_.find(p);
    if (it == live_.end()) return false;
    const size_t n = it->second.first;
    const int c = it->second.second;
    live_.erase(it);
    if (c >= 0) {  // back to its size class; slabs are kept
        small_free_[c].push_back(p);
        return true;
    }
    free_.emplace(n, p);
    free_bytes_ += n;
    // over kKeepBytes, free the smallest kept buffers, but never the one just
    // released: a caller repeating a search whose rows alone pass the limit
    // reuses it instead of pinning gigabytes again
    while (free_bytes_ > kKeepBytes && free_.size() > 1) {
        auto victim = free_.begin();
        if (victim->second == p) ++victim;
        free_bytes_ -= victim->first;
        cudaFreeHost(victim->second);
        free_.erase(victim);
    }
    return true;
}

}  // namespace cof
