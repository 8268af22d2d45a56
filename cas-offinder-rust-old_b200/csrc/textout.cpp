// textout.cpp -- result text from device memory to the caller (textout.h).
#include "textout.h"

#include <algorithm>
#include <cstring>
#include <string>

namespace cof {

namespace {
int cuda_fail(Error &err, cudaError_t e, const char *what) {
    err = {kCuda, std::string(what) + ": " + cudaGetErrorString(e)};
    return err.code;
}
}  // namespace

TextOut::~TextOut() {
    // no copy may still write into a buffer that is released here
    if (in_flight_) cudaStreamSynchronize(cs_);
    for (Pending &pc : pending_)
        if (pc.done) events_.push_back(pc.done);
    for (cudaEvent_t e : events_) cudaEventDestroy(e);
}

int TextOut::grow(size_t req, size_t need, Error &err) {
    if (need <= cap_[req]) return kOk;
    if (in_flight_) {  // copies into the old buffer finish first
        const cudaError_t e = cudaStreamSynchronize(cs_);
        if (e != cudaSuccess) return cuda_fail(err, e, "result copy");
        in_flight_ = false;
    }
    const size_t want = std::max(need, cap_[req] + cap_[req] / 2);
    PooledText nb;
    nb.p = PinnedPool::get().acquire(want);
    if (!nb.p) {
        err = {kOom, "out of page-locked host memory for result text"};
        return err.code;
    }
    Result &r = out_[req];
    if (r.pooled.p && len_[req]) std::memcpy(nb.p, r.pooled.p, len_[req]);
    r.pooled = std::move(nb);
    r.text = r.pooled.p;
    cap_[req] = want;
    return kOk;
}

int TextOut::reserve(size_t req, size_t bytes, Error &err) {
    if (sink_) return kOk;
    return grow(req, bytes + 1, err);
}

int TextOut::put(size_t req, const char *d_text, size_t len, uint64_t n_rows,
                 const MatchRec *d_recs, cudaEvent_t ready, Error &err) {
    cudaError_t e = cudaStreamWaitEvent(cs_, ready, 0);
    if (e != cudaSuccess) return cuda_fail(err, e, "result copy wait");
    if (!sink_) {
        if (grow(req, len_[req] + len + 1, err)) return err.code;
        if (len) {
            e = cudaMemcpyAsync(out_[req].pooled.p + len_[req], d_text, len,
                                cudaMemcpyDeviceToHost, cs_);
            if (e != cudaSuccess) return cuda_fail(err, e, "result copy");
            in_flight_ = true;
        }
        len_[req] += len;
        out_[req].n_rows += n_rows;
        copied_ += len;
        return kOk;
    }
    if (!len && !n_rows) return kOk;  // nothing to hand on
    Pending pc;
    pc.req = req;
    pc.len = len;
    pc.n_rows = n_rows;
    pc.text.p = PinnedPool::get().acquire(len + 1);
    const bool recs = sink_->records && n_rows;
    if (recs) pc.recs.p = PinnedPool::get().acquire(n_rows * sizeof(MatchRec));
    if (!pc.text.p || (recs && !pc.recs.p)) {
        err = {kOom, "out of page-locked host memory for a result piece"};
        return err.code;
    }
    if (len) {
        e = cudaMemcpyAsync(pc.text.p, d_text, len, cudaMemcpyDeviceToHost, cs_);
        if (e != cudaSuccess) return cuda_fail(err, e, "result piece copy");
        in_flight_ = true;
    }
    if (recs) {
        e = cudaMemcpyAsync(pc.recs.p, d_recs, n_rows * sizeof(MatchRec), cudaMemcpyDeviceToHost,
                            cs_);
        if (e != cudaSuccess) return cuda_fail(err, e, "match record copy");
        in_flight_ = true;
    }
    if (events_.empty()) {
        cudaEvent_t ev = nullptr;
        e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        if (e != cudaSuccess) return cuda_fail(err, e, "piece event");
        events_.push_back(ev);
    }
    pc.done = events_.back();
    events_.pop_back();
    e = cudaEventRecord(pc.done, cs_);
    if (e != cudaSuccess) {
        events_.push_back(pc.done);
        return cuda_fail(err, e, "piece event");
    }
    out_[req].n_rows += n_rows;
    copied_ += len + (recs ? n_rows * sizeof(MatchRec) : 0);
    pending_.push_back(std::move(pc));
    return kOk;
}

int TextOut::deliver(Pending &pc, Error &err) {
    events_.push_back(pc.done);
    pc.done = nullptr;
    pc.text.p[pc.len] = 0;
    Piece piece;
    piece.request = pc.req;
    piece.text = pc.text.p;
    piece.text_len = pc.len;
    piece.n_rows = pc.n_rows;
    piece.recs = reinterpret_cast<const MatchRec *>(pc.recs.p);
    if (sink_->fn(piece)) {
        for (Pending &q : pending_)
            if (q.done) events_.push_back(q.done);
        pending_.clear();
        err = {kCancelled, "the result sink stopped the search"};
        return err.code;
    }
    return kOk;
}

int TextOut::poll(Error &err) {
    while (sink_ && !pending_.empty()) {
        const cudaError_t e = cudaEventQuery(pending_.front().done);
        if (e == cudaErrorNotReady) return kOk;
        if (e != cudaSuccess) return cuda_fail(err, e, "result piece copy");
        Pending pc = std::move(pending_.front());
        pending_.pop_front();
        if (deliver(pc, err)) return err.code;
    }
    return kOk;
}

int TextOut::drain(Error &err) {
    if (in_flight_) {
        const cudaError_t e = cudaStreamSynchronize(cs_);
        if (e != cudaSuccess) return cuda_fail(err, e, "result copy");
        in_flight_ = false;
    }
    while (!pending_.empty()) {
        Pending pc = std::move(pending_.front());
        pending_.pop_front();
        if (deliver(pc, err)) return err.code;
    }
    return kOk;
}

int TextOut::finish(Error &err) {
    if (drain(err)) return err.code;
    if (!sink_) {
        for (size_t r = 0; r < out_.size(); ++r) {
            if (grow(r, len_[r] + 1, err)) return err.code;
            out_[r].text = out_[r].pooled.p;
            out_[r].text_len = len_[r];
            out_[r].pooled.p[len_[r]] = 0;
        }
    }
    return kOk;
}

}  // namespace cof
