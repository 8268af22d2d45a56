// textout.h -- result text (and match records) from device memory to the
// caller, beside the next slice's or chunk's device work.
//
// A search pass produces its output in pieces: a popcount slice, a bulge
// candidate chunk, or a whole pass split by request.  Each piece's device
// text is copied on the copy stream once the compute stream has written it
// (an event), so the copy runs while the GPU works on the next piece.  Two
// modes:
//   assemble : every request's pieces are appended, in order, to one
//              page-locked result buffer of its own (the cof_result text);
//              a buffer whose size estimate falls short grows (the copies
//              into it are waited for, the bytes kept).
//   sink     : every piece lands in a page-locked staging buffer and is
//              handed to the caller's sink once its copy is done (drain());
//              nothing accumulates, so results larger than host memory can
//              stream through.  This is the dest channel of search()
//              (search.rs:1490-1500), which moves Vec<Match> batches to the
//              writer as they are found.
#pragma once

#include <cuda_runtime.h>

#include <deque>
#include <vector>

#include "cof_engine.h"

namespace cof {

class TextOut {
  public:
    // out: one Result per request (assemble mode fills text, text_len and
    // n_rows; sink mode only n_rows).
    TextOut(cudaStream_t copy_stream, const Sink *sink, std::vector<Result> &out)
        : cs_(copy_stream), sink_(sink), out_(out), cap_(out.size(), 0), len_(out.size(), 0) {}
    ~TextOut();
    TextOut(const TextOut &) = delete;
    TextOut &operator=(const TextOut &) = delete;

    bool streaming() const { return sink_ != nullptr; }
    bool records() const { return sink_ && sink_->records; }
    // Assemble mode: at least `bytes` of text are expected for request req
    // in total (a larger buffer is allocated now, keeping what is there).
    int reserve(size_t req, size_t bytes, Error &err);
    // After `ready` (an event recorded on the compute stream once the text
    // is written), copies `len` bytes of device text holding `n_rows` rows
    // of request `req`; in sink mode with records also the n_rows records at
    // d_recs.  The device text must stay unchanged until drain() returns.
    int put(size_t req, const char *d_text, size_t len, uint64_t n_rows, const MatchRec *d_recs,
            cudaEvent_t ready, Error &err);
    // Waits for every copy in flight; sink mode then hands the copied pieces
    // to the sink in the order they were put.  A sink that returns nonzero
    // cancels the search (kCancelled).
    int drain(Error &err);
    // Sink mode: hands on the pieces, in order, whose copies have finished,
    // without waiting for the others (nothing in assemble mode).
    int poll(Error &err);
    // drain(), then NUL-terminates the assembled texts.
    int finish(Error &err);
    uint64_t bytes_copied() const { return copied_; }

  private:
    struct Pending {
        size_t req;
        size_t len;
        uint64_t n_rows;
        PooledText text, recs;
        cudaEvent_t done = nullptr;  // recorded on the copy stream after its copies
    };
    int grow(size_t req, size_t need, Error &err);
    int deliver(Pending &pc, Error &err);
    std::vector<cudaEvent_t> events_;  // spare completion events
    cudaStream_t cs_;
    const Sink *sink_;
    std::vector<Result> &out_;
    std::vector<size_t> cap_, len_;
    std::deque<Pending> pending_;
    uint64_t copied_ = 0;
    bool in_flight_ = false;
};

}  // namespace cof
