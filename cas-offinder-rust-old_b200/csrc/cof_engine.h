// cof_engine.h -- host-side engine of the B200 off-target search.
//
// Internal C++ interface shared by the C ABI (cabi.cpp), the command-line
// front (cli.cpp) and the CUDA orchestration (engine.cu).
#pragma once

#include <cstddef>
#include <cstdint>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>

#include <pthread.h>
#include <vector>

namespace cof {

constexpr uint32_t kChunkSize = 65536;           // chrom_chunk.rs:1
constexpr uint32_t kChunkBytes = kChunkSize / 2;  // chrom_chunk.rs:2
constexpr uint32_t kDefaultCps = 16384;          // search.rs:22 (GPU batch)
constexpr uint32_t kMaxPatternLen = 64;          // every path (Myers: one u64, myers.rs:3)
constexpr uint32_t kScanWindow = 32;             // cells a scan window holds (one
                                                 // 32-bit plane word); also the
                                                 // planes' leading padding

// Status codes mirrored from include/cof.h.
enum Status : int {
    kOk = 0,
    kBadInput = -1,
    kOom = -2,
    kCuda = -3,
    kIo = -4,
    kUnsupported = -5,
    kState = -6,
    kTimeout = -7,
    kCancelled = -8,
};

struct Error {
    int code = kOk;
    std::string msg;
};

// bit4 one-hot code tables of cas-offinder-lib/src/bit4ops.rs:1-121.
struct Bit4Tables {
    uint8_t str2b4[2][256];  // [mixed_base][char]
    char b4str[16];          // nibble -> uppercase IUPAC char (0 -> NUL)
    Bit4Tables();
};
const Bit4Tables &bit4();
inline uint8_t comp4(uint8_t v) { return (uint8_t)(((v << 2) | (v >> 2)) & 0xF); }
char complement_char(char c);  // bit4ops.rs:211-221
bool is_mixed_base(char c);    // bit4ops.rs:201-203

// The chunk stream of the reference (ChromChunkInfo), tight-packed the way
// chunks_to_searchchunk lays a search batch out (search.rs:1376-1427): chunk
// k occupies bytes [boff[k], boff[k+1]) of `data`.
// The bases of a .2bit file, as its chunks will hold them: for each chunk
// the file offset of its packed bases, its byte offset in the genome's bit4
// stream, its length, and the N ranges (nucleotides relative to the chunk,
// [lo, hi) pairs in nr) that the reference's N-block loop (read_2bit.rs)
// writes into it.  Built from the file's index and N blocks without touching
// a base; the bases are decoded later, on the host or on the device.
struct TwoBitPlan {
    struct Piece {
        uint64_t raw, out;  // file offset of the packed bases; bit4 byte offset
        uint32_t rs, nr;    // nucleotides; first N range (index into nr / 2)
    };
    std::string path;
    uint64_t file_bytes = 0;
    std::vector<Piece> pieces;  // one per chunk, plus a sentinel (nr = end)
    std::vector<uint32_t> nr;
    uint64_t raw_begin = 0, raw_end = 0;  // file bytes holding every chunk's bases
};

// A FASTA file whose chunks are decided (read_fasta.rs) but whose bases are
// not yet converted: the chunks as ranges of the file's lines, [first line,
// next chunk's first line), with their bit4 byte offsets.  Lines are counted
// as the reader counts them: every '\n' ends one, and a last line without
// '\n' counts too.
struct FastaPlan {
    std::string path;
    uint64_t file_bytes = 0;
    uint64_t n_lines = 0;
    std::vector<uint64_t> first_line;  // per chunk, ascending
    std::vector<uint64_t> last_line;   // per chunk: one past its last line
    std::vector<uint64_t> out;         // per chunk: bit4 byte offset
    std::vector<uint32_t> nt;          // per chunk: nucleotides
};

struct HostGenome {
    std::vector<std::string> names;
    std::vector<uint32_t> name_idx;  // per chunk
    std::vector<uint64_t> start, end, boff{0};
    std::vector<uint8_t> data;
    // a .2bit file loaded into an empty genome: its bases are decoded on the
    // device at upload (data stays empty); any other change to the genome
    // first decodes them on the host (materialize)
    std::shared_ptr<TwoBitPlan> deferred;
    std::shared_ptr<FastaPlan> deferred_fa;  // the same for one FASTA file

    size_t n_chunks() const { return start.size(); }
    uint64_t n_nucl() const;
    uint64_t n_bytes() const { return boff.back(); }
    int add_chunk(uint32_t name, uint64_t cs, uint64_t ce, const uint8_t *bytes, Error &err);
    uint32_t add_name(const char *s, size_t n);
    int materialize(Error &err);
};

// Genome loaders (read_fasta.rs, read_2bit.rs, read_fasta_folder.rs,
// dispatch of main.rs:106-121).
int load_genome_path(HostGenome &g, const std::string &path, Error &err);

// One compiled search request.
struct Request {
    std::string filter;
    std::vector<std::string> patterns;  // all patterns, fwd half then reverse half
    uint32_t max_mm = 0, max_db = 0, max_rb = 0;
    uint32_t cps = kDefaultCps;
    uint64_t pam_len = 0;               // main.rs:80-91
    bool raw = false;                   // search()'s raw Match stream, not rows
};
// Validates a cof_request-like description and builds a Request.
int make_request(const char *filter, size_t pattern_len, const char *const *patterns,
                 size_t n_patterns, uint32_t mm, uint32_t db, uint32_t rb, uint32_t flags,
                 uint32_t cps, Request &out, Error &err);

// Page-locked host buffers for result text.  The device copies each
// request's rows straight into one of them, and that buffer becomes the
// caller's cof_result.text; cof_result_free hands it back.  Freed buffers
// are kept (up to kKeepBytes, and always the one returned last) and reused,
// so a steady stream of searches neither pins nor first-touches new host
// pages.
//
// Results of up to kSmallMax bytes (the rows of a few guides) are blocks of
// a power-of-two size class cut from page-locked slabs of at least
// kSlabBytes, so that a pass over hundreds of small requests pins memory
// once instead of once per request.  Slabs stay until exit, kSmallCap bytes
// at most; beyond that small results are allocated like large ones.
class PinnedPool {
  public:
    static constexpr size_t kKeepBytes = size_t(4) << 30;
    static constexpr size_t kMinBlock = size_t(4) << 10;
    static constexpr int kClasses = 9;  // 4 KiB .. 1 MiB
    static constexpr size_t kSmallMax = kMinBlock << (kClasses - 1);
    static constexpr size_t kSlabBytes = size_t(8) << 20;
    static constexpr size_t kSmallCap = size_t(1) << 30;
    static PinnedPool &get();
    char *acquire(size_t bytes);  // nullptr when page-locked memory runs out
    bool release(char *p);        // false when p did not come from the pool

  private:
    char *alloc_large(size_t want);
    std::mutex mu_;
    // live buffer -> (bytes, size class; -1 for a buffer of its own)
    std::unordered_map<char *, std::pair<size_t, int>> live_;
    std::multimap<size_t, char *> free_;
    size_t free_bytes_ = 0;
    std::vector<char *> small_free_[kClasses];
    size_t slab_bytes_ = 0;
};

// A pool buffer owned by one result (move-only; returned to the pool when
// dropped unless taken).
struct PooledText {
    char *p = nullptr;
    PooledText() = default;
    PooledText(const PooledText &) = delete;
    PooledText &operator=(const PooledText &) = delete;
    PooledText(PooledText &&o) noexcept : p(o.p) { o.p = nullptr; }
    PooledText &operator=(PooledText &&o) noexcept {
        if (this != &o) {
            reset();
            p = o.p;
            o.p = nullptr;
        }
        return *this;
    }
    ~PooledText() { reset(); }
    void reset() {
        if (p) PinnedPool::get().release(p);
        p = nullptr;
    }
    char *take() {
        char *q = p;
        p = nullptr;
        return q;
    }
};

// Rows of one request.  `text` points into `pooled` (NUL-terminated, the
// usual case), into `owned`, or -- for the views the engine hands between
// its own stages -- into an engine buffer valid until its next search.
struct Result {
    const char *text = nullptr;
    size_t text_len = 0;
    uint64_t n_rows = 0;
    double device_ms = 0;
    std::string owned;
    PooledText pooled;
};

// One Match of search()'s stream as plain data (cof_match of include/cof.h,
// chrom_chunk.rs:19-29): 32 bytes.
struct MatchRec {
    uint64_t chrom_idx;    // position of the site's first cell in its record
    uint64_t text_offset;  // this match's line in its piece's text
    uint32_t record;       // record (name) index
    uint32_t pattern_idx;  // index in the request's full pattern list
    uint8_t mismatches, dna_bulge_size, rna_bulge_size, is_forward;
    uint32_t pad;
};
static_assert(sizeof(MatchRec) == 32, "MatchRec is cof_match");

// A piece of one request's output, handed to a streaming caller: rows (or
// raw Match lines) in the order of the request's result, valid only during
// the call.
struct Piece {
    size_t request = 0;
    const char *text = nullptr;
    size_t text_len = 0;
    uint64_t n_rows = 0;
    const MatchRec *recs = nullptr;  // n_rows records when Sink::records
};
// Receiver of a streamed search; a nonzero return stops the search.
struct Sink {
    std::function<int(const Piece &)> fn;
    bool records = false;  // pieces carry MatchRec records
};

// Part of the genome a search covers, in global nucleotide coordinates of
// the chunk stream: pattern starts [lo, hi) on the popcount path (rows and
// raw Match lines), alignment end positions [lo, hi) on the bulge path.
// Searches over consecutive ranges partition a whole search's rows; on the
// popcount path their texts, concatenated in range order, are the whole
// search's text.
struct SearchRange {
    uint64_t lo = 0, hi = ~0ull;
};

// Per-stage device timings of the last search (milliseconds, CUDA events).
struct StageTimes {
    double scan_ms = 0, verify_ms = 0, format_ms = 0, d2h_ms = 0, total_ms = 0;
    uint64_t candidates = 0, pairs = 0, raw_hits = 0, rows = 0, kernel_launches = 0;
    int scan_variant = -1;        // tile shape the scan ran with
    int slices = 0;               // slices of a sliced scan (0: one pass)
    std::string scan_shape;
};

// Scan tile-shape choices per request shape.  Enabled unless COF_AUTOTUNE=0;
// if COF_TUNE_CACHE names a file, choices are read from and appended to it.
class Tuner {
  public:
    bool enabled() const;
    bool lookup(const std::string &key, int &variant);
    void store(const std::string &key, int variant);
    std::string report() const;  // JSON object key -> variant index

  private:
    void load();
    std::map<std::string, int> cache_;
    bool loaded_ = false;
};

// Sets the message returned by cof_last_error() on this thread; returns code.
int set_last_error(int code, const std::string &msg);

class DeviceGenome;  // engine.cu

// A genome bound to one GPU: host chunk stream + resident device copy.
class Engine {
  public:
    explicit Engine(int device);
    ~Engine();
    Engine(const Engine &) = delete;
    Engine &operator=(const Engine &) = delete;

    HostGenome &host() { return host_; }
    const HostGenome &host() const { return host_; }
    bool uploaded() const { return dev_ != nullptr; }
    int upload(Error &err);
    // With a sink, the rows are handed to it piece by piece and `out` only
    // receives each request's row count.
    int search(const std::vector<Request> &reqs, std::vector<Result> &out, Error &err,
               const Sink *sink = nullptr, const SearchRange *range = nullptr);
    int free_device_bytes(uint64_t *free_bytes, Error &err);
    const StageTimes &last_times() const { return times_; }
    Tuner &tuner() { return tuner_; }
    int device() const { return device_; }

  private:
    int run_popcount(const std::vector<Request> &reqs, std::vector<Result> &out, Error &err,
                     const Sink *sink, const SearchRange &range);
    int run_bulge(const std::vector<Request> &reqs, std::vector<Result> &out, Error &err,
                  const Sink *sink, const SearchRange &range);
    int run_raw(const Request &req, Result &out, Error &err, const SearchRange &range);
    int device_;
    uint64_t slice_text_hint_ = 0;  // bytes of the last sliced result (+2 %)
    int scan_occ_[16] = {};          // resident CTAs per SM of each scan shape (0: not set up)
    // creates the device's CUDA context while the caller reads the genome
    // file; joined before the first device call, and only by the process
    // that started it (a forked child holds a copy of this object but not
    // the thread)
    pthread_t warm_{};
    bool warm_live_ = false;
    int warm_pid_ = 0;
    void join_warm();
    HostGenome host_;
    DeviceGenome *dev_ = nullptr;
    StageTimes times_;
    Tuner tuner_;
};

}  // namespace cof
