// cabi.cpp -- extern "C" entry points of libcof.so (declared in include/cof.h).
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>
#include <algorithm>

#include "../../include/cof.h"
#include "cof_engine.h"

struct cof_genome {
    cof::Engine engine;
    std::mutex mu;
    explicit cof_genome(int dev) : engine(dev) {}
};

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}
int fail(const cof::Error &e) { return fail(e.code, e.msg); }

int to_requests(const cof_request *reqs, size_t n, std::vector<cof::Request> &out,
                cof::Error &err) {
    out.resize(n);
    for (size_t i = 0; i < n; ++i) {
        const cof_request &r = reqs[i];
        if (cof::make_request(r.search_filter, r.pattern_len, r.patterns, r.n_patterns,
                              r.max_mismatches, r.max_dna_bulges, r.max_rna_bulges, r.flags,
                              r.chunks_per_search, out[i], err))
            return err.code;
    }
    return 0;
}

// Copies a result out of the engine's pinned buffer (large copies are split
// across threads: one host thread moves ~10 GB/s).
void parallel_copy(char *dst, const char *src, size_t n) {
    const size_t kPiece = 16u << 20;
    if (n < 2 * kPiece) {
        std::memcpy(dst, src, n);
        return;
    }
    unsigned nt = std::min<unsigned>(8, std::max(1u, std::thread::hardware_concurrency()));
    std::vector<std::thread> th;
    const size_t per = (n + nt - 1) / nt;
    for (unsigned t = 0; t < nt; ++t) {
        const size_t a = t * per, b = std::min(n, a + per);
        if (a >= b) break;
        th.emplace_back([=] { std::memcpy(dst + a, src + a, b - a); });
    }
    for (auto &x : th) x.join();
}

// Hands a result to the caller: a page-locked pool buffer changes owner as
// it is (cof_result_free returns it to the pool); anything else is copied
// into malloc'd memory.
int fill_result(cof::Result &r, cof_result *out) {
    if (r.pooled.p && r.text == r.pooled.p) {
        out->text = r.pooled.take();
    } else {
        out->text = (char *)std::malloc(r.text_len + 1);
        if (!out->text) return fail(COF_E_OOM, "out of host memory for result text");
        if (r.text_len) parallel_copy(out->text, r.text, r.text_len);
        out->text[r.text_len] = 0;
    }
    out->text_len = r.text_len;
    out->n_rows = r.n_rows;
    out->device_ms = r.device_ms;
    return COF_OK;
}

}  // namespace

namespace cof {
// Records a failure for cof_last_error() from code outside this file.
int set_last_error(int code, const std::string &msg) { return fail(code, msg); }

// Entry points of the request server (server.cpp) into a genome handle.
// A result that is neither pooled nor owned points into an engine buffer
// that the next search on this genome overwrites, so it becomes owned
// before the lock is let go.
int genome_search(cof_genome *g, const std::vector<Request> &reqs, std::vector<Result> &out,
                  Error &err, const SearchRange *range) {
    std::lock_guard<std::mutex> lk(g->mu);
    const int rc = g->engine.search(reqs, out, err, nullptr, range);
    if (rc) return rc;
    for (Result &r : out) {
        if (r.text && r.text != r.owned.data() && r.text != r.pooled.p) {
            r.owned.assign(r.text, r.text_len);
            r.text = r.owned.data();
        }
    }
    return rc;
}
uint64_t genome_nucl(const cof_genome *g) { return g->engine.host().n_nucl(); }
// Length of the genome's chunk stream (2 x its bytes: odd chunks leave a
// pad nibble), the coordinate space of SearchRange.
uint64_t genome_stream_nt(const cof_genome *g) { return 2 * g->engine.host().n_bytes(); }
int genome_free_device_bytes(cof_genome *g, uint64_t *free_bytes, Error &err) {
    std::lock_guard<std::mutex> lk(g->mu);
    if (g->engine.upload(err)) return err.code;
    return g->engine.free_device_bytes(free_bytes, err);
}
}  // namespace cof

extern "C" {

COF_API int cof_abi_version(void) { return COF_ABI_VERSION; }

COF_API const char *cof_last_error(void) { return g_last_error.c_str(); }

COF_API int cof_genome_create(int device, cof_genome **out) {
    if (!out) return fail(COF_E_BADINPUT, "null output handle");
    *out = nullptr;
    cof_genome *g = new (std::nothrow) cof_genome(device);
    if (!g) return fail(COF_E_OOM, "out of host memory");
    *out = g;
    g_last_error.clear();
    return COF_OK;
}

COF_API int cof_genome_add_chunk(cof_genome *g, const char *chr_name, const uint8_t *bit4,
                                 uint64_t chunk_start, uint64_t chunk_end) {
    if (!g || !chr_name || (!bit4 && chunk_end > chunk_start))
        return fail(COF_E_BADINPUT, "null argument");
    std::lock_guard<std::mutex> lk(g->mu);
    if (g->engine.uploaded()) return fail(COF_E_STATE, "genome already uploaded");
    cof::HostGenome &h = g->engine.host();
    if (chunk_end == chunk_start) return COF_OK;  // empty chunks carry nothing
    uint32_t name;
    if (chunk_start != 0 && !h.name_idx.empty() && h.names[h.name_idx.back()] == chr_name)
        name = h.name_idx.back();  // next chunk of the same record
    else
        name = h.add_name(chr_name, std::strlen(chr_name));
    cof::Error err;
    if (h.add_chunk(name, chunk_start, chunk_end, bit4, err)) return fail(err);
    return COF_OK;
}

COF_API int cof_genome_load(cof_genome *g, const char *path) {
    if (!g || !path) return fail(COF_E_BADINPUT, "null argument");
    std::lock_guard<std::mutex> lk(g->mu);
    if (g->engine.uploaded()) return fail(COF_E_STATE, "genome already uploaded");
    cof::Error err;
    if (cof::load_genome_path(g->engine.host(), path, err)) return fail(err);
    return COF_OK;
}

COF_API int cof_genome_upload(cof_genome *g) {
    if (!g) return fail(COF_E_BADINPUT, "null genome");
    std::lock_guard<std::mutex> lk(g->mu);
    cof::Error err;
    if (g->engine.upload(err)) return fail(err);
    return COF_OK;
}

COF_API uint64_t cof_genome_n_nucl(const cof_genome *g) {
    return g ? g->engine.host().n_nucl() : 0;
}

COF_API uint64_t cof_genome_n_chunks(const cof_genome *g) {
    return g ? g->engine.host().n_chunks() : 0;
}

COF_API void cof_genome_free(cof_genome *g) { delete g; }

COF_API int cof_search_batch(cof_genome *g, const cof_request *reqs, size_t n_reqs,
                             cof_result *outs) {
    if (!g || (!reqs && n_reqs) || (!outs && n_reqs)) return fail(COF_E_BADINPUT, "null argument");
    for (size_t i = 0; i < n_reqs; ++i) outs[i] = cof_result{nullptr, 0, 0, 0.0};
    cof::Error err;
    std::vector<cof::Request> rq;
    if (to_requests(reqs, n_reqs, rq, err)) return fail(err);
    std::vector<cof::Result> res;
    std::lock_guard<std::mutex> lk(g->mu);
    if (g->engine.search(rq, res, err)) return fail(err);
    for (size_t i = 0; i < n_reqs; ++i) {
        if (int rc = fill_result(res[i], &outs[i])) {
            for (size_t j = 0; j < i; ++j) cof_result_free(&outs[j]);
            return rc;
        }
    }
    return COF_OK;
}

COF_API int cof_search(cof_genome *g, const cof_request *req, cof_result *out) {
    return cof_search_batch(g, req, 1, out);
}

static_assert(sizeof(cof_match) == sizeof(cof::MatchRec) &&
                  offsetof(cof_match, text_offset) == offsetof(cof::MatchRec, text_offset) &&
                  offsetof(cof_match, record) == offsetof(cof::MatchRec, record) &&
                  offsetof(cof_match, mismatches) == offsetof(cof::MatchRec, mismatches) &&
                  offsetof(cof_match, is_forward) == offsetof(cof::MatchRec, is_forward),
              "cof_match and the engine's match record differ");

COF_API int cof_search_stream(cof_genome *g, const cof_request *reqs, size_t n_reqs,
                              uint32_t stream_flags, cof_sink sink, void *user,
                              uint64_t *n_rows) {
    if (!g || (!reqs && n_reqs) || !sink) return fail(COF_E_BADINPUT, "null argument");
    if (stream_flags & ~COF_STREAM_MATCHES) return fail(COF_E_BADINPUT, "unknown stream flag");
    cof::Error err;
    std::vector<cof::Request> rq;
    if (to_requests(reqs, n_reqs, rq, err)) return fail(err);
    cof::Sink sk;
    sk.records = (stream_flags & COF_STREAM_MATCHES) != 0;
    sk.fn = [sink, user](const cof::Piece &p) {
        cof_piece c;
        c.request = p.request;
        c.text = p.text;
        c.text_len = p.text_len;
        c.n_rows = p.n_rows;
        c.matches = reinterpret_cast<const cof_match *>(p.recs);
        return sink(user, &c);
    };
    std::vector<cof::Result> res;
    std::lock_guard<std::mutex> lk(g->mu);
    if (g->engine.search(rq, res, err, &sk)) return fail(err);
    if (n_rows)
        for (size_t i = 0; i < n_reqs; ++i) n_rows[i] = res[i].n_rows;
    return COF_OK;
}

COF_API uint32_t cof_genome_n_records(const cof_genome *g) {
    return g ? (uint32_t)g->engine.host().names.size() : 0;
}

COF_API const char *cof_genome_record_name(const cof_genome *g, uint32_t record) {
    if (!g || record >= g->engine.host().names.size()) return nullptr;
    return g->engine.host().names[record].c_str();
}

COF_API void cof_result_free(cof_result *r) {
    if (!r) return;
    if (!cof::PinnedPool::get().release(r->text)) std::free(r->text);
    r->text = nullptr;
    r->text_len = 0;
    r->n_rows = 0;
}

// Stage timings of the last search on a genome (milliseconds / counts), for
// benchmarking and profiling: scan, verify, format, d2h, total; PAM-passing
// windows, window x pattern pairs, scan candidates, rows, kernel launches.
// Not part of the reference interface.
COF_API int cof_genome_last_stats(const cof_genome *g, double *ms5, uint64_t *counts5) {
    if (!g || !ms5 || !counts5) return fail(COF_E_BADINPUT, "null argument");
    const cof::StageTimes &t = g->engine.last_times();
    ms5[0] = t.scan_ms;
    ms5[1] = t.verify_ms;
    ms5[2] = t.format_ms;
    ms5[3] = t.d2h_ms;
    ms5[4] = t.total_ms;
    counts5[0] = t.candidates;
    counts5[1] = t.pairs;
    counts5[2] = t.raw_hits;
    counts5[3] = t.rows;
    counts5[4] = t.kernel_launches;
    return COF_OK;
}

// Autotuner state of a genome: JSON {"last": tile shape of the last scan,
// "variant": its index, "slices": slices the last scan ran in (0: one pass),
// "cache": {shape key: variant index}}.  No reference counterpart.
COF_API int cof_genome_tuning(cof_genome *g, char *buf, size_t len) {
    if (!g || !buf || !len) return fail(COF_E_BADINPUT, "null argument");
    std::lock_guard<std::mutex> lk(g->mu);
    const cof::StageTimes &t = g->engine.last_times();
    std::string js = "{\"last\": \"" + t.scan_shape + "\", \"variant\": " +
                     std::to_string(t.scan_variant) + ", \"slices\": " +
                     std::to_string(t.slices) + ", \"cache\": " +
                     g->engine.tuner().report() + "}";
    std::snprintf(buf, len, "%s", js.c_str());
    return js.size() < len ? COF_OK : fail(COF_E_BADINPUT, "buffer too small");
}

}  // extern "C"
