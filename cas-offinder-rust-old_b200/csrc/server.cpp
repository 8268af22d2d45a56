// server.cpp -- continuous-batching request loop over a resident genome
// (cof_server_*, declared in include/cof.h).  No reference counterpart: the
// reference runs one filter per process (cli_utils.rs:97-108).
//
// A worker thread owns the GPU work.  It walks the genome as a ring of
// slices, one slice per step.  Before each step it admits queued requests in
// arrival order while their estimated device memory for candidate and row
// buffers fits the budget (and while the step has room, if a per-pass
// request limit is set); the step then searches its slice for every active
// request as one batched pass (one launch per kernel stage, scan groups
// shared by requests with the same filter).  A request that arrives while
// others are on the GPU thus joins them at the next slice boundary instead
// of waiting for a whole pass, and its work shares their launches.  After
// one full turn of the ring its slices' rows, joined in genome order, are
// its result, and its waiter is woken.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/cof.h"
#include "cof_engine.h"

struct cof_genome;  // cabi.cpp
namespace cof {
int genome_search(cof_genome *g, const std::vector<Request> &reqs, std::vector<Result> &out,
                  Error &err, const SearchRange *range);
uint64_t genome_nucl(const cof_genome *g);
uint64_t genome_stream_nt(const cof_genome *g);
int genome_free_device_bytes(cof_genome *g, uint64_t *free_bytes, Error &err);
}  // namespace cof

namespace {

using Clock = std::chrono::steady_clock;

double ms_since(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

struct Pending {
    uint64_t ticket;
    cof::Request req;
    uint64_t est_bytes;
    Clock::time_point t_submit;
};

struct Done {
    int status = COF_OK;
    std::string err;
    cof::PooledText pooled;  // the rows, when the engine delivered them pooled
    std::string text;        // the rows otherwise
    size_t text_len = 0;
    uint64_t n_rows = 0;
    double device_ms = 0;
    double latency_ms = 0;
    uint64_t pass = 0;
};

// A request on the ring: the slices searched so far, each slice's rows.
struct Active {
    Pending p;
    uint32_t searched = 0;
    std::vector<cof::Result> piece;  // per slice
    double device_ms = 0;
};

}  // namespace

struct cof_server {
    cof_genome *g = nullptr;
    uint32_t max_per_pass = 0;
    uint64_t budget = 0;
    uint64_t genome_nt = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Pending> queue;
    std::unordered_map<uint64_t, Done> done;
    uint64_t next_ticket = 1;
    uint64_t passes = 0, completed = 0, max_pass_size = 0;
    bool stop = false;
    std::thread worker;

    // Device bytes a request may need for candidates and rows: ~48 B per
    // expected row, rows expected at ~1 per pattern per Mbp (popcount) and
    // ~1000x that with bulges, plus 1 MiB of tables.
    uint64_t estimate(const cof::Request &r) const {
        const double mbp = (double)genome_nt / 1e6;
        const double per = (r.max_db || r.max_rb) ? 1000.0 : 1.0;
        return (uint64_t)(48.0 * per * mbp * (double)r.patterns.size()) + (1u << 20);
    }

    // The ring: n_slices slices of the chunk stream, cut[j] the first
    // coordinate of slice j.
    uint32_t n_slices = 1;
    std::vector<uint64_t> cut;

    // A finished request's result: its slices' rows in genome order.
    static Done assemble(Active &a, uint64_t step, Clock::time_point now) {
        Done d;
        d.pass = step;
        d.device_ms = a.device_ms;
        d.latency_ms = ms_since(a.p.t_submit, now);
        auto src = [](const cof::Result &r) -> const char * {
            return r.pooled.p ? r.pooled.p : r.owned.data();
        };
        if (a.piece.size() == 1) {
            cof::Result &r = a.piece[0];
            d.text_len = r.text_len;
            d.n_rows = r.n_rows;
            if (r.pooled.p) d.pooled = std::move(r.pooled);
            else d.text = std::move(r.owned);
            return d;
        }
        size_t total = 0;
        for (const cof::Result &r : a.piece) {
            total += r.text_len;
            d.n_rows += r.n_rows;
        }
        d.pooled.p = cof::PinnedPool::get().acquire(total + 1);
        if (!d.pooled.p) {
            d.status = COF_E_OOM;
            d.err = "out of page-locked host memory for a result";
            return d;
        }
        size_t at = 0;
        for (cof::Result &r : a.piece) {
            if (r.text_len) std::memcpy(d.pooled.p + at, src(r), r.text_len);
            at += r.text_len;
            r.pooled.reset();
            r.owned.clear();
        }
        d.pooled.p[total] = 0;
        d.text_len = total;
        return d;
    }

    void loop() {
        std::vector<Active> active;
        uint32_t cur = 0;  // the slice the next step searches
        std::unique_lock<std::mutex> lk(mu);
        while (true) {
            cv_work.wait(lk, [&] { return stop || !queue.empty() || !active.empty(); });
            if (stop && queue.empty() && active.empty()) return;
            // admission at this slice boundary: arrival order, memory
            // budget, per-step limit; with nothing active the first queued
            // request is always admitted so that none can starve
            uint64_t bytes = 0;
            for (const Active &x : active) bytes += x.p.est_bytes;
            while (!queue.empty()) {
                const Pending &p = queue.front();
                if (!active.empty() && (bytes + p.est_bytes > budget ||
                                        (max_per_pass && active.size() >= max_per_pass)))
                    break;
                if (!active.empty() && p.req.cps != active[0].p.req.cps) break;
                bytes += p.est_bytes;
                Active x;
                x.p = std::move(queue.front());
                queue.pop_front();
                x.piece.resize(n_slices);
                active.push_back(std::move(x));
            }
            const uint64_t step = ++passes;
            max_pass_size = std::max<uint64_t>(max_pass_size, active.size());
            lk.unlock();
            std::vector<cof::Request> reqs;
            for (const Active &x : active) reqs.push_back(x.p.req);
            std::vector<cof::Result> res;
            cof::Error err;
            const cof::SearchRange rg{cut[cur], cur + 1 == n_slices ? ~0ull : cut[cur + 1]};
            const int rc = cof::genome_search(g, reqs, res, err, n_slices > 1 ? &rg : nullptr);
            const auto now = Clock::now();
            std::vector<std::pair<uint64_t, Done>> fin;
            std::vector<Active> keep;
            for (size_t i = 0; i < active.size(); ++i) {
                Active &x = active[i];
                if (rc) {  // the step failed: every request on the ring fails
                    Done d;
                    d.status = rc;
                    d.err = err.msg;
                    d.pass = step;
                    d.latency_ms = ms_since(x.p.t_submit, now);
                    fin.emplace_back(x.p.ticket, std::move(d));
                    continue;
                }
                x.device_ms += res[i].device_ms;
                x.piece[cur] = std::move(res[i]);
                if (++x.searched == n_slices)
                    fin.emplace_back(x.p.ticket, assemble(x, step, now));
                else
                    keep.push_back(std::move(x));
            }
            active = std::move(keep);
            cur = (cur + 1) % n_slices;
            lk.lock();
            for (auto &f : fin) done[f.first] = std::move(f.second);
            completed += fin.size();
            if (!fin.empty()) cv_done.notify_all();
        }
    }
};

namespace cof {
int set_last_error(int code, const std::string &msg);
}

extern "C" {

COF_API int cof_server_create(cof_genome *g, const cof_server_config *cfg, cof_server **out) {
    if (!g || !out) return cof::set_last_error(COF_E_BADINPUT, "null argument");
    *out = nullptr;
    cof_server *s = new cof_server();
    s->g = g;
    s->genome_nt = cof::genome_nucl(g);
    s->max_per_pass = cfg ? cfg->max_requests_per_pass : 0;
    uint64_t budget = cfg ? cfg->memory_budget_bytes : 0;
    if (budget == 0) {
        uint64_t free_b = 0;
        cof::Error err;
        if (cof::genome_free_device_bytes(g, &free_b, err)) {
            delete s;
            return cof::set_last_error(err.code, err.msg);
        }
        budget = free_b / 2;  // half of what is free once the genome is resident
    }
    s->budget = budget;
    // the ring: about one slice per 512 Mnt unless set; whole-genome passes
    // for the plain one-request-per-pass loop
    const uint64_t nt = cof::genome_stream_nt(g);
    uint32_t k = cfg ? cfg->ring_slices : 0;
    if (k == 0) k = (uint32_t)std::min<uint64_t>(16, std::max<uint64_t>(1, (nt + (512ull << 20) - 1) >> 29));
    if (s->max_per_pass == 1) k = 1;
    k = (uint32_t)std::min<uint64_t>(k, std::max<uint64_t>(1, nt));
    s->n_slices = k;
    for (uint32_t j = 0; j < k; ++j) s->cut.push_back(nt * j / k);
    s->worker = std::thread([s] { s->loop(); });
    *out = s;
    return COF_OK;
}

COF_API int cof_server_submit(cof_server *s, const cof_request *r, uint64_t *ticket) {
    if (!s || !r || !ticket) return cof::set_last_error(COF_E_BADINPUT, "null argument");
    Pending p;
    cof::Error err;
    if (cof::make_request(r->search_filter, r->pattern_len, r->patterns, r->n_patterns,
                          r->max_mismatches, r->max_dna_bulges, r->max_rna_bulges, r->flags,
                          r->chunks_per_search, p.req, err))
        return cof::set_last_error(err.code, err.msg);
    p.t_submit = Clock::now();
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return cof::set_last_error(COF_E_STATE, "server is shutting down");
    p.est_bytes = s->estimate(p.req);
    p.ticket = s->next_ticket++;
    *ticket = p.ticket;
    s->queue.push_back(std::move(p));
    s->cv_work.notify_one();
    return COF_OK;
}

COF_API int cof_server_wait(cof_server *s, uint64_t ticket, int64_t timeout_ms, cof_result *out,
                            double *latency_ms) {
    if (!s || !out) return cof::set_last_error(COF_E_BADINPUT, "null argument");
    *out = cof_result{nullptr, 0, 0, 0.0};
    std::unique_lock<std::mutex> lk(s->mu);
    if (ticket == 0 || ticket >= s->next_ticket)
        return cof::set_last_error(COF_E_BADINPUT, "unknown ticket");
    auto ready = [&] { return s->done.count(ticket) != 0; };
    if (timeout_ms < 0) {
        s->cv_done.wait(lk, ready);
    } else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) {
        return cof::set_last_error(COF_E_TIMEOUT, "request still pending");
    }
    Done d = std::move(s->done[ticket]);
    s->done.erase(ticket);
    lk.unlock();
    if (latency_ms) *latency_ms = d.latency_ms;
    if (d.status) return cof::set_last_error(d.status, d.err);
    if (d.pooled.p) {  // handed over as it is; cof_result_free returns it
        out->text = d.pooled.take();
    } else {
        out->text = (char *)std::malloc(d.text.size() + 1);
        if (!out->text) return cof::set_last_error(COF_E_OOM, "out of host memory");
        std::memcpy(out->text, d.text.data(), d.text.size());
        out->text[d.text.size()] = 0;
    }
    out->text_len = d.text_len;
    out->n_rows = d.n_rows;
    out->device_ms = d.device_ms;
    return COF_OK;
}

COF_API int cof_server_stats(cof_server *s, uint64_t *stats4) {
    if (!s || !stats4) return cof::set_last_error(COF_E_BADINPUT, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    stats4[0] = s->passes;
    stats4[1] = s->completed;
    stats4[2] = s->queue.size();
    stats4[3] = s->max_pass_size;
    return COF_OK;
}

COF_API void cof_server_free(cof_server *s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    delete s;
}

}  // extern "C"
