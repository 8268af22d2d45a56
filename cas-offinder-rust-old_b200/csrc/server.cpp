// server.cpp -- continuous-batching request loop over a resident genome
// (cof_server_*, declared in include/cof.h).  No reference counterpart: the
// reference runs one filter per process (cli_utils.rs:97-108).
//
// A worker thread owns the GPU work.  Each pass takes the queued requests in
// arrival order while their estimated device memory for candidate and row
// buffers fits the budget (and while the pass has room, if a per-pass request
// limit is set), runs them as one batched search (one launch per kernel
// stage, scan groups shared by requests with the same filter), copies every
// request's rows into its own result and wakes its waiter.  Requests that
// arrive while a pass is on the GPU are admitted by the next pass.
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
                  Error &err);
uint64_t genome_nucl(const cof_genome *g);
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

    void loop() {
        std::unique_lock<std::mutex> lk(mu);
        while (true) {
            cv_work.wait(lk, [&] { return stop || !queue.empty(); });
            if (stop && queue.empty()) return;
            // admission: arrival order, memory budget, per-pass limit; the
            // first request is always admitted so that none can starve
            std::vector<Pending> batch;
            uint64_t bytes = 0;
            while (!queue.empty()) {
                const Pending &p = queue.front();
                if (!batch.empty() && (bytes + p.est_bytes > budget ||
                                       (max_per_pass && batch.size() >= max_per_pass)))
                    break;
                if (!batch.empty() && p.req.cps != batch[0].req.cps) break;
                bytes += p.est_bytes;
                batch.push_back(std::move(queue.front()));
                queue.pop_front();
            }
            const uint64_t pass = ++passes;
            max_pass_size = std::max<uint64_t>(max_pass_size, batch.size());
            lk.unlock();
            std::vector<cof::Request> reqs;
            for (auto &p : batch) reqs.push_back(p.req);
            std::vector<cof::Result> res;
            cof::Error err;
            const int rc = cof::genome_search(g, reqs, res, err);
            std::vector<Done> out(batch.size());
            const auto now = Clock::now();
            for (size_t i = 0; i < batch.size(); ++i) {
                Done &d = out[i];
                d.status = rc;
                d.pass = pass;
                if (rc) {
                    d.err = err.msg;
                } else {
                    if (res[i].pooled.p && res[i].text == res[i].pooled.p)
                        d.pooled = std::move(res[i].pooled);
                    else
                        d.text.assign(res[i].text ? res[i].text : "", res[i].text_len);
                    d.text_len = res[i].text_len;
                    d.n_rows = res[i].n_rows;
                    d.device_ms = res[i].device_ms;
                }
                d.latency_ms = ms_since(batch[i].t_submit, now);
            }
            lk.lock();
            for (size_t i = 0; i < batch.size(); ++i) done[batch[i].ticket] = std::move(out[i]);
            completed += batch.size();
            cv_done.notify_all();
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
