// Batched and served proving (lg_server_*, lg_prove_batch).
//
// A server owns `workers` threads, each with its own context (stream,
// arenas, cached RS tables) on one device.  Requests queue FIFO and are
// admitted when their device footprint fits the HBM budget next to the
// requests already in flight; an admitted request is proved by the next
// free worker, so requests that arrive while others run start as soon as a
// worker and memory free up, and their kernels and host transcript work
// overlap with the others'.  A server with one worker is the FIFO loop of
// the plain prover.
//
// Admission charges each request its peak device footprint, and the server
// charges what its contexts keep between requests (arenas, FFT tables and
// the device's shared code tables), so that the budget bounds the device
// memory in use.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/ligerito_b200.h"
#include "lg_host.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    uint64_t id = 0;
    lg_config cfg{};
    const uint32_t *poly = nullptr;
    uint64_t len = 0;
    int on_device = 0;
    std::vector<uint32_t> owned;  // copy of host input when asked for
    uint64_t mem = 0;             // admission footprint
    Clock::time_point t_submit, t_start, t_done;
    int worker = -1;      // the worker that must prove it (-1: any)
    int waiters = 0;      // threads inside lg_server_wait for it
    bool claimed = false; // its result was handed out
    bool done = false;
    lg_status st = LG_OK;
    lg_proof *proof = nullptr;
};

// Device bytes one proof holds at its peak: the input when it is on the
// host, the first encoded matrix (16 bytes per coefficient), its tree (4
// per coefficient), the scaled columns the encoding reads (4 per
// coefficient), the folded vectors and the per-context arenas.
uint64_t footprint(const lg_config &c, uint64_t len, int on_device) {
    uint64_t b = 16 * len + 4 * len + 4 * len + (len >> c.initial_k) * 4 * 4 + (48ull << 20);
    if (!on_device) b += 4 * len;
    return b;
}

}  // namespace

struct lg_server {
    int device = 0;
    uint64_t budget = 0, in_flight = 0;
    std::vector<lg_ctx *> ctxs;
    std::vector<std::thread> threads;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request *> pending;
    std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs;
    uint64_t next_id = 1, completed = 0;
    uint32_t max_batch = 1;  // same-config requests a worker proves in lockstep
    bool stop = false;
    Clock::time_point t0 = Clock::now();

    // device bytes the contexts keep between requests: each one's arena and
    // FFT tables, and the code tables they share
    uint64_t cached() const {
        uint64_t b = lg_device_table_bytes(device);
        for (auto *c : ctxs) b += lg_ctx_device_bytes_cached(c);
        return b;
    }

    // the first queued request this worker may take (FIFO among those)
    std::deque<Request *>::iterator next_for(int w) {
        for (auto it = pending.begin(); it != pending.end(); ++it)
            if ((*it)->worker < 0 || (*it)->worker == w) return it;
        return pending.end();
    }
    bool admissible(const Request *r) const {
        return budget == 0 || in_flight == 0 || r->mem + in_flight + cached() <= budget;
    }

    static bool same_shape(const Request *a, const Request *b) {
        return a->len == b->len && a->on_device == b->on_device && std::memcmp(&a->cfg, &b->cfg, sizeof a->cfg) == 0;
    }

    void worker(int w, lg_ctx *ctx) {
        std::vector<Request *> batch;
        std::vector<const uint32_t *> polys;
        std::vector<lg_proof *> outs;
        for (;;) {
            Request *r = nullptr;
            batch.clear();
            {
                std::unique_lock<std::mutex> lk(mu);
                std::deque<Request *>::iterator it;
                cv_work.wait(lk, [&] {
                    if (stop && pending.empty()) return true;
                    it = next_for(w);
                    return it != pending.end() && admissible(*it);
                });
                if (stop && pending.empty()) return;
                r = *it;
                pending.erase(it);
                in_flight += r->mem;
                batch.push_back(r);
                // queued requests of the same config join it, in queue
                // order, while they fit the budget
                for (auto jt = pending.begin(); jt != pending.end() && batch.size() < max_batch;) {
                    Request *x = *jt;
                    if ((x->worker < 0 || x->worker == w) && same_shape(x, r) && admissible(x)) {
                        in_flight += x->mem;
                        batch.push_back(x);
                        jt = pending.erase(jt);
                    } else {
                        ++jt;
                    }
                }
                const auto now = Clock::now();
                for (auto *x : batch) x->t_start = now;
            }
            outs.assign(batch.size(), nullptr);
            lg_status st;
            if (batch.size() == 1) {
                st = lg_prove(ctx, &r->cfg, r->poly, r->len, r->on_device, &outs[0]);
            } else {
                polys.clear();
                for (auto *x : batch) polys.push_back(x->poly);
                st = lg_prove_lockstep(ctx, &r->cfg, polys.data(), r->len, (uint32_t)batch.size(), r->on_device,
                                       outs.data());
            }
            {
                std::lock_guard<std::mutex> lk(mu);
                const auto now = Clock::now();
                for (size_t i = 0; i < batch.size(); ++i) {
                    Request *x = batch[i];
                    in_flight -= x->mem;
                    x->proof = outs[i];
                    x->st = outs[i] ? LG_OK : (st != LG_OK ? st : LG_ERR_PROVER_ASSERT);
                    x->t_done = now;
                    x->done = true;
                    x->owned.clear();
                    x->owned.shrink_to_fit();
                    ++completed;
                }
            }
            cv_done.notify_all();
            cv_work.notify_all();
        }
    }
};

extern "C" {

lg_status lg_server_create(int device, uint64_t hbm_budget_bytes, uint32_t workers, lg_server **out) {
    if (!out || workers == 0 || workers > 256) return LG_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    auto *s = new (std::nothrow) lg_server;
    if (!s) return LG_ERR_OUT_OF_MEMORY;
    s->device = device;
    s->budget = hbm_budget_bytes;
    for (uint32_t i = 0; i < workers; ++i) {
        lg_ctx *c = nullptr;
        lg_status st = lg_ctx_create(device, 0, &c);
        if (st != LG_OK) {
            for (auto *x : s->ctxs) lg_ctx_destroy(x);
            delete s;
            return st;
        }
        s->ctxs.push_back(c);
    }
    for (uint32_t i = 0; i < workers; ++i) {
        lg_ctx *c = s->ctxs[i];
        s->threads.emplace_back([s, i, c] { s->worker((int)i, c); });
    }
    *out = s;
    return LG_OK;
}

lg_status lg_server_set_max_batch(lg_server *s, uint32_t max_batch) {
    if (!s || max_batch == 0 || max_batch > 64) return LG_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(s->mu);
    s->max_batch = max_batch;
    return LG_OK;
}

lg_status lg_server_submit(lg_server *s, const lg_config *cfg, const uint32_t *poly, uint64_t len,
                           int poly_on_device, int copy_input, uint64_t *ticket) {
    if (!s || !cfg || !poly || !ticket) return LG_ERR_INVALID_ARGUMENT;
    lg_status st = lg::config_check(*cfg, len);
    if (st != LG_OK) return st;
    auto r = std::make_unique<Request>();
    r->cfg = *cfg;
    r->len = len;
    r->on_device = poly_on_device;
    if (copy_input && !poly_on_device) {
        r->owned.assign(poly, poly + len);
        r->poly = r->owned.data();
    } else {
        r->poly = poly;
    }
    r->mem = footprint(*cfg, len, poly_on_device);
    r->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        r->id = s->next_id++;
        *ticket = r->id;
        s->pending.push_back(r.get());
        s->reqs.emplace(r->id, std::move(r));
    }
    s->cv_work.notify_all();
    return LG_OK;
}

lg_status lg_server_wait(lg_server *s, uint64_t ticket, int64_t timeout_ms, lg_proof **proof, double *latency_ms,
                         double *queue_ms) {
    if (!s || !proof) return LG_ERR_INVALID_ARGUMENT;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end() || it->second->claimed) return LG_ERR_INVALID_ARGUMENT;
    Request *r = it->second.get();
    // the request stays in the map while any thread waits on it; the last
    // one out after it was claimed erases it
    ++r->waiters;
    auto ready = [&] { return r->done || r->claimed; };
    bool ok = true;
    if (timeout_ms < 0) s->cv_done.wait(lk, ready);
    else ok = s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready);
    --r->waiters;
    lg_status st;
    if (r->claimed) {
        st = LG_ERR_INVALID_ARGUMENT;  // another waiter took the result
    } else if (!ok) {
        return LG_ERR_TIMEOUT;
    } else {
        r->claimed = true;
        *proof = r->proof;
        r->proof = nullptr;
        if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
        if (queue_ms) *queue_ms = std::chrono::duration<double, std::milli>(r->t_start - r->t_submit).count();
        st = r->st;
        s->cv_done.notify_all();  // other waiters on this ticket learn it was claimed
    }
    if (r->waiters == 0) s->reqs.erase(r->id);
    return st;
}

lg_status lg_server_stats(lg_server *s, uint64_t *completed, uint64_t *queued, uint64_t *in_flight_bytes) {
    if (!s) return LG_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(s->mu);
    if (completed) *completed = s->completed;
    if (queued) *queued = s->pending.size();
    if (in_flight_bytes) *in_flight_bytes = s->in_flight;
    return LG_OK;
}

void lg_server_destroy(lg_server *s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    for (auto &t : s->threads) t.join();
    for (auto &kv : s->reqs)
        if (kv.second->proof) lg_proof_free(kv.second->proof);
    for (auto *c : s->ctxs) lg_ctx_destroy(c);
    delete s;
}

lg_status lg_server_warm(lg_server *s, const lg_config *cfgs, uint32_t count) {
    if (!s || (!cfgs && count)) return LG_ERR_INVALID_ARGUMENT;
    uint64_t maxlen = 0;
    for (uint32_t i = 0; i < count; ++i) {
        const uint64_t len = 1ull << (cfgs[i].initial_log_m + cfgs[i].initial_log_n);
        if (lg::config_check(cfgs[i], len) != LG_OK) return LG_ERR_INVALID_CONFIG;
        maxlen = std::max(maxlen, len);
    }
    if (!count) return LG_OK;
    // one device input of the largest size; every warm-up proof reads a prefix
    uint32_t *d = nullptr;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(s->device);
    if (cudaMalloc(&d, 4 * maxlen) != cudaSuccess) {
        cudaGetLastError();
        cudaSetDevice(prev);
        return LG_ERR_OUT_OF_MEMORY;
    }
    lg_status st = lg_fill_splitmix(s->ctxs[0], 0, d, maxlen);
    if (st == LG_OK) st = lg_ctx_synchronize(s->ctxs[0]);
    std::vector<uint64_t> tickets;
    if (st == LG_OK) {
        std::lock_guard<std::mutex> lk(s->mu);
        for (uint32_t i = 0; i < count; ++i)
            for (size_t w = 0; w < s->ctxs.size(); ++w) {
                auto r = std::make_unique<Request>();
                r->cfg = cfgs[i];
                r->len = 1ull << (cfgs[i].initial_log_m + cfgs[i].initial_log_n);
                r->poly = d;
                r->on_device = 1;
                r->worker = (int)w;
                r->mem = 0;  // warm-up runs outside the budget
                r->t_submit = Clock::now();
                r->id = s->next_id++;
                tickets.push_back(r->id);
                s->pending.push_back(r.get());
                s->reqs.emplace(r->id, std::move(r));
            }
    }
    s->cv_work.notify_all();
    for (uint64_t t : tickets) {
        lg_proof *p = nullptr;
        lg_status x = lg_server_wait(s, t, -1, &p, nullptr, nullptr);
        if (p) lg_proof_free(p);
        if (x != LG_OK && st == LG_OK) st = x;
    }
    cudaFree(d);
    cudaSetDevice(prev);
    return st;
}

// same-config proofs lg_prove_batch runs in lockstep on one worker
constexpr uint32_t kBatchLockstep = 8;

lg_status lg_prove_batch(int device, uint32_t workers, const lg_config *cfgs, const uint32_t *const *polys,
                         const uint64_t *lens, int polys_on_device, uint32_t count, lg_proof **out) {
    if (!cfgs || !polys || !lens || !out) return LG_ERR_INVALID_ARGUMENT;
    for (uint32_t i = 0; i < count; ++i) out[i] = nullptr;
    lg_server *s = nullptr;
    lg_status st = lg_server_create(device, 0, std::max<uint32_t>(1, std::min(workers, count)), &s);
    if (st != LG_OK) return st;
    lg_server_set_max_batch(s, kBatchLockstep);
    std::vector<uint64_t> tickets(count);
    lg_status first = LG_OK;
    for (uint32_t i = 0; i < count; ++i) {
        st = lg_server_submit(s, &cfgs[i], polys[i], lens[i], polys_on_device, 0, &tickets[i]);
        if (st != LG_OK) { first = st; tickets[i] = 0; }
    }
    for (uint32_t i = 0; i < count; ++i) {
        if (!tickets[i]) continue;
        st = lg_server_wait(s, tickets[i], -1, &out[i], nullptr, nullptr);
        if (st != LG_OK && first == LG_OK) first = st;
    }
    lg_server_destroy(s);
    return first;
}

}  // extern "C"
