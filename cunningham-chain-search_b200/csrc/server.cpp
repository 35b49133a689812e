// Served path: continuous batching of range requests over the batched
// executor (ccs_batch_*).  The reference has no server; its closest shape is
// the double-buffered batch loop of v13:3719-4057, which runs one range at a
// time.  Here a scheduler thread keeps up to max_active requests in flight:
// each tick gives every admitted request one chunk of tiles, runs all chunks
// in one graph replay, routes survivors and chains back to their requests by
// the range index carried in each record, and admits queued requests as soon
// as slots and the memory budget allow.
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/ccs.h"

namespace {

double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct Request {
    uint64_t id = 0;
    ccs_range rg{};
    uint64_t done_tiles = 0;
    uint64_t reserved = 0;
    uint32_t state = CCS_PENDING;       // CCS_PENDING (queued/active), CCS_OK, CCS_ERR_CANCELLED, CCS_OVERFLOW
    bool admitted = false;
    bool cancel = false;
    ccs_request_result res{};
    std::vector<ccs_survivor> surv;
    std::vector<ccs_chain> chains;
};

}  // namespace

struct ccs_server {
    std::vector<ccs_engine*> prof;
    ccs_server_config cfg{};
    ccs_batch* batch = nullptr;
    std::thread worker;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    bool stop = false;
    uint64_t next_id = 1;
    uint64_t reserved = 0;
    std::deque<Request*> pending;
    std::vector<Request*> active;
    std::unordered_map<uint64_t, Request*> all;
    uint64_t st_submitted = 0, st_admitted = 0, st_completed = 0, st_cancelled = 0, st_ticks = 0;
    std::vector<ccs_range> tick_ranges;
    std::vector<Request*> tick_req;
    std::vector<uint64_t> tick_off;
    std::vector<ccs_range_result> tick_res;
    std::vector<ccs_survivor> tick_surv;
    std::vector<ccs_chain> tick_chains;
    uint64_t surv_cap = 0, chain_cap = 0;
    std::string err;
    bool tune_pending = false;          // batch tuning to apply before the next tick
    ccs_batch_tuning tune{};
};

namespace {

uint64_t reserve_bytes(const ccs_range& rg) {
    // result buffers of one request: a generous per-tile allowance plus a floor
    return 4096 + rg.n_tiles / 64;
}

void finish(ccs_server* s, Request* r, uint32_t status) {
    r->state = status;
    r->res.status = status;
    r->res.done_s = now_s();
    s->reserved -= r->reserved;
    r->reserved = 0;
    if (status == CCS_ERR_CANCELLED) s->st_cancelled++;
    else s->st_completed++;
}

void worker_loop(ccs_server* s) {
    std::unique_lock<std::mutex> lk(s->mu);
    while (!s->stop) {
        // admit queued requests while slots and the memory budget allow
        while (!s->pending.empty() && s->active.size() < s->cfg.max_active) {
            Request* r = s->pending.front();
            if (r->cancel) {
                s->pending.pop_front();
                finish(s, r, CCS_ERR_CANCELLED);
                continue;
            }
            uint64_t need = reserve_bytes(r->rg);
            if (!s->active.empty() && s->reserved + need > s->cfg.mem_cap_bytes) break;
            s->pending.pop_front();
            r->reserved = need;
            s->reserved += need;
            r->admitted = true;
            r->res.admit_s = now_s();
            s->active.push_back(r);
            s->st_admitted++;
        }
        // drop cancelled active requests
        for (size_t i = 0; i < s->active.size();) {
            if (s->active[i]->cancel) {
                finish(s, s->active[i], CCS_ERR_CANCELLED);
                s->active.erase(s->active.begin() + i);
            } else {
                i++;
            }
        }
        if (s->active.empty()) {
            s->cv_done.notify_all();
            s->cv_work.wait(lk, [&] { return s->stop || !s->pending.empty(); });
            continue;
        }
        // one chunk of every active request
        s->tick_ranges.clear();
        s->tick_req.clear();
        s->tick_off.clear();
        for (Request* r : s->active) {
            uint64_t left = r->rg.n_tiles - r->done_tiles;
            uint64_t n = left < s->cfg.chunk_tiles ? left : s->cfg.chunk_tiles;
            unsigned __int128 ts = (((unsigned __int128)r->rg.tile_start_hi << 64) | r->rg.tile_start_lo) +
                                   r->done_tiles;
            ccs_range c = r->rg;
            c.tile_start_lo = (uint64_t)ts;
            c.tile_start_hi = (uint64_t)(ts >> 64);
            c.n_tiles = n;
            s->tick_ranges.push_back(c);
            s->tick_req.push_back(r);
            s->tick_off.push_back(r->done_tiles);
        }
        const uint32_t n = (uint32_t)s->tick_ranges.size();
        const bool retune = s->tune_pending;
        const ccs_batch_tuning tune = s->tune;
        s->tune_pending = false;
        lk.unlock();
        ccs_status st = retune ? ccs_batch_set_tuning(s->batch, &tune) : CCS_OK;
        if (st == CCS_OK)
            st = ccs_batch_run(s->batch, s->tick_ranges.data(), n, s->tick_res.data(),
                               s->tick_surv.data(), s->tick_chains.data(), nullptr);
        lk.lock();
        s->st_ticks++;
        if (st != CCS_OK && st != CCS_OVERFLOW) {
            s->err = ccs_last_error();
            for (Request* r : s->active) finish(s, r, st);
            s->active.clear();
            s->cv_done.notify_all();
            continue;
        }
        uint64_t ns = 0, nc = 0;
        for (uint32_t i = 0; i < n; i++) { ns += s->tick_res[i].n_survivors; nc += s->tick_res[i].n_chains; }
        if (ns > s->surv_cap) ns = s->surv_cap;
        if (nc > s->chain_cap) nc = s->chain_cap;
        // route records: survivor word 3 = range index within the tick
        for (uint64_t i = 0; i < ns; i++) {
            ccs_survivor v = s->tick_surv[i];
            uint32_t ri = v._pad;
            if (ri >= n) continue;
            v.tile_idx += (uint32_t)s->tick_off[ri];
            v._pad = 0;
            s->tick_req[ri]->surv.push_back(v);
        }
        for (uint64_t i = 0; i < nc; i++) {
            ccs_chain c = s->tick_chains[i];
            if (c.survivor >= ns) continue;
            uint32_t ri = s->tick_surv[c.survivor]._pad;
            if (ri >= n) continue;
            c.tile_idx += (uint32_t)s->tick_off[ri];
            s->tick_req[ri]->chains.push_back(c);
        }
        for (uint32_t i = 0; i < n; i++) {
            Request* r = s->tick_req[i];
            r->res.n_survivors += s->tick_res[i].n_survivors;
            r->res.n_chains += s->tick_res[i].n_chains;
            r->res.n_primes += s->tick_res[i].n_primes;
            r->res.candidates += s->tick_res[i].candidates;
            r->res.ticks++;
            r->done_tiles += s->tick_ranges[i].n_tiles;
            if (s->tick_res[i].status == CCS_OVERFLOW) r->state = CCS_OVERFLOW;
        }
        for (size_t i = 0; i < s->active.size();) {
            Request* r = s->active[i];
            if (r->done_tiles >= r->rg.n_tiles) {
                finish(s, r, r->state == CCS_OVERFLOW ? CCS_OVERFLOW : CCS_OK);
                s->active.erase(s->active.begin() + i);
            } else {
                i++;
            }
        }
        s->cv_done.notify_all();
    }
}

}  // namespace

extern "C" {

ccs_status ccs_server_create(ccs_engine* const* profiles, uint32_t n_profiles, const ccs_server_config* cfg,
                             ccs_server** out) {
    if (!profiles || !n_profiles || !out) return CCS_ERR_INVALID;
    *out = nullptr;
    ccs_server* s = new ccs_server();
    s->prof.assign(profiles, profiles + n_profiles);
    ccs_server_config c{};
    c.max_active = 256;
    c.chunk_tiles = 1u << 20;
    c.mem_cap_bytes = 120ull << 30;
    c.max_pending = 1u << 20;
    if (cfg) {
        if (cfg->max_active) c.max_active = cfg->max_active;
        if (cfg->chunk_tiles) c.chunk_tiles = cfg->chunk_tiles;
        if (cfg->mem_cap_bytes) c.mem_cap_bytes = cfg->mem_cap_bytes;
        if (cfg->max_pending) c.max_pending = cfg->max_pending;
    }
    s->cfg = c;
    s->surv_cap = 1u << 22;
    s->chain_cap = 1u << 20;
    ccs_status st = ccs_batch_create(profiles, n_profiles, c.max_active, s->surv_cap, s->chain_cap, &s->batch);
    if (st != CCS_OK) { delete s; return st; }
    s->tick_res.resize(c.max_active);
    s->tick_surv.resize(s->surv_cap);
    s->tick_chains.resize(s->chain_cap);
    s->worker = std::thread(worker_loop, s);
    *out = s;
    return CCS_OK;
}

ccs_status ccs_server_destroy(ccs_server* s) {
    if (!s) return CCS_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    ccs_batch_destroy(s->batch);
    for (auto& kv : s->all) delete kv.second;
    delete s;
    return CCS_OK;
}

ccs_status ccs_submit(ccs_server* s, const ccs_range* rg, uint64_t* id) {
    if (!s || !rg || !id) return CCS_ERR_INVALID;
    if (rg->profile >= s->prof.size() || rg->n_tiles >= (1ull << 32)) return CCS_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->pending.size() >= s->cfg.max_pending) return CCS_ERR_BUSY;
    Request* r = new Request();
    r->id = s->next_id++;
    r->rg = *rg;
    r->res.submit_s = now_s();
    r->res.status = CCS_PENDING;
    if (rg->n_tiles == 0) {
        r->state = CCS_OK;
        r->res.status = CCS_OK;
        r->res.admit_s = r->res.done_s = r->res.submit_s;
        s->st_completed++;
    } else {
        s->pending.push_back(r);
    }
    s->all[r->id] = r;
    s->st_submitted++;
    *id = r->id;
    s->cv_work.notify_one();
    return CCS_OK;
}

ccs_status ccs_poll(ccs_server* s, uint64_t id, ccs_request_result* res, ccs_survivor* surv_host,
                    uint64_t surv_cap, ccs_chain* chains_host, uint64_t chain_cap) {
    if (!s) return CCS_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return CCS_ERR_NOT_FOUND;
    Request* r = it->second;
    if (r->state == CCS_PENDING) {
        if (res) *res = r->res;
        return CCS_PENDING;
    }
    if (res) *res = r->res;
    uint64_t ns = r->surv.size() < surv_cap ? r->surv.size() : surv_cap;
    uint64_t nc = r->chains.size() < chain_cap ? r->chains.size() : chain_cap;
    if (surv_host && ns) memcpy(surv_host, r->surv.data(), sizeof(ccs_survivor) * ns);
    if (chains_host && nc) memcpy(chains_host, r->chains.data(), sizeof(ccs_chain) * nc);
    ccs_status st = (ccs_status)r->state;
    if (st == CCS_OK && (r->surv.size() > surv_cap || r->chains.size() > chain_cap)) st = CCS_OVERFLOW;
    s->all.erase(it);
    delete r;
    return st;
}

ccs_status ccs_wait(ccs_server* s, uint64_t id, uint32_t timeout_ms) {
    if (!s) return CCS_ERR_INVALID;
    std::unique_lock<std::mutex> lk(s->mu);
    auto done = [&] {
        auto it = s->all.find(id);
        return it == s->all.end() || it->second->state != CCS_PENDING;
    };
    if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), done)) return CCS_ERR_TIMEOUT;
    return s->all.count(id) ? CCS_OK : CCS_ERR_NOT_FOUND;
}

ccs_status ccs_cancel(ccs_server* s, uint64_t id) {
    if (!s) return CCS_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return CCS_ERR_NOT_FOUND;
    if (it->second->state == CCS_PENDING) it->second->cancel = true;
    s->cv_work.notify_one();
    return CCS_OK;
}

ccs_status ccs_server_set_batch_tuning(ccs_server* s, const ccs_batch_tuning* t) {
    if (!s || !t) return CCS_ERR_INVALID;
    if (t->block_threads && t->block_threads != 128 && t->block_threads != 256) return CCS_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    s->tune = *t;
    s->tune_pending = true;
    return CCS_OK;
}

ccs_status ccs_server_stats(ccs_server* s, uint64_t* out6) {
    if (!s || !out6) return CCS_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    out6[0] = s->st_submitted;
    out6[1] = s->st_admitted;
    out6[2] = s->st_completed;
    out6[3] = s->st_cancelled;
    out6[4] = s->st_ticks;
    out6[5] = s->pending.size();
    return CCS_OK;
}

}  // extern "C"
