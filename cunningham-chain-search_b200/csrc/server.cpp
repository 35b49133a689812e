// Served path: continuous batching of range requests over the batched
// executor (ccs_batch_*).  The reference has no server; its closest shape is
// the double-buffered batch loop of v13:3719-4057, which runs one range at a
// time.  Here a scheduler thread keeps up to max_active requests in flight:
// each tick gives every admitted request one chunk of tiles and runs all
// chunks in one graph replay; ticks alternate between two batch executors,
// so tick k is launched before the results of tick k - 1 are collected and
// routed back to their requests (by the range index carried in each record):
// the GPU works on one tick while the host finishes the previous one.
// Queued requests are admitted as soon as a slot is free and the device
// bytes they will hold (their residue rows and their share of the survivor
// and chain buffers of two ticks in flight) fit the memory budget.
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
    uint64_t sched_tiles = 0;           // tiles handed to ticks
    uint64_t done_tiles = 0;            // tiles whose results are routed back
    uint32_t inflight = 0;              // ticks holding a chunk of this request
    uint64_t reserved = 0;
    uint64_t surv_slots = 0;            // survivor records reserved per tick
    uint32_t state = CCS_PENDING;       // CCS_PENDING (queued/active), CCS_OK, CCS_ERR_CANCELLED, CCS_OVERFLOW
    bool overflow = false;              // a tick dropped records of this request (it still runs to the end)
    uint32_t error = CCS_OK;            // a failed tick ends the request with this status
    bool admitted = false;
    bool cancel = false;
    ccs_request_result res{};
    std::vector<ccs_survivor> surv;
    std::vector<ccs_chain> chains;
};

}  // namespace

// one scheduling tick: the chunks it runs and where their results go
struct Tick {
    std::vector<ccs_range> ranges;
    std::vector<Request*> req;
    std::vector<uint64_t> off;
    std::vector<ccs_range_result> res;
    bool live = false;
};

struct ccs_server {
    std::vector<ccs_engine*> prof;
    ccs_server_config cfg{};
    ccs_batch* batch[2] = {nullptr, nullptr};
    Tick tick[2];
    std::vector<double> surv_per_tile;  // expected survivors per tile, per profile
    std::vector<uint64_t> row_bytes;    // device bytes of one residue row, per profile
    uint64_t reserved_peak = 0;
    uint64_t slots_reserved = 0;
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
    std::vector<ccs_survivor> tick_surv;
    std::vector<ccs_chain> tick_chains;
    uint64_t surv_cap = 0, chain_cap = 0;
    std::string err;
    bool tune_pending[2] = {false, false};   // batch tuning to apply before each executor's next tick
    ccs_batch_tuning tune{};
};

namespace {

// Device bytes a request holds while admitted: its residue row (J0 mod q
// for every filter prime, recomputed on the device per chunk) in each of the
// two ticks in flight, plus survivor and chain record slots for the
// survivors its chunk is expected to produce (4x the expectation + 64, for
// each of the two ticks).
void plan_reservation(const ccs_server* s, Request* r) {
    const uint32_t p = r->rg.profile;
    const uint64_t chunk = r->rg.n_tiles < s->cfg.chunk_tiles ? r->rg.n_tiles : s->cfg.chunk_tiles;
    const double expect = s->surv_per_tile[p] * (double)chunk;
    r->surv_slots = (uint64_t)(4.0 * expect) + 64;
    r->reserved = 2 * (s->row_bytes[p] + r->surv_slots * (sizeof(ccs_survivor) + sizeof(ccs_chain)));
}

void finish(ccs_server* s, Request* r, uint32_t status) {
    r->state = status;
    r->res.status = status;
    r->res.done_s = now_s();
    s->reserved -= r->reserved;
    s->slots_reserved -= r->surv_slots;
    r->reserved = 0;
    r->surv_slots = 0;
    if (status == CCS_ERR_CANCELLED) s->st_cancelled++;
    else s->st_completed++;
}

// routes the records of a collected tick back to its requests (lock held)
void route(ccs_server* s, Tick& t, ccs_status st) {
    const uint32_t n = (uint32_t)t.ranges.size();
    if (st != CCS_OK && st != CCS_OVERFLOW) {
        s->err = ccs_last_error();
        for (uint32_t i = 0; i < n; i++) {
            Request* r = t.req[i];
            r->inflight--;
            r->done_tiles += t.ranges[i].n_tiles;
            if (r->error == CCS_OK) r->error = st;
        }
    } else {
        uint64_t ns = 0, nc = 0;
        for (uint32_t i = 0; i < n; i++) { ns += t.res[i].n_survivors; nc += t.res[i].n_chains; }
        if (ns > s->surv_cap) ns = s->surv_cap;
        if (nc > s->chain_cap) nc = s->chain_cap;
        // survivor word 3 = range index within the tick
        for (uint64_t i = 0; i < ns; i++) {
            ccs_survivor v = s->tick_surv[i];
            uint32_t ri = v._pad;
            if (ri >= n) continue;
            v.tile_idx += (uint32_t)t.off[ri];
            v._pad = 0;
            t.req[ri]->surv.push_back(v);
        }
        for (uint64_t i = 0; i < nc; i++) {
            ccs_chain c = s->tick_chains[i];
            if (c.survivor >= ns) continue;
            uint32_t ri = s->tick_surv[c.survivor]._pad;
            if (ri >= n) continue;
            c.tile_idx += (uint32_t)t.off[ri];
            t.req[ri]->chains.push_back(c);
        }
        for (uint32_t i = 0; i < n; i++) {
            Request* r = t.req[i];
            r->res.n_survivors += t.res[i].n_survivors;
            r->res.n_chains += t.res[i].n_chains;
            r->res.n_primes += t.res[i].n_primes;
            r->res.candidates += t.res[i].candidates;
            r->res.ticks++;
            r->inflight--;
            r->done_tiles += t.ranges[i].n_tiles;
            if (t.res[i].status == CCS_OVERFLOW) r->overflow = true;
        }
    }
    t.live = false;
    // requests with every chunk collected (or cancelled / failed, with none in flight)
    for (size_t i = 0; i < s->active.size();) {
        Request* r = s->active[i];
        const bool done = r->done_tiles >= r->rg.n_tiles;
        if (r->inflight == 0 && (done || r->cancel || r->error != CCS_OK)) {
            uint32_t fin = r->cancel ? CCS_ERR_CANCELLED
                         : r->error != CCS_OK ? r->error
                         : r->overflow ? CCS_OVERFLOW : CCS_OK;
            finish(s, r, fin);
            s->active.erase(s->active.begin() + i);
        } else {
            i++;
        }
    }
    s->cv_done.notify_all();
}

void worker_loop(ccs_server* s) {
    std::unique_lock<std::mutex> lk(s->mu);
    int k = 0;                          // executor of the next tick
    while (!s->stop) {
        // admit queued requests while slots and the memory budget allow
        while (!s->pending.empty() && s->active.size() < s->cfg.max_active) {
            Request* r = s->pending.front();
            if (r->cancel) {
                s->pending.pop_front();
                finish(s, r, CCS_ERR_CANCELLED);
                continue;
            }
            plan_reservation(s, r);
            if (!s->active.empty() && (s->reserved + r->reserved > s->cfg.mem_cap_bytes ||
                                       s->slots_reserved + r->surv_slots > s->surv_cap)) {
                r->reserved = 0;
                r->surv_slots = 0;
                break;
            }
            s->pending.pop_front();
            s->reserved += r->reserved;
            s->slots_reserved += r->surv_slots;
            if (s->reserved > s->reserved_peak) s->reserved_peak = s->reserved;
            r->admitted = true;
            r->res.admit_s = now_s();
            s->active.push_back(r);
            s->st_admitted++;
        }
        // cancelled active requests with nothing in flight end now
        for (size_t i = 0; i < s->active.size();) {
            if (s->active[i]->cancel && s->active[i]->inflight == 0) {
                finish(s, s->active[i], CCS_ERR_CANCELLED);
                s->active.erase(s->active.begin() + i);
            } else {
                i++;
            }
        }
        // tick k: the next chunk of every active request that has tiles left
        Tick& t = s->tick[k];
        Tick& prev = s->tick[k ^ 1];
        t.ranges.clear();
        t.req.clear();
        t.off.clear();
        for (Request* r : s->active) {
            if (r->cancel || r->error != CCS_OK || r->sched_tiles >= r->rg.n_tiles) continue;
            uint64_t left = r->rg.n_tiles - r->sched_tiles;
            uint64_t n = left < s->cfg.chunk_tiles ? left : s->cfg.chunk_tiles;
            unsigned __int128 ts = (((unsigned __int128)r->rg.tile_start_hi << 64) | r->rg.tile_start_lo) +
                                   r->sched_tiles;
            ccs_range c = r->rg;
            c.tile_start_lo = (uint64_t)ts;
            c.tile_start_hi = (uint64_t)(ts >> 64);
            c.n_tiles = n;
            t.ranges.push_back(c);
            t.req.push_back(r);
            t.off.push_back(r->sched_tiles);
            r->sched_tiles += n;
            r->inflight++;
        }
        if (t.ranges.empty() && !prev.live) {
            if (s->active.empty()) s->cv_done.notify_all();
            s->cv_work.wait(lk, [&] { return s->stop || !s->pending.empty(); });
            continue;
        }
        // a new batch tuning reaches each executor before its next launch
        const bool retune = s->tune_pending[k] && !t.ranges.empty();
        const ccs_batch_tuning tune = s->tune;
        if (retune) s->tune_pending[k] = false;
        lk.unlock();
        ccs_status st = CCS_OK;
        if (!t.ranges.empty()) {
            if (retune) st = ccs_batch_set_tuning(s->batch[k], &tune);
            if (st == CCS_OK) st = ccs_batch_launch(s->batch[k], t.ranges.data(), (uint32_t)t.ranges.size());
        }
        // collect the previous tick while this one runs on the GPU
        ccs_status pst = CCS_OK;
        if (prev.live)
            pst = ccs_batch_wait(s->batch[k ^ 1], prev.res.data(), s->tick_surv.data(), s->tick_chains.data());
        lk.lock();
        if (prev.live) route(s, prev, pst);
        if (!t.ranges.empty()) {
            s->st_ticks++;
            if (st != CCS_OK) route(s, t, st);     // the launch failed: its chunks end their requests
            else t.live = true;
        }
        k ^= 1;
    }
    // collect a tick still in flight
    for (int i = 0; i < 2; i++) {
        if (!s->tick[i].live) continue;
        lk.unlock();
        ccs_status pst = ccs_batch_wait(s->batch[i], s->tick[i].res.data(), s->tick_surv.data(),
                                        s->tick_chains.data());
        lk.lock();
        route(s, s->tick[i], pst);
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
    for (uint32_t i = 0; i < n_profiles; i++) {
        ccs_info inf;
        ccs_status st = ccs_get_info(profiles[i], &inf);
        if (st != CCS_OK) { delete s; return st; }
        s->surv_per_tile.push_back((double)inf.candidates_per_tile * inf.pass_rate);
        s->row_bytes.push_back(4ull * (inf.n_filter_primes + 64));
    }
    for (int i = 0; i < 2; i++) {
        ccs_status st = ccs_batch_create(profiles, n_profiles, c.max_active, s->surv_cap, s->chain_cap,
                                         &s->batch[i]);
        if (st != CCS_OK) {
            if (i) ccs_batch_destroy(s->batch[0]);
            delete s;
            return st;
        }
        s->tick[i].res.resize(c.max_active);
    }
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
    ccs_batch_destroy(s->batch[0]);
    ccs_batch_destroy(s->batch[1]);
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
    s->tune_pending[0] = s->tune_pending[1] = true;
    return CCS_OK;
}

ccs_status ccs_server_memory(ccs_server* s, uint64_t* reserved_now, uint64_t* reserved_peak) {
    if (!s || !reserved_now || !reserved_peak) return CCS_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    *reserved_now = s->reserved;
    *reserved_peak = s->reserved_peak;
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
