// psx_serve.cpp -- the served loop: segmented searches of uneven transform
// length, DM count and acceleration range, admitted as they arrive while
// others are on the GPU.
//
// The reference searches one observation per process with one Worker per
// GPU (src/pipeline_multi.cu:111-303, 523-535); nothing here replaces a
// reference function.  Each admitted request runs through one search
// instance (psx_search_block, the Worker's DM loop) on its own CUDA streams,
// so the GPU work of concurrent requests overlaps.  Admission is FIFO and
// by device memory: a request is admitted when a worker slot is free and
// the bytes it needs fit the budget.  Instances outlive their requests in a
// pool keyed by what their buffers and plans depend on (transform length,
// mode, batch, harmonic shape; not the fold count, which only selects the
// harmonic kernel at launch); a later request with the same key is
// retargeted onto a pooled instance (psx_search_retarget) instead of
// allocating, and idle pooled instances are destroyed, oldest first, when a
// new one needs their memory.
//
// Between running requests, the one with the least work (acceleration
// trials times transform length, summed over its DM trials) runs at the
// device's greatest stream priority: a short request admitted beside a long
// one finishes close to its isolated time, and the long one loses only the
// short one's work.  The exclusive policy runs one request at a time
// instead (a batched search fills the device by itself, so sharing it adds
// latency to every request it overlaps), choosing the pending request with
// the least work, or one that has been passed over kMaxPassedOver times.
// (Building the next request's instance while the current one runs was
// measured slower: the allocations and frees of the build stall the
// running request.)
#include <cuda_runtime.h>
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>
#include "peasoup_b200.h"

namespace psx {
void set_error(const char* fmt, ...);
void clear_error();
}  // namespace psx

namespace {

using Clock = std::chrono::steady_clock;

// Exclusive policy: admissions that may go ahead of a pending request
// before it is admitted regardless of its work (no starvation).
constexpr int kMaxPassedOver = 8;

struct EngineKey {
    size_t n;
    int mode, batch, shape, callback, lanes, form, group;
    bool operator==(const EngineKey& o) const
    {
        return n == o.n && mode == o.mode && batch == o.batch &&
               shape == o.shape && callback == o.callback && lanes == o.lanes &&
               form == o.form && group == o.group;
    }
};

EngineKey key_of(const psx_search_config& c)
{
    return {c.fft_size, c.mode, c.batch, c.harm_shape,
            c.mode == PSX_MODE_BATCHED && c.use_fft_callback ? 1 : 0, c.lanes, c.fft_form,
            c.group_dms};
}

struct Engine {
    psx_search* s = nullptr;
    EngineKey key{};
    size_t bytes = 0;
};

struct Request {
    long long id = 0;
    double work = 0;  // sum over DM trials of (acceleration trials + 3) * N
    psx_search_config cfg{};
    std::vector<float> bf, bw;
    std::vector<const float*> series;
    size_t nsamps = 0;
    int on_device = 0;
    std::vector<float> dms;
    std::vector<int> dm_idx;
    // results
    std::vector<psx_candidate> out;
    std::vector<int> nassoc, dm_of;
    psx_request_stats st{};
    std::string error;
    bool done = false;
    int passed_over = 0;  // exclusive policy: admissions that went ahead of it
};

}  // namespace

struct psx_server {
    psx_server_config cfg{};
    Clock::time_point t0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<std::shared_ptr<Request>> pending;
    std::map<long long, std::shared_ptr<Request>> requests;
    std::list<Engine> idle;  // pooled instances, least recently used first
    size_t used = 0;         // bytes of every live instance (busy and pooled)
    int active = 0;
    long long next_id = 1;
    bool stop = false;
    std::vector<std::thread> workers;
    // Requests running on the device (by admission order) with their work:
    // the one with the least work runs at the higher stream priority (the
    // older one on a tie), so a short request is not held back by a long
    // one, and the long one shares the GPU only for the short one's work.
    struct Running {
        psx_search* s;
        double work;
    };
    std::map<long long, Running> running;
    long long admit_seq = 0;
    void reprioritise()  // under `mu`
    {
        // every instance at the normal level (one runs at a time when exclusive)
        if (cfg.policy != PSX_SERVE_LEAST_WORK) return;
        auto best = running.end();
        for (auto it = running.begin(); it != running.end(); ++it)
            if (best == running.end() || it->second.work < best->second.work) best = it;
        for (auto it = running.begin(); it != running.end(); ++it)
            psx_search_set_priority(it->second.s, it == best ? 1 : 0);
    }

    double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
    void worker();
    // Under `mu`: decide whether the head of the queue can start.  Returns
    // 1 when it is admitted (popped; *eng is a pooled instance, eng->s set,
    // or a reservation of eng->bytes for a new one), 2 when the head was
    // failed because it can never fit (the queue changed: look again), 0
    // when it has to wait.
    int admit_head(std::shared_ptr<Request>* req, Engine* eng, std::vector<Engine>* evict);
};

int psx_server::admit_head(std::shared_ptr<Request>* req, Engine* eng,
                           std::vector<Engine>* evict)
{
    if (pending.empty() || active >= cfg.max_active) return 0;
    auto pick = pending.begin();
    if (cfg.policy == PSX_SERVE_EXCLUSIVE) {
        if (active > 0) return 0;  // one request on the device at a time
        // the oldest request passed over too often, else the least work
        // (the oldest on a tie)
        auto starved = pending.end();
        for (auto it = pending.begin(); it != pending.end(); ++it) {
            if ((*it)->passed_over >= kMaxPassedOver && starved == pending.end()) starved = it;
            if ((*it)->work < (*pick)->work) pick = it;
        }
        if (starved != pending.end()) pick = starved;
    }
    std::shared_ptr<Request> r = *pick;
    // every pending request ahead of the pick in arrival order was passed
    // over once more (counted when the pick is admitted)
    auto admitted = [&]() {
        for (auto it = pending.begin(); it != pick; ++it) ++(*it)->passed_over;
        pending.erase(pick);
    };
    const EngineKey k = key_of(r->cfg);
    for (auto it = idle.begin(); it != idle.end(); ++it) {
        if (it->key == k) {
            *eng = *it;
            idle.erase(it);
            admitted();
            *req = r;
            ++active;
            return 1;
        }
    }
    const size_t need = psx_search_footprint(&r->cfg);
    // free pooled instances, oldest first, until the new one fits
    while (used + need > cfg.hbm_budget && !idle.empty()) {
        evict->push_back(idle.front());
        used -= idle.front().bytes;
        idle.pop_front();
    }
    if (used + need > cfg.hbm_budget) {
        if (active == 0) {  // can never fit: fail it rather than wait forever
            pending.erase(pick);
            r->st.status = PSX_ERR_ALLOC;
            r->error = "server: request needs " + std::to_string(need) + " bytes, budget is " +
                       std::to_string(cfg.hbm_budget);
            r->st.t_admit = r->st.t_done = now();
            r->done = true;
            cv_done.notify_all();
            return 2;
        }
        return 0;
    }
    used += need;
    eng->s = nullptr;
    eng->key = k;
    eng->bytes = need;
    admitted();
    *req = r;
    ++active;
    return 1;
}

void psx_server::worker()
{
    cudaSetDevice(cfg.device);
    for (;;) {
        std::shared_ptr<Request> r;
        Engine eng;
        std::vector<Engine> evict;
        long long my_seq = 0;
        {
            std::unique_lock<std::mutex> lock(mu);
            for (;;) {
                if (stop && pending.empty()) return;
                const int a = admit_head(&r, &eng, &evict);
                if (a == 1) break;
                if (!evict.empty()) break;  // destroy outside the lock, then retry
                if (a == 2) continue;
                cv_work.wait(lock);
            }
            if (r) {
                r->st.t_admit = now();
                my_seq = ++admit_seq;
            }
        }
        for (Engine& e : evict) psx_search_destroy(e.s);
        evict.clear();
        if (!r) continue;

        int rc = PSX_OK;
        psx::clear_error();
        r->st.footprint = eng.s ? 0 : eng.bytes;
        r->st.engine_reused = eng.s ? 1 : 0;
        if (eng.s) {
            rc = psx_search_retarget(eng.s, &r->cfg);
            if (rc != PSX_OK) {  // cannot happen for equal keys; start afresh
                psx_search_destroy(eng.s);
                eng.s = nullptr;
                rc = PSX_OK;
            }
        }
        if (!eng.s) rc = psx_search_create(&r->cfg, &eng.s);
        if (rc == PSX_OK) {
            std::lock_guard<std::mutex> lock(mu);
            running[my_seq] = Running{eng.s, r->work};
            reprioritise();
        }
        if (rc == PSX_OK) {
            psx_search_info info{};
            size_t cap = (size_t)4096 * r->dms.size(), n = 0;
            for (int attempt = 0; attempt < 2; ++attempt) {
                r->out.resize(cap);
                r->nassoc.resize(cap);
                r->dm_of.resize(cap);
                rc = psx_search_block(eng.s, r->series.data(), r->nsamps, r->on_device,
                                      r->dms.data(), r->dm_idx.data(), (int)r->dms.size(),
                                      PSX_OUT_DM, r->out.data(), r->nassoc.data(), nullptr,
                                      r->dm_of.data(), cap, &n);
                if (rc != PSX_ERR_OVERFLOW) break;
                cap = n;
            }
            if (rc == PSX_OK) {
                r->out.resize(n);
                r->nassoc.resize(n);
                r->dm_of.resize(n);
                if (psx_search_last_info(eng.s, &info) == PSX_OK) r->st.ntrials = info.ntrials;
            }
        }
        if (rc != PSX_OK) r->error = psx_last_error();
        {
            std::lock_guard<std::mutex> lock(mu);
            if (running.erase(my_seq)) reprioritise();
            if (eng.s) psx_search_set_priority(eng.s, 0);  // pooled at the normal level
            if (eng.s) {
                idle.push_back(eng);
            } else {
                used -= eng.bytes;  // the reservation of an instance that failed to build
            }
            --active;
            r->st.status = rc;
            r->st.t_done = now();
            r->done = true;
        }
        cv_done.notify_all();
        cv_work.notify_all();
    }
}

extern "C" {

int psx_server_create(const psx_server_config* cfg, psx_server** out)
{
    psx::clear_error();
    if (!cfg || !out || cfg->max_active < 1 || cfg->max_active > 64 || cfg->max_queue < 1 ||
        cfg->hbm_budget == 0 ||
        (cfg->policy != PSX_SERVE_LEAST_WORK && cfg->policy != PSX_SERVE_EVEN &&
         cfg->policy != PSX_SERVE_EXCLUSIVE)) {
        psx::set_error("server_create: bad configuration (max_active 1..64, max_queue >= 1, "
                       "hbm_budget > 0, policy 0, 1 or 2)");
        return PSX_ERR_INVALID;
    }
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || cfg->device < 0 || cfg->device >= ndev) {
        psx::set_error("server_create: no CUDA device %d", cfg->device);
        return PSX_ERR_CUDA;
    }
    psx_server* s = new (std::nothrow) psx_server;
    if (!s) return PSX_ERR_ALLOC;
    s->cfg = *cfg;
    s->t0 = Clock::now();
    for (int i = 0; i < cfg->max_active; ++i) s->workers.emplace_back([s] { s->worker(); });
    *out = s;
    return PSX_OK;
}

int psx_server_destroy(psx_server* s)
{
    if (!s) return PSX_OK;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        // requests not yet admitted are failed; admitted ones finish
        for (auto& r : s->pending) {
            r->st.status = PSX_ERR_BUSY;
            r->error = "server: shut down before admission";
            r->done = true;
        }
        s->pending.clear();
        s->stop = true;
    }
    s->cv_work.notify_all();
    s->cv_done.notify_all();
    for (auto& t : s->workers) t.join();
    int dev = 0;
    cudaGetDevice(&dev);
    cudaSetDevice(s->cfg.device);
    for (Engine& e : s->idle) psx_search_destroy(e.s);
    cudaSetDevice(dev);
    delete s;
    return PSX_OK;
}

double psx_server_clock(psx_server* s) { return s ? s->now() : 0.0; }

int psx_server_submit(psx_server* s, const psx_search_config* cfg, const float* const* series,
                      size_t nsamps, int series_on_device, const float* dms, const int* dm_idx,
                      int ndm, long long* ticket)
{
    psx::clear_error();
    if (!s || !cfg || !series || !dms || !ticket || ndm <= 0 || nsamps == 0) {
        psx::set_error("server_submit: bad arguments");
        return PSX_ERR_INVALID;
    }
    for (int d = 0; d < ndm; ++d)
        if (!series[d]) {
            psx::set_error("server_submit: null series %d", d);
            return PSX_ERR_INVALID;
        }
    const size_t fp = psx_search_footprint(cfg);
    if (fp == 0) return PSX_ERR_INVALID;  // psx_search_footprint rejected the config
    if (fp > s->cfg.hbm_budget) {
        psx::set_error("server_submit: request needs %zu bytes, budget is %zu", fp,
                       s->cfg.hbm_budget);
        return PSX_ERR_ALLOC;
    }
    auto r = std::make_shared<Request>();
    r->cfg = *cfg;
    if (cfg->nbirdies) {
        r->bf.assign(cfg->birdie_freqs, cfg->birdie_freqs + cfg->nbirdies);
        r->bw.assign(cfg->birdie_widths, cfg->birdie_widths + cfg->nbirdies);
        r->cfg.birdie_freqs = r->bf.data();
        r->cfg.birdie_widths = r->bw.data();
    }
    r->series.assign(series, series + ndm);
    r->nsamps = nsamps;
    r->on_device = series_on_device ? 1 : 0;
    r->dms.assign(dms, dms + ndm);
    r->dm_idx.resize(ndm);
    for (int d = 0; d < ndm; ++d) r->dm_idx[d] = dm_idx ? dm_idx[d] : d;
    r->st.ndm = ndm;
    // work estimate for the scheduling between running requests: every DM
    // trial's acceleration trials plus about three trials' worth of
    // prologue, times the transform length
    for (int d = 0; d < ndm; ++d) {
        size_t nacc = 0;
        if (psx_accel_list(cfg->acc_lo, cfg->acc_hi, cfg->acc_tol, cfg->acc_pulse_width,
                           cfg->fft_size, cfg->tsamp, cfg->cfreq_hz, cfg->ch_bw_hz, dms[d],
                           cfg->cdm, nullptr, 0, &nacc) != PSX_OK)
            nacc = 1;
        r->work += (double)(nacc + 3) * (double)cfg->fft_size;
    }
    psx::clear_error();
    {
        std::lock_guard<std::mutex> lock(s->mu);
        if (s->stop) {
            psx::set_error("server_submit: server is shutting down");
            return PSX_ERR_BUSY;
        }
        if ((int)s->pending.size() >= s->cfg.max_queue) {
            psx::set_error("server_submit: queue full (%d pending)", (int)s->pending.size());
            return PSX_ERR_BUSY;
        }
        r->id = s->next_id++;
        r->st.t_submit = s->now();
        r->st.status = -1;
        s->pending.push_back(r);
        s->requests[r->id] = r;
        *ticket = r->id;
    }
    s->cv_work.notify_one();
    return PSX_OK;
}

int psx_server_wait(psx_server* s, long long ticket, double timeout_s, psx_candidate* h_out,
                    int* h_nassoc, int* h_dm, size_t cap, size_t* n_out, psx_request_stats* stats)
{
    psx::clear_error();
    if (!s || !n_out) {
        psx::set_error("server_wait: bad arguments");
        return PSX_ERR_INVALID;
    }
    *n_out = 0;
    std::shared_ptr<Request> r;
    {
        std::unique_lock<std::mutex> lock(s->mu);
        auto it = s->requests.find(ticket);
        if (it == s->requests.end()) {
            psx::set_error("server_wait: unknown ticket %lld", ticket);
            return PSX_ERR_INVALID;
        }
        r = it->second;
        auto ready = [&] { return r->done; };
        if (timeout_s < 0) {
            s->cv_done.wait(lock, ready);
        } else if (!s->cv_done.wait_for(lock, std::chrono::duration<double>(timeout_s), ready)) {
            psx::set_error("server_wait: request %lld still running", ticket);
            return PSX_ERR_BUSY;
        }
        if (stats) *stats = r->st;
        if (r->st.status != PSX_OK) {
            psx::set_error("%s", r->error.c_str());
            s->requests.erase(it);
            return r->st.status;
        }
        *n_out = r->out.size();
        if (r->out.size() > cap || (!h_out && !r->out.empty())) {
            psx::set_error("server_wait: %zu candidates, buffer holds %zu", r->out.size(), cap);
            return PSX_ERR_OVERFLOW;  // the request stays; call again with room
        }
        s->requests.erase(it);
    }
    if (!r->out.empty()) {
        std::memcpy(h_out, r->out.data(), sizeof(psx_candidate) * r->out.size());
        if (h_nassoc) std::memcpy(h_nassoc, r->nassoc.data(), sizeof(int) * r->out.size());
        if (h_dm) std::memcpy(h_dm, r->dm_of.data(), sizeof(int) * r->out.size());
    }
    return PSX_OK;
}

int psx_server_status(psx_server* s, size_t* used_bytes, int* active, int* pending, int* pooled)
{
    if (!s) return PSX_ERR_INVALID;
    std::lock_guard<std::mutex> lock(s->mu);
    if (used_bytes) *used_bytes = s->used;
    if (active) *active = s->active;
    if (pending) *pending = (int)s->pending.size();
    if (pooled) *pooled = (int)s->idle.size();
    return PSX_OK;
}

}  // extern "C"
