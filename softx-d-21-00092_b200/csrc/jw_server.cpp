// jw_server.cpp -- continuous-batching evolution server over the batched engine.
//
// A request is one event: MV initial condition (main_optimized.cpp:178-191),
// `steps` Langevin steps (:243-304) and a final dipole measurement
// (:321-334) returned as the angle-averaged S(r) and Q_s.  A worker thread
// owns the device:
//   admit   first fit over the queue by device footprint (the engine's budget);
//           requests that do not fit wait, later smaller ones may pass them;
//   tick    the chosen resident events advance together, one launch group
//           per lattice size, by k = min(max_steps_per_tick, fewest remaining
//           steps in the group) steps.  Chosen are all of them, or with
//           options.tick_sites the ones with the least remaining work first
//           (shortest remaining work, as many as fit in tick_sites lattice
//           sites, at least one); an event's MV initial condition runs when it
//           is first chosen;
//   retire  finished events are measured, their S(r) copied out and their
//           device memory released, which lets queued requests in.
// Requests that arrive while others are on the GPU join at the next tick.
// Each event's result is independent of what else is resident: the noise is a
// function of (seed, step, site) and every kernel treats events separately.
//
// The scheduler talks to a Backend: the engine, or (options.fake_device) a
// host-only stand-in with the same admission arithmetic and a fixed cost per
// site-step, so the scheduling and failure paths run without a GPU.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/jimwlk.h"

#define JW_EXPORT extern "C" __attribute__((visibility("default")))

namespace {

using Clock = std::chrono::steady_clock;

struct Backend {
    virtual ~Backend() {}
    virtual jw_status add(const jw_event_desc& d, int* id) = 0;
    virtual jw_status init_mv(const std::vector<int>& ids) = 0;
    virtual jw_status step(const std::vector<int>& ids, int k) = 0;
    virtual jw_status sync() = 0;
    // measure, then S(r) bins and Q_s
    virtual jw_status finish(int id, std::vector<double>& sb, std::vector<double>& rb, double* qs) = 0;
    virtual jw_status remove(int id) = 0;
    // the stream the backend's device work runs on (null: no device)
    virtual cudaStream_t stream() { return nullptr; }
};

struct EngineBackend : Backend {
    jw_engine* e = nullptr;
    std::map<int, int> n_of;
    ~EngineBackend() override {
        if (e) jw_engine_destroy(e);
    }
    jw_status add(const jw_event_desc& d, int* id) override {
        jw_status s = jw_engine_add_event(e, &d, id);
        if (!s) n_of[*id] = d.N;
        return s;
    }
    jw_status init_mv(const std::vector<int>& ids) override {
        return jw_engine_init_mv(e, ids.data(), (int)ids.size());
    }
    jw_status step(const std::vector<int>& ids, int k) override {
        return jw_engine_step(e, ids.data(), (int)ids.size(), k);
    }
    jw_status sync() override { return jw_engine_sync(e); }
    jw_status finish(int id, std::vector<double>& sb, std::vector<double>& rb, double* qs) override {
        jw_status s = jw_engine_measure(e, &id, 1);
        if (s) return s;
        const int nb = n_of[id] / 2 + 1;
        sb.assign(nb, 0.0);
        rb.assign(nb, 0.0);
        int n = 0;
        return jw_engine_dipole(e, id, nullptr, sb.data(), rb.data(), nullptr, nb, &n, qs);
    }
    jw_status remove(int id) override {
        n_of.erase(id);
        return jw_engine_remove_event(e, id);
    }
    cudaStream_t stream() override { return static_cast<cudaStream_t>(jw_engine_stream(e)); }
};

// Host-only stand-in: the engine's per-event footprint formula and budget,
// a fixed nanosecond cost per site-step, S(r) = exp(-r^2 / r0^2) with r0 set
// by the request so results are checkable.
struct FakeBackend : Backend {
    size_t budget = 0, used = 0;
    double ns_per_site_step = 0.05;
    int next = 1;
    struct Ev { jw_event_desc d; size_t bytes; long steps = 0; bool mv = false; };
    std::map<int, Ev> ev;
    static size_t bytes_of(const jw_event_desc& d) { return (size_t)d.N * d.N * (144 + 32 + 192); }
    jw_status add(const jw_event_desc& d, int* id) override {
        if (d.N < 8 || d.N > 2048 || (d.N & (d.N - 1))) return JW_EUNSUPPORTED;
        const size_t b = bytes_of(d);
        if (used + b > budget) return JW_ENOMEM;
        used += b;
        *id = next++;
        ev[*id] = Ev{d, b};
        return JW_OK;
    }
    jw_status init_mv(const std::vector<int>& ids) override {
        for (int i : ids) ev[i].mv = true;
        return JW_OK;
    }
    jw_status step(const std::vector<int>& ids, int k) override {
        double sites = 0;
        for (int i : ids) {
            ev[i].steps += k;
            sites += (double)ev[i].d.N * ev[i].d.N;
        }
        std::this_thread::sleep_for(std::chrono::nanoseconds((long)(sites * k * ns_per_site_step)));
        return JW_OK;
    }
    jw_status sync() override { return JW_OK; }
    jw_status finish(int id, std::vector<double>& sb, std::vector<double>& rb, double* qs) override {
        const Ev& v = ev[id];
        const int nb = v.d.N / 2 + 1;
        const double r0 = 1.0 + 0.01 * (double)v.steps + (double)(v.d.seed % 7);
        sb.resize(nb);
        rb.resize(nb);
        for (int b = 0; b < nb; ++b) {
            rb[b] = b;
            sb[b] = std::exp(-(double)b * b / (r0 * r0));
        }
        *qs = std::sqrt(2.0) / (r0 * std::sqrt(0.5));
        return v.mv ? JW_OK : JW_EINVAL;
    }
    jw_status remove(int id) override {
        used -= ev[id].bytes;
        ev.erase(id);
        return JW_OK;
    }
};

struct Request {
    jw_request_desc d{};
    int status = JW_OK;
    bool done = false;
    int eid = -1;
    long remaining = 0;
    bool mv = false;  // MV initial condition done
    double t_submit = 0, t_admit = 0, t_done = 0;
    std::vector<double> sb, rb;
    double qs = 0;
};

}  // namespace

struct jw_server {
    jw_server_options opt{};
    int device = 0;
    std::unique_ptr<Backend> be;
    std::thread worker;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<int64_t> queue;
    std::unordered_map<int64_t, Request> reqs;
    std::vector<Request*> active;  // worker only; nodes of reqs, whose addresses are stable
    bool stop = false;
    int64_t next_id = 1;
    Clock::time_point t0 = Clock::now();
    // statistics (under mu)
    int64_t submitted = 0, completed = 0, failed = 0;
    double site_steps = 0;
    int max_active_seen = 0;
    double t_admit = 0, t_mv = 0, t_step = 0, t_retire = 0;  // worker phases (under mu)
    // per lattice size (under mu): site-steps, device ms of steps and MV, ticks
    struct SizeStats { double site_steps = 0, step_ms = 0, mv_ms = 0; int64_t ticks = 0; };
    std::map<int, SizeStats> by_size;
    double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
};

namespace {

// CUDA events bracketing one size's launches within a tick (engine backend).
struct SizeTimer {
    int N = 0;
    cudaEvent_t a = nullptr, b = nullptr;
};

void timer_begin(cudaStream_t st, std::vector<SizeTimer>& v, int N) {
    if (!st) return;
    SizeTimer t;
    t.N = N;
    if (cudaEventCreate(&t.a) != cudaSuccess) return;
    if (cudaEventCreate(&t.b) != cudaSuccess) {
        cudaEventDestroy(t.a);
        return;
    }
    cudaEventRecord(t.a, st);
    v.push_back(t);
}

void timer_end(cudaStream_t st, std::vector<SizeTimer>& v) {
    if (st && !v.empty()) cudaEventRecord(v.back().b, st);
}

// After the stream has synchronised: the milliseconds of each bracket.
void timers_collect(std::vector<SizeTimer>& v, std::map<int, double>& ms) {
    for (SizeTimer& t : v) {
        float x = 0.0f;
        if (cudaEventElapsedTime(&x, t.a, t.b) == cudaSuccess) ms[t.N] += x;
        cudaEventDestroy(t.a);
        cudaEventDestroy(t.b);
    }
    v.clear();
}

}  // namespace

namespace {

// The last touch of a request by the worker: after this, jw_server_wait may
// erase it.
void retire(jw_server* s, Request* rp, int status) {
    std::lock_guard<std::mutex> lk(s->mu);
    Request& r = *rp;
    r.status = status;
    r.done = true;
    r.t_done = s->now();
    if (status == JW_OK) ++s->completed;
    else ++s->failed;
    s->cv_done.notify_all();
}

void worker_loop(jw_server* s) {
    const int K = std::max(1, s->opt.max_steps_per_tick);
    for (;;) {
        std::vector<Request*> admitted;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            if (s->stop) break;
            if (s->active.empty() && s->queue.empty()) {
                s->cv_work.wait_for(lk, std::chrono::milliseconds(20));
                continue;
            }
            // first fit over the queue
            const double ta = s->now();
            for (auto it = s->queue.begin(); it != s->queue.end();) {
                if (s->opt.max_active > 0 && (int)(s->active.size() + admitted.size()) >= s->opt.max_active) break;
                Request* r = &s->reqs[*it];
                jw_event_desc d{};
                d.N = r->d.N;
                d.ny_slices = r->d.ny_slices;
                d.mu = r->d.mu;
                d.mass = r->d.mass;
                d.step = r->d.step;
                d.coupling = r->d.coupling;
                d.kernel = r->d.kernel;
                d.seed = r->d.seed;
                int eid = -1;
                const jw_status st = s->be->add(d, &eid);
                if (st == JW_OK) {
                    r->eid = eid;
                    r->remaining = r->d.steps;
                    r->t_admit = s->now();
                    admitted.push_back(r);
                    it = s->queue.erase(it);
                } else if (st == JW_ENOMEM) {
                    ++it;  // waits for memory; smaller requests behind it may pass
                } else {
                    r->status = st;
                    r->done = true;
                    r->t_done = s->now();
                    ++s->failed;
                    s->cv_done.notify_all();
                    it = s->queue.erase(it);
                }
            }
            s->max_active_seen = std::max(s->max_active_seen, (int)(s->active.size() + admitted.size()));
            s->t_admit += s->now() - ta;
        }
        // device work runs outside the lock: only this thread uses the backend
        for (Request* r : admitted) s->active.push_back(r);
        if (s->active.empty()) continue;
        // choose this tick's events
        std::vector<Request*> sel;
        if (s->opt.tick_sites == 0) {
            sel = s->active;
        } else {
            auto work = [](const Request* r) {
                return (double)r->d.N * r->d.N * (double)(r->remaining + (r->mv ? 0 : r->d.ny_slices));
            };
            std::vector<Request*> order = s->active;
            std::stable_sort(order.begin(), order.end(),
                             [&](const Request* a, const Request* b) { return work(a) < work(b); });
            double sites = 0;
            for (Request* r : order) {
                const double n2 = (double)r->d.N * r->d.N;
                if (!sel.empty() && sites + n2 > (double)s->opt.tick_sites) continue;
                sel.push_back(r);
                sites += n2;
            }
        }
        // MV initial conditions of the chosen events that have none yet
        {
            std::vector<int> eids;
            std::vector<Request*> fresh;
            for (Request* r : sel)
                if (!r->mv) {
                    eids.push_back(r->eid);
                    fresh.push_back(r);
                }
            if (!eids.empty()) {
                const double tm = s->now();
                // one call per lattice size, each timed on the device
                std::map<int, std::vector<int>> mv_by_n;
                for (Request* r : fresh) mv_by_n[r->d.N].push_back(r->eid);
                std::vector<SizeTimer> timers;
                jw_status st = JW_OK;
                for (auto& kv : mv_by_n) {
                    timer_begin(s->be->stream(), timers, kv.first);
                    const jw_status sn = s->be->init_mv(kv.second);
                    timer_end(s->be->stream(), timers);
                    if (sn && !st) st = sn;
                }
                const jw_status sy = s->be->sync();
                std::map<int, double> ms;
                timers_collect(timers, ms);
                {
                    std::lock_guard<std::mutex> lk(s->mu);
                    s->t_mv += s->now() - tm;
                    for (auto& kv : ms) s->by_size[kv.first].mv_ms += kv.second;
                }
                for (Request* r : fresh) r->mv = (st == JW_OK && sy == JW_OK);
                if (st || sy) {
                    std::vector<Request*> keep;
                    for (Request* r : s->active) {
                        if (std::find(fresh.begin(), fresh.end(), r) != fresh.end()) {
                            s->be->remove(r->eid);
                            retire(s, r, st ? st : sy);
                        } else {
                            keep.push_back(r);
                        }
                    }
                    s->active.swap(keep);
                    continue;
                }
            }
        }
        // tick: one launch group per lattice size
        const double tt = s->now();
        std::map<int, std::vector<Request*>> by_n;
        for (Request* r : sel) by_n[r->d.N].push_back(r);
        double ss = 0;
        jw_status tick_status = JW_OK;
        std::vector<SizeTimer> timers;
        std::map<int, double> ss_by_n;
        for (auto& kv : by_n) {
            long k = K;
            for (Request* r : kv.second) k = std::min(k, r->remaining);
            if (k <= 0) continue;
            std::vector<int> eids;
            for (Request* r : kv.second) eids.push_back(r->eid);
            timer_begin(s->be->stream(), timers, kv.first);
            const jw_status st = s->be->step(eids, (int)k);
            timer_end(s->be->stream(), timers);
            if (st && !tick_status) tick_status = st;
            for (Request* r : kv.second) r->remaining -= k;
            const double n_ss = (double)kv.first * kv.first * (double)k * kv.second.size();
            ss += n_ss;
            ss_by_n[kv.first] += n_ss;
        }
        const jw_status sst = s->be->sync();
        if (!tick_status) tick_status = sst;
        const double tr = s->now();
        std::map<int, double> ms;
        timers_collect(timers, ms);
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->site_steps += ss;
            s->t_step += tr - tt;
            for (auto& kv : ss_by_n) {
                jw_server::SizeStats& z = s->by_size[kv.first];
                z.site_steps += kv.second;
                z.ticks += 1;
            }
            for (auto& kv : ms) s->by_size[kv.first].step_ms += kv.second;
        }
        // retire finished events (all of this tick's events if the tick failed)
        std::vector<Request*> keep;
        for (Request* r : s->active) {
            if (tick_status != JW_OK) {
                s->be->remove(r->eid);
                retire(s, r, tick_status);
            } else if (r->remaining <= 0 && r->mv) {
                std::vector<double> sb, rb;
                double qs = 0;
                const jw_status st = s->be->finish(r->eid, sb, rb, &qs);
                s->be->remove(r->eid);
                {
                    std::lock_guard<std::mutex> lk(s->mu);
                    r->sb.swap(sb);
                    r->rb.swap(rb);
                    r->qs = qs;
                }
                retire(s, r, st);
            } else {
                keep.push_back(r);
            }
        }
        s->active.swap(keep);
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->t_retire += s->now() - tr;
        }
    }
}

}  // namespace

JW_EXPORT jw_status jw_server_create(const jw_server_options* opt, int device, jw_server** out) {
    if (!opt || !out) return JW_EINVAL;
    *out = nullptr;
    auto* s = new jw_server();
    s->opt = *opt;
    s->device = device;
    if (opt->fake_device) {
        auto fb = std::make_unique<FakeBackend>();
        fb->budget = opt->max_bytes ? opt->max_bytes : ((size_t)1 << 30);
        if (opt->fake_ns_per_site_step > 0) fb->ns_per_site_step = opt->fake_ns_per_site_step;
        s->be = std::move(fb);
    } else {
        auto eb = std::make_unique<EngineBackend>();
        // launch groups (and their workspaces) no larger than a tick; column
        // tiles autotuned per lattice size
        jw_engine_options eo{opt->precision, opt->reunitarize, opt->max_bytes, 0, opt->tick_sites, 1};
        const jw_status st = jw_engine_create(&eo, device, &eb->e);
        if (st) {
            delete s;
            return st;
        }
        s->be = std::move(eb);
    }
    s->worker = std::thread([s]() {
        if (!s->opt.fake_device) cudaSetDevice(s->device);
        worker_loop(s);
    });
    *out = s;
    return JW_OK;
}

JW_EXPORT jw_status jw_server_destroy(jw_server* s) {
    if (!s) return JW_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->cv_work.notify_all();
    }
    if (s->worker.joinable()) s->worker.join();
    delete s;  // releases the backend (engine and its device memory)
    return JW_OK;
}

JW_EXPORT jw_status jw_server_submit(jw_server* s, const jw_request_desc* d, int64_t* rid) {
    if (!s || !d || !rid) return JW_EINVAL;
    *rid = -1;
    if (d->N < 8 || d->N > 2048 || (d->N & (d->N - 1))) return JW_EUNSUPPORTED;
    if (d->kernel != JW_SIN_KERNEL) return JW_EUNSUPPORTED;
    if (d->coupling != JW_SQRT_COUPLING_CONSTANT && d->coupling != JW_NOISE_COUPLING_CONSTANT &&
        d->coupling != JW_FIXED_COUPLING_CONSTANT)
        return JW_EUNSUPPORTED;
    if (d->steps < 0 || d->ny_slices < 0 || !(d->step >= 0.0) || !std::isfinite(d->mu) || !std::isfinite(d->mass))
        return JW_EINVAL;
    const size_t need = (size_t)d->N * d->N * (144 + 32 + 192);
    if (s->opt.max_bytes && need > s->opt.max_bytes) return JW_ENOMEM;  // could never be admitted
    std::lock_guard<std::mutex> lk(s->mu);
    const int64_t id = s->next_id++;
    Request& r = s->reqs[id];
    r.d = *d;
    r.t_submit = s->now();
    s->queue.push_back(id);
    ++s->submitted;
    s->cv_work.notify_all();
    *rid = id;
    return JW_OK;
}

JW_EXPORT jw_status jw_server_wait(jw_server* s, int64_t rid, double timeout_s, jw_request_result* res,
                                   double* S_bins, double* r_bins, int nbins_cap) {
    if (!s || !res) return JW_EINVAL;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(rid);
    if (it == s->reqs.end()) return JW_ENOTFOUND;
    const auto deadline = Clock::now() + std::chrono::duration_cast<Clock::duration>(
                                             std::chrono::duration<double>(timeout_s < 0 ? 0 : timeout_s));
    while (!s->reqs[rid].done) {
        if (s->cv_done.wait_until(lk, deadline) == std::cv_status::timeout && !s->reqs[rid].done) return JW_ETIMEOUT;
    }
    Request& r = s->reqs[rid];
    res->status = r.status;
    res->N = r.d.N;
    res->steps = r.d.steps;
    res->t_submit = r.t_submit;
    res->t_admit = r.t_admit;
    res->t_done = r.t_done;
    res->Qs = r.qs;
    res->nbins = (int)r.sb.size();
    if (S_bins && nbins_cap >= (int)r.sb.size()) {
        std::memcpy(S_bins, r.sb.data(), sizeof(double) * r.sb.size());
        if (r_bins) std::memcpy(r_bins, r.rb.data(), sizeof(double) * r.rb.size());
    }
    s->reqs.erase(rid);
    return JW_OK;
}

JW_EXPORT jw_status jw_server_size_stats(jw_server* s, int* N, double* site_steps, double* step_ms, double* mv_ms,
                                         int64_t* ticks, int cap, int* count) {
    if (!s || !count || cap < 0) return JW_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    int i = 0;
    for (auto& kv : s->by_size) {
        if (i < cap) {
            if (N) N[i] = kv.first;
            if (site_steps) site_steps[i] = kv.second.site_steps;
            if (step_ms) step_ms[i] = kv.second.step_ms;
            if (mv_ms) mv_ms[i] = kv.second.mv_ms;
            if (ticks) ticks[i] = kv.second.ticks;
        }
        ++i;
    }
    *count = i;
    return JW_OK;
}

JW_EXPORT jw_status jw_server_get_stats(jw_server* s, jw_server_stats* st) {
    if (!s || !st) return JW_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    st->submitted = s->submitted;
    st->completed = s->completed;
    st->failed = s->failed;
    st->queued = (int64_t)s->queue.size();
    st->site_steps = s->site_steps;
    st->max_active = s->max_active_seen;
    st->now = s->now();
    st->t_admit = s->t_admit;
    st->t_mv = s->t_mv;
    st->t_step = s->t_step;
    st->t_retire = s->t_retire;
    return JW_OK;
}
