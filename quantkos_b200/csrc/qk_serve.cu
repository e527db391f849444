// Continuous-batching request loop.
//
// Requests are queued by qk_serve_submit (any thread).  Lanes — host threads, each
// with its own handle, CUDA stream and grow-only device arenas on the same device —
// take the requests that have arrived, in arrival order, as one wave: a wave is
// closed when its estimated GPU time reaches the larger of the wave budget (a few
// milliseconds) and the lane's share of the backlog, when it reaches max_batch
// requests, or when the HBM its requests need (LSM slabs and tile records) would
// exceed what the budget has free.  Short queues thus give short waves (latency),
// long queues long ones (throughput).  A wave is planned,
// uploaded (each request's descriptors are copied to the device once, when its wave
// starts) and priced as one persistent launch per kernel kind plus the LSM jobs of
// its American contracts.  With several lanes, several waves are on the GPU at once:
// a request that arrives while others are being priced is admitted into the next
// wave as soon as a lane is free, its kernels overlap the waves already running, and
// memory returns to the budget as each wave completes.  A request larger than the
// whole budget is rejected (QK_ERR_CAPACITY).  The reference has no serving layer
// (one contract per process run, include/core/engine/Distpatcher.hpp:78-83).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "qk_engine.h"
#include "qk_host.h"
#include "qk_kernels.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    int64_t ticket;
    qk_contract c;
    qk_greeks g;
    size_t bytes;
    double est_us;
    Clock::time_point t_submit;
};

struct Finished {
    qk_result r;
    qk_status status;
    double latency_ms;
};

bool is_american(const qk_contract &c) {
    for (int k = 0; k < c.n_payoffs; ++k)
        if (c.payoffs[k].type == QK_AMERICAN) return true;
    return false;
}

// HBM a request holds while it is being priced: LSM slabs and cash flows for
// American contracts, per-tile moment records and descriptors otherwise.
size_t footprint(const qk_contract &c, const qk_greeks &g) {
    const size_t roles = qk::roles_for(g.mask ? &g : nullptr, c.T).size();
    const size_t esz = c.precision == QK_FP32 ? 4 : 8;
    size_t bytes = roles * (sizeof(qk::TaskDev) + 64);
    if (is_american(c)) {
        const size_t D = c.lsm_dates > 0 ? c.lsm_dates : c.n_steps;
        const size_t ld = (static_cast<size_t>(c.n_paths) + 3) / 4 * 4;
        const size_t slabs = c.lsm_basis == QK_LSM_POLY_SV ? 2 : 1;
        // the bumps of one request run on up to kLsmLanes streams at once, each with its own slabs
        const size_t concurrent = std::min<size_t>(roles, qk::kLsmLanes);
        bytes += concurrent * (D * ld * esz * slabs + ld * esz);
    } else {
        const size_t tiles = (static_cast<size_t>(c.n_paths) + qk::kWarpTilePaths - 1) / qk::kWarpTilePaths;
        bytes += roles * tiles * c.n_payoffs * sizeof(qk::Moments);
    }
    return bytes;
}

// Estimated GPU time of a request in microseconds: path-steps of all its pricing tasks
// at the measured rate of the FP32 Heston-Euler kernel (5.4e11 path-steps/s), weighted
// by the kind's relative cost (QE, jumps, FP64), plus for an American contract its
// backward sweep (16 bytes per path and date at 3e12 B/s, and a fixed 10 us per date).
double estimate_us(const qk_contract &c, const qk_greeks &g) {
    const double roles = static_cast<double>(qk::roles_for(g.mask ? &g : nullptr, c.T).size());
    double f = 1.0;
    if (c.scheme == QK_ANDERSEN_QE) f *= 1.7;
    if (c.scheme == QK_IMPLICIT_MILSTEIN) f *= 1.06;
    if (c.model == QK_BATES) f *= 1.2;
    if (c.precision == QK_FP64) f *= 6.0;
    double us = roles * static_cast<double>(c.n_paths) * c.n_steps * f / 5.4e5;
    if (is_american(c)) {
        const double D = c.lsm_dates > 0 ? c.lsm_dates : c.n_steps;
        us += roles * (16.0 * static_cast<double>(c.n_paths) * D / 3e6 + 10.0 * D);
    }
    return us;
}

}  // namespace

struct qk_server {
    int device = 0;
    size_t budget = 0, in_use = 0;
    int max_batch = 256;
    double wave_us = 2500.0;  // GPU-time budget of one wave (the least a wave is allowed to hold)
    double queued_us = 0.0;   // estimated GPU time of the requests waiting for admission
    int n_lanes = 1;
    size_t reserved = 0;  // bytes held in the device pool for the lanes (pool_reserve)
    bool plain = false;   // one request per wave, priced by the plain FP64 method
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request> queue;
    std::unordered_map<int64_t, Finished> done;
    int64_t next_ticket = 1;
    bool stop = false;
    std::vector<std::thread> lanes;
    std::vector<qk_handle *> handles;
    // statistics; the per-request records are a window over the most recent
    // kRecordWindow completed requests (a ring once full: rec_head is its oldest)
    static constexpr size_t kRecordWindow = size_t(1) << 20;
    std::vector<qk_serve_record> records;
    size_t rec_head = 0;
    int64_t next_wave = 0;
    int64_t submitted = 0, completed = 0, rejected = 0, batches = 0;
    double path_steps = 0.0, busy_s = 0.0;
    bool have_first = false;
    Clock::time_point t_first, t_last;
};

static void lane_loop(qk_server *s, qk_handle *h, int lane) {
    std::vector<Request> batch;
    std::vector<qk_contract> cs;
    std::vector<qk_greeks> gs;
    std::vector<qk_result> rs;
    for (;;) {
        batch.clear();
        size_t bytes = 0;
        double est = 0.0;
        int64_t wave = 0;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            for (;;) {
                if (s->stop && s->queue.empty()) return;
                // wave size: the budget, or this lane's share of the backlog when that is larger
                // (small waves while the queue is short, large ones under load)
                const double cap = std::max(s->wave_us, s->queued_us / s->n_lanes);
                est = 0.0;
                const int wave_max = s->plain ? 1 : s->max_batch;
                while (!s->queue.empty() && static_cast<int>(batch.size()) < wave_max &&
                       s->in_use + bytes + s->queue.front().bytes <= s->budget &&
                       (batch.empty() || est + s->queue.front().est_us <= cap)) {
                    bytes += s->queue.front().bytes;
                    est += s->queue.front().est_us;
                    s->queued_us -= s->queue.front().est_us;
                    batch.push_back(s->queue.front());
                    s->queue.pop_front();
                }
                if (s->queue.empty()) s->queued_us = 0.0;  // no drift from rounding
                if (!batch.empty()) break;
                s->cv_work.wait_for(lk, std::chrono::milliseconds(50));
            }
            s->in_use += bytes;
            wave = s->next_wave++;
        }
        cs.resize(batch.size());
        gs.resize(batch.size());
        rs.resize(batch.size());
        for (size_t i = 0; i < batch.size(); ++i) {
            cs[i] = batch[i].c;
            gs[i] = batch[i].g;
        }
        const auto t0 = Clock::now();
        const qk_status st =
            qk::price_contracts(h, cs.data(), static_cast<int32_t>(cs.size()), gs.data(), rs.data(), s->plain);
        const auto t1 = Clock::now();
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->in_use -= bytes;
            s->batches++;
            s->busy_s += std::chrono::duration<double>(t1 - t0).count();
            for (size_t i = 0; i < batch.size(); ++i) {
                Finished f;
                f.status = st;
                f.r = rs[i];
                if (st != QK_OK) f.r.status = st;
                f.latency_ms = std::chrono::duration<double, std::milli>(t1 - batch[i].t_submit).count();
                qk_serve_record rec;
                rec.ticket = batch[i].ticket;
                rec.wave = wave;
                rec.lane = lane;
                rec.wave_requests = static_cast<int32_t>(batch.size());
                rec.submit_s = std::chrono::duration<double>(batch[i].t_submit - s->t_first).count();
                rec.admit_ms = std::chrono::duration<double, std::milli>(t0 - batch[i].t_submit).count();
                rec.latency_ms = f.latency_ms;
                rec.wave_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
                rec.wave_est_ms = est * 1e-3;
                rec.est_ms = batch[i].est_us * 1e-3;
                if (s->records.size() < qk_server::kRecordWindow) {
                    s->records.push_back(rec);
                } else {
                    s->records[s->rec_head] = rec;
                    s->rec_head = (s->rec_head + 1) % qk_server::kRecordWindow;
                }
                s->completed++;
                if (st == QK_OK) s->path_steps += rs[i].path_steps;
                s->done[batch[i].ticket] = f;
            }
            s->t_last = t1;
        }
        s->cv_done.notify_all();
        s->cv_work.notify_all();
    }
}

extern "C" {

qk_status qk_serve_start(qk_handle *h, int64_t hbm_budget_mib, int32_t max_batch, qk_server **out) {
    qk_serve_options o;
    std::memset(&o, 0, sizeof(o));
    o.hbm_budget_mib = hbm_budget_mib;
    o.max_batch = max_batch;
    return qk_serve_start_ex(h, &o, out);
}

qk_status qk_serve_start_ex(qk_handle *h, const qk_serve_options *opt, qk_server **out) {
    if (!h || !opt || !out) return qk::fail(QK_ERR_INVALID_ARG, "NULL argument");
    *out = nullptr;
    if (opt->lanes < 0 || opt->lanes > 16) return qk::fail(QK_ERR_INVALID_ARG, "lanes must be in [0, 16] (0 = 4)");
    if (opt->wave_ms < 0.0) return qk::fail(QK_ERR_INVALID_ARG, "wave_ms must be >= 0 (0 = 2.5 ms)");
    if (opt->reserve_mib < -1) return qk::fail(QK_ERR_INVALID_ARG, "reserve_mib must be >= -1 (0 = the budget, -1 = none)");
    const int64_t hbm_budget_mib = opt->hbm_budget_mib;
    const int32_t max_batch = opt->max_batch;
    if (cudaSetDevice(h->device) != cudaSuccess) return qk::fail(QK_ERR_CUDA, "cudaSetDevice failed");
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return qk::fail(QK_ERR_CUDA, "cudaMemGetInfo failed");
    qk_server *s = new qk_server();
    s->device = h->device;
    s->budget = hbm_budget_mib > 0 ? static_cast<size_t>(hbm_budget_mib) << 20 : static_cast<size_t>(free_b * 0.8);
    s->max_batch = max_batch > 0 ? max_batch : 256;
    s->wave_us = opt->wave_ms > 0.0 ? opt->wave_ms * 1e3 : 2500.0;
    s->plain = opt->plain_fp64 != 0;
    const int lanes = opt->lanes > 0 ? opt->lanes : 4;
    s->n_lanes = lanes;
    const size_t reserve = opt->reserve_mib > 0 ? static_cast<size_t>(opt->reserve_mib) << 20
                           : opt->reserve_mib == 0 ? s->budget : 0;
    if (reserve > 0) {
        const qk_status st = qk::pool_reserve(h->device, h->stream, reserve);
        if (st == QK_OK) {
            s->reserved = reserve;
        } else if (opt->reserve_mib > 0) {
            delete s;
            return st;
        } else {
            qk::g_last_error.clear();  // a default reservation that does not fit is skipped, not an error
        }
    }
    for (int i = 0; i < lanes; ++i) {
        qk_handle *lh = nullptr;
        const qk_status st = qk_create(h->device, &lh);
        if (st != QK_OK) {
            for (qk_handle *x : s->handles) qk_destroy(x);
            qk::pool_release(s->device, s->reserved);
            delete s;
            return st;
        }
        // the lanes price with the caller's launch shapes (defaults, or those set by
        // qk_autotune / qk_tune_set on h before the start)
        lh->tune_tpw = h->tune_tpw;
        lh->tune_tail = h->tune_tail;
        lh->tune_lanes = h->tune_lanes;
        lh->tune_block = h->tune_block;
        s->handles.push_back(lh);
    }
    for (size_t i = 0; i < s->handles.size(); ++i) s->lanes.emplace_back(lane_loop, s, s->handles[i], static_cast<int>(i));
    *out = s;
    return QK_OK;
}

qk_status qk_serve_submit(qk_server *s, const qk_contract *c, const qk_greeks *g, int64_t *ticket) {
    if (!s || !c || !ticket) return qk::fail(QK_ERR_INVALID_ARG, "NULL argument");
    const qk_status v = qk::validate_contract(*c, g);
    if (v != QK_OK) return v;
    Request r;
    r.c = *c;
    if (g) r.g = *g;
    else std::memset(&r.g, 0, sizeof(r.g));
    r.bytes = footprint(r.c, r.g);
    r.est_us = estimate_us(r.c, r.g);
    r.t_submit = Clock::now();
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return qk::fail(QK_ERR_STATE, "server stopped");
    if (!s->have_first) {
        s->have_first = true;
        s->t_first = r.t_submit;
    }
    s->submitted++;
    if (r.bytes > s->budget) {
        s->rejected++;
        return qk::fail(QK_ERR_CAPACITY, "request needs more HBM than the admission budget");
    }
    r.ticket = s->next_ticket++;
    *ticket = r.ticket;
    s->queued_us += r.est_us;
    s->queue.push_back(r);
    s->cv_work.notify_one();
    return QK_OK;
}

qk_status qk_serve_poll(qk_server *s, int64_t ticket, int32_t wait_ms, int32_t *done, qk_result *out) {
    if (!s || !done) return qk::fail(QK_ERR_INVALID_ARG, "NULL argument");
    *done = 0;
    std::unique_lock<std::mutex> lk(s->mu);
    if (ticket <= 0 || ticket >= s->next_ticket) return qk::fail(QK_ERR_STATE, "unknown ticket");
    auto ready = [&] { return s->done.count(ticket) > 0; };
    if (!ready() && wait_ms > 0) s->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), ready);
    auto it = s->done.find(ticket);
    if (it == s->done.end()) return QK_OK;
    *done = 1;
    if (out) *out = it->second.r;
    const qk_status st = it->second.status;
    s->done.erase(it);
    if (st == QK_ERR_CANCELLED) return qk::fail(st, "qk_serve_poll: request cancelled before admission");
    if (st != QK_OK) return qk::fail(st, "qk_serve_poll: request failed while pricing, status " + std::to_string(st));
    return st;
}

qk_status qk_serve_cancel(qk_server *s, int64_t ticket, int32_t *cancelled) {
    if (!s || !cancelled) return qk::fail(QK_ERR_INVALID_ARG, "NULL argument");
    *cancelled = 0;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (ticket <= 0 || ticket >= s->next_ticket) return qk::fail(QK_ERR_STATE, "unknown ticket");
        auto it = std::find_if(s->queue.begin(), s->queue.end(), [&](const Request &r) { return r.ticket == ticket; });
        if (it == s->queue.end()) return QK_OK;  // admitted already (or finished): it completes
        s->queued_us = std::max(0.0, s->queued_us - it->est_us);
        s->queue.erase(it);
        Finished f;
        std::memset(&f.r, 0, sizeof(f.r));
        f.r.status = QK_ERR_CANCELLED;
        f.status = QK_ERR_CANCELLED;
        f.latency_ms = 0.0;
        s->done[ticket] = f;
        *cancelled = 1;
    }
    s->cv_done.notify_all();
    return QK_OK;
}

qk_status qk_serve_stats_get(qk_server *s, qk_serve_stats *out) {
    if (!s || !out) return qk::fail(QK_ERR_INVALID_ARG, "NULL argument");
    std::lock_guard<std::mutex> lk(s->mu);
    std::memset(out, 0, sizeof(*out));
    out->submitted = s->submitted;
    out->completed = s->completed;
    out->rejected = s->rejected;
    out->batches = s->batches;
    out->busy_s = s->busy_s;
    out->reserved_mib = static_cast<int64_t>(s->reserved >> 20);
    if (!s->records.empty()) {
        std::vector<double> l(s->records.size());
        for (size_t i = 0; i < l.size(); ++i) l[i] = s->records[i].latency_ms;
        std::sort(l.begin(), l.end());
        auto pct = [&](double p) { return l[std::min(l.size() - 1, static_cast<size_t>(p * (l.size() - 1) + 0.5))]; };
        out->p50_ms = pct(0.50);
        out->p99_ms = pct(0.99);
        out->p999_ms = pct(0.999);
        out->max_ms = l.back();
        const double span = std::chrono::duration<double>(s->t_last - s->t_first).count();
        if (span > 0.0) {
            out->contracts_per_s = static_cast<double>(s->completed) / span;
            out->path_steps_per_s = s->path_steps / span;
        }
    }
    return QK_OK;
}

qk_status qk_serve_records(qk_server *s, qk_serve_record *out, int64_t capacity, int64_t *count) {
    if (!s || !count || (capacity > 0 && !out)) return qk::fail(QK_ERR_INVALID_ARG, "NULL argument");
    std::lock_guard<std::mutex> lk(s->mu);
    const size_t n = s->records.size();
    const size_t m = std::min(n, static_cast<size_t>(std::max<int64_t>(capacity, 0)));
    for (size_t i = 0; i < m; ++i) out[i] = s->records[(s->rec_head + i) % n];
    *count = static_cast<int64_t>(n);
    return QK_OK;
}

qk_status qk_serve_stop(qk_server *s) {
    if (!s) return QK_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    for (auto &t : s->lanes) t.join();
    for (qk_handle *h : s->handles) qk_destroy(h);
    qk::pool_release(s->device, s->reserved);
    delete s;
    return QK_OK;
}

}  // extern "C"
