/* cb_pool.cpp -- a request loop that keeps runs resident on the GPU.
 *
 * No counterpart in the reference (one run per process, main.cpp). Callers
 * submit runs (parameters, initial-condition seed, number of steps); a worker
 * thread admits them against a device-memory budget and a slot limit, builds
 * their initial conditions on the device (cb_create_from_seed), and advances
 * every admitted run concurrently on its own stream in chunks that end at the
 * run's output steps, where it records the box averages. Runs that arrive
 * while others are on the GPU join as soon as a slot and their memory are
 * free (continuous batching); a finished run's memory is released at once.
 * Each run's arithmetic does not depend on the others', so a result is the
 * same alone and in a mix.
 */
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <exception>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "cb_handle.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    int64_t id = 0;
    cb_request req{};
    std::string xns_in;
    int state = CB_REQ_QUEUED;
    std::string err;
    cb_handle *h = nullptr;
    int steps_done = 0;
    int64_t footprint = 0;
    bool cancel = false;
    Clock::time_point t_submit, t_admit, t_done;
    std::vector<cb_sums> lines;
    std::vector<float> phi, pi;
};

double seconds(Clock::time_point a, Clock::time_point b) { return std::chrono::duration<double>(b - a).count(); }

}  // namespace

struct cb_pool {
    std::mutex mu;
    std::condition_variable changed;   /* a request changed state */
    std::condition_variable work;      /* new work for the worker */
    std::thread worker;
    bool stop = false;
    bool broken = false;
    std::string broken_why;
    int64_t budget = 0, used = 0;
    int max_active = 0;
    int device = 0;
    int64_t next_id = 1;
    std::deque<Request *> queue;
    std::vector<Request *> active;
    std::map<int64_t, Request *> all;
    int inject = 0;                    /* test hook: CB_INJECT_* */
    Clock::time_point t0;
    double site_updates = 0.0;
    int64_t completed = 0, failed = 0, cancelled = 0, admitted = 0;
    double busy_s = 0.0;
};

namespace {

int64_t footprint_of(const cb_params &p) {
    int64_t f = cb_footprint_bytes(&p);
    if (f < 0) return f;
    size_t N = 1;
    for (int i = 0; i < p.d; ++i) N *= (size_t)p.n_grids;
    return f + (int64_t)(N * sizeof(double)) * 2;   /* the initial condition's transient buffers */
}

void finish(cb_pool *P, Request *r, int state, const std::string &why) {
    /* called with P->mu held */
    r->state = state;
    r->err = why;
    r->t_done = Clock::now();
    P->used -= r->footprint;
    r->footprint = 0;
    if (state == CB_REQ_DONE) P->completed++;
    else if (state == CB_REQ_FAILED) P->failed++;
    else if (state == CB_REQ_CANCELLED) P->cancelled++;
    P->changed.notify_all();
}

/* Admit from the head of the queue while a slot and the memory are free. */
void admit(cb_pool *P) {
    for (;;) {
        Request *r = nullptr;
        {
            std::lock_guard<std::mutex> lock(P->mu);
            if (P->queue.empty() || (int)P->active.size() >= P->max_active) return;
            Request *head = P->queue.front();
            if (head->footprint > P->budget) {
                P->queue.pop_front();
                finish(P, head, CB_REQ_FAILED, "run needs more memory than the pool's whole budget");
                continue;
            }
            if (P->used + head->footprint > P->budget) return;   /* first come, first served */
            P->queue.pop_front();
            P->used += head->footprint;
            head->state = CB_REQ_RUNNING;
            head->t_admit = Clock::now();
            P->admitted++;
            r = head;
        }
        int st = CB_OK;
        std::string why;
        bool injected = false;
        {
            std::lock_guard<std::mutex> lock(P->mu);
            if (P->inject == CB_INJECT_ADMISSION_FAILURE) {
                P->inject = 0;
                injected = true;
            }
        }
        if (injected) {
            st = CB_ENOMEM;
            why = "injected admission failure";
        } else {
            cb_sums first;
            st = cb_create_from_seed(&r->req.params, &r->req.ic, r->xns_in.empty() ? nullptr : r->xns_in.c_str(),
                                     &first, nullptr, 0, nullptr, &r->h);
            if (st != CB_OK) why = cb_last_error(nullptr);
        }
        std::lock_guard<std::mutex> lock(P->mu);
        if (st != CB_OK) {
            r->h = nullptr;
            finish(P, r, CB_REQ_FAILED, why);
            continue;
        }
        P->active.push_back(r);
    }
}

/* One tick: every active run advances to its next output step (or its end). */
void tick(cb_pool *P) {
    std::vector<Request *> act;
    {
        std::lock_guard<std::mutex> lock(P->mu);
        act = P->active;
    }
    if (act.empty()) return;
    {
        std::lock_guard<std::mutex> lock(P->mu);
        if (P->inject == CB_INJECT_WORKER_EXCEPTION) {
            P->inject = 0;
            throw std::runtime_error("injected worker failure");
        }
    }
    const auto t_start = Clock::now();
    std::vector<int> chunk(act.size(), 0);
    for (size_t i = 0; i < act.size(); ++i) {
        Request *r = act[i];
        if (r->cancel) continue;
        const int every = r->req.sums_every > 0 ? r->req.sums_every : r->req.nt;
        const int to_event = every - (r->steps_done % every);
        const int k = std::min(to_event, r->req.nt - r->steps_done);
        const bool event = (r->steps_done + k) % every == 0 && r->req.sums_every > 0;
        if (cb::step_impl(r->h, k, event ? CB_STEP_SUMS : 0, false) != CB_OK) {
            chunk[i] = -1;
            continue;
        }
        chunk[i] = k;
    }
    double updates = 0.0;
    for (size_t i = 0; i < act.size(); ++i) {
        Request *r = act[i];
        std::string why;
        int state = -1;
        if (r->cancel) {
            state = CB_REQ_CANCELLED;
        } else if (chunk[i] < 0) {
            state = CB_REQ_FAILED;
            why = r->h->err;
        } else {
            const bool event = r->req.sums_every > 0 && (r->steps_done + chunk[i]) % r->req.sums_every == 0;
            cb_sums line;
            int st = event ? cb_get_sums(r->h, &line) : cb_sync(r->h);
            if (st != CB_OK) {
                state = CB_REQ_FAILED;
                why = r->h->err;
            } else {
                if (event) r->lines.push_back(line);
                r->steps_done += chunk[i];
                updates += (double)r->h->N * chunk[i];
                if (r->steps_done >= r->req.nt) {
                    if (r->req.want_fields) {
                        r->phi.resize(r->h->N);
                        r->pi.resize(r->h->N);
                        st = cb_get_fields_f32(r->h, r->phi.data(), r->pi.data(), nullptr, nullptr, nullptr);
                    }
                    state = st == CB_OK ? CB_REQ_DONE : CB_REQ_FAILED;
                    if (st != CB_OK) why = r->h->err;
                }
            }
        }
        if (state >= 0) {
            cb_destroy(r->h);
            r->h = nullptr;
            std::lock_guard<std::mutex> lock(P->mu);
            P->active.erase(std::find(P->active.begin(), P->active.end(), r));
            finish(P, r, state, why);
        }
    }
    std::lock_guard<std::mutex> lock(P->mu);
    P->site_updates += updates;
    P->busy_s += seconds(t_start, Clock::now());
}

void run_worker(cb_pool *P) {
    try {
        if (cb_set_device(P->device) != CB_OK) throw std::runtime_error(cb_last_error(nullptr));
        for (;;) {
            {
                std::unique_lock<std::mutex> lock(P->mu);
                if (P->stop) break;
                if (P->queue.empty() && P->active.empty())
                    P->work.wait_for(lock, std::chrono::milliseconds(20));
                if (P->stop) break;
            }
            admit(P);
            tick(P);
        }
    } catch (const std::exception &ex) {
        std::lock_guard<std::mutex> lock(P->mu);
        P->broken = true;
        P->broken_why = std::string("pool worker stopped: ") + ex.what();
        for (Request *r : P->active) {
            if (r->h) { cb_destroy(r->h); r->h = nullptr; }
            finish(P, r, CB_REQ_FAILED, P->broken_why);
        }
        P->active.clear();
        for (Request *r : P->queue) finish(P, r, CB_REQ_FAILED, P->broken_why);
        P->queue.clear();
        P->changed.notify_all();
    }
}

}  // namespace

extern "C" {

int cb_pool_create(int64_t budget_bytes, int max_active, cb_pool **out) {
    if (budget_bytes <= 0 || max_active < 1 || !out) return cb::fail(nullptr, CB_EINVAL, "cb_pool_create: bad arguments");
    cb_pool *P = new cb_pool();
    P->budget = budget_bytes;
    P->max_active = max_active;
    P->t0 = Clock::now();
    if (cudaGetDevice(&P->device) != cudaSuccess) { cudaGetLastError(); P->device = 0; }
    P->worker = std::thread(run_worker, P);
    *out = P;
    return CB_OK;
}

int cb_pool_submit(cb_pool *P, const cb_request *req, const char *xns_in, int64_t *id) {
    if (!P || !req || !id) return cb::fail(nullptr, CB_EINVAL, "cb_pool_submit: bad arguments");
    std::string why;
    if (req->nt < 1) return cb::fail(nullptr, CB_EINVAL, "cb_pool_submit: nt must be at least 1");
    if (req->sums_every < 0) return cb::fail(nullptr, CB_EINVAL, "cb_pool_submit: sums_every must be >= 0");
    const int64_t fp = footprint_of(req->params);
    if (fp < 0) return cb::fail(nullptr, CB_EINVAL, "cb_pool_submit: invalid run parameters");
    Request *r = new Request();
    r->req = *req;
    if (xns_in) r->xns_in = xns_in;
    r->footprint = fp;
    r->t_submit = Clock::now();
    std::lock_guard<std::mutex> lock(P->mu);
    if (P->broken) {
        delete r;
        return cb::fail(nullptr, CB_EDEVICE, P->broken_why);
    }
    r->id = P->next_id++;
    P->all[r->id] = r;
    P->queue.push_back(r);
    *id = r->id;
    P->work.notify_one();
    return CB_OK;
}

int cb_pool_status(cb_pool *P, int64_t id, int *state, int *steps_done) {
    if (!P) return CB_EINVAL;
    std::lock_guard<std::mutex> lock(P->mu);
    auto it = P->all.find(id);
    if (it == P->all.end()) return cb::fail(nullptr, CB_ENOTFOUND, "unknown run id");
    if (state) *state = it->second->state;
    if (steps_done) *steps_done = it->second->steps_done;
    return CB_OK;
}

int cb_pool_wait(cb_pool *P, int64_t id, int timeout_ms) {
    if (!P) return CB_EINVAL;
    std::unique_lock<std::mutex> lock(P->mu);
    auto it = P->all.find(id);
    if (it == P->all.end()) return cb::fail(nullptr, CB_ENOTFOUND, "unknown run id");
    Request *r = it->second;
    const auto until = Clock::now() + std::chrono::milliseconds(timeout_ms < 0 ? 0 : timeout_ms);
    while (r->state == CB_REQ_QUEUED || r->state == CB_REQ_RUNNING) {
        if (P->changed.wait_until(lock, until) == std::cv_status::timeout &&
            (r->state == CB_REQ_QUEUED || r->state == CB_REQ_RUNNING))
            return cb::fail(nullptr, CB_ETIMEOUT, "run not finished within the timeout");
    }
    return CB_OK;
}

int cb_pool_result(cb_pool *P, int64_t id, cb_sums *lines, int max_lines, int *nlines, float *phi, float *pi,
                   double *latency_s, char *err, size_t err_cap) {
    if (!P) return CB_EINVAL;
    std::lock_guard<std::mutex> lock(P->mu);
    auto it = P->all.find(id);
    if (it == P->all.end()) return cb::fail(nullptr, CB_ENOTFOUND, "unknown run id");
    Request *r = it->second;
    if (r->state == CB_REQ_QUEUED || r->state == CB_REQ_RUNNING)
        return cb::fail(nullptr, CB_EBUSY, "run not finished");
    if (nlines) *nlines = (int)r->lines.size();
    if (lines)
        for (int i = 0; i < (int)r->lines.size() && i < max_lines; ++i) lines[i] = r->lines[i];
    if (phi && !r->phi.empty()) std::memcpy(phi, r->phi.data(), r->phi.size() * sizeof(float));
    if (pi && !r->pi.empty()) std::memcpy(pi, r->pi.data(), r->pi.size() * sizeof(float));
    if (latency_s) *latency_s = seconds(r->t_submit, r->t_done);
    if (err && err_cap) {
        std::strncpy(err, r->err.c_str(), err_cap - 1);
        err[err_cap - 1] = 0;
    }
    return r->state == CB_REQ_DONE ? CB_OK : (r->state == CB_REQ_CANCELLED ? CB_ENOTFOUND : CB_EDEVICE);
}

int cb_pool_cancel(cb_pool *P, int64_t id) {
    if (!P) return CB_EINVAL;
    std::lock_guard<std::mutex> lock(P->mu);
    auto it = P->all.find(id);
    if (it == P->all.end()) return cb::fail(nullptr, CB_ENOTFOUND, "unknown run id");
    Request *r = it->second;
    if (r->state == CB_REQ_QUEUED) {
        P->queue.erase(std::find(P->queue.begin(), P->queue.end(), r));
        finish(P, r, CB_REQ_CANCELLED, "cancelled");
    } else if (r->state == CB_REQ_RUNNING) {
        r->cancel = true;
    }
    return CB_OK;
}

int cb_pool_get_stats(cb_pool *P, cb_pool_stats *out) {
    if (!P || !out) return CB_EINVAL;
    std::lock_guard<std::mutex> lock(P->mu);
    out->queued = (int64_t)P->queue.size();
    out->active = (int64_t)P->active.size();
    out->completed = P->completed;
    out->failed = P->failed;
    out->cancelled = P->cancelled;
    out->admitted = P->admitted;
    out->used_bytes = P->used;
    out->budget_bytes = P->budget;
    out->site_updates = P->site_updates;
    out->busy_s = P->busy_s;
    out->wall_s = seconds(P->t0, Clock::now());
    return CB_OK;
}

int cb_pool_inject_failure(cb_pool *P, int kind) {
    if (!P || (kind != CB_INJECT_ADMISSION_FAILURE && kind != CB_INJECT_WORKER_EXCEPTION)) return CB_EINVAL;
    std::lock_guard<std::mutex> lock(P->mu);
    P->inject = kind;
    P->work.notify_one();
    return CB_OK;
}

int cb_pool_destroy(cb_pool *P) {
    if (!P) return CB_EINVAL;
    {
        std::lock_guard<std::mutex> lock(P->mu);
        P->stop = true;
        P->work.notify_all();
    }
    if (P->worker.joinable()) P->worker.join();
    for (auto &kv : P->all) {
        if (kv.second->h) cb_destroy(kv.second->h);
        delete kv.second;
    }
    delete P;
    return CB_OK;
}

}  // extern "C"
