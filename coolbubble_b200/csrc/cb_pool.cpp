/* cb_pool.cpp -- a request loop that keeps runs resident on the GPU.
 *
 * No counterpart in the reference (one run per process, main.cpp). Callers
 * submit runs (parameters, initial-condition seed, number of steps). Two
 * threads serve them:
 *
 *  - the admission thread takes runs in arrival order while a slot and their
 *    memory fit the device-memory budget and builds each start on the device
 *    (cb_create_from_seed) on the run's own stream, so drawing a start on the
 *    host never holds up the runs already stepping;
 *  - the stepping thread keeps every admitted run's stream fed: each run has
 *    up to RING chunks queued (a chunk ends at the run's next output step and
 *    is followed by an asynchronous copy of its step record and an event);
 *    as soon as a run's oldest chunk completes its box averages are taken
 *    from the record and another chunk is queued. Runs never wait for one
 *    another, and a finished run's memory goes back to the budget at once
 *    (released in stream order, without a device-wide synchronise).
 *
 * Runs that arrive while others are on the GPU join as soon as a slot and
 * their memory are free (continuous batching). Each run's arithmetic does not
 * depend on the others', so a result is the same alone and in a mix.
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

constexpr int RING = 2;   /* chunks a run may have queued on its stream */

struct Chunk {
    int steps = 0;
    bool report = false;   /* the chunk ends at an output step */
    double t = 0.0;        /* the run's time after the chunk */
};

struct Request {
    int64_t id = 0;
    cb_request req{};
    std::string xns_in;
    int state = CB_REQ_QUEUED;
    std::string err;
    cb_handle *h = nullptr;
    int steps_done = 0;     /* steps whose chunk has completed */
    int steps_queued = 0;   /* steps queued on the stream */
    int64_t footprint = 0;
    bool cancel = false;
    bool building = false;  /* the admission thread owns it */
    int slot = -1;          /* pinned step records and events of the run */
    Chunk ring[RING];
    int ring_head = 0, ring_count = 0;
    int fail_status = CB_OK;
    std::string fail_why;
    Clock::time_point t_submit, t_admit, t_done;
    std::vector<cb_sums> lines;
    std::vector<float> phi, pi;
};

double seconds(Clock::time_point a, Clock::time_point b) { return std::chrono::duration<double>(b - a).count(); }

}  // namespace

struct cb_pool {
    std::mutex mu;
    std::condition_variable changed;   /* a request changed state */
    std::condition_variable work;      /* new work for either thread */
    std::thread admitter, stepper;
    bool stop = false;
    bool broken = false;
    std::string broken_why;
    int64_t budget = 0, used = 0;
    int max_active = 0;
    int device = 0;
    int64_t next_id = 1;
    std::deque<Request *> queue;
    std::vector<Request *> active;     /* admitted: being built or stepping */
    std::vector<Request *> ready;      /* built, not yet taken by the stepping thread */
    std::map<int64_t, Request *> all;
    std::vector<int> free_slots;
    cb::DevState *records = nullptr;   /* pinned, max_active * RING */
    std::vector<cudaEvent_t> events;   /* max_active * RING, made by the stepping thread */
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
    if (r->slot >= 0) {
        P->free_slots.push_back(r->slot);
        r->slot = -1;
    }
    auto it = std::find(P->active.begin(), P->active.end(), r);
    if (it != P->active.end()) P->active.erase(it);
    if (state == CB_REQ_DONE) P->completed++;
    else if (state == CB_REQ_FAILED) P->failed++;
    else if (state == CB_REQ_CANCELLED) P->cancelled++;
    P->changed.notify_all();
    P->work.notify_all();   /* memory and a slot are free again */
}

/* Called with P->mu held: the head of the queue, if it can be admitted now. */
Request *admissible_head(cb_pool *P) {
    while (!P->queue.empty()) {
        Request *head = P->queue.front();
        if (head->footprint > P->budget) {
            P->queue.pop_front();
            finish(P, head, CB_REQ_FAILED, "run needs more memory than the pool's whole budget");
            continue;
        }
        if ((int)P->active.size() >= P->max_active || P->free_slots.empty()) return nullptr;
        if (P->used + head->footprint > P->budget) return nullptr;   /* first come, first served */
        return head;
    }
    return nullptr;
}

void run_admitter(cb_pool *P) {
    if (cb_set_device(P->device) != CB_OK) {
        std::lock_guard<std::mutex> lock(P->mu);
        if (!P->broken) {
            P->broken = true;
            P->broken_why = std::string("pool admission stopped: ") + cb_last_error(nullptr);
        }
        P->work.notify_all();
        return;
    }
    for (;;) {
        Request *r = nullptr;
        bool injected = false;
        {
            std::unique_lock<std::mutex> lock(P->mu);
            P->work.wait(lock, [&] { return P->stop || P->broken || admissible_head(P) != nullptr; });
            if (P->stop || P->broken) return;
            r = P->queue.front();
            P->queue.pop_front();
            P->used += r->footprint;
            r->state = CB_REQ_RUNNING;
            r->building = true;
            r->t_admit = Clock::now();
            r->slot = P->free_slots.back();
            P->free_slots.pop_back();
            P->active.push_back(r);
            P->admitted++;
            if (P->inject == CB_INJECT_ADMISSION_FAILURE) {
                P->inject = 0;
                injected = true;
            }
        }
        int st = CB_OK;
        std::string why;
        cb_handle *h = nullptr;
        if (injected) {
            st = CB_ENOMEM;
            why = "injected admission failure";
        } else {
            cb_sums first;
            st = cb_create_from_seed(&r->req.params, &r->req.ic, r->xns_in.empty() ? nullptr : r->xns_in.c_str(),
                                     &first, nullptr, 0, nullptr, &h);
            if (st != CB_OK) why = cb_last_error(nullptr);
        }
        std::lock_guard<std::mutex> lock(P->mu);
        r->building = false;
        if (st != CB_OK) {
            finish(P, r, CB_REQ_FAILED, why);
        } else if (P->broken) {
            cb_destroy(h);
            finish(P, r, CB_REQ_FAILED, P->broken_why);
        } else if (r->cancel) {
            cb_destroy(h);
            finish(P, r, CB_REQ_CANCELLED, "cancelled");
        } else {
            r->h = h;
            P->ready.push_back(r);
            P->work.notify_all();
        }
    }
}

/* Queue the run's next chunk: up to its next output step or its end, then a
 * copy of its step record and an event. */
int queue_chunk(cb_pool *P, Request *r) {
    const int every = r->req.sums_every > 0 ? r->req.sums_every : r->req.nt;
    const int to_event = every - (r->steps_queued % every);
    const int k = std::min(to_event, r->req.nt - r->steps_queued);
    const bool report = r->req.sums_every > 0 && (r->steps_queued + k) % every == 0;
    int st = cb::step_impl(r->h, k, report ? CB_STEP_SUMS : 0, false);
    const int at = (r->ring_head + r->ring_count) % RING;
    const int idx = r->slot * RING + at;
    if (st == CB_OK) st = cb::enqueue_record_copy(r->h, &P->records[idx]);
    if (st == CB_OK) {
        cudaError_t e = cudaEventRecord(P->events[idx], r->h->stream);
        if (e != cudaSuccess) st = cb::cuda_fail(r->h, e, "recording an event");
    }
    if (st != CB_OK) return st;
    Chunk &c = r->ring[at];
    c.steps = k;
    c.report = report;
    c.t = r->h->t;
    r->ring_count++;
    r->steps_queued += k;
    return CB_OK;
}

/* Take the run's oldest chunk if it has completed. 1: taken, 0: not yet, <0: failed. */
int take_chunk(cb_pool *P, Request *r) {
    const int idx = r->slot * RING + r->ring_head;
    cudaError_t e = cudaEventQuery(P->events[idx]);
    if (e == cudaErrorNotReady) return 0;
    const Chunk c = r->ring[r->ring_head];
    r->ring_head = (r->ring_head + 1) % RING;
    r->ring_count--;
    if (e != cudaSuccess) {
        r->fail_status = cb::cuda_fail(r->h, e, "running a chunk of steps");
        r->fail_why = r->h->err;
        return -1;
    }
    cb_sums line;
    int st = cb::sums_from_record(r->h, P->records[idx], c.t, c.report ? &line : nullptr);
    if (st != CB_OK) {
        r->fail_status = st;
        r->fail_why = r->h->err;
        return -1;
    }
    std::lock_guard<std::mutex> lock(P->mu);
    if (c.report) r->lines.push_back(line);
    r->steps_done += c.steps;
    P->site_updates += (double)r->h->N * c.steps;
    return 1;
}

void retire(cb_pool *P, Request *r, int state, const std::string &why) {
    cb_destroy(r->h);   /* stream-ordered releases: no device-wide wait */
    r->h = nullptr;
    std::lock_guard<std::mutex> lock(P->mu);
    finish(P, r, state, why);
}

void fail_everything(cb_pool *P, std::vector<Request *> &mine, const std::string &why) {
    std::lock_guard<std::mutex> lock(P->mu);
    P->broken = true;
    P->broken_why = why;
    for (Request *r : P->ready) mine.push_back(r);
    P->ready.clear();
    for (Request *r : mine) {
        if (r->h) cb_destroy(r->h);
        r->h = nullptr;
        finish(P, r, CB_REQ_FAILED, why);
    }
    mine.clear();
    for (Request *r : P->queue) finish(P, r, CB_REQ_FAILED, why);
    P->queue.clear();
    /* a run the admission thread is still building fails when it returns */
    P->changed.notify_all();
    P->work.notify_all();
}

void run_stepper(cb_pool *P) {
    std::vector<Request *> mine;
    try {
        if (cb_set_device(P->device) != CB_OK) throw std::runtime_error(cb_last_error(nullptr));
        for (auto &ev : P->events)
            if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
                cudaGetLastError();
                throw std::runtime_error("creating the pool's events failed");
            }
        for (;;) {
            {
                std::unique_lock<std::mutex> lock(P->mu);
                if (P->stop) break;
                if (mine.empty() && P->ready.empty())
                    P->work.wait_for(lock, std::chrono::milliseconds(20),
                                     [&] { return P->stop || !P->ready.empty() || P->inject == CB_INJECT_WORKER_EXCEPTION; });
                if (P->stop) break;
                for (Request *r : P->ready) mine.push_back(r);
                P->ready.clear();
                if (!mine.empty() && P->inject == CB_INJECT_WORKER_EXCEPTION) {
                    P->inject = 0;
                    throw std::runtime_error("injected worker failure");
                }
            }
            if (mine.empty()) continue;
            const auto t_start = Clock::now();
            bool in_flight = false, progressed = false;
            for (size_t i = 0; i < mine.size();) {
                Request *r = mine[i];
                int got;
                while (r->ring_count > 0 && (got = take_chunk(P, r)) != 0) {
                    progressed = true;
                    if (got < 0) break;
                }
                if (r->ring_count > 0 && r->fail_status == CB_OK && !r->cancel) in_flight = true;
                bool cancel;
                {
                    std::lock_guard<std::mutex> lock(P->mu);
                    cancel = r->cancel;
                }
                /* top the run's queue up, unless it is winding down */
                while (r->fail_status == CB_OK && !cancel && r->ring_count < RING && r->steps_queued < r->req.nt) {
                    int st = queue_chunk(P, r);
                    if (st != CB_OK) {
                        r->fail_status = st;
                        r->fail_why = r->h->err;
                    }
                    progressed = true;
                    in_flight = true;
                }
                int state = -1;
                std::string why;
                if (r->ring_count == 0) {
                    if (r->fail_status != CB_OK) {
                        state = CB_REQ_FAILED;
                        why = r->fail_why;
                    } else if (cancel) {
                        state = CB_REQ_CANCELLED;
                        why = "cancelled";
                    } else if (r->steps_done >= r->req.nt) {
                        int st = CB_OK;
                        if (r->req.want_fields) {
                            r->phi.resize(r->h->N);
                            r->pi.resize(r->h->N);
                            st = cb_get_fields_f32(r->h, r->phi.data(), r->pi.data(), nullptr, nullptr, nullptr);
                        }
                        state = st == CB_OK ? CB_REQ_DONE : CB_REQ_FAILED;
                        if (st != CB_OK) why = r->h->err;
                    }
                }
                if (state >= 0) {
                    retire(P, r, state, why);
                    mine.erase(mine.begin() + i);
                    progressed = true;
                    continue;
                }
                ++i;
            }
            if (!progressed) std::this_thread::sleep_for(std::chrono::microseconds(20));
            if (in_flight) {
                std::lock_guard<std::mutex> lock(P->mu);
                P->busy_s += seconds(t_start, Clock::now());
            }
        }
    } catch (const std::exception &ex) {
        fail_everything(P, mine, std::string("pool worker stopped: ") + ex.what());
    }
}

}  // namespace

extern "C" {

int cb_pool_create(int64_t budget_bytes, int max_active, cb_pool **out) {
    if (budget_bytes <= 0 || max_active < 1 || max_active > 4096 || !out)
        return cb::fail(nullptr, CB_EINVAL, "cb_pool_create: bad arguments");
    cb_pool *P = new cb_pool();
    P->budget = budget_bytes;
    P->max_active = max_active;
    P->t0 = Clock::now();
    if (cudaGetDevice(&P->device) != cudaSuccess) { cudaGetLastError(); P->device = 0; }
    cudaError_t e = cudaMallocHost(&P->records, (size_t)max_active * RING * sizeof(cb::DevState));
    if (e != cudaSuccess) {
        cudaGetLastError();
        delete P;
        return cb::fail(nullptr, CB_ENOMEM, "cb_pool_create: pinned step records");
    }
    P->events.assign((size_t)max_active * RING, nullptr);
    for (int s = max_active - 1; s >= 0; --s) P->free_slots.push_back(s);
    P->stepper = std::thread(run_stepper, P);
    P->admitter = std::thread(run_admitter, P);
    *out = P;
    return CB_OK;
}

int cb_pool_submit(cb_pool *P, const cb_request *req, const char *xns_in, int64_t *id) {
    if (!P || !req || !id) return cb::fail(nullptr, CB_EINVAL, "cb_pool_submit: bad arguments");
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
    P->work.notify_all();
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
    P->work.notify_all();
    return CB_OK;
}

int cb_pool_destroy(cb_pool *P) {
    if (!P) return CB_EINVAL;
    {
        std::lock_guard<std::mutex> lock(P->mu);
        P->stop = true;
        P->work.notify_all();
    }
    if (P->admitter.joinable()) P->admitter.join();
    if (P->stepper.joinable()) P->stepper.join();
    for (auto &kv : P->all) {
        if (kv.second->h) cb_destroy(kv.second->h);
        delete kv.second;
    }
    for (cudaEvent_t ev : P->events)
        if (ev) cudaEventDestroy(ev);
    cudaFreeHost(P->records);
    delete P;
    return CB_OK;
}

}  // extern "C"
