// se_serve.cu -- a request loop over one GPU: queued Spectral Ewald solves
// admitted by free slot and device-memory footprint, overlapping on their own
// streams, with plans cached and kept resident between requests.
//
// Threads: callers submit and poll from any thread; one dispatcher thread
// owns every plan, stream and event.  The mutex guards only the queue, the
// completion list and the counters, so no CUDA call is made under it.
//
// A request's life: queued -> admitted (a slot and a plan are bound; the
// inputs are copied to the plan's staging buffers when they are host memory;
// se_solve_system runs; the result and the plan's input-error flag are copied
// back; an event is recorded) -> completed (the dispatcher sees the event,
// reads the flag, frees the slot and returns the plan to the idle cache).
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>

#include "se_internal.h"

namespace {

using Clock = std::chrono::steady_clock;

constexpr int MAX_SLOTS = 64;

double seconds(Clock::time_point a, Clock::time_point b)
{
    return std::chrono::duration<double>(b - a).count();
}

int out_width(const se_system& s) { return s.mode == SE_FORCE ? 3 : 1; }

// Particle capacity class of a plan: the next power of two >= N (>= 1024), so
// a plan serves every request of its class and the ones below it.
int capacity_class(int N)
{
    int c = 1024;
    while (c < N && c < (1 << 30)) c <<= 1;
    return c;
}

se_config config_of(const se_system& s, int cap, int precision)
{
    se_config c;
    c.M = s.M;
    c.P = s.P;
    c.L = s.L;
    c.xi = s.xi;
    c.m = s.m;
    c.mode = s.mode;
    c.precision = precision;
    c.max_particles = cap;
    return c;
}

size_t plan_bytes(const se_system& s, int cap, int precision)
{
    se_config c = config_of(s, cap, precision);
    // the plan's own buffers + the staging copies of x, q and out
    return se_plan_device_bytes(&c) + (size_t)cap * 8 * (4 + out_width(s));
}

struct PlanEntry {
    se_plan plan = nullptr;
    int M = 0, P = 0, mode = 0, cap = 0;
    size_t bytes = 0;
    double* d_x = nullptr;
    double* d_q = nullptr;
    double* d_out = nullptr;
    bool busy = false;
    unsigned long long last_used = 0;
};

struct Pending {
    long long ticket;
    se_request req;
    Clock::time_point t_submit;
};

struct Slot {
    cudaStream_t st = nullptr;
    cudaEvent_t done = nullptr;
    int* h_err = nullptr;   // pinned: the plan's input-error flag after the solve
    bool busy = false;
    PlanEntry* plan = nullptr;
    long long ticket = 0;
    Clock::time_point t_submit, t_admit;
    int launch_status = SE_OK;
};

}  // namespace

struct se_server_s {
    se_server_config cfg{};
    int device = 0;
    // guarded by mu
    std::mutex mu;
    std::condition_variable cv_work;   // dispatcher: new requests or stop
    std::condition_variable cv_done;   // drain: completions
    std::deque<Pending> queue;
    std::deque<se_completion> done;
    long long next_ticket = 1;
    long long submitted = 0, completed = 0, failed = 0;
    int in_flight = 0;
    int nplans = 0;
    long long plans_created = 0, plans_evicted = 0;
    size_t hbm_used = 0, hbm_peak = 0;
    bool stop = false;
    std::vector<se_system> reserve_req;   // handed to the dispatcher
    int reserve_status = SE_OK;
    bool reserve_pending = false;
    // dispatcher-owned
    std::vector<Slot> slots;
    std::vector<PlanEntry*> plans;
    unsigned long long use_clock = 0;
    std::thread worker;
};

namespace {

int free_plan(se_server s, PlanEntry* pe)
{
    if (pe->plan) se_plan_destroy(pe->plan);
    if (pe->d_x) cudaFree(pe->d_x);
    if (pe->d_q) cudaFree(pe->d_q);
    if (pe->d_out) cudaFree(pe->d_out);
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->hbm_used -= pe->bytes;
        s->nplans--;
    }
    delete pe;
    return SE_OK;
}

// A new plan for (M, P, mode) of capacity cap; the caller has checked the budget.
int make_plan(se_server s, const se_system& sys, int cap, PlanEntry** out)
{
    PlanEntry* pe = new PlanEntry();
    pe->M = sys.M;
    pe->P = sys.P;
    pe->mode = sys.mode;
    pe->cap = cap;
    pe->bytes = plan_bytes(sys, cap, s->cfg.precision);
    se_config c = config_of(sys, cap, s->cfg.precision);
    int r = se_plan_create(&pe->plan, &c);
    cudaError_t e = cudaSuccess;
    if (r == SE_OK) e = cudaMalloc(&pe->d_x, sizeof(double) * 3 * cap);
    if (r == SE_OK && e == cudaSuccess) e = cudaMalloc(&pe->d_q, sizeof(double) * cap);
    if (r == SE_OK && e == cudaSuccess)
        e = cudaMalloc(&pe->d_out, sizeof(double) * out_width(sys) * cap);
    if (r == SE_OK && e != cudaSuccess) r = se::cuda_fail(e, "cudaMalloc", __FILE__, __LINE__);
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->hbm_used += pe->bytes;
        s->nplans++;
    }
    if (r != SE_OK) {
        free_plan(s, pe);
        return r;
    }
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->plans_created++;
        s->hbm_peak = std::max(s->hbm_peak, s->hbm_used);
    }
    s->plans.push_back(pe);
    *out = pe;
    return SE_OK;
}

size_t used_bytes(se_server s)
{
    std::lock_guard<std::mutex> g(s->mu);
    return s->hbm_used;
}

// The idle cached plan of the smallest capacity that serves sys, or a new one
// when the budget allows (after freeing idle plans, least recently used
// first).  *pe == nullptr with SE_OK: nothing fits until running solves end.
int acquire_plan(se_server s, const se_system& sys, PlanEntry** pe)
{
    *pe = nullptr;
    PlanEntry* best = nullptr;
    for (PlanEntry* p : s->plans)
        if (!p->busy && p->M == sys.M && p->P == sys.P && p->mode == sys.mode && p->cap >= sys.N &&
            (!best || p->cap < best->cap))
            best = p;
    if (best) {
        *pe = best;
        return SE_OK;
    }
    const int cap = capacity_class(sys.N);
    const size_t need = plan_bytes(sys, cap, s->cfg.precision);
    while (used_bytes(s) + need > s->cfg.hbm_budget) {
        PlanEntry* lru = nullptr;
        for (PlanEntry* p : s->plans)
            if (!p->busy && (!lru || p->last_used < lru->last_used)) lru = p;
        if (!lru) return SE_OK;   // wait for running solves
        s->plans.erase(std::find(s->plans.begin(), s->plans.end(), lru));
        free_plan(s, lru);
        std::lock_guard<std::mutex> g(s->mu);
        s->plans_evicted++;
    }
    return make_plan(s, sys, cap, pe);
}

int launch(se_server s, Slot& sl, PlanEntry* pe, const se_request& rq)
{
    const se_system& sys = rq.sys;
    const int N = sys.N;
    cudaStream_t st = sl.st;
    if (rq.where == SE_WHERE_HOST) {
        SE_CUDA(cudaMemcpyAsync(pe->d_x, rq.x, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, st));
        SE_CUDA(cudaMemcpyAsync(pe->d_q, rq.q, sizeof(double) * N, cudaMemcpyHostToDevice, st));
        SE_TRY(se_solve_system(pe->plan, &sys, pe->d_x, pe->d_q, pe->d_out, nullptr, st));
        SE_CUDA(cudaMemcpyAsync(rq.out, pe->d_out, sizeof(double) * out_width(sys) * N,
                                cudaMemcpyDeviceToHost, st));
    } else {
        SE_TRY(se_solve_system(pe->plan, &sys, rq.x, rq.q, rq.out, nullptr, st));
    }
    SE_CUDA(cudaMemcpyAsync(sl.h_err, se::plan_error_flag(pe->plan), sizeof(int),
                            cudaMemcpyDeviceToHost, st));
    SE_CUDA(cudaEventRecord(sl.done, st));
    return SE_OK;
}

void complete(se_server s, long long ticket, int status, Clock::time_point t_submit,
              Clock::time_point t_admit)
{
    const Clock::time_point now = Clock::now();
    se_completion c;
    c.ticket = ticket;
    c.status = status;
    c.queue_s = seconds(t_submit, t_admit);
    c.latency_s = seconds(t_submit, now);
    std::lock_guard<std::mutex> g(s->mu);
    s->done.push_back(c);
    s->completed++;
    if (status != SE_OK) s->failed++;
    s->cv_done.notify_all();
}

void finish_slot(se_server s, Slot& sl, int status)
{
    if (status == SE_OK && *sl.h_err) status = SE_ERR_INPUT;
    sl.plan->busy = false;
    sl.plan->last_used = ++s->use_clock;
    sl.busy = false;
    sl.plan = nullptr;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->in_flight--;
    }
    complete(s, sl.ticket, status, sl.t_submit, sl.t_admit);
}

void do_reserve(se_server s, const std::vector<se_system>& req)
{
    int status = SE_OK;
    for (const se_system& sys : req) {
        bool have = false;
        const int cap = capacity_class(sys.N);
        for (PlanEntry* p : s->plans)
            have = have || (p->M == sys.M && p->P == sys.P && p->mode == sys.mode && p->cap == cap);
        if (have) continue;
        if (used_bytes(s) + plan_bytes(sys, cap, s->cfg.precision) > s->cfg.hbm_budget) {
            status = SE_ERR_NOMEM;
            continue;
        }
        PlanEntry* pe = nullptr;
        const int r = make_plan(s, sys, cap, &pe);
        if (r != SE_OK) status = r;
        else pe->last_used = ++s->use_clock;
    }
    std::lock_guard<std::mutex> g(s->mu);
    s->reserve_status = status;
    s->reserve_pending = false;
    s->cv_done.notify_all();
}

void dispatcher(se_server s)
{
    cudaSetDevice(s->device);
    for (;;) {
        bool progressed = false;
        // completions
        for (Slot& sl : s->slots) {
            if (!sl.busy) continue;
            if (sl.launch_status != SE_OK) {
                // what the failed launch did queue must end before the plan is reused
                cudaStreamSynchronize(sl.st);
                finish_slot(s, sl, sl.launch_status);
                progressed = true;
                continue;
            }
            const cudaError_t e = cudaEventQuery(sl.done);
            if (e == cudaErrorNotReady) continue;
            finish_slot(s, sl, e == cudaSuccess ? SE_OK
                                                : se::cuda_fail(e, "solve", __FILE__, __LINE__));
            progressed = true;
        }
        // plan reservations
        std::vector<se_system> reserve;
        {
            std::lock_guard<std::mutex> g(s->mu);
            if (s->reserve_pending) reserve.swap(s->reserve_req);
        }
        if (!reserve.empty()) {
            do_reserve(s, reserve);
            progressed = true;
        }
        // admissions, first come first served
        for (;;) {
            Slot* free_slot = nullptr;
            for (Slot& sl : s->slots)
                if (!sl.busy) {
                    free_slot = &sl;
                    break;
                }
            if (!free_slot) break;
            Pending head;
            {
                std::lock_guard<std::mutex> g(s->mu);
                if (s->queue.empty()) break;
                head = s->queue.front();
            }
            PlanEntry* pe = nullptr;
            const int r = acquire_plan(s, head.req.sys, &pe);
            if (r == SE_OK && !pe) break;   // memory frees when running solves end
            {
                std::lock_guard<std::mutex> g(s->mu);
                s->queue.pop_front();
                if (r == SE_OK) s->in_flight++;
            }
            const Clock::time_point t_admit = Clock::now();
            if (r != SE_OK) {
                complete(s, head.ticket, r, head.t_submit, t_admit);
                progressed = true;
                continue;
            }
            Slot& sl = *free_slot;
            sl.busy = true;
            sl.plan = pe;
            pe->busy = true;
            sl.ticket = head.ticket;
            sl.t_submit = head.t_submit;
            sl.t_admit = t_admit;
            *sl.h_err = 0;
            sl.launch_status = launch(s, sl, pe, head.req);
            progressed = true;
        }
        if (progressed) continue;
        std::unique_lock<std::mutex> lk(s->mu);
        if (s->stop && s->queue.empty() && s->in_flight == 0 && !s->reserve_pending) break;
        if (s->in_flight == 0) {
            s->cv_work.wait(lk, [&] { return s->stop || !s->queue.empty() || s->reserve_pending; });
        } else {
            lk.unlock();
            std::this_thread::sleep_for(std::chrono::microseconds(20));
        }
    }
}

bool valid_request(const se_request* r)
{
    if (!r || (r->where != SE_WHERE_HOST && r->where != SE_WHERE_DEVICE)) return false;
    const se_system& s = r->sys;
    if (s.N < 0 || s.M < 2 || s.M > 1024 || s.P < 1 || s.P > 32 || !(s.L > 0) || !(s.xi > 0) ||
        !(s.m > 0) || (s.mode != SE_POTENTIAL && s.mode != SE_FORCE))
        return false;
    return s.N == 0 || (r->x && r->q && r->out);
}

}  // namespace

extern "C" size_t se_server_request_bytes(const se_system* sys, int precision)
{
    if (!sys) return 0;
    return plan_bytes(*sys, capacity_class(sys->N), precision);
}

extern "C" int se_server_create(se_server* out, const se_server_config* cfg)
{
    if (!out || !cfg || cfg->slots < 1 || cfg->slots > MAX_SLOTS || cfg->max_queue < 0 ||
        (cfg->precision != SE_FP32 && cfg->precision != SE_FP64 &&
         cfg->precision != SE_FP32_FFT32) || cfg->hbm_budget == 0)
        return SE_ERR_INVALID;
    se_server s = new se_server_s();
    s->cfg = *cfg;
    cudaError_t e = cudaGetDevice(&s->device);
    s->slots.resize(cfg->slots);
    for (Slot& sl : s->slots) {
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&sl.st, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaMallocHost(&sl.h_err, sizeof(int));
    }
    if (e != cudaSuccess) {
        const int r = se::cuda_fail(e, "se_server_create", __FILE__, __LINE__);
        for (Slot& sl : s->slots) {
            if (sl.st) cudaStreamDestroy(sl.st);
            if (sl.done) cudaEventDestroy(sl.done);
            if (sl.h_err) cudaFreeHost(sl.h_err);
        }
        delete s;
        return r;
    }
    s->worker = std::thread(dispatcher, s);
    *out = s;
    return SE_OK;
}

extern "C" int se_server_reserve(se_server s, const se_system* systems, int n)
{
    if (!s || n < 0 || (n > 0 && !systems)) return SE_ERR_INVALID;
    std::unique_lock<std::mutex> lk(s->mu);
    s->cv_done.wait(lk, [&] { return !s->reserve_pending; });
    s->reserve_req.assign(systems, systems + n);
    s->reserve_pending = true;
    s->cv_work.notify_all();
    s->cv_done.wait(lk, [&] { return !s->reserve_pending; });
    return s->reserve_status;
}

extern "C" int se_server_submit(se_server s, const se_request* req, long long* ticket)
{
    if (!s || !valid_request(req)) return SE_ERR_INVALID;
    if (plan_bytes(req->sys, capacity_class(req->sys.N), s->cfg.precision) > s->cfg.hbm_budget)
        return SE_ERR_NOMEM;
    std::lock_guard<std::mutex> g(s->mu);
    if (s->stop) return SE_ERR_INVALID;
    if (s->cfg.max_queue > 0 && (int)s->queue.size() >= s->cfg.max_queue) return SE_ERR_BUSY;
    Pending p;
    p.ticket = s->next_ticket++;
    p.req = *req;
    p.t_submit = Clock::now();
    s->queue.push_back(p);
    s->submitted++;
    if (ticket) *ticket = p.ticket;
    s->cv_work.notify_all();
    return SE_OK;
}

extern "C" int se_server_poll(se_server s, se_completion* out, int max, int* n_done)
{
    if (!s || !n_done || max < 0 || (max > 0 && !out)) return SE_ERR_INVALID;
    std::lock_guard<std::mutex> g(s->mu);
    int n = 0;
    while (n < max && !s->done.empty()) {
        out[n++] = s->done.front();
        s->done.pop_front();
    }
    *n_done = n;
    return SE_OK;
}

extern "C" int se_server_drain(se_server s, double timeout_s)
{
    if (!s) return SE_ERR_INVALID;
    std::unique_lock<std::mutex> lk(s->mu);
    auto idle = [&] { return s->completed == s->submitted; };
    if (timeout_s < 0) {
        s->cv_done.wait(lk, idle);
        return SE_OK;
    }
    const bool ok = s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), idle);
    return ok ? SE_OK : SE_ERR_TIMEOUT;
}

extern "C" int se_server_get_stats(se_server s, se_server_stats* st)
{
    if (!s || !st) return SE_ERR_INVALID;
    std::lock_guard<std::mutex> g(s->mu);
    st->submitted = s->submitted;
    st->completed = s->completed;
    st->failed = s->failed;
    st->queued = (int)s->queue.size();
    st->in_flight = s->in_flight;
    st->plans = s->nplans;
    st->plans_created = s->plans_created;
    st->plans_evicted = s->plans_evicted;
    st->hbm_used = s->hbm_used;
    st->hbm_peak = s->hbm_peak;
    return SE_OK;
}

extern "C" int se_server_destroy(se_server s)
{
    if (!s) return SE_OK;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->stop = true;
        s->cv_work.notify_all();
    }
    s->worker.join();
    for (PlanEntry* pe : s->plans) free_plan(s, pe);
    s->plans.clear();
    for (Slot& sl : s->slots) {
        cudaStreamDestroy(sl.st);
        cudaEventDestroy(sl.done);
        cudaFreeHost(sl.h_err);
    }
    delete s;
    return SE_OK;
}
