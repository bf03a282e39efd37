// Request server: single solves arriving over time, continuously batched on
// one GPU.
//
// The reference has no serving path (one solve per process run,
// src/main.cpp:73-134).  Here a dispatcher thread admits queued requests in
// arrival order while a stream slot is free and the request's workspace fits
// the HBM budget; handles (plans, twiddles, workspaces) are pooled per shape
// and stay resident between requests, idle ones are evicted least recently
// used when a new shape needs room.  Each admitted request runs H2D -> solve
// -> D2H asynchronously on its slot's stream, so requests that arrive while
// others are on the GPU overlap with them; a host function enqueued after the
// D2H copy marks completion, and latency is measured from submit to that
// point.  Host buffers should be page-locked (pp_host_alloc) for the copies to
// overlap.
//
// The host function takes no lock: the dispatcher holds the server mutex
// across CUDA calls that may wait for the device (cudaFree inside a handle's
// buffer resize, for one), and a host function blocked on that mutex would
// keep the device from ever going idle.  It stores the completion time and an
// atomic flag and wakes the dispatcher.
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "../../include/pittpack_b200.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Req {
    unsigned long long ticket;
    pp_request r;
    Clock::time_point t_submit;
};

struct Result {
    bool done = false;
    int status = PP_SUCCESS;
    int precision = 0;
    double latency_ms = 0.0;
};

using ShapeKey = std::tuple<int, int, int, std::string>;

struct PooledHandle {
    pp_handle h;
    ShapeKey key;
    size_t bytes;
    Clock::time_point last_use;
};

struct Slot {
    cudaStream_t stream = nullptr;
    bool busy = false;
    unsigned long long ticket = 0;
    PooledHandle* ph = nullptr;
    int precision = 0;
    Clock::time_point t_submit;
    int status = PP_SUCCESS;       // PP_CUDA_ERROR when the completion could not be awaited
    Clock::time_point t_done;      // written by the host function
    std::atomic<int> finished{0};  // set by the host function after t_done
    struct pp_server_s* server = nullptr;
};

}  // namespace

struct pp_server_s {
    int device = 0;
    size_t budget = 0, pool_bytes = 0;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<Req> pending;
    std::map<unsigned long long, Result> results;
    std::list<PooledHandle> pool;  // every handle the server owns
    std::vector<std::unique_ptr<Slot>> slots;
    unsigned long long next_ticket = 1;
    bool stop = false;
    std::thread worker;
    long long n_done = 0;
    int max_inflight = 0;
    long long n_created = 0, n_evicted = 0;  // pooled handles made / freed
};

namespace {

// enqueued on the slot's stream after the D2H copy
void CUDART_CB on_complete(void* p)
{
    Slot* s = static_cast<Slot*>(p);
    s->t_done = Clock::now();
    s->finished.store(1, std::memory_order_release);
    s->server->cv.notify_all();
}

bool handle_busy(const pp_server_s* S, const PooledHandle* ph)
{
    for (const auto& sl : S->slots)
        if (sl->busy && sl->ph == ph) return true;
    return false;
}

// an idle pooled handle for the shape, or a new one if it fits the budget
// (evicting idle handles of other shapes, least recently used first);
// null with *rc == PP_SUCCESS: wait for completions.  A second handle of a
// shape that already has one (busy) is made only when it fits without
// evicting: an eviction frees device memory, which waits for the whole
// device, so waiting for the shape's own handle is the cheaper stall.
PooledHandle* acquire(pp_server_s* S, const pp_request& r, const ShapeKey& key, int* rc)
{
    *rc = PP_SUCCESS;
    bool have_shape = false;
    for (auto& ph : S->pool) {
        if (ph.key != key) continue;
        if (!handle_busy(S, &ph)) return &ph;
        have_shape = true;
    }
    // a handle holds four 2-complex-per-point buffers plus tables
    const size_t need = (size_t)r.nx * r.ny * r.nz * 8 * sizeof(double) + (1u << 20);
    if (have_shape && S->pool_bytes + need > S->budget) return nullptr;
    while (S->pool_bytes + need > S->budget) {
        auto victim = S->pool.end();
        for (auto it = S->pool.begin(); it != S->pool.end(); ++it) {
            if (handle_busy(S, &*it)) continue;
            if (victim == S->pool.end() || it->last_use < victim->last_use) victim = it;
        }
        if (victim == S->pool.end()) {
            // nothing to evict: wait, unless nothing is running (never fits)
            bool any = false;
            for (const auto& sl : S->slots) any |= sl->busy;
            if (!any) *rc = PP_ALLOCATION_FAIL;
            return nullptr;
        }
        S->pool_bytes -= victim->bytes;
        pp_destroy(victim->h);
        S->pool.erase(victim);
        S->n_evicted++;
    }
    pp_handle h = nullptr;
    if ((*rc = pp_create(r.nx, r.ny, r.nz, &h)) != PP_SUCCESS) return nullptr;
    if ((*rc = pp_set_box(h, r.box)) != PP_SUCCESS || (*rc = pp_assign_boundary(h, r.bc)) != PP_SUCCESS) {
        pp_destroy(h);
        return nullptr;
    }
    size_t bytes = 0;
    pp_workspace_bytes(h, &bytes);
    S->pool.push_back(PooledHandle{h, key, bytes, Clock::now()});
    S->pool_bytes += bytes;
    S->n_created++;
    return &S->pool.back();
}

void retire(pp_server_s* S, Slot& s)
{
    Result& res = S->results[s.ticket];
    res.done = true;
    res.status = s.status;
    res.precision = s.precision;
    res.latency_ms = std::chrono::duration<double, std::milli>(s.t_done - s.t_submit).count();
    s.finished.store(0, std::memory_order_relaxed);
    s.ph->last_use = Clock::now();
    s.busy = false;
    s.ph = nullptr;
    S->n_done++;
}

void fail(pp_server_s* S, unsigned long long ticket, int rc)
{
    Result& res = S->results[ticket];
    res.done = true;
    res.status = rc;
    S->cv.notify_all();
}

// start a request on a free slot; false if it cannot be admitted now
bool admit(pp_server_s* S, const Req& q)
{
    Slot* slot = nullptr;
    for (auto& sl : S->slots)
        if (!sl->busy) {
            slot = sl.get();
            break;
        }
    if (!slot) return false;
    const pp_request& r = q.r;
    const ShapeKey key(r.nx, r.ny, r.nz, std::string(r.bc, 6));
    int rc = PP_SUCCESS;
    PooledHandle* ph = acquire(S, r, key, &rc);
    if (!ph) {
        if (rc == PP_SUCCESS) return false;  // memory: wait for completions
        fail(S, q.ticket, rc);
        return true;
    }
    Slot& s = *slot;
    const int prec = r.precision == PP_PRECISION_MIXED ? PP_PRECISION_MIXED : PP_PRECISION_FP64;
    pp_options o;
    pp_default_options(&o);
    o.precision = prec;
    o.max_sweeps = r.sweeps;
    o.compat_zero_mode = prec == PP_PRECISION_MIXED ? 0 : 1;
    pp_handle h = ph->h;
    rc = pp_set_options(h, &o);
    if (rc == PP_SUCCESS) rc = pp_set_stream(h, s.stream);
    if (rc == PP_SUCCESS) rc = pp_assign_rhs_async(h, r.rhs);
    if (rc == PP_SUCCESS) rc = pp_solve(h);
    if (rc == PP_SUCCESS) rc = r.output_real ? pp_get_solution_real_async(h, r.P) : pp_get_solution_async(h, r.P);
    if (rc != PP_SUCCESS) {
        fail(S, q.ticket, rc);
        return true;
    }
    s.busy = true;
    s.ticket = q.ticket;
    s.ph = ph;
    s.precision = prec;
    s.t_submit = q.t_submit;
    s.status = PP_SUCCESS;
    if (cudaLaunchHostFunc(s.stream, on_complete, &s) != cudaSuccess) {
        // no completion callback: wait here, and fail the request if even that fails
        if (cudaStreamSynchronize(s.stream) != cudaSuccess) s.status = PP_CUDA_ERROR;
        s.t_done = Clock::now();
        s.finished.store(1, std::memory_order_release);
    }
    int inflight = 0;
    for (auto& x : S->slots) inflight += x->busy;
    if (inflight > S->max_inflight) S->max_inflight = inflight;
    return true;
}

void run(pp_server_s* S)
{
    cudaSetDevice(S->device);
    std::unique_lock<std::mutex> lk(S->mu);
    for (;;) {
        bool retired = false;
        for (auto& sl : S->slots)
            if (sl->busy && sl->finished.load(std::memory_order_acquire)) {
                retire(S, *sl);
                retired = true;
            }
        if (retired) S->cv.notify_all();
        // admit in arrival order while slots and memory allow
        while (!S->pending.empty() && admit(S, S->pending.front())) S->pending.pop_front();
        if (S->stop) {
            bool busy = false;
            for (auto& s : S->slots) busy |= s->busy;
            if (!busy && S->pending.empty()) break;
        }
        // a wake-up from a host function can slip in between the scan above and
        // this wait (it takes no lock); the short bound keeps that cheap
        S->cv.wait_for(lk, std::chrono::microseconds(500));
    }
}

}  // namespace

extern "C" int pp_server_create(int streams, double hbm_fraction, pp_server* out)
{
    if (!out || streams < 1 || streams > 64 || !(hbm_fraction > 0.0) || hbm_fraction > 0.95) return PP_INPUT_ARGS;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return PP_GPU_INIT_FAILURE;
    pp_server_s* S = new (std::nothrow) pp_server_s;
    if (!S) return PP_ALLOCATION_FAIL;
    cudaGetDevice(&S->device);
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    S->budget = (size_t)(hbm_fraction * (double)fr);
    for (int i = 0; i < streams; ++i) {
        S->slots.emplace_back(new Slot);
        S->slots[i]->server = S;
        if (cudaStreamCreateWithFlags(&S->slots[i]->stream, cudaStreamNonBlocking) != cudaSuccess) {
            for (int k = 0; k < i; ++k) cudaStreamDestroy(S->slots[k]->stream);
            delete S;
            return PP_CUDA_ERROR;
        }
    }
    S->worker = std::thread(run, S);
    *out = S;
    return PP_SUCCESS;
}

extern "C" int pp_server_submit(pp_server S, const pp_request* r, unsigned long long* ticket)
{
    if (!S) return PP_INVALID_HANDLE;
    if (!r || !ticket || !r->rhs || !r->P || r->nx < 2 || r->ny < 2 || r->nz < 3) return PP_INPUT_ARGS;
    if (r->sweeps < 0 || r->sweeps > 16 || (r->output_real != 0 && r->output_real != 1)) return PP_INPUT_ARGS;
    std::lock_guard<std::mutex> g(S->mu);
    if (S->stop) return PP_NOT_READY;
    const unsigned long long t = S->next_ticket++;
    S->pending.push_back(Req{t, *r, Clock::now()});
    S->results[t] = Result{};
    *ticket = t;
    S->cv.notify_all();
    return PP_SUCCESS;
}

extern "C" int pp_server_wait(pp_server S, unsigned long long ticket, double* latency_ms, int* precision)
{
    if (!S) return PP_INVALID_HANDLE;
    std::unique_lock<std::mutex> lk(S->mu);
    if (S->results.find(ticket) == S->results.end()) return PP_INPUT_ARGS;
    // a ticket is collected once: a second waiter on it (another thread) sees
    // its entry vanish and returns PP_INPUT_ARGS instead of waiting for good
    auto it = S->results.end();
    S->cv.wait(lk, [&] {
        it = S->results.find(ticket);
        return it == S->results.end() || it->second.done;
    });
    if (it == S->results.end()) return PP_INPUT_ARGS;
    const Result res = it->second;
    S->results.erase(it);
    if (latency_ms) *latency_ms = res.latency_ms;
    if (precision) *precision = res.precision;
    return res.status;
}

extern "C" int pp_server_stats(pp_server S, long long* completed, int* max_inflight, size_t* pool_bytes)
{
    if (!S) return PP_INVALID_HANDLE;
    std::lock_guard<std::mutex> g(S->mu);
    if (completed) *completed = S->n_done;
    if (max_inflight) *max_inflight = S->max_inflight;
    if (pool_bytes) *pool_bytes = S->pool_bytes;
    return PP_SUCCESS;
}

extern "C" int pp_server_pool_stats(pp_server S, long long* created, long long* evicted)
{
    if (!S) return PP_INVALID_HANDLE;
    std::lock_guard<std::mutex> g(S->mu);
    if (created) *created = S->n_created;
    if (evicted) *evicted = S->n_evicted;
    return PP_SUCCESS;
}

extern "C" int pp_server_destroy(pp_server S)
{
    if (!S) return PP_INVALID_HANDLE;
    {
        std::lock_guard<std::mutex> g(S->mu);
        S->stop = true;
        S->cv.notify_all();
    }
    S->worker.join();
    cudaSetDevice(S->device);
    // returns after each host function has run to its end
    for (auto& s : S->slots) cudaStreamSynchronize(s->stream);
    // the handles still name the slot streams: release them first
    for (auto& ph : S->pool) pp_destroy(ph.h);
    for (auto& s : S->slots) cudaStreamDestroy(s->stream);
    delete S;
    return PP_SUCCESS;
}
