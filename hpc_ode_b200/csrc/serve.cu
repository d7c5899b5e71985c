// serve.cu -- the request loop of include/b200ode.h (b200ode_server_*,
// b200ode_submit, b200ode_poll): continuous batching of chemistry requests on
// one GPU.
//
// Threads: callers submit and poll; one dispatcher thread owns the GPU side.
// The dispatcher
//   1. retires requests whose end event has completed (pinned staging ->
//      caller buffers, device range back to the arena, slot freed);
//   2. admits queued requests while a slot (stream) is free and the request's
//      footprint fits in the arena (first fit; FIFO with bounded backfill);
//   3. for each admitted request, chunk by chunk (at most chunk_cells cells
//      each): caller buffers -> pinned staging, one H2D copy of T|Y (+ P), the
//      persistent BDF kernel, one D2H copy of T|Y|status and the call totals,
//      an end event.  The next chunk is launched only when the previous one has
//      finished, so thread blocks of other requests take SMs in between: a
//      256k-cell request no longer holds the whole GPU until it is done, and
//      its device footprint is one chunk's.
// Device layout of a request's range, sized for one chunk of m cells (each part
// 256-byte aligned):
//   T[m] | Y[nsp*m] | status[m] | P[m] (if per-cell) | ctl[16] | per-warp scratch
// and the pinned staging buffer mirrors its first part (T|Y|status|P|totals);
// staging gathers a chunk's cells out of the caller's n-cell arrays and
// scatters the results back.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/b200ode.h"
#include "b200ode_internal.h"
#include "serve_arena.hpp"

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

size_t al(size_t b) { return b200::RangeArena::round_up(b); }

// Byte offsets of one request's parts, identical in device range and pinned staging.
struct Layout {
    size_t T = 0, Y = 0, status = 0, P = 0, ctl = 0, wg = 0, total = 0;
    size_t in_bytes = 0;    // T|Y contiguous input copy
    size_t out_bytes = 0;   // T|Y|status contiguous output copy
    Layout() = default;
    Layout(int64_t n, int nsp, bool per_cell_P, size_t wg_bytes) {
        T = 0;
        Y = al(n * sizeof(double));
        status = Y + al((size_t)n * nsp * sizeof(double));
        P = status + al(n * sizeof(int32_t));
        ctl = P + (per_cell_P ? al(n * sizeof(double)) : 0);
        wg = ctl + al(b200::kCtlWords * sizeof(unsigned long long));
        total = wg + al(wg_bytes);
        in_bytes = status;
        out_bytes = P;
    }
};

struct Request {
    uint64_t id = 0;
    b200ode_handle* h = nullptr;
    int nsp = 0;
    int64_t n = 0;
    const double* P = nullptr;
    double P_scalar = 0.0;
    double* T = nullptr;
    double* Y = nullptr;
    int32_t* status = nullptr;
    double t0 = 0.0, t1 = 0.0;
    Layout lay;              // one chunk's layout (chunk cells)
    int64_t chunk = 0;       // cells per chunk
    int64_t next_c0 = 0;     // first cell of the chunk in flight
    int64_t cur_m = 0;       // cells of the chunk in flight
    size_t offset = 0;
    int slot = -1;
    int bypassed = 0;
    bool done = false;
    b200ode_status rc = B200ODE_OK;
    std::string err;
    Clock::time_point t_submit, t_admit, t_done;
    b200ode_request_info info{};
};

struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_start = nullptr, ev_end = nullptr;
    unsigned char* pinned = nullptr;
    size_t pinned_bytes = 0;
    Request* req = nullptr;
};

double percentile(std::vector<double> v, double q) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const double pos = q * (double)(v.size() - 1);
    const size_t i = (size_t)pos;
    const double f = pos - (double)i;
    return i + 1 < v.size() ? v[i] * (1.0 - f) + v[i + 1] * f : v[i];
}

}  // namespace

struct b200ode_server {
    b200ode_server_options opt{};
    int device = 0;
    unsigned char* base = nullptr;   // device budget, reserved once
    b200::RangeArena arena;
    std::vector<Slot> slots;
    std::map<std::string, b200ode_handle*> handles;   // canonical mechanism name -> handle

    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request*> pending;
    std::map<uint64_t, std::unique_ptr<Request>> reqs;
    std::thread worker;
    bool stop = false;
    uint64_t next_id = 1;
    int inflight = 0;

    // report
    int64_t submitted = 0, completed = 0, failed = 0, cells = 0;
    std::vector<double> latencies, queue_ms;
    bool any_submit = false;
    Clock::time_point first_submit, last_done;
    int max_concurrent = 0;

    void run();
    bool admit_one(std::unique_lock<std::mutex>& lk);
    void start_request(Slot& s, Request* r);
    bool launch_chunk(Slot& s, Request* r);
    bool retire_chunk(Slot& s, Request* r);
    void finish_request(Slot& s, Request* r, cudaError_t e);
};

namespace {

std::string canonical_mech(const char* name) {
    if (!name) return std::string();
    std::string s(name);
    if (s.size() > 5 && s.substr(s.size() - 5) == ".yaml") s = s.substr(0, s.size() - 5);
    else if (s.size() > 4 && s.substr(s.size() - 4) == ".xml") s = s.substr(0, s.size() - 4);
    return s;
}

// Grows a slot's pinned staging buffer (dispatcher thread only, outside any launch).
cudaError_t ensure_pinned(Slot& s, size_t bytes) {
    if (bytes <= s.pinned_bytes) return cudaSuccess;
    if (s.pinned) cudaFreeHost(s.pinned);
    s.pinned = nullptr;
    s.pinned_bytes = 0;
    size_t cap = 1 << 20;
    while (cap < bytes) cap *= 2;
    cudaError_t e = cudaMallocHost(&s.pinned, cap);
    if (e == cudaSuccess) s.pinned_bytes = cap;
    return e;
}

// Makes the server's device current in a caller's thread and restores the
// caller's device afterwards.
struct ServerDeviceGuard {
    int prev = -1;
    explicit ServerDeviceGuard(int device) {
        if (cudaGetDevice(&prev) != cudaSuccess || prev == device) prev = -1;
        else cudaSetDevice(device);
    }
    ~ServerDeviceGuard() { if (prev >= 0) cudaSetDevice(prev); }
};

}  // namespace

// Starts a request: its first chunk.  Runs on the dispatcher thread without
// the lock: an admitted request belongs to the dispatcher until it is done.
void b200ode_server::start_request(Slot& s, Request* r) {
    r->next_c0 = 0;
    launch_chunk(s, r);   // on failure the request is already finished
}

// Stages cells [next_c0, next_c0 + m) and enqueues copies + kernel + end
// event on the slot's stream.  Returns false (the request finished with an
// error) if anything failed.
bool b200ode_server::launch_chunk(Slot& s, Request* r) {
    const Layout& L = r->lay;
    unsigned char* d = base + r->offset;
    const int64_t c0 = r->next_c0, m = std::min<int64_t>(r->chunk, r->n - c0);
    r->cur_m = m;
    auto fail_now = [&](cudaError_t e) {
        finish_request(s, r, e ? e : cudaErrorUnknown);
        return false;
    };
    cudaError_t e = ensure_pinned(s, L.ctl + b200::kCtlWords * sizeof(unsigned long long));
    if (e != cudaSuccess) return fail_now(e);
    // chunk SoA in staging (stride m), the layout the kernel sees for m cells
    std::memcpy(s.pinned + L.T, r->T + c0, m * sizeof(double));
    for (int k = 0; k < r->nsp; ++k)
        std::memcpy(s.pinned + L.Y + (size_t)k * m * sizeof(double), r->Y + (size_t)k * r->n + c0, m * sizeof(double));
    if (r->P) std::memcpy(s.pinned + L.P, r->P + c0, m * sizeof(double));
    if (c0 == 0) e = cudaEventRecord(s.ev_start, s.stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d, s.pinned, L.in_bytes, cudaMemcpyHostToDevice, s.stream);
    if (e == cudaSuccess && r->P)
        e = cudaMemcpyAsync(d + L.P, s.pinned + L.P, m * sizeof(double), cudaMemcpyHostToDevice, s.stream);
    if (e != cudaSuccess) return fail_now(e);
    auto* ctl = reinterpret_cast<unsigned long long*>(d + L.ctl);
    b200ode_status rc = b200::launch_persistent(
        r->h, m, r->P ? reinterpret_cast<const double*>(d + L.P) : nullptr, r->P_scalar,
        reinterpret_cast<double*>(d + L.T), reinterpret_cast<double*>(d + L.Y),
        reinterpret_cast<int32_t*>(d + L.status), r->t0, r->t1, ctl, d + L.wg, s.stream);
    if (rc != B200ODE_OK) {
        r->rc = rc;
        r->err = b200ode_last_error();
        finish_request(s, r, cudaSuccess);
        return false;
    }
    e = cudaMemcpyAsync(s.pinned, d, L.out_bytes, cudaMemcpyDeviceToHost, s.stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(s.pinned + L.ctl, ctl, b200::kCtlWords * sizeof(unsigned long long),
                            cudaMemcpyDeviceToHost, s.stream);
    if (e == cudaSuccess) e = cudaEventRecord(s.ev_end, s.stream);
    if (e != cudaSuccess) return fail_now(e);
    return true;
}

// The chunk in flight has finished: results to the caller's buffers, totals
// accumulated; launches the next chunk.  Returns true when the request is
// complete.
bool b200ode_server::retire_chunk(Slot& s, Request* r) {
    const Layout& L = r->lay;
    const int64_t c0 = r->next_c0, m = r->cur_m;
    std::memcpy(r->T + c0, s.pinned + L.T, m * sizeof(double));
    for (int k = 0; k < r->nsp; ++k)
        std::memcpy(r->Y + (size_t)k * r->n + c0, s.pinned + L.Y + (size_t)k * m * sizeof(double), m * sizeof(double));
    if (r->status) std::memcpy(r->status + c0, s.pinned + L.status, m * sizeof(int32_t));
    const auto* tot = reinterpret_cast<const unsigned long long*>(s.pinned + L.ctl) + 1;
    r->info.total_nst += (int64_t)tot[0];
    r->info.total_nni += (int64_t)tot[4];
    r->info.n_failed += (int64_t)tot[7];
    r->next_c0 = c0 + m;
    if (r->next_c0 >= r->n) return true;
    launch_chunk(s, r);   // on failure the request is already finished
    return false;
}

// Completes a request: results to the caller (when the GPU side succeeded),
// device range back to the arena, slot freed, pollers woken.
void b200ode_server::finish_request(Slot& s, Request* r, cudaError_t e) {
    // nothing of a failed request may still be in flight when its range is reused
    if (e != cudaSuccess || r->rc != B200ODE_OK) cudaStreamSynchronize(s.stream);
    if (e != cudaSuccess) {
        r->rc = B200ODE_ERR_CUDA;
        r->err = std::string("request ") + std::to_string(r->id) + ": " + cudaGetErrorString(e);
    }
    if (r->rc == B200ODE_OK) {
        float ms = 0.f;   // first chunk's start to last chunk's end
        if (cudaEventElapsedTime(&ms, s.ev_start, s.ev_end) == cudaSuccess) r->info.device_ms = ms;
    }
    const Clock::time_point now = Clock::now();
    std::lock_guard<std::mutex> lk(mu);
    arena.release(r->offset, r->lay.total);
    s.req = nullptr;
    --inflight;
    r->t_done = now;
    r->info.n_cells = r->n;
    r->info.footprint_bytes = (int64_t)r->lay.total;
    r->info.queue_ms = ms_between(r->t_submit, r->t_admit);
    r->info.latency_ms = ms_between(r->t_submit, now);
    r->done = true;
    ++completed;
    if (r->rc != B200ODE_OK) ++failed;
    else cells += r->n;
    latencies.push_back(r->info.latency_ms);
    queue_ms.push_back(r->info.queue_ms);
    last_done = now;
    cv_done.notify_all();
}

// Admits the first queued request that fits (FIFO; later requests may pass a
// head that does not fit at most 8 times).  Called with the lock held; drops it
// while the request is started.
bool b200ode_server::admit_one(std::unique_lock<std::mutex>& lk) {
    int slot = -1;
    for (size_t i = 0; i < slots.size(); ++i)
        if (!slots[i].req) { slot = (int)i; break; }
    if (slot < 0 || pending.empty()) return false;
    Request* head = pending.front();
    size_t off = 0;
    Request* pick = nullptr;
    auto pos = pending.begin();
    if (arena.alloc(head->lay.total, &off)) {
        pick = head;
    } else if (head->bypassed < 8) {
        for (auto it = std::next(pending.begin()); it != pending.end(); ++it)
            if (arena.alloc((*it)->lay.total, &off)) { pick = *it; pos = it; break; }
        if (pick) ++head->bypassed;
    }
    if (!pick) return false;
    pending.erase(pos);
    pick->offset = off;
    pick->slot = slot;
    pick->t_admit = Clock::now();
    Slot& s = slots[slot];
    s.req = pick;
    ++inflight;
    max_concurrent = std::max(max_concurrent, inflight);
    lk.unlock();
    start_request(s, pick);
    lk.lock();
    return true;
}

void b200ode_server::run() {
    cudaSetDevice(device);
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
        // 1. retire
        std::vector<std::pair<Slot*, cudaError_t>> finished;
        for (Slot& s : slots) {
            if (!s.req || s.req->done) continue;
            const cudaError_t q = cudaEventQuery(s.ev_end);
            if (q == cudaErrorNotReady) continue;
            finished.emplace_back(&s, q);
        }
        if (!finished.empty()) {
            lk.unlock();
            for (auto& f : finished) {
                Request* r = f.first->req;
                if (f.second != cudaSuccess) finish_request(*f.first, r, f.second);
                else if (retire_chunk(*f.first, r)) finish_request(*f.first, r, cudaSuccess);
            }
            lk.lock();
        }
        // 2. admit
        while (admit_one(lk)) {
        }
        // 3. wait
        if (stop && inflight == 0) break;
        if (inflight == 0 && pending.empty()) {
            cv_work.wait(lk, [&] { return stop || !pending.empty(); });
        } else {
            lk.unlock();
            std::this_thread::sleep_for(std::chrono::microseconds(50));
            lk.lock();
        }
    }
}

extern "C" {

void b200ode_default_server_options(b200ode_server_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    b200ode_default_options(&o->solver);
    o->hbm_budget_bytes = 0;
    o->max_inflight = 4;
    o->max_queued = 4096;
    o->chunk_cells = 32768;
}

b200ode_status b200ode_server_create(const b200ode_server_options* opts, b200ode_server** out) {
    if (!out) return b200::set_error(B200ODE_ERR_INVALID, "null output pointer");
    *out = nullptr;
    b200ode_server_options o;
    b200ode_default_server_options(&o);
    if (opts) o = *opts;
    if (o.max_inflight <= 0) o.max_inflight = 4;
    if (o.max_queued <= 0) o.max_queued = 4096;
    if (o.chunk_cells <= 0) o.chunk_cells = 32768;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return b200::set_error(B200ODE_ERR_NO_DEVICE, "no CUDA device available");
    }
    auto srv = std::make_unique<b200ode_server>();
    srv->opt = o;
    if (o.solver.device >= 0 && cudaSetDevice(o.solver.device) != cudaSuccess)
        return b200::set_error(B200ODE_ERR_CUDA, "cudaSetDevice failed");
    cudaGetDevice(&srv->device);
    srv->opt.solver.device = srv->device;
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess)
        return b200::set_error(B200ODE_ERR_CUDA, "cudaMemGetInfo failed");
    size_t budget = o.hbm_budget_bytes > 0 ? (size_t)o.hbm_budget_bytes : free_b / 4;
    budget = budget / b200::RangeArena::kAlign * b200::RangeArena::kAlign;
    if (budget == 0 || budget > free_b)
        return b200::set_error(B200ODE_ERR_ALLOC, "server budget of " + std::to_string(budget) +
                                                      " bytes does not fit in free device memory (" +
                                                      std::to_string(free_b) + ")");
    if (cudaMalloc(&srv->base, budget) != cudaSuccess)
        return b200::set_error(B200ODE_ERR_ALLOC, "cudaMalloc of the server budget failed");
    srv->arena.reset(budget);
    srv->slots.resize(o.max_inflight);
    for (Slot& s : srv->slots) {
        if (cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreate(&s.ev_start) != cudaSuccess || cudaEventCreate(&s.ev_end) != cudaSuccess) {
            b200ode_server_destroy(srv.release());
            return b200::set_error(B200ODE_ERR_CUDA, "stream/event creation failed");
        }
    }
    b200ode_server* raw = srv.release();
    raw->worker = std::thread([raw] { raw->run(); });
    *out = raw;
    return B200ODE_OK;
}

void b200ode_server_destroy(b200ode_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->pending.clear();
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    for (Slot& sl : s->slots) {
        if (sl.stream) cudaStreamSynchronize(sl.stream);
        if (sl.pinned) cudaFreeHost(sl.pinned);
        if (sl.ev_start) cudaEventDestroy(sl.ev_start);
        if (sl.ev_end) cudaEventDestroy(sl.ev_end);
        if (sl.stream) cudaStreamDestroy(sl.stream);
    }
    if (s->base) cudaFree(s->base);
    for (auto& kv : s->handles) b200ode_destroy(kv.second);
    delete s;
}

b200ode_status b200ode_submit(b200ode_server* s, const char* mech_name, int64_t n, const double* P,
                              double Ps, double* T, double* Y, double t0, double t1, int32_t* cell_status,
                              uint64_t* request_id) {
    if (!s || !request_id) return b200::set_error(B200ODE_ERR_INVALID, "null server or request id");
    if (n < 0) return b200::set_error(B200ODE_ERR_INVALID, "n_cells < 0");
    if (n > 0 && (!T || !Y)) return b200::set_error(B200ODE_ERR_INVALID, "null T or Y");
    if (n > 0 && !P && !(Ps > 0.0)) return b200::set_error(B200ODE_ERR_INVALID, "pressure must be > 0");
    if (!(t0 == t0) || !(t1 == t1)) return b200::set_error(B200ODE_ERR_INVALID, "t0/t1 not finite");
    const std::string mech = canonical_mech(mech_name);
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->stop) return b200::set_error(B200ODE_ERR_INVALID, "server is shutting down");
    if ((int64_t)s->pending.size() >= s->opt.max_queued)
        return b200::set_error(B200ODE_ERR_BUSY, "request queue full (" + std::to_string(s->opt.max_queued) + ")");
    ServerDeviceGuard guard(s->device);
    auto it = s->handles.find(mech);
    if (it == s->handles.end()) {
        b200ode_handle* h = nullptr;
        const b200ode_status rc = b200ode_create(mech_name, &s->opt.solver, &h);
        if (rc != B200ODE_OK) return rc;
        it = s->handles.emplace(mech, h).first;
    }
    b200ode_handle* h = it->second;
    const int nsp = b200ode_num_species(h);
    Layout lay;
    int64_t chunk = 0;
    if (n > 0) {
        chunk = std::min<int64_t>(n, s->opt.chunk_cells);
        const size_t wg = b200::persistent_scratch_bytes(h, chunk);
        if (wg == 0) return B200ODE_ERR_CUDA;
        lay = Layout(chunk, nsp, P != nullptr, wg);
        if (lay.total > s->arena.capacity())
            return b200::set_error(B200ODE_ERR_INVALID, "request of " + std::to_string(n) + " cells needs " +
                                                            std::to_string(lay.total) +
                                                            " device bytes; the server budget is " +
                                                            std::to_string(s->arena.capacity()));
    }
    auto r = std::make_unique<Request>();
    r->lay = lay;
    r->chunk = chunk;
    r->id = s->next_id++;
    r->h = h;
    r->nsp = nsp;
    r->n = n;
    r->P = P;
    r->P_scalar = Ps;
    r->T = T;
    r->Y = Y;
    r->status = cell_status;
    r->t0 = t0;
    r->t1 = t1;
    r->t_submit = Clock::now();
    if (!s->any_submit) {
        s->any_submit = true;
        s->first_submit = r->t_submit;
    }
    ++s->submitted;
    *request_id = r->id;
    if (n == 0) {   // nothing to do on the GPU
        r->done = true;
        r->t_admit = r->t_done = r->t_submit;
        ++s->completed;
        s->reqs.emplace(r->id, std::move(r));
        s->cv_done.notify_all();
        return B200ODE_OK;
    }
    s->pending.push_back(r.get());
    s->reqs.emplace(r->id, std::move(r));
    lk.unlock();
    s->cv_work.notify_all();
    return B200ODE_OK;
}

b200ode_status b200ode_poll(b200ode_server* s, uint64_t id, int32_t wait_ms, b200ode_request_info* info) {
    if (!s) return b200::set_error(B200ODE_ERR_INVALID, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end())
        return b200::set_error(B200ODE_ERR_INVALID, "unknown or already retired request " + std::to_string(id));
    Request* r = it->second.get();
    if (!r->done && wait_ms != 0) {
        auto pred = [&] { return r->done; };
        if (wait_ms < 0) s->cv_done.wait(lk, pred);
        else s->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), pred);
    }
    if (!r->done) return B200ODE_ERR_NOT_READY;
    if (info) *info = r->info;
    const b200ode_status rc = r->rc;
    const std::string err = r->err;
    s->reqs.erase(it);
    if (rc != B200ODE_OK) return b200::set_error(rc, err);
    return B200ODE_OK;
}

b200ode_status b200ode_server_get_report(b200ode_server* s, b200ode_server_report* rep) {
    if (!s || !rep) return b200::set_error(B200ODE_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    std::memset(rep, 0, sizeof(*rep));
    rep->submitted = s->submitted;
    rep->completed = s->completed;
    rep->failed_requests = s->failed;
    rep->cells_completed = s->cells;
    rep->p50_latency_ms = percentile(s->latencies, 0.50);
    rep->p99_latency_ms = percentile(s->latencies, 0.99);
    rep->max_latency_ms = s->latencies.empty() ? 0.0 : *std::max_element(s->latencies.begin(), s->latencies.end());
    double q = 0.0;
    for (double v : s->queue_ms) q += v;
    rep->mean_queue_ms = s->queue_ms.empty() ? 0.0 : q / (double)s->queue_ms.size();
    const double span = (s->any_submit && s->completed) ? ms_between(s->first_submit, s->last_done) : 0.0;
    rep->cells_per_sec = span > 0.0 ? (double)s->cells / (span * 1e-3) : 0.0;
    rep->max_concurrent = s->max_concurrent;
    rep->budget_bytes = (int64_t)s->arena.capacity();
    rep->peak_bytes = (int64_t)s->arena.peak();
    return B200ODE_OK;
}

}  // extern "C"
