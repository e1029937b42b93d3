// Serving loop of librcabf (rcabf_server_*): continuous batching of
// beamforming requests on one device.
//
// * Requests reference caller-owned device buffers (channel data, output,
//   mask) and a geometry handle; their workspace comes from an arena that the
//   server allocates once (the HBM budget).  A request whose workspace is
//   larger than the whole budget is refused at submit (RCABF_ERR_OOM_ADMISSION);
//   one that does not fit the free part waits until earlier requests release
//   theirs.
// * A scheduler thread admits queued requests in arrival order as launch
//   slots (streams) and arena space free up.  Requests whose launch plans
//   share one kernel variant (same table mode, interpolation, storage, frame
//   block and voxel blocking) are fused into one persistent launch
//   (rcabf_beamform_batch), so requests that arrive while others run are
//   picked up by the next launch and their work overlaps on the device.
// * Completion is signalled by a host function enqueued behind each launch;
//   it releases the workspace and the slot and records the request's latency
//   (submit to completion, host clock).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <set>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/rcabf.h"
#include "geometry.h"
#include "launchers.h"
#include "plan.h"

using Clock = std::chrono::steady_clock;

namespace rcabf {

struct DeviceState;
DeviceState *device_state(int dev, bool with_err);   // api.cpp

// First-fit allocator over one device allocation (offsets, 256-byte aligned).
class Arena {
public:
    void reset(size_t bytes)
    {
        free_.clear();
        if (bytes) free_[0] = bytes;
        size_ = bytes;
        used_ = peak_ = 0;
    }
    bool alloc(size_t bytes, size_t &off)
    {
        bytes = round(bytes);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < bytes) continue;
            off = it->first;
            const size_t rest = it->second - bytes;
            free_.erase(it);
            if (rest) free_[off + bytes] = rest;
            used_ += bytes;
            peak_ = std::max(peak_, used_);
            return true;
        }
        return false;
    }
    void release(size_t off, size_t bytes)
    {
        bytes = round(bytes);
        used_ -= bytes;
        auto it = free_.emplace(off, bytes).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
    size_t size() const { return size_; }
    size_t used() const { return used_; }
    size_t peak() const { return peak_; }
    static size_t round(size_t b) { return (std::max<size_t>(b, 1) + 255) / 256 * 256; }

private:
    std::map<size_t, size_t> free_;
    size_t size_ = 0, used_ = 0, peak_ = 0;
};

struct Request {
    uint64_t ticket = 0;
    rcabf_geometry *g = nullptr;
    rcabf_beamform_args a{};
    Plan plan;
    size_t ws_off = 0, ws_bytes = 0;
    double units = 0.0;
    Clock::time_point t_submit;
    int status = RCABF_ERR_PENDING;
    bool done = false;
    bool batchable = false;   // runs as one job of a fused multi-request launch
};

struct Launch;

}  // namespace rcabf

struct rcabf_server {
    rcabf_server_config cfg{};
    void *arena_base = nullptr;
    rcabf::Arena arena;
    std::vector<cudaStream_t> streams;
    std::vector<int> slot_busy;

    std::mutex mu;
    std::condition_variable cv;           // scheduler: new work or a completion
    std::condition_variable cv_done;      // waiters: a completion
    std::deque<rcabf::Request *> queue;
    std::map<uint64_t, rcabf::Request *> all;
    // outputs (and masks) of launches in flight: a request writing one of
    // them waits, so accumulating requests apply in arrival order
    std::multiset<const void *> busy_out;
    uint64_t next_ticket = 1;
    bool stop = false;
    std::thread thread;

    // statistics
    int64_t submitted = 0, completed = 0, rejected = 0, launches = 0, in_flight = 0;
    std::vector<double> latency_ms;
    double units_done = 0.0;
    double busy_s = 0.0;
    Clock::time_point busy_since;
    Clock::time_point first_submit, last_done;
    bool any_submit = false;
};

namespace rcabf {

struct Launch {
    rcabf_server *srv;
    int slot;
    std::vector<Request *> reqs;
};

// Requests fused into one launch must run one kernel variant.
static bool same_variant(const Request *a, const Request *b)
{
    return a->batchable && b->batchable && a->g->device == b->g->device && a->g->mode == b->g->mode && a->g->kind == b->g->kind &&
           a->a.storage == b->a.storage && a->plan.kernel == RCABF_KERNEL_FUSED &&
           b->plan.kernel == RCABF_KERNEL_FUSED && a->plan.fb == b->plan.fb && a->plan.vb == b->plan.vb &&
           a->plan.d == b->plan.d && a->plan.tc == b->plan.tc;
}

static void finish_locked(rcabf_server *s, Request *r, int status, Clock::time_point now)
{
    r->status = status;
    r->done = true;
    if (r->ws_bytes) s->arena.release(r->ws_off, r->ws_bytes);
    r->ws_bytes = 0;
    s->completed += 1;
    if (status == RCABF_OK) {
        s->latency_ms.push_back(std::chrono::duration<double, std::milli>(now - r->t_submit).count());
        s->units_done += r->units;
    }
    s->last_done = now;
}

// Host function run by CUDA when a launch's stream reaches it: no CUDA calls here.
static void CUDART_CB on_launch_done(void *p)
{
    Launch *L = static_cast<Launch *>(p);
    rcabf_server *s = L->srv;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        const auto now = Clock::now();
        for (Request *r : L->reqs) {
            finish_locked(s, r, RCABF_OK, now);
            s->busy_out.erase(s->busy_out.find(r->a.out));
            if (r->a.mask) s->busy_out.erase(s->busy_out.find(r->a.mask));
        }
        s->slot_busy[L->slot] = 0;
        s->in_flight -= 1;
        if (s->in_flight == 0) s->busy_s += std::chrono::duration<double>(now - s->busy_since).count();
    }
    s->cv.notify_all();
    s->cv_done.notify_all();
    delete L;
}

// Admits queued requests while a slot and arena space are free; returns
// whether anything was launched.  Called with the lock held.
static bool dispatch_locked(rcabf_server *s)
{
    bool any = false;
    while (!s->queue.empty()) {
        int slot = -1;
        for (int i = 0; i < (int)s->slot_busy.size(); ++i)
            if (!s->slot_busy[i]) { slot = i; break; }
        if (slot < 0) break;
        // a request may start when no launch in flight and no earlier queued
        // request writes its output or mask (requests that accumulate into one
        // buffer apply in arrival order)
        auto conflicts = [&](const Request *r, const std::vector<Request *> &before) {
            if (s->busy_out.count(r->a.out) || (r->a.mask && s->busy_out.count(r->a.mask))) return true;
            for (const Request *o : before)
                if (o->a.out == r->a.out || (r->a.mask && o->a.mask == r->a.mask)) return true;
            return false;
        };
        std::vector<Request *> before;
        auto hit = s->queue.begin();
        for (; hit != s->queue.end(); ++hit) {
            if (!conflicts(*hit, before)) break;
            before.push_back(*hit);
        }
        if (hit == s->queue.end()) break;
        Request *head = *hit;
        if (!s->arena.alloc(head->ws_bytes ? head->ws_bytes : 1, head->ws_off)) break;   // wait for space
        Launch *L = new Launch{s, slot, {head}};
        s->queue.erase(hit);
        // fuse later arrivals that run the same kernel variant and fit
        if (head->plan.kernel == RCABF_KERNEL_FUSED) {
            before.push_back(head);
            for (auto it = s->queue.begin(); it != s->queue.end() && (int)L->reqs.size() < s->cfg.max_batch;) {
                Request *r = *it;
                size_t off = 0;
                if (same_variant(head, r) && !conflicts(r, before) &&
                    s->arena.alloc(r->ws_bytes ? r->ws_bytes : 1, off)) {
                    r->ws_off = off;
                    L->reqs.push_back(r);
                    before.push_back(r);
                    it = s->queue.erase(it);
                } else {
                    before.push_back(r);
                    ++it;
                }
            }
        }
        for (Request *r : L->reqs) {
            if (!r->ws_bytes) r->ws_bytes = 1;   // the arena block reserved above
            r->a.workspace = static_cast<char *>(s->arena_base) + r->ws_off;
            r->a.workspace_bytes = Arena::round(r->ws_bytes);
            r->a.stage_events = nullptr;
        }
        cudaStream_t st = s->streams[slot];
        int status;
        if (L->reqs.size() == 1) {
            status = rcabf_beamform(L->reqs[0]->g, &L->reqs[0]->a, st);
        } else {
            std::vector<const rcabf_geometry *> gs;
            std::vector<rcabf_beamform_args> as;
            for (Request *r : L->reqs) {
                gs.push_back(r->g);
                as.push_back(r->a);
            }
            status = rcabf_beamform_batch((int)gs.size(), gs.data(), as.data(), st);
        }
        if (status == RCABF_OK) status = cudaLaunchHostFunc(st, on_launch_done, L) == cudaSuccess ? RCABF_OK
                                                                                                  : RCABF_ERR_CUDA;
        if (status != RCABF_OK) {
            // part of the launch may have been enqueued: let it drain before
            // the workspace goes back to the arena
            cudaStreamSynchronize(st);
            cudaGetLastError();
            const auto now = Clock::now();
            for (Request *r : L->reqs) finish_locked(s, r, status, now);
            delete L;
            s->cv_done.notify_all();
            continue;
        }
        for (Request *r : L->reqs) {
            s->busy_out.insert(r->a.out);
            if (r->a.mask) s->busy_out.insert(r->a.mask);
        }
        if (s->in_flight == 0) s->busy_since = Clock::now();
        s->in_flight += 1;
        s->launches += 1;
        s->slot_busy[slot] = 1;
        any = true;
    }
    return any;
}

static void scheduler(rcabf_server *s)
{
    cudaSetDevice(s->cfg.device);
    std::unique_lock<std::mutex> lk(s->mu);
    while (true) {
        if (s->stop && s->queue.empty() && s->in_flight == 0) break;
        // a short batching window lets requests arriving together share a launch
        if (s->cfg.batch_window_us > 0 && !s->queue.empty() && s->in_flight == 0) {
            const auto t0 = s->queue.front()->t_submit;
            const auto until = t0 + std::chrono::microseconds(s->cfg.batch_window_us);
            if (Clock::now() < until && !s->stop) {
                s->cv.wait_until(lk, until);
                continue;
            }
        }
        dispatch_locked(s);
        s->cv.wait_for(lk, std::chrono::milliseconds(5));
    }
}

}  // namespace rcabf

using namespace rcabf;

extern "C" {

int rcabf_server_create(const rcabf_server_config *cfg, rcabf_server **out)
{
    if (!cfg || !out || cfg->struct_size != (int32_t)sizeof(rcabf_server_config)) return RCABF_ERR_INVALID_ARGUMENT;
    if (cfg->n_streams < 1 || cfg->n_streams > 64 || cfg->max_queue < 1 || cfg->max_batch < 1 ||
        cfg->max_batch > MAX_JOBS || cfg->batch_window_us < 0 || cfg->hbm_budget_bytes == 0)
        return RCABF_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(cfg->device) != cudaSuccess) return RCABF_ERR_CUDA;
    // the library's per-device state (its error counter is a device
    // allocation) is made now: nothing may allocate once launches and their
    // completion callbacks are in flight
    device_state(cfg->device, true);
    rcabf_server *s = new rcabf_server();
    s->cfg = *cfg;
    int status = RCABF_OK;
    if (cudaMalloc(&s->arena_base, cfg->hbm_budget_bytes) != cudaSuccess) {
        cudaGetLastError();
        status = RCABF_ERR_OOM_ADMISSION;   // the budget itself does not fit the device
    }
    for (int i = 0; status == RCABF_OK && i < cfg->n_streams; ++i) {
        cudaStream_t st;
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) status = RCABF_ERR_CUDA;
        else s->streams.push_back(st);
    }
    cudaSetDevice(prev);
    if (status != RCABF_OK) {
        for (cudaStream_t st : s->streams) cudaStreamDestroy(st);
        if (s->arena_base) cudaFree(s->arena_base);
        delete s;
        return status;
    }
    s->arena.reset(cfg->hbm_budget_bytes / 256 * 256);
    s->slot_busy.assign(cfg->n_streams, 0);
    s->thread = std::thread(scheduler, s);
    *out = s;
    return RCABF_OK;
}

int rcabf_server_submit(rcabf_server *s, const rcabf_geometry *g, const rcabf_beamform_args *a, uint64_t *ticket)
{
    if (!s) return RCABF_ERR_BAD_HANDLE;
    if (!g) return RCABF_ERR_BAD_HANDLE;
    if (!a || !ticket) return RCABF_ERR_INVALID_ARGUMENT;
    rcabf_geometry *gg = const_cast<rcabf_geometry *>(g);
    if (gg->device != s->cfg.device) return RCABF_ERR_INVALID_ARGUMENT;
    Request *r = new Request();
    r->g = gg;
    r->a = *a;
    r->a.workspace = nullptr;
    r->a.workspace_bytes = 0;
    r->a.stage_events = nullptr;
    int st = plan_beamform(gg, &r->a, r->plan);
    if (st == RCABF_OK && (!r->a.iq || !r->a.out)) st = RCABF_ERR_INVALID_ARGUMENT;
    if (st == RCABF_OK && r->plan.kernel == RCABF_KERNEL_FUSED && r->a.frames_per_block == 0) {
        // pin the frame block the planner chose, so the request runs the same
        // kernel variant alone or fused with others; a request whose plan
        // would change under the pin is never fused
        rcabf_beamform_args pinned = r->a;
        pinned.frames_per_block = r->plan.fb;
        Plan p2;
        if (plan_beamform(gg, &pinned, p2) == RCABF_OK && p2.vb == r->plan.vb && p2.d == r->plan.d &&
            p2.tc == r->plan.tc && p2.fb == r->plan.fb && p2.total == r->plan.total) {
            r->a = pinned;
            r->batchable = true;
        }
    } else if (st == RCABF_OK && r->plan.kernel == RCABF_KERNEL_FUSED) {
        r->batchable = true;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    if (st == RCABF_OK && Arena::round(r->plan.total) > s->arena.size()) st = RCABF_ERR_OOM_ADMISSION;
    if (st == RCABF_OK && s->stop) st = RCABF_ERR_CANCELLED;
    if (st == RCABF_OK && (int64_t)s->queue.size() >= s->cfg.max_queue) st = RCABF_ERR_BUSY;
    if (st != RCABF_OK) {
        s->rejected += 1;
        delete r;
        return st;
    }
    r->ws_bytes = r->plan.total;
    r->units = (double)g->n_pix * g->n_ele * g->n_tx * (double)a->n_frame;
    r->t_submit = Clock::now();
    r->ticket = s->next_ticket++;
    if (!s->any_submit) { s->first_submit = r->t_submit; s->any_submit = true; }
    s->queue.push_back(r);
    s->all[r->ticket] = r;
    s->submitted += 1;
    *ticket = r->ticket;
    s->cv.notify_all();
    return RCABF_OK;
}

// Done requests are forgotten once their status has been returned.
static int take_locked(rcabf_server *s, uint64_t ticket, int *status, bool *found)
{
    auto it = s->all.find(ticket);
    *found = it != s->all.end();
    if (!*found) return RCABF_ERR_INVALID_ARGUMENT;
    Request *r = it->second;
    if (!r->done) return RCABF_ERR_PENDING;
    if (status) *status = r->status;
    s->all.erase(it);
    delete r;
    return RCABF_OK;
}

int rcabf_server_poll(rcabf_server *s, uint64_t ticket, int *status)
{
    if (!s) return RCABF_ERR_BAD_HANDLE;
    std::lock_guard<std::mutex> lk(s->mu);
    bool found;
    return take_locked(s, ticket, status, &found);
}

int rcabf_server_wait_for(rcabf_server *s, uint64_t ticket, double timeout_s, int *status)
{
    if (!s) return RCABF_ERR_BAD_HANDLE;
    if (!(timeout_s >= 0.0)) return RCABF_ERR_INVALID_ARGUMENT;
    const auto until = Clock::now() + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(
                                          std::min(timeout_s, 1.0e6)));
    std::unique_lock<std::mutex> lk(s->mu);
    while (true) {
        bool found;
        const int st = take_locked(s, ticket, status, &found);
        if (st != RCABF_ERR_PENDING) return st;
        if (s->cv_done.wait_until(lk, until) == std::cv_status::timeout) {
            const int st2 = take_locked(s, ticket, status, &found);
            return st2 == RCABF_ERR_PENDING ? RCABF_ERR_TIMEOUT : st2;
        }
    }
}

static double percentile(std::vector<double> v, double q)
{
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const double pos = q * (double)(v.size() - 1);
    const size_t i = (size_t)pos;
    const double f = pos - (double)i;
    return i + 1 < v.size() ? v[i] * (1.0 - f) + v[i + 1] * f : v[i];
}

int rcabf_server_get_stats(rcabf_server *s, rcabf_server_stats *st)
{
    if (!s) return RCABF_ERR_BAD_HANDLE;
    if (!st || st->struct_size != (int32_t)sizeof(rcabf_server_stats)) return RCABF_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(s->mu);
    const int32_t sz = st->struct_size;
    std::memset(st, 0, sizeof(*st));
    st->struct_size = sz;
    st->submitted = s->submitted;
    st->completed = s->completed;
    st->rejected = s->rejected;
    st->launches = s->launches;
    st->in_flight = s->in_flight;
    st->queued = (int64_t)s->queue.size();
    st->p50_ms = percentile(s->latency_ms, 0.50);
    st->p95_ms = percentile(s->latency_ms, 0.95);
    st->p99_ms = percentile(s->latency_ms, 0.99);
    double sum = 0.0, mx = 0.0;
    for (double x : s->latency_ms) { sum += x; mx = std::max(mx, x); }
    st->mean_ms = s->latency_ms.empty() ? 0.0 : sum / (double)s->latency_ms.size();
    st->max_ms = mx;
    st->units_done = s->units_done;
    double busy = s->busy_s;
    if (s->in_flight > 0) busy += std::chrono::duration<double>(Clock::now() - s->busy_since).count();
    st->busy_s = busy;
    st->span_s = s->any_submit ? std::chrono::duration<double>(s->last_done - s->first_submit).count() : 0.0;
    st->arena_bytes = s->arena.size();
    st->arena_peak_bytes = s->arena.peak();
    return RCABF_OK;
}

int rcabf_server_destroy(rcabf_server *s)
{
    if (!s) return RCABF_ERR_BAD_HANDLE;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;   // queued requests still run; new submits are refused
    }
    s->cv.notify_all();
    if (s->thread.joinable()) s->thread.join();
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(s->cfg.device);
    for (cudaStream_t st : s->streams) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    if (s->arena_base) cudaFree(s->arena_base);
    cudaSetDevice(prev);
    for (auto &kv : s->all) delete kv.second;
    delete s;
    return RCABF_OK;
}

}  // extern "C"
