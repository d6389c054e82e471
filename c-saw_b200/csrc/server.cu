// server.cu -- request loop with continuous batching (csaw_server_*).
//
// The reference serves one synchronous Sampler() call per process
// (non-stream/main.cu:196-308, called from mpi_main.cpp:40): it allocates,
// samples and returns a time.  Here a graph stays resident and a worker
// thread serves a stream of independent requests:
//
//   submit (any thread)  -> request queued with its own copy of params/seeds
//   worker: admission    -> a free slot (job context + stream) and room in the
//                           device arena for the request's seeds and outputs
//                           (first-fit in arrival order; a request waiting
//                           longer than max_wait_us blocks later ones)
//   worker: launch       -> seeds H2D from the slot's page-locked staging,
//                           the sampling kernels, counter read-back, event
//   worker: poll events  -> phase 1 done: edge count known, outputs D2H into
//                           the caller's buffers (direct when page-locked,
//                           else through the slot's staging), event
//                           phase 2 done: result complete, arena and slot
//                           released, waiters woken
//
// Requests on different slots overlap on the device; the work of a request
// is keyed only by its params and seeds (counter-based Philox draws, global
// sample ids), so a result is the same alone and in any mix.  Device memory
// for requests comes from one arena allocated at creation, so admission
// never calls cudaMalloc; job-context scratch grows on a slot's first
// requests and is then reused.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "csaw.h"
#include "csaw_host.h"

namespace {

using Clock = std::chrono::steady_clock;

double now_s() { return std::chrono::duration<double>(Clock::now().time_since_epoch()).count(); }

constexpr int64_t ARENA_ALIGN = 256;
constexpr int64_t DEFAULT_BUDGET = 1ll << 30;
constexpr int DEFAULT_MAX_WAIT_US = 2000;
constexpr int MAX_SLOTS = 64;

int64_t round_up(int64_t n, int64_t a) { return (n + a - 1) / a * a; }

// First-fit allocator over the offsets [0, size) of the device arena, with
// coalescing on release.
class Arena {
  public:
    void reset(int64_t size) {
        free_.clear();
        if (size > 0) free_[0] = size;
        size_ = size;
        used_ = peak_ = 0;
    }
    int64_t alloc(int64_t n) {
        n = round_up(n < 1 ? 1 : n, ARENA_ALIGN);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < n) continue;
            const int64_t off = it->first, rem = it->second - n;
            free_.erase(it);
            if (rem > 0) free_[off + n] = rem;
            used_ += n;
            peak_ = std::max(peak_, used_);
            return off;
        }
        return -1;
    }
    void release(int64_t off, int64_t n) {
        n = round_up(n < 1 ? 1 : n, ARENA_ALIGN);
        used_ -= n;
        auto it = free_.emplace(off, n).first;
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
    int64_t peak() const { return peak_; }

  private:
    std::map<int64_t, int64_t> free_;
    int64_t size_ = 0, used_ = 0, peak_ = 0;
};

struct Request {
    uint64_t id = 0;
    csaw_params p{};
    std::vector<int32_t> seeds;
    int32_t *out[4] = {};   // caller's host buffers: src, dst, sample, depth
    bool pinned = false;    // all non-null outputs page-locked
    int64_t cap = 0;        // caller's capacity
    int64_t dcap = 0;       // device capacity: the edge bound
    int64_t n_seeds = 0;
    int64_t seed_bytes = 0, bytes = 0, off = -1;
    int status = -1;        // -1 while unfinished
    std::string err;
    int64_t n_out = 0;
    double t_submit = 0, t_admit = 0, t_launched = 0, t_sampled = 0, t_done = 0;
};

struct Slot {
    void *job = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t ev = nullptr;
    int32_t *pin_seeds = nullptr;
    int64_t pin_seeds_n = 0;
    int32_t *pin_out = nullptr;
    int64_t pin_out_n = 0;
    Request *req = nullptr;
    int phase = 0;   // 0 free, 1 sampling, 2 copying out
};

bool host_pinned(const void *p) {
    if (!p) return true;
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// Grows a page-locked staging buffer to at least n int32 (doubling).
int grow_pinned(int32_t **buf, int64_t *have, int64_t n) {
    if (*have >= n) return 0;
    int64_t want = std::max<int64_t>(n, *have * 2);
    if (*buf) cudaFreeHost(*buf);
    *buf = nullptr;
    *have = 0;
    cudaError_t e = cudaHostAlloc((void **)buf, sizeof(int32_t) * (size_t)want, cudaHostAllocDefault);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *buf = nullptr;
        return csaw_host_fail(CSAW_ERR_NOMEM, "page-locked staging allocation failed");
    }
    *have = want;
    return 0;
}

}  // namespace

struct csaw_server_s {
    csaw_graph g = nullptr;
    int device = 0;
    csaw_server_config cfg{};
    unsigned char *arena_base = nullptr;
    Arena arena;
    std::vector<Slot> slots;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request *> queue;
    std::unordered_map<uint64_t, Request *> reqs;
    uint64_t next_id = 1;
    int busy = 0;
    bool stop = false;
    std::thread worker;
    int64_t submitted = 0, completed = 0, failed = 0, edges = 0;
    std::vector<double> lat_ms, queue_ms, launch_ms, gpu_ms;
    double first_submit = 0, last_done = 0;
    double max_call_ms = 0;        // longest worker step (launch or completion) since reset
    int64_t calls_over_1ms = 0;
};

namespace {

// Next request to admit (under the lock): first-fit in arrival order, unless
// the head has waited longer than the bound.  Reserves its arena bytes.
Request *pick(csaw_server_s *s) {
    if (s->queue.empty()) return nullptr;
    const double wait_s = (double)s->cfg.max_wait_us * 1e-6;
    const bool head_only = now_s() - s->queue.front()->t_submit > wait_s;
    for (auto it = s->queue.begin(); it != s->queue.end(); ++it) {
        Request *r = *it;
        const int64_t off = s->arena.alloc(r->bytes);
        if (off >= 0) {
            r->off = off;
            s->queue.erase(it);
            return r;
        }
        if (head_only) break;
    }
    return nullptr;
}

// Marks r finished (under the lock) and releases its slot and arena bytes.
void finish(csaw_server_s *s, Slot *sl, Request *r, int status, const char *err) {
    r->status = status;
    if (status != CSAW_OK && err) r->err = err;
    r->t_done = now_s();
    if (r->off >= 0) s->arena.release(r->off, r->bytes);
    r->off = -1;
    if (sl) {
        sl->req = nullptr;
        sl->phase = 0;
        --s->busy;
    }
    if (status == CSAW_OK) {
        ++s->completed;
        s->edges += r->n_out;
        s->lat_ms.push_back((r->t_done - r->t_submit) * 1e3);
        s->queue_ms.push_back((r->t_admit - r->t_submit) * 1e3);
        s->launch_ms.push_back((r->t_launched - r->t_admit) * 1e3);
        s->gpu_ms.push_back((r->t_sampled - r->t_launched) * 1e3);
        s->last_done = r->t_done;
    } else {
        ++s->failed;
    }
    s->cv_done.notify_all();
}

int32_t *dev_array(csaw_server_s *s, const Request *r, int k) {
    int32_t *base = (int32_t *)(s->arena_base + r->off + r->seed_bytes);
    int idx = 0;
    for (int j = 0; j < k; ++j)
        if (j < 2 || r->out[j]) ++idx;   // src and dst always have device arrays
    return base + (int64_t)idx * r->dcap;
}

// Phase 1 launch (lock not held): seeds in, sampling kernels, event.
int launch(csaw_server_s *s, Slot *sl) {
    Request *r = sl->req;
    if (r->n_seeds > 0) {
        if (grow_pinned(&sl->pin_seeds, &sl->pin_seeds_n, r->n_seeds)) return CSAW_ERR_NOMEM;
        std::memcpy(sl->pin_seeds, r->seeds.data(), sizeof(int32_t) * (size_t)r->n_seeds);
        cudaError_t e = cudaMemcpyAsync(s->arena_base + r->off, sl->pin_seeds, sizeof(int32_t) * (size_t)r->n_seeds,
                                        cudaMemcpyHostToDevice, sl->st);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return csaw_host_fail(CSAW_ERR_CUDA, cudaGetErrorString(e));
        }
    }
    const int32_t *seeds = (const int32_t *)(s->arena_base + r->off);
    int32_t *o[4];
    for (int k = 0; k < 4; ++k) o[k] = (k < 2 || r->out[k]) ? dev_array(s, r, k) : nullptr;
    int rc = csaw_host_job_enqueue(s->g, sl->job, &r->p, seeds, o[0], o[1], o[2], o[3], r->dcap);
    if (rc) return rc;
    cudaError_t e = cudaEventRecord(sl->ev, sl->st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return csaw_host_fail(CSAW_ERR_CUDA, cudaGetErrorString(e));
    }
    sl->phase = 1;
    return 0;
}

// Advances a slot whose event completed (lock not held).  Returns true when
// the request is finished (status in *rc).
bool advance(csaw_server_s *s, Slot *sl, int *rc) {
    Request *r = sl->req;
    if (sl->phase == 1) {
        r->t_sampled = now_s();
        int64_t n = 0;
        *rc = csaw_host_job_finish(s->g, sl->job, r->dcap, &n);
        r->n_out = n;
        if (*rc == 0 && n > r->cap) *rc = csaw_host_fail(CSAW_ERR_CAPACITY, "output capacity too small");
        if (*rc || n == 0) return true;
        const bool staged = !r->pinned;
        int narr = 0;
        for (int k = 0; k < 4; ++k) narr += r->out[k] != nullptr;
        if (staged && grow_pinned(&sl->pin_out, &sl->pin_out_n, n * narr)) {
            *rc = CSAW_ERR_NOMEM;
            return true;
        }
        int j = 0;
        for (int k = 0; k < 4; ++k) {
            if (!r->out[k]) continue;
            void *dst = staged ? (void *)(sl->pin_out + (int64_t)j * n) : (void *)r->out[k];
            cudaError_t e = cudaMemcpyAsync(dst, dev_array(s, r, k), sizeof(int32_t) * (size_t)n,
                                            cudaMemcpyDeviceToHost, sl->st);
            if (e != cudaSuccess) {
                cudaGetLastError();
                *rc = csaw_host_fail(CSAW_ERR_CUDA, cudaGetErrorString(e));
                return true;
            }
            ++j;
        }
        cudaError_t e = cudaEventRecord(sl->ev, sl->st);
        if (e != cudaSuccess) {
            cudaGetLastError();
            *rc = csaw_host_fail(CSAW_ERR_CUDA, cudaGetErrorString(e));
            return true;
        }
        sl->phase = 2;
        return false;
    }
    // phase 2: outputs are in host memory
    if (!r->pinned) {
        int j = 0;
        for (int k = 0; k < 4; ++k) {
            if (!r->out[k]) continue;
            std::memcpy(r->out[k], sl->pin_out + (int64_t)j * r->n_out, sizeof(int32_t) * (size_t)r->n_out);
            ++j;
        }
    }
    *rc = 0;
    return true;
}

// Records the duration of one worker step (under the lock).
void note_call(csaw_server_s *s, double seconds) {
    const double ms = seconds * 1e3;
    if (ms > s->max_call_ms) s->max_call_ms = ms;
    if (ms > 1.0) ++s->calls_over_1ms;
}

void worker_main(csaw_server_s *s) {
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        bool progressed = false;
        // admissions
        for (auto &sl : s->slots) {
            if (sl.phase != 0) continue;
            Request *r = pick(s);
            if (!r) break;
            sl.req = r;
            sl.phase = 1;
            ++s->busy;
            r->t_admit = now_s();
            lk.unlock();
            const int rc = launch(s, &sl);
            r->t_launched = now_s();
            const std::string err = rc ? csaw_last_error() : "";
            lk.lock();
            note_call(s, r->t_launched - r->t_admit);
            if (rc) finish(s, &sl, r, rc, err.c_str());
            progressed = true;
        }
        // completions
        for (auto &sl : s->slots) {
            if (sl.phase == 0) continue;
            const cudaError_t q = cudaEventQuery(sl.ev);
            if (q == cudaErrorNotReady) continue;
            lk.unlock();
            const double t0 = now_s();
            int rc = 0;
            bool done;
            if (q != cudaSuccess) {
                cudaGetLastError();
                rc = csaw_host_fail(CSAW_ERR_CUDA, cudaGetErrorString(q));
                done = true;
            } else {
                done = advance(s, &sl, &rc);
            }
            const std::string err = rc ? csaw_last_error() : "";
            const double t1 = now_s();
            lk.lock();
            note_call(s, t1 - t0);
            if (done) finish(s, &sl, sl.req, rc, err.c_str());
            progressed = true;
        }
        if (s->stop && s->queue.empty() && s->busy == 0) break;
        if (progressed) continue;
        if (s->busy > 0) {   // kernels in flight: poll again shortly
            lk.unlock();
            std::this_thread::yield();
            lk.lock();
        } else {
            s->cv_work.wait(lk, [&] { return s->stop || !s->queue.empty(); });
        }
    }
}

void free_server(csaw_server_s *s) {
    for (auto &sl : s->slots) {
        if (sl.job) csaw_host_job_destroy(sl.job);
        if (sl.ev) cudaEventDestroy(sl.ev);
        if (sl.pin_seeds) cudaFreeHost(sl.pin_seeds);
        if (sl.pin_out) cudaFreeHost(sl.pin_out);
    }
    if (s->arena_base) cudaFree(s->arena_base);
    for (auto &kv : s->reqs) delete kv.second;
    delete s;
}

}  // namespace

extern "C" int csaw_server_create(csaw_graph g, const csaw_server_config *cfg, csaw_server *out) {
    if (!g || !out) return csaw_host_fail(CSAW_ERR_INVALID, "NULL argument");
    csaw_server_config c = cfg ? *cfg : csaw_server_config{};
    if (c.n_slots == 0) c.n_slots = 8;
    if (c.n_slots < 1 || c.n_slots > MAX_SLOTS) return csaw_host_fail(CSAW_ERR_INVALID, "n_slots must be in [1, 64]");
    if (c.max_wait_us <= 0) c.max_wait_us = DEFAULT_MAX_WAIT_US;
    if (c.device_budget == 0) c.device_budget = DEFAULT_BUDGET;
    if (c.device_budget < 0) return csaw_host_fail(CSAW_ERR_INVALID, "device_budget < 0");
    auto *s = new csaw_server_s();
    s->g = g;
    s->device = csaw_host_graph_device(g);
    s->cfg = c;
    cudaError_t e = cudaSetDevice(s->device);
    if (e == cudaSuccess) e = cudaMalloc((void **)&s->arena_base, (size_t)c.device_budget);
    if (e != cudaSuccess) {
        cudaGetLastError();
        s->arena_base = nullptr;
        free_server(s);
        return csaw_host_fail(CSAW_ERR_NOMEM, "server arena allocation failed");
    }
    s->arena.reset(c.device_budget);
    s->slots.resize((size_t)c.n_slots);
    for (auto &sl : s->slots) {
        int rc = csaw_host_job_create(g, &sl.job, &sl.st);
        if (rc == 0 && cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            rc = csaw_host_fail(CSAW_ERR_CUDA, "event creation failed");
        }
        if (rc) {
            free_server(s);
            return rc;
        }
    }
    s->worker = std::thread(worker_main, s);
    *out = s;
    return 0;
}

extern "C" int csaw_server_destroy(csaw_server s) {
    if (!s) return csaw_host_fail(CSAW_ERR_INVALID, "server is NULL");
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    free_server(s);
    return 0;
}

extern "C" int csaw_server_submit(csaw_server s, const csaw_params *p, const int32_t *seeds, int32_t *out_src,
                                  int32_t *out_dst, int32_t *out_sample, int32_t *out_depth, int64_t capacity,
                                  uint64_t *ticket) {
    if (!s || !p || !ticket) return csaw_host_fail(CSAW_ERR_INVALID, "NULL argument");
    if (capacity < 0) return csaw_host_fail(CSAW_ERR_INVALID, "capacity < 0");
    if (capacity > 0 && (!out_src || !out_dst)) return csaw_host_fail(CSAW_ERR_INVALID, "out_src/out_dst are NULL");
    int64_t bound = 0, ns = 0;
    int rc = csaw_host_edge_bound(s->g, p, &bound, &ns);
    if (rc) return rc;
    if (ns > 0 && !seeds) return csaw_host_fail(CSAW_ERR_INVALID, "seeds is NULL");
    auto *r = new Request();
    r->p = *p;
    r->seeds.assign(seeds, seeds + ns);
    r->out[0] = out_src;
    r->out[1] = out_dst;
    r->out[2] = out_sample;
    r->out[3] = out_depth;
    r->pinned = host_pinned(out_src) && host_pinned(out_dst) && host_pinned(out_sample) && host_pinned(out_depth);
    r->cap = capacity;
    // the device buffers hold every edge the request can emit, so an
    // undersized host capacity still reports the needed count
    r->dcap = bound;
    r->n_seeds = ns;
    const int narr = 2 + (out_sample != nullptr) + (out_depth != nullptr);
    r->seed_bytes = round_up(sizeof(int32_t) * (ns > 0 ? ns : 1), ARENA_ALIGN);
    r->bytes = r->seed_bytes + (int64_t)sizeof(int32_t) * narr * r->dcap;
    if (r->bytes > s->cfg.device_budget) {
        const int64_t need = r->bytes;
        delete r;
        return csaw_host_fail(CSAW_ERR_CAPACITY, ("request needs " + std::to_string(need) +
                                                  " device bytes, above the server budget").c_str());
    }
    {
        std::lock_guard<std::mutex> lk(s->mu);
        r->id = s->next_id++;
        r->t_submit = now_s();
        if (s->submitted == 0) s->first_submit = r->t_submit;
        ++s->submitted;
        s->reqs[r->id] = r;
        s->queue.push_back(r);
        *ticket = r->id;
    }
    s->cv_work.notify_one();
    return 0;
}

extern "C" int csaw_server_wait(csaw_server s, uint64_t ticket, int64_t timeout_us, int64_t *n_out,
                                double *latency_ms) {
    if (!s) return csaw_host_fail(CSAW_ERR_INVALID, "server is NULL");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return csaw_host_fail(CSAW_ERR_INVALID, "unknown or already reported ticket");
    Request *r = it->second;
    auto ready = [&] { return r->status >= 0; };
    if (timeout_us < 0) s->cv_done.wait(lk, ready);
    else s->cv_done.wait_for(lk, std::chrono::microseconds(timeout_us), ready);
    if (!ready()) return CSAW_PENDING;
    if (n_out) *n_out = r->n_out;
    if (latency_ms) *latency_ms = (r->t_done - r->t_submit) * 1e3;
    const int rc = r->status;
    if (rc) csaw_host_fail(rc, r->err.c_str());
    s->reqs.erase(it);
    delete r;
    return rc;
}

extern "C" int csaw_server_get_stats(csaw_server s, int reset, csaw_server_stats *out) {
    if (!s || !out) return csaw_host_fail(CSAW_ERR_INVALID, "NULL argument");
    std::lock_guard<std::mutex> lk(s->mu);
    csaw_server_stats st{};
    st.submitted = s->submitted;
    st.completed = s->completed;
    st.failed = s->failed;
    st.queued = (int64_t)s->queue.size();
    st.in_flight = s->busy;
    st.edges = s->edges;
    st.peak_device_bytes = s->arena.peak();
    for (const auto &sl : s->slots) st.workspace_bytes += csaw_host_job_workspace(sl.job);
    auto pct = [](std::vector<double> v, double q) {   // nearest rank
        if (v.empty()) return 0.0;
        std::sort(v.begin(), v.end());
        size_t k = (size_t)std::ceil(q * (double)v.size());
        return v[k == 0 ? 0 : k - 1];
    };
    if (!s->lat_ms.empty()) {
        st.p50_ms = pct(s->lat_ms, 0.50);
        st.p90_ms = pct(s->lat_ms, 0.90);
        st.p99_ms = pct(s->lat_ms, 0.99);
        st.max_ms = pct(s->lat_ms, 1.0);
        double sum = 0;
        for (double x : s->lat_ms) sum += x;
        st.mean_ms = sum / (double)s->lat_ms.size();
        st.p99_queue_ms = pct(s->queue_ms, 0.99);
        st.p99_launch_ms = pct(s->launch_ms, 0.99);
        st.p99_gpu_ms = pct(s->gpu_ms, 0.99);
    }
    st.first_submit_s = s->first_submit;
    st.last_done_s = s->last_done;
    st.max_worker_call_ms = s->max_call_ms;
    st.worker_calls_over_1ms = s->calls_over_1ms;
    if (reset) {
        s->max_call_ms = 0;
        s->calls_over_1ms = 0;
        s->lat_ms.clear();
        s->queue_ms.clear();
        s->launch_ms.clear();
        s->gpu_ms.clear();
        s->submitted = s->completed = s->failed = s->edges = 0;
    }
    *out = st;
    return 0;
}
