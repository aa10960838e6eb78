// gqis_serve.cu - native sweep server (C ABI in include/gqis_serve.h).
//
// One scheduler thread per server, with the server's device current, does all CUDA work:
//   admit    - first-in-first-out, while the admitted requests' stated bytes fit the memory budget
//              and fewer than max_inflight requests run; the request's model module is loaded
//              (dlopen, once per path) and its info read; its points are cut into chunks;
//   dispatch - one chunk of each running request per pass, oldest request first, onto the
//              least-loaded stream, at most two chunks queued per stream; a chunk is the caller's
//              descriptor restricted to [point_begin + b, point_begin + b + n) with the per-point
//              pointers (results, rho0, trace, step_counts) offset to that slice, and for the
//              adaptive integrators a zeroed work counter of its own. The next chunks of all
//              running adaptive requests of one module go out together as one batch grid
//              (gqis_sweep_launch_batch, one zeroed counter): the persistent lanes take points of
//              every request from that counter, so work is stolen across requests;
//   complete - chunks end when their event has completed; a request ends when its last chunk has.
// A launch the module rejects fails its own request only (with the module's error text).
// Host threads submit, poll, wait and cancel under one mutex.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <stdarg.h>
#include <stdio.h>

#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "gqis_b200.h"
#include "gqis_serve.h"

namespace {

thread_local char g_serve_error[512] = "";

int fail(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_serve_error, sizeof(g_serve_error), fmt, ap);
    va_end(ap);
    return code;
}

using launch_fn = int (*)(const gqis_sweep_desc*, void*);
using batch_fn = int (*)(const gqis_sweep_desc*, int32_t, uint32_t*, void*);
using info_fn = int (*)(gqis_model_info*);
using error_fn = const char* (*)(void);

struct Module {
    void* handle = nullptr;
    launch_fn launch = nullptr;
    batch_fn batch = nullptr;  // gqis_sweep_launch_batch (absent from older modules)
    error_fn last_error = nullptr;
    gqis_model_info info{};
};

// One launch on the device. A batch launch is shared by the requests whose chunks it carries: its
// event, stream slot and counter are released when the last of them has seen it complete.
struct Launch {
    cudaEvent_t event;
    int stream;
    int counter;  // index into the server's work counters, or -1
    int holders;  // requests still holding this launch
};

struct InFlight {
    std::shared_ptr<Launch> launch;
};

struct Request {
    int64_t id = 0;
    std::string path;
    gqis_sweep_desc desc{};
    int64_t bytes = 0;
    Module* module = nullptr;
    std::deque<std::pair<int64_t, int64_t>> chunks;  // (begin, count) relative to desc.point_begin
    std::vector<InFlight> inflight;
    int32_t state = GQIS_REQ_QUEUED;
    bool cancel = false;
    std::string error;
};

bool adaptive(const gqis_model_info& info) {
    return info.solver == GQIS_SOLVER_TSIT5A || info.solver == GQIS_SOLVER_DOP853A;
}

}  // namespace

struct gqis_server {
    int device = 0, nstreams = 1, max_inflight = 1;
    int64_t chunk_points = 1, budget = 0, used = 0, next_id = 1;
    std::vector<cudaStream_t> streams;
    std::vector<int> load;
    unsigned int* counters = nullptr;  // device: one uint32 per possible chunk in flight
    std::vector<int> free_counters;
    std::map<std::string, std::unique_ptr<Module>> modules;
    std::map<int64_t, std::shared_ptr<Request>> requests;
    std::deque<std::shared_ptr<Request>> queue;
    std::vector<std::shared_ptr<Request>> active;
    std::mutex mu;
    std::condition_variable cv;
    std::thread thread;
    bool stop = false;

    // ---- scheduler (holds mu)
    Module* load_module(const std::string& path, std::string& error) {
        auto it = modules.find(path);
        if (it != modules.end()) return it->second.get();
        void* h = dlopen(path.c_str(), RTLD_NOW | RTLD_LOCAL);
        if (!h) {
            const char* e = dlerror();
            error = std::string("cannot load module: ") + (e ? e : path.c_str());
            return nullptr;
        }
        auto m = std::make_unique<Module>();
        m->handle = h;
        m->launch = reinterpret_cast<launch_fn>(dlsym(h, "gqis_sweep_launch"));
        m->batch = reinterpret_cast<batch_fn>(dlsym(h, "gqis_sweep_launch_batch"));
        m->last_error = reinterpret_cast<error_fn>(dlsym(h, "gqis_last_error"));
        info_fn info = reinterpret_cast<info_fn>(dlsym(h, "gqis_model_info_get"));
        if (!m->launch || !m->last_error || !info) {
            error = "not a model module (gqis_sweep_launch / gqis_model_info_get missing): " + path;
            return nullptr;
        }
        if (info(&m->info) != GQIS_OK) {
            error = std::string("gqis_model_info_get failed: ") + m->last_error();
            return nullptr;
        }
        Module* raw = m.get();
        modules[path] = std::move(m);
        return raw;
    }

    void end(const std::shared_ptr<Request>& r, int32_t state) {
        r->state = state;
        used -= r->bytes;
        for (size_t i = 0; i < active.size(); ++i)
            if (active[i] == r) {
                active.erase(active.begin() + (long)i);
                break;
            }
        cv.notify_all();
    }

    void admit() {
        while (!queue.empty() && (int)active.size() < max_inflight) {
            auto r = queue.front();
            if (budget > 0 && used + r->bytes > budget && !active.empty()) return;  // waits for memory
            queue.pop_front();
            used += r->bytes;
            std::string error;
            r->module = load_module(r->path, error);
            if (!r->module) {
                r->error = error;
                r->state = GQIS_REQ_FAILED;
                used -= r->bytes;
                cv.notify_all();
                continue;
            }
            for (int64_t b = 0; b < r->desc.point_count; b += chunk_points)
                r->chunks.emplace_back(b, std::min(chunk_points, r->desc.point_count - b));
            r->state = GQIS_REQ_RUNNING;
            active.push_back(r);
        }
    }

    gqis_sweep_desc chunk_desc(const Request& r, int64_t b, int64_t n) const {
        const gqis_model_info& in = r.module->info;
        const int64_t esz = in.form == GQIS_FORM_FP64 ? 8 : 4;
        const int64_t width = (in.output_mode == GQIS_OUT_MEAN || in.output_mode == GQIS_OUT_FINAL) ? 2 : in.state_size;
        gqis_sweep_desc d = r.desc;
        d.point_begin = r.desc.point_begin + b;
        d.point_count = n;
        d.results = static_cast<char*>(r.desc.results) + b * width * esz;
        if (r.desc.rho0) d.rho0 = static_cast<const char*>(r.desc.rho0) + b * (int64_t)in.state_size * esz;
        if (in.trace_mode != GQIS_TRACE_NONE && r.desc.trace) {
            const int64_t tw = in.trace_mode == GQIS_TRACE_OBSERVABLE ? 2 : in.state_size;
            d.trace = static_cast<char*>(r.desc.trace) + b * (int64_t)r.desc.num_trace * tw * esz;
        }
        if (r.desc.step_counts) d.step_counts = r.desc.step_counts + b * 2;
        return d;
    }

    int least_loaded() const {
        int s = 0;
        for (int i = 1; i < nstreams; ++i)
            if (load[i] < load[s]) s = i;
        return s;
    }

    // The next chunk of each request in rs (adaptive, one module) as one batch grid on stream s.
    void dispatch_batch(Module* m, const std::vector<std::shared_ptr<Request>>& rs, int s) {
        std::vector<gqis_sweep_desc> ds;
        for (const auto& r : rs) {
            const auto chunk = r->chunks.front();
            r->chunks.pop_front();
            ds.push_back(chunk_desc(*r, chunk.first, chunk.second));
        }
        const int counter = free_counters.back();
        free_counters.pop_back();
        cudaMemsetAsync(counters + counter, 0, sizeof(unsigned int), streams[s]);
        const int rc = m->batch(ds.data(), (int32_t)ds.size(), counters + counter, streams[s]);
        if (rc != GQIS_OK) {
            for (const auto& r : rs) {
                r->error = m->last_error();
                r->cancel = true;
            }
            free_counters.push_back(counter);
            return;
        }
        cudaEvent_t ev;
        if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventRecord(ev, streams[s]) != cudaSuccess) {
            cudaStreamSynchronize(streams[s]);  // no event: wait here instead
            free_counters.push_back(counter);
            return;
        }
        load[s] += 1;
        auto launch = std::make_shared<Launch>(Launch{ev, s, counter, (int)rs.size()});
        for (const auto& r : rs) r->inflight.push_back({launch});
    }

    bool dispatch() {
        bool progressed = false;
        std::map<Module*, std::vector<std::shared_ptr<Request>>> batched;  // adaptive requests by module
        for (auto& r : std::vector<std::shared_ptr<Request>>(active)) {
            if (r->cancel || r->chunks.empty()) continue;
            if (adaptive(r->module->info) && r->module->batch) {
                batched[r->module].push_back(r);
                continue;
            }
            const int s = least_loaded();
            if (load[s] >= 2) break;
            const auto chunk = r->chunks.front();
            r->chunks.pop_front();
            gqis_sweep_desc d = chunk_desc(*r, chunk.first, chunk.second);
            int counter = -1;
            if (adaptive(r->module->info)) {
                counter = free_counters.back();
                free_counters.pop_back();
                d.work_counter = counters + counter;
                cudaMemsetAsync(d.work_counter, 0, sizeof(unsigned int), streams[s]);
            }
            const int rc = r->module->launch(&d, streams[s]);
            if (rc != GQIS_OK) {
                r->error = r->module->last_error();
                r->cancel = true;
                if (counter >= 0) free_counters.push_back(counter);
                progressed = true;
                continue;
            }
            cudaEvent_t ev;
            if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess ||
                cudaEventRecord(ev, streams[s]) != cudaSuccess) {
                cudaStreamSynchronize(streams[s]);  // no event: wait here instead
                if (counter >= 0) free_counters.push_back(counter);
                progressed = true;
                continue;
            }
            load[s] += 1;
            r->inflight.push_back({std::make_shared<Launch>(Launch{ev, s, counter, 1})});
            progressed = true;
        }
        for (auto& group : batched) {
            const int s = least_loaded();
            if (load[s] >= 2 || free_counters.empty()) break;
            std::vector<std::shared_ptr<Request>>& rs = group.second;
            if (rs.size() > (size_t)GQIS_BATCH_MAX) rs.resize(GQIS_BATCH_MAX);
            dispatch_batch(group.first, rs, s);
            progressed = true;
        }
        return progressed;
    }

    bool complete() {
        bool progressed = false;
        for (auto& r : std::vector<std::shared_ptr<Request>>(active)) {
            std::vector<InFlight> still;
            for (const InFlight& f : r->inflight) {
                Launch& l = *f.launch;
                const cudaError_t q = cudaEventQuery(l.event);
                if (q == cudaErrorNotReady) {
                    still.push_back(f);
                    continue;
                }
                if (q != cudaSuccess && r->error.empty()) {
                    r->error = std::string("chunk failed on the device: ") + cudaGetErrorString(q);
                    r->cancel = true;
                }
                if (--l.holders == 0) {  // the last request of a shared batch releases its launch
                    cudaEventDestroy(l.event);
                    load[l.stream] -= 1;
                    if (l.counter >= 0) free_counters.push_back(l.counter);
                }
                progressed = true;
            }
            r->inflight.swap(still);
            if (!r->inflight.empty()) continue;
            if (r->cancel) {
                end(r, r->error.empty() ? GQIS_REQ_CANCELLED : GQIS_REQ_FAILED);
                progressed = true;
            } else if (r->chunks.empty()) {
                end(r, GQIS_REQ_DONE);
                progressed = true;
            }
        }
        return progressed;
    }

    void run() {
        cudaSetDevice(device);
        for (;;) {
            bool progressed;
            {
                std::lock_guard<std::mutex> lock(mu);
                if (stop) {
                    for (auto& r : queue) {
                        r->state = GQIS_REQ_CANCELLED;
                    }
                    queue.clear();
                    for (auto& r : active) r->cancel = true;
                    cv.notify_all();
                }
                admit();
                progressed = dispatch();
                progressed = complete() || progressed;
                if (stop && active.empty() && queue.empty()) return;
            }
            if (!progressed) std::this_thread::sleep_for(std::chrono::microseconds(50));
        }
    }
};

extern "C" {

__attribute__((visibility("default"))) const char* gqis_serve_last_error(void) { return g_serve_error; }

__attribute__((visibility("default"))) int gqis_serve_open(int device, int streams, int max_inflight,
                                                           int64_t chunk_points, int64_t memory_budget,
                                                           gqis_server** out) {
    if (!out) return fail(GQIS_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (streams < 1 || streams > 64 || max_inflight < 1 || chunk_points < 1 || memory_budget < 0)
        return fail(GQIS_ERR_INVALID, "invalid server sizes (streams %d, max_inflight %d, chunk_points %lld)", streams,
                    max_inflight, (long long)chunk_points);
    int prev = 0;
    cudaError_t e = cudaGetDevice(&prev);
    if (e != cudaSuccess) return fail(GQIS_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    if ((e = cudaSetDevice(device)) != cudaSuccess) return fail(GQIS_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e));
    auto s = std::make_unique<gqis_server>();
    s->device = device;
    s->nstreams = streams;
    s->max_inflight = max_inflight;
    s->chunk_points = chunk_points;
    s->budget = memory_budget;
    s->load.assign(streams, 0);
    int rc = GQIS_OK;
    for (int i = 0; i < streams && rc == GQIS_OK; ++i) {
        cudaStream_t st;
        if ((e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) != cudaSuccess)
            rc = fail(GQIS_ERR_CUDA, "cudaStreamCreate: %s", cudaGetErrorString(e));
        else
            s->streams.push_back(st);
    }
    const int ncounters = 2 * streams;  // at most two chunks queued per stream
    if (rc == GQIS_OK &&
        (e = cudaMalloc(reinterpret_cast<void**>(&s->counters), ncounters * sizeof(unsigned int))) != cudaSuccess)
        rc = fail(GQIS_ERR_CUDA, "cudaMalloc(work counters): %s", cudaGetErrorString(e));
    cudaSetDevice(prev);
    if (rc != GQIS_OK) {
        for (cudaStream_t st : s->streams) cudaStreamDestroy(st);
        return rc;
    }
    for (int i = ncounters - 1; i >= 0; --i) s->free_counters.push_back(i);
    gqis_server* raw = s.release();
    raw->thread = std::thread([raw] { raw->run(); });
    *out = raw;
    return GQIS_OK;
}

__attribute__((visibility("default"))) int gqis_serve_submit(gqis_server* s, const char* module_path,
                                                             const gqis_sweep_desc* desc, int64_t bytes,
                                                             int64_t* request_id) {
    if (!s || !module_path || !desc || !request_id || bytes < 0) return fail(GQIS_ERR_INVALID, "NULL argument");
    if (desc->abi_version != GQIS_ABI_VERSION)
        return fail(GQIS_ERR_INVALID, "descriptor ABI version %d, server expects %d", desc->abi_version, GQIS_ABI_VERSION);
    if (desc->point_count < 0 || !desc->results) return fail(GQIS_ERR_INVALID, "invalid point range or results");
    if (s->budget > 0 && bytes > s->budget)
        return fail(GQIS_ERR_TOO_LARGE, "request of %lld bytes exceeds the memory budget of %lld", (long long)bytes,
                    (long long)s->budget);
    auto r = std::make_shared<Request>();
    r->path = module_path;
    r->desc = *desc;
    r->bytes = bytes;
    std::lock_guard<std::mutex> lock(s->mu);
    if (s->stop) return fail(GQIS_ERR_INVALID, "server is closing");
    r->id = s->next_id++;
    s->requests[r->id] = r;
    s->queue.push_back(r);
    *request_id = r->id;
    return GQIS_OK;
}

__attribute__((visibility("default"))) int gqis_serve_poll(gqis_server* s, int64_t id, int32_t* state) {
    if (!s || !state) return fail(GQIS_ERR_INVALID, "NULL argument");
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->requests.find(id);
    if (it == s->requests.end()) return fail(GQIS_ERR_INVALID, "unknown request %lld", (long long)id);
    *state = it->second->state;
    return GQIS_OK;
}

__attribute__((visibility("default"))) int gqis_serve_wait(gqis_server* s, int64_t id, double timeout_s,
                                                           int32_t* state) {
    if (!s || !state || !(timeout_s >= 0.0)) return fail(GQIS_ERR_INVALID, "invalid argument");
    std::unique_lock<std::mutex> lock(s->mu);
    auto it = s->requests.find(id);
    if (it == s->requests.end()) return fail(GQIS_ERR_INVALID, "unknown request %lld", (long long)id);
    auto r = it->second;
    const bool ended = s->cv.wait_for(lock, std::chrono::duration<double>(timeout_s),
                                      [&] { return r->state >= GQIS_REQ_DONE; });
    *state = r->state;
    return ended ? GQIS_OK : fail(GQIS_ERR_TIMEOUT, "request %lld still running after %g s", (long long)id, timeout_s);
}

__attribute__((visibility("default"))) int gqis_serve_cancel(gqis_server* s, int64_t id) {
    if (!s) return fail(GQIS_ERR_INVALID, "NULL server");
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->requests.find(id);
    if (it == s->requests.end()) return fail(GQIS_ERR_INVALID, "unknown request %lld", (long long)id);
    auto r = it->second;
    if (r->state == GQIS_REQ_QUEUED) {
        for (size_t i = 0; i < s->queue.size(); ++i)
            if (s->queue[i] == r) {
                s->queue.erase(s->queue.begin() + (long)i);
                break;
            }
        r->state = GQIS_REQ_CANCELLED;
        s->cv.notify_all();
    } else if (r->state == GQIS_REQ_RUNNING) {
        r->cancel = true;
    }
    return GQIS_OK;
}

__attribute__((visibility("default"))) int gqis_serve_request_error(gqis_server* s, int64_t id, char* buf,
                                                                    int64_t len) {
    if (!s || !buf || len < 1) return fail(GQIS_ERR_INVALID, "invalid argument");
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->requests.find(id);
    if (it == s->requests.end()) return fail(GQIS_ERR_INVALID, "unknown request %lld", (long long)id);
    snprintf(buf, (size_t)len, "%s", it->second->error.c_str());
    return GQIS_OK;
}

__attribute__((visibility("default"))) int gqis_serve_close(gqis_server* s) {
    if (!s) return fail(GQIS_ERR_INVALID, "NULL server");
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stop = true;
    }
    if (s->thread.joinable()) s->thread.join();
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(s->device);
    for (cudaStream_t st : s->streams) cudaStreamDestroy(st);
    cudaFree(s->counters);
    cudaSetDevice(prev);
    delete s;  // loaded modules stay mapped (other servers or the host may use them)
    return GQIS_OK;
}

}  // extern "C"
