// cv_server.cu -- a persistent request loop over a filter batch
// (continuous batching of streamed constant-velocity filters).
//
// No counterpart in the reference (vSMC drives one Sampler per filter from
// the caller's thread, core/sampler.hpp:450-483).  Clients open filter
// requests of any particle count and stream observations to them, from any
// thread.  One loop thread owns a vsmc_cuda_cv_batch on its own stream and
// repeats a tick:
//
//   1. release the slots of requests that are closed and fully processed;
//   2. admit waiting requests in arrival order while a slot and the HBM
//      budget allow (a request that does not fit waits for memory to free);
//   3. take up to kCatchUp of the oldest pending observations of every
//      admitted request and run them together: append them, step every
//      filter through its own (one launch sequence per step over the
//      filters still stepping), read the steps back once;
//   4. publish one result per observation with its arrival and completion
//      times.
//
// A request whose observations arrive faster than ticks complete catches
// up several steps in one tick instead of one per tick, so the loop's fixed
// cost per tick (staging, the read-back, the host round trip) is shared by
// more steps as the load rises.
//
// Requests that arrive while a tick runs join the next tick, so their work
// shares launches with the filters already on the device.  Each filter's
// results equal those of the filter run alone (the batch guarantees that),
// whatever it was batched with.
#include "../../include/vsmc_cuda.h"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

namespace vsmc_b200 {
void set_last_error(const std::string &msg);
int cuda_status(cudaError_t e, const char *what);
} // namespace vsmc_b200

using namespace vsmc_b200;

namespace {

struct PendingObs {
    double x, y;
    int64_t submit_ns;
};

struct Request {
    uint64_t N = 0, T_max = 0;
    uint32_t seed = 0, stream_id = 0;
    int64_t slot = -1;      // -1 until admitted
    uint64_t submitted = 0; // observations accepted
    uint64_t stepped = 0;   // observations processed
    std::deque<PendingObs> pending;
    bool closed = false;
    int32_t status = VSMC_CUDA_OK;
    double logz = 0.0; // running log-evidence, summed as the device sums it
};

constexpr uint32_t kCatchUp = 32; // steps per request per tick at most

} // namespace

struct vsmc_cuda_cv_server {
    vsmc_cuda_cv_config model;
    uint32_t max_filters;
    uint64_t budget;
    int device;
    cudaStream_t stream;
    vsmc_cuda_cv_batch *batch;
    std::chrono::steady_clock::time_point t0;

    std::mutex mu;
    std::condition_variable work_cv;   // new requests / observations / stop
    std::condition_variable result_cv; // new results / drained
    bool stop;
    uint64_t next_id;
    std::unordered_map<uint64_t, Request> reqs;
    std::deque<uint64_t> waiting; // not yet admitted, arrival order
    std::vector<uint64_t> active; // admitted, admission order
    std::deque<vsmc_cuda_cv_result> results;
    uint64_t obs_submitted, obs_done;
    vsmc_cuda_cv_server_counters st;
    int loop_status;
    std::string loop_error;
    std::thread loop;

    int64_t now_ns() const
    {
        return std::chrono::duration_cast<std::chrono::nanoseconds>(
                   std::chrono::steady_clock::now() - t0)
            .count();
    }

    void run();
};

void vsmc_cuda_cv_server::run()
{
    cudaSetDevice(device);
    std::vector<uint32_t> release, tick_slots, counts, round_slots;
    std::vector<uint64_t> tick_ids, tick_t;
    std::vector<double> xs, ys, rx, ry, ess, dz;
    std::vector<int32_t> res, status;
    std::vector<int64_t> sub;
    struct Candidate {
        uint64_t id, N, T_max;
        uint32_t seed, stream_id;
    };
    std::vector<Candidate> cand;
    bool blocked = false; // admission waits for a release
    for (;;) {
        release.clear();
        cand.clear();
        {
            std::unique_lock<std::mutex> lk(mu);
            for (;;) {
                if (stop)
                    return;
                // 1. finished requests
                for (size_t k = 0; k < active.size();) {
                    Request &r = reqs[active[k]];
                    if (r.closed && r.pending.empty()) {
                        release.push_back((uint32_t)r.slot);
                        reqs.erase(active[k]);
                        active.erase(active.begin() + (long)k);
                        ++st.completed;
                    } else {
                        ++k;
                    }
                }
                while (!waiting.empty()) {
                    auto it = reqs.find(waiting.front());
                    if (it != reqs.end() && !(it->second.closed &&
                                              it->second.pending.empty()))
                        break;
                    if (it != reqs.end()) { // closed before admission
                        reqs.erase(it);
                        ++st.completed;
                    }
                    waiting.pop_front();
                }
                for (uint64_t id : waiting) {
                    const Request &r = reqs[id];
                    cand.push_back(
                        Candidate{id, r.N, r.T_max, r.seed, r.stream_id});
                }
                bool pending = false;
                for (uint64_t id : active)
                    if (!reqs[id].pending.empty()) {
                        pending = true;
                        break;
                    }
                if (!release.empty())
                    blocked = false;
                if (!release.empty() || pending ||
                    (!cand.empty() && !blocked &&
                     active.size() < max_filters))
                    break;
                cand.clear();
                work_cv.wait(lk);
            }
        }
        // 2. release, then admit in arrival order
        for (uint32_t s : release)
            vsmc_cuda_cv_batch_release(batch, s);
        std::vector<std::pair<uint64_t, uint32_t>> got;
        int refused = VSMC_CUDA_OK;
        for (const Candidate &c : cand) {
            uint32_t slot = 0;
            const int rc = vsmc_cuda_cv_batch_admit(batch, c.N, c.T_max,
                                                    c.seed, c.stream_id,
                                                    &slot);
            if (rc != VSMC_CUDA_OK) {
                // no slot or memory: wait for releases (in arrival order)
                refused = rc;
                blocked = true;
                break;
            }
            got.emplace_back(c.id, slot);
        }
        // 3. up to kCatchUp observations of each admitted request with any
        // pending, packed request by request
        tick_slots.clear();
        tick_ids.clear();
        tick_t.clear();
        counts.clear();
        xs.clear();
        ys.clear();
        sub.clear();
        {
            std::lock_guard<std::mutex> lk(mu);
            for (auto &g : got) {
                Request &r = reqs[g.first];
                r.slot = g.second;
                active.push_back(g.first);
                waiting.pop_front();
                ++st.admitted;
            }
            if (refused != VSMC_CUDA_OK && active.empty() &&
                !waiting.empty()) {
                // nothing on the device will free memory: the request at
                // the head can never be admitted; fail it
                const uint64_t id = waiting.front();
                waiting.pop_front();
                Request &r = reqs[id];
                const int64_t now = now_ns();
                for (uint64_t t = 0; t < r.pending.size(); ++t) {
                    vsmc_cuda_cv_result e;
                    std::memset(&e, 0, sizeof(e));
                    e.request = id;
                    e.t = t;
                    e.status = refused;
                    e.submit_ns = r.pending[t].submit_ns;
                    e.done_ns = now;
                    results.push_back(e);
                }
                obs_done += r.pending.size();
                r.pending.clear();
                r.status = refused;
                r.closed = true;
                reqs.erase(id);
                ++st.completed;
                blocked = false;
                result_cv.notify_all();
            }
            for (uint64_t id : active) {
                Request &r = reqs[id];
                if (r.pending.empty())
                    continue;
                const uint32_t m = (uint32_t)std::min<size_t>(
                    r.pending.size(), (size_t)kCatchUp);
                tick_slots.push_back((uint32_t)r.slot);
                tick_ids.push_back(id);
                tick_t.push_back(r.stepped);
                counts.push_back(m);
                for (uint32_t j = 0; j < m; ++j) {
                    const PendingObs o = r.pending.front();
                    r.pending.pop_front();
                    xs.push_back(o.x);
                    ys.push_back(o.y);
                    sub.push_back(o.submit_ns);
                }
                r.stepped += m;
            }
            if (active.size() > st.max_active)
                st.max_active = active.size();
        }
        if (tick_slots.empty())
            continue;
        const int64_t begin = now_ns();
        const uint32_t n = (uint32_t)tick_slots.size();
        const size_t total = xs.size();
        uint32_t maxm = 0;
        for (uint32_t m : counts)
            maxm = std::max(maxm, m);
        ess.assign(total, 0.0);
        dz.assign(total, 0.0);
        res.assign(total, 0);
        status.assign(n, 0);
        // append round j: observation j of every request with more than j
        int rc = VSMC_CUDA_OK;
        for (uint32_t j = 0; j < maxm && rc == VSMC_CUDA_OK; ++j) {
            round_slots.clear();
            rx.clear();
            ry.clear();
            size_t off = 0;
            for (uint32_t k = 0; k < n; ++k) {
                if (counts[k] > j) {
                    round_slots.push_back(tick_slots[k]);
                    rx.push_back(xs[off + j]);
                    ry.push_back(ys[off + j]);
                }
                off += counts[k];
            }
            rc = vsmc_cuda_cv_batch_append_observations(
                batch, (uint32_t)round_slots.size(), round_slots.data(),
                rx.data(), ry.data());
        }
        // every filter steps through its appended observations
        if (rc == VSMC_CUDA_OK)
            rc = vsmc_cuda_cv_batch_run(batch, n, tick_slots.data());
        if (rc == VSMC_CUDA_OK || rc == VSMC_CUDA_EDEGENERATE)
            rc = vsmc_cuda_cv_batch_read_steps(batch, n, tick_slots.data(),
                                               counts.data(), ess.data(),
                                               dz.data(), res.data(),
                                               status.data());
        const int64_t done = now_ns();
        const bool fatal = rc != VSMC_CUDA_OK && rc != VSMC_CUDA_EDEGENERATE;
        uint64_t psteps = 0;
        {
            std::lock_guard<std::mutex> lk(mu);
            if (fatal && loop_status == VSMC_CUDA_OK) {
                loop_status = rc;
                loop_error = "tick failed (status " + std::to_string(rc) + ")";
            }
            size_t off = 0;
            for (uint32_t k = 0; k < n; ++k) {
                auto it = reqs.find(tick_ids[k]);
                double lz = it != reqs.end() ? it->second.logz : 0.0;
                for (uint32_t j = 0; j < counts[k]; ++j) {
                    const size_t i = off + j;
                    vsmc_cuda_cv_result r;
                    r.request = tick_ids[k];
                    r.t = tick_t[k] + j;
                    r.ess = ess[i];
                    r.logz_inc = dz[i];
                    lz = lz + dz[i];
                    r.log_evidence = lz;
                    r.resampled = res[i];
                    // a step's status: the slot's sticky status from the
                    // step whose ESS it made undefined (the weights turned
                    // degenerate there), and on the tick's last step
                    const bool hit = ess[i] != ess[i] || j + 1 == counts[k];
                    r.status = fatal ? rc
                                     : (hit ? status[k] : VSMC_CUDA_OK);
                    r.submit_ns = sub[i];
                    r.done_ns = done;
                    results.push_back(r);
                    if (it != reqs.end() && r.status != VSMC_CUDA_OK)
                        it->second.status = r.status;
                }
                if (it != reqs.end()) {
                    it->second.logz = lz;
                    psteps += it->second.N * counts[k];
                }
                off += counts[k];
            }
            obs_done += total;
            ++st.ticks;
            st.steps += total;
            st.particle_steps += psteps;
            st.busy_seconds += (double)(done - begin) * 1e-9;
        }
        result_cv.notify_all();
    }
}

extern "C" {

int vsmc_cuda_cv_server_create(const vsmc_cuda_cv_config *model,
                               uint32_t max_filters, uint64_t hbm_budget,
                               vsmc_cuda_cv_server **out)
{
    if (out == nullptr || model == nullptr || max_filters == 0) {
        set_last_error("vsmc_cuda_cv_server_create: invalid arguments");
        return VSMC_CUDA_EINVAL;
    }
    *out = nullptr;
    vsmc_cuda_cv_server *s = new (std::nothrow) vsmc_cuda_cv_server();
    if (s == nullptr)
        return VSMC_CUDA_ENOMEM;
    s->model = *model;
    s->max_filters = max_filters;
    s->budget = hbm_budget;
    s->stop = false;
    s->next_id = 1;
    s->obs_submitted = s->obs_done = 0;
    std::memset(&s->st, 0, sizeof(s->st));
    s->loop_status = VSMC_CUDA_OK;
    s->t0 = std::chrono::steady_clock::now();
    cudaError_t e = cudaGetDevice(&s->device);
    if (e == cudaSuccess)
        e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete s;
        return cuda_status(e, "vsmc_cuda_cv_server_create");
    }
    int rc = vsmc_cuda_cv_batch_create(model, max_filters, hbm_budget,
                                       s->stream, &s->batch);
    if (rc != VSMC_CUDA_OK) {
        cudaStreamDestroy(s->stream);
        delete s;
        return rc;
    }
    // ticks differ in their filters and step counts: direct launches
    vsmc_cuda_cv_batch_set_graphs(s->batch, 0);
    try {
        s->loop = std::thread([s] { s->run(); });
    } catch (...) {
        vsmc_cuda_cv_batch_destroy(s->batch);
        cudaStreamDestroy(s->stream);
        delete s;
        set_last_error("vsmc_cuda_cv_server_create: no loop thread");
        return VSMC_CUDA_ENOMEM;
    }
    *out = s;
    return VSMC_CUDA_OK;
}

int vsmc_cuda_cv_server_destroy(vsmc_cuda_cv_server *s)
{
    if (s == nullptr)
        return VSMC_CUDA_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->work_cv.notify_all();
    s->result_cv.notify_all();
    if (s->loop.joinable())
        s->loop.join();
    int rc = vsmc_cuda_cv_batch_destroy(s->batch);
    cudaStreamDestroy(s->stream);
    delete s;
    return rc;
}

int64_t vsmc_cuda_cv_server_now_ns(vsmc_cuda_cv_server *s)
{
    return s == nullptr ? 0 : s->now_ns();
}

int vsmc_cuda_cv_server_open(vsmc_cuda_cv_server *s, uint64_t N,
                             uint64_t T_max, uint32_t seed,
                             uint32_t stream_id, uint64_t *request)
{
    if (s == nullptr || request == nullptr || N < 2 || N > (1ull << 30) ||
        T_max < 1 || T_max > (1ull << 31)) {
        set_last_error("vsmc_cuda_cv_server_open: invalid arguments");
        return VSMC_CUDA_EINVAL;
    }
    if (s->budget != 0 &&
        vsmc_cuda_cv_batch_slot_bytes(&s->model, N, T_max) > s->budget) {
        set_last_error("vsmc_cuda_cv_server_open: the filter alone exceeds "
                       "the HBM budget");
        return VSMC_CUDA_ENOMEM;
    }
    {
        std::lock_guard<std::mutex> lk(s->mu);
        const uint64_t id = s->next_id++;
        Request &r = s->reqs[id];
        r.N = N;
        r.T_max = T_max;
        r.seed = seed;
        r.stream_id = stream_id;
        s->waiting.push_back(id);
        ++s->st.opened;
        *request = id;
    }
    s->work_cv.notify_one();
    return VSMC_CUDA_OK;
}

int vsmc_cuda_cv_server_observe(vsmc_cuda_cv_server *s, uint32_t n,
                                const uint64_t *requests, const double *x,
                                const double *y, const int64_t *submit_ns)
{
    if (s == nullptr || (n > 0 && (requests == nullptr || x == nullptr ||
                                   y == nullptr))) {
        set_last_error("vsmc_cuda_cv_server_observe: invalid arguments");
        return VSMC_CUDA_EINVAL;
    }
    const int64_t now = s->now_ns();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        for (uint32_t k = 0; k < n; ++k) {
            auto it = s->reqs.find(requests[k]);
            if (it == s->reqs.end() || it->second.closed ||
                it->second.submitted >= it->second.T_max) {
                set_last_error("vsmc_cuda_cv_server_observe: request " +
                               std::to_string(requests[k]) +
                               " is unknown, closed or full");
                return VSMC_CUDA_EINVAL;
            }
        }
        for (uint32_t k = 0; k < n; ++k) {
            Request &r = s->reqs[requests[k]];
            r.pending.push_back(
                PendingObs{x[k], y[k], submit_ns ? submit_ns[k] : now});
            ++r.submitted;
        }
        s->obs_submitted += n;
    }
    s->work_cv.notify_one();
    return VSMC_CUDA_OK;
}

int vsmc_cuda_cv_server_close(vsmc_cuda_cv_server *s, uint64_t request)
{
    if (s == nullptr)
        return VSMC_CUDA_EINVAL;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->reqs.find(request);
        if (it == s->reqs.end() || it->second.closed) {
            set_last_error("vsmc_cuda_cv_server_close: unknown request");
            return VSMC_CUDA_EINVAL;
        }
        it->second.closed = true;
    }
    s->work_cv.notify_one();
    return VSMC_CUDA_OK;
}

int vsmc_cuda_cv_server_poll(vsmc_cuda_cv_server *s, vsmc_cuda_cv_result *out,
                             uint32_t max, uint32_t *n, int wait_ms)
{
    if (s == nullptr || n == nullptr || (max > 0 && out == nullptr))
        return VSMC_CUDA_EINVAL;
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->results.empty() && wait_ms > 0)
        s->result_cv.wait_for(lk, std::chrono::milliseconds(wait_ms), [s] {
            return !s->results.empty() || s->stop ||
                   s->loop_status != VSMC_CUDA_OK;
        });
    uint32_t k = 0;
    while (k < max && !s->results.empty()) {
        out[k++] = s->results.front();
        s->results.pop_front();
    }
    *n = k;
    if (s->loop_status != VSMC_CUDA_OK) {
        set_last_error("vsmc_cuda_cv_server: " + s->loop_error);
        return s->loop_status;
    }
    return VSMC_CUDA_OK;
}

int vsmc_cuda_cv_server_drain(vsmc_cuda_cv_server *s, int timeout_ms)
{
    if (s == nullptr)
        return VSMC_CUDA_EINVAL;
    std::unique_lock<std::mutex> lk(s->mu);
    const bool ok = s->result_cv.wait_for(
        lk, std::chrono::milliseconds(timeout_ms), [s] {
            return s->obs_done == s->obs_submitted ||
                   s->loop_status != VSMC_CUDA_OK;
        });
    if (s->loop_status != VSMC_CUDA_OK) {
        set_last_error("vsmc_cuda_cv_server: " + s->loop_error);
        return s->loop_status;
    }
    if (!ok) {
        set_last_error("vsmc_cuda_cv_server_drain: timed out");
        return VSMC_CUDA_ETIMEOUT;
    }
    return VSMC_CUDA_OK;
}

int vsmc_cuda_cv_server_stats(vsmc_cuda_cv_server *s,
                              vsmc_cuda_cv_server_counters *out)
{
    if (s == nullptr || out == nullptr)
        return VSMC_CUDA_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    *out = s->st;
    out->waiting = s->waiting.size();
    out->active = s->active.size();
    return VSMC_CUDA_OK;
}

} // extern "C"
