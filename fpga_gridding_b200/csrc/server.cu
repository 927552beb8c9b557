// Resident gridding server: continuous batching of independent jobs on one
// device.
//
// A server thread owns `num_slots` slots, each a workspace with two streams
// (the workspace's own, and one of the device's highest priority).
// Submitted jobs wait in arrival order.  Whenever a slot is free the thread
// takes the head job plus the following queued jobs that fit in the same
// launch (same precision and kernel storage, at most max_batch jobs and
// kBatchPoints visibilities) and that fit the HBM budget, allocates and
// zeroes their output grids, and enqueues one batched gridding call
// (run_batch).  Slots run concurrently, so jobs that arrive while others are
// on the device start as soon as a slot and memory are free.  Completion is
// detected by polling a CUDA event per slot; the job's skip count, norm and
// status are copied back through pinned memory.
//
// Large jobs must not hold up small ones.  A persistent gridding kernel
// keeps every SM until its task queue is empty, and a running CTA is never
// preempted, so three rules keep latency bounded under mixed sizes:
//   * a batch of at most kSmallPoints visibilities runs on the slot's
//     high-priority stream;
//   * a larger batch grids in time slices (about kSlicePoints visibilities
//     each, at most kMaxBands): its CTAs retire at each slice boundary and
//     the SMs go to waiting high-priority work first;
//   * with three or more slots the last slot takes small jobs only (the
//     first small jobs in the queue, passing large ones), so a small job
//     never waits for a slot while large jobs occupy the others.
#include <algorithm>
#include <cmath>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

#include "common.cuh"
#include "internal.h"

using namespace b200;

namespace {

constexpr size_t kBatchPoints = 8u << 20;   // visibilities per merged launch
constexpr size_t kSmallPoints = 2u << 20;   // small: high-priority stream
constexpr size_t kSlicePoints = 4u << 20;   // visibilities per time slice

struct Pending
{
    oskar_B200Request req;
    double submit_s;
    size_t grid_bytes;
};

struct Running
{
    Pending p;
    void* grid;
};

struct Slot
{
    oskar_B200Workspace* ws = nullptr;
    cudaStream_t hi = nullptr;  // highest-priority stream (small batches)
    bool small_only = false;    // reserved for small jobs
    bool busy = false;
    cudaEvent_t done = nullptr;
    DeviceBuffer outs;          // per job: skipped (u64), norm (f64)
    void* h_outs = nullptr;     // pinned mirror
    std::vector<Running> jobs;
    double start_s = 0.0;
};

// Workspace bytes a batch of n points needs (run_batch's buffers).
size_t workspace_need(size_t n)
{
    // keys and indices (twice), records, task starts and jobs, and the
    // sort's scratch: 44 bytes per point in either precision
    return n * 44u + (8u << 20);
}

}  // namespace

struct oskar_B200Server
{
    int device = 0;
    size_t budget = 0;
    int max_batch = 1;
    oskar_B200Options opt{};
    std::vector<Slot> slots;
    std::thread thread;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    bool stop = false;
    int startup_status = OSKAR_B200_OK;
    std::deque<Pending> queue;
    std::deque<oskar_B200Completion> done;
    std::unordered_map<unsigned long long, std::pair<void*, size_t>> live;
    std::multimap<size_t, void*> pool;   // released grids kept for reuse
    size_t grid_bytes = 0;               // live + pooled grid bytes
    std::chrono::steady_clock::time_point t0;

    double now() const
    {
        return std::chrono::duration<double>(
                   std::chrono::steady_clock::now() - t0).count();
    }

    size_t in_use() const
    {
        size_t b = grid_bytes;
        for (const Slot& s : slots) b += oskar_b200_workspace_bytes(s.ws);
        return b;
    }

    // A grid of `bytes` from the pool or a fresh allocation (lock held).
    void* take_grid(size_t bytes)
    {
        auto it = pool.find(bytes);
        if (it != pool.end())
        {
            void* p = it->second;
            pool.erase(it);
            return p;
        }
        void* p = nullptr;
        if (cudaMalloc(&p, bytes) != cudaSuccess)
        {
            cudaGetLastError();
            return nullptr;
        }
        grid_bytes += bytes;
        return p;
    }

    // Frees pooled grids until `need` more bytes fit the budget.
    void trim_pool(size_t need)
    {
        while (!pool.empty() && in_use() + need > budget)
        {
            auto it = pool.begin();
            cudaFree(it->second);
            grid_bytes -= it->first;
            pool.erase(it);
        }
    }

    void finish_slot(Slot& s)
    {
        const unsigned long long* c =
            static_cast<const unsigned long long*>(s.ws->h_counters);
        const int dev_status = c[CNT_STATUS]
            ? ((c[CNT_STATUS] & DEV_ERR_TIMEOUT) ? OSKAR_B200_ERR_TIMEOUT
                                    : OSKAR_B200_ERR_DEVICE_CHECK)
            : OSKAR_B200_OK;
        const cudaError_t e = cudaEventQuery(s.done);
        const int status = e == cudaSuccess ? dev_status : status_from_cuda(e);
        const double t = now();
        const unsigned long long* outs =
            static_cast<const unsigned long long*>(s.h_outs);
        for (size_t i = 0; i < s.jobs.size(); ++i)
        {
            oskar_B200Completion c1{};
            c1.tag = s.jobs[i].p.req.tag;
            c1.status = status;
            c1.num_skipped = outs[2 * i];
            double nrm;
            memcpy(&nrm, &outs[2 * i + 1], sizeof(nrm));
            c1.norm = nrm;
            c1.grid = s.jobs[i].grid;
            c1.submit_s = s.jobs[i].p.submit_s;
            c1.start_s = s.start_s;
            c1.end_s = t;
            c1.batch_size = (int)s.jobs.size();
            done.push_back(c1);
        }
        s.jobs.clear();
        s.busy = false;
    }

    void fail_head(int status)
    {
        Pending p = queue.front();
        queue.pop_front();
        oskar_B200Completion c1{};
        c1.tag = p.req.tag;
        c1.status = status;
        c1.submit_s = p.submit_s;
        c1.start_s = c1.end_s = now();
        done.push_back(c1);
    }

    // Admits queued jobs onto free slots (lock held).  Returns true if any
    // slot was started.
    bool admit()
    {
        bool started = false;
        for (Slot& s : slots)
        {
            if (s.busy || queue.empty()) continue;
            // The batch: a general slot takes the head and the following
            // compatible jobs that fit; a small-only slot takes the first
            // small job and the following compatible small ones, passing
            // large ones.
            std::vector<size_t> pick;
            const oskar_B200Cube* c0 = nullptr;
            size_t n = 0, gbytes = 0;
            const size_t have = oskar_b200_workspace_bytes(s.ws);
            for (size_t qi = 0; qi < queue.size(); ++qi)
            {
                const Pending& p = queue[qi];
                if (s.small_only && p.req.num_points > kSmallPoints) continue;
                if ((int)pick.size() >= max_batch) break;
                if (c0 && (p.req.cube->data_is_double != c0->data_is_double ||
                           p.req.cube->kernel_type != c0->kernel_type))
                {
                    if (s.small_only) continue;
                    break;
                }
                if (!pick.empty() && n + p.req.num_points > kBatchPoints) break;
                const size_t ws_need = workspace_need(n + p.req.num_points);
                const size_t grow = ws_need > have ? ws_need - have : 0;
                trim_pool(grow + gbytes + p.grid_bytes);
                if (in_use() + grow + gbytes + p.grid_bytes > budget) break;
                if (!c0) c0 = p.req.cube;
                n += p.req.num_points;
                gbytes += p.grid_bytes;
                pick.push_back(qi);
            }
            if (pick.empty())
            {
                if (s.small_only) continue;
                // The head does not fit now; if nothing runs it never will.
                bool any_busy = false;
                for (const Slot& o : slots) any_busy |= o.busy;
                if (!any_busy)
                {
                    fail_head(OSKAR_B200_ERR_OVER_BUDGET);
                    started = true;
                }
                break;
            }
            // Take the picked jobs out of the queue, keeping the order of
            // the others.
            std::vector<Pending> batch;
            batch.reserve(pick.size());
            for (size_t k = pick.size(); k-- > 0;)
            {
                batch.push_back(queue[pick[k]]);
                queue.erase(queue.begin() + (std::ptrdiff_t)pick[k]);
            }
            std::reverse(batch.begin(), batch.end());
            const size_t count = batch.size();
            const bool small = n <= kSmallPoints;
            const int slices = small ? 1 : (int)std::min<size_t>(
                (size_t)kMaxBands, (n + kSlicePoints - 1) / kSlicePoints);
            std::vector<HostJob> jobs(count);
            s.jobs.clear();
            cudaStream_t st = small ? s.hi : s.ws->stream;
            bool ok = true;
            for (size_t i = 0; i < count; ++i)
            {
                Pending p = batch[i];
                void* g = take_grid(p.grid_bytes);
                if (!g || cudaMemsetAsync(g, 0, p.grid_bytes, st) != cudaSuccess)
                {
                    // Put this job and the rest back at the head.
                    ok = false;
                    for (size_t r = count; r-- > i;)
                        queue.push_front(batch[r]);
                    break;
                }
                live[p.req.tag] = std::make_pair(g, p.grid_bytes);
                s.jobs.push_back(Running{p, g});
                unsigned long long* outs =
                    static_cast<unsigned long long*>(s.outs.ptr) + 2 * i;
                jobs[i] = HostJob{p.req.cube, p.req.num_points, p.req.uu,
                                  p.req.vv, p.req.ww, p.req.vis, p.req.weight,
                                  p.req.cell_size_rad, p.req.w_scale,
                                  p.req.grid_size, g, outs,
                                  reinterpret_cast<double*>(outs + 1),
                                  p.req.frequency_hz};
            }
            if (!ok && s.jobs.empty()) break;
            jobs.resize(s.jobs.size());
            cudaMemsetAsync(s.outs.ptr, 0, 16 * jobs.size(), st);
            int rs = run_batch(s.ws, &opt, (int)jobs.size(), jobs.data(), st,
                               false, nullptr, slices);
            if (rs == OSKAR_B200_OK)
            {
                cudaMemcpyAsync(s.h_outs, s.outs.ptr, 16 * jobs.size(),
                                cudaMemcpyDeviceToHost, st);
                cudaEventRecord(s.done, st);
                s.start_s = now();
                s.busy = true;
            }
            else
            {
                const double t = now();
                for (const Running& r : s.jobs)
                {
                    oskar_B200Completion c1{};
                    c1.tag = r.p.req.tag;
                    c1.status = rs;
                    c1.grid = r.grid;
                    c1.submit_s = r.p.submit_s;
                    c1.start_s = c1.end_s = t;
                    c1.batch_size = (int)s.jobs.size();
                    done.push_back(c1);
                }
                s.jobs.clear();
            }
            started = true;
        }
        return started;
    }

    void loop()
    {
        cudaSetDevice(device);
        std::unique_lock<std::mutex> lock(mu);
        for (;;)
        {
            bool any_busy = false, finished = false;
            for (Slot& s : slots)
            {
                if (!s.busy) continue;
                const cudaError_t e = cudaEventQuery(s.done);
                if (e == cudaErrorNotReady)
                {
                    any_busy = true;
                    continue;
                }
                finish_slot(s);
                finished = true;
            }
            const bool started = admit();
            if (finished || started) cv_done.notify_all();
            for (const Slot& s : slots) any_busy |= s.busy;
            if (stop && queue.empty() && !any_busy) break;
            if (!any_busy && !started)
            {
                // Idle: sleep until a submit, a release or stop.
                cv_work.wait_for(lock, std::chrono::milliseconds(50));
            }
            else
            {
                // Jobs in flight: poll their events about every 10 us.
                lock.unlock();
                std::this_thread::sleep_for(std::chrono::microseconds(10));
                lock.lock();
            }
        }
    }
};

extern "C" {

int oskar_b200_server_create(int device, size_t hbm_budget_bytes,
                             int num_slots, int max_batch_jobs,
                             const oskar_B200Options* opt,
                             oskar_B200Server** server)
{
    if (!server || num_slots < 1 || num_slots > 64 || max_batch_jobs < 1 ||
        max_batch_jobs > 1024 || hbm_budget_bytes == 0)
        return OSKAR_B200_ERR_INVALID_ARGUMENT;
    *server = nullptr;
    auto* s = new (std::nothrow) oskar_B200Server();
    if (!s) return OSKAR_B200_ERR_OUT_OF_MEMORY;
    s->device = device;
    s->budget = hbm_budget_bytes;
    s->max_batch = max_batch_jobs;
    oskar_b200_options_init(&s->opt);
    if (opt) s->opt = *opt;
    s->slots.resize((size_t)num_slots);
    int prev = 0;
    cudaGetDevice(&prev);
    int st = OSKAR_B200_OK;
    int least_prio = 0, greatest_prio = 0;
    for (Slot& sl : s->slots)
    {
        st = oskar_b200_workspace_create(device, &sl.ws);
        if (st) break;
        cudaSetDevice(device);
        cudaDeviceGetStreamPriorityRange(&least_prio, &greatest_prio);
        if (cudaStreamCreateWithPriority(&sl.hi, cudaStreamNonBlocking,
                                         greatest_prio) != cudaSuccess)
        {
            cudaGetLastError();
            st = OSKAR_B200_ERR_CUDA;
            break;
        }
        if (cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming) !=
                cudaSuccess ||
            sl.outs.ensure(16 * (size_t)max_batch_jobs) != cudaSuccess ||
            cudaMallocHost(&sl.h_outs, 16 * (size_t)max_batch_jobs) !=
                cudaSuccess)
        {
            st = OSKAR_B200_ERR_OUT_OF_MEMORY;
            break;
        }
    }
    cudaSetDevice(prev);
    if (st)
    {
        for (Slot& sl : s->slots)
        {
            if (sl.done) cudaEventDestroy(sl.done);
            if (sl.hi) cudaStreamDestroy(sl.hi);
            if (sl.h_outs) cudaFreeHost(sl.h_outs);
            sl.outs.release();
            if (sl.ws) oskar_b200_workspace_free(sl.ws);
        }
        delete s;
        return st;
    }
    if (num_slots >= 3) s->slots.back().small_only = true;
    s->t0 = std::chrono::steady_clock::now();
    s->thread = std::thread([s] { s->loop(); });
    *server = s;
    return OSKAR_B200_OK;
}

int oskar_b200_server_submit(oskar_B200Server* s, const oskar_B200Request* r)
{
    if (!s || !r || !r->cube || r->cube->device != s->device ||
        r->grid_size < 1 || r->grid_size > 65535 ||
        (r->num_points && (!r->uu || !r->vv || !r->ww || !r->vis)) ||
        (s->opt.apply_weight && r->num_points && !r->weight) ||
        !(r->frequency_hz >= 0.0) || !std::isfinite(r->frequency_hz))
        return OSKAR_B200_ERR_INVALID_ARGUMENT;
    Pending p;
    p.req = *r;
    p.grid_bytes = (size_t)r->grid_size * r->grid_size * 2 *
                   (r->cube->data_is_double ? sizeof(double) : sizeof(float));
    {
        std::lock_guard<std::mutex> lock(s->mu);
        if (s->stop) return OSKAR_B200_ERR_INVALID_ARGUMENT;
        p.submit_s = s->now();
        s->queue.push_back(p);
    }
    s->cv_work.notify_one();
    return OSKAR_B200_OK;
}

int oskar_b200_server_poll(oskar_B200Server* s, oskar_B200Completion* out,
                           int max_out, int* num_out, double timeout_s)
{
    if (!s || !out || !num_out || max_out < 1)
        return OSKAR_B200_ERR_INVALID_ARGUMENT;
    std::unique_lock<std::mutex> lock(s->mu);
    if (s->done.empty() && timeout_s > 0)
        s->cv_done.wait_for(lock, std::chrono::duration<double>(timeout_s),
                            [s] { return !s->done.empty(); });
    int n = 0;
    while (n < max_out && !s->done.empty())
    {
        out[n++] = s->done.front();
        s->done.pop_front();
    }
    *num_out = n;
    return OSKAR_B200_OK;
}

int oskar_b200_server_release(oskar_B200Server* s, unsigned long long tag)
{
    if (!s) return OSKAR_B200_ERR_INVALID_ARGUMENT;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        auto it = s->live.find(tag);
        if (it == s->live.end()) return OSKAR_B200_ERR_INVALID_ARGUMENT;
        s->pool.insert(std::make_pair(it->second.second, it->second.first));
        s->live.erase(it);
    }
    s->cv_work.notify_one();
    return OSKAR_B200_OK;
}

double oskar_b200_server_clock(oskar_B200Server* s)
{
    return s ? s->now() : 0.0;
}

int oskar_b200_server_memory(oskar_B200Server* s, size_t* bytes_in_use,
                             size_t* budget)
{
    if (!s) return OSKAR_B200_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(s->mu);
    if (bytes_in_use) *bytes_in_use = s->in_use();
    if (budget) *budget = s->budget;
    return OSKAR_B200_OK;
}

int oskar_b200_server_free(oskar_B200Server* s)
{
    if (!s) return OSKAR_B200_OK;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->thread.joinable()) s->thread.join();
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(s->device);
    for (auto& kv : s->live) cudaFree(kv.second.first);
    for (auto& kv : s->pool) cudaFree(kv.second);
    for (Slot& sl : s->slots)
    {
        if (sl.done) cudaEventDestroy(sl.done);
        if (sl.hi) cudaStreamDestroy(sl.hi);
        if (sl.h_outs) cudaFreeHost(sl.h_outs);
        sl.outs.release();
        oskar_b200_workspace_free(sl.ws);
    }
    cudaSetDevice(prev);
    delete s;
    return OSKAR_B200_OK;
}

}  // extern "C"
