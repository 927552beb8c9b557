// Gridding of a batch of jobs on device-resident data:
//   prep (placement, keys, norms, skip counts, plane histograms)
//   -> one radix sort of (key, index) over all jobs (job in the top bits)
//   -> task list (tasks never cross a job, tile or plane)
//   -> one persistent Romein gridding launch over every task of every job;
//      each task gathers its points' records and visibilities through the
//      sorted index (no separate permutation pass).
// A single oskar_b200_grid call is a batch of one job.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "grid_romein.cuh"
#include "internal.h"
#include "prep.cuh"

namespace b200 {

int status_from_cuda(cudaError_t e)
{
    switch (e)
    {
    case cudaSuccess: return OSKAR_B200_OK;
    case cudaErrorMemoryAllocation: return OSKAR_B200_ERR_OUT_OF_MEMORY;
    case cudaErrorNoDevice:
    case cudaErrorInsufficientDriver:
    case cudaErrorNoKernelImageForDevice: return OSKAR_B200_ERR_NO_DEVICE;
    case cudaErrorInvalidValue: return OSKAR_B200_ERR_INVALID_ARGUMENT;
    default: return OSKAR_B200_ERR_CUDA;
    }
}

// Allocation failures injected for tests (oskar_b200_testing_fail_allocation):
// the number of device allocations still to succeed before one fails, or -1.
std::atomic<long long> g_alloc_countdown{-1};

cudaError_t DeviceBuffer::ensure(size_t n)
{
    if (n <= bytes && ptr) return cudaSuccess;
    release();
    long long left = g_alloc_countdown.load();
    while (left >= 0 &&
           !g_alloc_countdown.compare_exchange_weak(left, left - 1))
    {
    }
    if (left == 0) return cudaErrorMemoryAllocation;
    const size_t granule = 2u << 20;
    const size_t want = n == 0 ? granule : (n + granule - 1) / granule * granule;
    cudaError_t e = cudaMalloc(&ptr, want);
    if (e != cudaSuccess)
    {
        ptr = nullptr;
        bytes = 0;
        cudaGetLastError();  // clear the allocation error
        return e;
    }
    bytes = want;
    return cudaSuccess;
}

void DeviceBuffer::release()
{
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
}

DeviceBuffer::~DeviceBuffer() { release(); }

#define B200_TRY(expr)                                      \
    do {                                                    \
        const cudaError_t e_ = (expr);                      \
        if (e_ != cudaSuccess) return status_from_cuda(e_); \
    } while (0)

double coord_scale_of(double frequency_hz)
{
    return frequency_hz > 0.0 ? frequency_hz / 299792458.0 : 1.0;
}

int run_batch(oskar_B200Workspace* ws, const oskar_B200Options* opt,
              int num_jobs, const HostJob* jobs, cudaStream_t st,
              bool degrid, BandPlan* bands, int time_slices)
{
    if (time_slices < 1 || time_slices > kMaxBands ||
        (time_slices > 1 && (bands || degrid)))
        return OSKAR_B200_ERR_INVALID_ARGUMENT;
    // (the error grid is folded in after the last band: not band-ordered)
    if (bands && (num_jobs != 1 || degrid || !bands->events ||
                  opt->accum_mode == OSKAR_B200_ACCUM_COMPENSATED))
        return OSKAR_B200_ERR_INVALID_ARGUMENT;
    const oskar_B200Cube* c0 = jobs[0].cube;
    const bool dbl = c0->data_is_double != 0;
    const bool comp = !degrid &&
                      opt->accum_mode == OSKAR_B200_ACCUM_COMPENSATED;
    int launches = 0;
    ws->last_launches = 0;
    ws->events_recorded = 0;
    const bool timing = ws->stage_timing != 0;
    auto mark = [&](int i) -> cudaError_t {
        return timing ? cudaEventRecord(ws->events[i], st) : cudaSuccess;
    };

    // Job table (host, pinned: it is the source of an async upload).
    size_t n = 0, max_points = 0, comp_floats = 0;
    int max_grid = 1, max_planes = 1;
    unsigned max_block = 0;
    for (int j = 0; j < num_jobs; ++j)
    {
        n += jobs[j].num_points;
        max_points = std::max(max_points, jobs[j].num_points);
        max_grid = std::max(max_grid, jobs[j].grid_size);
        max_planes = std::max(max_planes, jobs[j].cube->num_planes);
        max_block = std::max(max_block, jobs[j].cube->max_block_bytes);
        if (comp)
            comp_floats += 2 * (size_t)jobs[j].grid_size * jobs[j].grid_size;
    }
    if (n >= 0xffffffffull) return OSKAR_B200_ERR_INVALID_ARGUMENT;
    ws->last_points = n;
    KeyLayout kl;
    // Launch shape: the options', else the workspace's tuned one.
    const int tile_shift = opt->tile_shift > 0 ? opt->tile_shift
                           : ws->tuned_launch ? ws->tuned_tile_shift : 0;
    if (!make_key_layout(max_grid, max_planes, num_jobs, &kl, tile_shift))
        return OSKAR_B200_ERR_UNSUPPORTED;
    if (bands)
    {
        bands->row_shift = kl.coarse_shift;
        bands->num_bands = (max_grid + (1 << kl.coarse_shift) - 1) >>
                           kl.coarse_shift;
        bands->halo = c0->max_support;
        if (bands->num_bands > kMaxBands) return OSKAR_B200_ERR_UNSUPPORTED;
        for (int i = 0, lo = 0, hi = bands->num_bands - 1; lo <= hi; ++i)
            bands->order[i] = (i & 1) ? hi-- : lo++;
        // (the layout already holds: at most 16 coarse tiles per axis)
        B200_TRY(ws->bands.ensure(256));
    }
    if (time_slices > 1) B200_TRY(ws->bands.ensure(256));
    // Every band event is recorded on every successful path.
    auto record_bands = [&]() -> cudaError_t {
        if (!bands) return cudaSuccess;
        for (int b = 0; b < bands->num_bands; ++b)
        {
            const cudaError_t e = cudaEventRecord(bands->events[b], st);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    };
    const size_t job_bytes = sizeof(JobDesc) * num_jobs;
    cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
    B200_TRY(cudaStreamIsCapturing(st, &capture));
    const bool capturing = capture != cudaStreamCaptureStatusNone;
    // The job table goes up from the next pinned buffer of the ring; the
    // upload that last read that buffer must have happened before it is
    // rewritten.  (A caller capturing a graph has synchronised.)
    // Every buffer of the ring is (re)allocated together, so that a call
    // being captured into a graph after one that sized them allocates
    // nothing; in steps of 64 KiB (256 jobs), since freeing pinned memory
    // can wait for the whole device (a server growing its batches one job
    // at a time stalled every slot on each step).
    const size_t ring_bytes = (job_bytes + 65535) / 65536 * 65536;
    if (ws->h_jobs_bytes[0] < job_bytes)
    {
        for (int r = 0; r < kJobRing; ++r)
        {
            if (ws->jobs_event_pending[r] && !capturing)
                B200_TRY(cudaEventSynchronize(ws->jobs_event[r]));
            ws->jobs_event_pending[r] = 0;
            if (ws->h_jobs[r]) cudaFreeHost(ws->h_jobs[r]);
            ws->h_jobs[r] = nullptr;
            ws->h_jobs_bytes[r] = 0;
        }
        for (int r = 0; r < kJobRing; ++r)
        {
            B200_TRY(cudaMallocHost(&ws->h_jobs[r], ring_bytes));
            ws->h_jobs_bytes[r] = ring_bytes;
        }
    }
    const int slot = ws->jobs_slot;
    ws->jobs_slot = (slot + 1) % kJobRing;
    if (ws->jobs_event_pending[slot] && !capturing)
        B200_TRY(cudaEventSynchronize(ws->jobs_event[slot]));
    ws->jobs_event_pending[slot] = 0;
    if (comp) B200_TRY(ws->comp_grid.ensure(comp_floats * sizeof(float)));
    JobDesc* hj = static_cast<JobDesc*>(ws->h_jobs[slot]);
    size_t first = 0, comp_off = 0;
    for (int j = 0; j < num_jobs; ++j)
    {
        const HostJob& h = jobs[j];
        const oskar_B200Cube* c = h.cube;
        JobDesc d{};
        d.uu = h.uu;
        d.vv = h.vv;
        d.ww = h.ww;
        d.vis = h.vis;
        d.weight = h.weight;
        d.grid = h.grid;
        d.comp = comp ? static_cast<float*>(ws->comp_grid.ptr) + comp_off
                      : nullptr;
        d.planes = static_cast<const PlaneDesc*>(c->d_planes.ptr);
        d.slabs = c->d_slabs.ptr;
        d.norm_table = static_cast<const double*>(c->d_norm_table.ptr);
        d.support = static_cast<const int*>(c->d_support.ptr);
        d.d_norm = h.d_norm;
        d.d_skipped = h.d_num_skipped;
        d.grid_scale = (double)h.grid_size * h.cell_size_rad;
        d.w_scale = h.w_scale;
        // The reference's float path computes grid_size * cell_size_rad in
        // float (oskar_grid_wproj.c:150).
        d.grid_scale_f = (float)h.grid_size * (float)h.cell_size_rad;
        d.w_scale_f = (float)h.w_scale;
        d.coord_scale = coord_scale_of(h.frequency_hz);
        d.coord_scale_f = (float)d.coord_scale;
        d.first = first;
        d.n = h.num_points;
        d.grid_size = h.grid_size;
        d.num_planes = c->num_planes;
        d.oversample = c->oversample;
        d.half = c->half;
        hj[j] = d;
        first += h.num_points;
        if (comp) comp_off += 2 * (size_t)h.grid_size * h.grid_size;
    }
    const int bpj = prep_blocks_per_job(max_points, num_jobs, ws->num_sms);
    B200_TRY(ws->counters.ensure(sizeof(unsigned long long) * CNT_COUNT));
    B200_TRY(ws->jobs.ensure(job_bytes));
    B200_TRY(ws->job_skipped.ensure(sizeof(unsigned long long) * num_jobs));
    B200_TRY(ws->plane_counts.ensure(sizeof(unsigned long long) * num_jobs *
                                     max_planes));
    B200_TRY(ws->partials.ensure(sizeof(double) * num_jobs * bpj));
    unsigned long long* counters =
        static_cast<unsigned long long*>(ws->counters.ptr);
    B200_TRY(cudaMemsetAsync(counters, 0,
                             sizeof(unsigned long long) * CNT_COUNT, st));
    B200_TRY(cudaMemsetAsync(ws->job_skipped.ptr, 0,
                             sizeof(unsigned long long) * num_jobs, st));
    B200_TRY(cudaMemsetAsync(ws->plane_counts.ptr, 0,
                             sizeof(unsigned long long) * num_jobs * max_planes,
                             st));
    B200_TRY(cudaMemcpyAsync(ws->jobs.ptr, hj, job_bytes,
                             cudaMemcpyHostToDevice, st));
    {
        // Outside stream capture, remember when the upload has happened.
        if (!capturing)
        {
            if (!ws->jobs_event[slot])
                B200_TRY(cudaEventCreateWithFlags(&ws->jobs_event[slot],
                                                  cudaEventDisableTiming));
            B200_TRY(cudaEventRecord(ws->jobs_event[slot], st));
            ws->jobs_event_pending[slot] = 1;
        }
    }
    const JobDesc* d_jobs = static_cast<const JobDesc*>(ws->jobs.ptr);

    if (n > 0)
    {
        B200_TRY(ws->keys[0].ensure(4 * n));
        B200_TRY(ws->keys[1].ensure(4 * n));
        B200_TRY(ws->vals[0].ensure(4 * n));
        B200_TRY(ws->vals[1].ensure(4 * n));
        B200_TRY(ws->rec.ensure(16 * n));
        if (!degrid)
        {
            B200_TRY(ws->flags.ensure(8 * task_tiles(n)));
            B200_TRY(ws->task_start.ensure(4 * (n + 2)));
            B200_TRY(ws->task_job.ensure(4 * (n + 2)));
        }
        B200_TRY(ws->scan_tmp.ensure(std::max(radix_sort_temp_bytes(n),
                                              scan_temp_bytes(n))));
    }

    PrepArgs pa{};
    pa.jobs = d_jobs;
    pa.num_jobs = num_jobs;
    pa.blocks_per_job = bpj;
    pa.max_planes = max_planes;
    // (the norm is not a degridding output)
    pa.apply_weight = degrid ? 0 : opt->apply_weight;
    pa.key = kl;
    pa.rec = static_cast<int4*>(ws->rec.ptr);
    uint32_t* keys[2] = {static_cast<uint32_t*>(ws->keys[0].ptr),
                         static_cast<uint32_t*>(ws->keys[1].ptr)};
    uint32_t* vals[2] = {static_cast<uint32_t*>(ws->vals[0].ptr),
                         static_cast<uint32_t*>(ws->vals[1].ptr)};
    pa.keys = keys[0];
    pa.vals = vals[0];
    pa.counters = counters;
    pa.job_skipped = static_cast<unsigned long long*>(ws->job_skipped.ptr);
    pa.norm_partials = static_cast<double*>(ws->partials.ptr);
    pa.plane_counts = static_cast<unsigned long long*>(ws->plane_counts.ptr);

    B200_TRY(mark(0));
    if (n > 0)
    {
        B200_TRY(launch_prep(pa, dbl, opt->coord_mode, st));
        launches += 1;
    }
    else
    {
        B200_TRY(cudaMemsetAsync(pa.norm_partials, 0,
                                 sizeof(double) * num_jobs * bpj, st));
    }
    // Norms, skip counts and grid updates of every job (also when empty).
    B200_TRY(launch_finalize_prep(pa, st));
    launches += 1;
    B200_TRY(mark(1));
    if (n == 0)
    {
        B200_TRY(mark(2));
        B200_TRY(mark(3));
        B200_TRY(record_bands());
        B200_TRY(mark(4));
        ws->events_recorded = timing ? 1 : 0;
        ws->last_launches = launches;
        B200_TRY(cudaMemcpyAsync(ws->h_counters, counters,
                                 sizeof(unsigned long long) * CNT_COUNT,
                                 cudaMemcpyDeviceToHost, st));
        return OSKAR_B200_OK;
    }

    int which = 0;
    B200_TRY(radix_sort_pairs(keys, vals, n, kl.total_bits + 1,
                              ws->scan_tmp.ptr, st, &which, &launches));
    B200_TRY(mark(2));
    if (degrid)
    {
        B200_TRY(mark(3));
        B200_TRY(launch_degrid(vals[which], keys[which], pa.rec, d_jobs,
                               kl.job_shift, opt->apply_weight, counters, n,
                               dbl, c0->kernel_type, ws->num_sms, st));
        launches += 1;
        B200_TRY(mark(4));
        ws->events_recorded = timing ? 1 : 0;
        ws->last_launches = launches;
        B200_TRY(cudaMemcpyAsync(ws->h_counters, counters,
                                 sizeof(unsigned long long) * CNT_COUNT,
                                 cudaMemcpyDeviceToHost, st));
        return OSKAR_B200_OK;
    }
    B200_TRY(launch_tasks(keys[which], n, counters, 2 * kl.fine_bits,
                          kl.job_shift, kTaskMax,
                          static_cast<uint32_t*>(ws->flags.ptr),
                          ws->scan_tmp.ptr,
                          static_cast<uint32_t*>(ws->task_start.ptr),
                          static_cast<uint32_t*>(ws->task_job.ptr), st,
                          &launches));

    GridArgs ga{};
    ga.order = vals[which];
    ga.rec = pa.rec;
    ga.apply_weight = opt->apply_weight;
    ga.task_start = static_cast<const uint32_t*>(ws->task_start.ptr);
    ga.task_job = static_cast<const uint32_t*>(ws->task_job.ptr);
    ga.jobs = d_jobs;
    ga.counters = counters;
    ga.comp_radius = opt->compensate_radius >= 0 ? opt->compensate_radius
                     : ws->tuned_launch ? ws->tuned_comp_radius : 0;
    // Counting the grid atomics costs an instruction per tap: only when the
    // caller asked for it (statistics level bit 1).
    ga.count_flushes = (ws->stage_timing & 2) ? 1 : 0;
    if (opt->classes_per_thread >= 1 && opt->classes_per_thread <= 6)
        memset(ga.cpt, opt->classes_per_thread, sizeof(ga.cpt));
    else if (ws->tuned)
        memcpy(ga.cpt, ws->tune, sizeof(ga.cpt));
    else
        default_tune_table(ga.cpt);
    // Kernel values are read through L1 unless staging is asked for: on
    // plain_large the L1 path is as fast as staging each row-offset run's
    // W-row block into shared memory (24.2 ms vs 24.8 ms with FP16 slabs,
    // 30.2 ms with FP32 slabs, whose blocks cap residency at 2 CTAs/SM).
    const bool staged = opt->staging == 1 ||
                        (opt->staging == 0 && !comp && ws->tuned_launch &&
                         ws->tuned_staging == 1);
    if (staged && grid_smem_bytes(dbl, max_block, true) > ws->smem_optin)
        return OSKAR_B200_ERR_UNSUPPORTED;
    if (comp)
        B200_TRY(cudaMemsetAsync(ws->comp_grid.ptr, 0,
                                 comp_floats * sizeof(float), st));
    int ctas = 0;
    if (bands)
    {
        uint32_t* band_first = static_cast<uint32_t*>(ws->bands.ptr);
        unsigned long long* queues = reinterpret_cast<unsigned long long*>(
            static_cast<unsigned char*>(ws->bands.ptr) + 128);
        B200_TRY(launch_band_first(keys[which], ga.task_start, n, counters,
                                   kl, bands->num_bands, band_first,
                                   ws->num_sms, st));
        B200_TRY(cudaMemsetAsync(queues, 0,
                                 sizeof(unsigned long long) * kMaxBands, st));
        launches += 1;
        B200_TRY(mark(3));
        for (int i = 0; i < bands->num_bands; ++i)
        {
            const int b = bands->order[i];
            ga.range = band_first + b;
            ga.queue = queues + b;
            B200_TRY(launch_grid(ga, dbl, c0->kernel_type, max_block, staged,
                                 comp, ws->num_sms, st, &ctas));
            B200_TRY(cudaEventRecord(bands->events[i], st));
            launches += 1;
        }
    }
    else if (time_slices > 1)
    {
        // The task list in time_slices contiguous ranges, one launch each:
        // the persistent CTAs of one launch retire when its range is done,
        // so work queued on other streams (of higher priority) gets SMs
        // between slices instead of waiting for the whole job.
        uint32_t* first = static_cast<uint32_t*>(ws->bands.ptr);
        unsigned long long* queues = reinterpret_cast<unsigned long long*>(
            static_cast<unsigned char*>(ws->bands.ptr) + 128);
        B200_TRY(launch_slice_bounds(counters, time_slices, first, queues,
                                     st));
        launches += 1;
        B200_TRY(mark(3));
        for (int k = 0; k < time_slices; ++k)
        {
            ga.range = first + k;
            ga.queue = queues + k;
            B200_TRY(launch_grid(ga, dbl, c0->kernel_type, max_block, staged,
                                 comp, ws->num_sms, st, &ctas));
            launches += 1;
        }
    }
    else
    {
        B200_TRY(mark(3));
        B200_TRY(launch_grid(ga, dbl, c0->kernel_type, max_block, staged,
                             comp, ws->num_sms, st, &ctas));
        launches += 1;
    }
    if (comp)
    {
        B200_TRY(launch_fold_jobs(d_jobs, num_jobs, ws->num_sms, st));
        launches += 1;
    }
    B200_TRY(mark(4));
    ws->events_recorded = timing ? 1 : 0;
    ws->last_launches = launches;
    B200_TRY(cudaMemcpyAsync(ws->h_counters, counters,
                             sizeof(unsigned long long) * CNT_COUNT,
                             cudaMemcpyDeviceToHost, st));
    return OSKAR_B200_OK;
}

int run_grid(oskar_B200Workspace* ws, const oskar_B200Cube* cube,
             const oskar_B200Options* opt, size_t n, const void* uu,
             const void* vv, const void* ww, const void* vis,
             const void* weight, double cell_size_rad, double w_scale,
             int grid_size, void* grid, unsigned long long* d_num_skipped,
             double* d_norm, cudaStream_t st)
{
    HostJob j{};
    j.cube = cube;
    j.num_points = n;
    j.uu = uu;
    j.vv = vv;
    j.ww = ww;
    j.vis = vis;
    j.weight = weight;
    j.cell_size_rad = cell_size_rad;
    j.w_scale = w_scale;
    j.grid_size = grid_size;
    j.grid = grid;
    j.d_num_skipped = d_num_skipped;
    j.d_norm = d_norm;
    j.frequency_hz = opt->frequency_hz;
    return run_batch(ws, opt, 1, &j, st);
}

int run_place(oskar_B200Workspace* ws, int data_is_double, int coord_mode,
              const int* d_support, int num_planes, int oversample,
              size_t num_points, const void* uu, const void* vv,
              const void* ww, double cell_size_rad, double w_scale,
              int grid_size, int32_t* gu, int32_t* gv, int32_t* plane,
              int32_t* off_u, int32_t* off_v, int32_t* conj,
              int32_t* skipped, cudaStream_t st)
{
    PlaceConsts pc{};
    pc.grid_scale = (double)grid_size * cell_size_rad;
    pc.w_scale = w_scale;
    pc.grid_scale_f = (float)grid_size * (float)cell_size_rad;
    pc.w_scale_f = (float)w_scale;
    pc.grid_size = grid_size;
    pc.centre = grid_size / 2;
    pc.num_planes = num_planes;
    pc.oversample = oversample;
    if (num_points == 0) return OSKAR_B200_OK;
    return status_from_cuda(launch_place(data_is_double, coord_mode, uu, vv,
                                         ww, num_points, pc, d_support, gu,
                                         gv, plane, off_u, off_v, conj,
                                         skipped, ws->num_sms, st));
}

namespace {

// Complex-FP32 atomic-rate probe: each warp adds to 32 consecutive cells of
// a pseudo-random row per round (the access shape of a gridding flush).
__global__ void atomic_rate_kernel(float* __restrict__ grid, int grid_size,
                                   int iters)
{
    const unsigned lane = threadIdx.x & 31;
    const unsigned warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned cols = (unsigned)grid_size / 32u;
    unsigned h = warp * 2654435761u + 12345u;
    for (int it = 0; it < iters; ++it)
    {
        h ^= h << 13;
        h ^= h >> 17;
        h ^= h << 5;
        const unsigned row = h % (unsigned)grid_size;
        const unsigned col = ((h >> 8) % cols) * 32u + lane;
        red_add_c(grid + 2 * ((size_t)row * grid_size + col), 1.0f, 1.0f);
    }
}

// Self-test of the bounded waits: one CTA waits on an mbarrier phase that
// nothing completes (no arrival is ever made), gives up after `spins`
// try_wait attempts and records DEV_ERR_TIMEOUT, exactly as the gridding
// kernel does when a staged copy never lands.
__global__ void bounded_wait_probe_kernel(unsigned spins,
                                          unsigned long long* status)
{
    __shared__ uint64_t bar;
    if (threadIdx.x == 0)
    {
        mbar_init(&bar, 1);
        mbar_fence_init();
    }
    __syncthreads();
    const bool ok = mbar_wait_bounded(&bar, 0, spins);
    if (!__syncthreads_and(ok) && threadIdx.x == 0)
        atomicOr(status, (unsigned long long)DEV_ERR_TIMEOUT);
}

// dst = this call's contributions, src = the caller's values.  Where the
// call added nothing (dst is zero) the caller's value is kept as it is, as
// the reference leaves cells no footprint reaches (a -0.0 stays -0.0, a
// NaN keeps its bits).
template <typename T>
__global__ void add_kernel(T* __restrict__ dst, const T* __restrict__ src,
                           size_t n)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
    {
        const T a = dst[i], b = src[i];
        dst[i] = a == T(0) ? b : a + b;
    }
}

__global__ void status_or_kernel(const unsigned long long* counters,
                                 unsigned long long* acc)
{
    if (counters[CNT_STATUS]) *acc |= counters[CNT_STATUS];
}

// first[k] = floor(T * k / K) for k in [0, K], T the task count of the
// gridding launch; the K work-queue heads are zeroed.
__global__ void slice_bounds_kernel(const unsigned long long* counters,
                                    int k_slices, uint32_t* first,
                                    unsigned long long* queues)
{
    const unsigned long long t = counters[CNT_TASKS];
    for (int k = threadIdx.x; k <= k_slices; k += blockDim.x)
    {
        first[k] = (uint32_t)(t * (unsigned long long)k /
                              (unsigned long long)k_slices);
        if (k < k_slices) queues[k] = 0;
    }
}

}  // namespace

cudaError_t launch_slice_bounds(const unsigned long long* counters,
                                int k_slices, uint32_t* first,
                                unsigned long long* queues, cudaStream_t st)
{
    slice_bounds_kernel<<<1, 32, 0, st>>>(counters, k_slices, first, queues);
    return cudaGetLastError();
}

cudaError_t launch_add(void* dst, const void* src, size_t n, int is_double,
                       int num_sms, cudaStream_t st)
{
    if (n == 0) return cudaSuccess;
    const size_t want = (n + 255) / 256, cap = (size_t)num_sms * 8;
    const unsigned blocks = (unsigned)(want < cap ? want : cap);
    if (is_double)
        add_kernel<double><<<blocks, 256, 0, st>>>(
            static_cast<double*>(dst), static_cast<const double*>(src), n);
    else
        add_kernel<float><<<blocks, 256, 0, st>>>(
            static_cast<float*>(dst), static_cast<const float*>(src), n);
    return cudaGetLastError();
}

cudaError_t launch_status_or(oskar_B200Workspace* ws,
                             unsigned long long* acc, cudaStream_t st)
{
    status_or_kernel<<<1, 1, 0, st>>>(
        static_cast<const unsigned long long*>(ws->counters.ptr), acc);
    return cudaGetLastError();
}

int selftest_bounded_wait(oskar_B200Workspace* ws, unsigned spins,
                          int* device_status)
{
    B200_TRY(ws->counters.ensure(sizeof(unsigned long long) * CNT_COUNT));
    unsigned long long* c = static_cast<unsigned long long*>(ws->counters.ptr);
    B200_TRY(cudaMemsetAsync(c, 0, sizeof(unsigned long long) * CNT_COUNT,
                             ws->stream));
    bounded_wait_probe_kernel<<<1, 128, 0, ws->stream>>>(spins,
                                                         c + CNT_STATUS);
    B200_TRY(cudaGetLastError());
    unsigned long long s = 0;
    B200_TRY(cudaMemcpyAsync(&s, c + CNT_STATUS, sizeof(s),
                             cudaMemcpyDeviceToHost, ws->stream));
    B200_TRY(cudaStreamSynchronize(ws->stream));
    *device_status = (s & DEV_ERR_TIMEOUT) ? OSKAR_B200_ERR_TIMEOUT
                                           : OSKAR_B200_OK;
    return OSKAR_B200_OK;
}

int measure_atomic_rate(oskar_B200Workspace* ws, void* grid, int grid_size,
                        int iters, double* updates_per_s)
{
    if (grid_size < 32 || iters < 1) return OSKAR_B200_ERR_INVALID_ARGUMENT;
    const int blocks = ws->num_sms * 8, threads = 256;
    cudaEvent_t a, b;
    B200_TRY(cudaEventCreate(&a));
    B200_TRY(cudaEventCreate(&b));
    float* g = static_cast<float*>(grid);
    // warm-up, then timed
    atomic_rate_kernel<<<blocks, threads, 0, ws->stream>>>(g, grid_size, 8);
    cudaEventRecord(a, ws->stream);
    atomic_rate_kernel<<<blocks, threads, 0, ws->stream>>>(g, grid_size,
                                                           iters);
    cudaEventRecord(b, ws->stream);
    cudaError_t e = cudaEventSynchronize(b);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (e != cudaSuccess) return status_from_cuda(e);
    *updates_per_s = (double)blocks * threads * iters / (ms * 1e-3);
    return OSKAR_B200_OK;
}

}  // namespace b200
