// One gridding job on device-resident data:
//   prep (placement, keys, norm, skip count, plane histogram)
//   -> radix sort of (key, index)
//   -> permute records and visibilities into sorted order
//   -> task list
//   -> Romein gridding kernel.
#include <algorithm>
#include <cstring>

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

cudaError_t DeviceBuffer::ensure(size_t n)
{
    if (n <= bytes && ptr) return cudaSuccess;
    release();
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

namespace {

#define B200_TRY(expr)                                   \
    do {                                                 \
        const cudaError_t e_ = (expr);                   \
        if (e_ != cudaSuccess) return status_from_cuda(e_); \
    } while (0)

}  // namespace

int run_grid(oskar_B200Workspace* ws, const oskar_B200Cube* cube,
             const oskar_B200Options* opt, size_t n, const void* uu,
             const void* vv, const void* ww, const void* vis,
             const void* weight, double cell_size_rad, double w_scale,
             int grid_size, void* grid, unsigned long long* d_num_skipped,
             double* d_norm, cudaStream_t st)
{
    const bool dbl = cube->data_is_double != 0;
    const int P = cube->num_planes;
    const size_t vsz = dbl ? sizeof(double) : sizeof(float);
    int launches = 0;
    ws->last_points = n;
    ws->last_launches = 0;
    ws->events_recorded = 0;
    const bool timing = ws->stage_timing != 0;
    auto mark = [&](int i) -> cudaError_t {
        return timing ? cudaEventRecord(ws->events[i], st) : cudaSuccess;
    };

    B200_TRY(ws->counters.ensure(sizeof(unsigned long long) * CNT_COUNT));
    B200_TRY(ws->plane_counts.ensure(sizeof(unsigned long long) * P));
    unsigned long long* counters =
        static_cast<unsigned long long*>(ws->counters.ptr);
    B200_TRY(cudaMemsetAsync(counters, 0,
                             sizeof(unsigned long long) * CNT_COUNT, st));
    B200_TRY(cudaMemsetAsync(ws->plane_counts.ptr, 0,
                             sizeof(unsigned long long) * P, st));
    if (n == 0)
    {
        if (d_num_skipped)
            B200_TRY(cudaMemsetAsync(d_num_skipped, 0, sizeof(*d_num_skipped),
                                     st));
        B200_TRY(cudaMemcpyAsync(ws->h_counters, counters,
                                 sizeof(unsigned long long) * CNT_COUNT,
                                 cudaMemcpyDeviceToHost, st));
        return OSKAR_B200_OK;
    }

    B200_TRY(ws->keys[0].ensure(4 * n));
    B200_TRY(ws->keys[1].ensure(4 * n));
    B200_TRY(ws->vals[0].ensure(4 * n));
    B200_TRY(ws->vals[1].ensure(4 * n));
    B200_TRY(ws->rec.ensure(16 * n));
    B200_TRY(ws->srec.ensure(16 * n));
    B200_TRY(ws->svis.ensure(2 * vsz * n));
    B200_TRY(ws->flags.ensure(4 * n));
    B200_TRY(ws->task_start.ensure(4 * (n + 2)));
    B200_TRY(ws->scan_tmp.ensure(std::max(radix_sort_temp_bytes(n),
                                          scan_temp_bytes(n))));
    const unsigned blocks = prep_num_blocks(n, ws->num_sms);
    B200_TRY(ws->partials.ensure(sizeof(double) * blocks));

    const KeyLayout kl = make_key_layout(grid_size, P);
    PrepArgs pa{};
    pa.uu = uu;
    pa.vv = vv;
    pa.ww = ww;
    pa.weight = weight;
    pa.n = n;
    pa.pc.grid_scale = (double)grid_size * cell_size_rad;
    pa.pc.w_scale = w_scale;
    // The reference's float path computes grid_size * cell_size_rad in float.
    pa.pc.grid_scale_f = (float)grid_size * (float)cell_size_rad;
    pa.pc.w_scale_f = (float)w_scale;
    pa.pc.grid_size = grid_size;
    pa.pc.centre = grid_size / 2;
    pa.pc.num_planes = P;
    pa.pc.oversample = cube->oversample;
    pa.support = static_cast<const int*>(cube->d_support.ptr);
    pa.num_planes = P;
    pa.half = cube->half;
    pa.apply_weight = opt->apply_weight;
    pa.norm_table = static_cast<const double*>(cube->d_norm_table.ptr);
    pa.key = kl;
    pa.rec = static_cast<int4*>(ws->rec.ptr);
    uint32_t* keys[2] = {static_cast<uint32_t*>(ws->keys[0].ptr),
                         static_cast<uint32_t*>(ws->keys[1].ptr)};
    uint32_t* vals[2] = {static_cast<uint32_t*>(ws->vals[0].ptr),
                         static_cast<uint32_t*>(ws->vals[1].ptr)};
    pa.keys = keys[0];
    pa.vals = vals[0];
    pa.counters = counters;
    pa.norm_partials = static_cast<double*>(ws->partials.ptr);
    pa.plane_counts = static_cast<unsigned long long*>(ws->plane_counts.ptr);
    B200_TRY(mark(0));
    B200_TRY(launch_prep(pa, dbl, opt->coord_mode, blocks, st));
    B200_TRY(launch_finalize_prep(pa.norm_partials, (int)blocks,
                                  pa.plane_counts, pa.support, P, counters,
                                  d_norm, d_num_skipped, st));
    launches += 2;

    B200_TRY(mark(1));
    int which = 0;
    B200_TRY(radix_sort_pairs(keys, vals, n, kl.total_bits + 1,
                              ws->scan_tmp.ptr, st, &which, &launches));
    B200_TRY(mark(2));
    B200_TRY(launch_permute(vals[which], n, counters, pa.rec, vis, weight,
                            opt->apply_weight, dbl,
                            static_cast<int4*>(ws->srec.ptr), ws->svis.ptr,
                            ws->num_sms, st));
    launches += 1;
    B200_TRY(launch_tasks(keys[which], n, counters, 2 * kl.fine_bits,
                          kTaskMax, static_cast<uint32_t*>(ws->flags.ptr),
                          keys[which ^ 1], ws->scan_tmp.ptr,
                          static_cast<uint32_t*>(ws->task_start.ptr),
                          ws->num_sms, st, &launches));

    GridArgs ga{};
    ga.srec = static_cast<const int4*>(ws->srec.ptr);
    ga.svis = ws->svis.ptr;
    ga.task_start = static_cast<const uint32_t*>(ws->task_start.ptr);
    ga.planes = static_cast<const PlaneDesc*>(cube->d_planes.ptr);
    ga.slabs = cube->d_slabs.ptr;
    ga.grid = grid;
    ga.counters = counters;
    ga.grid_size = grid_size;
    ga.oversample = cube->oversample;
    ga.half = cube->half;
    if (opt->classes_per_thread == 1 || opt->classes_per_thread == 2 ||
        opt->classes_per_thread == 4)
        memset(ga.cpt, opt->classes_per_thread, sizeof(ga.cpt));
    else
        default_tune_table(ga.cpt);
    // Auto staging reads the kernel slabs through L1: on plain_large it ran
    // the gridding kernel 2.3x faster than staging each task's slab into
    // shared memory, whose size caps residency at one CTA per SM.
    const bool fits = grid_smem_bytes(cube, true) <= ws->smem_optin;
    const bool staged = opt->staging == 1;
    if (staged && !fits) return OSKAR_B200_ERR_UNSUPPORTED;
    const bool comp = opt->accum_mode == OSKAR_B200_ACCUM_COMPENSATED;
    const size_t cells = (size_t)grid_size * (size_t)grid_size;
    if (comp)
    {
        // Error grid of this job: zeroed here, folded into the grid below.
        B200_TRY(ws->comp_grid.ensure(cells * 2 * sizeof(float)));
        B200_TRY(cudaMemsetAsync(ws->comp_grid.ptr, 0,
                                 cells * 2 * sizeof(float), st));
        ga.comp = ws->comp_grid.ptr;
    }
    int ctas = 0;
    B200_TRY(mark(3));
    B200_TRY(launch_grid(ga, cube, staged, comp, ws->num_sms, st, &ctas));
    launches += 1;
    if (comp)
    {
        B200_TRY(launch_fold(static_cast<float*>(grid),
                             static_cast<float*>(ws->comp_grid.ptr), cells,
                             ws->num_sms, st));
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

}  // namespace

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

}  // namespace b200
