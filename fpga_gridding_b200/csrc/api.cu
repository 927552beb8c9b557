// Public C ABI of the B200 gridder: the drop-in oskar_grid_wproj_{d,f}
// replacements and the extended device-resident API.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <new>
#include <vector>

#include "band_rows.h"
#include "ingest_plan.h"
#include "common.cuh"
#include "prep.cuh"
#include "grid_romein.cuh"
#include "internal.h"

#define B200_STR2(x) #x
#define B200_STR(x) B200_STR2(x)

using namespace b200;

namespace {

thread_local int tls_status = OSKAR_B200_OK;

// Makes `device` current for the scope of a call and restores the caller's.
struct DeviceGuard
{
    int prev = -1;
    bool changed = false;
    explicit DeviceGuard(int device)
    {
        if (cudaGetDevice(&prev) == cudaSuccess && prev != device)
            changed = cudaSetDevice(device) == cudaSuccess;
    }
    ~DeviceGuard()
    {
        if (changed) cudaSetDevice(prev);
    }
};

// The caller's current device, if it is a usable sm_100 device.
int current_device(int* device)
{
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
    {
        cudaGetLastError();
        return OSKAR_B200_ERR_NO_DEVICE;
    }
    if (cudaGetDevice(device) != cudaSuccess) return OSKAR_B200_ERR_NO_DEVICE;
    int major = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, *device);
    // The kernels are built for sm_100a only.
    if (major != 10) return OSKAR_B200_ERR_NO_DEVICE;
    return OSKAR_B200_OK;
}

int workspace_create(int device, oskar_B200Workspace** out)
{
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 ||
        device >= count)
    {
        cudaGetLastError();
        return OSKAR_B200_ERR_NO_DEVICE;
    }
    int major = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device);
    if (major != 10) return OSKAR_B200_ERR_NO_DEVICE;
    DeviceGuard g(device);
    auto* ws = new (std::nothrow) oskar_B200Workspace();
    if (!ws) return OSKAR_B200_ERR_OUT_OF_MEMORY;
    ws->device = device;
    int smem = 0;
    cudaDeviceGetAttribute(&ws->num_sms, cudaDevAttrMultiProcessorCount, device);
    cudaDeviceGetAttribute(&smem, cudaDevAttrMaxSharedMemoryPerBlockOptin,
                           device);
    ws->smem_optin = (size_t)smem;
    cudaError_t e = cudaStreamCreateWithFlags(&ws->stream,
                                              cudaStreamNonBlocking);
    if (e == cudaSuccess)
        e = cudaMallocHost(&ws->h_counters,
                           sizeof(unsigned long long) * CNT_COUNT);
    if (e != cudaSuccess)
    {
        if (ws->stream) cudaStreamDestroy(ws->stream);
        delete ws;
        cudaGetLastError();
        return status_from_cuda(e);
    }
    memset(ws->h_counters, 0, sizeof(unsigned long long) * CNT_COUNT);
    *out = ws;
    return OSKAR_B200_OK;
}

void workspace_free(oskar_B200Workspace* ws)
{
    if (!ws) return;
    DeviceGuard g(ws->device);
    if (ws->stream) cudaStreamSynchronize(ws->stream);
    if (ws->copy_stream) cudaStreamSynchronize(ws->copy_stream);
    if (ws->d2h_stream) cudaStreamSynchronize(ws->d2h_stream);
    for (cudaEvent_t& e : ws->events)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t& e : ws->ingest_events)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t& e : ws->band_events)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t& e : ws->piece_events)
        if (e) cudaEventDestroy(e);
    if (ws->copy_stream) cudaStreamDestroy(ws->copy_stream);
    if (ws->d2h_stream) cudaStreamDestroy(ws->d2h_stream);
    for (int r = 0; r < kJobRing; ++r)
    {
        if (ws->jobs_event[r]) cudaEventDestroy(ws->jobs_event[r]);
        if (ws->h_jobs[r]) cudaFreeHost(ws->h_jobs[r]);
    }
    if (ws->h_counters) cudaFreeHost(ws->h_counters);
    if (ws->stream) cudaStreamDestroy(ws->stream);
    delete ws;  // DeviceBuffer destructors free device memory
}

// Per-thread cache of the drop-in path: a workspace for the current device
// and a cube object whose device buffers are reused across calls.
struct ThreadCache
{
    oskar_B200Workspace* ws = nullptr;
    oskar_B200Cube* cube = nullptr;
    void release()
    {
        if (ws)
        {
            DeviceGuard g(ws->device);
            delete cube;
            workspace_free(ws);
        }
        else
        {
            delete cube;
        }
        ws = nullptr;
        cube = nullptr;
    }
    ~ThreadCache() { release(); }
};
thread_local ThreadCache tls_cache;

int validate_cube_args(size_t num_w_planes, const int* support,
                       int oversample, int conv_size_half,
                       const void* conv_func)
{
    if (num_w_planes == 0 || num_w_planes > (1u << 15) || !support ||
        !conv_func || oversample < 1 || oversample > 32 ||
        conv_size_half < 1)
        return OSKAR_B200_ERR_INVALID_ARGUMENT;
    const long long csh = conv_size_half;
    const long long total = (long long)num_w_planes * csh * csh;
    const int half = (oversample + 1) / 2;
    for (size_t p = 0; p < num_w_planes; ++p)
    {
        const long long s = support[p];
        if (s < 0) return OSKAR_B200_ERR_INVALID_ARGUMENT;
        // The gridding kernel lays a footprint's 2S+1 columns across one
        // 256-thread CTA.
        if (s > 127) return OSKAR_B200_ERR_UNSUPPORTED;
        // Largest flat index the reference reads on this plane
        // (oskar_grid_wproj.c:110-116) must lie inside the cube.
        const long long e = oversample * s + half;
        if ((long long)p * csh * csh + e * csh + e >= total)
            return OSKAR_B200_ERR_INVALID_ARGUMENT;
    }
    return OSKAR_B200_OK;
}

// Builds (or rebuilds) `cube` in place from a device copy of the cube.
int cube_init(oskar_B200Cube* c, int device, size_t num_w_planes,
              const int* support, int oversample, int conv_size_half,
              const void* d_conv, const void* d_conv_im, int conv_is_double,
              int data_is_double, int kernel_type, cudaStream_t st)
{
    c->device = device;
    c->num_planes = (int)num_w_planes;
    c->oversample = oversample;
    c->half = (oversample + 1) / 2;
    c->conv_size_half = conv_size_half;
    c->data_is_double = data_is_double;
    c->kernel_type = kernel_type;
    if (data_is_double)
        c->elem_bytes = 16;
    else
        c->elem_bytes = kernel_type == OSKAR_B200_KERNEL_NATIVE ? 8 : 4;
    c->planes.assign(num_w_planes, PlaneDesc{});
    c->max_support = 0;
    for (size_t p = 0; p < num_w_planes; ++p)
    {
        c->planes[p].support = support[p];
        if (support[p] > c->max_support) c->max_support = support[p];
    }
    cudaError_t e = c->d_support.ensure(sizeof(int) * num_w_planes);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(c->d_support.ptr, support,
                            sizeof(int) * num_w_planes,
                            cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return status_from_cuda(e);
    return cube_build(c, d_conv, d_conv_im, conv_is_double, st);
}


int check_grid_args(size_t num_points, const void* uu, const void* vv,
                    const void* ww, const void* vis, const void* weight,
                    int apply_weight, int grid_size, const void* grid)
{
    if (grid_size < 1 || grid_size > 65535 || !grid)
        return OSKAR_B200_ERR_INVALID_ARGUMENT;
    if (num_points >= 0xffffffffull) return OSKAR_B200_ERR_INVALID_ARGUMENT;
    if (num_points && (!uu || !vv || !ww || !vis))
        return OSKAR_B200_ERR_INVALID_ARGUMENT;
    if (num_points && apply_weight && !weight)
        return OSKAR_B200_ERR_INVALID_ARGUMENT;
    return OSKAR_B200_OK;
}

// The drop-in's device pipeline.  Streams: s grids, c uploads (the cube, the
// chunks in order, then the caller's grid band by band), d adds each
// finished band of the caller's grid to the accumulated contributions and
// copies it back.  The caller's grid on the device (in_grid) is never
// modified, so a job whose device status reports a failure is undone by
// copying it back over the rows already returned.
template <typename T>
int drop_in(size_t num_w_planes, const int* support, int oversample,
            int conv_size_half, const T* conv_func, size_t num_points,
            const T* uu, const T* vv, const T* ww, const T* vis,
            double cell_size_rad, double w_scale, int grid_size,
            size_t* num_skipped, double* norm, T* grid)
{
    const bool dbl = sizeof(T) == sizeof(double);
    if (!num_skipped || !norm || !grid) return OSKAR_B200_ERR_INVALID_ARGUMENT;
    int st = validate_cube_args(num_w_planes, support, oversample,
                                conv_size_half, conv_func);
    if (st) return st;
    st = check_grid_args(num_points, uu, vv, ww, vis, nullptr, 0, grid_size,
                         grid);
    if (st) return st;
    int device = 0;
    st = current_device(&device);
    if (st) return st;
    ThreadCache& tc = tls_cache;
    if (tc.ws && tc.ws->device != device) tc.release();
    if (!tc.ws)
    {
        st = workspace_create(device, &tc.ws);
        if (st) return st;
    }
    if (!tc.cube)
    {
        tc.cube = new (std::nothrow) oskar_B200Cube();
        if (!tc.cube) return OSKAR_B200_ERR_OUT_OF_MEMORY;
    }
    oskar_B200Workspace* ws = tc.ws;
    cudaStream_t s = ws->stream;
    const size_t n = num_points;
    const size_t cube_elems = num_w_planes * (size_t)conv_size_half *
                              conv_size_half * 2;
    const size_t row_elems = 2 * (size_t)grid_size;
    const size_t grid_elems = row_elems * grid_size;
    // Chunk k covers points [bound[k], bound[k + 1]); the last is the tail.
    // (One event per chunk after the cube's: at most kIngestEvents - 1.)
    size_t bound[kIngestEvents];
    const int chunks = ingest_chunks(n, kIngestEvents - 1, bound);
    size_t rows_back = 0;   // rows of the caller's grid already overwritten
    auto sync_all = [&]() {
        cudaStreamSynchronize(s);
        if (ws->copy_stream) cudaStreamSynchronize(ws->copy_stream);
        if (ws->d2h_stream) cudaStreamSynchronize(ws->d2h_stream);
    };
    // Puts back the caller's rows already overwritten (when the device can
    // still do it) and reports `status`.
    auto fail = [&](int status) -> int {
        sync_all();
        cudaGetLastError();
        if (rows_back &&
            cudaMemcpyAsync(grid, ws->in_grid.ptr,
                            rows_back * row_elems * sizeof(T),
                            cudaMemcpyDeviceToHost, s) == cudaSuccess)
            cudaStreamSynchronize(s);
        cudaGetLastError();
        return status;
    };
#define B200_CHECK(expr)                                            \
    do {                                                            \
        const cudaError_t e_ = (expr);                              \
        if (e_ != cudaSuccess) return fail(status_from_cuda(e_));   \
    } while (0)
    if (!ws->copy_stream)
        B200_CHECK(cudaStreamCreateWithFlags(&ws->copy_stream,
                                             cudaStreamNonBlocking));
    if (!ws->d2h_stream)
        B200_CHECK(cudaStreamCreateWithFlags(&ws->d2h_stream,
                                             cudaStreamNonBlocking));
    for (cudaEvent_t& e : ws->ingest_events)
        if (!e) B200_CHECK(cudaEventCreateWithFlags(&e,
                                                    cudaEventDisableTiming));
    for (int b = 0; b < kMaxBands; ++b)
    {
        if (!ws->band_events[b])
            B200_CHECK(cudaEventCreateWithFlags(&ws->band_events[b],
                                                cudaEventDisableTiming));
        if (!ws->piece_events[b])
            B200_CHECK(cudaEventCreateWithFlags(&ws->piece_events[b],
                                                cudaEventDisableTiming));
    }
    cudaStream_t c = ws->copy_stream;
    cudaStream_t d = ws->d2h_stream;
    cudaEvent_t ev_cube = ws->ingest_events[0];
    cudaEvent_t* ev_chunk = ws->ingest_events + 1;
    B200_CHECK(ws->in_cube.ensure(cube_elems * sizeof(T)));
    B200_CHECK(ws->in_grid.ensure(grid_elems * sizeof(T)));
    B200_CHECK(ws->acc_grid.ensure(grid_elems * sizeof(T)));
    // [norm, device status of every chunk OR-ed, skip count of each chunk]
    const size_t slots = 2 + (size_t)chunks;
    B200_CHECK(ws->in_norm.ensure(sizeof(double) * slots));
    if (n)
    {
        B200_CHECK(ws->in_uu.ensure(n * sizeof(T)));
        B200_CHECK(ws->in_vv.ensure(n * sizeof(T)));
        B200_CHECK(ws->in_ww.ensure(n * sizeof(T)));
        B200_CHECK(ws->in_vis.ensure(2 * n * sizeof(T)));
    }
    // The previous call's copies were waited for before it returned.
    B200_CHECK(cudaMemcpyAsync(ws->in_cube.ptr, conv_func,
                               cube_elems * sizeof(T),
                               cudaMemcpyHostToDevice, c));
    B200_CHECK(cudaEventRecord(ev_cube, c));
    B200_CHECK(cudaStreamWaitEvent(s, ev_cube, 0));
    st = cube_init(tc.cube, device, num_w_planes, support, oversample,
                   conv_size_half, ws->in_cube.ptr, nullptr, dbl, dbl,
                   OSKAR_B200_KERNEL_NATIVE, s);
    if (st) return fail(st);
    B200_CHECK(cudaMemsetAsync(ws->in_norm.ptr, 0, sizeof(double) * slots,
                               s));
    B200_CHECK(cudaMemsetAsync(ws->acc_grid.ptr, 0, grid_elems * sizeof(T),
                               s));
    oskar_B200Options opt;
    oskar_b200_options_init(&opt);
    double* d_norm = static_cast<double*>(ws->in_norm.ptr);
    unsigned long long* d_status =
        reinterpret_cast<unsigned long long*>(d_norm + 1);
    unsigned long long* d_skip = d_status + 1;
    T* acc = static_cast<T*>(ws->acc_grid.ptr);
    T* in_grid = static_cast<T*>(ws->in_grid.ptr);
    BandPlan plan{};
    plan.events = ws->band_events;
    for (int k = 0; k < chunks; ++k)
    {
        const bool last = k == chunks - 1;
        const size_t b = bound[k], e = bound[k + 1];
        const size_t m = e - b;
        T* du = static_cast<T*>(ws->in_uu.ptr) + b;
        T* dv = static_cast<T*>(ws->in_vv.ptr) + b;
        T* dw = static_cast<T*>(ws->in_ww.ptr) + b;
        T* dz = static_cast<T*>(ws->in_vis.ptr) + 2 * b;
        if (m)
        {
            B200_CHECK(cudaMemcpyAsync(du, uu + b, m * sizeof(T),
                                       cudaMemcpyHostToDevice, c));
            B200_CHECK(cudaMemcpyAsync(dv, vv + b, m * sizeof(T),
                                       cudaMemcpyHostToDevice, c));
            B200_CHECK(cudaMemcpyAsync(dw, ww + b, m * sizeof(T),
                                       cudaMemcpyHostToDevice, c));
            B200_CHECK(cudaMemcpyAsync(dz, vis + 2 * b, 2 * m * sizeof(T),
                                       cudaMemcpyHostToDevice, c));
        }
        B200_CHECK(cudaEventRecord(ev_chunk[k], c));
        B200_CHECK(cudaStreamWaitEvent(s, ev_chunk[k], 0));
        HostJob j{};
        j.cube = tc.cube;
        j.num_points = m;
        j.uu = du;
        j.vv = dv;
        j.ww = dw;
        j.vis = dz;
        j.cell_size_rad = cell_size_rad;
        j.w_scale = w_scale;
        j.grid_size = grid_size;
        j.grid = acc;
        j.d_num_skipped = d_skip + k;
        j.d_norm = d_norm;
        st = run_batch(ws, &opt, 1, &j, s, false, last ? &plan : nullptr);
        if (st) return fail(st);
        // Each chunk resets the workspace's status word: keep its bits.
        B200_CHECK(launch_status_or(ws, d_status, s));
    }
    // The caller's grid goes up band by band after the visibilities, in the
    // order the bands are gridded.
    const int nb = plan.num_bands;
    const int rs = plan.row_shift;
    const size_t G = (size_t)grid_size;
    auto band_rows = [&](int b, size_t* r0, size_t* r1) {
        *r0 = std::min(G, (size_t)b << rs);
        *r1 = std::min(G, (size_t)(b + 1) << rs);
    };
    cudaEvent_t piece_of_band[kMaxBands] = {};
    for (int i = 0; i < nb; ++i)
    {
        const int b = plan.order[i];
        size_t r0, r1;
        band_rows(b, &r0, &r1);
        B200_CHECK(cudaMemcpyAsync(in_grid + r0 * row_elems,
                                   grid + r0 * row_elems,
                                   (r1 - r0) * row_elems * sizeof(T),
                                   cudaMemcpyHostToDevice, c));
        B200_CHECK(cudaEventRecord(ws->piece_events[i], c));
        piece_of_band[b] = ws->piece_events[i];
    }
    // After each band, the rows that just became final (no later band can
    // reach them) get the caller's values added and go back.  (The caller's
    // rows have all gone up before any of them comes back: each returned
    // run waits for the uploads of its own bands.)
    int waited_step = -1;
    for (const FinalRows& f : final_rows(nb, plan.order, rs, plan.halo,
                                         (long long)G))
    {
        if (f.step != waited_step)
        {
            B200_CHECK(cudaStreamWaitEvent(d, ws->band_events[f.step], 0));
            waited_step = f.step;
        }
        for (long long x = f.r0 >> rs; x <= (f.r1 - 1) >> rs; ++x)
            B200_CHECK(cudaStreamWaitEvent(d, piece_of_band[x], 0));
        const size_t off = (size_t)f.r0 * row_elems;
        const size_t cnt = (size_t)(f.r1 - f.r0) * row_elems;
        B200_CHECK(launch_add(acc + off, in_grid + off, cnt, dbl,
                              ws->num_sms, d));
        rows_back = G;   // (fail() puts back every row from here on)
        B200_CHECK(cudaMemcpyAsync(grid + off, acc + off, cnt * sizeof(T),
                                   cudaMemcpyDeviceToHost, d));
    }
    B200_CHECK(cudaStreamSynchronize(s));
    B200_CHECK(cudaStreamSynchronize(c));
    B200_CHECK(cudaStreamSynchronize(d));
    B200_CHECK(cudaGetLastError());
    std::vector<unsigned long long> out(slots);
    B200_CHECK(cudaMemcpyAsync(out.data(), d_norm,
                               sizeof(double) * slots,
                               cudaMemcpyDeviceToHost, s));
    B200_CHECK(cudaStreamSynchronize(s));
    if (out[1]) return fail(out[1] & DEV_ERR_TIMEOUT ? OSKAR_B200_ERR_TIMEOUT
                                                     : OSKAR_B200_ERR_DEVICE_CHECK);
#undef B200_CHECK
    unsigned long long skipped = 0;
    for (int k = 0; k < chunks; ++k) skipped += out[2 + k];
    double nrm;
    memcpy(&nrm, &out[0], sizeof(nrm));
    *norm += nrm;
    *num_skipped = (size_t)skipped;
    return OSKAR_B200_OK;
}

}  // namespace

namespace b200 {

int check_options(const oskar_B200Options* opt, int data_is_double)
{
    if (opt->coord_mode != OSKAR_B200_COORDS_F64 &&
        opt->coord_mode != OSKAR_B200_COORDS_REFERENCE_F32)
        return OSKAR_B200_ERR_INVALID_ARGUMENT;
    if (data_is_double && opt->coord_mode != OSKAR_B200_COORDS_F64)
        return OSKAR_B200_ERR_UNSUPPORTED;
    if (opt->accum_mode != OSKAR_B200_ACCUM_PLAIN &&
        opt->accum_mode != OSKAR_B200_ACCUM_COMPENSATED)
        return OSKAR_B200_ERR_INVALID_ARGUMENT;
    if (opt->accum_mode == OSKAR_B200_ACCUM_COMPENSATED &&
        (data_is_double || opt->staging == 1))
        return OSKAR_B200_ERR_UNSUPPORTED;
    if (opt->staging < 0 || opt->staging > 2)
        return OSKAR_B200_ERR_INVALID_ARGUMENT;
    if (opt->compensate_radius < -1 ||
        (opt->tile_shift != 0 && (opt->tile_shift < 6 || opt->tile_shift > 15)))
        return OSKAR_B200_ERR_INVALID_ARGUMENT;
    if (!(opt->frequency_hz >= 0.0) || !std::isfinite(opt->frequency_hz))
        return OSKAR_B200_ERR_INVALID_ARGUMENT;
    return OSKAR_B200_OK;
}

}  // namespace b200

// ---------------------------------------------------------------------------
// Drop-in entry points
// ---------------------------------------------------------------------------
extern "C" {

void oskar_grid_wproj_d(const size_t num_w_planes, const int* support,
                        const int oversample, const int conv_size_half,
                        const double* conv_func, const size_t num_points,
                        const double* uu, const double* vv, const double* ww,
                        const double* vis, const double* weight,
                        const double cell_size_rad, const double w_scale,
                        const int grid_size, size_t* num_skipped,
                        double* norm, double* grid)
{
    (void)weight;  // ignored, as in oskar_grid_wproj.c:80-81
    tls_status = drop_in<double>(num_w_planes, support, oversample,
                                 conv_size_half, conv_func, num_points, uu,
                                 vv, ww, vis, cell_size_rad, w_scale,
                                 grid_size, num_skipped, norm, grid);
}

void oskar_grid_wproj_f(const size_t num_w_planes, const int* support,
                        const int oversample, const int conv_size_half,
                        const float* conv_func, const size_t num_points,
                        const float* uu, const float* vv, const float* ww,
                        const float* vis, const float* weight,
                        const float cell_size_rad, const float w_scale,
                        const int grid_size, size_t* num_skipped,
                        double* norm, float* grid)
{
    (void)weight;  // ignored, as in oskar_grid_wproj.c:184-185
    tls_status = drop_in<float>(num_w_planes, support, oversample,
                                conv_size_half, conv_func, num_points, uu, vv,
                                ww, vis, (double)cell_size_rad,
                                (double)w_scale, grid_size, num_skipped, norm,
                                grid);
}

int oskar_grid_wproj_b200_last_error(void) { return tls_status; }

const char* oskar_grid_wproj_b200_error_string(int status)
{
    switch (status)
    {
    case OSKAR_B200_OK: return "ok";
    case OSKAR_B200_ERR_INVALID_ARGUMENT: return "invalid argument";
    case OSKAR_B200_ERR_NO_DEVICE: return "no usable sm_100 CUDA device";
    case OSKAR_B200_ERR_OUT_OF_MEMORY: return "out of memory";
    case OSKAR_B200_ERR_CUDA: return "CUDA runtime error";
    case OSKAR_B200_ERR_UNSUPPORTED: return "unsupported option combination";
    case OSKAR_B200_ERR_DEVICE_CHECK: return "device-side bounds check failed";
    case OSKAR_B200_ERR_TIMEOUT: return "bounded device wait expired";
    case OSKAR_B200_ERR_OVER_BUDGET: return "job exceeds the memory budget";
    default: return "unknown status";
    }
}

void oskar_grid_wproj_b200_release_thread_cache(void) { tls_cache.release(); }

// ---------------------------------------------------------------------------
// Extended API
// ---------------------------------------------------------------------------

void oskar_b200_options_init(oskar_B200Options* opt)
{
    if (!opt) return;
    memset(opt, 0, sizeof(*opt));
    opt->coord_mode = OSKAR_B200_COORDS_F64;
    opt->kernel_type = OSKAR_B200_KERNEL_NATIVE;
    opt->accum_mode = OSKAR_B200_ACCUM_PLAIN;
}

int oskar_b200_workspace_create(int device, oskar_B200Workspace** ws)
{
    if (!ws) return OSKAR_B200_ERR_INVALID_ARGUMENT;
    return workspace_create(device, ws);
}

int oskar_b200_workspace_free(oskar_B200Workspace* ws)
{
    workspace_free(ws);
    return OSKAR_B200_OK;
}

size_t oskar_b200_workspace_bytes(const oskar_B200Workspace* ws)
{
    if (!ws) return 0;
    const DeviceBuffer* bufs[] = {
        &ws->keys[0], &ws->keys[1], &ws->vals[0], &ws->vals[1], &ws->rec,
        &ws->scan_tmp, &ws->flags, &ws->task_start, &ws->task_job,
        &ws->counters, &ws->partials, &ws->plane_counts, &ws->in_uu,
        &ws->in_vv, &ws->in_ww, &ws->in_vis, &ws->in_weight, &ws->in_grid,
        &ws->in_cube, &ws->in_norm, &ws->comp_grid};
    size_t t = 0;
    for (const DeviceBuffer* b : bufs) t += b->bytes;
    return t;
}

}  // extern "C"

namespace {

// Shared body of the cube constructors: conv_im == nullptr means conv_func is
// the interleaved complex cube; otherwise conv_func / conv_im are the real /
// imaginary parts.
int cube_create_impl(oskar_B200Workspace* ws, size_t num_w_planes,
                     const int* support, int oversample, int conv_size_half,
                     const void* conv_func, const void* conv_im,
                     int conv_func_is_double, int conv_func_on_device,
                     int data_is_double, int kernel_type, void* stream,
                     oskar_B200Cube** cube)
{
    if (!ws || !cube) return OSKAR_B200_ERR_INVALID_ARGUMENT;
    *cube = nullptr;
    int st = validate_cube_args(num_w_planes, support, oversample,
                                conv_size_half, conv_func);
    if (st) return st;
    if (kernel_type < OSKAR_B200_KERNEL_NATIVE ||
        kernel_type > OSKAR_B200_KERNEL_BF16)
        return OSKAR_B200_ERR_INVALID_ARGUMENT;
    if (data_is_double && kernel_type != OSKAR_B200_KERNEL_NATIVE)
        return OSKAR_B200_ERR_UNSUPPORTED;
    DeviceGuard g(ws->device);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ws->stream;
    auto* c = new (std::nothrow) oskar_B200Cube();
    if (!c) return OSKAR_B200_ERR_OUT_OF_MEMORY;
    const size_t parts = conv_im ? 1 : 2;
    const size_t bytes = num_w_planes * (size_t)conv_size_half *
                         conv_size_half * parts *
                         (conv_func_is_double ? sizeof(double) : sizeof(float));
    const void* d_conv = conv_func;
    const void* d_im = conv_im;
    DeviceBuffer staging, staging_im;
    if (!conv_func_on_device)
    {
        cudaError_t e = staging.ensure(bytes);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(staging.ptr, conv_func, bytes,
                                cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess && conv_im)
        {
            e = staging_im.ensure(bytes);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(staging_im.ptr, conv_im, bytes,
                                    cudaMemcpyHostToDevice, s);
        }
        if (e != cudaSuccess) { delete c; return status_from_cuda(e); }
        d_conv = staging.ptr;
        d_im = conv_im ? staging_im.ptr : nullptr;
    }
    st = cube_init(c, ws->device, num_w_planes, support, oversample,
                   conv_size_half, d_conv, d_im, conv_func_is_double,
                   data_is_double, kernel_type, s);
    // The staging copies must outlive the kernels that read them.
    cudaError_t e = cudaStreamSynchronize(s);
    if (!st && e != cudaSuccess) st = status_from_cuda(e);
    if (st) { delete c; return st; }
    *cube = c;
    return OSKAR_B200_OK;
}

}  // namespace

extern "C" {

int oskar_b200_cube_create(oskar_B200Workspace* ws, size_t num_w_planes,
                           const int* support, int oversample,
                           int conv_size_half, const void* conv_func,
                           int conv_func_is_double, int conv_func_on_device,
                           int data_is_double, int kernel_type, void* stream,
                           oskar_B200Cube** cube)
{
    return cube_create_impl(ws, num_w_planes, support, oversample,
                            conv_size_half, conv_func, nullptr,
                            conv_func_is_double, conv_func_on_device,
                            data_is_double, kernel_type, stream, cube);
}

int oskar_b200_cube_create_planar(oskar_B200Workspace* ws,
                                  size_t num_w_planes, const int* support,
                                  int oversample, int conv_size_half,
                                  const void* conv_re, const void* conv_im,
                                  int conv_is_double, int conv_on_device,
                                  int data_is_double, int kernel_type,
                                  void* stream, oskar_B200Cube** cube)
{
    if (!conv_im) return OSKAR_B200_ERR_INVALID_ARGUMENT;
    return cube_create_impl(ws, num_w_planes, support, oversample,
                            conv_size_half, conv_re, conv_im, conv_is_double,
                            conv_on_device, data_is_double, kernel_type,
                            stream, cube);
}

int oskar_b200_cube_free(oskar_B200Cube* cube)
{
    if (!cube) return OSKAR_B200_OK;
    DeviceGuard g(cube->device);
    delete cube;
    return OSKAR_B200_OK;
}

size_t oskar_b200_cube_bytes(const oskar_B200Cube* cube)
{
    if (!cube) return 0;
    return cube->d_slabs.bytes + cube->d_planes.bytes +
           cube->d_norm_table.bytes + cube->d_support.bytes;
}

int oskar_b200_grid(oskar_B200Workspace* ws, const oskar_B200Cube* cube,
                    const oskar_B200Options* opt, size_t num_points,
                    const void* uu, const void* vv, const void* ww,
                    const void* vis, const void* weight, double cell_size_rad,
                    double w_scale, int grid_size, void* grid,
                    unsigned long long* d_num_skipped, double* d_norm,
                    void* stream)
{
    if (!ws || !cube) return OSKAR_B200_ERR_INVALID_ARGUMENT;
    oskar_B200Options defaults;
    oskar_b200_options_init(&defaults);
    if (!opt) opt = &defaults;
    int st = check_options(opt, cube->data_is_double);
    if (st) return st;
    st = check_grid_args(num_points, uu, vv, ww, vis, weight,
                         opt->apply_weight, grid_size, grid);
    if (st) return st;
    if (cube->device != ws->device) return OSKAR_B200_ERR_INVALID_ARGUMENT;
    DeviceGuard g(ws->device);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ws->stream;
    return run_grid(ws, cube, opt, num_points, uu, vv, ww, vis, weight,
                    cell_size_rad, w_scale, grid_size, grid, d_num_skipped,
                    d_norm, s);
}

int oskar_b200_degrid(oskar_B200Workspace* ws, const oskar_B200Cube* cube,
                      const oskar_B200Options* opt, size_t num_points,
                      const void* uu, const void* vv, const void* ww,
                      const void* weight, double cell_size_rad,
                      double w_scale, int grid_size, const void* grid,
                      void* vis, unsigned long long* d_num_skipped,
                      void* stream)
{
    if (!ws || !cube) return OSKAR_B200_ERR_INVALID_ARGUMENT;
    oskar_B200Options defaults;
    oskar_b200_options_init(&defaults);
    if (!opt) opt = &defaults;
    int st = check_options(opt, cube->data_is_double);
    if (st) return st;
    if (opt->accum_mode != OSKAR_B200_ACCUM_PLAIN)
        return OSKAR_B200_ERR_UNSUPPORTED;
    st = check_grid_args(num_points, uu, vv, ww, vis, weight,
                         opt->apply_weight, grid_size, grid);
    if (st) return st;
    if (cube->device != ws->device) return OSKAR_B200_ERR_INVALID_ARGUMENT;
    DeviceGuard g(ws->device);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ws->stream;
    HostJob j{};
    j.cube = cube;
    j.num_points = num_points;
    j.uu = uu;
    j.vv = vv;
    j.ww = ww;
    j.vis = vis;               // written
    j.weight = weight;
    j.cell_size_rad = cell_size_rad;
    j.w_scale = w_scale;
    j.grid_size = grid_size;
    j.grid = const_cast<void*>(grid);   // read
    j.d_num_skipped = d_num_skipped;
    j.d_norm = nullptr;
    j.frequency_hz = opt->frequency_hz;
    return run_batch(ws, opt, 1, &j, s, true);
}

int oskar_b200_grid_batch(oskar_B200Workspace* ws,
                          const oskar_B200Options* opt, int num_jobs,
                          const oskar_B200Job* jobs, void* stream)
{
    if (!ws || !jobs || num_jobs < 1 || num_jobs > (1 << 15))
        return OSKAR_B200_ERR_INVALID_ARGUMENT;
    oskar_B200Options defaults;
    oskar_b200_options_init(&defaults);
    if (!opt) opt = &defaults;
    const oskar_B200Cube* c0 = jobs[0].cube;
    if (!c0) return OSKAR_B200_ERR_INVALID_ARGUMENT;
    int st = check_options(opt, c0->data_is_double);
    if (st) return st;
    std::vector<HostJob> hj((size_t)num_jobs);
    for (int j = 0; j < num_jobs; ++j)
    {
        const oskar_B200Job& in = jobs[j];
        if (!in.cube || in.cube->device != ws->device ||
            in.cube->data_is_double != c0->data_is_double ||
            in.cube->kernel_type != c0->kernel_type)
            return OSKAR_B200_ERR_INVALID_ARGUMENT;
        st = check_grid_args(in.num_points, in.uu, in.vv, in.ww, in.vis,
                             in.weight, opt->apply_weight, in.grid_size,
                             in.grid);
        if (st) return st;
        if (!(in.frequency_hz >= 0.0) || !std::isfinite(in.frequency_hz))
            return OSKAR_B200_ERR_INVALID_ARGUMENT;
        hj[j] = HostJob{in.cube, in.num_points, in.uu, in.vv, in.ww, in.vis,
                        in.weight, in.cell_size_rad, in.w_scale,
                        in.grid_size, in.grid, in.d_num_skipped, in.d_norm,
                        in.frequency_hz};
    }
    DeviceGuard g(ws->device);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ws->stream;
    return run_batch(ws, opt, num_jobs, hj.data(), s);
}

int oskar_b200_place(oskar_B200Workspace* ws, int data_is_double,
                     int coord_mode, size_t num_w_planes, const int* support,
                     int oversample, size_t num_points, const void* uu,
                     const void* vv, const void* ww, double cell_size_rad,
                     double w_scale, int grid_size, int32_t* gu, int32_t* gv,
                     int32_t* plane, int32_t* off_u, int32_t* off_v,
                     int32_t* conj, int32_t* skipped, void* stream)
{
    if (!ws || !support || num_w_planes == 0 || oversample < 1 ||
        grid_size < 1 || (num_points && (!uu || !vv || !ww)))
        return OSKAR_B200_ERR_INVALID_ARGUMENT;
    if (coord_mode != OSKAR_B200_COORDS_F64 &&
        coord_mode != OSKAR_B200_COORDS_REFERENCE_F32)
        return OSKAR_B200_ERR_INVALID_ARGUMENT;
    if (data_is_double && coord_mode != OSKAR_B200_COORDS_F64)
        return OSKAR_B200_ERR_UNSUPPORTED;
    DeviceGuard g(ws->device);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ws->stream;
    DeviceBuffer d_support;
    cudaError_t e = d_support.ensure(sizeof(int) * num_w_planes);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_support.ptr, support, sizeof(int) * num_w_planes,
                            cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return status_from_cuda(e);
    int st = run_place(ws, data_is_double, coord_mode,
                       static_cast<const int*>(d_support.ptr),
                       (int)num_w_planes, oversample, num_points, uu, vv, ww,
                       cell_size_rad, w_scale, grid_size, gu, gv, plane,
                       off_u, off_v, conj, skipped, s);
    e = cudaStreamSynchronize(s);  // d_support is freed on return
    if (!st && e != cudaSuccess) st = status_from_cuda(e);
    return st;
}

int oskar_b200_last_stats(oskar_B200Workspace* ws, oskar_B200Stats* stats)
{
    if (!ws || !stats) return OSKAR_B200_ERR_INVALID_ARGUMENT;
    const unsigned long long* c =
        static_cast<const unsigned long long*>(ws->h_counters);
    memset(stats, 0, sizeof(*stats));
    stats->num_points = ws->last_points;
    stats->num_gridded = ws->last_points - c[CNT_SKIPPED];
    stats->grid_updates = c[CNT_UPDATES];
    stats->num_tasks = c[CNT_TASKS];
    stats->atomic_flushes = c[CNT_FLUSHES];
    stats->status = c[CNT_STATUS] ? (c[CNT_STATUS] & DEV_ERR_TIMEOUT
                                         ? OSKAR_B200_ERR_TIMEOUT
                                         : OSKAR_B200_ERR_DEVICE_CHECK)
                                  : OSKAR_B200_OK;
    stats->kernel_launches = ws->last_launches;
    if (ws->events_recorded)
    {
        DeviceGuard g(ws->device);
        float* out[4] = {&stats->prep_ms, &stats->sort_ms, &stats->tasks_ms,
                         &stats->grid_ms};
        for (int i = 0; i < 4; ++i)
            if (cudaEventElapsedTime(out[i], ws->events[i],
                                     ws->events[i + 1]) != cudaSuccess)
            {
                cudaGetLastError();
                *out[i] = 0.f;
            }
    }
    return OSKAR_B200_OK;
}

int oskar_b200_autotune(oskar_B200Workspace* ws, const oskar_B200Cube* cube,
                        const oskar_B200Options* opt, size_t num_points,
                        const void* uu, const void* vv, const void* ww,
                        const void* vis, double cell_size_rad,
                        double w_scale, int grid_size, void* grid,
                        unsigned char* table_out)
{
    if (!ws || !cube) return OSKAR_B200_ERR_INVALID_ARGUMENT;
    oskar_B200Options defaults;
    oskar_b200_options_init(&defaults);
    if (!opt) opt = &defaults;
    int st = check_options(opt, cube->data_is_double);
    if (st) return st;
    st = check_grid_args(num_points, uu, vv, ww, vis, nullptr, 0, grid_size,
                         grid);
    if (st) return st;
    if (cube->device != ws->device) return OSKAR_B200_ERR_INVALID_ARGUMENT;
    DeviceGuard g(ws->device);
    return run_autotune(ws, cube, opt, num_points, uu, vv, ww, vis,
                        cell_size_rad, w_scale, grid_size, grid, table_out);
}

int oskar_b200_tune_table(oskar_B200Workspace* ws, const unsigned char* table,
                          unsigned char* current)
{
    if (!ws) return OSKAR_B200_ERR_INVALID_ARGUMENT;
    if (table)
    {
        for (int s = 0; s < 128; ++s)
            if (!(table[s] >= 1 && table[s] <= 6))
                return OSKAR_B200_ERR_INVALID_ARGUMENT;
        memcpy(ws->tune, table, sizeof(ws->tune));
        ws->tuned = 1;
    }
    if (current)
    {
        if (ws->tuned)
            memcpy(current, ws->tune, sizeof(ws->tune));
        else
            default_tune_table(current);
    }
    return OSKAR_B200_OK;
}

int oskar_b200_tune_launch(oskar_B200Workspace* ws, const int* set,
                           int* current)
{
    if (!ws) return OSKAR_B200_ERR_INVALID_ARGUMENT;
    if (set)
    {
        if ((set[0] != 0 && (set[0] < 6 || set[0] > 15)) ||
            (set[1] != 1 && set[1] != 2) || set[2] < 0)
            return OSKAR_B200_ERR_INVALID_ARGUMENT;
        ws->tuned_tile_shift = set[0];
        ws->tuned_staging = set[1];
        ws->tuned_comp_radius = set[2];
        ws->tuned_launch = 1;
    }
    if (current)
    {
        current[0] = ws->tuned_launch ? ws->tuned_tile_shift : 0;
        current[1] = ws->tuned_launch ? ws->tuned_staging : 2;
        current[2] = ws->tuned_launch ? ws->tuned_comp_radius : 0;
    }
    return OSKAR_B200_OK;
}

int oskar_b200_set_stage_timing(oskar_B200Workspace* ws, int enable)
{
    if (!ws) return OSKAR_B200_ERR_INVALID_ARGUMENT;
    DeviceGuard g(ws->device);
    if (enable)
        for (cudaEvent_t& e : ws->events)
            if (!e)
            {
                const cudaError_t r = cudaEventCreate(&e);
                if (r != cudaSuccess) return status_from_cuda(r);
            }
    ws->stage_timing = enable & 3;
    ws->events_recorded = 0;
    return OSKAR_B200_OK;
}

int oskar_b200_measure_atomic_rate(oskar_B200Workspace* ws, void* grid,
                                   int grid_size, int iters,
                                   double* updates_per_s)
{
    if (!ws || !grid || !updates_per_s) return OSKAR_B200_ERR_INVALID_ARGUMENT;
    DeviceGuard g(ws->device);
    return measure_atomic_rate(ws, grid, grid_size, iters, updates_per_s);
}

const char* oskar_b200_build_info(void)
{
    return "fpga_gridding_b200 gridder; sm_100a; CUDA "
#if defined(CUDART_VERSION)
           B200_STR(CUDART_VERSION)
#endif
        ;
}

}  // extern "C"

extern "C" int oskar_b200_testing_fail_allocation(long long after)
{
    if (after < -1) return OSKAR_B200_ERR_INVALID_ARGUMENT;
    g_alloc_countdown.store(after);
    return OSKAR_B200_OK;
}

extern "C" int oskar_b200_selftest_bounded_wait(oskar_B200Workspace* ws,
                                                unsigned spins,
                                                int* device_status)
{
    if (!ws || !device_status || spins == 0)
        return OSKAR_B200_ERR_INVALID_ARGUMENT;
    DeviceGuard g(ws->device);
    return selftest_bounded_wait(ws, spins, device_status);
}

// ---------------------------------------------------------------------------
// Uniform weighting: drop-ins for utils/oskar_grid_weights.c and the
// device-resident calls.
// ---------------------------------------------------------------------------
namespace {

int check_weights_args(size_t num_points, const void* uu, const void* vv,
                       const void* weight, int grid_size, const void* grid)
{
    if (grid_size < 1 || grid_size > 65535 || !grid)
        return OSKAR_B200_ERR_INVALID_ARGUMENT;
    if (num_points >= 0xffffffffull) return OSKAR_B200_ERR_INVALID_ARGUMENT;
    if (num_points && (!uu || !vv || !weight))
        return OSKAR_B200_ERR_INVALID_ARGUMENT;
    return OSKAR_B200_OK;
}

// The calling thread's cached workspace on its current device.
int dropin_workspace(oskar_B200Workspace** out)
{
    int device = 0;
    int st = current_device(&device);
    if (st) return st;
    ThreadCache& tc = tls_cache;
    if (tc.ws && tc.ws->device != device) tc.release();
    if (!tc.ws)
    {
        st = workspace_create(device, &tc.ws);
        if (st) return st;
    }
    *out = tc.ws;
    return OSKAR_B200_OK;
}

#define B200_WCHECK(expr)                                           \
    do {                                                            \
        const cudaError_t e_ = (expr);                              \
        if (e_ != cudaSuccess) { cudaStreamSynchronize(s);          \
                                 cudaGetLastError();                \
                                 return status_from_cuda(e_); }     \
    } while (0)

// Chunks of the pipelined host-array calls (weights drop-ins, host
// degridding): about kIngestChunk points each.
int pipeline_chunks(size_t n)
{
    if (n == 0) return 1;
    return (int)std::min<size_t>(kIngestEvents - 2,
                                 (n + kIngestChunk - 1) / kIngestChunk);
}

// Copy streams and events of the pipelined host-array calls (created on
// first use).
cudaError_t pipeline_streams(oskar_B200Workspace* ws)
{
    cudaError_t e = cudaSuccess;
    if (!ws->copy_stream)
        e = cudaStreamCreateWithFlags(&ws->copy_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess && !ws->d2h_stream)
        e = cudaStreamCreateWithFlags(&ws->d2h_stream, cudaStreamNonBlocking);
    for (cudaEvent_t& ev : ws->ingest_events)
        if (e == cudaSuccess && !ev)
            e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    for (cudaEvent_t& ev : ws->band_events)
        if (e == cudaSuccess && !ev)
            e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    return e;
}

// oskar_grid_weights_write_{d,f} on host arrays: ordered (bit-exact) write.
// The caller's grid goes up first, then the points in chunks on the copy
// stream; each chunk is written into the grid as it lands, in order (so
// every cell still sums its weights in input order, starting from the
// caller's value), while the next chunk crosses PCIe.
template <typename T>
int weights_write_drop_in(size_t n, const T* uu, const T* vv,
                          const T* weight, double cell_size_rad,
                          int grid_size, size_t* num_skipped, T* grid)
{
    if (!num_skipped) return OSKAR_B200_ERR_INVALID_ARGUMENT;
    int st = check_weights_args(n, uu, vv, weight, grid_size, grid);
    if (st) return st;
    oskar_B200Workspace* ws = nullptr;
    st = dropin_workspace(&ws);
    if (st) return st;
    cudaStream_t s = ws->stream;
    auto sync_all = [&]() {
        cudaStreamSynchronize(s);
        if (ws->copy_stream) cudaStreamSynchronize(ws->copy_stream);
        if (ws->d2h_stream) cudaStreamSynchronize(ws->d2h_stream);
        cudaGetLastError();
    };
#define B200_PCHECK(expr)                                           \
    do {                                                            \
        const cudaError_t e_ = (expr);                              \
        if (e_ != cudaSuccess) { sync_all();                        \
                                 return status_from_cuda(e_); }     \
    } while (0)
    B200_PCHECK(pipeline_streams(ws));
    cudaStream_t c = ws->copy_stream;
    const size_t grid_bytes = (size_t)grid_size * grid_size * sizeof(T);
    const int chunks = pipeline_chunks(n);
    B200_PCHECK(ws->in_grid.ensure(grid_bytes));
    B200_PCHECK(ws->in_norm.ensure(sizeof(unsigned long long) * chunks));
    if (n)
    {
        B200_PCHECK(ws->in_uu.ensure(n * sizeof(T)));
        B200_PCHECK(ws->in_vv.ensure(n * sizeof(T)));
        B200_PCHECK(ws->in_weight.ensure(n * sizeof(T)));
    }
    B200_PCHECK(cudaMemcpyAsync(ws->in_grid.ptr, grid, grid_bytes,
                                cudaMemcpyHostToDevice, c));
    unsigned long long* d_skip =
        static_cast<unsigned long long*>(ws->in_norm.ptr);
    for (int k = 0; k < chunks; ++k)
    {
        const size_t b = n * (size_t)k / (size_t)chunks;
        const size_t m = n * (size_t)(k + 1) / (size_t)chunks - b;
        T* du = static_cast<T*>(ws->in_uu.ptr) + b;
        T* dv = static_cast<T*>(ws->in_vv.ptr) + b;
        T* dw = static_cast<T*>(ws->in_weight.ptr) + b;
        if (m)
        {
            B200_PCHECK(cudaMemcpyAsync(du, uu + b, m * sizeof(T),
                                        cudaMemcpyHostToDevice, c));
            B200_PCHECK(cudaMemcpyAsync(dv, vv + b, m * sizeof(T),
                                        cudaMemcpyHostToDevice, c));
            B200_PCHECK(cudaMemcpyAsync(dw, weight + b, m * sizeof(T),
                                        cudaMemcpyHostToDevice, c));
        }
        B200_PCHECK(cudaEventRecord(ws->ingest_events[k], c));
        B200_PCHECK(cudaStreamWaitEvent(s, ws->ingest_events[k], 0));
        st = run_weights_write(ws, sizeof(T) == sizeof(double), 1, m, du, dv,
                               dw, cell_size_rad, grid_size, ws->in_grid.ptr,
                               d_skip + k, 0.0, s);
        if (st) { sync_all(); return st; }
    }
    B200_PCHECK(cudaStreamSynchronize(s));
    B200_PCHECK(cudaStreamSynchronize(c));
    std::vector<unsigned long long> skips(chunks);
    B200_PCHECK(cudaMemcpyAsync(skips.data(), d_skip,
                                sizeof(unsigned long long) * chunks,
                                cudaMemcpyDeviceToHost, s));
    B200_PCHECK(cudaMemcpyAsync(grid, ws->in_grid.ptr, grid_bytes,
                                cudaMemcpyDeviceToHost, s));
    B200_PCHECK(cudaStreamSynchronize(s));
    unsigned long long skipped = 0;
    for (unsigned long long x : skips) skipped += x;
    *num_skipped = (size_t)skipped;
    return OSKAR_B200_OK;
}

// oskar_grid_weights_read_{d,f} on host arrays.  weight_out is uploaded as
// well: the entries of skipped points keep their previous values.  The
// caller's grid goes up first, then the points in chunks; each chunk is
// read as it lands and its weight_out goes back on a third stream while
// later chunks still cross PCIe.
template <typename T>
int weights_read_drop_in(size_t n, const T* uu, const T* vv,
                         const T* weight_in, T* weight_out,
                         double cell_size_rad, int grid_size,
                         size_t* num_skipped, const T* grid)
{
    if (!num_skipped || (n && !weight_out))
        return OSKAR_B200_ERR_INVALID_ARGUMENT;
    int st = check_weights_args(n, uu, vv, weight_in, grid_size, grid);
    if (st) return st;
    oskar_B200Workspace* ws = nullptr;
    st = dropin_workspace(&ws);
    if (st) return st;
    cudaStream_t s = ws->stream;
    auto sync_all = [&]() {
        cudaStreamSynchronize(s);
        if (ws->copy_stream) cudaStreamSynchronize(ws->copy_stream);
        if (ws->d2h_stream) cudaStreamSynchronize(ws->d2h_stream);
        cudaGetLastError();
    };
    B200_PCHECK(pipeline_streams(ws));
    cudaStream_t c = ws->copy_stream;
    cudaStream_t d = ws->d2h_stream;
    const size_t grid_bytes = (size_t)grid_size * grid_size * sizeof(T);
    const int chunks = pipeline_chunks(n);
    B200_PCHECK(ws->in_grid.ensure(grid_bytes));
    B200_PCHECK(ws->in_norm.ensure(sizeof(unsigned long long) * chunks));
    if (n)
    {
        B200_PCHECK(ws->in_uu.ensure(n * sizeof(T)));
        B200_PCHECK(ws->in_vv.ensure(n * sizeof(T)));
        B200_PCHECK(ws->in_weight.ensure(n * sizeof(T)));
        B200_PCHECK(ws->in_vis.ensure(n * sizeof(T)));
    }
    B200_PCHECK(cudaMemcpyAsync(ws->in_grid.ptr, grid, grid_bytes,
                                cudaMemcpyHostToDevice, c));
    unsigned long long* d_skip =
        static_cast<unsigned long long*>(ws->in_norm.ptr);
    for (int k = 0; k < chunks; ++k)
    {
        const size_t b = n * (size_t)k / (size_t)chunks;
        const size_t m = n * (size_t)(k + 1) / (size_t)chunks - b;
        T* du = static_cast<T*>(ws->in_uu.ptr) + b;
        T* dv = static_cast<T*>(ws->in_vv.ptr) + b;
        T* dw = static_cast<T*>(ws->in_weight.ptr) + b;
        T* dout = static_cast<T*>(ws->in_vis.ptr) + b;
        if (m)
        {
            B200_PCHECK(cudaMemcpyAsync(du, uu + b, m * sizeof(T),
                                        cudaMemcpyHostToDevice, c));
            B200_PCHECK(cudaMemcpyAsync(dv, vv + b, m * sizeof(T),
                                        cudaMemcpyHostToDevice, c));
            B200_PCHECK(cudaMemcpyAsync(dw, weight_in + b, m * sizeof(T),
                                        cudaMemcpyHostToDevice, c));
            B200_PCHECK(cudaMemcpyAsync(dout, weight_out + b, m * sizeof(T),
                                        cudaMemcpyHostToDevice, c));
        }
        B200_PCHECK(cudaEventRecord(ws->ingest_events[k], c));
        B200_PCHECK(cudaStreamWaitEvent(s, ws->ingest_events[k], 0));
        st = run_weights_read(ws, sizeof(T) == sizeof(double), m, du, dv, dw,
                              dout, cell_size_rad, grid_size, ws->in_grid.ptr,
                              d_skip + k, 0.0, s);
        if (st) { sync_all(); return st; }
        if (m)
        {
            // (every upload of this chunk happened before the event above,
            // so its host rows are read before they are overwritten)
            B200_PCHECK(cudaEventRecord(ws->band_events[k], s));
            B200_PCHECK(cudaStreamWaitEvent(d, ws->band_events[k], 0));
            B200_PCHECK(cudaMemcpyAsync(weight_out + b, dout, m * sizeof(T),
                                        cudaMemcpyDeviceToHost, d));
        }
    }
    B200_PCHECK(cudaStreamSynchronize(s));
    B200_PCHECK(cudaStreamSynchronize(c));
    B200_PCHECK(cudaStreamSynchronize(d));
    std::vector<unsigned long long> skips(chunks);
    B200_PCHECK(cudaMemcpyAsync(skips.data(), d_skip,
                                sizeof(unsigned long long) * chunks,
                                cudaMemcpyDeviceToHost, s));
    B200_PCHECK(cudaStreamSynchronize(s));
    unsigned long long skipped = 0;
    for (unsigned long long x : skips) skipped += x;
    *num_skipped = (size_t)skipped;
    return OSKAR_B200_OK;
}

#undef B200_PCHECK

// oskar_grid_wproj_f_diagnostics on the caller's host arrays: the gridding
// (grid, norm, skip count) as oskar_grid_wproj_f with the reference's float
// coordinate arithmetic, then the hit counts (diagnostics.cu).  Histogram
// sizes: num_vis_per_wsupport covers support values 0 .. max(support),
// num_vis_per_wplane the unclamped plane indices of the points, as the
// reference indexes them.  Every result goes back only after the device
// work has succeeded.
int diagnostics_drop_in(size_t num_w_planes, const int* support,
                        int oversample, int conv_size_half,
                        const float* conv_func, size_t n, const float* uu,
                        const float* vv, const float* ww, const float* vis,
                        float cell_size_rad, float w_scale, int grid_size,
                        size_t* num_skipped, double* norm, float* grid,
                        long long* num_vis_per_wsupport,
                        long long* num_vis_per_wplane,
                        long long* num_vis_per_grid,
                        float* avg_wsupport_per_grid)
{
    if (!num_skipped || !norm || !grid || !num_vis_per_wsupport ||
        !num_vis_per_wplane || !num_vis_per_grid || !avg_wsupport_per_grid)
        return OSKAR_B200_ERR_INVALID_ARGUMENT;
    int st = validate_cube_args(num_w_planes, support, oversample,
                                conv_size_half, conv_func);
    if (st) return st;
    st = check_grid_args(n, uu, vv, ww, vis, nullptr, 0, grid_size, grid);
    if (st) return st;
    oskar_B200Workspace* ws = nullptr;
    st = dropin_workspace(&ws);
    if (st) return st;
    ThreadCache& tc = tls_cache;
    if (!tc.cube)
    {
        tc.cube = new (std::nothrow) oskar_B200Cube();
        if (!tc.cube) return OSKAR_B200_ERR_OUT_OF_MEMORY;
    }
    cudaStream_t s = ws->stream;
#define B200_DCHECK(expr)                                           \
    do {                                                            \
        const cudaError_t e_ = (expr);                              \
        if (e_ != cudaSuccess) { cudaStreamSynchronize(s);          \
                                 cudaGetLastError();                \
                                 return status_from_cuda(e_); }     \
    } while (0)
    const size_t G = (size_t)grid_size, cells = G * G;
    const size_t cube_elems = num_w_planes * (size_t)conv_size_half *
                              conv_size_half * 2;
    int max_support = 0;
    for (size_t p = 0; p < num_w_planes; ++p)
        max_support = std::max(max_support, support[p]);
    const size_t ns = (size_t)max_support + 1;
    B200_DCHECK(ws->in_cube.ensure(cube_elems * sizeof(float)));
    B200_DCHECK(ws->in_grid.ensure(2 * cells * sizeof(float)));
    B200_DCHECK(ws->in_norm.ensure(8 * sizeof(unsigned long long)));
    if (n)
    {
        B200_DCHECK(ws->in_uu.ensure(n * sizeof(float)));
        B200_DCHECK(ws->in_vv.ensure(n * sizeof(float)));
        B200_DCHECK(ws->in_ww.ensure(n * sizeof(float)));
        B200_DCHECK(ws->in_vis.ensure(2 * n * sizeof(float)));
    }
    DeviceBuffer d_per_support, d_per_plane, d_per_cell, d_cell_sum;
    B200_DCHECK(d_per_support.ensure(ns * sizeof(long long)));
    B200_DCHECK(d_per_cell.ensure(cells * sizeof(long long)));
    B200_DCHECK(d_cell_sum.ensure(cells * sizeof(float)));
    const float* du = static_cast<const float*>(ws->in_uu.ptr);
    const float* dv = static_cast<const float*>(ws->in_vv.ptr);
    const float* dw = static_cast<const float*>(ws->in_ww.ptr);
    unsigned long long* small =
        static_cast<unsigned long long*>(ws->in_norm.ptr);
    // small: [0] norm (double), [1] skip count, [2] device status,
    // [3] largest unclamped plane, [4] unusable plane flag
    B200_DCHECK(cudaMemcpyAsync(ws->in_cube.ptr, conv_func,
                                cube_elems * sizeof(float),
                                cudaMemcpyHostToDevice, s));
    st = cube_init(tc.cube, ws->device, num_w_planes, support, oversample,
                   conv_size_half, ws->in_cube.ptr, nullptr, 0, 0,
                   OSKAR_B200_KERNEL_NATIVE, s);
    if (st) { cudaStreamSynchronize(s); cudaGetLastError(); return st; }
    if (n)
    {
        B200_DCHECK(cudaMemcpyAsync(ws->in_uu.ptr, uu, n * sizeof(float),
                                    cudaMemcpyHostToDevice, s));
        B200_DCHECK(cudaMemcpyAsync(ws->in_vv.ptr, vv, n * sizeof(float),
                                    cudaMemcpyHostToDevice, s));
        B200_DCHECK(cudaMemcpyAsync(ws->in_ww.ptr, ww, n * sizeof(float),
                                    cudaMemcpyHostToDevice, s));
        B200_DCHECK(cudaMemcpyAsync(ws->in_vis.ptr, vis,
                                    2 * n * sizeof(float),
                                    cudaMemcpyHostToDevice, s));
    }
    // The largest unclamped plane index sizes num_vis_per_wplane.
    const float w_scale_f = w_scale;
    B200_DCHECK(launch_diag_max_plane(dw, n, w_scale_f, small + 3,
                                      ws->num_sms, s));
    unsigned long long plane_info[2] = {0, 0};
    B200_DCHECK(cudaMemcpyAsync(plane_info, small + 3, sizeof(plane_info),
                                cudaMemcpyDeviceToHost, s));
    B200_DCHECK(cudaStreamSynchronize(s));
    if (plane_info[1]) return OSKAR_B200_ERR_INVALID_ARGUMENT;
    const size_t np = n ? (size_t)plane_info[0] + 1 : 0;
    if (np) B200_DCHECK(d_per_plane.ensure(np * sizeof(long long)));
    // The caller's arrays accumulate: their current contents go up.
    B200_DCHECK(cudaMemcpyAsync(ws->in_grid.ptr, grid,
                                2 * cells * sizeof(float),
                                cudaMemcpyHostToDevice, s));
    B200_DCHECK(cudaMemcpyAsync(d_per_support.ptr, num_vis_per_wsupport,
                                ns * sizeof(long long),
                                cudaMemcpyHostToDevice, s));
    if (np)
        B200_DCHECK(cudaMemcpyAsync(d_per_plane.ptr, num_vis_per_wplane,
                                    np * sizeof(long long),
                                    cudaMemcpyHostToDevice, s));
    B200_DCHECK(cudaMemcpyAsync(d_per_cell.ptr, num_vis_per_grid,
                                cells * sizeof(long long),
                                cudaMemcpyHostToDevice, s));
    B200_DCHECK(cudaMemcpyAsync(d_cell_sum.ptr, avg_wsupport_per_grid,
                                cells * sizeof(float),
                                cudaMemcpyHostToDevice, s));
    B200_DCHECK(cudaMemsetAsync(small, 0, 3 * sizeof(unsigned long long),
                                s));
    double* d_norm = reinterpret_cast<double*>(small);
    oskar_B200Options opt;
    oskar_b200_options_init(&opt);
    opt.coord_mode = OSKAR_B200_COORDS_REFERENCE_F32;
    HostJob j{};
    j.cube = tc.cube;
    j.num_points = n;
    j.uu = du;
    j.vv = dv;
    j.ww = dw;
    j.vis = ws->in_vis.ptr;
    j.cell_size_rad = cell_size_rad;
    j.w_scale = w_scale;
    j.grid_size = grid_size;
    j.grid = ws->in_grid.ptr;
    j.d_num_skipped = small + 1;
    j.d_norm = d_norm;
    st = run_batch(ws, &opt, 1, &j, s, false, nullptr);
    if (st) { cudaStreamSynchronize(s); cudaGetLastError(); return st; }
    B200_DCHECK(launch_status_or(ws, small + 2, s));
    PlaceConsts pc{};
    pc.grid_scale = (double)grid_size * (double)cell_size_rad;
    pc.w_scale = w_scale;
    pc.grid_scale_f = (float)grid_size * cell_size_rad;
    pc.w_scale_f = w_scale_f;
    pc.grid_size = grid_size;
    pc.centre = grid_size / 2;
    pc.num_planes = (int)num_w_planes;
    pc.oversample = oversample;
    B200_DCHECK(launch_diag_counts(
        du, dv, dw, n, pc, static_cast<const int*>(tc.cube->d_support.ptr),
        static_cast<unsigned long long*>(d_per_support.ptr),
        static_cast<unsigned long long*>(d_per_plane.ptr),
        static_cast<unsigned long long*>(d_per_cell.ptr),
        static_cast<float*>(d_cell_sum.ptr), ws->num_sms, s));
    unsigned long long res[3];
    B200_DCHECK(cudaMemcpyAsync(res, small, sizeof(res),
                                cudaMemcpyDeviceToHost, s));
    B200_DCHECK(cudaStreamSynchronize(s));
    if (res[2]) return res[2] & DEV_ERR_TIMEOUT ? OSKAR_B200_ERR_TIMEOUT
                                                : OSKAR_B200_ERR_DEVICE_CHECK;
    B200_DCHECK(cudaMemcpyAsync(grid, ws->in_grid.ptr,
                                2 * cells * sizeof(float),
                                cudaMemcpyDeviceToHost, s));
    B200_DCHECK(cudaMemcpyAsync(num_vis_per_wsupport, d_per_support.ptr,
                                ns * sizeof(long long),
                                cudaMemcpyDeviceToHost, s));
    if (np)
        B200_DCHECK(cudaMemcpyAsync(num_vis_per_wplane, d_per_plane.ptr,
                                    np * sizeof(long long),
                                    cudaMemcpyDeviceToHost, s));
    B200_DCHECK(cudaMemcpyAsync(num_vis_per_grid, d_per_cell.ptr,
                                cells * sizeof(long long),
                                cudaMemcpyDeviceToHost, s));
    B200_DCHECK(cudaMemcpyAsync(avg_wsupport_per_grid, d_cell_sum.ptr,
                                cells * sizeof(float),
                                cudaMemcpyDeviceToHost, s));
    B200_DCHECK(cudaStreamSynchronize(s));
#undef B200_DCHECK
    double nrm;
    memcpy(&nrm, &res[0], sizeof(nrm));
    *norm += nrm;
    *num_skipped = (size_t)res[1];
    return OSKAR_B200_OK;
}

#undef B200_WCHECK

}  // namespace

extern "C" {

void oskar_grid_wproj_f_diagnostics(const size_t num_w_planes,
        const int* support, const int oversample, const int conv_size_half,
        const float* conv_func, const size_t num_points, const float* uu,
        const float* vv, const float* ww, const float* vis,
        const float* weight, const float cell_size_rad, const float w_scale,
        const int grid_size, size_t* num_skipped, double* norm, float* grid,
        long long int* num_vis_per_wsupport, long long int* num_vis_per_wplane,
        long long int* num_vis_per_grid, float* avg_wsupport_per_grid,
        float* avg_wplane_per_grid)
{
    (void)weight;               // ignored, as in oskar_grid_wproj.c:299-300
    (void)avg_wplane_per_grid;  // never written by the reference either
    tls_status = diagnostics_drop_in(
        num_w_planes, support, oversample, conv_size_half, conv_func,
        num_points, uu, vv, ww, vis, cell_size_rad, w_scale, grid_size,
        num_skipped, norm, grid, num_vis_per_wsupport, num_vis_per_wplane,
        num_vis_per_grid, avg_wsupport_per_grid);
}

void oskar_grid_weights_write_d(const size_t num_points, const double* uu,
                                const double* vv, const double* weight,
                                const double cell_size_rad,
                                const int grid_size, size_t* num_skipped,
                                double* grid)
{
    tls_status = weights_write_drop_in<double>(num_points, uu, vv, weight,
                                               cell_size_rad, grid_size,
                                               num_skipped, grid);
}

void oskar_grid_weights_read_d(const size_t num_points, const double* uu,
                               const double* vv, const double* weight_in,
                               double* weight_out, const double cell_size_rad,
                               const int grid_size, size_t* num_skipped,
                               const double* grid)
{
    tls_status = weights_read_drop_in<double>(num_points, uu, vv, weight_in,
                                              weight_out, cell_size_rad,
                                              grid_size, num_skipped, grid);
}

void oskar_grid_weights_write_f(const size_t num_points, const float* uu,
                                const float* vv, const float* weight,
                                const float cell_size_rad,
                                const int grid_size, size_t* num_skipped,
                                float* grid)
{
    tls_status = weights_write_drop_in<float>(num_points, uu, vv, weight,
                                              (double)cell_size_rad,
                                              grid_size, num_skipped, grid);
}

void oskar_grid_weights_read_f(const size_t num_points, const float* uu,
                               const float* vv, const float* weight_in,
                               float* weight_out, const float cell_size_rad,
                               const int grid_size, size_t* num_skipped,
                               const float* grid)
{
    tls_status = weights_read_drop_in<float>(num_points, uu, vv, weight_in,
                                             weight_out,
                                             (double)cell_size_rad,
                                             grid_size, num_skipped, grid);
}

int oskar_b200_weights_write(oskar_B200Workspace* ws, int data_is_double,
                             int ordered, size_t num_points, const void* uu,
                             const void* vv, const void* weight,
                             double cell_size_rad, int grid_size, void* grid,
                             unsigned long long* d_num_skipped,
                             double frequency_hz, void* stream)
{
    if (!ws || !(frequency_hz >= 0.0) || !std::isfinite(frequency_hz))
        return OSKAR_B200_ERR_INVALID_ARGUMENT;
    int st = check_weights_args(num_points, uu, vv, weight, grid_size, grid);
    if (st) return st;
    DeviceGuard g(ws->device);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ws->stream;
    return run_weights_write(ws, data_is_double ? 1 : 0, ordered ? 1 : 0,
                             num_points, uu, vv, weight, cell_size_rad,
                             grid_size, grid, d_num_skipped, frequency_hz, s);
}

int oskar_b200_weights_read(oskar_B200Workspace* ws, int data_is_double,
                            size_t num_points, const void* uu,
                            const void* vv, const void* weight_in,
                            void* weight_out, double cell_size_rad,
                            int grid_size, const void* grid,
                            unsigned long long* d_num_skipped,
                            double frequency_hz, void* stream)
{
    if (!ws || (num_points && !weight_out) || !(frequency_hz >= 0.0) ||
        !std::isfinite(frequency_hz))
        return OSKAR_B200_ERR_INVALID_ARGUMENT;
    int st = check_weights_args(num_points, uu, vv, weight_in, grid_size,
                                grid);
    if (st) return st;
    DeviceGuard g(ws->device);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ws->stream;
    return run_weights_read(ws, data_is_double ? 1 : 0, num_points, uu, vv,
                            weight_in, weight_out, cell_size_rad, grid_size,
                            grid, d_num_skipped, frequency_hz, s);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Degridding of host arrays, with the copies overlapped
// ---------------------------------------------------------------------------
extern "C" {

// The caller's grid goes up first (every chunk reads all of it), then the
// visibilities' coordinates (and their current values: skipped ones keep
// them) in chunks on the copy stream; each chunk is degridded as it lands
// and its predicted visibilities go back on a third stream while later
// chunks still cross PCIe.
int oskar_b200_degrid_host(oskar_B200Workspace* ws, const oskar_B200Cube* cube,
                           const oskar_B200Options* opt, size_t num_points,
                           const void* uu, const void* vv, const void* ww,
                           const void* weight, double cell_size_rad,
                           double w_scale, int grid_size, const void* grid,
                           void* vis, size_t* num_skipped)
{
    if (!ws || !cube || !num_skipped) return OSKAR_B200_ERR_INVALID_ARGUMENT;
    oskar_B200Options defaults;
    oskar_b200_options_init(&defaults);
    if (!opt) opt = &defaults;
    int st = check_options(opt, cube->data_is_double);
    if (st) return st;
    if (opt->accum_mode != OSKAR_B200_ACCUM_PLAIN)
        return OSKAR_B200_ERR_UNSUPPORTED;
    st = check_grid_args(num_points, uu, vv, ww, vis, weight,
                         opt->apply_weight, grid_size, grid);
    if (st) return st;
    if (cube->device != ws->device) return OSKAR_B200_ERR_INVALID_ARGUMENT;
    DeviceGuard g(ws->device);
    cudaStream_t s = ws->stream;
    auto sync_all = [&]() {
        cudaStreamSynchronize(s);
        if (ws->copy_stream) cudaStreamSynchronize(ws->copy_stream);
        if (ws->d2h_stream) cudaStreamSynchronize(ws->d2h_stream);
        cudaGetLastError();
    };
#define B200_DCHECK(expr)                                           \
    do {                                                            \
        const cudaError_t e_ = (expr);                              \
        if (e_ != cudaSuccess) { sync_all();                        \
                                 return status_from_cuda(e_); }     \
    } while (0)
    B200_DCHECK(pipeline_streams(ws));
    cudaStream_t c = ws->copy_stream;
    cudaStream_t d = ws->d2h_stream;
    const size_t n = num_points;
    const size_t T = cube->data_is_double ? sizeof(double) : sizeof(float);
    const bool weighted = opt->apply_weight != 0;
    const size_t grid_bytes = 2 * (size_t)grid_size * grid_size * T;
    const int chunks = pipeline_chunks(n);
    // [status of every chunk OR-ed, skip count of each chunk]
    B200_DCHECK(ws->in_norm.ensure(sizeof(unsigned long long) *
                                   (1 + (size_t)chunks)));
    B200_DCHECK(ws->in_grid.ensure(grid_bytes));
    if (n)
    {
        B200_DCHECK(ws->in_uu.ensure(n * T));
        B200_DCHECK(ws->in_vv.ensure(n * T));
        B200_DCHECK(ws->in_ww.ensure(n * T));
        B200_DCHECK(ws->in_vis.ensure(2 * n * T));
        if (weighted) B200_DCHECK(ws->in_weight.ensure(n * T));
    }
    unsigned long long* d_status =
        static_cast<unsigned long long*>(ws->in_norm.ptr);
    unsigned long long* d_skip = d_status + 1;
    B200_DCHECK(cudaMemsetAsync(d_status, 0,
                                sizeof(unsigned long long) * (1 + chunks), s));
    B200_DCHECK(cudaMemcpyAsync(ws->in_grid.ptr, grid, grid_bytes,
                                cudaMemcpyHostToDevice, c));
    cudaEvent_t ev_grid = ws->ingest_events[kIngestEvents - 1];
    B200_DCHECK(cudaEventRecord(ev_grid, c));
    B200_DCHECK(cudaStreamWaitEvent(s, ev_grid, 0));
    const unsigned char* h_uu = static_cast<const unsigned char*>(uu);
    const unsigned char* h_vv = static_cast<const unsigned char*>(vv);
    const unsigned char* h_ww = static_cast<const unsigned char*>(ww);
    const unsigned char* h_w = static_cast<const unsigned char*>(weight);
    unsigned char* h_vis = static_cast<unsigned char*>(vis);
    for (int k = 0; k < chunks; ++k)
    {
        const size_t b = n * (size_t)k / (size_t)chunks;
        const size_t m = n * (size_t)(k + 1) / (size_t)chunks - b;
        unsigned char* du = static_cast<unsigned char*>(ws->in_uu.ptr) + b * T;
        unsigned char* dv = static_cast<unsigned char*>(ws->in_vv.ptr) + b * T;
        unsigned char* dw = static_cast<unsigned char*>(ws->in_ww.ptr) + b * T;
        unsigned char* dz = static_cast<unsigned char*>(ws->in_vis.ptr) +
                            2 * b * T;
        unsigned char* dwt = weighted
            ? static_cast<unsigned char*>(ws->in_weight.ptr) + b * T
            : nullptr;
        if (m)
        {
            B200_DCHECK(cudaMemcpyAsync(du, h_uu + b * T, m * T,
                                        cudaMemcpyHostToDevice, c));
            B200_DCHECK(cudaMemcpyAsync(dv, h_vv + b * T, m * T,
                                        cudaMemcpyHostToDevice, c));
            B200_DCHECK(cudaMemcpyAsync(dw, h_ww + b * T, m * T,
                                        cudaMemcpyHostToDevice, c));
            B200_DCHECK(cudaMemcpyAsync(dz, h_vis + 2 * b * T, 2 * m * T,
                                        cudaMemcpyHostToDevice, c));
            if (weighted)
                B200_DCHECK(cudaMemcpyAsync(dwt, h_w + b * T, m * T,
                                            cudaMemcpyHostToDevice, c));
        }
        B200_DCHECK(cudaEventRecord(ws->ingest_events[k], c));
        B200_DCHECK(cudaStreamWaitEvent(s, ws->ingest_events[k], 0));
        HostJob j{};
        j.cube = cube;
        j.num_points = m;
        j.uu = du;
        j.vv = dv;
        j.ww = dw;
        j.vis = dz;
        j.weight = dwt;
        j.cell_size_rad = cell_size_rad;
        j.w_scale = w_scale;
        j.grid_size = grid_size;
        j.grid = ws->in_grid.ptr;
        j.d_num_skipped = d_skip + k;
        j.d_norm = nullptr;
        j.frequency_hz = opt->frequency_hz;
        st = run_batch(ws, opt, 1, &j, s, true);
        if (st) { sync_all(); return st; }
        // Each chunk resets the workspace's status word: keep its bits.
        B200_DCHECK(launch_status_or(ws, d_status, s));
        if (m)
        {
            B200_DCHECK(cudaEventRecord(ws->band_events[k], s));
            B200_DCHECK(cudaStreamWaitEvent(d, ws->band_events[k], 0));
            B200_DCHECK(cudaMemcpyAsync(h_vis + 2 * b * T, dz, 2 * m * T,
                                        cudaMemcpyDeviceToHost, d));
        }
    }
    B200_DCHECK(cudaStreamSynchronize(s));
    B200_DCHECK(cudaStreamSynchronize(c));
    B200_DCHECK(cudaStreamSynchronize(d));
    std::vector<unsigned long long> out(1 + (size_t)chunks);
    B200_DCHECK(cudaMemcpyAsync(out.data(), d_status,
                                sizeof(unsigned long long) * out.size(),
                                cudaMemcpyDeviceToHost, s));
    B200_DCHECK(cudaStreamSynchronize(s));
#undef B200_DCHECK
    if (out[0]) return out[0] & DEV_ERR_TIMEOUT ? OSKAR_B200_ERR_TIMEOUT
                                                : OSKAR_B200_ERR_DEVICE_CHECK;
    unsigned long long skipped = 0;
    for (int k = 0; k < chunks; ++k) skipped += out[1 + k];
    *num_skipped = (size_t)skipped;
    return OSKAR_B200_OK;
}

}  // extern "C"
