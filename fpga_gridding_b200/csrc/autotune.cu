// Empirical tuning of the gridding kernel's classes per thread (CPT: how
// many footprint rows one thread owns, which sets how the W x W classes of a
// support fill a CTA).  For each support size of a cube, the visibilities of
// a sample job that land on planes of that support are gridded alone with
// every built CPT, timed with CUDA events around the gridding kernel, and
// the fastest is kept in the workspace; supports without enough sample
// points keep the cost-model choice (default_tune_table).  Later gridding
// calls on the workspace with classes_per_thread = 0 use the table.
#include <algorithm>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "grid_romein.cuh"
#include "internal.h"

namespace b200 {

namespace {

constexpr int kChoices[] = {1, 2, 3, 4, 5, 6, 8};
constexpr size_t kMinPoints = 2000;   // fewer: keep the model's choice
constexpr int kRepeats = 3;           // best of three launches

#define B200_TRY(expr)                                      \
    do {                                                    \
        const cudaError_t e_ = (expr);                      \
        if (e_ != cudaSuccess) return status_from_cuda(e_); \
    } while (0)

}  // namespace

int run_autotune(oskar_B200Workspace* ws, const oskar_B200Cube* cube,
                 const oskar_B200Options* opt_in, size_t n, const void* uu,
                 const void* vv, const void* ww, const void* vis,
                 double cell_size_rad, double w_scale, int grid_size,
                 void* grid, unsigned char* table_out)
{
    cudaStream_t st = ws->stream;
    const size_t elem = cube->data_is_double ? sizeof(double) : sizeof(float);
    const int P = cube->num_planes;
    // Placement of the sample (w-plane of each visibility).
    DeviceBuffer d_plane, d_skip;
    B200_TRY(d_plane.ensure(sizeof(int32_t) * (n ? n : 1)));
    B200_TRY(d_skip.ensure(sizeof(int32_t) * (n ? n : 1)));
    oskar_B200Options opt = *opt_in;
    opt.coord_mode = cube->data_is_double ? OSKAR_B200_COORDS_F64
                                          : opt.coord_mode;
    int rs = run_place(ws, cube->data_is_double, opt.coord_mode,
                       static_cast<const int*>(cube->d_support.ptr), P,
                       cube->oversample, n, uu, vv, ww, cell_size_rad,
                       w_scale, grid_size, nullptr, nullptr,
                       static_cast<int32_t*>(d_plane.ptr), nullptr, nullptr,
                       nullptr, static_cast<int32_t*>(d_skip.ptr), st);
    if (rs) return rs;
    std::vector<int32_t> plane(n), skipped(n);
    std::vector<unsigned char> h_uu(n * elem), h_vv(n * elem), h_ww(n * elem),
        h_vis(2 * n * elem);
    if (n)
    {
        B200_TRY(cudaMemcpyAsync(plane.data(), d_plane.ptr, 4 * n,
                                 cudaMemcpyDeviceToHost, st));
        B200_TRY(cudaMemcpyAsync(skipped.data(), d_skip.ptr, 4 * n,
                                 cudaMemcpyDeviceToHost, st));
        B200_TRY(cudaMemcpyAsync(h_uu.data(), uu, n * elem,
                                 cudaMemcpyDeviceToHost, st));
        B200_TRY(cudaMemcpyAsync(h_vv.data(), vv, n * elem,
                                 cudaMemcpyDeviceToHost, st));
        B200_TRY(cudaMemcpyAsync(h_ww.data(), ww, n * elem,
                                 cudaMemcpyDeviceToHost, st));
        B200_TRY(cudaMemcpyAsync(h_vis.data(), vis, 2 * n * elem,
                                 cudaMemcpyDeviceToHost, st));
    }
    B200_TRY(cudaStreamSynchronize(st));

    unsigned char table[kTuneMax];
    default_tune_table(table);
    // Sample indices per support size.
    std::vector<std::vector<uint32_t>> by_support(kTuneMax);
    for (size_t i = 0; i < n; ++i)
    {
        if (skipped[i]) continue;
        const int s = cube->planes[(size_t)plane[i]].support;
        if (s < kTuneMax) by_support[s].push_back((uint32_t)i);
    }
    size_t largest = 0;
    for (const auto& v : by_support) largest = std::max(largest, v.size());
    DeviceBuffer s_uu, s_vv, s_ww, s_vis;
    if (largest)
    {
        B200_TRY(s_uu.ensure(largest * elem));
        B200_TRY(s_vv.ensure(largest * elem));
        B200_TRY(s_ww.ensure(largest * elem));
        B200_TRY(s_vis.ensure(2 * largest * elem));
    }
    std::vector<unsigned char> g_uu, g_vv, g_ww, g_vis;
    const int saved_timing = ws->stage_timing;
    for (cudaEvent_t& e : ws->events)
        if (!e) B200_TRY(cudaEventCreate(&e));
    ws->stage_timing = 1;
    int status = OSKAR_B200_OK;
    for (int s = 0; s < kTuneMax && !status; ++s)
    {
        const auto& idx = by_support[s];
        if (idx.size() < kMinPoints) continue;
        const size_t m = idx.size();
        g_uu.resize(m * elem);
        g_vv.resize(m * elem);
        g_ww.resize(m * elem);
        g_vis.resize(2 * m * elem);
        for (size_t k = 0; k < m; ++k)
        {
            const size_t i = idx[k];
            memcpy(&g_uu[k * elem], &h_uu[i * elem], elem);
            memcpy(&g_vv[k * elem], &h_vv[i * elem], elem);
            memcpy(&g_ww[k * elem], &h_ww[i * elem], elem);
            memcpy(&g_vis[2 * k * elem], &h_vis[2 * i * elem], 2 * elem);
        }
        B200_TRY(cudaMemcpyAsync(s_uu.ptr, g_uu.data(), m * elem,
                                 cudaMemcpyHostToDevice, st));
        B200_TRY(cudaMemcpyAsync(s_vv.ptr, g_vv.data(), m * elem,
                                 cudaMemcpyHostToDevice, st));
        B200_TRY(cudaMemcpyAsync(s_ww.ptr, g_ww.data(), m * elem,
                                 cudaMemcpyHostToDevice, st));
        B200_TRY(cudaMemcpyAsync(s_vis.ptr, g_vis.data(), 2 * m * elem,
                                 cudaMemcpyHostToDevice, st));
        float best_ms = 1e30f;
        int best = table[s];
        for (int c : kChoices)
        {
            opt.classes_per_thread = c;
            float t_min = 1e30f;
            for (int r = 0; r < kRepeats && !status; ++r)
            {
                status = run_grid(ws, cube, &opt, m, s_uu.ptr, s_vv.ptr,
                                  s_ww.ptr, s_vis.ptr, nullptr,
                                  cell_size_rad, w_scale, grid_size, grid,
                                  nullptr, nullptr, st);
                if (status) break;
                const cudaError_t e = cudaStreamSynchronize(st);
                if (e != cudaSuccess) { status = status_from_cuda(e); break; }
                float ms = 0.f;
                if (cudaEventElapsedTime(&ms, ws->events[3], ws->events[4]) ==
                    cudaSuccess)
                    t_min = std::min(t_min, ms);
                else
                    cudaGetLastError();
            }
            if (t_min < best_ms)
            {
                best_ms = t_min;
                best = c;
            }
        }
        table[s] = (unsigned char)best;
    }
    ws->stage_timing = saved_timing;
    if (status) return status;
    memcpy(ws->tune, table, sizeof(table));
    ws->tuned = 1;
    if (table_out) memcpy(table_out, table, sizeof(table));
    return OSKAR_B200_OK;
}

}  // namespace b200
