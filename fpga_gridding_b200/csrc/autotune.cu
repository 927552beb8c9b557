// Empirical tuning of the gridding launch on a sample job.
//  1. Classes per thread (CPT: how many footprint rows one thread owns,
//     which sets how the W x W classes of a support fill a CTA).  For each
//     support size of a cube, the visibilities of the sample that land on
//     planes of that support are gridded alone with every built CPT, timed
//     with CUDA events around the gridding kernel, and the fastest is kept;
//     supports without enough sample points keep the cost-model choice
//     (default_tune_table).
//  2. Tile width and kernel-value path: the whole sample is gridded with
//     the coarse tile (the unit the sort orders work by, hence what a task
//     covers) at the automatic width, half and twice it, each with kernel
//     values read through L1 and staged in shared memory, and the fastest
//     pipeline (prep to gridding) is kept.
//  3. Flush policy, for compensated accumulation: the sample is gridded
//     with compensation everywhere and nowhere, then within the radii
//     holding 50, 75 and 90 % of its visibilities; the smallest radius whose
//     grid lies within a quarter of the uncompensated grid's distance from
//     the fully compensated grid is kept.
// Later gridding calls on the workspace that leave these choices to it use
// the results.  The reference's tiled gridder fixes the corresponding
// choices at compile time (OskarTuningParams,
// oskar_grid_wproj_gpu.cu.old:1646-1655).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "grid_romein.cuh"
#include "internal.h"

namespace b200 {

namespace {

constexpr int kChoices[] = {1, 2, 3, 4, 5, 6};
constexpr size_t kMinPoints = 2000;   // fewer: keep the model's choice
constexpr int kRepeats = 3;           // best of three launches

#define B200_TRY(expr)                                      \
    do {                                                    \
        const cudaError_t e_ = (expr);                      \
        if (e_ != cudaSuccess) return status_from_cuda(e_); \
    } while (0)

// out[0] += sum (a - b)^2, out[1] += sum b^2 over n floats (FP64 sums).
__global__ void diff_norms_kernel(const float* __restrict__ a,
                                  const float* __restrict__ b, size_t n,
                                  double* out)
{
    double d2 = 0.0, b2 = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
    {
        const double d = (double)a[i] - (double)b[i];
        d2 += d * d;
        b2 += (double)b[i] * (double)b[i];
    }
    d2 = warp_sum(d2);
    b2 = warp_sum(b2);
    if ((threadIdx.x & 31) == 0)
    {
        atomicAdd(&out[0], d2);
        atomicAdd(&out[1], b2);
    }
}

// ||a - b|| / ||b|| of two FP32 grids of n floats (synchronous on st).
int grid_distance(const float* a, const float* b, size_t n, int num_sms,
                  double* sums, cudaStream_t st, double* rel)
{
    B200_TRY(cudaMemsetAsync(sums, 0, 2 * sizeof(double), st));
    diff_norms_kernel<<<num_sms * 4, 256, 0, st>>>(a, b, n, sums);
    B200_TRY(cudaGetLastError());
    double h[2] = {0.0, 0.0};
    B200_TRY(cudaMemcpyAsync(h, sums, sizeof(h), cudaMemcpyDeviceToHost, st));
    B200_TRY(cudaStreamSynchronize(st));
    *rel = h[1] > 0.0 ? std::sqrt(h[0] / h[1]) : std::sqrt(h[0]);
    return OSKAR_B200_OK;
}

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
    if (status)
    {
        ws->stage_timing = saved_timing;
        return status;
    }
    memcpy(ws->tune, table, sizeof(table));
    ws->tuned = 1;
    if (table_out) memcpy(table_out, table, sizeof(table));

    // (2) Tile width x kernel-value path on the whole sample, the table
    // above in use; the pipeline from prep to the end of gridding is timed.
    const bool comp = opt_in->accum_mode == OSKAR_B200_ACCUM_COMPENSATED;
    KeyLayout kl;
    if (!make_key_layout(grid_size, P, 1, &kl))
    {
        ws->stage_timing = saved_timing;
        return OSKAR_B200_ERR_UNSUPPORTED;
    }
    int gbits = 0;
    while ((1 << gbits) < grid_size) ++gbits;
    std::vector<int> shifts = {kl.coarse_shift};
    if (kl.coarse_shift - 1 >= 6) shifts.push_back(kl.coarse_shift - 1);
    if (kl.coarse_shift + 1 <= std::max(gbits, 6))
        shifts.push_back(kl.coarse_shift + 1);
    std::vector<int> paths = {2};
    if (!comp && grid_smem_bytes(cube->data_is_double, cube->max_block_bytes,
                                 true) <= ws->smem_optin)
        paths.push_back(1);
    int best_shift = 0, best_path = 2;
    float best_ms = 1e30f;
    oskar_B200Options o2 = *opt_in;
    o2.coord_mode = opt.coord_mode;
    o2.classes_per_thread = 0;
    o2.accum_mode = OSKAR_B200_ACCUM_PLAIN;
    o2.compensate_radius = 0;
    for (int sh : shifts)
        for (int path : paths)
        {
            o2.tile_shift = sh;
            o2.staging = path;
            float t_min = 1e30f;
            for (int r = 0; r < kRepeats && !status; ++r)
            {
                status = run_grid(ws, cube, &o2, n, uu, vv, ww, vis, nullptr,
                                  cell_size_rad, w_scale, grid_size, grid,
                                  nullptr, nullptr, st);
                if (status) break;
                const cudaError_t e = cudaStreamSynchronize(st);
                if (e != cudaSuccess) { status = status_from_cuda(e); break; }
                float ms = 0.f;
                if (cudaEventElapsedTime(&ms, ws->events[0], ws->events[4]) ==
                    cudaSuccess)
                    t_min = std::min(t_min, ms);
                else
                    cudaGetLastError();
            }
            if (!status && t_min < best_ms)
            {
                best_ms = t_min;
                best_shift = sh == kl.coarse_shift ? 0 : sh;
                best_path = path;
            }
        }
    ws->stage_timing = saved_timing;
    if (status) return status;

    // (3) Flush policy: the compensation radius.
    int radius = 0;
    if (comp && !cube->data_is_double && n > 0)
    {
        DeviceBuffer d_gu, d_gv, full, plain, sums;
        const size_t floats = 2 * (size_t)grid_size * grid_size;
        B200_TRY(d_gu.ensure(sizeof(int32_t) * n));
        B200_TRY(d_gv.ensure(sizeof(int32_t) * n));
        B200_TRY(full.ensure(sizeof(float) * floats));
        B200_TRY(plain.ensure(sizeof(float) * floats));
        B200_TRY(sums.ensure(2 * sizeof(double)));
        rs = run_place(ws, 0, opt.coord_mode,
                       static_cast<const int*>(cube->d_support.ptr), P,
                       cube->oversample, n, uu, vv, ww, cell_size_rad,
                       w_scale, grid_size, static_cast<int32_t*>(d_gu.ptr),
                       static_cast<int32_t*>(d_gv.ptr), nullptr, nullptr,
                       nullptr, nullptr, static_cast<int32_t*>(d_skip.ptr),
                       st);
        if (rs) return rs;
        std::vector<int32_t> gu(n), gv(n);
        B200_TRY(cudaMemcpyAsync(gu.data(), d_gu.ptr, 4 * n,
                                 cudaMemcpyDeviceToHost, st));
        B200_TRY(cudaMemcpyAsync(gv.data(), d_gv.ptr, 4 * n,
                                 cudaMemcpyDeviceToHost, st));
        B200_TRY(cudaMemcpyAsync(skipped.data(), d_skip.ptr, 4 * n,
                                 cudaMemcpyDeviceToHost, st));
        B200_TRY(cudaStreamSynchronize(st));
        // Chebyshev distance of each kept visibility from the grid centre
        // (the measure the gridding kernel tests a task's radius with).
        std::vector<int> dist;
        dist.reserve(n);
        const int c = grid_size / 2;
        for (size_t i = 0; i < n; ++i)
            if (!skipped[i])
                dist.push_back(std::max(std::abs(gu[i] - c),
                                        std::abs(gv[i] - c)));
        std::sort(dist.begin(), dist.end());
        oskar_B200Options o3 = *opt_in;
        o3.coord_mode = opt.coord_mode;
        o3.classes_per_thread = 0;
        o3.tile_shift = best_shift;
        o3.staging = 2;
        auto grid_into = [&](void* g, int accum, int rad) -> int {
            o3.accum_mode = accum;
            o3.compensate_radius = rad;
            B200_TRY(cudaMemsetAsync(g, 0, sizeof(float) * floats, st));
            return run_grid(ws, cube, &o3, n, uu, vv, ww, vis, nullptr,
                            cell_size_rad, w_scale, grid_size, g, nullptr,
                            nullptr, st);
        };
        status = grid_into(full.ptr, OSKAR_B200_ACCUM_COMPENSATED, 0);
        if (!status) status = grid_into(plain.ptr, OSKAR_B200_ACCUM_PLAIN, 0);
        double d_plain = 0.0;
        if (!status)
            status = grid_distance(static_cast<const float*>(plain.ptr),
                                   static_cast<const float*>(full.ptr), floats,
                                   ws->num_sms, static_cast<double*>(sums.ptr),
                                   st, &d_plain);
        if (status) return status;
        if (!dist.empty() && d_plain > 0.0)
        {
            for (double q : {0.5, 0.75, 0.9})
            {
                const size_t k = std::min(dist.size() - 1,
                                          (size_t)(q * (double)dist.size()));
                const int rad = std::max(1, dist[k]);
                status = grid_into(grid, OSKAR_B200_ACCUM_COMPENSATED, rad);
                double d = 0.0;
                if (!status)
                    status = grid_distance(static_cast<const float*>(grid),
                                           static_cast<const float*>(full.ptr),
                                           floats, ws->num_sms,
                                           static_cast<double*>(sums.ptr), st,
                                           &d);
                if (status) return status;
                if (d <= 0.25 * d_plain)
                {
                    radius = rad;
                    break;
                }
            }
        }
    }
    ws->tuned_tile_shift = best_shift;
    ws->tuned_staging = best_path;
    ws->tuned_comp_radius = radius;
    ws->tuned_launch = 1;
    return OSKAR_B200_OK;
}

}  // namespace b200
