// Hit counts of oskar_grid_wproj_f_diagnostics (oskar_grid_wproj.c:245-370)
// on the GPU.  The gridding itself (grid, norm, skip count) runs through the
// ordinary pipeline with the reference's float coordinate arithmetic; these
// kernels add what the diagnostics variant counts besides:
//   per point (skipped or not): num_vis_per_wsupport[w_support] += 1 and
//     num_vis_per_wplane[grid_w] += 1, grid_w = round(sqrt(|w * w_scale|))
//     before it is clamped to the last plane (:317-318);
//   per tap of a kept point, at its grid cell: num_vis_per_grid += 1 and
//     avg_wsupport_per_grid += w_support, then += grid_w (:358-360; both
//     sums go to the same array, as in the reference).
// The per-cell counts are integer atomics; the per-cell sums are float
// atomics of small integers, exact (and so equal to the reference's
// sequential sum) while every partial sum stays below 2^24.
#include "common.cuh"
#include "internal.h"
#include "prep.cuh"

namespace b200 {
namespace {

// grid_w in the reference's float arithmetic (oskar_grid_wproj.c:286), the
// same operations as place_one's plane before its clamp.
__device__ __forceinline__ float raw_plane_f(float w, float w_scale_f)
{
    return roundf(sqrtf(fabsf(__fmul_rn(w, w_scale_f))));
}

// out[0] = max grid_w over the points; out[1] = 1 if any grid_w is not a
// finite value below kDiagMaxPlanes.
__global__ void diag_max_plane_kernel(const float* __restrict__ ww, size_t n,
                                      float w_scale_f,
                                      unsigned long long* __restrict__ out)
{
    unsigned long long mx = 0, bad = 0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
    {
        const float r = raw_plane_f(ww[i], w_scale_f);
        if (r < (float)kDiagMaxPlanes)
            mx = max(mx, (unsigned long long)r);
        else
            bad = 1;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
    {
        mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        bad |= __shfl_xor_sync(0xffffffffu, bad, o);
    }
    if ((threadIdx.x & 31) == 0)
    {
        if (mx) atomicMax(&out[0], mx);
        if (bad) atomicOr(&out[1], 1ull);
    }
}

// One warp per point: lane 0 counts the point's support and plane, the
// lanes walk its footprint's taps row-major, 32 at a time.
__global__ void diag_counts_kernel(const float* __restrict__ uu,
                                   const float* __restrict__ vv,
                                   const float* __restrict__ ww, size_t n,
                                   PlaceConsts pc,
                                   const int* __restrict__ support,
                                   unsigned long long* __restrict__ per_support,
                                   unsigned long long* __restrict__ per_plane,
                                   unsigned long long* __restrict__ per_cell,
                                   float* __restrict__ cell_sum)
{
    const int lane = threadIdx.x & 31;
    const size_t warps = (size_t)gridDim.x * (blockDim.x >> 5);
    for (size_t i = (size_t)blockIdx.x * (blockDim.x >> 5) +
                    (threadIdx.x >> 5);
         i < n; i += warps)
    {
        const Placed p = place_one<float, COORD_REF_F32>(uu[i], vv[i], ww[i],
                                                         pc, support);
        const int s = support[p.plane];
        const unsigned long long raw =
            (unsigned long long)raw_plane_f(ww[i], pc.w_scale_f);
        if (lane == 0)
        {
            atomicAdd(&per_support[s], 1ull);
            atomicAdd(&per_plane[raw], 1ull);
        }
        if (p.skipped) continue;
        const int w = 2 * s + 1, taps = w * w;
        const float fs = (float)s, fr = (float)raw;
        const size_t G = (size_t)pc.grid_size;
        const size_t corner = (size_t)(p.gv - s) * G + (size_t)(p.gu - s);
        for (int t = lane; t < taps; t += 32)
        {
            const int j = t / w, k = t - j * w;
            const size_t cell = corner + (size_t)j * G + (size_t)k;
            atomicAdd(&per_cell[cell], 1ull);
            atomicAdd(&cell_sum[cell], fs);
            atomicAdd(&cell_sum[cell], fr);
        }
    }
}

}  // namespace

cudaError_t launch_diag_max_plane(const float* ww, size_t n, float w_scale_f,
                                  unsigned long long* out, int num_sms,
                                  cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(out, 0, 2 * sizeof(unsigned long long),
                                    st);
    if (e != cudaSuccess || n == 0) return e;
    const size_t want = (n + 255) / 256, cap = (size_t)num_sms * 8;
    diag_max_plane_kernel<<<(unsigned)(want < cap ? want : cap), 256, 0,
                            st>>>(ww, n, w_scale_f, out);
    return cudaGetLastError();
}

cudaError_t launch_diag_counts(const float* uu, const float* vv,
                               const float* ww, size_t n,
                               const PlaceConsts& pc, const int* support,
                               unsigned long long* per_support,
                               unsigned long long* per_plane,
                               unsigned long long* per_cell, float* cell_sum,
                               int num_sms, cudaStream_t st)
{
    if (n == 0) return cudaSuccess;
    const size_t want = (n + 7) / 8;
    const size_t cap = (size_t)num_sms * 8;
    const unsigned blocks = (unsigned)(want < cap ? want : cap);
    diag_counts_kernel<<<blocks, 256, 0, st>>>(uu, vv, ww, n, pc, support,
                                                per_support, per_plane,
                                                per_cell, cell_sum);
    return cudaGetLastError();
}

}  // namespace b200
