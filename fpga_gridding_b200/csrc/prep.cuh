// Placement of one visibility and the prep launch interface.
#pragma once

#include <climits>

#include "common.cuh"
#include "internal.h"

namespace b200 {

enum { COORD_F64 = 0, COORD_REF_F32 = 1 };

struct PlaceConsts
{
    double grid_scale;    // grid_size * cell_size_rad in FP64
    double w_scale;
    float grid_scale_f;   // grid_size * cell_size_rad rounded as in float C
    float w_scale_f;
    int grid_size;
    int centre;           // grid_size / 2
    int num_planes;
    int oversample;
};

struct Placed
{
    int gu, gv;                 // valid when !skipped
    int gu_report, gv_report;   // saturated to int32 for inspection
    int plane;                  // clamped to the last plane
    int off_u, off_v;
    int conj;                   // -1 when w > 0, else +1
    int skipped;
};

__device__ __forceinline__ int sat_i32(long long x)
{
    return x > INT_MAX ? INT_MAX : (x < INT_MIN ? INT_MIN : (int)x);
}

// oskar_grid_wproj.c:70-101 (FP64) or :168-212 (float, MODE ==
// COORD_REF_F32).  Every rounding step is an explicit IEEE operation so
// the result is bit-identical to the C code on the same inputs:
//   pos = -u * grid_scale, v * grid_scale
//   grid_w = round(sqrt(|w * w_scale|)), clamped to the last plane
//   grid_u = (int)round(pos_u) + grid_size / 2     (same for v)
//   off_u = (int)round((round(pos_u) - pos_u) * oversample)
//   skipped when grid_u +- S or grid_v +- S leaves [0, grid_size).
// round() is half-away-from-zero on both sides.  A coordinate whose rounded
// value is outside the int range (or NaN) is placed at INT_MIN, as x86-64's
// truncating conversion does, and is therefore skipped.
template <typename T, int MODE>
__device__ __forceinline__ Placed place_one(T u, T v, T w,
                                            const PlaceConsts& c,
                                            const int* __restrict__ support)
{
    Placed p;
    long long gu, gv;
    if (MODE == COORD_F64)
    {
        const double du = (double)u, dv = (double)v, dw = (double)w;
        const double pos_u = __dmul_rn(-du, c.grid_scale);
        const double pos_v = __dmul_rn(dv, c.grid_scale);
        p.conj = dw > 0.0 ? -1 : 1;
        const double wr = round(sqrt(fabs(__dmul_rn(dw, c.w_scale))));
        p.plane = wr < (double)c.num_planes ? (int)wr : c.num_planes - 1;
        const double ru = round(pos_u), rv = round(pos_v);
        const bool oku = ru > -2147483649.0 && ru < 2147483648.0;
        const bool okv = rv > -2147483649.0 && rv < 2147483648.0;
        gu = (oku ? (long long)ru : (long long)INT_MIN) + c.centre;
        gv = (okv ? (long long)rv : (long long)INT_MIN) + c.centre;
        p.off_u = (int)round(__dmul_rn(__dsub_rn(ru, pos_u),
                                       (double)c.oversample));
        p.off_v = (int)round(__dmul_rn(__dsub_rn(rv, pos_v),
                                       (double)c.oversample));
    }
    else
    {
        const float fu = (float)u, fv = (float)v, fw = (float)w;
        const float pos_u = __fmul_rn(-fu, c.grid_scale_f);
        const float pos_v = __fmul_rn(fv, c.grid_scale_f);
        p.conj = fw > 0.0f ? -1 : 1;
        const float wr = roundf(sqrtf(fabsf(__fmul_rn(fw, c.w_scale_f))));
        p.plane = wr < (float)c.num_planes ? (int)wr : c.num_planes - 1;
        const float ru = roundf(pos_u), rv = roundf(pos_v);
        const bool oku = ru > -2147483649.0f && ru < 2147483648.0f;
        const bool okv = rv > -2147483649.0f && rv < 2147483648.0f;
        gu = (oku ? (long long)ru : (long long)INT_MIN) + c.centre;
        gv = (okv ? (long long)rv : (long long)INT_MIN) + c.centre;
        p.off_u = (int)roundf(__fmul_rn(__fsub_rn(ru, pos_u),
                                        (float)c.oversample));
        p.off_v = (int)roundf(__fmul_rn(__fsub_rn(rv, pos_v),
                                        (float)c.oversample));
    }
    const int s = support[p.plane];
    p.skipped = (gu + s >= c.grid_size) || (gu - s < 0) ||
                (gv + s >= c.grid_size) || (gv - s < 0);
    p.gu = (int)gu;
    p.gv = (int)gv;
    p.gu_report = sat_i32(gu);
    p.gv_report = sat_i32(gv);
    return p;
}

// Metres to wavelengths as scale_coords (utils/read_vis.c:51-73) does on the
// host: one multiplication in the data's precision (the FP64 scale rounded
// to float for FP32 data).  The scale is exactly 1 when no frequency is
// given, and x * 1 == x.
__device__ __forceinline__ double scale_coord(double x, const JobDesc& jd)
{
    return __dmul_rn(x, jd.coord_scale);
}
__device__ __forceinline__ float scale_coord(float x, const JobDesc& jd)
{
    return __fmul_rn(x, jd.coord_scale_f);
}

// Prep of a batch: launch grid (blocks_per_job, num_jobs), block (x, j)
// walks job j's points.
struct PrepArgs
{
    const JobDesc* jobs;
    int num_jobs;
    int blocks_per_job;
    int max_planes;          // row stride of plane_counts
    int apply_weight;
    KeyLayout key;
    int4* rec;               // [total points], global index
    uint32_t* keys;
    uint32_t* vals;
    unsigned long long* counters;     // CNT_SKIPPED: all jobs
    unsigned long long* job_skipped;  // [num_jobs]
    double* norm_partials;            // [num_jobs][blocks_per_job]
    unsigned long long* plane_counts; // [num_jobs][max_planes]
};

// Blocks per job: about 8 per SM over the whole batch, at least one per job,
// no more than the largest job needs.
int prep_blocks_per_job(size_t max_points, int num_jobs, int num_sms);
cudaError_t launch_prep(const PrepArgs& a, int data_is_double, int coord_mode,
                        cudaStream_t st);
// Per job: norm += sum of its partials; skip count; grid updates.
cudaError_t launch_finalize_prep(const PrepArgs& a, cudaStream_t st);
// Task list: a task starts where (job, coarse tile, plane) changes and every
// task_max positions; task_job[t] is the job of task t.  tile_counts holds
// 2 * task_tiles(n) entries; scan_tmp as exclusive_scan_u32 needs for
// task_tiles(n) values.
size_t task_tiles(size_t n);
cudaError_t launch_tasks(const uint32_t* sorted_keys, size_t n,
                         unsigned long long* counters, int fine_key_bits,
                         int job_shift, int task_max, uint32_t* tile_counts,
                         void* scan_tmp, uint32_t* task_start,
                         uint32_t* task_job, cudaStream_t st, int* launches);
// Bands of a single job's task list: band b holds the tasks of coarse-tile
// row b; band_first[b] (b <= num_bands) is its first task.
cudaError_t launch_band_first(const uint32_t* sorted_keys,
                              const uint32_t* task_start, size_t n,
                              const unsigned long long* counters,
                              const KeyLayout& kl, int num_bands,
                              uint32_t* band_first, int num_sms,
                              cudaStream_t st);
// oskar_grid_wproj_f_diagnostics (diagnostics.cu).  Unclamped w-plane
// indices at or above kDiagMaxPlanes are refused.
constexpr unsigned kDiagMaxPlanes = 1u << 24;
// out[0] = the largest unclamped w-plane index of the points, out[1] = 1
// when any index is not finite or not below kDiagMaxPlanes.
cudaError_t launch_diag_max_plane(const float* ww, size_t n, float w_scale_f,
                                  unsigned long long* out, int num_sms,
                                  cudaStream_t st);
// The per-support, per-plane and per-cell counts and the per-cell support +
// plane sums of the diagnostics gridder, with its float placement.
cudaError_t launch_diag_counts(const float* uu, const float* vv,
                               const float* ww, size_t n,
                               const PlaceConsts& pc, const int* support,
                               unsigned long long* per_support,
                               unsigned long long* per_plane,
                               unsigned long long* per_cell, float* cell_sum,
                               int num_sms, cudaStream_t st);
cudaError_t launch_place(int data_is_double, int coord_mode, const void* uu,
                         const void* vv, const void* ww, size_t n,
                         const PlaceConsts& pc, const int* support,
                         int32_t* gu, int32_t* gv, int32_t* plane,
                         int32_t* off_u, int32_t* off_v, int32_t* conj,
                         int32_t* skipped, int num_sms, cudaStream_t st);

}  // namespace b200
