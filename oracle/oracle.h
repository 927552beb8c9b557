/*
 * oracle.h -- CPU restatement of the reference W-projection gridder.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this code.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg use it, and only as the checker / the timed CPU baseline.
 *
 * Parity of this restatement is pinned two ways:
 *   - bit-exact against the reference's own oskar_grid_wproj_d / _f compiled
 *     from its sources into oracle/_ref/ (see oracle/Makefile);
 *   - against golden fixtures generated from that compiled reference and
 *     committed under tests/golden/ (tests/golden/make_golden.py).
 *
 * Reference: oskar_grid_wproj.c (OxfordSKA/FPGA_Gridding).
 */
#ifndef FPGA_GRIDDING_ORACLE_H_
#define FPGA_GRIDDING_ORACLE_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Restates oskar_grid_wproj_d, oskar_grid_wproj.c:39-126. Same arguments,
 * same in/out semantics (num_skipped reset, norm and grid accumulate,
 * weight ignored). */
void orc_grid_wproj_d(size_t num_w_planes, const int* support, int oversample,
        int conv_size_half, const double* conv_func, size_t num_points,
        const double* uu, const double* vv, const double* ww,
        const double* vis, const double* weight, double cell_size_rad,
        double w_scale, int grid_size, size_t* num_skipped, double* norm,
        double* grid);

/* Restates oskar_grid_wproj_f, oskar_grid_wproj.c:128-243, over all
 * num_points.  The shipped reference loops a fixed 10000 points and prints
 * progress (oskar_grid_wproj.c:154-157); those two debugging lines are the
 * only deviation.  All coordinate arithmetic is float, as in the reference. */
/* FP64 gridding with each visibility scaled by its weight and the norm
 * adding tap sum x weight: the weighting of the reference's tiled CUDA
 * gridder (oskar_grid_wproj_gpu.cu.old:718-724, :799), on the arithmetic
 * of oskar_grid_wproj_d.  Unit weights give orc_grid_wproj_d exactly. */
void orc_grid_wproj_weighted_d(size_t num_w_planes, const int* support,
        int oversample, int conv_size_half, const double* conv_func,
        size_t num_points, const double* uu, const double* vv,
        const double* ww, const double* vis, const double* weight,
        double cell_size_rad, double w_scale, int grid_size,
        size_t* num_skipped, double* norm, double* grid);

void orc_grid_wproj_f(size_t num_w_planes, const int* support, int oversample,
        int conv_size_half, const float* conv_func, size_t num_points,
        const float* uu, const float* vv, const float* ww,
        const float* vis, const float* weight, float cell_size_rad,
        float w_scale, int grid_size, size_t* num_skipped, double* norm,
        float* grid);

/* Restates oskar_grid_wproj_f_diagnostics, oskar_grid_wproj.c:245-370:
 * oskar_grid_wproj_f's float gridding of all num_points plus per-support,
 * per-plane (unclamped) and per-cell hit counts and the per-cell sum of
 * support + plane of every tap (in avg_wsupport_per_grid, as the reference
 * writes it; avg_wplane_per_grid is not touched). */
void orc_grid_wproj_f_diagnostics(size_t num_w_planes, const int* support,
        int oversample, int conv_size_half, const float* conv_func,
        size_t num_points, const float* uu, const float* vv,
        const float* ww, const float* vis, const float* weight,
        float cell_size_rad, float w_scale, int grid_size,
        size_t* num_skipped, double* norm, float* grid,
        long long* num_vis_per_wsupport, long long* num_vis_per_wplane,
        long long* num_vis_per_grid, float* avg_wsupport_per_grid,
        float* avg_wplane_per_grid);

/* Per-visibility placement tuple, FP64 coordinate arithmetic of
 * oskar_grid_wproj.c:70-101.  plane is the clamped w-plane actually used
 * (min(grid_w, num_w_planes-1)); raw_plane is grid_w before clamping
 * (saturated to INT32_MAX).  skipped[i] = 1 when the footprint leaves the grid. */
void orc_vis_place_d(size_t num_w_planes, const int* support, int oversample,
        size_t num_points, const double* uu, const double* vv,
        const double* ww, double cell_size_rad, double w_scale,
        int grid_size, int32_t* gu, int32_t* gv, int32_t* plane,
        int32_t* raw_plane, int32_t* off_u, int32_t* off_v, int8_t* conj,
        uint8_t* skipped);

/* Same with the float coordinate arithmetic of oskar_grid_wproj.c:168-212. */
void orc_vis_place_f(size_t num_w_planes, const int* support, int oversample,
        size_t num_points, const float* uu, const float* vv, const float* ww,
        float cell_size_rad, float w_scale, int grid_size, int32_t* gu,
        int32_t* gv, int32_t* plane, int32_t* raw_plane, int32_t* off_u,
        int32_t* off_v, int8_t* conj, uint8_t* skipped);

/* Row-band multi-threaded restatement of oskar_grid_wproj_d / _f.  Each
 * thread owns a band of grid rows and walks every visibility in input order,
 * applying only the taps that land in its rows, so every grid cell receives
 * exactly the same sequence of additions as the serial loop: results are
 * bit-identical to orc_grid_wproj_d / _f for any thread count. */
void orc_grid_wproj_d_banded(size_t num_w_planes, const int* support,
        int oversample, int conv_size_half, const double* conv_func,
        size_t num_points, const double* uu, const double* vv,
        const double* ww, const double* vis, const double* weight,
        double cell_size_rad, double w_scale, int grid_size,
        size_t* num_skipped, double* norm, double* grid, int num_threads);
void orc_grid_wproj_f_banded(size_t num_w_planes, const int* support,
        int oversample, int conv_size_half, const float* conv_func,
        size_t num_points, const float* uu, const float* vv,
        const float* ww, const float* vis, const float* weight,
        float cell_size_rad, float w_scale, int grid_size,
        size_t* num_skipped, double* norm, float* grid, int num_threads);

/* Uniform-weighting helpers, restating utils/oskar_grid_weights.c:38-172. */
void orc_grid_weights_write_d(size_t num_points, const double* uu,
        const double* vv, const double* weight, double cell_size_rad,
        int grid_size, size_t* num_skipped, double* grid);
void orc_grid_weights_read_d(size_t num_points, const double* uu,
        const double* vv, const double* weight_in, double* weight_out,
        double cell_size_rad, int grid_size, size_t* num_skipped,
        const double* grid);
void orc_grid_weights_write_f(size_t num_points, const float* uu,
        const float* vv, const float* weight, float cell_size_rad,
        int grid_size, size_t* num_skipped, float* grid);
void orc_grid_weights_read_f(size_t num_points, const float* uu,
        const float* vv, const float* weight_in, float* weight_out,
        float cell_size_rad, int grid_size, size_t* num_skipped,
        const float* grid);

/* Degridding: the adjoint of oskar_grid_wproj_d.  The reference has no
 * degridder (Defines.h:48 only reserves the switch), so this is defined
 * here: with the gridder's placement and skip test
 * (oskar_grid_wproj.c:70-101) and its tap kernel value
 * Kt = conj?(K[plane][|off_v + j*os|][|off_u + k*os|]) (conjugated for
 * w > 0, :110-122), each kept visibility becomes
 *   vis[i] = sum over the (2S+1)^2 taps of grid[(gv+j)*G + gu+k] * conj(Kt)
 * summed in FP64, rows j outer, columns k inner.  Skipped visibilities keep
 * their vis_out value; num_skipped counts them. */
void orc_degrid_wproj_d(size_t num_w_planes, const int* support,
        int oversample, int conv_size_half, const double* conv_func,
        size_t num_points, const double* uu, const double* vv,
        const double* ww, double cell_size_rad, double w_scale,
        int grid_size, const double* grid, size_t* num_skipped,
        double* vis_out);

/* Coordinates in metres to wavelengths, restating utils/read_vis.c:51-73:
 * every coordinate times freq_hz / c, in the data's precision (the double
 * scale is rounded to float for FP32 data).  is_double selects the type. */
void orc_scale_coords(double freq_hz, int is_double, size_t num_coords,
        void* uu, void* vv, void* ww);

/* ------------------------------------------------------------------------
 * CPU baseline harness.  Runs a gridding function (the compiled reference's
 * or this restatement's, passed as a pointer) on num_threads threads, each
 * on its own contiguous slice of the visibilities with a private grid, and
 * returns the longest per-thread wall time of the gridding calls alone.
 * Private grids are allocated and zeroed before timing starts.
 *
 * chunk_points > 0 makes each thread call fn on consecutive sub-slices of
 * exactly chunk_points points; a final short sub-slice is padded with points
 * placed far outside the grid (which the gridder skips and counts).  This is
 * how the shipped reference oskar_grid_wproj_f, which always processes a
 * fixed 10000 points, is driven over a whole workload.  While fn runs,
 * stdout is redirected to /dev/null (the shipped _f prints progress).
 *
 * On return, grid_out (if not NULL) holds the sum of the private grids,
 * *norm_out the sum of the norms and *skipped_out the skip count net of
 * padding. Returns seconds, or a negative value on allocation failure.
 * ------------------------------------------------------------------------ */
typedef void (*orc_grid_fn_d)(size_t, const int*, int, int, const double*,
        size_t, const double*, const double*, const double*, const double*,
        const double*, double, double, int, size_t*, double*, double*);
typedef void (*orc_grid_fn_f)(size_t, const int*, int, int, const float*,
        size_t, const float*, const float*, const float*, const float*,
        const float*, float, float, int, size_t*, double*, float*);

typedef void (*orc_wwrite_fn_f)(size_t, const float*, const float*,
        const float*, float, int, size_t*, float*);
typedef void (*orc_wread_fn_f)(size_t, const float*, const float*,
        const float*, float*, float, int, size_t*, const float*);

/* Uniform-weighting CPU baseline (FP32): num_threads threads run wfn on
 * contiguous slices into private grids, sum the private grids into
 * grid_out in parallel (in thread order), then run rfn on the slices
 * against grid_out.  Returns the seconds of the whole pass (or -1). */
double orc_time_weights_parallel_f(orc_wwrite_fn_f wfn, orc_wread_fn_f rfn,
        int num_threads, size_t num_points, const float* uu, const float* vv,
        const float* w_in, float cell_size_rad, int grid_size,
        float* grid_out, float* w_out, size_t* skipped_w, size_t* skipped_r);

double orc_time_parallel_d(orc_grid_fn_d fn, int num_threads,
        size_t chunk_points, size_t num_w_planes, const int* support,
        int oversample, int conv_size_half, const double* conv_func,
        size_t num_points, const double* uu, const double* vv,
        const double* ww, const double* vis, const double* weight,
        double cell_size_rad, double w_scale, int grid_size,
        size_t* skipped_out, double* norm_out, double* grid_out);
double orc_time_parallel_f(orc_grid_fn_f fn, int num_threads,
        size_t chunk_points, size_t num_w_planes, const int* support,
        int oversample, int conv_size_half, const float* conv_func,
        size_t num_points, const float* uu, const float* vv,
        const float* ww, const float* vis, const float* weight,
        float cell_size_rad, float w_scale, int grid_size,
        size_t* skipped_out, double* norm_out, float* grid_out);

/* Number of grid updates (kernel taps) the reference applies:
 * sum over non-skipped points of (2*support+1)^2, FP64 placement. */
uint64_t orc_count_taps_d(size_t num_w_planes, const int* support,
        int oversample, size_t num_points, const double* uu,
        const double* vv, const double* ww, double cell_size_rad,
        double w_scale, int grid_size);

#ifdef __cplusplus
}
#endif

#endif /* FPGA_GRIDDING_ORACLE_H_ */
