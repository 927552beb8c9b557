/*
 * oskar_grid_wproj_b200.h -- B200 (sm_100a) W-projection gridder, C ABI.
 *
 * Library: fpga_gridding_b200/libgridder_b200.so
 *
 * 1. Drop-in entry points with exactly the reference's signatures
 *    (oskar_grid_wproj.h:69-86 and :114-131 of OxfordSKA/FPGA_Gridding).
 *    All pointers are host memory, the call is synchronous, num_skipped is
 *    reset, norm and grid accumulate, weight is ignored (as the reference
 *    hard-codes weight 1.0, oskar_grid_wproj.c:80-81).  Like the reference
 *    they return void; a failure leaves grid/norm untouched and is readable
 *    with oskar_grid_wproj_b200_last_error() from the same thread.  (Rows of
 *    grid are copied back while later rows still grid; after a failure
 *    they are restored from the device copy of the caller's grid, so only
 *    a fault that loses the CUDA context can leave some of them updated.)
 *
 * 2. An extended, asynchronous API on device-resident buffers with explicit
 *    stream, workspace, resident kernel cubes and precision options.  Every
 *    extended function returns an oskar_B200Status.
 *
 * There is no CPU fallback: without a usable CUDA device every entry point
 * fails with OSKAR_B200_ERR_NO_DEVICE.
 */
#ifndef OSKAR_GRID_WPROJ_B200_H_
#define OSKAR_GRID_WPROJ_B200_H_

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define OSKAR_B200_EXPORT __attribute__((visibility("default")))
#else
#define OSKAR_B200_EXPORT
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------------- */
/* Status codes                                                           */
/* ---------------------------------------------------------------------- */
typedef enum
{
    OSKAR_B200_OK = 0,
    OSKAR_B200_ERR_INVALID_ARGUMENT = 1, /* sizes, null pointers, cube extent */
    OSKAR_B200_ERR_NO_DEVICE = 2,        /* no usable CUDA device */
    OSKAR_B200_ERR_OUT_OF_MEMORY = 3,    /* device or pinned host allocation */
    OSKAR_B200_ERR_CUDA = 4,             /* any other CUDA runtime error */
    OSKAR_B200_ERR_UNSUPPORTED = 5,      /* option combination not built */
    OSKAR_B200_ERR_DEVICE_CHECK = 6,     /* a kernel's own bounds check fired */
    OSKAR_B200_ERR_TIMEOUT = 7,          /* a bounded device-side wait expired */
    OSKAR_B200_ERR_OVER_BUDGET = 8       /* job exceeds the HBM budget */
} oskar_B200Status;

/* ---------------------------------------------------------------------- */
/* 1. Drop-in replacements                                                */
/* ---------------------------------------------------------------------- */

/* Replaces oskar_grid_wproj_d (oskar_grid_wproj.h:69-86).  FP64 data,
 * FP64 grid, FP64 coordinates; grid within 1e-12 relative RMS of the
 * reference, num_skipped and every placement bit-exact. */
OSKAR_B200_EXPORT
void oskar_grid_wproj_d(
        const size_t num_w_planes,
        const int* support,
        const int oversample,
        const int conv_size_half,
        const double* conv_func,
        const size_t num_points,
        const double* uu,
        const double* vv,
        const double* ww,
        const double* vis,
        const double* weight,
        const double cell_size_rad,
        const double w_scale,
        const int grid_size,
        size_t* num_skipped,
        double* norm,
        double* grid);

/* Replaces oskar_grid_wproj_f (oskar_grid_wproj.h:114-131).  FP32 data,
 * kernel and grid; grid coordinates, w-plane and oversample offsets are
 * computed in FP64 from the float inputs (so placements equal the FP64
 * reference's on the same inputs); norm is FP64.  The reference's float
 * coordinate arithmetic is available through the extended API
 * (OSKAR_B200_COORDS_REFERENCE_F32). */
OSKAR_B200_EXPORT
void oskar_grid_wproj_f(
        const size_t num_w_planes,
        const int* support,
        const int oversample,
        const int conv_size_half,
        const float* conv_func,
        const size_t num_points,
        const float* uu,
        const float* vv,
        const float* ww,
        const float* vis,
        const float* weight,
        const float cell_size_rad,
        const float w_scale,
        const int grid_size,
        size_t* num_skipped,
        double* norm,
        float* grid);

/* Replaces oskar_grid_wproj_f_diagnostics (oskar_grid_wproj.c:245-370;
 * defined there, declared in no reference header): oskar_grid_wproj_f over
 * all num_points with the reference's float coordinate arithmetic, plus hit
 * counts, all accumulating into the caller's arrays:
 *   num_vis_per_wsupport[w_support] += 1 and num_vis_per_wplane[grid_w] += 1
 *     for every point, skipped or not, where grid_w =
 *     round(sqrt(|w * w_scale|)) before it is clamped to the last plane and
 *     w_support is the support of the plane actually used;
 *   for every tap of a kept point, at its grid cell (grid_size^2 arrays,
 *     row-major in v): num_vis_per_grid += 1, avg_wsupport_per_grid +=
 *     w_support + grid_w (both into the same array, as the reference
 *     does); avg_wplane_per_grid is never written.
 * num_vis_per_wsupport must hold max(support) + 1 entries and
 * num_vis_per_wplane the largest grid_w of the points + 1, as the
 * reference's indexing requires; a point whose grid_w is not finite or not
 * below 2^24 fails the call with OSKAR_B200_ERR_INVALID_ARGUMENT.  Counts
 * are exact; the per-cell sums are exact while they stay below 2^24 (the
 * reference's own float sums round beyond that).  Synchronous; on failure
 * the outputs are untouched and the status is available from
 * oskar_grid_wproj_b200_last_error(). */
OSKAR_B200_EXPORT
void oskar_grid_wproj_f_diagnostics(
        const size_t num_w_planes,
        const int* support,
        const int oversample,
        const int conv_size_half,
        const float* conv_func,
        const size_t num_points,
        const float* uu,
        const float* vv,
        const float* ww,
        const float* vis,
        const float* weight,
        const float cell_size_rad,
        const float w_scale,
        const int grid_size,
        size_t* num_skipped,
        double* norm,
        float* grid,
        long long int* num_vis_per_wsupport,
        long long int* num_vis_per_wplane,
        long long int* num_vis_per_grid,
        float* avg_wsupport_per_grid,
        float* avg_wplane_per_grid);

/* Replace oskar_grid_weights_{write,read}_{d,f} (utils/oskar_grid_weights.h:
 * 60-65, 84-89, 107-112, 131-136): the "uniform" weighting histogram and its
 * density lookup, computed on the GPU on the caller's host arrays.  Same
 * arguments and results as the reference, bit for bit:
 *   write: grid (real, grid_size^2, row-major in v) += weight of every point
 *     at cell (round(-u * grid_size * cell) + grid_size / 2,
 *     round(v * grid_size * cell) + grid_size / 2); each cell's weights are
 *     added in point order (a stable sort by cell on the device, then one
 *     sequential sum per cell); num_skipped counts points outside the grid.
 *   read: weight_out[i] = weight_in[i] / grid[cell], or 0 where the cell
 *     is empty; skipped points keep their weight_out value.
 * The _f variants do the coordinate arithmetic in float, as the reference's.
 * Synchronous; on failure the outputs are untouched and the status is
 * available from oskar_grid_wproj_b200_last_error(). */
OSKAR_B200_EXPORT
void oskar_grid_weights_write_d(const size_t num_points, const double* uu,
        const double* vv, const double* weight, const double cell_size_rad,
        const int grid_size, size_t* num_skipped, double* grid);
OSKAR_B200_EXPORT
void oskar_grid_weights_read_d(const size_t num_points, const double* uu,
        const double* vv, const double* weight_in, double* weight_out,
        const double cell_size_rad, const int grid_size, size_t* num_skipped,
        const double* grid);
OSKAR_B200_EXPORT
void oskar_grid_weights_write_f(const size_t num_points, const float* uu,
        const float* vv, const float* weight, const float cell_size_rad,
        const int grid_size, size_t* num_skipped, float* grid);
OSKAR_B200_EXPORT
void oskar_grid_weights_read_f(const size_t num_points, const float* uu,
        const float* vv, const float* weight_in, float* weight_out,
        const float cell_size_rad, const int grid_size, size_t* num_skipped,
        const float* grid);

/* Status of the calling thread's most recent drop-in call. */
OSKAR_B200_EXPORT int oskar_grid_wproj_b200_last_error(void);

/* Static description of a status code. */
OSKAR_B200_EXPORT const char* oskar_grid_wproj_b200_error_string(int status);

/* Frees the calling thread's cached device buffers and stream (the drop-ins
 * keep them between calls to avoid re-allocation). */
OSKAR_B200_EXPORT void oskar_grid_wproj_b200_release_thread_cache(void);

/* ---------------------------------------------------------------------- */
/* 2. Extended API                                                        */
/* ---------------------------------------------------------------------- */

/* Coordinate arithmetic for (grid_u, grid_v, w-plane, offsets). */
enum
{
    OSKAR_B200_COORDS_F64 = 0,            /* oskar_grid_wproj.c:70-93, FP64 */
    OSKAR_B200_COORDS_REFERENCE_F32 = 1   /* oskar_grid_wproj.c:168-204, float */
};

/* Storage type of the resident W-kernel cube. */
enum
{
    OSKAR_B200_KERNEL_NATIVE = 0,  /* same as the data: FP32 or FP64 */
    OSKAR_B200_KERNEL_F16 = 1,     /* FP16 with a per-plane scale */
    OSKAR_B200_KERNEL_BF16 = 2     /* BF16 with a per-plane scale */
};

/* Grid accumulation for FP32 data.  COMPENSATED: every grid atomic returns
 * the old value, the exact rounding error of the addition (TwoSum) goes to
 * an FP32 error grid in the workspace (grid_size^2 complex), and the error
 * grid is added into the grid at the end of the call. */
enum
{
    OSKAR_B200_ACCUM_PLAIN = 0,        /* FP32 register sums, FP32 atomics */
    OSKAR_B200_ACCUM_COMPENSATED = 1   /* plus the compensated grid atomics */
};

typedef struct oskar_B200Options
{
    int coord_mode;      /* OSKAR_B200_COORDS_* */
    int kernel_type;     /* OSKAR_B200_KERNEL_* */
    int accum_mode;      /* OSKAR_B200_ACCUM_* */
    int apply_weight;    /* 0: ignore weight (reference); 1: vis and norm x weight */
    int classes_per_thread; /* 0: autotuned table; 1-6 forces it */
    int staging;         /* 0: auto (the workspace's tuned choice, else L1);
                          * 1: TMA bulk copy to shared; 2: L1 reads */
    int compensate_radius; /* ACCUM_COMPENSATED: compensate only work whose
                            * footprint centre lies within this many cells of
                            * the grid centre (the heavily hit cells);
                            * 0: everywhere; -1: the workspace's tuned
                            * radius (everywhere until tuned) */
    int tile_shift;      /* log2 of the coarse grid tile side in cells that
                          * orders the work (6-15); 0: the workspace's
                          * tuned value, else grid_size / 16 (at least 64) */
    double frequency_hz; /* > 0: uu, vv, ww are in metres; they are scaled to
                          * wavelengths by frequency_hz / c in the data's
                          * precision before placement, exactly as
                          * scale_coords (utils/read_vis.c:51-73) does on the
                          * host; 0: they are in wavelengths already */
    int reserved[6];
} oskar_B200Options;

/* Fills the defaults (FP64 coordinates, native kernels, plain accumulation,
 * weight ignored, autotuned launch shape). */
OSKAR_B200_EXPORT void oskar_b200_options_init(oskar_B200Options* opt);

/* Opaque workspace: a device, a set of grow-only device buffers and a
 * default stream.  One workspace must not be used by two calls that can
 * overlap in time; give each concurrent stream its own. */
typedef struct oskar_B200Workspace oskar_B200Workspace;

OSKAR_B200_EXPORT int oskar_b200_workspace_create(int device,
        oskar_B200Workspace** ws);
OSKAR_B200_EXPORT int oskar_b200_workspace_free(oskar_B200Workspace* ws);
/* Bytes of device memory currently held by the workspace. */
OSKAR_B200_EXPORT size_t oskar_b200_workspace_bytes(
        const oskar_B200Workspace* ws);

/* Opaque resident kernel cube: the W-kernels re-laid for the gridding
 * kernel (per-plane, phase-major quadrant slabs in the chosen storage
 * type) and the per-(plane, offset) norm table.  Build once, grid many. */
typedef struct oskar_B200Cube oskar_B200Cube;

/* conv_func: [num_w_planes][conv_size_half][conv_size_half][2] in the
 * reference layout, FP32 (is_double = 0) or FP64 (is_double = 1), on the
 * host (conv_func_on_device = 0) or device.  support[] is host memory.
 * data_is_double selects the gridding precision the cube serves. */
OSKAR_B200_EXPORT int oskar_b200_cube_create(oskar_B200Workspace* ws,
        size_t num_w_planes, const int* support, int oversample,
        int conv_size_half, const void* conv_func, int conv_func_is_double,
        int conv_func_on_device, int data_is_double, int kernel_type,
        void* stream, oskar_B200Cube** cube);
/* The same from the separate real and imaginary cubes
 * ([num_w_planes][conv_size_half][conv_size_half] each) that read_kernel
 * returns for the *_KERNELS_REAL / _IMAG FITS files (utils/read_kernel.c:
 * 36-118, main.cpp:182-189): the interleave of main.cpp:197-201 happens in
 * the re-layout kernel instead of on the host. */
OSKAR_B200_EXPORT int oskar_b200_cube_create_planar(oskar_B200Workspace* ws,
        size_t num_w_planes, const int* support, int oversample,
        int conv_size_half, const void* conv_re, const void* conv_im,
        int conv_is_double, int conv_on_device, int data_is_double,
        int kernel_type, void* stream, oskar_B200Cube** cube);
OSKAR_B200_EXPORT int oskar_b200_cube_free(oskar_B200Cube* cube);
OSKAR_B200_EXPORT size_t oskar_b200_cube_bytes(const oskar_B200Cube* cube);

/* Grid num_points visibilities with a resident cube, asynchronously on
 * `stream` (NULL: the workspace's stream).  uu, vv, ww, vis (interleaved),
 * weight and grid are DEVICE pointers of the cube's data precision (float
 * or double).  d_num_skipped (device, uint64) is overwritten with this
 * call's skip count; d_norm (device, double) is incremented.  Either may be
 * NULL.  The grid accumulates. */
OSKAR_B200_EXPORT int oskar_b200_grid(oskar_B200Workspace* ws,
        const oskar_B200Cube* cube, const oskar_B200Options* opt,
        size_t num_points, const void* uu, const void* vv, const void* ww,
        const void* vis, const void* weight, double cell_size_rad,
        double w_scale, int grid_size, void* grid,
        unsigned long long* d_num_skipped, double* d_norm, void* stream);

/* One job of a batch: the arguments of oskar_b200_grid. */
typedef struct oskar_B200Job
{
    const oskar_B200Cube* cube;
    size_t num_points;
    const void* uu;
    const void* vv;
    const void* ww;
    const void* vis;
    const void* weight;
    double cell_size_rad;
    double w_scale;
    int grid_size;
    void* grid;
    unsigned long long* d_num_skipped;
    double* d_norm;
    double frequency_hz;   /* as oskar_B200Options::frequency_hz, per job */
} oskar_B200Job;

/* Grids many independent jobs (channels, snapshots) with uneven sizes and
 * their own cubes and grids in one pipeline: one sort over all
 * visibilities and one persistent gridding launch that takes work from a
 * device queue spanning every job.  All cubes must share the data precision
 * and storage type.  Each job's result equals oskar_b200_grid on that job
 * alone (up to floating-point summation order).  The call only enqueues
 * device work on `stream`, so it can be captured into a CUDA graph once its
 * buffers have been sized by an earlier call with the same jobs. */
OSKAR_B200_EXPORT int oskar_b200_grid_batch(oskar_B200Workspace* ws,
        const oskar_B200Options* opt, int num_jobs, const oskar_B200Job* jobs,
        void* stream);

/* Degridding: the adjoint of oskar_b200_grid (no counterpart in the
 * reference, whose Defines.h:48 only reserves a DEGRIDDING switch).  With
 * the gridder's placement, skip test and tap kernel value
 * Kt = conj?(K[plane][|off_v + j*os|][|off_u + k*os|]) (conjugated for
 * w > 0), each kept visibility gets
 *   vis[i] = sum over its (2S+1)^2 taps of grid[(gv+j)*G + gu+k] * conj(Kt)
 * (times weight[i] with apply_weight), so that for any v and g
 * <grid(v), g> = <v, degrid(g)>.  Device pointers; `grid` is read, `vis`
 * (interleaved complex) written for kept visibilities, skipped ones keep
 * their value and are counted in *d_num_skipped.  Options as
 * oskar_b200_grid (plain accumulation only).  Asynchronous on `stream`. */
OSKAR_B200_EXPORT int oskar_b200_degrid(oskar_B200Workspace* ws,
        const oskar_B200Cube* cube, const oskar_B200Options* opt,
        size_t num_points, const void* uu, const void* vv, const void* ww,
        const void* weight, double cell_size_rad, double w_scale,
        int grid_size, const void* grid, void* vis,
        unsigned long long* d_num_skipped, void* stream);

/* Degridding of host arrays (no counterpart in the reference): the same
 * result as oskar_b200_degrid, with uu, vv, ww, weight (read only with
 * apply_weight), grid and vis in host memory (float arrays for an FP32
 * cube, double for FP64) and the call synchronous.  The grid is uploaded
 * first; the visibilities then cross PCIe in chunks of about 5 M that are
 * degridded as they land, their predictions copied back while later
 * chunks still upload.  Skipped visibilities keep their value in `vis`;
 * *num_skipped receives their count.  On failure `vis` may be partly
 * written.  Pinned host memory makes the copies several times faster. */
OSKAR_B200_EXPORT int oskar_b200_degrid_host(oskar_B200Workspace* ws,
        const oskar_B200Cube* cube, const oskar_B200Options* opt,
        size_t num_points, const void* uu, const void* vv, const void* ww,
        const void* weight, double cell_size_rad, double w_scale,
        int grid_size, const void* grid, void* vis, size_t* num_skipped);

/* Per-visibility placement exactly as the gridder computes it (device
 * pointers, int32 outputs, any may be NULL): grid cell, clamped w-plane,
 * oversample offsets, conjugation sign (+1/-1) and skip flag (0/1). */
OSKAR_B200_EXPORT int oskar_b200_place(oskar_B200Workspace* ws,
        int data_is_double, int coord_mode, size_t num_w_planes,
        const int* support, int oversample, size_t num_points,
        const void* uu, const void* vv, const void* ww,
        double cell_size_rad, double w_scale, int grid_size,
        int32_t* gu, int32_t* gv, int32_t* plane, int32_t* off_u,
        int32_t* off_v, int32_t* conj, int32_t* skipped, void* stream);

/* Uniform weighting on device arrays (FP64 when data_is_double, else FP32
 * with the reference's float coordinate arithmetic), asynchronous on
 * `stream`.  *d_num_skipped (device, may be NULL) is reset, then counts the
 * points outside the grid.  frequency_hz > 0: uu, vv are in metres and are
 * scaled as scale_coords does first (see oskar_B200Options).
 * write: grid (device, grid_size^2 reals) accumulates the weights.
 *   ordered = 1 adds each cell's weights in point order, bit-identical to
 *   oskar_grid_weights_write_{d,f} (stable sort by cell, then one
 *   sequential sum per cell); ordered = 0 issues one atomic add per point
 *   (faster; cell sums depend on the order the atomics land in, exact when
 *   every partial sum is, e.g. unit weights).
 * read: weight_out[i] = weight_in[i] / grid[cell] (0 for an empty cell);
 *   skipped points keep their weight_out value. */
OSKAR_B200_EXPORT int oskar_b200_weights_write(oskar_B200Workspace* ws,
        int data_is_double, int ordered, size_t num_points, const void* uu,
        const void* vv, const void* weight, double cell_size_rad,
        int grid_size, void* grid, unsigned long long* d_num_skipped,
        double frequency_hz, void* stream);
OSKAR_B200_EXPORT int oskar_b200_weights_read(oskar_B200Workspace* ws,
        int data_is_double, size_t num_points, const void* uu, const void* vv,
        const void* weight_in, void* weight_out, double cell_size_rad,
        int grid_size, const void* grid, unsigned long long* d_num_skipped,
        double frequency_hz, void* stream);

/* Block ingest: visibility blocks in host memory (pageable or pinned), as
 * the reference's main loop reads them (main.cpp:413-535), gridded into one
 * device grid.  Each pushed block is copied to the device on a copy stream
 * and gridded on the workspace's stream when its copy lands, with the
 * metres-to-wavelengths scaling of scale_coords (utils/read_vis.c:51-73)
 * done in the prep kernel when frequency_hz > 0.  push() returns once the
 * block's data has been copied (the caller may then refill its buffers)
 * while the block grids; the next push uploads while it grids.  `grid` and
 * `d_norm` (device, d_norm may be NULL) accumulate.  The workspace is busy
 * until finish(), which waits for every block and returns the total skip
 * count.  Options as oskar_b200_grid (frequency_hz there is ignored). */
typedef struct oskar_B200Blocks oskar_B200Blocks;
OSKAR_B200_EXPORT int oskar_b200_blocks_create(oskar_B200Workspace* ws,
        const oskar_B200Cube* cube, const oskar_B200Options* opt,
        double cell_size_rad, double w_scale, int grid_size, void* grid,
        double* d_norm, oskar_B200Blocks** blocks);
OSKAR_B200_EXPORT int oskar_b200_blocks_push(oskar_B200Blocks* blocks,
        size_t num_points, const void* uu, const void* vv, const void* ww,
        const void* vis, const void* weight, double frequency_hz);
OSKAR_B200_EXPORT int oskar_b200_blocks_finish(oskar_B200Blocks* blocks,
        unsigned long long* num_skipped);
OSKAR_B200_EXPORT int oskar_b200_blocks_free(oskar_B200Blocks* blocks);

/* Statistics of the most recent oskar_b200_grid call on this workspace
 * (valid once its stream has been synchronised). */
typedef struct oskar_B200Stats
{
    unsigned long long num_points;     /* visibilities given */
    unsigned long long num_gridded;    /* not skipped */
    unsigned long long grid_updates;   /* sum of (2S+1)^2 over gridded */
    unsigned long long num_tasks;      /* gridding work items */
    unsigned long long atomic_flushes; /* grid atomics issued (counted only
                                          with statistics level bit 1) */
    int status;                        /* device-side check status */
    int kernel_launches;               /* kernels the call launched */
    /* Stage durations in ms (CUDA events on the call's stream), filled
     * when stage timing is enabled on the workspace, else 0: placement and
     * keys, radix sort, task list, gridding kernel. */
    float prep_ms, sort_ms, tasks_ms, grid_ms;
} oskar_B200Stats;

OSKAR_B200_EXPORT int oskar_b200_last_stats(oskar_B200Workspace* ws,
        oskar_B200Stats* stats);

/* Autotuner.  (1) Threads per grid point: for each support size of `cube`,
 * grids the sample job's visibilities on planes of that support alone with
 * every built classes-per-thread choice (1-6: how many footprint rows a
 * thread of the gridding kernel owns), times the gridding kernel with CUDA
 * events (best of three) and keeps the fastest per support.  Supports with
 * fewer than 2000 sample visibilities keep the cost-model choice.  (2) Tile
 * width and kernel-value path: grids the whole sample with the coarse tile
 * at the automatic width, half and twice it, each with kernel values read
 * through L1 and staged in shared memory (plain accumulation only), and
 * keeps the fastest pipeline.  (3) Flush policy, with ACCUM_COMPENSATED in
 * `opt`: grids the sample with compensation everywhere, nowhere, and within
 * the radii (cells from the grid centre) holding 50, 75 and 90 % of its
 * visibilities, and keeps the smallest radius whose grid is within a
 * quarter of the uncompensated grid's distance from the fully compensated
 * one (two extra grids of scratch device memory).  Later calls on this
 * workspace that leave these to it (classes_per_thread 0, tile_shift 0,
 * staging 0, compensate_radius -1) use the results; oskar_b200_tune_launch
 * reads (2) and (3).  Device arrays as oskar_b200_grid; `grid` is scratch
 * (its contents are destroyed).  Synchronous.  table_out (host, 128
 * entries, indexed by support, may be NULL) receives the classes-per-thread
 * table. */
OSKAR_B200_EXPORT int oskar_b200_autotune(oskar_B200Workspace* ws,
        const oskar_B200Cube* cube, const oskar_B200Options* opt,
        size_t num_points, const void* uu, const void* vv, const void* ww,
        const void* vis, double cell_size_rad, double w_scale, int grid_size,
        void* grid, unsigned char* table_out);
/* Sets the workspace's classes-per-thread table (128 entries indexed by
 * support, each 1-6; NULL leaves it) and/or copies the table in use
 * into `current` (the cost model's until one is set or tuned). */
OSKAR_B200_EXPORT int oskar_b200_tune_table(oskar_B200Workspace* ws,
        const unsigned char* table, unsigned char* current);

/* The launch shape oskar_b200_autotune picks beside the table, used by
 * later calls whose options leave it to the workspace (tile_shift 0,
 * staging 0, compensate_radius -1): {tile_shift, staging, compensate_radius}
 * with staging 1 (shared) or 2 (L1).  `set` (3 ints, NULL leaves them)
 * installs a shape; `current` (3 ints, may be NULL) receives the shape in
 * use, {0, 2, 0} (automatic tiles, L1, compensation everywhere) until one is
 * tuned or set.  The reference's tiled gridder fixes its tile shape at
 * compile time (OskarTuningParams, oskar_grid_wproj_gpu.cu.old:1646-1655). */
OSKAR_B200_EXPORT int oskar_b200_tune_launch(oskar_B200Workspace* ws,
        const int* set, int* current);

/* Statistics level of every later gridding call on this workspace:
 * 0 = none; bit 0 (1) = CUDA events between the stages (stage times in
 * oskar_B200Stats); bit 1 (2) = also count the grid atomics the gridding
 * kernel issues (atomic_flushes; costs an instruction per tap, so leave it
 * off when timing). */
OSKAR_B200_EXPORT int oskar_b200_set_stage_timing(oskar_B200Workspace* ws,
        int enable);

/* Measures the device's complex-FP32 grid-atomic rate: `iters` rounds in
 * which every warp of a persistent grid issues red.global.add.v2.f32 to 32
 * consecutive cells at a pseudo-random row of `grid` (grid_size^2 complex
 * FP32 cells, device memory, contents destroyed).  Synchronous; returns
 * complex updates per second in *updates_per_s. */
OSKAR_B200_EXPORT int oskar_b200_measure_atomic_rate(oskar_B200Workspace* ws,
        void* grid, int grid_size, int iters, double* updates_per_s);

/* Gridding that allocates no device memory.  No counterpart in the
 * reference (whose CPU gridder needs no device memory at all).
 *
 * For callers that must not call cudaMalloc: code running inside a memory
 * pool fixed up front, a service whose device memory is provisioned by an
 * operator or scheduler, or a thread that must not take the allocator's
 * locks or risk its implicit device synchronisation while other streams
 * run.  Grids one FP32 job (FP64 placement, as oskar_grid_wproj_f) into
 * `grid` (device, accumulates), adding to *d_norm and writing
 * *d_num_skipped (device, either may be NULL).  conv_func, uu, vv, ww, vis
 * are device pointers; support is host memory; weight is ignored as in the
 * reference.  All scratch (the re-laid cube, sort keys, records, task list)
 * comes from one static device array of 64 MiB that every GPU loading this
 * library holds until the process exits: enough for about 1.5 million
 * visibilities with a small cube.  A job that does not fit returns
 * OSKAR_B200_ERR_OVER_BUDGET and touches nothing.  The array's device
 * address is looked up on the first call on each device (with that device
 * current), so make that first call outside any stream capture.  Every call
 * shares the array: calls whose device work can overlap (other streams,
 * other threads) race and must be serialised by the caller.  Asynchronous on
 * `stream` (NULL: the legacy default stream).  The return value covers the
 * arguments and the enqueueing only; the kernels' own checks land in a
 * status word inside the static array, read with
 * oskar_b200_grid_f_static_status.  The library holds the array's address
 * for the life of the process, so resetting the device (cudaDeviceReset)
 * after the first call is not supported. */
OSKAR_B200_EXPORT int oskar_b200_grid_f_static(size_t num_w_planes,
        const int* support, int oversample, int conv_size_half,
        const float* conv_func, size_t num_points, const float* uu,
        const float* vv, const float* ww, const float* vis,
        float cell_size_rad, float w_scale, int grid_size, float* grid,
        unsigned long long* d_num_skipped, double* d_norm, void* stream);

/* Device-side outcome of the latest oskar_b200_grid_f_static call on the
 * current device (no counterpart in the reference, whose CPU gridder cannot
 * fail).  Each call clears the status word in the static array before its
 * kernels run, and the kernels' bounds checks and bounded waits OR their
 * findings into it.  This copies the word back on `stream` (the stream of
 * the call, or one ordered after it), waits for that copy, and writes
 * *status: OSKAR_B200_OK, OSKAR_B200_ERR_DEVICE_CHECK (a bounds check
 * fired; the grid may be incomplete) or OSKAR_B200_ERR_TIMEOUT (a bounded
 * wait expired).  Allocates nothing.  A later call overwrites the word, so
 * read it before the next call; a call refused by its return value runs no
 * kernels and leaves the word as it was. */
OSKAR_B200_EXPORT int oskar_b200_grid_f_static_status(void* stream,
        int* status);

/* ---------------------------------------------------------------------- */
/* 3. Serving                                                             */
/* ---------------------------------------------------------------------- */

/* A resident gridding server on one device.  A server thread admits
 * submitted jobs in arrival order as slots and memory free up: each of
 * `num_slots` slots owns a workspace and a stream, so admitted jobs run
 * concurrently on the device; queued jobs that fit together are merged into
 * one batched launch (continuous batching).  Large jobs do not hold up
 * small ones: batches of up to 2^21 visibilities run on a stream of the
 * device's highest priority, larger batches grid in time slices of about
 * 2^22 visibilities whose SMs go to waiting high-priority work first, and
 * with three or more slots the last slot takes only such small jobs
 * (passing large ones in the queue).  The server owns each job's
 * output grid, allocated (zeroed) at admission; the HBM budget covers the
 * slots' workspaces and the live output grids, and a job waits until it
 * fits.  Cubes and input visibilities stay the caller's (device memory). */
typedef struct oskar_B200Server oskar_B200Server;

typedef struct oskar_B200Request
{
    unsigned long long tag;        /* caller's id, echoed in the completion */
    const oskar_B200Cube* cube;    /* resident, may be shared by requests */
    size_t num_points;
    const void* uu;                /* device pointers, cube's precision */
    const void* vv;
    const void* ww;
    const void* vis;
    const void* weight;
    double cell_size_rad;
    double w_scale;
    int grid_size;
    double frequency_hz;           /* as oskar_B200Options::frequency_hz */
} oskar_B200Request;

typedef struct oskar_B200Completion
{
    unsigned long long tag;
    int status;                    /* oskar_B200Status of the job */
    unsigned long long num_skipped;
    double norm;
    void* grid;                    /* device grid owned by the server until
                                      oskar_b200_server_release(tag) */
    double submit_s, start_s, end_s;   /* server clock (oskar_b200_server_clock) */
    int batch_size;                /* jobs in the launch that ran it */
} oskar_B200Completion;

OSKAR_B200_EXPORT int oskar_b200_server_create(int device,
        size_t hbm_budget_bytes, int num_slots, int max_batch_jobs,
        const oskar_B200Options* opt, oskar_B200Server** server);
/* Queues a job (non-blocking). */
OSKAR_B200_EXPORT int oskar_b200_server_submit(oskar_B200Server* server,
        const oskar_B200Request* request);
/* Returns up to max_out completed jobs, waiting up to timeout_s for the
 * first one; *num_out may be 0 on timeout. */
OSKAR_B200_EXPORT int oskar_b200_server_poll(oskar_B200Server* server,
        oskar_B200Completion* out, int max_out, int* num_out,
        double timeout_s);
/* Returns a completed job's grid to the server (and its budget). */
OSKAR_B200_EXPORT int oskar_b200_server_release(oskar_B200Server* server,
        unsigned long long tag);
/* Seconds since the server started (the clock of the completions). */
OSKAR_B200_EXPORT double oskar_b200_server_clock(oskar_B200Server* server);
/* Device bytes the server holds now, and its budget. */
OSKAR_B200_EXPORT int oskar_b200_server_memory(oskar_B200Server* server,
        size_t* bytes_in_use, size_t* budget);
/* Drains all jobs, frees every grid and workspace, stops the thread. */
OSKAR_B200_EXPORT int oskar_b200_server_free(oskar_B200Server* server);

/* Self-test of the device-side bounded waits: a kernel waits on a barrier
 * phase that nothing completes, gives up after `spins` attempts and records
 * a timeout in the workspace's status word, leaving the context usable.
 * *device_status receives OSKAR_B200_ERR_TIMEOUT when the wait expired as
 * designed.  Synchronous. */
OSKAR_B200_EXPORT int oskar_b200_selftest_bounded_wait(
        oskar_B200Workspace* ws, unsigned spins, int* device_status);

/* Testing aid for failure handling (the reference has no counterpart: it
 * aborts on errors).  After `after` more device allocations by this library
 * succeed, the next one fails as if the device were out of memory, once;
 * -1 disarms.  Lets a test check that a call reports
 * OSKAR_B200_ERR_OUT_OF_MEMORY and leaves the caller's outputs untouched
 * without exhausting a shared GPU.  Process-wide; not for production use. */
OSKAR_B200_EXPORT int oskar_b200_testing_fail_allocation(long long after);

/* Testing aid for oskar_b200_grid_f_static_status (no counterpart in the
 * reference): enqueues on `stream` a write of `bits` (device check bits:
 * 1 grid index, 2 slab index, 4 wait timeout, 8 task bounds) into the
 * static array's status word on the current device, as a kernel whose check
 * fired would.  Lets a test see the reader report a failure, and the next
 * gridding call clear it, without provoking a fault on the GPU. */
OSKAR_B200_EXPORT int oskar_b200_testing_set_static_status(
        unsigned long long bits, void* stream);

/* Library build description (arch, version). */
OSKAR_B200_EXPORT const char* oskar_b200_build_info(void);

#ifdef __cplusplus
}
#endif

#endif /* OSKAR_GRID_WPROJ_B200_H_ */
