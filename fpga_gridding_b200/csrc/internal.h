// Internal host-side declarations of the B200 gridder.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <atomic>
#include <vector>

#include "oskar_grid_wproj_b200.h"

namespace b200 {

// ---------------------------------------------------------------------------
// Re-laid kernel cube.
//
// The reference stores, per w-plane, the non-negative quadrant of the
// oversampled kernel, indexed by |off + tap * oversample| in each axis
// (oskar_grid_wproj.c:110-117).  Each plane becomes one "slab":
//   columns: quadrant column x goes to position (x % os) * L + x / os,
//     L = ceil(E / os), E = os * S + ceil(os / 2) + 1 (the entries the plane
//     can use).  The taps k = -S..S of one visibility then read consecutive
//     positions (an ascending run for off + k * os >= 0, a descending run
//     for the rest), so a warp's kernel reads are contiguous.
//   rows: expanded per row offset.  Row (off_v + H) * W + (j + S),
//     W = 2S + 1, H = ceil(os / 2), holds quadrant row |off_v + j * os|.
//     A visibility's tap rows j = -S..S are then W consecutive slab rows, so
//     the row part of a tap's index is linear in the tap row.
// ---------------------------------------------------------------------------
struct PlaneDesc
{
    int support;        // S
    int extent;         // E
    int L;              // column positions per oversample phase
    int pitch;          // row length of the slab in elements (os * L)
    int rows;           // slab rows: (2H + 1) * (2S + 1)
    long long offset;   // element offset of the slab in the slab array
    unsigned bytes;     // slab bytes, rounded up to 16
    float scale;        // stored value = true value / scale (1 unless F16/BF16)
};

// One gridding job of a batch, as the device kernels see it.  A single
// oskar_b200_grid call is a batch of one.
struct JobDesc
{
    const void* uu;
    const void* vv;
    const void* ww;
    const void* vis;
    const void* weight;
    void* grid;
    void* comp;                   // error grid (ACCUM_COMPENSATED) or null
    const PlaneDesc* planes;
    const void* slabs;
    const double* norm_table;
    const int* support;
    double* d_norm;               // caller's norm accumulator (device) or null
    unsigned long long* d_skipped;// caller's skip count (device) or null
    double grid_scale;            // grid_size * cell_size_rad, FP64
    double w_scale;
    float grid_scale_f;           // the same rounded as float C computes it
    float w_scale_f;
    double coord_scale = 1.0;     // uu, vv, ww multiplier (frequency / c, or 1)
    float coord_scale_f = 1.0f;   // the same rounded to float (FP32 data)
    unsigned long long first;     // global index of the job's first point
    unsigned long long n;         // points of the job
    int grid_size;
    int num_planes;
    int oversample;
    int half;                     // ceil(oversample / 2)
};

struct DeviceBuffer
{
    void* ptr = nullptr;
    size_t bytes = 0;
    cudaError_t ensure(size_t n);  // grow-only; contents not preserved
    void release();
    ~DeviceBuffer();
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    DeviceBuffer(DeviceBuffer&& o) noexcept : ptr(o.ptr), bytes(o.bytes)
    {
        o.ptr = nullptr;
        o.bytes = 0;
    }
};

// Injected device-allocation failures (testing aid), see pipeline.cu.
extern std::atomic<long long> g_alloc_countdown;

// Events of the drop-in's pipelined upload: cube and up to 15 chunks.
constexpr int kIngestEvents = 16;
// Bands of grid rows (rows of coarse tiles, at most 16 per grid).
constexpr int kMaxBands = 16;
// Pinned host job tables per workspace (see oskar_B200Workspace::h_jobs).
constexpr int kJobRing = 8;

// Band-ordered gridding of one job: the gridding kernel runs once per band
// of coarse-tile rows, bands taken in `order`, and events[i] (created by the
// caller) is recorded on the stream after the i-th of them.  Band b covers
// grid rows [b << row_shift, (b + 1) << row_shift); the footprints of its
// tasks reach at most `halo` rows beyond it.  The order is outside-in
// (0, last, 1, last - 1, ...): visibilities concentrate near the uv origin,
// so the light outer bands finish first and the heavy central ones last.
struct BandPlan
{
    cudaEvent_t* events;      // kMaxBands of them
    int num_bands;            // set by run_batch
    int row_shift;            // set by run_batch
    int halo;                 // set by run_batch: the cube's largest support
    int order[kMaxBands];     // set by run_batch
};

}  // namespace b200

// Opaque public types.
struct oskar_B200Workspace
{
    int device = 0;
    int num_sms = 0;
    size_t smem_optin = 0;
    cudaStream_t stream = nullptr;
    // per-visibility work arrays
    b200::DeviceBuffer keys[2], vals[2], rec, scan_tmp, flags;
    b200::DeviceBuffer task_start, task_job;
    // small arrays: counters, partial sums, per-job plane histograms and
    // skip counts, the job table
    b200::DeviceBuffer counters, partials, plane_counts, job_skipped, jobs;
    // pinned host copies of the job table (the sources of its uploads), a
    // ring of them so that a call rarely waits for an earlier call's upload,
    // each with the event after which that upload has read it
    void* h_jobs[b200::kJobRing] = {};
    size_t h_jobs_bytes[b200::kJobRing] = {};
    cudaEvent_t jobs_event[b200::kJobRing] = {};
    int jobs_event_pending[b200::kJobRing] = {};
    int jobs_slot = 0;
    // drop-in staging of the caller's host arrays
    b200::DeviceBuffer in_uu, in_vv, in_ww, in_vis, in_weight, in_grid,
        in_cube, in_norm;
    // error grid of ACCUM_COMPENSATED
    b200::DeviceBuffer comp_grid;
    // drop-in pipelined upload: copy stream, its events (cube, one per
    // chunk) and the zeroed grid the chunks accumulate into
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ingest_events[b200::kIngestEvents] = {};
    b200::DeviceBuffer acc_grid;
    // band-ordered last chunk: per band, the event after its gridding and
    // the event after the upload of its rows of the caller's grid; the
    // stream that adds finished rows to the caller's grid and copies them
    // back; band_first[kMaxBands + 1] (uint32) then the bands' work-queue
    // counters (uint64) at byte 128
    cudaStream_t d2h_stream = nullptr;
    cudaEvent_t band_events[b200::kMaxBands] = {};
    cudaEvent_t piece_events[b200::kMaxBands] = {};
    b200::DeviceBuffer bands;
    // pinned host mirror of the device counters (stats)
    void* h_counters = nullptr;
    unsigned long long last_points = 0;
    int last_launches = 0;
    // statistics level (oskar_b200_set_stage_timing): bit 0 stage events,
    // bit 1 atomic counting
    int stage_timing = 0;
    int events_recorded = 0;
    cudaEvent_t events[5] = {};
    // classes-per-thread table measured by oskar_b200_autotune
    unsigned char tune[128] = {};
    int tuned = 0;
    // launch shape picked by oskar_b200_autotune (or set): coarse tile
    // shift (0: automatic), staging (1 shared, 2 L1), compensation radius
    int tuned_launch = 0;
    int tuned_tile_shift = 0;
    int tuned_staging = 2;
    int tuned_comp_radius = 0;
};

struct oskar_B200Cube
{
    int device = 0;
    int num_planes = 0;
    int oversample = 0;
    int half = 0;            // ceil(oversample / 2): offsets lie in [-half, half]
    int conv_size_half = 0;
    int data_is_double = 0;
    int kernel_type = OSKAR_B200_KERNEL_NATIVE;
    int elem_bytes = 0;      // bytes per stored complex value
    unsigned max_slab_bytes = 0;
    unsigned max_block_bytes = 0;   // largest W-row block (one row offset)
    int max_support = 0;
    std::vector<b200::PlaneDesc> planes;
    b200::DeviceBuffer d_planes, d_slabs, d_norm_table, d_support;
};

namespace b200 {

// Counter slots in oskar_B200Workspace::counters (unsigned long long each).
enum CounterSlot
{
    CNT_SKIPPED = 0,
    CNT_TASKS = 1,
    CNT_TASK_NEXT = 2,   // work-queue head of the gridding kernel
    CNT_FLUSHES = 3,
    CNT_STATUS = 4,      // DEV_ERR_* bits
    CNT_UPDATES = 5,     // grid updates (taps) of gridded points
    CNT_COUNT = 8
};

// ---- radix_sort.cu --------------------------------------------------------
size_t scan_temp_bytes(size_t n);
// Exclusive prefix sum of n uint32 values (out must not alias in).
cudaError_t exclusive_scan_u32(const uint32_t* in, uint32_t* out, size_t n,
                               void* temp, cudaStream_t st, int* launches);
size_t radix_sort_temp_bytes(size_t n);
// Stable LSD sort of (key, value) pairs on the low num_bits of the keys.
// The sorted pairs end in keys[*which] / vals[*which].
cudaError_t radix_sort_pairs(uint32_t* keys[2], uint32_t* vals[2], size_t n,
                             int num_bits, void* temp, cudaStream_t st,
                             int* which, int* launches);

// ---- cube.cu ----------------------------------------------------------------
// d_conv_im == nullptr: d_conv_func is the interleaved complex cube;
// otherwise d_conv_func / d_conv_im hold the real / imaginary parts.
int cube_build(oskar_B200Cube* cube, const void* d_conv_func,
               const void* d_conv_im, int conv_func_is_double,
               cudaStream_t st);

// ---- prep.cu / grid_romein.cu ---------------------------------------------
// Sort key, most significant first:
//   job | coarse tile (row-major: row, column) | w-plane |
//   cell inside the tile (Morton)
// with a skip flag above all of them.
struct KeyLayout
{
    int coarse_shift;  // log2 of the coarse tile side (cells)
    int coarse_bits;   // bits per axis of the coarse tile index
    int fine_shift;    // cells dropped inside a coarse tile
    int fine_bits;     // bits per axis of the fine index
    int plane_bits;
    int job_bits;
    int job_shift;     // position of the job field
    int total_bits;    // key bits below the skip flag
};
// Layout for the largest grid and plane count of the batch; false if the
// fields cannot fit 31 bits.
// tile_shift > 0 sets the coarse tile side to 2^tile_shift cells (at least
// 64, at most the grid); 0 picks grid_size / 16.
bool make_key_layout(int grid_size, int num_planes, int num_jobs,
                     KeyLayout* out, int tile_shift = 0);

// One job of a batch, host side.
struct HostJob
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
    double frequency_hz;          // 0: coordinates in wavelengths
};

// Grids a batch of jobs that share precision and kernel storage type, with
// one sort and one persistent gridding launch.  degrid: the same placement
// and sort, then the adjoint (degrid.cu): each job's `grid` is read and its
// `vis` written.
// time_slices > 1 (at most kMaxBands; not with bands or degrid): the
// gridding kernel runs as that many launches over contiguous ranges of the
// task list, so that the device can schedule other streams' work between
// them (the server's large batches).
int run_batch(oskar_B200Workspace* ws, const oskar_B200Options* opt,
              int num_jobs, const HostJob* jobs, cudaStream_t st,
              bool degrid = false, BandPlan* bands = nullptr,
              int time_slices = 1);
// first[0..k_slices] = the bounds of k_slices equal ranges of the task
// list; queues[0..k_slices) = 0.
cudaError_t launch_slice_bounds(const unsigned long long* counters,
                                int k_slices, uint32_t* first,
                                unsigned long long* queues, cudaStream_t st);

// ---- degrid.cu ------------------------------------------------------------
cudaError_t launch_degrid(const uint32_t* order, const uint32_t* sorted_keys,
                          const int4* rec, const JobDesc* jobs, int job_shift,
                          int apply_weight, unsigned long long* counters,
                          size_t n, int data_is_double, int kernel_type,
                          int num_sms, cudaStream_t st);

int run_grid(oskar_B200Workspace* ws, const oskar_B200Cube* cube,
             const oskar_B200Options* opt, size_t num_points, const void* uu,
             const void* vv, const void* ww, const void* vis,
             const void* weight, double cell_size_rad, double w_scale,
             int grid_size, void* grid, unsigned long long* d_num_skipped,
             double* d_norm, cudaStream_t st);

int run_place(oskar_B200Workspace* ws, int data_is_double, int coord_mode,
              const int* d_support, int num_planes, int oversample,
              size_t num_points, const void* uu, const void* vv,
              const void* ww, double cell_size_rad, double w_scale,
              int grid_size, int32_t* gu, int32_t* gv, int32_t* plane,
              int32_t* off_u, int32_t* off_v, int32_t* conj,
              int32_t* skipped, cudaStream_t st);

int measure_atomic_rate(oskar_B200Workspace* ws, void* grid, int grid_size,
                        int iters, double* updates_per_s);

// ---- weights.cu -------------------------------------------------------------
// Uniform weighting (utils/oskar_grid_weights.c:38-172) on device arrays.
// *d_num_skipped (or a workspace counter when null) is reset, then counts.
int run_weights_write(oskar_B200Workspace* ws, int data_is_double,
                      int ordered, size_t n, const void* uu, const void* vv,
                      const void* weight, double cell_size_rad,
                      int grid_size, void* grid,
                      unsigned long long* d_num_skipped, double frequency_hz,
                      cudaStream_t st);
int run_weights_read(oskar_B200Workspace* ws, int data_is_double, size_t n,
                     const void* uu, const void* vv, const void* weight_in,
                     void* weight_out, double cell_size_rad, int grid_size,
                     const void* grid, unsigned long long* d_num_skipped,
                     double frequency_hz, cudaStream_t st);

// Coordinate multiplier of scale_coords (utils/read_vis.c:54): frequency
// over the speed of light, or 1 when frequency_hz is 0.
double coord_scale_of(double frequency_hz);

int selftest_bounded_wait(oskar_B200Workspace* ws, unsigned spins,
                          int* device_status);

// ---- autotune.cu ------------------------------------------------------------
int run_autotune(oskar_B200Workspace* ws, const oskar_B200Cube* cube,
                 const oskar_B200Options* opt, size_t n, const void* uu,
                 const void* vv, const void* ww, const void* vis,
                 double cell_size_rad, double w_scale, int grid_size,
                 void* grid, unsigned char* table_out);

// dst[i] += src[i] for n reals (FP64 when is_double, else FP32); where
// dst[i] is zero the result is src[i] itself (sign of zero and NaN bits
// kept).
cudaError_t launch_add(void* dst, const void* src, size_t n, int is_double,
                       int num_sms, cudaStream_t st);
// *acc |= the workspace's device status word (after a run_batch on st).
cudaError_t launch_status_or(oskar_B200Workspace* ws,
                             unsigned long long* acc, cudaStream_t st);

int status_from_cuda(cudaError_t e);

// Validates an options struct for data of the given precision.
int check_options(const oskar_B200Options* opt, int data_is_double);

}  // namespace b200
