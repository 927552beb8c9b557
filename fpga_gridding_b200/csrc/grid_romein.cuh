// Launch interface of the Romein gridding kernel.
#pragma once

#include "internal.h"

namespace b200 {

constexpr int kGridThreads = 256;   // threads per CTA
// Resident CTAs per SM the gridding kernel's registers are bounded for:
// 4 for FP32 grids (64 registers), 3 for FP64 (80; its accumulators and
// coefficients are twice as wide and spill at 64).
template <typename GT>
constexpr int grid_ctas_per_sm() { return sizeof(GT) == 8 ? 3 : 4; }
constexpr int kTaskMax = 256;       // visibilities per task
constexpr int kTuneMax = 128;       // supports covered by the tune table
constexpr unsigned kBulkChunk = 32768;  // bytes per cp.async.bulk
constexpr int kMaxOffsets = 33;     // 2 * ceil(oversample / 2) + 1, oversample <= 32

struct GridArgs
{
    const uint32_t* order;      // sorted position -> point (global index)
    const int4* rec;            // placement record of each point
    int apply_weight;           // visibilities x weight (see JobDesc)
    const uint32_t* task_start; // [num_tasks + 1]
    const uint32_t* task_job;   // [num_tasks]: job of each task
    const JobDesc* jobs;        // cube, grid and geometry of each job
    unsigned long long* counters;
    unsigned block_smem_bytes;  // set by launch_grid
    int comp_radius;            // see oskar_B200Options::compensate_radius
    int count_flushes;          // count grid atomics (statistics)
    unsigned char cpt[kTuneMax];
    // Optional task range [range[0], range[1]) with its own work-queue
    // counter (one launch per band of grid rows); null: every task, queue
    // head counters[CNT_TASK_NEXT].
    const uint32_t* range;
    unsigned long long* queue;
};

void default_tune_table(unsigned char* cpt);
size_t grid_smem_bytes(int data_is_double, unsigned max_block_bytes,
                       bool staged);
cudaError_t launch_grid(const GridArgs& a, int data_is_double,
                        int kernel_type, unsigned max_block_bytes, bool staged,
                        bool compensated, int num_sms, cudaStream_t st,
                        int* ctas_out);
// For every job with an error grid: grid += comp, comp = 0.
cudaError_t launch_fold_jobs(const JobDesc* jobs, int num_jobs, int num_sms,
                             cudaStream_t st);

}  // namespace b200
