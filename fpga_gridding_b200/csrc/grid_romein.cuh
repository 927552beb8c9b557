// Launch interface of the Romein gridding kernel.
#pragma once

#include "internal.h"

namespace b200 {

constexpr int kGridThreads = 256;   // threads per CTA
constexpr int kTaskMax = 256;       // visibilities per task
constexpr int kTuneMax = 128;       // supports covered by the tune table
constexpr unsigned kBulkChunk = 32768;  // bytes per cp.async.bulk
constexpr int kMaxOffsets = 33;     // 2 * ceil(oversample / 2) + 1, oversample <= 32

struct GridArgs
{
    const int4* srec;           // sorted placement records
    const void* svis;           // sorted visibilities (float2 / double2)
    const uint32_t* task_start; // [num_tasks + 1]
    const PlaneDesc* planes;
    const void* slabs;
    void* grid;
    void* comp;                 // compensation grid (ACCUM_COMPENSATED) or null
    unsigned long long* counters;
    int grid_size;
    int oversample;
    int half;
    unsigned block_smem_bytes;  // set by launch_grid
    unsigned char cpt[kTuneMax];
};

void default_tune_table(unsigned char* cpt);
size_t grid_smem_bytes(const oskar_B200Cube* cube, bool staged);
cudaError_t launch_grid(const GridArgs& a, const oskar_B200Cube* cube,
                        bool staged, bool compensated, int num_sms,
                        cudaStream_t st, int* ctas_out);
// grid[i] += comp[i]; comp[i] = 0 over 2 * cells floats.
cudaError_t launch_fold(float* grid, float* comp, size_t cells,
                        int num_sms, cudaStream_t st);

}  // namespace b200
