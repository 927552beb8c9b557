// Uniform weighting on the device: the weights-grid histogram ("write") and
// the density lookup ("read") of utils/oskar_grid_weights.c:38-172.
//
// Both steps place a point at the cell
//   grid_u = (int)round(-u * grid_size * cell) + grid_size / 2,
//   grid_v = (int)round( v * grid_size * cell) + grid_size / 2
// (u, v first scaled from metres to wavelengths as scale_coords does, when a
// frequency is given)
// and skip it when the cell is outside the grid.  The weights grid is real
// (one value per cell), row-major in v.
//
// write, ordered (the default, bit-exact): the reference adds the weights of
//   a cell in point order, so a stable radix sort of (cell, point index)
//   gathers each cell's points in that order, and they are added one after
//   the other onto the cell's previous value (by one thread, or by one warp
//   for a cell with more than 32 points).  The sums are the reference's to
//   the bit for any weights.
// write, atomic: one fire-and-forget reduction per point.  Cell sums then
//   depend on the order the reductions land in; they are exact whenever the
//   partial sums are (e.g. unit weights below 2^24 per cell in FP32).
// read: one thread per point; out = in / grid[cell] (IEEE division), 0 where
//   the cell is empty, and skipped points keep their previous output value.
#include <climits>

#include "common.cuh"
#include "internal.h"

namespace b200 {
namespace {

struct WeightConsts
{
    double grid_scale;   // grid_size * cell_size_rad, FP64
    float grid_scale_f;  // the same product in float arithmetic
    double coord_scale;  // metres to wavelengths (scale_coords), or 1
    float coord_scale_f;
    int grid_size;
    int centre;
};

// Cell index of a point, or -1 when it is skipped.  A rounded coordinate
// outside the int range (or NaN) converts to INT_MIN, as x86-64's truncating
// conversion does, and is therefore skipped.
template <typename T>
__device__ __forceinline__ long long weight_cell(T u, T v,
                                                 const WeightConsts& c)
{
    long long gu, gv;
    if (sizeof(T) == sizeof(double))
    {
        const double us = __dmul_rn((double)u, c.coord_scale);
        const double vs = __dmul_rn((double)v, c.coord_scale);
        const double ru = round(__dmul_rn(-us, c.grid_scale));
        const double rv = round(__dmul_rn(vs, c.grid_scale));
        gu = (ru > -2147483649.0 && ru < 2147483648.0 ? (long long)ru
                                                        : (long long)INT_MIN);
        gv = (rv > -2147483649.0 && rv < 2147483648.0 ? (long long)rv
                                                        : (long long)INT_MIN);
    }
    else
    {
        const float us = __fmul_rn((float)u, c.coord_scale_f);
        const float vs = __fmul_rn((float)v, c.coord_scale_f);
        const float ru = roundf(__fmul_rn(-us, c.grid_scale_f));
        const float rv = roundf(__fmul_rn(vs, c.grid_scale_f));
        gu = (ru > -2147483649.0f && ru < 2147483648.0f ? (long long)ru
                                                          : (long long)INT_MIN);
        gv = (rv > -2147483649.0f && rv < 2147483648.0f ? (long long)rv
                                                          : (long long)INT_MIN);
    }
    gu += c.centre;
    gv += c.centre;
    if (gu < 0 || gu >= c.grid_size || gv < 0 || gv >= c.grid_size) return -1;
    return gv * c.grid_size + gu;
}

__device__ __forceinline__ double add_rn(double a, double b)
{
    return __dadd_rn(a, b);
}
__device__ __forceinline__ float add_rn(float a, float b)
{
    return __fadd_rn(a, b);
}
__device__ __forceinline__ double div_rn(double a, double b)
{
    return __ddiv_rn(a, b);
}
__device__ __forceinline__ float div_rn(float a, float b)
{
    return __fdiv_rn(a, b);
}

__device__ __forceinline__ void count_skipped(unsigned local,
                                              unsigned long long* skipped)
{
    local = warp_sum(local);
    if ((threadIdx.x & 31) == 0 && local)
        atomicAdd(skipped, (unsigned long long)local);
}

template <typename T>
__global__ void __launch_bounds__(256)
weights_write_atomic_kernel(size_t n, const T* __restrict__ uu,
                            const T* __restrict__ vv,
                            const T* __restrict__ weight, WeightConsts c,
                            T* __restrict__ grid,
                            unsigned long long* __restrict__ skipped)
{
    unsigned local = 0;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += stride)
    {
        const long long t = weight_cell(uu[i], vv[i], c);
        if (t < 0)
            ++local;
        else
            atomicAdd(grid + t, weight[i]);
    }
    count_skipped(local, skipped);
}

// Sort keys for the ordered write: the cell, or `sentinel` (= grid_size^2,
// above every cell) for a skipped point; values are the point indices.
template <typename T>
__global__ void __launch_bounds__(256)
weights_key_kernel(size_t n, const T* __restrict__ uu,
                   const T* __restrict__ vv, WeightConsts c,
                   uint32_t sentinel, uint32_t* __restrict__ keys,
                   uint32_t* __restrict__ vals,
                   unsigned long long* __restrict__ skipped)
{
    unsigned local = 0;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += stride)
    {
        const long long t = weight_cell(uu[i], vv[i], c);
        local += t < 0;
        keys[i] = t < 0 ? sentinel : (uint32_t)t;
        vals[i] = (uint32_t)i;
    }
    count_skipped(local, skipped);
}

// Sums each run of equal keys (one cell's points, in point order) onto the
// cell's previous value.  A warp takes 32 sorted positions at a time; a lane
// holding the first element of a run of at most 32 sums it alone, and runs
// longer than 32 (the dense cells near the grid centre, up to ~10^4 points)
// are summed by the whole warp: 32 weights are gathered at once (the next 32
// already in flight) and added in order through warp shuffles, every lane
// keeping the same running sum.  Either way the additions are exactly the
// reference's, in its order.
template <typename T>
__global__ void __launch_bounds__(256)
weights_run_sum_kernel(size_t n, const uint32_t* __restrict__ keys,
                       const uint32_t* __restrict__ vals,
                       const T* __restrict__ weight, uint32_t sentinel,
                       T* __restrict__ grid)
{
    const int lane = threadIdx.x & 31;
    const size_t warp0 = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const size_t warps = ((size_t)gridDim.x * blockDim.x) >> 5;
    for (size_t base = warp0 * 32; base < n; base += warps * 32)
    {
        const size_t i = base + lane;
        const uint32_t k = i < n ? keys[i] : sentinel;
        const bool head = k != sentinel && (i == 0 || keys[i - 1] != k);
        // Sorted keys: the run is longer than 32 iff position i + 32 holds
        // the same key.
        const bool longrun = head && i + 32 < n && keys[i + 32] == k;
        if (head && !longrun)
        {
            T acc = grid[k];
            for (size_t j = i; j < i + 32; j += 4)
            {
                uint32_t kk[4];
                T ww[4];
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    kk[q] = j + q < n ? keys[j + q] : sentinel;
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    ww[q] = kk[q] == k ? weight[vals[j + q]] : T(0);
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    if (kk[q] == k) acc = add_rn(acc, ww[q]);
                if (kk[3] != k) break;
            }
            grid[k] = acc;
        }
        unsigned pending = __ballot_sync(0xffffffffu, longrun);
        while (pending)
        {
            const int src = __ffs(pending) - 1;
            pending &= pending - 1;
            const size_t b = base + (size_t)src;
            const uint32_t key = __shfl_sync(0xffffffffu, k, src);
            T acc = grid[key];
            size_t j = b + lane;
            uint32_t kk = j < n ? keys[j] : sentinel;
            T v = kk == key ? weight[vals[j]] : T(0);
            for (;;)
            {
                const unsigned match = __ballot_sync(0xffffffffu, kk == key);
                const int cnt = __popc(match);
                // next chunk in flight while this one is summed
                const size_t jn = j + 32;
                uint32_t kn = sentinel;
                T vn = T(0);
                if (cnt == 32)
                {
                    kn = jn < n ? keys[jn] : sentinel;
                    vn = kn == key ? weight[vals[jn]] : T(0);
                }
#pragma unroll
                for (int t = 0; t < 32; ++t)
                {
                    const T x = __shfl_sync(0xffffffffu, v, t);
                    if (t < cnt) acc = add_rn(acc, x);
                }
                if (cnt < 32) break;
                j = jn;
                kk = kn;
                v = vn;
            }
            if (lane == 0) grid[key] = acc;
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(256)
weights_read_kernel(size_t n, const T* __restrict__ uu,
                    const T* __restrict__ vv,
                    const T* __restrict__ weight_in,
                    T* __restrict__ weight_out, WeightConsts c,
                    const T* __restrict__ grid,
                    unsigned long long* __restrict__ skipped)
{
    unsigned local = 0;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += stride)
    {
        const long long t = weight_cell(uu[i], vv[i], c);
        if (t < 0)
        {
            ++local;
            continue;
        }
        const T g = grid[t];
        weight_out[i] = g != T(0) ? div_rn(weight_in[i], g) : T(0);
    }
    count_skipped(local, skipped);
}

WeightConsts make_consts(int data_is_double, double cell_size_rad,
                         int grid_size, double frequency_hz)
{
    WeightConsts c;
    c.grid_scale = grid_size * cell_size_rad;
    // C evaluates int * float in float (FLT_EVAL_METHOD 0 on x86-64).
    c.grid_scale_f = (float)grid_size * (float)cell_size_rad;
    c.coord_scale = coord_scale_of(frequency_hz);
    c.coord_scale_f = (float)c.coord_scale;
    (void)data_is_double;
    c.grid_size = grid_size;
    c.centre = grid_size / 2;
    return c;
}

int bit_length(unsigned long long x)
{
    int b = 0;
    while (x) { ++b; x >>= 1; }
    return b;
}

int launch_blocks(const oskar_B200Workspace* ws, size_t n)
{
    const size_t want = (n + 255) / 256;
    const size_t cap = (size_t)ws->num_sms * 8;
    return (int)(want < cap ? (want ? want : 1) : cap);
}

#define B200_TRY(expr)                                      \
    do {                                                    \
        const cudaError_t e_ = (expr);                      \
        if (e_ != cudaSuccess) return status_from_cuda(e_); \
    } while (0)

unsigned long long* skip_counter(oskar_B200Workspace* ws,
                                 unsigned long long* d_num_skipped)
{
    if (d_num_skipped) return d_num_skipped;
    return static_cast<unsigned long long*>(ws->counters.ptr) + CNT_SKIPPED;
}

}  // namespace

int run_weights_write(oskar_B200Workspace* ws, int data_is_double,
                      int ordered, size_t n, const void* uu, const void* vv,
                      const void* weight, double cell_size_rad,
                      int grid_size, void* grid,
                      unsigned long long* d_num_skipped, double frequency_hz,
                      cudaStream_t st)
{
    B200_TRY(ws->counters.ensure(sizeof(unsigned long long) * CNT_COUNT));
    unsigned long long* skipped = skip_counter(ws, d_num_skipped);
    B200_TRY(cudaMemsetAsync(skipped, 0, sizeof(unsigned long long), st));
    int launches = 0;
    if (n == 0)
    {
        ws->last_launches = 0;
        return OSKAR_B200_OK;
    }
    const WeightConsts c = make_consts(data_is_double, cell_size_rad,
                                       grid_size, frequency_hz);
    const int blocks = launch_blocks(ws, n);
    if (!ordered)
    {
        if (data_is_double)
            weights_write_atomic_kernel<double><<<blocks, 256, 0, st>>>(
                n, (const double*)uu, (const double*)vv,
                (const double*)weight, c, (double*)grid, skipped);
        else
            weights_write_atomic_kernel<float><<<blocks, 256, 0, st>>>(
                n, (const float*)uu, (const float*)vv, (const float*)weight,
                c, (float*)grid, skipped);
        B200_TRY(cudaGetLastError());
        ws->last_launches = 1;
        return OSKAR_B200_OK;
    }
    B200_TRY(ws->keys[0].ensure(4 * n));
    B200_TRY(ws->keys[1].ensure(4 * n));
    B200_TRY(ws->vals[0].ensure(4 * n));
    B200_TRY(ws->vals[1].ensure(4 * n));
    B200_TRY(ws->scan_tmp.ensure(radix_sort_temp_bytes(n)));
    uint32_t* keys[2] = {static_cast<uint32_t*>(ws->keys[0].ptr),
                         static_cast<uint32_t*>(ws->keys[1].ptr)};
    uint32_t* vals[2] = {static_cast<uint32_t*>(ws->vals[0].ptr),
                         static_cast<uint32_t*>(ws->vals[1].ptr)};
    const unsigned long long cells =
        (unsigned long long)grid_size * (unsigned long long)grid_size;
    const uint32_t sentinel = (uint32_t)cells;
    if (data_is_double)
        weights_key_kernel<double><<<blocks, 256, 0, st>>>(
            n, (const double*)uu, (const double*)vv, c, sentinel, keys[0],
            vals[0], skipped);
    else
        weights_key_kernel<float><<<blocks, 256, 0, st>>>(
            n, (const float*)uu, (const float*)vv, c, sentinel, keys[0],
            vals[0], skipped);
    B200_TRY(cudaGetLastError());
    ++launches;
    int which = 0;
    B200_TRY(radix_sort_pairs(keys, vals, n, bit_length(cells),
                              ws->scan_tmp.ptr, st, &which, &launches));
    if (data_is_double)
        weights_run_sum_kernel<double><<<blocks, 256, 0, st>>>(
            n, keys[which], vals[which], (const double*)weight, sentinel,
            (double*)grid);
    else
        weights_run_sum_kernel<float><<<blocks, 256, 0, st>>>(
            n, keys[which], vals[which], (const float*)weight, sentinel,
            (float*)grid);
    B200_TRY(cudaGetLastError());
    ++launches;
    ws->last_launches = launches;
    return OSKAR_B200_OK;
}

int run_weights_read(oskar_B200Workspace* ws, int data_is_double, size_t n,
                     const void* uu, const void* vv, const void* weight_in,
                     void* weight_out, double cell_size_rad, int grid_size,
                     const void* grid, unsigned long long* d_num_skipped,
                     double frequency_hz, cudaStream_t st)
{
    B200_TRY(ws->counters.ensure(sizeof(unsigned long long) * CNT_COUNT));
    unsigned long long* skipped = skip_counter(ws, d_num_skipped);
    B200_TRY(cudaMemsetAsync(skipped, 0, sizeof(unsigned long long), st));
    ws->last_launches = 0;
    if (n == 0) return OSKAR_B200_OK;
    const WeightConsts c = make_consts(data_is_double, cell_size_rad,
                                       grid_size, frequency_hz);
    const int blocks = launch_blocks(ws, n);
    if (data_is_double)
        weights_read_kernel<double><<<blocks, 256, 0, st>>>(
            n, (const double*)uu, (const double*)vv,
            (const double*)weight_in, (double*)weight_out, c,
            (const double*)grid, skipped);
    else
        weights_read_kernel<float><<<blocks, 256, 0, st>>>(
            n, (const float*)uu, (const float*)vv, (const float*)weight_in,
            (float*)weight_out, c, (const float*)grid, skipped);
    B200_TRY(cudaGetLastError());
    ws->last_launches = 1;
    return OSKAR_B200_OK;
}

}  // namespace b200
