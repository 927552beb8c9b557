// Per-visibility preparation of a batch of jobs: placement (grid cell,
// w-plane, oversample offsets, conjugation, skip test) exactly as
// oskar_grid_wproj.c:70-101 computes it, the sort key, the skip counts, the
// norms and the plane histograms; then, after the sort, the gridding work
// list (tasks).
#include <algorithm>

#include "common.cuh"
#include "internal.h"
#include "prep.cuh"

namespace b200 {

// Sort key bits (skip flag included) that the fine cell index may fill.
// Coarser fine cells sort faster but grid slower: at plain_large, 24 bits
// (three 8-bit passes) gave sort 2.17 -> 1.47 ms, gridding 20.3 -> 22.2 ms.
constexpr int kKeyBits = 32;

bool make_key_layout(int grid_size, int num_planes, int num_jobs,
                     KeyLayout* out, int tile_shift)
{
    KeyLayout k{};
    int gbits = 0;
    while ((1 << gbits) < grid_size) ++gbits;
    // Coarse tiles: at most 16 per axis and at least 64 cells wide, so the
    // visibilities in flight at any time touch a few coarse tiles of grid
    // (or the width asked for, within 64 cells and the grid).
    k.coarse_shift = gbits - 4 > 6 ? gbits - 4 : 6;
    if (tile_shift > 0)
        k.coarse_shift = std::max(6, std::min(tile_shift, std::max(gbits, 6)));
    const int ctiles = (grid_size + (1 << k.coarse_shift) - 1) >> k.coarse_shift;
    while ((1 << k.coarse_bits) < ctiles) ++k.coarse_bits;
    while ((1 << k.plane_bits) < num_planes) ++k.plane_bits;
    while ((1 << k.job_bits) < num_jobs) ++k.job_bits;
    k.fine_shift = 0;
    k.fine_bits = k.coarse_shift;
    const int fixed = k.job_bits + 2 * k.coarse_bits + k.plane_bits + 1;
    if (fixed > 32) return false;
    while (fixed + 2 * k.fine_bits > kKeyBits && k.fine_bits > 0)
    {
        ++k.fine_shift;
        --k.fine_bits;
    }
    k.job_shift = 2 * k.coarse_bits + k.plane_bits + 2 * k.fine_bits;
    k.total_bits = k.job_shift + k.job_bits;
    *out = k;
    return true;
}

int prep_blocks_per_job(size_t max_points, int num_jobs, int num_sms)
{
    const size_t need = (max_points + 255) / 256;
    size_t want = (size_t)num_sms * 8 / (size_t)(num_jobs > 0 ? num_jobs : 1);
    if (want < 1) want = 1;
    if (want > need) want = need > 0 ? need : 1;
    return (int)want;
}

namespace {

constexpr int kPrepThreads = 256;
constexpr int kMaxSmemPlanes = 4096;

// Spreads the low 16 bits of x to the even bit positions.
__device__ __forceinline__ uint32_t spread_bits(uint32_t x)
{
    x &= 0xffffu;
    x = (x | (x << 8)) & 0x00ff00ffu;
    x = (x | (x << 4)) & 0x0f0f0f0fu;
    x = (x | (x << 2)) & 0x33333333u;
    x = (x | (x << 1)) & 0x55555555u;
    return x;
}

__device__ __forceinline__ uint32_t make_key(const KeyLayout& k, int job,
                                             int gu, int gv, int plane)
{
    const uint32_t cu = (uint32_t)gu >> k.coarse_shift;
    const uint32_t cv = (uint32_t)gv >> k.coarse_shift;
    const uint32_t in_mask = (1u << k.coarse_shift) - 1u;
    const uint32_t fu = ((uint32_t)gu & in_mask) >> k.fine_shift;
    const uint32_t fv = ((uint32_t)gv & in_mask) >> k.fine_shift;
    // Coarse tiles in row-major order: tasks of one row of tiles are
    // contiguous, so a band of grid rows is complete once its tasks and its
    // neighbours' are (the drop-in streams such bands back to the host).
    const uint32_t coarse = (cv << k.coarse_bits) | cu;
    const uint32_t fine = spread_bits(fu) | (spread_bits(fv) << 1);
    return ((uint32_t)job << k.job_shift) |
           (coarse << (k.plane_bits + 2 * k.fine_bits)) |
           ((uint32_t)plane << (2 * k.fine_bits)) | fine;
}

__device__ __forceinline__ PlaceConsts place_consts(const JobDesc& jd)
{
    PlaceConsts pc;
    pc.grid_scale = jd.grid_scale;
    pc.w_scale = jd.w_scale;
    pc.grid_scale_f = jd.grid_scale_f;
    pc.w_scale_f = jd.w_scale_f;
    pc.grid_size = jd.grid_size;
    pc.centre = jd.grid_size / 2;
    pc.num_planes = jd.num_planes;
    pc.oversample = jd.oversample;
    return pc;
}

template <typename T, int MODE>
__global__ void __launch_bounds__(kPrepThreads)
prep_kernel(const PrepArgs a)
{
    const int job = blockIdx.y;
    const JobDesc& jd = a.jobs[job];
    const T* __restrict__ uu = static_cast<const T*>(jd.uu);
    const T* __restrict__ vv = static_cast<const T*>(jd.vv);
    const T* __restrict__ ww = static_cast<const T*>(jd.ww);
    const T* __restrict__ wt = static_cast<const T*>(jd.weight);
    const PlaceConsts pc = place_consts(jd);
    const int num_planes = jd.num_planes, half = jd.half;
    const unsigned long long first = jd.first, n = jd.n;
    __shared__ unsigned s_hist[kMaxSmemPlanes];
    __shared__ double s_norm[kPrepThreads / 32];
    __shared__ unsigned s_skip[kPrepThreads / 32];
    const bool smem_hist = num_planes <= kMaxSmemPlanes;
    if (smem_hist)
        for (int p = threadIdx.x; p < num_planes; p += blockDim.x)
            s_hist[p] = 0;
    __syncthreads();

    const int span = 2 * half + 1;
    const uint32_t skip_key = 1u << a.key.total_bits;
    const int lane = threadIdx.x & 31;
    unsigned long long* job_hist = a.plane_counts + (size_t)job * a.max_planes;
    double norm = 0.0;
    unsigned skipped = 0;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t base = (size_t)blockIdx.x * blockDim.x; base < n;
         base += stride)
    {
        const size_t i = base + threadIdx.x;
        const bool in_range = i < n;
        const size_t g = first + i;
        Placed p{};
        if (in_range)
            p = place_one<T, MODE>(scale_coord(uu[i], jd),
                                   scale_coord(vv[i], jd),
                                   scale_coord(ww[i], jd), pc, jd.support);
        const bool keep = in_range && !p.skipped;
        if (in_range)
        {
            if (keep)
            {
                a.rec[g] = make_int4(p.gu, p.gv,
                                     p.plane | (p.conj < 0 ? (int)0x80000000 : 0),
                                     (p.off_u + half) | ((p.off_v + half) << 16));
                a.keys[g] = make_key(a.key, job, p.gu, p.gv, p.plane);
                double s = jd.norm_table[((size_t)p.plane * span +
                                          (p.off_v + half)) * span +
                                         (p.off_u + half)];
                if (a.apply_weight) s *= (double)wt[i];
                norm += s;
            }
            else
            {
                a.keys[g] = skip_key;
            }
            a.vals[g] = (uint32_t)g;
        }
        skipped += in_range && !keep;
        // plane histogram, aggregated across equal planes in the warp
        const unsigned pl = keep ? (unsigned)p.plane : 0xffffffffu;
        const unsigned peers = __match_any_sync(0xffffffffu, pl);
        if (keep && lane == __ffs(peers) - 1)
        {
            if (smem_hist) atomicAdd(&s_hist[pl], (unsigned)__popc(peers));
            else atomicAdd(&job_hist[pl], (unsigned long long)__popc(peers));
        }
    }
    norm = warp_sum(norm);
    skipped = warp_sum(skipped);
    if (lane == 0)
    {
        s_norm[threadIdx.x >> 5] = norm;
        s_skip[threadIdx.x >> 5] = skipped;
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        double t = 0.0;
        unsigned long long k = 0;
        for (int w = 0; w < kPrepThreads / 32; ++w)
        {
            t += s_norm[w];
            k += s_skip[w];
        }
        a.norm_partials[(size_t)job * gridDim.x + blockIdx.x] = t;
        if (k)
        {
            atomicAdd(&a.job_skipped[job], k);
            atomicAdd(&a.counters[CNT_SKIPPED], k);
        }
    }
    if (smem_hist)
        for (int p = threadIdx.x; p < num_planes; p += blockDim.x)
            if (s_hist[p])
                atomicAdd(&job_hist[p], (unsigned long long)s_hist[p]);
}

// One block per job: sums the job's norm partials in a fixed order
// (deterministic), adds them to the caller's norm, publishes the skip count,
// and counts grid updates from the plane histogram.
__global__ void finalize_prep_kernel(const PrepArgs a)
{
    const int job = blockIdx.x;
    const JobDesc& jd = a.jobs[job];
    __shared__ double s_v[32];
    __shared__ unsigned long long s_u[32];
    double t = 0.0;
    for (int i = threadIdx.x; i < a.blocks_per_job; i += blockDim.x)
        t += a.norm_partials[(size_t)job * a.blocks_per_job + i];
    unsigned long long up = 0;
    const unsigned long long* hist = a.plane_counts + (size_t)job * a.max_planes;
    for (int p = threadIdx.x; p < jd.num_planes; p += blockDim.x)
    {
        const unsigned long long w = 2ull * jd.support[p] + 1ull;
        up += hist[p] * w * w;
    }
    t = warp_sum(t);
    up = warp_sum(up);
    if ((threadIdx.x & 31) == 0)
    {
        s_v[threadIdx.x >> 5] = t;
        s_u[threadIdx.x >> 5] = up;
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        double s = 0.0;
        unsigned long long u = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
        {
            s += s_v[w];
            u += s_u[w];
        }
        if (jd.d_norm) *jd.d_norm += s;
        if (jd.d_skipped) *jd.d_skipped = a.job_skipped[job];
        atomicAdd(&a.counters[CNT_UPDATES], u);
    }
}

// Task list in two passes over the sorted keys, tiles of kTaskTile
// positions: each tile counts its task starts, the tile counts are scanned,
// and each tile writes its starts at its offset.  A task starts at sorted
// position s < valid when s == 0, s % task_max == 0, or the key above the
// fine cell bits changes.
constexpr int kTaskTile = 4096;
constexpr int kTaskThreads = 256;

__device__ __forceinline__ bool task_starts_at(const uint32_t* keys, size_t s,
                                               size_t valid, int fine_bits,
                                               int task_max)
{
    return s < valid &&
           (s == 0 || s % (size_t)task_max == 0 ||
            (keys[s] >> fine_bits) != (keys[s - 1] >> fine_bits));
}

__global__ void __launch_bounds__(kTaskThreads)
task_count_kernel(const uint32_t* __restrict__ keys, size_t n,
                  const unsigned long long* __restrict__ counters,
                  int fine_key_bits, int task_max,
                  uint32_t* __restrict__ tile_counts)
{
    const size_t valid = n - counters[CNT_SKIPPED];
    const size_t tile0 = (size_t)blockIdx.x * kTaskTile;
    unsigned c = 0;
    for (int k = threadIdx.x; k < kTaskTile; k += kTaskThreads)
        c += task_starts_at(keys, tile0 + k, valid, fine_key_bits, task_max);
    c = warp_sum(c);
    __shared__ unsigned s_w[kTaskThreads / 32];
    if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0)
    {
        unsigned t = 0;
        for (int w = 0; w < kTaskThreads / 32; ++w) t += s_w[w];
        tile_counts[blockIdx.x] = t;
    }
}

// tile_offsets: exclusive scan of tile_counts (the last tile also needs its
// own count to close the list).
__global__ void __launch_bounds__(kTaskThreads)
task_write_kernel(const uint32_t* __restrict__ keys, size_t n,
                  unsigned long long* __restrict__ counters,
                  int fine_key_bits, int task_max, int job_shift,
                  const uint32_t* __restrict__ tile_counts,
                  const uint32_t* __restrict__ tile_offsets,
                  uint32_t* __restrict__ task_start,
                  uint32_t* __restrict__ task_job)
{
    const size_t valid = n - counters[CNT_SKIPPED];
    const size_t tile0 = (size_t)blockIdx.x * kTaskTile;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __shared__ unsigned s_w[kTaskThreads / 32];
    uint32_t base = tile_offsets[blockIdx.x];
    // rounds of kTaskThreads consecutive positions, in order
    for (int r = 0; r < kTaskTile; r += kTaskThreads)
    {
        const size_t pos = tile0 + r + threadIdx.x;
        const bool f = task_starts_at(keys, pos, valid, fine_key_bits,
                                      task_max);
        const unsigned ball = __ballot_sync(0xffffffffu, f);
        if (lane == 0) s_w[warp] = __popc(ball);
        __syncthreads();
        unsigned before = 0, total = 0;
#pragma unroll
        for (int w = 0; w < kTaskThreads / 32; ++w)
        {
            before += w < warp ? s_w[w] : 0u;
            total += s_w[w];
        }
        if (f)
        {
            const uint32_t t = base + before +
                               __popc(ball & ((1u << lane) - 1u));
            task_start[t] = (uint32_t)pos;
            task_job[t] = keys[pos] >> job_shift;
        }
        base += total;
        __syncthreads();   // s_w is rewritten by the next round
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0)
    {
        const uint32_t num_tasks = tile_offsets[blockIdx.x] +
                                   tile_counts[blockIdx.x];
        counters[CNT_TASKS] = num_tasks;
        task_start[num_tasks] = (uint32_t)valid;
    }
}

// Placement only, for inspection (oskar_b200_place).
template <typename T, int MODE>
__global__ void place_kernel(const T* __restrict__ uu, const T* __restrict__ vv,
                             const T* __restrict__ ww, size_t n,
                             PlaceConsts pc, const int* __restrict__ support,
                             int32_t* gu, int32_t* gv, int32_t* plane,
                             int32_t* off_u, int32_t* off_v, int32_t* conj,
                             int32_t* skipped)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
    {
        const Placed p = place_one<T, MODE>(uu[i], vv[i], ww[i], pc, support);
        if (gu) gu[i] = p.gu_report;
        if (gv) gv[i] = p.gv_report;
        if (plane) plane[i] = p.plane;
        if (off_u) off_u[i] = p.off_u;
        if (off_v) off_v[i] = p.off_v;
        if (conj) conj[i] = p.conj;
        if (skipped) skipped[i] = p.skipped;
    }
}

unsigned grid_blocks(size_t n, int num_sms, int per_sm, int threads)
{
    const size_t need = (n + threads - 1) / threads;
    const size_t cap = (size_t)num_sms * per_sm;
    return (unsigned)(need < cap ? (need > 0 ? need : 1) : cap);
}

}  // namespace

cudaError_t launch_prep(const PrepArgs& a, int data_is_double, int coord_mode,
                        cudaStream_t st)
{
    const dim3 grid(a.blocks_per_job, a.num_jobs);
    if (data_is_double)
        prep_kernel<double, COORD_F64><<<grid, kPrepThreads, 0, st>>>(a);
    else if (coord_mode == OSKAR_B200_COORDS_REFERENCE_F32)
        prep_kernel<float, COORD_REF_F32><<<grid, kPrepThreads, 0, st>>>(a);
    else
        prep_kernel<float, COORD_F64><<<grid, kPrepThreads, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_finalize_prep(const PrepArgs& a, cudaStream_t st)
{
    finalize_prep_kernel<<<a.num_jobs, 256, 0, st>>>(a);
    return cudaGetLastError();
}

size_t task_tiles(size_t n) { return (n + kTaskTile - 1) / kTaskTile; }

cudaError_t launch_tasks(const uint32_t* sorted_keys, size_t n,
                         unsigned long long* counters, int fine_key_bits,
                         int job_shift, int task_max, uint32_t* tile_counts,
                         void* scan_tmp, uint32_t* task_start,
                         uint32_t* task_job, cudaStream_t st, int* launches)
{
    const size_t tiles = task_tiles(n);
    if (tiles == 0) return cudaSuccess;
    uint32_t* tile_offsets = tile_counts + tiles;
    task_count_kernel<<<(unsigned)tiles, kTaskThreads, 0, st>>>(
        sorted_keys, n, counters, fine_key_bits, task_max, tile_counts);
    cudaError_t e = exclusive_scan_u32(tile_counts, tile_offsets, tiles,
                                       scan_tmp, st, launches);
    if (e != cudaSuccess) return e;
    if (launches) *launches += 2;
    task_write_kernel<<<(unsigned)tiles, kTaskThreads, 0, st>>>(
        sorted_keys, n, counters, fine_key_bits, task_max, job_shift,
        tile_counts, tile_offsets, task_start, task_job);
    return cudaGetLastError();
}

namespace {

__device__ __forceinline__ int band_of_task(const uint32_t* keys,
                                            const uint32_t* task_start,
                                            unsigned t, int band_shift,
                                            uint32_t band_mask)
{
    return (int)((keys[task_start[t]] >> band_shift) & band_mask);
}

// band_first[b] = first task whose band is >= b, for b in [0, num_bands];
// tasks are in key order, so bands are non-decreasing along the list.
__global__ void band_first_kernel(const uint32_t* __restrict__ sorted_keys,
                                  const uint32_t* __restrict__ task_start,
                                  const unsigned long long* __restrict__ counters,
                                  int band_shift, uint32_t band_mask,
                                  int num_bands, uint32_t* __restrict__ band_first)
{
    const unsigned nt = (unsigned)counters[CNT_TASKS];
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t <= nt;
         t += (size_t)gridDim.x * blockDim.x)
    {
        int b = t < nt ? band_of_task(sorted_keys, task_start, (unsigned)t,
                                      band_shift, band_mask)
                       : num_bands;
        b = b < num_bands ? b : num_bands;
        int prev = t > 0 ? band_of_task(sorted_keys, task_start,
                                        (unsigned)t - 1, band_shift, band_mask)
                         : -1;
        prev = prev < num_bands ? prev : num_bands;
        for (int c = prev + 1; c <= b; ++c) band_first[c] = (uint32_t)t;
    }
}

}  // namespace

cudaError_t launch_band_first(const uint32_t* sorted_keys,
                              const uint32_t* task_start, size_t n,
                              const unsigned long long* counters,
                              const KeyLayout& kl, int num_bands,
                              uint32_t* band_first, int num_sms,
                              cudaStream_t st)
{
    const int shift = kl.plane_bits + 2 * kl.fine_bits + kl.coarse_bits;
    const uint32_t mask = (1u << kl.coarse_bits) - 1u;
    const unsigned blocks = grid_blocks(n + 1, num_sms, 8, 256);
    band_first_kernel<<<blocks, 256, 0, st>>>(sorted_keys, task_start,
                                              counters, shift, mask, num_bands,
                                              band_first);
    return cudaGetLastError();
}

cudaError_t launch_place(int data_is_double, int coord_mode, const void* uu,
                         const void* vv, const void* ww, size_t n,
                         const PlaceConsts& pc, const int* support,
                         int32_t* gu, int32_t* gv, int32_t* plane,
                         int32_t* off_u, int32_t* off_v, int32_t* conj,
                         int32_t* skipped, int num_sms, cudaStream_t st)
{
    const unsigned blocks = grid_blocks(n, num_sms, 8, 256);
    if (data_is_double)
        place_kernel<double, COORD_F64><<<blocks, 256, 0, st>>>(
            static_cast<const double*>(uu), static_cast<const double*>(vv),
            static_cast<const double*>(ww), n, pc, support, gu, gv, plane,
            off_u, off_v, conj, skipped);
    else if (coord_mode == OSKAR_B200_COORDS_REFERENCE_F32)
        place_kernel<float, COORD_REF_F32><<<blocks, 256, 0, st>>>(
            static_cast<const float*>(uu), static_cast<const float*>(vv),
            static_cast<const float*>(ww), n, pc, support, gu, gv, plane,
            off_u, off_v, conj, skipped);
    else
        place_kernel<float, COORD_F64><<<blocks, 256, 0, st>>>(
            static_cast<const float*>(uu), static_cast<const float*>(vv),
            static_cast<const float*>(ww), n, pc, support, gu, gv, plane,
            off_u, off_v, conj, skipped);
    return cudaGetLastError();
}

}  // namespace b200
