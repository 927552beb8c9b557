// Romein-style W-projection scatter kernel for sm_100a.
//
// Work arrives as tasks: runs of <= kTaskMax sorted visibilities that share
// a w-plane (hence a support S and footprint width W = 2S+1) and a coarse
// grid tile.  A persistent CTA pulls tasks from a device work queue.  For a
// task it
//   1. stages the plane's re-laid kernel slab into shared memory with one
//      TMA bulk copy (cp.async.bulk + mbarrier), skipped when the previous
//      task of this CTA used the same plane,
//   2. turns each visibility into a small tap record in shared memory,
//   3. lets each thread own "classes" (a, b) in [0, W)^2: for every
//      visibility, the class's grid point is the unique footprint cell
//      (u, v) with u = a (mod W) and v = b (mod W).  Consecutive (spatially
//      sorted) visibilities mostly map a class to the same cell, so the
//      thread accumulates vis * kernel in registers and issues one atomic
//      (red.global.add.v2.f32, or two red.f64) only when its cell changes.
// Each grid cell receives exactly the reference's terms
//   grid[v][u] += vis * (conj ? conj(K) : K)(|off_v + j*os|, |off_u + k*os|)
// (oskar_grid_wproj.c:104-123), summed in a different order.
#include <algorithm>

#include "common.cuh"
#include "grid_romein.cuh"
#include "internal.h"

namespace b200 {
namespace {

template <typename GT> struct Vec2;
template <> struct Vec2<float> { using type = float2; };
template <> struct Vec2<double> { using type = double2; };

// Per-visibility tap record.  For a class (a, b) of a task with footprint W:
//   ru = (a + mu) mod W, rv = (b + mv) mod W   (offsets inside the footprint)
//   column = ru >= tu ? cp + ru : cn - ru      (slab position, see PlaneDesc)
//   rowoff = rv >= tv ? rp + rv * pitch : rn - rv * pitch
//   cell   = origin + ru + rv * grid_size
template <typename GT>
struct __align__(16) TapVis
{
    unsigned origin;
    int mu, mv, tuv;   // tuv = tu | tv << 16
    int cp, cn, rp, rn;
    GT ar, ai, bi, br; // re += ar*Kre - ai*Kim; im += bi*Kre + br*Kim
};

template <typename GT>
__device__ __forceinline__ TapVis<GT> derive(const int4 rec,
                                             const typename Vec2<GT>::type vis,
                                             const PlaneDesc& d, int grid_size,
                                             int oversample, int half)
{
    TapVis<GT> t;
    const int s = d.support, w = 2 * s + 1, os = oversample;
    const int conj = rec.z < 0 ? -1 : 1;
    // Offsets lie in [-half, half] by construction; the clamp only guards
    // the slab bounds against a corrupted record.
    const int off_u = min(max((rec.w & 0xffff) - half, -half), half);
    const int off_v = min(max((rec.w >> 16) - half, -half), half);
    const int u0 = rec.x - s, v0 = rec.y - s;
    t.origin = (unsigned)u0 + (unsigned)v0 * (unsigned)grid_size;
    t.mu = (w - u0 % w) % w;
    t.mv = (w - v0 % w) % w;
    // Taps k >= k0 have off + k*os >= 0 (the ascending run of positions).
    const int tu = s + (off_u < 0 ? 1 : 0);
    const int tv = s + (off_v < 0 ? 1 : 0);
    t.tuv = tu | (tv << 16);
    const int rpu = ((off_u % os) + os) % os, rnu = ((-off_u % os) + os) % os;
    const int rpv = ((off_v % os) + os) % os, rnv = ((-off_v % os) + os) % os;
    t.cp = rpu * d.L + (off_u - rpu) / os - s;
    t.cn = rnu * d.L + (-off_u - rnu) / os + s;
    t.rp = (rpv * d.L + (off_v - rpv) / os - s) * d.pitch;
    t.rn = (rnv * d.L + (-off_v - rnv) / os + s) * d.pitch;
    const GT sc = (GT)d.scale;
    const GT vr = vis.x * sc, vi = vis.y * sc;
    t.ar = vr;
    t.ai = conj * vi;
    t.bi = vi;
    t.br = conj * vr;
    return t;
}

template <typename GT>
__device__ __forceinline__ void flush(GT* grid, unsigned cell, unsigned cells,
                                      GT re, GT im, unsigned long long* status)
{
    if (cell < cells)
        red_add_c(grid + 2 * (size_t)cell, re, im);
    else
        atomicOr(status, (unsigned long long)DEV_ERR_GRID_INDEX);
}

// One task: every class of the W x W footprint over the task's visibilities.
template <typename GT, typename KT, int CPT>
__device__ __forceinline__ void process_task(const TapVis<GT>* __restrict__ s_vis,
                                             int m, int w, int pitch,
                                             const KT* __restrict__ slab,
                                             GT* __restrict__ grid,
                                             int grid_size, unsigned cells,
                                             unsigned long long* status,
                                             unsigned& flushes)
{
    const int classes = w * w;
    const int tps = min(kGridThreads, (classes + CPT - 1) / CPT);
    int slices = kGridThreads / tps;
    if (slices > m) slices = m;
    const int r = threadIdx.x / tps, l = threadIdx.x - r * tps;
    if (r >= slices) return;
    const int i0 = (r * m) / slices, i1 = ((r + 1) * m) / slices;
    const int per_pass = tps * CPT;
    for (int base = 0; base < classes; base += per_pass)
    {
        int ca[CPT], cb[CPT];
        bool act[CPT];
        GT are[CPT], aim[CPT];
        unsigned cur[CPT];
#pragma unroll
        for (int q = 0; q < CPT; ++q)
        {
            const int c = base + q * tps + l;
            act[q] = c < classes;
            const int cc = act[q] ? c : 0;
            cb[q] = cc / w;
            ca[q] = cc - cb[q] * w;
            are[q] = aim[q] = GT(0);
            cur[q] = 0xffffffffu;
        }
        for (int i = i0; i < i1; ++i)
        {
            const TapVis<GT> v = s_vis[i];
            const int tu = v.tuv & 0xffff, tv = v.tuv >> 16;
#pragma unroll
            for (int q = 0; q < CPT; ++q)
            {
                if (!act[q]) continue;
                int ru = ca[q] + v.mu;
                ru = ru >= w ? ru - w : ru;
                int rv = cb[q] + v.mv;
                rv = rv >= w ? rv - w : rv;
                const int col = ru >= tu ? v.cp + ru : v.cn - ru;
                const int roff = rv >= tv ? v.rp + rv * pitch : v.rn - rv * pitch;
                const auto k = KernelLoad<KT>::get(slab[roff + col]);
                const unsigned cell = v.origin + (unsigned)ru +
                                      (unsigned)rv * (unsigned)grid_size;
                if (cell != cur[q])
                {
                    if (cur[q] != 0xffffffffu)
                    {
                        flush(grid, cur[q], cells, are[q], aim[q], status);
                        ++flushes;
                    }
                    are[q] = aim[q] = GT(0);
                    cur[q] = cell;
                }
                are[q] = fma(v.ar, (GT)k.x, are[q]);
                are[q] = fma(-v.ai, (GT)k.y, are[q]);
                aim[q] = fma(v.bi, (GT)k.x, aim[q]);
                aim[q] = fma(v.br, (GT)k.y, aim[q]);
            }
        }
#pragma unroll
        for (int q = 0; q < CPT; ++q)
            if (act[q] && cur[q] != 0xffffffffu)
            {
                flush(grid, cur[q], cells, are[q], aim[q], status);
                ++flushes;
            }
    }
}

template <typename GT, typename KT, bool STAGED>
__global__ void __launch_bounds__(kGridThreads)
romein_grid_kernel(const GridArgs a)
{
    using V2 = typename Vec2<GT>::type;
    extern __shared__ __align__(128) unsigned char smem[];
    KT* s_slab = reinterpret_cast<KT*>(smem);
    TapVis<GT>* s_vis = reinterpret_cast<TapVis<GT>*>(
        smem + (STAGED ? a.slab_smem_bytes : 0));
    __shared__ uint64_t s_bar;
    __shared__ unsigned s_task;

    const V2* __restrict__ svis = static_cast<const V2*>(a.svis);
    const KT* __restrict__ slabs = static_cast<const KT*>(a.slabs);
    GT* __restrict__ grid = static_cast<GT*>(a.grid);
    unsigned long long* status = &a.counters[CNT_STATUS];
    const unsigned num_tasks = (unsigned)a.counters[CNT_TASKS];
    const unsigned cells = (unsigned)a.grid_size * (unsigned)a.grid_size;

    if (STAGED && threadIdx.x == 0)
    {
        mbar_init(&s_bar, 1);
        mbar_fence_init();
    }
    __syncthreads();

    uint32_t phase = 0;
    int cur_plane = -1;
    unsigned flushes = 0;
    for (;;)
    {
        if (threadIdx.x == 0)
            s_task = (unsigned)atomicAdd(&a.counters[CNT_TASK_NEXT], 1ull);
        // Also: every thread has finished with the previous task's records
        // and slab before they are overwritten below.
        __syncthreads();
        const unsigned task = s_task;
        if (task >= num_tasks) break;
        const uint32_t begin = a.task_start[task];
        const int m = (int)(a.task_start[task + 1] - begin);
        if (m <= 0 || m > kTaskMax)
        {
            if (threadIdx.x == 0)
                atomicOr(status, (unsigned long long)DEV_ERR_TASK);
            continue;
        }
        const int plane = a.srec[begin].z & 0x7fffffff;
        const PlaneDesc d = a.planes[plane];
        const bool load = STAGED && plane != cur_plane;
        if (load && threadIdx.x == 0)
        {
            fence_proxy_async_shared();
            mbar_arrive_expect_tx(&s_bar, d.bytes);
            const unsigned char* src =
                reinterpret_cast<const unsigned char*>(slabs + d.offset);
            for (unsigned off = 0; off < d.bytes; off += kBulkChunk)
                bulk_copy_g2s(smem + off, src + off,
                              min(kBulkChunk, d.bytes - off), &s_bar);
        }
        for (int i = threadIdx.x; i < m; i += kGridThreads)
            s_vis[i] = derive<GT>(a.srec[begin + i], svis[begin + i], d,
                                  a.grid_size, a.oversample, a.half);
        if (load)
        {
            const bool ok = mbar_wait_bounded(&s_bar, phase);
            if (!__syncthreads_and(ok))
            {
                // Record the failure, let the copy drain (bounded), leave.
                if (threadIdx.x == 0)
                    atomicOr(status, (unsigned long long)DEV_ERR_TIMEOUT);
                mbar_wait_bounded(&s_bar, phase);
                return;
            }
            phase ^= 1u;
            cur_plane = plane;
        }
        else
        {
            __syncthreads();
        }
        const KT* slab = STAGED ? s_slab : slabs + d.offset;
        const int w = 2 * d.support + 1;
        const int cpt = d.support < kTuneMax ? a.cpt[d.support] : 4;
        if (cpt == 1)
            process_task<GT, KT, 1>(s_vis, m, w, d.pitch, slab, grid,
                                    a.grid_size, cells, status, flushes);
        else if (cpt == 2)
            process_task<GT, KT, 2>(s_vis, m, w, d.pitch, slab, grid,
                                    a.grid_size, cells, status, flushes);
        else
            process_task<GT, KT, 4>(s_vis, m, w, d.pitch, slab, grid,
                                    a.grid_size, cells, status, flushes);
    }
    const unsigned long long f = warp_sum((unsigned long long)flushes);
    if ((threadIdx.x & 31) == 0 && f)
        atomicAdd(&a.counters[CNT_FLUSHES], f);
}

template <typename GT, typename KT, bool STAGED>
cudaError_t launch_variant(const GridArgs& a, int num_sms, size_t smem,
                           cudaStream_t st, int* ctas_out)
{
    auto fn = romein_grid_kernel<GT, KT, STAGED>;
    cudaError_t e = cudaFuncSetAttribute(
        fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn,
                                                      kGridThreads, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    const int ctas = num_sms * per_sm;
    if (ctas_out) *ctas_out = ctas;
    fn<<<ctas, kGridThreads, smem, st>>>(a);
    return cudaGetLastError();
}

}  // namespace

// Classes-per-thread for each support: the choice that keeps the most
// thread slots busy (W^2 classes over 256 threads, sliced over the task's
// visibilities when W^2 is small), preferring more classes per thread on
// ties for the extra independent work per tap record.
void default_tune_table(unsigned char* cpt)
{
    for (int s = 0; s < kTuneMax; ++s)
    {
        const int classes = (2 * s + 1) * (2 * s + 1);
        double best = -1.0;
        int pick = 1;
        for (int c : {1, 2, 4})
        {
            const int tps = std::min(kGridThreads, (classes + c - 1) / c);
            const int slices = kGridThreads / tps;
            const int passes = (classes + tps * c - 1) / (tps * c);
            const double util = (double)classes * slices /
                                ((double)kGridThreads * c * passes);
            if (util >= best - 1e-9)
            {
                best = util;
                pick = c;
            }
        }
        cpt[s] = (unsigned char)pick;
    }
}

size_t grid_smem_bytes(const oskar_B200Cube* cube, bool staged)
{
    const size_t rec = cube->data_is_double ? sizeof(TapVis<double>)
                                            : sizeof(TapVis<float>);
    const size_t slab = staged ? ((cube->max_slab_bytes + 127) / 128) * 128 : 0;
    return slab + rec * kTaskMax;
}

cudaError_t launch_grid(const GridArgs& a, const oskar_B200Cube* cube,
                        bool staged, int num_sms, cudaStream_t st,
                        int* ctas_out)
{
    const size_t smem = grid_smem_bytes(cube, staged);
    GridArgs args = a;
    args.slab_smem_bytes = staged ? (unsigned)(((cube->max_slab_bytes + 127) /
                                                128) * 128)
                                  : 0u;
    if (cube->data_is_double)
    {
        if (cube->kernel_type != OSKAR_B200_KERNEL_NATIVE)
            return cudaErrorInvalidValue;
        return staged ? launch_variant<double, double2, true>(args, num_sms, smem, st, ctas_out)
                      : launch_variant<double, double2, false>(args, num_sms, smem, st, ctas_out);
    }
    switch (cube->kernel_type)
    {
    case OSKAR_B200_KERNEL_F16:
        return staged ? launch_variant<float, __half2, true>(args, num_sms, smem, st, ctas_out)
                      : launch_variant<float, __half2, false>(args, num_sms, smem, st, ctas_out);
    case OSKAR_B200_KERNEL_BF16:
        return staged ? launch_variant<float, __nv_bfloat162, true>(args, num_sms, smem, st, ctas_out)
                      : launch_variant<float, __nv_bfloat162, false>(args, num_sms, smem, st, ctas_out);
    default:
        return staged ? launch_variant<float, float2, true>(args, num_sms, smem, st, ctas_out)
                      : launch_variant<float, float2, false>(args, num_sms, smem, st, ctas_out);
    }
}

}  // namespace b200
