// Romein-style W-projection scatter kernel for sm_100a.
//
// Work arrives as tasks: runs of <= kTaskMax sorted visibilities that share
// a w-plane (hence a support S and footprint width W = 2S+1) and a coarse
// grid tile.  A persistent CTA pulls tasks from a device work queue.  For a
// task it
//   0. gathers the task's placement records and visibilities through the
//      sort's index array (sorted position -> point),
//   1. orders the task's visibilities by cell (and kernel row offset) and
//      turns each into a small tap record in shared memory, merging records
//      whose taps are identical,
//   2. reads kernel values through L1 (default) or, with staging on, copies
//      the W-row block of each kernel row offset into shared memory with
//      TMA bulk copies (cp.async.bulk + mbarrier) before that offset's run,
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
#include <mutex>
#include <type_traits>

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
//   column = ru >= tu ? cp + ru : cn - ru      (slab column, see PlaneDesc)
//   kernel index = rowbase + column + rv * pitch
//   cell         = origin + ru + rv * grid_size
template <typename GT>
struct __align__(16) TapVis
{
    unsigned origin;
    int mu, mv, tu;
    int cp, cn, rowbase, unused;
    // re += c0.x * Kre + c1.x * Kim;  im += c0.y * Kre + c1.y * Kim
    typename Vec2<GT>::type c0, c1;
};

// A task's visibility as gathered from the caller's order: its placement
// record and its visibility (times its weight when asked for).  The task's
// raw records occupy the start of the tap-record array until derive() has
// read them.
template <typename GT>
struct __align__(16) RawVis
{
    int4 rec;
    typename Vec2<GT>::type vis;
};

// acc += c0 * k.x + c1 * k.y, component-wise, one rounding per product
// added (fma), in that order.  FP32: two packed fma.rn.f32x2 instead of
// four scalar fma, the same roundings.
__device__ __forceinline__ void cmac(float2& acc, const float2 c0,
                                     const float2 c1, const float2 k)
{
    acc = __ffma2_rn(c0, make_float2(k.x, k.x), acc);
    acc = __ffma2_rn(c1, make_float2(k.y, k.y), acc);
}

__device__ __forceinline__ void cmac(double2& acc, const double2 c0,
                                     const double2 c1, const double2 k)
{
    acc.x = fma(c0.x, k.x, acc.x);
    acc.x = fma(c1.x, k.y, acc.x);
    acc.y = fma(c0.y, k.x, acc.y);
    acc.y = fma(c1.y, k.y, acc.y);
}

template <typename GT>
__device__ __forceinline__ TapVis<GT> derive(const int4 rec,
                                             const typename Vec2<GT>::type vis,
                                             const PlaneDesc& d, int grid_size,
                                             int oversample, int half,
                                             unsigned long long* status)
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
    // Column taps k >= 0 (k >= 1 when off_u < 0) have off_u + k*os >= 0:
    // the ascending run of slab columns.
    t.tu = s + (off_u < 0 ? 1 : 0);
    const int rpu = ((off_u % os) + os) % os, rnu = ((-off_u % os) + os) % os;
    t.cp = rpu * d.L + (off_u - rpu) / os - s;
    t.cn = rnu * d.L + (-off_u - rnu) / os + s;
    // First of the W slab rows holding this row offset's taps.
    t.rowbase = (off_v + half) * w * d.pitch;
    t.unused = 0;
    GT sc = (GT)d.scale;
    // The prep kernel only keeps points whose footprint lies inside the
    // grid; a record that breaks this is reported and neutralised (zero
    // weight at cell 0) so no flush can leave the grid.
    if (u0 < 0 || v0 < 0 || u0 + w > grid_size || v0 + w > grid_size)
    {
        atomicOr(status, (unsigned long long)DEV_ERR_GRID_INDEX);
        t.origin = 0;
        t.mu = t.mv = 0;
        sc = GT(0);
    }
    const GT vr = vis.x * sc, vi = vis.y * sc;
    t.c0.x = vr;
    t.c0.y = vi;
    t.c1.x = -(conj * vi);
    t.c1.y = conj * vr;
    return t;
}

// Spreads the low 9 bits of x to the even bit positions.
__device__ __forceinline__ uint32_t spread9(uint32_t x)
{
    x &= 0x1ffu;
    x = (x | (x << 8)) & 0x00ff00ffu;
    x = (x | (x << 4)) & 0x0f0f0f0fu;
    x = (x | (x << 2)) & 0x33333333u;
    x = (x | (x << 1)) & 0x55555555u;
    return x;
}

// Layout of the in-task order key, most significant first:
//   row-offset major (staged kernel values: each row offset's run reads one
//   W-row block):  (off_v + H) | Morton(gu, gv) | (off_u + H) | index
//   cell major (kernel values through L1):  Morton(gu, gv) | (off_v + H) |
//   (off_u + H) | index.  Neighbouring visibilities then share most class
//   cells, which halves the grid atomics at plain_large (6.6e9 -> 3.4e9)
//   and is 1.7 % faster there than row-offset major.
// The offsets take `ob` bits each (the bit width of 2H, H = ceil(os / 2)),
// the index the low 8 bits, and the Morton code of the low `mb` (<= 9) bits
// of gu and gv what is left.  Records with identical taps are adjacent in
// either order.
struct TaskKey
{
    int ob, mb;
    bool cell_major;
    __device__ __forceinline__ TaskKey(int half, bool cell_major_order)
    {
        ob = 32 - __clz(2 * half);
        mb = min(9, (32 - 8 - 2 * ob) / 2);
        cell_major = cell_major_order;
    }
    __device__ __forceinline__ uint32_t make(const int4 r, unsigned t) const
    {
        const uint32_t mask = (1u << mb) - 1u;
        const uint32_t morton = spread9((uint32_t)r.x & mask) |
                                (spread9((uint32_t)r.y & mask) << 1);
        const uint32_t ov = (uint32_t)(r.w >> 16), ou = (uint32_t)(r.w & 0xffff);
        if (cell_major)
            return (morton << (8 + 2 * ob)) | (ov << (8 + ob)) | (ou << 8) | t;
        return (ov << (32 - ob)) | (morton << (8 + ob)) | (ou << 8) | t;
    }
    __device__ __forceinline__ int row_offset(uint32_t key) const
    {
        return (int)(key >> (32 - ob));
    }
};

// Returns, for thread t < m, the key of the t-th visibility of the task in
// TaskKey order; its low 8 bits are the task-relative index of that
// visibility.  Bitonic sort of one key
// per thread (m <= 256); strides below 32 use warp shuffles, larger ones go
// through shared memory.  All threads of the CTA must call it.
__device__ __forceinline__ uint32_t task_order(uint32_t key,
                                               uint32_t* s_order)
{
    static_assert(kTaskMax == kGridThreads, "one key per thread");
    const unsigned t = threadIdx.x;
#pragma unroll
    for (unsigned k = 2; k <= (unsigned)kGridThreads; k <<= 1)
    {
#pragma unroll
        for (unsigned j = k >> 1; j > 0; j >>= 1)
        {
            uint32_t other;
            if (j >= 32)
            {
                s_order[t] = key;
                __syncthreads();
                other = s_order[t ^ j];
                __syncthreads();
            }
            else
            {
                other = __shfl_xor_sync(0xffffffffu, key, j);
            }
            const bool ascending = (t & k) == 0;
            const bool take_min = ((t & j) == 0) == ascending;
            key = take_min ? min(key, other) : max(key, other);
        }
    }
    return key;
}

// Two records that read the same kernel values into the same cells.  Their
// contributions are vis_a * Kt + vis_b * Kt = (vis_a + vis_b) * Kt: the tap
// coefficients (which fold in the conjugation) can simply be added.
template <typename GT>
__device__ __forceinline__ bool same_taps(const TapVis<GT>& a,
                                          const TapVis<GT>& b)
{
    return a.origin == b.origin && a.mu == b.mu && a.mv == b.mv &&
           a.tu == b.tu && a.cp == b.cp && a.cn == b.cn &&
           a.rowbase == b.rowbase;
}

// Predicated complex flush: one vector reduction when `pred` holds, no
// branch (the flush decision differs from lane to lane on most taps).
__device__ __forceinline__ void red_add_c_if(bool pred, float* addr, float re,
                                             float im)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %3, 0;\n\t"
                 "@p red.relaxed.gpu.global.add.v2.f32 [%0], {%1, %2};\n\t}"
                 :: "l"(addr), "f"(re), "f"(im), "r"((int)pred) : "memory");
}

__device__ __forceinline__ void red_add_c_if(bool pred, double* addr,
                                             double re, double im)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %3, 0;\n\t"
                 "@p red.relaxed.gpu.global.add.f64 [%0], %1;\n\t"
                 "@p red.relaxed.gpu.global.add.f64 [%4], %2;\n\t}"
                 :: "l"(addr), "d"(re), "d"(im), "r"((int)pred), "l"(addr + 1)
                 : "memory");
}

// Thread layout of one task.  The W x W classes are split into W columns
// (a) and ceil(W / CPT) row groups of CPT consecutive rows; a work item is
// one (column, row group) pair, so the column arithmetic of a tap is done
// once per visibility and shared by the item's CPT classes, and the 32
// lanes of a warp hold consecutive columns (contiguous kernel reads,
// coalesced flushes).  The last row group of a column is moved up to rows
// W - CPT .. W - 1 and its first slots, which repeat rows of the group
// before, are masked, so every slot reads an in-bounds kernel row.  When
// the items fit the CTA several times, `slices` copies of the layout split
// the task's visibilities between them; otherwise the CTA's threads take
// the items in passes of kGridThreads.  Against one column per thread with
// rows strided by the number of threads per column (the thread count per
// column capped at 256 / W, so wide footprints left up to a third of the
// CTA idle in their last pass), the plain_large gridding kernel went from
// 15.3 to 14.4 ms: fewer idle thread slots, and no per-slot row registers.
struct TaskLayout
{
    int items, slices, per_slice;
};

template <int CPT>
__device__ __forceinline__ TaskLayout task_layout(int w)
{
    TaskLayout t;
    t.items = w * ((w + CPT - 1) / CPT);
    if (t.items <= kGridThreads)
    {
        t.slices = kGridThreads / t.items;
        t.per_slice = t.items;
    }
    else
    {
        t.slices = 1;
        t.per_slice = kGridThreads;
    }
    return t;
}

// Grid flush policies.  PlainFlush: one predicated vector reduction.
// CompensatedFlush (FP32): the addition returns the old value; Knuth's
// TwoSum recovers the exact rounding error of old + x (the atomic rounds to
// nearest even), which is added to a compensation grid folded into the grid
// at the end of the job.  Its branch is taken only when the lane flushes.
template <typename GT>
struct PlainFlush
{
    GT* grid;
    // FP32: the compare, the predicated reduction and the reset of the
    // running sum in one block of PTX.  When `valid` and cell != cur, the
    // sum goes to cur's grid cell and restarts from zero.
    __device__ __forceinline__ void flush_reset(int valid, unsigned cell,
                                                unsigned cur, float& ax,
                                                float& ay) const
    {
        asm volatile("{\n\t.reg .pred v, p;\n\t"
                     "setp.ne.s32 v, %5, 0;\n\t"
                     "setp.ne.and.u32 p, %2, %3, v;\n\t"
                     "@p red.relaxed.gpu.global.add.v2.f32 [%4], {%0, %1};\n\t"
                     "@p mov.f32 %0, 0f00000000;\n\t"
                     "@p mov.f32 %1, 0f00000000;\n\t}"
                     : "+f"(ax), "+f"(ay)
                     : "r"(cell), "r"(cur),
                       "l"(reinterpret_cast<float*>(grid) + 2 * (size_t)cur),
                       "r"(valid));
    }
    __device__ __forceinline__ void operator()(bool pred, unsigned cell, GT re,
                                               GT im) const
    {
        red_add_c_if(pred, grid + 2 * (size_t)cell, re, im);
    }
};

__device__ __forceinline__ float two_sum_err(float a, float b)
{
    const float s = __fadd_rn(a, b);
    const float bb = __fsub_rn(s, a);
    return __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
}

struct CompensatedFlush
{
    float* grid;
    float* comp;
    bool active;   // false: this task's cells are not compensated
    __device__ __forceinline__ void operator()(bool pred, unsigned cell,
                                               float re, float im) const
    {
        if (!active)
        {
            red_add_c_if(pred, grid + 2 * (size_t)cell, re, im);
            return;
        }
        if (!pred) return;
        float ore, oim;
        asm volatile("atom.relaxed.gpu.global.add.v2.f32 {%0, %1}, [%2], {%3, %4};"
                     : "=f"(ore), "=f"(oim)
                     : "l"(grid + 2 * (size_t)cell), "f"(re), "f"(im)
                     : "memory");
        const float er = two_sum_err(ore, re), ei = two_sum_err(oim, im);
        if (er != 0.f || ei != 0.f)
            red_add_c(comp + 2 * (size_t)cell, er, ei);
    }
};

// One task: every class of the W x W footprint over the task's visibilities.
// Each class keeps a running sum for its current cell and flushes it when
// the cell changes (and at the end).  Every cell a class visits lies inside
// the grid: the prep kernel keeps only footprints inside the grid, derive()
// moves a record that breaks this to cell 0 with zero weight, and tasks
// whose footprint is wider than the grid are rejected before this point.
// Kernel values: read-only global memory (the L1 path, through the
// non-coherent load) or the staged shared-memory block.
template <bool GMEM, typename KT>
__device__ __forceinline__ KT load_kernel(const KT* p)
{
    if constexpr (GMEM) return __ldg(p);
    else return *p;
}

template <typename GT, typename KT, int CPT, bool COUNT, bool GMEM,
          typename FL>
__device__ __forceinline__ void process_task(const TapVis<GT>* __restrict__ s_vis,
                                             int m, int w, int pitch,
                                             int row_shift,
                                             const KT* __restrict__ slab,
                                             const FL& flush,
                                             int grid_size, unsigned& flushes)
{
    const TaskLayout lay = task_layout<CPT>(w);
    int slices = lay.slices < m ? lay.slices : m;
    const int r = threadIdx.x / lay.per_slice;
    if (r >= slices) return;
    const int l = threadIdx.x - r * lay.per_slice;
    const int i0 = (r * m) / slices, i1 = ((r + 1) * m) / slices;
    const unsigned pitch_b = (unsigned)pitch * (unsigned)sizeof(KT);
    for (int it = l; it < lay.items; it += kGridThreads)
    {
        const int a = it % w;
        // Rows b0 .. b0 + CPT - 1; slots q < skip repeat the previous
        // group's rows and never flush (CPT <= W).
        int b0 = (it / w) * CPT, skip = 0;
        if (b0 + CPT > w)
        {
            skip = b0 + CPT - w;
            b0 = w - CPT;
        }
        // Every slot runs the same straight-line code (a per-slot `break`
        // cost a branch and convergence barriers per tap: 19.9 -> 16.8 ms
        // at plain_large without it); masked slots never flush.
        typename Vec2<GT>::type acc[CPT];   // (re, im) of each row's cell
        unsigned cur[CPT];
        constexpr bool kFused =
            std::is_same<FL, PlainFlush<float>>::value && !COUNT;
        {
            // The first visibility's cells: its taps flush nothing.
            const TapVis<GT> v = s_vis[i0];
            const unsigned ru = min((unsigned)(a + v.mu),
                                    (unsigned)(a + v.mu - w));
            const unsigned xb = (unsigned)(b0 + v.mv);
#pragma unroll
            for (int q = 0; q < CPT; ++q)
            {
                const unsigned rv = min(xb + q, xb + q - (unsigned)w);
                cur[q] = v.origin + ru + rv * (unsigned)grid_size;
                acc[q].x = acc[q].y = GT(0);
            }
        }
        // Two visibilities per iteration: the running cells then alternate
        // between registers instead of being moved (15.7 -> 15.2 ms at
        // plain_large).
#pragma unroll 2
        for (int i = i0; i < i1; ++i)
        {
            const TapVis<GT> v = s_vis[i];
            // (a + mu) mod W for a + mu in [0, 2W): min over unsigned wraps
            const unsigned ru = min((unsigned)(a + v.mu),
                                    (unsigned)(a + v.mu - w));
            const int col = (int)ru >= v.tu ? v.cp + (int)ru : v.cn - (int)ru;
            // The kernel row base of this visibility's column, as a byte
            // address: each tap's address is then one wide multiply-add of
            // its row by the row pitch in bytes.
            const char* __restrict__ kp = reinterpret_cast<const char*>(
                slab + (unsigned)(v.rowbase - row_shift + col));
            const unsigned cell0 = v.origin + ru;
            // All of this visibility's kernel values for the thread's rows
            // are requested before any is used.
            unsigned rvs[CPT];
            typename KernelLoad<KT>::Wide kv[CPT];
            const unsigned xb = (unsigned)(b0 + v.mv);
#pragma unroll
            for (int q = 0; q < CPT; ++q)
            {
                rvs[q] = min(xb + q, xb + q - (unsigned)w);
                kv[q] = KernelLoad<KT>::get(load_kernel<GMEM>(
                    reinterpret_cast<const KT*>(kp + (size_t)rvs[q] * pitch_b)));
            }
#pragma unroll
            for (int q = 0; q < CPT; ++q)
            {
                const unsigned cell = cell0 + rvs[q] * (unsigned)grid_size;
                if constexpr (kFused)
                {
                    flush.flush_reset(q >= skip, cell, cur[q], acc[q].x,
                                      acc[q].y);
                }
                else
                {
                    const bool change = q >= skip && cell != cur[q];
                    flush(change, cur[q], acc[q].x, acc[q].y);
                    if (COUNT) flushes += change;
                    acc[q].x = change ? GT(0) : acc[q].x;
                    acc[q].y = change ? GT(0) : acc[q].y;
                }
                cur[q] = cell;
                typename Vec2<GT>::type kk;
                kk.x = (GT)kv[q].x;
                kk.y = (GT)kv[q].y;
                cmac(acc[q], v.c0, v.c1, kk);
            }
        }
#pragma unroll
        for (int q = 0; q < CPT; ++q)
            flush(q >= skip, cur[q], acc[q].x, acc[q].y);
        if (COUNT) flushes += CPT - skip;
    }
}

template <typename GT, typename KT, bool COUNT, bool GMEM, typename FL>
__device__ __forceinline__ void dispatch_cpt(int cpt, const TapVis<GT>* s_vis,
                                             int m, int w, int pitch,
                                             int row_shift, const KT* slab,
                                             const FL& fl, int grid_size,
                                             unsigned& flushes)
{
#define B200_CPT(C)                                                         \
    process_task<GT, KT, C, COUNT, GMEM, FL>(s_vis, m, w, pitch, row_shift, \
                                             slab, fl, grid_size, flushes)
    // A row group never has more rows than the footprint (W = 1, 3, 5
    // take CPT = W).
    if (cpt > w) cpt = w;
    switch (cpt)
    {
    case 1: B200_CPT(1); break;
    case 2: B200_CPT(2); break;
    case 3: B200_CPT(3); break;
    case 4: B200_CPT(4); break;
    case 6: B200_CPT(6); break;
    default: B200_CPT(5); break;
    }
#undef B200_CPT
}

template <typename GT, bool COMP> struct FlushFor { using type = PlainFlush<GT>; };
template <> struct FlushFor<float, true> { using type = CompensatedFlush; };

template <typename GT, bool COMP>
__device__ __forceinline__ typename FlushFor<GT, COMP>::type
make_flush(void* grid, void* comp, bool active);
template <>
__device__ __forceinline__ PlainFlush<float> make_flush<float, false>(void* grid, void*, bool)
{
    return PlainFlush<float>{static_cast<float*>(grid)};
}
template <>
__device__ __forceinline__ PlainFlush<double> make_flush<double, false>(void* grid, void*, bool)
{
    return PlainFlush<double>{static_cast<double*>(grid)};
}
template <>
__device__ __forceinline__ CompensatedFlush make_flush<float, true>(void* grid, void* comp,
                                                                    bool active)
{
    return CompensatedFlush{static_cast<float*>(grid), static_cast<float*>(comp),
                            active};
}

// At least grid_ctas_per_sm<GT>() CTAs per SM.  FP32: with the
// straight-line row slots and at most 6 rows per thread, 4 CTAs (64
// registers) measured 16.28 ms at plain_large against 16.76 ms for 3 (and
// 16.94-17.74 ms for 5 or 6 CTAs with at most 4 or 3 rows per thread).
template <typename GT, typename KT, bool STAGED, bool COMP, bool COUNT>
__global__ void __launch_bounds__(kGridThreads, grid_ctas_per_sm<GT>())
romein_grid_kernel(const GridArgs a)
{
    using V2 = typename Vec2<GT>::type;
    extern __shared__ __align__(128) unsigned char smem[];
    // STAGED: [row block of the current run][tap records]; else [records]
    KT* s_block = reinterpret_cast<KT*>(smem);
    TapVis<GT>* s_vis = reinterpret_cast<TapVis<GT>*>(
        smem + (STAGED ? a.block_smem_bytes : 0));
    __shared__ uint64_t s_bar;
    __shared__ unsigned long long s_task;
    __shared__ uint32_t s_order[kGridThreads];
    __shared__ int s_run_begin[kMaxOffsets], s_run_end[kMaxOffsets];
    __shared__ unsigned char s_head[kTaskMax];
    __shared__ int s_warp_heads[kGridThreads / 32];

    unsigned long long* status = &a.counters[CNT_STATUS];
    const unsigned num_tasks = (unsigned)a.counters[CNT_TASKS];
    unsigned long long first = 0, end = num_tasks;
    unsigned long long* queue = &a.counters[CNT_TASK_NEXT];
    if (a.range)
    {
        first = a.range[0];
        end = min((unsigned long long)a.range[1], end);
        queue = a.queue;
    }

    if (STAGED && threadIdx.x == 0)
    {
        mbar_init(&s_bar, 1);
        mbar_fence_init();
    }
    __syncthreads();

    uint32_t phase = 0;
    unsigned flushes = 0;
    for (;;)
    {
        if (threadIdx.x == 0) s_task = first + atomicAdd(queue, 1ull);
        if (threadIdx.x < kMaxOffsets)
        {
            s_run_begin[threadIdx.x] = 0;
            s_run_end[threadIdx.x] = 0;
        }
        // Also: every thread has finished with the previous task's records
        // and row block before they are overwritten below.
        __syncthreads();
        if (s_task >= end) break;
        const unsigned task = (unsigned)s_task;
        const uint32_t begin = a.task_start[task];
        int m = (int)(a.task_start[task + 1] - begin);
        if (m <= 0 || m > kTaskMax)
        {
            if (threadIdx.x == 0)
                atomicOr(status, (unsigned long long)DEV_ERR_TASK);
            __syncthreads();   // s_task is read before thread 0 rewrites it
            continue;
        }
        // The task's job: its cube, grid and geometry.
        const JobDesc& jd = a.jobs[a.task_job[task]];
        const TaskKey tk(jd.half, !STAGED);
        const int t = threadIdx.x;
        // Gather the task's visibilities (sorted positions begin .. begin +
        // m - 1) straight from the caller's arrays: record, visibility and
        // weight of each point.  Against a separate pass that permuted
        // records and visibilities into sorted order: plain_large step
        // 19.15 -> 18.25 ms (the 1.6 ms pass gone, the gridding kernel
        // 0.7 ms slower with the gathers in its task set-up; prefetching
        // the next task's points into L2 cost more than it hid).
        static_assert(sizeof(RawVis<GT>) <= sizeof(TapVis<GT>),
                      "raw records fit the tap-record array");
        RawVis<GT>* s_raw = reinterpret_cast<RawVis<GT>*>(s_vis);
        uint32_t key = 0xffffffffu;
        if (t < m)
        {
            const uint32_t i = a.order[begin + t];
            RawVis<GT> rv;
            rv.rec = a.rec[i];
            const size_t local = i - jd.first;
            const GT* __restrict__ vis = static_cast<const GT*>(jd.vis);
            GT re = vis[2 * local], im = vis[2 * local + 1];
            if (a.apply_weight)
            {
                const GT wt = static_cast<const GT*>(jd.weight)[local];
                re *= wt;
                im *= wt;
            }
            rv.vis.x = re;
            rv.vis.y = im;
            s_raw[t] = rv;
            key = tk.make(rv.rec, t);
        }
        // Order the task's visibilities by (row offset, cell): each run of
        // one row offset reads one W-row block of the plane's slab, and
        // consecutive visibilities are neighbours.  (Its block barriers also
        // publish the raw records.)
        static_assert(kGridThreads >= 64, "task_order has a block barrier");
        key = task_order(key, s_order);
        const KT* __restrict__ slabs = static_cast<const KT*>(jd.slabs);
        const int4 r0 = s_raw[0].rec;
        // Compensation is limited to tasks near the grid centre when a
        // radius is set (a task is a compact run of one coarse tile).
        bool comp_here = true;
        if (COMP && a.comp_radius > 0)
        {
            const int c = jd.grid_size / 2;
            comp_here = abs(r0.x - c) <= a.comp_radius &&
                        abs(r0.y - c) <= a.comp_radius;
        }
        const auto fl = make_flush<GT, COMP>(jd.grid, jd.comp, comp_here);
        const int grid_size = jd.grid_size;
        const int offsets = 2 * jd.half + 1;
        const int plane = r0.z & 0x7fffffff;
        const PlaneDesc d = static_cast<const PlaneDesc*>(jd.planes)[plane];
        const int w = 2 * d.support + 1;
        // No kept footprint is wider than its grid; a task that says
        // otherwise is malformed (and its cells could leave the grid).
        if (w > grid_size)
        {
            if (threadIdx.x == 0)
                atomicOr(status, (unsigned long long)DEV_ERR_TASK);
            __syncthreads();   // s_task is read before thread 0 rewrites it
            continue;
        }
        const int cpt = d.support < kTuneMax ? a.cpt[d.support] : 5;

        RawVis<GT> mine;
        if (t < m) mine = s_raw[key & 0xffu];
        __syncthreads();   // every raw record is read before it is overwritten
        TapVis<GT> tv;
        if (t < m)
        {
            tv = derive<GT>(mine.rec, mine.vis, d, grid_size, jd.oversample,
                            jd.half, status);
            s_vis[t] = tv;
        }
        __syncthreads();
        // Merge runs of records with the same taps (the same cell, plane
        // and offsets: adjacent in this order): their coefficients add.
        // Dense cells hold many visibilities with identical placements; at
        // plain_large this removes a sixth of the taps.
        const bool head = t < m && (t == 0 || !same_taps(tv, s_vis[t - 1]));
        s_head[t] = head ? 1 : 0;
        const unsigned ball = __ballot_sync(0xffffffffu, head);
        if ((t & 31) == 0) s_warp_heads[t >> 5] = __popc(ball);
        __syncthreads();
        int pos = __popc(ball & ((1u << (t & 31)) - 1u)), merged = 0;
#pragma unroll
        for (int wi = 0; wi < kGridThreads / 32; ++wi)
        {
            pos += wi < (t >> 5) ? s_warp_heads[wi] : 0;
            merged += s_warp_heads[wi];
        }
        if (head)
        {
            for (int q = t + 1; q < m && !s_head[q]; ++q)
            {
                tv.c0.x += s_vis[q].c0.x;
                tv.c0.y += s_vis[q].c0.y;
                tv.c1.x += s_vis[q].c1.x;
                tv.c1.y += s_vis[q].c1.y;
            }
        }
        __syncthreads();   // every run has been read
        if (head)
        {
            s_vis[pos] = tv;
            s_order[pos] = key;
        }
        __syncthreads();
        m = merged;
        if (STAGED && t < m)
        {
            key = s_order[t];
            const int ov = tk.row_offset(key);
            if (t == 0 || tk.row_offset(s_order[t - 1]) != ov)
                s_run_begin[ov] = t;
            if (t == m - 1 || tk.row_offset(s_order[t + 1]) != ov)
                s_run_end[ov] = t + 1;
        }
        __syncthreads();

        if (!STAGED)
        {
            dispatch_cpt<GT, KT, COUNT, true>(cpt, s_vis, m, w, d.pitch, 0,
                                        slabs + d.offset, fl, grid_size,
                                        flushes);
            continue;
        }
        const unsigned block_elems = (unsigned)w * (unsigned)d.pitch;
        const unsigned block_bytes = block_elems * (unsigned)sizeof(KT);
        for (int ov = 0; ov < offsets; ++ov)
        {
            const int rb = s_run_begin[ov], re = s_run_end[ov];
            if (re <= rb) continue;
            if (threadIdx.x == 0)
            {
                // Every thread finished reading the previous block (barrier
                // below / above); order that before the async-proxy write.
                fence_proxy_async_shared();
                mbar_arrive_expect_tx(&s_bar, block_bytes);
                const unsigned char* src = reinterpret_cast<const unsigned char*>(
                    slabs + d.offset + (long long)ov * block_elems);
                for (unsigned off = 0; off < block_bytes; off += kBulkChunk)
                    bulk_copy_g2s(reinterpret_cast<unsigned char*>(s_block) + off,
                                  src + off, min(kBulkChunk, block_bytes - off),
                                  &s_bar);
            }
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
            dispatch_cpt<GT, KT, COUNT, false>(cpt, s_vis + rb, re - rb, w,
                                        d.pitch, ov * (int)block_elems,
                                        s_block, fl, grid_size, flushes);
            __syncthreads();
        }
    }
    if (COUNT)
    {
        const unsigned long long f = warp_sum((unsigned long long)flushes);
        if ((threadIdx.x & 31) == 0 && f)
            atomicAdd(&a.counters[CNT_FLUSHES], f);
    }
}

template <typename GT, typename KT, bool STAGED, bool COMP = false,
          bool COUNT = false>
cudaError_t launch_variant(const GridArgs& a, int num_sms, size_t smem,
                           cudaStream_t st, int* ctas_out)
{
    auto fn = romein_grid_kernel<GT, KT, STAGED, COMP, COUNT>;
    // Function attributes and occupancy are looked up once per (variant,
    // device, shared-memory size), not on every launch.
    static std::mutex mu;
    static int cached_dev = -1;
    static size_t cached_smem = 0;
    static int cached_per_sm = 0;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    {
        std::lock_guard<std::mutex> lock(mu);
        if (dev == cached_dev && smem == cached_smem)
        {
            per_sm = cached_per_sm;
        }
        else
        {
            e = cudaFuncSetAttribute(
                fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
            if (!STAGED)
            {
                // Only the shared memory grid_ctas_per_sm CTAs need; the
                // rest of the SM's unified L1/shared storage caches kernel
                // values (measured 19.88 -> 19.66 ms at plain_large against
                // the default carveout).
                cudaFuncAttributes fa{};
                e = cudaFuncGetAttributes(&fa, fn);
                if (e != cudaSuccess) return e;
                const size_t per = smem + fa.sharedSizeBytes + 1024;
                int pct = (int)((100 * grid_ctas_per_sm<GT>() * per +
                                 228 * 1024 - 1) /
                                (228 * 1024));
                pct = pct > 100 ? 100 : pct;
                e = cudaFuncSetAttribute(
                    fn, cudaFuncAttributePreferredSharedMemoryCarveout, pct);
                if (e != cudaSuccess) return e;
            }
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                &per_sm, fn, kGridThreads, smem);
            if (e != cudaSuccess) return e;
            cached_dev = dev;
            cached_smem = smem;
            cached_per_sm = per_sm;
        }
    }
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    const int ctas = num_sms * per_sm;
    if (ctas_out) *ctas_out = ctas;
    fn<<<ctas, kGridThreads, smem, st>>>(a);
    return cudaGetLastError();
}

}  // namespace

// Rows-per-thread (CPT) for each support, from a cost model of
// process_task: per visibility a thread does ~12 instructions of shared
// column work plus ~20 per class, so the cost of a tap is
// (12 / CPT + 20) / utilisation, utilisation being the fraction of the
// CTA's thread slots (threads x CPT x passes) holding a live class under
// the (column, row group) layout of process_task.
void default_tune_table(unsigned char* cpt)
{
    const int choices[] = {1, 2, 3, 4, 5, 6};
    for (int s = 0; s < kTuneMax; ++s)
    {
        const int w = 2 * s + 1;
        double best = 1e30;
        int pick = 1;
        for (int c : choices)
        {
            if (c > w) continue;
            const int items = w * ((w + c - 1) / c);
            const int slices = items <= kGridThreads ? kGridThreads / items : 1;
            const int passes = (items + kGridThreads - 1) / kGridThreads;
            const double util = (double)w * w * slices /
                                ((double)kGridThreads * c * passes);
            const double cost = (12.0 / c + 20.0) / util;
            if (cost < best - 1e-9)
            {
                best = cost;
                pick = c;
            }
        }
        cpt[s] = (unsigned char)pick;
    }
}

namespace {

// Block (x, j) folds part of job j's error grid into its grid.
__global__ void fold_kernel(const JobDesc* __restrict__ jobs)
{
    const JobDesc& jd = jobs[blockIdx.y];
    if (!jd.comp) return;
    float2* grid = static_cast<float2*>(jd.grid);
    float2* comp = static_cast<float2*>(jd.comp);
    const size_t cells = (size_t)jd.grid_size * (size_t)jd.grid_size;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < cells;
         i += (size_t)gridDim.x * blockDim.x)
    {
        const float2 c = comp[i];
        if (c.x != 0.f || c.y != 0.f)
        {
            float2 g = grid[i];
            g.x += c.x;
            g.y += c.y;
            grid[i] = g;
            comp[i] = make_float2(0.f, 0.f);
        }
    }
}

}  // namespace

cudaError_t launch_fold_jobs(const JobDesc* jobs, int num_jobs, int num_sms,
                             cudaStream_t st)
{
    int bx = num_sms * 8 / (num_jobs > 0 ? num_jobs : 1);
    if (bx < 4) bx = 4;
    fold_kernel<<<dim3(bx, num_jobs), 256, 0, st>>>(jobs);
    return cudaGetLastError();
}

size_t grid_smem_bytes(int data_is_double, unsigned max_block_bytes,
                       bool staged)
{
    const size_t rec = data_is_double ? sizeof(TapVis<double>)
                                      : sizeof(TapVis<float>);
    const size_t block = staged ? ((max_block_bytes + 127) / 128) * 128 : 0;
    return block + rec * kTaskMax;
}

cudaError_t launch_grid(const GridArgs& a, int data_is_double,
                        int kernel_type, unsigned max_block_bytes, bool staged,
                        bool compensated, int num_sms, cudaStream_t st,
                        int* ctas_out)
{
    const size_t smem = grid_smem_bytes(data_is_double, max_block_bytes,
                                        staged);
    GridArgs args = a;
    args.block_smem_bytes = staged ? (unsigned)(((max_block_bytes + 127) /
                                                  128) * 128)
                                    : 0u;
    if (compensated)
    {
        // FP32 grids only; kernel values read through L1.
        if (data_is_double || staged) return cudaErrorInvalidValue;
        switch (kernel_type)
        {
        case OSKAR_B200_KERNEL_F16:
            return a.count_flushes
                ? launch_variant<float, __half2, false, true, true>(args, num_sms, smem, st, ctas_out)
                : launch_variant<float, __half2, false, true>(args, num_sms, smem, st, ctas_out);
        case OSKAR_B200_KERNEL_BF16:
            return a.count_flushes
                ? launch_variant<float, __nv_bfloat162, false, true, true>(args, num_sms, smem, st, ctas_out)
                : launch_variant<float, __nv_bfloat162, false, true>(args, num_sms, smem, st, ctas_out);
        default:
            return a.count_flushes
                ? launch_variant<float, float2, false, true, true>(args, num_sms, smem, st, ctas_out)
                : launch_variant<float, float2, false, true>(args, num_sms, smem, st, ctas_out);
        }
    }
    // Flushes are counted (statistics) on the L1 path only.
    const bool count = a.count_flushes && !staged;
    if (data_is_double)
    {
        if (kernel_type != OSKAR_B200_KERNEL_NATIVE)
            return cudaErrorInvalidValue;
        if (staged) return launch_variant<double, double2, true>(args, num_sms, smem, st, ctas_out);
        return count ? launch_variant<double, double2, false, false, true>(args, num_sms, smem, st, ctas_out)
                     : launch_variant<double, double2, false>(args, num_sms, smem, st, ctas_out);
    }
    switch (kernel_type)
    {
    case OSKAR_B200_KERNEL_F16:
        if (staged) return launch_variant<float, __half2, true>(args, num_sms, smem, st, ctas_out);
        return count ? launch_variant<float, __half2, false, false, true>(args, num_sms, smem, st, ctas_out)
                     : launch_variant<float, __half2, false>(args, num_sms, smem, st, ctas_out);
    case OSKAR_B200_KERNEL_BF16:
        if (staged) return launch_variant<float, __nv_bfloat162, true>(args, num_sms, smem, st, ctas_out);
        return count ? launch_variant<float, __nv_bfloat162, false, false, true>(args, num_sms, smem, st, ctas_out)
                     : launch_variant<float, __nv_bfloat162, false>(args, num_sms, smem, st, ctas_out);
    default:
        if (staged) return launch_variant<float, float2, true>(args, num_sms, smem, st, ctas_out);
        return count ? launch_variant<float, float2, false, false, true>(args, num_sms, smem, st, ctas_out)
                     : launch_variant<float, float2, false>(args, num_sms, smem, st, ctas_out);
    }
}

}  // namespace b200
