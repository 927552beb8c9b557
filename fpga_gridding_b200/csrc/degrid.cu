// Degridding: the adjoint of the W-projection gridder.  The reference has
// no degridder (Defines.h:48 only reserves the switch); this one is defined
// as the exact adjoint of the gridding path of this library: with the
// gridder's placement, skip test and tap kernel value
//   Kt = conj?(K[plane][|off_v + j*os|][|off_u + k*os|])
// (conjugated for w > 0, oskar_grid_wproj.c:70-122), each kept visibility
// becomes
//   vis = sum over the (2S+1)^2 taps of grid[(gv+j)*G + gu+k] * conj(Kt).
//
// The visibilities arrive in the gridder's sort order (coarse tile, plane,
// fine cell); each CTA takes chunks of consecutive ones from a work queue,
// so its warps read neighbouring grid rows and the same kernel slab rows
// from L1.  A group of 16 lanes takes one visibility (2 per warp): its
// lanes walk the footprint's taps in row-major order, 16 at a time (busy
// whatever the support; the per-visibility set-up and reduction serve 2
// visibilities at once), and the lane sums are reduced within the group.
// Measured at plain_large: 16 lanes 28.5 ms, 8 lanes 30.2, 4 lanes 33.8,
// 32 lanes 40.9.
// The result goes to the visibility's own slot (the sort's values are the
// original indices).
#include "common.cuh"
#include "internal.h"

namespace b200 {
namespace {

template <typename GT> struct Cplx;
template <> struct Cplx<float> { using type = float2; };
template <> struct Cplx<double> { using type = double2; };

constexpr int kDegridWarps = 8;     // warps per CTA
constexpr int kGroup = 16;          // lanes per visibility
constexpr int kGroups = 32 / kGroup;
constexpr int kDegridMaxW = 255;   // footprint width for support <= 127
constexpr int kDegridChunk = 128;  // visibilities per work-queue item

// Sum over taps of grid * conj(Kt), Kt = (kr, sgn * ki).  FP32: two packed
// FMAs per tap, A += g * kr and B += g * ki, with the sign applied once at
// the end (re = A.x + sgn B.y, im = A.y - sgn B.x).  FP64: four FMAs per
// tap in the order of the definition.
template <typename GT> struct DegridAcc;
template <> struct DegridAcc<float>
{
    float2 a = make_float2(0.f, 0.f), b = make_float2(0.f, 0.f);
    float sgn;
    __device__ __forceinline__ explicit DegridAcc(float s) : sgn(s) {}
    __device__ __forceinline__ void add(const float2 g, float kr, float ki)
    {
        a = __ffma2_rn(g, make_float2(kr, kr), a);
        b = __ffma2_rn(g, make_float2(ki, ki), b);
    }
    __device__ __forceinline__ void finish(float& re, float& im) const
    {
        re = fmaf(sgn, b.y, a.x);
        im = fmaf(-sgn, b.x, a.y);
    }
};
template <> struct DegridAcc<double>
{
    double re = 0.0, im = 0.0, sgn;
    __device__ __forceinline__ explicit DegridAcc(double s) : sgn(s) {}
    __device__ __forceinline__ void add(const double2 g, double kr, double ki)
    {
        ki *= sgn;
        re = fma(g.x, kr, fma(g.y, ki, re));
        im = fma(g.y, kr, fma(-g.x, ki, im));
    }
    __device__ __forceinline__ void finish(double& r, double& i) const
    {
        r = re;
        i = im;
    }
};

// Slab column of footprint column k: the quadrant column |off_u + (k - S) os|
// in the phase-major layout, (x mod os) * L + x / os.  For k >= tu the
// argument is non-negative and the column is cp + k; below, cn - k.  With
// |off_u| <= os the remainders and quotients need no division.
struct ColumnMap
{
    int tu, cp, cn;
    __device__ __forceinline__ ColumnMap(int off_u, int S, int os, int L)
    {
        const int rp = off_u < 0 ? off_u + os : (off_u >= os ? off_u - os : off_u);
        const int qp = off_u < 0 ? -1 : (off_u >= os ? 1 : 0);
        const int on = -off_u;
        const int rn = on < 0 ? on + os : (on >= os ? on - os : on);
        const int qn = on < 0 ? -1 : (on >= os ? 1 : 0);
        tu = S + (off_u < 0 ? 1 : 0);
        cp = rp * L + qp - S;
        cn = rn * L + qn + S;
    }
    __device__ __forceinline__ int operator()(int k) const
    {
        return k >= tu ? cp + k : cn - k;
    }
};

// Rows in the outer loop, each lane of a group owning the footprint columns
// k = gl + kGroup * m, m < M: the byte addresses of each column's kernel
// value and grid cell in the first row are registers, so a tap costs two
// wide multiply-adds (row times the row pitch in bytes), two loads and the
// packed multiply-adds.  Used for footprints kGroup to 5 * kGroup wide
// (narrower ones would leave lanes idle; wider ones take the flattened
// walk).  The slab and the grid are read-only here: non-coherent loads.
template <int M, typename GT, typename KT, typename C2>
__device__ __forceinline__ void degrid_rows(const KT* __restrict__ slab,
                                            const C2* __restrict__ grid,
                                            int W, int pitch, int G,
                                            const ColumnMap& cm, int gl,
                                            DegridAcc<GT>& acc)
{
    const char* kc[M];
    const char* gc[M];
    bool ok[M];
#pragma unroll
    for (int m = 0; m < M; ++m)
    {
        const int k = gl + kGroup * m;
        ok[m] = k < W;
        kc[m] = reinterpret_cast<const char*>(slab + (ok[m] ? cm(k) : 0));
        gc[m] = reinterpret_cast<const char*>(grid + (ok[m] ? k : 0));
    }
    const unsigned kb = (unsigned)pitch * (unsigned)sizeof(KT);
    const unsigned gb = (unsigned)G * (unsigned)sizeof(C2);
    for (int j = 0; j < W; ++j)
    {
#pragma unroll
        for (int m = 0; m < M; ++m)
        {
            if (!ok[m]) continue;
            const auto kv = KernelLoad<KT>::get(__ldg(
                reinterpret_cast<const KT*>(kc[m] + (size_t)j * kb)));
            const C2 g = __ldg(
                reinterpret_cast<const C2*>(gc[m] + (size_t)j * gb));
            acc.add(g, (GT)kv.x, (GT)kv.y);
        }
    }
}

// apply_weight: the adjoint of gridding weight * vis, i.e. the degridded
// value times the visibility's weight.
// Registers bounded for 4 resident CTAs (32 warps) per SM.  FP32 at
// plain_large: 2 CTAs 30.3 ms, 3: 23.2, 4: 20.8, 5: 22.1, 6: 23.3 (more
// warps share the same L1 for their kernel rows and grid lines).
template <typename GT, typename KT>
__global__ void __launch_bounds__(kDegridWarps * 32, 4)
degrid_kernel(const uint32_t* __restrict__ order,
              const uint32_t* __restrict__ sorted_keys,
              const int4* __restrict__ rec, const JobDesc* __restrict__ jobs,
              int job_shift, int apply_weight,
              unsigned long long* __restrict__ counters, size_t n)
{
    using C2 = typename Cplx<GT>::type;
    __shared__ unsigned long long s_chunk;
    const size_t valid = n - counters[CNT_SKIPPED];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int group = lane / kGroup, gl = lane % kGroup;
    // A CTA takes chunks of kDegridChunk consecutive sorted visibilities
    // from a work queue: its warps work on neighbouring footprints and share
    // grid lines and kernel rows in L1, and the uneven cost of the chunks
    // (footprints of 81 to 5329 taps) balances across CTAs.
    for (;;)
    {
        if (threadIdx.x == 0)
            s_chunk = atomicAdd(&counters[CNT_TASK_NEXT], 1ull);
        __syncthreads();
        const size_t begin = (size_t)s_chunk * kDegridChunk;
        __syncthreads();   // every thread has read s_chunk
        if (begin >= valid) break;
        const size_t end = min(valid, begin + (size_t)kDegridChunk);
        // Each warp takes kGroups visibilities at a time, one per group of
        // kGroup lanes (the loop bounds are the same for the whole warp).
        for (size_t base = begin + (size_t)warp * kGroups; base < end;
             base += (size_t)kDegridWarps * kGroups)
        {
            const size_t s = base + group;
            bool active = s < end;
            uint32_t i = 0;
            const JobDesc* jd = nullptr;
            int4 r = make_int4(0, 0, 0, 0);
            if (active)
            {
                i = order[s];
                jd = &jobs[sorted_keys[s] >> job_shift];
                r = rec[i];
            }
            int S = 0, W = 0, u0 = 0, v0 = 0, off_u = 0, off_v = 0, half = 0;
            int os = 1, G = 1;
            PlaneDesc d{};
            GT sgn = GT(1);
            if (active)
            {
                const int plane = r.z & 0x7fffffff;
                sgn = r.z < 0 ? GT(-1) : GT(1);
                half = jd->half;
                os = jd->oversample;
                off_u = min(max((r.w & 0xffff) - half, -half), half);
                off_v = min(max((r.w >> 16) - half, -half), half);
                d = static_cast<const PlaneDesc*>(jd->planes)[plane];
                S = d.support;
                W = 2 * S + 1;
                G = jd->grid_size;
                u0 = r.x - S;
                v0 = r.y - S;
                // The prep kernel keeps only footprints inside the grid; a
                // record that says otherwise is reported and skipped.
                if (u0 < 0 || v0 < 0 || u0 + W > G || v0 + W > G ||
                    W > kDegridMaxW)
                {
                    if (gl == 0)
                        atomicOr(&counters[CNT_STATUS],
                                 (unsigned long long)DEV_ERR_GRID_INDEX);
                    active = false;
                    W = 0;
                }
            }
            const ColumnMap cm(off_u, S, os, d.L);
            DegridAcc<GT> acc(sgn);
            if (active)
            {
                const KT* __restrict__ slab =
                    static_cast<const KT*>(jd->slabs) + d.offset +
                    (long long)(off_v + half) * W * d.pitch;
                const C2* __restrict__ grid =
                    static_cast<const C2*>(jd->grid) + (size_t)v0 * G + u0;
                // The group's lanes walk the W * W taps in row-major order,
                // kGroup at a time (contiguous grid reads within a row).
                const int mc = (W + kGroup - 1) / kGroup;
                if (W >= kGroup && mc <= 5)
                {
                    // rows outer, columns per lane (plain_large degrid
                    // 26.5 -> 25.2 ms)
                    switch (mc)
                    {
                    case 1: degrid_rows<1, GT>(slab, grid, W, d.pitch, G, cm, gl, acc); break;
                    case 2: degrid_rows<2, GT>(slab, grid, W, d.pitch, G, cm, gl, acc); break;
                    case 3: degrid_rows<3, GT>(slab, grid, W, d.pitch, G, cm, gl, acc); break;
                    case 4: degrid_rows<4, GT>(slab, grid, W, d.pitch, G, cm, gl, acc); break;
                    default: degrid_rows<5, GT>(slab, grid, W, d.pitch, G, cm, gl, acc); break;
                    }
                }
                else
                {
                    // The lane's tap (j, k) is tracked as 32-bit running
                    // offsets (grid cell j * G + k, kernel row j * pitch),
                    // stepped kGroup taps at a time with k wrapping past W: the
                    // 64-bit index arithmetic per tap cost 28.4 -> 26.5 ms at
                    // plain_large.
                    const int taps = W * W, dj = kGroup / W, dk = kGroup % W;
                    const int j0 = gl / W;
                    int k = gl - j0 * W;
                    unsigned goff = (unsigned)j0 * (unsigned)G + (unsigned)k;
                    unsigned krow = (unsigned)j0 * (unsigned)d.pitch;
                    const unsigned gstep = (unsigned)dj * (unsigned)G + (unsigned)dk;
                    const unsigned kstep = (unsigned)dj * (unsigned)d.pitch;
                    const unsigned gwrap = (unsigned)G - (unsigned)W;
                    const unsigned kwrap = (unsigned)d.pitch;
#pragma unroll 4
                    for (int t = gl; t < taps; t += kGroup)
                    {
                        const auto kv =
                            KernelLoad<KT>::get(__ldg(slab + krow + cm(k)));
                        const C2 g = __ldg(grid + goff);
                        acc.add(g, (GT)kv.x, (GT)kv.y);
                        k += dk;
                        goff += gstep;
                        krow += kstep;
                        const bool wrap = k >= W;
                        k = wrap ? k - W : k;
                        goff += wrap ? gwrap : 0u;
                        krow += wrap ? kwrap : 0u;
                    }
                }
            }
            GT are, aim;
            acc.finish(are, aim);
#pragma unroll
            for (int o = kGroup / 2; o > 0; o >>= 1)
            {
                are += __shfl_xor_sync(0xffffffffu, are, o);
                aim += __shfl_xor_sync(0xffffffffu, aim, o);
            }
            if (active && gl == 0)
            {
                const size_t local = i - jd->first;
                GT sc = (GT)d.scale;
                if (apply_weight)
                    sc *= static_cast<const GT*>(jd->weight)[local];
                GT* out = static_cast<GT*>(const_cast<void*>(jd->vis));
                out[2 * local] = are * sc;
                out[2 * local + 1] = aim * sc;
            }
        }
        __syncthreads();   // before thread 0 takes the next chunk
    }
}

}  // namespace

cudaError_t launch_degrid(const uint32_t* order, const uint32_t* sorted_keys,
                          const int4* rec, const JobDesc* jobs, int job_shift,
                          int apply_weight, unsigned long long* counters,
                          size_t n,
                          int data_is_double, int kernel_type, int num_sms,
                          cudaStream_t st)
{
    // up to 8 CTAs of 8 warps per SM, persistent over the work queue
    const size_t want = (n + kDegridChunk - 1) / kDegridChunk;
    const size_t cap = (size_t)num_sms * 8;
    const unsigned blocks = (unsigned)(want < cap ? (want ? want : 1) : cap);
    if (data_is_double)
    {
        if (kernel_type != OSKAR_B200_KERNEL_NATIVE)
            return cudaErrorInvalidValue;
        degrid_kernel<double, double2><<<blocks, kDegridWarps * 32, 0, st>>>(
            order, sorted_keys, rec, jobs, job_shift, apply_weight, counters, n);
    }
    else if (kernel_type == OSKAR_B200_KERNEL_F16)
        degrid_kernel<float, __half2><<<blocks, kDegridWarps * 32, 0, st>>>(
            order, sorted_keys, rec, jobs, job_shift, apply_weight, counters, n);
    else if (kernel_type == OSKAR_B200_KERNEL_BF16)
        degrid_kernel<float, __nv_bfloat162><<<blocks, kDegridWarps * 32, 0, st>>>(
            order, sorted_keys, rec, jobs, job_shift, apply_weight, counters, n);
    else
        degrid_kernel<float, float2><<<blocks, kDegridWarps * 32, 0, st>>>(
            order, sorted_keys, rec, jobs, job_shift, apply_weight, counters, n);
    return cudaGetLastError();
}

}  // namespace b200
