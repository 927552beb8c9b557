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
// fine cell), so consecutive warps read neighbouring grid rows and the same
// kernel slab rows from L1/L2.  One warp takes one visibility: its lanes
// take footprint columns (32 at a time) and walk the footprint rows, so a
// row's grid cells and kernel values are read as contiguous runs; the lane
// sums are then reduced across the warp.  The result goes to the
// visibility's own slot (the sort's values are the original indices).
#include "common.cuh"
#include "internal.h"

namespace b200 {
namespace {

template <typename GT> struct Cplx;
template <> struct Cplx<float> { using type = float2; };
template <> struct Cplx<double> { using type = double2; };

// apply_weight: the adjoint of gridding weight * vis, i.e. the degridded
// value times the visibility's weight.
template <typename GT, typename KT>
__global__ void __launch_bounds__(256)
degrid_kernel(const uint32_t* __restrict__ order,
              const uint32_t* __restrict__ sorted_keys,
              const int4* __restrict__ rec, const JobDesc* __restrict__ jobs,
              int job_shift, int apply_weight,
              unsigned long long* __restrict__ counters, size_t n)
{
    using C2 = typename Cplx<GT>::type;
    const size_t valid = n - counters[CNT_SKIPPED];
    const int lane = threadIdx.x & 31;
    const size_t warp0 = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const size_t warps = ((size_t)gridDim.x * blockDim.x) >> 5;
    for (size_t s = warp0; s < valid; s += warps)
    {
        const uint32_t i = order[s];
        const JobDesc& jd = jobs[sorted_keys[s] >> job_shift];
        const int4 r = rec[i];
        const int plane = r.z & 0x7fffffff;
        const GT sgn = r.z < 0 ? GT(-1) : GT(1);
        const int half = jd.half, os = jd.oversample;
        const int off_u = min(max((r.w & 0xffff) - half, -half), half);
        const int off_v = min(max((r.w >> 16) - half, -half), half);
        const PlaneDesc d = static_cast<const PlaneDesc*>(jd.planes)[plane];
        const int S = d.support, W = 2 * S + 1, G = jd.grid_size;
        const int u0 = r.x - S, v0 = r.y - S;
        // The prep kernel keeps only footprints inside the grid; a record
        // that says otherwise is reported and produces nothing.
        if (u0 < 0 || v0 < 0 || u0 + W > G || v0 + W > G)
        {
            if (lane == 0)
                atomicOr(&counters[CNT_STATUS],
                         (unsigned long long)DEV_ERR_GRID_INDEX);
            continue;
        }
        const KT* __restrict__ slab =
            static_cast<const KT*>(jd.slabs) + d.offset +
            (long long)(off_v + half) * W * d.pitch;
        const C2* __restrict__ grid = static_cast<const C2*>(jd.grid);
        GT are = GT(0), aim = GT(0);
        for (int k = lane; k < W; k += 32)
        {
            // quadrant column |off_u + (k - S) * os|, phase-major position
            const int x = abs(off_u + (k - S) * os);
            const int pos = (x % os) * d.L + x / os;
            const KT* kp = slab + pos;
            const C2* gp = grid + (size_t)v0 * G + u0 + k;
#pragma unroll 4
            for (int j = 0; j < W; ++j)
            {
                const auto kv = KernelLoad<KT>::get(kp[(long long)j * d.pitch]);
                const C2 g = gp[(size_t)j * G];
                const GT kr = (GT)kv.x, ki = sgn * (GT)kv.y;
                // grid * conj(Kt), Kt = (kr, ki)
                are = fma(g.x, kr, fma(g.y, ki, are));
                aim = fma(g.y, kr, fma(-g.x, ki, aim));
            }
        }
        are = warp_sum(are);
        aim = warp_sum(aim);
        if (lane == 0)
        {
            const size_t local = i - jd.first;
            GT sc = (GT)d.scale;
            if (apply_weight) sc *= static_cast<const GT*>(jd.weight)[local];
            GT* out = static_cast<GT*>(const_cast<void*>(jd.vis));
            out[2 * local] = are * sc;
            out[2 * local + 1] = aim * sc;
        }
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
    const size_t want = (n * 32 + 255) / 256;
    const size_t cap = (size_t)num_sms * 8;
    const unsigned blocks = (unsigned)(want < cap ? (want ? want : 1) : cap);
    if (data_is_double)
    {
        if (kernel_type != OSKAR_B200_KERNEL_NATIVE)
            return cudaErrorInvalidValue;
        degrid_kernel<double, double2><<<blocks, 256, 0, st>>>(
            order, sorted_keys, rec, jobs, job_shift, apply_weight, counters, n);
    }
    else if (kernel_type == OSKAR_B200_KERNEL_F16)
        degrid_kernel<float, __half2><<<blocks, 256, 0, st>>>(
            order, sorted_keys, rec, jobs, job_shift, apply_weight, counters, n);
    else if (kernel_type == OSKAR_B200_KERNEL_BF16)
        degrid_kernel<float, __nv_bfloat162><<<blocks, 256, 0, st>>>(
            order, sorted_keys, rec, jobs, job_shift, apply_weight, counters, n);
    else
        degrid_kernel<float, float2><<<blocks, 256, 0, st>>>(
            order, sorted_keys, rec, jobs, job_shift, apply_weight, counters, n);
    return cudaGetLastError();
}

}  // namespace b200
