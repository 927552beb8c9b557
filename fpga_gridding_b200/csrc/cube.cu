// Kernel-cube ingest: re-lays the reference's W-kernel cube into
// phase-major per-plane slabs (see PlaneDesc in internal.h) in the storage
// type the gridding kernel reads, and tabulates the per-(plane, offset) norm
// contribution.
#include <cmath>
#include <vector>

#include "common.cuh"
#include "internal.h"

namespace b200 {
namespace {

template <typename KT> struct Store;
template <> struct Store<float2>
{
    __device__ static float2 make(double re, double im, float inv)
    {
        return make_float2((float)re, (float)im);
    }
};
template <> struct Store<double2>
{
    __device__ static double2 make(double re, double im, float inv)
    {
        return make_double2(re, im);
    }
};
template <> struct Store<__half2>
{
    __device__ static __half2 make(double re, double im, float inv)
    {
        return __floats2half2_rn((float)re * inv, (float)im * inv);
    }
};
template <> struct Store<__nv_bfloat162>
{
    __device__ static __nv_bfloat162 make(double re, double im, float inv)
    {
        return __floats2bfloat162_rn((float)re * inv, (float)im * inv);
    }
};

// The reference's cube as the kernels read it: the real and imaginary part
// of flat element f (plane * csh^2 + row * csh + column) at re[f * stride]
// and im[f * stride].  Interleaved (the reference's complex array,
// main.cpp:197-201): im = re + 1, stride 2.  Planar (the separate real and
// imaginary cubes read_kernel returns, main.cpp:182-189): stride 1.
template <typename IN>
struct CubeSrc
{
    const IN* re;
    const IN* im;
    int stride;
    __device__ __forceinline__ double real(long long f) const
    {
        return (double)re[f * stride];
    }
    __device__ __forceinline__ double imag(long long f) const
    {
        return (double)im[f * stride];
    }
};

template <typename IN>
CubeSrc<IN> cube_src(const void* re, const void* im)
{
    CubeSrc<IN> c;
    c.re = static_cast<const IN*>(re);
    if (im)
    {
        c.im = static_cast<const IN*>(im);
        c.stride = 1;
    }
    else
    {
        c.im = c.re + 1;
        c.stride = 2;
    }
    return c;
}

// Largest |re| or |im| over each plane's used quadrant [0, E)^2, following
// the reference's flat indexing (an index past the row end reads the next
// row, as oskar_grid_wproj.c:110-116 does).
template <typename IN>
__global__ void plane_maxabs_kernel(const CubeSrc<IN> cube,
                                    const PlaneDesc* __restrict__ planes,
                                    int conv_size_half, float* __restrict__ out)
{
    const int p = blockIdx.x;
    const PlaneDesc d = planes[p];
    const long long base = (long long)p * conv_size_half * conv_size_half;
    float m = 0.f;
    for (int e = threadIdx.x; e < d.extent * d.extent; e += blockDim.x)
    {
        const int xv = e / d.extent, xu = e % d.extent;
        const long long f = base + (long long)xv * conv_size_half + xu;
        m = fmaxf(m, fmaxf(fabsf((float)cube.real(f)),
                           fabsf((float)cube.imag(f))));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    __shared__ float s_m[32];
    if ((threadIdx.x & 31) == 0) s_m[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0)
    {
        float t = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t = fmaxf(t, s_m[w]);
        out[p] = t;
    }
}

template <typename IN, typename KT>
__global__ void relayout_kernel(const CubeSrc<IN> cube,
                                const PlaneDesc* __restrict__ planes,
                                int oversample, int half, int conv_size_half,
                                KT* __restrict__ slabs)
{
    const int p = blockIdx.y;
    const PlaneDesc d = planes[p];
    const long long base = (long long)p * conv_size_half * conv_size_half;
    const int w = 2 * d.support + 1;
    const int total = d.rows * d.pitch;
    const float inv = 1.0f / d.scale;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += gridDim.x * blockDim.x)
    {
        const int row = e / d.pitch, col = e % d.pitch;
        // row = (off_v + H) * W + (j + S)  ->  quadrant row |off_v + j * os|
        const int off_v = row / w - half, j = row % w - d.support;
        const int xv = abs(off_v + j * oversample);
        // column position = (x % os) * L + x / os  <=>
        // x = (pos % L) * os + pos / L
        const int xu = (col % d.L) * oversample + col / d.L;
        double re = 0.0, im = 0.0;
        // Columns past os * L are padding.
        if (col < oversample * d.L && xu < d.extent)
        {
            const long long f = base + (long long)xv * conv_size_half + xu;
            re = cube.real(f);
            im = cube.imag(f);
        }
        slabs[d.offset + e] = Store<KT>::make(re, im, inv);
    }
}

// Norm contribution of one visibility on plane p with offsets (off_u,
// off_v): the real parts of its (2S+1)^2 taps summed in FP64 in the
// reference's order (dv outer, du inner; oskar_grid_wproj.c:104-123), so a
// per-visibility sum is bit-identical to the reference's `sum`.
template <typename IN>
__global__ void norm_table_kernel(const CubeSrc<IN> cube,
                                  const PlaneDesc* __restrict__ planes,
                                  int num_planes, int oversample, int half,
                                  int conv_size_half, double* __restrict__ table)
{
    const int span = 2 * half + 1;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= num_planes * span * span) return;
    const int p = idx / (span * span);
    const int ov = (idx / span) % span - half;
    const int ou = idx % span - half;
    const int s = planes[p].support;
    const long long base = (long long)p * conv_size_half * conv_size_half;
    double acc = 0.0;
    for (int dv = -s; dv <= s; ++dv)
    {
        const long long krow = base +
            (long long)abs(ov + dv * oversample) * conv_size_half;
        for (int du = -s; du <= s; ++du)
            acc += cube.real(krow + abs(ou + du * oversample));
    }
    table[idx] = acc;
}

template <typename IN, typename KT>
void launch_relayout(const oskar_B200Cube* c, const void* conv,
                     const void* conv_im, cudaStream_t st)
{
    dim3 grid(64, c->num_planes);
    relayout_kernel<IN, KT><<<grid, 256, 0, st>>>(
        cube_src<IN>(conv, conv_im),
        static_cast<const PlaneDesc*>(c->d_planes.ptr), c->oversample,
        c->half, c->conv_size_half, static_cast<KT*>(c->d_slabs.ptr));
}

}  // namespace

int cube_build(oskar_B200Cube* c, const void* d_conv, const void* d_conv_im,
               int conv_is_double, cudaStream_t st)
{
    const int P = c->num_planes, os = c->oversample;
    // Slab geometry and offsets (host).
    long long off = 0;
    unsigned max_bytes = 0;
    c->max_block_bytes = 0;
    const size_t align_elems = 16 / c->elem_bytes > 0 ? 16 / c->elem_bytes : 1;
    for (int p = 0; p < P; ++p)
    {
        PlaneDesc& d = c->planes[p];
        d.extent = os * d.support + c->half + 1;
        d.L = (d.extent + os - 1) / os;
        // Rows padded to 4 elements: every W-row block is then a multiple
        // of 16 bytes and starts 16-byte aligned (bulk-copy rules).
        d.pitch = (os * d.L + 3) / 4 * 4;
        d.rows = (2 * c->half + 1) * (2 * d.support + 1);
        const unsigned block = (unsigned)((2 * d.support + 1) * d.pitch *
                                          c->elem_bytes);
        if (block > c->max_block_bytes) c->max_block_bytes = block;
        d.offset = off;
        const size_t elems = (size_t)d.rows * d.pitch;
        const size_t padded = (elems + align_elems - 1) / align_elems *
                              align_elems;
        d.bytes = (unsigned)(padded * c->elem_bytes);
        d.scale = 1.0f;
        off += (long long)padded;
        if (d.bytes > max_bytes) max_bytes = d.bytes;
    }
    c->max_slab_bytes = max_bytes;
    cudaError_t e = c->d_planes.ensure(sizeof(PlaneDesc) * P);
    if (e == cudaSuccess) e = c->d_slabs.ensure((size_t)off * c->elem_bytes);
    if (e == cudaSuccess)
        e = c->d_norm_table.ensure(sizeof(double) * P * (2 * c->half + 1) *
                                   (2 * c->half + 1));
    if (e != cudaSuccess) return status_from_cuda(e);

    const bool scaled = c->kernel_type != OSKAR_B200_KERNEL_NATIVE;
    if (scaled)
    {
        // Per-plane scale so the reduced-precision values use their full
        // range: stored = value / max|value|.
        e = cudaMemcpyAsync(c->d_planes.ptr, c->planes.data(),
                            sizeof(PlaneDesc) * P, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return status_from_cuda(e);
        DeviceBuffer d_max;
        e = d_max.ensure(sizeof(float) * P);
        if (e != cudaSuccess) return status_from_cuda(e);
        if (conv_is_double)
            plane_maxabs_kernel<double><<<P, 256, 0, st>>>(
                cube_src<double>(d_conv, d_conv_im),
                static_cast<const PlaneDesc*>(c->d_planes.ptr),
                c->conv_size_half, static_cast<float*>(d_max.ptr));
        else
            plane_maxabs_kernel<float><<<P, 256, 0, st>>>(
                cube_src<float>(d_conv, d_conv_im),
                static_cast<const PlaneDesc*>(c->d_planes.ptr),
                c->conv_size_half, static_cast<float*>(d_max.ptr));
        std::vector<float> h_max(P);
        e = cudaMemcpyAsync(h_max.data(), d_max.ptr, sizeof(float) * P,
                            cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return status_from_cuda(e);
        for (int p = 0; p < P; ++p)
            c->planes[p].scale = h_max[p] > 0.f ? h_max[p] : 1.0f;
    }
    e = cudaMemcpyAsync(c->d_planes.ptr, c->planes.data(),
                        sizeof(PlaneDesc) * P, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return status_from_cuda(e);

    if (conv_is_double)
    {
        switch (c->kernel_type)
        {
        case OSKAR_B200_KERNEL_F16:
            launch_relayout<double, __half2>(c, d_conv, d_conv_im, st); break;
        case OSKAR_B200_KERNEL_BF16:
            launch_relayout<double, __nv_bfloat162>(c, d_conv, d_conv_im, st); break;
        default:
            if (c->data_is_double) launch_relayout<double, double2>(c, d_conv, d_conv_im, st);
            else launch_relayout<double, float2>(c, d_conv, d_conv_im, st);
        }
    }
    else
    {
        switch (c->kernel_type)
        {
        case OSKAR_B200_KERNEL_F16:
            launch_relayout<float, __half2>(c, d_conv, d_conv_im, st); break;
        case OSKAR_B200_KERNEL_BF16:
            launch_relayout<float, __nv_bfloat162>(c, d_conv, d_conv_im, st); break;
        default:
            if (c->data_is_double) launch_relayout<float, double2>(c, d_conv, d_conv_im, st);
            else launch_relayout<float, float2>(c, d_conv, d_conv_im, st);
        }
    }
    const int span = 2 * c->half + 1;
    const int entries = P * span * span;
    const int blocks = (entries + 127) / 128;
    if (conv_is_double)
        norm_table_kernel<double><<<blocks, 128, 0, st>>>(
            cube_src<double>(d_conv, d_conv_im),
            static_cast<const PlaneDesc*>(c->d_planes.ptr), P, os, c->half,
            c->conv_size_half, static_cast<double*>(c->d_norm_table.ptr));
    else
        norm_table_kernel<float><<<blocks, 128, 0, st>>>(
            cube_src<float>(d_conv, d_conv_im),
            static_cast<const PlaneDesc*>(c->d_planes.ptr), P, os, c->half,
            c->conv_size_half, static_cast<double*>(c->d_norm_table.ptr));
    return status_from_cuda(cudaGetLastError());
}

// Host-side slab geometry of an FP32 cube (the same layout cube_build
// gives), for callers that place the re-laid cube in memory they provide.
size_t static_cube_geometry(int num_planes, const int* support,
                            int oversample, std::vector<PlaneDesc>* planes,
                            unsigned* max_block_bytes)
{
    const int half = (oversample + 1) / 2;
    const int elem = (int)sizeof(float2);
    long long off = 0;
    unsigned max_block = 0;
    planes->assign((size_t)num_planes, PlaneDesc{});
    for (int p = 0; p < num_planes; ++p)
    {
        PlaneDesc& d = (*planes)[p];
        d.support = support[p];
        d.extent = oversample * d.support + half + 1;
        d.L = (d.extent + oversample - 1) / oversample;
        d.pitch = (oversample * d.L + 3) / 4 * 4;
        d.rows = (2 * half + 1) * (2 * d.support + 1);
        const unsigned block = (unsigned)((2 * d.support + 1) * d.pitch * elem);
        if (block > max_block) max_block = block;
        d.offset = off;
        const size_t elems = ((size_t)d.rows * d.pitch + 1) / 2 * 2;
        d.bytes = (unsigned)(elems * elem);
        d.scale = 1.0f;
        off += (long long)elems;
    }
    *max_block_bytes = max_block;
    return (size_t)off * elem;
}

// Re-lays an FP32 cube (device, reference layout) into d_slabs and fills
// the norm table, using only the memory given: d_planes must already hold
// `planes` (see static_cube_geometry).
int static_cube_fill(const float* d_conv, int num_planes, int oversample,
                     int conv_size_half, const PlaneDesc* d_planes,
                     float2* d_slabs, double* d_norm_table, cudaStream_t st)
{
    const int half = (oversample + 1) / 2;
    relayout_kernel<float, float2><<<dim3(64, num_planes), 256, 0, st>>>(
        cube_src<float>(d_conv, nullptr), d_planes, oversample, half,
        conv_size_half, d_slabs);
    const int span = 2 * half + 1;
    const int entries = num_planes * span * span;
    norm_table_kernel<float><<<(entries + 127) / 128, 128, 0, st>>>(
        cube_src<float>(d_conv, nullptr), d_planes, num_planes, oversample,
        half, conv_size_half, d_norm_table);
    return status_from_cuda(cudaGetLastError());
}

}  // namespace b200
