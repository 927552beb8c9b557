// Block ingest: visibility blocks in host memory, as the reference's main
// loop reads them (main.cpp:413-535: read a block's coordinates, scale them
// to wavelengths with scale_coords, grid the block), streamed through the
// device.  Each pushed block is copied straight from the caller's buffers to
// one of two device slots on a copy stream; its gridding (with the
// metres-to-wavelengths scaling done inside the prep kernel) runs on the
// workspace's stream as soon as its copy lands.  push() returns once the
// block's copy is complete, so the caller can read the next block into the
// same buffers while this one grids and the next one crosses PCIe.
#include <cmath>
#include <new>

#include "common.cuh"
#include "internal.h"

using namespace b200;

struct oskar_B200Blocks
{
    oskar_B200Workspace* ws = nullptr;
    const oskar_B200Cube* cube = nullptr;
    oskar_B200Options opt{};
    double cell_size_rad = 0.0, w_scale = 0.0;
    int grid_size = 0;
    void* grid = nullptr;
    double* d_norm = nullptr;
    cudaStream_t copy = nullptr;
    struct Slot
    {
        DeviceBuffer uu, vv, ww, vis, weight;
        cudaEvent_t uploaded = nullptr;  // copy stream: data in the slot
        cudaEvent_t consumed = nullptr;  // compute stream: gridding done
        bool used = false;
    } slots[2];
    // [0] skipped points of every block, [1] device status bits of every
    // block, [2 + k] skip count of the block in slot k
    DeviceBuffer acc;
    unsigned long long pushes = 0;
};

namespace {

__global__ void block_accumulate_kernel(unsigned long long* acc, int slot,
                                        const unsigned long long* counters)
{
    acc[0] += acc[2 + slot];
    acc[1] |= counters[CNT_STATUS];
}

int fail(cudaError_t e)
{
    cudaGetLastError();
    return status_from_cuda(e);
}

struct Guard
{
    int prev = -1;
    bool changed = false;
    explicit Guard(int device)
    {
        if (cudaGetDevice(&prev) == cudaSuccess && prev != device)
            changed = cudaSetDevice(device) == cudaSuccess;
    }
    ~Guard()
    {
        if (changed) cudaSetDevice(prev);
    }
};

}  // namespace

extern "C" {

int oskar_b200_blocks_create(oskar_B200Workspace* ws,
                             const oskar_B200Cube* cube,
                             const oskar_B200Options* opt,
                             double cell_size_rad, double w_scale,
                             int grid_size, void* grid, double* d_norm,
                             oskar_B200Blocks** out)
{
    if (!out) return OSKAR_B200_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (!ws || !cube || cube->device != ws->device || !grid ||
        grid_size < 1 || grid_size > 65535)
        return OSKAR_B200_ERR_INVALID_ARGUMENT;
    if (opt)
    {
        const int st = check_options(opt, cube->data_is_double);
        if (st) return st;
    }
    Guard g(ws->device);
    auto* b = new (std::nothrow) oskar_B200Blocks();
    if (!b) return OSKAR_B200_ERR_OUT_OF_MEMORY;
    b->ws = ws;
    b->cube = cube;
    if (opt)
        b->opt = *opt;
    else
        oskar_b200_options_init(&b->opt);
    b->cell_size_rad = cell_size_rad;
    b->w_scale = w_scale;
    b->grid_size = grid_size;
    b->grid = grid;
    b->d_norm = d_norm;
    cudaError_t e = cudaStreamCreateWithFlags(&b->copy, cudaStreamNonBlocking);
    for (auto& s : b->slots)
    {
        if (e == cudaSuccess)
            e = cudaEventCreateWithFlags(&s.uploaded, cudaEventDisableTiming);
        if (e == cudaSuccess)
            e = cudaEventCreateWithFlags(&s.consumed, cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = b->acc.ensure(4 * sizeof(unsigned long long));
    if (e == cudaSuccess)
        e = cudaMemsetAsync(b->acc.ptr, 0, 4 * sizeof(unsigned long long),
                            ws->stream);
    if (e != cudaSuccess)
    {
        oskar_b200_blocks_free(b);
        return fail(e);
    }
    *out = b;
    return OSKAR_B200_OK;
}

int oskar_b200_blocks_push(oskar_B200Blocks* b, size_t num_points,
                           const void* uu, const void* vv, const void* ww,
                           const void* vis, const void* weight,
                           double frequency_hz)
{
    if (!b || num_points >= 0xffffffffull ||
        (num_points && (!uu || !vv || !ww || !vis)) ||
        (num_points && b->opt.apply_weight && !weight) ||
        !(frequency_hz >= 0.0) || !std::isfinite(frequency_hz))
        return OSKAR_B200_ERR_INVALID_ARGUMENT;
    oskar_B200Workspace* ws = b->ws;
    Guard g(ws->device);
    const int k = (int)(b->pushes & 1);
    auto& sl = b->slots[k];
    const size_t n = num_points;
    const size_t elem = b->cube->data_is_double ? sizeof(double) : sizeof(float);
    cudaError_t e = cudaSuccess;
    // The block two pushes ago has finished with this slot's buffers.
    if (sl.used) e = cudaEventSynchronize(sl.consumed);
    if (e == cudaSuccess && n)
    {
        e = sl.uu.ensure(n * elem);
        if (e == cudaSuccess) e = sl.vv.ensure(n * elem);
        if (e == cudaSuccess) e = sl.ww.ensure(n * elem);
        if (e == cudaSuccess) e = sl.vis.ensure(2 * n * elem);
        if (e == cudaSuccess && weight) e = sl.weight.ensure(n * elem);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(sl.uu.ptr, uu, n * elem,
                                cudaMemcpyHostToDevice, b->copy);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(sl.vv.ptr, vv, n * elem,
                                cudaMemcpyHostToDevice, b->copy);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(sl.ww.ptr, ww, n * elem,
                                cudaMemcpyHostToDevice, b->copy);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(sl.vis.ptr, vis, 2 * n * elem,
                                cudaMemcpyHostToDevice, b->copy);
        if (e == cudaSuccess && weight)
            e = cudaMemcpyAsync(sl.weight.ptr, weight, n * elem,
                                cudaMemcpyHostToDevice, b->copy);
    }
    if (e == cudaSuccess) e = cudaEventRecord(sl.uploaded, b->copy);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ws->stream, sl.uploaded, 0);
    if (e != cudaSuccess) return fail(e);
    unsigned long long* acc = static_cast<unsigned long long*>(b->acc.ptr);
    HostJob j{};
    j.cube = b->cube;
    j.num_points = n;
    j.uu = sl.uu.ptr;
    j.vv = sl.vv.ptr;
    j.ww = sl.ww.ptr;
    j.vis = sl.vis.ptr;
    j.weight = weight ? sl.weight.ptr : nullptr;
    j.cell_size_rad = b->cell_size_rad;
    j.w_scale = b->w_scale;
    j.grid_size = b->grid_size;
    j.grid = b->grid;
    j.d_num_skipped = acc + 2 + k;
    j.d_norm = b->d_norm;
    j.frequency_hz = frequency_hz;
    int st = run_batch(ws, &b->opt, 1, &j, ws->stream);
    if (st) return st;
    block_accumulate_kernel<<<1, 1, 0, ws->stream>>>(
        acc, k, static_cast<const unsigned long long*>(ws->counters.ptr));
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaEventRecord(sl.consumed, ws->stream);
    sl.used = true;
    ++b->pushes;
    // The caller may reuse its buffers once the copy has landed.
    if (e == cudaSuccess) e = cudaEventSynchronize(sl.uploaded);
    return e == cudaSuccess ? OSKAR_B200_OK : fail(e);
}

int oskar_b200_blocks_finish(oskar_B200Blocks* b,
                             unsigned long long* num_skipped)
{
    if (!b) return OSKAR_B200_ERR_INVALID_ARGUMENT;
    Guard g(b->ws->device);
    unsigned long long h[2] = {0, 0};
    cudaError_t e = cudaStreamSynchronize(b->ws->stream);
    if (e == cudaSuccess)
        e = cudaMemcpy(h, b->acc.ptr, sizeof(h), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return fail(e);
    if (num_skipped) *num_skipped = h[0];
    if (h[1]) return h[1] & DEV_ERR_TIMEOUT ? OSKAR_B200_ERR_TIMEOUT
                                            : OSKAR_B200_ERR_DEVICE_CHECK;
    return OSKAR_B200_OK;
}

int oskar_b200_blocks_free(oskar_B200Blocks* b)
{
    if (!b) return OSKAR_B200_OK;
    Guard g(b->ws->device);
    if (b->ws->stream) cudaStreamSynchronize(b->ws->stream);
    if (b->copy) cudaStreamSynchronize(b->copy);
    for (auto& s : b->slots)
    {
        if (s.uploaded) cudaEventDestroy(s.uploaded);
        if (s.consumed) cudaEventDestroy(s.consumed);
    }
    if (b->copy) cudaStreamDestroy(b->copy);
    delete b;  // device buffers free themselves
    return OSKAR_B200_OK;
}

}  // extern "C"
