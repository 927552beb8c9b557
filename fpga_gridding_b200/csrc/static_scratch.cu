// Gridding without any device allocation.
//
// Some callers cannot allocate device memory: code running inside a
// pre-allocated memory pool that must not grow, a pipeline whose memory is
// fixed up front by an operator or scheduler, or a thread that must not take
// the allocator's global locks (or trigger the implicit device
// synchronisation cudaMalloc/cudaFree may cause) while other streams run.
// For them, oskar_b200_grid_f_static grids one FP32 job using only a
// scratch area that lives in a file-scope __device__ array of
// kStaticScratchBytes, which the module holds on every device that loads it
// until the process exits.  The caller still passes all inputs and outputs
// as device pointers (and the support array on the host).
//
// The array's name is a host-side stand-in, not a device address: the
// device address is fetched with cudaGetSymbolAddress the first time the
// entry point runs on each device (with that device current) and cached.
// That first call must therefore not happen inside a stream capture.
// Every call uses the same array, and it keeps the previous call's
// contents: the counters and histograms are cleared each call, and two
// calls whose work overlaps on the GPU (different streams, or different
// threads) race on the array, so callers must serialise them.
#include <algorithm>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "grid_romein.cuh"
#include "internal.h"
#include "prep.cuh"

namespace b200 {

size_t static_cube_geometry(int num_planes, const int* support,
                            int oversample, std::vector<PlaneDesc>* planes,
                            unsigned* max_block_bytes);
int static_cube_fill(const float* d_conv, int num_planes, int oversample,
                     int conv_size_half, const PlaneDesc* d_planes,
                     float2* d_slabs, double* d_norm_table, cudaStream_t st);

namespace {

// 64 MiB: about 1.5 million visibilities with a small cube (~41 bytes of
// scratch per visibility plus the re-laid cube).
constexpr size_t kStaticScratchBytes = size_t(64) << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

std::mutex g_addr_mu;
void* g_addr[kMaxDevices] = {};

// Device address of the scratch array on `device` (the current device),
// looked up once per device.
int scratch_address(int device, unsigned char** out)
{
    if (device < 0 || device >= kMaxDevices) return OSKAR_B200_ERR_NO_DEVICE;
    std::lock_guard<std::mutex> lock(g_addr_mu);
    if (!g_addr[device])
    {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess || !p)
        {
            cudaGetLastError();
            return e == cudaSuccess ? OSKAR_B200_ERR_CUDA : status_from_cuda(e);
        }
        g_addr[device] = p;
    }
    *out = static_cast<unsigned char*>(g_addr[device]);
    return OSKAR_B200_OK;
}

// Bump allocator over the scratch array (256-byte aligned regions).  The
// first region is always the counters (CNT_COUNT words), so the status word
// sits at a fixed place whatever the size of the job that carved the rest.
struct Carver
{
    unsigned char* base;
    size_t used = 0;
    template <typename T>
    T* take(size_t bytes)
    {
        T* p = reinterpret_cast<T*>(base + used);
        used += (bytes + 255) / 256 * 256;
        return p;
    }
};

}  // namespace

}  // namespace b200

using namespace b200;

extern "C" int oskar_b200_grid_f_static(
        size_t num_w_planes, const int* support, int oversample,
        int conv_size_half, const float* conv_func, size_t num_points,
        const float* uu, const float* vv, const float* ww, const float* vis,
        float cell_size_rad, float w_scale, int grid_size, float* grid,
        unsigned long long* d_num_skipped, double* d_norm, void* stream)
{
    // Arguments: the same rules as the other entry points.
    if (num_w_planes == 0 || num_w_planes > 4096 || !support || !conv_func ||
        oversample < 1 || oversample > 32 || conv_size_half < 1 ||
        grid_size < 1 || grid_size > 65535 || !grid ||
        num_points >= 0xffffffffull ||
        (num_points && (!uu || !vv || !ww || !vis)))
        return OSKAR_B200_ERR_INVALID_ARGUMENT;
    const int P = (int)num_w_planes, half = (oversample + 1) / 2;
    const long long csh = conv_size_half;
    for (int p = 0; p < P; ++p)
    {
        if (support[p] < 0) return OSKAR_B200_ERR_INVALID_ARGUMENT;
        if (support[p] > 127) return OSKAR_B200_ERR_UNSUPPORTED;
        const long long e = (long long)oversample * support[p] + half;
        if ((long long)p * csh * csh + e * csh + e >= (long long)P * csh * csh)
            return OSKAR_B200_ERR_INVALID_ARGUMENT;
    }
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return OSKAR_B200_ERR_NO_DEVICE;
    int major = 0, num_sms = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device);
    cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device);
    if (major != 10) return OSKAR_B200_ERR_NO_DEVICE;
    KeyLayout kl;
    if (!make_key_layout(grid_size, P, 1, &kl)) return OSKAR_B200_ERR_UNSUPPORTED;

    // Carve the scratch; refuse jobs that do not fit.
    std::vector<PlaneDesc> planes;
    unsigned max_block = 0;
    const size_t slab_bytes = static_cube_geometry(P, support, oversample,
                                                   &planes, &max_block);
    const size_t n = num_points;
    const int bpj = prep_blocks_per_job(n, 1, num_sms);
    const int span = 2 * half + 1;
    unsigned char* base = nullptr;
    int st = scratch_address(device, &base);
    if (st) return st;
    Carver cv{base};
    auto* counters = cv.take<unsigned long long>(8 * CNT_COUNT);
    auto* d_job = cv.take<JobDesc>(sizeof(JobDesc));
    auto* job_skipped = cv.take<unsigned long long>(8);
    auto* d_planes = cv.take<PlaneDesc>(sizeof(PlaneDesc) * P);
    auto* d_support = cv.take<int>(sizeof(int) * P);
    auto* d_norm_table = cv.take<double>(sizeof(double) * P * span * span);
    auto* plane_counts = cv.take<unsigned long long>(8 * (size_t)P);
    auto* partials = cv.take<double>(8 * (size_t)bpj);
    auto* slabs = cv.take<float2>(slab_bytes);
    uint32_t* keys[2] = {cv.take<uint32_t>(4 * n), cv.take<uint32_t>(4 * n)};
    uint32_t* vals[2] = {cv.take<uint32_t>(4 * n), cv.take<uint32_t>(4 * n)};
    auto* rec = cv.take<int4>(16 * n);
    auto* tile_counts = cv.take<uint32_t>(8 * task_tiles(n));
    auto* task_start = cv.take<uint32_t>(4 * (n + 2));
    auto* task_job = cv.take<uint32_t>(4 * (n + 2));
    const size_t tmp = std::max(radix_sort_temp_bytes(n > 0 ? n : 1),
                                scan_temp_bytes(n > 0 ? n : 1));
    void* scan_tmp = cv.take<unsigned char>(tmp);
    if (cv.used > kStaticScratchBytes) return OSKAR_B200_ERR_OVER_BUDGET;
    if (grid_smem_bytes(0, max_block, false) > 227 * 1024)
        return OSKAR_B200_ERR_UNSUPPORTED;

    cudaStream_t s = static_cast<cudaStream_t>(stream);
    for (PlaneDesc& d : planes) d.scale = 1.0f;
    JobDesc jd{};
    jd.uu = uu;
    jd.vv = vv;
    jd.ww = ww;
    jd.vis = vis;
    jd.weight = nullptr;
    jd.grid = grid;
    jd.planes = d_planes;
    jd.slabs = slabs;
    jd.norm_table = d_norm_table;
    jd.support = d_support;
    jd.d_norm = d_norm;
    jd.d_skipped = d_num_skipped;
    jd.grid_scale = (double)grid_size * (double)cell_size_rad;
    jd.w_scale = w_scale;
    jd.grid_scale_f = (float)grid_size * cell_size_rad;
    jd.w_scale_f = w_scale;
    jd.coord_scale = 1.0;       // coordinates are in wavelengths
    jd.coord_scale_f = 1.0f;
    jd.first = 0;
    jd.n = n;
    jd.grid_size = grid_size;
    jd.num_planes = P;
    jd.oversample = oversample;
    jd.half = half;

#define B200_S(expr)                                                 \
    do {                                                             \
        const cudaError_t e_ = (expr);                               \
        if (e_ != cudaSuccess) return status_from_cuda(e_);          \
    } while (0)
    // Small tables from pageable host memory: each copy returns once the
    // host data is staged, so the host vectors may go out of scope.
    B200_S(cudaMemcpyAsync(d_planes, planes.data(), sizeof(PlaneDesc) * P,
                           cudaMemcpyHostToDevice, s));
    const std::vector<int> support_copy(support, support + P);
    B200_S(cudaMemcpyAsync(d_support, support_copy.data(), sizeof(int) * P,
                           cudaMemcpyHostToDevice, s));
    B200_S(cudaMemcpyAsync(d_job, &jd, sizeof(JobDesc),
                           cudaMemcpyHostToDevice, s));
    // The array keeps the last call's contents: clear what accumulates.
    B200_S(cudaMemsetAsync(counters, 0, 8 * CNT_COUNT, s));
    B200_S(cudaMemsetAsync(job_skipped, 0, 8, s));
    B200_S(cudaMemsetAsync(plane_counts, 0, 8 * (size_t)P, s));
    st = static_cube_fill(conv_func, P, oversample, conv_size_half, d_planes,
                          slabs, d_norm_table, s);
    if (st) return st;

    PrepArgs pa{};
    pa.jobs = d_job;
    pa.num_jobs = 1;
    pa.blocks_per_job = bpj;
    pa.max_planes = P;
    pa.apply_weight = 0;
    pa.key = kl;
    pa.rec = rec;
    pa.keys = keys[0];
    pa.vals = vals[0];
    pa.counters = counters;
    pa.job_skipped = job_skipped;
    pa.norm_partials = partials;
    pa.plane_counts = plane_counts;
    if (n > 0)
        B200_S(launch_prep(pa, 0, OSKAR_B200_COORDS_F64, s));
    else
        B200_S(cudaMemsetAsync(partials, 0, 8 * (size_t)bpj, s));
    B200_S(launch_finalize_prep(pa, s));
    if (n == 0) return OSKAR_B200_OK;
    int which = 0;
    B200_S(radix_sort_pairs(keys, vals, n, kl.total_bits + 1, scan_tmp, s,
                            &which, nullptr));
    B200_S(launch_tasks(keys[which], n, counters, 2 * kl.fine_bits,
                        kl.job_shift, kTaskMax, tile_counts, scan_tmp,
                        task_start, task_job, s, nullptr));
    GridArgs ga{};
    ga.order = vals[which];
    ga.rec = rec;
    ga.apply_weight = 0;
    ga.task_start = task_start;
    ga.task_job = task_job;
    ga.jobs = d_job;
    ga.counters = counters;
    ga.comp_radius = 0;
    default_tune_table(ga.cpt);
    int ctas = 0;
    B200_S(launch_grid(ga, 0, OSKAR_B200_KERNEL_NATIVE, max_block, false,
                       false, num_sms, s, &ctas));
    return OSKAR_B200_OK;
}

namespace {

// Device address of the status word of the static counters.
int static_status_word(unsigned long long** word)
{
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return OSKAR_B200_ERR_NO_DEVICE;
    unsigned char* base = nullptr;
    const int st = scratch_address(device, &base);
    if (st) return st;
    *word = reinterpret_cast<unsigned long long*>(base) + CNT_STATUS;
    return OSKAR_B200_OK;
}

}  // namespace

extern "C" int oskar_b200_grid_f_static_status(void* stream, int* status)
{
    if (!status) return OSKAR_B200_ERR_INVALID_ARGUMENT;
    unsigned long long* word = nullptr;
    const int st = static_status_word(&word);
    if (st) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned long long bits = 0;
    B200_S(cudaMemcpyAsync(&bits, word, sizeof(bits), cudaMemcpyDeviceToHost,
                           s));
    B200_S(cudaStreamSynchronize(s));
    *status = bits == 0 ? OSKAR_B200_OK
              : (bits & DEV_ERR_TIMEOUT) ? OSKAR_B200_ERR_TIMEOUT
                                         : OSKAR_B200_ERR_DEVICE_CHECK;
    return OSKAR_B200_OK;
}

extern "C" int oskar_b200_testing_set_static_status(unsigned long long bits,
                                                    void* stream)
{
    unsigned long long* word = nullptr;
    const int st = static_status_word(&word);
    if (st) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // From pageable memory: the copy has staged `bits` when this returns.
    B200_S(cudaMemcpyAsync(word, &bits, sizeof(bits), cudaMemcpyHostToDevice,
                           s));
    return OSKAR_B200_OK;
}
#undef B200_S
