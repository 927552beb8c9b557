/*
 * oracle.c -- CPU restatement of the reference W-projection gridder.
 *
 * TEST INFRASTRUCTURE ONLY: the product library never links or calls this.
 * Compiled with -ffp-contract=off so that every floating-point operation is
 * rounded separately, as in the reference built for plain x86-64 SSE.
 *
 * Algorithm: OxfordSKA/FPGA_Gridding oskar_grid_wproj.c.  For each
 * visibility: map (u, v) to the nearest grid cell, pick the w-plane as
 * round(sqrt(|w| * w_scale)) clamped to the last plane, find the oversampled
 * sub-cell offset, skip the point if its (2S+1)^2 footprint leaves the grid,
 * otherwise add vis * kernel (conjugated for w > 0) into every footprint cell
 * and add the real parts of the kernel taps into norm.
 */
#define _GNU_SOURCE
#include "oracle.h"

#include <fcntl.h>
#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

/* ------------------------------------------------------------------ */
/* Placement: the per-visibility part of oskar_grid_wproj.c:70-101.     */
/* ------------------------------------------------------------------ */

typedef struct
{
    int64_t gu, gv;      /* grid cell of the footprint centre */
    size_t plane;        /* clamped w-plane */
    size_t raw_plane;    /* grid_w before clamping */
    int off_u, off_v;    /* oversampled sub-cell offsets */
    int conj;            /* -1 when w > 0, else +1 */
    int support;         /* support of the plane used */
    int skipped;
} Place;

/* (int)round(x) as the reference computes it on x86-64: values outside the
 * int range (and NaN) become INT_MIN, which cvttsd2si produces. */
static int64_t round_to_int_d(double x)
{
    const double r = round(x);
    if (!(r > -2147483649.0 && r < 2147483648.0)) return INT32_MIN;
    return (int64_t)r;
}

static int64_t round_to_int_f(float x)
{
    const float r = roundf(x);
    if (!(r > -2147483649.0f && r < 2147483648.0f)) return INT32_MIN;
    return (int64_t)r;
}

/* (size_t)round(...) for a non-negative value; non-finite or huge values
 * saturate, and saturated values are clamped to the last plane anyway. */
static size_t plane_from_double(double r)
{
    if (!(r < 4294967296.0)) return (size_t)0xFFFFFFFFu;
    return (size_t)r;
}

static void place_d(size_t num_w_planes, const int* support, int oversample,
        double grid_scale, int grid_size, double w_scale,
        double u, double v, double w, Place* p)
{
    const int grid_centre = grid_size / 2;
    /* oskar_grid_wproj.c:71-77 */
    const double pos_u = -u * grid_scale;
    const double pos_v = v * grid_scale;
    p->conj = (w > 0.0) ? -1 : 1;
    p->raw_plane = plane_from_double(round(sqrt(fabs(w * w_scale))));
    p->gu = round_to_int_d(pos_u) + grid_centre;
    p->gv = round_to_int_d(pos_v) + grid_centre;
    /* oskar_grid_wproj.c:86-87 */
    p->off_u = (int)round_to_int_d((round(pos_u) - pos_u) * oversample);
    p->off_v = (int)round_to_int_d((round(pos_v) - pos_v) * oversample);
    /* oskar_grid_wproj.c:90-93: clamp to the last plane */
    p->plane = p->raw_plane < num_w_planes ? p->raw_plane : num_w_planes - 1;
    p->support = support[p->plane];
    /* oskar_grid_wproj.c:96-101 */
    p->skipped = (p->gu + p->support >= grid_size || p->gu - p->support < 0 ||
            p->gv + p->support >= grid_size || p->gv - p->support < 0);
}

static void place_f(size_t num_w_planes, const int* support, int oversample,
        float grid_scale, int grid_size, float w_scale,
        float u, float v, float w, Place* p)
{
    const int grid_centre = grid_size / 2;
    /* oskar_grid_wproj.c:169-176, all in float */
    const float pos_u = -u * grid_scale;
    const float pos_v = v * grid_scale;
    p->conj = (w > 0.0f) ? -1 : 1;
    p->raw_plane = plane_from_double((double)roundf(sqrtf(fabsf(w * w_scale))));
    p->gu = round_to_int_f(pos_u) + grid_centre;
    p->gv = round_to_int_f(pos_v) + grid_centre;
    /* oskar_grid_wproj.c:195-196 */
    p->off_u = (int)round_to_int_f((roundf(pos_u) - pos_u) * oversample);
    p->off_v = (int)round_to_int_f((roundf(pos_v) - pos_v) * oversample);
    p->plane = p->raw_plane < num_w_planes ? p->raw_plane : num_w_planes - 1;
    p->support = support[p->plane];
    p->skipped = (p->gu + p->support >= grid_size || p->gu - p->support < 0 ||
            p->gv + p->support >= grid_size || p->gv - p->support < 0);
}

/* ------------------------------------------------------------------ */
/* Serial gridders: oskar_grid_wproj.c:39-126 and :128-243.             */
/* ------------------------------------------------------------------ */

void orc_grid_wproj_d(size_t num_w_planes, const int* support, int oversample,
        int conv_size_half, const double* conv_func, size_t num_points,
        const double* uu, const double* vv, const double* ww,
        const double* vis, const double* weight, double cell_size_rad,
        double w_scale, int grid_size, size_t* num_skipped, double* norm,
        double* grid)
{
    const size_t plane_elems = (size_t)conv_size_half * conv_size_half;
    const double grid_scale = grid_size * cell_size_rad;
    size_t n;
    (void)weight; /* the reference hard-codes weight 1 (:80-81) */
    *num_skipped = 0;
    for (n = 0; n < num_points; ++n)
    {
        Place p;
        double tap_sum = 0.0;
        int dv, du;
        place_d(num_w_planes, support, oversample, grid_scale, grid_size,
                w_scale, uu[n], vv[n], ww[n], &p);
        if (p.skipped) { *num_skipped += 1; continue; }
        {
            const double a_re = vis[2 * n], a_im = vis[2 * n + 1];
            const double sgn = (double)p.conj;
            const size_t plane_base = p.plane * plane_elems;
            for (dv = -p.support; dv <= p.support; ++dv)
            {
                const size_t row = (size_t)(p.gv + dv) * (size_t)grid_size;
                const size_t krow = plane_base + (size_t)abs(p.off_v +
                        dv * oversample) * (size_t)conv_size_half;
                for (du = -p.support; du <= p.support; ++du)
                {
                    const size_t ki = 2 * (krow +
                            (size_t)abs(p.off_u + du * oversample));
                    const size_t gi = 2 * (row + (size_t)(p.gu + du));
                    const double k_re = conv_func[ki];
                    const double k_im = conv_func[ki + 1] * sgn;
                    grid[gi]     += (a_re * k_re - a_im * k_im);
                    grid[gi + 1] += (a_im * k_re + a_re * k_im);
                    tap_sum += k_re;
                }
            }
        }
        *norm += tap_sum;
    }
}

/* Weighted FP64 gridding: the weighting of the reference's tiled CUDA
 * gridder (oskar_grid_wproj_gpu.cu.old:718-724 and :965-978 scale each
 * visibility by its weight before the tap loop; :799 and :1261 add the
 * tap sum times the weight to the norm), on the FP64 placement and tap
 * arithmetic of oskar_grid_wproj_d above.  With unit weights it equals
 * orc_grid_wproj_d bit for bit. */
void orc_grid_wproj_weighted_d(size_t num_w_planes, const int* support,
        int oversample, int conv_size_half, const double* conv_func,
        size_t num_points, const double* uu, const double* vv,
        const double* ww, const double* vis, const double* weight,
        double cell_size_rad, double w_scale, int grid_size,
        size_t* num_skipped, double* norm, double* grid)
{
    const size_t plane_elems = (size_t)conv_size_half * conv_size_half;
    const double grid_scale = grid_size * cell_size_rad;
    size_t n;
    *num_skipped = 0;
    for (n = 0; n < num_points; ++n)
    {
        Place p;
        double tap_sum = 0.0;
        int dv, du;
        place_d(num_w_planes, support, oversample, grid_scale, grid_size,
                w_scale, uu[n], vv[n], ww[n], &p);
        if (p.skipped) { *num_skipped += 1; continue; }
        {
            const double w = weight[n];
            const double a_re = vis[2 * n] * w, a_im = vis[2 * n + 1] * w;
            const double sgn = (double)p.conj;
            const size_t plane_base = p.plane * plane_elems;
            for (dv = -p.support; dv <= p.support; ++dv)
            {
                const size_t row = (size_t)(p.gv + dv) * (size_t)grid_size;
                const size_t krow = plane_base + (size_t)abs(p.off_v +
                        dv * oversample) * (size_t)conv_size_half;
                for (du = -p.support; du <= p.support; ++du)
                {
                    const size_t ki = 2 * (krow +
                            (size_t)abs(p.off_u + du * oversample));
                    const size_t gi = 2 * (row + (size_t)(p.gu + du));
                    const double k_re = conv_func[ki];
                    const double k_im = conv_func[ki + 1] * sgn;
                    grid[gi]     += (a_re * k_re - a_im * k_im);
                    grid[gi + 1] += (a_im * k_re + a_re * k_im);
                    tap_sum += k_re;
                }
            }
            *norm += tap_sum * w;
        }
    }
}

void orc_grid_wproj_f(size_t num_w_planes, const int* support, int oversample,
        int conv_size_half, const float* conv_func, size_t num_points,
        const float* uu, const float* vv, const float* ww,
        const float* vis, const float* weight, float cell_size_rad,
        float w_scale, int grid_size, size_t* num_skipped, double* norm,
        float* grid)
{
    const size_t plane_elems = (size_t)conv_size_half * conv_size_half;
    const float grid_scale = grid_size * cell_size_rad;
    size_t n;
    (void)weight;
    *num_skipped = 0;
    for (n = 0; n < num_points; ++n)
    {
        Place p;
        double tap_sum = 0.0;
        int dv, du;
        place_f(num_w_planes, support, oversample, grid_scale, grid_size,
                w_scale, uu[n], vv[n], ww[n], &p);
        if (p.skipped) { *num_skipped += 1; continue; }
        {
            const float a_re = vis[2 * n], a_im = vis[2 * n + 1];
            const float sgn = (float)p.conj;
            const size_t plane_base = p.plane * plane_elems;
            for (dv = -p.support; dv <= p.support; ++dv)
            {
                const size_t row = (size_t)(p.gv + dv) * (size_t)grid_size;
                const size_t krow = plane_base + (size_t)abs(p.off_v +
                        dv * oversample) * (size_t)conv_size_half;
                for (du = -p.support; du <= p.support; ++du)
                {
                    const size_t ki = 2 * (krow +
                            (size_t)abs(p.off_u + du * oversample));
                    const size_t gi = 2 * (row + (size_t)(p.gu + du));
                    const float k_re = conv_func[ki];
                    const float k_im = conv_func[ki + 1] * sgn;
                    grid[gi]     += (a_re * k_re - a_im * k_im);
                    grid[gi + 1] += (a_im * k_re + a_re * k_im);
                    tap_sum += k_re;
                }
            }
        }
        *norm += tap_sum;
    }
}

/* oskar_grid_wproj_f_diagnostics, oskar_grid_wproj.c:245-370: the float
 * gridder of oskar_grid_wproj_f over all num_points, plus hit counts.  For
 * every point (skipped or not), with grid_w = round(sqrt(|w * w_scale|))
 * before clamping and w_support the support of the clamped plane:
 *   num_vis_per_wsupport[w_support] += 1, num_vis_per_wplane[grid_w] += 1
 * (:317-318); for every tap of a kept point, at its grid cell:
 *   num_vis_per_grid += 1, avg_wsupport_per_grid += w_support, then
 *   avg_wsupport_per_grid += grid_w (:358-360: both sums go to the same
 *   array); avg_wplane_per_grid is never written. */
void orc_grid_wproj_f_diagnostics(size_t num_w_planes, const int* support,
        int oversample, int conv_size_half, const float* conv_func,
        size_t num_points, const float* uu, const float* vv,
        const float* ww, const float* vis, const float* weight,
        float cell_size_rad, float w_scale, int grid_size,
        size_t* num_skipped, double* norm, float* grid,
        long long* num_vis_per_wsupport, long long* num_vis_per_wplane,
        long long* num_vis_per_grid, float* avg_wsupport_per_grid,
        float* avg_wplane_per_grid)
{
    const size_t plane_elems = (size_t)conv_size_half * conv_size_half;
    const float grid_scale = grid_size * cell_size_rad;
    size_t n;
    (void)weight;
    (void)avg_wplane_per_grid;
    *num_skipped = 0;
    for (n = 0; n < num_points; ++n)
    {
        Place p;
        double tap_sum = 0.0;
        int dv, du;
        place_f(num_w_planes, support, oversample, grid_scale, grid_size,
                w_scale, uu[n], vv[n], ww[n], &p);
        num_vis_per_wsupport[p.support] += 1;
        num_vis_per_wplane[p.raw_plane] += 1;
        if (p.skipped) { *num_skipped += 1; continue; }
        {
            const float a_re = vis[2 * n], a_im = vis[2 * n + 1];
            const float sgn = (float)p.conj;
            const size_t plane_base = p.plane * plane_elems;
            for (dv = -p.support; dv <= p.support; ++dv)
            {
                const size_t row = (size_t)(p.gv + dv) * (size_t)grid_size;
                const size_t krow = plane_base + (size_t)abs(p.off_v +
                        dv * oversample) * (size_t)conv_size_half;
                for (du = -p.support; du <= p.support; ++du)
                {
                    const size_t ki = 2 * (krow +
                            (size_t)abs(p.off_u + du * oversample));
                    const size_t cell = row + (size_t)(p.gu + du);
                    const float k_re = conv_func[ki];
                    const float k_im = conv_func[ki + 1] * sgn;
                    grid[2 * cell]     += (a_re * k_re - a_im * k_im);
                    grid[2 * cell + 1] += (a_im * k_re + a_re * k_im);
                    num_vis_per_grid[cell] += 1;
                    avg_wsupport_per_grid[cell] += (float)p.support;
                    avg_wsupport_per_grid[cell] += (float)p.raw_plane;
                    tap_sum += k_re;
                }
            }
        }
        *norm += tap_sum;
    }
}

/* ------------------------------------------------------------------ */
/* Placement tuples.                                                    */
/* ------------------------------------------------------------------ */

static int32_t sat32(int64_t x)
{
    return x > INT32_MAX ? INT32_MAX : (x < INT32_MIN ? INT32_MIN : (int32_t)x);
}

static void store_place(const Place* p, size_t n, int32_t* gu, int32_t* gv,
        int32_t* plane, int32_t* raw_plane, int32_t* off_u, int32_t* off_v,
        int8_t* conj, uint8_t* skipped)
{
    gu[n] = sat32(p->gu);
    gv[n] = sat32(p->gv);
    plane[n] = (int32_t)p->plane;
    raw_plane[n] = p->raw_plane > (size_t)INT32_MAX ? INT32_MAX :
            (int32_t)p->raw_plane;
    off_u[n] = p->off_u;
    off_v[n] = p->off_v;
    conj[n] = (int8_t)p->conj;
    skipped[n] = (uint8_t)p->skipped;
}

void orc_vis_place_d(size_t num_w_planes, const int* support, int oversample,
        size_t num_points, const double* uu, const double* vv,
        const double* ww, double cell_size_rad, double w_scale,
        int grid_size, int32_t* gu, int32_t* gv, int32_t* plane,
        int32_t* raw_plane, int32_t* off_u, int32_t* off_v, int8_t* conj,
        uint8_t* skipped)
{
    const double grid_scale = grid_size * cell_size_rad;
    size_t n;
    for (n = 0; n < num_points; ++n)
    {
        Place p;
        place_d(num_w_planes, support, oversample, grid_scale, grid_size,
                w_scale, uu[n], vv[n], ww[n], &p);
        store_place(&p, n, gu, gv, plane, raw_plane, off_u, off_v, conj,
                skipped);
    }
}

void orc_vis_place_f(size_t num_w_planes, const int* support, int oversample,
        size_t num_points, const float* uu, const float* vv, const float* ww,
        float cell_size_rad, float w_scale, int grid_size, int32_t* gu,
        int32_t* gv, int32_t* plane, int32_t* raw_plane, int32_t* off_u,
        int32_t* off_v, int8_t* conj, uint8_t* skipped)
{
    const float grid_scale = grid_size * cell_size_rad;
    size_t n;
    for (n = 0; n < num_points; ++n)
    {
        Place p;
        place_f(num_w_planes, support, oversample, grid_scale, grid_size,
                w_scale, uu[n], vv[n], ww[n], &p);
        store_place(&p, n, gu, gv, plane, raw_plane, off_u, off_v, conj,
                skipped);
    }
}

uint64_t orc_count_taps_d(size_t num_w_planes, const int* support,
        int oversample, size_t num_points, const double* uu,
        const double* vv, const double* ww, double cell_size_rad,
        double w_scale, int grid_size)
{
    const double grid_scale = grid_size * cell_size_rad;
    uint64_t taps = 0;
    size_t n;
    for (n = 0; n < num_points; ++n)
    {
        Place p;
        place_d(num_w_planes, support, oversample, grid_scale, grid_size,
                w_scale, uu[n], vv[n], ww[n], &p);
        if (!p.skipped)
            taps += (uint64_t)(2 * p.support + 1) * (2 * p.support + 1);
    }
    return taps;
}

/* ------------------------------------------------------------------ */
/* Row-band threaded restatement (bit-identical to the serial loop).    */
/* ------------------------------------------------------------------ */

/* Offsets lie in [-half, half] with half = ceil(oversample / 2). */
static int offset_half(int oversample) { return (oversample + 1) / 2; }

typedef struct
{
    /* shared, read-only */
    const Place* place;
    size_t num_points;
    int oversample, conv_size_half, grid_size;
    const void* conv_func;
    const void* vis;
    void* grid;
    int is_double;
    /* this thread's rows [row0, row1) */
    int64_t row0, row1;
} BandJob;

#define BAND_TAPS(T)                                                   \
    {                                                                       \
        const T* cf = (const T*)job->conv_func;                             \
        const T* vs = (const T*)job->vis;                                   \
        T* gr = (T*)job->grid;                                              \
        const size_t plane_elems = (size_t)job->conv_size_half *            \
                job->conv_size_half;                                        \
        size_t n;                                                           \
        for (n = 0; n < job->num_points; ++n)                               \
        {                                                                   \
            const Place* p = &job->place[n];                                \
            int64_t dv_lo, dv_hi, dv;                                       \
            int du;                                                         \
            if (p->skipped) continue;                                       \
            dv_lo = job->row0 - p->gv;                                      \
            dv_hi = job->row1 - 1 - p->gv;                                  \
            if (dv_lo < -p->support) dv_lo = -p->support;                   \
            if (dv_hi > p->support) dv_hi = p->support;                     \
            if (dv_lo > dv_hi) continue;                                    \
            {                                                               \
                const T a_re = vs[2 * n], a_im = vs[2 * n + 1];             \
                const T sgn = (T)p->conj;                                   \
                const size_t plane_base = p->plane * plane_elems;           \
                for (dv = dv_lo; dv <= dv_hi; ++dv)                         \
                {                                                           \
                    const size_t row = (size_t)(p->gv + dv) *               \
                            (size_t)job->grid_size;                         \
                    const size_t krow = plane_base + (size_t)abs(           \
                            p->off_v + (int)dv * job->oversample) *         \
                            (size_t)job->conv_size_half;                    \
                    for (du = -p->support; du <= p->support; ++du)          \
                    {                                                       \
                        const size_t ki = 2 * (krow + (size_t)abs(          \
                                p->off_u + du * job->oversample));          \
                        const size_t gi = 2 * (row + (size_t)(p->gu + du)); \
                        const T k_re = cf[ki];                              \
                        const T k_im = cf[ki + 1] * sgn;                    \
                        gr[gi]     += (a_re * k_re - a_im * k_im);          \
                        gr[gi + 1] += (a_im * k_re + a_re * k_im);          \
                    }                                                       \
                }                                                           \
            }                                                               \
        }                                                                   \
    }

static void* band_worker(void* arg)
{
    const BandJob* job = (const BandJob*)arg;
    if (job->is_double) BAND_TAPS(double)
    else BAND_TAPS(float)
    return NULL;
}

/* Norm contribution of one point: the reference sums the real parts of the
 * taps in (dv outer, du inner) order into a double (oskar_grid_wproj.c:121),
 * which depends only on (plane, off_u, off_v).  Tabulating it in that order
 * gives bit-identical per-point sums. */
static double* norm_table(size_t num_w_planes, const int* support,
        int oversample, int conv_size_half, const void* conv_func,
        int is_double)
{
    const int h = offset_half(oversample);
    const int span = 2 * h + 1;
    const size_t plane_elems = (size_t)conv_size_half * conv_size_half;
    double* t = (double*)calloc(num_w_planes * span * span, sizeof(double));
    size_t pl;
    if (!t) return NULL;
    for (pl = 0; pl < num_w_planes; ++pl)
    {
        int ov, ou, dv, du;
        const int s = support[pl];
        for (ov = -h; ov <= h; ++ov)
            for (ou = -h; ou <= h; ++ou)
            {
                double acc = 0.0;
                for (dv = -s; dv <= s; ++dv)
                {
                    const size_t krow = pl * plane_elems + (size_t)abs(ov +
                            dv * oversample) * (size_t)conv_size_half;
                    for (du = -s; du <= s; ++du)
                    {
                        const size_t ki = 2 * (krow + (size_t)abs(ou +
                                du * oversample));
                        acc += is_double ? ((const double*)conv_func)[ki] :
                                (double)((const float*)conv_func)[ki];
                    }
                }
                t[(pl * span + (ov + h)) * span + (ou + h)] = acc;
            }
    }
    return t;
}

static void banded_common(size_t num_w_planes, const int* support,
        int oversample, int conv_size_half, const void* conv_func,
        size_t num_points, const Place* place, const void* vis,
        int grid_size, size_t* num_skipped, double* norm, void* grid,
        int num_threads, int is_double)
{
    const int h = offset_half(oversample);
    const int span = 2 * h + 1;
    double* table;
    int64_t* row_work;
    pthread_t* th;
    BandJob* jobs;
    size_t n;
    int t;
    int64_t total = 0, acc = 0, row;

    if (num_threads < 1) num_threads = 1;
    if (num_threads > grid_size) num_threads = grid_size > 0 ? grid_size : 1;

    /* num_skipped and norm, in input order. */
    table = norm_table(num_w_planes, support, oversample, conv_size_half,
            conv_func, is_double);
    *num_skipped = 0;
    for (n = 0; n < num_points; ++n)
    {
        const Place* p = &place[n];
        if (p->skipped) { *num_skipped += 1; continue; }
        *norm += table[(p->plane * span + (p->off_v + h)) * span +
                (p->off_u + h)];
    }
    free(table);

    /* Balance bands by the number of tap rows that land in each grid row. */
    row_work = (int64_t*)calloc((size_t)grid_size + 1, sizeof(int64_t));
    for (n = 0; n < num_points; ++n)
    {
        const Place* p = &place[n];
        if (p->skipped) continue;
        row_work[p->gv - p->support] += 2 * p->support + 1;
        row_work[p->gv + p->support + 1] -= 2 * p->support + 1;
    }
    for (row = 0; row < grid_size; ++row)
    {
        acc += row_work[row];
        row_work[row] = acc;  /* per-row work */
        total += acc;
    }
    jobs = (BandJob*)calloc((size_t)num_threads, sizeof(BandJob));
    th = (pthread_t*)calloc((size_t)num_threads, sizeof(pthread_t));
    {
        int64_t r = 0, done = 0;
        for (t = 0; t < num_threads; ++t)
        {
            const int64_t target = (total * (t + 1)) / num_threads;
            jobs[t].row0 = r;
            while (r < grid_size && (done < target || t == num_threads - 1))
                done += row_work[r++];
            jobs[t].row1 = r;
        }
    }
    for (t = 0; t < num_threads; ++t)
    {
        jobs[t].place = place;
        jobs[t].num_points = num_points;
        jobs[t].oversample = oversample;
        jobs[t].conv_size_half = conv_size_half;
        jobs[t].grid_size = grid_size;
        jobs[t].conv_func = conv_func;
        jobs[t].vis = vis;
        jobs[t].grid = grid;
        jobs[t].is_double = is_double;
        pthread_create(&th[t], NULL, band_worker, &jobs[t]);
    }
    for (t = 0; t < num_threads; ++t) pthread_join(th[t], NULL);
    free(th);
    free(jobs);
    free(row_work);
}

void orc_grid_wproj_d_banded(size_t num_w_planes, const int* support,
        int oversample, int conv_size_half, const double* conv_func,
        size_t num_points, const double* uu, const double* vv,
        const double* ww, const double* vis, const double* weight,
        double cell_size_rad, double w_scale, int grid_size,
        size_t* num_skipped, double* norm, double* grid, int num_threads)
{
    const double grid_scale = grid_size * cell_size_rad;
    Place* place = (Place*)malloc((num_points ? num_points : 1) * sizeof(Place));
    size_t n;
    (void)weight;
    for (n = 0; n < num_points; ++n)
        place_d(num_w_planes, support, oversample, grid_scale, grid_size,
                w_scale, uu[n], vv[n], ww[n], &place[n]);
    banded_common(num_w_planes, support, oversample, conv_size_half,
            conv_func, num_points, place, vis, grid_size, num_skipped, norm,
            grid, num_threads, 1);
    free(place);
}

void orc_grid_wproj_f_banded(size_t num_w_planes, const int* support,
        int oversample, int conv_size_half, const float* conv_func,
        size_t num_points, const float* uu, const float* vv,
        const float* ww, const float* vis, const float* weight,
        float cell_size_rad, float w_scale, int grid_size,
        size_t* num_skipped, double* norm, float* grid, int num_threads)
{
    const float grid_scale = grid_size * cell_size_rad;
    Place* place = (Place*)malloc((num_points ? num_points : 1) * sizeof(Place));
    size_t n;
    (void)weight;
    for (n = 0; n < num_points; ++n)
        place_f(num_w_planes, support, oversample, grid_scale, grid_size,
                w_scale, uu[n], vv[n], ww[n], &place[n]);
    banded_common(num_w_planes, support, oversample, conv_size_half,
            conv_func, num_points, place, vis, grid_size, num_skipped, norm,
            grid, num_threads, 0);
    free(place);
}

/* ------------------------------------------------------------------ */
/* Uniform weighting: utils/oskar_grid_weights.c:38-172.                */
/* ------------------------------------------------------------------ */

void orc_grid_weights_write_d(size_t num_points, const double* uu,
        const double* vv, const double* weight, double cell_size_rad,
        int grid_size, size_t* num_skipped, double* grid)
{
    const int centre = grid_size / 2;
    const double scale = grid_size * cell_size_rad;
    size_t n;
    *num_skipped = 0;
    for (n = 0; n < num_points; ++n)
    {
        const int64_t gu = round_to_int_d(-uu[n] * scale) + centre;
        const int64_t gv = round_to_int_d(vv[n] * scale) + centre;
        if (gu >= grid_size || gu < 0 || gv >= grid_size || gv < 0)
        { *num_skipped += 1; continue; }
        grid[(size_t)gv * grid_size + gu] += weight[n];
    }
}

void orc_grid_weights_read_d(size_t num_points, const double* uu,
        const double* vv, const double* weight_in, double* weight_out,
        double cell_size_rad, int grid_size, size_t* num_skipped,
        const double* grid)
{
    const int centre = grid_size / 2;
    const double scale = grid_size * cell_size_rad;
    size_t n;
    *num_skipped = 0;
    for (n = 0; n < num_points; ++n)
    {
        const int64_t gu = round_to_int_d(-uu[n] * scale) + centre;
        const int64_t gv = round_to_int_d(vv[n] * scale) + centre;
        double density;
        if (gu >= grid_size || gu < 0 || gv >= grid_size || gv < 0)
        { *num_skipped += 1; continue; }
        density = grid[(size_t)gv * grid_size + gu];
        weight_out[n] = (density != 0.0) ? weight_in[n] / density : 0.0;
    }
}

void orc_grid_weights_write_f(size_t num_points, const float* uu,
        const float* vv, const float* weight, float cell_size_rad,
        int grid_size, size_t* num_skipped, float* grid)
{
    const int centre = grid_size / 2;
    const float scale = grid_size * cell_size_rad;
    size_t n;
    *num_skipped = 0;
    for (n = 0; n < num_points; ++n)
    {
        const int64_t gu = round_to_int_f(-uu[n] * scale) + centre;
        const int64_t gv = round_to_int_f(vv[n] * scale) + centre;
        if (gu >= grid_size || gu < 0 || gv >= grid_size || gv < 0)
        { *num_skipped += 1; continue; }
        grid[(size_t)gv * grid_size + gu] += weight[n];
    }
}

void orc_grid_weights_read_f(size_t num_points, const float* uu,
        const float* vv, const float* weight_in, float* weight_out,
        float cell_size_rad, int grid_size, size_t* num_skipped,
        const float* grid)
{
    const int centre = grid_size / 2;
    const float scale = grid_size * cell_size_rad;
    size_t n;
    *num_skipped = 0;
    for (n = 0; n < num_points; ++n)
    {
        const int64_t gu = round_to_int_f(-uu[n] * scale) + centre;
        const int64_t gv = round_to_int_f(vv[n] * scale) + centre;
        float density;
        if (gu >= grid_size || gu < 0 || gv >= grid_size || gv < 0)
        { *num_skipped += 1; continue; }
        density = grid[(size_t)gv * grid_size + gu];
        /* the reference compares the float against 0.0 and divides in float */
        weight_out[n] = (density != 0.0) ? weight_in[n] / density : 0.0f;
    }
}

/* ------------------------------------------------------------------ */
/* CPU baseline harness: private-grid threads over contiguous slices.   */
/* ------------------------------------------------------------------ */

static double now_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

typedef struct
{
    int is_double;
    void* fn;
    size_t chunk_points;
    size_t num_w_planes;
    const int* support;
    int oversample, conv_size_half, grid_size;
    const void* conv_func;
    size_t begin, end;
    const void *uu, *vv, *ww, *vis, *weight;
    double cell_size_rad, w_scale;
    void* grid;          /* private grid */
    size_t grid_bytes;
    int failed;
    double norm;
    size_t skipped;      /* net of padding */
    double seconds;
    pthread_barrier_t* barrier;
} TimedJob;

/* One thread's timed run: either a single call over its slice, or
 * consecutive calls of exactly chunk_points points with a padded tail. */
#define TIMED_RUN(T, FNT)                                                    \
    {                                                                        \
        FNT fn = (FNT)job->fn;                                               \
        const T* uu = (const T*)job->uu;                                     \
        const T* vv = (const T*)job->vv;                                     \
        const T* ww = (const T*)job->ww;                                     \
        const T* vis = (const T*)job->vis;                                   \
        const T* wt = (const T*)job->weight;                                 \
        const size_t total = job->end - job->begin;                          \
        const size_t c = job->chunk_points ? job->chunk_points : total;      \
        const size_t tail = c ? total % c : 0;                               \
        T *pu = 0, *pv = 0, *pw = 0, *pz = 0, *pwt = 0;                      \
        size_t done, i, sk = 0;                                              \
        double t0;                                                           \
        if (tail)                                                            \
        {                                                                    \
            /* padding points sit 4 grid widths off-centre: always skipped */\
            const T far_u = (T)(4.0 / job->cell_size_rad);                   \
            pu = (T*)calloc(c, sizeof(T)); pv = (T*)calloc(c, sizeof(T));    \
            pw = (T*)calloc(c, sizeof(T)); pz = (T*)calloc(2 * c, sizeof(T));\
            pwt = (T*)calloc(c, sizeof(T));                                  \
            for (i = 0; i < c; ++i) pu[i] = far_u;                           \
            for (i = 0; i < tail; ++i)                                       \
            {                                                                \
                const size_t s = job->begin + total - tail + i;              \
                pu[i] = uu[s]; pv[i] = vv[s]; pw[i] = ww[s];                 \
                pz[2 * i] = vis[2 * s]; pz[2 * i + 1] = vis[2 * s + 1];      \
                pwt[i] = wt[s];                                              \
            }                                                                \
        }                                                                    \
        pthread_barrier_wait(job->barrier);                                  \
        t0 = now_s();                                                        \
        for (done = 0; c && done + c <= total; done += c)                    \
        {                                                                    \
            const size_t s = job->begin + done;                              \
            fn(job->num_w_planes, job->support, job->oversample,             \
                    job->conv_size_half, (const T*)job->conv_func, c,        \
                    uu + s, vv + s, ww + s, vis + 2 * s, wt + s,             \
                    (T)job->cell_size_rad, (T)job->w_scale, job->grid_size,  \
                    &sk, &job->norm, (T*)job->grid);                         \
            job->skipped += sk;                                              \
        }                                                                    \
        if (tail)                                                            \
        {                                                                    \
            fn(job->num_w_planes, job->support, job->oversample,             \
                    job->conv_size_half, (const T*)job->conv_func, c,        \
                    pu, pv, pw, pz, pwt, (T)job->cell_size_rad,              \
                    (T)job->w_scale, job->grid_size, &sk, &job->norm,        \
                    (T*)job->grid);                                          \
            job->skipped += sk - (c - tail);                                 \
        }                                                                    \
        job->seconds = now_s() - t0;                                         \
        free(pu); free(pv); free(pw); free(pz); free(pwt);                   \
    }

static void* timed_worker(void* arg)
{
    TimedJob* job = (TimedJob*)arg;
    /* Private grid, allocated and zeroed (every page touched) by this
     * thread before the timed region. */
    job->grid = malloc(job->grid_bytes);
    if (job->grid) memset(job->grid, 0, job->grid_bytes);
    if (!job->grid)
    {
        job->failed = 1;
        pthread_barrier_wait(job->barrier);
        return NULL;
    }
    if (job->is_double) TIMED_RUN(double, orc_grid_fn_d)
    else TIMED_RUN(float, orc_grid_fn_f)
    return NULL;
}

static double time_parallel(int is_double, void* fn, int num_threads,
        size_t chunk_points, size_t num_w_planes, const int* support,
        int oversample, int conv_size_half, const void* conv_func,
        size_t num_points, const void* uu, const void* vv, const void* ww,
        const void* vis, const void* weight, double cell_size_rad,
        double w_scale, int grid_size, size_t* skipped_out,
        double* norm_out, void* grid_out)
{
    const size_t elem = is_double ? sizeof(double) : sizeof(float);
    const size_t cells = (size_t)grid_size * (size_t)grid_size;
    TimedJob* jobs;
    pthread_t* th;
    pthread_barrier_t barrier;
    double worst = 0.0;
    int t, saved_stdout = -1, devnull = -1;

    if (num_threads < 1) num_threads = 1;
    jobs = (TimedJob*)calloc((size_t)num_threads, sizeof(TimedJob));
    th = (pthread_t*)calloc((size_t)num_threads, sizeof(pthread_t));
    if (!jobs || !th) { free(jobs); free(th); return -1.0; }
    for (t = 0; t < num_threads; ++t)
    {
        TimedJob* j = &jobs[t];
        j->grid_bytes = 2 * cells * elem;
        j->is_double = is_double;
        j->fn = fn;
        j->chunk_points = chunk_points;
        j->num_w_planes = num_w_planes;
        j->support = support;
        j->oversample = oversample;
        j->conv_size_half = conv_size_half;
        j->grid_size = grid_size;
        j->conv_func = conv_func;
        j->begin = (num_points * (size_t)t) / (size_t)num_threads;
        j->end = (num_points * (size_t)(t + 1)) / (size_t)num_threads;
        j->uu = uu; j->vv = vv; j->ww = ww; j->vis = vis; j->weight = weight;
        j->cell_size_rad = cell_size_rad;
        j->w_scale = w_scale;
        j->barrier = &barrier;
    }
    pthread_barrier_init(&barrier, NULL, (unsigned)num_threads);
    if (chunk_points)
    {
        fflush(stdout);
        saved_stdout = dup(1);
        devnull = open("/dev/null", O_WRONLY);
        if (devnull >= 0) dup2(devnull, 1);
    }
    for (t = 0; t < num_threads; ++t)
        pthread_create(&th[t], NULL, timed_worker, &jobs[t]);
    for (t = 0; t < num_threads; ++t) pthread_join(th[t], NULL);
    if (chunk_points)
    {
        fflush(stdout);
        if (saved_stdout >= 0) { dup2(saved_stdout, 1); close(saved_stdout); }
        if (devnull >= 0) close(devnull);
    }
    pthread_barrier_destroy(&barrier);

    if (skipped_out) *skipped_out = 0;
    if (norm_out) *norm_out = 0.0;
    for (t = 0; t < num_threads; ++t)
        if (jobs[t].failed) worst = -1.0;
    for (t = 0; t < num_threads; ++t)
    {
        TimedJob* j = &jobs[t];
        if (worst < 0.0 || !j->grid) { free(j->grid); continue; }
        if (j->seconds > worst) worst = j->seconds;
        if (skipped_out) *skipped_out += j->skipped;
        if (norm_out) *norm_out += j->norm;
        if (grid_out)
        {
            size_t c;
            if (is_double)
            {
                double* dst = (double*)grid_out;
                const double* src = (const double*)j->grid;
                for (c = 0; c < 2 * cells; ++c) dst[c] += src[c];
            }
            else
            {
                float* dst = (float*)grid_out;
                const float* src = (const float*)j->grid;
                for (c = 0; c < 2 * cells; ++c) dst[c] += src[c];
            }
        }
        free(j->grid);
    }
    free(jobs);
    free(th);
    return worst;
}

double orc_time_parallel_d(orc_grid_fn_d fn, int num_threads,
        size_t chunk_points, size_t num_w_planes, const int* support,
        int oversample, int conv_size_half, const double* conv_func,
        size_t num_points, const double* uu, const double* vv,
        const double* ww, const double* vis, const double* weight,
        double cell_size_rad, double w_scale, int grid_size,
        size_t* skipped_out, double* norm_out, double* grid_out)
{
    return time_parallel(1, (void*)fn, num_threads, chunk_points,
            num_w_planes, support, oversample, conv_size_half, conv_func,
            num_points, uu, vv, ww, vis, weight, cell_size_rad, w_scale,
            grid_size, skipped_out, norm_out, grid_out);
}

double orc_time_parallel_f(orc_grid_fn_f fn, int num_threads,
        size_t chunk_points, size_t num_w_planes, const int* support,
        int oversample, int conv_size_half, const float* conv_func,
        size_t num_points, const float* uu, const float* vv,
        const float* ww, const float* vis, const float* weight,
        float cell_size_rad, float w_scale, int grid_size,
        size_t* skipped_out, double* norm_out, float* grid_out)
{
    return time_parallel(0, (void*)fn, num_threads, chunk_points,
            num_w_planes, support, oversample, conv_size_half, conv_func,
            num_points, uu, vv, ww, vis, weight, (double)cell_size_rad,
            (double)w_scale, grid_size, skipped_out, norm_out, grid_out);
}

/* ------------------------------------------------------------------ */
/* CPU baseline harness for uniform weighting (FP32): the weights write */
/* on private grids over contiguous slices, a parallel sum of the       */
/* private grids, then the read over slices of the summed grid.         */
/* ------------------------------------------------------------------ */

typedef struct
{
    orc_wwrite_fn_f wfn;
    orc_wread_fn_f rfn;
    int t, num_threads;
    size_t begin, end, num_points, cells;
    const float *uu, *vv, *w_in;
    float* w_out;
    float cell_size_rad;
    int grid_size;
    float* grid;            /* private grid */
    float** grids;          /* every thread's private grid */
    float* grid_out;        /* summed grid */
    size_t skipped_w, skipped_r;
    int failed;
    double seconds;
    pthread_barrier_t* barrier;
} WeightsJob;

static void* weights_worker(void* arg)
{
    WeightsJob* job = (WeightsJob*)arg;
    const size_t n = job->end - job->begin;
    size_t c, c0, c1, sk = 0;
    double t0;
    int k;
    job->grid = (float*)malloc(job->cells * sizeof(float));
    if (job->grid) memset(job->grid, 0, job->cells * sizeof(float));
    else job->failed = 1;
    job->grids[job->t] = job->grid;
    pthread_barrier_wait(job->barrier);
    t0 = now_s();
    if (job->grid)
    {
        job->wfn(n, job->uu + job->begin, job->vv + job->begin,
                 job->w_in + job->begin, job->cell_size_rad, job->grid_size,
                 &sk, job->grid);
        job->skipped_w = sk;
    }
    pthread_barrier_wait(job->barrier);
    /* this thread's share of the cells, summed over all private grids in
     * thread order */
    c0 = (job->cells * (size_t)job->t) / (size_t)job->num_threads;
    c1 = (job->cells * (size_t)(job->t + 1)) / (size_t)job->num_threads;
    for (k = 0; k < job->num_threads; ++k)
    {
        const float* src = job->grids[k];
        if (!src) continue;
        for (c = c0; c < c1; ++c) job->grid_out[c] += src[c];
    }
    pthread_barrier_wait(job->barrier);
    job->rfn(n, job->uu + job->begin, job->vv + job->begin,
             job->w_in + job->begin, job->w_out + job->begin,
             job->cell_size_rad, job->grid_size, &sk, job->grid_out);
    job->skipped_r = sk;
    job->seconds = now_s() - t0;
    return NULL;
}

double orc_time_weights_parallel_f(orc_wwrite_fn_f wfn, orc_wread_fn_f rfn,
        int num_threads, size_t num_points, const float* uu, const float* vv,
        const float* w_in, float cell_size_rad, int grid_size,
        float* grid_out, float* w_out, size_t* skipped_w, size_t* skipped_r)
{
    const size_t cells = (size_t)grid_size * (size_t)grid_size;
    WeightsJob* jobs;
    pthread_t* th;
    float** grids;
    pthread_barrier_t barrier;
    double worst = 0.0;
    int t;
    if (num_threads < 1) num_threads = 1;
    jobs = (WeightsJob*)calloc((size_t)num_threads, sizeof(WeightsJob));
    th = (pthread_t*)calloc((size_t)num_threads, sizeof(pthread_t));
    grids = (float**)calloc((size_t)num_threads, sizeof(float*));
    if (!jobs || !th || !grids)
    {
        free(jobs); free(th); free(grids);
        return -1.0;
    }
    pthread_barrier_init(&barrier, NULL, (unsigned)num_threads);
    for (t = 0; t < num_threads; ++t)
    {
        WeightsJob* j = &jobs[t];
        j->wfn = wfn;
        j->rfn = rfn;
        j->t = t;
        j->num_threads = num_threads;
        j->begin = (num_points * (size_t)t) / (size_t)num_threads;
        j->end = (num_points * (size_t)(t + 1)) / (size_t)num_threads;
        j->num_points = num_points;
        j->cells = cells;
        j->uu = uu; j->vv = vv; j->w_in = w_in; j->w_out = w_out;
        j->cell_size_rad = cell_size_rad;
        j->grid_size = grid_size;
        j->grids = grids;
        j->grid_out = grid_out;
        j->barrier = &barrier;
    }
    for (t = 0; t < num_threads; ++t)
        pthread_create(&th[t], NULL, weights_worker, &jobs[t]);
    for (t = 0; t < num_threads; ++t) pthread_join(th[t], NULL);
    pthread_barrier_destroy(&barrier);
    *skipped_w = *skipped_r = 0;
    for (t = 0; t < num_threads; ++t)
    {
        if (jobs[t].failed) worst = -1.0;
        if (worst >= 0.0 && jobs[t].seconds > worst) worst = jobs[t].seconds;
        *skipped_w += jobs[t].skipped_w;
        *skipped_r += jobs[t].skipped_r;
        free(jobs[t].grid);
    }
    free(jobs);
    free(th);
    free(grids);
    return worst;
}

/* ------------------------------------------------------------------ */
/* Coordinate scaling (utils/read_vis.c:51-73).                         */
/* ------------------------------------------------------------------ */

void orc_scale_coords(double freq_hz, int is_double, size_t num_coords,
        void* uu, void* vv, void* ww)
{
    size_t i;
    /* metres to wavelengths: times frequency over the speed of light */
    const double s = freq_hz / 299792458.0;
    if (is_double)
    {
        double* u = (double*)uu; double* v = (double*)vv; double* w = (double*)ww;
        for (i = 0; i < num_coords; ++i)
        {
            u[i] = u[i] * s;
            v[i] = v[i] * s;
            w[i] = w[i] * s;
        }
    }
    else
    {
        const float sf = (float)s;
        float* u = (float*)uu; float* v = (float*)vv; float* w = (float*)ww;
        for (i = 0; i < num_coords; ++i)
        {
            u[i] = u[i] * sf;
            v[i] = v[i] * sf;
            w[i] = w[i] * sf;
        }
    }
}

/* ------------------------------------------------------------------ */
/* Degridding (adjoint of the gridder; see oracle.h).                   */
/* ------------------------------------------------------------------ */

void orc_degrid_wproj_d(size_t num_w_planes, const int* support,
        int oversample, int conv_size_half, const double* conv_func,
        size_t num_points, const double* uu, const double* vv,
        const double* ww, double cell_size_rad, double w_scale,
        int grid_size, const double* grid, size_t* num_skipped,
        double* vis_out)
{
    const size_t plane_elems = (size_t)conv_size_half * conv_size_half;
    const double grid_scale = grid_size * cell_size_rad;
    size_t n;
    *num_skipped = 0;
    for (n = 0; n < num_points; ++n)
    {
        Place p;
        double re = 0.0, im = 0.0;
        int dv, du;
        place_d(num_w_planes, support, oversample, grid_scale, grid_size,
                w_scale, uu[n], vv[n], ww[n], &p);
        if (p.skipped) { *num_skipped += 1; continue; }
        {
            const double sgn = (double)p.conj;
            const size_t plane_base = p.plane * plane_elems;
            for (dv = -p.support; dv <= p.support; ++dv)
            {
                const size_t row = (size_t)(p.gv + dv) * (size_t)grid_size;
                const size_t krow = plane_base + (size_t)abs(p.off_v +
                        dv * oversample) * (size_t)conv_size_half;
                for (du = -p.support; du <= p.support; ++du)
                {
                    const size_t ki = 2 * (krow +
                            (size_t)abs(p.off_u + du * oversample));
                    const size_t gi = 2 * (row + (size_t)(p.gu + du));
                    /* tap value Kt = (k_re, sgn * k_im); add grid * conj(Kt) */
                    const double k_re = conv_func[ki];
                    const double k_im = conv_func[ki + 1] * sgn;
                    const double g_re = grid[gi], g_im = grid[gi + 1];
                    re += g_re * k_re + g_im * k_im;
                    im += g_im * k_re - g_re * k_im;
                }
            }
        }
        vis_out[2 * n] = re;
        vis_out[2 * n + 1] = im;
    }
}
