// es_context.cu - the C ABI of include/es_cuda.h: context, grid upload,
// sector setup and the per-field pass (stage a, then stages b+c per
// temperature group).
//
// Host arithmetic that must agree with the reference bit for bit (phase
// angles, velocities, bound angles, sigma prefactors) is compiled for the host
// without FMA contraction (-Xcompiler -ffp-contract=off) and uses the host libm,
// exactly like the reference's CPU code.
#include "es_cuda.h"
#include "es_host_math.h"
#include "es_nvtx.h"
#include "es_internal.h"
#include "es_upload.h"

#include <cfloat>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

namespace {

using es::host::kHALF_PI;

thread_local char g_create_error[512] = "";

}  // namespace

struct es_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    es_sim_desc desc{};
    char err[512] = "";
    int64_t launches = 0;

    // grid
    double2* d_imps = nullptr;
    int64_t imps_cap = 0;
    int64_t n_imps = 0;
    int* d_cell_end = nullptr;
    int64_t cells_cap = 0;
    es_impurity_settings is{};
    uint64_t generation = 0;
    bool has_grid = false;
    es::Staging staging;  // pinned ring for grids uploaded from pageable host memory

    // sector (Simulation::InitSample state)
    es_settings settings{};
    int coherent = 0;
    bool has_sample = false;
    double phi_start = 0, phi_step = 0, area = 0, phi_integrand_factor = 0;

    // per-pass state
    int64_t n_orbits = 0;
    int n_phase = 0;
    int n_pos = 0;
    double* d_lifetimes = nullptr;
    es::PhaseOrbit* d_phase_orbit = nullptr;
    double4* d_orbit_table = nullptr;  // split precision: the pass's per-phase orbit table
    es::PhaseSigma* d_phase_sigma = nullptr;
    unsigned long long* d_metrics = nullptr;
    int* d_error = nullptr;
    double* d_partial = nullptr;
    double* d_sigma = nullptr;        // 2 * kMaxTChunk scratch for blocking calls
    double* h_sigma = nullptr;        // pinned
    double* d_pos = nullptr;          // images: 3 * pos_cap doubles
    int64_t pos_cap = 0;
    double last_w = 0;                // angular speed of the resident lifetimes
    // split precision
    float2* d_imps32 = nullptr;            // cell-local FP32 impurities
    int64_t imps32_cap = 0;
    long long* d_retrace = nullptr;        // orbits for the FP64 re-trace
    unsigned long long* d_retrace_count = nullptr;
    long long retrace_cap = 0;
    es_tuning tuning{es::kLifetimePerThreadDefer};
    int finish_retrace_every = 0;  // es_debug_finish_retrace
    bool lifetimes_valid = false;
    int row0 = 0, row1 = 0;  // start rows [row0, row1) of the passes (es_set_rows); row1 = dim by default
};

namespace {

es_status fail(es_ctx* c, es_status st, const char* fmt, ...)
{
    char* buf = c ? c->err : g_create_error;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, 512, fmt, ap);
    va_end(ap);
    return st;
}

es_status cuda_fail(es_ctx* c, cudaError_t e, const char* what)
{
    const es_status st = (e == cudaErrorMemoryAllocation) ? ES_ERR_OOM : ES_ERR_LAUNCH;
    return fail(c, st, "%s: %s", what, cudaGetErrorString(e));
}

#define ES_CUDA(call, what)                                   \
    do {                                                      \
        cudaError_t e_ = (call);                              \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, what); \
    } while (0)

es_status bind(es_ctx* ctx)
{
    if (!ctx) return ES_ERR_BAD_ARG;
    ES_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    return ES_OK;
}

double integrand_factor(const es_ctx* ctx, double w, double tau)
{
    return es::host::integrand_factor(ctx->settings.particle_speed, ctx->desc.positions_per_row,
                                      ctx->phi_integrand_factor, w, tau);
}

double get_tau(const es_ctx* ctx, double temperature)
{
    return es::host::get_tau(ctx->coherent != 0, ctx->settings.tau, temperature);
}

es_status check_ready(es_ctx* ctx)
{
    if (!ctx->has_grid) return fail(ctx, ES_ERR_NO_GRID, "es_upload_grid has not been called");
    if (!ctx->has_sample) return fail(ctx, ES_ERR_NO_SAMPLE, "es_init_sample has not been called");
    return ES_OK;
}

// Launch constants of one sector pass at field B on the resident grid.
es::LifetimeLaunch make_launch(const es_ctx* ctx, double magnetic_field, double speed, int clockwise, int coherent)
{
    // SimulationCPU::ComputeLifetimes, src/sim/SimulationCPU.cpp:107-108
    const double w = es::host::angular_speed(magnetic_field);
    es::LifetimeLaunch L{};
    L.imps = ctx->d_imps;
    L.cell_end = ctx->d_cell_end;
    L.phase = ctx->d_phase_orbit;
    L.out = ctx->d_lifetimes;
    L.out32 = nullptr;
    L.metrics = ctx->d_metrics;
    L.error = ctx->d_error;
    L.spawn_start = ctx->is.spawn_region_start;
    L.spawn_size = ctx->is.spawn_region_size;
    L.cell_size = ctx->is.cell_size;
    L.imp_radius = ctx->is.impurity_radius;
    L.speed = speed;
    L.radius = speed / w;  // CreateParticle, src/sim/es/lifetime.h:48
    L.radius_sq = L.radius * L.radius;
    L.w = w;
    L.dist = ctx->desc.region_size / (double)(ctx->desc.positions_per_row - 1);
    L.off_x = ctx->desc.grid_cell_size * 0.01;
    L.off_y = ctx->desc.grid_cell_size * 0.005;
    L.n_orbits = (int64_t)(ctx->row1 - ctx->row0) * ctx->desc.positions_per_row * ctx->n_phase;
    L.cpr = ctx->is.cells_per_row;
    L.dim = ctx->desc.positions_per_row;
    L.n_phase = ctx->n_phase;
    L.clockwise = clockwise;
    L.coherent = coherent;
    L.walk_cap = es::host::walk_cap_for(L.radius, L.cell_size);
    L.row0 = ctx->row0;
    L.variant = ctx->tuning.lifetime_variant;
    L.imps32 = ctx->d_imps32;
    L.retrace = ctx->d_retrace;
    L.retrace_count = ctx->d_retrace_count;
    L.retrace_cap = ctx->retrace_cap;
    L.orbit_table = ctx->d_orbit_table;
    L.finish_retrace_every = ctx->finish_retrace_every;
    es::host::split_constants(L);
    return L;
}

// Stage (a) for the whole sector pass at field B.
es_status enqueue_lifetimes(es_ctx* ctx, double magnetic_field)
{
    if (!(magnetic_field > 0.0) || !std::isfinite(magnetic_field))
        return fail(ctx, ES_ERR_BAD_ARG, "magnetic field must be positive and finite (got %g)", magnetic_field);
    const es::LifetimeLaunch L =
        make_launch(ctx, magnetic_field, ctx->settings.particle_speed, ctx->settings.is_clockwise ? 1 : 0, ctx->coherent);
    if (es::split_walk(ctx->desc.precision)) {
        const bool defer = es::host::long_walks(ctx->n_imps, ctx->is.cells_per_row, ctx->is.cell_size,
                                                ctx->is.impurity_radius);
        ctx->lifetimes_valid = false;  // set again once every launch of the pass is made
        ES_CUDA(es::launch_lifetimes_split(L, defer, ctx->stream), "split lifetime kernel launch");
        ctx->launches += defer ? 4 : 3;  // orbit table, lifetime walk, (winner finish,) FP64 re-trace
    } else {
        ctx->lifetimes_valid = false;
        ES_CUDA(es::launch_lifetimes_fp64(L, ctx->stream), "lifetime kernel launch");
        ctx->launches++;
    }
    ctx->last_w = L.w;
    ctx->lifetimes_valid = true;
    return ES_OK;
}

// Every temperature of a call is checked before its first launch, so an
// ES_ERR_BAD_ARG return means nothing of the call was enqueued.
es_status check_temperatures(es_ctx* ctx, const double* temperatures, int32_t n_t)
{
    if (n_t < 0 || (n_t > 0 && !temperatures)) return fail(ctx, ES_ERR_BAD_ARG, "bad temperature list");
    for (int32_t k = 0; k < n_t; k++) {
        const double T = temperatures[k];
        if (!ctx->coherent && !(T > 0.0))
            return fail(ctx, ES_ERR_BAD_ARG, "temperature %g: the incoherent sector needs T > 0", T);
        if (!std::isfinite(T) && !ctx->coherent)
            return fail(ctx, ES_ERR_BAD_ARG, "temperature %g is not finite", T);
    }
    return ES_OK;
}

// Stages (b)+(c) for all temperatures on the resident lifetimes; results to a
// device array of 2*n_t doubles. pos != nullptr also writes the image maps.
es_status enqueue_integrate(es_ctx* ctx, const double* temperatures, int32_t n_t, double* d_out, double* pos)
{
    es_status st = check_temperatures(ctx, temperatures, n_t);
    if (st != ES_OK) return st;
    const double w = ctx->last_w;
    const double w_signed = ctx->settings.is_clockwise ? -w : w;  // SimulationCPU.cpp:108
    for (int32_t t0 = 0; t0 < n_t; t0 += es::kMaxTChunk) {
        const int nc = (n_t - t0) < es::kMaxTChunk ? (n_t - t0) : es::kMaxTChunk;
        es::IntegrateLaunch L{};
        L.lifetimes = ctx->d_lifetimes;
        L.phase = ctx->d_phase_sigma;
        for (int k = 0; k < nc; k++) {
            const double tau = get_tau(ctx, temperatures[t0 + k]);
            L.tau[k] = tau;
            L.max_lt[k] = 15.0 * tau;  // GetDefaultMaxLifetime, Simulation.h:91
            L.inv_tau[k] = 1.0 / tau;
            L.factor[k] = integrand_factor(ctx, w, tau);
        }
        if (pos) {
            L.pos_lt = pos + (int64_t)t0 * ctx->n_pos;
            L.pos_xx = pos + ctx->pos_cap + (int64_t)t0 * ctx->n_pos;
            L.pos_xy = pos + 2 * ctx->pos_cap + (int64_t)t0 * ctx->n_pos;
        }
        L.partial = ctx->d_partial;
        L.sigma_out = d_out + 2 * t0;
        L.w_signed = w_signed;
        L.phi_integrand_factor = ctx->phi_integrand_factor;
        L.dim = ctx->desc.positions_per_row;
        L.n_phase = ctx->n_phase;
        L.n_t = nc;
        L.row0 = ctx->row0;
        L.rows = ctx->row1 - ctx->row0;
        L.n_blocks = es::kIntegrateBlocks;
        L.fp32 = es::fp32_integrand(ctx->desc.precision) ? 1 : 0;
        ES_CUDA(es::launch_integrate(L, ctx->stream), "integration kernel launch");
        ctx->launches += 2;
    }
    return ES_OK;
}

es_status read_device_error(es_ctx* ctx)
{
    int h_err = 0;
    ES_CUDA(es::copy_async(&h_err, ctx->d_error, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream), "error readback");
    ES_CUDA(cudaStreamSynchronize(ctx->stream), "stream synchronize");
    if (h_err) {
        ES_CUDA(cudaMemsetAsync(ctx->d_error, 0, sizeof(int), ctx->stream), "error reset");
        if (h_err & es::kErrRetraceOverflow)
            return fail(ctx, ES_ERR_LAUNCH, "split precision: the FP64 re-trace list overflowed; results are invalid");
        if (h_err & es::kErrWalkCap)
            return fail(ctx, ES_ERR_WALK_CAP, "an orbit exceeded the cell-walk step bound (its lifetime was set to 0)");
        return fail(ctx, ES_ERR_BAD_ARG, "a start position lies outside the impurity grid");
    }
    return ES_OK;
}

es_status read_metrics_into(es_ctx* ctx, es_metrics* out, bool reset)
{
    unsigned long long h[es::kMetCount];
    ES_CUDA(es::copy_async(h, ctx->d_metrics, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream), "metrics readback");
    if (reset) ES_CUDA(cudaMemsetAsync(ctx->d_metrics, 0, sizeof(h), ctx->stream), "metrics reset");
    ES_CUDA(cudaStreamSynchronize(ctx->stream), "stream synchronize");
    if (out) {
        out->cells_passed = (int64_t)h[es::kMetCells];
        out->impurities_tested = (int64_t)h[es::kMetImps];
        out->particles_inside_impurity = (int64_t)h[es::kMetInside];
        out->particles_escaped = (int64_t)h[es::kMetEscaped];
        out->particles_at_bound = (int64_t)h[es::kMetAtBound];
        out->max_impurities_tested = (int64_t)h[es::kMetMaxImps];
        out->max_cells_passed = (int64_t)h[es::kMetMaxCells];
        out->crossings_tested = (int64_t)h[es::kMetCrossings];
        out->start_cell_tests = (int64_t)h[es::kMetStartTests];
        out->retraced_fp64 = (int64_t)h[es::kMetRetraced];
    }
    return ES_OK;
}

es_status ensure_pos(es_ctx* ctx, int32_t n_t)
{
    const int64_t need = (int64_t)n_t * ctx->n_pos;
    if (need <= ctx->pos_cap) return ES_OK;
    if (ctx->d_pos) cudaFree(ctx->d_pos);
    ctx->d_pos = nullptr;
    ctx->pos_cap = 0;
    ES_CUDA(es::dev_malloc(&ctx->d_pos, sizeof(double) * 3 * need), "image buffers");
    ctx->pos_cap = need;
    return ES_OK;
}

void release(es_ctx* ctx)
{
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    cudaFree(ctx->d_imps);
    cudaFree(ctx->d_cell_end);
    cudaFree(ctx->d_lifetimes);
    cudaFree(ctx->d_phase_orbit);
    cudaFree(ctx->d_orbit_table);
    cudaFree(ctx->d_phase_sigma);
    cudaFree(ctx->d_metrics);
    cudaFree(ctx->d_error);
    cudaFree(ctx->d_partial);
    cudaFree(ctx->d_sigma);
    cudaFree(ctx->d_pos);
    cudaFree(ctx->d_imps32);
    cudaFree(ctx->d_retrace);
    cudaFree(ctx->d_retrace_count);
    if (ctx->h_sigma) cudaFreeHost(ctx->h_sigma);
    ctx->staging.release();
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

es_status upload_arrays(es_ctx* ctx, const double* imp_xy, int64_t n_indexed, const int32_t* cell_end,
                        const es_impurity_settings* is, uint64_t generation, cudaMemcpyKind kind);

}  // namespace

extern "C" {

es_status es_create(const es_sim_desc* desc, es_ctx** out)
{
    es::Range nvtx_range("create");
    if (!desc || !out) return fail(nullptr, ES_ERR_BAD_ARG, "null argument");
    *out = nullptr;
    if (desc->positions_per_row < 3 || desc->positions_per_row % 2 == 0)
        return fail(nullptr, ES_ERR_BAD_ARG, "positions_per_row must be odd and >= 3 (got %d)", desc->positions_per_row);
    if (desc->particles_per_quadrant < 3 || desc->particles_per_quadrant % 2 == 0)
        return fail(nullptr, ES_ERR_BAD_ARG, "particles_per_quadrant must be odd and >= 3 (got %d)",
                    desc->particles_per_quadrant);
    if (!(desc->region_size > 0.0) || !(desc->grid_cell_size > 0.0))
        return fail(nullptr, ES_ERR_BAD_ARG, "region_size and grid_cell_size must be positive");
    if (!es::precision_known(desc->precision))
        return fail(nullptr, ES_ERR_BAD_ARG, "unknown precision %d", desc->precision);
    const int64_t n_phase = 4LL * desc->particles_per_quadrant;
    const int64_t n_pos = (int64_t)desc->positions_per_row * desc->positions_per_row;
    if (n_pos > 2000000000LL / 1 || n_pos * n_phase > (1LL << 40))
        return fail(nullptr, ES_ERR_BAD_ARG, "problem too large");

    int n_dev = 0;
    if (cudaGetDeviceCount(&n_dev) != cudaSuccess || n_dev == 0)
        return fail(nullptr, ES_ERR_DEVICE, "no CUDA device is visible");
    if (desc->device_ordinal < 0 || desc->device_ordinal >= n_dev)
        return fail(nullptr, ES_ERR_DEVICE, "device ordinal %d out of range (%d devices)", desc->device_ordinal, n_dev);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, desc->device_ordinal) != cudaSuccess)
        return fail(nullptr, ES_ERR_DEVICE, "cudaGetDeviceProperties failed");
    if (prop.major != 10)
        return fail(nullptr, ES_ERR_DEVICE, "device %d is sm_%d%d; this library is built for sm_100a only",
                    desc->device_ordinal, prop.major, prop.minor);

    es_ctx* ctx = new (std::nothrow) es_ctx();
    if (!ctx) return fail(nullptr, ES_ERR_OOM, "host allocation failed");
    ctx->device = desc->device_ordinal;
    ctx->desc = *desc;
    ctx->n_phase = (int)n_phase;
    ctx->n_pos = (int)n_pos;
    ctx->n_orbits = n_pos * n_phase;
    ctx->row0 = 0;
    ctx->row1 = desc->positions_per_row;

    cudaError_t e = cudaSetDevice(ctx->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = es::dev_malloc(&ctx->d_lifetimes, sizeof(double) * ctx->n_orbits);
    if (e == cudaSuccess) e = es::dev_malloc(&ctx->d_phase_orbit, sizeof(es::PhaseOrbit) * n_phase);
    if (e == cudaSuccess && es::split_walk(desc->precision))
        e = es::dev_malloc(&ctx->d_orbit_table, sizeof(double4) * n_phase);
    if (e == cudaSuccess) e = es::dev_malloc(&ctx->d_phase_sigma, sizeof(es::PhaseSigma) * n_phase);
    if (e == cudaSuccess) e = es::dev_malloc(&ctx->d_metrics, sizeof(unsigned long long) * es::kMetCount);
    if (e == cudaSuccess) e = es::dev_malloc(&ctx->d_error, sizeof(int));
    if (e == cudaSuccess && es::split_walk(desc->precision)) {
        // Re-traced orbits are a small fraction (guard-band decisions); a quarter
        // of the pass is a generous bound, and overflow is reported, not ignored.
        ctx->retrace_cap = ctx->n_orbits / 4 + 1024;
        e = es::dev_malloc(&ctx->d_retrace, sizeof(long long) * ctx->retrace_cap);
        if (e == cudaSuccess) e = es::dev_malloc(&ctx->d_retrace_count, sizeof(unsigned long long));
    }
    if (e == cudaSuccess) e = es::dev_malloc(&ctx->d_partial, sizeof(double) * 2 * es::kMaxTChunk * es::kIntegrateBlocks);
    if (e == cudaSuccess) e = es::dev_malloc(&ctx->d_sigma, sizeof(double) * 2 * es::kMaxTChunk);
    if (e == cudaSuccess) e = es::host_malloc(&ctx->h_sigma, sizeof(double) * 2 * es::kMaxTChunk);
    if (e == cudaSuccess) e = cudaMemsetAsync(ctx->d_metrics, 0, sizeof(unsigned long long) * es::kMetCount, ctx->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(ctx->d_error, 0, sizeof(int), ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        fail(nullptr, e == cudaErrorMemoryAllocation ? ES_ERR_OOM : ES_ERR_LAUNCH, "es_create: %s",
             cudaGetErrorString(e));
        release(ctx);
        return e == cudaErrorMemoryAllocation ? ES_ERR_OOM : ES_ERR_LAUNCH;
    }
    *out = ctx;
    return ES_OK;
}

es_status es_destroy(es_ctx* ctx)
{
    if (!ctx) return ES_ERR_BAD_ARG;
    release(ctx);
    return ES_OK;
}

const char* es_last_error(const es_ctx* ctx) { return ctx ? ctx->err : g_create_error; }

}  // extern "C"

void es::set_global_error(const char* msg) { snprintf(g_create_error, sizeof g_create_error, "%s", msg ? msg : ""); }

namespace {

es_status upload_arrays(es_ctx* ctx, const double* imp_xy, int64_t n_indexed, const int32_t* cell_end,
                        const es_impurity_settings* is, uint64_t generation, cudaMemcpyKind kind)
{
    const int64_t n_cells = (int64_t)is->cells_per_row * is->cells_per_row;
    // Until this upload completes the context holds no usable grid: a failure
    // below leaves it asking for es_upload_grid again, so no launch can pair
    // the old grid's settings with partly replaced arrays.
    ctx->has_grid = false;
    ctx->lifetimes_valid = false;
    if (n_indexed > ctx->imps_cap) {
        cudaFree(ctx->d_imps);
        ctx->d_imps = nullptr;
        ctx->imps_cap = 0;
        ES_CUDA(es::dev_malloc(&ctx->d_imps, sizeof(double2) * (n_indexed > 0 ? n_indexed : 1)), "impurity buffer");
        ctx->imps_cap = n_indexed;
    }
    if (n_cells > ctx->cells_cap) {
        cudaFree(ctx->d_cell_end);
        ctx->d_cell_end = nullptr;
        ctx->cells_cap = 0;
        ES_CUDA(es::dev_malloc(&ctx->d_cell_end, sizeof(int) * n_cells), "cell index buffer");
        ctx->cells_cap = n_cells;
    }
    auto upload = [&](void* dst, const void* src, size_t bytes) {
        return kind == cudaMemcpyHostToDevice ? ctx->staging.h2d(dst, src, bytes, ctx->stream)
                                              : es::copy_async(dst, src, bytes, kind, ctx->stream);
    };
    if (n_indexed > 0) ES_CUDA(upload(ctx->d_imps, imp_xy, sizeof(double2) * n_indexed), "impurity upload");
    ES_CUDA(upload(ctx->d_cell_end, cell_end, sizeof(int) * n_cells), "cell index upload");
    if (es::split_walk(ctx->desc.precision)) {
        if (n_indexed > ctx->imps32_cap) {
            cudaFree(ctx->d_imps32);
            ctx->d_imps32 = nullptr;
            ctx->imps32_cap = 0;
            ES_CUDA(es::dev_malloc(&ctx->d_imps32, sizeof(float2) * (n_indexed > 0 ? n_indexed : 1)), "FP32 impurity buffer");
            ctx->imps32_cap = n_indexed;
        }
        ES_CUDA(es::launch_local_impurities(ctx->d_imps, ctx->d_cell_end, ctx->d_imps32, is->spawn_region_start,
                                            is->cell_size, is->cells_per_row, ctx->stream),
                "FP32 impurity conversion");
        ctx->launches++;
    }
    ES_CUDA(cudaStreamSynchronize(ctx->stream), "grid upload");
    ctx->n_imps = n_indexed;
    ctx->is = *is;
    ctx->generation = generation;
    ctx->has_grid = true;
    ctx->lifetimes_valid = false;
    return ES_OK;
}

}  // namespace

extern "C" {

es_status es_get_tuning(const es_ctx* ctx, es_tuning* out)
{
    if (!ctx || !out) return ES_ERR_BAD_ARG;
    *out = ctx->tuning;
    return ES_OK;
}

es_status es_set_tuning(es_ctx* ctx, const es_tuning* tuning)
{
    if (!ctx || !tuning) return ES_ERR_BAD_ARG;
    if (!es::lifetime_variant_known(tuning->lifetime_variant))
        return fail(ctx, ES_ERR_BAD_ARG, "unknown lifetime variant %d", tuning->lifetime_variant);
    ctx->tuning = *tuning;
    return ES_OK;
}

es_status es_set_rows(es_ctx* ctx, int32_t j0, int32_t j1)
{
    if (!ctx) return ES_ERR_BAD_ARG;
    if (j0 < 0 || j1 <= j0 || j1 > ctx->desc.positions_per_row)
        return fail(ctx, ES_ERR_BAD_ARG, "es_set_rows: rows [%d, %d) outside 0..%d", j0, j1,
                    ctx->desc.positions_per_row);
    ctx->row0 = j0;
    ctx->row1 = j1;
    ctx->lifetimes_valid = false;
    return ES_OK;
}

es_status es_upload_grid(es_ctx* ctx, const double* imp_xy, int64_t n_indexed, const int32_t* cell_end,
                         const es_impurity_settings* is, uint64_t generation)
{
    es::Range nvtx_range("upload_grid");
    es_status st = bind(ctx);
    if (st != ES_OK) return st;
    if (!is || !cell_end || n_indexed < 0 || (n_indexed > 0 && !imp_xy))
        return fail(ctx, ES_ERR_BAD_ARG, "es_upload_grid: null or negative argument");
    if (is->cells_per_row < 1 || !(is->cell_size > 0.0) || !(is->spawn_region_size > 0.0))
        return fail(ctx, ES_ERR_BAD_ARG, "es_upload_grid: invalid impurity settings");
    if (ctx->has_grid && generation != 0 && generation == ctx->generation) return ES_OK;

    const int64_t n_cells = (int64_t)is->cells_per_row * is->cells_per_row;
    // The kernels index impurities through cell_end: validate it once here so
    // that no device load can leave the impurity array.
    int64_t prev = 0;
    for (int64_t c = 0; c < n_cells; c++) {
        if (cell_end[c] < prev) return fail(ctx, ES_ERR_BAD_ARG, "cell index is not monotone at cell %lld", (long long)c);
        prev = cell_end[c];
    }
    if (prev != n_indexed)
        return fail(ctx, ES_ERR_BAD_ARG, "cell index ends at %lld but %lld impurities were given", (long long)prev,
                    (long long)n_indexed);
    return upload_arrays(ctx, imp_xy, n_indexed, cell_end, is, generation, cudaMemcpyHostToDevice);
}

es_status es_upload_dgrid(es_ctx* ctx, const es_dgrid* g)
{
    es::Range nvtx_range("upload_grid");
    es_status st = bind(ctx);
    if (st != ES_OK) return st;
    if (!g) return fail(ctx, ES_ERR_BAD_ARG, "es_upload_dgrid: null grid");
    const double2* imps;
    const int* cell_end;
    int64_t n_indexed;
    es_impurity_settings is;
    uint64_t generation;
    int device;
    es::dgrid_arrays(g, &imps, &cell_end, &n_indexed, &is, &generation, &device);
    if (device != ctx->device)
        return fail(ctx, ES_ERR_BAD_ARG, "es_upload_dgrid: the grid lives on device %d, the context on %d", device,
                    ctx->device);
    if (ctx->has_grid && generation == ctx->generation) return ES_OK;
    // the cell index is monotone and ends at n_indexed by construction
    return upload_arrays(ctx, reinterpret_cast<const double*>(imps), n_indexed, cell_end, &is, generation,
                         cudaMemcpyDeviceToDevice);
}

es_status es_init_sample(es_ctx* ctx, const es_settings* s, int32_t coherent)
{
    es::Range nvtx_range("init_sample");
    es_status st = bind(ctx);
    if (st != ES_OK) return st;
    if (!s) return fail(ctx, ES_ERR_BAD_ARG, "es_init_sample: null settings");
    if (!ctx->has_grid) return fail(ctx, ES_ERR_NO_GRID, "es_upload_grid must precede es_init_sample");
    if (!(s->particle_speed > 0.0)) return fail(ctx, ES_ERR_BAD_ARG, "particle_speed must be positive");
    if (coherent && !(s->tau > 0.0)) return fail(ctx, ES_ERR_BAD_ARG, "tau must be positive");

    // Every start position must lie in the impurity grid (the reference reads
    // out of bounds otherwise). Positions grow monotonically with i, j.
    {
        const int dim = ctx->desc.positions_per_row;
        const double dist = ctx->desc.region_size / (double)(dim - 1);
        const double ox = ctx->desc.grid_cell_size * 0.01, oy = ctx->desc.grid_cell_size * 0.005;
        const double xs[2] = {0.0 * dist + ox, (double)(dim - 1) * dist + ox};
        const double ys[2] = {0.0 * dist + oy, (double)(dim - 1) * dist + oy};
        for (double x : xs)
            for (double y : ys) {
                const int cx = (int)((x - ctx->is.spawn_region_start) / ctx->is.spawn_region_size * (double)ctx->is.cells_per_row);
                const int cy = (int)((y - ctx->is.spawn_region_start) / ctx->is.spawn_region_size * (double)ctx->is.cells_per_row);
                if (cx < 0 || cy < 0 || cx >= ctx->is.cells_per_row || cy >= ctx->is.cells_per_row)
                    return fail(ctx, ES_ERR_BAD_ARG,
                                "start position (%g, %g) lies outside the impurity grid; increase region_extends", x, y);
            }
    }

    ctx->has_sample = false;  // until the phase tables below are on the device
    ctx->lifetimes_valid = false;
    ctx->settings = *s;
    ctx->coherent = coherent ? 1 : 0;

    // Simulation::InitSample, src/sim/Simulation.h:111-126
    const int ppq = ctx->desc.particles_per_quadrant;
    const es::host::Sector sec = es::host::sector(s->alpha, ppq, coherent != 0);
    ctx->area = sec.area;
    ctx->phi_integrand_factor = sec.phi_integrand_factor;
    ctx->phi_start = sec.phi_start;
    ctx->phi_step = sec.phi_step;

    std::vector<es::PhaseOrbit> po((size_t)ctx->n_phase);
    std::vector<es::PhaseSigma> psg((size_t)ctx->n_phase);
    es::host::phase_tables(sec, ppq, s->particle_speed, s->alpha, s->is_clockwise != 0, po.data(), psg.data());
    ES_CUDA(es::copy_async(ctx->d_phase_orbit, po.data(), sizeof(es::PhaseOrbit) * po.size(), cudaMemcpyHostToDevice,
                            ctx->stream),
            "phase table upload");
    ES_CUDA(es::copy_async(ctx->d_phase_sigma, psg.data(), sizeof(es::PhaseSigma) * psg.size(),
                            cudaMemcpyHostToDevice, ctx->stream),
            "phase table upload");
    ES_CUDA(cudaStreamSynchronize(ctx->stream), "phase table upload");
    ctx->has_sample = true;
    ctx->lifetimes_valid = false;
    return ES_OK;
}

es_status es_compute_lifetimes(es_ctx* ctx, double magnetic_field, double* out_lifetimes, es_metrics* out_metrics)
{
    es::Range nvtx_range("lifetimes");
    es_status st = bind(ctx);
    if (st != ES_OK) return st;
    if ((st = check_ready(ctx)) != ES_OK) return st;
    ES_CUDA(cudaMemsetAsync(ctx->d_metrics, 0, sizeof(unsigned long long) * es::kMetCount, ctx->stream), "metrics reset");
    if ((st = enqueue_lifetimes(ctx, magnetic_field)) != ES_OK) return st;
    if (out_lifetimes)
        ES_CUDA(es::copy_async(out_lifetimes, ctx->d_lifetimes, sizeof(double) * ctx->n_orbits, cudaMemcpyDeviceToHost,
                                ctx->stream),
                "lifetime readback");
    if ((st = read_metrics_into(ctx, out_metrics, true)) != ES_OK) return st;
    return read_device_error(ctx);
}

es_status es_read_lifetimes(es_ctx* ctx, int64_t first, int64_t count, double* out)
{
    es_status st = bind(ctx);
    if (st != ES_OK) return st;
    if (!ctx->lifetimes_valid) return fail(ctx, ES_ERR_BAD_ARG, "no resident lifetimes: call es_compute_lifetimes first");
    if (first < 0 || count < 0 || first > ctx->n_orbits || count > ctx->n_orbits - first || (count > 0 && !out))
        return fail(ctx, ES_ERR_BAD_ARG, "es_read_lifetimes: range [%lld, +%lld) outside the %lld orbits of the pass",
                    (long long)first, (long long)count, (long long)ctx->n_orbits);
    if (count == 0) return ES_OK;
    ES_CUDA(es::copy_async(out, ctx->d_lifetimes + first, sizeof(double) * count, cudaMemcpyDeviceToHost, ctx->stream),
            "lifetime readback");
    ES_CUDA(cudaStreamSynchronize(ctx->stream), "lifetime readback");
    return ES_OK;
}

es_status es_derive_temperatures(es_ctx* ctx, const double* temperatures, int32_t n_t, double* out_sigma)
{
    es::Range nvtx_range("temperatures");
    es_status st = bind(ctx);
    if (st != ES_OK) return st;
    if ((st = check_ready(ctx)) != ES_OK) return st;
    if (!ctx->lifetimes_valid) return fail(ctx, ES_ERR_BAD_ARG, "no resident lifetimes: call es_compute_lifetimes first");
    if (n_t > 0 && !out_sigma) return fail(ctx, ES_ERR_BAD_ARG, "bad temperature list");
    if ((st = check_temperatures(ctx, temperatures, n_t)) != ES_OK) return st;
    for (int32_t t0 = 0; t0 < n_t; t0 += es::kMaxTChunk) {
        const int nc = (n_t - t0) < es::kMaxTChunk ? (n_t - t0) : es::kMaxTChunk;
        if ((st = enqueue_integrate(ctx, temperatures + t0, nc, ctx->d_sigma, nullptr)) != ES_OK) return st;
        ES_CUDA(es::copy_async(ctx->h_sigma, ctx->d_sigma, sizeof(double) * 2 * nc, cudaMemcpyDeviceToHost, ctx->stream),
                "sigma readback");
        ES_CUDA(cudaStreamSynchronize(ctx->stream), "sigma readback");
        std::memcpy(out_sigma + 2 * t0, ctx->h_sigma, sizeof(double) * 2 * nc);
    }
    return ES_OK;
}

es_status es_compute_sigmas(es_ctx* ctx, double magnetic_field, const double* temperatures, int32_t n_t,
                            double* out_sigma, es_metrics* out_metrics)
{
    es::Range nvtx_range("compute_sigmas");
    es_status st = bind(ctx);
    if (st != ES_OK) return st;
    if ((st = check_ready(ctx)) != ES_OK) return st;
    if (n_t > 0 && !out_sigma) return fail(ctx, ES_ERR_BAD_ARG, "bad temperature list");
    if ((st = check_temperatures(ctx, temperatures, n_t)) != ES_OK) return st;
    st = es_compute_lifetimes(ctx, magnetic_field, nullptr, out_metrics);
    if (st != ES_OK) return st;
    return es_derive_temperatures(ctx, temperatures, n_t, out_sigma);
}

es_status es_compute_sigmas_images(es_ctx* ctx, double magnetic_field, const double* temperatures, int32_t n_t,
                                   double* out_sigma, double* lifetime_pos, double* sigma_xx_pos,
                                   double* sigma_xy_pos, es_metrics* out_metrics)
{
    es::Range nvtx_range("compute_sigmas_images");
    es_status st = bind(ctx);
    if (st != ES_OK) return st;
    if ((st = check_ready(ctx)) != ES_OK) return st;
    if (n_t < 0 || (n_t > 0 && (!temperatures || !out_sigma || !lifetime_pos || !sigma_xx_pos || !sigma_xy_pos)))
        return fail(ctx, ES_ERR_BAD_ARG, "bad image arguments");
    if (ctx->row0 != 0 || ctx->row1 != ctx->desc.positions_per_row)
        return fail(ctx, ES_ERR_BAD_ARG, "the per-position maps need every start row (es_set_rows)");
    if ((st = check_temperatures(ctx, temperatures, n_t)) != ES_OK) return st;
    st = es_compute_lifetimes(ctx, magnetic_field, nullptr, out_metrics);
    if (st != ES_OK) return st;
    if ((st = ensure_pos(ctx, es::kMaxTChunk)) != ES_OK) return st;
    for (int32_t t0 = 0; t0 < n_t; t0 += es::kMaxTChunk) {
        const int nc = (n_t - t0) < es::kMaxTChunk ? (n_t - t0) : es::kMaxTChunk;
        if ((st = enqueue_integrate(ctx, temperatures + t0, nc, ctx->d_sigma, ctx->d_pos)) != ES_OK) return st;
        const size_t bytes = sizeof(double) * (size_t)nc * ctx->n_pos;
        ES_CUDA(es::copy_async(lifetime_pos + (int64_t)t0 * ctx->n_pos, ctx->d_pos, bytes, cudaMemcpyDeviceToHost,
                                ctx->stream),
                "image readback");
        ES_CUDA(es::copy_async(sigma_xx_pos + (int64_t)t0 * ctx->n_pos, ctx->d_pos + ctx->pos_cap, bytes,
                                cudaMemcpyDeviceToHost, ctx->stream),
                "image readback");
        ES_CUDA(es::copy_async(sigma_xy_pos + (int64_t)t0 * ctx->n_pos, ctx->d_pos + 2 * ctx->pos_cap, bytes,
                                cudaMemcpyDeviceToHost, ctx->stream),
                "image readback");
        ES_CUDA(es::copy_async(ctx->h_sigma, ctx->d_sigma, sizeof(double) * 2 * nc, cudaMemcpyDeviceToHost, ctx->stream),
                "sigma readback");
        ES_CUDA(cudaStreamSynchronize(ctx->stream), "image readback");
        std::memcpy(out_sigma + 2 * t0, ctx->h_sigma, sizeof(double) * 2 * nc);
    }
    return ES_OK;
}

es_status es_enqueue_sigmas(es_ctx* ctx, double magnetic_field, const double* temperatures, int32_t n_t,
                            double* d_out_sigma)
{
    es::Range nvtx_range("enqueue_sigmas");
    es_status st = bind(ctx);
    if (st != ES_OK) return st;
    if ((st = check_ready(ctx)) != ES_OK) return st;
    if (n_t < 0 || (n_t > 0 && (!temperatures || !d_out_sigma))) return fail(ctx, ES_ERR_BAD_ARG, "bad temperature list");
    if ((st = check_temperatures(ctx, temperatures, n_t)) != ES_OK) return st;
    if ((st = enqueue_lifetimes(ctx, magnetic_field)) != ES_OK) return st;
    return enqueue_integrate(ctx, temperatures, n_t, d_out_sigma, nullptr);
}

es_status es_enqueue_derive_temperatures(es_ctx* ctx, const double* temperatures, int32_t n_t, double* d_out_sigma)
{
    es::Range nvtx_range("enqueue_temperatures");
    es_status st = bind(ctx);
    if (st != ES_OK) return st;
    if ((st = check_ready(ctx)) != ES_OK) return st;
    if (!ctx->lifetimes_valid) return fail(ctx, ES_ERR_BAD_ARG, "no resident lifetimes: call es_compute_lifetimes first");
    if (n_t > 0 && !d_out_sigma) return fail(ctx, ES_ERR_BAD_ARG, "bad temperature list");
    return enqueue_integrate(ctx, temperatures, n_t, d_out_sigma, nullptr);
}

es_status es_enqueue_lifetimes(es_ctx* ctx, double magnetic_field)
{
    es::Range nvtx_range("enqueue_lifetimes");
    es_status st = bind(ctx);
    if (st != ES_OK) return st;
    if ((st = check_ready(ctx)) != ES_OK) return st;
    return enqueue_lifetimes(ctx, magnetic_field);
}

es_status es_average_lifetime(es_ctx* ctx, double* out_average)
{
    es::Range nvtx_range("average_lifetime");
    es_status st = bind(ctx);
    if (st != ES_OK) return st;
    if (!out_average) return fail(ctx, ES_ERR_BAD_ARG, "es_average_lifetime: null output");
    if (ctx->row0 != 0 || ctx->row1 != ctx->desc.positions_per_row)
        return fail(ctx, ES_ERR_BAD_ARG, "es_average_lifetime needs every start row (es_set_rows)");
    if (!ctx->lifetimes_valid) return fail(ctx, ES_ERR_BAD_ARG, "no resident lifetimes: call es_compute_lifetimes first");
    ES_CUDA(es::launch_lifetime_sum(ctx->d_lifetimes, ctx->n_orbits, ctx->d_partial, ctx->d_sigma, ctx->stream),
            "lifetime sum");
    ctx->launches += 2;
    ES_CUDA(es::copy_async(ctx->h_sigma, ctx->d_sigma, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream),
            "lifetime sum readback");
    ES_CUDA(cudaStreamSynchronize(ctx->stream), "lifetime sum");
    *out_average = ctx->h_sigma[0] / (double)ctx->n_orbits;  // Simulation::AverageLifetime
    return ES_OK;
}

es_status es_synchronize(es_ctx* ctx)
{
    es_status st = bind(ctx);
    if (st != ES_OK) return st;
    return read_device_error(ctx);
}

es_status es_read_metrics(es_ctx* ctx, es_metrics* out, int32_t reset)
{
    es_status st = bind(ctx);
    if (st != ES_OK) return st;
    return read_metrics_into(ctx, out, reset != 0);
}

void* es_stream(es_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int64_t es_launch_count(const es_ctx* ctx) { return ctx ? ctx->launches : 0; }

es_status es_debug_trace(es_ctx* ctx, double px, double py, int32_t q, int32_t p, double magnetic_field,
                         double phi_start, double phi_step_size, double alpha, double particle_speed,
                         int32_t is_clockwise, int32_t is_coherent, double* out_lifetime)
{
    es_status st = bind(ctx);
    if (st != ES_OK) return st;
    if (!ctx->has_grid) return fail(ctx, ES_ERR_NO_GRID, "es_upload_grid has not been called");
    if (!out_lifetime || !(magnetic_field > 0.0) || !(particle_speed > 0.0))
        return fail(ctx, ES_ERR_BAD_ARG, "es_debug_trace: bad argument");
    const es::LifetimeLaunch L = make_launch(ctx, magnetic_field, particle_speed, is_clockwise ? 1 : 0, is_coherent ? 1 : 0);
    // CreateParticle, src/sim/es/lifetime.h:39-52
    es::PhaseOrbit ph;
    ph.phi = phi_start + q * kHALF_PI + p * phi_step_size;
    ph.vel_x = std::cos(ph.phi) * particle_speed;
    ph.vel_y = std::sin(ph.phi) * particle_speed;
    const double remaining = es::host::smod(ph.phi + alpha, kHALF_PI);
    ph.bound_dphi = is_clockwise ? remaining : (2.0 * alpha - remaining);
    double* d = nullptr;
    ES_CUDA(es::dev_malloc(&d, sizeof(double)), "debug buffer");
    cudaError_t e = es::launch_debug_trace(L, ph, px, py, d, ctx->stream);
    if (e == cudaSuccess) ctx->launches++;
    if (e == cudaSuccess) e = es::copy_async(out_lifetime, d, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(d);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "es_debug_trace");
    if (*out_lifetime < 0.0) return fail(ctx, ES_ERR_BAD_ARG, "es_debug_trace: position outside the impurity grid");
    return ES_OK;
}

es_status es_debug_finish_retrace(es_ctx* ctx, int32_t every)
{
    if (!ctx) return ES_ERR_BAD_ARG;
    if (every < 0) return fail(ctx, ES_ERR_BAD_ARG, "es_debug_finish_retrace: every must be >= 0 (got %d)", every);
    ctx->finish_retrace_every = every;
    ctx->lifetimes_valid = false;
    return ES_OK;
}

es_status es_debug_next_cell(es_ctx* ctx, double center_x, double center_y, double radius, int32_t clockwise,
                             double phi, const es_impurity_settings* is, const double* in6, double* out6,
                             int32_t* out_available)
{
    es_status st = bind(ctx);
    if (st != ES_OK) return st;
    if (!is || !in6 || !out6 || !out_available) return fail(ctx, ES_ERR_BAD_ARG, "null argument");
    double* d = nullptr;
    int* d_avail = nullptr;
    ES_CUDA(es::dev_malloc(&d, sizeof(double) * 12), "debug buffers");
    cudaError_t e = es::dev_malloc(&d_avail, sizeof(int));
    if (e == cudaSuccess) e = es::copy_async(d, in6, sizeof(double) * 6, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess)
        e = es::launch_debug_next_cell(center_x, center_y, radius, clockwise, phi, is->spawn_region_start,
                                       is->spawn_region_size, is->cell_size, is->cells_per_row, d, d + 6, d_avail,
                                       ctx->stream);
    if (e == cudaSuccess) ctx->launches++;
    int avail = 0;
    if (e == cudaSuccess) e = es::copy_async(out6, d + 6, sizeof(double) * 6, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = es::copy_async(&avail, d_avail, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(d);
    cudaFree(d_avail);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "es_debug_next_cell");
    *out_available = avail;
    return ES_OK;
}

}  // extern "C"
