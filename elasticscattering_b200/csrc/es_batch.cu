// es_batch.cu - batched sweeps: many (sample, field, sector) passes, each with
// its own temperature list, in one replay of a CUDA graph.
//
// Modes (es_batch_mode). ES_BATCH_PASS_KERNELS, the default, records for each
// pass in turn the single-pass path's kernels (es_lifetime_split.cu or
// es_lifetime_fp64.cu, then es_integrate.cu) on shared device scratch: the
// lean lifetime kernel without the integrand is 12-16% faster on B200 than the
// fused kernel below on passes of 129^2 start positions and up, and the 16
// bytes per orbit it moves through HBM are ~1% of its time. ES_BATCH_PERSISTENT
// fuses stages (b) and (c) into one persistent lifetime kernel over every pass,
// as described next; it wins on sweeps of many small passes (the surrogate's
// training runs of 65^2 x 100 orbits), where per-pass launches dominate. Two
// block-per-work-item modes (one grid over every pass, one graph node per pass)
// never won on B200 and were removed.
//
// No reference counterpart: the reference runs one pass at a time
// (SimulationRunner::RunSample, src/SimulationRunner.cpp:103-151, calling
// Simulation::ComputeSigmas per field and sector). Each batched pass computes
// exactly what that call computes -- stage (a) TraceOrbit lifetimes, then per
// temperature GetTruncatedLifetimes / GetSigma / the two Simpson integrals
// (src/sim/Simulation.h:78-91, src/sim/es/util.h:34-46,
// src/sim/SimulationCPU.cpp:178-222) -- with stages (b) and (c) fused into the
// lifetime kernel, so no lifetime is ever written to memory.
//
// Work decomposition. Pass k covers orbits [0, n_k) in the reference's
// [j][i][q][p] order, cut into work items of 32 * chunk_iters consecutive
// orbits. Warps of a persistent grid take work items from one global counter
// (any pass, heaviest passes first), trace 32 orbits per iteration (one per
// lane: 32 phases of one start position), and add each orbit's Simpson-
// weighted Boltzmann kernel value to a lane-private FP64 slot in shared memory.
// At the end of a work item the warp reduces its slots with a fixed shuffle
// tree and adds the sum, rounded to a per-pass fixed-point scale, to the pass's
// 64-bit integer accumulators. Integer addition is associative, so the
// result does not depend on which warp ran which work item: runs are
// bit-reproducible.
//
// Precision ES_PRECISION_SPLIT: stage (a) is the FP32 walk of es_orbit_split.cuh
// (orbits it cannot settle are re-traced in FP64 on the spot, by the same lane);
// the Boltzmann kernel is evaluated in FP32 in a cancellation-free form (below);
// the orbit phase (phi + w t) is accumulated and reduced in FP64, and every sum
// is FP64. ES_PRECISION_FP64: stage (a) is the plain FP64 TraceOrbit and the
// Boltzmann kernel is the FP64 expression of the per-pass path (es_integrate.cu).
#include "es_cuda.h"
#include "es_nvtx.h"
#include "es_host_math.h"
#include "es_orbit_split.cuh"
#include "es_sigma32.cuh"
#include "es_upload.h"

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <new>
#include <numeric>
#include <tuple>
#include <vector>

namespace es {

constexpr int kBatchMaxTau = 4;     // distinct relaxation times per pass
constexpr int kBatchWarps = 8;      // warps per block (256 threads)

// One pass of the batch, as the kernel sees it.
struct __align__(16) BatchInstanceD {
    LifetimeLaunch L;                 // geometry and orbit constants (L.out unused)
    const PhaseSigma* phase_sigma;
    unsigned long long* acc;          // [2 * kBatchMaxTau] fixed-point sums (xx, xy per tau)
    unsigned long long* metrics;      // kMetCount counters of this pass
    long long chunk_begin;            // first work item of this pass
    double fx_scale;                  // fixed-point scale: a power of two
    double w_signed;                  // signed angular speed (SimulationCPU.cpp:108)
    double tau[kBatchMaxTau];
    double inv_tau[kBatchMaxTau];
    double max_lt[kBatchMaxTau];      // 15 tau (GetDefaultMaxLifetime, Simulation.h:91)
    double wtau[kBatchMaxTau];        // w_signed * tau
    int n_tau;
    int pad[3];
};
static_assert(sizeof(BatchInstanceD) % 16 == 0, "instance records are copied as int4");

struct BatchLaunch {
    const BatchInstanceD* inst;
    const long long* chunk_begin;     // n_inst + 1 entries; the last is the work-item count
    const long long* n_inst;          // device scalar, so a captured graph serves any table
    unsigned long long* counter;      // work-item counter, zeroed before each run
    int* error;
    int chunk_iters;
    // split precision: orbits for the FP64 re-trace, as (pass << 40) | orbit
    unsigned long long* retrace;
    unsigned long long* retrace_count;
    long long retrace_cap;
};

constexpr int kRetraceOrbitBits = 40;   // orbit index bits of a re-trace entry (passes < 2^40 orbits)

namespace {

__device__ __forceinline__ double warp_sum_d(double v)
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    return v;
}

// SimpsonWeight, src/sim/es/util.h:24-28
__device__ __forceinline__ double simpson_w(int i, int dim)
{
    const double main_multiplier = (i % 2 == 0) ? 2.0 : 4.0;
    return (i == 0 || i == dim - 1) ? 1.0 : main_multiplier;
}

// GetSigma of pass I's temperature k for one orbit (sigma_fp32).
__device__ __forceinline__ void kernel_fp32(const BatchInstanceD& I, int k, double raw, const PhaseSigma& ph,
                                            float& r_xx, float& r_xy)
{
    sigma_fp32(raw, I.max_lt[k], I.inv_tau[k], I.w_signed, I.wtau[k], ph, r_xx, r_xy);
}

__device__ __forceinline__ void add_kernel_fp32(const BatchInstanceD& I, double raw, const PhaseSigma& ph,
                                                double wgt, double* slots)
{
    const int n_tau = I.n_tau;
#pragma unroll 1
    for (int k = 0; k < n_tau; k++) {
        float r_xx, r_xy;
        kernel_fp32(I, k, raw, ph, r_xx, r_xy);
        slots[(2 * k) * 32] += wgt * (double)r_xx;
        slots[(2 * k + 1) * 32] += wgt * (double)r_xy;
    }
}

// The per-pass path's FP64 expression (es_integrate.cu), orbit by orbit.
__device__ __forceinline__ void add_kernel_fp64(const BatchInstanceD& I, double raw, const PhaseSigma& ph,
                                                double wpos, double* slots)
{
    double sa_raw, ca_raw;
    sincos(ph.phi + I.w_signed * raw, &sa_raw, &ca_raw);
#pragma unroll 1
    for (int k = 0; k < I.n_tau; k++) {
        const bool keep = raw < I.max_lt[k];
        const double lt = keep ? raw : I.max_lt[k];
        double sa = sa_raw, ca = ca_raw;
        if (!keep) sincos(ph.phi + I.w_signed * lt, &sa, &ca);
        const double z = exp(-lt / I.tau[k]);
        double r = ph.cos_phi - ca * z;
        r += I.wtau[k] * sa * z;
        r -= I.wtau[k] * ph.sin_phi;
        slots[(2 * k) * 32] += ((r * ph.cos_phi) * ph.weight) * wpos;
        slots[(2 * k + 1) * 32] += ((r * ph.sin_phi) * ph.weight) * wpos;
    }
}

// Plain FP64 TraceOrbit of orbit g, with the start-cell check.
__device__ __forceinline__ double fp64_lifetime(const LifetimeLaunch& P, long long g, OrbitCounters* cnt, int* flags)
{
    GridD gr;
    gr.imps = P.imps;
    gr.cell_end = P.cell_end;
    gr.start = P.spawn_start;
    gr.size = P.spawn_size;
    gr.cell = P.cell_size;
    gr.imp_r = P.imp_radius;
    gr.cpr = P.cpr;
    dv2 pos;
    const OrbitD o = make_orbit(P, g, pos);
    OrbitCounters c = {0, 0, 0, 0};
    int f = kTraceOk;
    const iv2 c0 = get_cell(pos, gr.start, gr.size, gr.cpr);
    double lt = 0.0;
    if (!within_bounds(c0, gr.cpr)) {
        atomicOr(P.error, kErrStartCell);
    } else {
        lt = trace_orbit(o, pos, o.particle_angle, P.w, gr, P.walk_cap, c, f);
        if (f & kTraceWalkCap) atomicOr(P.error, kErrWalkCap);
    }
    *cnt = c;
    *flags = f;
    return lt;
}

template <int kPrec, int kMinBlocks>
__global__ void __launch_bounds__(kBatchWarps * 32, kMinBlocks) batch_kernel(BatchLaunch B)
{
    __shared__ BatchInstanceD s_inst[kBatchWarps];
    __shared__ double s_acc[kBatchWarps][2 * kBatchMaxTau][32];
    __shared__ unsigned long long s_met[kBatchWarps][kMetCount];

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    BatchInstanceD& I = s_inst[warp];
    double* slots = &s_acc[warp][0][lane];
    unsigned long long* met = s_met[warp];
    const long long n_inst = *B.n_inst;
    const long long n_items = B.chunk_begin[n_inst];
    const long long item_orbits = 32LL * B.chunk_iters;
    long long cur = -1;

    for (;;) {
        long long item = 0;
        if (lane == 0) item = (long long)atomicAdd(B.counter, 1ull);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= n_items) break;
        // the pass holding this item: the last k with chunk_begin[k] <= item
        long long lo = 0, hi = n_inst - 1;
        while (lo < hi) {
            const long long mid = (lo + hi + 1) >> 1;
            if (__ldg(B.chunk_begin + mid) <= item) lo = mid;
            else hi = mid - 1;
        }
        __syncwarp();
        if (lo != cur) {
            const int4* src = reinterpret_cast<const int4*>(B.inst + lo);
            int4* dst = reinterpret_cast<int4*>(&I);
            for (int k = lane; k < (int)(sizeof(BatchInstanceD) / 16); k += 32) dst[k] = src[k];
            cur = lo;
        }
#pragma unroll
        for (int k = 0; k < 2 * kBatchMaxTau; k++) slots[k * 32] = 0.0;
        if (lane < kMetCount) met[lane] = 0ull;
        __syncwarp();

        const long long g0 = (item - I.chunk_begin) * item_orbits;
        for (int it = 0; it < B.chunk_iters; it++) {
            const long long g = g0 + (long long)it * 32 + lane;
            const bool active = g < I.L.n_orbits;
            const unsigned amask = __ballot_sync(0xffffffffu, active);
            if (amask == 0u) break;
            unsigned cells = 0, imps = 0, cross = 0, starts = 0;
            int flags = kTraceOk;
            bool retrace = false;
            if (active) {
                double lt = 0.0;
                if (kPrec == ES_PRECISION_SPLIT) {
                    SplitCounters sc;
                    retrace = split_orbit(SharedFields{&I.L}, g, sc, flags, lt, amask);
                    cells = sc.cells, imps = sc.imps, cross = sc.crossings, starts = sc.start_tests;
                } else {
                    OrbitCounters oc;
                    lt = fp64_lifetime(I.L, g, &oc, &flags);
                    cells = oc.cells, imps = oc.imps, cross = oc.crossings, starts = oc.start_tests;
                }
                if (!retrace) {
                    const int n_phase = I.L.n_phase, dim = I.L.dim;
                    const int v = (int)(g % n_phase);
                    const long long pidx = g / n_phase;
                    const int i = (int)(pidx % dim);
                    const int j = (int)(pidx / dim);
                    const double wpos = simpson_w(j, dim) * simpson_w(i, dim);
                    const PhaseSigma ph = I.phase_sigma[v];
                    if (kPrec == ES_PRECISION_SPLIT) add_kernel_fp32(I, lt, ph, wpos * ph.weight, slots);
                    else add_kernel_fp64(I, lt, ph, wpos, slots);
                }
            }
            if (kPrec == ES_PRECISION_SPLIT) {
                // uncertain orbits go to the FP64 re-trace list (one atomic per warp);
                // the re-trace kernel counts and integrates them
                const unsigned want = __ballot_sync(0xffffffffu, retrace);
                if (want) {
                    unsigned long long base = 0;
                    if (lane == 0) base = atomicAdd(B.retrace_count, (unsigned long long)__popc(want));
                    base = __shfl_sync(0xffffffffu, base, 0);
                    if (retrace) {
                        const unsigned long long slot = base + __popc(want & ((1u << lane) - 1u));
                        if (slot < (unsigned long long)B.retrace_cap)
                            B.retrace[slot] = ((unsigned long long)cur << kRetraceOrbitBits) | (unsigned long long)g;
                        else
                            atomicOr(B.error, kErrRetraceOverflow);
                    }
                }
            }
            const unsigned s_cells = __reduce_add_sync(0xffffffffu, cells);
            const unsigned s_imps = __reduce_add_sync(0xffffffffu, imps);
            const unsigned s_cross = __reduce_add_sync(0xffffffffu, cross);
            const unsigned s_start = __reduce_add_sync(0xffffffffu, starts);
            const unsigned s_inside = __reduce_add_sync(0xffffffffu, (flags & kTraceInside) ? 1u : 0u);
            const unsigned s_escaped = __reduce_add_sync(0xffffffffu, (flags & kTraceEscaped) ? 1u : 0u);
            const unsigned s_bound = __reduce_add_sync(0xffffffffu, (flags & kTraceAtBound) ? 1u : 0u);
            const unsigned m_cells = __reduce_max_sync(0xffffffffu, cells);
            const unsigned m_imps = __reduce_max_sync(0xffffffffu, imps);
            if (lane == 0) {
                met[kMetCells] += s_cells;
                met[kMetImps] += s_imps;
                met[kMetCrossings] += s_cross;
                met[kMetStartTests] += s_start;
                met[kMetInside] += s_inside;
                met[kMetEscaped] += s_escaped;
                met[kMetAtBound] += s_bound;
                met[kMetMaxCells] = max(met[kMetMaxCells], (unsigned long long)m_cells);
                met[kMetMaxImps] = max(met[kMetMaxImps], (unsigned long long)m_imps);
            }
        }
        __syncwarp();

        // Work-item flush: fixed-order tree, then fixed-point integer atomics.
#pragma unroll
        for (int k = 0; k < 2 * kBatchMaxTau; k++) {
            if (k < 2 * I.n_tau) {
                const double sum = warp_sum_d(slots[k * 32]);
                if (lane == 0) {
                    const long long q = __double2ll_rn(sum * I.fx_scale);
                    if (q != 0) atomicAdd(I.acc + k, (unsigned long long)q);
                }
            }
        }
        if (lane < kMetCount) {
            const unsigned long long m = met[lane];
            if (m != 0) {
                if (lane == kMetMaxCells || lane == kMetMaxImps) atomicMax(I.metrics + lane, m);
                else atomicAdd(I.metrics + lane, m);
            }
        }
    }
}

// The listed orbits of a split run, in FP64 (TraceOrbit, src/sim/es/lifetime.h:78-148),
// then integrated like every other orbit. Each warp takes a contiguous slice of
// the list (entries are appended in roughly pass order), its lanes accumulate
// fixed-point sums and metrics per pass and add them when the pass changes.
__global__ void __launch_bounds__(256, 2) batch_retrace_kernel(BatchLaunch B)
{
    const unsigned long long n = min(*B.retrace_count, (unsigned long long)B.retrace_cap);
    const unsigned long long warps = (unsigned long long)gridDim.x * (blockDim.x / 32);
    const unsigned long long wid = (unsigned long long)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    const unsigned long long per = (n + warps - 1) / warps;
    const unsigned long long e_begin = wid * per;
    const unsigned long long e_end = min(n, e_begin + per);
    constexpr unsigned long long kOrbitMask = (1ull << kRetraceOrbitBits) - 1ull;

    long long cur = -1;
    long long acc[2 * kBatchMaxTau];
    unsigned long long m_sum[8], m_cells = 0, m_imps = 0;
    auto flush = [&]() {
        if (cur < 0) return;
        const BatchInstanceD& I = B.inst[cur];
#pragma unroll
        for (int k = 0; k < 2 * kBatchMaxTau; k++)
            if (acc[k] != 0) atomicAdd(I.acc + k, (unsigned long long)acc[k]);
        const int slot[8] = {kMetCells, kMetImps, kMetCrossings, kMetStartTests, kMetInside, kMetEscaped, kMetAtBound,
                             kMetRetraced};
#pragma unroll
        for (int k = 0; k < 8; k++)
            if (m_sum[k] != 0) atomicAdd(I.metrics + slot[k], m_sum[k]);
        if (m_cells) atomicMax(I.metrics + kMetMaxCells, m_cells);
        if (m_imps) atomicMax(I.metrics + kMetMaxImps, m_imps);
    };
    for (unsigned long long e = e_begin + lane; e < e_end; e += 32) {
        const unsigned long long ent = B.retrace[e];
        const long long inst = (long long)(ent >> kRetraceOrbitBits);
        const long long g = (long long)(ent & kOrbitMask);
        if (inst != cur) {
            flush();
            cur = inst;
#pragma unroll
            for (int k = 0; k < 2 * kBatchMaxTau; k++) acc[k] = 0;
#pragma unroll
            for (int k = 0; k < 8; k++) m_sum[k] = 0;
            m_cells = m_imps = 0;
        }
        const BatchInstanceD& I = B.inst[inst];
        OrbitCounters oc;
        int flags = kTraceOk;
        const double lt = fp64_lifetime(I.L, g, &oc, &flags);
        const int v = (int)(g % I.L.n_phase);
        const long long pidx = g / I.L.n_phase;
        const int i = (int)(pidx % I.L.dim);
        const int j = (int)(pidx / I.L.dim);
        const PhaseSigma ph = I.phase_sigma[v];
        const double wgt = simpson_w(j, I.L.dim) * simpson_w(i, I.L.dim) * ph.weight;
#pragma unroll
        for (int k = 0; k < kBatchMaxTau; k++) {
            if (k < I.n_tau) {
                float r_xx, r_xy;
                kernel_fp32(I, k, lt, ph, r_xx, r_xy);
                acc[2 * k] += __double2ll_rn(wgt * (double)r_xx * I.fx_scale);
                acc[2 * k + 1] += __double2ll_rn(wgt * (double)r_xy * I.fx_scale);
            }
        }
        m_sum[0] += (unsigned)oc.cells;
        m_sum[1] += (unsigned)oc.imps;
        m_sum[2] += (unsigned)oc.crossings;
        m_sum[3] += (unsigned)oc.start_tests;
        m_sum[4] += (flags & kTraceInside) ? 1u : 0u;
        m_sum[5] += (flags & kTraceEscaped) ? 1u : 0u;
        m_sum[6] += (flags & kTraceAtBound) ? 1u : 0u;
        m_sum[7] += 1u;
        m_cells = max(m_cells, (unsigned long long)oc.cells);
        m_imps = max(m_imps, (unsigned long long)oc.imps);
    }
    flush();
}

template <int kPrec, int kMinBlocks>
cudaError_t launch_batch_t(const BatchLaunch& B, int n_sm, cudaStream_t s)
{
    batch_kernel<kPrec, kMinBlocks><<<n_sm * kMinBlocks, kBatchWarps * 32, 0, s>>>(B);
    return es::launched(s);
}

// ES_BATCH_PERSISTENT: the one kernel over every pass.
cudaError_t launch_batch(const BatchLaunch& B, int precision, int blocks_per_sm, int n_sm, cudaStream_t s)
{
    if (precision == ES_PRECISION_SPLIT)
        return (blocks_per_sm == 3) ? launch_batch_t<ES_PRECISION_SPLIT, 3>(B, n_sm, s)
                                    : launch_batch_t<ES_PRECISION_SPLIT, 4>(B, n_sm, s);
    return (blocks_per_sm == 3) ? launch_batch_t<ES_PRECISION_FP64, 3>(B, n_sm, s)
                                : launch_batch_t<ES_PRECISION_FP64, 4>(B, n_sm, s);
}

// Split precision: the FP64 re-trace of the run's list.
cudaError_t launch_retrace(const BatchLaunch& B, int n_sm, cudaStream_t s)
{
    batch_retrace_kernel<<<n_sm * 2, 256, 0, s>>>(B);
    return es::launched(s);
}

}  // namespace
}  // namespace es

// ---------------------------------------------------------------------------
// Host side: the es_batch object of include/es_cuda.h.

struct es_batch_grid {
    double2* d_imps = nullptr;
    float2* d_imps32 = nullptr;
    int* d_cell_end = nullptr;
    int64_t n_indexed = 0;
    es_impurity_settings is{};
    int64_t imps_cap = 0, cells_cap = 0;  // allocated impurities and cells
};

struct es_batch_phase {
    es::PhaseOrbit* d_orbit = nullptr;
    es::PhaseSigma* d_sigma = nullptr;
    double phi_integrand_factor = 0;
};

struct es_batch {
    int device = 0;
    int n_sm = 0;
    cudaStream_t stream = nullptr;
    char err[512] = "";
    int64_t launches = 0;
    // measured best on B200 for passes of 129^2 to 513^2 start positions x 516 phases
    // (12-16% ahead of ES_BATCH_PERSISTENT; the autotuner may choose otherwise)
    es_batch_tuning tuning{32, 4, ES_PRECISION_SPLIT, ES_BATCH_PASS_KERNELS};
    std::vector<long long> pass_items;        // work items per pass, kernel order

    std::vector<es_batch_grid> grids;
    // Device memory of the grids es_batch_clear released, reused by the next
    // es_batch_add_grid calls (smallest that fits): a sweep that clears and adds
    // grids of the same sizes every step allocates and frees nothing.
    std::vector<es_batch_grid> spare;
    es::Staging staging;  // pinned ring for grids copied from pageable host memory
    std::map<std::tuple<int, int, double, double, int>, es_batch_phase> phases;  // (ppq, coherent, alpha, speed, cw)

    // instances (caller order) and their host-side constants
    std::vector<es_batch_instance> inst;
    std::vector<int> order;                   // kernel position -> caller index
    std::vector<std::vector<double>> factor;  // per caller instance, per distinct tau
    std::vector<std::vector<int>> t_slot;     // per caller instance, per temperature: distinct-tau slot
    std::vector<double> fx_scale;             // per caller instance
    int64_t total_orbits = 0;
    int64_t total_items = 0;

    // device table: [n_inst (1) | chunk_begin (cap + 1) | pad] then BatchInstanceD[cap]
    int64_t cap = 0;
    unsigned char* h_table = nullptr;  // pinned
    unsigned char* d_table = nullptr;
    size_t table_bytes = 0, inst_offset = 0;
    unsigned long long* d_acc = nullptr;      // cap * 2 * kBatchMaxTau
    unsigned long long* d_metrics = nullptr;  // cap * kMetCount
    unsigned long long* h_acc = nullptr;      // pinned
    unsigned long long* h_metrics = nullptr;  // pinned
    unsigned long long* d_counter = nullptr;
    int* d_error = nullptr;
    int* h_error = nullptr;                   // pinned
    // split precision: FP64 re-trace list (one 8-byte entry per uncertain orbit)
    unsigned long long* d_retrace = nullptr;
    long long retrace_cap = 0;
    unsigned long long* d_retrace_count = nullptr;
    unsigned long long* h_retrace_count = nullptr;  // pinned
    int64_t retrace_regrows = 0;

    // ES_BATCH_PASS_KERNELS: per-pass sigma (cap * 2 * kBatchMaxTau doubles, one
    // slot per distinct tau) and the scratch the single-pass kernels share
    double* d_psigma = nullptr;
    double* h_psigma = nullptr;                // pinned
    double* d_lt = nullptr;                    // one pass's lifetimes
    long long lt_cap = 0;
    double4* d_otab = nullptr;                 // one pass's orbit table (split)
    long long otab_cap = 0;
    double* d_partial = nullptr;               // integration block partials
    std::vector<double> pass_phi_factor;       // per kernel position: the sector's phi_integrand_factor

    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int64_t graph_kernels = 0;                 // kernel nodes of the recorded graph
    bool graph_dirty = true;
    bool has_instances = false;
};

namespace {

es_status bfail(es_batch* b, es_status st, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(b->err, sizeof b->err, fmt, ap);
    va_end(ap);
    return st;
}

es_status bcuda(es_batch* b, cudaError_t e, const char* what)
{
    return bfail(b, e == cudaErrorMemoryAllocation ? ES_ERR_OOM : ES_ERR_LAUNCH, "%s: %s", what,
                 cudaGetErrorString(e));
}

#define ES_BCUDA(call, what)                                  \
    do {                                                      \
        cudaError_t e_ = (call);                              \
        if (e_ != cudaSuccess) return bcuda(b, e_, what);     \
    } while (0)

void drop_graph(es_batch* b)
{
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    b->graph_dirty = true;
}

// The recorded graph no longer matches the batch's buffers or instances: it
// is recorded again before the next launch. The executable graph is kept (and
// never launched meanwhile) so that the new recording can update it in place.
void invalidate_graph(es_batch* b) { b->graph_dirty = true; }

void free_tables(es_batch* b)
{
    cudaFree(b->d_table);
    cudaFree(b->d_acc);
    cudaFree(b->d_metrics);
    if (b->h_table) cudaFreeHost(b->h_table);
    if (b->h_acc) cudaFreeHost(b->h_acc);
    if (b->h_metrics) cudaFreeHost(b->h_metrics);
    cudaFree(b->d_psigma);
    if (b->h_psigma) cudaFreeHost(b->h_psigma);
    b->d_table = b->h_table = nullptr;
    b->d_acc = b->d_metrics = b->h_acc = b->h_metrics = nullptr;
    b->d_psigma = b->h_psigma = nullptr;
    b->cap = 0;
}

void free_pass_scratch(es_batch* b)
{
    cudaFree(b->d_lt);
    cudaFree(b->d_otab);
    cudaFree(b->d_partial);
    b->d_lt = nullptr;
    b->d_otab = nullptr;
    b->d_partial = nullptr;
    b->lt_cap = b->otab_cap = 0;
}

void free_grid(es_batch_grid& g)
{
    cudaFree(g.d_imps);
    cudaFree(g.d_imps32);
    cudaFree(g.d_cell_end);
    g = es_batch_grid{};
}

void free_grids(es_batch* b)
{
    for (auto& g : b->grids) free_grid(g);
    b->grids.clear();
    for (auto& g : b->spare) free_grid(g);
    b->spare.clear();
    for (auto& kv : b->phases) {
        cudaFree(kv.second.d_orbit);
        cudaFree(kv.second.d_sigma);
    }
    b->phases.clear();
}

es_status ensure_capacity(es_batch* b, int64_t n)
{
    if (n <= b->cap) return ES_OK;
    invalidate_graph(b);
    free_tables(b);
    int64_t cap = 64;
    while (cap < n) cap *= 2;
    b->inst_offset = (size_t)((1 + cap + 1) * sizeof(long long) + 255) & ~(size_t)255;
    b->table_bytes = b->inst_offset + sizeof(es::BatchInstanceD) * (size_t)cap;
    ES_BCUDA(es::dev_malloc(&b->d_table, b->table_bytes), "batch table");
    ES_BCUDA(es::host_malloc(&b->h_table, b->table_bytes), "batch table (host)");
    ES_BCUDA(es::dev_malloc(&b->d_acc, sizeof(unsigned long long) * 2 * es::kBatchMaxTau * cap), "batch accumulators");
    ES_BCUDA(es::dev_malloc(&b->d_metrics, sizeof(unsigned long long) * es::kMetCount * cap), "batch metrics");
    ES_BCUDA(es::host_malloc(&b->h_acc, sizeof(unsigned long long) * 2 * es::kBatchMaxTau * cap), "batch accumulators");
    ES_BCUDA(es::host_malloc(&b->h_metrics, sizeof(unsigned long long) * es::kMetCount * cap), "batch metrics");
    ES_BCUDA(es::dev_malloc(&b->d_psigma, sizeof(double) * 2 * es::kBatchMaxTau * cap), "per-pass sigma");
    ES_BCUDA(es::host_malloc(&b->h_psigma, sizeof(double) * 2 * es::kBatchMaxTau * cap), "per-pass sigma (host)");
    std::memset(b->h_table, 0, b->table_bytes);
    b->cap = cap;
    return ES_OK;
}

// Re-trace list of at least `want` entries (the graph records its address).
es_status ensure_retrace(es_batch* b, long long want)
{
    if (want <= b->retrace_cap) return ES_OK;
    invalidate_graph(b);
    cudaFree(b->d_retrace);
    b->d_retrace = nullptr;
    b->retrace_cap = 0;
    ES_BCUDA(es::dev_malloc(&b->d_retrace, sizeof(unsigned long long) * (size_t)want), "re-trace list");
    b->retrace_cap = want;
    return ES_OK;
}

// ES_BATCH_PASS_KERNELS: scratch for the largest pass (allocated before the
// capture; the graph records the addresses).
es_status ensure_pass_scratch(es_batch* b)
{
    const es::BatchInstanceD* hi = reinterpret_cast<const es::BatchInstanceD*>(b->h_table + b->inst_offset);
    long long max_orbits = 1, max_phase = 1;
    for (size_t pos = 0; pos < b->inst.size(); pos++) {
        max_orbits = std::max(max_orbits, hi[pos].L.n_orbits);
        max_phase = std::max(max_phase, (long long)hi[pos].L.n_phase);
    }
    if (max_orbits <= b->lt_cap && max_phase <= b->otab_cap && b->d_partial) return ES_OK;
    invalidate_graph(b);
    free_pass_scratch(b);
    ES_BCUDA(es::dev_malloc(&b->d_lt, sizeof(double) * (size_t)max_orbits), "pass lifetimes");
    ES_BCUDA(es::dev_malloc(&b->d_otab, sizeof(double4) * (size_t)max_phase), "pass orbit table");
    ES_BCUDA(es::dev_malloc(&b->d_partial, sizeof(double) * 2 * es::kMaxTChunk * es::kIntegrateBlocks),
             "integration partials");
    b->lt_cap = max_orbits;
    b->otab_cap = max_phase;
    return ES_OK;
}

int64_t count_kernel_nodes(cudaGraph_t g);

// ES_BATCH_PASS_KERNELS: each pass in turn through the single-pass path's
// kernels -- orbit table, lifetime walk and FP64 re-trace (split), or the FP64
// lifetime kernel, then stages (b)+(c) for the pass's distinct relaxation
// times -- into the pass's metrics slot and sigma slot.
cudaError_t record_pass_kernels(es_batch* b)
{
    const es::BatchInstanceD* hi = reinterpret_cast<const es::BatchInstanceD*>(b->h_table + b->inst_offset);
    cudaError_t e = cudaSuccess;
    for (size_t pos = 0; e == cudaSuccess && pos < b->inst.size(); pos++) {
        const es::BatchInstanceD& d = hi[pos];
        const int k = b->order[pos];
        const es_batch_grid& g = b->grids[(size_t)b->inst[(size_t)k].grid];
        es::LifetimeLaunch L = d.L;
        L.out = b->d_lt;
        L.out32 = nullptr;
        L.metrics = d.metrics;
        L.row0 = 0;
        L.variant = es::kLifetimePerThreadDefer;
        L.retrace = reinterpret_cast<long long*>(b->d_retrace);
        L.retrace_count = b->d_retrace_count;
        L.retrace_cap = b->retrace_cap;
        L.orbit_table = b->d_otab;
        if (es::split_walk(b->tuning.precision))
            e = es::launch_lifetimes_split(
                L, es::host::long_walks(g.n_indexed, g.is.cells_per_row, g.is.cell_size, g.is.impurity_radius),
                b->stream);
        else
            e = es::launch_lifetimes_fp64(L, b->stream);
        if (e != cudaSuccess) break;
        es::IntegrateLaunch I{};
        I.lifetimes = b->d_lt;
        I.phase = d.phase_sigma;
        for (int u = 0; u < d.n_tau; u++) {
            I.tau[u] = d.tau[u];
            I.max_lt[u] = d.max_lt[u];
            I.inv_tau[u] = d.inv_tau[u];
            I.factor[u] = b->factor[(size_t)k][(size_t)u];
        }
        I.partial = b->d_partial;
        I.sigma_out = b->d_psigma + pos * 2 * es::kBatchMaxTau;
        I.w_signed = d.w_signed;
        I.phi_integrand_factor = b->pass_phi_factor[pos];
        I.dim = L.dim;
        I.n_phase = L.n_phase;
        I.n_t = d.n_tau;
        I.n_blocks = es::kIntegrateBlocks;
        I.fp32 = es::fp32_integrand(b->tuning.precision) ? 1 : 0;
        e = es::launch_integrate(I, b->stream);
    }
    return e;
}

// Records the run sequence on the batch stream: table upload, clears, the
// pass kernels, the FP64 re-trace, readbacks.
es_status capture(es_batch* b)
{
    es::Range nvtx_range("batch_record");
    if (b->graph) cudaGraphDestroy(b->graph);
    b->graph = nullptr;
    b->graph_dirty = true;
    es_status st = ES_OK;
    if (b->tuning.mode == ES_BATCH_PASS_KERNELS && (st = ensure_pass_scratch(b)) != ES_OK) return st;
    const int64_t cap = b->cap;
    es::BatchLaunch L{};
    L.inst = reinterpret_cast<const es::BatchInstanceD*>(b->d_table + b->inst_offset);
    L.n_inst = reinterpret_cast<const long long*>(b->d_table);
    L.chunk_begin = reinterpret_cast<const long long*>(b->d_table) + 1;
    L.counter = b->d_counter;
    L.error = b->d_error;
    L.chunk_iters = b->tuning.chunk_iters;
    L.retrace = b->d_retrace;
    L.retrace_count = b->d_retrace_count;
    L.retrace_cap = b->retrace_cap;
    const size_t acc_bytes = sizeof(unsigned long long) * 2 * es::kBatchMaxTau * cap;
    const size_t met_bytes = sizeof(unsigned long long) * es::kMetCount * cap;

    ES_BCUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "graph capture");
    cudaError_t e = es::copy_async(b->d_table, b->h_table, b->table_bytes, cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->d_acc, 0, acc_bytes, b->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->d_metrics, 0, met_bytes, b->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->d_counter, 0, sizeof(unsigned long long), b->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->d_retrace_count, 0, sizeof(unsigned long long), b->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->d_error, 0, sizeof(int), b->stream);
    if (e == cudaSuccess) {
        if (b->tuning.mode == ES_BATCH_PASS_KERNELS) e = record_pass_kernels(b);
        else e = es::launch_batch(L, b->tuning.precision, b->tuning.blocks_per_sm, b->n_sm, b->stream);
    }
    if (e == cudaSuccess && es::split_walk(b->tuning.precision) && b->tuning.mode != ES_BATCH_PASS_KERNELS)
        e = es::launch_retrace(L, b->n_sm, b->stream);
    if (e == cudaSuccess && b->tuning.mode == ES_BATCH_PASS_KERNELS)
        e = es::copy_async(b->h_psigma, b->d_psigma, sizeof(double) * 2 * es::kBatchMaxTau * cap,
                            cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess) e = es::copy_async(b->h_acc, b->d_acc, acc_bytes, cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess) e = es::copy_async(b->h_metrics, b->d_metrics, met_bytes, cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess) e = es::copy_async(b->h_error, b->d_error, sizeof(int), cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess)
        e = es::copy_async(b->h_retrace_count, b->d_retrace_count, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                            b->stream);
    cudaGraph_t g = nullptr;
    const cudaError_t e_end = cudaStreamEndCapture(b->stream, &g);
    if (e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return bcuda(b, e, "batch graph recording");
    }
    if (e_end != cudaSuccess) return bcuda(b, e_end, "batch graph capture");
    b->graph = g;
    b->graph_kernels = count_kernel_nodes(g);
    if (b->exec) {
        // Same node sequence as the last recording (same passes, mode and
        // precision): update the executable graph's parameters in place, which
        // costs far less than instantiating it again.
        cudaGraphExecUpdateResultInfo info;
        if (cudaGraphExecUpdate(b->exec, b->graph, &info) == cudaSuccess) {
            b->graph_dirty = false;
            return ES_OK;
        }
        cudaGetLastError();  // the failed update is not an error of a later call
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
    ES_BCUDA(cudaGraphInstantiate(&b->exec, b->graph, 0), "batch graph instantiation");
    b->graph_dirty = false;
    return ES_OK;
}

// Kernel nodes of a recorded graph: the kernels one replay launches.
int64_t count_kernel_nodes(cudaGraph_t g)
{
    size_t n = 0;
    if (cudaGraphGetNodes(g, nullptr, &n) != cudaSuccess) return 0;
    std::vector<cudaGraphNode_t> nodes(n);
    if (n == 0 || cudaGraphGetNodes(g, nodes.data(), &n) != cudaSuccess) return 0;
    int64_t k = 0;
    for (size_t i = 0; i < n; i++) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nodes[i], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) k++;
    }
    return k;
}

es_status bind_batch(es_batch* b)
{
    if (!b) return ES_ERR_BAD_ARG;
    ES_BCUDA(cudaSetDevice(b->device), "cudaSetDevice");
    return ES_OK;
}

// Fixed-point scale of a pass: a power of two with the largest possible sum
// below 2^62. |kernel value| <= 3 (1 + |w tau|) in both forms, and the Simpson
// weights sum to 3 (dim - 1) per position axis and 4 * 3 (ppq - 1) over phase.
double fixed_point_scale(int dim, int ppq, double max_wtau)
{
    const double bound = 9.0 * (dim - 1.0) * (dim - 1.0) * 12.0 * (ppq - 1.0) * 3.0 * (1.0 + max_wtau) * 1.0625;
    int ex = 0;
    std::frexp(std::ldexp(1.0, 62) / bound, &ex);
    return std::ldexp(1.0, ex - 1);
}

es_status add_grid_arrays(es_batch* b, const double* imp_xy, int64_t n_indexed, const int32_t* cell_end,
                          const es_impurity_settings* is, cudaMemcpyKind kind, int32_t* out_grid);
es_status lay_instances(es_batch* b, const es_batch_instance* inst, int32_t n);

}  // namespace

extern "C" {

es_status es_batch_create(int32_t device_ordinal, es_batch** out)
{
    es::Range nvtx_range("batch_create");
    if (!out) return ES_ERR_BAD_ARG;
    *out = nullptr;
    int n_dev = 0;
    if (cudaGetDeviceCount(&n_dev) != cudaSuccess || n_dev == 0) {
        es::set_global_error("no CUDA device is visible");
        return ES_ERR_DEVICE;
    }
    if (device_ordinal < 0 || device_ordinal >= n_dev) {
        es::set_global_error("device ordinal out of range");
        return ES_ERR_DEVICE;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device_ordinal) != cudaSuccess || prop.major != 10) {
        es::set_global_error("the batched path is built for sm_100a only");
        return ES_ERR_DEVICE;
    }
    es_batch* b = new (std::nothrow) es_batch();
    if (!b) return ES_ERR_OOM;
    b->device = device_ordinal;
    b->n_sm = prop.multiProcessorCount;
    cudaError_t e = cudaSetDevice(device_ordinal);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = es::dev_malloc(&b->d_counter, sizeof(unsigned long long));
    if (e == cudaSuccess) e = es::dev_malloc(&b->d_error, sizeof(int));
    if (e == cudaSuccess) e = es::host_malloc(&b->h_error, sizeof(int));
    if (e == cudaSuccess) e = es::dev_malloc(&b->d_retrace_count, sizeof(unsigned long long));
    if (e == cudaSuccess) e = es::host_malloc(&b->h_retrace_count, sizeof(unsigned long long));
    if (e == cudaSuccess) {
        *b->h_error = 0;
        *b->h_retrace_count = 0;
    }
    if (e != cudaSuccess) {
        char msg[256];
        snprintf(msg, sizeof msg, "es_batch_create: %s", cudaGetErrorString(e));
        es::set_global_error(msg);
        es_batch_destroy(b);
        return e == cudaErrorMemoryAllocation ? ES_ERR_OOM : ES_ERR_LAUNCH;
    }
    *out = b;
    return ES_OK;
}

es_status es_batch_destroy(es_batch* b)
{
    if (!b) return ES_ERR_BAD_ARG;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    drop_graph(b);
    free_tables(b);
    free_pass_scratch(b);
    free_grids(b);
    cudaFree(b->d_counter);
    cudaFree(b->d_error);
    cudaFree(b->d_retrace);
    cudaFree(b->d_retrace_count);
    if (b->h_error) cudaFreeHost(b->h_error);
    if (b->h_retrace_count) cudaFreeHost(b->h_retrace_count);
    b->staging.release();
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return ES_OK;
}

const char* es_batch_last_error(const es_batch* b) { return b ? b->err : es_last_error(nullptr); }

es_status es_batch_get_tuning(const es_batch* b, es_batch_tuning* out)
{
    if (!b || !out) return ES_ERR_BAD_ARG;
    *out = b->tuning;
    return ES_OK;
}

es_status es_batch_set_tuning(es_batch* b, const es_batch_tuning* t)
{
    if (!b || !t) return ES_ERR_BAD_ARG;
    if (t->chunk_iters < 1 || t->chunk_iters > 4096)
        return bfail(b, ES_ERR_BAD_ARG, "chunk_iters must be in [1, 4096] (got %d)", t->chunk_iters);
    if (t->blocks_per_sm != 3 && t->blocks_per_sm != 4)
        return bfail(b, ES_ERR_BAD_ARG, "blocks_per_sm must be 3 or 4 (got %d)", t->blocks_per_sm);
    if (!es::precision_known(t->precision))
        return bfail(b, ES_ERR_BAD_ARG, "unknown precision %d", t->precision);
    if (t->precision == ES_PRECISION_SPLIT_EXACT && t->mode != ES_BATCH_PASS_KERNELS)
        return bfail(b, ES_ERR_BAD_ARG, "ES_PRECISION_SPLIT_EXACT runs in ES_BATCH_PASS_KERNELS mode only");
    if (t->mode != ES_BATCH_PERSISTENT && t->mode != ES_BATCH_PASS_KERNELS)
        return bfail(b, ES_ERR_BAD_ARG, "unknown batch mode %d", t->mode);
    auto item_orbits = [](const es_batch_tuning& x) {
        return x.mode == ES_BATCH_PERSISTENT ? 32LL * x.chunk_iters : 32LL * es::kBatchWarps;
    };
    const bool items_change = item_orbits(*t) != item_orbits(b->tuning);
    const es_batch_tuning old = b->tuning;
    b->tuning = *t;
    b->graph_dirty = true;
    if (items_change && !b->inst.empty()) {
        // work-item boundaries depend on the mode and chunk_iters: re-lay the table.
        // On failure the old tuning stays and the instance list is kept, so the
        // same call can be repeated; until then the batch runs nothing.
        std::vector<es_batch_instance> copy = b->inst;
        const es_status st = lay_instances(b, copy.data(), (int32_t)copy.size());
        if (st != ES_OK) {
            b->tuning = old;
            b->inst = copy;
        }
        return st;
    }
    return ES_OK;
}

es_status es_batch_add_grid(es_batch* b, const double* imp_xy, int64_t n_indexed, const int32_t* cell_end,
                            const es_impurity_settings* is, int32_t* out_grid)
{
    es::Range nvtx_range("batch_add_grid");
    es_status st = bind_batch(b);
    if (st != ES_OK) return st;
    if (!is || !cell_end || !out_grid || n_indexed < 0 || (n_indexed > 0 && !imp_xy))
        return bfail(b, ES_ERR_BAD_ARG, "es_batch_add_grid: null or negative argument");
    if (is->cells_per_row < 1 || !(is->cell_size > 0.0) || !(is->spawn_region_size > 0.0))
        return bfail(b, ES_ERR_BAD_ARG, "es_batch_add_grid: invalid impurity settings");
    const int64_t n_cells = (int64_t)is->cells_per_row * is->cells_per_row;
    int64_t prev = 0;
    for (int64_t c = 0; c < n_cells; c++) {
        if (cell_end[c] < prev)
            return bfail(b, ES_ERR_BAD_ARG, "cell index is not monotone at cell %lld", (long long)c);
        prev = cell_end[c];
    }
    if (prev != n_indexed)
        return bfail(b, ES_ERR_BAD_ARG, "cell index ends at %lld but %lld impurities were given", (long long)prev,
                     (long long)n_indexed);
    return add_grid_arrays(b, imp_xy, n_indexed, cell_end, is, cudaMemcpyHostToDevice, out_grid);
}

es_status es_batch_add_dgrid(es_batch* b, const es_dgrid* grid, int32_t* out_grid)
{
    es::Range nvtx_range("batch_add_grid");
    es_status st = bind_batch(b);
    if (st != ES_OK) return st;
    if (!grid || !out_grid) return bfail(b, ES_ERR_BAD_ARG, "es_batch_add_dgrid: null argument");
    const double2* imps;
    const int* cell_end;
    int64_t n_indexed;
    es_impurity_settings is;
    uint64_t generation;
    int device;
    es::dgrid_arrays(grid, &imps, &cell_end, &n_indexed, &is, &generation, &device);
    if (device != b->device)
        return bfail(b, ES_ERR_BAD_ARG, "es_batch_add_dgrid: the grid lives on device %d, the batch on %d", device,
                     b->device);
    // the cell index is monotone and ends at n_indexed by construction
    return add_grid_arrays(b, reinterpret_cast<const double*>(imps), n_indexed, cell_end, &is,
                           cudaMemcpyDeviceToDevice, out_grid);
}

}  // extern "C"

namespace {

es_status add_grid_arrays(es_batch* b, const double* imp_xy, int64_t n_indexed, const int32_t* cell_end,
                          const es_impurity_settings* is, cudaMemcpyKind kind, int32_t* out_grid)
{
    const int64_t n_cells = (int64_t)is->cells_per_row * is->cells_per_row;
    const int64_t n_alloc = n_indexed > 0 ? n_indexed : 1;
    es_batch_grid g;
    // the smallest cleared allocation that holds this grid; when none does, the
    // cleared ones are released before a new one is made
    int best = -1;
    for (size_t k = 0; k < b->spare.size(); k++) {
        const es_batch_grid& c = b->spare[k];
        if (c.imps_cap >= n_alloc && c.cells_cap >= n_cells && (best < 0 || c.imps_cap < b->spare[(size_t)best].imps_cap))
            best = (int)k;
    }
    cudaError_t e = cudaSuccess;
    if (best >= 0) {
        g = b->spare[(size_t)best];
        b->spare.erase(b->spare.begin() + best);
    } else {
        for (auto& c : b->spare) free_grid(c);
        b->spare.clear();
        e = es::dev_malloc(&g.d_imps, sizeof(double2) * (size_t)n_alloc);
        if (e == cudaSuccess) e = es::dev_malloc(&g.d_imps32, sizeof(float2) * (size_t)n_alloc);
        if (e == cudaSuccess) e = es::dev_malloc(&g.d_cell_end, sizeof(int) * (size_t)n_cells);
        g.imps_cap = n_alloc;
        g.cells_cap = n_cells;
    }
    g.n_indexed = n_indexed;
    g.is = *is;
    auto upload = [&](void* dst, const void* src, size_t bytes) {
        return kind == cudaMemcpyHostToDevice ? b->staging.h2d(dst, src, bytes, b->stream)
                                              : es::copy_async(dst, src, bytes, kind, b->stream);
    };
    if (e == cudaSuccess && n_indexed > 0) e = upload(g.d_imps, imp_xy, sizeof(double2) * (size_t)n_indexed);
    if (e == cudaSuccess) e = upload(g.d_cell_end, cell_end, sizeof(int) * (size_t)n_cells);
    if (e == cudaSuccess)
        e = es::launch_local_impurities(g.d_imps, g.d_cell_end, g.d_imps32, is->spawn_region_start, is->cell_size,
                                        is->cells_per_row, b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) {
        free_grid(g);
        return bcuda(b, e, "es_batch_add_grid");
    }
    b->launches++;
    b->grids.push_back(g);
    *out_grid = (int32_t)(b->grids.size() - 1);
    return ES_OK;
}

}  // namespace

extern "C" {

es_status es_batch_clear(es_batch* b)
{
    es_status st = bind_batch(b);
    if (st != ES_OK) return st;
    ES_BCUDA(cudaStreamSynchronize(b->stream), "stream synchronize");
    for (auto& g : b->grids) b->spare.push_back(g);
    b->grids.clear();
    b->inst.clear();
    b->has_instances = false;
    return ES_OK;
}

es_status es_batch_set_instances(es_batch* b, const es_batch_instance* inst, int32_t n)
{
    es::Range nvtx_range("batch_set_instances");
    const es_status st = lay_instances(b, inst, n);
    // a failure after the table was touched leaves no instances to run
    if (st != ES_OK && b && !b->has_instances) b->inst.clear();
    return st;
}

}  // extern "C"

namespace {

es_status lay_instances(es_batch* b, const es_batch_instance* inst, int32_t n)
{
    namespace H = es::host;
    es_status st = bind_batch(b);
    if (st != ES_OK) return st;
    if (n < 1 || !inst) return bfail(b, ES_ERR_BAD_ARG, "es_batch_set_instances: need at least one instance");
    ES_BCUDA(cudaStreamSynchronize(b->stream), "stream synchronize");

    // validate, and set up the phase tables
    std::vector<std::vector<double>> taus((size_t)n);
    std::vector<std::vector<int>> t_slot((size_t)n);
    std::vector<es_batch_phase*> ph((size_t)n);
    for (int32_t k = 0; k < n; k++) {
        const es_batch_instance& x = inst[k];
        if (x.grid < 0 || x.grid >= (int32_t)b->grids.size())
            return bfail(b, ES_ERR_BAD_ARG, "instance %d: unknown grid %d", k, x.grid);
        if (x.positions_per_row < 3 || x.positions_per_row % 2 == 0)
            return bfail(b, ES_ERR_BAD_ARG, "instance %d: positions_per_row must be odd and >= 3", k);
        if (x.particles_per_quadrant < 3 || x.particles_per_quadrant % 2 == 0)
            return bfail(b, ES_ERR_BAD_ARG, "instance %d: particles_per_quadrant must be odd and >= 3", k);
        if (!(x.region_size > 0.0) || !(x.grid_cell_size > 0.0) || !(x.settings.particle_speed > 0.0))
            return bfail(b, ES_ERR_BAD_ARG, "instance %d: region_size, grid_cell_size and particle_speed must be positive", k);
        if (!(x.magnetic_field > 0.0) || !std::isfinite(x.magnetic_field))
            return bfail(b, ES_ERR_BAD_ARG, "instance %d: magnetic field must be positive and finite", k);
        if (x.n_t < 1 || x.n_t > ES_BATCH_MAX_T)
            return bfail(b, ES_ERR_BAD_ARG, "instance %d: n_t must be in [1, %d]", k, ES_BATCH_MAX_T);
        if (x.coherent && !(x.settings.tau > 0.0)) return bfail(b, ES_ERR_BAD_ARG, "instance %d: tau must be positive", k);
        const int64_t n_orbits = (int64_t)x.positions_per_row * x.positions_per_row * 4 * x.particles_per_quadrant;
        if (n_orbits >= (1LL << 40)) return bfail(b, ES_ERR_BAD_ARG, "instance %d: too many orbits", k);
        for (int t = 0; t < x.n_t; t++) {
            const double T = x.temperatures[t];
            if (!x.coherent && !(T > 0.0))
                return bfail(b, ES_ERR_BAD_ARG, "instance %d: temperature %g: the incoherent sector needs T > 0", k, T);
            const double tau = H::get_tau(x.coherent != 0, x.settings.tau, T);
            int slot = -1;
            for (size_t u = 0; u < taus[k].size(); u++)
                if (taus[k][u] == tau) slot = (int)u;
            if (slot < 0) {
                if ((int)taus[k].size() == es::kBatchMaxTau)
                    return bfail(b, ES_ERR_BAD_ARG, "instance %d: more than %d distinct relaxation times; split its temperatures",
                                 k, es::kBatchMaxTau);
                slot = (int)taus[k].size();
                taus[k].push_back(tau);
            }
            t_slot[k].push_back(slot);
        }
        // start positions inside the grid (the reference reads out of bounds otherwise)
        const es_impurity_settings& is = b->grids[(size_t)x.grid].is;
        const int dim = x.positions_per_row;
        const double dist = x.region_size / (double)(dim - 1);
        const double ox = x.grid_cell_size * 0.01, oy = x.grid_cell_size * 0.005;
        const double xs[2] = {0.0 * dist + ox, (double)(dim - 1) * dist + ox};
        const double ys[2] = {0.0 * dist + oy, (double)(dim - 1) * dist + oy};
        for (double px : xs)
            for (double py : ys) {
                const int cx = (int)((px - is.spawn_region_start) / is.spawn_region_size * (double)is.cells_per_row);
                const int cy = (int)((py - is.spawn_region_start) / is.spawn_region_size * (double)is.cells_per_row);
                if (cx < 0 || cy < 0 || cx >= is.cells_per_row || cy >= is.cells_per_row)
                    return bfail(b, ES_ERR_BAD_ARG, "instance %d: start position (%g, %g) lies outside its grid", k, px, py);
            }
        const auto key = std::make_tuple(x.particles_per_quadrant, x.coherent ? 1 : 0, x.settings.alpha,
                                         x.settings.particle_speed, x.settings.is_clockwise ? 1 : 0);
        auto it = b->phases.find(key);
        if (it == b->phases.end()) {
            const int ppq = x.particles_per_quadrant;
            const H::Sector sec = H::sector(x.settings.alpha, ppq, x.coherent != 0);
            std::vector<es::PhaseOrbit> po((size_t)(4 * ppq));
            std::vector<es::PhaseSigma> psg((size_t)(4 * ppq));
            H::phase_tables(sec, ppq, x.settings.particle_speed, x.settings.alpha, x.settings.is_clockwise != 0,
                            po.data(), psg.data());
            es_batch_phase p;
            p.phi_integrand_factor = sec.phi_integrand_factor;
            cudaError_t e = es::dev_malloc(&p.d_orbit, sizeof(es::PhaseOrbit) * po.size());
            if (e == cudaSuccess) e = es::dev_malloc(&p.d_sigma, sizeof(es::PhaseSigma) * psg.size());
            if (e == cudaSuccess)
                e = es::copy_sync(p.d_orbit, po.data(), sizeof(es::PhaseOrbit) * po.size(), cudaMemcpyHostToDevice);
            if (e == cudaSuccess)
                e = es::copy_sync(p.d_sigma, psg.data(), sizeof(es::PhaseSigma) * psg.size(), cudaMemcpyHostToDevice);
            if (e != cudaSuccess) {
                cudaFree(p.d_orbit);
                cudaFree(p.d_sigma);
                return bcuda(b, e, "phase tables");
            }
            it = b->phases.emplace(key, p).first;
        }
        ph[(size_t)k] = &it->second;
    }

    // From here the instance table is rewritten: until it is complete the batch
    // has no instances, so a failure below leaves nothing that es_batch_enqueue
    // would run.
    b->has_instances = false;
    if ((st = ensure_capacity(b, n)) != ES_OK) return st;

    // kernel order: largest passes first, so the tail of the run is made of small work items
    std::vector<int> order((size_t)n);
    std::iota(order.begin(), order.end(), 0);
    auto orbits_of = [&](int k) {
        return (int64_t)inst[k].positions_per_row * inst[k].positions_per_row * 4 * inst[k].particles_per_quadrant;
    };
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return orbits_of(a) > orbits_of(c); });

    const int64_t item_orbits =
        b->tuning.mode == ES_BATCH_PERSISTENT ? 32LL * b->tuning.chunk_iters : 32LL * es::kBatchWarps;
    b->pass_items.assign((size_t)n, 0);
    long long* hdr = reinterpret_cast<long long*>(b->h_table);
    es::BatchInstanceD* hi = reinterpret_cast<es::BatchInstanceD*>(b->h_table + b->inst_offset);
    b->factor.assign((size_t)n, {});
    b->fx_scale.assign((size_t)n, 0.0);
    b->pass_phi_factor.assign((size_t)n, 0.0);
    long long items = 0;
    int64_t total = 0;
    for (int32_t pos = 0; pos < n; pos++) {
        const int k = order[(size_t)pos];
        const es_batch_instance& x = inst[k];
        const es_batch_grid& g = b->grids[(size_t)x.grid];
        const es_batch_phase& p = *ph[(size_t)k];
        es::BatchInstanceD d;
        std::memset(&d, 0, sizeof d);
        es::LifetimeLaunch& L = d.L;
        // make_launch of the per-pass path (es_context.cu), same arithmetic
        const double w = H::angular_speed(x.magnetic_field);
        L.imps = g.d_imps;
        L.cell_end = g.d_cell_end;
        L.phase = p.d_orbit;
        L.error = b->d_error;
        L.spawn_start = g.is.spawn_region_start;
        L.spawn_size = g.is.spawn_region_size;
        L.cell_size = g.is.cell_size;
        L.imp_radius = g.is.impurity_radius;
        L.speed = x.settings.particle_speed;
        L.radius = x.settings.particle_speed / w;
        L.radius_sq = L.radius * L.radius;
        L.w = w;
        L.dist = x.region_size / (double)(x.positions_per_row - 1);
        L.off_x = x.grid_cell_size * 0.01;
        L.off_y = x.grid_cell_size * 0.005;
        L.n_orbits = orbits_of(k);
        L.cpr = g.is.cells_per_row;
        L.dim = x.positions_per_row;
        L.n_phase = 4 * x.particles_per_quadrant;
        L.clockwise = x.settings.is_clockwise ? 1 : 0;
        L.coherent = x.coherent ? 1 : 0;
        L.walk_cap = H::walk_cap_for(L.radius, L.cell_size);
        L.imps32 = g.d_imps32;
        H::split_constants(L);
        d.phase_sigma = p.d_sigma;
        d.acc = b->d_acc + (size_t)pos * 2 * es::kBatchMaxTau;
        d.metrics = b->d_metrics + (size_t)pos * es::kMetCount;
        d.chunk_begin = items;
        d.w_signed = x.settings.is_clockwise ? -w : w;
        d.n_tau = (int)taus[k].size();
        double max_wtau = 0.0;
        std::vector<double> fac;
        for (int u = 0; u < d.n_tau; u++) {
            const double tau = taus[k][(size_t)u];
            d.tau[u] = tau;
            d.inv_tau[u] = 1.0 / tau;
            d.max_lt[u] = 15.0 * tau;
            d.wtau[u] = d.w_signed * tau;
            max_wtau = std::max(max_wtau, std::fabs(d.wtau[u]));
            fac.push_back(H::integrand_factor(x.settings.particle_speed, x.positions_per_row, p.phi_integrand_factor, w,
                                              tau));
        }
        d.fx_scale = fixed_point_scale(x.positions_per_row, x.particles_per_quadrant, max_wtau);
        hi[pos] = d;
        hdr[1 + pos] = items;
        b->pass_items[(size_t)pos] = (L.n_orbits + item_orbits - 1) / item_orbits;
        items += b->pass_items[(size_t)pos];
        total += L.n_orbits;
        b->factor[(size_t)k] = fac;
        b->fx_scale[(size_t)k] = d.fx_scale;
        b->pass_phi_factor[(size_t)pos] = p.phi_integrand_factor;
    }
    hdr[0] = n;
    hdr[1 + n] = items;
    b->inst.assign(inst, inst + n);
    b->order = order;
    b->t_slot = t_slot;
    b->total_orbits = total;
    b->total_items = items;
    // Re-traced orbits are a small fraction (observed ~0.05%); the list starts
    // at 1/1024 of the run and grows on overflow (es_batch_collect re-runs).
    if (es::split_walk(b->tuning.precision))
        if ((st = ensure_retrace(b, total / 1024 + 262144)) != ES_OK) return st;
    b->has_instances = true;
    // pass records are kernel parameters in this mode: record the graph again
    if (b->tuning.mode == ES_BATCH_PASS_KERNELS) b->graph_dirty = true;
    return ES_OK;
}

}  // namespace

extern "C" {

es_status es_batch_enqueue(es_batch* b)
{
    es::Range nvtx_range("batch_enqueue");
    es_status st = bind_batch(b);
    if (st != ES_OK) return st;
    if (!b->has_instances) return bfail(b, ES_ERR_BAD_ARG, "es_batch_set_instances has not been called");
    if (es::split_walk(b->tuning.precision) && b->retrace_cap == 0)
        if ((st = ensure_retrace(b, b->total_orbits / 1024 + 262144)) != ES_OK) return st;
    if (b->graph_dirty || !b->exec)
        if ((st = capture(b)) != ES_OK) return st;
    ES_BCUDA(cudaGraphLaunch(b->exec, b->stream), "batch graph launch");
    b->launches++;
    return ES_OK;
}

es_status es_batch_collect(es_batch* b, double* out_sigma, es_metrics* out_metrics)
{
    es::Range nvtx_range("batch_collect");
    es_status st = bind_batch(b);
    if (st != ES_OK) return st;
    if (!b->has_instances) return bfail(b, ES_ERR_BAD_ARG, "es_batch_set_instances has not been called");
    ES_BCUDA(cudaStreamSynchronize(b->stream), "batch synchronize");
    if (*b->h_error & es::kErrRetraceOverflow) {
        // the list was too short for this run: grow it to fit and run again
        // (in ES_BATCH_PASS_KERNELS the count read back is the last pass's only)
        const long long need = b->tuning.mode == ES_BATCH_PASS_KERNELS
                                   ? std::max((long long)*b->h_retrace_count, 2 * b->retrace_cap)
                                   : (long long)*b->h_retrace_count;
        if ((st = ensure_retrace(b, need + need / 4 + 1024)) != ES_OK) return st;
        b->retrace_regrows++;
        if ((st = es_batch_enqueue(b)) != ES_OK) return st;
        ES_BCUDA(cudaStreamSynchronize(b->stream), "batch synchronize");
        if (*b->h_error & es::kErrRetraceOverflow)
            return bfail(b, ES_ERR_LAUNCH, "split precision: the FP64 re-trace list overflowed twice");
    }
    const int h_err = *b->h_error;
    if (h_err & es::kErrWalkCap)
        return bfail(b, ES_ERR_WALK_CAP, "an orbit exceeded the cell-walk step bound (its lifetime was set to 0)");
    if (h_err) return bfail(b, ES_ERR_BAD_ARG, "a start position lies outside its impurity grid");
    const int32_t n = (int32_t)b->inst.size();
    for (int32_t pos = 0; pos < n; pos++) {
        const int k = b->order[(size_t)pos];
        const es_batch_instance& x = b->inst[(size_t)k];
        const unsigned long long* acc = b->h_acc + (size_t)pos * 2 * es::kBatchMaxTau;
        if (out_sigma) {
            double* o = out_sigma + (size_t)k * ES_BATCH_MAX_T * 2;
            for (int t = 0; t < ES_BATCH_MAX_T * 2; t++) o[t] = 0.0;
            const double* ps = b->h_psigma + (size_t)pos * 2 * es::kBatchMaxTau;
            for (int t = 0; t < x.n_t; t++) {
                const int u = b->t_slot[(size_t)k][(size_t)t];
                for (int c = 0; c < 2; c++) {
                    if (b->tuning.mode == ES_BATCH_PASS_KERNELS) {
                        o[2 * t + c] = ps[2 * u + c];
                    } else {
                        const long long q = (long long)acc[2 * u + c];
                        o[2 * t + c] = ((double)q / b->fx_scale[(size_t)k]) * b->factor[(size_t)k][(size_t)u];
                    }
                }
            }
        }
        if (out_metrics) {
            const unsigned long long* m = b->h_metrics + (size_t)pos * es::kMetCount;
            es_metrics& om = out_metrics[k];
            om.cells_passed = (int64_t)m[es::kMetCells];
            om.impurities_tested = (int64_t)m[es::kMetImps];
            om.particles_inside_impurity = (int64_t)m[es::kMetInside];
            om.particles_escaped = (int64_t)m[es::kMetEscaped];
            om.particles_at_bound = (int64_t)m[es::kMetAtBound];
            om.max_impurities_tested = (int64_t)m[es::kMetMaxImps];
            om.max_cells_passed = (int64_t)m[es::kMetMaxCells];
            om.crossings_tested = (int64_t)m[es::kMetCrossings];
            om.start_cell_tests = (int64_t)m[es::kMetStartTests];
            om.retraced_fp64 = (int64_t)m[es::kMetRetraced];
        }
    }
    return ES_OK;
}

es_status es_batch_run(es_batch* b, double* out_sigma, es_metrics* out_metrics)
{
    es_status st = es_batch_enqueue(b);
    if (st != ES_OK) return st;
    return es_batch_collect(b, out_sigma, out_metrics);
}

void* es_batch_stream(es_batch* b) { return b ? (void*)b->stream : nullptr; }

int64_t es_batch_launch_count(const es_batch* b) { return b ? b->launches : 0; }

int64_t es_batch_graph_kernels(const es_batch* b) { return b ? b->graph_kernels : 0; }

int64_t es_batch_total_orbits(const es_batch* b) { return b ? b->total_orbits : 0; }

}  // extern "C"
