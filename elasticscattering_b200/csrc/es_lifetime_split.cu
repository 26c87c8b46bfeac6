// es_lifetime_split.cu - stage (a), FP32/FP64 split precision: the single-pass kernels.
//
// lifetime_split_kernel walks one orbit per thread with the FP32 cell walk of
// es_orbit_split.cuh, recomputes the winning crossing in FP64 and appends the
// orbits whose FP32 decision is not certain to a re-trace list;
// lifetime_retrace_kernel then runs the exact FP64 TraceOrbit
// (src/sim/es/lifetime.h:78-148) on that list. The lifetimes are the FP64
// path's, orbit for orbit.
#include "es_orbit_split.cuh"

namespace es {
namespace {

// kSplitFinish: the walk stops at the winning disk(s) and leaves them in the
// orbit's lifetime slot for lifetime_finish_kernel (split_orbit_walk), for
// passes whose walks end after differing numbers of cell steps; otherwise the
// winner's FP64 time is taken inside the walk (split_orbit), for passes where
// nearly every walk ends in its first cell.
template <int kMinBlocks, bool kSplitFinish>
__global__ void __launch_bounds__(256, kMinBlocks) lifetime_split_kernel(LifetimeLaunch P)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = t < P.n_orbits;
    const unsigned mask = __ballot_sync(0xffffffffu, active);
    if (!active) return;
    const long long g = (long long)P.row0 * P.dim * P.n_phase + t;

    SplitCounters cnt;
    int flags;
    double lt;
    bool retrace;
    if constexpr (kSplitFinish) {
        int2 win;
        const int st = split_orbit_walk(LaunchFields{P}, g, mask, cnt, flags, lt, win);
        retrace = st == kSplitRetrace;
        // every slot is written, so that the finish kernel reads no stale hit
        P.out[g] = st == kSplitHit ? encode_hit(win) : lt;
    } else {
        retrace = split_orbit(LaunchFields{P}, g, cnt, flags, lt, mask);
        if (!retrace) P.out[g] = lt;
    }
    if (retrace) {
        const unsigned long long slot = atomicAdd(P.retrace_count, 1ull);
        if (slot < (unsigned long long)P.retrace_cap) P.retrace[slot] = g;
        else atomicOr(P.error, kErrRetraceOverflow);
    }
    // re-traced orbits are counted by the FP64 kernel; a hit's at-bound flag by
    // the finish kernel
    flush_split_metrics(P.metrics, mask, cnt, flags, !retrace);
}

// LaunchFields with the FP64 crossing code inline: the finish kernel has no
// walk whose body it would lengthen.
struct FinishFields : LaunchFields {
    static constexpr bool kCrossOutOfLine = false;
};

// The winners' FP64 times of a split-finish pass (lifetime_split_kernel<.., true>):
// for every slot holding a hit, the reference's GetCrossPoints/GetAngle/
// GetCrossAngle time of the first crossing of the winning disk (the earlier of
// two near-equal ones), clamped to the sector bound (src/sim/es/lifetime.h:
// 138-146), as the walk would have taken it. A winner whose crossing point
// the reference drops (NaN) goes to the FP64 re-trace, marked as already
// counted. At-bound hits are counted here, one atomic per warp. Five blocks
// per SM (48 registers, a few spills) hide more of the FP64 latency than four
// (52 registers): 0.6% per config-1 pass on B200.
__global__ void __launch_bounds__(256, 5) lifetime_finish_kernel(LifetimeLaunch P)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned bound = 0;
    if (t < P.n_orbits) {
        const long long g = (long long)P.row0 * P.dim * P.n_phase + t;
        int2 win;
        if (decode_hit(P.out[g], win)) {
            const FinishFields f{{P}};
            dv2 pos;
            const OrbitD o = make_orbit(f, g, pos);
            int flags;
            const double lt = finish_hit<FinishFields, true>(f, o, win.x, win.y, flags);
            if (lt != lt || (P.finish_retrace_every > 0 && g % P.finish_retrace_every == 0)) {
                P.out[g] = 0.0;
                const unsigned long long slot = atomicAdd(P.retrace_count, 1ull);
                if (slot < (unsigned long long)P.retrace_cap) P.retrace[slot] = g | kRetraceFromFinish;
                else atomicOr(P.error, kErrRetraceOverflow);
            } else {
                P.out[g] = lt;
                bound = (flags & kTraceAtBound) ? 1u : 0u;
            }
        }
    }
    const unsigned n_bound = __reduce_add_sync(0xffffffffu, bound);
    if ((threadIdx.x & 31) == 0 && n_bound) atomicAdd(P.metrics + kMetAtBound, (unsigned long long)n_bound);
}

// The pass's orbit table: per phase, CreateParticle's centre shift and bound
// time (src/sim/es/lifetime.h:36-58, details.h:243-250) at this pass's radius
// and w -- the FP64 quotients make_orbit would otherwise form for every orbit.
__global__ void orbit_table_kernel(LifetimeLaunch P)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= P.n_phase) return;
    const PhaseOrbit ph = P.phase[v];
    const double shift_x = (ph.vel_y * P.radius) / P.speed;
    const double shift_y = (-ph.vel_x * P.radius) / P.speed;
    const double bound_time = P.coherent ? kINF : ph.bound_dphi / P.w;
    P.orbit_table[v] = make_double4(shift_x, shift_y, bound_time, ph.phi);
}

// Exact FP64 re-trace of the listed orbits (the list length is a device count).
// The list is short (0.01-0.2 % of a pass) and each entry is a long FP64 walk,
// so entries go to warps first: entry e runs in warp e mod W (W = the grid's
// warps), lane (e / W) mod 32. A list of a few thousand orbits then spreads
// over every SM, one walk per warp, instead of filling the first few blocks.
// The counters are summed per warp, then per block in shared memory, and the
// block adds them to the pass's counters with one atomic each (per-orbit
// atomics on the same ten addresses serialised in L2). An entry from the
// finish kernel was counted by the walk: its walk counters are subtracted
// (the FP64 walk passes at least the cells and disks the split walk did, so
// the maxima the walk recorded stay below the FP64 ones).
__global__ void __launch_bounds__(256, 4) lifetime_retrace_kernel(LifetimeLaunch P)
{
    __shared__ unsigned long long s_sum[8];  // two's complement sums
    __shared__ unsigned s_max[2];
    const unsigned long long n_list = min(*P.retrace_count, (unsigned long long)P.retrace_cap);
    const unsigned long long warps = (unsigned long long)gridDim.x * (blockDim.x / 32);
    const unsigned long long wid = (unsigned long long)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const unsigned long long lane = threadIdx.x & 31;
    if (threadIdx.x < 8) s_sum[threadIdx.x] = 0ull;
    if (threadIdx.x < 2) s_max[threadIdx.x] = 0u;
    __syncthreads();
    OrbitCounters cnt = {0, 0, 0, 0};
    unsigned in = 0, esc = 0, bound = 0, mc = 0, mi = 0, n = 0;
    for (unsigned long long e = lane * warps + wid; e < n_list; e += 32 * warps) {
        const long long entry = P.retrace[e];
        const long long g = entry & ~kRetraceFromFinish;
        if (entry & kRetraceFromFinish) {
            const SplitCounters w = split_walk_counters(P, g);
            cnt.cells -= w.cells;
            cnt.imps -= w.imps;
            cnt.crossings -= w.crossings;
            cnt.start_tests -= w.start_tests;
        }
        retrace_orbit(P, g, cnt, in, esc, bound, mc, mi);
        n++;
    }
    const int v[8] = {(int)cnt.cells, (int)cnt.imps, (int)cnt.crossings, (int)cnt.start_tests,
                      (int)in, (int)esc, (int)bound, (int)n};
    int r[8];
#pragma unroll
    for (int k = 0; k < 8; k++) r[k] = __reduce_add_sync(0xffffffffu, v[k]);
    const unsigned rmc = __reduce_max_sync(0xffffffffu, mc), rmi = __reduce_max_sync(0xffffffffu, mi);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < 8; k++)
            if (r[k]) atomicAdd(&s_sum[k], (unsigned long long)(long long)r[k]);
        atomicMax(&s_max[0], rmc);
        atomicMax(&s_max[1], rmi);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int slot[8] = {kMetCells, kMetImps, kMetCrossings, kMetStartTests, kMetInside, kMetEscaped, kMetAtBound,
                             kMetRetraced};
#pragma unroll
        for (int k = 0; k < 8; k++)
            if (s_sum[k]) atomicAdd(P.metrics + slot[k], s_sum[k]);
        if (s_max[0]) atomicMax(P.metrics + kMetMaxCells, (unsigned long long)s_max[0]);
        if (s_max[1]) atomicMax(P.metrics + kMetMaxImps, (unsigned long long)s_max[1]);
    }
}

// Cell-local FP32 copy of the ordered impurities: x - (start + cx L), y - (start + cy L).
__global__ void local_impurities_kernel(const double2* imps, const int* cell_end, float2* out, double start,
                                        double cell, int cpr)
{
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (long long)cpr * cpr) return;
    const int cx = (int)(c % cpr), cy = (int)(c / cpr);
    const double ox = start + cx * cell, oy = start + cy * cell;
    const int k0 = (c == 0) ? 0 : cell_end[c - 1];
    const int k1 = cell_end[c];
    for (int k = k0; k < k1; k++) {
        const double2 q = imps[k];
        out[k] = make_float2((float)(q.x - ox), (float)(q.y - oy));
    }
}

}  // namespace

cudaError_t launch_lifetimes_split(const LifetimeLaunch& L, bool split_finish, cudaStream_t s)
{
    if (L.n_orbits <= 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(L.retrace_count, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    if (L.orbit_table != nullptr) {
        orbit_table_kernel<<<(unsigned)((L.n_phase + 127) / 128), 128, 0, s>>>(L);
        if ((e = es::launched(s)) != cudaSuccess) return e;
    }
    const long long blocks = (L.n_orbits + 255) / 256;
    if (split_finish) {
        lifetime_split_kernel<4, true><<<(unsigned)blocks, 256, 0, s>>>(L);
        if ((e = es::launched(s)) != cudaSuccess) return e;
        lifetime_finish_kernel<<<(unsigned)blocks, 256, 0, s>>>(L);
    } else {
        lifetime_split_kernel<4, false><<<(unsigned)blocks, 256, 0, s>>>(L);
    }
    if ((e = es::launched(s)) != cudaSuccess) return e;
    lifetime_retrace_kernel<<<148 * 4, 256, 0, s>>>(L);
    return es::launched(s);
}

cudaError_t launch_local_impurities(const double2* imps, const int* cell_end, float2* out, double start, double cell,
                                    int cpr, cudaStream_t s)
{
    const long long n = (long long)cpr * cpr;
    local_impurities_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(imps, cell_end, out, start, cell, cpr);
    return es::launched(s);
}

}  // namespace es
