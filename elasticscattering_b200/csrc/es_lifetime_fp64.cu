// es_lifetime_fp64.cu - stage (a), plain FP64: one orbit lifetime per thread.
//
// Replaces the OpenCL `lifetime` kernel (src/sim/cl/scatter.cl:26-96) and the
// CPU loop of SimulationCPU::ComputeLifetimes (src/sim/SimulationCPU.cpp:103-141).
// Compiled with -fmad=false (see es_orbit_fp64.cuh).
//
// Mapping: consecutive threads take consecutive orbits in [j][i][q][p] order,
// so a warp covers 32 phases of one start position (same start cell, same
// start-cell impurity scan, coalesced 8-byte stores). Per-orbit constants come
// from the host-built phase table. Metrics are summed per warp with
// __reduce_*_sync and added with one atomic per warp and counter instead of
// the reference's atomic per cell step (src/sim/es/device_macros.h:33-36).
#include "es_internal.h"
#include "es_orbit_fp64.cuh"

namespace es {

namespace {

__device__ __forceinline__ void warp_flush(unsigned long long* metrics, unsigned mask, OrbitCounters c, int flags,
                                           bool active)
{
    const unsigned cells = active ? (unsigned)c.cells : 0u;
    const unsigned imps = active ? (unsigned)c.imps : 0u;
    const unsigned cross = active ? (unsigned)c.crossings : 0u;
    const unsigned start_tests = active ? (unsigned)c.start_tests : 0u;
    const unsigned inside = (active && (flags & kTraceInside)) ? 1u : 0u;
    const unsigned escaped = (active && (flags & kTraceEscaped)) ? 1u : 0u;
    const unsigned bound = (active && (flags & kTraceAtBound)) ? 1u : 0u;

    const unsigned s_cells = __reduce_add_sync(mask, cells);
    const unsigned s_imps = __reduce_add_sync(mask, imps);
    const unsigned s_cross = __reduce_add_sync(mask, cross);
    const unsigned s_start = __reduce_add_sync(mask, start_tests);
    const unsigned s_inside = __reduce_add_sync(mask, inside);
    const unsigned s_escaped = __reduce_add_sync(mask, escaped);
    const unsigned s_bound = __reduce_add_sync(mask, bound);
    const unsigned m_cells = __reduce_max_sync(mask, cells);
    const unsigned m_imps = __reduce_max_sync(mask, imps);

    if ((threadIdx.x & 31) == (__ffs(mask) - 1)) {
        if (s_cells) atomicAdd(metrics + kMetCells, (unsigned long long)s_cells);
        if (s_imps) atomicAdd(metrics + kMetImps, (unsigned long long)s_imps);
        if (s_cross) atomicAdd(metrics + kMetCrossings, (unsigned long long)s_cross);
        if (s_start) atomicAdd(metrics + kMetStartTests, (unsigned long long)s_start);
        if (s_inside) atomicAdd(metrics + kMetInside, (unsigned long long)s_inside);
        if (s_escaped) atomicAdd(metrics + kMetEscaped, (unsigned long long)s_escaped);
        if (s_bound) atomicAdd(metrics + kMetAtBound, (unsigned long long)s_bound);
        if (m_cells) atomicMax(metrics + kMetMaxCells, (unsigned long long)m_cells);
        if (m_imps) atomicMax(metrics + kMetMaxImps, (unsigned long long)m_imps);
    }
}

// Lanes take consecutive orbits of the storage order, i.e. 32 phases of one
// start position. kDefer > 0 parks crossing disks in shared memory and takes
// their crossing points after the cheap tests of the cell (trace_orbit).
template <int kMinBlocks, int kDefer>
__global__ void __launch_bounds__(256, kMinBlocks) lifetime_fp64_kernel(LifetimeLaunch P)
{
    __shared__ int s_defer[kDefer > 0 ? kDefer * kDeferStride : 1];
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = t < P.n_orbits;
    const unsigned mask = __ballot_sync(0xffffffffu, active);
    if (!active) return;

    const long long g = (long long)P.row0 * P.dim * P.n_phase + t;
    const int v = (int)(g % P.n_phase);
    const long long pidx = g / P.n_phase;
    const int i = (int)(pidx % P.dim);
    const int j = (int)(pidx / P.dim);

    // Simulation position grid, src/sim/SimulationCPU.cpp:114:
    // v2(i, j) * distance_between_positions + small_offset
    const dv2 position = {(double)i * P.dist + P.off_x, (double)j * P.dist + P.off_y};

    const PhaseOrbit ph = P.phase[v];
    OrbitD o;
    o.radius = P.radius;
    o.radius_sq = P.radius_sq;
    o.clockwise = P.clockwise != 0;
    // GetCyclotronOrbitCenter, src/sim/es/details.h:243-250:
    // shift = (vel.y, -vel.x) * radius / speed
    const double shift_x = (ph.vel_y * P.radius) / P.speed;
    const double shift_y = (-ph.vel_x * P.radius) / P.speed;
    if (o.clockwise) {
        o.center = dv2{position.x - shift_x, position.y - shift_y};
    } else {
        o.center = dv2{position.x + shift_x, position.y + shift_y};
    }
    // GetBoundTime, src/sim/es/details.h:219-228 (INF when coherent)
    o.bound_time = P.coherent ? kINF : ph.bound_dphi / P.w;
    o.particle_angle = ph.phi;

    GridD gr;
    gr.imps = P.imps;
    gr.cell_end = P.cell_end;
    gr.start = P.spawn_start;
    gr.size = P.spawn_size;
    gr.cell = P.cell_size;
    gr.imp_r = P.imp_radius;
    gr.cpr = P.cpr;

    OrbitCounters cnt = {0, 0, 0, 0};
    int flags = kTraceOk;
    double lt = 0.0;
    const iv2 c0 = get_cell(position, gr.start, gr.size, gr.cpr);
    const bool in_grid = within_bounds(c0, gr.cpr);
    // The start-cell scan depends on the start position only: when the warp's
    // lanes all start at one position, they share it.
    StartScan start{-1, false};
    {
        const int src = __ffs(mask) - 1;
        const long long p0 = __shfl_sync(mask, pidx, src);
        if (__all_sync(mask, pidx == p0 && in_grid))
            start = start_scan_shared64(gr.imps, gr.cell_end, c0.y * gr.cpr + c0.x, position, gr.imp_r, mask);
    }
    if (!in_grid) {
        atomicOr(P.error, kErrStartCell);
    } else {
        lt = trace_orbit<kDefer>(o, position, ph.phi, P.w, gr, P.walk_cap, cnt, flags, s_defer + threadIdx.x, start);
        if (flags & kTraceWalkCap) atomicOr(P.error, kErrWalkCap);
    }
    P.out[g] = lt;
    if (P.out32) P.out32[g] = (float)lt;

    warp_flush(P.metrics, mask, cnt, flags, true);
}

__global__ void debug_next_cell_kernel(double cx, double cy, double r, int clockwise, double phi, double start,
                                       double size, double cell, int cpr, const double* in6, double* out6,
                                       int* avail)
{
    OrbitD o;
    o.center = dv2{cx, cy};
    o.radius = r;
    o.radius_sq = r * r;
    o.clockwise = clockwise != 0;
    o.bound_time = 0;
    o.particle_angle = 0;
    GridD g;
    g.imps = nullptr;
    g.cell_end = nullptr;
    g.start = start;
    g.size = size;
    g.cell = cell;
    g.imp_r = 0;
    g.cpr = cpr;
    Isect last, next;
    last.position = dv2{in6[0], in6[1]};
    last.incident_angle = in6[2];
    last.dphi = in6[3];
    last.cell = iv2{(int)in6[4], (int)in6[5]};
    *avail = next_cell(o, phi, g, last, next) ? 1 : 0;
    out6[0] = next.position.x;
    out6[1] = next.position.y;
    out6[2] = next.incident_angle;
    out6[3] = next.dphi;
    out6[4] = next.cell.x;
    out6[5] = next.cell.y;
}

// One orbit with explicit particle constants (phase table row, field,
// position); the grid and geometry fields of P are used as in the pass kernel.
__global__ void debug_trace_kernel(LifetimeLaunch P, PhaseOrbit ph, double px, double py, double* out)
{
    const dv2 position = {px, py};
    OrbitD o;
    o.radius = P.radius;
    o.radius_sq = P.radius_sq;
    o.clockwise = P.clockwise != 0;
    const double shift_x = (ph.vel_y * P.radius) / P.speed;
    const double shift_y = (-ph.vel_x * P.radius) / P.speed;
    o.center = o.clockwise ? dv2{position.x - shift_x, position.y - shift_y}
                           : dv2{position.x + shift_x, position.y + shift_y};
    o.bound_time = P.coherent ? kINF : ph.bound_dphi / P.w;
    o.particle_angle = ph.phi;
    GridD gr;
    gr.imps = P.imps;
    gr.cell_end = P.cell_end;
    gr.start = P.spawn_start;
    gr.size = P.spawn_size;
    gr.cell = P.cell_size;
    gr.imp_r = P.imp_radius;
    gr.cpr = P.cpr;
    OrbitCounters cnt = {0, 0, 0, 0};
    int flags = kTraceOk;
    const iv2 c0 = get_cell(position, gr.start, gr.size, gr.cpr);
    *out = within_bounds(c0, gr.cpr) ? trace_orbit(o, position, ph.phi, P.w, gr, P.walk_cap, cnt, flags) : -1.0;
}

}  // namespace

cudaError_t launch_debug_trace(const LifetimeLaunch& L, const PhaseOrbit& ph, double px, double py, double* d_out,
                               cudaStream_t s)
{
    debug_trace_kernel<<<1, 1, 0, s>>>(L, ph, px, py, d_out);
    return es::launched(s);
}

namespace {

template <int kMinBlocks, int kDefer>
cudaError_t launch_per_thread(const LifetimeLaunch& L, cudaStream_t s)
{
    const long long blocks = (L.n_orbits + 255) / 256;
    lifetime_fp64_kernel<kMinBlocks, kDefer><<<(unsigned)blocks, 256, 0, s>>>(L);
    return es::launched(s);
}

}  // namespace

cudaError_t launch_lifetimes_fp64(const LifetimeLaunch& L, cudaStream_t s)
{
    if (L.n_orbits <= 0) return cudaSuccess;
    switch (L.variant) {
        case kLifetimePerThread: return launch_per_thread<3, 0>(L, s);
        case kLifetimePerThreadLean: return launch_per_thread<4, 0>(L, s);
        case kLifetimePerThreadDefer: return launch_per_thread<4, 4>(L, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_debug_next_cell(double cx, double cy, double r, int clockwise, double phi, double start,
                                   double size, double cell, int cpr, const double* d_in6, double* d_out6,
                                   int* d_avail, cudaStream_t s)
{
    debug_next_cell_kernel<<<1, 1, 0, s>>>(cx, cy, r, clockwise, phi, start, size, cell, cpr, d_in6, d_out6, d_avail);
    return es::launched(s);
}

}  // namespace es
