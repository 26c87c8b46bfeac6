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

// kPositionMajor = false: lanes take consecutive orbits of the storage order,
// i.e. 32 phases of one start position. kPositionMajor = true: lanes take 32
// neighbouring start positions of one row at the same phase; their orbits are
// parallel shifts of each other (by the position spacing, a fraction of a
// cell), so they cross the same cells and edges and scan the same impurity
// lists, which keeps the warp converged. Stores are then strided.
template <int kMinBlocks, bool kPositionMajor, int kDefer>
__global__ void __launch_bounds__(256, kMinBlocks) lifetime_fp64_kernel(LifetimeLaunch P)
{
    __shared__ int s_defer[kDefer > 0 ? kDefer * kDeferStride : 1];
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool active = t < P.n_orbits;
    const unsigned mask = __ballot_sync(0xffffffffu, active);
    if (!active) return;

    int v, i, j;
    long long g;
    if (kPositionMajor) {
        // t = ((row * n_phase) + v) * dim + i over the rows of this launch
        i = (int)(t % P.dim);
        const long long rv = t / P.dim;
        v = (int)(rv % P.n_phase);
        j = P.row0 + (int)(rv / P.n_phase);
        g = ((long long)j * P.dim + i) * P.n_phase + v;
    } else {
        g = (long long)P.row0 * P.dim * P.n_phase + t;
        v = (int)(g % P.n_phase);
        const long long pidx = g / P.n_phase;
        i = (int)(pidx % P.dim);
        j = (int)(pidx / P.dim);
    }

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
    if (!within_bounds(c0, gr.cpr)) {
        atomicOr(P.error, kErrStartCell);
    } else {
        lt = trace_orbit<kDefer>(o, position, ph.phi, P.w, gr, P.walk_cap, cnt, flags, s_defer + threadIdx.x);
        if (flags & kTraceWalkCap) atomicOr(P.error, kErrWalkCap);
    }
    P.out[g] = lt;
    if (P.out32) P.out32[g] = (float)lt;

    warp_flush(P.metrics, mask, cnt, flags, true);
}

// ---------------------------------------------------------------------------
// Lane-refill variant: persistent warps. A lane owns one orbit at a time and
// advances it one cell step per iteration; when its orbit finishes it takes the
// next orbit of the warp's chunk, so a warp no longer idles while its longest
// orbit walks on (orbits range from 0 to tens of cell steps). Warps take chunks
// of kRefillChunk consecutive orbits from a global counter. Every orbit runs
// exactly the reference's TraceOrbit sequence (trace_orbit in
// es_orbit_fp64.cuh, unrolled into steps), so results are identical to the
// one-thread-per-orbit kernel.
constexpr int kRefillChunk = 128;

struct LaneTally {
    unsigned long long cells = 0, imps = 0, cross = 0, start = 0;
    unsigned inside = 0, escaped = 0, bound = 0, max_cells = 0, max_imps = 0;
};

template <int kMinBlocks>
__global__ void __launch_bounds__(256, kMinBlocks) lifetime_fp64_refill_kernel(LifetimeLaunch P)
{
    const unsigned kFull = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;

    GridD gr;
    gr.imps = P.imps;
    gr.cell_end = P.cell_end;
    gr.start = P.spawn_start;
    gr.size = P.spawn_size;
    gr.cell = P.cell_size;
    gr.imp_r = P.imp_radius;
    gr.cpr = P.cpr;

    long long g = -1;  // orbit owned by this lane, -1 when idle
    OrbitD o;
    o.radius = P.radius;
    o.radius_sq = P.radius_sq;
    o.clockwise = P.clockwise != 0;
    dv2 pos = {0.0, 0.0};
    Isect next;
    double lifetime = kINF;
    int steps = 0, o_cells = 0, o_imps = 0;
    bool started = false;
    LaneTally tally;

    long long chunk_next = 0, chunk_end = 0;  // warp-uniform
    bool exhausted = false;                   // warp-uniform

    for (;;) {
        // ---- refill idle lanes from the warp's chunk ----
        unsigned idle = __ballot_sync(kFull, g < 0);
        while (idle != 0u && !exhausted) {
            if (chunk_next >= chunk_end) {
                unsigned long long base = 0;
                if (lane == 0) base = atomicAdd(P.work, (unsigned long long)kRefillChunk);
                base = __shfl_sync(kFull, base, 0);
                if ((long long)base >= P.n_orbits) {
                    exhausted = true;
                    break;
                }
                chunk_next = (long long)base;
                chunk_end = min((long long)base + kRefillChunk, P.n_orbits);
            }
            const long long avail = chunk_end - chunk_next;
            const int r = __popc(idle & lt_mask);
            if (g < 0 && r < avail) {
                g = chunk_next + r;
                // CreateParticle + TraceOrbit set-up (see lifetime_fp64_kernel)
                const long long gg = (long long)P.row0 * P.dim * P.n_phase + g;
                const int v = (int)(gg % P.n_phase);
                const long long pidx = gg / P.n_phase;
                const int i = (int)(pidx % P.dim);
                const int j = (int)(pidx / P.dim);
                pos = dv2{(double)i * P.dist + P.off_x, (double)j * P.dist + P.off_y};
                const PhaseOrbit ph = P.phase[v];
                const double shift_x = (ph.vel_y * P.radius) / P.speed;
                const double shift_y = (-ph.vel_x * P.radius) / P.speed;
                o.center = o.clockwise ? dv2{pos.x - shift_x, pos.y - shift_y} : dv2{pos.x + shift_x, pos.y + shift_y};
                o.bound_time = P.coherent ? kINF : ph.bound_dphi / P.w;
                o.particle_angle = ph.phi;
                next.position = pos;
                next.cell = get_cell(pos, gr.start, gr.size, gr.cpr);
                next.dphi = kPI2;
                next.incident_angle = ph.phi;
                lifetime = kINF;
                steps = o_cells = o_imps = 0;
                started = false;
            }
            chunk_next += min((long long)__popc(idle), avail);
            idle = __ballot_sync(kFull, g < 0);
        }
        if (__all_sync(kFull, g < 0)) break;
        if (g < 0) continue;

        // ---- one step of the owned orbit ----
        int k0 = 0, k1 = 0;
        bool avail_next = false;
        double vr_x = 0.0, vr_y = 0.0;
        bool finish = false;
        double result = 0.0;
        if (!started) {
            if (!within_bounds(next.cell, gr.cpr)) {
                atomicOr(P.error, kErrStartCell);
                finish = true;
            } else {
                const int pci = next.cell.y * gr.cpr + next.cell.x;
                k0 = (pci == 0) ? 0 : __ldg(gr.cell_end + pci - 1);
                k1 = __ldg(gr.cell_end + pci);
            }
        } else {
            Isect entry = next;
            avail_next = next_cell(o, o.particle_angle, gr, entry, next);
            vr_x = entry.incident_angle;
            vr_y = avail_next ? next.incident_angle : o.particle_angle;
            const int ci = entry.cell.y * gr.cpr + entry.cell.x;
            k0 = (ci > 0) ? __ldg(gr.cell_end + ci - 1) : 0;
            k1 = __ldg(gr.cell_end + ci);
            o_cells += 1;
            o_imps += k1 - k0;
        }

        bool inside = false;
        for (int k = k0; k < k1; k++) {
            const double2 imp = __ldg(gr.imps + k);
            const dv2 ip = {imp.x, imp.y};
            if (!started) {
                tally.start += 1;
                if (inside_impurity(pos, ip, gr.imp_r)) {
                    inside = true;
                    break;
                }
            } else if (circles_cross(o, ip, gr.imp_r)) {
                tally.cross += 1;
                const double t = first_cross_time(o, ip, gr.imp_r, P.w, vr_x, vr_y);
                lifetime = (t < lifetime) ? t : lifetime;
            }
        }

        if (!finish) {
            if (!started) {
                if (inside) {
                    tally.inside += 1;
                    finish = true;  // result 0
                } else {
                    started = true;
                }
            } else {
                bool clamp = false;
                if (lifetime < kINF) {
                    finish = clamp = true;
                    result = lifetime;
                } else if (!avail_next) {
                    tally.escaped += 1;
                    finish = clamp = true;  // result 0, then the bound check
                } else if (++steps >= P.walk_cap) {
                    atomicOr(P.error, kErrWalkCap);
                    finish = true;
                }
                if (clamp && result > o.bound_time) {
                    tally.bound += 1;
                    result = o.bound_time;
                }
            }
        }
        if (finish) {
            P.out[(long long)P.row0 * P.dim * P.n_phase + g] = result;
            if (P.out32) P.out32[(long long)P.row0 * P.dim * P.n_phase + g] = (float)result;
            tally.cells += (unsigned)o_cells;
            tally.imps += (unsigned)o_imps;
            tally.max_cells = max(tally.max_cells, (unsigned)o_cells);
            tally.max_imps = max(tally.max_imps, (unsigned)o_imps);
            g = -1;
        }
    }

    // ---- per-warp metric flush (all 32 lanes are here) ----
    unsigned long long s_cells = tally.cells, s_imps = tally.imps, s_cross = tally.cross, s_start = tally.start;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        s_cells += __shfl_xor_sync(kFull, s_cells, off);
        s_imps += __shfl_xor_sync(kFull, s_imps, off);
        s_cross += __shfl_xor_sync(kFull, s_cross, off);
        s_start += __shfl_xor_sync(kFull, s_start, off);
    }
    const unsigned s_inside = __reduce_add_sync(kFull, tally.inside);
    const unsigned s_escaped = __reduce_add_sync(kFull, tally.escaped);
    const unsigned s_bound = __reduce_add_sync(kFull, tally.bound);
    const unsigned m_cells = __reduce_max_sync(kFull, tally.max_cells);
    const unsigned m_imps = __reduce_max_sync(kFull, tally.max_imps);
    if (lane == 0) {
        if (s_cells) atomicAdd(P.metrics + kMetCells, s_cells);
        if (s_imps) atomicAdd(P.metrics + kMetImps, s_imps);
        if (s_cross) atomicAdd(P.metrics + kMetCrossings, s_cross);
        if (s_start) atomicAdd(P.metrics + kMetStartTests, s_start);
        if (s_inside) atomicAdd(P.metrics + kMetInside, (unsigned long long)s_inside);
        if (s_escaped) atomicAdd(P.metrics + kMetEscaped, (unsigned long long)s_escaped);
        if (s_bound) atomicAdd(P.metrics + kMetAtBound, (unsigned long long)s_bound);
        if (m_cells) atomicMax(P.metrics + kMetMaxCells, (unsigned long long)m_cells);
        if (m_imps) atomicMax(P.metrics + kMetMaxImps, (unsigned long long)m_imps);
    }
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
    return cudaGetLastError();
}

namespace {

template <int kMinBlocks>
cudaError_t launch_refill(const LifetimeLaunch& L, cudaStream_t s)
{
    static int blocks_per_sm = 0, sms = 0;
    if (blocks_per_sm == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, lifetime_fp64_refill_kernel<kMinBlocks>, 256, 0);
        if (blocks_per_sm < 1) blocks_per_sm = 1;
    }
    cudaError_t e = cudaMemsetAsync(L.work, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    const long long warps_needed = (L.n_orbits + kRefillChunk - 1) / kRefillChunk;
    long long blocks = (long long)sms * blocks_per_sm;
    if (blocks * 8 > warps_needed) blocks = (warps_needed + 7) / 8;
    lifetime_fp64_refill_kernel<kMinBlocks><<<(unsigned)blocks, 256, 0, s>>>(L);
    return cudaGetLastError();
}

template <int kMinBlocks, bool kPositionMajor, int kDefer>
cudaError_t launch_per_thread(const LifetimeLaunch& L, cudaStream_t s)
{
    const long long blocks = (L.n_orbits + 255) / 256;
    lifetime_fp64_kernel<kMinBlocks, kPositionMajor, kDefer><<<(unsigned)blocks, 256, 0, s>>>(L);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_lifetimes_fp64(const LifetimeLaunch& L, cudaStream_t s)
{
    if (L.n_orbits <= 0) return cudaSuccess;
    switch (L.variant) {
        case kLifetimePerThread: return launch_per_thread<3, false, 0>(L, s);
        case kLifetimeRefill: return launch_refill<2>(L, s);
        case kLifetimePerThreadLean: return launch_per_thread<4, false, 0>(L, s);
        case kLifetimeRefillLean: return launch_refill<3>(L, s);
        case kLifetimePositionMajor: return launch_per_thread<4, true, 0>(L, s);
        case kLifetimePositionMajorDefer: return launch_per_thread<4, true, 4>(L, s);
        case kLifetimePerThreadDefer: return launch_per_thread<4, false, 4>(L, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_debug_next_cell(double cx, double cy, double r, int clockwise, double phi, double start,
                                   double size, double cell, int cpr, const double* d_in6, double* d_out6,
                                   int* d_avail, cudaStream_t s)
{
    debug_next_cell_kernel<<<1, 1, 0, s>>>(cx, cy, r, clockwise, phi, start, size, cell, cpr, d_in6, d_out6, d_avail);
    return cudaGetLastError();
}

}  // namespace es
