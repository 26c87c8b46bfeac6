// es_orbit_fp64.cuh - FP64 orbit geometry and cell walk on the device.
//
// Restates the reference's header-only numerical core operation by operation
// (src/sim/es/details.h, src/sim/es/cell_grid.h, src/sim/es/lifetime.h) so that
// the plain FP64 kernel takes the same decisions as the reference's CPU code.
// Translation units that include this header are compiled with -fmad=false:
// no multiply-add contraction, IEEE division and square root, so that only the
// libm-dependent asin differs in its last bits from the reference.
//
// What is NOT evaluated here: cos/sin of the phase angle, the orbit-centre
// shift and the sector bound time. They depend only on (phase, B) and are
// tabulated on the host with the reference's own expressions
// (es_phase_table in es_context.cu), which makes particle creation bit-exact.
#pragma once

#include <cfloat>
#include <cstdint>

namespace es {

// src/sim/es/constants.h:23-35 (same literals)
constexpr double kPI = 3.141592653589793238463;
constexpr double kPI2 = 6.283185307179586;
constexpr double kHALF_PI = 1.570796326794896619231;
constexpr double kINF = DBL_MAX;

struct dv2 {
    double x, y;
};
struct iv2 {
    int x, y;
};

// Intersection, src/sim/es/cell_grid.h:31-45
struct Isect {
    dv2 position;
    double incident_angle;
    double dphi;
    iv2 cell;
};

// Orbit, src/sim/es/details.h:31-62 (bound_phi is never read by TraceOrbit)
struct OrbitD {
    dv2 center;
    double radius;
    double radius_sq;
    double bound_time;
    double particle_angle;
    bool clockwise;
};

struct GridD {
    const double2* __restrict__ imps;
    const int* __restrict__ cell_end;
    double start;     // spawn_region_start
    double size;      // spawn_region_size
    double cell;      // cell_size
    double imp_r;     // impurity_radius
    int cpr;          // cells_per_row
};

// smod, details.h:79-83
__device__ __forceinline__ double smod(double a, double b) { return a - b * floor(a / b); }

// AngleVelocity, details.h:85-90
__device__ __forceinline__ double angle_velocity(double pos_angle, bool clockwise)
{
    const double offset = clockwise ? kHALF_PI : -kHALF_PI;
    return smod(pos_angle + offset, kPI2);
}

// GetAngle, details.h:93-107
__device__ __forceinline__ double get_angle(dv2 pos, const OrbitD& o)
{
    const double y_dist = pos.y - o.center.y;
    const bool left_side = pos.x < o.center.x;
    double angle;
    if (fabs(y_dist) > (1e-10 * o.radius)) {
        angle = asin(y_dist / o.radius);
        angle = left_side ? kPI - angle : angle;
    } else {
        angle = left_side ? kPI : 0.0;
    }
    return angle_velocity(angle, o.clockwise);
}

// GetCrossAngle, details.h:111-116
__device__ __forceinline__ double cross_angle(double p, double q, bool clockwise)
{
    const double g = clockwise ? (p - q) : (q - p);
    return smod(g, kPI2);
}

// AngleInRange, details.h:119-136
__device__ __forceinline__ bool angle_in_range(double phi, double rx, double ry, bool clockwise)
{
    if (fabs(rx - ry) < 1e-10) return true;
    const double low = clockwise ? ry : rx;
    double high = clockwise ? rx : ry;
    high = (high < low) ? (high + kPI2) : high;
    return (low < phi && phi < high) || (low < (phi + kPI2) && (phi + kPI2) < high);
}

// CirclesCross, details.h:141-151
__device__ __forceinline__ bool circles_cross(const OrbitD& o, dv2 p2, double r2)
{
    const double qx = o.center.x - p2.x;
    const double qy = o.center.y - p2.y;
    const double dist_sq = qx * qx + qy * qy;
    const double r_add = o.radius + r2;
    const double r_min = o.radius - r2;
    return (dist_sq < r_add * r_add) && (dist_sq > r_min * r_min);
}

// GetFirstCrossTime + GetCrossPoints, details.h:153-206
__device__ __forceinline__ double first_cross_time(const OrbitD& o, dv2 ip, double ir, double w, double vr_x,
                                                   double vr_y)
{
    const double qx = o.center.x - ip.x;
    const double qy = o.center.y - ip.y;
    const double dist_sq = qx * qx + qy * qy;
    const double dist = sqrt(dist_sq);
    const double xs = (dist_sq + o.radius_sq - ir * ir) / (2.0 * dist);
    const double ys = sqrt(o.radius_sq - xs * xs);
    const double ux = (ip.x - o.center.x) / dist;
    const double uy = (ip.y - o.center.y) / dist;

    const dv2 p1 = {o.center.x + ux * xs + uy * ys, o.center.y + uy * xs + -ux * ys};
    const dv2 p2 = {o.center.x + ux * xs + -uy * ys, o.center.y + uy * xs + ux * ys};

    // Crossing point 1, then 2 (the order of the reference's min updates).
    double t_min = kINF;
#pragma unroll 1
    for (int k = 0; k < 2; k++) {
        const double phi_k = get_angle(k == 0 ? p1 : p2, o);
        if (angle_in_range(phi_k, vr_x, vr_y, o.clockwise)) {
            const double t = cross_angle(o.particle_angle, phi_k, o.clockwise) / w;
            t_min = (t_min < t) ? t_min : t;
        }
    }
    return t_min;
}

// InsideImpurity, details.h:208-213
__device__ __forceinline__ bool inside_impurity(dv2 pos, dv2 imp, double r)
{
    const double dx = pos.x - imp.x;
    const double dy = pos.y - imp.y;
    return (r * r) > (dx * dx + dy * dy);
}

// get_cell, cell_grid.h:52-58
__device__ __forceinline__ iv2 get_cell(dv2 pos, double start, double size, int cpr)
{
    return iv2{(int)((pos.x - start) / size * (double)cpr), (int)((pos.y - start) / size * (double)cpr)};
}

__device__ __forceinline__ bool within_bounds(iv2 p, int cpr)
{
    return (p.x >= 0 && p.x < cpr) && (p.y >= 0 && p.y < cpr);
}

// PointInSegment, cell_grid.h:69-72
__device__ __forceinline__ bool point_in_segment(double point, double l0, double l1)
{
    return (point > l0 && point < l1) || (point < l0 && point > l1);
}

// DifferentPoint, cell_grid.h:74-77
__device__ __forceinline__ bool different_point(dv2 a, dv2 b, double L)
{
    return fabs(a.x - b.x) > 1e-6 * L || fabs(a.y - b.y) > 1e-6 * L;
}

// Update_Best_Intersect, cell_grid.h:80-89
__device__ __forceinline__ void update_best(const OrbitD& o, dv2 ip, iv2 next_cell, const Isect& last, Isect& closest,
                                            double L)
{
    const double incident = get_angle(ip, o);
    const double dphi = cross_angle(last.incident_angle, incident, o.clockwise);
    if (dphi < closest.dphi && different_point(ip, last.position, L)) {
        closest.position = ip;
        closest.cell = next_cell;
        closest.incident_angle = incident;
        closest.dphi = dphi;
    }
}

// UpdateFirstBoundaryIntersect, cell_grid.h:91-129
__device__ __forceinline__ void update_first_boundary(const OrbitD& o, int offx, int offy, dv2 p1, dv2 p2, double L,
                                                      const Isect& last, Isect& closest)
{
    const double ux = (p2.x - p1.x) / L;
    const double uy = (p2.y - p1.y) / L;
    const double pd = ux * (o.center.x - p1.x) + uy * (o.center.y - p1.y);
    const dv2 proj = {p1.x + ux * pd, p1.y + uy * pd};
    const double dx = proj.x - o.center.x;
    const double dy = proj.y - o.center.y;
    const double pcd = dx * dx + dy * dy;
    if (pcd >= o.radius_sq) return;

    const double s = sqrt(o.radius_sq - pcd);
    const double tex = ux * s, tey = uy * s;
    const dv2 i1 = {proj.x + tex, proj.y + tey};
    const dv2 i2 = {proj.x - tex, proj.y - tey};

    const bool horizontal = fabs(ux) > fabs(uy);
    const bool i1_valid = horizontal ? point_in_segment(i1.x, p1.x, p2.x) : point_in_segment(i1.y, p1.y, p2.y);
    const bool i2_valid = horizontal ? point_in_segment(i2.x, p1.x, p2.x) : point_in_segment(i2.y, p1.y, p2.y);

    const iv2 next_cell = {last.cell.x + offx, last.cell.y + offy};
    // i1 then i2, as the reference; one loop body keeps a single inlined copy
    // of GetAngle (asin) instead of two per edge.
#pragma unroll 1
    for (int k = 0; k < 2; k++) {
        const bool valid = k == 0 ? i1_valid : i2_valid;
        if (valid) update_best(o, k == 0 ? i1 : i2, next_cell, last, closest, L);
    }
}

// GetNextCell, cell_grid.h:132-181
__device__ __forceinline__ bool next_cell(const OrbitD& o, double phi, const GridD& g, Isect& last, Isect& next)
{
    last.dphi = kPI2;
    next = last;

    const double L = g.cell;
    const dv2 ll = {g.start + last.cell.x * L, g.start + last.cell.y * L};
    const dv2 lr = {ll.x + L, ll.y + 0.0};
    const dv2 tr = {ll.x + L, ll.y + L};
    const dv2 tl = {ll.x + 0.0, ll.y + L};

    // Edges in the reference's order: top (tl->tr), bottom (ll->lr),
    // right (lr->tr), left (ll->tl). One loop body, one inlined copy.
#pragma unroll 1
    for (int e = 0; e < 4; e++) {
        const dv2 p1 = e == 0 ? tl : (e == 2 ? lr : ll);
        const dv2 p2 = e == 0 ? tr : (e == 1 ? lr : (e == 2 ? tr : tl));
        const int offx = e < 2 ? 0 : (e == 2 ? 1 : -1);
        const int offy = e == 0 ? 1 : (e == 1 ? -1 : 0);
        update_first_boundary(o, offx, offy, p1, p2, L, last, next);
    }

    {
        const double delta = 1e-7 * L;
        const bool is_xlow = (next.position.x - ll.x) < delta;
        const bool is_xtop = (-next.position.x + L + ll.x) < delta;
        const bool is_ylow = (next.position.y - ll.y) < delta;
        const bool is_ytop = (-next.position.y + L + ll.y) < delta;

        int ox = next.cell.x - last.cell.x, oy = next.cell.y - last.cell.y;
        if (is_xtop && is_ylow) { ox = 1; oy = -1; }
        if (is_xlow && is_ylow) { ox = -1; oy = -1; }
        if (is_xlow && is_ytop) { ox = -1; oy = 1; }
        if (is_xtop && is_ytop) { ox = 1; oy = 1; }
        next.cell.x = last.cell.x + ox;
        next.cell.y = last.cell.y + oy;
    }

    const bool same_cell = next.cell.x == last.cell.x && next.cell.y == last.cell.y;
    return !same_cell && within_bounds(next.cell, g.cpr) &&
           !angle_in_range(phi, last.incident_angle, next.incident_angle, o.clockwise);
}

// The start-cell InsideImpurity scan (lifetime.h:90-99): the disks tested (up
// to and including the first that holds the start) and whether one does.
// tests < 0: not yet scanned.
struct StartScan {
    int tests;
    bool inside;
};

// The FP64 scan shared by the lanes of `mask`, which all start at `position`
// in cell `pci` (the phases of one start position): the lane of rank r tests
// disks k0 + r, k0 + r + n, ... (n lanes), and a ballot per round finds the
// first disk that holds the start. Each test is InsideImpurity on the same
// operands as the per-lane scan, so the decision and the count are its own.
__device__ __forceinline__ StartScan start_scan_shared64(const double2* imps, const int* cell_end, int pci,
                                                         dv2 position, double imp_r, unsigned mask)
{
    const unsigned lane = threadIdx.x & 31u;
    const int rank = __popc(mask & ((1u << lane) - 1u));
    const int n = __popc(mask);
    const int k0 = (pci == 0) ? 0 : __ldg(cell_end + pci - 1);
    const int k1 = __ldg(cell_end + pci);
    for (int base = k0; base < k1; base += n) {  // the same trip count on every lane of mask
        const int k = base + rank;
        bool inside = false;
        if (k < k1) {
            const double2 imp = __ldg(imps + k);
            inside = inside_impurity(position, dv2{imp.x, imp.y}, imp_r);
        }
        const unsigned hit = __ballot_sync(mask, inside);
        if (hit) {
            const int first = __popc(mask & ((1u << (__ffs(hit) - 1)) - 1u));
            return StartScan{base - k0 + first + 1, true};
        }
    }
    return StartScan{k1 - k0, false};
}

// Per-orbit counters; summed per warp before any global atomic.
struct OrbitCounters {
    int cells;
    int imps;
    int crossings;
    int start_tests;  // InsideImpurity evaluations of the start-cell scan
};

enum TraceFlag : int { kTraceOk = 0, kTraceInside = 1, kTraceEscaped = 2, kTraceAtBound = 4, kTraceWalkCap = 8 };

// TraceOrbit, src/sim/es/lifetime.h:78-148. `phi` is the particle's phase
// angle, `w` the unsigned angular speed. The loop is bounded by walk_cap cell
// steps (the reference loops while(1)); exceeding it flags kTraceWalkCap and
// returns 0.
//
// kDefer > 0: the cell's impurity scan first runs the cheap CirclesCross test
// over all impurities and parks the indices of crossing ones in `defer`
// (kDefer slots per thread, stride kDeferStride ints, shared memory); the
// expensive GetFirstCrossTime then runs over the parked indices only. A warp
// then executes the expensive branch about max-over-lanes(crossings) times per
// cell instead of once per impurity position that any lane crosses. The
// lifetime is a min over the same set of crossing times, so the result is
// identical.
constexpr int kDeferStride = 256;

//
// start: the start-cell scan when the caller's lanes shared it
// (start_scan_shared64), else tests < 0 and the scan runs here.
template <int kDefer = 0>
__device__ __forceinline__ double trace_orbit(const OrbitD& o, dv2 position, double phi, double w, const GridD& g,
                                              int walk_cap, OrbitCounters& cnt, int& flags, int* defer = nullptr,
                                              StartScan start = StartScan{-1, false})
{
    double lifetime = kINF;
    Isect next;
    next.position = position;
    next.cell = get_cell(position, g.start, g.size, g.cpr);
    next.dphi = kPI2;
    next.incident_angle = phi;

    if (start.tests >= 0) {
        cnt.start_tests += start.tests;
        if (start.inside) {
            flags = kTraceInside;
            return 0.0;
        }
    } else {
        const int pci = next.cell.y * g.cpr + next.cell.x;
        const int start = (pci == 0) ? 0 : __ldg(g.cell_end + pci - 1);
        const int end = __ldg(g.cell_end + pci);
        for (int k = start; k < end; k++) {
            const double2 imp = __ldg(g.imps + k);
            cnt.start_tests += 1;
            if (inside_impurity(position, dv2{imp.x, imp.y}, g.imp_r)) {
                flags = kTraceInside;
                return 0.0;
            }
        }
    }

    int steps = 0;
    for (;;) {
        Isect entry = next;
        const bool avail = next_cell(o, phi, g, entry, next);
        const double vr_x = entry.incident_angle;
        const double vr_y = avail ? next.incident_angle : phi;

        const int ci = entry.cell.y * g.cpr + entry.cell.x;
        const int start = (ci > 0) ? __ldg(g.cell_end + ci - 1) : 0;
        const int end = __ldg(g.cell_end + ci);
        cnt.cells += 1;
        cnt.imps += end - start;

        if (kDefer == 0) {
            for (int k = start; k < end; k++) {
                const double2 imp = __ldg(g.imps + k);
                const dv2 ip = {imp.x, imp.y};
                if (circles_cross(o, ip, g.imp_r)) {
                    cnt.crossings += 1;
                    const double t = first_cross_time(o, ip, g.imp_r, w, vr_x, vr_y);
                    lifetime = (t < lifetime) ? t : lifetime;
                }
            }
        } else {
            int parked = 0;
            for (int k = start; k < end; k++) {
                const double2 imp = __ldg(g.imps + k);
                if (circles_cross(o, dv2{imp.x, imp.y}, g.imp_r)) {
                    cnt.crossings += 1;
                    defer[parked * kDeferStride] = k;
                    if (++parked == kDefer) {
#pragma unroll 1
                        for (int c = 0; c < parked; c++) {
                            const double2 pi = __ldg(g.imps + defer[c * kDeferStride]);
                            const double t = first_cross_time(o, dv2{pi.x, pi.y}, g.imp_r, w, vr_x, vr_y);
                            lifetime = (t < lifetime) ? t : lifetime;
                        }
                        parked = 0;
                    }
                }
            }
#pragma unroll 1
            for (int c = 0; c < parked; c++) {
                const double2 pi = __ldg(g.imps + defer[c * kDeferStride]);
                const double t = first_cross_time(o, dv2{pi.x, pi.y}, g.imp_r, w, vr_x, vr_y);
                lifetime = (t < lifetime) ? t : lifetime;
            }
        }
        if (lifetime < kINF) break;
        if (!avail) {
            flags = kTraceEscaped;
            lifetime = 0.0;
            break;
        }
        if (++steps >= walk_cap) {
            flags = kTraceWalkCap;
            return 0.0;
        }
    }

    if (lifetime > o.bound_time) {
        flags |= kTraceAtBound;
        return o.bound_time;
    }
    return lifetime;
}

}  // namespace es
