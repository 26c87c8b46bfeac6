// es_orbit_split.cuh - stage (a), FP32/FP64 split precision: the per-orbit
// walk shared by the single-pass kernel (es_lifetime_split.cu) and the batched
// kernel (es_batch.cu).
//
// Same result as the plain FP64 kernel (the reference's TraceOrbit,
// src/sim/es/lifetime.h:78-148) but with the bulk of the work in FP32:
//
// 1. The reference's walk returns the first crossing, along the orbit, of any
//    impurity disk listed in the cells it visits before it stops: impurities
//    are filed under every cell they overlap (src/sim/Grid.cpp:112-180), so a
//    crossing point in a visited cell is always found in that visit. It stops
//    after the first visit holding an accepted crossing, and it stops early
//    (lifetime 0) when the next cell leaves the grid or the orbit comes full
//    circle -- then only the last cell's disks count, over the rest of the
//    circle (valid range [entry, start angle], lifetime.h:106).
// 2. This kernel walks the same cells in FP32, in angle space relative to the
//    orbit centre: the exit of a (convex) cell is the first crossing of any of
//    its four edge lines. Disks are tested in FP32 on cell-local coordinates
//    (CirclesCross decided in FP64 inside a tangency band) and their first
//    crossing advance is kept in FP32.
// 3. The winning disk's crossing time is then recomputed in FP64 with the
//    reference's own GetCrossPoints/GetAngle/GetCrossAngle arithmetic, and
//    clamped to the sector bound in FP64 -- the same bits as the plain path.
// 4. Every decision that FP32 cannot settle with margin -- an exit within a
//    guard angle of a corner, a cell arc shorter than the guard (where the
//    reference's 1e-6 L DifferentPoint rule can stop the walk), a start point
//    near an edge, two winners or a winner and an exit within the guard, the
//    walk bound -- sends the whole orbit to a list that the plain FP64 kernel
//    re-traces afterwards.
#pragma once

#include "es_internal.h"
#include "es_orbit_fp64.cuh"

namespace es {

namespace {

constexpr float kTwoPiF = 6.2831853071795864769f;
constexpr float kPiF = 3.1415926535897932385f;
constexpr float kGuard = 4e-6f;        // angle guard (rad): ~40x the FP32 angle error
constexpr double kPolarGuard = 4e-6;   // |x_line - x_centre| / r below which a vertical edge is re-traced
constexpr float kPolarMark = -2.0f;    // crossing value that marks such an edge (a miss is -1)

// Where the walk reads its per-pass constants. LaunchFields: from a
// LifetimeLaunch passed as the kernel parameter, whose fields are constant-bank
// operands and cost no registers. SharedFields: from a LifetimeLaunch in shared
// memory (the batched kernels), loaded where the compiler chooses.
struct LaunchFields {
    static constexpr bool kCrossOutOfLine = true;  // see first_cross_angle
    static constexpr bool kOrbitTable = true;      // see make_orbit
    static constexpr bool kTwoPassDisks = true;    // see trace_split
    const LifetimeLaunch& P;
    __device__ __forceinline__ const int* cell_end() const { return P.cell_end; }
    __device__ __forceinline__ const float2* imps32() const { return P.imps32; }
    __device__ __forceinline__ const double2* imps() const { return P.imps; }
    __device__ __forceinline__ const PhaseOrbit* phase() const { return P.phase; }
    __device__ __forceinline__ int* error() const { return P.error; }
    __device__ __forceinline__ double spawn_start() const { return P.spawn_start; }
    __device__ __forceinline__ double spawn_size() const { return P.spawn_size; }
    __device__ __forceinline__ double cell_size() const { return P.cell_size; }
    __device__ __forceinline__ double imp_radius() const { return P.imp_radius; }
    __device__ __forceinline__ double speed() const { return P.speed; }
    __device__ __forceinline__ double radius() const { return P.radius; }
    __device__ __forceinline__ double radius_sq() const { return P.radius_sq; }
    __device__ __forceinline__ double w() const { return P.w; }
    __device__ __forceinline__ double dist() const { return P.dist; }
    __device__ __forceinline__ double off_x() const { return P.off_x; }
    __device__ __forceinline__ double off_y() const { return P.off_y; }
    __device__ __forceinline__ int cpr() const { return P.cpr; }
    __device__ __forceinline__ int dim() const { return P.dim; }
    __device__ __forceinline__ int n_phase() const { return P.n_phase; }
    __device__ __forceinline__ int clockwise() const { return P.clockwise; }
    __device__ __forceinline__ int coherent() const { return P.coherent; }
    __device__ __forceinline__ int walk_cap() const { return P.walk_cap; }
    __device__ __forceinline__ const double4* orbit_table() const { return P.orbit_table; }
    // the pass's FP32 walk constants, host-computed launch parameters
    __device__ __forceinline__ float r32() const { return P.sc_r; }
    __device__ __forceinline__ float inv_r32() const { return P.sc_inv_r; }
    __device__ __forceinline__ float ir32() const { return P.sc_ir; }
    __device__ __forceinline__ float lo2() const { return P.sc_lo2; }
    __device__ __forceinline__ float hi2() const { return P.sc_hi2; }
    __device__ __forceinline__ float eps2() const { return P.sc_eps2; }
    __device__ __forceinline__ float band_d() const { return P.sc_band_d; }
    __device__ __forceinline__ float inv4r() const { return P.sc_inv4r; }
    __device__ __forceinline__ float tangent_tol() const { return P.sc_tangent_tol; }
    __device__ __forceinline__ unsigned long long inv_phase() const { return P.inv_phase; }
    __device__ __forceinline__ unsigned long long inv_dim() const { return P.inv_dim; }
};

struct SharedFields {
    static constexpr bool kCrossOutOfLine = false;
    static constexpr bool kOrbitTable = false;
    static constexpr bool kTwoPassDisks = false;
    const LifetimeLaunch* P;  // shared memory
    __device__ __forceinline__ const int* cell_end() const { return P->cell_end; }
    __device__ __forceinline__ const float2* imps32() const { return P->imps32; }
    __device__ __forceinline__ const double2* imps() const { return P->imps; }
    __device__ __forceinline__ const PhaseOrbit* phase() const { return P->phase; }
    __device__ __forceinline__ int* error() const { return P->error; }
    __device__ __forceinline__ double spawn_start() const { return P->spawn_start; }
    __device__ __forceinline__ double spawn_size() const { return P->spawn_size; }
    __device__ __forceinline__ double cell_size() const { return P->cell_size; }
    __device__ __forceinline__ double imp_radius() const { return P->imp_radius; }
    __device__ __forceinline__ double speed() const { return P->speed; }
    __device__ __forceinline__ double radius() const { return P->radius; }
    __device__ __forceinline__ double radius_sq() const { return P->radius_sq; }
    __device__ __forceinline__ double w() const { return P->w; }
    __device__ __forceinline__ double dist() const { return P->dist; }
    __device__ __forceinline__ double off_x() const { return P->off_x; }
    __device__ __forceinline__ double off_y() const { return P->off_y; }
    __device__ __forceinline__ int cpr() const { return P->cpr; }
    __device__ __forceinline__ int dim() const { return P->dim; }
    __device__ __forceinline__ int n_phase() const { return P->n_phase; }
    __device__ __forceinline__ int clockwise() const { return P->clockwise; }
    __device__ __forceinline__ int coherent() const { return P->coherent; }
    __device__ __forceinline__ int walk_cap() const { return P->walk_cap; }
    __device__ __forceinline__ const double4* orbit_table() const { return nullptr; }
    __device__ __forceinline__ float r32() const { return P->sc_r; }
    __device__ __forceinline__ float inv_r32() const { return P->sc_inv_r; }
    __device__ __forceinline__ float ir32() const { return P->sc_ir; }
    __device__ __forceinline__ float lo2() const { return P->sc_lo2; }
    __device__ __forceinline__ float hi2() const { return P->sc_hi2; }
    __device__ __forceinline__ float eps2() const { return P->sc_eps2; }
    __device__ __forceinline__ float band_d() const { return P->sc_band_d; }
    __device__ __forceinline__ float inv4r() const { return P->sc_inv4r; }
    __device__ __forceinline__ float tangent_tol() const { return P->sc_tangent_tol; }
    __device__ __forceinline__ unsigned long long inv_phase() const { return P->inv_phase; }
    __device__ __forceinline__ unsigned long long inv_dim() const { return P->inv_dim; }
};

__device__ __forceinline__ float wrap2pi(float a) { return a - kTwoPiF * floorf(a * (1.0f / kTwoPiF)); }

// Advance (angle travelled since the start, in [0, 2pi)) of position angle psi.
__device__ __forceinline__ float advance(float psi, float psi0, float dir) { return wrap2pi(dir * (psi - psi0)); }

// atan(t) for t in [0, 1] as t * P(t^2), a least-squares polynomial fitted
// for this kernel (max abs error 1.2e-7 rad evaluated in FP32).
__device__ __forceinline__ float atan_unit(float t)
{
    const float z = t * t;
    float p = 0.0024682495277374983f;
    p = fmaf(p, z, -0.01445870939642191f);
    p = fmaf(p, z, 0.03989958390593529f);
    p = fmaf(p, z, -0.07247953116893768f);
    p = fmaf(p, z, 0.10507321357727051f);
    p = fmaf(p, z, -0.14164334535598755f);
    p = fmaf(p, z, 0.19986537098884583f);
    p = fmaf(p, z, -0.3333265781402588f);
    p = fmaf(p, z, 0.9999998807907104f);
    return t * p;
}

// atan2 by octant reduction onto atan_unit; (0, 0) never reaches it.
__device__ __forceinline__ float fast_atan2(float y, float x)
{
    const float ax = fabsf(x), ay = fabsf(y);
    const float a0 = atan_unit(__fdividef(fminf(ax, ay), fmaxf(ax, ay)));
    float a = ay > ax ? 0.5f * kPiF - a0 : a0;
    a = x < 0.0f ? kPiF - a : a;
    return copysignf(a, y);
}

// 2 asin(sqrt(s2)): the crossing half-angle, a series for the usual tiny s2.
__device__ __forceinline__ float half_angle(float s2)
{
    const float x = sqrtf(s2);
    if (s2 < 0.01f) {
        // asin(x) = x (1 + z/6 + 3 z^2/40 + 5 z^3/112 + ...), z = x^2
        const float p = fmaf(fmaf(fmaf(0.044642857142857144f, s2, 0.075f), s2, 0.16666666666666666f), s2, 1.0f);
        return 2.0f * x * p;
    }
    return 2.0f * fast_atan2(x, sqrtf(1.0f - s2));
}

// The two crossing advances of the circle (radius r, centre at the origin)
// with an edge line at signed distance c64 (x = c for vertical lines, y = c for
// horizontal ones); both -1 when the line misses the circle. acos(|c| / r) is
// taken as atan2(sqrt(m (2 - m)), 1 - m) with m = (r - |c|) / r from FP64, which
// stays accurate near tangency. Returns 1 when the line lies within
// tangent_tol of tangency (| r - |c| | < tangent_tol).
__device__ __forceinline__ unsigned line_crossings(double c64, double r64, float inv_r, bool horizontal, float psi0,
                                                   float dir, float tangent_tol, float& a1, float& a2)
{
    const double m64 = r64 - fabs(c64);
    const unsigned near_tangent = fabsf((float)m64) < tangent_tol ? 1u : 0u;
    if (!(m64 > 0.0)) {
        a1 = a2 = -1.0f;
        return near_tangent;
    }
    const float m = (float)m64 * inv_r;
    const float ths = fast_atan2(sqrtf(m * (2.0f - m)), 1.0f - m);  // acos(|u|)
    float p1, p2;
    if (!horizontal) {
        const float acu = c64 >= 0.0 ? ths : kPiF - ths;
        p1 = acu;
        p2 = -acu;
    } else {
        const float asu = c64 >= 0.0 ? (0.5f * kPiF - ths) : (ths - 0.5f * kPiF);
        p1 = asu;
        p2 = kPiF - asu;
    }
    a1 = advance(p1, psi0, dir);
    a2 = advance(p2, psi0, dir);
    return near_tangent;
}

// FP64 GetFirstCrossTime without the valid-range filter, as an angle: the
// earlier of the two crossings' GetCrossAngle (src/sim/es/details.h:153-206).
// Divided by w this is the reference's time for the disk that holds the first
// crossing of the orbit. NaN when either crossing point's GetAngle is NaN:
// for a point at the very top or bottom of the orbit, rounding can make
// |y - c_y| / r exceed 1 and asin return NaN; the reference then drops that
// point (AngleInRange is false for NaN), which only the FP64 walk reproduces.
__device__ __forceinline__ double first_cross_angle_open(const OrbitD& o, dv2 ip, double ir)
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
    double a_min = kINF;
#pragma unroll 1
    for (int k = 0; k < 2; k++) {
        const double a = cross_angle(o.particle_angle, get_angle(k == 0 ? p1 : p2, o), o.clockwise);
        if (a != a) return a;
        a_min = (a_min < a) ? a_min : a;
    }
    return a_min;
}

// first_cross_angle_open as one out-of-line copy: the FP32 walk reaches it once
// or twice per orbit (the winner) and for grazing disks. In the single-pass
// kernel, keeping its FP64 sqrt/asin/division code out of the walk's body is
// 3-7% faster on B200 despite the spills around the call; in the batched
// kernel the spills cost more than the shorter body saves (measured 4-8%
// slower), so there it stays inline (F::kCrossOutOfLine).
__device__ __noinline__ double first_cross_angle_call(double cx, double cy, double radius, double radius_sq,
                                                      double particle_angle, int clockwise, double ipx, double ipy,
                                                      double ir)
{
    OrbitD o;
    o.center = dv2{cx, cy};
    o.radius = radius;
    o.radius_sq = radius_sq;
    o.bound_time = 0.0;
    o.particle_angle = particle_angle;
    o.clockwise = clockwise != 0;
    return first_cross_angle_open(o, dv2{ipx, ipy}, ir);
}

// first_cross_angle_open for lifetime_finish_kernel, with one GetAngle
// instead of two where that gives the same bits. p1 lies at the centre angle
// theta_u - beta of the disk direction theta_u and p2 at theta_u + beta
// (beta = atan2(ys, xs)). Travelling counter-clockwise the orbit reaches p1
// first, clockwise p2, unless the start angle lies between them. When that
// point's travel angle plus the arc 2 beta stays 1e-5 rad clear of 2 pi, and
// the arc is longer than 1e-5 rad, the other point's travel angle is the larger
// (FP32 arc, error below 1e-6 rad), so the minimum is this one. Otherwise both
// are computed as in first_cross_angle_open. A NaN first point returns NaN. A
// NaN second point, past the shortcut's test, is one the reference drops
// (AngleInRange is false), leaving the first.
__device__ __forceinline__ double first_cross_angle_first(const OrbitD& o, dv2 ip, double ir)
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
    const double af = cross_angle(o.particle_angle, get_angle(o.clockwise ? p2 : p1, o), o.clockwise);
    if (af != af) return af;
    const float arc = 2.0f * fast_atan2((float)ys, (float)xs);
    if (arc > 1e-5f && (float)af + arc < kTwoPiF - 1e-5f) return af;
    const double as = cross_angle(o.particle_angle, get_angle(o.clockwise ? p1 : p2, o), o.clockwise);
    if (as != as) return as;
    const double a1 = o.clockwise ? as : af, a2 = o.clockwise ? af : as;  // the angles of p1, p2
    return (a1 < a2) ? a1 : a2;
}

template <class F>
__device__ __forceinline__ double first_cross_angle(const OrbitD& o, dv2 ip, double ir)
{
    if (F::kCrossOutOfLine)
        return first_cross_angle_call(o.center.x, o.center.y, o.radius, o.radius_sq, o.particle_angle,
                                      o.clockwise ? 1 : 0, ip.x, ip.y, ir);
    return first_cross_angle_open(o, ip, ir);
}

struct SplitCounters {
    int cells, imps, crossings, start_tests;
};

// One disk of the scan: FP32 d^2 against r_i^2, decided in FP64 within a
// relative 1e-4 band of the edge.
template <class F>
__device__ __forceinline__ bool start_inside(const F& f, dv2 pos, float plx, float ply, float ir2, int k)
{
    const float2 q = __ldg(f.imps32() + k);
    const float dx = plx - q.x, dy = ply - q.y;
    const float d2 = fmaf(dx, dx, dy * dy);
    bool inside = d2 < ir2;
    if (fabsf(d2 - ir2) <= 1e-4f * ir2) {
        const double2 q64 = __ldg(f.imps() + k);
        inside = inside_impurity(pos, dv2{q64.x, q64.y}, f.imp_radius());
    }
    return inside;
}

// The scan by one lane: the disks of the start cell in order.
template <class F>
__device__ __forceinline__ StartScan start_scan_lane(const F& f, dv2 pos, int cx, int cy)
{
    const int c = cy * f.cpr() + cx;
    const int k0 = (c == 0) ? 0 : __ldg(f.cell_end() + c - 1);
    const int k1 = __ldg(f.cell_end() + c);
    const float plx = (float)(pos.x - (f.spawn_start() + cx * f.cell_size()));
    const float ply = (float)(pos.y - (f.spawn_start() + cy * f.cell_size()));
    const float ir = f.ir32();
    const float ir2 = ir * ir;
    for (int k = k0; k < k1; k++)
        if (start_inside(f, pos, plx, ply, ir2, k)) return StartScan{k - k0 + 1, true};
    return StartScan{k1 - k0, false};
}

// The same scan shared by the lanes of `mask`, which all start at `pos` (the
// phases of one start position): the lane of rank r tests disks k0 + r,
// k0 + r + n, ... (n lanes), and a ballot per round finds the first disk that
// holds the start. Each disk's test is start_inside, so the decision and the
// count are the per-lane scan's; the scan takes ceil(disks / n) rounds instead
// of one round per disk.
template <class F>
__device__ __forceinline__ StartScan start_scan_shared(const F& f, dv2 pos, int cx, int cy, unsigned mask)
{
    const unsigned lane = threadIdx.x & 31u;
    const int rank = __popc(mask & ((1u << lane) - 1u));
    const int n = __popc(mask);
    const int c = cy * f.cpr() + cx;
    const int k0 = (c == 0) ? 0 : __ldg(f.cell_end() + c - 1);
    const int k1 = __ldg(f.cell_end() + c);
    const float plx = (float)(pos.x - (f.spawn_start() + cx * f.cell_size()));
    const float ply = (float)(pos.y - (f.spawn_start() + cy * f.cell_size()));
    const float ir = f.ir32();
    const float ir2 = ir * ir;
    for (int base = k0; base < k1; base += n) {  // the same trip count on every lane of mask
        const int k = base + rank;
        const bool inside = k < k1 && start_inside(f, pos, plx, ply, ir2, k);
        const unsigned hit = __ballot_sync(mask, inside);
        if (hit) {
            const int first = __popc(mask & ((1u << (__ffs(hit) - 1)) - 1u));
            return StartScan{base - k0 + first + 1, true};
        }
    }
    return StartScan{k1 - k0, false};
}

// kSplitHit: the walk found its winning disk (and a near-equal runner-up);
// the FP64 time of the crossing is still to be computed (finish_hit).
enum SplitOutcome : int { kSplitDone = 0, kSplitRetrace = 1, kSplitHit = 2 };

// The winning disk's reference time (FP64) and the bound clamp. kFirstPoint:
// the crossing angles by first_cross_angle_first (lifetime_finish_kernel).
template <class F, bool kFirstPoint = false>
__device__ __forceinline__ double finish_hit(const F& f, const OrbitD& o, int win_k, int alt_k, int& flags)
{
    auto angle = [&](double2 q) {
        return kFirstPoint ? first_cross_angle_first(o, dv2{q.x, q.y}, f.imp_radius())
                           : first_cross_angle<F>(o, dv2{q.x, q.y}, f.imp_radius());
    };
    double t = angle(__ldg(f.imps() + win_k)) / f.w();
    if (alt_k >= 0) {
        const double t2 = angle(__ldg(f.imps() + alt_k)) / f.w();
        t = (t < t2) ? t : t2;
    }
    flags = kTraceOk;
    if (t > o.bound_time) {  // lifetime.h:142-146
        flags |= kTraceAtBound;
        t = o.bound_time;
    }
    return t;
}

// FP32 walk of one orbit. Returns kSplitDone with `out` set (and flags for the
// metrics), or kSplitRetrace when the orbit must be re-traced in FP64. With
// kDefer it returns kSplitHit instead of computing the winner's FP64 time: the
// winning disk in win.x, a near-equal second in win.y (else -1), for
// finish_hit in lifetime_finish_kernel.
template <class F, bool kDefer = false>
__device__ __forceinline__ int trace_split(const F& f, const OrbitD& o, dv2 pos, int cx, int cy, SplitCounters& cnt,
                                           int& flags, double& out, int2& win, StartScan start = StartScan{-1, false})
{
    const double r64 = o.radius;
    // The pass's FP32 constants (split_constants, es_host_math.h): r, 1/r, r_i;
    // CirclesCross in d^2: anything outside [lo2 - eps2, hi2 + eps2] misses for
    // sure (the FP32 d^2 error is below 3e-7 r^2), where lo2 = (r - r_i)^2 and
    // hi2 = (r + r_i)^2 in FP64 rounded once, eps2 = 2e-6 r^2; inside, |d - r|
    // decides, and within band_d = 0.02 r_i of the edge the decision and the
    // angle are taken in FP64; inv4r = 1 / (4 r).
    const float r = f.r32();
    const float inv_r = f.inv_r32();
    const float ir = f.ir32();
    const float lo2 = f.lo2(), hi2 = f.hi2();
    const float eps2 = f.eps2();
    const float band_d = f.band_d();
    const float inv4r = f.inv4r();
    // Position angle of the start: C = pos -/+ r (sin phi, -cos phi) (details.h:243-250).
    const float dir = o.clockwise ? -1.0f : 1.0f;
    const float psi0 = (float)(o.clockwise ? o.particle_angle - kHALF_PI : o.particle_angle + kHALF_PI);

    // (cx, cy): the start cell, (int)((pos - start) / size * cpr) per axis, from the caller.

    // Start-cell InsideImpurity scan (lifetime.h:90-99), FP32 with an FP64 band,
    // unless the caller's lanes shared it (start_scan_shared).
    if (start.tests < 0) start = start_scan_lane(f, pos, cx, cy);
    cnt.start_tests += start.tests;
    if (start.inside) {
        flags = kTraceInside;
        out = 0.0;
        return kSplitDone;
    }

    // Crossing advances of the current cell's four edge lines (x-lo, x-hi,
    // y-lo, y-hi), two per line, -1 when the line misses the circle. Moving to
    // a neighbour keeps three of the four lines, so one line is new per step.
    //
    // A vertical line that passes within kPolarGuard r of the centre's x meets
    // the circle within ~kPolarGuard rad of its top or bottom, where the
    // reference's GetAngle (asin(dy / r), |dy| ~ r) can round to NaN and
    // GetNextCell then drops that crossing (cell_grid.h:80-89) -- the walk stops
    // or takes another edge. Such lines get the crossing value kPolarMark, and a
    // cell that has one hands the orbit to the FP64 re-trace.
    //
    // Bit e of `tangent` marks a line within tangent_tol of tangency
    // (| r - |c| | < tangent_tol). GetNextCell's corner rule (cell_grid.h:154-167)
    // moves diagonally when the exit point lies within 1e-7 L of a
    // perpendicular edge. Where that edge's line is not near tangency, the
    // circle crosses it within 2e-7 L / (r |cos phi|) < 2e-6 rad of the exit
    // point (2x margin; |cos phi| > 0.1 L / r), so the exit-angle guards already
    // hand the orbit to the FP64 re-trace; a line with |cos phi| <= 0.1 L / r
    // at such a point has r - |c| <= r (0.1 L / r)^2 + 2e-7 L = tangent_tol.
    float la[4], lb[4];
    unsigned tangent = 0;
    const float tangent_tol = f.tangent_tol();  // r (0.1 L / r)^2 + 2e-7 L
    {
        const double L = f.cell_size();
        const double llx0 = f.spawn_start() + cx * L, lly0 = f.spawn_start() + cy * L;
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const double c64 = e == 0 ? llx0 - o.center.x
                                      : (e == 1 ? (llx0 + L) - o.center.x
                                                : (e == 2 ? lly0 - o.center.y : (lly0 + L) - o.center.y));
            tangent |= line_crossings(c64, r64, inv_r, e >= 2, psi0, dir, tangent_tol, la[e], lb[e]) << e;
            if (e < 2 && fabs(c64) < kPolarGuard * r64) la[e] = kPolarMark;
        }
    }

    float a_cur = 0.0f;        // advance at which the current cell was entered
    int entry_line = -1;       // edge line crossed to enter
    float global_a = 3.0e38f;  // earliest disk crossing seen in any visited cell
    int steps = 0;

    for (;;) {
        // ---- exit of this cell: first edge-line crossing after a_cur ----
        float ex = kTwoPiF, ex2 = kTwoPiF;
        int ex_line = -1, ex2_line = -1;
        bool ambiguous = false;
#pragma unroll
        for (int e = 0; e < 4; e++) {
            float a1 = la[e], a2 = lb[e];
            if (a1 < 0.0f) {
                if (a1 < -1.5f) ambiguous = true;  // kPolarMark: crossing at the top or bottom of the orbit
                continue;
            }
            if (e == entry_line) {
                // one of the two is the entry crossing itself
                const float d1 = fabsf(a1 - a_cur), d2 = fabsf(a2 - a_cur);
                if (fminf(d1, kTwoPiF - d1) < fminf(d2, kTwoPiF - d2)) a1 = -1.0f; else a2 = -1.0f;
            }
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const float a = h == 0 ? a1 : a2;
                if (a < 0.0f) continue;
                if (fabsf(a - a_cur) < kGuard || a > kTwoPiF - kGuard) {
                    ambiguous = true;  // crossing at the entry point (corner) or at the start angle
                    continue;
                }
                if (a < a_cur) continue;
                if (a < ex) {
                    ex2 = ex;
                    ex2_line = ex_line;
                    ex = a;
                    ex_line = e;
                } else if (a < ex2) {
                    ex2 = a;
                    ex2_line = e;
                }
            }
        }
        if (ambiguous) return kSplitRetrace;
        if (ex_line >= 0) {
            if (ex - a_cur < kGuard) return kSplitRetrace;                                        // tiny arc
            if (ex2_line >= 0 && ex2_line != ex_line && ex2 - ex < kGuard) return kSplitRetrace;  // corner
        }
        // Next cell across the exit line; a final visit when the orbit comes
        // full circle or the next cell leaves the grid.
        int nx = cx, ny = cy;
        if (ex_line == 0) nx -= 1;
        if (ex_line == 1) nx += 1;
        if (ex_line == 2) ny -= 1;
        if (ex_line == 3) ny += 1;
        const bool final_visit = ex_line < 0 || nx < 0 || ny < 0 || nx >= f.cpr() || ny >= f.cpr();

        // ---- disks of this cell ----
        const int c = cy * f.cpr() + cx;
        const int k0 = (c == 0) ? 0 : __ldg(f.cell_end() + c - 1);
        const int k1 = __ldg(f.cell_end() + c);
        cnt.cells += 1;
        cnt.imps += k1 - k0;
        // cell corner relative to the orbit centre
        const float ox = (float)((f.spawn_start() + cx * f.cell_size()) - o.center.x);
        const float oy = (float)((f.spawn_start() + cy * f.cell_size()) - o.center.y);
        if (ex_line >= 0 && (tangent & (ex_line < 2 ? 0xCu : 0x3u)) != 0) {
            // A perpendicular edge near tangency: the orbit runs almost parallel
            // to it, so the exit point can lie within 1e-7 L of it (the corner
            // rule) while its own crossing is far away in angle. The exit line's
            // two crossing points are checked against both perpendicular edges
            // (2x margin): first in FP32 from the cell-local centre offset with a
            // bound on its error (1e-5 r, valid while the exit line is not within
            // 5% of tangency), then, only if that cannot exclude it, in FP64.
            const float Lf = (float)f.cell_size();
            const bool horiz = ex_line >= 2;
            const float dl = horiz ? (ex_line == 2 ? oy : oy + Lf) : (ex_line == 0 ? ox : ox + Lf);
            const float h32 = sqrtf(fmaxf(fmaf(-dl, dl, r * r), 0.0f));
            const float cp = horiz ? -ox : -oy;
            const float tol32 = 2e-7f * Lf + 1e-5f * r;
            if (h32 < 0.05f * r || fabsf(cp + h32) < tol32 || fabsf(cp + h32 - Lf) < tol32 || fabsf(cp - h32) < tol32 ||
                fabsf(cp - h32 - Lf) < tol32) {
                const double L = f.cell_size();
                const double llx = f.spawn_start() + cx * L, lly = f.spawn_start() + cy * L;
                const double lv = horiz ? (ex_line == 2 ? lly : lly + L) : (ex_line == 0 ? llx : llx + L);
                const double d = lv - (horiz ? o.center.y : o.center.x);
                const double h = sqrt(fmax(o.radius_sq - d * d, 0.0));
                const double c_perp = horiz ? o.center.x : o.center.y;
                const double lo = horiz ? llx : lly;
                const double tol = 2e-7 * L;
                const double p1 = c_perp + h, p2 = c_perp - h;
                if (fabs(p1 - lo) < tol || fabs(p1 - (lo + L)) < tol || fabs(p2 - lo) < tol ||
                    fabs(p2 - (lo + L)) < tol)
                    return kSplitRetrace;
            }
        }
        const float2* const imps32 = f.imps32();
        float v1 = 3.0e38f, v2 = 3.0e38f, v3 = 3.0e38f;  // best three crossing advances of this visit
        int k1st = -1, k2nd = -1;
        // The crossing test of one disk appears twice below, identical in both
        // loop forms (kept inline: as a shared function or lambda it compiled
        // to more spills in the batched kernel).
        if constexpr (F::kTwoPassDisks) {
            // Two passes per 32 disks. The annulus reject is cheap and rejects
            // most disks; the crossing test behind it is ~50 instructions. In one
            // loop a warp runs that test for every disk that some lane has in
            // its annulus, with few lanes active. Pass 1 only marks each lane's
            // candidates in a bit mask, and pass 2 runs the test per candidate in
            // disk order, so the warp runs it as often as its busiest lane has
            // candidates: 1.5% (B = 20 T) to 4% (B = 1 T; 1e16 m^-2) faster per
            // pass on B200. The batched kernel keeps one loop (1.3% slower there).
            // The annulus test d^2 in [lo2 - eps2, hi2 + eps2] on the bit patterns:
            // d^2 >= +0 and the bounds are finite, so the unsigned difference of
            // the patterns orders like the floats (a lower bound below zero, which
            // rejects nothing, is taken as +0). Two disks per step in sm_100
            // packed FP32x2 operations, each element the scalar fmaf/add/mul.
            const float alo = lo2 - eps2;
            const unsigned blo = alo > 0.0f ? __float_as_uint(alo) : 0u;
            const unsigned bspan = __float_as_uint(hi2 + eps2) - blo;
            const float2 ox2 = make_float2(ox, ox), oy2 = make_float2(oy, oy);
            for (int kb = k0; kb < k1; kb += 32) {
                const int kn = min(32, k1 - kb);
                unsigned cand = 0u;
                int t = 0;
                for (; t + 1 < kn; t += 2) {
                    const float2 qa = __ldg(imps32 + kb + t), qb = __ldg(imps32 + kb + t + 1);
                    const float2 dx = __fadd2_rn(make_float2(qa.x, qb.x), ox2);
                    const float2 dy = __fadd2_rn(make_float2(qa.y, qb.y), oy2);
                    const float2 d2 = __ffma2_rn(dx, dx, __fmul2_rn(dy, dy));
                    cand |= (unsigned)(__float_as_uint(d2.x) - blo <= bspan) << t;
                    cand |= (unsigned)(__float_as_uint(d2.y) - blo <= bspan) << (t + 1);
                }
                if (t < kn) {
                    const float2 q = __ldg(imps32 + kb + t);
                    const float dx = q.x + ox, dy = q.y + oy;
                    const float d2 = fmaf(dx, dx, dy * dy);
                    cand |= (unsigned)(__float_as_uint(d2) - blo <= bspan) << t;
                }
                while (cand != 0u) {
                    const int k = kb + __ffs(cand) - 1;
                    cand &= cand - 1u;
                    const float2 q = __ldg(imps32 + k);
                    const float dx = q.x + ox, dy = q.y + oy;
                    const float d2 = fmaf(dx, dx, dy * dy);
                    const float d = d2 * rsqrtf(d2);
                    const float delta = d - r;
                    float a;
                    if (fabsf(fabsf(delta) - ir) <= band_d) {
                        // grazing disk: CirclesCross and the crossing angle in FP64
                        const double2 q64 = __ldg(f.imps() + k);
                        if (!circles_cross(o, dv2{q64.x, q64.y}, f.imp_radius())) continue;
                        const double a64 = first_cross_angle<F>(o, dv2{q64.x, q64.y}, f.imp_radius());
                        if (a64 != a64) return kSplitRetrace;  // a crossing point the reference drops
                        a = (float)a64;
                    } else {
                        if (!(fabsf(delta) < ir)) continue;
                        // crossing half-angle at the orbit centre:
                        // sin^2(beta / 2) = (ir - delta)(ir + delta) / (4 d r)
                        const float s2 = __fdividef((ir - delta) * (ir + delta) * inv4r, d);
                        const float beta = half_angle(s2);
                        // The disk's arc on the orbit is [ac - beta, ac + beta] in advance;
                        // one that touches the start angle is left to FP64 (taking the min
                        // of two separately wrapped FP32 advances could pick the wrong end).
                        const float ac = advance(fast_atan2(dy, dx), psi0, dir);
                        if (ac - beta < kGuard || ac + beta > kTwoPiF - kGuard) return kSplitRetrace;
                        a = ac - beta;
                    }
                    cnt.crossings += 1;
                    if (a < v1) {
                        v3 = v2;
                        v2 = v1;
                        k2nd = k1st;
                        v1 = a;
                        k1st = k;
                    } else if (a < v2) {
                        v3 = v2;
                        v2 = a;
                        k2nd = k;
                    } else if (a < v3) {
                        v3 = a;
                    }
                }
            }
        } else {
            for (int k = k0; k < k1; k++) {
                const float2 q = __ldg(imps32 + k);
                const float dx = q.x + ox, dy = q.y + oy;
                const float d2 = fmaf(dx, dx, dy * dy);
                if (d2 < lo2 - eps2 || d2 > hi2 + eps2) continue;
                const float d = d2 * rsqrtf(d2);
                const float delta = d - r;
                float a;
                if (fabsf(fabsf(delta) - ir) <= band_d) {
                    // grazing disk: CirclesCross and the crossing angle in FP64
                    const double2 q64 = __ldg(f.imps() + k);
                    if (!circles_cross(o, dv2{q64.x, q64.y}, f.imp_radius())) continue;
                    const double a64 = first_cross_angle<F>(o, dv2{q64.x, q64.y}, f.imp_radius());
                    if (a64 != a64) return kSplitRetrace;  // a crossing point the reference drops
                    a = (float)a64;
                } else {
                    if (!(fabsf(delta) < ir)) continue;
                    // crossing half-angle at the orbit centre:
                    // sin^2(beta / 2) = (ir - delta)(ir + delta) / (4 d r)
                    const float s2 = __fdividef((ir - delta) * (ir + delta) * inv4r, d);
                    const float beta = half_angle(s2);
                    // The disk's arc on the orbit is [ac - beta, ac + beta] in advance;
                    // one that touches the start angle is left to FP64 (taking the min
                    // of two separately wrapped FP32 advances could pick the wrong end).
                    const float ac = advance(fast_atan2(dy, dx), psi0, dir);
                    if (ac - beta < kGuard || ac + beta > kTwoPiF - kGuard) return kSplitRetrace;
                    a = ac - beta;
                }
                cnt.crossings += 1;
                if (a < v1) {
                    v3 = v2;
                    v2 = v1;
                    k2nd = k1st;
                    v1 = a;
                    k1st = k;
                } else if (a < v2) {
                    v3 = v2;
                    v2 = a;
                    k2nd = k;
                } else if (a < v3) {
                    v3 = a;
                }
            }
        }
        global_a = fminf(global_a, v1);

        if (!final_visit && !(global_a < ex + kGuard)) {
            if (++steps >= f.walk_cap()) return kSplitRetrace;
            // Enter the neighbour: the crossed line becomes its opposite line,
            // the parallel line moves by one cell, the other two are shared.
            entry_line = ex_line ^ 1;
            la[entry_line] = la[ex_line];
            lb[entry_line] = lb[ex_line];
            tangent = (tangent & ~(3u << (ex_line & 2))) | (((tangent >> ex_line) & 1u) << entry_line);
            cx = nx;
            cy = ny;
            {
                const double L = f.cell_size();
                const double nllx = f.spawn_start() + cx * L, nlly = f.spawn_start() + cy * L;
                const int e = ex_line;  // the new cell's line on the far side has the same index
                const double c64 = e == 0 ? nllx - o.center.x
                                          : (e == 1 ? (nllx + L) - o.center.x
                                                    : (e == 2 ? nlly - o.center.y : (nlly + L) - o.center.y));
                tangent |= line_crossings(c64, r64, inv_r, e >= 2, psi0, dir, tangent_tol, la[e], lb[e]) << e;
                if (e < 2 && fabs(c64) < kPolarGuard * r64) la[e] = kPolarMark;
            }
            a_cur = ex;
            continue;
        }
        // This visit ends the walk: a crossing at or before the exit (or the
        // final visit). The reference accepts this cell's disks only, over
        // [entry, exit] -- or over the rest of the circle in a final visit.
        if (!final_visit && global_a > ex - kGuard) return kSplitRetrace;  // winner at the exit
        if (k1st < 0) {
            if (global_a < ex + kGuard) return kSplitRetrace;  // a crossing before the exit but not in this cell
            flags = kTraceEscaped;                             // lifetime.h:131-136, then the bound check
            out = 0.0;
            if (out > o.bound_time) {
                flags |= kTraceAtBound;
                out = o.bound_time;
            }
            return kSplitDone;
        }
        if (global_a < v1 - kGuard) return kSplitRetrace;  // an earlier cell's crossing inside this visit
        if (v3 < v1 + kGuard) return kSplitRetrace;         // three near-equal winners
        // The first visit's valid range starts at, and a final visit's range ends
        // at, the particle's raw phase angle (lifetime.h:84,106), which is
        // negative for the incoherent sector's first quadrant. AngleInRange
        // (details.h:119-136) then tests x and x + 2pi only and rejects some
        // crossings the geometry accepts: clockwise in the final visit,
        // counter-clockwise in the first. The FP64 walk reproduces that.
        if (o.particle_angle < 0.0 && (o.clockwise ? final_visit : entry_line < 0)) return kSplitRetrace;
        if constexpr (kDefer) {
            win = make_int2(k1st, v2 < v1 + kGuard ? k2nd : -1);
            return kSplitHit;
        }
        out = finish_hit(f, o, k1st, v2 < v1 + kGuard ? k2nd : -1, flags);
        if (out != out) return kSplitRetrace;  // the winner's crossing point is one the reference drops
        return kSplitDone;
    }
}

// Orbit g of pass P (CreateParticle, src/sim/es/lifetime.h:36-58, with the
// host-tabulated phase constants).
template <class F>
__device__ __forceinline__ OrbitD make_orbit(const F& f, long long g, dv2& pos)
{
    int v, i, j;
    if (F::kOrbitTable && (unsigned long long)g < (1ull << 32)) {
        // 32-bit index arithmetic (every pass below 2^32 orbits): a 64-bit
        // division by a run-time divisor is a long instruction sequence, a
        // 32-bit one a shorter one, a multiply-high by ceil(2^64 / divisor)
        // (split_constants) one instruction pair
        const unsigned g32 = (unsigned)g, np = (unsigned)f.n_phase(), d = (unsigned)f.dim();
        const unsigned long long mp = f.inv_phase(), md = f.inv_dim();
        const unsigned pidx = mp ? (unsigned)__umul64hi((unsigned long long)g32, mp) : g32 / np;
        v = (int)(g32 - pidx * np);
        const unsigned row = md ? (unsigned)__umul64hi((unsigned long long)pidx, md) : pidx / d;
        i = (int)(pidx - row * d);
        j = (int)row;
    } else {
        v = (int)(g % f.n_phase());
        const long long pidx = g / f.n_phase();
        i = (int)(pidx % f.dim());
        j = (int)(pidx / f.dim());
    }
    pos = dv2{(double)i * f.dist() + f.off_x(), (double)j * f.dist() + f.off_y()};
    OrbitD o;
    o.radius = f.radius();
    o.radius_sq = f.radius_sq();
    o.clockwise = f.clockwise() != 0;
    if (F::kOrbitTable && f.orbit_table() != nullptr) {
        // the pass's table holds the same FP64 quotients (orbit_table_kernel)
        const double2* t = reinterpret_cast<const double2*>(f.orbit_table() + v);
        const double2 shift = __ldg(t), rest = __ldg(t + 1);  // (shift_x, shift_y), (bound_time, phi)
        o.center = o.clockwise ? dv2{pos.x - shift.x, pos.y - shift.y} : dv2{pos.x + shift.x, pos.y + shift.y};
        o.bound_time = rest.x;
        o.particle_angle = rest.y;
        return o;
    }
    const PhaseOrbit ph = f.phase()[v];
    const double shift_x = (ph.vel_y * o.radius) / f.speed();
    const double shift_y = (-ph.vel_x * o.radius) / f.speed();
    o.center = o.clockwise ? dv2{pos.x - shift_x, pos.y - shift_y} : dv2{pos.x + shift_x, pos.y + shift_y};
    o.bound_time = f.coherent() ? kINF : ph.bound_dphi / f.w();
    o.particle_angle = ph.phi;
    return o;
}

__device__ __forceinline__ OrbitD make_orbit(const LifetimeLaunch& P, long long g, dv2& pos)
{
    return make_orbit(LaunchFields{P}, g, pos);
}

// The start scan of the lanes of `mask` (0: none), shared when they all start
// at the same position inside the grid, else left to each lane (tests < 0).
// Every lane of a nonzero mask calls this.
template <class F>
__device__ __forceinline__ StartScan warp_start_scan(const F& f, dv2 pos, int cx, int cy, bool in_grid,
                                                     unsigned mask)
{
    if (mask == 0u) return StartScan{-1, false};
    const int src = __ffs(mask) - 1;
    const double x0 = __shfl_sync(mask, pos.x, src), y0 = __shfl_sync(mask, pos.y, src);
    if (!__all_sync(mask, pos.x == x0 && pos.y == y0 && in_grid)) return StartScan{-1, false};
    return start_scan_shared(f, pos, cx, cy, mask);
}

// The split walk of orbit g. Returns true when the orbit must be re-traced in
// FP64 (cnt and flags are then cleared); otherwise lt holds its lifetime.
// `mask`: the warp's lanes that call this together (their start scan is
// shared when they start at one position), or 0.
template <class F>
__device__ __forceinline__ bool split_orbit(const F& f, long long g, SplitCounters& cnt, int& flags, double& lt,
                                            unsigned mask = 0u)
{
    dv2 pos;
    const OrbitD o = make_orbit(f, g, pos);
    cnt = SplitCounters{0, 0, 0, 0};
    flags = kTraceOk;
    lt = 0.0;
    const int cx = (int)((pos.x - f.spawn_start()) / f.spawn_size() * (double)f.cpr());
    const int cy = (int)((pos.y - f.spawn_start()) / f.spawn_size() * (double)f.cpr());
    const bool in_grid = !(cx < 0 || cy < 0 || cx >= f.cpr() || cy >= f.cpr());
    const StartScan start = warp_start_scan(f, pos, cx, cy, in_grid, mask);
    if (!in_grid) {
        atomicOr(f.error(), kErrStartCell);
        return false;
    }
    int2 win;
    if (trace_split(f, o, pos, cx, cy, cnt, flags, lt, win, start) == kSplitRetrace) {
        cnt = SplitCounters{0, 0, 0, 0};
        flags = kTraceOk;
        return true;
    }
    return false;
}

// Lifetime slot of an orbit whose walk found its winning disk(s) but whose
// FP64 time is still to be taken (lifetime_finish_kernel): a negative double
// (lifetimes are >= 0) with the first disk in the low word and the second + 1
// (0: none) in the high word's low 31 bits.
__device__ __forceinline__ double encode_hit(int2 win)
{
    return __hiloint2double((int)(0x80000000u | (unsigned)(win.y + 1)), win.x);
}

__device__ __forceinline__ bool decode_hit(double v, int2& win)
{
    const long long b = __double_as_longlong(v);
    if (b >= 0) return false;
    win.x = (int)(unsigned)(b & 0xffffffffLL);
    win.y = (int)(((unsigned long long)b >> 32) & 0x7fffffffu) - 1;
    return true;
}

// A re-trace list entry made by lifetime_finish_kernel (an orbit whose walk
// was already counted): bit 62 of the orbit index.
constexpr long long kRetraceFromFinish = 1LL << 62;

// The split walk of orbit g up to its winning disk(s), for passes whose walks
// end after differing numbers of cell steps: the FP64 time of the winner --
// sqrt, asin and divisions of the reference's GetCrossPoints/GetAngle -- is
// left to lifetime_finish_kernel, which runs it for every such orbit of the
// pass with all lanes busy and none of the walk's registers live. Returns
// kSplitDone (lt set), kSplitHit (win set) or kSplitRetrace (cnt and flags
// cleared). `mask`: the warp's lanes that call this together (their start scan
// is shared when they start at one position).
template <class F>
__device__ __forceinline__ int split_orbit_walk(const F& f, long long g, unsigned mask, SplitCounters& cnt, int& flags,
                                                double& lt, int2& win)
{
    dv2 pos;
    const OrbitD o = make_orbit(f, g, pos);
    cnt = SplitCounters{0, 0, 0, 0};
    flags = kTraceOk;
    lt = 0.0;
    win = make_int2(-1, -1);
    const int cx = (int)((pos.x - f.spawn_start()) / f.spawn_size() * (double)f.cpr());
    const int cy = (int)((pos.y - f.spawn_start()) / f.spawn_size() * (double)f.cpr());
    const bool in_grid = !(cx < 0 || cy < 0 || cx >= f.cpr() || cy >= f.cpr());
    const StartScan start = warp_start_scan(f, pos, cx, cy, in_grid, mask);
    if (!in_grid) {
        atomicOr(f.error(), kErrStartCell);
        return kSplitDone;
    }
    const int st = trace_split<F, true>(f, o, pos, cx, cy, cnt, flags, lt, win, start);
    if (st == kSplitRetrace) {
        cnt = SplitCounters{0, 0, 0, 0};
        flags = kTraceOk;
    }
    return st;
}

// The counters split_orbit_walk gave orbit g (the walk is deterministic):
// what the pass already counted for an orbit that lifetime_finish_kernel
// hands to the FP64 re-trace.
__device__ __forceinline__ SplitCounters split_walk_counters(const LifetimeLaunch& P, long long g)
{
    SplitCounters cnt;
    int flags;
    double lt;
    int2 win;
    split_orbit_walk(LaunchFields{P}, g, 0u, cnt, flags, lt, win);
    return cnt;
}

// Exact FP64 TraceOrbit of orbit g (src/sim/es/lifetime.h:78-148): writes the
// lifetime and adds the orbit's counters to `cnt` (and its flags' counts to
// `in`, `esc`, `bound`, its maxima to `max_cells`, `max_imps`).
__device__ __forceinline__ void retrace_orbit(const LifetimeLaunch& P, long long g, OrbitCounters& cnt,
                                              unsigned& in, unsigned& esc, unsigned& bound, unsigned& max_cells,
                                              unsigned& max_imps)
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
    int flags = kTraceOk;
    const double lt = trace_orbit(o, pos, o.particle_angle, P.w, gr, P.walk_cap, c, flags);
    if (flags & kTraceWalkCap) atomicOr(P.error, kErrWalkCap);
    P.out[g] = lt;
    cnt.cells += c.cells;
    cnt.imps += c.imps;
    cnt.crossings += c.crossings;
    cnt.start_tests += c.start_tests;
    in += (flags & kTraceInside) ? 1u : 0u;
    esc += (flags & kTraceEscaped) ? 1u : 0u;
    bound += (flags & kTraceAtBound) ? 1u : 0u;
    max_cells = max(max_cells, (unsigned)c.cells);
    max_imps = max(max_imps, (unsigned)c.imps);
}

// Metrics of the lanes in `mask` (one instance), one atomic per warp and counter.
__device__ __forceinline__ void flush_split_metrics(unsigned long long* metrics, unsigned mask, const SplitCounters& cnt,
                                                    int flags, bool live)
{
    const unsigned l = live ? 1u : 0u;
    const unsigned s_cells = __reduce_add_sync(mask, (unsigned)cnt.cells);
    const unsigned s_imps = __reduce_add_sync(mask, (unsigned)cnt.imps);
    const unsigned s_cross = __reduce_add_sync(mask, (unsigned)cnt.crossings);
    const unsigned s_start = __reduce_add_sync(mask, (unsigned)cnt.start_tests);
    const unsigned s_inside = __reduce_add_sync(mask, (flags & kTraceInside) ? l : 0u);
    const unsigned s_escaped = __reduce_add_sync(mask, (flags & kTraceEscaped) ? l : 0u);
    const unsigned s_bound = __reduce_add_sync(mask, (flags & kTraceAtBound) ? l : 0u);
    const unsigned m_cells = __reduce_max_sync(mask, (unsigned)cnt.cells);
    const unsigned m_imps = __reduce_max_sync(mask, (unsigned)cnt.imps);
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

}  // namespace

}  // namespace es
