/* es_oracle.c - CPU restatement of ElasticScattering's FP64 real-space
 * conductivity path (impurity grid, orbit lifetimes, Simpson integration).
 *
 * TEST INFRASTRUCTURE ONLY: the oracle for the CUDA path. Loaded by tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg; never by the product.
 *
 * Every function restates the reference operation by operation (same operand
 * order, no FMA contraction, glibc libm), so that on this toolchain it agrees
 * bit for bit with the reference's own CPU code (checked by
 * tests/test_oracle_pin.py against oracle/_ref/libes_ref.so). Citations are to
 * files of the reference project.
 */
#include "es_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* src/sim/es/constants.h:23-35 (same literals). */
#define ES_M0 9.10938188e-31
#define ES_M (5.0 * ES_M0)
#define ES_E 1.60217646e-19
#define ES_HBAR 1.05457148e-34
#define ES_C1 1.15e-9
#define ES_KB 1.380649e-23
#define ES_PI 3.141592653589793238463
#define ES_PI2 6.283185307179586
#define ES_HALF_PI 1.570796326794896619231
#define ES_INF (DBL_MAX)

typedef struct { double x, y; } v2;
typedef struct { int x, y; } v2i;

typedef struct {
    v2 position;
    double incident_angle;
    double dphi;
    v2i entering_cell;
} isect; /* Intersection, src/sim/es/cell_grid.h:31-45 */

typedef struct {
    v2 center;
    double radius;
    double radius_squared;
    double bound_time;
    double particle_angle;
    int clockwise;
} orbit_t; /* Orbit, src/sim/es/details.h:31-62 */

/* ---- src/sim/es/details.h ----------------------------------------------- */

/* smod, details.h:79-83 */
static double smod(double a, double b) { return a - b * floor(a / b); }

/* AngleVelocity, details.h:85-90 */
static double angle_velocity(double pos_angle, int clockwise)
{
    double offset = clockwise ? ES_HALF_PI : -ES_HALF_PI;
    return smod(pos_angle + offset, ES_PI2);
}

/* GetAngle, details.h:93-107 */
static double get_angle(v2 pos, const orbit_t* o)
{
    const double y_dist = pos.y - o->center.y;
    const int left_side = pos.x < o->center.x;
    double angle = 0;
    if (fabs(y_dist) > (1e-10 * o->radius)) {
        angle = asin(y_dist / o->radius);
        angle = left_side ? ES_PI - angle : angle;
    } else {
        angle = left_side ? ES_PI : 0;
    }
    return angle_velocity(angle, o->clockwise);
}

/* GetCrossAngle, details.h:111-116 */
static double cross_angle(double p, double q, int clockwise)
{
    const double g = clockwise ? (p - q) : (q - p);
    return smod(g, ES_PI2);
}

/* AngleInRange, details.h:119-136 */
static int angle_in_range(double phi, v2 range, int clockwise)
{
    if (fabs(range.x - range.y) < 1e-10) return 1;
    double low = clockwise ? range.y : range.x;
    double high = clockwise ? range.x : range.y;
    high = (high < low) ? (high + ES_PI2) : high;
    return (low < phi && phi < high) || (low < (phi + ES_PI2) && (phi + ES_PI2) < high);
}

/* CirclesCross, details.h:141-151 (the reference's dot is a.x*b.x + b.y*b.y,
 * only ever called as dot(q, q)). */
static int circles_cross(const orbit_t* o, v2 p2, double r2)
{
    const v2 q = {o->center.x - p2.x, o->center.y - p2.y};
    const double dist_squared = q.x * q.x + q.y * q.y;
    const double r_add = o->radius + r2;
    const double r_min = o->radius - r2;
    return (dist_squared < r_add * r_add) && (dist_squared > r_min * r_min);
}

/* GetFirstCrossTime + GetCrossPoints, details.h:153-206 */
static double first_cross_time(const orbit_t* o, v2 ip, double ir, double w, v2 valid_range)
{
    const v2 q = {o->center.x - ip.x, o->center.y - ip.y};
    const double dist_squared = q.x * q.x + q.y * q.y;
    const double dist = sqrt(dist_squared);
    const double xs = (dist_squared + o->radius_squared - ir * ir) / (2.0 * dist);
    const double ys = sqrt(o->radius_squared - xs * xs);
    const v2 u = {(ip.x - o->center.x) / dist, (ip.y - o->center.y) / dist};

    const v2 p1 = {o->center.x + u.x * xs + u.y * ys, o->center.y + u.y * xs + -u.x * ys};
    const v2 p2 = {o->center.x + u.x * xs + -u.y * ys, o->center.y + u.y * xs + u.x * ys};

    const double phi1 = get_angle(p1, o);
    const double phi2 = get_angle(p2, o);

    double traversal_time = ES_INF;
    if (angle_in_range(phi1, valid_range, o->clockwise)) {
        const double t = cross_angle(o->particle_angle, phi1, o->clockwise) / w;
        traversal_time = (traversal_time < t) ? traversal_time : t;
    }
    if (angle_in_range(phi2, valid_range, o->clockwise)) {
        const double t = cross_angle(o->particle_angle, phi2, o->clockwise) / w;
        traversal_time = (traversal_time < t) ? traversal_time : t;
    }
    return traversal_time;
}

/* InsideImpurity, details.h:208-213 */
static int inside_impurity(v2 pos, v2 imp, double r)
{
    const v2 d = {pos.x - imp.x, pos.y - imp.y};
    return (r * r) > (d.x * d.x + d.y * d.y);
}

/* GetBoundTime, details.h:219-228 */
static double bound_time(double phi, double alpha, double w, int coherent, int is_electron, int is_future)
{
    if (coherent) return ES_INF;
    const double remaining = smod(phi + alpha, ES_HALF_PI);
    double dphi = (is_electron != is_future) ? remaining : (2.0 * alpha - remaining);
    return dphi / w;
}

/* ---- src/sim/es/cell_grid.h --------------------------------------------- */

/* get_cell, cell_grid.h:52-58 */
static v2i get_cell(v2 pos, double start, double size, int cpr)
{
    v2i c = {(int)((pos.x - start) / size * (double)(cpr)), (int)((pos.y - start) / size * (double)(cpr))};
    return c;
}

/* to_world, cell_grid.h:60-63 */
static v2 to_world(v2i c, double start, double cell_size)
{
    v2 r = {start + c.x * cell_size, start + c.y * cell_size};
    return r;
}

static int within_bounds(v2i p, int cpr) { return (p.x >= 0 && p.x < cpr) && (p.y >= 0 && p.y < cpr); }

/* PointInSegment, cell_grid.h:69-72 */
static int point_in_segment(double point, double l0, double l1)
{
    return (point > l0 && point < l1) || (point < l0 && point > l1);
}

/* DifferentPoint, cell_grid.h:74-77 */
static int different_point(v2 p1, v2 p2, double L)
{
    return fabs(p1.x - p2.x) > 1e-6 * L || fabs(p1.y - p2.y) > 1e-6 * L;
}

/* Update_Best_Intersect, cell_grid.h:80-89 */
static void update_best(const orbit_t* o, v2 ip, v2i next_cell, const isect* last, isect* closest, double L)
{
    const double incident = get_angle(ip, o);
    const double dphi = cross_angle(last->incident_angle, incident, o->clockwise);
    if (dphi < closest->dphi && different_point(ip, last->position, L)) {
        closest->position = ip;
        closest->entering_cell = next_cell;
        closest->incident_angle = incident;
        closest->dphi = dphi;
    }
}

/* UpdateFirstBoundaryIntersect, cell_grid.h:91-129 (pow(d, 2) is d*d). */
static void update_first_boundary(const orbit_t* o, v2i off, v2 p1, v2 p2, double L, const isect* last,
                                  isect* closest)
{
    const v2 u = {(p2.x - p1.x) / L, (p2.y - p1.y) / L};
    const double pd = u.x * (o->center.x - p1.x) + u.y * (o->center.y - p1.y);
    const v2 proj = {p1.x + u.x * pd, p1.y + u.y * pd};
    const double dx = proj.x - o->center.x;
    const double dy = proj.y - o->center.y;
    const double pcd = dx * dx + dy * dy;
    if (pcd >= o->radius_squared) return;

    const double s = sqrt(o->radius_squared - pcd);
    const v2 te = {u.x * s, u.y * s};
    const v2 i1 = {proj.x + te.x, proj.y + te.y};
    const v2 i2 = {proj.x - te.x, proj.y - te.y};

    const int horizontal = fabs(u.x) > fabs(u.y);
    const int i1_valid = horizontal ? point_in_segment(i1.x, p1.x, p2.x) : point_in_segment(i1.y, p1.y, p2.y);
    const int i2_valid = horizontal ? point_in_segment(i2.x, p1.x, p2.x) : point_in_segment(i2.y, p1.y, p2.y);

    const v2i next_cell = {last->entering_cell.x + off.x, last->entering_cell.y + off.y};
    if (i1_valid) update_best(o, i1, next_cell, last, closest, L);
    if (i2_valid) update_best(o, i2, next_cell, last, closest, L);
}

/* GetNextCell, cell_grid.h:132-181 */
static int next_cell(const orbit_t* o, double phi, const orc_impurity_settings* is, isect* last, isect* next)
{
    last->dphi = ES_PI2;
    *next = *last;

    const double L = is->cell_size;
    const v2 ll = to_world(last->entering_cell, is->spawn_region_start, L);
    const v2 lr = {ll.x + L, ll.y + 0};
    const v2 tr = {ll.x + L, ll.y + L};
    const v2 tl = {ll.x + 0, ll.y + L};

    const v2i up = {0, 1}, down = {0, -1}, right = {1, 0}, left = {-1, 0};
    update_first_boundary(o, up, tl, tr, L, last, next);
    update_first_boundary(o, down, ll, lr, L, last, next);
    update_first_boundary(o, right, lr, tr, L, last, next);
    update_first_boundary(o, left, ll, tl, L, last, next);

    {
        const double delta = 1e-7 * L;
        const int is_xlow = (next->position.x - ll.x) < delta;
        const int is_xtop = (-next->position.x + L + ll.x) < delta;
        const int is_ylow = (next->position.y - ll.y) < delta;
        const int is_ytop = (-next->position.y + L + ll.y) < delta;

        v2i offset = {next->entering_cell.x - last->entering_cell.x, next->entering_cell.y - last->entering_cell.y};
        if (is_xtop && is_ylow) { offset.x = 1; offset.y = -1; }
        if (is_xlow && is_ylow) { offset.x = -1; offset.y = -1; }
        if (is_xlow && is_ytop) { offset.x = -1; offset.y = 1; }
        if (is_xtop && is_ytop) { offset.x = 1; offset.y = 1; }
        next->entering_cell.x = last->entering_cell.x + offset.x;
        next->entering_cell.y = last->entering_cell.y + offset.y;
    }

    const int same_cell = next->entering_cell.x == last->entering_cell.x && next->entering_cell.y == last->entering_cell.y;
    const v2 range = {last->incident_angle, next->incident_angle};
    return !same_cell && within_bounds(next->entering_cell, is->cells_per_row) && !angle_in_range(phi, range, o->clockwise);
}

/* ---- src/sim/es/lifetime.h ---------------------------------------------- */

typedef struct {
    int64_t cells;
    int64_t imps;
} orbit_counts;

/* CreateParticle (lifetime.h:36-58) followed by TraceOrbit (lifetime.h:78-148). */
static double trace(const orc_sim* s, const orc_impurity_settings* is, const v2* imps, const int32_t* cell_end,
                    double w, v2 position, int q, int p, double phi_start, double phi_step, orc_metrics* m,
                    orbit_counts* cnt)
{
    /* CreateParticle */
    const double phi = phi_start + q * ES_HALF_PI + p * phi_step;
    const v2 vel = {cos(phi) * s->particle_speed, sin(phi) * s->particle_speed};
    orbit_t o;
    o.clockwise = s->is_clockwise;
    o.radius = s->particle_speed / w;
    o.radius_squared = o.radius * o.radius;
    {
        /* GetCyclotronOrbitCenter, details.h:243-250 */
        const v2 shift = {(vel.y * o.radius) / s->particle_speed, (-vel.x * o.radius) / s->particle_speed};
        if (s->is_clockwise) {
            o.center.x = position.x - shift.x;
            o.center.y = position.y - shift.y;
        } else {
            o.center.x = position.x + shift.x;
            o.center.y = position.y + shift.y;
        }
    }
    o.bound_time = bound_time(phi, s->alpha, w, s->is_coherent, s->is_clockwise, 0);
    o.particle_angle = phi;

    /* TraceOrbit */
    double lifetime = ES_INF;
    isect next;
    next.position = position;
    next.entering_cell = get_cell(position, is->spawn_region_start, is->spawn_region_size, is->cells_per_row);
    next.dphi = ES_PI2;
    next.incident_angle = phi;

    const int pci = next.entering_cell.y * is->cells_per_row + next.entering_cell.x;
    {
        const int start = (pci == 0) ? 0 : cell_end[pci - 1];
        const int end = cell_end[pci];
        for (int i = start; i < end; i++) {
            if (inside_impurity(position, imps[i], is->impurity_radius)) {
                m->particles_inside_impurity++;
                return 0;
            }
        }
    }

    for (;;) {
        isect entry = next;
        const int avail = next_cell(&o, phi, is, &entry, &next);
        const v2 valid = {entry.incident_angle, avail ? next.incident_angle : phi};

        const int ci = entry.entering_cell.y * is->cells_per_row + entry.entering_cell.x;
        const int start = (ci > 0) ? cell_end[ci - 1] : 0;
        const int end = cell_end[ci];
        m->cells_passed++;
        m->impurities_tested += end - start;
        cnt->cells++;
        cnt->imps += end - start;

        for (int i = start; i < end; i++) {
            if (circles_cross(&o, imps[i], is->impurity_radius)) {
                const double t = first_cross_time(&o, imps[i], is->impurity_radius, w, valid);
                lifetime = (t < lifetime) ? t : lifetime;
            }
        }
        if (lifetime < ES_INF) break;
        if (!avail) {
            m->particles_escaped++;
            lifetime = 0;
            break;
        }
    }

    if (lifetime > o.bound_time) {
        m->particles_at_bound++;
        return o.bound_time;
    }
    return lifetime;
}

/* Phase layout of Simulation::InitSample, src/sim/Simulation.h:111-126. */
static void sector_phase(const orc_sim* s, double* phi_start, double* phi_step, double* area)
{
    const double base_area = s->alpha * 2.0;
    *area = !s->is_coherent ? base_area : (ES_HALF_PI - base_area);
    *phi_start = (!s->is_coherent ? -s->alpha : s->alpha);
    *phi_step = *area / (s->particles_per_quadrant - 1);
}

void orc_lifetimes(const orc_sim* s, const orc_impurity_settings* is, const double* imp_xy,
                   const int32_t* cell_end, double magnetic_field, int32_t j0, int32_t j1, double* out,
                   orc_metrics* m)
{
    /* SimulationCPU::ComputeLifetimes, src/sim/SimulationCPU.cpp:103-141 */
    const double w = ES_E * magnetic_field / ES_M;
    const double dist = s->region_size / (double)(s->positions_per_row - 1);
    const v2 off = {s->grid_cell_size * 0.01, s->grid_cell_size * 0.005};
    double phi_start, phi_step, area;
    sector_phase(s, &phi_start, &phi_step, &area);
    const v2* imps = (const v2*)imp_xy;
    int64_t k = 0;
    for (int j = j0; j < j1; j++) {
        for (int i = 0; i < s->positions_per_row; i++) {
            const v2 position = {i * dist + off.x, j * dist + off.y};
            for (int q = 0; q < 4; q++) {
                for (int p = 0; p < s->particles_per_quadrant; p++) {
                    orbit_counts c = {0, 0};
                    out[k++] = trace(s, is, imps, cell_end, w, position, q, p, phi_start, phi_step, m, &c);
                    if (m->max_cells_passed < c.cells) m->max_cells_passed = c.cells;
                    if (m->max_impurities_tested < c.imps) m->max_impurities_tested = c.imps;
                }
            }
        }
    }
}

double orc_trace_one(const orc_sim* s, const orc_impurity_settings* is, const double* imp_xy,
                     const int32_t* cell_end, double magnetic_field, double px, double py, int32_t q,
                     int32_t p, orc_metrics* m)
{
    const double w = ES_E * magnetic_field / ES_M;
    double phi_start, phi_step, area;
    sector_phase(s, &phi_start, &phi_step, &area);
    orbit_counts c = {0, 0};
    const v2 pos = {px, py};
    return trace(s, is, (const v2*)imp_xy, cell_end, w, pos, q, p, phi_start, phi_step, m, &c);
}

double orc_trace_explicit(const orc_impurity_settings* is, const double* imp_xy, const int32_t* cell_end,
                          double magnetic_field, double px, double py, int32_t q, int32_t p, double phi_start,
                          double phi_step, double alpha, double particle_speed, int32_t is_clockwise,
                          int32_t is_coherent)
{
    orc_sim s;
    memset(&s, 0, sizeof(s));
    s.particle_speed = particle_speed;
    s.alpha = alpha;
    s.is_clockwise = is_clockwise;
    s.is_coherent = is_coherent;
    const double w = ES_E * magnetic_field / ES_M;
    orc_metrics m;
    memset(&m, 0, sizeof(m));
    orbit_counts c = {0, 0};
    const v2 pos = {px, py};
    return trace(&s, is, (const v2*)imp_xy, cell_end, w, pos, q, p, phi_start, phi_step, &m, &c);
}

/* ---- src/sim/es/util.h and the integration in SimulationCPU.cpp --------- */

/* SimpsonWeight, util.h:24-28 */
double orc_simpson_weight(int i, int dim)
{
    const double main_multiplier = (i % 2 == 0) ? 2.0 : 4.0;
    const int is_edge = (i == 0) || i == (dim - 1);
    return is_edge ? 1.0 : main_multiplier;
}

/* GetSigma, util.h:34-46 */
static double get_sigma(double lt, double phi, double tau, double w)
{
    const double z = exp(-lt / tau);
    double r = cos(phi) - cos(phi + w * lt) * z;
    r += w * tau * sin(phi + w * lt) * z;
    r -= w * tau * sin(phi);
    return r;
}

/* SigmaFactor and GetSigmaIntegrandFactor, src/sim/Simulation.h:69-76,88 */
static double integrand_factor(const orc_sim* s, double w, double tau)
{
    double area, ps0, step;
    sector_phase(s, &ps0, &step, &area);
    const double phi_integrand_factor = area / ((s->particles_per_quadrant - 1) * 3.0);
    const double kf = ES_M * s->particle_speed / ES_HBAR;
    double outside = (ES_E * ES_E * kf * kf) / (2.0 * ES_PI * ES_PI * ES_M * ES_C1);
    const double wct = w * tau;
    outside *= tau / (1.0 + wct * wct);
    const double a = 1.0 / (3.0 * (s->positions_per_row - 1));
    return a * a * phi_integrand_factor * outside * 1e-8;
}

/* GetTau, src/sim/Simulation.h:90 */
static double get_tau(const orc_sim* s, double temperature)
{
    return s->is_coherent ? s->tau : ES_HBAR / (ES_KB * temperature);
}

static void apply_sigma(const orc_sim* s, double w_signed, double tau, const double* raw, double* xx, double* xy,
                        double* lt_trunc)
{
    /* GetTruncatedLifetimes (Simulation.h:78-86) + ApplySigma (SimulationCPU.cpp:178-204) */
    const double max_lt = 15.0 * tau;
    double phi_start, phi_step, area;
    sector_phase(s, &phi_start, &phi_step, &area);
    const int dim = s->positions_per_row, ppq = s->particles_per_quadrant;
    for (int j = 0; j < dim; j++)
        for (int i = 0; i < dim; i++)
            for (int q = 0; q < 4; q++)
                for (int p = 0; p < ppq; p++) {
                    const int64_t idx = ((int64_t)j * dim + i) * 4 * ppq + q * ppq + p;
                    const double lt = (raw[idx] < max_lt) ? raw[idx] : max_lt;
                    if (lt_trunc) lt_trunc[idx] = lt;
                    const double phi = phi_start + q * ES_HALF_PI + p * phi_step;
                    const double base = get_sigma(lt, phi, tau, w_signed);
                    xx[idx] = base * cos(phi);
                    xy[idx] = base * sin(phi);
                }
}

/* IntegrateResult, SimulationCPU.cpp:206-222 (without the factor) */
static double integrate_result(const orc_sim* s, const double* v)
{
    const int dim = s->positions_per_row, ppq = s->particles_per_quadrant;
    double total = 0;
    for (int j = 0; j < dim; j++) {
        const double wy = orc_simpson_weight(j, dim);
        for (int i = 0; i < dim; i++) {
            const double wp = wy * orc_simpson_weight(i, dim);
            for (int q = 0; q < 4; q++)
                for (int p = 0; p < ppq; p++)
                    total += v[((int64_t)j * dim + i) * 4 * ppq + q * ppq + p] * (wp * orc_simpson_weight(p, ppq));
        }
    }
    return total;
}

/* IntegratePosition, SimulationCPU.cpp:224-243 */
static void integrate_position(const orc_sim* s, const double* v, double* out)
{
    const int dim = s->positions_per_row, ppq = s->particles_per_quadrant;
    double ps0, step, area;
    sector_phase(s, &ps0, &step, &area);
    const double phi_integrand_factor = area / ((ppq - 1) * 3.0);
    for (int j = 0; j < dim; j++)
        for (int i = 0; i < dim; i++) {
            double total = 0;
            for (int q = 0; q < 4; q++)
                for (int p = 0; p < ppq; p++)
                    total += v[((int64_t)j * dim + i) * 4 * ppq + q * ppq + p] * orc_simpson_weight(p, ppq);
            out[j * dim + i] = total * phi_integrand_factor;
        }
}

void orc_derive_temperature(const orc_sim* s, double magnetic_field, double temperature,
                            const double* raw_lifetimes, double* out_xx_xy)
{
    const double w = ES_E * magnetic_field / ES_M;
    const double w_signed = s->is_clockwise ? -w : w;
    const double tau = get_tau(s, temperature);
    const int64_t n = (int64_t)s->positions_per_row * s->positions_per_row * 4 * s->particles_per_quadrant;
    double* xx = (double*)malloc(sizeof(double) * n);
    double* xy = (double*)malloc(sizeof(double) * n);
    apply_sigma(s, w_signed, tau, raw_lifetimes, xx, xy, NULL);
    const double f = integrand_factor(s, w, tau);
    out_xx_xy[0] = integrate_result(s, xx) * f;
    out_xx_xy[1] = integrate_result(s, xy) * f;
    free(xx);
    free(xy);
}

void orc_derive_temperature_images(const orc_sim* s, double magnetic_field, double temperature,
                                   const double* raw_lifetimes, double* out_xx_xy, double* lt_pos,
                                   double* xx_pos, double* xy_pos)
{
    const double w = ES_E * magnetic_field / ES_M;
    const double w_signed = s->is_clockwise ? -w : w;
    const double tau = get_tau(s, temperature);
    const int64_t n = (int64_t)s->positions_per_row * s->positions_per_row * 4 * s->particles_per_quadrant;
    double* xx = (double*)malloc(sizeof(double) * n);
    double* xy = (double*)malloc(sizeof(double) * n);
    double* lt = (double*)malloc(sizeof(double) * n);
    apply_sigma(s, w_signed, tau, raw_lifetimes, xx, xy, lt);
    integrate_position(s, lt, lt_pos);
    integrate_position(s, xx, xx_pos);
    integrate_position(s, xy, xy_pos);
    const double f = integrand_factor(s, w, tau);
    out_xx_xy[0] = integrate_result(s, xx) * f;
    out_xx_xy[1] = integrate_result(s, xy) * f;
    free(xx);
    free(xy);
    free(lt);
}

/* ---- src/sim/Grid.cpp --------------------------------------------------- */

/* libstdc++'s std::default_random_engine is minstd_rand0 (x <- 16807 x mod 2^31-1);
 * Grid::GenerateImpurities passes the seed through an `int` parameter
 * (src/sim/Grid.cpp:61). */
static uint64_t minstd_seed(uint32_t seed)
{
    const uint64_t s = (uint64_t)(int64_t)(int32_t)seed;
    const uint64_t x = s % 2147483647ULL;
    return x == 0 ? 1 : x;
}

static uint64_t minstd_next(uint64_t* x)
{
    *x = (*x * 16807ULL) % 2147483647ULL;
    return *x;
}

/* std::generate_canonical<double, 53> for a generator with range
 * r = max - min + 1 = 2147483646: two draws (k = ceil(53 / floor(log2 r))),
 * the scale accumulated in long double and stored as double. */
static double canonical(uint64_t* x)
{
    const long double r = 2147483646.0L;
    double sum = 0, tmp = 1;
    for (int k = 0; k < 2; k++) {
        sum += (double)(minstd_next(x) - 1) * tmp;
        tmp = (double)((long double)tmp * r);
    }
    double ret = sum / tmp;
    if (ret >= 1.0) ret = nextafter(1.0, 0.0);
    return ret;
}

void orc_generate_impurities(uint32_t seed, int64_t count, double a, double b, double* xy)
{
    /* Grid::GenerateImpurities, src/sim/Grid.cpp:61-75: x then y per impurity,
     * uniform_real_distribution returns canonical * (b - a) + a. */
    uint64_t x = minstd_seed(seed);
    for (int64_t i = 0; i < 2 * count; i++) xy[i] = (canonical(&x) * (b - a)) + a;
}

int orc_grid_seed_sizes(double region_size, double region_extends, double density,
                        int32_t target_cell_population, int64_t* unique_count, int32_t* cells_per_row)
{
    /* Grid::Grid(seed, ...), src/sim/Grid.cpp:28-46 */
    const double lo = -region_extends, hi = region_size + region_extends;
    const double area_length = hi - lo;
    const double proposal = area_length * area_length * density;
    if (proposal > 1e7) return 1;
    if (proposal < 1) return 2;
    long u = (long)ceil(proposal);
    if (u < 1) u = 1;
    *unique_count = u;
    int c = (int)round(sqrt(u / (double)target_cell_population));
    *cells_per_row = c > 1 ? c : 1;
    return 0;
}

void orc_grid_settings(double region_size, double region_extends, double impurity_radius,
                       int32_t cells_per_row, orc_impurity_settings* is)
{
    /* Grid::GetSettings, src/sim/Grid.h:77-86 */
    const double lo = -region_extends, hi = region_size + region_extends;
    is->impurity_radius = impurity_radius;
    is->spawn_region_start = lo;
    is->spawn_region_size = hi - lo;
    is->cells_per_row = cells_per_row;
    is->cell_size = is->spawn_region_size / (double)cells_per_row;
}

typedef struct {
    double lo, size, cell_size;
    int cpr;
} grid_geo;

static v2i grid_cell(const grid_geo* g, double x, double y)
{
    /* Grid::get_cell, src/sim/Grid.cpp:182-188 */
    v2i c = {(int)((x - g->lo) / g->size * (double)(g->cpr)), (int)((y - g->lo) / g->size * (double)(g->cpr))};
    return c;
}

/* Cells one impurity is filed under, in the reference's push order
 * (add_to_overlapping_cells, src/sim/Grid.cpp:112-180). Returns the count. */
static int overlapping_cells(const grid_geo* g, v2 pos, double r, int* cells)
{
    const v2i probes[5] = {grid_cell(g, pos.x, pos.y), grid_cell(g, pos.x + r, pos.y), grid_cell(g, pos.x - r, pos.y),
                           grid_cell(g, pos.x, pos.y + r), grid_cell(g, pos.x, pos.y - r)};
    int n = 0;
    v2i added[5];
    int n_added = 0;
    for (int i = 0; i < 5; i++) {
        const v2i c = probes[i];
        int seen = 0;
        for (int k = 0; k < n_added; k++)
            if (added[k].x == c.x && added[k].y == c.y) seen = 1;
        if (!seen && within_bounds(c, g->cpr)) {
            added[n_added++] = c;
            cells[n++] = c.y * g->cpr + c.x;
        }
    }

    /* to_world uses spawn_range.x for both axes (src/sim/Grid.h:48-51). */
    const v2 ll = {g->lo + probes[0].x * g->cell_size, g->lo + probes[0].y * g->cell_size};
    const v2 lr = {g->cell_size + ll.x, 0 + ll.y};
    const v2 tl = {0 + ll.x, g->cell_size + ll.y};
    const v2 tr = {g->cell_size + ll.x, g->cell_size + ll.y};
    const double ir2 = r * r;
    const v2i cell = grid_cell(g, pos.x, pos.y);

    const v2 corners[4] = {tl, tr, ll, lr};
    const v2i offs[4] = {{-1, 1}, {1, 1}, {-1, -1}, {1, -1}};
    for (int k = 0; k < 4; k++) {
        const double dx = corners[k].x - pos.x, dy = corners[k].y - pos.y;
        if (dx * dx + dy * dy < ir2) {
            const v2i nc = {cell.x + offs[k].x, cell.y + offs[k].y};
            if (within_bounds(nc, g->cpr)) cells[n++] = nc.y * g->cpr + nc.x;
        }
    }
    return n;
}

int64_t orc_grid_build(const double* xy, int64_t n, double region_extends, double region_size,
                       double impurity_radius, int32_t cells_per_row, double* out_xy, int32_t* cell_end)
{
    /* GenerateImpurityCells + ConvertToIndex (src/sim/Grid.cpp:77-110): a stable
     * counting sort by cell reproduces the per-cell push order. */
    grid_geo g;
    g.lo = -region_extends;
    g.size = (region_size + region_extends) - (-region_extends);
    g.cpr = cells_per_row;
    g.cell_size = g.size / (double)cells_per_row;
    const int64_t ncell = (int64_t)cells_per_row * cells_per_row;
    int64_t* count = (int64_t*)calloc((size_t)ncell + 1, sizeof(int64_t));
    int cells[9];
    int64_t total = 0;
    for (int64_t i = 0; i < n; i++) {
        const v2 pos = {xy[2 * i], xy[2 * i + 1]};
        const int k = overlapping_cells(&g, pos, impurity_radius, cells);
        for (int c = 0; c < k; c++) count[cells[c]]++;
        total += k;
    }
    if (cell_end) {
        int64_t acc = 0;
        for (int64_t c = 0; c < ncell; c++) {
            acc += count[c];
            cell_end[c] = (int32_t)acc;
        }
    }
    if (out_xy) {
        int64_t* cursor = (int64_t*)malloc(sizeof(int64_t) * (size_t)ncell);
        int64_t acc = 0;
        for (int64_t c = 0; c < ncell; c++) {
            cursor[c] = acc;
            acc += count[c];
        }
        for (int64_t i = 0; i < n; i++) {
            const v2 pos = {xy[2 * i], xy[2 * i + 1]};
            const int k = overlapping_cells(&g, pos, impurity_radius, cells);
            for (int c = 0; c < k; c++) {
                const int64_t at = cursor[cells[c]]++;
                out_xy[2 * at] = pos.x;
                out_xy[2 * at + 1] = pos.y;
            }
        }
        free(cursor);
    }
    free(count);
    return total;
}

/* ---- geometry helpers for known-answer tests ---------------------------- */

static orbit_t mk_orbit(double cx, double cy, double r, int clockwise)
{
    orbit_t o;
    o.center.x = cx;
    o.center.y = cy;
    o.radius = r;
    o.radius_squared = r * r;
    o.clockwise = clockwise;
    o.bound_time = 0;
    o.particle_angle = 0;
    return o;
}

double orc_get_angle(double px, double py, double cx, double cy, double radius, int clockwise)
{
    orbit_t o = mk_orbit(cx, cy, radius, clockwise);
    v2 p = {px, py};
    return get_angle(p, &o);
}

int orc_angle_in_range(double phi, double lo, double hi, int clockwise)
{
    v2 r = {lo, hi};
    return angle_in_range(phi, r, clockwise);
}

double orc_cross_angle(double p, double q, int clockwise) { return cross_angle(p, q, clockwise); }

double orc_bound_time(double phi, double alpha, double w, int coherent, int is_electron, int is_future)
{
    return bound_time(phi, alpha, w, coherent, is_electron, is_future);
}

int orc_circles_cross(double cx, double cy, double r, double px, double py, double r2)
{
    orbit_t o = mk_orbit(cx, cy, r, 1);
    v2 p = {px, py};
    return circles_cross(&o, p, r2);
}

double orc_first_cross_time(double cx, double cy, double r, int clockwise, double particle_angle, double ix,
                            double iy, double ir, double w, double lo, double hi)
{
    orbit_t o = mk_orbit(cx, cy, r, clockwise);
    o.particle_angle = particle_angle;
    v2 ip = {ix, iy}, vr = {lo, hi};
    return first_cross_time(&o, ip, ir, w, vr);
}

int orc_next_cell(double cx, double cy, double r, int clockwise, double phi, const orc_impurity_settings* is,
                  double* inout6, double* next6)
{
    orbit_t o = mk_orbit(cx, cy, r, clockwise);
    isect last, next;
    last.position.x = inout6[0];
    last.position.y = inout6[1];
    last.incident_angle = inout6[2];
    last.dphi = inout6[3];
    last.entering_cell.x = (int)inout6[4];
    last.entering_cell.y = (int)inout6[5];
    const int avail = next_cell(&o, phi, is, &last, &next);
    next6[0] = next.position.x;
    next6[1] = next.position.y;
    next6[2] = next.incident_angle;
    next6[3] = next.dphi;
    next6[4] = next.entering_cell.x;
    next6[5] = next.entering_cell.y;
    return avail;
}
