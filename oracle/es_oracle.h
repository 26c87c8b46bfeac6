/* es_oracle.h - CPU restatement of ElasticScattering's FP64 real-space
 * conductivity path.
 *
 * TEST INFRASTRUCTURE ONLY. The oracle verifies the CUDA path: only
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load it. The
 * product (libes_cuda.so, the host runtime) never links or calls it.
 *
 * Parity: pinned bit for bit against the reference's own CPU code built from
 * its sources (oracle/_ref/libes_ref.so, see oracle/Makefile) and against the
 * reference's golden vectors (tests/golden/, generated by
 * tests/golden/make_golden.py from the reference's test files).
 */
#ifndef ES_ORACLE_H
#define ES_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Reference layouts (src/sim/es/settings.h:76-122, src/sim/es/particle_metrics.h:22-44). */
typedef struct orc_impurity_settings {
    double spawn_region_start;
    double spawn_region_size;
    double cell_size;
    int32_t cells_per_row;
    double impurity_radius;
} orc_impurity_settings;

typedef struct orc_metrics {
    int64_t cells_passed;
    int64_t impurities_tested;
    int64_t particles_inside_impurity;
    int64_t particles_escaped;
    int64_t particles_at_bound;
    int64_t max_impurities_tested;
    int64_t max_cells_passed;
} orc_metrics;

/* Sector/sample description: the fields Simulation's constructor and
 * InitSample derive (src/sim/Simulation.h:111-146). */
typedef struct orc_sim {
    int32_t positions_per_row;      /* dim (odd) */
    int32_t particles_per_quadrant; /* phi_steps (odd) */
    double region_size;
    double grid_cell_size;          /* GridInformation::cell_size, sets small_offset */
    double particle_speed;
    double alpha;
    double tau;                     /* coherent tau */
    int32_t is_clockwise;
    int32_t is_coherent;
} orc_sim;

/* ---- impurity grid (src/sim/Grid.cpp) ------------------------------------ */

/* libstdc++ std::default_random_engine (minstd_rand0) driving
 * std::uniform_real_distribution<double>(a, b): fills 2*count doubles x0,y0,x1,... */
void orc_generate_impurities(uint32_t seed, int64_t count, double a, double b, double* xy);

/* Sizes of Grid(seed, ...) (src/sim/Grid.cpp:28-46): returns 0 on success, 1 for
 * "Woah!" (>1e7 impurities), 2 for "No impurities". */
int orc_grid_seed_sizes(double region_size, double region_extends, double density,
                        int32_t target_cell_population, int64_t* unique_count, int32_t* cells_per_row);

/* Bins impurities into cells_per_row^2 cells with the reference's overlap rules
 * (src/sim/Grid.cpp:77-180) and flattens them (src/sim/Grid.cpp:92-110).
 * Pass out_xy == NULL to get only the total indexed count. Returns the total
 * indexed impurity count. cell_end has cells_per_row^2 entries. */
int64_t orc_grid_build(const double* xy, int64_t n, double region_extends, double region_size,
                       double impurity_radius, int32_t cells_per_row, double* out_xy, int32_t* cell_end);

void orc_grid_settings(double region_size, double region_extends, double impurity_radius,
                       int32_t cells_per_row, orc_impurity_settings* is);

/* ---- stage (a): lifetimes ----------------------------------------------- */

/* Raw lifetimes of every orbit in start-position rows [j0, j1) in the
 * reference's [j][i][q][p] order (src/sim/SimulationCPU.cpp:103-141). */
void orc_lifetimes(const orc_sim* s, const orc_impurity_settings* is, const double* imp_xy,
                   const int32_t* cell_end, double magnetic_field, int32_t j0, int32_t j1, double* out,
                   orc_metrics* m);

/* One orbit: CreateParticle + TraceOrbit (src/sim/es/lifetime.h:36-148). */
double orc_trace_one(const orc_sim* s, const orc_impurity_settings* is, const double* imp_xy,
                     const int32_t* cell_end, double magnetic_field, double px, double py, int32_t q,
                     int32_t p, orc_metrics* m);

/* One orbit with explicit ParticleSettings fields (src/sim/es/settings.h:87-98),
 * as the reference's LifetimeTests build them (tests/es/LifetimeTests.h:19-34). */
double orc_trace_explicit(const orc_impurity_settings* is, const double* imp_xy, const int32_t* cell_end,
                          double magnetic_field, double px, double py, int32_t q, int32_t p, double phi_start,
                          double phi_step, double alpha, double particle_speed, int32_t is_clockwise,
                          int32_t is_coherent);

/* ---- stages (b),(c): integration ---------------------------------------- */

/* SimulationCPU::DeriveTemperature (src/sim/SimulationCPU.cpp:143-155): sigma xx, xy
 * for one temperature from raw lifetimes of a full sector pass. */
void orc_derive_temperature(const orc_sim* s, double magnetic_field, double temperature,
                            const double* raw_lifetimes, double* out_xx_xy);

/* SimulationCPU::DeriveTemperatureWithImages (src/sim/SimulationCPU.cpp:157-172):
 * per-position maps (dim*dim each) and the sigmas. */
void orc_derive_temperature_images(const orc_sim* s, double magnetic_field, double temperature,
                                   const double* raw_lifetimes, double* out_xx_xy, double* lt_pos,
                                   double* xx_pos, double* xy_pos);

/* Helpers exposed for known-answer tests of the geometry (src/sim/es/details.h). */
double orc_get_angle(double px, double py, double cx, double cy, double radius, int clockwise);
int orc_angle_in_range(double phi, double lo, double hi, int clockwise);
double orc_cross_angle(double p, double q, int clockwise);
double orc_bound_time(double phi, double alpha, double w, int coherent, int is_electron, int is_future);
int orc_circles_cross(double cx, double cy, double r, double px, double py, double r2);
double orc_first_cross_time(double cx, double cy, double r, int clockwise, double particle_angle,
                            double ix, double iy, double ir, double w, double lo, double hi);
double orc_simpson_weight(int i, int dim);

/* One GetNextCell step (src/sim/es/cell_grid.h:132-181) on an explicit orbit.
 * in/out intersection = (pos.x, pos.y, incident_angle, dphi, cell.x, cell.y). */
int orc_next_cell(double cx, double cy, double r, int clockwise, double phi,
                  const orc_impurity_settings* is, double* inout6, double* next6);

#ifdef __cplusplus
}
#endif

#endif
