/* C-callable harness around the reference's own CPU implementation.
 *
 * TEST INFRASTRUCTURE ONLY. This file is compiled together with the
 * reference's unmodified sources (src/sim/Grid.cpp, src/sim/SimulationCPU.cpp
 * and the header-only numerical core src/sim/es/*.h) read in place from the
 * reference tree, by oracle/Makefile, into oracle/_ref/libes_ref.so. It lets
 * the tests pin the oracle restatement (oracle/es_oracle.c) against the
 * reference bit for bit, and lets bench.py time the reference's CPU path
 * (`--impl reference`). No product code links it.
 *
 * Entry points mirror the reference's call sites:
 *   - Grid(seed, ...) / Grid(vector<v2>, ...)         src/sim/Grid.cpp:28-59
 *   - Simulation::InitSample                          src/sim/Simulation.h:111-126
 *   - SimulationCPU::ComputeLifetimes (private)       src/sim/SimulationCPU.cpp:103-141
 *   - SimulationCPU::ComputeSigmas                    src/sim/SimulationCPU.cpp:33-60
 *   - SimulationCPU::ComputeSigmasWithImages          src/sim/SimulationCPU.cpp:63-86
 */

/* ComputeLifetimes, DeriveTemperature and the settings structs are private or
 * protected members of SimulationCPU (class-default access); the harness reaches
 * them without editing the reference. */
#define class struct
#define private public
#define protected public
#include "src/sim/Simulation.h"
#include "src/sim/es/lifetime.h"
#undef private
#undef protected
#undef class

#include <cstdint>
#include <cstring>
#include <vector>

namespace {

struct RefSim {
    Grid* grid = nullptr;
    SimulationCPU* sim = nullptr;
    Settings settings{};
};

GridInformation info_of(const Grid& g, double region_size, double region_extends)
{
    /* Same construction as src/SimulationRunner.cpp:72-77 and
     * tests/sim/SigmaIntegrationTest.h:32-37. */
    GridInformation gi;
    gi.cell_size = g.GetSettings().cell_size;
    gi.indexed_impurity_count = g.GetTotalImpurityCount();
    gi.index_size = (int)g.GetIndex().size();
    gi.region_size = region_size;
    gi.region_extends = region_extends;
    return gi;
}

}  // namespace

extern "C" {

/* Grid(seed, region_size, region_extends, density, radius, target_cell_population). */
void* ref_grid_new_seed(unsigned int seed, double region_size, double region_extends, double density,
                        double impurity_radius, int target_cell_population)
{
    return new Grid(seed, region_size, region_extends, density, impurity_radius, target_cell_population);
}

/* Grid(vector<v2>, region_size, region_extends, radius, target_cell_population). */
void* ref_grid_new_list(const double* xy, int n, double region_size, double region_extends,
                        double impurity_radius, int target_cell_population)
{
    std::vector<v2> imps((size_t)n);
    for (int i = 0; i < n; i++) imps[i] = v2(xy[2 * i], xy[2 * i + 1]);
    return new Grid(imps, region_size, region_extends, impurity_radius, target_cell_population);
}

void ref_grid_free(void* g) { delete (Grid*)g; }

/* Sizes: cells_per_row, total indexed impurities, unique impurities, and the
 * ImpuritySettings fields (start, size, cell_size, radius). */
void ref_grid_info(void* gp, int* cells_per_row, int* total_indexed, int* unique_count, double* spawn_start,
                   double* spawn_size, double* cell_size, double* radius)
{
    Grid* g = (Grid*)gp;
    ImpuritySettings is = g->GetSettings();
    *cells_per_row = g->GetCellsPerRow();
    *total_indexed = g->GetTotalImpurityCount();
    *unique_count = g->GetUniqueImpurityCount();
    *spawn_start = is.spawn_region_start;
    *spawn_size = is.spawn_region_size;
    *cell_size = is.cell_size;
    *radius = is.impurity_radius;
}

/* Copies ordered impurities (x,y interleaved) and the cumulative cell index. */
void ref_grid_copy(void* gp, double* xy, int* cell_end)
{
    Grid* g = (Grid*)gp;
    const auto& imps = g->GetImpurities();
    const auto& idx = g->GetIndex();
    for (size_t i = 0; i < imps.size(); i++) {
        xy[2 * i] = imps[i].x;
        xy[2 * i + 1] = imps[i].y;
    }
    std::memcpy(cell_end, idx.data(), sizeof(int) * idx.size());
}

/* A SimulationCPU bound to a grid, as src/SimulationRunner.cpp:79-84 builds it. */
void* ref_sim_new(void* gp, int positions_per_row, int phi_steps, double tau, double alpha, int is_clockwise,
                  double particle_speed, double region_size, double region_extends)
{
    RefSim* rs = new RefSim();
    rs->grid = (Grid*)gp;
    rs->settings.tau = tau;
    rs->settings.alpha = alpha;
    rs->settings.is_clockwise = is_clockwise != 0;
    rs->settings.particle_speed = particle_speed;
    rs->settings.region_size = region_size;
    rs->settings.region_extends = region_extends;
    rs->settings.impurity_density = 0;
    rs->settings.impurity_radius = rs->grid->GetSettings().impurity_radius;
    rs->settings.target_cell_population = 0;
    rs->sim = new SimulationCPU(positions_per_row, phi_steps, info_of(*rs->grid, region_size, region_extends));
    return rs;
}

void ref_sim_free(void* p)
{
    RefSim* rs = (RefSim*)p;
    delete rs->sim;
    delete rs;
}

void ref_sim_init_sample(void* p, int coherent)
{
    RefSim* rs = (RefSim*)p;
    rs->sim->InitSample(*rs->grid, rs->settings, coherent != 0);
}

static void copy_metrics(const ParticleMetrics& pm, int* out7)
{
    if (!out7) return;
    out7[0] = pm.cells_passed;
    out7[1] = pm.impurities_tested;
    out7[2] = pm.particles_inside_impurity;
    out7[3] = pm.particles_escaped;
    out7[4] = pm.particles_at_bound;
    out7[5] = pm.max_impurities_tested;
    out7[6] = pm.max_cells_passed;
}

/* SimulationCPU::ComputeLifetimes: raw per-orbit lifetimes in [j][i][q][p] order. */
int ref_sim_lifetimes(void* p, double magnetic_field, double* out, int* metrics7)
{
    RefSim* rs = (RefSim*)p;
    Metrics m;
    std::vector<double> lt = rs->sim->ComputeLifetimes(magnetic_field, *rs->grid, m);
    std::memcpy(out, lt.data(), sizeof(double) * lt.size());
    copy_metrics(m.particle_metrics, metrics7);
    return (int)lt.size();
}

/* The body of SimulationCPU::ComputeLifetimes (src/sim/SimulationCPU.cpp:105-135)
 * restricted to start-position rows [j0, j1): used to time a bounded sample of a
 * large sector pass on the CPU, and to split a pass over many processes. Writes
 * (j1-j0)*dim*4*ppq lifetimes and the rows' counters, the per-orbit maxima
 * included. */
long long ref_sim_lifetimes_rows(void* p, double magnetic_field, int j0, int j1, double* out, int* metrics7)
{
    RefSim* rs = (RefSim*)p;
    SimulationCPU& s = *rs->sim;
    s.ps.angular_speed = E * magnetic_field / M;
    s.ss.signed_angular_speed = s.ps.is_clockwise ? -s.ps.angular_speed : s.ps.angular_speed;
    ParticleMetrics pm;
    long long k = 0;
    for (int j = j0; j < j1; j++) {
        for (int i = 0; i < s.ss.positions_per_row; i++) {
            const v2 position = v2(i, j) * s.ss.distance_between_positions + s.ss.small_offset;
            for (int q = 0; q < 4; q++) {
                for (int pp = 0; pp < s.ss.particles_per_quadrant; pp++) {
                    auto particle = CreateParticle(q, pp, position, &s.ps);
                    const int last_cells = pm.cells_passed, last_tested = pm.impurities_tested;
                    double lt = TraceOrbit(&particle, &s.is, rs->grid->GetImpurities(), rs->grid->GetIndex(), pm);
                    if (out) out[k] = lt;
                    k++;
                    /* the per-orbit maxima, as src/sim/SimulationCPU.cpp:123-131 keeps them */
                    if (pm.max_cells_passed < pm.cells_passed - last_cells)
                        pm.max_cells_passed = pm.cells_passed - last_cells;
                    if (pm.max_impurities_tested < pm.impurities_tested - last_tested)
                        pm.max_impurities_tested = pm.impurities_tested - last_tested;
                }
            }
        }
    }
    copy_metrics(pm, metrics7);
    return k;
}

/* SimulationCPU::ComputeSigmas: out = [xx0, xy0, xx1, xy1, ...] per temperature. */
int ref_sim_sigmas(void* p, double magnetic_field, const double* temperatures, int n_t, double* out, int* metrics7)
{
    RefSim* rs = (RefSim*)p;
    std::vector<double> ts(temperatures, temperatures + n_t);
    SampleMetrics sm(0, false, 0);
    std::vector<Sigma> r = rs->sim->ComputeSigmas(magnetic_field, ts, *rs->grid, sm);
    for (int t = 0; t < n_t; t++) {
        out[2 * t] = r[t].xx;
        out[2 * t + 1] = r[t].xy;
    }
    if (!sm.iteration_metrics.empty()) copy_metrics(sm.iteration_metrics[0].particle_metrics, metrics7);
    return n_t;
}

/* SimulationCPU::ComputeSigmasWithImages: sigmas plus per-position maps
 * (lifetime, xx, xy), each dim*dim per temperature, temperature-major. */
int ref_sim_sigmas_images(void* p, double magnetic_field, const double* temperatures, int n_t, double* out,
                          double* lt_pos, double* xx_pos, double* xy_pos)
{
    RefSim* rs = (RefSim*)p;
    std::vector<double> ts(temperatures, temperatures + n_t);
    SampleMetrics sm(0, false, 0);
    std::vector<IterationResult> r = rs->sim->ComputeSigmasWithImages(magnetic_field, ts, *rs->grid, sm);
    const size_t np = (size_t)rs->sim->ss.total_positions;
    for (int t = 0; t < n_t; t++) {
        out[2 * t] = r[t].result.xx;
        out[2 * t + 1] = r[t].result.xy;
        std::memcpy(lt_pos + t * np, r[t].particle_lifetimes.data(), sizeof(double) * np);
        std::memcpy(xx_pos + t * np, r[t].sigmas.xx_buffer.data(), sizeof(double) * np);
        std::memcpy(xy_pos + t * np, r[t].sigmas.xy_buffer.data(), sizeof(double) * np);
    }
    return n_t;
}

/* SimulationCPU::DeriveTemperature on caller-provided raw lifetimes. */
void ref_sim_derive(void* p, double magnetic_field, double temperature, const double* raw, double* out2)
{
    RefSim* rs = (RefSim*)p;
    SimulationCPU& s = *rs->sim;
    s.ps.angular_speed = E * magnetic_field / M;
    s.ss.signed_angular_speed = s.ps.is_clockwise ? -s.ps.angular_speed : s.ps.angular_speed;
    std::vector<double> lt(raw, raw + s.ss.total_particles);
    Sigma r = s.DeriveTemperature(temperature, lt);
    out2[0] = r.xx;
    out2[1] = r.xy;
}

}  // extern "C"
