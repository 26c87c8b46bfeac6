/* C-callable harness around the reference-side binding SimulationCUDA.
 *
 * TEST INFRASTRUCTURE ONLY. Compiled by oracle/Makefile with the reference's
 * unmodified sources (src/sim/Grid.cpp, src/sim/SimulationCPU.cpp and the
 * headers they include, read in place) and elasticscattering_b200/refbind/
 * SimulationCUDA.h, linked against libes_cuda.so, into
 * oracle/_ref/libes_refbind.so. It runs the reference's own sweep loop --
 * RunSimulation / RunSample (src/SimulationRunner.cpp:54-151): one Simulation
 * object for all samples, the grid rebuilt per sample, InitSample per sector,
 * ComputeSigmas (or ComputeSigmasWithImages) per field -- through a
 * `Simulation*` that is either the reference's SimulationCPU or the binding's
 * SimulationCUDA, so a test can compare the two backends behind the
 * reference's own interface.
 */
#include "src/sim/Simulation.h"

#include "SimulationCUDA.h"

#include <cstring>
#include <vector>

extern "C" {

/* out: [sample][sector: coherent, incoherent][field][temperature][xx, xy];
 * metrics: [sample][sector][field][7] (the ParticleMetrics counters, in
 * src/sim/es/particle_metrics.h order); avg_lt: [sample][sector][field].
 * images != 0 runs ComputeSigmasWithImages and also fills maps
 * [sample][sector][field][temperature][3][dim*dim] (lifetime, xx, xy) if maps is
 * not NULL. Returns 0, or -1 for an unknown backend. */
int rb_sweep(int backend, const unsigned* seeds, int n_samples, double region_size, double region_extends,
             double density, double impurity_radius, int target_cell_population, int positions_per_row,
             int phi_steps, double tau, double alpha, int is_clockwise, double particle_speed, const double* fields,
             int n_fields, const double* temperatures, int n_t, int images, double* out, int* metrics,
             double* avg_lt, double* maps)
{
    if (backend != 0 && backend != 1) return -1;
    Settings s;
    s.tau = tau;
    s.alpha = alpha;
    s.is_clockwise = is_clockwise != 0;
    s.particle_speed = particle_speed;
    s.region_size = region_size;
    s.region_extends = region_extends;
    s.impurity_density = density;
    s.impurity_radius = impurity_radius;
    s.target_cell_population = target_cell_population;
    const std::vector<double> temps(temperatures, temperatures + n_t);

    /* src/SimulationRunner.cpp:60,72-84 */
    auto grid = Grid(seeds[0], region_size, region_extends, density, impurity_radius, target_cell_population);
    GridInformation gi;
    gi.cell_size = grid.GetSettings().cell_size;
    gi.indexed_impurity_count = grid.GetTotalImpurityCount();
    gi.index_size = grid.GetIndex().size();
    gi.region_size = region_size;
    gi.region_extends = region_extends;
    Simulation* es;
    if (backend == 1) es = new SimulationCUDA(positions_per_row, phi_steps, gi);
    else es = new SimulationCPU(positions_per_row, phi_steps, gi);

    const size_t np = (size_t)positions_per_row * positions_per_row;
    for (int i = 0; i < n_samples; i++) {
        for (int sector = 0; sector < 2; sector++) {
            const bool coherent = sector == 0;
            es->InitSample(grid, s, coherent); /* src/SimulationRunner.cpp:112 */
            SampleMetrics sm(i, coherent, 0);
            for (int f = 0; f < n_fields; f++) {
                const size_t base = ((size_t)i * 2 + sector) * n_fields + f;
                if (!images) {
                    const std::vector<Sigma> r = es->ComputeSigmas(fields[f], temps, grid, sm);
                    for (int t = 0; t < n_t; t++) {
                        out[(base * n_t + t) * 2] = r[t].xx;
                        out[(base * n_t + t) * 2 + 1] = r[t].xy;
                    }
                } else {
                    const std::vector<IterationResult> r = es->ComputeSigmasWithImages(fields[f], temps, grid, sm);
                    for (int t = 0; t < n_t; t++) {
                        out[(base * n_t + t) * 2] = r[t].result.xx;
                        out[(base * n_t + t) * 2 + 1] = r[t].result.xy;
                        if (maps) {
                            double* m = maps + ((base * n_t + t) * 3) * np;
                            std::memcpy(m, r[t].particle_lifetimes.data(), sizeof(double) * np);
                            std::memcpy(m + np, r[t].sigmas.xx_buffer.data(), sizeof(double) * np);
                            std::memcpy(m + 2 * np, r[t].sigmas.xy_buffer.data(), sizeof(double) * np);
                        }
                    }
                }
                const Metrics& mt = sm.iteration_metrics.back();
                const ParticleMetrics& pm = mt.particle_metrics;
                int* mo = metrics + base * 7;
                mo[0] = pm.cells_passed;
                mo[1] = pm.impurities_tested;
                mo[2] = pm.particles_inside_impurity;
                mo[3] = pm.particles_escaped;
                mo[4] = pm.particles_at_bound;
                mo[5] = pm.max_impurities_tested;
                mo[6] = pm.max_cells_passed;
                avg_lt[base] = mt.avg_particle_lifetime;
            }
        }
        /* src/SimulationRunner.cpp:96-97 */
        if (i < n_samples - 1)
            grid = Grid(seeds[i + 1], region_size, region_extends, density, impurity_radius, target_cell_population);
    }
    delete es;
    return 0;
}

}  // extern "C"
