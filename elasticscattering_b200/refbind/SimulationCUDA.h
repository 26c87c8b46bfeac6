/* SimulationCUDA.h - the reference-side binding of the B200 backend.
 *
 * A third backend beside the reference's SimulationCPU and SimulationCL: a
 * subclass of the reference's own `class Simulation` (src/sim/Simulation.h:56-147)
 * that forwards to the C ABI of include/es_cuda.h (libes_cuda.so). A maintainer
 * adds this header to the reference tree and picks it in
 * SimulationRunner::RunSimulation (src/SimulationRunner.cpp:82-84):
 *
 *     if (cfg.use_gpu) es = new SimulationCUDA(cfg.positions_per_row, cfg.particles_per_quadrant, gi);
 *
 * It compiles against the reference's headers unchanged (this repository
 * builds it that way into oracle/_ref/libes_refbind.so and drives it through a
 * `Simulation*` in a GPU test).
 *
 * Simulation::InitSample is not virtual in the reference: the base class keeps
 * the sector in its protected settings (ss, ps, is), and this class hands that
 * sector and the grid to the device on the next ComputeSigmas call when either
 * changed. Errors print and exit(0) as the reference's ErrorMacros do
 * (src/utils/ErrorMacros.h:22-38).
 */
#pragma once

#include "src/sim/Simulation.h"

#include "es_cuda.h"

#include <cstdint>
#include <cstdlib>
#include <iostream>
#include <vector>

class SimulationCUDA : public Simulation {
    es_ctx* ctx = nullptr;

    // what the device holds: the grid (its identity) and the sector
    struct GridKey {
        const void* data = nullptr;
        size_t n = 0;
        unsigned int seed = 0;
        int cells_per_row = 0;
        double first_x = 0, last_y = 0;
        bool operator==(const GridKey& o) const
        {
            return data == o.data && n == o.n && seed == o.seed && cells_per_row == o.cells_per_row &&
                   first_x == o.first_x && last_y == o.last_y;
        }
    } grid_key;
    uint64_t generation = 0;
    bool has_sector = false;
    es_settings sector{};
    int sector_coherent = -1;

    static void Check(const es_ctx* c, es_status st)
    {
        if (st != ES_OK) {
            std::cout << "CUDA error: " << es_last_error(c) << std::endl;
            exit(0);
        }
    }

    // The grid and sector the base class's InitSample recorded, on the device.
    void Sync(const Grid& grid)
    {
        const std::vector<v2>& imps = grid.GetImpurities();
        GridKey k;
        k.data = imps.data();
        k.n = imps.size();
        k.seed = grid.GetSeed();
        k.cells_per_row = grid.GetCellsPerRow();
        k.first_x = imps.empty() ? 0.0 : imps.front().x;
        k.last_y = imps.empty() ? 0.0 : imps.back().y;
        if (generation == 0 || !(k == grid_key)) {
            const ImpuritySettings g = grid.GetSettings();
            es_impurity_settings s{g.spawn_region_start, g.spawn_region_size, g.cell_size, g.cells_per_row,
                                   g.impurity_radius};
            // v2 is two doubles (src/sim/es/v2.h), the ABI's x,y pairs
            Check(ctx, es_upload_grid(ctx, imps.empty() ? nullptr : &imps[0].x, (int64_t)imps.size(),
                                      grid.GetIndex().data(), &s, ++generation));
            grid_key = k;
            has_sector = false;  // es_init_sample follows every upload
        }
        es_settings st{};
        st.tau = ss.coherent_tau;
        st.alpha = ps.alpha;
        st.is_clockwise = ps.is_clockwise ? 1 : 0;
        st.particle_speed = ps.particle_speed;
        st.region_size = ss.region_size;
        st.region_extends = ss.region_extended_area;
        st.impurity_radius = is.impurity_radius;
        const int coherent = ps.is_coherent ? 1 : 0;
        if (!has_sector || coherent != sector_coherent || st.tau != sector.tau || st.alpha != sector.alpha ||
            st.is_clockwise != sector.is_clockwise || st.particle_speed != sector.particle_speed) {
            Check(ctx, es_init_sample(ctx, &st, coherent));
            sector = st;
            sector_coherent = coherent;
            has_sector = true;
        }
    }

    Metrics ToMetrics(const es_metrics& m) const
    {
        Metrics metrics;
        metrics.particle_metrics.cells_passed = (int)m.cells_passed;
        metrics.particle_metrics.impurities_tested = (int)m.impurities_tested;
        metrics.particle_metrics.particles_inside_impurity = (int)m.particles_inside_impurity;
        metrics.particle_metrics.particles_escaped = (int)m.particles_escaped;
        metrics.particle_metrics.particles_at_bound = (int)m.particles_at_bound;
        metrics.particle_metrics.max_impurities_tested = (int)m.max_impurities_tested;
        metrics.particle_metrics.max_cells_passed = (int)m.max_cells_passed;
        metrics.real_particles = ss.total_particles - metrics.particle_metrics.particles_inside_impurity;
        return metrics;
    }

public:
    SimulationCUDA(int p_positions_per_row, int p_particles_per_quadrant, const GridInformation& grid_info,
                   int device_ordinal = 0, int precision = ES_PRECISION_FP64)
        : Simulation(p_positions_per_row, p_particles_per_quadrant, grid_info)
    {
        es_sim_desc d{p_positions_per_row, p_particles_per_quadrant, grid_info.region_size, grid_info.region_extends,
                      grid_info.cell_size, device_ordinal, precision};
        Check(nullptr, es_create(&d, &ctx));
    }

    ~SimulationCUDA() { es_destroy(ctx); }

    virtual std::vector<Sigma> ComputeSigmas(const double magnetic_field, const std::vector<double>& temperatures,
                                             const Grid& grid, SampleMetrics& sample_metrics) override
    {
        Sync(grid);
        es_metrics m{};
        QueryPerformanceCounter(&pc.lifetimeBegin);
        Check(ctx, es_compute_lifetimes(ctx, magnetic_field, nullptr, &m));
        QueryPerformanceCounter(&pc.lifetimeEnd);
        Metrics metrics = ToMetrics(m);
        metrics.time_elapsed_lifetimes = GetElapsedTime(pc.lifetimeBegin, pc.lifetimeEnd);
        Check(ctx, es_average_lifetime(ctx, &metrics.avg_particle_lifetime));

        QueryPerformanceCounter(&pc.temperaturesBegin);
        std::vector<double> out(2 * temperatures.size());
        if (!temperatures.empty())
            Check(ctx, es_derive_temperatures(ctx, temperatures.data(), (int32_t)temperatures.size(), out.data()));
        QueryPerformanceCounter(&pc.temperaturesEnd);
        metrics.time_elapsed_temperatures = GetElapsedTime(pc.temperaturesBegin, pc.temperaturesEnd);
        sample_metrics.iteration_metrics.push_back(metrics);

        std::vector<Sigma> results(temperatures.size());
        for (size_t t = 0; t < temperatures.size(); t++) results[t] = Sigma(out[2 * t], out[2 * t + 1]);
        return results;
    }

    virtual std::vector<IterationResult> ComputeSigmasWithImages(const double magnetic_field,
                                                                 const std::vector<double>& temperatures,
                                                                 const Grid& grid,
                                                                 SampleMetrics& sample_metrics) override
    {
        Sync(grid);
        const size_t nt = temperatures.size(), np = (size_t)ss.total_positions;
        std::vector<double> out(2 * nt), lt(nt * np), xx(nt * np), xy(nt * np);
        es_metrics m{};
        QueryPerformanceCounter(&pc.lifetimeBegin);
        Check(ctx, es_compute_sigmas_images(ctx, magnetic_field, temperatures.data(), (int32_t)nt, out.data(),
                                            lt.data(), xx.data(), xy.data(), &m));
        QueryPerformanceCounter(&pc.lifetimeEnd);
        Metrics metrics = ToMetrics(m);
        // lifetimes and temperatures run in one call on the device
        metrics.time_elapsed_lifetimes = GetElapsedTime(pc.lifetimeBegin, pc.lifetimeEnd);
        Check(ctx, es_average_lifetime(ctx, &metrics.avg_particle_lifetime));
        sample_metrics.iteration_metrics.push_back(metrics);

        std::vector<IterationResult> results(nt);
        for (size_t t = 0; t < nt; t++) {
            results[t].particle_lifetimes.assign(lt.begin() + t * np, lt.begin() + (t + 1) * np);
            results[t].sigmas.xx_buffer.assign(xx.begin() + t * np, xx.begin() + (t + 1) * np);
            results[t].sigmas.xy_buffer.assign(xy.begin() + t * np, xy.begin() + (t + 1) * np);
            results[t].result = Sigma(out[2 * t], out[2 * t + 1]);
        }
        return results;
    }
};
