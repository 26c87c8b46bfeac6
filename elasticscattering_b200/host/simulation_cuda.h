// simulation_cuda.h - the B200 backend behind the reference's Simulation interface.
//
// class Simulation (src/sim/Simulation.h:56-147) with its result and metrics
// types (src/SimulationResult.h, src/Metrics.h), forwarding to the C ABI of
// include/es_cuda.h. Failures of the ABI throw SimulationError with the
// library's message (the reference prints and exits, src/utils/ErrorMacros.h).
#pragma once

#include <stdexcept>
#include <string>
#include <vector>

#include "es_cuda.h"
#include "grid.h"

namespace es_host {

struct SimulationError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// src/SimulationResult.h:24-52
struct Sigma {
    double xx = 0, xy = 0;
    Sigma() = default;
    Sigma(double a, double b) : xx(a), xy(b) {}
    Sigma operator+(const Sigma& a) const { return Sigma(a.xx + xx, a.xy + xy); }
    Sigma& operator+=(const Sigma& a)
    {
        xx += a.xx;
        xy += a.xy;
        return *this;
    }
};

// src/SimulationResult.h:54-74: results[field][temperature]
struct SampleResult {
    std::vector<std::vector<Sigma>> results;
    SampleResult() = default;
    SampleResult(int T, int N) : results((size_t)N, std::vector<Sigma>((size_t)T)) {}
};

// src/SimulationResult.h:76-87
struct IterationResult {
    std::vector<double> particle_lifetimes, xx_buffer, xy_buffer;
    Sigma result;
};

// src/SimulationResult.h:89-114
struct DataRow {
    double temperature = 0, magnetic_field = 0;
    Sigma incoherent, coherent;
    double xxd = 0;
};

// src/Metrics.h:24-42 (ParticleMetrics widened to 64 bits)
struct Metrics {
    es_metrics particle_metrics{};
    int64_t real_particles = 0;
    double time_elapsed_lifetimes = 0;
    double time_elapsed_temperatures = 0;
    double avg_particle_lifetime = 0;
};

// src/Metrics.h:44-51
struct GlobalMetrics {
    int particles_per_row = 0;
    int phi_steps = 0;
    int64_t unique_impurity_count = 0;
    int cells_per_row = 0;
    double grid_creation_time = 0;
};

// src/Metrics.h:53-80
struct SampleMetrics {
    int sample_index = 0;
    int64_t total_particles = 0;
    int64_t total_cells = 0;
    int64_t impurity_count = 0;
    unsigned int seed = 0;
    int64_t total_indexed_impurities = 0;
    bool coherent = false;
    std::vector<Metrics> iteration_metrics;
    SampleMetrics(int index, bool coh, int64_t nlt) : sample_index(index), total_particles(nlt), coherent(coh) {}
};

// GridInformation, src/sim/es/settings.h:65-73
struct GridInformation {
    double region_size = 0, region_extends = 0, cell_size = 0;
    int64_t indexed_impurity_count = 0, index_size = 0;
};

class SimulationCUDA {
public:
    SimulationCUDA(int positions_per_row, int phi_steps, const GridInformation& gi, int device = 0,
                   int precision = ES_PRECISION_FP64);
    ~SimulationCUDA();
    SimulationCUDA(const SimulationCUDA&) = delete;
    SimulationCUDA& operator=(const SimulationCUDA&) = delete;

    // Simulation::InitSample, src/sim/Simulation.h:111-126
    void InitSample(const Grid& grid, const es_settings& settings, bool coherent);
    // Simulation::ComputeSigmas / ComputeSigmasWithImages, src/sim/Simulation.h:128-129
    std::vector<Sigma> ComputeSigmas(double magnetic_field, const std::vector<double>& temperatures, const Grid& grid,
                                     SampleMetrics& sample_metrics);
    std::vector<IterationResult> ComputeSigmasWithImages(double magnetic_field, const std::vector<double>& temperatures,
                                                         const Grid& grid, SampleMetrics& sample_metrics);

    es_ctx* context() { return ctx_; }

private:
    void check(es_status st) const;
    Metrics LifetimeMetrics(const es_metrics& m, double seconds);

    es_ctx* ctx_ = nullptr;
    int positions_per_row_ = 0, phi_steps_ = 0;
    int64_t total_particles_ = 0;
    bool want_average_ = true;
};

}  // namespace es_host
