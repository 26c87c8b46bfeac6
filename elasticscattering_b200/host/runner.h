// runner.h - SimulationRunner (src/SimulationRunner.h:24-57): a .config sweep over
// samples, magnetic fields and temperatures, with the reference's results folder.
#pragma once

#include <ostream>
#include <string>
#include <vector>

#include "config.h"
#include "simulation_cuda.h"

namespace es_host {

struct SimulationResult {
    std::vector<SampleResult> coherent, incoherent;
};

class SimulationRunner {
public:
    explicit SimulationRunner(std::ostream& log) : log_(log) {}
    // Run(InitParameters) of src/SimulationRunner.cpp:31-50; returns the results
    // (per sample and sector) after writing the files the config asks for.
    SimulationResult Run(const std::string& config_path);
    SimulationResult Run(const RunConfig& cfg);
    const RunConfig& config() const { return cfg_; }

private:
    SimulationResult RunSimulation();
    SimulationResult RunBatched();
    SampleResult RunSample(SimulationCUDA& es, int sample_index, bool coherent, const Grid& grid);
    void FinishResults(const SimulationResult& sr) const;
    void CreateOutputDirectory() const;
    void CreateSampleOutputDirectory(int sample_index) const;

    std::string ResultPath(int t) const { return cfg_.output_directory + "/T" + std::to_string(t) + ".dat"; }
    std::string SamplePath(int s) const { return cfg_.output_directory + "/Sample " + std::to_string(s); }
    std::string SampleResultsPath(int s) const { return SamplePath(s) + "/sample_results.dat"; }
    std::string ImagePath(int t, int m, int s, bool coherent) const
    {
        return SamplePath(s) + (coherent ? "/Coherent/" : "/Incoherent/") + "T" + std::to_string(t) + " MF" +
               std::to_string(m) + ".png";
    }
    std::string MetricsPath() const { return cfg_.output_directory + "/Metrics.txt"; }

    RunConfig cfg_;
    std::ostream& log_;
};

}  // namespace es_host
