// runner.h - SimulationRunner (src/SimulationRunner.h:24-57): a .config sweep over
// samples, magnetic fields and temperatures, with the reference's results folder.
#pragma once

#include <memory>
#include <ostream>
#include <string>
#include <vector>

#include "config.h"
#include "journal.h"
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
    // Passes of the last Run taken from the journal / computed.
    int64_t resumed_passes() const { return resumed_; }
    int64_t computed_passes() const { return computed_; }

private:
    SimulationResult RunSimulation();
    SimulationResult RunBatched();
    SampleResult RunSample(std::unique_ptr<SimulationCUDA>& es, const GridInformation& gi, int sample_index,
                           bool coherent, const Grid& grid);
    void Record(int sample_index, bool coherent, double field, const std::vector<Sigma>& sigma, const Metrics& m);
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
    std::unique_ptr<Journal> journal_;
    int64_t resumed_ = 0, computed_ = 0;
};

}  // namespace es_host
