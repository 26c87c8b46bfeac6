// logger.h - the results folder's files in the reference's formats (src/Logger.cpp):
// T<j>.dat per temperature, Sample <i>/sample_results.dat, Metrics.txt and the
// per-position PNG maps, so that the reference's plotting scripts read them
// unchanged.
#pragma once

#include <string>
#include <vector>

#include "config.h"
#include "simulation_cuda.h"

namespace es_host {

struct Logger {
    static constexpr int result_precision = 6;
    static constexpr int rw = result_precision + 10;

    static void CreateResultLog(const std::string& path, const RunConfig& cfg, double temperature);
    static void LogResult(const std::string& path, const DataRow& row);
    static void CreateSampleResultLog(const std::string& path);
    static void LogSampleResults(const std::string& path, const SampleResult& coherent, const SampleResult& incoherent);
    static void CreateSampleMetricsLog(const std::string& path, const GlobalMetrics& gm);
    static void LogSampleMetrics(const std::string& path, const SampleMetrics& sm);
    static void LogImages(const std::string& path, int dim, const IterationResult& it);
};

// RGB8 PNG (stored, uncompressed deflate); returns false on I/O failure.
bool WritePng(const std::string& path, int width, int height, const std::vector<unsigned char>& rgb);

}  // namespace es_host
