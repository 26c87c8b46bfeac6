// config.h - the reference's .config file, parsed with its rules.
//
// Same keys, defaults and validation as SimulationConfiguration::ParseFromeFile
// (src/SimulationConfiguration.h:79-228). Errors are reported (ConfigError)
// instead of the reference's print-and-exit; the CLI turns them into a
// non-zero exit code.
//
// Keys this runtime adds (ignored by the reference): `precision
// fp64|split|split_exact` (default fp64: the reference's arithmetic;
// split_exact: the split walk with FP64 integration, the same sigma as fp64),
// `batched 0|1` (1: every sample,
// field and sector in one batched run), `device_ordinal n`, `journal <path>`
// (the per-pass results journal that lets a stopped sweep resume; journal.h).
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "es_cuda.h"

namespace es_host {

struct ConfigError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

enum class OutputType { Nothing, Results, All };

struct RunConfig {
    int num_samples = 0;
    int positions_per_row = 0;       // `dimension`
    int particles_per_quadrant = 0;  // `phi_steps`
    bool print_info = false;
    OutputType output_type = OutputType::All;
    std::string device = "";         // `device` as written (the reference selects OpenCL with "gpu")
    es_settings settings{};
    std::vector<double> magnetic_fields;
    std::vector<double> temperatures;
    std::vector<unsigned int> sample_seeds;
    std::string config_path;
    std::string base_output_directory;
    std::string output_directory;
    int digits_in_sample_num = 0;
    // additions
    int precision = ES_PRECISION_FP64;
    bool batched = false;
    int device_ordinal = 0;
    std::string journal_path;  // empty: no journal
};

// Key/value lines as the reference reads them: empty lines and lines starting
// with '#' or ":/" are skipped, the key runs to the first space, and the first
// occurrence of a key wins.
std::unordered_map<std::string, std::string> ReadConfigValues(const std::string& text);

RunConfig ParseConfigFile(const std::string& file_path);
RunConfig ParseConfigText(const std::string& text, const std::string& file_path);
// The parsed values as a JSON object.
std::string DescribeConfig(const RunConfig& cfg);

}  // namespace es_host
