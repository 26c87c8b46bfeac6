// config.cpp - .config parsing with the reference's rules
// (SimulationConfiguration::ParseFromeFile, src/SimulationConfiguration.h:79-228).
#include "config.h"

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <random>
#include <sstream>

namespace es_host {

std::unordered_map<std::string, std::string> ReadConfigValues(const std::string& text)
{
    std::unordered_map<std::string, std::string> values;
    std::istringstream in(text);
    std::string raw;
    while (std::getline(in, raw)) {
        // the reference re-reads each line through a stringstream, which only
        // drops what follows an embedded '\n'; a trailing '\r' stays
        std::istringstream is_line(raw);
        std::string line;
        if (!std::getline(is_line, line)) continue;
        if (line.empty() || line[0] == '\n' || line[0] == '#' || (line.size() > 1 && line[0] == ':' && line[1] == '/'))
            continue;
        const size_t pos = line.find(' ');
        const std::string key = line.substr(0, pos);
        // substr(npos + 1) wraps to substr(0): a line without a space maps to itself
        const std::string value = line.substr(pos + 1);
        values.emplace(key, value);  // the first occurrence wins
    }
    return values;
}

namespace {

const std::string& need(const std::unordered_map<std::string, std::string>& v, const char* key)
{
    auto it = v.find(key);
    if (it == v.end()) throw ConfigError(std::string("missing config key '") + key + "'");
    return it->second;
}

bool has(const std::unordered_map<std::string, std::string>& v, const char* key) { return v.find(key) != v.end(); }

}  // namespace

RunConfig ParseConfigText(const std::string& text, const std::string& file_path)
{
    const auto values = ReadConfigValues(text);
    RunConfig cfg;
    cfg.config_path = file_path;

    cfg.output_type = OutputType::All;
    if (has(values, "output_type")) {
        const auto& v = values.at("output_type");
        if (v == "nothing") cfg.output_type = OutputType::Nothing;
        else if (v == "results") cfg.output_type = OutputType::Results;
    }
    if (cfg.output_type == OutputType::Nothing) {
        cfg.base_output_directory = "";
        cfg.output_directory = "";
    } else {
        cfg.base_output_directory = has(values, "output_directory") ? values.at("output_directory") : "ESLogs";
        const std::string base = cfg.base_output_directory + "/Result_";
        for (unsigned n = 0;; n++) {
            const std::string dir = base + std::to_string(n);
            if (!std::filesystem::exists(dir)) {
                cfg.output_directory = dir;
                break;
            }
        }
    }

    cfg.device = has(values, "device") ? values.at("device") : "";
    cfg.print_info = has(values, "print_info") && std::atoi(values.at("print_info").c_str()) == 1;

    cfg.num_samples = std::atoi(need(values, "num_samples").c_str());
    if (cfg.num_samples <= 0) throw ConfigError("Samples must be greater than 0.");
    cfg.particles_per_quadrant = std::atoi(need(values, "phi_steps").c_str());
    if (cfg.particles_per_quadrant % 2 == 0) throw ConfigError("Phi steps must be odd.");
    cfg.positions_per_row = std::atoi(need(values, "dimension").c_str());
    if (cfg.positions_per_row % 2 == 0) throw ConfigError("Dimension must be odd.");

    if (has(values, "magnetic_field")) {
        cfg.magnetic_fields.push_back(std::atof(values.at("magnetic_field").c_str()));
    } else {
        const double mf_min = std::atof(need(values, "magnetic_field_min").c_str());
        const double mf_max = std::atof(need(values, "magnetic_field_max").c_str());
        const double mf_n = std::atoi(need(values, "magnetic_field_n").c_str());
        if (mf_n < 2)
            throw ConfigError(
                "Tried to declare magnetic field range with n<2. Use 'magnetic_field x' when using only one value.");
        const int n = (int)mf_n;
        const double step = (mf_max - mf_min) / (double)(mf_n - 1);
        cfg.magnetic_fields.resize((size_t)n);
        for (int i = 0; i < n; i++) cfg.magnetic_fields[(size_t)i] = mf_min + i * step;
    }

    {
        std::stringstream ss(need(values, "temperatures"));
        while (ss.good()) {
            std::string a;
            std::getline(ss, a, ' ');
            const double t = std::atof(a.c_str());
            if (t > 0) cfg.temperatures.push_back(t);  // the reference drops T <= 0
        }
    }

    cfg.settings.particle_speed = std::atof(need(values, "particle_speed").c_str());
    cfg.settings.tau = std::atof(need(values, "tau").c_str());
    cfg.settings.alpha = std::atof(need(values, "alpha").c_str());
    cfg.settings.is_clockwise = std::atoi(need(values, "clockwise").c_str()) > 0 ? 1 : 0;

    unsigned int seed;
    if (has(values, "start_seed")) {
        seed = (unsigned int)std::atoi(values.at("start_seed").c_str());
    } else {
        std::random_device rd;
        seed = rd();
    }
    cfg.sample_seeds.resize((size_t)cfg.num_samples);
    for (int i = 0; i < cfg.num_samples; i++) cfg.sample_seeds[(size_t)i] = (seed + 100) * (unsigned)(i + 1);

    cfg.settings.region_size = std::atof(need(values, "region_size").c_str());
    cfg.settings.region_extends = std::atof(need(values, "region_extends").c_str());
    cfg.settings.impurity_density = std::atof(need(values, "impurity_density").c_str());
    cfg.settings.impurity_radius = std::atof(need(values, "impurity_radius").c_str());
    cfg.settings.target_cell_population =
        has(values, "target_cell_population") ? std::atoi(values.at("target_cell_population").c_str()) : 15;

    int x = cfg.num_samples;
    cfg.digits_in_sample_num = 0;
    while (x > 0) {
        x = (int)std::floor(x / 10);
        cfg.digits_in_sample_num++;
    }

    if (has(values, "precision")) {
        const auto& p = values.at("precision");
        if (p == "split") cfg.precision = ES_PRECISION_SPLIT;
        else if (p == "split_exact") cfg.precision = ES_PRECISION_SPLIT_EXACT;
        else if (p == "fp64") cfg.precision = ES_PRECISION_FP64;
        else throw ConfigError("precision must be 'fp64', 'split' or 'split_exact'");
    }
    cfg.batched = has(values, "batched") && std::atoi(values.at("batched").c_str()) == 1;
    cfg.device_ordinal = has(values, "device_ordinal") ? std::atoi(values.at("device_ordinal").c_str()) : 0;
    cfg.journal_path = has(values, "journal") ? values.at("journal") : "";
    return cfg;
}

RunConfig ParseConfigFile(const std::string& file_path)
{
    std::ifstream f(file_path, std::ios::in | std::ios::binary);
    if (!f) throw ConfigError("Could not load config file '" + file_path + "'");
    std::stringstream ss;
    ss << f.rdbuf();
    return ParseConfigText(ss.str(), file_path);
}

std::string DescribeConfig(const RunConfig& c)
{
    std::ostringstream o;
    o.precision(17);
    auto list = [&](const char* name, const auto& v) {
        o << "\"" << name << "\": [";
        for (size_t i = 0; i < v.size(); i++) o << (i ? ", " : "") << v[i];
        o << "]";
    };
    o << "{\"num_samples\": " << c.num_samples << ", \"dimension\": " << c.positions_per_row
      << ", \"phi_steps\": " << c.particles_per_quadrant << ", \"print_info\": " << (c.print_info ? 1 : 0)
      << ", \"output_type\": \""
      << (c.output_type == OutputType::Nothing ? "nothing" : c.output_type == OutputType::Results ? "results" : "all")
      << "\", \"device\": \"" << c.device << "\", ";
    list("magnetic_fields", c.magnetic_fields);
    o << ", ";
    list("temperatures", c.temperatures);
    o << ", ";
    list("sample_seeds", c.sample_seeds);
    o << ", \"particle_speed\": " << c.settings.particle_speed << ", \"tau\": " << c.settings.tau
      << ", \"alpha\": " << c.settings.alpha << ", \"clockwise\": " << c.settings.is_clockwise
      << ", \"region_size\": " << c.settings.region_size << ", \"region_extends\": " << c.settings.region_extends
      << ", \"impurity_density\": " << c.settings.impurity_density
      << ", \"impurity_radius\": " << c.settings.impurity_radius
      << ", \"target_cell_population\": " << c.settings.target_cell_population
      << ", \"output_directory\": \"" << c.output_directory << "\", \"digits_in_sample_num\": "
      << c.digits_in_sample_num << ", \"precision\": " << c.precision << ", \"batched\": " << (c.batched ? 1 : 0)
      << ", \"device_ordinal\": " << c.device_ordinal << ", \"journal\": \"" << c.journal_path << "\"}";
    return o.str();
}

}  // namespace es_host

void es_host_set_error(const char* msg);

extern "C" es_status es_config_describe(const char* config_path, char* out_json, int32_t out_len)
{
    if (!config_path || !out_json || out_len <= 0) {
        es_host_set_error("es_config_describe: bad arguments");
        return ES_ERR_BAD_ARG;
    }
    try {
        const std::string s = es_host::DescribeConfig(es_host::ParseConfigFile(config_path));
        if ((int64_t)s.size() + 1 > out_len) {
            es_host_set_error("es_config_describe: output buffer too small");
            return ES_ERR_BAD_ARG;
        }
        std::memcpy(out_json, s.c_str(), s.size() + 1);
        return ES_OK;
    } catch (const std::exception& e) {
        es_host_set_error(e.what());
        return ES_ERR_BAD_ARG;
    }
}
