// runner.cpp - the .config sweep of SimulationRunner (src/SimulationRunner.cpp:31-221)
// on the CUDA backend, and its C ABI (es_run_config, include/es_host.h).
//
// Per-pass mode follows the reference call for call: per sample one Grid, the
// coherent then the incoherent sector, per field one ComputeSigmas (or
// ComputeSigmasWithImages when every output is requested), then the sample
// averages and delta_xx of FinishResults. `batched 1` runs every (sample,
// field, sector) pass of the config in one batched graph replay instead and
// writes the same files (without the per-position images, which the batched
// path does not materialise).
//
// With `journal <path>` every finished pass is appended to the journal, and a
// pass already there (same run inputs, sample seed, sector and field) is taken
// from it instead of being computed (journal.h). A resumed pass writes no
// per-position images: they are in the results folder of the run that
// computed it. The device context of the per-pass mode is created at the first
// pass to compute, so a sweep found whole in the journal needs no GPU.
#include "runner.h"

#include <chrono>
#include <cmath>
#include <cstring>
#include <filesystem>
#include <iostream>
#include <memory>
#include <sstream>

#include "es_host.h"
#include "es_nvtx.h"
#include "logger.h"

void es_host_set_error(const char* msg);

namespace es_host {

namespace {
double now_s()
{
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

Grid make_grid(const RunConfig& cfg, int sample)
{
    const es_settings& s = cfg.settings;
    return Grid(cfg.sample_seeds[(size_t)sample], s.region_size, s.region_extends, s.impurity_density,
                s.impurity_radius, s.target_cell_population);
}
}  // namespace

SimulationResult SimulationRunner::Run(const std::string& config_path) { return Run(ParseConfigFile(config_path)); }

SimulationResult SimulationRunner::Run(const RunConfig& cfg)
{
    es::Range nvtx_range("sweep");
    cfg_ = cfg;
    resumed_ = computed_ = 0;
    journal_.reset();
    log_ << "Starting simulation (" << cfg_.config_path << ")" << std::endl;
    if (!cfg_.journal_path.empty()) {
        journal_ = std::make_unique<Journal>(cfg_.journal_path, cfg_);
        log_ << "Journal: " << cfg_.journal_path << " (" << journal_->size() << " passes of this run)" << std::endl;
    }
    if (cfg_.output_type != OutputType::Nothing) {
        log_ << "Output directory: " << cfg_.output_directory << std::endl;
        CreateOutputDirectory();
    }
    log_ << std::endl;
    const double t0 = now_s();
    SimulationResult sr = cfg_.batched ? RunBatched() : RunSimulation();
    log_ << std::endl << "Finished! (" << (now_s() - t0) << "s)" << std::endl;
    if (journal_) log_ << "Passes: " << computed_ << " computed, " << resumed_ << " from the journal" << std::endl;
    if (cfg_.output_type != OutputType::Nothing) FinishResults(sr);
    return sr;
}

SimulationResult SimulationRunner::RunSimulation()
{
    const double tg = now_s();
    auto grid = std::make_unique<Grid>(make_grid(cfg_, 0));
    const double grid_time = now_s() - tg;
    if (cfg_.output_type != OutputType::Nothing) {
        GlobalMetrics gm;
        gm.particles_per_row = cfg_.positions_per_row;
        gm.phi_steps = 4 * cfg_.particles_per_quadrant;
        gm.cells_per_row = grid->GetCellsPerRow();
        gm.unique_impurity_count = grid->GetUniqueImpurityCount();
        gm.grid_creation_time = grid_time;
        Logger::CreateSampleMetricsLog(MetricsPath(), gm);
    }
    GridInformation gi;
    gi.cell_size = grid->GetSettings().cell_size;
    gi.indexed_impurity_count = grid->GetTotalImpurityCount();
    gi.index_size = (int64_t)grid->GetIndex().size();
    gi.region_size = cfg_.settings.region_size;
    gi.region_extends = cfg_.settings.region_extends;
    std::unique_ptr<SimulationCUDA> es;  // created at the first pass to compute

    SimulationResult sr;
    for (int i = 0; i < cfg_.num_samples; i++) {
        if (cfg_.output_type == OutputType::All) CreateSampleOutputDirectory(i);
        sr.coherent.push_back(RunSample(es, gi, i, true, *grid));
        sr.incoherent.push_back(RunSample(es, gi, i, false, *grid));
        if (cfg_.output_type == OutputType::All)
            Logger::LogSampleResults(SampleResultsPath(i), sr.coherent[(size_t)i], sr.incoherent[(size_t)i]);
        if (i + 1 < cfg_.num_samples) grid = std::make_unique<Grid>(make_grid(cfg_, i + 1));
    }
    return sr;
}

void SimulationRunner::Record(int sample_index, bool coherent, double field, const std::vector<Sigma>& sigma,
                              const Metrics& m)
{
    computed_++;
    if (!journal_) return;
    JournalEntry e;
    e.sample = sample_index;
    e.seed = cfg_.sample_seeds[(size_t)sample_index];
    e.coherent = coherent;
    e.field = field;
    e.sigma = sigma;
    e.metrics = m;
    journal_->Append(e);
}

SampleResult SimulationRunner::RunSample(std::unique_ptr<SimulationCUDA>& es, const GridInformation& gi,
                                         int sample_index, bool coherent, const Grid& grid)
{
    const int T = (int)cfg_.temperatures.size();
    const int N = (int)cfg_.magnetic_fields.size();
    SampleResult sr(T, N);
    const int64_t nlifetimes = (int64_t)cfg_.positions_per_row * cfg_.positions_per_row * 4 * cfg_.particles_per_quadrant;
    const std::string range = "sample " + std::to_string(sample_index) + (coherent ? " coherent" : " incoherent");
    es::Range nvtx_range(range.c_str());
    std::vector<const JournalEntry*> done((size_t)N, nullptr);
    int n_done = 0;
    if (journal_)
        for (int i = 0; i < N; i++)
            if ((done[(size_t)i] = journal_->Find(sample_index, cfg_.sample_seeds[(size_t)sample_index], coherent,
                                                 cfg_.magnetic_fields[(size_t)i])) != nullptr)
                n_done++;
    if (n_done < N) {
        if (!es)
            es = std::make_unique<SimulationCUDA>(cfg_.positions_per_row, cfg_.particles_per_quadrant, gi,
                                                  cfg_.device_ordinal, cfg_.precision);
        es->InitSample(grid, cfg_.settings, coherent);
    }
    SampleMetrics sm(sample_index, coherent, nlifetimes);
    sm.total_indexed_impurities = grid.GetTotalImpurityCount();
    sm.impurity_count = grid.GetUniqueImpurityCount();
    sm.total_cells = (int64_t)grid.GetCellsPerRow() * grid.GetCellsPerRow();
    sm.seed = grid.GetSeed();
    {
        const std::string raw = std::to_string(sample_index + 1);
        const std::string tag =
            std::string((size_t)std::max(0, cfg_.digits_in_sample_num - (int)raw.size()), '0') + raw +
            (coherent ? " C" : " I") + " [";
        log_ << '\r' << tag << std::string((size_t)N, '.') << "]" << '\r' << tag << std::flush;
    }
    for (int i = 0; i < N; i++) {
        const double B = cfg_.magnetic_fields[(size_t)i];
        if (const JournalEntry* d = done[(size_t)i]) {
            sr.results[(size_t)i] = d->sigma;
            sm.iteration_metrics.push_back(d->metrics);
            resumed_++;
            log_ << "j" << std::flush;
            continue;
        }
        if (cfg_.output_type != OutputType::All) {
            sr.results[(size_t)i] = es->ComputeSigmas(B, cfg_.temperatures, grid, sm);
        } else {
            auto it = es->ComputeSigmasWithImages(B, cfg_.temperatures, grid, sm);
            for (int j = 0; j < T; j++) {
                sr.results[(size_t)i][(size_t)j] = it[(size_t)j].result;
                Logger::LogImages(ImagePath(j, i, sample_index, coherent), cfg_.positions_per_row, it[(size_t)j]);
            }
        }
        Record(sample_index, coherent, B, sr.results[(size_t)i], sm.iteration_metrics.back());
        log_ << "x" << std::flush;
    }
    if (cfg_.output_type != OutputType::Nothing) Logger::LogSampleMetrics(MetricsPath(), sm);
    return sr;
}

SimulationResult SimulationRunner::RunBatched()
{
    es::Range nvtx_range("batched_sweep");
    const int S = cfg_.num_samples, N = (int)cfg_.magnetic_fields.size(), T = (int)cfg_.temperatures.size();
    if (T > ES_BATCH_MAX_T) throw SimulationError("batched runs take at most 8 temperatures");
    es_batch* b = nullptr;
    if (es_batch_create(cfg_.device_ordinal, &b) != ES_OK) throw SimulationError(es_last_error(nullptr));
    std::unique_ptr<es_batch, es_status (*)(es_batch*)> guard(b, es_batch_destroy);
    auto check = [&](es_status st) {
        if (st != ES_OK) throw SimulationError(es_batch_last_error(b));
    };
    es_batch_tuning tu{};
    check(es_batch_get_tuning(b, &tu));
    tu.precision = cfg_.precision;
    check(es_batch_set_tuning(b, &tu));

    // Every sample's Grid (src/SimulationRunner.cpp:60,96-97) built on the GPU
    // (es_dgrid: the host Grid's arrays bit for bit) and copied into the batch.
    struct SampleGrid {
        es_impurity_settings is{};
        int64_t indexed = 0, unique = 0;
        uint32_t seed = 0;
    };
    std::vector<SampleGrid> grids((size_t)S);
    std::vector<int32_t> ids((size_t)S);
    const double tg = now_s();
    for (int s = 0; s < S; s++) {
        const es_settings& st = cfg_.settings;
        es_dgrid* dg = nullptr;
        if (es_dgrid_create_seeded(cfg_.device_ordinal, cfg_.sample_seeds[(size_t)s], st.region_size,
                                   st.region_extends, st.impurity_density, st.impurity_radius,
                                   st.target_cell_population, 0, &dg) != ES_OK)
            throw SimulationError(es_last_error(nullptr));
        std::unique_ptr<es_dgrid, es_status (*)(es_dgrid*)> dguard(dg, es_dgrid_destroy);
        SampleGrid& g = grids[(size_t)s];
        if (es_dgrid_info(dg, &g.is, &g.indexed, &g.unique) != ES_OK) throw SimulationError(es_last_error(nullptr));
        g.seed = cfg_.sample_seeds[(size_t)s];
        check(es_batch_add_dgrid(b, dg, &ids[(size_t)s]));
    }
    const double grid_time = (now_s() - tg) / S;
    if (cfg_.output_type != OutputType::Nothing) {
        GlobalMetrics gm;
        gm.particles_per_row = cfg_.positions_per_row;
        gm.phi_steps = 4 * cfg_.particles_per_quadrant;
        gm.cells_per_row = grids[0].is.cells_per_row;
        gm.unique_impurity_count = grids[0].unique;
        gm.grid_creation_time = grid_time;
        Logger::CreateSampleMetricsLog(MetricsPath(), gm);
    }
    // The reference takes GridInformation::cell_size from the first sample's grid
    // for every sample (src/SimulationRunner.cpp:76-86).
    const double cell0 = grids[0].is.cell_size;
    std::vector<es_batch_instance> inst;
    // per (sample, sector, field): the journal's entry, or the batch instance
    std::vector<const JournalEntry*> done;
    std::vector<size_t> slot;
    for (int s = 0; s < S; s++)
        for (int coh = 1; coh >= 0; coh--)
            for (int i = 0; i < N; i++) {
                const JournalEntry* d =
                    journal_ ? journal_->Find(s, cfg_.sample_seeds[(size_t)s], coh == 1, cfg_.magnetic_fields[(size_t)i])
                             : nullptr;
                done.push_back(d);
                slot.push_back(inst.size());
                if (d) continue;
                es_batch_instance x{};
                x.grid = ids[(size_t)s];
                x.positions_per_row = cfg_.positions_per_row;
                x.particles_per_quadrant = cfg_.particles_per_quadrant;
                x.coherent = coh;
                x.region_size = cfg_.settings.region_size;
                x.grid_cell_size = cell0;
                x.magnetic_field = cfg_.magnetic_fields[(size_t)i];
                x.settings = cfg_.settings;
                x.n_t = T;
                for (int t = 0; t < T; t++) x.temperatures[t] = cfg_.temperatures[(size_t)t];
                inst.push_back(x);
            }
    std::vector<double> out(inst.size() * ES_BATCH_MAX_T * 2);
    std::vector<es_metrics> mets(inst.size());
    double run_s = 0;
    if (!inst.empty()) {
        check(es_batch_set_instances(b, inst.data(), (int32_t)inst.size()));
        const double t0 = now_s();
        check(es_batch_run(b, out.data(), mets.data()));
        run_s = now_s() - t0;
    }
    log_ << "Batched run: " << inst.size() << " passes in " << run_s << "s" << std::endl;

    SimulationResult sr;
    const int64_t nlt = (int64_t)cfg_.positions_per_row * cfg_.positions_per_row * 4 * cfg_.particles_per_quadrant;
    size_t k = 0;
    for (int s = 0; s < S; s++) {
        for (int coh = 1; coh >= 0; coh--) {
            SampleResult res(T, N);
            SampleMetrics sm(s, coh == 1, nlt);
            const SampleGrid& g = grids[(size_t)s];
            sm.total_indexed_impurities = g.indexed;
            sm.impurity_count = g.unique;
            sm.total_cells = (int64_t)g.is.cells_per_row * g.is.cells_per_row;
            sm.seed = g.seed;
            for (int i = 0; i < N; i++, k++) {
                if (const JournalEntry* d = done[k]) {
                    res.results[(size_t)i] = d->sigma;
                    sm.iteration_metrics.push_back(d->metrics);
                    resumed_++;
                    continue;
                }
                const size_t q = slot[k];
                for (int t = 0; t < T; t++)
                    res.results[(size_t)i][(size_t)t] = Sigma(out[(q * ES_BATCH_MAX_T + t) * 2],
                                                              out[(q * ES_BATCH_MAX_T + t) * 2 + 1]);
                Metrics m;
                m.particle_metrics = mets[q];
                m.real_particles = nlt - mets[q].particles_inside_impurity;
                m.time_elapsed_lifetimes = run_s / (double)inst.size();  // the batch's mean time per pass
                sm.iteration_metrics.push_back(m);
                Record(s, coh == 1, cfg_.magnetic_fields[(size_t)i], res.results[(size_t)i], m);
            }
            if (cfg_.output_type != OutputType::Nothing) Logger::LogSampleMetrics(MetricsPath(), sm);
            (coh ? sr.coherent : sr.incoherent).push_back(res);
        }
        if (cfg_.output_type == OutputType::All) {
            CreateSampleOutputDirectory(s);
            Logger::LogSampleResults(SampleResultsPath(s), sr.coherent[(size_t)s], sr.incoherent[(size_t)s]);
        }
    }
    return sr;
}

void SimulationRunner::FinishResults(const SimulationResult& sr) const
{
    const double S = (double)cfg_.num_samples;
    for (size_t j = 0; j < cfg_.temperatures.size(); j++) {
        const double temperature = cfg_.temperatures[j];
        const std::string file = ResultPath((int)j);
        Logger::CreateResultLog(file, cfg_, temperature);
        for (size_t i = 0; i < cfg_.magnetic_fields.size(); i++) {
            Sigma coherent, incoherent;
            double dxx_squared = 0;
            for (int s = 0; s < cfg_.num_samples; s++) {
                const Sigma coh = sr.coherent[(size_t)s].results[i][j];
                const Sigma inc = sr.incoherent[(size_t)s].results[i][j];
                coherent += coh;
                incoherent += inc;
                dxx_squared += std::pow(coh.xx + inc.xx, 2);
            }
            coherent.xx /= S;
            coherent.xy /= S;
            incoherent.xx /= S;
            incoherent.xy /= S;
            DataRow row;
            row.temperature = temperature;
            row.magnetic_field = cfg_.magnetic_fields[i];
            row.coherent = coherent;
            row.incoherent = incoherent;
            if (cfg_.num_samples == 1) {
                row.xxd = 0;
            } else {
                // src/SimulationRunner.cpp:183-193
                const double sq_exp = dxx_squared / S;
                const double exp = coherent.xx + incoherent.xx;
                const double stdev = std::sqrt((sq_exp - exp * exp) / (S - 1.0));
                row.xxd = stdev / exp;
            }
            Logger::LogResult(file, row);
        }
    }
}

void SimulationRunner::CreateSampleOutputDirectory(int sample_index) const
{
    const std::string p = SamplePath(sample_index);
    std::filesystem::create_directory(p);
    std::filesystem::create_directory(p + "/Incoherent/");
    std::filesystem::create_directory(p + "/Coherent/");
    Logger::CreateSampleResultLog(SampleResultsPath(sample_index));
}

void SimulationRunner::CreateOutputDirectory() const
{
    if (!std::filesystem::exists(cfg_.base_output_directory))
        std::filesystem::create_directories(cfg_.base_output_directory);
    std::filesystem::create_directory(cfg_.output_directory);
    const auto slash = cfg_.config_path.rfind('/');
    const std::string name = slash != std::string::npos ? cfg_.config_path.substr(slash) : cfg_.config_path;
    std::filesystem::copy_file(cfg_.config_path, cfg_.output_directory + "/" + name,
                               std::filesystem::copy_options::overwrite_existing);
}

}  // namespace es_host

extern "C" es_status es_run_config(const char* config_path, char* out_directory, int32_t out_len, int32_t quiet)
{
    if (!config_path) {
        es_host_set_error("es_run_config: null config path");
        return ES_ERR_BAD_ARG;
    }
    std::ostringstream sink;
    std::ostream& log = quiet ? static_cast<std::ostream&>(sink) : std::cout;
    try {
        es_host::SimulationRunner runner(log);
        runner.Run(std::string(config_path));
        if (out_directory && out_len > 0) {
            std::strncpy(out_directory, runner.config().output_directory.c_str(), (size_t)out_len - 1);
            out_directory[out_len - 1] = '\0';
        }
        return ES_OK;
    } catch (const es_host::ConfigError& e) {
        es_host_set_error(e.what());
        return ES_ERR_BAD_ARG;
    } catch (const std::exception& e) {
        es_host_set_error(e.what());
        return ES_ERR_LAUNCH;
    }
}
