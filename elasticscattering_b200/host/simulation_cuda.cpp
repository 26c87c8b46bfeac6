// simulation_cuda.cpp - Simulation's methods on the C ABI (include/es_cuda.h).
#include "simulation_cuda.h"

#include <chrono>

namespace es_host {

namespace {
double now_s()
{
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}
}  // namespace

SimulationCUDA::SimulationCUDA(int positions_per_row, int phi_steps, const GridInformation& gi, int device,
                               int precision)
    : positions_per_row_(positions_per_row), phi_steps_(phi_steps)
{
    es_sim_desc d{};
    d.positions_per_row = positions_per_row;
    d.particles_per_quadrant = phi_steps;
    d.region_size = gi.region_size;
    d.region_extends = gi.region_extends;
    d.grid_cell_size = gi.cell_size;
    d.device_ordinal = device;
    d.precision = precision;
    const es_status st = es_create(&d, &ctx_);
    if (st != ES_OK) throw SimulationError(std::string("es_create: ") + es_last_error(nullptr));
    total_particles_ = (int64_t)positions_per_row * positions_per_row * 4 * phi_steps;
}

SimulationCUDA::~SimulationCUDA()
{
    if (ctx_) es_destroy(ctx_);
}

void SimulationCUDA::check(es_status st) const
{
    if (st != ES_OK) throw SimulationError(es_last_error(ctx_));
}

void SimulationCUDA::InitSample(const Grid& grid, const es_settings& settings, bool coherent)
{
    const es_impurity_settings is = grid.GetSettings();
    const auto& imps = grid.GetImpurities();
    check(es_upload_grid(ctx_, imps.empty() ? nullptr : &imps[0].x, grid.GetTotalImpurityCount(),
                         grid.GetIndex().data(), &is, grid.Generation()));
    check(es_init_sample(ctx_, &settings, coherent ? 1 : 0));
}

Metrics SimulationCUDA::LifetimeMetrics(const es_metrics& m, double seconds)
{
    Metrics out;
    out.particle_metrics = m;
    out.time_elapsed_lifetimes = seconds;
    // SimulationCPU::ComputeSigmas, src/sim/SimulationCPU.cpp:41
    out.real_particles = total_particles_ - m.particles_inside_impurity;
    check(es_average_lifetime(ctx_, &out.avg_particle_lifetime));
    return out;
}

std::vector<Sigma> SimulationCUDA::ComputeSigmas(double magnetic_field, const std::vector<double>& temperatures,
                                                 const Grid&, SampleMetrics& sample_metrics)
{
    es_metrics m{};
    const double t0 = now_s();
    check(es_compute_lifetimes(ctx_, magnetic_field, nullptr, &m));
    const double t1 = now_s();
    Metrics metrics = LifetimeMetrics(m, t1 - t0);
    std::vector<double> out(2 * temperatures.size());
    const double t2 = now_s();
    check(es_derive_temperatures(ctx_, temperatures.data(), (int32_t)temperatures.size(), out.data()));
    metrics.time_elapsed_temperatures = now_s() - t2;
    sample_metrics.iteration_metrics.push_back(metrics);
    std::vector<Sigma> res(temperatures.size());
    for (size_t t = 0; t < temperatures.size(); t++) res[t] = Sigma(out[2 * t], out[2 * t + 1]);
    return res;
}

std::vector<IterationResult> SimulationCUDA::ComputeSigmasWithImages(double magnetic_field,
                                                                     const std::vector<double>& temperatures,
                                                                     const Grid&, SampleMetrics& sample_metrics)
{
    const size_t nt = temperatures.size();
    const size_t npos = (size_t)positions_per_row_ * positions_per_row_;
    std::vector<double> out(2 * nt), lt(nt * npos), xx(nt * npos), xy(nt * npos);
    es_metrics m{};
    const double t0 = now_s();
    check(es_compute_sigmas_images(ctx_, magnetic_field, temperatures.data(), (int32_t)nt, out.data(), lt.data(),
                                   xx.data(), xy.data(), &m));
    const double t1 = now_s();
    Metrics metrics = LifetimeMetrics(m, t1 - t0);
    sample_metrics.iteration_metrics.push_back(metrics);
    std::vector<IterationResult> res(nt);
    for (size_t t = 0; t < nt; t++) {
        res[t].particle_lifetimes.assign(lt.begin() + t * npos, lt.begin() + (t + 1) * npos);
        res[t].xx_buffer.assign(xx.begin() + t * npos, xx.begin() + (t + 1) * npos);
        res[t].xy_buffer.assign(xy.begin() + t * npos, xy.begin() + (t + 1) * npos);
        res[t].result = Sigma(out[2 * t], out[2 * t + 1]);
    }
    return res;
}

}  // namespace es_host
