// logger.cpp - results files in the reference's formats (src/Logger.cpp:42-334).
//
// Text layout, column widths and number formats follow the reference so that
// its loaders (reproduce_graphs/*/view_result.py) read these files unchanged.
// Metrics.txt is written as UTF-8 bytes with the C locale: the reference writes
// it through a wide stream imbued with en_US.UTF-8, which gives the same box
// characters; numbers here are never digit-grouped.
#include "logger.h"

#include <cmath>
#include <cstdint>
#include <fstream>
#include <iomanip>
#include <sstream>

namespace es_host {

namespace {

std::string repeat(const char* s, int n)
{
    std::string r;
    for (int i = 0; i < n; i++) r += s;
    return r;
}

}  // namespace

void Logger::CreateResultLog(const std::string& path, const RunConfig& cfg, double temperature)
{
    std::ofstream f(path);
    f << "# Elastic Scattering results summary." << std::endl;
    f << std::endl;
    f << "Temperature " << std::fixed << std::setprecision(4) << temperature << std::endl;
    f << std::endl;
    f << "MF values   " << cfg.magnetic_fields.size() << std::endl;
    f << "Samples     " << cfg.num_samples << std::endl;
    f << "Positions   " << cfg.positions_per_row << " x " << cfg.positions_per_row << std::endl;
    f << "Phi steps   " << cfg.particles_per_quadrant << std::endl;
    f << std::endl;
    f << "# Results #" << std::endl << std::endl;
    f << std::left << std::setw(8) << "B" << std::setw(rw) << "sigma_xx_inc" << std::setw(rw) << "sigma_xx_coh"
      << std::setw(rw) << "sigma_xy_inc" << std::setw(rw) << "sigma_xy_coh" << std::setw(rw) << "delta_xx" << std::endl;
}

void Logger::LogResult(const std::string& path, const DataRow& row)
{
    std::ofstream f(path, std::ios_base::app);
    f << std::left << std::setw(8) << std::setprecision(2) << std::fixed << row.magnetic_field << std::scientific
      << std::setprecision(result_precision) << std::setw(rw) << row.incoherent.xx << std::setw(rw) << row.coherent.xx
      << std::setw(rw) << row.incoherent.xy << std::setw(rw) << row.coherent.xy << std::setw(rw) << std::setprecision(4)
      << std::defaultfloat << row.xxd << std::endl;
}

void Logger::CreateSampleResultLog(const std::string& path)
{
    std::ofstream f(path);
    f << "# Elastic Scattering sample results summary." << std::endl << std::endl;
    f << std::left << std::setw(4) << "T" << std::setw(4) << "B" << std::setw(rw) << "sigma_xx_inc" << std::setw(rw)
      << "sigma_xx_coh" << std::setw(rw) << "sigma_xy_inc" << std::setw(rw) << "sigma_xy_coh" << std::endl;
}

void Logger::LogSampleResults(const std::string& path, const SampleResult& coherent, const SampleResult& incoherent)
{
    std::ofstream f(path, std::ios_base::app);
    f << std::setprecision(result_precision);
    const size_t T = coherent.results.empty() ? 0 : coherent.results[0].size();
    const size_t B = coherent.results.size();
    for (size_t j = 0; j < T; j++) {
        for (size_t i = 0; i < B; i++) {
            const auto& coh = coherent.results[i];
            const auto& inc = incoherent.results[i];
            f << std::left << std::setw(4) << j << std::setw(4) << i << std::setw(rw) << std::scientific << inc[j].xx
              << std::setw(rw) << std::scientific << coh[j].xx << std::setw(rw) << std::scientific << inc[j].xy
              << std::setw(rw) << std::scientific << coh[j].xy << std::endl;
        }
        f << std::endl;
    }
}

void Logger::CreateSampleMetricsLog(const std::string& path, const GlobalMetrics& gm)
{
    std::ofstream f(path);
    f << "# Metrics collected during particle lifetime computation." << std::endl << std::endl;
    f << "Positions  " << gm.particles_per_row << " x " << gm.particles_per_row << std::endl;
    f << "Phi values " << gm.phi_steps << std::endl;
    f << "Lifetimes  " << ((int64_t)gm.particles_per_row * gm.particles_per_row * gm.phi_steps) << std::endl;
    f << "Impurities " << gm.unique_impurity_count << std::endl;
    f << "Cells      " << gm.cells_per_row << " x " << gm.cells_per_row << std::endl;
    f << "Index time " << std::fixed << std::setprecision(1) << gm.grid_creation_time * 1000.0 << "ms" << std::endl;
    f << std::endl;
}

void Logger::LogSampleMetrics(const std::string& path, const SampleMetrics& sm)
{
    std::ofstream f(path, std::ios_base::app);
    const int mw = 26;  // metric column
    const int vw = 12;  // value columns
    const auto& m = sm.iteration_metrics;
    const int n = (int)m.size();

    if (sm.coherent) {  // the coherent sector precedes the incoherent one
        f << std::endl << std::endl << std::endl;
        f << "---------------------------------------------------------" << std::endl;
        f << "Sample " << sm.sample_index << (sm.coherent ? " Coherent" : " Incoherent") << std::endl;
        f << "---------------------------------------------------------" << std::endl;
        f << "Seed                      " << sm.seed << std::endl;
        f << "Total indexed impurities  " << std::setprecision(2) << (double)sm.total_indexed_impurities / 1000000.0
          << " mil (" << std::setprecision(4) << (sm.total_indexed_impurities - sm.impurity_count) << " overlapped)"
          << std::endl;
        f << "Avg. impurities per cell  " << std::setprecision(2)
          << (double)sm.total_indexed_impurities / (double)sm.total_cells << std::endl;
        f << "Positions inside impurity " << std::setprecision(2)
          << (100 * ((double)(n ? m[0].particle_metrics.particles_inside_impurity : 0) / (double)sm.total_particles))
          << "%" << std::endl;
    }

    auto blank_row = [&]() {
        f << "│" << std::string((size_t)mw, ' ');
        for (int i = 0; i < n; i++) f << "│" << std::string((size_t)vw, ' ');
        f << "│" << std::endl;
    };

    f << std::endl;
    f << "┌" << repeat("─", mw);
    for (int i = 0; i < n; i++) f << "┬" << repeat("─", vw);
    f << "┐" << std::endl;
    f << "│" << std::setw(mw) << std::left << (sm.coherent ? " Metric (Coherent)" : " Metric (Incoherent)");
    for (int i = 0; i < n; i++) f << "│" << std::setw(vw) << std::left << (" MF " + std::to_string(i));
    f << "│" << std::endl;
    f << "├" << repeat("─", mw);
    for (int i = 0; i < n; i++) f << "┼" << repeat("─", vw);
    f << "┤" << std::endl;

    f << "│" << std::setw(mw) << std::left << " Avg. particle lifetime";
    for (int i = 0; i < n; i++) f << "│" << std::setw(vw) << std::right << std::setprecision(3) << m[i].avg_particle_lifetime;
    f << "│" << std::endl;
    f << "│" << std::setw(mw) << std::left << "Time spent on";
    for (int i = 0; i < n; i++) f << "│" << std::string((size_t)vw, ' ');
    f << "│" << std::endl;
    f << "│" << std::setw(mw - 2) << std::left << "\t Lifetimes";
    for (int i = 0; i < n; i++)
        f << "│" << std::setw(vw - 2) << std::right << std::setprecision(3) << (m[i].time_elapsed_lifetimes * 1000.0)
          << "ms";
    f << "│" << std::endl;
    f << "│" << std::setw(mw - 2) << std::left << "\t Temperatures";
    for (int i = 0; i < n; i++)
        f << "│" << std::setw(vw - 2) << std::right << std::setprecision(3) << (m[i].time_elapsed_temperatures * 1000.0)
          << "ms";
    f << "│" << std::endl;
    f << "│" << std::setw(mw) << std::left << " Particles escaped";
    for (int i = 0; i < n; i++) f << "│" << std::setw(vw) << std::right << (double)m[i].particle_metrics.particles_escaped;
    f << "│" << std::endl;
    f << "│" << std::setw(mw) << std::left << " Particles at bound";
    for (int i = 0; i < n; i++) f << "│" << std::setw(vw) << std::right << (double)m[i].particle_metrics.particles_at_bound;
    f << "│" << std::endl;
    blank_row();

    f << "│" << std::setw(mw) << std::left << " Total impurities tested";
    for (int i = 0; i < n; i++)
        f << "│" << std::setw(vw - 4) << std::right << std::setprecision(3)
          << ((double)m[i].particle_metrics.impurities_tested / 1000000.0) << " mil";
    f << "│" << std::endl;
    f << "│" << std::setw(mw - 2) << std::left << "\t Average";
    for (int i = 0; i < n; i++)
        f << "│" << std::setw(vw) << std::right << std::setprecision(2)
          << ((double)m[i].particle_metrics.impurities_tested / (double)m[i].real_particles);
    f << "│" << std::endl;
    f << "│" << std::setw(mw - 2) << std::left << "\t Average %";
    for (int i = 0; i < n; i++)
        f << "│" << std::setw(vw - 1) << std::right << std::setprecision(2)
          << (100 * ((double)m[i].particle_metrics.impurities_tested / (double)m[i].real_particles) /
              (double)sm.impurity_count)
          << "%";
    f << "│" << std::endl;
    blank_row();

    f << "│" << std::setw(mw) << std::left << " Grid cells passed";
    for (int i = 0; i < n; i++)
        f << "│" << std::setw(vw - 4) << std::right << std::setprecision(3)
          << ((double)m[i].particle_metrics.cells_passed / 1000000.0) << " mil";
    f << "│" << std::endl;
    f << "│" << std::setw(mw - 2) << std::left << "\t Average";
    for (int i = 0; i < n; i++)
        f << "│" << std::setw(vw) << std::right << std::setprecision(2)
          << ((double)m[i].particle_metrics.cells_passed / (double)m[i].real_particles);
    f << "│" << std::endl;
    f << "│" << std::setw(mw - 2) << std::left << "\t Average %";
    for (int i = 0; i < n; i++)
        f << "│" << std::setw(vw - 1) << std::right << std::setprecision(2)
          << (100 * ((double)m[i].particle_metrics.cells_passed / (double)m[i].real_particles) / (double)sm.total_cells)
          << "%";
    f << "│" << std::endl;

    f << "└" << repeat("─", mw);
    for (int i = 0; i < n; i++) f << "┴" << repeat("─", vw);
    f << "┘" << std::endl;
}

namespace {

// One third of the image: a grey map (or, coloured, red for positive and blue
// for negative values) scaled by the extremes, as WriteImageSection does
// (src/Logger.cpp:278-318).
void image_section(std::vector<unsigned char>& px, const std::vector<double>& v, int dim, int id, bool colored)
{
    const int width = dim * 3 * 3;
    const int offset = id * dim * 3;
    double lo = 1.7976931348623157e308, hi = -1.7976931348623157e308;
    for (double k : v) {
        if (k < lo) lo = k;
        if (k > hi) hi = k;
    }
    for (int j = 0; j < dim; j++)
        for (int i = 0; i < dim; i++) {
            const int idx = j * width + i * 3 + offset;
            const double c = v[(size_t)j * dim + i];
            if (!colored) {
                const auto k = (unsigned char)((c - lo) / hi * 255.0);
                px[(size_t)idx] = px[(size_t)idx + 1] = px[(size_t)idx + 2] = k;
            } else if (c < 0) {
                px[(size_t)idx] = 0;
                px[(size_t)idx + 1] = 0;
                px[(size_t)idx + 2] = (unsigned char)(c / lo * 255.0);
            } else {
                px[(size_t)idx] = (unsigned char)(c / hi * 255.0);
                px[(size_t)idx + 1] = 0;
                px[(size_t)idx + 2] = 0;
            }
        }
}

uint32_t crc32(const unsigned char* p, size_t n, uint32_t crc = 0)
{
    static uint32_t table[256];
    static bool init = false;
    if (!init) {
        for (uint32_t i = 0; i < 256; i++) {
            uint32_t c = i;
            for (int k = 0; k < 8; k++) c = (c & 1) ? 0xEDB88320u ^ (c >> 1) : c >> 1;
            table[i] = c;
        }
        init = true;
    }
    crc = ~crc;
    for (size_t i = 0; i < n; i++) crc = table[(crc ^ p[i]) & 0xFF] ^ (crc >> 8);
    return ~crc;
}

void put32(std::string& s, uint32_t v)
{
    s += (char)(v >> 24);
    s += (char)(v >> 16);
    s += (char)(v >> 8);
    s += (char)v;
}

void chunk(std::ofstream& f, const char* type, const std::string& data)
{
    std::string c;
    put32(c, (uint32_t)data.size());
    std::string body = std::string(type, 4) + data;
    c += body;
    put32(c, crc32((const unsigned char*)body.data(), body.size()));
    f.write(c.data(), (std::streamsize)c.size());
}

}  // namespace

bool WritePng(const std::string& path, int width, int height, const std::vector<unsigned char>& rgb)
{
    std::ofstream f(path, std::ios::binary);
    if (!f) return false;
    static const unsigned char sig[8] = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1A, '\n'};
    f.write((const char*)sig, 8);
    std::string ihdr;
    put32(ihdr, (uint32_t)width);
    put32(ihdr, (uint32_t)height);
    ihdr += (char)8;  // bit depth
    ihdr += (char)2;  // RGB
    ihdr += (char)0;
    ihdr += (char)0;
    ihdr += (char)0;
    chunk(f, "IHDR", ihdr);
    // scanlines with filter byte 0, in a zlib stream of stored deflate blocks
    std::string raw;
    for (int y = 0; y < height; y++) {
        raw += (char)0;
        raw.append((const char*)&rgb[(size_t)y * width * 3], (size_t)width * 3);
    }
    std::string z;
    z += (char)0x78;
    z += (char)0x01;
    uint32_t a = 1, b = 0;  // Adler-32
    for (unsigned char c : raw) {
        a = (a + c) % 65521u;
        b = (b + a) % 65521u;
    }
    size_t pos = 0;
    do {
        const size_t len = std::min<size_t>(65535, raw.size() - pos);
        const bool last = pos + len == raw.size();
        z += (char)(last ? 1 : 0);
        z += (char)(len & 0xFF);
        z += (char)(len >> 8);
        z += (char)(~len & 0xFF);
        z += (char)((~len >> 8) & 0xFF);
        z.append(raw, pos, len);
        pos += len;
    } while (pos < raw.size());
    put32(z, (b << 16) | a);
    chunk(f, "IDAT", z);
    chunk(f, "IEND", "");
    return (bool)f;
}

void Logger::LogImages(const std::string& path, int dim, const IterationResult& it)
{
    const int width = dim * 3, height = dim;
    std::vector<unsigned char> px((size_t)width * height * 3);
    image_section(px, it.particle_lifetimes, dim, 0, false);
    image_section(px, it.xx_buffer, dim, 1, false);
    image_section(px, it.xy_buffer, dim, 2, true);
    WritePng(path, width, height, px);
}

}  // namespace es_host
