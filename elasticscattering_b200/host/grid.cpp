// grid.cpp - impurity field + cell index (reference: src/sim/Grid.cpp).
//
// The reference files each impurity into up to 9 per-cell std::vectors
// (std::set-deduplicated probes, then corner checks) and concatenates them
// row-major. This runtime computes the same cells per impurity and places the
// impurities with a two-pass stable counting sort, which yields the identical
// ordered array and cumulative index without per-cell containers.
#include "grid.h"

#include <atomic>
#include <cmath>
#include <cstring>
#include <random>
#include <string>

#include "es_host.h"

namespace es_host {

namespace {

std::atomic<uint64_t> g_generation{1};

struct Geo {
    double lo, size, cell_size;
    int cpr;

    // Grid::get_cell, src/sim/Grid.cpp:182-188 (truncation toward zero)
    void cell(double x, double y, int& cx, int& cy) const
    {
        cx = (int)((x - lo) / size * (double)(cpr));
        cy = (int)((y - lo) / size * (double)(cpr));
    }
    bool within(int cx, int cy) const { return cx >= 0 && cx < cpr && cy >= 0 && cy < cpr; }
};

// The cells add_to_overlapping_cells (src/sim/Grid.cpp:112-180) files one
// impurity under, in its push order. Returns how many (at most 9).
int overlapping_cells(const Geo& g, v2 pos, double r, int* out)
{
    int px[5], py[5];
    g.cell(pos.x, pos.y, px[0], py[0]);
    g.cell(pos.x + r, pos.y, px[1], py[1]);
    g.cell(pos.x - r, pos.y, px[2], py[2]);
    g.cell(pos.x, pos.y + r, px[3], py[3]);
    g.cell(pos.x, pos.y - r, px[4], py[4]);

    int n = 0;
    int ax[5], ay[5], na = 0;
    for (int i = 0; i < 5; i++) {
        bool seen = false;
        for (int k = 0; k < na; k++) seen |= (ax[k] == px[i] && ay[k] == py[i]);
        if (!seen && g.within(px[i], py[i])) {
            ax[na] = px[i];
            ay[na] = py[i];
            na++;
            out[n++] = py[i] * g.cpr + px[i];
        }
    }

    // Grid::to_world uses spawn_range.x for both axes (src/sim/Grid.h:48-51).
    const double llx = g.lo + px[0] * g.cell_size, lly = g.lo + py[0] * g.cell_size;
    const double cxs[4] = {0 + llx, g.cell_size + llx, llx, g.cell_size + llx};  // tl, tr, ll, lr
    const double cys[4] = {g.cell_size + lly, g.cell_size + lly, lly, 0 + lly};
    const int ox[4] = {-1, 1, -1, 1}, oy[4] = {1, 1, -1, -1};
    const double ir2 = r * r;
    int cx, cy;
    g.cell(pos.x, pos.y, cx, cy);
    for (int k = 0; k < 4; k++) {
        const double dx = cxs[k] - pos.x, dy = cys[k] - pos.y;
        if (dx * dx + dy * dy < ir2 && g.within(cx + ox[k], cy + oy[k])) out[n++] = (cy + oy[k]) * g.cpr + (cx + ox[k]);
    }
    return n;
}

}  // namespace

Grid::Grid(uint32_t seed, double region_size, double region_extends, double density, double impurity_radius,
           int target_cell_population, int64_t max_impurities)
{
    seed_used_ = seed;
    impurity_radius_ = impurity_radius;
    lo_ = -region_extends;
    hi_ = region_size + region_extends;
    const double area_length = hi_ - lo_;
    const double proposal = area_length * area_length * density;
    if (proposal > (double)max_impurities) throw std::runtime_error("Woah!");
    if (proposal < 1) throw std::runtime_error("No impurities");
    if (target_cell_population < 1) throw std::runtime_error("target_cell_population must be >= 1");

    unique_impurity_count_ = std::max<int64_t>(1, (int64_t)std::ceil(proposal));
    cells_per_row_ = std::max((int)std::round(std::sqrt(unique_impurity_count_ / (double)target_cell_population)), 1);
    cell_size_ = (hi_ - lo_) / (double)cells_per_row_;

    // GenerateImpurities, src/sim/Grid.cpp:61-75: the seed passes through an int.
    std::vector<v2> imps((size_t)unique_impurity_count_);
    std::uniform_real_distribution<double> unif(lo_, hi_);
    std::default_random_engine re((int)seed);
    for (auto& p : imps) {
        const double x = unif(re);
        const double y = unif(re);
        p = v2{x, y};
    }
    Build(imps);
}

Grid::Grid(const std::vector<v2>& impurities, double region_size, double region_extends, double impurity_radius,
           int target_cell_population)
{
    impurity_radius_ = impurity_radius;
    lo_ = -region_extends;
    hi_ = region_size + region_extends;
    if (target_cell_population < 1) throw std::runtime_error("target_cell_population must be >= 1");
    unique_impurity_count_ = (int64_t)impurities.size();
    cells_per_row_ = std::max((int)std::round(std::sqrt(unique_impurity_count_ / (double)target_cell_population)), 1);
    cell_size_ = (hi_ - lo_) / (double)cells_per_row_;
    Build(impurities);
}

void Grid::Build(const std::vector<v2>& imps)
{
    // GenerateImpurityCells + ConvertToIndex, src/sim/Grid.cpp:77-110
    Geo g{lo_, hi_ - lo_, cell_size_, cells_per_row_};
    const size_t n_cells = (size_t)cells_per_row_ * (size_t)cells_per_row_;
    std::vector<int64_t> count(n_cells, 0);
    int cells[9];
    int64_t total = 0;
    for (const v2& p : imps) {
        const int k = overlapping_cells(g, p, impurity_radius_, cells);
        for (int c = 0; c < k; c++) count[(size_t)cells[c]]++;
        total += k;
    }
    if (total > INT32_MAX) throw std::runtime_error("indexed impurity count exceeds the int32 cell index");
    imp_index_.resize(n_cells);
    std::vector<int64_t> cursor(n_cells);
    int64_t acc = 0;
    for (size_t c = 0; c < n_cells; c++) {
        cursor[c] = acc;
        acc += count[c];
        imp_index_[c] = (int32_t)acc;
    }
    ordered_impurities_.resize((size_t)total);
    for (const v2& p : imps) {
        const int k = overlapping_cells(g, p, impurity_radius_, cells);
        for (int c = 0; c < k; c++) ordered_impurities_[(size_t)cursor[(size_t)cells[c]]++] = p;
    }
    generation_ = g_generation.fetch_add(1);
}

es_impurity_settings Grid::GetSettings() const
{
    // Grid::GetSettings, src/sim/Grid.h:77-86
    es_impurity_settings is;
    is.impurity_radius = impurity_radius_;
    is.spawn_region_start = lo_;
    is.spawn_region_size = hi_ - lo_;
    is.cells_per_row = cells_per_row_;
    is.cell_size = is.spawn_region_size / (double)cells_per_row_;
    return is;
}

}  // namespace es_host

// ---- C ABI -----------------------------------------------------------------

struct es_grid {
    es_host::Grid grid;
};

namespace {
thread_local std::string g_host_error;
}

void es_host_set_error(const char* msg) { g_host_error = msg ? msg : ""; }

extern "C" {

const char* es_host_last_error(void) { return g_host_error.c_str(); }

es_status es_grid_create_seeded(uint32_t seed, double region_size, double region_extends, double density,
                                double impurity_radius, int32_t target_cell_population, int64_t max_impurities,
                                es_grid** out)
{
    if (!out) return ES_ERR_BAD_ARG;
    *out = nullptr;
    try {
        *out = new es_grid{es_host::Grid(seed, region_size, region_extends, density, impurity_radius,
                                         target_cell_population, max_impurities > 0 ? max_impurities : 10000000)};
    } catch (const std::bad_alloc&) {
        g_host_error = "host allocation failed";
        return ES_ERR_OOM;
    } catch (const std::exception& e) {
        g_host_error = e.what();
        return ES_ERR_BAD_ARG;
    }
    return ES_OK;
}

es_status es_grid_create_from_list(const double* xy, int64_t n, double region_size, double region_extends,
                                   double impurity_radius, int32_t target_cell_population, es_grid** out)
{
    if (!out || n < 0 || (n > 0 && !xy)) return ES_ERR_BAD_ARG;
    *out = nullptr;
    try {
        std::vector<es_host::v2> imps((size_t)n);
        for (int64_t i = 0; i < n; i++) imps[(size_t)i] = es_host::v2{xy[2 * i], xy[2 * i + 1]};
        *out = new es_grid{es_host::Grid(imps, region_size, region_extends, impurity_radius, target_cell_population)};
    } catch (const std::bad_alloc&) {
        g_host_error = "host allocation failed";
        return ES_ERR_OOM;
    } catch (const std::exception& e) {
        g_host_error = e.what();
        return ES_ERR_BAD_ARG;
    }
    return ES_OK;
}

void es_grid_destroy(es_grid* g) { delete g; }

const double* es_grid_impurities(const es_grid* g)
{
    return g ? reinterpret_cast<const double*>(g->grid.GetImpurities().data()) : nullptr;
}
const int32_t* es_grid_index(const es_grid* g) { return g ? g->grid.GetIndex().data() : nullptr; }
int64_t es_grid_indexed_count(const es_grid* g) { return g ? g->grid.GetTotalImpurityCount() : 0; }
int64_t es_grid_unique_count(const es_grid* g) { return g ? g->grid.GetUniqueImpurityCount() : 0; }
int32_t es_grid_cells_per_row(const es_grid* g) { return g ? g->grid.GetCellsPerRow() : 0; }
uint32_t es_grid_seed(const es_grid* g) { return g ? g->grid.GetSeed() : 0; }
uint64_t es_grid_generation(const es_grid* g) { return g ? g->grid.Generation() : 0; }
void es_grid_settings(const es_grid* g, es_impurity_settings* out)
{
    if (g && out) *out = g->grid.GetSettings();
}

}  // extern "C"
