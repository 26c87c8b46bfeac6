// grid.h - impurity field and cell index, the host half of the path's input.
//
// Same interface as the reference's Grid (src/sim/Grid.h:55-94): uniform
// random impurities from a seed (or a given list), binned into
// cells_per_row^2 cells with the reference's overlap rules and flattened to
// (ordered impurities, cumulative end index per cell).
#pragma once

#include <cstdint>
#include <stdexcept>
#include <vector>

#include "es_cuda.h"

namespace es_host {

struct v2 {
    double x, y;
};

class Grid {
public:
    // Grid(seed, ...), src/sim/Grid.cpp:28-46. Throws std::runtime_error for the
    // reference's config errors ("Woah!" above max_impurities, "No impurities").
    Grid(uint32_t seed, double region_size, double region_extends, double density, double impurity_radius,
         int target_cell_population, int64_t max_impurities = 10000000);
    // Grid(vector<v2>, ...), src/sim/Grid.cpp:48-59.
    Grid(const std::vector<v2>& impurities, double region_size, double region_extends, double impurity_radius,
         int target_cell_population);

    const std::vector<v2>& GetImpurities() const { return ordered_impurities_; }
    const std::vector<int32_t>& GetIndex() const { return imp_index_; }
    int64_t GetUniqueImpurityCount() const { return unique_impurity_count_; }
    int64_t GetTotalImpurityCount() const { return (int64_t)ordered_impurities_.size(); }
    int GetCellsPerRow() const { return cells_per_row_; }
    uint32_t GetSeed() const { return seed_used_; }
    es_impurity_settings GetSettings() const;
    // Monotone identity of this impurity field, used as the upload key of the
    // device copy (the reference keys on the seed, which is 0 for file grids).
    uint64_t Generation() const { return generation_; }

private:
    void Build(const std::vector<v2>& impurities);

    std::vector<v2> ordered_impurities_;
    std::vector<int32_t> imp_index_;
    int64_t unique_impurity_count_ = 0;
    double lo_ = 0, hi_ = 0;
    int cells_per_row_ = 0;
    double cell_size_ = 0;
    double impurity_radius_ = 0;
    uint32_t seed_used_ = 0;
    uint64_t generation_ = 0;
};

}  // namespace es_host
