/* es_host.h - C ABI of the host runtime that surrounds the CUDA backend:
 * the impurity field + cell index (the reference's Grid, src/sim/Grid.h:55-94)
 * and the .config sweep driver (src/SimulationRunner.cpp).
 *
 * The Grid is host C++ like the reference's and makes the same standard
 * library calls (std::default_random_engine + std::uniform_real_distribution,
 * src/sim/Grid.cpp:61-75), so a seed gives the same impurity field as the
 * reference built with the same C++ standard library.
 */
#ifndef ES_HOST_H
#define ES_HOST_H

#include <stdint.h>

#include "es_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct es_grid es_grid;

/* Replaces Grid(seed, region_size, region_extends, density, radius,
 * target_cell_population) (src/sim/Grid.cpp:28-46). max_impurities caps the
 * impurity count like the reference's "Woah!" check (src/sim/Grid.cpp:36);
 * pass 0 for the reference's 1e7. */
es_status es_grid_create_seeded(uint32_t seed, double region_size, double region_extends, double density,
                                double impurity_radius, int32_t target_cell_population, int64_t max_impurities,
                                es_grid** out);

/* Replaces Grid(vector<v2> impurities, ...) (src/sim/Grid.cpp:48-59). */
es_status es_grid_create_from_list(const double* xy, int64_t n, double region_size, double region_extends,
                                   double impurity_radius, int32_t target_cell_population, es_grid** out);

void es_grid_destroy(es_grid* g);

/* Grid::GetImpurities / GetIndex / GetSettings / GetCellsPerRow / GetSeed /
 * GetUniqueImpurityCount / GetTotalImpurityCount (src/sim/Grid.h:74-91). */
const double* es_grid_impurities(const es_grid* g);   /* x,y pairs, es_grid_indexed_count of them */
const int32_t* es_grid_index(const es_grid* g);        /* cells_per_row^2 cumulative ends */
int64_t es_grid_indexed_count(const es_grid* g);
int64_t es_grid_unique_count(const es_grid* g);
int32_t es_grid_cells_per_row(const es_grid* g);
uint32_t es_grid_seed(const es_grid* g);
void es_grid_settings(const es_grid* g, es_impurity_settings* out);
/* Process-unique, never reused identity of this impurity field: the key to
 * pass to es_upload_grid so a resident copy is reused only for this grid. */
uint64_t es_grid_generation(const es_grid* g);

/* Replaces SimulationRunner::Run (src/SimulationRunner.cpp:31-50) and the
 * executable around it (src/main.cpp): parses a reference .config file with the
 * reference's rules (src/SimulationConfiguration.h:79-228), runs the sweep over
 * samples, magnetic fields and temperatures on the CUDA backend, and writes the
 * reference's results folder (<output_directory>/Result_<n>/ with the config,
 * T<j>.dat, Metrics.txt and Sample <i>/ with sample_results.dat and the PNG
 * maps). The folder used is copied to out_directory (out_len bytes, may be
 * NULL). quiet != 0 suppresses the progress output. Errors, including config
 * errors the reference exits on, return non-OK with es_host_last_error().
 * With the added key `journal <path>` every finished (sample, sector, field)
 * pass is appended to that file as one JSON line, and passes already there
 * (same run inputs) are taken from it instead of being computed, so a stopped
 * sweep resumes; a sweep found whole in the journal makes no device call. */
es_status es_run_config(const char* config_path, char* out_directory, int32_t out_len, int32_t quiet);

/* The parsed form of a .config file (the values es_run_config would use) as a
 * JSON object in out_json (out_len bytes). No reference counterpart: a dry run
 * of SimulationConfiguration::ParseFromeFile (src/SimulationConfiguration.h:79-228). */
es_status es_config_describe(const char* config_path, char* out_json, int32_t out_len);

/* Message of the last failed es_grid_* or es_run_config call on this thread. */
const char* es_host_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* ES_HOST_H */
