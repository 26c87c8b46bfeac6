// journal.h - the per-pass results journal of a .config sweep (config key
// `journal <path>`).
//
// Every finished (sample, sector, field) pass appends one JSON line: its sigma
// at every temperature and its metrics. A sweep that stopped part way -- a
// killed job, a crash, a failed call -- is run again with the same config and
// journal, and every pass found there is taken from the journal instead of
// being computed. No reference counterpart: the reference has no resume
// (src/SimulationRunner.cpp:88-98 runs every pass every time).
//
// Line format (one object per line, keys in this order):
//   {"journal":1,"run":"<16 hex digits>","sample":S,"seed":U,"coherent":0|1,
//    "field":B,"sigma":[[xx,xy],...],"metrics":{<the es_metrics counters>},
//    "real_particles":N,"avg_particle_lifetime":X,"time_lifetimes":X,
//    "time_temperatures":X}
// Doubles are written with 17 significant digits, so they read back bit for
// bit. "run" is a hash of every input that decides a pass's sigma (start grid,
// phases, precision, per-pass or batched mode, Settings, temperatures); lines
// of other runs, and a torn last line, are ignored. A line is appended with
// one write(2) on a file opened O_APPEND: it survives the process, not the
// machine.
#pragma once

#include <cstdint>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "config.h"
#include "simulation_cuda.h"

namespace es_host {

struct JournalEntry {
    int sample = 0;
    unsigned int seed = 0;
    bool coherent = false;
    double field = 0;
    std::vector<Sigma> sigma;  // one per temperature of the run
    Metrics metrics;
};

class Journal {
public:
    // Reads the entries of `path` that belong to this run (the file need not
    // exist) and opens it for appending.
    Journal(const std::string& path, const RunConfig& cfg);
    ~Journal();
    Journal(const Journal&) = delete;
    Journal& operator=(const Journal&) = delete;

    const JournalEntry* Find(int sample, unsigned int seed, bool coherent, double field) const;
    void Append(const JournalEntry& e);
    size_t size() const { return entries_.size(); }

    // The run key: FNV-1a (64 bit) over the inputs that decide a pass's sigma.
    static uint64_t RunKey(const RunConfig& cfg);
    // One journal line (no newline) and its parse; Parse returns false for a
    // line that is not a complete entry of run `key`.
    static std::string Format(uint64_t key, const JournalEntry& e);
    static bool Parse(const std::string& line, uint64_t key, size_t n_temperatures, JournalEntry& out);

private:
    using Key = std::tuple<int, unsigned int, int, uint64_t>;
    static Key KeyOf(int sample, unsigned int seed, bool coherent, double field);

    std::string path_;
    uint64_t run_ = 0;
    size_t n_t_ = 0;
    int fd_ = -1;
    std::map<Key, JournalEntry> entries_;
};

}  // namespace es_host
