// journal.cpp - the per-pass results journal (journal.h).
#include "journal.h"

#include <fcntl.h>
#include <unistd.h>

#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>

namespace es_host {

namespace {

// ---- a small JSON reader for the journal's own lines ----------------------

struct JVal {
    enum Type { Null, Bool, Num, Str, Arr, Obj } type = Null;
    std::string text;  // number text or string value
    std::vector<JVal> items;
    std::vector<std::pair<std::string, JVal>> fields;

    const JVal* get(const char* key) const
    {
        for (const auto& f : fields)
            if (f.first == key) return &f.second;
        return nullptr;
    }
};

struct Reader {
    const char* p;
    const char* end;

    void ws()
    {
        while (p < end && (*p == ' ' || *p == '\t' || *p == '\r' || *p == '\n')) p++;
    }
    bool lit(const char* s)
    {
        const size_t n = std::strlen(s);
        if ((size_t)(end - p) < n || std::strncmp(p, s, n) != 0) return false;
        p += n;
        return true;
    }
    bool string(std::string& out)
    {
        if (p >= end || *p != '"') return false;
        p++;
        out.clear();
        while (p < end && *p != '"') {
            if (*p == '\\') {
                if (++p >= end) return false;
                switch (*p) {
                    case '"': out += '"'; break;
                    case '\\': out += '\\'; break;
                    case '/': out += '/'; break;
                    case 'n': out += '\n'; break;
                    case 't': out += '\t'; break;
                    default: return false;  // the journal writes no other escapes
                }
                p++;
            } else {
                out += *p++;
            }
        }
        if (p >= end) return false;
        p++;
        return true;
    }
    bool value(JVal& v, int depth)
    {
        if (depth > 8) return false;
        ws();
        if (p >= end) return false;
        if (*p == '{') {
            p++;
            v.type = JVal::Obj;
            ws();
            if (p < end && *p == '}') return ++p, true;
            for (;;) {
                ws();
                std::string key;
                if (!string(key)) return false;
                ws();
                if (p >= end || *p != ':') return false;
                p++;
                JVal item;
                if (!value(item, depth + 1)) return false;
                v.fields.emplace_back(std::move(key), std::move(item));
                ws();
                if (p < end && *p == ',') {
                    p++;
                    continue;
                }
                if (p < end && *p == '}') return ++p, true;
                return false;
            }
        }
        if (*p == '[') {
            p++;
            v.type = JVal::Arr;
            ws();
            if (p < end && *p == ']') return ++p, true;
            for (;;) {
                JVal item;
                if (!value(item, depth + 1)) return false;
                v.items.push_back(std::move(item));
                ws();
                if (p < end && *p == ',') {
                    p++;
                    continue;
                }
                if (p < end && *p == ']') return ++p, true;
                return false;
            }
        }
        if (*p == '"') {
            v.type = JVal::Str;
            return string(v.text);
        }
        if (lit("true") || lit("false")) {
            v.type = JVal::Bool;
            return true;
        }
        if (lit("null")) {
            v.type = JVal::Null;
            return true;
        }
        const char* s = p;
        while (p < end && (std::strchr("+-0123456789.eE", *p) != nullptr)) p++;
        if (p == s) return false;
        v.type = JVal::Num;
        v.text.assign(s, p);
        return true;
    }
};

bool as_double(const JVal* v, double& out)
{
    if (!v || v->type != JVal::Num) return false;
    char* e = nullptr;
    out = std::strtod(v->text.c_str(), &e);
    return e && *e == '\0';
}

bool as_int(const JVal* v, long long& out)
{
    if (!v || v->type != JVal::Num) return false;
    char* e = nullptr;
    errno = 0;
    out = std::strtoll(v->text.c_str(), &e, 10);
    return e && *e == '\0' && errno == 0;
}

// The es_metrics counters, in struct order.
const char* const kCounters[] = {"cells_passed",      "impurities_tested",     "particles_inside_impurity",
                                 "particles_escaped", "particles_at_bound",    "max_impurities_tested",
                                 "max_cells_passed",  "crossings_tested",      "start_cell_tests",
                                 "retraced_fp64"};
constexpr int kNumCounters = 10;
static_assert(sizeof(es_metrics) == kNumCounters * sizeof(int64_t), "es_metrics is ten int64 counters");

int64_t* counter(es_metrics& m, int k) { return reinterpret_cast<int64_t*>(&m) + k; }
int64_t counter(const es_metrics& m, int k) { return reinterpret_cast<const int64_t*>(&m)[k]; }

struct Fnv {
    uint64_t h = 1469598103934665603ULL;
    void bytes(const void* p, size_t n)
    {
        const unsigned char* c = static_cast<const unsigned char*>(p);
        for (size_t i = 0; i < n; i++) {
            h ^= c[i];
            h *= 1099511628211ULL;
        }
    }
    void d(double x) { bytes(&x, sizeof x); }
    void i(int64_t x) { bytes(&x, sizeof x); }
};

void put_double(std::string& s, double x)
{
    char buf[40];
    std::snprintf(buf, sizeof buf, "%.17g", x);
    s += buf;
}

}  // namespace

uint64_t Journal::RunKey(const RunConfig& cfg)
{
    Fnv f;
    const char tag[] = "es-journal-1";
    f.bytes(tag, sizeof tag);
    f.i(cfg.positions_per_row);
    f.i(cfg.particles_per_quadrant);
    f.i(cfg.precision);
    f.i(cfg.batched ? 1 : 0);  // the batched sums round differently from the per-pass ones
    const es_settings& s = cfg.settings;
    f.d(s.tau);
    f.d(s.alpha);
    f.i(s.is_clockwise);
    f.d(s.particle_speed);
    f.d(s.region_size);
    f.d(s.region_extends);
    f.d(s.impurity_density);
    f.d(s.impurity_radius);
    f.i(s.target_cell_population);
    f.i((int64_t)cfg.temperatures.size());
    for (double t : cfg.temperatures) f.d(t);
    return f.h;
}

Journal::Key Journal::KeyOf(int sample, unsigned int seed, bool coherent, double field)
{
    uint64_t bits = 0;
    std::memcpy(&bits, &field, sizeof bits);
    return Key(sample, seed, coherent ? 1 : 0, bits);
}

std::string Journal::Format(uint64_t key, const JournalEntry& e)
{
    char head[160];
    std::snprintf(head, sizeof head, "{\"journal\":1,\"run\":\"%016llx\",\"sample\":%d,\"seed\":%u,\"coherent\":%d,\"field\":",
                  (unsigned long long)key, e.sample, e.seed, e.coherent ? 1 : 0);
    std::string s = head;
    put_double(s, e.field);
    s += ",\"sigma\":[";
    for (size_t t = 0; t < e.sigma.size(); t++) {
        s += t ? ",[" : "[";
        put_double(s, e.sigma[t].xx);
        s += ",";
        put_double(s, e.sigma[t].xy);
        s += "]";
    }
    s += "],\"metrics\":{";
    for (int k = 0; k < kNumCounters; k++) {
        s += k ? ",\"" : "\"";
        s += kCounters[k];
        s += "\":" + std::to_string((long long)counter(e.metrics.particle_metrics, k));
    }
    s += "},\"real_particles\":" + std::to_string((long long)e.metrics.real_particles);
    s += ",\"avg_particle_lifetime\":";
    put_double(s, e.metrics.avg_particle_lifetime);
    s += ",\"time_lifetimes\":";
    put_double(s, e.metrics.time_elapsed_lifetimes);
    s += ",\"time_temperatures\":";
    put_double(s, e.metrics.time_elapsed_temperatures);
    s += "}";
    return s;
}

bool Journal::Parse(const std::string& line, uint64_t key, size_t n_temperatures, JournalEntry& out)
{
    Reader r{line.data(), line.data() + line.size()};
    JVal v;
    if (!r.value(v, 0) || v.type != JVal::Obj) return false;
    r.ws();
    if (r.p != r.end) return false;
    long long version = 0, sample = 0, seed = 0, coherent = 0, real = 0;
    if (!as_int(v.get("journal"), version) || version != 1) return false;
    const JVal* run = v.get("run");
    char want[24];
    std::snprintf(want, sizeof want, "%016llx", (unsigned long long)key);
    if (!run || run->type != JVal::Str || run->text != want) return false;
    if (!as_int(v.get("sample"), sample) || !as_int(v.get("seed"), seed) || !as_int(v.get("coherent"), coherent))
        return false;
    if (sample < 0 || seed < 0 || seed > 0xFFFFFFFFLL || (coherent != 0 && coherent != 1)) return false;
    JournalEntry e;
    e.sample = (int)sample;
    e.seed = (unsigned int)seed;
    e.coherent = coherent == 1;
    if (!as_double(v.get("field"), e.field)) return false;
    const JVal* sig = v.get("sigma");
    if (!sig || sig->type != JVal::Arr || sig->items.size() != n_temperatures) return false;
    for (const JVal& pair : sig->items) {
        if (pair.type != JVal::Arr || pair.items.size() != 2) return false;
        Sigma s;
        if (!as_double(&pair.items[0], s.xx) || !as_double(&pair.items[1], s.xy)) return false;
        e.sigma.push_back(s);
    }
    const JVal* m = v.get("metrics");
    if (!m || m->type != JVal::Obj) return false;
    for (int k = 0; k < kNumCounters; k++) {
        long long c = 0;
        if (!as_int(m->get(kCounters[k]), c)) return false;
        *counter(e.metrics.particle_metrics, k) = c;
    }
    if (!as_int(v.get("real_particles"), real)) return false;
    e.metrics.real_particles = real;
    if (!as_double(v.get("avg_particle_lifetime"), e.metrics.avg_particle_lifetime) ||
        !as_double(v.get("time_lifetimes"), e.metrics.time_elapsed_lifetimes) ||
        !as_double(v.get("time_temperatures"), e.metrics.time_elapsed_temperatures))
        return false;
    out = std::move(e);
    return true;
}

Journal::Journal(const std::string& path, const RunConfig& cfg)
    : path_(path), run_(RunKey(cfg)), n_t_(cfg.temperatures.size())
{
    {
        std::ifstream in(path);
        std::string line;
        while (std::getline(in, line)) {
            JournalEntry e;
            if (Parse(line, run_, n_t_, e)) entries_[KeyOf(e.sample, e.seed, e.coherent, e.field)] = e;
        }
    }
    fd_ = ::open(path.c_str(), O_WRONLY | O_APPEND | O_CREAT | O_CLOEXEC, 0644);
    if (fd_ < 0) throw SimulationError("cannot open the journal " + path + ": " + std::strerror(errno));
    // A torn last line (no newline) must not glue onto the next entry.
    std::ifstream tail(path, std::ios::binary | std::ios::ate);
    if (tail && tail.tellg() > 0) {
        tail.seekg(-1, std::ios::end);
        char c = 0;
        tail.get(c);
        if (c != '\n' && ::write(fd_, "\n", 1) != 1)
            throw SimulationError("cannot write the journal " + path + ": " + std::strerror(errno));
    }
}

Journal::~Journal()
{
    if (fd_ >= 0) ::close(fd_);
}

const JournalEntry* Journal::Find(int sample, unsigned int seed, bool coherent, double field) const
{
    auto it = entries_.find(KeyOf(sample, seed, coherent, field));
    return it == entries_.end() ? nullptr : &it->second;
}

void Journal::Append(const JournalEntry& e)
{
    const std::string line = Format(run_, e) + "\n";
    const ssize_t n = ::write(fd_, line.data(), line.size());
    if (n != (ssize_t)line.size())
        throw SimulationError("cannot write the journal " + path_ + ": " + std::strerror(n < 0 ? errno : EIO));
    entries_[KeyOf(e.sample, e.seed, e.coherent, e.field)] = e;
}

}  // namespace es_host
