// es_fault.cu - the armed fault-injection plan and its C ABI
// (es_fault_inject, es_fault_counts; include/es_cuda.h). No reference
// counterpart: the reference prints and exits on every error
// (src/utils/ErrorMacros.h:22-38) and has no way to provoke one.
#include "es_fault.h"

#include <atomic>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "es_cuda.h"
#include "es_internal.h"

namespace {

struct Rule {
    es::fault::Kind kind;
    int64_t nth;       // 1-based index among operations of `kind`
    bool and_later;    // "kind:n+": the n-th and every later one
};

std::mutex g_mu;
std::vector<Rule> g_rules;
std::atomic<bool> g_armed{false};
std::atomic<int64_t> g_count[es::fault::kKinds];
std::atomic<int64_t> g_fired{0};
std::once_flag g_env_once;

bool parse(const char* spec, std::vector<Rule>& out)
{
    out.clear();
    if (!spec) return true;
    std::string s(spec);
    size_t at = 0;
    while (at < s.size()) {
        size_t end = s.find(',', at);
        if (end == std::string::npos) end = s.size();
        std::string item = s.substr(at, end - at);
        at = end + 1;
        while (!item.empty() && item.front() == ' ') item.erase(item.begin());
        while (!item.empty() && item.back() == ' ') item.pop_back();
        if (item.empty()) continue;
        const size_t colon = item.find(':');
        if (colon == std::string::npos) return false;
        const std::string kind = item.substr(0, colon);
        std::string num = item.substr(colon + 1);
        Rule r{};
        if (kind == "alloc") r.kind = es::fault::kAlloc;
        else if (kind == "copy") r.kind = es::fault::kCopy;
        else if (kind == "launch") r.kind = es::fault::kLaunch;
        else return false;
        r.and_later = !num.empty() && num.back() == '+';
        if (r.and_later) num.pop_back();
        if (num.empty() || num.size() > 15) return false;
        for (char c : num)
            if (c < '0' || c > '9') return false;
        r.nth = std::strtoll(num.c_str(), nullptr, 10);
        if (r.nth < 1) return false;
        out.push_back(r);
    }
    return true;
}

void arm(std::vector<Rule>&& rules)
{
    std::lock_guard<std::mutex> lock(g_mu);
    g_rules = std::move(rules);
    for (auto& c : g_count) c.store(0);
    g_fired.store(0);
    g_armed.store(!g_rules.empty());
}

void read_env()
{
    std::vector<Rule> rules;
    const char* spec = std::getenv("ES_FAULT_INJECT");
    if (spec && parse(spec, rules)) arm(std::move(rules));
}

}  // namespace

bool es::fault::fire(Kind kind)
{
    std::call_once(g_env_once, read_env);
    const int64_t n = g_count[kind].fetch_add(1) + 1;
    if (!g_armed.load(std::memory_order_acquire)) return false;
    std::lock_guard<std::mutex> lock(g_mu);
    for (const Rule& r : g_rules)
        if (r.kind == kind && (n == r.nth || (r.and_later && n > r.nth))) {
            g_fired.fetch_add(1);
            return true;
        }
    return false;
}

cudaError_t es::fault::after(Kind kind, cudaStream_t s)
{
    if (!fire(kind)) return cudaSuccess;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (s != nullptr) cudaStreamIsCapturing(s, &cap);
    if (cap == cudaStreamCaptureStatusNone) {
        // the operation completes before its failure is reported
        if (s != nullptr) cudaStreamSynchronize(s);
        else cudaDeviceSynchronize();
    }
    return kind == kLaunch ? cudaErrorLaunchFailure : cudaErrorUnknown;
}

extern "C" {

es_status es_fault_inject(const char* spec)
{
    std::call_once(g_env_once, [] {});  // an explicit plan replaces the environment's
    std::vector<Rule> rules;
    if (!parse(spec, rules)) {
        es::set_global_error("es_fault_inject: expected comma-separated alloc|copy|launch:N[+] items");
        return ES_ERR_BAD_ARG;
    }
    arm(std::move(rules));
    return ES_OK;
}

es_status es_fault_counts(int64_t* out_counts)
{
    if (!out_counts) return ES_ERR_BAD_ARG;
    for (int k = 0; k < es::fault::kKinds; k++) out_counts[k] = g_count[k].load();
    out_counts[es::fault::kKinds] = g_fired.load();
    return ES_OK;
}

}  // extern "C"
