// es_noalloc.cu - stages (b)+(c) for callers that cannot allocate device memory.
//
// Some callers of this library cannot call cudaMalloc: a host framework that
// owns all device memory through its own pool (or has reserved it all), or a
// caller on a path where the implicit device synchronisation of a driver
// allocation is not allowed. es_derive_temperatures_noalloc serves them: the
// caller passes the lifetimes and the output as device pointers, and the
// scratch the integration needs -- the per-phase table and the per-block
// partial sums -- lives in g_noalloc_scratch below, a fixed array that every
// GPU which loads this library holds until the process exits.
//
// Set-up: the first call in a CUDA context (per device, with that device
// current) looks up the array's device address in that context
// (cudaGetSymbolAddress) and caches it under the context's unique id, so a
// context created later on the same device (after cudaDeviceReset, or a
// caller's own cuCtxCreate context) gets its own lookup. Make the first call
// in each context before any stream capture. Later calls only launch kernels
// on the caller's stream.
#include "es_cuda.h"
#include "es_host_math.h"
#include "es_nvtx.h"
#include "es_internal.h"

#include <cuda.h>

#include <cmath>
#include <cstdio>
#include <mutex>

namespace {

// Stated maximum: phi_steps <= 1025, i.e. 4100 phases.
constexpr int kNoAllocMaxPhiSteps = 1025;
constexpr int kNoAllocMaxPhases = 4 * kNoAllocMaxPhiSteps;
constexpr size_t kPhaseBytes = sizeof(es::PhaseSigma) * kNoAllocMaxPhases;                       // 131,200 B
constexpr size_t kPartialOffset = (kPhaseBytes + 255) / 256 * 256;
constexpr size_t kPartialBytes = sizeof(double) * 2 * es::kMaxTChunk * es::kIntegrateBlocks;     // 37,888 B
constexpr size_t kScratchBytes = kPartialOffset + kPartialBytes;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Device address of g_noalloc_scratch per CUDA context, keyed by the context's
// process-unique id (cuCtxGetId).
struct ScratchEntry {
    unsigned long long ctx_id;
    void* addr;
};
constexpr int kMaxContexts = 64;
std::mutex g_setup_mutex;
ScratchEntry g_scratch[kMaxContexts] = {};
int g_scratch_n = 0;
int g_scratch_next = 0;  // round-robin slot once the table is full

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);
CtxGetCurrentFn g_ctx_get_current = nullptr;
CtxGetIdFn g_ctx_get_id = nullptr;

// Phase table of one sector (ApplySigma, src/sim/SimulationCPU.cpp:186-192),
// written into the scratch array by the device. phi is formed with the host
// table's operations (this file is compiled without contraction); cos and sin
// come from the device libm, so the table can differ from the host-built one
// of es_init_sample in the last bit.
__global__ void noalloc_phase_table_kernel(es::PhaseSigma* table, int ppq, double phi_start, double phi_step)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= 4 * ppq) return;
    const int q = v / ppq, p = v % ppq;
    const double phi = phi_start + q * es::host::kHALF_PI + p * phi_step;
    double s, c;
    sincos(phi, &s, &c);
    const double main_multiplier = (p % 2 == 0) ? 2.0 : 4.0;  // SimpsonWeight, src/sim/es/util.h:24-28
    table[v] = es::PhaseSigma{phi, c, s, (p == 0 || p == ppq - 1) ? 1.0 : main_multiplier};
}

es_status set_error(es_status st, const char* what, cudaError_t e = cudaSuccess)
{
    char msg[256];
    if (e != cudaSuccess) snprintf(msg, sizeof msg, "es_derive_temperatures_noalloc: %s: %s", what, cudaGetErrorString(e));
    else snprintf(msg, sizeof msg, "es_derive_temperatures_noalloc: %s", what);
    es::set_global_error(msg);
    return st;
}

// The unique id of the context current on this thread (binding the current
// device's primary context first if none is current).
es_status current_context_id(unsigned long long* out)
{
    if (!g_ctx_get_current || !g_ctx_get_id) {
        void* f1 = nullptr;
        void* f2 = nullptr;
        cudaDriverEntryPointQueryResult q1 = cudaDriverEntryPointSymbolNotFound, q2 = cudaDriverEntryPointSymbolNotFound;
        cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1);
        if (e == cudaSuccess) e = cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2);
        if (e != cudaSuccess || q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess || !f1 || !f2)
            return set_error(ES_ERR_DEVICE, "driver entry points cuCtxGetCurrent/cuCtxGetId unavailable", e);
        g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(f1);
        g_ctx_get_id = reinterpret_cast<CtxGetIdFn>(f2);
    }
    CUcontext ctx = nullptr;
    if (g_ctx_get_current(&ctx) != CUDA_SUCCESS || !ctx) {
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaSetDevice(dev);  // binds the device's primary context
        if (e != cudaSuccess) return set_error(ES_ERR_DEVICE, "no usable current CUDA device", e);
        if (g_ctx_get_current(&ctx) != CUDA_SUCCESS || !ctx)
            return set_error(ES_ERR_DEVICE, "no current CUDA context");
    }
    if (g_ctx_get_id(ctx, out) != CUDA_SUCCESS) return set_error(ES_ERR_DEVICE, "cuCtxGetId failed");
    return ES_OK;
}

es_status scratch_for_current_context(void** out)
{
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    unsigned long long id = 0;
    es_status st = current_context_id(&id);
    if (st != ES_OK) return st;
    for (int k = 0; k < g_scratch_n; k++) {
        if (g_scratch[k].ctx_id == id) {
            *out = g_scratch[k].addr;
            return ES_OK;
        }
    }
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) return set_error(ES_ERR_DEVICE, "cudaGetSymbolAddress failed", e);
    // A bounded table: beyond kMaxContexts contexts the entries are reused in turn.
    const int slot = g_scratch_n < kMaxContexts ? g_scratch_n++ : (g_scratch_next++ % kMaxContexts);
    g_scratch[slot] = ScratchEntry{id, p};
    *out = p;
    return ES_OK;
}

}  // namespace

extern "C" es_status es_derive_temperatures_noalloc(const double* d_lifetimes, int32_t positions_per_row,
                                                    int32_t phi_steps, const es_settings* s, int32_t coherent,
                                                    double magnetic_field, const double* temperatures, int32_t n_t,
                                                    double* d_out_sigma, void* stream)
{
    es::Range nvtx_range("temperatures_noalloc");
    // Every argument is checked before anything is enqueued: an error return
    // means no work was queued and d_out_sigma is untouched.
    if (!d_lifetimes || !d_out_sigma || !s || (n_t > 0 && !temperatures) || n_t < 0)
        return set_error(ES_ERR_BAD_ARG, "null or negative argument");
    if (positions_per_row < 3 || positions_per_row % 2 == 0 || phi_steps < 3 || phi_steps % 2 == 0)
        return set_error(ES_ERR_BAD_ARG, "positions_per_row and phi_steps must be odd and >= 3");
    if (phi_steps > kNoAllocMaxPhiSteps) {
        char msg[160];
        snprintf(msg, sizeof msg, "phi_steps %d exceeds the fixed scratch maximum of %d", phi_steps,
                 kNoAllocMaxPhiSteps);
        return set_error(ES_ERR_BAD_ARG, msg);
    }
    if (!(magnetic_field > 0.0) || !std::isfinite(magnetic_field) || !(s->particle_speed > 0.0) ||
        (coherent && !(s->tau > 0.0)))
        return set_error(ES_ERR_BAD_ARG, "field, speed and tau must be positive");
    for (int32_t k = 0; k < n_t; k++) {
        if (!coherent && !(temperatures[k] > 0.0)) {
            char msg[160];
            snprintf(msg, sizeof msg, "temperature %d (%g): the incoherent sector needs T > 0", k, temperatures[k]);
            return set_error(ES_ERR_BAD_ARG, msg);
        }
    }
    if (n_t == 0) return ES_OK;
    void* scratch = nullptr;
    es_status st = scratch_for_current_context(&scratch);
    if (st != ES_OK) return st;
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    es::PhaseSigma* table = reinterpret_cast<es::PhaseSigma*>(scratch);
    double* partial = reinterpret_cast<double*>(static_cast<unsigned char*>(scratch) + kPartialOffset);

    // Simulation::InitSample, src/sim/Simulation.h:114-125
    const es::host::Sector sec = es::host::sector(s->alpha, phi_steps, coherent != 0);
    const int n_phase = 4 * phi_steps;
    noalloc_phase_table_kernel<<<(n_phase + 127) / 128, 128, 0, cs>>>(table, phi_steps, sec.phi_start, sec.phi_step);
    cudaError_t e = es::launched(cs);

    // SimulationCPU::ComputeLifetimes, src/sim/SimulationCPU.cpp:107-108
    const double w = es::host::angular_speed(magnetic_field);
    const double w_signed = s->is_clockwise ? -w : w;
    for (int32_t t0 = 0; e == cudaSuccess && t0 < n_t; t0 += es::kMaxTChunk) {
        const int nc = (n_t - t0) < es::kMaxTChunk ? (n_t - t0) : es::kMaxTChunk;
        es::IntegrateLaunch L{};
        L.lifetimes = d_lifetimes;
        L.phase = table;
        for (int k = 0; k < nc; k++) {
            const double tau = es::host::get_tau(coherent != 0, s->tau, temperatures[t0 + k]);
            L.tau[k] = tau;
            L.max_lt[k] = 15.0 * tau;  // GetDefaultMaxLifetime, Simulation.h:91
            L.inv_tau[k] = 1.0 / tau;
            L.factor[k] = es::host::integrand_factor(s->particle_speed, positions_per_row, sec.phi_integrand_factor,
                                                     w, tau);
        }
        L.partial = partial;
        L.sigma_out = d_out_sigma + 2 * t0;
        L.w_signed = w_signed;
        L.phi_integrand_factor = sec.phi_integrand_factor;
        L.dim = positions_per_row;
        L.n_phase = n_phase;
        L.n_t = nc;
        L.n_blocks = es::kIntegrateBlocks;
        e = es::launch_integrate(L, cs);
    }
    if (e != cudaSuccess) return set_error(ES_ERR_LAUNCH, "launch failed", e);
    return ES_OK;
}
