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
// Set-up: the first call on a device, with that device current, looks up the
// array's device address (cudaGetSymbolAddress) and caches it; make that first
// call before any stream capture. Later calls only launch kernels on the
// caller's stream.
#include "es_cuda.h"
#include "es_internal.h"

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

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void* g_scratch_addr[kMaxDevices] = {};

// src/sim/es/constants.h:23-32
constexpr double kM0 = 9.10938188e-31;
constexpr double kM = (5.0 * kM0);
constexpr double kE = 1.60217646e-19;
constexpr double kHBAR = 1.05457148e-34;
constexpr double kC1 = 1.15e-9;
constexpr double kKB = 1.380649e-23;
constexpr double kPI = 3.141592653589793238463;
constexpr double kHALF_PI = 1.570796326794896619231;

// Phase table of one sector (ApplySigma, src/sim/SimulationCPU.cpp:186-192),
// written into the scratch array by the device.
__global__ void noalloc_phase_table_kernel(es::PhaseSigma* table, int ppq, double phi_start, double phi_step)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= 4 * ppq) return;
    const int q = v / ppq, p = v % ppq;
    const double phi = phi_start + q * kHALF_PI + p * phi_step;
    double s, c;
    sincos(phi, &s, &c);
    const double main_multiplier = (p % 2 == 0) ? 2.0 : 4.0;  // SimpsonWeight, src/sim/es/util.h:24-28
    table[v] = es::PhaseSigma{phi, c, s, (p == 0 || p == ppq - 1) ? 1.0 : main_multiplier};
}

es_status scratch_for_current_device(void** out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        es::set_global_error("es_derive_temperatures_noalloc: no usable current CUDA device");
        return ES_ERR_DEVICE;
    }
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            char msg[256];
            snprintf(msg, sizeof msg, "es_derive_temperatures_noalloc: cudaGetSymbolAddress failed: %s",
                     cudaGetErrorString(e));
            es::set_global_error(msg);
            return ES_ERR_DEVICE;
        }
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return ES_OK;
}

}  // namespace

extern "C" es_status es_derive_temperatures_noalloc(const double* d_lifetimes, int32_t positions_per_row,
                                                    int32_t phi_steps, const es_settings* s, int32_t coherent,
                                                    double magnetic_field, const double* temperatures, int32_t n_t,
                                                    double* d_out_sigma, void* stream)
{
    if (!d_lifetimes || !d_out_sigma || !s || (n_t > 0 && !temperatures) || n_t < 0) {
        es::set_global_error("es_derive_temperatures_noalloc: null or negative argument");
        return ES_ERR_BAD_ARG;
    }
    if (positions_per_row < 3 || positions_per_row % 2 == 0 || phi_steps < 3 || phi_steps % 2 == 0) {
        es::set_global_error("es_derive_temperatures_noalloc: positions_per_row and phi_steps must be odd and >= 3");
        return ES_ERR_BAD_ARG;
    }
    if (phi_steps > kNoAllocMaxPhiSteps) {
        char msg[160];
        snprintf(msg, sizeof msg, "es_derive_temperatures_noalloc: phi_steps %d exceeds the fixed scratch maximum of %d",
                 phi_steps, kNoAllocMaxPhiSteps);
        es::set_global_error(msg);
        return ES_ERR_BAD_ARG;
    }
    if (!(magnetic_field > 0.0) || !(s->particle_speed > 0.0) || (coherent && !(s->tau > 0.0))) {
        es::set_global_error("es_derive_temperatures_noalloc: field, speed and tau must be positive");
        return ES_ERR_BAD_ARG;
    }
    void* scratch = nullptr;
    es_status st = scratch_for_current_device(&scratch);
    if (st != ES_OK) return st;
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    es::PhaseSigma* table = reinterpret_cast<es::PhaseSigma*>(scratch);
    double* partial = reinterpret_cast<double*>(static_cast<unsigned char*>(scratch) + kPartialOffset);

    // Simulation::InitSample, src/sim/Simulation.h:114-125
    const double base_area = s->alpha * 2.0;
    const double area = !coherent ? base_area : (kHALF_PI - base_area);
    const double phi_integrand_factor = area / ((phi_steps - 1) * 3.0);
    const double phi_start = !coherent ? -s->alpha : s->alpha;
    const double phi_step = area / (phi_steps - 1);
    const int n_phase = 4 * phi_steps;
    noalloc_phase_table_kernel<<<(n_phase + 127) / 128, 128, 0, cs>>>(table, phi_steps, phi_start, phi_step);
    cudaError_t e = cudaGetLastError();

    // SimulationCPU::ComputeLifetimes, src/sim/SimulationCPU.cpp:107-108
    const double w = kE * magnetic_field / kM;
    const double w_signed = s->is_clockwise ? -w : w;
    // SigmaFactor / GetSigmaIntegrandFactor, src/sim/Simulation.h:69-76,88
    const double kf = kM * s->particle_speed / kHBAR;
    const double outside0 = (kE * kE * kf * kf) / (2.0 * kPI * kPI * kM * kC1);
    const double pos_w = std::pow(1.0 / (3.0 * (positions_per_row - 1)), 2);
    for (int32_t t0 = 0; e == cudaSuccess && t0 < n_t; t0 += es::kMaxTChunk) {
        const int nc = (n_t - t0) < es::kMaxTChunk ? (n_t - t0) : es::kMaxTChunk;
        es::IntegrateLaunch L{};
        L.lifetimes = d_lifetimes;
        L.phase = table;
        for (int k = 0; k < nc; k++) {
            const double T = temperatures[t0 + k];
            if (!coherent && !(T > 0.0)) {
                es::set_global_error("es_derive_temperatures_noalloc: the incoherent sector needs T > 0");
                return ES_ERR_BAD_ARG;
            }
            const double tau = coherent ? s->tau : kHBAR / (kKB * T);  // GetTau, Simulation.h:90
            const double wct = w * tau;
            double outside = outside0;
            outside *= tau / (1.0 + wct * wct);
            L.tau[k] = tau;
            L.max_lt[k] = 15.0 * tau;
            L.factor[k] = pos_w * phi_integrand_factor * outside * 1e-8;
        }
        L.partial = partial;
        L.sigma_out = d_out_sigma + 2 * t0;
        L.w_signed = w_signed;
        L.phi_integrand_factor = phi_integrand_factor;
        L.dim = positions_per_row;
        L.n_phase = n_phase;
        L.n_t = nc;
        L.n_blocks = es::kIntegrateBlocks;
        e = es::launch_integrate(L, cs);
    }
    if (e != cudaSuccess) {
        char msg[256];
        snprintf(msg, sizeof msg, "es_derive_temperatures_noalloc: launch failed: %s", cudaGetErrorString(e));
        es::set_global_error(msg);
        return ES_ERR_LAUNCH;
    }
    return ES_OK;
}
