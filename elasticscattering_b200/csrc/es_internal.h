// es_internal.h - launch interfaces shared by the translation units of
// libes_cuda.so. Not part of the public ABI (include/es_cuda.h).
#pragma once

#include <cuda_runtime.h>

#include "es_cuda.h"
#include "es_fault.h"

#include <cstdint>

namespace es {

// Precision modes: the FP32/FP64 split walk (ES_PRECISION_SPLIT and
// ES_PRECISION_SPLIT_EXACT) and the FP32 integrand (ES_PRECISION_SPLIT only).
inline bool split_walk(int precision) { return precision == ES_PRECISION_SPLIT || precision == ES_PRECISION_SPLIT_EXACT; }
inline bool fp32_integrand(int precision) { return precision == ES_PRECISION_SPLIT; }
inline bool precision_known(int precision)
{
    return precision == ES_PRECISION_FP64 || precision == ES_PRECISION_SPLIT || precision == ES_PRECISION_SPLIT_EXACT;
}

// Device-side metric slots (es_metrics order).
enum MetricSlot : int {
    kMetCells = 0,
    kMetImps = 1,
    kMetInside = 2,
    kMetEscaped = 3,
    kMetAtBound = 4,
    kMetMaxImps = 5,
    kMetMaxCells = 6,
    kMetCrossings = 7,
    kMetStartTests = 8,
    kMetRetraced = 9,
    kMetCount = 10
};

// Device error bits (written with atomicOr, read by es_synchronize).
enum DeviceError : int { kErrWalkCap = 1, kErrStartCell = 2, kErrRetraceOverflow = 4 };

// Per-phase constants of one sector, tabulated on the host by es_init_sample
// with the reference's expressions (CreateParticle, src/sim/es/lifetime.h:36-58):
// phi, velocity (cos(phi) * v, sin(phi) * v) from the host libm, and the
// angle to the sector bound (GetBoundTime's dphi, src/sim/es/details.h:219-228;
// unused for the coherent sector, whose bound time is INF). The field-dependent parts
// (orbit-centre shift, bound time = dphi / w) are finished in the kernel with
// the same IEEE operations.
struct PhaseOrbit {
    double phi, vel_x, vel_y, bound_dphi;
};

// Per-phase integration constants (ApplySigma, src/sim/SimulationCPU.cpp:186-192):
// phi, cos(phi), sin(phi) (host libm) and the phase Simpson weight.
struct PhaseSigma {
    double phi, cos_phi, sin_phi, weight;
};

struct LifetimeLaunch {
    const double2* imps;
    const int* cell_end;
    const PhaseOrbit* phase;
    double* out;                  // n_orbits raw lifetimes, [j][i][q][p]
    float* out32;                 // optional FP32 copy (split path), may be null
    unsigned long long* metrics;  // kMetCount slots
    int* error;
    double spawn_start, spawn_size, cell_size, imp_radius;
    double speed, radius, radius_sq, w, dist, off_x, off_y;
    long long n_orbits;
    int cpr, dim, n_phase, clockwise, coherent, walk_cap;
    int row0;                     // first start-position row of this launch
    int variant;                  // LifetimeVariant
    // split precision
    const float2* imps32;         // cell-local FP32 copy of imps
    long long* retrace;           // orbits handed to the FP64 re-trace
    unsigned long long* retrace_count;
    long long retrace_cap;
    // Per-pass orbit table of the split kernels, [n_phase] x {shift_x, shift_y,
    // bound_time, phi}: CreateParticle's per-phase quantities at this pass's
    // radius and w, written by orbit_table_kernel before the lifetime kernel
    // (null: computed per orbit).
    double4* orbit_table;
    // The split walk's FP32 constants of this pass (split_constants in
    // es_host_math.h): as kernel parameters they are constant-bank operands
    // instead of registers.
    float sc_r, sc_inv_r, sc_ir, sc_lo2, sc_hi2, sc_eps2, sc_band_d, sc_inv4r, sc_tangent_tol;
    // ceil(2^64 / n_phase) and ceil(2^64 / dim) (split_constants): the 32-bit
    // quotients of an orbit index by them as one multiply-high each (exact for
    // dividends and divisors below 2^32); 0: divide.
    unsigned long long inv_phase, inv_dim;
    // Test hook (es_debug_finish_retrace): the finish kernel hands the hit of
    // every orbit whose index is a multiple of this to the FP64 re-trace, as it
    // does a NaN finish (0: none).
    int finish_retrace_every;
};

// FP64 lifetime kernel choices (es_tuning.lifetime_variant). The values 1, 3,
// 4 and 5 named variants that measured slower on B200 and were removed (lane
// refill, 19.8 ms against 15.3 ms per 257^2 x 516 pass; lanes over
// neighbouring positions, 55 ms); es_set_tuning rejects them.
enum LifetimeVariant : int {
    kLifetimePerThread = 0,      // one orbit per thread, <= 80 registers (3 blocks of 256 per SM)
    kLifetimePerThreadLean = 2,  // one orbit per thread, <= 64 registers (4 blocks per SM)
    kLifetimePerThreadDefer = 6, // as 2, crossing computations deferred past the cheap tests (default)
};

inline bool lifetime_variant_known(int v)
{
    return v == kLifetimePerThread || v == kLifetimePerThreadLean || v == kLifetimePerThreadDefer;
}

constexpr int kIntegrateBlocks = 296;   // 2 x 148 SMs; fixed so the reduction order is fixed
constexpr int kIntegrateThreads = 256;   // threads per block for 3+ temperatures; 1-2 temperatures use 512
constexpr int kMaxTChunk = 8;           // temperatures integrated per pass over the lifetimes

// One group of up to kMaxTChunk temperatures; all per-temperature constants
// travel by value in the launch, so no device parameter buffers are needed.
struct IntegrateLaunch {
    const double* lifetimes;      // raw lifetimes, [pos][phase]
    const PhaseSigma* phase;
    double tau[kMaxTChunk];       // GetTau per temperature
    double max_lt[kMaxTChunk];    // GetDefaultMaxLifetime = 15 * tau
    double inv_tau[kMaxTChunk];   // 1 / tau (the FP32 kernel)
    double factor[kMaxTChunk];    // GetSigmaIntegrandFactor
    double* pos_lt;               // optional per-position maps [t][pos] (images), may be null
    double* pos_xx;
    double* pos_xy;
    double* partial;              // [t][block][2] block partial sums (xx, xy), scratch
    double* sigma_out;            // [t][2] for this group
    double w_signed;
    double phi_integrand_factor;
    int dim, n_phase, n_t;        // n_t <= kMaxTChunk
    int row0, rows;               // start rows [row0, row0 + rows) of the pass (rows 0: every row)
    int n_blocks;                 // partial blocks per temperature
    int fp32;                     // 1: the FP32 Boltzmann kernel of the split path (es_sigma32.cuh)
    // Filled by launch_integrate from the fields above (FP32 split kernel):
    // 1 / tau and w tau in FP32, and sin h, cos h (h = w 15 tau / 2) and
    // 1 - exp(-15) of a lifetime truncated at 15 tau.
    float inv_tau_f[kMaxTChunk];
    float wtau_f[kMaxTChunk];
    float trunc_sh[kMaxTChunk];
    float trunc_ch[kMaxTChunk];
    float trunc_e1[kMaxTChunk];
};

// Message returned by es_last_error(NULL), for entry points without a context.
void set_global_error(const char* msg);

// The device arrays of a grid built by es_dgrid_create_seeded (es_grid_build.cu).
void dgrid_arrays(const es_dgrid* g, const double2** imps, const int** cell_end, int64_t* n_indexed,
                  es_impurity_settings* is, uint64_t* generation, int* device);

cudaError_t launch_lifetimes_fp64(const LifetimeLaunch& L, cudaStream_t s);
// Split precision: the orbit table, the FP32 walk, then the FP64 re-trace of
// the listed orbits. split_finish (passes with long walks): the walk leaves
// each winner's FP64 time to a finish kernel between walk and re-trace (see
// lifetime_split_kernel); otherwise the walk takes it.
cudaError_t launch_lifetimes_split(const LifetimeLaunch& L, bool split_finish, cudaStream_t s);
cudaError_t launch_local_impurities(const double2* imps, const int* cell_end, float2* out, double start, double cell,
                                    int cpr, cudaStream_t s);
// Stages (b)+(c) for one temperature group: two launches.
cudaError_t launch_integrate(const IntegrateLaunch& L, cudaStream_t s);
// Sum of n raw lifetimes into *out (device), fixed order; partial holds kIntegrateBlocks doubles.
cudaError_t launch_lifetime_sum(const double* lifetimes, long long n, double* partial, double* out, cudaStream_t s);
cudaError_t launch_debug_trace(const LifetimeLaunch& L, const PhaseOrbit& ph, double px, double py, double* d_out,
                               cudaStream_t s);
cudaError_t launch_debug_next_cell(double cx, double cy, double r, int clockwise, double phi, double start,
                                   double size, double cell, int cpr, const double* d_in6, double* d_out6,
                                   int* d_avail, cudaStream_t s);

}  // namespace es
