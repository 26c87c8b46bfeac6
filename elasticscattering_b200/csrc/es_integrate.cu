// es_integrate.cu - stages (b) and (c): Simpson integration of the Boltzmann
// kernel over phase angle, then over the start-position grid, in FP64.
//
// Replaces the OpenCL kernels apply_max_lifetime, apply_sigma_component,
// apply_simpson_weights, integrate_to_position and sum
// (src/sim/cl/integration.cl:25-112) and their CPU counterparts
// GetTruncatedLifetimes / ApplySigma / IntegratePosition / IntegrateResult
// (src/sim/Simulation.h:78-86, src/sim/SimulationCPU.cpp:178-243).
//
// The five reference passes (each reading and writing N doubles, twice for xx
// and xy) become one read of the N lifetimes per group of up to kMaxTChunk
// temperatures: a warp owns one start position, its lanes stride over the 4*ppq
// phases, truncate at 15 tau, evaluate GetSigma once per (orbit, T) with one
// sincos per orbit shared by every T that does not truncate, weight by the
// phase Simpson weight and reduce with a fixed shuffle tree. Each block then
// accumulates its positions with the position weights w_i*w_j and writes one
// partial per temperature; a second single-block kernel sums the partials in a
// fixed order and applies GetSigmaIntegrandFactor. Every summation order is
// fixed, so results are bit-reproducible run to run.
//
// Split-precision contexts (fp32 = 1) evaluate GetSigma in FP32 (es_sigma32.cuh:
// cancellation-free form, angles formed and reduced in FP64) and keep every
// sum in FP64, as the north-star split asks of the Simpson integrals; the
// plain path keeps the reference's FP64 expression operation by operation.
#include "es_internal.h"
#include "es_sigma32.cuh"

namespace es {

namespace {

// SimpsonWeight, src/sim/es/util.h:24-28
__device__ __forceinline__ double simpson_weight(int i, int dim)
{
    const double main_multiplier = (i % 2 == 0) ? 2.0 : 4.0;
    const bool is_edge = (i == 0) || i == (dim - 1);
    return is_edge ? 1.0 : main_multiplier;
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    return v;
}

// kThreads: 512 for one or two temperatures (two blocks of 16 warps per SM at
// <= 64 registers: the lifetime loads of 32 warps in flight per SM), 256 above
// (more accumulators per thread).
template <int NT, bool kFP32, int kThreads>
__global__ void __launch_bounds__(kThreads, 2) integrate_positions_kernel(IntegrateLaunch P)
{
    constexpr int kWarps = kThreads / 32;
    __shared__ double s_acc[kWarps][NT][2];

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int n_pos = P.dim * P.dim;

    double tau[NT], max_lt[NT], wtau[NT];
#pragma unroll
    for (int k = 0; k < NT; k++) {
        tau[k] = P.tau[k];
        max_lt[k] = P.max_lt[k];
        wtau[k] = P.w_signed * tau[k];
    }

    double blk_xx[NT], blk_xy[NT];
#pragma unroll
    for (int k = 0; k < NT; k++) blk_xx[k] = blk_xy[k] = 0.0;

    for (int pidx = blockIdx.x * kWarps + warp; pidx < n_pos; pidx += gridDim.x * kWarps) {
        const double* lts = P.lifetimes + (long long)pidx * P.n_phase;
        double acc_xx[NT], acc_xy[NT], acc_lt[NT];
#pragma unroll
        for (int k = 0; k < NT; k++) acc_xx[k] = acc_xy[k] = acc_lt[k] = 0.0;

        for (int v = lane; v < P.n_phase; v += 32) {
            const double raw = __ldg(lts + v);
            const PhaseSigma ph = P.phase[v];
            if (kFP32) {
                const SigmaAngles a_raw = sigma_angles(raw, P.w_signed, ph);
#pragma unroll
                for (int k = 0; k < NT; k++) {
                    const bool keep = raw < max_lt[k];
                    const double lt = keep ? raw : max_lt[k];
                    const SigmaAngles a = keep ? a_raw : sigma_angles(lt, P.w_signed, ph);
                    float r_xx, r_xy;
                    sigma_fp32_at(a, lt, P.inv_tau[k], wtau[k], ph, r_xx, r_xy);
                    acc_xx[k] += (double)r_xx * ph.weight;
                    acc_xy[k] += (double)r_xy * ph.weight;
                    acc_lt[k] += lt * ph.weight;
                }
                continue;
            }
            double sa_raw, ca_raw;
            sincos(ph.phi + P.w_signed * raw, &sa_raw, &ca_raw);
#pragma unroll
            for (int k = 0; k < NT; k++) {
                // GetTruncatedLifetimes: min(raw, 15 tau)
                const bool keep = raw < max_lt[k];
                const double lt = keep ? raw : max_lt[k];
                double sa = sa_raw, ca = ca_raw;
                if (!keep) sincos(ph.phi + P.w_signed * lt, &sa, &ca);
                // GetSigma, src/sim/es/util.h:34-46
                const double z = exp(-lt / tau[k]);
                double r = ph.cos_phi - ca * z;
                r += wtau[k] * sa * z;
                r -= wtau[k] * ph.sin_phi;
                acc_xx[k] += (r * ph.cos_phi) * ph.weight;
                acc_xy[k] += (r * ph.sin_phi) * ph.weight;
                acc_lt[k] += lt * ph.weight;
            }
        }

        const int i = pidx % P.dim;
        const int j = pidx / P.dim;
        const double wpos = simpson_weight(j, P.dim) * simpson_weight(i, P.dim);
#pragma unroll
        for (int k = 0; k < NT; k++) {
            const double sx = warp_sum(acc_xx[k]);
            const double sy = warp_sum(acc_xy[k]);
            blk_xx[k] += sx * wpos;
            blk_xy[k] += sy * wpos;
            if (P.pos_xx != nullptr) {
                const double sl = warp_sum(acc_lt[k]);
                if (lane == 0) {
                    const long long o = (long long)k * n_pos + pidx;
                    P.pos_lt[o] = sl * P.phi_integrand_factor;
                    P.pos_xx[o] = sx * P.phi_integrand_factor;
                    P.pos_xy[o] = sy * P.phi_integrand_factor;
                }
            }
        }
    }

    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < NT; k++) {
            s_acc[warp][k][0] = blk_xx[k];
            s_acc[warp][k][1] = blk_xy[k];
        }
    }
    __syncthreads();
    if (threadIdx.x < 2 * NT) {
        const int k = threadIdx.x >> 1, c = threadIdx.x & 1;
        double s = 0.0;
        for (int w = 0; w < kWarps; w++) s += s_acc[w][k][c];
        P.partial[((long long)k * P.n_blocks + blockIdx.x) * 2 + c] = s;
    }
}

// One block: per temperature and component, a fixed-order tree over the block
// partials, times GetSigmaIntegrandFactor (src/sim/Simulation.h:88).
__global__ void __launch_bounds__(256) reduce_partials_kernel(IntegrateLaunch P)
{
    __shared__ double s_red[256];
    for (int tc = 0; tc < 2 * P.n_t; tc++) {
        const int t = tc >> 1, c = tc & 1;
        double s = 0.0;
        for (int b = threadIdx.x; b < P.n_blocks; b += blockDim.x) s += P.partial[((long long)t * P.n_blocks + b) * 2 + c];
        s_red[threadIdx.x] = s;
        __syncthreads();
        for (int stride = blockDim.x / 2; stride > 0; stride >>= 1) {
            if (threadIdx.x < stride) s_red[threadIdx.x] += s_red[threadIdx.x + stride];
            __syncthreads();
        }
        if (threadIdx.x == 0) P.sigma_out[2 * t + c] = s_red[0] * P.factor[t];
        __syncthreads();
    }
}

// Sum of the raw lifetimes (Simulation::AverageLifetime's numerator,
// src/sim/Simulation.h:93-106): kIntegrateBlocks grid-stride partial sums, then
// one block adds them in a fixed order.
__global__ void __launch_bounds__(256) lifetime_sum_kernel(const double* lt, long long n, double* partial)
{
    __shared__ double s[256];
    double acc = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        acc += lt[i];
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = s[0];
}

__global__ void __launch_bounds__(256) sum_partials_kernel(const double* partial, int n, double* out)
{
    __shared__ double s[256];
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) acc += partial[i];
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = s[0];
}

template <int NT>
cudaError_t launch_group(const IntegrateLaunch& L, cudaStream_t s)
{
    constexpr int kThreads = NT <= 2 ? 2 * kIntegrateThreads : kIntegrateThreads;
    if (L.fp32) integrate_positions_kernel<NT, true, kThreads><<<L.n_blocks, kThreads, 0, s>>>(L);
    else integrate_positions_kernel<NT, false, kThreads><<<L.n_blocks, kThreads, 0, s>>>(L);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_integrate(const IntegrateLaunch& L, cudaStream_t s)
{
    cudaError_t e;
    switch (L.n_t) {
        case 1: e = launch_group<1>(L, s); break;
        case 2: e = launch_group<2>(L, s); break;
        case 3: e = launch_group<3>(L, s); break;
        case 4: e = launch_group<4>(L, s); break;
        case 5: e = launch_group<5>(L, s); break;
        case 6: e = launch_group<6>(L, s); break;
        case 7: e = launch_group<7>(L, s); break;
        case 8: e = launch_group<8>(L, s); break;
        default: return cudaErrorInvalidValue;
    }
    if (e != cudaSuccess) return e;
    reduce_partials_kernel<<<1, 256, 0, s>>>(L);
    return cudaGetLastError();
}

cudaError_t launch_lifetime_sum(const double* lifetimes, long long n, double* partial, double* out, cudaStream_t s)
{
    lifetime_sum_kernel<<<kIntegrateBlocks, 256, 0, s>>>(lifetimes, n, partial);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    sum_partials_kernel<<<1, 256, 0, s>>>(partial, kIntegrateBlocks, out);
    return cudaGetLastError();
}

}  // namespace es
