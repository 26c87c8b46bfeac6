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
// Sigma-only calls (no per-position maps) use integrate_flat_kernel instead:
// the N lifetimes as one flat array, four consecutive orbits per thread step
// (one 32-byte load: 4 * phi_steps phases per position is a multiple of 4, so
// the four share a start position), several steps in flight per thread, and
// the phase table in shared memory. It is bound by HBM on the split path.
//
// Split-precision contexts (fp32 = 1) evaluate GetSigma in FP32 (es_sigma32.cuh:
// cancellation-free form, angles formed and reduced in FP64) and keep every
// sum in FP64: the Simpson integrals in FP32 with FP64 accumulation; the
// plain path keeps the reference's FP64 expression operation by operation.
#include "es_internal.h"
#include "es_sigma32.cuh"

#include <cmath>
#include <cstdint>

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
    const int n_pos = P.rows * P.dim;  // the launch's positions, from row P.row0 on

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
        const double* lts = P.lifetimes + ((long long)P.row0 * P.dim + pidx) * P.n_phase;
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
        const int j = P.row0 + pidx / P.dim;
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

// Phases whose table fits the flat kernel's shared memory beside its reduction
// slots within 48 KB (no opt-in): 16-byte float entries on the split path, the
// 32-byte FP64 table on the plain path. Larger tables take integrate_positions_kernel.
constexpr int kFlatPhasesSplit = 2900;
constexpr int kFlatPhasesFP64 = 1400;

struct PhaseF {
    float c, s, w, pad;  // cos(phi), sin(phi), phase Simpson weight
};

// Stages (b)+(c) over the flat lifetime array ([pos][phase], pos = j*dim + i).
// Thread step g covers orbits 4g..4g+3: four phases of one start position,
// read as two 16-byte loads; the next step's loads are issued before this
// step's arithmetic. Per step
// the four integrands are weighted by their phase weights, summed, weighted by
// the position's w_i * w_j and added to the thread's FP64 sums; the block then
// reduces in a fixed order. The grid size is fixed, so every summation order is
// fixed and results are bit-reproducible.
//
// Split path (kFP32): GetSigma in FP32 in the cancellation-free form of
// es_sigma32.cuh. sin h and cos h (h = w t / 2) come from one FP32 evaluation
// after an FP64 quadrant reduction; sin(phi + h) and cos(phi + h) follow from
// the angle-addition formulas with the phase table's cos(phi), sin(phi). A
// lifetime truncated at 15 tau has h and 1 - exp(-15) fixed per temperature, so
// those are taken once per thread. The four weighted values of a step are
// summed in FP32 before the FP64 accumulation.
// Plain path: the reference's FP64 GetSigma operation by operation, as
// integrate_positions_kernel.
template <int NT, bool kFP32, int kThreads>
__global__ void __launch_bounds__(kThreads, 2) integrate_flat_kernel(IntegrateLaunch P)
{
    extern __shared__ __align__(16) unsigned char s_raw[];
    __shared__ double s_acc[kThreads / 32][NT][2];
    const int n_phase = P.n_phase;
    if (kFP32) {
        PhaseF* tab = reinterpret_cast<PhaseF*>(s_raw);
        for (int v = threadIdx.x; v < n_phase; v += kThreads) {
            const PhaseSigma ph = P.phase[v];
            tab[v] = PhaseF{(float)ph.cos_phi, (float)ph.sin_phi, (float)ph.weight, 0.0f};
        }
    } else {
        PhaseSigma* tab = reinterpret_cast<PhaseSigma*>(s_raw);
        for (int v = threadIdx.x; v < n_phase; v += kThreads) tab[v] = P.phase[v];
    }
    __syncthreads();

    const unsigned dim = (unsigned)P.dim;
    const unsigned row0 = (unsigned)P.row0;
    const unsigned long long n_steps = (unsigned long long)P.rows * dim * (unsigned)n_phase / 4ull;

    // Per-temperature constants are read from the launch parameters (constant
    // bank operands) where they are used, which keeps them out of registers.
    double acc_xx[NT], acc_xy[NT];
#pragma unroll
    for (int k = 0; k < NT; k++) acc_xx[k] = acc_xy[k] = 0.0;

    // one step: four orbits of start position (i, j), phases v0..v0+3
    auto step = [&](unsigned i, unsigned j, unsigned v0, double2 a, double2 b) {
        const double wpos = simpson_weight((int)(row0 + j), (int)dim) * simpson_weight((int)i, (int)dim);
        const double raw4[4] = {a.x, a.y, b.x, b.y};
        if (kFP32) {
            const PhaseF* tab = reinterpret_cast<const PhaseF*>(s_raw);
            float sx[NT], sy[NT];
#pragma unroll
            for (int k = 0; k < NT; k++) sx[k] = sy[k] = 0.0f;
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const double raw = raw4[u];
                const PhaseF ph = tab[v0 + u];
                float sh, ch;
                sincos_reduced_fast(0.5 * P.w_signed * raw, sh, ch);
                const float rawf = (float)raw;
#pragma unroll
                for (int k = 0; k < NT; k++) {
                    const bool keep = raw < P.max_lt[k];
                    const float hs = keep ? sh : P.trunc_sh[k], hc = keep ? ch : P.trunc_ch[k];
                    const float e1 = keep ? one_minus_exp_neg(rawf * P.inv_tau_f[k]) : P.trunc_e1[k];
                    // sin(phi + h), cos(phi + h) by angle addition
                    const float sp = fmaf(ph.s, hc, ph.c * hs);
                    const float cp = fmaf(ph.c, hc, -(ph.s * hs));
                    const float zs = 2.0f * (1.0f - e1) * hs;
                    const float r = fmaf(P.wtau_f[k], fmaf(zs, cp, -e1 * ph.s), fmaf(ph.c, e1, zs * sp));
                    const float rw = r * ph.w;
                    sx[k] = fmaf(rw, ph.c, sx[k]);
                    sy[k] = fmaf(rw, ph.s, sy[k]);
                }
            }
#pragma unroll
            for (int k = 0; k < NT; k++) {
                acc_xx[k] += (double)sx[k] * wpos;
                acc_xy[k] += (double)sy[k] * wpos;
            }
        } else {
            const PhaseSigma* tab = reinterpret_cast<const PhaseSigma*>(s_raw);
            double gx[NT], gy[NT];
#pragma unroll
            for (int k = 0; k < NT; k++) gx[k] = gy[k] = 0.0;
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const double raw = raw4[u];
                const PhaseSigma ph = tab[v0 + u];
                double sa_raw, ca_raw;
                sincos(ph.phi + P.w_signed * raw, &sa_raw, &ca_raw);
#pragma unroll
                for (int k = 0; k < NT; k++) {
                    // GetTruncatedLifetimes: min(raw, 15 tau)
                    const bool keep = raw < P.max_lt[k];
                    const double lt = keep ? raw : P.max_lt[k];
                    double sa = sa_raw, ca = ca_raw;
                    if (!keep) sincos(ph.phi + P.w_signed * lt, &sa, &ca);
                    // GetSigma, src/sim/es/util.h:34-46
                    const double wtau = P.w_signed * P.tau[k];
                    const double z = exp(-lt / P.tau[k]);
                    double r = ph.cos_phi - ca * z;
                    r += wtau * sa * z;
                    r -= wtau * ph.sin_phi;
                    gx[k] += (r * ph.cos_phi) * ph.weight;
                    gy[k] += (r * ph.sin_phi) * ph.weight;
                }
            }
#pragma unroll
            for (int k = 0; k < NT; k++) {
                acc_xx[k] += gx[k] * wpos;
                acc_xy[k] += gy[k] * wpos;
            }
        }
    };

    // The thread's position advances by the grid stride, 4 * stride orbits,
    // written in the mixed radix (j, i, v) of [j][i][phase]: no division in the
    // loop. The stride is below 2^31 orbits and dim, n_phase below 2^31, so
    // the 32-bit sums below do not overflow.
    const unsigned stride = gridDim.x * (unsigned)kThreads;
    const unsigned long long adv = 4ull * stride;
    const unsigned dv = (unsigned)(adv % (unsigned)n_phase);
    const unsigned long long adv_pos = adv / (unsigned)n_phase;
    const unsigned di = (unsigned)(adv_pos % dim);
    const unsigned long long dj = adv_pos / dim;
    unsigned long long g = (unsigned long long)blockIdx.x * kThreads + threadIdx.x;
    // Software pipeline: the next step's 32 bytes are requested before this
    // step's arithmetic, so every thread keeps a load in flight.
    const double2* lt2 = reinterpret_cast<const double2*>(P.lifetimes + (long long)row0 * dim * n_phase);
    if (g < n_steps) {
        const unsigned e0 = (unsigned)(g * 4ull);  // below 4 * stride
        unsigned pidx = e0 / (unsigned)n_phase, v0 = e0 - pidx * (unsigned)n_phase;
        unsigned j = pidx / dim, i = pidx - j * dim;
        double2 a = __ldcs(lt2 + 2 * g), b = __ldcs(lt2 + 2 * g + 1);
        for (;;) {
            const unsigned long long gn = g + stride;
            double2 an = a, bn = b;
            if (gn < n_steps) {
                an = __ldcs(lt2 + 2 * gn);
                bn = __ldcs(lt2 + 2 * gn + 1);
            }
            step(i, j, v0, a, b);
            if (gn >= n_steps) break;
            g = gn;
            a = an;
            b = bn;
            v0 += dv;
            const unsigned cv = v0 >= (unsigned)n_phase ? 1u : 0u;
            v0 -= cv * (unsigned)n_phase;
            i += di + cv;
            const unsigned ci = i >= dim ? 1u : 0u;
            i -= ci * dim;
            j += (unsigned)dj + ci;
        }
    }

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NT; k++) {
        const double sx = warp_sum(acc_xx[k]);
        const double sy = warp_sum(acc_xy[k]);
        if (lane == 0) {
            s_acc[warp][k][0] = sx;
            s_acc[warp][k][1] = sy;
        }
    }
    __syncthreads();
    if (threadIdx.x < 2 * NT) {
        const int k = threadIdx.x >> 1, c = threadIdx.x & 1;
        double sum = 0.0;
        for (int w = 0; w < kThreads / 32; w++) sum += s_acc[w][k][c];
        P.partial[((long long)k * P.n_blocks + blockIdx.x) * 2 + c] = sum;
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
    const bool flat = L.pos_xx == nullptr && (L.n_phase % 4) == 0 &&
                      (reinterpret_cast<uintptr_t>(L.lifetimes + (long long)L.row0 * L.dim * L.n_phase) % 16) == 0 &&
                      L.n_phase <= (L.fp32 ? kFlatPhasesSplit : kFlatPhasesFP64);
    if (flat) {
        // The FP64 integrand (sincos and exp in FP64) bounds the plain path by the
        // FP64 pipe, not by the loads: 256 threads with up to 128 registers.
        // Split path: 384 threads (24 warps per SM at two blocks, up to 85
        // registers) for one or two temperatures, 256 above.
        constexpr int kSplitThreads = NT <= 2 ? 384 : kIntegrateThreads;
        if (L.fp32)
            integrate_flat_kernel<NT, true, kSplitThreads>
                <<<L.n_blocks, kSplitThreads, sizeof(PhaseF) * L.n_phase, s>>>(L);
        else
            integrate_flat_kernel<NT, false, kIntegrateThreads>
                <<<L.n_blocks, kIntegrateThreads, sizeof(PhaseSigma) * L.n_phase, s>>>(L);
        return es::launched(s);
    }
    if (L.fp32) integrate_positions_kernel<NT, true, kThreads><<<L.n_blocks, kThreads, 0, s>>>(L);
    else integrate_positions_kernel<NT, false, kThreads><<<L.n_blocks, kThreads, 0, s>>>(L);
    return es::launched(s);
}

}  // namespace

cudaError_t launch_integrate(const IntegrateLaunch& L0, cudaStream_t s)
{
    IntegrateLaunch L = L0;
    if (L.rows == 0) {
        L.row0 = 0;
        L.rows = L.dim;
    }
    if (L.row0 < 0 || L.rows < 0 || L.row0 + L.rows > L.dim) return cudaErrorInvalidValue;
    for (int k = 0; k < L.n_t && k < kMaxTChunk; k++) {
        const double h = 0.5 * L.w_signed * L.max_lt[k];
        L.inv_tau_f[k] = (float)L.inv_tau[k];
        L.wtau_f[k] = (float)(L.w_signed * L.tau[k]);
        L.trunc_sh[k] = (float)std::sin(h);
        L.trunc_ch[k] = (float)std::cos(h);
        L.trunc_e1[k] = (float)(-std::expm1(-L.max_lt[k] / L.tau[k]));
    }
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
    return es::launched(s);
}

cudaError_t launch_lifetime_sum(const double* lifetimes, long long n, double* partial, double* out, cudaStream_t s)
{
    lifetime_sum_kernel<<<kIntegrateBlocks, 256, 0, s>>>(lifetimes, n, partial);
    cudaError_t e = es::launched(s);
    if (e != cudaSuccess) return e;
    sum_partials_kernel<<<1, 256, 0, s>>>(partial, kIntegrateBlocks, out);
    return es::launched(s);
}

}  // namespace es
