// es_mlp.cu - the learned surrogate: an ensemble of small MLPs that maps
// (log B, T, log density, impurity radius, log tau) to (sigma_xx, sigma_xy) / sigma_0.
//
// No reference counterpart. Architecture 5 -> 256 x 4 -> 2, GELU, one network per
// ensemble member. BF16 weights and activations, FP32 accumulation, FP32 master
// weights and Adam state. Training and inference are this file's kernels only:
//   - tc_gemm_kernel<TA, TB, EPI>: the three 256 x 256 layers on the
//     5th-generation tensor cores (tcgen05.mma, TMEM accumulators): the forward
//     pass (X W^T + b, GELU), the input gradient (dZ W times GELU'(Z_prev)) and
//     the weight gradient (dZ^T A), with the operands transposed into the
//     K-major shared-memory layout while staging;
//   - input_forward_kernel / input_wgrad_kernel: the 5 -> 256 input layer on the
//     CUDA cores (its K = 5 and N = 5 are below one tensor-core tile);
//   - the 256 -> 2 output head in FP32 on the FP32 master weights and FP32
//     activations, because its 256 terms cancel into a small output and BF16
//     rounding there measurably limited the fit (about 1% error in sigma);
//   - small kernels: minibatch gather, loss gradient, bias gradients, Adam,
//     ensemble mean and spread;
//   - es_mlp_query's kernels: a whole query (features, every layer of every
//     member, sigma, mean and spread) in one CUDA-core kernel for small batches
//     (query_small_kernel, latency first), or the features and the combination
//     around the batched tensor-core pass.
// Every minibatch and reduction order is fixed: training is bit-reproducible.
#include "es_cuda.h"
#include "es_internal.h"

#include <cuda_bf16.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

namespace es {
namespace {

constexpr int kIn = 5, kHidden = 256, kOut = 2, kLayers = 5;  // 4 hidden layers + output
constexpr int kDims[kLayers + 1] = {kIn, kHidden, kHidden, kHidden, kHidden, kOut};

enum Epilogue : int {
    kEpiHidden = 0,  // Z = acc + b (FP32 out), A = GELU(Z) (BF16 out2)
    kEpiDGelu = 2,   // acc * GELU'(Zprev) (BF16 out2)
    kEpiPlain = 3    // acc (FP32 out)
};

struct GemmArgs {
    const __nv_bfloat16* A;
    const __nv_bfloat16* B;
    long long strideA, strideB;  // per ensemble member (elements); 0 = shared
    int lda, ldb;
    int M, N, K;
    const float* bias;  // kEpiHidden
    long long strideBias;
    float* out;  // FP32 [M][N], row stride N
    __nv_bfloat16* out2;  // BF16 [M][N], row stride N
    long long strideOut;
    const float* zprev;  // kEpiDGelu: pre-activations, [M][N]
};

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }

__device__ __forceinline__ float gelu_grad(float x)
{
    const float cdf = 0.5f * (1.0f + erff(x * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * expf(-0.5f * x * x);
    return cdf + x * pdf;
}

// ---- The 5 -> 256 input layer on the CUDA cores ----
//
// K = 5 (forward) and N = 5 (weight gradient) are below one tensor-core tile,
// and the layer is 0.7 % of the network's multiply-adds: plain FP32 FMAs on the
// BF16 operands (exact products), in a fixed order.

// Z = X W0^T + b0 (FP32, written when z is not null) and GELU(Z) (BF16): one
// thread per (row, neuron), the five products summed in k order.
__global__ void input_forward_kernel(const __nv_bfloat16* x, long long stride_x, const __nv_bfloat16* w,
                                     long long stride_w, const float* b, long long stride_b, int M, float* z,
                                     __nv_bfloat16* act, long long stride_out)
{
    const int net = blockIdx.y;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)M * kHidden) return;
    const int m = (int)(i / kHidden), n = (int)(i % kHidden);
    const __nv_bfloat16* xr = x + net * stride_x + (long long)m * kIn;
    const __nv_bfloat16* wr = w + net * stride_w + n * kIn;
    float acc = 0.0f;
#pragma unroll
    for (int k = 0; k < kIn; k++) acc = fmaf(__bfloat162float(xr[k]), __bfloat162float(wr[k]), acc);
    const float zz = acc + b[net * stride_b + n];
    if (z) z[net * stride_out + i] = zz;
    act[net * stride_out + i] = __float2bfloat16(gelu(zz));
}

// dW0[n][k] = sum_m dZ0[m][n] A0[m][k]: block (32 neurons, member), lane = n,
// warp w sums rows w, w + 8, ..., the 8 partials added in warp order.
__global__ void input_wgrad_kernel(const __nv_bfloat16* dz, const __nv_bfloat16* a, int M, int cap, float* gw,
                                   long long stride_p)
{
    __shared__ float s_part[8][32][kIn];
    const int net = blockIdx.y;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n = blockIdx.x * 32 + lane;
    const __nv_bfloat16* d = dz + (long long)net * cap * kHidden;
    const __nv_bfloat16* ar = a + (long long)net * cap * kIn;
    float s[kIn] = {};
    for (int m = warp; m < M; m += 8) {
        const float g = __bfloat162float(d[(long long)m * kHidden + n]);
#pragma unroll
        for (int k = 0; k < kIn; k++) s[k] = fmaf(g, __bfloat162float(ar[(long long)m * kIn + k]), s[k]);
    }
#pragma unroll
    for (int k = 0; k < kIn; k++) s_part[warp][lane][k] = s[k];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < kIn; k++) {
            float t = 0.0f;
            for (int w = 0; w < 8; w++) t += s_part[w][lane][k];
            gw[net * stride_p + n * kIn + k] = t;
        }
    }
}

// ---- Hidden layers 1-3 (K = N = 256) on the 5th-generation tensor cores ----
//
// (The forward pass, as tc_gemm_kernel<false, false, kEpiHidden> below.)
// Z = A W^T + b and GELU(Z) for 128 rows x all 256 columns of
// one member per CTA (grid = row tiles x members, 512 threads), with tcgen05.mma:
//   - the CTA stages its A tile (128 x 256 BF16, 64 KB) and the member's W
//     (256 x 256, 128 KB, L2-resident: every row tile reads it) with 16-byte
//     cp.async copies in shared memory in the no-swizzle K-major layout of
//     the UMMA descriptors: 8-row x 16-byte core matrices of 128 contiguous
//     bytes, the K chunks of a row group adjacent (leading byte offset 128 B),
//     row groups 32 x 128 B apart (stride byte offset 4096 B);
//   - warp 0 allocates 256 TMEM columns (the 128 x 256 FP32 accumulator); one
//     thread issues the 16 MMAs of K = 16 (kind::f16, BF16 in, FP32 out,
//     M = 128, N = 256) and commits them to an mbarrier;
//   - 16 warps read the accumulator back with tcgen05.ld (each warp its lane
//     quarter's rows, a quarter of the columns), add the bias and write Z
//     (FP32; skipped when out is null) and GELU(Z) (BF16) with 16-byte
//     stores; warp 0 frees the TMEM. The GELU epilogue (erff per element) is
//     most of the kernel's instructions, hence the 16 warps.
// The wait on the MMAs is bounded: past its limit the kernel records
// kTcTimeout in *err, waits once more (also bounded) and frees the TMEM, so
// the caller gets an error instead of a hung device.
constexpr int kTcM = 128, kTcN = 256, kTcK = 256;
constexpr int kTcThreads = 512;  // 16 warps: warp w reads TMEM lanes 32 (w % 4).., columns 64 (w / 4)..
constexpr int kTcSmemA = kTcM * kTcK * 2, kTcSmemB = kTcN * kTcK * 2;
constexpr int kTcSmem = kTcSmemA + kTcSmemB;  // 192 KB dynamic shared memory
constexpr int kTcTimeout = 1;
constexpr unsigned kTcWaitLimit = 1u << 24;

// UMMA shared-memory descriptor, no swizzle (layout type 0), version 1 (sm_100).
__device__ __forceinline__ unsigned long long umma_desc(unsigned saddr, unsigned lbo, unsigned sbo)
{
    return (unsigned long long)((saddr >> 4) & 0x3FFFu) | ((unsigned long long)((lbo >> 4) & 0x3FFFu) << 16) |
           ((unsigned long long)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor: FP32 accumulator, BF16 A and B, both K-major, N >> 3, M >> 4.
constexpr unsigned kTcIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(kTcN >> 3) << 17) |
                              ((unsigned)(kTcM >> 4) << 24);

__device__ __forceinline__ bool mbar_try_wait(unsigned addr, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(addr), "r"(parity)
        : "memory");
    return ok != 0;
}

// Stages rows [r0, r0 + R) x reduction [k0, k0 + kTcK) of a GEMM operand X(r, k)
// into the no-swizzle K-major core-matrix layout at sdst (zero outside rows x
// [0, kmax)). !T: X(r, k) = src[r * ld + k], 16-byte cp.async copies (kmax a
// multiple of 8). T: X(r, k) = src[k * ld + r] -- the operand stored with the
// reduction index outermost, as the backward pass reads W (input gradient) and
// dZ and A (weight gradient) -- each thread loads 8 x 8 tiles with 16-byte loads
// along r, transposes them in registers and stores eight 16-byte rows (rows a
// multiple of 8). Returns after issuing (T: after storing); the caller waits
// for the cp.async group and fences before the MMAs read.
template <bool T, int R>
__device__ __forceinline__ void tc_stage(unsigned sdst, const __nv_bfloat16* src, int ld, int r0, int rows, int k0,
                                         int kmax, int tid)
{
    constexpr int kChunks = kTcK / 8;
    if (!T) {
        for (int q = tid; q < R * kChunks; q += kTcThreads) {
            const int r = q / kChunks, kc = q % kChunks;
            const bool in = r0 + r < rows && k0 + kc * 8 < kmax;
            const __nv_bfloat16* p = src + (in ? (long long)(r0 + r) * ld + k0 + kc * 8 : 0);
            const unsigned dst = sdst + ((r >> 3) * kChunks + kc) * 128 + (r & 7) * 16;
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" :: "r"(dst), "l"(p), "r"(in ? 16 : 0)
                         : "memory");
        }
    } else {
        constexpr int kRb = R / 8;
        for (int q = tid; q < kRb * kChunks; q += kTcThreads) {
            const int rb = q % kRb, kb = q / kRb;
            const bool rin = r0 + rb * 8 < rows;
            unsigned short t[8][8];
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const int k = k0 + kb * 8 + u;
                uint4 v = make_uint4(0u, 0u, 0u, 0u);
                if (rin && k < kmax) v = __ldg(reinterpret_cast<const uint4*>(src + (long long)k * ld + r0 + rb * 8));
                const unsigned w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                for (int c = 0; c < 4; c++) {
                    t[u][2 * c] = (unsigned short)(w[c] & 0xFFFFu);
                    t[u][2 * c + 1] = (unsigned short)(w[c] >> 16);
                }
            }
#pragma unroll
            for (int v = 0; v < 8; v++) {  // row rb * 8 + v: its 8 reduction values kb * 8 + 0..7
                const uint4 o = make_uint4((unsigned)t[0][v] | ((unsigned)t[1][v] << 16),
                                           (unsigned)t[2][v] | ((unsigned)t[3][v] << 16),
                                           (unsigned)t[4][v] | ((unsigned)t[5][v] << 16),
                                           (unsigned)t[6][v] | ((unsigned)t[7][v] << 16));
                const unsigned dst = sdst + (rb * kChunks + kb) * 128 + v * 16;
                asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" :: "r"(dst), "r"(o.x), "r"(o.y), "r"(o.z),
                             "r"(o.w) : "memory");
            }
        }
    }
}

// C[m][n] = sum_k A(m, k) B(n, k) for 128 rows x all 256 columns of one member
// per CTA (grid = row tiles x members, 512 threads) with tcgen05.mma, the
// reduction in steps of 256 accumulated in TMEM: the forward pass of the
// 256 x 256 layers (kEpiHidden: Z = C + b and GELU(Z)), the input gradient
// (TB, kEpiDGelu: C * GELU'(Z_prev) to BF16) and the weight gradient (TA, TB,
// kEpiPlain: C in FP32). Per reduction step the CTA stages its A tile (128 x
// 256 BF16, 64 KB) and B (256 x 256, 128 KB) in shared memory, one thread
// issues the 16 MMAs of K = 16 (kind::f16, BF16 in, FP32 out, M = 128, N =
// 256) and commits them to an mbarrier, and every thread waits (bounded) before
// the next step restages; 16 warps then read the accumulator with tcgen05.ld
// (each warp its lane quarter's rows, a quarter of the columns) for the
// epilogue, and warp 0 frees the TMEM. Past a wait's limit the kernel records
// kTcTimeout in *err, issues nothing more, waits once more (also bounded) and
// frees the TMEM, so the caller gets an error instead of a hung device.
template <bool TA, bool TB, int EPI>
__global__ void __launch_bounds__(kTcThreads, 1) tc_gemm_kernel(GemmArgs g, int* err)
{
    extern __shared__ __align__(1024) unsigned char tc_smem[];
    __shared__ __align__(8) unsigned long long mbar;
    __shared__ unsigned tmem_base;
    const int net = blockIdx.y;
    const int m0 = blockIdx.x * kTcM;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const __nv_bfloat16* A = g.A + net * g.strideA;
    const __nv_bfloat16* B = g.B + net * g.strideB;
    const unsigned sA = (unsigned)__cvta_generic_to_shared(tc_smem);
    const unsigned sB = sA + kTcSmemA;
    const unsigned sbar = (unsigned)__cvta_generic_to_shared(&mbar);
    constexpr int kChunks = kTcK / 8;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"((unsigned)__cvta_generic_to_shared(&tmem_base)), "r"(kTcN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(sbar));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    bool done = true;
    const int steps = (g.K + kTcK - 1) / kTcK;
    for (int c = 0; c < steps && done; c++) {
        const int k0 = c * kTcK;
        tc_stage<TA, kTcM>(sA, A, g.lda, m0, g.M, k0, g.K, tid);
        tc_stage<TB, kTcN>(sB, B, g.ldb, 0, g.N, k0, g.K, tid);
        asm volatile("cp.async.commit_group;" ::: "memory");
        asm volatile("cp.async.wait_all;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic-proxy writes -> MMA reads
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (tid == 0) {
            const unsigned tmem = tmem_base;
#pragma unroll 1
            for (int s = 0; s < kTcK / 16; s++) {
                // K step s covers chunks 2s and 2s + 1 of every row group
                const unsigned long long da = umma_desc(sA + 2 * s * 128, 128, kChunks * 128);
                const unsigned long long db = umma_desc(sB + 2 * s * 128, 128, kChunks * 128);
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                    :: "r"(tmem), "l"(da), "l"(db), "r"(kTcIdesc), "r"(c * 16 + s));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         :: "r"(sbar) : "memory");
        }
        bool ok = false;
        for (unsigned it = 0; it < kTcWaitLimit && !ok; it++) ok = mbar_try_wait(sbar, (unsigned)(c & 1));
        if (!ok) {
            atomicOr(err, kTcTimeout);
            for (unsigned it = 0; it < kTcWaitLimit && !ok; it++) ok = mbar_try_wait(sbar, (unsigned)(c & 1));
        }
        // the next step may restage only once every thread saw the MMAs finish
        done = __syncthreads_and(ok ? 1 : 0) != 0;
        if (!ok) done = false;
    }
    done = __all_sync(0xffffffffu, done);  // tcgen05.ld below is warp-collective
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

    if (done) {
        // Warp w may read only TMEM lanes 32 (w % 4) .. + 31: its rows. The four
        // warps of a lane quarter split the 256 columns, 64 each, read 32 at a
        // time; a thread holds 32 columns of its row and writes them with
        // 16-byte stores (Z skipped when out is null).
        const unsigned tmem = tmem_base;
        const int quarter = warp & 3;
        const int col0 = (warp >> 2) * 64;
        const int m = m0 + quarter * 32 + lane;
        float* out = g.out ? g.out + net * g.strideOut : nullptr;
        __nv_bfloat16* out2 = g.out2 ? g.out2 + net * g.strideOut : nullptr;
        const float* bias = EPI == kEpiHidden ? g.bias + net * g.strideBias : nullptr;
        const float* zprev = EPI == kEpiDGelu ? g.zprev + net * g.strideOut : nullptr;
#pragma unroll 1
        for (int c0 = col0; c0 < col0 + 64; c0 += 32) {
            unsigned v[32];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                  "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
                  "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
                  "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                : "r"(tmem + ((unsigned)(quarter * 32) << 16) + (unsigned)c0));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (m < g.M) {
                const long long o = (long long)m * g.N + c0;
#pragma unroll
                for (int j = 0; j < 32; j += 8) {
                    float z[8];
#pragma unroll
                    for (int u = 0; u < 8; u++) z[u] = __uint_as_float(v[j + u]);
                    if (EPI == kEpiHidden) {
#pragma unroll
                        for (int u = 0; u < 8; u++) z[u] += bias[c0 + j + u];
                    }
                    if (EPI == kEpiHidden && out) {
                        *reinterpret_cast<float4*>(out + o + j) = make_float4(z[0], z[1], z[2], z[3]);
                        *reinterpret_cast<float4*>(out + o + j + 4) = make_float4(z[4], z[5], z[6], z[7]);
                    }
                    if (EPI == kEpiPlain) {  // weight gradients: member strides are even, not multiples of 4
#pragma unroll
                        for (int u = 0; u < 8; u += 2)
                            *reinterpret_cast<float2*>(out + o + j + u) = make_float2(z[u], z[u + 1]);
                    }
                    if (EPI == kEpiHidden || EPI == kEpiDGelu) {
                        unsigned h[4];
#pragma unroll
                        for (int u = 0; u < 4; u++) {
                            float a0, a1;
                            if (EPI == kEpiHidden) {
                                a0 = gelu(z[2 * u]);
                                a1 = gelu(z[2 * u + 1]);
                            } else {
                                a0 = z[2 * u] * gelu_grad(zprev[o + j + 2 * u]);
                                a1 = z[2 * u + 1] * gelu_grad(zprev[o + j + 2 * u + 1]);
                            }
                            const __nv_bfloat162 pr = __floats2bfloat162_rn(a0, a1);
                            h[u] = *reinterpret_cast<const unsigned*>(&pr);
                        }
                        *reinterpret_cast<uint4*>(out2 + o + j) = make_uint4(h[0], h[1], h[2], h[3]);
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem_base), "r"(kTcN));
}

namespace {
bool al16(const void* p) { return ((unsigned long long)p & 15ull) == 0; }
}  // namespace

// Whether a GEMM can take the tensor-core kernel: N = 256 output columns, 16-byte
// aligned operand rows and member strides, and the layout each use needs --
// forward (kEpiHidden): A and B K-major, K = 256, lda = ldb = 256;
// input gradient (TB, kEpiDGelu): K = 256, lda = 256, B = W with ldb = 256;
// weight gradient (TA, TB, kEpiPlain): M a multiple of 8, any K (the rows),
// lda = M, ldb = 256, the FP32 output 8-byte aligned (its 8-byte stores).
bool tc_eligible(const GemmArgs& g)
{
    return g.K == kTcK && g.N == kTcN && g.lda == kTcK && g.ldb == kTcK && al16(g.A) && al16(g.B) &&
           (g.strideA * 2) % 16 == 0 && (g.strideB * 2) % 16 == 0 && g.bias && g.out2 && al16(g.out2) &&
           (g.out == nullptr || al16(g.out)) && g.strideOut % 8 == 0;
}

bool tc_eligible_dgelu(const GemmArgs& g)
{
    return g.K == kTcK && g.N == kTcN && g.lda == kTcK && g.ldb == kTcN && al16(g.A) && al16(g.B) &&
           (g.strideA * 2) % 16 == 0 && (g.strideB * 2) % 16 == 0 && g.out2 && al16(g.out2) && g.zprev &&
           g.strideOut % 8 == 0;
}

bool tc_eligible_wgrad(const GemmArgs& g)
{
    return g.N == kTcN && g.M % 8 == 0 && g.lda == g.M && g.ldb == kTcN && g.K >= 1 && al16(g.A) && al16(g.B) &&
           (g.strideA * 2) % 16 == 0 && (g.strideB * 2) % 16 == 0 && g.out &&
           ((unsigned long long)g.out & 7ull) == 0 && g.strideOut % 2 == 0;
}

template <bool TA, bool TB, int EPI>
cudaError_t gemm_tc(const GemmArgs& g, int nets, int* err, cudaStream_t s)
{
    static bool attr_set = false;  // per process and instantiation; the attribute is per function
    if (!attr_set) {
        const cudaError_t e =
            cudaFuncSetAttribute(tc_gemm_kernel<TA, TB, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem);
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    tc_gemm_kernel<TA, TB, EPI><<<dim3((g.M + kTcM - 1) / kTcM, nets), kTcThreads, kTcSmem, s>>>(g, err);
    return cudaGetLastError();
}

cudaError_t gemm_hidden_tc(const GemmArgs& g, int nets, int* err, cudaStream_t s)
{
    return gemm_tc<false, false, kEpiHidden>(g, nets, err, s);
}

// splitmix64: the minibatch index stream (counter-based, reproducible).
__device__ __forceinline__ unsigned long long mix64(unsigned long long z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Minibatch of member `net` at `step`: M rows drawn with replacement from the
// member's bootstrap view of the dataset.
__global__ void gather_kernel(const float* x, const float* y, long long n, int M, int cap, unsigned long long seed,
                              long long step, __nv_bfloat16* xb, float* yb)
{
    const int net = blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= M) return;
    const unsigned long long key = mix64(seed ^ mix64((unsigned long long)step * 0x100000001B3ull + net * 0x9E37ull + i));
    const long long row = (long long)(key % (unsigned long long)n);
#pragma unroll
    for (int k = 0; k < kIn; k++) xb[((long long)net * cap + i) * kIn + k] = __float2bfloat16(x[row * kIn + k]);
#pragma unroll
    for (int k = 0; k < kOut; k++) yb[((long long)net * cap + i) * kOut + k] = y[row * kOut + k];
}

// The output head (256 -> 2) in FP32: out = W4 GELU(Z3) + b4 with the FP32
// master weights and FP32 activations. One warp per row, lanes over the 256
// inputs, fixed shuffle tree.
__global__ void head_forward_kernel(const float* z3, const float* w, const float* b, long long stride_p, int M,
                                    int cap, float* out)
{
    const int net = blockIdx.y;
    const int m = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (m >= M) return;
    const float* z = z3 + ((long long)net * cap + m) * kHidden;
    const float* W = w + net * stride_p;
    float s0 = 0.0f, s1 = 0.0f;
#pragma unroll
    for (int i = 0; i < kHidden / 32; i++) {
        const int k = lane + 32 * i;
        const float a = gelu(z[k]);
        s0 += W[k] * a;
        s1 += W[kHidden + k] * a;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, off);
        s1 += __shfl_xor_sync(0xffffffffu, s1, off);
    }
    if (lane == 0) {
        const float* B = b + net * stride_p;
        out[((long long)net * cap + m) * kOut + 0] = s0 + B[0];
        out[((long long)net * cap + m) * kOut + 1] = s1 + B[1];
    }
}

// Head backward, part 1: dZ3 = (dY W4) * GELU'(Z3), rounded to BF16 for the trunk's GEMMs.
__global__ void head_backward_dz_kernel(const float* dy, const float* z3, const float* w, long long stride_p, int M,
                                        int cap, __nv_bfloat16* dz3)
{
    const int net = blockIdx.y;
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)M * kHidden) return;
    const int m = (int)(e / kHidden), k = (int)(e % kHidden);
    const float* W = w + net * stride_p;
    const long long row = (long long)net * cap + m;
    const float g = dy[row * kOut] * W[k] + dy[row * kOut + 1] * W[kHidden + k];
    dz3[row * kHidden + k] = __float2bfloat16(g * gelu_grad(z3[row * kHidden + k]));
}

// Head backward, part 2: dW4[j][k] = sum_m dY[m][j] GELU(Z3[m][k]) and
// db4[j] = sum_m dY[m][j], one thread per k (and per j for the bias), rows in order.
// Head backward, weights: gw[c][k] = sum_m dY[m][c] GELU(Z3[m][k]) and gb[c] =
// sum_m dY[m][c]. Block (k tile of 32, member): lane = k, warp w sums rows
// w, w + 8, ...; the 8 warp partials are added in warp order. Fixed order: the
// result does not depend on timing.
__global__ void head_backward_w_kernel(const float* dy, const float* z3, int M, int cap, float* gw, float* gb,
                                       long long stride_p)
{
    __shared__ float s_part[8][32][kOut];
    __shared__ float s_bias[8][kOut];
    const int net = blockIdx.y;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int k = blockIdx.x * 32 + lane;
    const float* dyn = dy + (long long)net * cap * kOut;
    const float* zn = z3 + (long long)net * cap * kHidden;
    float s0 = 0.0f, s1 = 0.0f, b0 = 0.0f, b1 = 0.0f;
    for (int m = warp; m < M; m += 8) {
        const float a = gelu(zn[(long long)m * kHidden + k]);
        const float d0 = dyn[(long long)m * kOut], d1 = dyn[(long long)m * kOut + 1];
        s0 += d0 * a;
        s1 += d1 * a;
        b0 += d0;
        b1 += d1;
    }
    s_part[warp][lane][0] = s0;
    s_part[warp][lane][1] = s1;
    if (lane == 0) {
        s_bias[warp][0] = b0;
        s_bias[warp][1] = b1;
    }
    __syncthreads();
    if (warp == 0) {
        float t0 = 0.0f, t1 = 0.0f;
        for (int w = 0; w < 8; w++) {
            t0 += s_part[w][lane][0];
            t1 += s_part[w][lane][1];
        }
        gw[net * stride_p + k] = t0;
        gw[net * stride_p + kHidden + k] = t1;
        if (blockIdx.x == 0 && lane < kOut) {
            float t = 0.0f;
            for (int w = 0; w < 8; w++) t += s_bias[w][lane];
            gb[net * stride_p + lane] = t;
        }
    }
}

// Loss (mean squared error over M x kOut) and its FP32 gradient. One block per
// member; fixed-order tree for the loss.
__global__ void loss_kernel(const float* pred, const float* target, int M, int cap, float* dpred, float* loss)
{
    __shared__ float s[256];
    const int net = blockIdx.x;
    const float scale = 2.0f / (float)(M * kOut);
    float acc = 0.0f;
    for (int e = threadIdx.x; e < M * kOut; e += blockDim.x) {
        const long long o = (long long)net * cap * kOut + e;
        const float d = pred[o] - target[o];
        acc += d * d;
        dpred[o] = scale * d;
    }
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) loss[net] = s[0] / (float)(M * kOut);
}

// db[n] = sum_m dZ[m][n] (BF16 values, FP32 sum in row order).
// Bias gradient db[n] = sum_m dZ[m][n]: block (column tile of 32, member), lane
// = n, warp w sums rows w, w + 8, ..., the 8 partials added in warp order.
__global__ void bias_grad_kernel(const __nv_bfloat16* dz, int M, int cap, int N, float* db, long long stride_db)
{
    __shared__ float s_part[8][32];
    const int net = blockIdx.y;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n = blockIdx.x * 32 + lane;
    const __nv_bfloat16* d = dz + (long long)net * cap * N;
    float s = 0.0f;
    if (n < N)
        for (int m = warp; m < M; m += 8) s += __bfloat162float(d[(long long)m * N + n]);
    s_part[warp][lane] = s;
    __syncthreads();
    if (warp == 0 && n < N) {
        float t = 0.0f;
        for (int w = 0; w < 8; w++) t += s_part[w][lane];
        db[net * stride_db + n] = t;
    }
}

// Adam on the FP32 master parameters; refreshes the BF16 weight copies.
__global__ void adam_kernel(float* p, const float* g, float* m1, float* m2, __nv_bfloat16* w16, const int* is_weight,
                            long long n, float lr, float b1, float b2, float eps, float c1, float c2)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float a = b1 * m1[i] + (1.0f - b1) * gi;
    const float b = b2 * m2[i] + (1.0f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = b;
    const float v = p[i] - lr * (a / c1) / (sqrtf(b / c2) + eps);
    p[i] = v;
    if (is_weight[i] >= 0) w16[is_weight[i]] = __float2bfloat16(v);
}

// Ensemble mean and spread (population standard deviation / |mean|) per query and output.
__global__ void ensemble_kernel(const float* pred, int nets, long long Q, float* mean, float* spread)
{
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= Q * kOut) return;
    float s = 0.0f;
    for (int k = 0; k < nets; k++) s += pred[(long long)k * Q * kOut + e];
    const float mu = s / (float)nets;
    float v = 0.0f;
    for (int k = 0; k < nets; k++) {
        const float d = pred[(long long)k * Q * kOut + e] - mu;
        v += d * d;
    }
    mean[e] = mu;
    spread[e] = sqrtf(v / (float)nets) / fmaxf(fabsf(mu), 1e-30f);
}

__global__ void to_bf16_kernel(const float* x, __nv_bfloat16* y, long long n)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = __float2bfloat16(x[i]);
}

// ---- Whole queries on the device (es_mlp_query) ----------------------------
//
// A query is (B, T, density, impurity radius, tau). Its features are the
// caller's maps, f = 2 (g(v) - g(lo)) / (g(hi) - g(lo)) - 1 with g = log or the
// identity, evaluated in FP64 and rounded to FP32; the members' outputs t are
// turned into sigma = exp(t) sigma_0 (1, w tau) / (1 + (w tau)^2) with
// sigma_0 = sigma0_per_tau * tau and w = w_per_b * B, in FP64; the answer is the
// members' mean and the spread is the largest over the two outputs of their
// standard deviation over |mean|.

struct QueryArgs {
    es_mlp_query_map map;
    const double* q;  // [n][kIn]
    long long n;
    const __nv_bfloat16* w16;
    long long w16_stride;
    long long w16_off[kLayers];
    const float* p;
    long long p_stride;
    long long b_off[kLayers], w_off[kLayers];
    float* t;           // member outputs [nets][n][kOut]
    unsigned* counter;  // per row tile: member blocks done
    double* sigma;      // [n][kOut]
    double* spread;     // [n]
    int nets;
};

__device__ __forceinline__ float query_feature(const es_mlp_query_map& mp, int k, double v)
{
    const double g = mp.log_scale[k] ? log(v) : v;
    return (float)(2.0 * (g - mp.g_lo[k]) / (mp.g_hi[k] - mp.g_lo[k]) - 1.0);
}

__device__ __forceinline__ float bf16_round(float x) { return __bfloat162float(__float2bfloat16(x)); }

// One query row from its members' outputs t(k) = t[k * member_stride + c].
__device__ __forceinline__ void combine_row(const es_mlp_query_map& mp, const double* qrow, const float* t,
                                            long long member_stride, int nets, double* sigma, double* spread)
{
    const double B = qrow[0], tau = qrow[kIn - 1];
    const double wt = mp.w_per_b * B * tau;
    const double d = 1.0 + wt * wt;
    const double s0 = mp.sigma0_per_tau * tau;
    const double shape[kOut] = {1.0 / d, wt / d};
    double worst = 0.0;
    for (int c = 0; c < kOut; c++) {
        double sum = 0.0;
        for (int k = 0; k < nets; k++) sum += exp((double)__ldcg(t + k * member_stride + c)) * s0 * shape[c];
        const double mu = sum / (double)nets;
        double ss = 0.0;
        for (int k = 0; k < nets; k++) {
            const double v = exp((double)__ldcg(t + k * member_stride + c)) * s0 * shape[c] - mu;
            ss += v * v;
        }
        sigma[c] = mu;
        worst = fmax(worst, sqrt(ss / (double)nets) / fmax(fabs(mu), 1e-300));
    }
    *spread = worst;
}

// Small batches, latency first: block (tile, member) runs R query rows through
// every layer of one member on the CUDA cores -- thread j owns neuron j, the
// activations stay in shared memory, rounded to BF16 between layers as on the
// tensor-core path, and the head is head_forward_kernel's warp-per-row sum --
// and the last member block of a tile to finish (a counter, no waiting)
// combines the members. Only the hidden layers' FP32 summation order differs
// from the batched path's.
template <int R>
__global__ void __launch_bounds__(256) query_small_kernel(QueryArgs a)
{
    __shared__ float s_act[2][R][kHidden];
    __shared__ float s_z[R][kHidden];
    __shared__ int s_last;
    const int tile = blockIdx.x, net = blockIdx.y, j = threadIdx.x;
    const long long r0 = (long long)tile * R;
    const int rows = (int)min((long long)R, a.n - r0);
    if (j < R * kIn) {
        const int r = j / kIn, k = j - r * kIn;
        s_act[0][r][k] = r < rows ? bf16_round(query_feature(a.map, k, a.q[(r0 + r) * kIn + k])) : 0.0f;
    }
    __syncthreads();
    const __nv_bfloat16* W16 = a.w16 + net * a.w16_stride;
    const float* P = a.p + net * a.p_stride;
    {  // 5 -> 256
        float acc[R];
#pragma unroll
        for (int r = 0; r < R; r++) acc[r] = 0.0f;
#pragma unroll
        for (int k = 0; k < kIn; k++) {
            const float w = __bfloat162float(W16[a.w16_off[0] + j * kIn + k]);
#pragma unroll
            for (int r = 0; r < R; r++) acc[r] = fmaf(w, s_act[0][r][k], acc[r]);
        }
        const float b = P[a.b_off[0] + j];
#pragma unroll
        for (int r = 0; r < R; r++) s_act[1][r][j] = bf16_round(gelu(acc[r] + b));
    }
    __syncthreads();
    int cur = 1;
    for (int l = 1; l < kLayers - 1; l++) {  // 256 -> 256
        const uint4* wrow = reinterpret_cast<const uint4*>(W16 + a.w16_off[l] + (long long)j * kHidden);
        float acc[R];
#pragma unroll
        for (int r = 0; r < R; r++) acc[r] = 0.0f;
        for (int k8 = 0; k8 < kHidden / 8; k8++) {
            const uint4 wv = __ldg(wrow + k8);
            const __nv_bfloat162* w2 = reinterpret_cast<const __nv_bfloat162*>(&wv);
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const float2 w = __bfloat1622float2(w2[u]);
#pragma unroll
                for (int r = 0; r < R; r++) {
                    acc[r] = fmaf(w.x, s_act[cur][r][k8 * 8 + 2 * u], acc[r]);
                    acc[r] = fmaf(w.y, s_act[cur][r][k8 * 8 + 2 * u + 1], acc[r]);
                }
            }
        }
        const float b = P[a.b_off[l] + j];
        if (l < kLayers - 2) {
#pragma unroll
            for (int r = 0; r < R; r++) s_act[cur ^ 1][r][j] = bf16_round(gelu(acc[r] + b));
        } else {
#pragma unroll
            for (int r = 0; r < R; r++) s_z[r][j] = acc[r] + b;
        }
        cur ^= 1;
        __syncthreads();
    }
    {  // 256 -> 2 in FP32, one warp per row
        const int warp = j >> 5, lane = j & 31;
        const float* W = P + a.w_off[kLayers - 1];
        const float* Bh = P + a.b_off[kLayers - 1];
        for (int r = warp; r < rows; r += 256 / 32) {
            float s0 = 0.0f, s1 = 0.0f;
#pragma unroll
            for (int i = 0; i < kHidden / 32; i++) {
                const int k = lane + 32 * i;
                const float x = gelu(s_z[r][k]);
                s0 += W[k] * x;
                s1 += W[kHidden + k] * x;
            }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                s0 += __shfl_xor_sync(0xffffffffu, s0, off);
                s1 += __shfl_xor_sync(0xffffffffu, s1, off);
            }
            if (lane == 0) {
                float* o = a.t + ((long long)net * a.n + r0 + r) * kOut;
                o[0] = s0 + Bh[0];
                o[1] = s1 + Bh[1];
            }
        }
    }
    __threadfence();
    __syncthreads();
    if (j == 0) s_last = atomicAdd(a.counter + tile, 1u) == (unsigned)(a.nets - 1);
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    if (j < rows)
        combine_row(a.map, a.q + (r0 + j) * kIn, a.t + (r0 + j) * kOut, a.n * kOut, a.nets, a.sigma + (r0 + j) * kOut,
                    a.spread + r0 + j);
}

// Large batches: the features into the shared BF16 input of the batched forward pass.
__global__ void query_features_kernel(es_mlp_query_map mp, const double* q, long long n, __nv_bfloat16* x)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * kIn) return;
    x[i] = __float2bfloat16(query_feature(mp, (int)(i % kIn), q[i]));
}

// Large batches: members' outputs (the head's, [nets][cap][kOut]) to sigma and spread.
__global__ void query_combine_kernel(QueryArgs a, const float* out, long long cap)
{
    const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.n) return;
    for (int k = 0; k < a.nets; k++)
        for (int c = 0; c < kOut; c++) a.t[((long long)k * a.n + r) * kOut + c] = out[((long long)k * cap + r) * kOut + c];
    combine_row(a.map, a.q + r * kIn, out + r * kOut, cap * kOut, a.nets, a.sigma + r * kOut, a.spread + r);
}

}  // namespace
}  // namespace es

// ---------------------------------------------------------------------------
// Host side.

namespace {

// Parameter layout of one member: for each layer l, W_l [N_l][K_l] then b_l [N_l].
struct Layout {
    long long w_off[es::kLayers], b_off[es::kLayers], w16_off[es::kLayers];
    long long n_params = 0, n_weights = 0;
    Layout()
    {
        for (int l = 0; l < es::kLayers; l++) {
            const long long K = es::kDims[l], N = es::kDims[l + 1];
            w_off[l] = n_params;
            w16_off[l] = n_weights;
            n_params += N * K;
            n_weights += N * K;
            b_off[l] = n_params;
            n_params += N;
        }
    }
};

const Layout& layout()
{
    static const Layout L;
    return L;
}

}  // namespace

struct es_mlp {
    int device = 0;
    int nets = 0;
    cudaStream_t stream = nullptr;
    char err[512] = "";
    int64_t launches = 0;
    long long step = 0;
    // parameters (FP32 master, Adam moments, gradients), BF16 weight copies
    float* d_p = nullptr;
    float* d_g = nullptr;
    float* d_m1 = nullptr;
    float* d_m2 = nullptr;
    __nv_bfloat16* d_w16 = nullptr;
    int* d_is_weight = nullptr;  // per parameter: index into w16 (per member) or -1
    // dataset
    float* d_x = nullptr;
    float* d_y = nullptr;
    long long n_data = 0;
    // work buffers for `cap` rows per member
    int cap = 0;
    __nv_bfloat16* d_act[es::kLayers] = {};  // A_l: [nets][cap][K_l]
    float* d_z[es::kLayers] = {};            // Z_l (hidden) / output (last): [nets][cap][N_l]
    __nv_bfloat16* d_dz[es::kLayers] = {};   // dZ_l: [nets][cap][N_l]
    float* d_yb = nullptr;                   // targets [nets][cap][kOut]
    float* d_dy = nullptr;                   // output gradient [nets][cap][kOut], FP32
    float* d_xin = nullptr;                  // query staging [cap][kIn], FP32
    float* d_loss = nullptr;                 // [nets]
    int* d_tc_err = nullptr;                 // tc_gemm_kernel's bounded-wait flag
    int* h_tc_err = nullptr;                 // pinned copy
    float* h_loss = nullptr;                 // pinned
    float* d_mean = nullptr;
    float* d_spread = nullptr;
    // es_mlp_query staging for `qcap` queries: device and pinned host
    long long qcap = 0;
    double* d_q = nullptr;
    float* d_qt = nullptr;       // member outputs [nets][qcap][kOut]
    double* d_qout = nullptr;    // sigma [qcap][kOut], then spread [qcap]
    unsigned* d_qcount = nullptr;  // per row tile of the small-batch kernel
    double* h_q = nullptr;
    double* h_qout = nullptr;
};

namespace {

es_status mfail(es_mlp* m, es_status st, const char* fmt, const char* what = "")
{
    snprintf(m->err, sizeof m->err, fmt, what);
    return st;
}

#define ES_MCUDA(call, what)                                                                              \
    do {                                                                                                  \
        cudaError_t e_ = (call);                                                                          \
        if (e_ != cudaSuccess) {                                                                          \
            snprintf(m->err, sizeof m->err, "%s: %s", what, cudaGetErrorString(e_));                      \
            return e_ == cudaErrorMemoryAllocation ? ES_ERR_OOM : ES_ERR_LAUNCH;                          \
        }                                                                                                 \
    } while (0)

void free_work(es_mlp* m)
{
    for (int l = 0; l < es::kLayers; l++) {
        cudaFree(m->d_act[l]);
        cudaFree(m->d_z[l]);
        cudaFree(m->d_dz[l]);
        m->d_act[l] = nullptr;
        m->d_z[l] = nullptr;
        m->d_dz[l] = nullptr;
    }
    cudaFree(m->d_yb);
    cudaFree(m->d_dy);
    cudaFree(m->d_xin);
    cudaFree(m->d_mean);
    cudaFree(m->d_spread);
    m->d_yb = m->d_dy = m->d_xin = m->d_mean = m->d_spread = nullptr;
    m->cap = 0;
}

es_status ensure_rows(es_mlp* m, long long rows)
{
    if (rows <= m->cap) return ES_OK;
    if (rows > 4000000) return mfail(m, ES_ERR_BAD_ARG, "at most 4,000,000 rows per call");
    free_work(m);
    const long long E = m->nets;
    for (int l = 0; l < es::kLayers; l++) {
        const long long K = es::kDims[l], N = es::kDims[l + 1];
        ES_MCUDA(cudaMalloc(&m->d_act[l], sizeof(__nv_bfloat16) * E * rows * K), "activations");
        ES_MCUDA(cudaMalloc(&m->d_z[l], sizeof(float) * E * rows * N), "pre-activations");
        ES_MCUDA(cudaMalloc(&m->d_dz[l], sizeof(__nv_bfloat16) * E * rows * N), "gradients");
    }
    ES_MCUDA(cudaMalloc(&m->d_yb, sizeof(float) * E * rows * es::kOut), "targets");
    ES_MCUDA(cudaMalloc(&m->d_dy, sizeof(float) * E * rows * es::kOut), "output gradient");
    ES_MCUDA(cudaMalloc(&m->d_xin, sizeof(float) * rows * es::kIn), "query staging");
    ES_MCUDA(cudaMalloc(&m->d_mean, sizeof(float) * rows * es::kOut), "ensemble mean");
    ES_MCUDA(cudaMalloc(&m->d_spread, sizeof(float) * rows * es::kOut), "ensemble spread");
    m->cap = (int)rows;
    return ES_OK;
}

void free_query(es_mlp* m)
{
    cudaFree(m->d_q);
    cudaFree(m->d_qt);
    cudaFree(m->d_qout);
    cudaFree(m->d_qcount);
    if (m->h_q) cudaFreeHost(m->h_q);
    if (m->h_qout) cudaFreeHost(m->h_qout);
    m->d_q = m->h_q = m->d_qout = m->h_qout = nullptr;
    m->d_qt = nullptr;
    m->d_qcount = nullptr;
    m->qcap = 0;
}

constexpr long long kSmallQuery = 256;  // es_mlp_query's CUDA-core kernel up to here
constexpr int kQueryRows = 8;           // query rows per block of that kernel

es_status ensure_query(es_mlp* m, long long n)
{
    if (n <= m->qcap) return ES_OK;
    if (n > 4000000) return mfail(m, ES_ERR_BAD_ARG, "at most 4,000,000 queries per call");
    free_query(m);
    long long cap = 256;
    while (cap < n) cap *= 2;
    const long long tiles = (kSmallQuery + kQueryRows - 1) / kQueryRows;
    ES_MCUDA(cudaMalloc(&m->d_q, sizeof(double) * cap * es::kIn), "query staging");
    ES_MCUDA(cudaMalloc(&m->d_qt, sizeof(float) * m->nets * cap * es::kOut), "member outputs");
    ES_MCUDA(cudaMalloc(&m->d_qout, sizeof(double) * cap * (es::kOut + 1)), "query answers");
    ES_MCUDA(cudaMalloc(&m->d_qcount, sizeof(unsigned) * tiles), "query counters");
    ES_MCUDA(cudaMallocHost(&m->h_q, sizeof(double) * cap * es::kIn), "query staging (host)");
    ES_MCUDA(cudaMallocHost(&m->h_qout, sizeof(double) * cap * (es::kOut + 1)), "query answers (host)");
    m->qcap = cap;
    return ES_OK;
}

es::GemmArgs args0() { return es::GemmArgs{}; }

// Forward pass of every member on rows already staged in d_act[0] (BF16
// [nets][rows][kIn], or [rows][kIn] shared when shared_input).
// keep_z: write every hidden layer's pre-activation Z (FP32), which the
// backward pass reads; a query pass (false) writes only the last one, the
// head's input.
cudaError_t forward(es_mlp* m, int rows, bool shared_input, bool keep_z)
{
    const Layout& L = layout();
    const long long P = L.n_params, W = L.n_weights;
    cudaError_t e = cudaSuccess;
    // the BF16 trunk on the tensor cores
    for (int l = 0; l + 1 < es::kLayers && e == cudaSuccess; l++) {
        const int K = es::kDims[l], N = es::kDims[l + 1];
        es::GemmArgs g = args0();
        g.A = m->d_act[l];
        g.strideA = (l == 0 && shared_input) ? 0 : (long long)m->cap * K;
        g.lda = K;
        g.B = m->d_w16 + L.w16_off[l];
        g.strideB = W;
        g.ldb = K;
        g.M = rows;
        g.N = N;
        g.K = K;
        g.bias = m->d_p + L.b_off[l];
        g.strideBias = P;
        g.strideOut = (long long)m->cap * N;
        g.out2 = m->d_act[l + 1];
        g.out = m->d_z[l];
        if (!keep_z && l + 2 < es::kLayers) g.out = nullptr;  // Z only where the backward pass or the head reads it
        if (l == 0) {
            const long long n = (long long)rows * N;
            es::input_forward_kernel<<<dim3((unsigned)((n + 255) / 256), m->nets), 256, 0, m->stream>>>(
                g.A, g.strideA, g.B, g.strideB, g.bias, g.strideBias, rows, g.out, g.out2, g.strideOut);
            e = cudaGetLastError();
        } else if (es::tc_eligible(g)) {
            e = es::gemm_hidden_tc(g, m->nets, m->d_tc_err, m->stream);
        } else {
            e = cudaErrorInvalidValue;  // every 256 x 256 layer meets the tensor-core kernel's layout
        }
        m->launches++;
    }
    // the FP32 head
    if (e == cudaSuccess) {
        const int last = es::kLayers - 1;
        es::head_forward_kernel<<<dim3((rows + 7) / 8, m->nets), 256, 0, m->stream>>>(
            m->d_z[last - 1], m->d_p + L.w_off[last], m->d_p + L.b_off[last], P, rows, m->cap, m->d_z[last]);
        m->launches++;
        e = cudaGetLastError();
    }
    return e;
}

// Backward pass from the FP32 output gradient in d_dy: the head in FP32, then
// the trunk's weight and bias gradients into d_g.
cudaError_t backward(es_mlp* m, int rows)
{
    const Layout& L = layout();
    const long long P = L.n_params, W = L.n_weights;
    cudaError_t e = cudaSuccess;
    {
        const int last = es::kLayers - 1;
        es::head_backward_w_kernel<<<dim3(es::kHidden / 32, m->nets), 256, 0, m->stream>>>(
            m->d_dy, m->d_z[last - 1], rows, m->cap, m->d_g + L.w_off[last], m->d_g + L.b_off[last], P);
        m->launches++;
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        const long long n = (long long)rows * es::kHidden;
        es::head_backward_dz_kernel<<<dim3((unsigned)((n + 255) / 256), m->nets), 256, 0, m->stream>>>(
            m->d_dy, m->d_z[last - 1], m->d_p + L.w_off[last], P, rows, m->cap, m->d_dz[last - 1]);
        m->launches++;
        e = cudaGetLastError();
    }
    for (int l = es::kLayers - 2; l >= 0 && e == cudaSuccess; l--) {
        const int K = es::kDims[l], N = es::kDims[l + 1];
        // dW_l[n][k] = sum_m dZ_l[m][n] A_l[m][k]
        es::GemmArgs gw = args0();
        gw.A = m->d_dz[l];
        gw.strideA = (long long)m->cap * N;
        gw.lda = N;
        gw.B = m->d_act[l];
        gw.strideB = (long long)m->cap * K;
        gw.ldb = K;
        gw.M = N;
        gw.N = K;
        gw.K = rows;
        gw.out = m->d_g + L.w_off[l];
        gw.strideOut = P;
        // out[n * K + k] with row stride = gw.N = K
        if (l == 0) {
            es::input_wgrad_kernel<<<dim3(es::kHidden / 32, m->nets), 256, 0, m->stream>>>(
                m->d_dz[0], m->d_act[0], rows, m->cap, m->d_g + L.w_off[0], P);
            e = cudaGetLastError();
        } else if (es::tc_eligible_wgrad(gw)) {
            e = es::gemm_tc<true, true, es::kEpiPlain>(gw, m->nets, m->d_tc_err, m->stream);
        } else {
            e = cudaErrorInvalidValue;
        }
        m->launches++;
        if (e != cudaSuccess) break;
        es::bias_grad_kernel<<<dim3((N + 31) / 32, m->nets), 256, 0, m->stream>>>(m->d_dz[l], rows, m->cap, N,
                                                                                     m->d_g + L.b_off[l], P);
        m->launches++;
        if ((e = cudaGetLastError()) != cudaSuccess) break;
        if (l == 0) break;
        // dZ_{l-1}[m][k] = (sum_n dZ_l[m][n] W_l[n][k]) * GELU'(Z_{l-1}[m][k])
        es::GemmArgs gx = args0();
        gx.A = m->d_dz[l];
        gx.strideA = (long long)m->cap * N;
        gx.lda = N;
        gx.B = m->d_w16 + L.w16_off[l];
        gx.strideB = W;
        gx.ldb = K;
        gx.M = rows;
        gx.N = K;
        gx.K = N;
        gx.out2 = m->d_dz[l - 1];
        gx.strideOut = (long long)m->cap * K;
        gx.zprev = m->d_z[l - 1];
        if (es::tc_eligible_dgelu(gx)) e = es::gemm_tc<false, true, es::kEpiDGelu>(gx, m->nets, m->d_tc_err, m->stream);
        else e = cudaErrorInvalidValue;
        m->launches++;
    }
    return e;
}

// The tensor-core kernel's flag (read back with the caller's synchronisation):
// a bounded wait ran out, so that call's outputs are not valid.
es_status check_tc(es_mlp* m)
{
    if (*m->h_tc_err == 0) return ES_OK;
    *m->h_tc_err = 0;
    cudaMemsetAsync(m->d_tc_err, 0, sizeof(int), m->stream);
    return mfail(m, ES_ERR_TIMEOUT, "tensor-core GEMM: the wait for the MMAs ran out");
}

es_status bind_mlp(es_mlp* m)
{
    if (!m) return ES_ERR_BAD_ARG;
    ES_MCUDA(cudaSetDevice(m->device), "cudaSetDevice");
    return ES_OK;
}

// Loss and gradients on the staged minibatch (d_act[0], d_yb).
es_status loss_and_grads(es_mlp* m, int rows)
{
    cudaError_t e = forward(m, rows, false, true);
    if (e == cudaSuccess) {
        es::loss_kernel<<<m->nets, 256, 0, m->stream>>>(m->d_z[es::kLayers - 1], m->d_yb, rows, m->cap, m->d_dy,
                                                        m->d_loss);
        m->launches++;
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = backward(m, rows);
    ES_MCUDA(e, "surrogate training step");
    return ES_OK;
}

}  // namespace

extern "C" {

int64_t es_mlp_param_count(void) { return layout().n_params; }

es_status es_mlp_create(int32_t n_nets, int32_t device_ordinal, es_mlp** out)
{
    if (!out || n_nets < 1 || n_nets > 64) return ES_ERR_BAD_ARG;
    *out = nullptr;
    int n_dev = 0;
    if (cudaGetDeviceCount(&n_dev) != cudaSuccess || device_ordinal < 0 || device_ordinal >= n_dev) {
        es::set_global_error("es_mlp_create: no such CUDA device");
        return ES_ERR_DEVICE;
    }
    es_mlp* m = new (std::nothrow) es_mlp();
    if (!m) return ES_ERR_OOM;
    m->device = device_ordinal;
    m->nets = n_nets;
    const Layout& L = layout();
    const long long P = L.n_params * n_nets, W = L.n_weights * n_nets;
    std::vector<int> is_w((size_t)P, -1);
    for (int k = 0; k < n_nets; k++)
        for (int l = 0; l < es::kLayers; l++) {
            const long long nk = (long long)es::kDims[l] * es::kDims[l + 1];
            for (long long i = 0; i < nk; i++)
                is_w[(size_t)(k * L.n_params + L.w_off[l] + i)] = (int)(k * L.n_weights + L.w16_off[l] + i);
        }
    cudaError_t e = cudaSetDevice(device_ordinal);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&m->d_p, sizeof(float) * P);
    if (e == cudaSuccess) e = cudaMalloc(&m->d_g, sizeof(float) * P);
    if (e == cudaSuccess) e = cudaMalloc(&m->d_m1, sizeof(float) * P);
    if (e == cudaSuccess) e = cudaMalloc(&m->d_m2, sizeof(float) * P);
    if (e == cudaSuccess) e = cudaMalloc(&m->d_w16, sizeof(__nv_bfloat16) * W);
    if (e == cudaSuccess) e = cudaMalloc(&m->d_is_weight, sizeof(int) * P);
    if (e == cudaSuccess) e = cudaMalloc(&m->d_loss, sizeof(float) * n_nets);
    if (e == cudaSuccess) e = cudaMalloc(&m->d_tc_err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(m->d_tc_err, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaMallocHost(&m->h_tc_err, sizeof(int));
    if (e == cudaSuccess) e = cudaMallocHost(&m->h_loss, sizeof(float) * n_nets);
    if (e == cudaSuccess)
        e = cudaMemcpy(m->d_is_weight, is_w.data(), sizeof(int) * P, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(m->d_p, 0, sizeof(float) * P);
    if (e == cudaSuccess) e = cudaMemset(m->d_m1, 0, sizeof(float) * P);
    if (e == cudaSuccess) e = cudaMemset(m->d_m2, 0, sizeof(float) * P);
    if (e == cudaSuccess) e = cudaMemset(m->d_w16, 0, sizeof(__nv_bfloat16) * W);
    if (e != cudaSuccess) {
        char msg[256];
        snprintf(msg, sizeof msg, "es_mlp_create: %s", cudaGetErrorString(e));
        es::set_global_error(msg);
        es_mlp_destroy(m);
        return e == cudaErrorMemoryAllocation ? ES_ERR_OOM : ES_ERR_LAUNCH;
    }
    *out = m;
    return ES_OK;
}

es_status es_mlp_destroy(es_mlp* m)
{
    if (!m) return ES_ERR_BAD_ARG;
    cudaSetDevice(m->device);
    if (m->stream) cudaStreamSynchronize(m->stream);
    free_work(m);
    free_query(m);
    cudaFree(m->d_p);
    cudaFree(m->d_g);
    cudaFree(m->d_m1);
    cudaFree(m->d_m2);
    cudaFree(m->d_w16);
    cudaFree(m->d_is_weight);
    cudaFree(m->d_x);
    cudaFree(m->d_y);
    cudaFree(m->d_loss);
    cudaFree(m->d_tc_err);
    cudaFreeHost(m->h_tc_err);
    if (m->h_loss) cudaFreeHost(m->h_loss);
    if (m->stream) cudaStreamDestroy(m->stream);
    delete m;
    return ES_OK;
}

const char* es_mlp_last_error(const es_mlp* m) { return m ? m->err : es_last_error(nullptr); }

es_status es_mlp_set_params(es_mlp* m, const float* params)
{
    es_status st = bind_mlp(m);
    if (st != ES_OK) return st;
    if (!params) return mfail(m, ES_ERR_BAD_ARG, "null parameters");
    const Layout& L = layout();
    const long long P = L.n_params * m->nets;
    ES_MCUDA(cudaMemcpyAsync(m->d_p, params, sizeof(float) * P, cudaMemcpyHostToDevice, m->stream), "parameter upload");
    ES_MCUDA(cudaMemsetAsync(m->d_m1, 0, sizeof(float) * P, m->stream), "Adam state");
    ES_MCUDA(cudaMemsetAsync(m->d_m2, 0, sizeof(float) * P, m->stream), "Adam state");
    for (int k = 0; k < m->nets; k++)
        for (int l = 0; l < es::kLayers; l++) {
            const long long nk = (long long)es::kDims[l] * es::kDims[l + 1];
            es::to_bf16_kernel<<<(unsigned)((nk + 255) / 256), 256, 0, m->stream>>>(
                m->d_p + k * L.n_params + L.w_off[l], m->d_w16 + k * L.n_weights + L.w16_off[l], nk);
            m->launches++;
        }
    ES_MCUDA(cudaGetLastError(), "weight conversion");
    ES_MCUDA(cudaStreamSynchronize(m->stream), "parameter upload");
    m->step = 0;
    return ES_OK;
}

es_status es_mlp_get_params(es_mlp* m, float* params)
{
    es_status st = bind_mlp(m);
    if (st != ES_OK) return st;
    if (!params) return mfail(m, ES_ERR_BAD_ARG, "null parameters");
    ES_MCUDA(cudaMemcpyAsync(params, m->d_p, sizeof(float) * layout().n_params * m->nets, cudaMemcpyDeviceToHost,
                             m->stream),
             "parameter readback");
    ES_MCUDA(cudaStreamSynchronize(m->stream), "parameter readback");
    return ES_OK;
}

es_status es_mlp_set_dataset(es_mlp* m, const float* x, const float* y, int64_t n)
{
    es_status st = bind_mlp(m);
    if (st != ES_OK) return st;
    if (!x || !y || n < 1) return mfail(m, ES_ERR_BAD_ARG, "empty dataset");
    cudaFree(m->d_x);
    cudaFree(m->d_y);
    m->d_x = m->d_y = nullptr;
    m->n_data = 0;
    ES_MCUDA(cudaMalloc(&m->d_x, sizeof(float) * n * es::kIn), "dataset");
    ES_MCUDA(cudaMalloc(&m->d_y, sizeof(float) * n * es::kOut), "dataset");
    ES_MCUDA(cudaMemcpyAsync(m->d_x, x, sizeof(float) * n * es::kIn, cudaMemcpyHostToDevice, m->stream), "dataset");
    ES_MCUDA(cudaMemcpyAsync(m->d_y, y, sizeof(float) * n * es::kOut, cudaMemcpyHostToDevice, m->stream), "dataset");
    ES_MCUDA(cudaStreamSynchronize(m->stream), "dataset");
    m->n_data = n;
    return ES_OK;
}

es_status es_mlp_train(es_mlp* m, int32_t steps, int32_t batch, float lr, uint64_t seed, float* out_loss)
{
    es_status st = bind_mlp(m);
    if (st != ES_OK) return st;
    if (m->n_data < 1) return mfail(m, ES_ERR_BAD_ARG, "es_mlp_set_dataset has not been called");
    if (steps < 0 || batch < 1 || batch > 65536 || !(lr > 0.0f))
        return mfail(m, ES_ERR_BAD_ARG, "bad training arguments");
    if ((st = ensure_rows(m, batch)) != ES_OK) return st;
    const Layout& L = layout();
    const long long P = L.n_params * m->nets;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int s = 0; s < steps; s++) {
        es::gather_kernel<<<dim3((batch + 255) / 256, m->nets), 256, 0, m->stream>>>(
            m->d_x, m->d_y, m->n_data, batch, m->cap, seed, m->step, m->d_act[0], m->d_yb);
        m->launches++;
        ES_MCUDA(cudaGetLastError(), "minibatch gather");
        if ((st = loss_and_grads(m, batch)) != ES_OK) return st;
        m->step++;
        const float c1 = 1.0f - std::pow(b1, (float)m->step), c2 = 1.0f - std::pow(b2, (float)m->step);
        es::adam_kernel<<<(unsigned)((P + 255) / 256), 256, 0, m->stream>>>(m->d_p, m->d_g, m->d_m1, m->d_m2, m->d_w16,
                                                                           m->d_is_weight, P, lr, b1, b2, eps, c1, c2);
        m->launches++;
        ES_MCUDA(cudaGetLastError(), "Adam update");
    }
    if (out_loss) {
        ES_MCUDA(cudaMemcpyAsync(m->h_loss, m->d_loss, sizeof(float) * m->nets, cudaMemcpyDeviceToHost, m->stream),
                 "loss readback");
    }
    ES_MCUDA(cudaMemcpyAsync(m->h_tc_err, m->d_tc_err, sizeof(int), cudaMemcpyDeviceToHost, m->stream), "flag readback");
    ES_MCUDA(cudaStreamSynchronize(m->stream), "training");
    if ((st = check_tc(m)) != ES_OK) return st;
    if (out_loss) std::memcpy(out_loss, m->h_loss, sizeof(float) * m->nets);
    return ES_OK;
}

es_status es_mlp_gradients(es_mlp* m, const float* x, const float* y, int32_t rows, float* out_grads, float* out_loss)
{
    es_status st = bind_mlp(m);
    if (st != ES_OK) return st;
    if (!x || !y || !out_grads || rows < 1) return mfail(m, ES_ERR_BAD_ARG, "bad gradient arguments");
    if ((st = ensure_rows(m, rows)) != ES_OK) return st;
    // x: [nets][rows][kIn] FP32 (rounded to BF16 here), y: [nets][rows][kOut]
    float* d_tmp = nullptr;
    const long long nx = (long long)m->nets * rows * es::kIn;
    ES_MCUDA(cudaMalloc(&d_tmp, sizeof(float) * nx), "gradient input");
    cudaError_t e = cudaMemcpyAsync(d_tmp, x, sizeof(float) * nx, cudaMemcpyHostToDevice, m->stream);
    if (e == cudaSuccess) {
        // rows are packed with stride `rows`; the work buffers use stride `cap`
        for (int k = 0; k < m->nets && e == cudaSuccess; k++) {
            es::to_bf16_kernel<<<(unsigned)((rows * es::kIn + 255) / 256), 256, 0, m->stream>>>(
                d_tmp + (long long)k * rows * es::kIn, m->d_act[0] + (long long)k * m->cap * es::kIn,
                (long long)rows * es::kIn);
            m->launches++;
            e = cudaGetLastError();
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(m->d_yb + (long long)k * m->cap * es::kOut, y + (long long)k * rows * es::kOut,
                                    sizeof(float) * rows * es::kOut, cudaMemcpyHostToDevice, m->stream);
        }
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
    cudaFree(d_tmp);
    ES_MCUDA(e, "gradient inputs");
    if ((st = loss_and_grads(m, rows)) != ES_OK) return st;
    ES_MCUDA(cudaMemcpyAsync(out_grads, m->d_g, sizeof(float) * layout().n_params * m->nets, cudaMemcpyDeviceToHost,
                             m->stream),
             "gradient readback");
    ES_MCUDA(cudaMemcpyAsync(m->h_loss, m->d_loss, sizeof(float) * m->nets, cudaMemcpyDeviceToHost, m->stream),
             "loss readback");
    ES_MCUDA(cudaMemcpyAsync(m->h_tc_err, m->d_tc_err, sizeof(int), cudaMemcpyDeviceToHost, m->stream), "flag readback");
    ES_MCUDA(cudaStreamSynchronize(m->stream), "gradients");
    if ((st = check_tc(m)) != ES_OK) return st;
    if (out_loss) std::memcpy(out_loss, m->h_loss, sizeof(float) * m->nets);
    return ES_OK;
}

es_status es_mlp_predict(es_mlp* m, const float* x, int64_t q, float* out_each, float* out_mean, float* out_spread)
{
    es_status st = bind_mlp(m);
    if (st != ES_OK) return st;
    if (!x || q < 1) return mfail(m, ES_ERR_BAD_ARG, "bad query arguments");
    if ((st = ensure_rows(m, q)) != ES_OK) return st;
    cudaError_t e = cudaMemcpyAsync(m->d_xin, x, sizeof(float) * q * es::kIn, cudaMemcpyHostToDevice, m->stream);
    if (e == cudaSuccess) {
        es::to_bf16_kernel<<<(unsigned)((q * es::kIn + 255) / 256), 256, 0, m->stream>>>(m->d_xin, m->d_act[0],
                                                                                         q * es::kIn);
        m->launches++;
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = forward(m, (int)q, true, false);
    if (e == cudaSuccess) {
        // outputs of member k are at d_z[last] + k * cap * kOut; pack them with stride q
        if (m->cap != q) {
            for (int k = 0; k < m->nets && e == cudaSuccess; k++)
                e = cudaMemcpyAsync(m->d_yb + (long long)k * q * es::kOut,
                                    m->d_z[es::kLayers - 1] + (long long)k * m->cap * es::kOut,
                                    sizeof(float) * q * es::kOut, cudaMemcpyDeviceToDevice, m->stream);
        } else {
            e = cudaMemcpyAsync(m->d_yb, m->d_z[es::kLayers - 1], sizeof(float) * m->nets * q * es::kOut,
                                cudaMemcpyDeviceToDevice, m->stream);
        }
    }
    if (e == cudaSuccess) {
        es::ensemble_kernel<<<(unsigned)((q * es::kOut + 255) / 256), 256, 0, m->stream>>>(m->d_yb, m->nets, q,
                                                                                           m->d_mean, m->d_spread);
        m->launches++;
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && out_each)
        e = cudaMemcpyAsync(out_each, m->d_yb, sizeof(float) * m->nets * q * es::kOut, cudaMemcpyDeviceToHost,
                            m->stream);
    if (e == cudaSuccess && out_mean)
        e = cudaMemcpyAsync(out_mean, m->d_mean, sizeof(float) * q * es::kOut, cudaMemcpyDeviceToHost, m->stream);
    if (e == cudaSuccess && out_spread)
        e = cudaMemcpyAsync(out_spread, m->d_spread, sizeof(float) * q * es::kOut, cudaMemcpyDeviceToHost, m->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(m->h_tc_err, m->d_tc_err, sizeof(int), cudaMemcpyDeviceToHost, m->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
    ES_MCUDA(e, "surrogate query");
    return check_tc(m);
}

es_status es_mlp_query(es_mlp* m, const es_mlp_query_map* map, const double* q, int64_t n, double* out_sigma,
                       double* out_spread, float* out_each)
{
    es_status st = bind_mlp(m);
    if (st != ES_OK) return st;
    if (!map || !q || n < 1) return mfail(m, ES_ERR_BAD_ARG, "es_mlp_query: null or empty argument");
    for (int k = 0; k < es::kIn; k++)
        if (!(map->g_hi[k] != map->g_lo[k]) || !std::isfinite(map->g_hi[k]) || !std::isfinite(map->g_lo[k]))
            return mfail(m, ES_ERR_BAD_ARG, "es_mlp_query: feature map needs finite g_lo != g_hi");
    for (int64_t i = 0; i < n; i++)
        for (int k = 0; k < es::kIn; k++) {
            const double v = q[i * es::kIn + k];
            if (!std::isfinite(v) || (map->log_scale[k] && !(v > 0.0)))
                return mfail(m, ES_ERR_BAD_ARG, "es_mlp_query: a query value is not finite (or not > 0 on a log feature)");
        }
    if ((st = ensure_query(m, n)) != ES_OK) return st;
    const Layout& L = layout();
    es::QueryArgs a{};
    a.map = *map;
    a.q = m->d_q;
    a.n = n;
    a.w16 = m->d_w16;
    a.w16_stride = L.n_weights;
    a.p = m->d_p;
    a.p_stride = L.n_params;
    for (int l = 0; l < es::kLayers; l++) {
        a.w16_off[l] = L.w16_off[l];
        a.b_off[l] = L.b_off[l];
        a.w_off[l] = L.w_off[l];
    }
    a.t = m->d_qt;
    a.counter = m->d_qcount;
    a.sigma = m->d_qout;
    a.spread = m->d_qout + n * es::kOut;
    a.nets = m->nets;
    std::memcpy(m->h_q, q, sizeof(double) * n * es::kIn);
    cudaError_t e = cudaMemcpyAsync(m->d_q, m->h_q, sizeof(double) * n * es::kIn, cudaMemcpyHostToDevice, m->stream);
    if (n <= kSmallQuery) {
        const unsigned tiles = (unsigned)((n + kQueryRows - 1) / kQueryRows);
        if (e == cudaSuccess) e = cudaMemsetAsync(m->d_qcount, 0, sizeof(unsigned) * tiles, m->stream);
        if (e == cudaSuccess) {
            if (n == 1) es::query_small_kernel<1><<<dim3(1, m->nets), 256, 0, m->stream>>>(a);
            else es::query_small_kernel<kQueryRows><<<dim3(tiles, m->nets), 256, 0, m->stream>>>(a);
            m->launches++;
            e = cudaGetLastError();
        }
    } else {
        if ((st = ensure_rows(m, n)) != ES_OK) return st;
        if (e == cudaSuccess) {
            es::query_features_kernel<<<(unsigned)((n * es::kIn + 255) / 256), 256, 0, m->stream>>>(
                a.map, m->d_q, n, m->d_act[0]);
            m->launches++;
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = forward(m, (int)n, true, false);
        if (e == cudaSuccess) {
            es::query_combine_kernel<<<(unsigned)((n + 255) / 256), 256, 0, m->stream>>>(
                a, m->d_z[es::kLayers - 1], m->cap);
            m->launches++;
            e = cudaGetLastError();
        }
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(m->h_qout, m->d_qout, sizeof(double) * n * (es::kOut + 1), cudaMemcpyDeviceToHost,
                            m->stream);
    if (e == cudaSuccess && out_each)
        e = cudaMemcpyAsync(out_each, m->d_qt, sizeof(float) * m->nets * n * es::kOut, cudaMemcpyDeviceToHost,
                            m->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(m->h_tc_err, m->d_tc_err, sizeof(int), cudaMemcpyDeviceToHost, m->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
    ES_MCUDA(e, "surrogate query");
    if ((st = check_tc(m)) != ES_OK) return st;
    if (out_sigma) std::memcpy(out_sigma, m->h_qout, sizeof(double) * n * es::kOut);
    if (out_spread) std::memcpy(out_spread, m->h_qout + n * es::kOut, sizeof(double) * n);
    return ES_OK;
}

int64_t es_mlp_launch_count(const es_mlp* m) { return m ? m->launches : 0; }

void* es_mlp_stream(es_mlp* m) { return m ? (void*)m->stream : nullptr; }

}  // extern "C"
