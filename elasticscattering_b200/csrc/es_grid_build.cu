// es_grid_build.cu - the seeded impurity grid built on the GPU
// (reference: Grid::Grid(seed, ...), GenerateImpurities, GenerateImpurityCells
// and ConvertToIndex, src/sim/Grid.cpp:28-110 and :112-188).
//
// The result is the host Grid's, bit for bit: the same impurity positions and
// the same cell-major ordered array and cumulative cell index.
//
// 1. Positions. The reference draws x then y per impurity from
//    std::uniform_real_distribution<double> over std::default_random_engine,
//    which libstdc++ defines as minstd_rand0 (x <- 16807 x mod 2^31 - 1).
//    Each double is std::generate_canonical<double, 53>: two draws u1, u2,
//    sum = (u1 - 1) + (u2 - 1) r with r = 2^31 - 2, divided by r^2 (rounded to
//    double), then mapped to [a, b) as c (b - a) + a. Impurity i consumes draws
//    4i+1 .. 4i+4, so each thread jumps straight to its draws with
//    16807^(4i) mod (2^31 - 1) and needs no sequential pass. Compiled with
//    -fmad=false, every operation rounds as the host's.
// 2. Cells. add_to_overlapping_cells files an impurity under up to 9 cells
//    (the unique in-grid cells of 5 probes, then the diagonal neighbours whose
//    shared corner lies inside the disk). The reference keeps one vector per
//    cell, filled in impurity order, and concatenates them row-major. Here: a
//    count kernel (atomics), an exclusive scan, a placement kernel (atomic
//    cursors: any order within a cell), then one warp per cell ranks its
//    entries by impurity index and writes the positions in that order -- the
//    stable order the reference produces.
#include <algorithm>
#include <cmath>
#include <cstdio>

#include "es_cuda.h"
#include "es_nvtx.h"
#include "es_internal.h"

struct es_dgrid {
    int device = 0;
    double2* d_imps = nullptr;   // ordered (cell-major) impurities, n_indexed
    int* d_cell_end = nullptr;   // cumulative ends, cells_per_row^2
    int64_t n_indexed = 0;
    int64_t n_unique = 0;
    es_impurity_settings is{};
    uint64_t generation = 0;
};

namespace es {

namespace {

constexpr unsigned long long kMinstdM = 2147483647ULL;  // 2^31 - 1
constexpr unsigned long long kMinstdA = 16807ULL;

// a b mod (2^31 - 1) for a, b < 2^31, by folding the 62-bit product.
__device__ __forceinline__ unsigned long long mulmod_m31(unsigned long long a, unsigned long long b)
{
    unsigned long long p = a * b;
    p = (p & kMinstdM) + (p >> 31);
    p = (p & kMinstdM) + (p >> 31);
    return p >= kMinstdM ? p - kMinstdM : p;
}

__device__ __forceinline__ unsigned long long powmod_m31(unsigned long long base, unsigned long long e)
{
    unsigned long long r = 1;
    while (e) {
        if (e & 1ULL) r = mulmod_m31(r, base);
        base = mulmod_m31(base, base);
        e >>= 1;
    }
    return r;
}

// std::generate_canonical<double, 53> over minstd_rand0 (min 1, max 2^31 - 2).
__device__ __forceinline__ double canonical53(unsigned long long& x)
{
    const double r = 2147483646.0;
    x = mulmod_m31(x, kMinstdA);
    double sum = 0.0 + (double)(x - 1ULL) * 1.0;
    x = mulmod_m31(x, kMinstdA);
    sum = sum + (double)(x - 1ULL) * r;
    const double tmp = r * r;
    double ret = sum / tmp;
    if (ret >= 1.0) ret = 0x1.fffffffffffffp-1;  // nextafter(1, 0)
    return ret;
}

__global__ void generate_kernel(unsigned long long x0, long long n, double a, double b, double2* out)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        unsigned long long x = mulmod_m31(x0, powmod_m31(kMinstdA, 4ULL * (unsigned long long)i));
        const double cx = canonical53(x);
        const double cy = canonical53(x);
        out[i] = make_double2((cx * (b - a)) + a, (cy * (b - a)) + a);
    }
}

struct Geo {
    double lo, size, cell_size;
    int cpr;
};

// Grid::get_cell (src/sim/Grid.cpp:182-188): truncation toward zero.
__device__ __forceinline__ int2 geo_cell(const Geo& g, double x, double y)
{
    return make_int2((int)((x - g.lo) / g.size * (double)g.cpr), (int)((y - g.lo) / g.size * (double)g.cpr));
}

__device__ __forceinline__ bool geo_within(const Geo& g, int2 c) { return c.x >= 0 && c.x < g.cpr && c.y >= 0 && c.y < g.cpr; }

// The cells add_to_overlapping_cells (src/sim/Grid.cpp:112-180) files one
// impurity under; returns how many (at most 9).
__device__ int overlapping_cells(const Geo& g, double2 p, double r, int* out)
{
    int2 pr[5];
    pr[0] = geo_cell(g, p.x, p.y);
    pr[1] = geo_cell(g, p.x + r, p.y);
    pr[2] = geo_cell(g, p.x - r, p.y);
    pr[3] = geo_cell(g, p.x, p.y + r);
    pr[4] = geo_cell(g, p.x, p.y - r);
    int n = 0;
#pragma unroll
    for (int i = 0; i < 5; i++) {
        bool seen = false;
#pragma unroll
        for (int k = 0; k < i; k++) seen |= (pr[k].x == pr[i].x && pr[k].y == pr[i].y && geo_within(g, pr[k]));
        if (!seen && geo_within(g, pr[i])) out[n++] = pr[i].y * g.cpr + pr[i].x;
    }
    // Grid::to_world uses spawn_range.x for both axes (src/sim/Grid.h:48-51);
    // corners in the order top-left, top-right, low-left, low-right.
    const double llx = g.lo + pr[0].x * g.cell_size, lly = g.lo + pr[0].y * g.cell_size;
    const double cxs[4] = {0 + llx, g.cell_size + llx, llx, g.cell_size + llx};
    const double cys[4] = {g.cell_size + lly, g.cell_size + lly, lly, 0 + lly};
    const int ox[4] = {-1, 1, -1, 1}, oy[4] = {1, 1, -1, -1};
    const double ir2 = r * r;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const double dx = cxs[k] - p.x, dy = cys[k] - p.y;
        const int2 nc = make_int2(pr[0].x + ox[k], pr[0].y + oy[k]);
        if (dx * dx + dy * dy < ir2 && geo_within(g, nc)) out[n++] = nc.y * g.cpr + nc.x;
    }
    return n;
}

__global__ void count_kernel(const double2* pos, long long n, Geo g, double r, unsigned int* count)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        int cells[9];
        const int k = overlapping_cells(g, pos[i], r, cells);
        for (int c = 0; c < k; c++) atomicAdd(count + cells[c], 1u);
    }
}

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

// Block-wide exclusive scan of a per-thread value; returns the block total.
__device__ unsigned long long block_exclusive_scan(unsigned long long v, unsigned long long& excl)
{
    __shared__ unsigned long long s_warp[kScanThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long inc = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const unsigned long long t = __shfl_up_sync(0xffffffffu, inc, off);
        if (lane >= off) inc += t;
    }
    if (lane == 31) s_warp[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        unsigned long long w = lane < kScanThreads / 32 ? s_warp[lane] : 0ULL;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const unsigned long long t = __shfl_up_sync(0xffffffffu, w, off);
            if (lane >= off) w += t;
        }
        if (lane < kScanThreads / 32) s_warp[lane] = w;  // inclusive over warps
    }
    __syncthreads();
    const unsigned long long warp_base = warp == 0 ? 0ULL : s_warp[warp - 1];
    excl = warp_base + inc - v;
    const unsigned long long total = s_warp[kScanThreads / 32 - 1];
    __syncthreads();
    return total;
}

// Tile scan: exclusive prefix within each tile of kScanTile counts, tile totals out.
__global__ void __launch_bounds__(kScanThreads) scan_tiles_kernel(const unsigned int* count, long long n,
                                                                  unsigned long long* prefix,
                                                                  unsigned long long* tile_sum)
{
    const long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
    unsigned int v[kScanItems];
    unsigned long long s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        v[k] = base + k < n ? count[base + k] : 0u;
        s += v[k];
    }
    unsigned long long excl;
    const unsigned long long total = block_exclusive_scan(s, excl);
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        if (base + k < n) prefix[base + k] = excl;
        excl += v[k];
    }
    if (threadIdx.x == 0) tile_sum[blockIdx.x] = total;
}

// One block: exclusive scan of the tile totals in place (any count of tiles).
__global__ void __launch_bounds__(kScanThreads) scan_totals_kernel(unsigned long long* tile_sum, long long n_tiles,
                                                                   unsigned long long* grand_total)
{
    unsigned long long carry = 0;
    for (long long b = 0; b < n_tiles; b += kScanThreads) {
        const long long i = b + threadIdx.x;
        const unsigned long long v = i < n_tiles ? tile_sum[i] : 0ULL;
        unsigned long long excl;
        const unsigned long long total = block_exclusive_scan(v, excl);
        if (i < n_tiles) tile_sum[i] = carry + excl;
        carry += total;
    }
    if (threadIdx.x == 0) *grand_total = carry;
}

// cursor = exclusive start of each cell (the placement cursor), cell_end = inclusive end.
__global__ void finish_scan_kernel(const unsigned int* count, const unsigned long long* prefix,
                                   const unsigned long long* tile_sum, long long n, unsigned int* cursor,
                                   int* cell_end)
{
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        const unsigned long long start = prefix[c] + tile_sum[c / kScanTile];
        cursor[c] = (unsigned int)start;
        cell_end[c] = (int)(start + count[c]);
    }
}

__global__ void place_kernel(const double2* pos, long long n, Geo g, double r, unsigned int* cursor, int* idx)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        int cells[9];
        const int k = overlapping_cells(g, pos[i], r, cells);
        for (int c = 0; c < k; c++) idx[atomicAdd(cursor + cells[c], 1u)] = (int)i;
    }
}

// One warp per cell: the rank of each entry among the cell's entries by
// impurity index is its place in the reference's per-cell vector.
__global__ void order_kernel(const double2* pos, const int* idx, const int* cell_end, long long n_cells,
                             double2* out)
{
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long c = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < n_cells; c += warps) {
        const int start = c == 0 ? 0 : cell_end[c - 1];
        const int cnt = cell_end[c] - start;
        for (int j0 = 0; j0 < cnt; j0 += 32) {
            const int j = j0 + lane;
            const int v = j < cnt ? idx[start + j] : 0x7fffffff;
            int rank = 0;
            for (int k0 = 0; k0 < cnt; k0 += 32) {
                const int w = k0 + lane < cnt ? idx[start + k0 + lane] : 0x7fffffff;
#pragma unroll 8
                for (int t = 0; t < 32; t++) rank += (__shfl_sync(0xffffffffu, w, t) < v) ? 1 : 0;
            }
            if (j < cnt) out[start + rank] = pos[v];
        }
    }
}

unsigned blocks_for(long long n, int threads)
{
    const long long b = (n + threads - 1) / threads;
    return (unsigned)(b < 1 ? 1 : (b > 148LL * 64 ? 148LL * 64 : b));
}

unsigned long long g_dgrid_generation = 1;

}  // namespace

}  // namespace es

namespace {

es_status dgrid_fail(es_status st, const char* fmt, long long a = 0, long long b = 0)
{
    char msg[512];
    snprintf(msg, sizeof msg, fmt, a, b);
    es::set_global_error(msg);
    return st;
}

#define ES_DG_CUDA(call, what)                                                                           \
    do {                                                                                                 \
        const cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) {                                                                         \
            char m_[512];                                                                                \
            snprintf(m_, sizeof m_, "%s: %s", what, cudaGetErrorString(e_));                             \
            es::set_global_error(m_);                                                                    \
            return e_ == cudaErrorMemoryAllocation ? ES_ERR_OOM : ES_ERR_LAUNCH;                         \
        }                                                                                                \
    } while (0)

struct Scratch {
    double2* d_pos = nullptr;
    unsigned int* d_count = nullptr;
    unsigned int* d_cursor = nullptr;
    unsigned long long* d_prefix = nullptr;
    unsigned long long* d_tiles = nullptr;
    unsigned long long* d_total = nullptr;
    int* d_idx = nullptr;
    cudaStream_t stream = nullptr;
    ~Scratch()
    {
        if (stream) cudaStreamSynchronize(stream);
        cudaFree(d_pos);
        cudaFree(d_count);
        cudaFree(d_cursor);
        cudaFree(d_prefix);
        cudaFree(d_tiles);
        cudaFree(d_total);
        cudaFree(d_idx);
        if (stream) cudaStreamDestroy(stream);
    }
};

es_status build(es_dgrid* g, uint32_t seed, double density, int32_t tcp, int64_t max_impurities)
{
    using namespace es;
    // Grid::Grid(seed, ...), src/sim/Grid.cpp:28-46
    const double lo = g->is.spawn_region_start;
    const double hi = lo + g->is.spawn_region_size;
    const double area_length = hi - lo;
    const double proposal = area_length * area_length * density;
    if (proposal > (double)max_impurities) return dgrid_fail(ES_ERR_BAD_ARG, "Woah!");
    if (proposal < 1) return dgrid_fail(ES_ERR_BAD_ARG, "No impurities");
    const int64_t n = std::max<int64_t>(1, (int64_t)std::ceil(proposal));
    const int cpr = std::max((int)std::round(std::sqrt(n / (double)tcp)), 1);
    g->n_unique = n;
    g->is.cells_per_row = cpr;
    g->is.cell_size = g->is.spawn_region_size / (double)cpr;
    const long long n_cells = (long long)cpr * cpr;
    const long long n_tiles = (n_cells + kScanTile - 1) / kScanTile;

    Scratch s;
    ES_DG_CUDA(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking), "stream");
    ES_DG_CUDA(es::dev_malloc(&s.d_pos, sizeof(double2) * (size_t)n), "impurity positions");
    ES_DG_CUDA(es::dev_malloc(&s.d_count, sizeof(unsigned int) * (size_t)n_cells), "cell counts");
    ES_DG_CUDA(es::dev_malloc(&s.d_cursor, sizeof(unsigned int) * (size_t)n_cells), "cell cursors");
    ES_DG_CUDA(es::dev_malloc(&s.d_prefix, sizeof(unsigned long long) * (size_t)n_cells), "cell prefix");
    ES_DG_CUDA(es::dev_malloc(&s.d_tiles, sizeof(unsigned long long) * (size_t)n_tiles), "scan tiles");
    ES_DG_CUDA(es::dev_malloc(&s.d_total, sizeof(unsigned long long)), "scan total");
    ES_DG_CUDA(es::dev_malloc(&g->d_cell_end, sizeof(int) * (size_t)n_cells), "cell index");

    // GenerateImpurities (src/sim/Grid.cpp:61-75): the seed passes through an
    // int, and minstd_rand0 maps a zero state to 1.
    const unsigned long long s64 = (unsigned long long)(long long)(int)seed;
    unsigned long long x0 = s64 % kMinstdM;
    if (x0 == 0) x0 = 1;
    generate_kernel<<<blocks_for(n, 256), 256, 0, s.stream>>>(x0, n, lo, hi, s.d_pos);
    ES_DG_CUDA(es::launched(s.stream), "generate_kernel");

    // GenerateImpurityCells + ConvertToIndex (src/sim/Grid.cpp:77-110)
    const Geo geo{lo, hi - lo, g->is.cell_size, cpr};
    const double r = g->is.impurity_radius;
    ES_DG_CUDA(cudaMemsetAsync(s.d_count, 0, sizeof(unsigned int) * (size_t)n_cells, s.stream), "count clear");
    count_kernel<<<blocks_for(n, 256), 256, 0, s.stream>>>(s.d_pos, n, geo, r, s.d_count);
    ES_DG_CUDA(es::launched(s.stream), "count_kernel");
    scan_tiles_kernel<<<(unsigned)n_tiles, kScanThreads, 0, s.stream>>>(s.d_count, n_cells, s.d_prefix, s.d_tiles);
    ES_DG_CUDA(es::launched(s.stream), "scan_tiles_kernel");
    scan_totals_kernel<<<1, kScanThreads, 0, s.stream>>>(s.d_tiles, n_tiles, s.d_total);
    ES_DG_CUDA(es::launched(s.stream), "scan_totals_kernel");
    unsigned long long total = 0;
    ES_DG_CUDA(es::copy_async(&total, s.d_total, sizeof total, cudaMemcpyDeviceToHost, s.stream), "scan total");
    ES_DG_CUDA(cudaStreamSynchronize(s.stream), "grid build");
    if (total > 0x7fffffffULL)
        return dgrid_fail(ES_ERR_BAD_ARG, "indexed impurity count %lld exceeds the int32 cell index", (long long)total);
    finish_scan_kernel<<<blocks_for(n_cells, 256), 256, 0, s.stream>>>(s.d_count, s.d_prefix, s.d_tiles, n_cells,
                                                                       s.d_cursor, g->d_cell_end);
    ES_DG_CUDA(es::launched(s.stream), "finish_scan_kernel");
    const size_t n_alloc = (size_t)(total > 0 ? total : 1);
    ES_DG_CUDA(es::dev_malloc(&s.d_idx, sizeof(int) * n_alloc), "placement index");
    ES_DG_CUDA(es::dev_malloc(&g->d_imps, sizeof(double2) * n_alloc), "ordered impurities");
    place_kernel<<<blocks_for(n, 256), 256, 0, s.stream>>>(s.d_pos, n, geo, r, s.d_cursor, s.d_idx);
    ES_DG_CUDA(es::launched(s.stream), "place_kernel");
    order_kernel<<<blocks_for(n_cells * 32, 256), 256, 0, s.stream>>>(s.d_pos, s.d_idx, g->d_cell_end, n_cells,
                                                                       g->d_imps);
    ES_DG_CUDA(es::launched(s.stream), "order_kernel");
    ES_DG_CUDA(cudaStreamSynchronize(s.stream), "grid build");
    g->n_indexed = (int64_t)total;
    return ES_OK;
}

}  // namespace

extern "C" {

es_status es_dgrid_create_seeded(int32_t device_ordinal, uint32_t seed, double region_size, double region_extends,
                                 double density, double impurity_radius, int32_t target_cell_population,
                                 int64_t max_impurities, es_dgrid** out)
{
    es::Range nvtx_range("grid_build");
    if (!out) return dgrid_fail(ES_ERR_BAD_ARG, "es_dgrid_create_seeded: null output");
    *out = nullptr;
    if (target_cell_population < 1) return dgrid_fail(ES_ERR_BAD_ARG, "target_cell_population must be >= 1");
    if (!(region_size > 0.0) || !(region_extends >= 0.0) || !(density > 0.0) || !(impurity_radius >= 0.0))
        return dgrid_fail(ES_ERR_BAD_ARG, "es_dgrid_create_seeded: invalid geometry or density");
    int n_dev = 0;
    if (cudaGetDeviceCount(&n_dev) != cudaSuccess || device_ordinal < 0 || device_ordinal >= n_dev)
        return dgrid_fail(ES_ERR_DEVICE, "no CUDA device %lld", device_ordinal);
    ES_DG_CUDA(cudaSetDevice(device_ordinal), "cudaSetDevice");
    es_dgrid* g = new es_dgrid;
    g->device = device_ordinal;
    g->is.spawn_region_start = -region_extends;
    g->is.spawn_region_size = (region_size + region_extends) - (-region_extends);
    g->is.impurity_radius = impurity_radius;
    const es_status st = build(g, seed, density, target_cell_population, max_impurities > 0 ? max_impurities : 10000000);
    if (st != ES_OK) {
        es_dgrid_destroy(g);
        return st;
    }
    g->generation = (1ULL << 63) | __atomic_fetch_add(&es::g_dgrid_generation, 1ULL, __ATOMIC_RELAXED);
    *out = g;
    return ES_OK;
}

es_status es_dgrid_destroy(es_dgrid* g)
{
    if (!g) return ES_OK;
    cudaSetDevice(g->device);
    cudaFree(g->d_imps);
    cudaFree(g->d_cell_end);
    delete g;
    return ES_OK;
}

es_status es_dgrid_info(const es_dgrid* g, es_impurity_settings* out_settings, int64_t* out_indexed,
                        int64_t* out_unique)
{
    if (!g) return dgrid_fail(ES_ERR_BAD_ARG, "es_dgrid_info: null grid");
    if (out_settings) *out_settings = g->is;
    if (out_indexed) *out_indexed = g->n_indexed;
    if (out_unique) *out_unique = g->n_unique;
    return ES_OK;
}

es_status es_dgrid_download(const es_dgrid* g, double* out_xy, int32_t* out_cell_end)
{
    if (!g) return dgrid_fail(ES_ERR_BAD_ARG, "es_dgrid_download: null grid");
    ES_DG_CUDA(cudaSetDevice(g->device), "cudaSetDevice");
    if (out_xy && g->n_indexed > 0)
        ES_DG_CUDA(es::copy_sync(out_xy, g->d_imps, sizeof(double2) * (size_t)g->n_indexed, cudaMemcpyDeviceToHost),
                   "impurity download");
    if (out_cell_end)
        ES_DG_CUDA(es::copy_sync(out_cell_end, g->d_cell_end,
                              sizeof(int) * (size_t)g->is.cells_per_row * (size_t)g->is.cells_per_row,
                              cudaMemcpyDeviceToHost),
                   "cell index download");
    return ES_OK;
}

}  // extern "C"

namespace es {

// The device arrays of a built grid, for es_upload_dgrid and es_batch_add_dgrid.
void dgrid_arrays(const es_dgrid* g, const double2** imps, const int** cell_end, int64_t* n_indexed,
                  es_impurity_settings* is, uint64_t* generation, int* device)
{
    *imps = g->d_imps;
    *cell_end = g->d_cell_end;
    *n_indexed = g->n_indexed;
    *is = g->is;
    *generation = g->generation;
    *device = g->device;
}

}  // namespace es
