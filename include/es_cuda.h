/* es_cuda.h - C ABI of the B200 (sm_100a) backend for ElasticScattering's
 * real-space conductivity path.
 *
 * The reference selects a backend behind `class Simulation`
 * (src/sim/Simulation.h:56-147; chosen at src/SimulationRunner.cpp:82-84) and
 * its GPU implementation is an OpenCL context with six kernels
 * (src/sim/SimulationCL.cpp and the .cl files of src/sim/cl). This header is the drop-in
 * replacement for that implementation: plain pointers and sizes, no C++ or
 * framework types. A host wrapper (SimulationCUDA, elasticscattering_b200/host)
 * maps the reference's `Simulation` methods onto these calls one to one.
 *
 * Conventions
 *  - Every call returns es_status; ES_OK == 0. After a failure, es_last_error()
 *    returns a message. The reference prints and exit(0)s instead
 *    (src/utils/ErrorMacros.h:22-38); the host wrapper restores that behaviour.
 *  - One context = one device + one CUDA stream. Calls on a context are
 *    serialised on its stream; distinct contexts share no state.
 *  - Host arrays are caller-owned. The context owns its device buffers.
 *  - Orbit order is the reference's [j][i][q][p]: index
 *    j*dim*4*ppq + i*4*ppq + q*ppq + p (src/sim/Simulation.h:67).
 */
#ifndef ES_CUDA_H
#define ES_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum es_status {
    ES_OK = 0,
    ES_ERR_BAD_ARG = 1,     /* invalid size, pointer or state */
    ES_ERR_OOM = 2,         /* device allocation failed */
    ES_ERR_LAUNCH = 3,      /* kernel launch or CUDA API failure */
    ES_ERR_WALK_CAP = 4,    /* an orbit exceeded the cell-walk step bound */
    ES_ERR_DEVICE = 5,      /* no usable CUDA device / wrong architecture */
    ES_ERR_NO_GRID = 6,     /* es_upload_grid has not been called */
    ES_ERR_NO_SAMPLE = 7,   /* es_init_sample has not been called */
    ES_ERR_TIMEOUT = 8      /* a bounded device wait ran out */
} es_status;

typedef enum es_precision {
    ES_PRECISION_FP64 = 0,       /* plain FP64, reference semantics operation by operation */
    ES_PRECISION_SPLIT = 1,      /* FP32 orbit stepping, FP64 tangency band, phase and reductions */
    ES_PRECISION_SPLIT_EXACT = 2 /* the split walk (its lifetimes are the FP64 walk's bit for bit:
                                    every decision FP32 cannot settle is taken in FP64) with the
                                    FP64 integration: sigma equals ES_PRECISION_FP64's. Batches:
                                    ES_BATCH_PASS_KERNELS only */
} es_precision;

/* Reference layout of ImpuritySettings (src/sim/es/settings.h:76-85). */
typedef struct es_impurity_settings {
    double spawn_region_start;
    double spawn_region_size;
    double cell_size;
    int32_t cells_per_row;
    double impurity_radius;
} es_impurity_settings;

/* The reference's Settings (src/ConfigSettings.h:22-34) with the bool widened
 * to int32 for a stable C layout. */
typedef struct es_settings {
    double tau;
    double alpha;
    int32_t is_clockwise;
    double particle_speed;
    double region_size;
    double region_extends;
    double impurity_density;
    double impurity_radius;
    int32_t target_cell_population;
} es_settings;

/* ParticleMetrics (src/sim/es/particle_metrics.h:22-44) with 64-bit counters
 * (the reference's int32 counters overflow beyond ~2^31 impurity tests). */
typedef struct es_metrics {
    int64_t cells_passed;
    int64_t impurities_tested;
    int64_t particles_inside_impurity;
    int64_t particles_escaped;
    int64_t particles_at_bound;
    int64_t max_impurities_tested;
    int64_t max_cells_passed;
    int64_t crossings_tested; /* orbit/impurity pairs that passed CirclesCross (FLOP model) */
    int64_t start_cell_tests; /* InsideImpurity tests of the start-cell scans (FLOP model) */
    int64_t retraced_fp64;    /* split precision: orbits re-traced by the FP64 kernel */
} es_metrics;

/* Constructor arguments of Simulation (src/sim/Simulation.h:131-146) plus
 * the GridInformation it reads (src/sim/es/settings.h:65-73). */
typedef struct es_sim_desc {
    int32_t positions_per_row;      /* dim, odd, >= 3 */
    int32_t particles_per_quadrant; /* phi_steps, odd, >= 3 */
    double region_size;
    double region_extends;
    double grid_cell_size;          /* GridInformation::cell_size (sets the start offset) */
    int32_t device_ordinal;
    int32_t precision;              /* es_precision */
} es_sim_desc;

typedef struct es_ctx es_ctx;

/* Kernel choices of a context. No reference counterpart (the reference's
 * OpenCL launch shape is fixed, src/sim/SimulationCL.cpp:412-431); the
 * autotuner picks these, the defaults are the measured best on B200. */
typedef struct es_tuning {
    int32_t lifetime_variant;  /* FP64 lifetime kernel: 0 = one orbit per thread (<= 80 registers),
                                  2 = the same at <= 64 registers, 6 = as 2 with the crossing points of
                                  a cell taken after its cheap tests (the default); other values are
                                  rejected */
} es_tuning;

/* Replaces SimulationCL::SimulationCL (src/sim/SimulationCL.cpp:386-475): binds a
 * device, creates the stream and the per-pass buffers. */
es_status es_create(const es_sim_desc* desc, es_ctx** out);

/* Replaces SimulationCL::~SimulationCL (src/sim/SimulationCL.cpp:477-508). */
es_status es_destroy(es_ctx* ctx);

/* Reads / sets the kernel choices of a context (see es_tuning). */
es_status es_get_tuning(const es_ctx* ctx, es_tuning* out);
es_status es_set_tuning(es_ctx* ctx, const es_tuning* tuning);

/* Message of the last failure on this context ("" if none). ctx may be NULL
 * for failures of es_create and es_derive_temperatures_noalloc. */
const char* es_last_error(const es_ctx* ctx);

/* Restricts the following passes of this context to start rows [j0, j1)
 * (0 <= j0 < j1 <= positions_per_row; the default is every row). Stage (a)
 * traces only those rows' orbits, whose lifetimes land at their usual place in
 * the pass's [j][i][q][p] order, and stages (b)+(c) return those rows' share of
 * sigma. The shares of a partition of the rows add up to the whole pass's
 * sigma: a sector pass too large for one GPU is split over GPUs this way, each
 * computing a row range, the shares summed in rank order. No reference
 * counterpart (the reference runs every pass on one device). The images path
 * (es_compute_sigmas_images) and es_average_lifetime need every row. */
es_status es_set_rows(es_ctx* ctx, int32_t j0, int32_t j1);

/* Replaces the impurity/index upload in SimulationCL::ComputeLifetimes
 * (src/sim/SimulationCL.cpp:119-125). imp_xy holds n_indexed ordered
 * impurities as x,y pairs (Grid::GetImpurities, src/sim/Grid.h:74), cell_end
 * the cumulative end index of each of cells_per_row^2 cells (Grid::GetIndex,
 * src/sim/Grid.h:75). The upload is skipped when `generation` equals the
 * generation already resident (the reference keys on the seed, which is 0 for
 * every file-loaded grid). Pageable host arrays are copied through a pinned
 * staging ring by several host threads; pinned arrays are copied directly. */
es_status es_upload_grid(es_ctx* ctx, const double* imp_xy, int64_t n_indexed, const int32_t* cell_end,
                         const es_impurity_settings* is, uint64_t generation);

/* Replaces Simulation::InitSample (src/sim/Simulation.h:111-126): sector
 * (coherent or incoherent) and carrier settings for the following passes. */
es_status es_init_sample(es_ctx* ctx, const es_settings* s, int32_t coherent);

/* Replaces Simulation::ComputeSigmas (src/sim/Simulation.h:128,
 * src/sim/SimulationCL.cpp:72-91): lifetimes of all orbits for field B
 * (stage a), then per temperature the phase Simpson integral (stage b) and the
 * start-position Simpson reduction (stage c). out_sigma receives
 * [xx_0, xy_0, xx_1, xy_1, ...] (2*n_t doubles). out_metrics may be NULL.
 * Blocks until the results are on the host. */
es_status es_compute_sigmas(es_ctx* ctx, double magnetic_field, const double* temperatures, int32_t n_t,
                            double* out_sigma, es_metrics* out_metrics);

/* Replaces Simulation::ComputeSigmasWithImages (src/sim/Simulation.h:129,
 * src/sim/SimulationCL.cpp:93-111): as es_compute_sigmas plus the per-position
 * maps of IntegratePosition (src/sim/SimulationCPU.cpp:224-243): truncated
 * lifetime, sigma_xx and sigma_xy integrated over phase, each dim*dim doubles
 * per temperature, temperature-major. */
es_status es_compute_sigmas_images(es_ctx* ctx, double magnetic_field, const double* temperatures, int32_t n_t,
                                   double* out_sigma, double* lifetime_pos, double* sigma_xx_pos,
                                   double* sigma_xy_pos, es_metrics* out_metrics);

/* Replaces SimulationCL::ComputeLifetimes (src/sim/SimulationCL.cpp:113-177):
 * stage (a) only. If out_lifetimes is non-NULL the dim^2*4*ppq raw lifetimes
 * are copied to it (the `dump_lifetimes` option of the reference's config,
 * examples/explanation.config:89-90). The lifetimes stay resident for
 * es_derive_temperatures. */
es_status es_compute_lifetimes(es_ctx* ctx, double magnetic_field, double* out_lifetimes, es_metrics* out_metrics);

/* Copies `count` raw lifetimes of the resident pass, starting at orbit `first`
 * ([j][i][q][p] order), to the host array out. No reference counterpart (the
 * reference reads whole buffers back, src/sim/SimulationCL.cpp:148); it reads
 * a band of start rows of a pass too large to copy out whole. */
es_status es_read_lifetimes(es_ctx* ctx, int64_t first, int64_t count, double* out);

/* Replaces the temperature loop of SimulationCL::ComputeSigmas
 * (src/sim/SimulationCL.cpp:82-84, DeriveTemperature :179-189) on the
 * lifetimes resident from the last es_compute_lifetimes. */
es_status es_derive_temperatures(es_ctx* ctx, const double* temperatures, int32_t n_t, double* out_sigma);

/* Asynchronous form of es_compute_sigmas for callers that keep results on the
 * device: enqueues stages (a)-(c) on the context stream and writes 2*n_t
 * doubles to the DEVICE pointer d_out_sigma. Metrics accumulate on the device
 * until es_read_metrics. No host synchronisation. */
es_status es_enqueue_sigmas(es_ctx* ctx, double magnetic_field, const double* temperatures, int32_t n_t,
                            double* d_out_sigma);

/* Asynchronous form of es_derive_temperatures: enqueues stages (b)+(c) for
 * every temperature on the resident lifetimes and writes 2*n_t doubles to the
 * DEVICE pointer d_out_sigma. No host synchronisation. */
es_status es_enqueue_derive_temperatures(es_ctx* ctx, const double* temperatures, int32_t n_t, double* d_out_sigma);

/* Asynchronous stage (a) only: enqueues the lifetime pass for field B on the
 * context stream (SimulationCL::ComputeLifetimes without its blocking copies,
 * src/sim/SimulationCL.cpp:113-177). The lifetimes stay resident. */
es_status es_enqueue_lifetimes(es_ctx* ctx, double magnetic_field);

/* Replaces Simulation::AverageLifetime (src/sim/Simulation.h:93-106): the mean
 * raw lifetime of the resident pass (the "Avg. particle lifetime" row of
 * Metrics.txt), summed on the device in a fixed order. */
es_status es_average_lifetime(es_ctx* ctx, double* out_average);

/* Waits for the context stream, then reports any device-side error flag. */
es_status es_synchronize(es_ctx* ctx);

/* Reads (and optionally resets) the device-side metrics accumulated by
 * es_enqueue_sigmas. Synchronises the stream. */
es_status es_read_metrics(es_ctx* ctx, es_metrics* out, int32_t reset);

/* The context's cudaStream_t, as an opaque pointer (for event timing). */
void* es_stream(es_ctx* ctx);

/* Number of kernel launches this context has issued since creation. */
int64_t es_launch_count(const es_ctx* ctx);

/* Test hook for the split path's finish kernel: on passes that leave their
 * winners to it (long walks), the hit of every orbit whose index is a multiple
 * of `every` goes to the FP64 re-trace as a winner whose crossing point the
 * reference drops would, and the re-trace subtracts the walk's counters. The
 * lifetimes and every counter but `retraced_fp64` must stay as without it.
 * 0 (the default) turns it off. No reference counterpart. */
es_status es_debug_finish_retrace(es_ctx* ctx, int32_t every);

/* Known-answer hook for the device geometry: one GetNextCell step
 * (src/sim/es/cell_grid.h:132-181) evaluated by the FP64 device code on one
 * thread. in6/out6 = (pos.x, pos.y, incident_angle, dphi, cell.x, cell.y).
 * Returns the step's "next cell available" flag in *out_available. */
es_status es_debug_next_cell(es_ctx* ctx, double center_x, double center_y, double radius, int32_t clockwise,
                             double phi, const es_impurity_settings* is, const double* in6, double* out6,
                             int32_t* out_available);

/* Known-answer hook for one orbit: CreateParticle(q, p, (px, py), ps) +
 * TraceOrbit (src/sim/es/lifetime.h:36-148) on the resident grid, evaluated by
 * the FP64 device code on one thread, with explicit ParticleSettings fields
 * (src/sim/es/settings.h:87-98) as the reference's LifetimeTests build them.
 * Writes the raw lifetime (seconds) to *out_lifetime. */
es_status es_debug_trace(es_ctx* ctx, double px, double py, int32_t q, int32_t p, double magnetic_field,
                         double phi_start, double phi_step_size, double alpha, double particle_speed,
                         int32_t is_clockwise, int32_t is_coherent, double* out_lifetime);

/* Stages (b)+(c) -- the phase and start-position Simpson integrals of
 * es_derive_temperatures -- without allocating any device memory. No
 * counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc: a framework that owns all device
 * memory through its own pool, or a path on which a driver allocation (and its
 * implicit synchronisation) is not allowed. The caller passes the raw lifetimes
 * of one sector pass (d_lifetimes, device memory, dim^2 * 4 * phi_steps doubles
 * in [j][i][q][p] order, e.g. as es_compute_lifetimes returns them), the
 * sector's settings, field and temperatures, and d_out_sigma (device memory,
 * 2 * n_t doubles: xx, xy per temperature). Work is enqueued on `stream`
 * (a cudaStream_t; NULL = the legacy default stream) and not waited for.
 * Every argument (each temperature included) is checked before anything is
 * enqueued: an error return means no work was queued and d_out_sigma is
 * untouched. n_t == 0 enqueues nothing.
 *
 * Results agree with es_derive_temperatures to about 1e-12 relative, not bit
 * for bit: this entry point builds its phase table on the device (device
 * cos/sin), the allocating path on the host (host libm).
 *
 * The scratch (phase table and block partial sums) is one fixed array of
 * 169 KB that every GPU which loads this library holds until the process
 * exits. Limit: phi_steps <= 1025; larger values return ES_ERR_BAD_ARG with a
 * message in es_last_error(NULL). The first call in a CUDA context (with that
 * context's device current) looks up the array's device address in that
 * context and caches it under the context's id; make that first call before
 * any stream capture. Every call shares the array and leaves its contents
 * behind; each call rewrites every slot it reads before reading it, so nothing
 * needs clearing between calls, but calls whose work overlaps on the GPU
 * (different streams, or threads) race on it. */
es_status es_derive_temperatures_noalloc(const double* d_lifetimes, int32_t positions_per_row, int32_t phi_steps,
                                         const es_settings* s, int32_t coherent, double magnetic_field,
                                         const double* temperatures, int32_t n_t, double* d_out_sigma,
                                         void* stream);

/* ---------------------------------------------------------------------------
 * Batched sweeps. No reference counterpart: the reference runs one
 * (sample, field, sector) pass per Simulation::ComputeSigmas call
 * (src/SimulationRunner.cpp:103-151). A batch holds many such passes -- each
 * with its own grid, start-position grid, phase count, field, sector and
 * temperature list -- and computes all of them in one persistent kernel,
 * launched from a CUDA graph that is recorded once and replayed; changing the
 * instance table does not re-record it. Lifetimes are not materialised:
 * stages (b) and (c) are fused into the lifetime kernel. Results are
 * bit-reproducible run to run (fixed-point accumulation).
 * ------------------------------------------------------------------------- */

#define ES_BATCH_MAX_T 8

typedef struct es_batch es_batch;

/* One pass: the arguments of es_create + es_init_sample + es_compute_sigmas
 * for one (sample, field, sector). */
typedef struct es_batch_instance {
    int32_t grid;                   /* index returned by es_batch_add_grid */
    int32_t positions_per_row;      /* dim, odd, >= 3 */
    int32_t particles_per_quadrant; /* phi_steps, odd, >= 3 */
    int32_t coherent;               /* sector */
    double region_size;
    double grid_cell_size;          /* GridInformation::cell_size (start offset), as es_sim_desc */
    double magnetic_field;
    es_settings settings;           /* tau, alpha, is_clockwise, particle_speed are read */
    int32_t n_t;                    /* 1..ES_BATCH_MAX_T temperatures, at most 4 distinct tau */
    double temperatures[ES_BATCH_MAX_T];
} es_batch_instance;

/* How a batch maps its passes onto kernels. In every mode one graph replay
 * runs the whole batch; the autotuner picks the mode. */
typedef enum es_batch_mode {
    /* values 0 and 1 named block-per-work-item modes that never won on B200 and were
       removed; es_batch_set_tuning rejects them */
    ES_BATCH_PERSISTENT = 2,  /* one persistent kernel: warps take work items of 32 * chunk_iters
                                 orbits of any pass from a global counter, stages (b)+(c) fused in */
    ES_BATCH_PASS_KERNELS = 3 /* the single-pass path's kernels for each pass in turn: the lifetime
                                 kernel (and, split, its FP64 re-trace) writes the pass's lifetimes
                                 to device scratch, the integration kernels reduce them to sigma;
                                 chunk_iters and blocks_per_sm are not used (the default) */
} es_batch_mode;

/* Launch choices of a batch (picked by the autotuner). */
typedef struct es_batch_tuning {
    int32_t chunk_iters;    /* ES_BATCH_PERSISTENT: orbits per work item = 32 * chunk_iters */
    int32_t blocks_per_sm;  /* ES_BATCH_PERSISTENT: resident blocks of 256 threads per SM, 3 or 4 */
    int32_t precision;      /* es_precision */
    int32_t mode;           /* es_batch_mode */
} es_batch_tuning;

es_status es_batch_create(int32_t device_ordinal, es_batch** out);
es_status es_batch_destroy(es_batch* b);
/* Message of the last failure on this batch ("" if none). */
const char* es_batch_last_error(const es_batch* b);
es_status es_batch_get_tuning(const es_batch* b, es_batch_tuning* out);
es_status es_batch_set_tuning(es_batch* b, const es_batch_tuning* t);

/* Copies one impurity grid (same arrays as es_upload_grid) to the device and
 * returns its index in *out_grid. Grids stay resident until es_batch_clear.
 * Host arrays in pageable memory are copied through a pinned staging ring by
 * several host threads; pinned arrays are copied directly. */
es_status es_batch_add_grid(es_batch* b, const double* imp_xy, int64_t n_indexed, const int32_t* cell_end,
                            const es_impurity_settings* is, int32_t* out_grid);

/* Releases every grid and instance of the batch. The grids' device memory is
 * kept and reused by later es_batch_add_grid calls (the smallest allocation
 * that fits; when none fits, all kept memory is freed before the new grid is
 * allocated), so a sweep that clears and adds same-sized grids every step
 * neither allocates nor frees. es_batch_destroy frees everything. */
es_status es_batch_clear(es_batch* b);

/* Sets the passes of the batch (validated as es_create / es_init_sample /
 * es_compute_sigmas validate them). */
es_status es_batch_set_instances(es_batch* b, const es_batch_instance* inst, int32_t n);

/* Runs every pass and blocks. out_sigma: n * ES_BATCH_MAX_T * 2 doubles,
 * [instance][temperature][xx, xy], as es_compute_sigmas returns them per pass.
 * out_metrics (n entries) may be NULL. */
es_status es_batch_run(es_batch* b, double* out_sigma, es_metrics* out_metrics);

/* es_batch_run in two halves: enqueue the graph on the batch stream (no host
 * wait), then wait and convert the results. */
es_status es_batch_enqueue(es_batch* b);
es_status es_batch_collect(es_batch* b, double* out_sigma, es_metrics* out_metrics);

/* The batch's cudaStream_t, as an opaque pointer (for event timing). */
void* es_batch_stream(es_batch* b);
/* Kernel launches issued by this batch (one per graph replay, one per grid copy). */
int64_t es_batch_launch_count(const es_batch* b);
/* Kernel nodes of the batch's recorded graph: the kernels one replay launches
 * (0 before the first run). */
int64_t es_batch_graph_kernels(const es_batch* b);
/* Orbits per run of the current instance table. */
int64_t es_batch_total_orbits(const es_batch* b);

/* ---------------------------------------------------------------------------
 * Grids built on the GPU. Replaces the host work of Grid::Grid(seed, ...)
 * (src/sim/Grid.cpp:28-46) with GenerateImpurities, GenerateImpurityCells and
 * ConvertToIndex (src/sim/Grid.cpp:61-110, :112-188) plus the upload of
 * es_upload_grid / es_batch_add_grid: the impurity positions are the
 * libstdc++ minstd_rand0 + generate_canonical draws the host Grid makes,
 * reproduced draw for draw, and the ordered array and cumulative cell index
 * are the host Grid's bit for bit. Failures before a grid exists report
 * through es_last_error(NULL).
 * ------------------------------------------------------------------------- */

typedef struct es_dgrid es_dgrid;

/* Grid(seed, region_size, region_extends, density, impurity_radius,
 * target_cell_population) on device_ordinal. max_impurities <= 0 means the
 * reference's 1e7 ("Woah!", src/sim/Grid.cpp:36). */
es_status es_dgrid_create_seeded(int32_t device_ordinal, uint32_t seed, double region_size, double region_extends,
                                 double density, double impurity_radius, int32_t target_cell_population,
                                 int64_t max_impurities, es_dgrid** out);
es_status es_dgrid_destroy(es_dgrid* g);
/* GetSettings (src/sim/Grid.h:77-86), GetTotalImpurityCount and the unique count. */
es_status es_dgrid_info(const es_dgrid* g, es_impurity_settings* out_settings, int64_t* out_indexed,
                        int64_t* out_unique);
/* GetImpurities / GetIndex as host copies: 2 * n_indexed doubles, cells_per_row^2 ints (either may be NULL). */
es_status es_dgrid_download(const es_dgrid* g, double* out_xy, int32_t* out_cell_end);
/* es_upload_grid from a device grid (device-to-device; skipped when already resident). */
es_status es_upload_dgrid(es_ctx* ctx, const es_dgrid* g);
/* es_batch_add_grid from a device grid (device-to-device copy; g may be destroyed afterwards). */
es_status es_batch_add_dgrid(es_batch* b, const es_dgrid* g, int32_t* out_grid);

/* ---------------------------------------------------------------------------
 * Learned surrogate. No reference counterpart: an ensemble of MLPs,
 * 5 -> 256 x 4 -> 2 with GELU; the hidden layers in BF16 weights and
 * activations with FP32 accumulation on the tensor cores, the 256 -> 2 head in
 * FP32; trained on the GPU by this library's own forward and backward kernels. Inputs are 5 normalised features per query, outputs 2
 * normalised targets per query and member; the normalisation and the fallback
 * to the simulator live with the caller.
 * Parameter layout of one member: for each of the 5 layers, W [N][K] row-major
 * then b [N], with (K, N) = (5, 256), (256, 256) x 3, (256, 2); members follow
 * each other.
 * ------------------------------------------------------------------------- */

typedef struct es_mlp es_mlp;

/* Parameters of one member (199,426). */
int64_t es_mlp_param_count(void);
es_status es_mlp_create(int32_t n_nets, int32_t device_ordinal, es_mlp** out);
es_status es_mlp_destroy(es_mlp* m);
const char* es_mlp_last_error(const es_mlp* m);
/* FP32 parameters of every member (n_nets * es_mlp_param_count() floats); resets Adam. */
es_status es_mlp_set_params(es_mlp* m, const float* params);
es_status es_mlp_get_params(es_mlp* m, float* params);
/* Training set: x [n][5], y [n][2] (host, FP32), copied to the device. */
es_status es_mlp_set_dataset(es_mlp* m, const float* x, const float* y, int64_t n);
/* `steps` Adam steps (beta 0.9 / 0.999, eps 1e-8) of every member on its own
 * bootstrap minibatches of `batch` rows (drawn from `seed` and the step count);
 * out_loss (n_nets floats, may be NULL) receives the last step's mean squared error. */
es_status es_mlp_train(es_mlp* m, int32_t steps, int32_t batch, float lr, uint64_t seed, float* out_loss);
/* Loss and gradients without an update, for checking: x [n_nets][rows][5],
 * y [n_nets][rows][2]; out_grads n_nets * es_mlp_param_count() floats. */
es_status es_mlp_gradients(es_mlp* m, const float* x, const float* y, int32_t rows, float* out_grads,
                           float* out_loss);
/* Every member on the same q queries x [q][5]: out_each [n_nets][q][2], out_mean
 * [q][2], out_spread [q][2] (ensemble standard deviation / |mean|); any output
 * pointer may be NULL. */
es_status es_mlp_predict(es_mlp* m, const float* x, int64_t q, float* out_each, float* out_mean, float* out_spread);
/* Whole queries on the device: q [n][5] = (B, T, density, impurity radius,
 * tau) -> the members' mean sigma out_sigma [n][2] and out_spread [n], the
 * largest over the two outputs of the members' standard deviation over |mean|;
 * out_each [n_nets][n][2] (may be NULL) receives the network outputs. The
 * features, the five layers of every member and the conversion of the outputs
 * to sigma (exp(t) sigma_0 (1, w tau) / (1 + (w tau)^2), FP64) run in one
 * kernel for n <= 256 (latency: CUDA cores, activations in shared memory) and
 * as the batched tensor-core pass plus two small kernels above. The two agree
 * to FP32 summation order in the hidden layers. Any output may be NULL. */
typedef struct es_mlp_query_map {
    double g_lo[5], g_hi[5]; /* feature k: 2 (g(v) - g_lo[k]) / (g_hi[k] - g_lo[k]) - 1 */
    int32_t log_scale[5];    /* g = log when nonzero (the query value must then be > 0), else the identity */
    double sigma0_per_tau;   /* sigma_0 = sigma0_per_tau * tau */
    double w_per_b;          /* omega = w_per_b * B */
} es_mlp_query_map;
es_status es_mlp_query(es_mlp* m, const es_mlp_query_map* map, const double* q, int64_t n, double* out_sigma,
                       double* out_spread, float* out_each);
int64_t es_mlp_launch_count(const es_mlp* m);
void* es_mlp_stream(es_mlp* m);

/* ---------------------------------------------------------------------------
 * Host-side fault injection, for testing callers' error handling. No
 * reference counterpart (the reference prints and exits on every error,
 * src/utils/ErrorMacros.h:22-38).
 *
 * spec: comma-separated items "kind:N" or "kind:N+", kind one of
 *   alloc   device and pinned-host allocations,
 *   copy    host<->device and device<->device copies,
 *   launch  kernel launches,
 * made by the lifetime, integration, batch, grid-build and no-alloc entry
 * points (the es_mlp_* surrogate calls are not counted). "kind:N" fails the
 * N-th such operation (1-based, counted from this call) once; "kind:N+" fails
 * the N-th and every later one. NULL or "" disarms. The environment variable
 * ES_FAULT_INJECT arms the same syntax at the first counted operation, unless
 * es_fault_inject was called first.
 *
 * An injected allocation failure makes nothing and returns ES_ERR_OOM. An
 * injected copy or launch failure is reported (ES_ERR_LAUNCH) after the real
 * operation was issued and its stream waited on, so memory holds what an
 * error-free call would have written and nothing is left in flight; no GPU
 * fault is ever provoked. After any failure the object stays usable: the call
 * can be repeated (a context whose es_upload_grid or es_init_sample failed
 * needs that call again first). */
es_status es_fault_inject(const char* spec);
/* Operations counted since the last es_fault_inject: out_counts[0] alloc,
 * [1] copy, [2] launch, [3] how many were failed. */
es_status es_fault_counts(int64_t* out_counts);

/* Measured FP64 FMA throughput of a device (TFLOP/s, 2 FLOP per FMA): the
 * denominator of the lifetime kernel's roofline. No reference counterpart
 * (the reference publishes no device figures). Runs for a few milliseconds. */
es_status es_probe_fp64_fma(int32_t device_ordinal, double* out_tflops);

/* Measured FP32 FMA throughput (TFLOP/s): the denominator of the split
 * kernel's roofline. No reference counterpart. */
es_status es_probe_fp32_fma(int32_t device_ordinal, double* out_tflops);

#ifdef __cplusplus
}
#endif

#endif /* ES_CUDA_H */
