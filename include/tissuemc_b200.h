/* tissuemc_b200.h — C ABI of the B200 (sm_100a) photon-walk engine.
 *
 * The engine is a drop-in for TissueMC's GPU engine, whose C++ boundary is
 *
 *     namespace tissuemc {
 *         bool cuda_available();                                            // cuda_engine.hpp:9-11
 *         RunResult run_cuda(const RunSpec &run, const EngineOptions &opt); // cuda_engine.hpp:13-14
 *     }
 *
 * (paths relative to the TissueMC project root: include/tissuemc/cuda_engine.hpp). The entry points
 * below carry the same information as plain C structs, pointers and sizes, so that the C++ shim
 * (tissuemc_b200/csrc/host/run_cuda.cpp), ctypes, or any other FFI can bind them. Results are
 * written into caller-allocated buffers whose sizes come from tmc_b200_query_sizes().
 *
 * Every entry point is synchronous at the boundary, uses the device given in the options (default
 * 0) and is NOT re-entrant: concurrent calls from several host threads must be serialised by the
 * caller, as with the reference engine (src/cuda/engine.cu:322-358 runs on the default stream of
 * device 0).
 *
 * Status codes follow the reference's error behaviour: an invalid run or invalid options is
 * TMC_BAD_CONFIG (the reference throws ConfigError, config.hpp:31-66 and engine.cu:328-350), a
 * missing device is TMC_NO_DEVICE ("no usable CUDA device found", engine.cu:351-353), a CUDA
 * failure is TMC_CUDA_ERROR ("CUDA error at file:line: ...", engine.cu:18-26). The message buffer
 * holds the same text the reference would put in the exception.
 */
#ifndef TISSUEMC_B200_H
#define TISSUEMC_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The library exports these entry points and nothing else (its C++ internals are hidden). */
#if defined(__GNUC__)
#define TMC_B200_API __attribute__((visibility("default")))
#else
#define TMC_B200_API
#endif

#define TMC_B200_MAX_LAYERS 16
#define TMC_B200_ABI_VERSION 2

typedef enum {
    TMC_OK = 0,
    TMC_BAD_CONFIG = 1,     /* invalid run description or options                           */
    TMC_NO_DEVICE = 2,      /* no usable CUDA device                                         */
    TMC_CUDA_ERROR = 3,     /* a CUDA runtime call failed                                    */
    TMC_DEVICE_TIMEOUT = 4, /* a bounded device-side wait gave up (sweep work queue)         */
    TMC_BAD_ARGUMENT = 5    /* a NULL pointer or a buffer too small for the run              */
} tmc_status_code;

typedef struct {
    int32_t code;       /* tmc_status_code */
    char message[512];  /* NUL-terminated; empty on success */
} tmc_status;

/* One tissue layer: refractive index, absorption and scattering coefficients [1/cm], anisotropy,
 * thickness [cm]. Mirrors LayerSpec (include/tissuemc/config.hpp:14-20). */
typedef struct {
    double n, mua, mus, g, d;
} tmc_layer;

/* One MCML run. Mirrors RunSpec (include/tissuemc/config.hpp:22-29); na, which the reference
 * parses but never uses, sets the number of exit-angle bins of R_d(r,a) and T_t(r,a). */
typedef struct {
    uint64_t photons;
    double dz, dr;
    int32_t nz, nr, na;
    double n_above, n_below;
    int32_t num_layers;
    tmc_layer layers[TMC_B200_MAX_LAYERS];
} tmc_run_spec;

/* Engine options. Mirrors EngineOptions (include/tissuemc/cpu_engine.hpp:18-30) where the fields
 * mean something to a GPU engine; zero-initialise and set what you need (tmc_b200_default_options
 * fills the reference's defaults). */
typedef struct {
    uint64_t seed;          /* Philox key; photon i always uses the stream (seed, i)           */
    int32_t batches;        /* >= 1 and <= photons; the unit of the standard error              */
    uint64_t photons;       /* if nonzero, overrides spec.photons                               */
    int32_t rung;           /* accepted for CLI compatibility: 0,1,3,5,6,7,8; one B200 kernel   */
    int32_t profiles;       /* 0: skip the profile tallies (diagnostic, rung 6 only)            */
    int32_t device;         /* CUDA device ordinal                                              */
    int32_t fast_math;      /* 1 (default): SFU intrinsics; 0: IEEE division/sqrt, libdevice    */
    int32_t threads_per_block; /* 0 = chosen by the planner                                     */
    int32_t blocks_per_sm;     /* 0 = chosen by the planner                                     */
    int32_t smem_budget;       /* bytes of shared memory per block for tallies; 0 = planner     */
    uint32_t step_cap;         /* a packet still alive after this many steps is ended and counted
                                  as an anomaly (0 = 2,000,000,000); no reference counterpart: the
                                  reference loops until the packet dies (physics.hpp:279-287) */
    /* Shared-memory tally tiles, for grids whose tallies do not all fit (tmc_b200_plan,
     * tmc_b200_autotune); they change where deposits are summed, never the results. */
    int32_t tile_tz;           /* depth bins of the shared core tile of A(r,z); its radial rows
                                  follow from the budget. 0 = planner (about 2 sqrt(tile words)),
                                  -1 = no core tile (only the cross, if any, in shared memory) */
    int32_t tile_ra_rows;      /* radial rows of R_d(r,a) and of T_t(r,a) kept in shared memory:
                                  0 = planner (an eighth of the budget each), -1 = none */
    int32_t tile_cross;        /* the clamped last row and last column of A(r,z) in shared memory:
                                  0 or 1 = when they fit (planner), -1 = never */
} tmc_options;

/* Element counts of every output buffer for a run (tmc_b200_query_sizes). */
typedef struct {
    uint64_t batches, layers, nz, nr, na;
    uint64_t absorbed; /* batches * layers */
    uint64_t a_rz;     /* nr * nz  */
    uint64_t ra;       /* nr * na  (each of rd_ra and tt_ra) */
    uint64_t tally_words; /* 64-bit words of the raw fixed-point tally buffer */
    uint64_t device_words; /* 64-bit words of the device buffer of tmc_b200_run_device and
                              tmc_b200_run_device_range: the tally words, then one word that holds
                              the call's photon-claim counter */
} tmc_sizes;

/* Caller-allocated host buffers for one run. Every pointer is required unless marked optional.
 * Weights are in units of launched packets (the sums the reference reports, not normalised per
 * area or solid angle). 2-D arrays are row-major with r as the slow index, as MCML's A_rz[ir][iz]
 * and Rd_ra[ir][ia]. */
typedef struct {
    uint64_t *first_photon, *photons; /* [batches]  BatchPlan (include/tissuemc/batching.hpp)   */
    double *rd, *tt;                  /* [batches]  weight leaving through the top / bottom     */
    double *absorbed;                 /* [batches * layers]                                      */
    uint64_t *events, *anomalies;     /* [batches]                                               */
    double *a_z, *rd_r;               /* [nz], [nr]  the reference's 1-D profiles                */
    double *tt_r;                     /* [nr]        optional                                    */
    double *a_rz;                     /* [nr * nz]   optional                                    */
    double *rd_ra, *tt_ra;            /* [nr * na]   optional                                    */
    uint64_t *raw;                    /* [tally_words] optional: the fixed-point tally buffer    */
    double specular;                  /* out: specular reflectance, computed in double           */
    double kernel_seconds;            /* out: device time of the walk and its reduction          */
    double wall_seconds;              /* out: host time of the whole call                        */
    char device[128];                 /* out: "NVIDIA B200 (sm_100)"                            */
} tmc_result;

/* Fixed-point scale of the tallies: a weight w is added as round(w * 2^32) into an unsigned
 * 64-bit integer, so every sum is exact and independent of scheduling. */
#define TMC_B200_FIXED_SCALE 4294967296.0

/* Largest photon count per run. A single tally word holds at most 2^32 launched packets' weight
 * (2^64 / 2^32); with the roulette's weight boost the headroom is kept at a factor of two. */
#define TMC_B200_MAX_PHOTONS (1ull << 31)

/* 1 if a CUDA device is present and usable (replaces tissuemc::cuda_available,
 * include/tissuemc/cuda_engine.hpp:9-11). */
TMC_B200_API int tmc_b200_available(void);

/* ABI version and the library's build string. */
TMC_B200_API int tmc_b200_abi_version(void);
TMC_B200_API const char *tmc_b200_version(void);

/* Options with the reference's defaults (seed 1, 10 batches, rung 0, profiles on; cpu_engine.hpp). */
TMC_B200_API void tmc_b200_default_options(tmc_options *opt);

/* Validate the run and options exactly as run_cuda does (include/tissuemc/config.hpp:38-66 and
 * src/cuda/engine.cu:322-350) and report every buffer size. No device is touched. */
TMC_B200_API int tmc_b200_query_sizes(const tmc_run_spec *spec, const tmc_options *opt, tmc_sizes *sizes,
                         tmc_status *status);

/* Run the photon walk on the GPU (replaces tissuemc::run_cuda, src/cuda/engine.cu:322-358). */
TMC_B200_API int tmc_b200_run(const tmc_run_spec *spec, const tmc_options *opt, tmc_result *result,
                 tmc_status *status);

/* Device-resident variant for callers that keep the tallies on the GPU: zeroes the buffer
 * `d_tally` (device memory, tmc_sizes.device_words 64-bit words: the tally_words fixed-point
 * tallies, then the launch's photon-claim counter), runs the walk on `stream` (a cudaStream_t,
 * NULL = the legacy default stream) and returns without synchronising; time it with events on
 * `stream`. Everything the launch writes is in `d_tally`, so calls on different streams into
 * different buffers may run at the same time on the GPU. */
TMC_B200_API int tmc_b200_run_device(const tmc_run_spec *spec, const tmc_options *opt, uint64_t *d_tally,
                        void *stream, tmc_status *status);

/* One shard of a run: walks only photons [first_photon, first_photon + count) of the run that
 * spec and opt describe (each with its own stream (seed, id) and its batch in the run's BatchPlan),
 * into `d_tally` like tmc_b200_run_device. The shards' tally buffers of a partition of [0, photons)
 * add up (unsigned 64-bit sums) to the whole run's buffer bit for bit, so a run spread over several
 * GPUs needs one integer all-reduce of the buffer. No reference counterpart (the reference runs on
 * one GPU, src/cuda/engine.cu:355). */
TMC_B200_API int tmc_b200_run_device_range(const tmc_run_spec *spec, const tmc_options *opt, uint64_t first_photon,
                                           uint64_t count, uint64_t *d_tally, void *stream, tmc_status *status);

/* Convert a raw fixed-point tally buffer (as returned in tmc_result.raw or copied back from
 * tmc_b200_run_device) into the result arrays; pure host code. */
TMC_B200_API int tmc_b200_decode(const tmc_run_spec *spec, const tmc_options *opt, const uint64_t *raw,
                    tmc_result *result, tmc_status *status);

/* Launch and shared-memory plan of a walk: block size, blocks per SM, grid, the shared tiles of
 * A(r,z) (core rows tr_a x depth bins tz_a, plus the clamped last row and column when cross = 1),
 * the shared rows of R_d(r,a) and T_t(r,a), whether the per-batch totals are in shared memory, and
 * the dynamic shared memory per block in bytes. */
typedef struct {
    int32_t threads, blocks_per_sm, grid, tr_a, tz_a, cross, tr_rd, tr_tt, batch_smem, smem_bytes;
} tmc_plan;

/* The plan tmc_b200_run would use on a device with these limits (cudaDeviceProp's
 * multiProcessorCount, sharedMemPerMultiprocessor, sharedMemPerBlockOptin,
 * reservedSharedMemPerBlock) when the register limit allows regs_blocks_per_sm blocks per SM.
 * Pure host code; no device is touched. */
TMC_B200_API int tmc_b200_plan(const tmc_run_spec *spec, const tmc_options *opt, int32_t sms, int64_t smem_per_sm,
                  int64_t smem_per_block_optin, int64_t reserved_per_block, int32_t regs_blocks_per_sm,
                  tmc_plan *plan, tmc_status *status);

/* Autotune the walk's launch and tally-tile plan for this run on its device: time candidate plans
 * (blocks per SM, block size, the shared A(r,z) core tile's shape, the shared rows of R_d(r,a) and
 * T_t(r,a), the shared "cross" of A(r,z)) by coordinate descent on a sample of the run
 * (min(photons, sample_photons) photons, the run's seed and batches), each the best of two timed
 * launches after one warm-up, and write the fastest into opt's threads_per_block, blocks_per_sm,
 * tile_tz, tile_ra_rows and tile_cross. The results of a run do not depend on the plan (integer
 * tallies). plan (optional) receives the chosen plan; default_seconds and best_seconds (optional)
 * the sample's kernel time with the planner's default plan and with the chosen one. Replaces the
 * fixed occupancy sizing of the reference's GPU engine (src/cuda/engine.cu:216-239). */
TMC_B200_API int tmc_b200_autotune(const tmc_run_spec *spec, tmc_options *opt, uint64_t sample_photons,
                                   tmc_plan *plan, double *default_seconds, double *best_seconds,
                                   tmc_status *status);

/* Capacity of the static scratch used by tmc_b200_run_static, in 64-bit tally words (512 KiB). */
#define TMC_B200_STATIC_SCRATCH_WORDS 65536u

/* Run the walk without allocating anything. No counterpart in the reference: it exists for callers
 * that cannot call cudaMalloc — a framework that owns every byte of device memory through its own
 * pool and does not let libraries allocate behind its back, or a plugin host that hands its
 * plugins a fixed memory budget and counts any cudaMalloc against them as a failure. Results are
 * as tmc_b200_run's, bit for bit.
 *
 * The walk's scratch (its photon-claim counter and the fixed-point tally accumulators) lives in a
 * static device array of the library, TMC_B200_STATIC_SCRATCH_WORDS words plus a 256-byte head,
 * which every GPU that loads the library holds until the process exits. Runs whose tally buffer
 * (tmc_sizes.tally_words) is larger are rejected with TMC_BAD_CONFIG. The caller passes every
 * output, including result->raw (tally_words host words), which receives the fixed-point tallies
 * and is then decoded into the other arrays. No cudaMalloc, cudaFree, stream or event creation,
 * and no host-side allocation on success.
 *
 * The first call on a device sets up that device (it looks up the array's device address and
 * raises the kernels' shared-memory limit). Each call clears the parts of the array it uses,
 * runs on the legacy default stream (which waits for, and is waited on by, the blocking streams
 * of the device) and returns when the tallies are in result->raw. The calling thread's current
 * device is the same on return as on entry. Every call shares the one array: calls serialise on
 * the host, and calls that could overlap on the GPU (from other code paths on other streams)
 * would race. kernel_seconds is host time from the launch to the end of the walk (a stream
 * synchronisation), without the copy of the tallies. */
TMC_B200_API int tmc_b200_run_static(const tmc_run_spec *spec, const tmc_options *opt, tmc_result *result,
                                     tmc_status *status);

/* ------------------------------------------------------------------ batched sweep
 * Thousands of independent tissue configurations in one persistent, CUDA-graph-captured launch.
 * No counterpart in the reference (an addition of this engine). Every configuration shares the
 * grid and batch count of the options; each runs its own photons with its own Philox seed, and
 * its tallies are bit for bit those of tmc_b200_run on that configuration alone (same seed,
 * photons, batches, grid and math). */
typedef struct {
    uint64_t photons;          /* >= batches */
    uint64_t seed;             /* Philox key of this configuration's photon streams */
    double n_above, n_below;   /* ambient refractive indices */
    int32_t num_layers;
    tmc_layer layers[TMC_B200_MAX_LAYERS];
} tmc_sweep_config;

typedef struct {
    double dz, dr;             /* grid shared by every configuration */
    int32_t nz, nr, na;
    int32_t batches;           /* per configuration */
    int32_t fast_math;         /* as tmc_options */
    int32_t profiles;          /* 0: totals only */
    int32_t device;
    int32_t threads_per_block; /* 0 = 256 */
    int32_t item_photons;      /* photons per work-queue item; 0 = 256 */
    int32_t tile_r, tile_z;    /* per-warp shared-memory tile of A(r,z): the first tile_r x tile_z
                                  bins of the configuration of the warp's current item (0 x 0 =
                                  none, the default; at most 32 KB of tiles per block) */
} tmc_sweep_options;

typedef struct {
    uint64_t words_per_config;   /* raw tally words per configuration: the single-run layout with
                                    max_layers layer slots in every batch row */
    uint64_t summary_per_config; /* nr + 3: R_d(r) per photon, then R_d, T_t, A per photon */
    int32_t max_layers;
} tmc_sweep_sizes;

/* Options for the sweep workload of this engine's benchmark: grid nr = nz = 64, dr = dz = 0.01 cm,
 * na = 1, 10 batches, fast math, 256 threads, 256 photons per item. */
TMC_B200_API void tmc_b200_sweep_default_options(tmc_sweep_options *opt);

/* Draw n configurations: 1-3 layers sharing one refractive index n ~ U[1.33, 1.5] in air;
 * per layer mua ~ logU[0.01, 10] /cm, reduced scattering mus' ~ logU[1, 50] /cm, g ~ U[0.7, 0.95]
 * (mus = mus' / (1 - g)), thickness ~ logU[0.01, 1] cm; photons ~ logU[1e4, 1e6]; a 64-bit seed
 * per configuration. Draws come from Philox keyed by master_seed with the configuration index in
 * the counter, so configuration c does not depend on n. */
TMC_B200_API int tmc_b200_sweep_sample(uint64_t master_seed, int32_t n, tmc_sweep_config *out, tmc_status *status);

/* Validate every configuration (messages name the configuration) and report buffer sizes. */
TMC_B200_API int tmc_b200_sweep_sizes(const tmc_sweep_config *cfgs, int32_t n, const tmc_sweep_options *opt,
                                      tmc_sweep_sizes *sizes, tmc_status *status);

/* The estimate of the steps a photon of each configuration takes, by which tmc_b200_sweep_run
 * orders the configurations inside its launch (largest first, so that long photons start early);
 * host only, for inspection. cost: n doubles. */
TMC_B200_API int tmc_b200_sweep_costs(const tmc_sweep_config *cfgs, int32_t n, double *cost, tmc_status *status);

/* Run the sweep: one captured graph (table upload, zeroing, the persistent sweep kernel, the
 * per-configuration summary kernel, summary download), cached per device and reused while the
 * shape allows. raw (optional, host): n * words_per_config words; summary (optional, host):
 * n * summary_per_config doubles, both in the order of cfgs; kernel_seconds (optional): device
 * time of the sweep kernel. */
TMC_B200_API int tmc_b200_sweep_run(const tmc_sweep_config *cfgs, int32_t n, const tmc_sweep_options *opt,
                                    uint64_t *raw, double *summary, double *kernel_seconds, tmc_status *status);

/* The baseline the sweep replaces: the same configurations as a loop of single-run launches of
 * the walk kernel on one stream (one launch per configuration). raw (optional) as above;
 * seconds: device time from the first launch to the end of the last. */
TMC_B200_API int tmc_b200_sweep_run_loop(const tmc_sweep_config *cfgs, int32_t n, const tmc_sweep_options *opt,
                                         uint64_t *raw, double *seconds, tmc_status *status);

/* Autotune the sweep's launch shape on these configurations: the caller's options, then block size
 * {128, 256} x photons per work item {64, 256, 1024}, then the per-warp shared tile of A(r,z)
 * {8 x 8, 16 x 16, 16 x 32} with the best of those, each timed on a second run; a candidate
 * replaces the best so far only when it is at least 1.5 % faster. Writes the choice into *opt. */
TMC_B200_API int tmc_b200_sweep_autotune(const tmc_sweep_config *cfgs, int32_t n, tmc_sweep_options *opt,
                                         double *best_seconds, tmc_status *status);

/* ------------------------------------------------------------------ tensor-core GEMM
 * D = A * B^T (+ bias) on the tcgen05 tensor cores: A is M x K and B is N x K, BF16, row-major with
 * K contiguous; D is M x N float32 row-major; bias (optional) has N entries; K a positive multiple
 * of 64. All pointers are device memory of the current device; runs on `stream` and synchronises
 * it. No counterpart in the reference (the surrogate's building block). TMC_DEVICE_TIMEOUT if a
 * bounded tensor-core wait gave up. */
TMC_B200_API int tmc_b200_gemm_bf16(const uint16_t *A, const uint16_t *B, const float *bias, float *D, int32_t M,
                                    int32_t N, int32_t K, void *stream, tmc_status *status);

/* Test of a bounded device wait that gives up (no counterpart in the reference). Runs the GEMM
 * kernel above on one 128 x 128 x 64 product (a few KB of device memory, allocated and freed here)
 * with its producer told to issue no loads, so that the MMA issuer's wait on a stage nobody fills
 * runs out after wait_limit polls (1 .. the production limit) with no copy and no MMA outstanding.
 * The kernel then skips its epilogue, frees its tensor memory and raises its status word. Returns
 * TMC_DEVICE_TIMEOUT when the status word reported the give-up (the expected result), TMC_OK if it
 * did not; the device stays usable either way. Synchronous. */
TMC_B200_API int tmc_b200_probe_wait_timeout(int32_t device, uint32_t wait_limit, tmc_status *status);

/* ------------------------------------------------------------------ surrogate network ops
 * The learned surrogate's building blocks (no counterpart in the reference). Device pointers of
 * the current device; launched on `stream` without synchronising, so a training step can be
 * captured in a CUDA graph. Matrices are row-major; "bf16" buffers are uint16_t bit patterns.
 * Every product runs on the tcgen05 tensor cores with FP32 accumulation (K multiple of 64).
 *
 * linear:        Z = X W^T + b (float32, optional), H = gelu(Z) or Z (bf16, optional), HT = H^T
 *                (bf16, N x M, optional: the operand of the weight gradient, written by the same
 *                kernel); X: M x K, W: N x K, b: N.
 * backward_data: dX = (dZ WT^T) * gelu'(Zprev) (bf16) and dXT = dX^T (N x M, optional); dZ: M x K,
 *                WT: N x K (the transposed weight, N = the layer's inputs), Zprev: M x N.
 * matmul_f32:    D = A B^T (float32); A: M x K, B: N x K (weight gradients from transposed
 *                activations).
 * matmul_f32_splitk: the same with K cut into `splits` equal ranges computed by separate CTAs
 *                (K / 64 a multiple of splits) into work (splits x M x N floats), then summed into
 *                D in a fixed order (deterministic); for long K and small M x N.
 * transpose:     Y = X^T for a rows x cols bf16 matrix.
 * colsum:        db[n] = sum_m dZ[m][n] (float32, overwritten), in a fixed order (deterministic)
 *                through `work`, which holds tmc_b200_nn_colsum_work(N) floats.
 * mse:           loss += scale * sum (pred - target)^2 over the first T of ld columns; dZ (bf16,
 *                optional) = 2 scale (pred - target), zero in the padded columns.
 * adam:          one Adam step on float32 master weights, writing the bf16 copy wb and its
 *                transpose wt (each optional). The bias-corrected step size is lr_t, or lr_dev[0]
 *                when lr_dev (device memory) is given, so that a captured CUDA graph reads each
 *                step's value; with avg given, avg = avg_beta avg + (1 - avg_beta) w afterwards
 *                (Polyak averaging fused into the step, the same bits as the separate ema).
 * adam_plan:     fill first_block of each tmc_adam_tensor of a host table (in order) and return
 *                the blocks a launch over all of them needs (-1 on an empty or invalid table).
 * adam_multi:    the adam step for every tensor of a planned table in one launch; `tab` is the
 *                table copied to device memory, `blocks` what adam_plan returned; each tensor's
 *                optional pointers (wb, wt, avg) may be NULL. The same bits as one adam call per
 *                tensor.
 * ema:           avg = beta avg + (1 - beta) w over n float32 values (Polyak averaging).
 * to_bf16:       wb = bf16(w) and wt = its transpose (each optional) for a rows x cols matrix.
 * status:        nonzero if a bounded tensor-core wait gave up since the last clear. */
TMC_B200_API int tmc_b200_nn_linear(const uint16_t *X, const uint16_t *W, const float *bias, float *Z, uint16_t *H,
                                    uint16_t *HT, int32_t M, int32_t N, int32_t K, int32_t gelu, void *stream,
                                    tmc_status *status);
TMC_B200_API int tmc_b200_nn_backward_data(const uint16_t *dZ, const uint16_t *WT, const float *Zprev, uint16_t *dX,
                                           uint16_t *dXT, int32_t M, int32_t N, int32_t K, void *stream,
                                           tmc_status *status);
TMC_B200_API int tmc_b200_nn_matmul_f32(const uint16_t *A, const uint16_t *B, float *D, int32_t M, int32_t N,
                                        int32_t K, void *stream, tmc_status *status);
TMC_B200_API int tmc_b200_nn_matmul_f32_splitk(const uint16_t *A, const uint16_t *B, float *D, float *work,
                                               int32_t M, int32_t N, int32_t K, int32_t splits, void *stream,
                                               tmc_status *status);
TMC_B200_API int tmc_b200_nn_transpose(const uint16_t *X, uint16_t *Y, int32_t rows, int32_t cols, void *stream,
                                       tmc_status *status);
TMC_B200_API int tmc_b200_nn_colsum(const uint16_t *dZ, float *db, int32_t M, int32_t N, float *work,
                                    void *stream, tmc_status *status);
TMC_B200_API int32_t tmc_b200_nn_colsum_work(int32_t N);
TMC_B200_API int tmc_b200_nn_mse(const float *pred, const float *target, uint16_t *dZ, float *loss, int32_t M,
                                 int32_t T, int32_t ld, float scale, void *stream, tmc_status *status);
TMC_B200_API int tmc_b200_nn_adam(float *w, const float *g, float *m, float *v, int32_t rows, int32_t cols,
                                  float lr_t, const float *lr_dev, float b1, float b2, float eps, float weight_decay,
                                  uint16_t *wb, uint16_t *wt, float *avg, float avg_beta, void *stream,
                                  tmc_status *status);
/* One parameter tensor of a many-tensor Adam step (device pointers; rows x cols float32). */
typedef struct {
    float *w;
    const float *g;
    float *m;
    float *v;
    uint16_t *wb;  /* bf16 copy (optional) */
    uint16_t *wt;  /* its transpose (optional) */
    float *avg;    /* Polyak average (optional) */
    int32_t rows, cols;
    float weight_decay;
    int32_t first_block; /* filled by tmc_b200_nn_adam_plan */
} tmc_adam_tensor;
TMC_B200_API int32_t tmc_b200_nn_adam_plan(tmc_adam_tensor *tab, int32_t count);
TMC_B200_API int tmc_b200_nn_adam_multi(const tmc_adam_tensor *tab, int32_t count, int32_t blocks, float lr_t,
                                        const float *lr_dev, float b1, float b2, float eps, float avg_beta,
                                        void *stream, tmc_status *status);
TMC_B200_API int tmc_b200_nn_ema(const float *w, float *avg, int64_t n, float beta, void *stream, tmc_status *status);
TMC_B200_API int tmc_b200_nn_to_bf16(const float *w, int32_t rows, int32_t cols, uint16_t *wb, uint16_t *wt,
                                     void *stream, tmc_status *status);
TMC_B200_API int tmc_b200_nn_status(int32_t clear);
/* encode: X (n x ld, bf16) = z-scored feats (n x nf, float32), zero-padded to ld columns.
 * gate:   per query, each member's diffuse reflectance on the grid from its normalised outputs
 *         Z[m] (n x ld float32, members member_stride elements apart), de-normalised with ymean,
 *         ystd (log10 R_d(r) per area in the first nbins columns) and weighted by the annulus
 *         areas; rd_mean (optional) gets the members' mean, spread (optional) their sample standard
 *         deviation over the mean, and route[q] = 1 when the spread exceeds threshold (the query
 *         goes to Monte Carlo). */
TMC_B200_API int tmc_b200_nn_encode(const float *feats, const float *mean, const float *stdv, uint16_t *X, int32_t n,
                                    int32_t nf, int32_t ld, void *stream, tmc_status *status);
TMC_B200_API int tmc_b200_nn_gate(const float *Z, int32_t members, int64_t member_stride, int32_t ld,
                                  const float *ymean, const float *ystd, const float *areas, int32_t nbins, int32_t n,
                                  float threshold, float *rd_mean, float *spread, uint8_t *route, void *stream,
                                  tmc_status *status);

/* Fused ensemble inference (serving): one persistent tcgen05 kernel runs all members of the
 * surrogate (64 -> 4 x 512 GELU -> 128, BF16 operands, FP32 accumulation in tensor memory) on
 * tiles of 128 queries, keeping activations on chip, and applies the gate above.
 *   packed_bytes: size of the packed weight stream for `members` networks (1,769,472 bytes each).
 *   pack:    weights[m * 5 + l] is member m's layer-l BF16 weight matrix (device, row-major, rows x
 *            cols = 512 x 64, 512 x 512 three times, 128 x 512; inputs zero-padded to 64 columns,
 *            outputs to 128 rows); the host array of pointers is read during the call. Re-pack after
 *            every weight update.
 *   infer:   bias = members x 2176 floats (the five bias vectors of each member, concatenated);
 *            feats = n x n_feat raw features, z-scored with x_mean / x_std; outputs de-normalised
 *            with y_mean / y_std; out (optional) = n x n_out ensemble mean; rd_mean, spread and
 *            route (optional) as in tmc_b200_nn_gate over the first nbins outputs. Asynchronous on
 *            `stream`; a bounded tensor-core wait that gives up raises tmc_b200_nn_status. */
TMC_B200_API int64_t tmc_b200_nn_packed_bytes(int32_t members);
TMC_B200_API int tmc_b200_nn_pack(const uint16_t *const *weights, int32_t members, uint8_t *packed, void *stream,
                                  tmc_status *status);
TMC_B200_API int tmc_b200_nn_ensemble_infer(const uint8_t *packed, const float *bias, int32_t members,
                                            const float *feats, int32_t n, int32_t n_feat, const float *x_mean,
                                            const float *x_std, int32_t n_out, const float *y_mean,
                                            const float *y_std, const float *areas, int32_t nbins, float threshold,
                                            float *out, float *rd_mean, float *spread, uint8_t *route, void *stream,
                                            tmc_status *status);

/* Physics probe: the walk's own device functions in isolation, on many Philox streams keyed by
 * (seed, thread), for unit tests of the GPU physics (TissueMC checks its CPU physics the same way,
 * tests/cpp/test_physics.cpp:91-160). One layer with anisotropy g and attenuation mu_t [1/cm];
 * fast_math as in tmc_options. out[5] (host): what 0 = Henyey-Greenstein cosines: sum, sum of
 * squares, min, max; what 1 = consecutive direction rotations (32 chains): worst |norm - 1|;
 * what 2 = free paths: sum, sum of squares. out[4] = the samples drawn (samples rounded up to a
 * multiple of the threads). No reference counterpart; allocates a 32-byte device buffer. */
TMC_B200_API int tmc_b200_probe_physics(int32_t what, double g, double mu_t, int64_t samples, uint64_t seed,
                                        int32_t fast_math, int32_t device, double *out, tmc_status *status);

/* Parse an MCML .mci file (the reference's parse_mci_file, src/io/mci.cpp:173-183): writes up to
 * `max_runs` runs and returns the number found in *n_runs. Errors carry the line number. */
TMC_B200_API int tmc_b200_parse_mci(const char *path, tmc_run_spec *runs, int32_t max_runs, int32_t *n_runs,
                       tmc_status *status);

/* Write a finished run as an MCML output file (.mco: InParm, RAT, A_l, A_z, Rd_r, Rd_a, Tt_r, Tt_a,
 * A_rz, Rd_ra, Tt_ra, scaled per area, solid angle and volume as the MCML manual defines them).
 * `result` must carry the batch totals and the optional 2-D arrays a_rz, rd_ra and tt_ra. No
 * reference counterpart: TissueMC writes JSON only (src/io/result.cpp). Pure host code. */
TMC_B200_API int tmc_b200_write_mco(const tmc_run_spec *spec, const tmc_options *opt, const tmc_result *result,
                                    const char *path, tmc_status *status);

#ifdef __cplusplus
}
#endif

#endif /* TISSUEMC_B200_H */
