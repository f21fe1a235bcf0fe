/*
 * vsmc_cuda.h -- C ABI of libvsmc_cuda, the B200 (sm_100a) SMC step.
 *
 * Plain pointers, sizes and status codes only.  Every entry point names the
 * vSMC interface it replaces (paths relative to the vSMC project root).
 * Device pointers are CUDA global-memory addresses on the current device;
 * `stream` is a cudaStream_t (NULL = legacy default stream).
 *
 * Errors: every function returns VSMC_CUDA_OK (0) or one of the codes below;
 * vsmc_cuda_last_error() gives the calling thread's last message.  This
 * replaces VSMC_RUNTIME_ASSERT (include/vsmc/internal/assert.hpp:60-99);
 * the C++ facade (include/vsmc_b200/vsmc.hpp) turns codes into exceptions.
 */
#ifndef VSMC_CUDA_H
#define VSMC_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VSMC_CUDA_ABI_VERSION 1

enum vsmc_cuda_status {
    VSMC_CUDA_OK = 0,
    VSMC_CUDA_EINVAL = 1,      /* bad argument (size, scheme, null pointer) */
    VSMC_CUDA_ENOMEM = 2,      /* device allocation or HBM budget exceeded */
    VSMC_CUDA_EDEGENERATE = 3, /* all log-weights -inf, or NaN/inf weights */
    VSMC_CUDA_ETIMEOUT = 4,    /* a bounded device-side wait gave up */
    VSMC_CUDA_ECUDA = 5        /* CUDA runtime error (message has details) */
};

/* Same values as vsmc::ResampleScheme (include/vsmc/resample/common.hpp:
 * 124-131). */
enum vsmc_cuda_scheme {
    VSMC_CUDA_MULTINOMIAL = 0,
    VSMC_CUDA_RESIDUAL = 1,
    VSMC_CUDA_STRATIFIED = 2,
    VSMC_CUDA_SYSTEMATIC = 3,
    VSMC_CUDA_RESIDUAL_STRATIFIED = 4,
    VSMC_CUDA_RESIDUAL_SYSTEMATIC = 5
};

/* Precision forms of the particle move. */
enum vsmc_cuda_form {
    VSMC_CUDA_FP64 = 0, /* everything in double (the reference's layout) */
    VSMC_CUDA_MIXED = 1 /* float state, move and log-weights; double
                           cumulative-weight scan and log-evidence */
};

const char *vsmc_cuda_status_string(int status);
const char *vsmc_cuda_last_error(void);
int vsmc_cuda_abi_version(void);

/* ------------------------------------------------------ device memory --- */

/* Plain device memory for callers built without the CUDA toolkit (the C++
 * interface in include/vsmc_b200/vsmc_cuda.hpp): cudaMalloc, cudaFree, and a
 * cudaMemcpyAsync on `stream` that returns once the copy is done.  No
 * counterpart in the reference (host memory only). */
enum {
    VSMC_CUDA_HOST_TO_DEVICE = 1,
    VSMC_CUDA_DEVICE_TO_HOST = 2,
    VSMC_CUDA_DEVICE_TO_DEVICE = 3
};

int vsmc_cuda_device_alloc(size_t bytes, void **ptr);
int vsmc_cuda_device_free(void *ptr);
int vsmc_cuda_memcpy(void *dst, const void *src, size_t bytes, int kind,
                     void *stream);
int vsmc_cuda_stream_synchronize(void *stream);

/* ------------------------------------------------------------- RNG ------ */

/* n successive outputs of PhiloxEngine<uint32_t,4,10>::operator()() after
 * key(key), ctr(ctr) and `skip` discarded draws, written to device `out`.
 * Replaces include/vsmc/rng/philox.hpp:367-395 (ctr/key/operator()). */
int vsmc_cuda_philox4x32_words(const uint32_t key[2], const uint32_t ctr[4],
                               uint64_t skip, uint64_t n, uint32_t *out,
                               void *stream);

/* Same for ThreefryEngine<uint64_t,4,20> (include/vsmc/rng/threefry.hpp:
 * 336-364). */
int vsmc_cuda_threefry4x64_words(const uint64_t key[4], const uint64_t ctr[4],
                                 uint64_t skip, uint64_t n, uint64_t *out,
                                 void *stream);

/* Position of a Threefry4x64 resample engine: the next word drawn is lane
 * (offset % 4) of block ctr + offset / 4 + 1.  A freshly seeded engine
 * (Threefry4x64(s)) is {key = {s,0,0,0}, ctr = 0, offset = 0}. */
typedef struct {
    uint64_t key[4];
    uint64_t ctr[4];
    uint64_t offset;
} vsmc_cuda_threefry_state;

/* ------------------------------------------------------------ weights --- */

/* WeightSet::set_log_weight (inc == NULL) or add_log_weight(inc) on device
 * arrays: log_weight += inc; log_weight -= max; weight = exp(log_weight) /
 * sum; *ess = 1 / sum(weight^2).  log_weight is updated in place (max-
 * normalised, as the reference stores it); weight may be NULL.  Blocks until
 * *ess is known.  Replaces include/vsmc/core/weight_set.hpp:297-331 and
 * post_set_log_weight :441-446. */
int vsmc_cuda_weight_add_log(uint64_t N, double *log_weight, double *weight,
                             const double *inc, double *ess, void *stream);

/* WeightSet::ess(first, use_log) (core/weight_set.hpp:132-146 and
 * compute_ess :385-409): the ESS the weights would have after an update by
 * the N incremental weights `inc` (device), without changing them.  With
 * use_log, inc are log increments added to the max-normalised log_weight;
 * otherwise inc multiply the normalised `weight`.  Blocks. */
int vsmc_cuda_weight_ess(uint64_t N, const double *log_weight,
                         const double *weight, const double *inc, int use_log,
                         double *ess, void *stream);

/* WeightSet::cess(first, use_log) (core/weight_set.hpp:160-174 and
 * compute_cess :411-431): the conditional ESS (sum W b)^2 / sum W b^2 of the
 * normalised `weight` and the incremental weights b = inc (or exp(inc) with
 * use_log), device arrays of N.  Blocks. */
int vsmc_cuda_weight_cess(uint64_t N, const double *weight, const double *inc,
                          int use_log, double *cess, void *stream);

/* ----------------------------------------------------------- resample --- */

/* Bytes of device workspace vsmc_cuda_resample needs for N particles. */
size_t vsmc_cuda_resample_workspace_size(uint64_t N);

/* Resample<Scheme>::operator()(N, N, rng, weight, replication) followed by
 * internal::cfrp_trans(N, N, replication, copy_from) (include/vsmc/resample/
 * *.hpp, common.hpp:57-118; Particle::resample, core/particle.hpp:230-250).
 *
 * weight: N normalised weights (device).  replication, copy_from: N int32
 * (device; copy_from may be NULL).  rng: the resample engine position; on
 * return it has advanced by exactly the words the reference would draw.
 * uniforms: NULL to draw the U01 sequence from rng on the device (bit-exact
 * words; the Multinomial sequence goes through log/exp and so matches to a
 * few ulps), or a device array of the sequence values u_0..u_{k-1} that the
 * reference's inversion would query (parity mode; k = n_uniforms, entries
 * beyond k are taken as +inf).  Blocks until the engine position is known.
 */
int vsmc_cuda_resample(int scheme, uint64_t N, const double *weight,
                       const double *uniforms, uint64_t n_uniforms,
                       vsmc_cuda_threefry_state *rng, int32_t *replication,
                       int32_t *copy_from, void *workspace,
                       size_t workspace_bytes, void *stream);

/* Bytes of device workspace vsmc_cuda_resample_mn needs. */
size_t vsmc_cuda_resample_mn_workspace_size(uint64_t M, uint64_t N);

/* Resample<Scheme>::operator()(M, N, rng, weight, replication) followed by
 * internal::cfrp_trans(M, N, replication, copy_from) for M weights and N
 * children (include/vsmc/resample/multinomial.hpp to residual_systematic.hpp;
 * common.hpp:57-118): replication has M entries
 * summing to N; copy_from (N entries, may be NULL) is, for M != N, the
 * cfrp_trans expansion (parent i repeated replication[i] times, in order)
 * and for M == N the same as vsmc_cuda_resample.  M >= 1; N = 0 leaves every
 * count at zero (a Systematic engine still draws its one word).  uniforms /
 * n_uniforms as vsmc_cuda_resample, with up to N values.  The engine
 * advances by exactly the words the reference draws.  Blocks until done. */
int vsmc_cuda_resample_mn(int scheme, uint64_t M, uint64_t N,
                          const double *weight, const double *uniforms,
                          uint64_t n_uniforms, vsmc_cuda_threefry_state *rng,
                          int32_t *replication, int32_t *copy_from,
                          void *workspace, size_t workspace_bytes,
                          void *stream);

/* Largest N accepted by vsmc_cuda_resample_noalloc. */
#define VSMC_CUDA_NOALLOC_MAX_N 262144

/* No counterpart in the reference.  vsmc_cuda_resample for callers that
 * cannot allocate device memory (a fixed HBM budget reserved up front, loops
 * where cudaMalloc/cudaFree would synchronise the device, or a plugin whose
 * host owns every allocation): the same kernels and results, with the
 * workspace (and the copy_from scratch when copy_from is NULL) taken from a
 * static device array the library holds for N <= VSMC_CUDA_NOALLOC_MAX_N
 * particles (about 7.4 MiB on every device that loads the library, kept
 * until exit).  Larger N returns VSMC_CUDA_EINVAL.  It calls no cudaMalloc
 * or cudaFree.  The first call on each device looks up the array's device
 * address (cudaGetSymbolAddress, with that device current) and caches it
 * with the device's current context (a context created anew, e.g. after
 * cudaDeviceReset, is looked up again); make that first call before any
 * stream capture.  Every call waits for `stream` before it returns (it reads
 * the engine position back).  All calls share the array: calls that overlap
 * on the GPU race and must be serialised by the caller. */
int vsmc_cuda_resample_noalloc(int scheme, uint64_t N, const double *weight,
                               const double *uniforms, uint64_t n_uniforms,
                               vsmc_cuda_threefry_state *rng,
                               int32_t *replication, int32_t *copy_from,
                               void *stream);

/* StateMatrix<ColMajor, dim, double>::copy(N, copy_from)
 * (include/vsmc/core/state_matrix.hpp:378-394): dst[d*N + i] =
 * src[d*N + copy_from[i]] for every column d (src != dst). */
int vsmc_cuda_copy_f64(uint64_t N, uint32_t dim, const double *src,
                       double *dst, const int32_t *copy_from, void *stream);

/* The library's FP64 natural logarithm (fn 0) and exponential (fn 1) --
 * the table-driven functions its kernels evaluate the move, the weights and
 * the sorted U01 sequence with (include/vsmc_b200/fastmath.cuh) -- on n
 * device values: out[i] = f(in[i]).  For checking them against other
 * implementations. */
int vsmc_cuda_math_eval(int fn, uint64_t n, const double *in, double *out,
                        void *stream);

/* ------------------------------------------------ CV Student-t filter ---- */

/* The constant-velocity Student-t bootstrap filter of example/pf
 * (include/pf_smp.hpp:73-258) as one device-resident object: Sampler<T>
 * with a StateMatrix<ColMajor,4> value, a Philox4x32 per-particle stream
 * (counter {block, step, id, stream_id}, key {seed+1, 0}) and the default
 * Threefry4x64 resample engine seeded seed+2 (Seed::set(seed) semantics,
 * include/vsmc/rng/seed.hpp:102,149; core/particle.hpp:64-70). */
typedef struct vsmc_cuda_cv_filter vsmc_cuda_cv_filter;

typedef struct {
    uint64_t N;          /* particles */
    uint64_t T_max;      /* capacity of the observation / history arrays */
    int scheme;          /* vsmc_cuda_scheme */
    int form;            /* vsmc_cuda_form */
    double threshold;    /* resample when ESS < threshold * N */
    uint32_t seed;       /* Seed::set(seed) */
    uint32_t stream_id;  /* 4th counter word, distinguishes filters */
    double dt, sd_pos, sd_vel, sd_pos0, sd_vel0, scale, nu;
} vsmc_cuda_cv_config;

/* N = 0, T_max = 0, Multinomial, FP64, threshold 0.5, seed 101, stream 0,
 * dt 0.1, sd_pos 0.02, sd_vel 0.5, sd_pos0 2, sd_vel0 1, scale 10, nu 10. */
void vsmc_cuda_cv_config_default(vsmc_cuda_cv_config *cfg);

/* Device bytes a filter with this configuration allocates. */
size_t vsmc_cuda_cv_device_bytes(const vsmc_cuda_cv_config *cfg);

/* Sampler<T>(N, scheme, threshold) (core/sampler.hpp:80-104).  All device
 * memory is allocated here; later calls allocate nothing.  A Multinomial
 * filter also creates a second, internal stream: the sorted U01 sequence of
 * the next resampling (which depends only on N and the engine position) is
 * drawn there while the step's move runs; it writes only the filter's own
 * workspace, and the filter's stream waits for it where it is read.  After
 * an iterate of more than one step the filter's stream also waits for the
 * sequence it left running. */
int vsmc_cuda_cv_create(const vsmc_cuda_cv_config *cfg, void *stream,
                        vsmc_cuda_cv_filter **out);
int vsmc_cuda_cv_destroy(vsmc_cuda_cv_filter *f);

/* Observations y_0..y_{T-1} (x and y coordinates), host or device memory
 * (cv_state::read_data, pf_smp.hpp:114-125).  Host arrays are copied
 * asynchronously on the filter's stream (pinned memory recommended). */
int vsmc_cuda_cv_set_observations(vsmc_cuda_cv_filter *f, const double *obs_x,
                                  const double *obs_y, uint64_t T,
                                  int on_device);

/* Sampler::initialize (core/sampler.hpp:450-463): reset histories, draw the
 * prior, weight by y_0, possibly resample.  Asynchronous. */
int vsmc_cuda_cv_initialize(vsmc_cuda_cv_filter *f);

/* Sampler::iterate(num) (core/sampler.hpp:471-483): num steps of move,
 * weight update, ESS test and resampling, monitor.  Asynchronous. */
int vsmc_cuda_cv_iterate(vsmc_cuda_cv_filter *f, uint64_t num);

/* Waits for the filter's stream and reports sticky device-side errors
 * (VSMC_CUDA_EDEGENERATE, VSMC_CUDA_ETIMEOUT). */
int vsmc_cuda_cv_synchronize(vsmc_cuda_cv_filter *f);

/* Number of completed steps (Sampler::iter_size). */
int vsmc_cuda_cv_iter_size(vsmc_cuda_cv_filter *f, uint64_t *iter_size);

/* Histories (host arrays of iter_size entries, each may be NULL):
 * Sampler::ess_history / resampled_history (core/sampler.hpp:293-307), the
 * per-step log-evidence increments (example/include/move_smc.hpp:63-71) and
 * the MonitorMCMC-stage importance-sampling estimates of the position
 * (Monitor::record, core/monitor.hpp:181-217).  Synchronises. */
int vsmc_cuda_cv_history(vsmc_cuda_cv_filter *f, double *ess,
                         int32_t *resampled, double *logz_inc, double *mean_x,
                         double *mean_y);

/* Monitor::eval of the last step (core/sampler.hpp:825-834) when that step
 * resampled: its posterior mean is taken over the gathered parents, which
 * the next move gathers anyway, so iterate leaves it to that move or to
 * this call (vsmc_cuda_cv_history makes it too).  Asynchronous; enqueues two
 * kernels that return at once when there is nothing to complete. */
int vsmc_cuda_cv_complete_monitor(vsmc_cuda_cv_filter *f);

/* Running log-evidence sum (host scalar).  Synchronises. */
int vsmc_cuda_cv_log_evidence(vsmc_cuda_cv_filter *f, double *logz);

/* Current particles in double, SoA host arrays of N (each may be NULL), and
 * the max-normalised log-weights (WeightSet::read_log_weight,
 * core/weight_set.hpp:199-211).  Synchronises. */
int vsmc_cuda_cv_read_state(vsmc_cuda_cv_filter *f, double *x, double *y,
                            double *vx, double *vy, double *log_weight);

/* Appends n observations after the ones already set (streaming use: one
 * per step as it arrives).  Host arrays are copied asynchronously on the
 * filter's stream and must stay valid until the stream reaches the copy. */
int vsmc_cuda_cv_append_observations(vsmc_cuda_cv_filter *f,
                                     const double *obs_x, const double *obs_y,
                                     uint64_t n, int on_device);

/* Enqueues device-to-host copies of step t's ESS, log-evidence increment and
 * resampled flag (each pointer may be NULL).  With synchronize != 0 it waits
 * and reports sticky device errors; otherwise the values are valid after
 * the filter's stream reaches the copies. */
int vsmc_cuda_cv_read_step(vsmc_cuda_cv_filter *f, uint64_t t, double *ess,
                           double *logz_inc, int32_t *resampled,
                           int synchronize);

/* Fixed-ancestry runs (precision comparisons, trajectory replay).  With
 * `record` (device, T_max x N int32) every step stores its copy_from in row
 * t (meaningful where the step resampled).  With `replay` (device, T_max x N)
 * and `replay_resampled` (device, T_max int32) the filter skips its own
 * resampling: step t resamples iff replay_resampled[t] != 0 and then takes
 * row t as copy_from, so a run in another precision form follows exactly
 * the recorded ancestry.  With all three, the filter follows `replay` and
 * still resamples on each step's own decision, writing its own copy_from
 * into row t of `record` (the engine advances by the words it draws): the
 * step-by-step comparison of the device's resampling with another run's
 * (the reference's) on a shared trajectory.  Pass NULLs to turn either off.
 * The arrays stay owned by the caller and must outlive the steps that use
 * them. */
int vsmc_cuda_cv_set_ancestry(vsmc_cuda_cv_filter *f, int32_t *record,
                              const int32_t *replay,
                              const int32_t *replay_resampled);

/* Kernel timing with CUDA events on the filter's stream.  While enabled,
 * every step records events around the move kernel and around the whole
 * step; vsmc_cuda_cv_timing returns the summed milliseconds of the move
 * kernels and of whole steps, and the number of steps, since enabling (it
 * synchronises).  *launches counts this library's kernel launches. */
int vsmc_cuda_cv_set_timing(vsmc_cuda_cv_filter *f, int enable);
int vsmc_cuda_cv_timing(vsmc_cuda_cv_filter *f, double *move_ms,
                        double *step_ms, uint64_t *steps, uint64_t *launches);

/* The workload's observation series: state (0,0,1,1), the configuration's
 * constant-velocity dynamics, positions plus Student-t(nu)/scale noise; step
 * t draws from Philox4x32-10 with key {obs_seed, 1} and counter
 * {0, t, 0, cfg->stream_id} through std::normal_distribution.  Host arrays;
 * truth (T x 4) may be NULL.  No device is used. */
int vsmc_cuda_cv_simulate(const vsmc_cuda_cv_config *cfg, uint32_t obs_seed,
                          uint64_t T, double *obs_x, double *obs_y,
                          double *truth);

/* Words drawn so far by the resample engine (Threefry4x64 offset). */
int vsmc_cuda_cv_resample_words(vsmc_cuda_cv_filter *f, uint64_t *words);

/* The filter's last copy_from vector (host, N int32) and whether the last
 * step resampled.  Synchronises. */
int vsmc_cuda_cv_copy_from(vsmc_cuda_cv_filter *f, int32_t *copy_from,
                           int32_t *resampled);

/* ---- the model-independent core of a device Sampler ---------------------
 *
 * For particle moves the caller compiles itself (nvcc, sm_100a) against
 * include/vsmc_b200/smc_device.cuh; include/vsmc_b200/smc.cuh wraps it as
 * vsmc::Sampler<T> with MoveCUDA / InitializeCUDA / MonitorEvalCUDA
 * functors.  The core holds what the reference's Sampler<T> keeps apart from
 * the value: the WeightSet (core/weight_set.hpp:96-454) as raw device
 * log-weights, the resample engine and Particle::resample's copy_from
 * (core/particle.hpp:230-250), and the ESS / resampled / accept histories
 * (core/sampler.hpp:725-741).  A step is the caller's kernels followed by
 * vsmc_cuda_smc_finish_step: normalisation, ESS, the log-evidence increment
 * (example/include/move_smc.hpp:63-71), the decision ESS < threshold * N
 * and the scheme's resampling, all on the device.
 *
 * Contract of a step's move kernel (what vsmc_cuda_smc_step describes): for
 * every particle i, with parent p = copy_from[i] if *resampled (the previous
 * step resampled; 0 <= p < N) else i, the move reads the parent's state,
 * writes particle i's new state, and sets log_weight[i] to
 *   (the previous step's log-weight, 0 after a resampling, else
 *    log_weight[i] - *lw_max) + the step's log-weight increment,
 * and writes one vsmc_b200::TileStats per tile of VSMC_CUDA_SMC_TILE
 * particles (the online log-sum-exp of its new log-weights).  The first step
 * (iter 0, Sampler::initialize) sets log_weight[i] to its increment. */
#define VSMC_CUDA_SMC_TILE 2048     /* particles per TileStats */
#define VSMC_CUDA_SMC_MAX_QUEUE 16  /* accept counters per step */

typedef struct vsmc_cuda_smc vsmc_cuda_smc;

typedef struct {
    uint64_t N;               /* particles */
    uint64_t ntiles;          /* tiles of VSMC_CUDA_SMC_TILE particles */
    uint64_t iter;            /* the step the next kernels compute */
    double *log_weight;       /* N raw log-weights (device) */
    const double *lw_max;     /* device: maximum raw log-weight of the last
                                 finished step (subtracted when it did not
                                 resample: WeightSet's max-normalisation) */
    const double *weight_s1;  /* device: sum exp(lw - lw_max) of that step */
    const int32_t *resampled; /* device flag: the last finished step
                                 resampled */
    const int32_t *copy_from; /* device: N parents of that resampling */
    void *tile_stats;         /* device: ntiles vsmc_b200::TileStats */
    uint64_t *accept;         /* device counters, step t, queue position k:
                                 accept[t * VSMC_CUDA_SMC_MAX_QUEUE + k]
                                 (Sampler::accept_history) */
    void *stream;             /* the core's cudaStream_t */
} vsmc_cuda_smc_step;

/* Sampler<T>(N, scheme, threshold)'s weight set and resampling for up to
 * T_max steps; the resample engine is Threefry4x64(resample_seed) (the
 * reference seeds it with the Seed::get() after the particle engines').
 * All device memory is allocated here. */
int vsmc_cuda_smc_create(uint64_t N, uint64_t T_max, int scheme,
                         double threshold, uint32_t resample_seed,
                         void *stream, vsmc_cuda_smc **out);
int vsmc_cuda_smc_destroy(vsmc_cuda_smc *s);

/* Sampler::initialize's reset (core/sampler.hpp:764-776): step 0, equal
 * weights, histories and accept counters cleared, running log-evidence 0;
 * the resample engine keeps its position.  Asynchronous. */
int vsmc_cuda_smc_reset(vsmc_cuda_smc *s);

/* The device pointers and step number a move kernel of the next step uses. */
int vsmc_cuda_smc_step_args(vsmc_cuda_smc *s, vsmc_cuda_smc_step *out);

/* Ends the step the kernels computed: Sampler::do_resample
 * (core/sampler.hpp:816-822) on the device.  Asynchronous. */
int vsmc_cuda_smc_finish_step(vsmc_cuda_smc *s);

/* Waits for the core's stream; reports sticky device errors. */
int vsmc_cuda_smc_synchronize(vsmc_cuda_smc *s);

int vsmc_cuda_smc_iter_size(vsmc_cuda_smc *s, uint64_t *iter_size);

/* Histories of the finished steps (host arrays of iter_size entries; accept
 * has iter_size x VSMC_CUDA_SMC_MAX_QUEUE; each may be NULL): ESS,
 * resampled flags, log-evidence increments, accept counts.  Synchronises. */
int vsmc_cuda_smc_history(vsmc_cuda_smc *s, double *ess, int32_t *resampled,
                          double *logz_inc, uint64_t *accept);

/* Running log-evidence sum.  Synchronises. */
int vsmc_cuda_smc_log_evidence(vsmc_cuda_smc *s, double *logz);

/* WeightSet::read_weight / read_log_weight after the last step (equal
 * weights when it resampled); host arrays of N, each may be NULL.
 * Synchronises. */
int vsmc_cuda_smc_read_weights(vsmc_cuda_smc *s, double *weight,
                               double *log_weight);

/* Words drawn so far by the resample engine. */
int vsmc_cuda_smc_resample_words(vsmc_cuda_smc *s, uint64_t *words);

/* Kernel launches the core has issued. */
int vsmc_cuda_smc_launches(vsmc_cuda_smc *s, uint64_t *launches);

/* ---- many filters on one device (batched runs and serving) -------------
 *
 * No counterpart in the reference, which runs one Sampler per filter
 * (core/sampler.hpp:450-483) and leaves many-filter programs to loop over
 * them.  A batch holds up to `capacity` constant-velocity filters in slots.
 * Each slot keeps its particles, weights, RNG counters, resampling state,
 * observations and histories resident in device memory (one allocation
 * from the batch's own memory pool, admitted against `hbm_budget` bytes;
 * 0 = no limit).  The scheme, form, threshold and model parameters come
 * from `model` and are shared by every slot; N, T_max, seed and stream_id
 * are per slot.  A step over a list of slots runs every listed filter's
 * next step in one launch per kernel; each filter's results equal those of
 * a vsmc_cuda_cv_filter with the same configuration, whatever else runs in
 * the same launch.  All calls are asynchronous on `stream` unless noted,
 * and the slot lists they take are copied before they return. */
typedef struct vsmc_cuda_cv_batch vsmc_cuda_cv_batch;

/* Device bytes one slot of N particles and T_max observations holds. */
uint64_t vsmc_cuda_cv_batch_slot_bytes(const vsmc_cuda_cv_config *model,
                                       uint64_t N, uint64_t T_max);

/* A batch of up to `capacity` slots.  hbm_budget > 0 caps the bytes the
 * admitted slots may hold (admission past it returns VSMC_CUDA_ENOMEM) and
 * is reserved in the batch's memory pool at creation when the device has
 * it, so admissions reuse held memory instead of growing the pool; 0 means
 * no cap and no reservation. */
int vsmc_cuda_cv_batch_create(const vsmc_cuda_cv_config *model,
                              uint32_t capacity, uint64_t hbm_budget,
                              void *stream, vsmc_cuda_cv_batch **out);
int vsmc_cuda_cv_batch_destroy(vsmc_cuda_cv_batch *b);

/* Admits a filter (Sampler<T>(N, ...) plus Seed::set(seed)) into a free
 * slot; VSMC_CUDA_ENOMEM when no slot is free or its bytes exceed the
 * remaining budget.  The filter starts at step 0. */
int vsmc_cuda_cv_batch_admit(vsmc_cuda_cv_batch *b, uint64_t N,
                             uint64_t T_max, uint32_t seed,
                             uint32_t stream_id, uint32_t *slot);

/* Frees a slot and returns its bytes to the budget (the memory stays in
 * the batch's pool for later admissions). */
int vsmc_cuda_cv_batch_release(vsmc_cuda_cv_batch *b, uint32_t slot);
int vsmc_cuda_cv_batch_bytes_in_use(vsmc_cuda_cv_batch *b, uint64_t *bytes);

/* Observations of n slots, packed: slot k's T[k] values follow those of
 * slots 0..k-1 in obs_x / obs_y (host or device memory).  Each series
 * replaces the slot's observations from index 0. */
int vsmc_cuda_cv_batch_set_observations(vsmc_cuda_cv_batch *b, uint32_t n,
                                        const uint32_t *slots,
                                        const uint64_t *T, const double *obs_x,
                                        const double *obs_y, int on_device);

/* One observation appended to each of n slots (host values). */
int vsmc_cuda_cv_batch_append_observations(vsmc_cuda_cv_batch *b,
                                           uint32_t n, const uint32_t *slots,
                                           const double *x, const double *y);

/* Restarts the listed filters at step 0 (Sampler::initialize's reset; the
 * resample engine position is kept, as in the reference). */
int vsmc_cuda_cv_batch_initialize(vsmc_cuda_cv_batch *b, uint32_t n,
                                  const uint32_t *slots);

/* One step of each listed filter: the first step of a filter is
 * Sampler::initialize, later ones Sampler::iterate(1).  Every listed slot
 * needs an observation for that step. */
int vsmc_cuda_cv_batch_step(vsmc_cuda_cv_batch *b, uint32_t n,
                            const uint32_t *slots);

/* Steps each listed filter until its observations are used up (the whole
 * run of a batch of series of different lengths). */
int vsmc_cuda_cv_batch_run(vsmc_cuda_cv_batch *b, uint32_t n,
                           const uint32_t *slots);

/* The last counts[k] steps of each listed slot, oldest first, packed in
 * list order (sum of counts entries per array): ESS, log-evidence
 * increment, resampled flag; status[k] is the slot's sticky device status
 * (host arrays; each may be NULL).  The running log-evidence after a step is
 * the previous one plus its increment, in that order (the device's own sum).
 * Synchronises; returns the first non-zero status. */
int vsmc_cuda_cv_batch_read_steps(vsmc_cuda_cv_batch *b, uint32_t n,
                                  const uint32_t *slots,
                                  const uint32_t *counts, double *ess,
                                  double *logz_inc, int32_t *resampled,
                                  int32_t *status);

/* The last step of each listed slot: ESS, log-evidence increment,
 * resampled flag, running log-evidence and the slot's sticky device status
 * (host arrays of n; each may be NULL).  Synchronises; returns the first
 * non-zero status of the listed slots (the arrays are filled either way). */
int vsmc_cuda_cv_batch_read_last(vsmc_cuda_cv_batch *b, uint32_t n,
                                 const uint32_t *slots, double *ess,
                                 double *logz_inc, int32_t *resampled,
                                 double *log_evidence, int32_t *status);

int vsmc_cuda_cv_batch_iter_size(vsmc_cuda_cv_batch *b, uint32_t slot,
                                 uint64_t *iter_size);

/* Histories of one slot, as vsmc_cuda_cv_history.  Synchronises. */
int vsmc_cuda_cv_batch_history(vsmc_cuda_cv_batch *b, uint32_t slot,
                               double *ess, int32_t *resampled,
                               double *logz_inc, double *mean_x,
                               double *mean_y);

int vsmc_cuda_cv_batch_synchronize(vsmc_cuda_cv_batch *b);

/* vsmc_cuda_cv_batch_run records its steps in a CUDA graph and launches
 * the graph (on by default); a run with the same slots and step counts as
 * the previous one relaunches the same graph. */
int vsmc_cuda_cv_batch_set_graphs(vsmc_cuda_cv_batch *b, int enable);

/* The launch shape of later steps: the move compiled for `move_blocks`
 * (2, 3 or 4) x 256 threads per SM, the finalize CTA at `final_threads` (1024 or
 * 256; 256 applies only while every admitted filter has at most 256 tiles
 * of 2048 particles).  No shape changes a result.  New batches start at
 * (4, 256). */
int vsmc_cuda_cv_batch_set_launch_shape(vsmc_cuda_cv_batch *b,
                                        int move_blocks, int final_threads);

/* Tiling of vsmc_cuda_cv_batch_run: filters of at most `block_tiles` tiles
 * (2048 particles each; 0 <= block_tiles <= 64) run block-per-filter -- one
 * persistent launch in which a CTA takes a filter and runs all of its
 * remaining steps with block barriers only, beside the grid-per-filter
 * steps of the larger filters on a second stream -- and the rest
 * grid-per-filter (one launch per kernel per step over every filter's
 * tiles).  0 (the default of a new batch) runs every filter grid-per-filter.
 * The tiling changes no result: both run the same per-tile code in the same
 * summation order. */
int vsmc_cuda_cv_batch_set_tiling(vsmc_cuda_cv_batch *b, int block_tiles);
int vsmc_cuda_cv_batch_tiling(vsmc_cuda_cv_batch *b, int *block_tiles);

/* The batch's autotuner: times a few steps of a trial copy of (a sample
 * of at most 256 of) the listed filters, with zero observations, under each
 * launch shape (the move compiled for 2, 3 or 4 x 256 threads per SM; the finalize
 * CTA at 1024 or 256 threads when every filter has at most 256 tiles) and
 * keeps the fastest for later steps; then, at that shape, times whole trial
 * runs under each tiling (block_tiles 0, 1, 2, 4, ... up to the largest
 * trial filter; vsmc_cuda_cv_batch_set_tiling) and keeps the fastest.  The
 * shapes and the tiling change no result, and the trial touches none of the
 * batch's filters.  Synchronises; reports the launch shape (each pointer
 * may be NULL; vsmc_cuda_cv_batch_tiling gives the tiling). */
int vsmc_cuda_cv_batch_autotune(vsmc_cuda_cv_batch *b, uint32_t n,
                                const uint32_t *slots, int *move_blocks,
                                int *final_threads);

/* Kernel launches this batch has issued. */
int vsmc_cuda_cv_batch_launches(vsmc_cuda_cv_batch *b, uint64_t *launches);

/* ---- serving: a persistent request loop over a batch ---------------------
 *
 * No counterpart in the reference.  A server owns a vsmc_cuda_cv_batch and
 * one loop thread on its own stream.  Clients (any thread) open filter
 * requests of any N and stream observations to them; each tick the loop
 * releases finished requests, admits waiting ones in arrival order while a
 * slot and the HBM budget allow, steps every admitted request that has a
 * pending observation in one batched step, and publishes one result per
 * observation.  A request's results equal those of the same filter run
 * alone. */
typedef struct vsmc_cuda_cv_server vsmc_cuda_cv_server;

typedef struct {
    uint64_t request;     /* id from vsmc_cuda_cv_server_open */
    uint64_t t;           /* step (observation index) */
    double ess;
    double logz_inc;      /* log-evidence increment of this step */
    double log_evidence;  /* running sum after this step */
    int32_t resampled;
    int32_t status;       /* VSMC_CUDA_OK or the request's error */
    int64_t submit_ns;    /* server clock: arrival of the observation */
    int64_t done_ns;      /* server clock: result available on the host */
} vsmc_cuda_cv_result;

typedef struct {
    uint64_t opened, admitted, completed; /* requests */
    uint64_t ticks, steps, particle_steps;
    uint64_t max_active;                  /* most filters on the device */
    uint64_t waiting, active;             /* now */
    double busy_seconds;                  /* loop time spent in ticks */
} vsmc_cuda_cv_server_counters;

/* Starts the loop thread on the current device.  model: shared scheme,
 * form, threshold and parameters; max_filters: slots; hbm_budget: bytes
 * the admitted filters may hold (0 = no limit). */
int vsmc_cuda_cv_server_create(const vsmc_cuda_cv_config *model,
                               uint32_t max_filters, uint64_t hbm_budget,
                               vsmc_cuda_cv_server **out);

/* Stops the loop (pending work is dropped) and frees everything. */
int vsmc_cuda_cv_server_destroy(vsmc_cuda_cv_server *s);

/* The server clock (steady, nanoseconds since creation). */
int64_t vsmc_cuda_cv_server_now_ns(vsmc_cuda_cv_server *s);

/* A new filter request; VSMC_CUDA_ENOMEM if it alone exceeds the budget. */
int vsmc_cuda_cv_server_open(vsmc_cuda_cv_server *s, uint64_t N,
                             uint64_t T_max, uint32_t seed,
                             uint32_t stream_id, uint64_t *request);

/* The next observation of each of n requests; submit_ns (may be NULL =
 * now) stamps their arrival on the server clock. */
int vsmc_cuda_cv_server_observe(vsmc_cuda_cv_server *s, uint32_t n,
                                const uint64_t *requests, const double *x,
                                const double *y, const int64_t *submit_ns);

/* No more observations: the slot is freed after the pending ones run. */
int vsmc_cuda_cv_server_close(vsmc_cuda_cv_server *s, uint64_t request);

/* Up to max results in completion order; waits up to wait_ms for one. */
int vsmc_cuda_cv_server_poll(vsmc_cuda_cv_server *s,
                             vsmc_cuda_cv_result *out, uint32_t max,
                             uint32_t *n, int wait_ms);

/* Waits until every submitted observation has a result. */
int vsmc_cuda_cv_server_drain(vsmc_cuda_cv_server *s, int timeout_ms);

int vsmc_cuda_cv_server_stats(vsmc_cuda_cv_server *s,
                              vsmc_cuda_cv_server_counters *stats);

/* ---- tempered SMC for a 1-D Gaussian mixture ----------------------------
 *
 * The sampler of example/gmm (gmm_smc.cpp) with the alpha_prior schedule
 * (example/include/move_alpha.hpp:120-140): Seed::set(seed);
 * Sampler<gmm_state>(N, scheme, threshold); init gmm_init (4 components);
 * move move_smc (alpha_t = (t / iters)^power, incremental weight
 * loglik * (alpha_t - alpha_{t-1}), example/include/move_smc.hpp:51-75);
 * `sweeps` sweeps of gmm_move_mu, gmm_move_lambda and gmm_move_weight
 * (example/gmm/include/gmm_move.hpp:35-117) with every block's proposal sd
 * `sd`; path_sampling(smc_path).  Each particle draws from its own
 * Threefry4x64 engine (RngSet<Threefry4x64, Vector>: engine i seeded with
 * the (i+1)-th Seed::get(), the resample engine with the (N+1)-th). */
typedef struct vsmc_cuda_gmm vsmc_cuda_gmm;

typedef struct {
    uint64_t N;       /* particles */
    uint64_t iters;   /* tempering steps after initialize */
    int power;        /* alpha_t = (t / iters)^power */
    int sweeps;       /* MH sweeps per step (<= 16) */
    double sd;        /* proposal sd of every block */
    int scheme;       /* vsmc_cuda_scheme */
    double threshold; /* resample when ESS < threshold * N */
    uint32_t seed;    /* Seed::set(seed) */
    int form;         /* VSMC_CUDA_FP64, or VSMC_CUDA_MIXED: each data
                         point's mixture density in float, the per-particle
                         sum of log terms in double */
    int group;        /* lanes per particle (1, 2, 4, 8, 16); 0 = pick the
                         fastest at initialize (results do not depend on it) */
} vsmc_cuda_gmm_config;

/* N 2^16, iters 100, power 4, sweeps 5, sd 0.1, Systematic, threshold 0.5,
 * seed 101, FP64, group 0. */
void vsmc_cuda_gmm_config_default(vsmc_cuda_gmm_config *cfg);

/* data: n host doubles (n <= 16384), gmm_state::read_data. */
int vsmc_cuda_gmm_create(const vsmc_cuda_gmm_config *cfg, const double *data,
                         uint64_t n, void *stream, vsmc_cuda_gmm **out);
int vsmc_cuda_gmm_destroy(vsmc_cuda_gmm *g);

/* Sampler::initialize / iterate(num) (at most iters steps in total). */
int vsmc_cuda_gmm_initialize(vsmc_cuda_gmm *g);
int vsmc_cuda_gmm_iterate(vsmc_cuda_gmm *g, uint64_t num);
int vsmc_cuda_gmm_iter_size(vsmc_cuda_gmm *g, uint64_t *iter_size);

/* Histories (host arrays of iter_size entries, each may be NULL): ESS,
 * resampled flags, log-evidence increments log sum_i W_i exp(inc_i), path
 * sampling integrand sum_i W_i loglik_i and grid alpha_t, and acceptance
 * counts (iter_size x (1 + 3 sweeps): move_smc's 0, then the MH moves in
 * queue order), as Sampler::accept_history.  Synchronises. */
int vsmc_cuda_gmm_history(vsmc_cuda_gmm *g, double *ess, int32_t *resampled,
                          double *zinc, double *integrand, double *grid,
                          int64_t *accept);

/* log-evidence estimates with the -n/2 log(2 pi) constant: the SMC product
 * of increments (zconst + log_likelihood_const, example/include/smc_do.hpp)
 * and path sampling.  Synchronises. */
int vsmc_cuda_gmm_log_evidence(vsmc_cuda_gmm *g, double *smc, double *path);

/* Particles (host, N x 14: mu[4], lambda[4], weight[4], log prior, log
 * likelihood), max-normalised log-weights and the words each particle's
 * engine has drawn (each may be NULL).  Synchronises. */
int vsmc_cuda_gmm_read_params(vsmc_cuda_gmm *g, double *params, double *lw,
                              uint64_t *words);

/* Log likelihood of every current particle evaluated in `form` (host, N
 * doubles), for precision comparisons.  Synchronises. */
int vsmc_cuda_gmm_loglik(vsmc_cuda_gmm *g, int form, double *out);

/* Lanes per particle in use (the autotuned value when group was 0). */
int vsmc_cuda_gmm_group(vsmc_cuda_gmm *g, int *group);

/* CUDA-event timing of the MCMC kernels (as vsmc_cuda_cv_set_timing). */
int vsmc_cuda_gmm_set_timing(vsmc_cuda_gmm *g, int enable);
int vsmc_cuda_gmm_timing(vsmc_cuda_gmm *g, double *mcmc_ms, uint64_t *steps,
                         uint64_t *launches);

/* The workload's mixture data: point i from component floor(4 u) of means
 * (-3, 0, 2, 5), unit sd; Philox4x32-10 keyed {seed, 3}. Host only. */
int vsmc_cuda_gmm_simulate(uint32_t seed, uint64_t n, double *out);

#ifdef __cplusplus
}
#endif

#endif /* VSMC_CUDA_H */
