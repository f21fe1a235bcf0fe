/*
 * smc_oracle.h -- CPU restatement of vSMC's SMC step (TEST INFRASTRUCTURE).
 *
 * This header and smc_oracle.c are the correctness oracle for the B200 SMC
 * step.  Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
 * reference legs may load them, and only as the checker: the product library
 * (libvsmc_cuda.so) never links or calls anything here.
 *
 * Every function restates the reference algorithm with the same sequence of
 * IEEE-754 double operations (built with -ffp-contract=off and no -march, so
 * no FMA contraction), so on the same CPU and libm it reproduces the vSMC
 * headers bit for bit.  That claim is pinned by tests/test_oracle.py against
 * fixtures generated from the unmodified vSMC headers (oracle/ref_harness.cpp,
 * built by oracle/Makefile into oracle/_ref/).
 *
 * Reference paths below are relative to the vSMC project root.
 */
#ifndef VSMC_B200_SMC_ORACLE_H
#define VSMC_B200_SMC_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- RNG -- */

/* One Philox4x32-10 block: include/vsmc/rng/philox.hpp:137-265, 504-523. */
void orc_philox4x32_block(const uint32_t ctr[4], const uint32_t key[2],
                          uint32_t out[4]);

/* One Threefry4x64-20 block: include/vsmc/rng/threefry.hpp:105-233,
 * 473-506 (key schedule :65-73, 491-506). */
void orc_threefry4x64_block(const uint64_t ctr[4], const uint64_t key[4],
                            uint64_t out[4]);

/* Stateful engines with the reference's (ctr, key, buffer, index)
 * semantics: operator()() increments the counter *before* generating a block
 * (philox.hpp:386-395, threefry.hpp:355-364, utility/counter.hpp:119-120). */
typedef struct {
    uint32_t key[2];
    uint32_t ctr[4];
    uint32_t buf[4];
    unsigned index;
} orc_philox;

typedef struct {
    uint64_t key[4];
    uint64_t ctr[4];
    uint64_t buf[4];
    unsigned index;
} orc_threefry;

/* seed(s): key = {s, 0...}, ctr = 0, index = K (philox.hpp:344-350,
 * threefry.hpp:301-309). */
void orc_philox_seed(orc_philox *e, uint32_t s);
void orc_threefry_seed(orc_threefry *e, uint64_t s);
/* key(k) / ctr(c): set and invalidate the buffer (philox.hpp:367-377). */
void orc_philox_set_key(orc_philox *e, const uint32_t key[2]);
void orc_philox_set_ctr(orc_philox *e, const uint32_t ctr[4]);
void orc_threefry_set_key(orc_threefry *e, const uint64_t key[4]);
void orc_threefry_set_ctr(orc_threefry *e, const uint64_t ctr[4]);
uint32_t orc_philox_next(orc_philox *e);
uint64_t orc_threefry_next(orc_threefry *e);
/* Number of words drawn since the counter was last zero:
 * (ctr-1)*K + index for ctr > 0. Valid while ctr fits in 64 bits. */
uint64_t orc_threefry_words_used(const orc_threefry *e);

/* Word streams (test helpers): n successive operator()() outputs of an
 * engine with the given key, whose counter starts at ctr0 with an empty
 * buffer, after discarding `skip` words. */
void orc_philox_stream(const uint32_t key[2], const uint32_t ctr0[4],
                       uint64_t skip, uint64_t n, uint32_t *out);
void orc_threefry_stream(const uint64_t key[4], const uint64_t ctr0[4],
                         uint64_t skip, uint64_t n, uint64_t *out);

/* ------------------------------------------------------------ U01 ------ */

/* include/vsmc/rng/u01.h:93-180 (the 53-bit double conversions). */
double orc_u01_closed_open_64_53(uint64_t u);
double orc_u01_open_closed_32_53(uint32_t u);

/* std::uniform_real_distribution<double>(0,1) over a 64-bit engine, as used by
 * U01Sequence* (rng/u01.hpp:185,228,261): libstdc++ generate_canonical with
 * one word: double(x) * 2^-64, clamped below 1. */
double orc_canonical_u64(uint64_t x);
/* ... over a 32-bit engine: two words a (first), b: (a + b*2^32) * 2^-64. */
double orc_canonical_u32x2(uint32_t a, uint32_t b);

/* std::normal_distribution<double> (libstdc++ Marsaglia polar method with a
 * cached second variate) driven by a Philox4x32 engine through
 * generate_canonical. Used by the CV model moves
 * (example/pf/include/pf_smp.hpp:154-155, 215-216). */
typedef struct {
    int saved_available;
    double saved;
} orc_normal;
void orc_normal_reset(orc_normal *nd);
double orc_normal_philox(orc_normal *nd, orc_philox *e, double mean,
                         double sd);

/* -------------------------------------------------------- weights ------ */

/* WeightSet::post_set_log_weight after add_log_weight
 * (core/weight_set.hpp:325-331, 441-446): lw += inc; lw -= max(lw);
 * w = exp(lw); w *= 1/asum(w); returns ESS = 1/dot(w,w). inc may be NULL
 * (set_log_weight semantics with lw already filled). */
double orc_add_log_weight(size_t N, double *lw, double *w, const double *inc);
/* set_equal_weight (weight_set.hpp:96-106): w = 1/N, lw = 0, returns N. */
double orc_set_equal_weight(size_t N, double *lw, double *w);

/* ------------------------------------------------------- resample ------ */

enum {
    ORC_MULTINOMIAL = 0,
    ORC_RESIDUAL = 1,
    ORC_STRATIFIED = 2,
    ORC_SYSTEMATIC = 3,
    ORC_RESIDUAL_STRATIFIED = 4,
    ORC_RESIDUAL_SYSTEMATIC = 5
}; /* resample/common.hpp:124-131 */

/* Resample<Scheme>::operator()(M, N, rng, weight, replication)
 * (resample/multinomial.hpp:53-59, residual.hpp:53-77, stratified.hpp:53-59,
 * systematic.hpp:53-59, residual_stratified.hpp:53-77,
 * residual_systematic.hpp:53-77) over internal::inversion
 * (common.hpp:57-84).  `uniforms`, when not NULL, receives every value of the
 * U01 sequence that inversion queried, in query order (at most N), and
 * *n_uniforms their count; *cdf_sum (if not NULL) receives the final accw. */
void orc_resample(int scheme, size_t M, size_t N, orc_threefry *rng,
                  const double *weight, int64_t *replication,
                  double *uniforms, size_t *n_uniforms);

/* Same as orc_resample's inversion step on caller-supplied U01 sequence
 * values (u[0..N-1]; entries past the ones inversion reads are ignored). */
void orc_inversion(size_t M, size_t N, const double *weight, const double *u,
                   int64_t *replication);

/* internal::cfrp_trans (resample/common.hpp:87-118). */
void orc_cfrp_trans(size_t M, size_t N, const int64_t *replication,
                    int64_t *copy_from);

/* -------------------------------------------------- CV model ---------- */

/* Constant-velocity Student-t model. Move, init and likelihood follow
 * example/pf/include/pf_smp.hpp:96-112 (log_likelihood), :150-173 (init),
 * :207-238 (move) with the workload's parameters and a non-aliasing counter
 * layout ctr = {block, step, particle id, stream}. */
typedef struct {
    double dt;      /* 0.1 */
    double sd_pos;  /* process noise sd on position, 0.02 */
    double sd_vel;  /* process noise sd on velocity, 0.5 */
    double sd_pos0; /* prior sd on position, 2 */
    double sd_vel0; /* prior sd on velocity, 1 */
    double scale;   /* likelihood multiplier on the residual, 10 */
    double nu;      /* Student-t degrees of freedom, 10 */
} orc_cv_param;

void orc_cv_default(orc_cv_param *p);
double orc_cv_loglik(const orc_cv_param *p, double x, double y, double ox,
                     double oy);
void orc_cv_init_particle(const orc_cv_param *p, const uint32_t key[2],
                          uint32_t id, uint32_t stream, double s[4]);
void orc_cv_move_particle(const orc_cv_param *p, const uint32_t key[2],
                          uint32_t iter, uint32_t id, uint32_t stream,
                          double s[4]);
/* Simulated observations: state starts at (0,0,1,1); obs_t = pos_t +
 * t_nu / scale, t_nu = z0 / sqrt(sum_{k=1..nu} z_k^2 / nu) (nu integer).
 * One Philox4x32 engine per step with key {obs_seed, 1} and ctr
 * {0, t, 0, stream}, one polar generator per step. */
void orc_cv_simulate(const orc_cv_param *p, uint32_t obs_seed,
                     uint32_t stream, size_t T, double *obs_x, double *obs_y,
                     double *truth /* T x 4, nullable */);

/* Full bootstrap filter, FP64: Sampler::initialize + iterate(T-1)
 * (core/sampler.hpp:450-483, 758-834) with Seed::set(seed) semantics
 * (rng/seed.hpp:102,149; particle.hpp:64-70): model key {seed+1, 0},
 * resample engine Threefry4x64 seeded seed+2.  Log-evidence follows
 * example/include/move_smc.hpp:63-71 (sum_i W_i exp(inc_i) before the add).
 * Per-step outputs (length T, nullable): ess (before resampling), resampled
 * (0/1), logz_inc, mean_x / mean_y (MonitorMCMC stage: after resampling,
 * ISIntegrate order).  final_state (4*N SoA, nullable), final_lw (nullable),
 * and words_used (resample engine words drawn, nullable).  Returns the
 * log-evidence. */
typedef struct {
    double *ess;
    int32_t *resampled;
    double *logz_inc;
    double *mean_x;
    double *mean_y;
    double *final_state;
    double *final_lw;
    uint64_t *words_used;
    /* When not NULL: per-step resampling record of the LAST resampling step
     * only: copy_from (N) and the uniforms inversion read. */
    int64_t *last_copy_from;
} orc_cv_out;

double orc_cv_filter(const orc_cv_param *p, size_t N, size_t T, int scheme,
                     double threshold, uint32_t seed, uint32_t stream,
                     const double *obs_x, const double *obs_y,
                     orc_cv_out *out);

#ifdef __cplusplus
}
#endif

#endif
