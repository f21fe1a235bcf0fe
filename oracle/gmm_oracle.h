/*
 * gmm_oracle.h -- CPU restatement of vSMC's tempered SMC sampler for a 1-D
 * Gaussian mixture (TEST INFRASTRUCTURE: loaded by tests/, smoke() and
 * bench.py's CPU legs only; never part of the product).
 *
 * Follows example/gmm/include/gmm_param.hpp, gmm_state.hpp, gmm_init.hpp,
 * gmm_move.hpp, example/include/move_smc.hpp, move_alpha.hpp (alpha_prior),
 * smc_path.hpp, and vSMC's Sampler / Path / WeightSet / RngSet for the run,
 * with libstdc++'s normal, lognormal, gamma and uniform distributions over
 * each particle's Threefry4x64 engine.  Pinned against oracle/ref_gmm.cpp,
 * the same sampler built from the reference's own classes.
 */
#ifndef VSMC_B200_GMM_ORACLE_H
#define VSMC_B200_GMM_ORACLE_H

#include "smc_oracle.h"

#ifdef __cplusplus
extern "C" {
#endif

/* std::gamma_distribution<double>(alpha, beta) (libstdc++ Marsaglia-Tsang)
 * over a Threefry4x64 engine; `nd` is the distribution's own normal (0, 1)
 * with its cached second value. */
double orc_gamma_threefry(orc_normal *nd, orc_threefry *e, double alpha,
                          double beta);
double orc_normal_threefry(orc_normal *nd, orc_threefry *e, double mean,
                           double sd);

/* The mixture data: n points, point i from component k = floor(4 u)
 * (u = std::uniform_real_distribution over a Philox4x32 engine keyed
 * {seed, 3}) with means (-3, 0, 2, 5) and unit sd
 * (std::normal_distribution(mean_k, 1) on the same engine). */
void orc_gmm_simulate(uint32_t seed, size_t n, double *out);

/* The whole run: Seed::set(seed); Sampler(N, scheme, threshold); initialize
 * with 4 components; `iters` iterations with alpha_t = (t / iters)^power,
 * each followed by `sweeps` sweeps of the mu, lambda and weight MH moves
 * with proposal sd `sd`.  Arrays of iters + 1 entries (each may be NULL):
 * ess, resampled, zinc (zconst_t - zconst_{t-1}, 0 at t = 0), integrand and
 * grid of the path sampler; accept is (iters + 1) x (1 + 3 sweeps); params
 * is N x 14 (mu[4], lambda[4], weight[4], log prior, log likelihood); lw is
 * the final log-weights; words the words each particle's engine drew.
 * Returns zconst + log_likelihood_const; *path_logz the path estimate. */
double orc_gmm_smc(const double *data, size_t n, size_t N, size_t iters,
                   int power, int sweeps, double sd, int scheme,
                   double threshold, uint32_t seed, double *ess,
                   int32_t *resampled, double *zinc, double *integrand,
                   double *grid, int64_t *accept, double *params, double *lw,
                   uint64_t *words, double *path_logz);

/* Log-likelihood of one parameter set (the gmm_state::log_likelihood sum
 * without the -n/2 log(2 pi) constant). */
double orc_gmm_loglik(const double *data, size_t n, const double *mu,
                      const double *lambda, const double *weight);

#ifdef __cplusplus
}
#endif

#endif
