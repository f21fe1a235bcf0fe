// ref_gmm.cpp -- test-only harness: vSMC's tempered SMC sampler for a 1-D
// Gaussian mixture, built from the unmodified vSMC headers and the
// reference's own example/gmm classes (gmm_param, gmm_state, gmm_init,
// gmm_move_mu / _lambda / _weight) and example/include helpers (move_smc,
// alpha_prior, smc_path).  It is the checker of the C restatement in
// oracle/gmm_oracle.c and of the device sampler; nothing in the product
// links it.
//
// The sampler is set up the way example/gmm/src/gmm_smc.cpp sets it up:
// Sampler<gmm_state>(N, scheme, threshold), init gmm_init, move
// move_smc<alpha_prior<Power>, proposal>, the three MH block moves as the
// MCMC queue (here repeated `sweeps` times), path_sampling(smc_path), and
// initialize(data_info) with 4 components.  The proposal scale is fixed
// (fixed_sd below, the only class written here): every block moves with the
// same sd, which is what a fixed "proposal sd per block" means; the
// example's own gmm_proposal derives the scales from alpha instead.
#define BASE_STATE vsmc::StateOMP
#define BASE_INIT vsmc::InitializeOMP
#define BASE_MOVE vsmc::MoveOMP
#define BASE_MONITOR vsmc::MonitorEvalOMP
#define BASE_PATH vsmc::PathEvalOMP

#include <vsmc/smp/backend_omp.hpp>
#include <vsmc/cxx11/cmath.hpp>

static const std::size_t InitCompNum = 4;
static const std::size_t MinCompNum = 1;
static const std::size_t MaxCompNum = 10;

#include "common.hpp"
#include "gmm_param.hpp"
#include "gmm_state.hpp"
#include "gmm_init.hpp"
#include "gmm_move.hpp"
#include "move_alpha.hpp"
#include "move_smc.hpp"
#include "smc_path.hpp"

#include <omp.h>

#include <chrono>
#include <cstdint>
#include <cstring>
#include <sstream>
#include <string>

namespace {

class fixed_sd
{
    public :

    typedef double value_type;

    fixed_sd (value_type sd = 0.1) : sd_(sd) {}

    void proposal_iter (std::size_t, vsmc::Particle<gmm_state> &particle)
        const
    {
        for (vsmc::Particle<gmm_state>::size_type i = 0;
                i != particle.size(); ++i) {
            particle.value().state(i, 0).mu_sd()     = sd_;
            particle.value().state(i, 0).lambda_sd() = sd_;
            particle.value().state(i, 0).weight_sd() = sd_;
        }
    }

    private :

    double sd_;
};

uint64_t words_used (const vsmc::Threefry4x64 &eng)
{
    std::stringstream ss;
    ss << eng;
    uint64_t v[13];
    for (int k = 0; k != 13; ++k)
        ss >> v[k];
    std::size_t index = 0;
    ss >> index;
    return v[0] == 0 ? 0 : (v[0] - 1) * 4 + index;
}

template <std::size_t Power>
double run (const double *data, uint64_t n, uint64_t N, uint64_t iters,
        int sweeps, double sd, int scheme, double threshold, unsigned seed,
        double *ess, int32_t *resampled, double *zinc, double *integrand,
        double *grid, int64_t *accept, double *params, double *lw,
        uint64_t *words, double *path_logz, double *seconds,
        std::string *summary)
{
    typedef move_smc<gmm_state, alpha_prior<gmm_state, Power>, fixed_sd>
        smc_move;
    vsmc::Seed::instance().set(seed);
    vsmc::Sampler<gmm_state> sampler(N,
            static_cast<vsmc::ResampleScheme>(scheme), threshold);
    sampler.init(gmm_init()).move(smc_move(iters, sd), false);
    for (int s = 0; s != sweeps; ++s) {
        sampler
            .mcmc(gmm_move_mu(), true)
            .mcmc(gmm_move_lambda(), true)
            .mcmc(gmm_move_weight(), true);
    }
    sampler.path_sampling(smc_path<gmm_state>());
    sampler.particle().value().comp_num(InitCompNum);

    data_info info(n, data);
    std::vector<double> z(iters + 1, 0.0);
    auto t0 = std::chrono::steady_clock::now();
    sampler.initialize(&info);
    z[0] = 0;
    for (uint64_t t = 1; t <= iters; ++t) {
        sampler.iterate(1);
        z[t] = sampler.particle().value().zconst();
    }
    auto t1 = std::chrono::steady_clock::now();
    if (seconds)
        *seconds = std::chrono::duration<double>(t1 - t0).count();

    const std::size_t T = sampler.iter_size();
    const std::size_t nacc = 1 + 3 * static_cast<std::size_t>(sweeps);
    for (std::size_t t = 0; t != T; ++t) {
        if (ess)
            ess[t] = sampler.ess_history(t);
        if (resampled)
            resampled[t] = sampler.resampled_history(t) ? 1 : 0;
        if (zinc)
            zinc[t] = t == 0 ? 0.0 : (t == 1 ? z[1] : z[t] - z[t - 1]);
        if (accept)
            for (std::size_t k = 0; k != nacc; ++k)
                accept[t * nacc + k] =
                    t == 0 && k > 0 ? 0 : static_cast<int64_t>(
                            sampler.accept_history(k, t));
    }
    if (integrand)
        sampler.path().read_integrand(integrand);
    if (grid)
        sampler.path().read_grid(grid);
    if (path_logz)
        *path_logz = sampler.path_sampling() +
            sampler.particle().value().log_likelihood_const();
    if (params)
        for (uint64_t i = 0; i != N; ++i) {
            const gmm_param &p = sampler.particle().value().state(i, 0);
            double *o = params + i * 14;
            for (std::size_t d = 0; d != 4; ++d) {
                o[d] = p.mu(d);
                o[4 + d] = p.lambda(d);
                o[8 + d] = p.weight(d);
            }
            o[12] = p.log_prior();
            o[13] = p.log_likelihood();
        }
    if (lw)
        sampler.particle().weight_set().read_log_weight(lw);
    if (words)
        for (uint64_t i = 0; i != N; ++i)
            words[i] = words_used(sampler.particle().rng(i));
    if (summary) {
        std::stringstream ss;
        ss << sampler;
        *summary = ss.str();
    }
    return sampler.particle().value().zconst() +
        sampler.particle().value().log_likelihood_const();
}

} // namespace

extern "C" {

// The tempered SMC run: initialize + `iters` iterations with alpha_t =
// (t / iters)^power (power 2, 4 or 5).  Histories have iters + 1 entries
// (zinc[t] = zconst after step t minus zconst after step t - 1, the only
// view of the increments the reference gives); accept is (iters + 1) x
// (1 + 3 sweeps) (move_smc first, then the MH moves in queue order; the
// init step's MH entries are 0); params is N x 14 (mu[4], lambda[4],
// weight[4], log prior, log likelihood).  Returns the SMC log-evidence
// estimate zconst + log_likelihood_const (example/include/smc_do.hpp);
// *path_logz gets the path-sampling one.
double ref_gmm_smc (const double *data, uint64_t n, uint64_t N,
        uint64_t iters, int power, int sweeps, double sd, int scheme,
        double threshold, unsigned seed, int nthreads, double *ess,
        int32_t *resampled, double *zinc, double *integrand, double *grid,
        int64_t *accept, double *params, double *lw, uint64_t *words,
        double *path_logz, double *seconds)
{
    if (nthreads > 0)
        omp_set_num_threads(nthreads);
    switch (power) {
        case 2 :
            return run<2>(data, n, N, iters, sweeps, sd, scheme, threshold,
                    seed, ess, resampled, zinc, integrand, grid, accept,
                    params, lw, words, path_logz, seconds, VSMC_NULLPTR);
        case 5 :
            return run<5>(data, n, N, iters, sweeps, sd, scheme, threshold,
                    seed, ess, resampled, zinc, integrand, grid, accept,
                    params, lw, words, path_logz, seconds, VSMC_NULLPTR);
        default :
            return run<4>(data, n, N, iters, sweeps, sd, scheme, threshold,
                    seed, ess, resampled, zinc, integrand, grid, accept,
                    params, lw, words, path_logz, seconds, VSMC_NULLPTR);
    }
}

// The summary table `os << sampler` (Sampler::print) of the same run with
// power 4, copied into buf (cap bytes, NUL-terminated); returns its length.
uint64_t ref_gmm_summary (const double *data, uint64_t n, uint64_t N,
        uint64_t iters, int sweeps, double sd, int scheme, double threshold,
        unsigned seed, char *buf, uint64_t cap)
{
    std::string text;
    run<4>(data, n, N, iters, sweeps, sd, scheme, threshold, seed,
            VSMC_NULLPTR, VSMC_NULLPTR, VSMC_NULLPTR, VSMC_NULLPTR,
            VSMC_NULLPTR, VSMC_NULLPTR, VSMC_NULLPTR, VSMC_NULLPTR,
            VSMC_NULLPTR, VSMC_NULLPTR, VSMC_NULLPTR, &text);
    if (buf && cap > 0) {
        const uint64_t k = text.size() < cap - 1 ? text.size() : cap - 1;
        std::memcpy(buf, text.data(), k);
        buf[k] = '\0';
    }
    return text.size();
}

} // extern "C"
