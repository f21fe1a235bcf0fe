/*
 * gmm_oracle.c -- CPU restatement of vSMC's tempered SMC sampler for the
 * 1-D Gaussian mixture (TEST INFRASTRUCTURE; see gmm_oracle.h).
 *
 * Built like smc_oracle.c (-O2 -ffp-contract=off, no -march): each double
 * expression below is written in the reference's evaluation order so that
 * the results equal vSMC's bit for bit on the same libm.  Citations are
 * relative to the vSMC project root; "libstdc++" refers to the
 * distributions of GCC 13's <random> (bits/random.tcc), which the example
 * uses through vsmc::cxx11.
 */
#include "gmm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define K 4 /* components (InitCompNum, example/gmm/include/gmm.hpp) */

/* vsmc::math::ln_pi_2<double>() = log(2 pi) (math/constants.hpp). */
#define ORC_LN_PI_2 1.8378770664093454835606594728112

/* ---------------------------------------------------- distributions -- */

static double canonical64(orc_threefry *e)
{
    return orc_canonical_u64(orc_threefry_next(e));
}

/* libstdc++ normal_distribution::operator(): Marsaglia polar method, the
 * second value of each pair cached in the distribution object. */
double orc_normal_threefry(orc_normal *nd, orc_threefry *e, double mean,
                           double sd)
{
    double ret;
    if (nd->saved_available) {
        nd->saved_available = 0;
        ret = nd->saved;
    } else {
        double x, y, r2;
        do {
            x = 2.0 * canonical64(e) - 1.0;
            y = 2.0 * canonical64(e) - 1.0;
            r2 = x * x + y * y;
        } while (r2 > 1.0 || r2 == 0.0);
        const double mult = sqrt(-2.0 * log(r2) / r2);
        nd->saved = x * mult;
        nd->saved_available = 1;
        ret = y * mult;
    }
    return ret * sd + mean;
}

/* libstdc++ gamma_distribution::operator() (Marsaglia and Tsang 2000):
 * param_type::_M_initialize gives malpha (alpha, or alpha + 1 below 1),
 * a1 = malpha - 1/3 and a2 = 1/sqrt(9 a1). */
double orc_gamma_threefry(orc_normal *nd, orc_threefry *e, double alpha,
                          double beta)
{
    const double malpha = alpha < 1.0 ? alpha + 1.0 : alpha;
    const double a1 = malpha - 1.0 / 3.0;
    const double a2 = 1.0 / sqrt(9.0 * a1);
    double u, v, n;
    do {
        do {
            n = orc_normal_threefry(nd, e, 0.0, 1.0);
            v = 1.0 + a2 * n;
        } while (v <= 0.0);
        v = v * v * v;
        u = canonical64(e);
    } while (u > 1.0 - 0.0331 * n * n * n * n &&
             log(u) > 0.5 * n * n + a1 * (1.0 - v + log(v)));
    if (alpha == malpha)
        return a1 * v * beta;
    do
        u = canonical64(e);
    while (u == 0.0);
    return pow(u, 1.0 / alpha) * a1 * v * beta;
}

/* ------------------------------------------------------------- data -- */

void orc_gmm_simulate(uint32_t seed, size_t n, double *out)
{
    static const double means[K] = {-3.0, 0.0, 2.0, 5.0};
    orc_philox e;
    uint32_t key[2] = {seed, 3u};
    orc_philox_seed(&e, 0);
    orc_philox_set_key(&e, key);
    orc_normal nd;
    orc_normal_reset(&nd);
    for (size_t i = 0; i != n; ++i) {
        const uint32_t a = orc_philox_next(&e);
        const uint32_t b = orc_philox_next(&e);
        const double u = orc_canonical_u32x2(a, b) * 1.0 + 0.0;
        int k = (int)(u * 4.0);
        k = k > K - 1 ? K - 1 : k;
        out[i] = orc_normal_philox(&nd, &e, means[k], 1.0);
    }
}

/* ------------------------------------------------------------ model -- */

typedef struct {
    double mu[K], lambda[K], log_lambda[K], weight[K];
    double mu_old[K], lambda_old[K], log_lambda_old[K], weight_old[K];
    double lp, ll, lt;
    double lp_old, ll_old, lt_old;
} gmm_param;

typedef struct {
    const double *obs;
    size_t n;
    double mu0, sd0, shape0, scale0;
    double alpha, alpha_inc;
} gmm_model;

/* gmm_state::read_data (gmm_state.hpp:118-157): prior hyper-parameters
 * from the data range. */
static void model_init(gmm_model *m, const double *obs, size_t n)
{
    m->obs = obs;
    m->n = n;
    double xmax = obs[0], xmin = obs[0];
    for (size_t i = 0; i != n; ++i) {
        if (obs[i] > xmax)
            xmax = obs[i];
        if (obs[i] < xmin)
            xmin = obs[i];
    }
    const double kappa = 1 / ((xmax - xmin) * (xmax - xmin));
    m->mu0 = 0.5 * (xmin + xmax);
    m->sd0 = 1 / sqrt(kappa);
    m->shape0 = 2;
    m->scale0 = 50 * kappa;
    m->alpha = 0;
    m->alpha_inc = 0;
}

/* gmm_state::log_prior (gmm_state.hpp:67-80) */
static double log_prior(const gmm_model *m, gmm_param *s)
{
    double lp = 0;
    for (int d = 0; d != K; ++d) {
        const double resid = s->mu[d] - m->mu0;
        lp += -0.5 * (resid * resid) / (m->sd0 * m->sd0);
        lp += (m->shape0 - 1) * log(s->lambda[d]) - s->lambda[d] / m->scale0;
    }
    return s->lp = lp;
}

double orc_gmm_loglik(const double *obs, size_t n, const double *mu,
                      const double *lambda, const double *weight)
{
    double log_lambda[K];
    for (int d = 0; d != K; ++d)
        log_lambda[d] = log(lambda[d]);
    double ll = 0;
    for (size_t i = 0; i != n; ++i) {
        double lli = 0;
        for (int d = 0; d != K; ++d) {
            const double resid = obs[i] - mu[d];
            lli += weight[d] * exp(0.5 * log_lambda[d] -
                                   0.5 * lambda[d] * resid * resid);
        }
        ll += log(lli + 1e-13);
    }
    return ll;
}

/* gmm_state::log_likelihood (gmm_state.hpp:82-103), which also refreshes
 * log_lambda (gmm_param::log_lambda()). */
static double log_likelihood(const gmm_model *m, gmm_param *s)
{
    for (int d = 0; d != K; ++d)
        s->log_lambda[d] = log(s->lambda[d]);
    double ll = 0;
    for (size_t i = 0; i != m->n; ++i) {
        double lli = 0;
        for (int d = 0; d != K; ++d) {
            const double resid = m->obs[i] - s->mu[d];
            lli += s->weight[d] * exp(0.5 * s->log_lambda[d] -
                                      0.5 * s->lambda[d] * resid * resid);
        }
        ll += log(lli + 1e-13);
    }
    return s->ll = ll;
}

/* gmm_state::log_target (gmm_state.hpp:105-110) */
static double log_target(const gmm_model *m, gmm_param *s)
{
    const double lp = log_prior(m, s);
    const double lt = lp + m->alpha * log_likelihood(m, s);
    return s->lt = lt;
}

/* gmm_param::save_old (gmm_param.hpp:176-192) */
static void save_old(const gmm_model *m, gmm_param *s)
{
    for (int i = 0; i != K; ++i) {
        s->mu_old[i] = s->mu[i];
        s->lambda_old[i] = s->lambda[i];
        s->log_lambda_old[i] = s->log_lambda[i];
        s->weight_old[i] = s->weight[i];
    }
    s->lp_old = s->lp;
    s->ll_old = s->ll;
    s->lt_old = s->lp + m->alpha * s->ll;
}

/* mh_reject_common (gmm_param.hpp:339-350) */
static void reject_common(gmm_param *s, double p, double u)
{
    if (p < u) {
        s->lp = s->lp_old;
        s->ll = s->ll_old;
        s->lt = s->lt_old;
    } else {
        s->lp_old = s->lp;
        s->ll_old = s->ll;
        s->lt_old = s->lt;
    }
}

/* gmm_move_mu::move_state (gmm_move.hpp:35-58) with ordered() false */
static int move_mu(const gmm_model *m, gmm_param *s, orc_threefry *e,
                   double sd)
{
    orc_normal rmu;
    orc_normal_reset(&rmu);
    save_old(m, s);
    for (int d = 0; d != K; ++d)
        s->mu[d] += orc_normal_threefry(&rmu, e, 0.0, sd);
    log_target(m, s);
    const double p = s->lt - s->lt_old;
    const double u = log(canonical64(e) * 1.0 + 0.0);
    reject_common(s, p, u);
    if (p < u) {
        for (int i = 0; i != K; ++i)
            s->mu[i] = s->mu_old[i];
        return 0;
    }
    for (int i = 0; i != K; ++i)
        s->mu_old[i] = s->mu[i];
    return 1;
}

/* gmm_move_lambda::move_state (gmm_move.hpp:61-83): lognormal_distribution
 * (0, sd) is exp(sd * n + 0) with n from its own normal (0, 1). */
static int move_lambda(const gmm_model *m, gmm_param *s, orc_threefry *e,
                       double sd)
{
    orc_normal nd;
    orc_normal_reset(&nd);
    save_old(m, s);
    for (int d = 0; d != K; ++d)
        s->lambda[d] *= exp(sd * orc_normal_threefry(&nd, e, 0.0, 1.0) + 0.0);
    log_target(m, s);
    double lld = 0; /* log_lambda_diff (gmm_param.hpp:204-211) */
    for (int i = 0; i != K; ++i)
        lld += s->log_lambda[i] - s->log_lambda_old[i];
    const double p = s->lt - s->lt_old + lld;
    const double u = log(canonical64(e) * 1.0 + 0.0);
    reject_common(s, p, u);
    if (p < u) {
        for (int i = 0; i != K; ++i) {
            s->lambda[i] = s->lambda_old[i];
            s->log_lambda[i] = s->log_lambda_old[i];
        }
        return 0;
    }
    for (int i = 0; i != K; ++i) {
        s->lambda_old[i] = s->lambda[i];
        s->log_lambda_old[i] = s->log_lambda[i];
    }
    return 1;
}

/* logit_weight_diff's per-vector term (gmm_param.hpp:221-248) */
static double logit_term(const double *w)
{
    double sum_lw = 1, sum_llw = 0;
    for (int d = 0; d != K - 1; ++d) {
        const double r = w[d] / w[K - 1];
        sum_lw += r;
        sum_llw += log(r);
    }
    sum_llw -= K * log(sum_lw);
    return sum_llw;
}

/* gmm_move_weight::move_state (gmm_move.hpp:86-117) */
static int move_weight(const gmm_model *m, gmm_param *s, orc_threefry *e,
                       double sd)
{
    orc_normal rw;
    orc_normal_reset(&rw);
    save_old(m, s);
    double sum_weight = 1;
    for (int d = 0; d != K - 1; ++d) {
        s->weight[d] = log(s->weight[d] / s->weight[K - 1]);
        s->weight[d] += orc_normal_threefry(&rw, e, 0.0, sd);
        s->weight[d] = exp(s->weight[d]);
        sum_weight += s->weight[d];
    }
    s->weight[K - 1] = 1;
    for (int d = 0; d != K; ++d)
        s->weight[d] /= sum_weight;
    log_target(m, s);
    const double p =
        s->lt - s->lt_old + (logit_term(s->weight) - logit_term(s->weight_old));
    const double u = log(canonical64(e) * 1.0 + 0.0);
    reject_common(s, p, u);
    if (p < u) {
        for (int i = 0; i != K; ++i)
            s->weight[i] = s->weight_old[i];
        return 0;
    }
    for (int i = 0; i != K; ++i)
        s->weight_old[i] = s->weight[i];
    return 1;
}

/* gmm_init::initialize_state (gmm_init.hpp:51-76) */
static void init_particle(const gmm_model *m, gmm_param *s, orc_threefry *e)
{
    orc_normal nmu, nlambda, nweight;
    orc_normal_reset(&nmu);
    orc_normal_reset(&nlambda);
    orc_normal_reset(&nweight);
    double sum_weight = 0;
    for (int d = 0; d != K; ++d) {
        s->mu[d] = orc_normal_threefry(&nmu, e, m->mu0, m->sd0);
        s->lambda[d] = orc_gamma_threefry(&nlambda, e, m->shape0, m->scale0);
        s->weight[d] = orc_gamma_threefry(&nweight, e, 1.0, 1.0);
        sum_weight += s->weight[d];
    }
    for (int d = 0; d != K; ++d)
        s->weight[d] /= sum_weight;
    log_target(m, s);
}

/* gmm_param's copy assignment (gmm_param.hpp:62-77): parameters and the
 * three log densities. */
static void copy_param(gmm_param *dst, const gmm_param *src)
{
    for (int i = 0; i != K; ++i) {
        dst->mu[i] = src->mu[i];
        dst->lambda[i] = src->lambda[i];
        dst->log_lambda[i] = src->log_lambda[i];
        dst->weight[i] = src->weight[i];
    }
    dst->lp = src->lp;
    dst->ll = src->ll;
    dst->lt = src->lt;
}

/* vsmc::Seed::get (rng/seed.hpp:102,149) */
static uint32_t seed_next(uint32_t s) { return s == 0xFFFFFFFFu ? 1u : s + 1u; }

double orc_gmm_smc(const double *data, size_t n, size_t N, size_t iters,
                   int power, int sweeps, double sd, int scheme,
                   double threshold, uint32_t seed, double *ess_out,
                   int32_t *res_out, double *zinc_out, double *integ_out,
                   double *grid_out, int64_t *acc_out, double *params,
                   double *lw_out, uint64_t *words, double *path_logz)
{
    gmm_model m;
    model_init(&m, data, n);
    gmm_param *s = (gmm_param *)calloc(N, sizeof(gmm_param));
    gmm_param *tmp = (gmm_param *)calloc(N, sizeof(gmm_param));
    orc_threefry *eng = (orc_threefry *)calloc(N, sizeof(orc_threefry));
    double *w = (double *)malloc(N * sizeof(double));
    double *lw = (double *)malloc(N * sizeof(double));
    double *inc = (double *)malloc(N * sizeof(double));
    int64_t *rep = (int64_t *)malloc(N * sizeof(int64_t));
    int64_t *cf = (int64_t *)malloc(N * sizeof(int64_t));
    const size_t nacc = 1 + 3 * (size_t)sweeps;

    /* Seed::set(seed); Particle: RngSet<Threefry4x64, Vector> takes one
     * Seed::get() per particle, then the resample engine one more
     * (core/particle.hpp:64-70, rng/rng_set.hpp:100-135). */
    uint32_t sg = (uint32_t)(seed % 0xFFFFFFFFu);
    for (size_t i = 0; i != N; ++i) {
        sg = seed_next(sg);
        orc_threefry_seed(&eng[i], sg);
    }
    orc_threefry rrng;
    sg = seed_next(sg);
    orc_threefry_seed(&rrng, sg);

    /* initialize: do_reset, gmm_init (alpha 0, equal weights), do_resample,
     * path evaluation (core/sampler.hpp:450-463, 758-781). */
    double ess = orc_set_equal_weight(N, lw, w);
    m.alpha = 0;
    m.alpha_inc = 0;
    for (size_t i = 0; i != N; ++i)
        init_particle(&m, &s[i], &eng[i]);
    double zconst = 0, plogz = 0, prev_grid = 0, prev_integ = 0;
    for (size_t t = 0; t <= iters; ++t) {
        int64_t acc[1 + 3 * 64];
        memset(acc, 0, sizeof(acc));
        if (t > 0) {
            /* move_smc::operator() (example/include/move_smc.hpp:51-75) */
            if (m.alpha <= 0)
                zconst = 0;
            const double b = (double)t / (double)iters;
            double a = 1;
            for (int p = 0; p != power; ++p)
                a *= b;
            /* gmm_state::alpha (gmm_state.hpp:159-168) */
            a = a < 1 ? a : 1;
            a = a > 0 ? a : 0;
            m.alpha_inc = a > 0 ? a - m.alpha : 0;
            m.alpha = a;
            double sum = 0;
            for (size_t i = 0; i != N; ++i) {
                inc[i] = s[i].ll * m.alpha_inc;
                sum += w[i] * exp(inc[i]);
            }
            const double before = zconst;
            zconst += log(sum);
            /* the increment as the difference of the running sums (the
             * reference's zconst() is only seen after each iterate) */
            if (zinc_out)
                zinc_out[t] = t == 1 ? zconst : zconst - before;
            ess = orc_add_log_weight(N, lw, w, inc);
        } else if (zinc_out) {
            zinc_out[0] = 0;
        }
        /* do_resample (core/sampler.hpp:816-822; particle.hpp:230-250) */
        const int resampled = ess < threshold * (double)N;
        if (ess_out)
            ess_out[t] = ess;
        if (res_out)
            res_out[t] = resampled;
        if (resampled) {
            orc_resample(scheme, N, N, &rrng, w, rep, NULL, NULL);
            orc_cfrp_trans(N, N, rep, cf);
            memcpy(tmp, s, N * sizeof(gmm_param));
            for (size_t i = 0; i != N; ++i)
                if ((size_t)cf[i] != i)
                    copy_param(&s[i], &tmp[cf[i]]);
            ess = orc_set_equal_weight(N, lw, w);
        }
        /* the MCMC queue: sweeps x (mu, lambda, weight) */
        if (t > 0) {
            for (size_t i = 0; i != N; ++i)
                for (int k = 0; k != sweeps; ++k) {
                    acc[1 + 3 * k] += move_mu(&m, &s[i], &eng[i], sd);
                    acc[2 + 3 * k] += move_lambda(&m, &s[i], &eng[i], sd);
                    acc[3 + 3 * k] += move_weight(&m, &s[i], &eng[i], sd);
                }
        }
        if (acc_out)
            for (size_t k = 0; k != nacc; ++k)
                acc_out[t * nacc + k] = acc[k];
        /* Path::eval + push_back (core/path.hpp:170-239): integrand
         * dot(W, log likelihood), grid alpha, trapezoid rule. */
        double integ = 0;
        for (size_t i = 0; i != N; ++i)
            integ += w[i] * s[i].ll;
        const double grid = m.alpha;
        if (t > 0)
            plogz += 0.5 * (grid - prev_grid) * (integ + prev_integ);
        prev_grid = grid;
        prev_integ = integ;
        if (integ_out)
            integ_out[t] = integ;
        if (grid_out)
            grid_out[t] = grid;
    }
    const double llc = -0.5 * (double)n * ORC_LN_PI_2;
    if (params)
        for (size_t i = 0; i != N; ++i) {
            double *o = params + i * 14;
            for (int d = 0; d != K; ++d) {
                o[d] = s[i].mu[d];
                o[4 + d] = s[i].lambda[d];
                o[8 + d] = s[i].weight[d];
            }
            o[12] = s[i].lp;
            o[13] = s[i].ll;
        }
    if (lw_out)
        memcpy(lw_out, lw, N * sizeof(double));
    if (words)
        for (size_t i = 0; i != N; ++i)
            words[i] = orc_threefry_words_used(&eng[i]);
    if (path_logz)
        *path_logz = plogz + llc;
    free(s);
    free(tmp);
    free(eng);
    free(w);
    free(lw);
    free(inc);
    free(rep);
    free(cf);
    return zconst + llc;
}
