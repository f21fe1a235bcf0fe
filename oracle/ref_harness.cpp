// ref_harness.cpp -- drives the UNMODIFIED vSMC headers (TEST INFRASTRUCTURE)
//
// Built by oracle/Makefile against the vSMC include tree into oracle/_ref/
// (git-ignored).  It is the pinned reference that the C restatement
// (smc_oracle.c) and the golden fixtures under tests/golden/ are checked
// against, and the timed CPU baseline of bench.py (StateOMP / StateSTD /
// StateSEQ backends).  Nothing in the product links it.
//
// Everything below is vSMC API use; the model is the constant-velocity
// Student-t particle filter of example/pf/include/pf_smp.hpp:73-258 with the
// workload's parameters (process sd 0.02 / 0.5, dt 0.1) and the counter
// layout {block, step, particle id, stream} (the example's (id<<16)+iter
// packing aliases once N >= 2^16).
#include <vsmc/core/sampler.hpp>
#include <vsmc/core/state_matrix.hpp>
#include <vsmc/resample/resample.hpp>
#include <vsmc/rng/philox.hpp>
#include <vsmc/rng/threefry.hpp>
#include <vsmc/rng/rng_set.hpp>
#include <vsmc/smp/adapter.hpp>
#include <vsmc/smp/backend_omp.hpp>
#include <vsmc/smp/backend_seq.hpp>
#include <vsmc/smp/backend_std.hpp>

#include <omp.h>

#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <sstream>
#include <string>
#include <vector>

namespace {

const std::size_t PosX = 0;
const std::size_t PosY = 1;
const std::size_t VelX = 2;
const std::size_t VelY = 3;
const std::size_t LogL = 4;

struct cv_param {
    double dt, sd_pos, sd_vel, sd_pos0, sd_vel0, scale, nu;
};

template <template <typename> class StateB>
class cv_state : public StateB<vsmc::StateMatrix<vsmc::ColMajor, 5, double> >
{
    public :

    typedef vsmc::RngSet<vsmc::Philox4x32, vsmc::Scalar> rng_set_type;
    typedef StateB<vsmc::StateMatrix<vsmc::ColMajor, 5, double> > base;
    typedef typename base::size_type size_type;

    cv_state (size_type N) : base(N), zconst(0), stream(0),
        rec_cf(VSMC_NULLPTR), rec_w(VSMC_NULLPTR), rec_w_step(0),
        words_before(VSMC_NULLPTR) {}

    // Particle::resample hands the value its copy_from vector here
    // (core/particle.hpp:245); the trace keeps each step's row before the
    // backend's own copy runs.
    template <typename IntType>
    void copy (size_type N, const IntType *copy_from)
    {
        if (rec_cf != VSMC_NULLPTR && copy_from != VSMC_NULLPTR) {
            const std::size_t row = zinc.size() - 1;
            for (size_type i = 0; i != N; ++i)
                rec_cf[row * N + i] = static_cast<int32_t>(copy_from[i]);
        }
        base::copy(N, copy_from);
    }

    double log_likelihood (std::size_t iter, size_type id) const
    {
        using std::log;
        double llh_x = prm.scale * (this->state(id, vsmc::Position<PosX>())
                - obs_x[iter]);
        double llh_y = prm.scale * (this->state(id, vsmc::Position<PosY>())
                - obs_y[iter]);
        llh_x = log(1 + llh_x * llh_x / prm.nu);
        llh_y = log(1 + llh_y * llh_y / prm.nu);
        return -0.5 * (prm.nu + 1) * (llh_x + llh_y);
    }

    cv_param prm;
    const double *obs_x;
    const double *obs_y;
    double zconst;
    std::vector<double> zinc;
    unsigned stream;

    // trace of a run (ref_cv_filter_trace): each step's copy_from (T x N),
    // the normalised weights one step resamples with, and the resample
    // engine's word count before each step's resampling
    int32_t *rec_cf;
    double *rec_w;
    std::size_t rec_w_step;
    uint64_t *words_before;
};

// Words drawn from a Threefry4x64 engine since its counter was zero.  The
// buffer index is private, so it is read back from the engine's stream form
// "ctr(4) par(5) buffer(4) index" (threefry.hpp:425-440).
uint64_t threefry_words_used (const vsmc::Threefry4x64 &eng)
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

// Per-particle engine: a copy of the particle's RngSet engine with the
// counter set to {0, step, id, stream} (pf_smp.hpp:159-164, 218-227).
template <typename T>
typename vsmc::Particle<T>::rng_type particle_engine (
        vsmc::SingleParticle<T> sp, std::size_t iter)
{
    typedef typename vsmc::Particle<T>::rng_type rng_type;
    rng_type eng(sp.rng());
    typename rng_type::ctr_type ctr;
    vsmc::Counter<typename rng_type::ctr_type>::reset(ctr);
    ctr[1] = static_cast<uint32_t>(iter);
    ctr[2] = static_cast<uint32_t>(sp.id());
    ctr[3] = static_cast<uint32_t>(sp.particle().value().stream);
    eng.ctr(ctr);
    return eng;
}

template <typename T>
void add_with_evidence (vsmc::Particle<T> &particle, std::vector<double> &w,
        std::vector<double> &inc, bool set)
{
    using std::exp;
    using std::log;
    inc.resize(particle.size());
    w.resize(particle.size());
    particle.value().read_state(vsmc::Position<LogL>(), &inc[0]);
    particle.weight_set().read_weight(&w[0]);
    double sum = 0;                       // example/include/move_smc.hpp:63-71
    for (std::size_t i = 0; i != inc.size(); ++i)
        sum += w[i] * exp(inc[i]);
    particle.value().zconst += log(sum);
    particle.value().zinc.push_back(log(sum));
    if (set)
        particle.weight_set().set_log_weight(&inc[0]);
    else
        particle.weight_set().add_log_weight(&inc[0]);
    T &value = particle.value();
    const std::size_t step = value.zinc.size() - 1;
    if (value.words_before != VSMC_NULLPTR)
        value.words_before[step] = threefry_words_used(particle.resample_rng());
    if (value.rec_w != VSMC_NULLPTR && step == value.rec_w_step)
        particle.weight_set().read_weight(value.rec_w);
}

template <template <typename> class StateB,
         template <typename, typename> class InitB>
class cv_init : public InitB<cv_state<StateB>, cv_init<StateB, InitB> >
{
    public :

    typedef cv_state<StateB> cv;

    std::size_t initialize_state (vsmc::SingleParticle<cv> sp)
    {
        const cv_param &p = sp.particle().value().prm;
        vsmc::cxx11::normal_distribution<> norm_pos(0, p.sd_pos0);
        vsmc::cxx11::normal_distribution<> norm_vel(0, p.sd_vel0);
        typename vsmc::Particle<cv>::rng_type eng = particle_engine(sp, 0);
        sp.template state<PosX>() = norm_pos(eng);
        sp.template state<PosY>() = norm_pos(eng);
        sp.template state<VelX>() = norm_vel(eng);
        sp.template state<VelY>() = norm_vel(eng);
        sp.template state<LogL>() =
            sp.particle().value().log_likelihood(0, sp.id());
        return 1;
    }

    void initialize_param (vsmc::Particle<cv> &, void *) {}

    void post_processor (vsmc::Particle<cv> &particle)
    {add_with_evidence(particle, w_, inc_, true);}

    private :

    std::vector<double> w_, inc_;
};

template <template <typename> class StateB,
         template <typename, typename> class MoveB>
class cv_move : public MoveB<cv_state<StateB>, cv_move<StateB, MoveB> >
{
    public :

    typedef cv_state<StateB> cv;

    std::size_t move_state (std::size_t iter, vsmc::SingleParticle<cv> sp)
    {
        const cv_param &p = sp.particle().value().prm;
        vsmc::cxx11::normal_distribution<> norm_pos(0, p.sd_pos);
        vsmc::cxx11::normal_distribution<> norm_vel(0, p.sd_vel);
        typename vsmc::Particle<cv>::rng_type eng = particle_engine(sp, iter);
        sp.state(vsmc::Position<PosX>()) += norm_pos(eng) +
            p.dt * sp.state(vsmc::Position<VelX>());
        sp.state(vsmc::Position<PosY>()) += norm_pos(eng) +
            p.dt * sp.state(vsmc::Position<VelY>());
        sp.state(vsmc::Position<VelX>()) += norm_vel(eng);
        sp.state(vsmc::Position<VelY>()) += norm_vel(eng);
        sp.state(vsmc::Position<LogL>()) =
            sp.particle().value().log_likelihood(iter, sp.id());
        return 1;
    }

    void post_processor (std::size_t, vsmc::Particle<cv> &particle)
    {add_with_evidence(particle, w_, inc_, false);}

    private :

    std::vector<double> w_, inc_;
};

template <typename T>
void cv_est (std::size_t, std::size_t, vsmc::ConstSingleParticle<T> csp,
        double *res)
{
    res[0] = csp.state(vsmc::Position<0>());
    res[1] = csp.state(vsmc::Position<1>());
}

struct run_out {
    double *ess;
    int32_t *resampled;
    double *logz_inc;
    double *mean_x;
    double *mean_y;
    double *final_state;
    double *final_lw;
    uint64_t *words_used;
    double *seconds;
    double *step_seconds;
    std::string *summary; // Sampler::print output (sampler.hpp:684-721)
    int32_t *rec_cf;      // trace: T x N copy_from rows (nullable)
    double *rec_w;        // trace: the weights step rec_w_step resamples
    uint64_t rec_w_step;
    uint64_t *words_before; // trace: T engine word counts (nullable)
};

template <template <typename> class StateB,
         template <typename, typename> class InitB,
         template <typename, typename> class MoveB,
         template <typename, typename> class MonB>
double run_filter (const cv_param &prm, std::size_t N, std::size_t T,
        int scheme, double threshold, unsigned seed, unsigned stream,
        const double *ox, const double *oy, run_out *out)
{
    typedef cv_state<StateB> cv;
    vsmc::Seed::instance().set(seed);
    vsmc::Sampler<cv> sampler(N, static_cast<vsmc::ResampleScheme>(scheme),
            threshold);
    sampler.particle().value().prm = prm;
    sampler.particle().value().obs_x = ox;
    sampler.particle().value().obs_y = oy;
    sampler.particle().value().stream = stream;
    if (out) {
        sampler.particle().value().rec_cf = out->rec_cf;
        sampler.particle().value().rec_w = out->rec_w;
        sampler.particle().value().rec_w_step = out->rec_w_step;
        sampler.particle().value().words_before = out->words_before;
    }
    sampler
        .init(cv_init<StateB, InitB>())
        .move(cv_move<StateB, MoveB>(), false)
        .monitor("pos", 2, vsmc::MonitorEvalAdapter<cv, MonB>(cv_est<cv>));

    auto t0 = std::chrono::steady_clock::now();
    sampler.initialize();
    auto tp = std::chrono::steady_clock::now();
    if (out && out->step_seconds)
        out->step_seconds[0] = std::chrono::duration<double>(tp - t0).count();
    for (std::size_t t = 1; t < T; ++t) {
        sampler.iterate(1);
        auto tn = std::chrono::steady_clock::now();
        if (out && out->step_seconds)
            out->step_seconds[t] = std::chrono::duration<double>(tn - tp).count();
        tp = tn;
    }
    auto t1 = std::chrono::steady_clock::now();

    if (out) {
        if (out->seconds)
            *out->seconds = std::chrono::duration<double>(t1 - t0).count();
        for (std::size_t t = 0; t != T; ++t) {
            if (out->ess)
                out->ess[t] = sampler.ess_history(t);
            if (out->resampled)
                out->resampled[t] = sampler.resampled_history(t) ? 1 : 0;
            if (out->logz_inc)
                out->logz_inc[t] = sampler.particle().value().zinc[t];
            if (out->mean_x)
                out->mean_x[t] = sampler.monitor("pos").record(0, t);
            if (out->mean_y)
                out->mean_y[t] = sampler.monitor("pos").record(1, t);
        }
        if (out->final_state)
            for (std::size_t d = 0; d != 4; ++d)
                for (std::size_t i = 0; i != N; ++i)
                    out->final_state[d * N + i] =
                        sampler.particle().value().state(i, d);
        if (out->final_lw)
            sampler.particle().weight_set().read_log_weight(out->final_lw);
        if (out->words_used) {
            *out->words_used =
                threefry_words_used(sampler.particle().resample_rng());
        }
        if (out->summary) {
            // monitor names as the pf example sets them (pf_smp_do.hpp)
            sampler.monitor("pos").name(0) = "pos.x";
            sampler.monitor("pos").name(1) = "pos.y";
            std::stringstream ss;
            ss << sampler;
            *out->summary = ss.str();
        }
    }
    return sampler.particle().value().zconst;
}

} // namespace

extern "C" {

// Word streams of the reference engines: `n` outputs of operator()() after
// key(k), ctr(c) and `skip` discarded draws (philox.hpp:367-395,
// threefry.hpp:336-364).
void ref_philox_stream (const uint32_t *key, const uint32_t *ctr,
        uint64_t skip, uint64_t n, uint32_t *out)
{
    vsmc::Philox4x32 eng;
    vsmc::Philox4x32::key_type k;
    k[0] = key[0];
    k[1] = key[1];
    vsmc::Philox4x32::ctr_type c;
    for (int i = 0; i != 4; ++i)
        c[i] = ctr[i];
    eng.key(k);
    eng.ctr(c);
    for (uint64_t i = 0; i != skip; ++i)
        eng();
    for (uint64_t i = 0; i != n; ++i)
        out[i] = eng();
}

void ref_threefry_stream (const uint64_t *key, const uint64_t *ctr,
        uint64_t skip, uint64_t n, uint64_t *out)
{
    vsmc::Threefry4x64 eng;
    vsmc::Threefry4x64::key_type k;
    vsmc::Threefry4x64::ctr_type c;
    for (int i = 0; i != 4; ++i) {
        k[i] = key[i];
        c[i] = ctr[i];
    }
    eng.key(k);
    eng.ctr(c);
    for (uint64_t i = 0; i != skip; ++i)
        eng();
    for (uint64_t i = 0; i != n; ++i)
        out[i] = eng();
}

// Resample<Scheme> + internal::cfrp_trans on given weights, with the
// resample engine Threefry4x64 seeded `seed` after `skip` discarded words
// (Particle::resample, particle.hpp:230-250).  Returns the words drawn.
uint64_t ref_resample (int scheme, uint64_t M, uint64_t N, uint64_t seed,
        uint64_t skip, const double *w, int64_t *rep, int64_t *copy_from)
{
    vsmc::Threefry4x64 rng(seed);
    for (uint64_t i = 0; i != skip; ++i)
        rng();
    std::vector<std::size_t> r(M), cf(N);
    switch (scheme) {
        case vsmc::Multinomial :
            vsmc::ResampleType<vsmc::Multinomial>::type()(M, N, rng, w, &r[0]);
            break;
        case vsmc::Residual :
            vsmc::ResampleType<vsmc::Residual>::type()(M, N, rng, w, &r[0]);
            break;
        case vsmc::Stratified :
            vsmc::ResampleType<vsmc::Stratified>::type()(M, N, rng, w, &r[0]);
            break;
        case vsmc::Systematic :
            vsmc::ResampleType<vsmc::Systematic>::type()(M, N, rng, w, &r[0]);
            break;
        case vsmc::ResidualStratified :
            vsmc::ResampleType<vsmc::ResidualStratified>::type()(
                    M, N, rng, w, &r[0]);
            break;
        case vsmc::ResidualSystematic :
            vsmc::ResampleType<vsmc::ResidualSystematic>::type()(
                    M, N, rng, w, &r[0]);
            break;
        default :
            return 0;
    }
    if (N > 0)
        vsmc::internal::cfrp_trans(M, N, &r[0], &cf[0]);
    for (uint64_t i = 0; i != M; ++i)
        rep[i] = static_cast<int64_t>(r[i]);
    if (copy_from)
        for (uint64_t i = 0; i != N; ++i)
            copy_from[i] = static_cast<int64_t>(cf[i]);
    return threefry_words_used(rng) - skip;
}

// WeightSet::set_log_weight(lw) then add_log_weight(inc) (when inc != 0)
// (weight_set.hpp:297-331, 441-446).  Returns ESS; writes the normalised
// weights and log weights.
double ref_weight_set (uint64_t N, const double *lw, const double *inc,
        double *w_out, double *lw_out)
{
    vsmc::WeightSet ws(N);
    ws.set_log_weight(lw);
    if (inc)
        ws.add_log_weight(inc);
    ws.read_weight(w_out);
    ws.read_log_weight(lw_out);
    return ws.ess();
}

// WeightSet::set_log_weight(lw) then ess(inc, use_log) or cess(inc,
// use_log) (weight_set.hpp:132-186, 385-431): the prospective ESS / CESS.
double ref_weight_prospective (uint64_t N, const double *lw, const double *inc,
        int use_log, int cess)
{
    vsmc::WeightSet ws(N);
    ws.set_log_weight(lw);
    return cess ? ws.cess(inc, use_log != 0) : ws.ess(inc, use_log != 0);
}

// The CV Student-t bootstrap filter through Sampler<T>; backend 0 = OMP
// (StateOMP/InitializeOMP/MoveOMP/MonitorEvalOMP), 1 = STD (std::thread),
// 2 = SEQ.  nthreads > 0 sets the OpenMP thread count (OMP backend).
// step_seconds (T entries, nullable): wall time of initialize and of each
// iterate(1).
double ref_cv_filter (int backend, int nthreads, const double *param,
        uint64_t N, uint64_t T, int scheme, double threshold, unsigned seed,
        unsigned stream, const double *ox, const double *oy,
        double *ess, int32_t *resampled, double *logz_inc, double *mean_x,
        double *mean_y, double *final_state, double *final_lw,
        uint64_t *words_used, double *seconds, double *step_seconds)
{
    cv_param prm = {param[0], param[1], param[2], param[3], param[4],
        param[5], param[6]};
    run_out out = {ess, resampled, logz_inc, mean_x, mean_y, final_state,
        final_lw, words_used, seconds, step_seconds, VSMC_NULLPTR,
        VSMC_NULLPTR, VSMC_NULLPTR, 0, VSMC_NULLPTR};
    if (nthreads > 0)
        omp_set_num_threads(nthreads);
    switch (backend) {
        case 0 :
            return run_filter<vsmc::StateOMP, vsmc::InitializeOMP,
                   vsmc::MoveOMP, vsmc::MonitorEvalOMP>(prm, N, T, scheme,
                           threshold, seed, stream, ox, oy, &out);
        case 1 :
            return run_filter<vsmc::StateSTD, vsmc::InitializeSTD,
                   vsmc::MoveSTD, vsmc::MonitorEvalSTD>(prm, N, T, scheme,
                           threshold, seed, stream, ox, oy, &out);
        default :
            return run_filter<vsmc::StateSEQ, vsmc::InitializeSEQ,
                   vsmc::MoveSEQ, vsmc::MonitorEvalSEQ>(prm, N, T, scheme,
                           threshold, seed, stream, ox, oy, &out);
    }
}

// The summary table `os << sampler` writes (Sampler::print, sampler.hpp:
// 684-721) for the CV filter on the SEQ backend, copied into `buf` (at most
// cap bytes, NUL-terminated).  Returns the full length.
uint64_t ref_cv_summary (const double *param, uint64_t N, uint64_t T,
        int scheme, double threshold, unsigned seed, unsigned stream,
        const double *ox, const double *oy, char *buf, uint64_t cap)
{
    cv_param prm = {param[0], param[1], param[2], param[3], param[4],
        param[5], param[6]};
    std::string text;
    run_out out = {VSMC_NULLPTR, VSMC_NULLPTR, VSMC_NULLPTR, VSMC_NULLPTR,
        VSMC_NULLPTR, VSMC_NULLPTR, VSMC_NULLPTR, VSMC_NULLPTR, VSMC_NULLPTR,
        VSMC_NULLPTR, &text, VSMC_NULLPTR, VSMC_NULLPTR, 0, VSMC_NULLPTR};
    run_filter<vsmc::StateSEQ, vsmc::InitializeSEQ, vsmc::MoveSEQ,
        vsmc::MonitorEvalSEQ>(prm, N, T, scheme, threshold, seed, stream, ox,
                oy, &out);
    if (buf && cap > 0) {
        const uint64_t n = text.size() < cap - 1 ? text.size() : cap - 1;
        std::memcpy(buf, text.data(), n);
        buf[n] = '\0';
    }
    return text.size();
}

// ref_cv_filter (OMP backend) plus a trace of the run: cf (T x N int32,
// nullable) receives each resampling step's copy_from row as
// Particle::resample hands it to the value (rows of steps that do not
// resample are left as they are); w (N doubles, nullable) the normalised
// weights step w_step resamples with; words_before (T, nullable) the resample
// engine's words drawn before each step's resampling.
double ref_cv_filter_trace (int nthreads, const double *param, uint64_t N,
        uint64_t T, int scheme, double threshold, unsigned seed,
        unsigned stream, const double *ox, const double *oy, double *ess,
        int32_t *resampled, double *logz_inc, double *mean_x, double *mean_y,
        uint64_t *words_used, int32_t *cf, double *w, uint64_t w_step,
        uint64_t *words_before, double *seconds)
{
    cv_param prm = {param[0], param[1], param[2], param[3], param[4],
        param[5], param[6]};
    run_out out = {ess, resampled, logz_inc, mean_x, mean_y, VSMC_NULLPTR,
        VSMC_NULLPTR, words_used, seconds, VSMC_NULLPTR, VSMC_NULLPTR, cf, w,
        w_step, words_before};
    if (nthreads > 0)
        omp_set_num_threads(nthreads);
    return run_filter<vsmc::StateOMP, vsmc::InitializeOMP, vsmc::MoveOMP,
           vsmc::MonitorEvalOMP>(prm, N, T, scheme, threshold, seed, stream,
                   ox, oy, &out);
}

int ref_max_threads (void) {return omp_get_max_threads();}

} // extern "C"
