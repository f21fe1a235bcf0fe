// generic_main.cu -- two user models written against vsmc::Sampler<T> with
// device moves (include/vsmc_b200/smc.cuh), the way a vSMC user writes them
// against the SMP backends:
//
//   cv     the constant-velocity Student-t filter of the repository's
//          reference harness (example/pf/include/pf_smp.hpp:73-258 with the
//          counter layout {block, step, id, stream}); RngSet<Philox4x32,
//          Scalar> positioned per particle and step;
//   paper  example/paper/src/paper_pf.cpp:44-161: sd sqrt(0.02) and
//          sqrt(0.001), the reference's default RngSet<Threefry4x64, Vector>
//          (one engine per particle slot), Stratified resampling.
//
// Usage: generic_main cv N T scheme obs.bin out.tsv
//        generic_main paper N T obs.bin out.tsv
// obs.bin holds T x-values then T y-values (doubles).  Writes `os <<
// sampler` to out.tsv and prints the log-evidence.  Compiled with
// --fmad=false so that the per-particle arithmetic rounds like the
// reference's x86 build (no contraction into FMAs).
#include <vsmc_b200/smc.cuh>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>

namespace {

struct cv_param {
    double dt, sd_pos, sd_vel, sd_pos0, sd_vel0, scale, nu;
};

// cv_state::log_likelihood as the harness writes it
__device__ double cv_log_likelihood(const cv_param &p, double x, double y,
                                    double ox, double oy)
{
    double llh_x = p.scale * (x - ox);
    double llh_y = p.scale * (y - oy);
    llh_x = log(1 + llh_x * llh_x / p.nu);
    llh_y = log(1 + llh_y * llh_y / p.nu);
    return -0.5 * (p.nu + 1) * (llh_x + llh_y);
}

class cv : public vsmc::StateCUDA<4>
{
  public:
    typedef vsmc::RngSet<vsmc::Philox4x32, vsmc::Scalar> rng_set_type;
    explicit cv(size_type N) : vsmc::StateCUDA<4>(N) {}
};

struct cv_data {
    cv_param prm;
    const double *obs_x;
    const double *obs_y;
    unsigned stream;
};

class cv_init : public vsmc::InitializeCUDA<cv, cv_init>
{
  public:
    explicit cv_init(const cv_data &d) : d_(d) {}

    __device__ std::size_t initialize_state(vsmc::SingleParticle<cv> sp)
    {
        vsmc::NormalDistribution norm_pos(0, d_.prm.sd_pos0);
        vsmc::NormalDistribution norm_vel(0, d_.prm.sd_vel0);
        vsmc::PhiloxEngineCUDA &eng = sp.rng();
        eng.ctr(make_uint4(0u, 0u, (unsigned)sp.id(), d_.stream));
        sp.state(0) = norm_pos(eng);
        sp.state(1) = norm_pos(eng);
        sp.state(2) = norm_vel(eng);
        sp.state(3) = norm_vel(eng);
        sp.set_log_weight(cv_log_likelihood(d_.prm, sp.state(0), sp.state(1),
                                            d_.obs_x[0], d_.obs_y[0]));
        return 1;
    }

  private:
    cv_data d_;
};

class cv_move : public vsmc::MoveCUDA<cv, cv_move>
{
  public:
    explicit cv_move(const cv_data &d) : d_(d) {}

    __device__ std::size_t move_state(std::size_t iter,
                                      vsmc::SingleParticle<cv> sp)
    {
        vsmc::NormalDistribution norm_pos(0, d_.prm.sd_pos);
        vsmc::NormalDistribution norm_vel(0, d_.prm.sd_vel);
        vsmc::PhiloxEngineCUDA &eng = sp.rng();
        eng.ctr(make_uint4(0u, (unsigned)iter, (unsigned)sp.id(), d_.stream));
        sp.state(0) += norm_pos(eng) + d_.prm.dt * sp.state(2);
        sp.state(1) += norm_pos(eng) + d_.prm.dt * sp.state(3);
        sp.state(2) += norm_vel(eng);
        sp.state(3) += norm_vel(eng);
        sp.add_log_weight(cv_log_likelihood(d_.prm, sp.state(0), sp.state(1),
                                            d_.obs_x[iter], d_.obs_y[iter]));
        return 1;
    }

  private:
    cv_data d_;
};

// the position monitor (cv_est of the harness; cv_monitor_state of
// paper_pf.cpp) for either value type
template <typename T>
class pos_est : public vsmc::MonitorEvalCUDA<T, pos_est<T> >
{
  public:
    __device__ void monitor_state(std::size_t, std::size_t dim,
                                  vsmc::ConstSingleParticle<T> csp,
                                  double *res) const
    {
        for (std::size_t d = 0; d != dim; ++d)
            res[d] = csp.state(d);
    }
};

// ---- example/paper/src/paper_pf.cpp ----------------------------------
class paper_cv : public vsmc::StateCUDA<4>
{
  public:
    explicit paper_cv(size_type N) : vsmc::StateCUDA<4>(N) {}
};

__device__ double paper_log_likelihood(double x, double y, double ox,
                                       double oy)
{
    const double scale = 10;
    const double nu = 10;
    double llh_x = scale * (x - ox);
    double llh_y = scale * (y - oy);
    llh_x = log(1 + llh_x * llh_x / nu);
    llh_y = log(1 + llh_y * llh_y / nu);
    return -0.5 * (nu + 1) * (llh_x + llh_y);
}

class paper_init : public vsmc::InitializeCUDA<paper_cv, paper_init>
{
  public:
    paper_init(const double *ox, const double *oy) : ox_(ox), oy_(oy) {}

    __device__ std::size_t
    initialize_state(vsmc::SingleParticle<paper_cv> sp)
    {
        const double sd_pos0 = 2;
        const double sd_vel0 = 1;
        vsmc::NormalDistribution norm_pos(0, sd_pos0);
        vsmc::NormalDistribution norm_vel(0, sd_vel0);
        sp.state(0) = norm_pos(sp.rng());
        sp.state(1) = norm_pos(sp.rng());
        sp.state(2) = norm_vel(sp.rng());
        sp.state(3) = norm_vel(sp.rng());
        sp.set_log_weight(
            paper_log_likelihood(sp.state(0), sp.state(1), ox_[0], oy_[0]));
        return 0;
    }

  private:
    const double *ox_, *oy_;
};

class paper_move : public vsmc::MoveCUDA<paper_cv, paper_move>
{
  public:
    paper_move(const double *ox, const double *oy) : ox_(ox), oy_(oy) {}

    __device__ std::size_t move_state(std::size_t iter,
                                      vsmc::SingleParticle<paper_cv> sp)
    {
        const double sd_pos = sqrt(0.02);
        const double sd_vel = sqrt(0.001);
        const double delta = 0.1;
        vsmc::NormalDistribution norm_pos(0, sd_pos);
        vsmc::NormalDistribution norm_vel(0, sd_vel);
        sp.state(0) += norm_pos(sp.rng()) + delta * sp.state(2);
        sp.state(1) += norm_pos(sp.rng()) + delta * sp.state(3);
        sp.state(2) += norm_vel(sp.rng());
        sp.state(3) += norm_vel(sp.rng());
        sp.add_log_weight(paper_log_likelihood(sp.state(0), sp.state(1),
                                               ox_[iter], oy_[iter]));
        return 0;
    }

  private:
    const double *ox_, *oy_;
};

std::vector<double> read_obs(const char *path, std::size_t T)
{
    std::vector<double> v(2 * T);
    std::FILE *f = std::fopen(path, "rb");
    if (f == nullptr || std::fread(v.data(), 8, 2 * T, f) != 2 * T) {
        std::fprintf(stderr, "cannot read %s\n", path);
        std::exit(1);
    }
    std::fclose(f);
    return v;
}

int run_cv(std::size_t N, std::size_t T, int scheme, const char *obs,
           const char *out)
{
    std::vector<double> o = read_obs(obs, T);
    vsmc_b200::DeviceVector<double> dobs(2 * T);
    dobs.upload(o.data(), 2 * T);
    cv_data d;
    d.prm = cv_param{0.1, 0.02, 0.5, 2.0, 1.0, 10.0, 10.0};
    d.obs_x = dobs.data();
    d.obs_y = dobs.data() + T;
    d.stream = 0;
    vsmc::Seed::instance().set(101);
    vsmc::Sampler<cv> sampler(N, static_cast<vsmc::ResampleScheme>(scheme),
                              0.5, T);
    sampler.init(cv_init(d)).move(cv_move(d), false);
    sampler.monitor("pos", 2, pos_est<cv>());
    sampler.monitor("pos").name(0) = "pos.x";
    sampler.monitor("pos").name(1) = "pos.y";
    sampler.initialize();
    sampler.iterate(T - 1);
    std::ofstream f(out);
    f << sampler;
    std::printf("%.17g\n", sampler.particle().log_evidence());
    return 0;
}

int run_paper(std::size_t N, std::size_t T, const char *obs, const char *out)
{
    std::vector<double> o = read_obs(obs, T);
    vsmc_b200::DeviceVector<double> dobs(2 * T);
    dobs.upload(o.data(), 2 * T);
    const double *ox = dobs.data(), *oy = dobs.data() + T;
    vsmc::Seed::instance().set(101);
    vsmc::Sampler<paper_cv> sampler(N, vsmc::Stratified, 0.5, T);
    sampler.init(paper_init(ox, oy));
    sampler.move(paper_move(ox, oy), false);
    sampler.monitor("pos", 2, pos_est<paper_cv>());
    sampler.initialize();
    sampler.iterate(T - 1);
    std::ofstream f(out);
    f << sampler;
    std::printf("%.17g\n", sampler.particle().log_evidence());
    return 0;
}

} // namespace

int main(int argc, char **argv)
{
    try {
        if (argc == 7 && std::string(argv[1]) == "cv")
            return run_cv(std::strtoull(argv[2], nullptr, 10),
                          std::strtoull(argv[3], nullptr, 10),
                          std::atoi(argv[4]), argv[5], argv[6]);
        if (argc == 6 && std::string(argv[1]) == "paper")
            return run_paper(std::strtoull(argv[2], nullptr, 10),
                             std::strtoull(argv[3], nullptr, 10), argv[4],
                             argv[5]);
    } catch (const std::exception &e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    std::fprintf(stderr, "usage: generic_main cv|paper ...\n");
    return 2;
}
