// cv_data.cu -- host-side simulation of the workloads' synthetic data.  The
// CV Student-t observation series: state (0, 0, 1, 1), constant-velocity
// moves with Gaussian noise, positions observed with Student-t(nu) noise of
// scale 1/scale.  Step t uses a Philox4x32-10 engine keyed {obs_seed, 1}
// with counter {0, t, 0, stream_id} and one std::normal_distribution, so the
// series is a pure function of (obs_seed, stream_id, parameters).
#include "../../include/vsmc_cuda.h"
#include "../../include/vsmc_b200/rng.hpp"

#include <cmath>
#include <random>

extern "C" int vsmc_cuda_cv_simulate(const vsmc_cuda_cv_config *c,
                                     uint32_t obs_seed, uint64_t T,
                                     double *obs_x, double *obs_y,
                                     double *truth)
{
    if (c == nullptr || obs_x == nullptr || obs_y == nullptr || T == 0 ||
        !(c->nu >= 1.0) || c->nu != std::floor(c->nu))
        return VSMC_CUDA_EINVAL;
    typedef std::normal_distribution<double> normal;
    double s[4] = {0, 0, 1, 1};
    const int k = static_cast<int>(c->nu);
    for (uint64_t t = 0; t != T; ++t) {
        vsmc_b200::Philox4x32 eng(
            vsmc_b200::Philox4x32::key_type{{obs_seed, 1u}});
        eng.ctr(vsmc_b200::Philox4x32::ctr_type{
            {0u, static_cast<uint32_t>(t), 0u, c->stream_id}});
        normal nd(0, 1);
        if (t > 0) {
            double n;
            n = nd(eng, normal::param_type(0, c->sd_pos));
            s[0] += n + c->dt * s[2];
            n = nd(eng, normal::param_type(0, c->sd_pos));
            s[1] += n + c->dt * s[3];
            n = nd(eng, normal::param_type(0, c->sd_vel));
            s[2] += n;
            n = nd(eng, normal::param_type(0, c->sd_vel));
            s[3] += n;
        }
        double tv[2];
        for (int d = 0; d != 2; ++d) {
            const double z0 = nd(eng);
            double chi = 0;
            for (int i = 0; i != k; ++i) {
                const double z = nd(eng);
                chi += z * z;
            }
            tv[d] = z0 / std::sqrt(chi / c->nu);
        }
        obs_x[t] = s[0] + tv[0] / c->scale;
        obs_y[t] = s[1] + tv[1] / c->scale;
        if (truth != nullptr)
            for (int d = 0; d != 4; ++d)
                truth[t * 4 + d] = s[d];
    }
    return VSMC_CUDA_OK;
}

// The mixture data of the tempered SMC workload: point i draws its
// component k = floor(4 u) (u from std::uniform_real_distribution) and then
// mean_k + std::normal_distribution(0, 1) noise, means (-3, 0, 2, 5), on one
// Philox4x32-10 engine keyed {seed, 3} with counter 0.
extern "C" int vsmc_cuda_gmm_simulate(uint32_t seed, uint64_t n, double *out)
{
    if (out == nullptr)
        return VSMC_CUDA_EINVAL;
    static const double means[4] = {-3.0, 0.0, 2.0, 5.0};
    vsmc_b200::Philox4x32 eng(vsmc_b200::Philox4x32::key_type{{seed, 3u}});
    std::uniform_real_distribution<double> u01(0, 1);
    typedef std::normal_distribution<double> normal;
    normal nd;
    for (uint64_t i = 0; i != n; ++i) {
        const double u = u01(eng);
        int k = static_cast<int>(u * 4.0);
        k = k > 3 ? 3 : k;
        out[i] = nd(eng, normal::param_type(means[k], 1.0));
    }
    return VSMC_CUDA_OK;
}
