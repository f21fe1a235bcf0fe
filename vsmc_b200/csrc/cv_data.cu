// cv_data.cu -- host-side simulation of the CV Student-t observation series
// (the workload's synthetic data): state (0, 0, 1, 1), constant-velocity
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
