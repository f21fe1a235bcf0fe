// Test driver for the C++ interface (include/vsmc_b200/vsmc_cuda.hpp).
// Written the way a vSMC program is, with the device types in place of the
// host ones.  Inputs and outputs are raw little-endian binary files so that
// tests/test_gpu_facade.py can compare them with the golden fixtures.
//
//   facade_main pf N T scheme form obs.bin out.tsv
//       Seed::set(101); CVSampler(N, scheme, 0.5) over the 2T observations
//       (x then y) in obs.bin; writes `os << sampler` (Sampler::print) and
//       prints the log-evidence.
//   facade_main resample scheme seed skip N1 w1.bin rep1.bin [N2 ...]
//       for each case: Resample<scheme>()(N, N, rng, w, rep) with a fresh
//       Threefry4x64(seed) after skip draws and rep as std::size_t, written
//       as int64; prints the words drawn per case.
//   facade_main weights N lw.bin inc.bin w.bin
//       WeightSetCUDA: set_log_weight(lw), add_log_weight(inc), read_weight;
//       prints the ESS.
//   facade_main gmm N iters sweeps scheme data.bin n out.tsv
//       Seed::set(101); GmmSampler over the n doubles of data.bin (alpha_t =
//       (t/iters)^4, sd 0.1, threshold 0.5); writes `os << sampler` and
//       prints the SMC and path log-evidence.
//   facade_main particle N scheme seed out.bin
//       ParticleCUDA<2>: state (i, -i), weights from log-weights
//       -((i mod 7) - 3)^2, resample(scheme, 1.0); writes the resampled
//       first column (N doubles) and prints the engine words drawn.
#include <vsmc_b200/vsmc_cuda.hpp>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

namespace {

template <typename T>
std::vector<T> read_bin(const char *path, std::size_t n)
{
    std::vector<T> v(n);
    std::ifstream f(path, std::ios::binary);
    f.read(reinterpret_cast<char *>(v.data()),
           static_cast<std::streamsize>(n * sizeof(T)));
    if (!f)
        throw std::runtime_error(std::string("cannot read ") + path);
    return v;
}

template <typename T>
void write_bin(const char *path, const std::vector<T> &v)
{
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char *>(v.data()),
            static_cast<std::streamsize>(v.size() * sizeof(T)));
}

template <vsmc_b200::ResampleScheme S>
void resample_with(std::size_t N, vsmc_b200::Threefry4x64 &rng,
                   const double *w, std::size_t *rep)
{
    vsmc_b200::Resample<S>()(N, N, rng, w, rep);
}

int pf(int argc, char **argv)
{
    if (argc != 8)
        return 2;
    const std::size_t N = std::strtoull(argv[2], nullptr, 10);
    const std::size_t T = std::strtoull(argv[3], nullptr, 10);
    const int scheme = std::atoi(argv[4]);
    const int form = std::atoi(argv[5]);
    std::vector<double> obs = read_bin<double>(argv[6], 2 * T);
    vsmc_b200::Seed::instance().set(101);
    vsmc_b200::CVSampler sampler(
        N, static_cast<vsmc_b200::ResampleScheme>(scheme), 0.5, T,
        static_cast<vsmc_b200::Form>(form));
    sampler.monitor_name(0) = "pos.x";
    sampler.monitor_name(1) = "pos.y";
    sampler.initialize(obs.data(), obs.data() + T, T);
    sampler.iterate(T - 1);
    std::ofstream est(argv[7]);
    est << sampler;
    std::printf("%.17g\n", sampler.log_evidence());
    return 0;
}

int resample(int argc, char **argv)
{
    if (argc < 8 || (argc - 5) % 3 != 0)
        return 2;
    const int scheme = std::atoi(argv[2]);
    const std::uint64_t seed = std::strtoull(argv[3], nullptr, 10);
    const std::uint64_t skip = std::strtoull(argv[4], nullptr, 10);
    for (int a = 5; a + 2 < argc; a += 3) {
        const std::size_t N = std::strtoull(argv[a], nullptr, 10);
        std::vector<double> w = read_bin<double>(argv[a + 1], N);
        vsmc_b200::Threefry4x64 rng(seed);
        rng.discard(skip);
        const std::uint64_t before = rng.words_used();
        std::vector<std::size_t> rep(N);
        switch (scheme) {
        case vsmc_b200::Multinomial:
            resample_with<vsmc_b200::Multinomial>(N, rng, w.data(),
                                                  rep.data());
            break;
        case vsmc_b200::Residual:
            resample_with<vsmc_b200::Residual>(N, rng, w.data(), rep.data());
            break;
        case vsmc_b200::Stratified:
            resample_with<vsmc_b200::Stratified>(N, rng, w.data(),
                                                 rep.data());
            break;
        case vsmc_b200::Systematic:
            resample_with<vsmc_b200::Systematic>(N, rng, w.data(),
                                                 rep.data());
            break;
        case vsmc_b200::ResidualStratified:
            resample_with<vsmc_b200::ResidualStratified>(N, rng, w.data(),
                                                         rep.data());
            break;
        default:
            resample_with<vsmc_b200::ResidualSystematic>(N, rng, w.data(),
                                                         rep.data());
            break;
        }
        std::vector<std::int64_t> out(rep.begin(), rep.end());
        write_bin(argv[a + 2], out);
        std::printf("%llu\n",
                    static_cast<unsigned long long>(rng.words_used() - before));
    }
    return 0;
}

int weights(int argc, char **argv)
{
    if (argc != 6)
        return 2;
    const std::size_t N = std::strtoull(argv[2], nullptr, 10);
    std::vector<double> lw = read_bin<double>(argv[3], N);
    std::vector<double> inc = read_bin<double>(argv[4], N);
    vsmc_b200::WeightSetCUDA ws(N);
    ws.set_log_weight(lw.begin());
    ws.add_log_weight(inc.begin());
    std::vector<double> w(N);
    ws.read_weight(w.begin());
    write_bin(argv[5], w);
    std::printf("%.17g\n", ws.ess());
    return 0;
}

int particle(int argc, char **argv)
{
    if (argc != 6)
        return 2;
    const std::size_t N = std::strtoull(argv[2], nullptr, 10);
    const int scheme = std::atoi(argv[3]);
    vsmc_b200::Seed::instance().set(std::strtoull(argv[4], nullptr, 10));
    vsmc_b200::ParticleCUDA<2> p(N);
    std::vector<double> c0(N), c1(N), lw(N);
    for (std::size_t i = 0; i != N; ++i) {
        c0[i] = static_cast<double>(i);
        c1[i] = -static_cast<double>(i);
        const double d = static_cast<double>(i % 7) - 3.0;
        lw[i] = -d * d;
    }
    p.value().write_state(0, c0.begin());
    p.value().write_state(1, c1.begin());
    p.weight_set().set_log_weight(lw.begin());
    const bool res =
        p.resample(static_cast<vsmc_b200::ResampleScheme>(scheme), 1.0);
    std::vector<double> out(N);
    p.value().read_state(0, out.begin());
    write_bin(argv[5], out);
    std::printf("%d %llu %.17g\n", res ? 1 : 0,
                static_cast<unsigned long long>(p.resample_rng().words_used()),
                p.weight_set().ess());
    return 0;
}

int gmm(int argc, char **argv)
{
    if (argc != 9)
        return 2;
    const std::size_t N = std::strtoull(argv[2], nullptr, 10);
    const std::size_t iters = std::strtoull(argv[3], nullptr, 10);
    const int sweeps = std::atoi(argv[4]);
    const int scheme = std::atoi(argv[5]);
    const std::size_t n = std::strtoull(argv[7], nullptr, 10);
    std::vector<double> data = read_bin<double>(argv[6], n);
    vsmc_b200::Seed::instance().set(101);
    vsmc_b200::GmmSampler sampler(
        data.data(), n, N, iters, 4, sweeps, 0.1,
        static_cast<vsmc_b200::ResampleScheme>(scheme), 0.5);
    sampler.initialize();
    sampler.iterate(iters);
    std::ofstream est(argv[8]);
    est << sampler;
    std::printf("%.17g %.17g\n", sampler.log_evidence(),
                sampler.path_log_evidence());
    return 0;
}

// Many filters through vsmc_b200::CVBatch: autotune, then the series fed
// three observations per filter at a time (append, run, read_steps).
// Writes each filter's ESS then its log-evidence increments (n x T each).
int batch(int argc, char **argv)
{
    if (argc != 6)
        return 2;
    const std::uint32_t n = static_cast<std::uint32_t>(std::atoi(argv[2]));
    const std::size_t T = std::strtoull(argv[3], nullptr, 10);
    std::vector<double> obs = read_bin<double>(argv[4], 2 * T);
    vsmc_b200::CVBatch b(n, vsmc_b200::Multinomial);
    std::vector<std::uint32_t> slots(n);
    for (std::uint32_t k = 0; k != n; ++k)
        slots[k] = b.admit(1000 + 517 * k, T, 101 + k, k);
    b.autotune(slots);
    std::vector<double> ess(n * T), dz(n * T);
    for (std::size_t t0 = 0; t0 < T; t0 += 3) {
        const std::size_t m = std::min<std::size_t>(3, T - t0);
        for (std::size_t j = 0; j != m; ++j)
            b.append(slots, std::vector<double>(n, obs[t0 + j]),
                     std::vector<double>(n, obs[T + t0 + j]));
        b.run(slots);
        const vsmc_b200::CVBatch::Steps r = b.read_steps(
            slots, std::vector<std::uint32_t>(n, static_cast<std::uint32_t>(m)));
        for (std::uint32_t k = 0; k != n; ++k)
            for (std::size_t j = 0; j != m; ++j) {
                ess[k * T + t0 + j] = r.ess[k * m + j];
                dz[k * T + t0 + j] = r.logz_inc[k * m + j];
            }
    }
    std::vector<double> out(ess);
    out.insert(out.end(), dz.begin(), dz.end());
    write_bin(argv[5], out);
    return 0;
}

} // namespace

int main(int argc, char **argv)
{
    if (argc < 2)
        return 2;
    const std::string cmd = argv[1];
    try {
        if (cmd == "pf")
            return pf(argc, argv);
        if (cmd == "resample")
            return resample(argc, argv);
        if (cmd == "weights")
            return weights(argc, argv);
        if (cmd == "particle")
            return particle(argc, argv);
        if (cmd == "gmm")
            return gmm(argc, argv);
        if (cmd == "batch")
            return batch(argc, argv);
    } catch (const vsmc_b200::RuntimeError &e) {
        std::fprintf(stderr, "RuntimeError %d: %s\n", e.status(), e.what());
        return 3;
    }
    return 2;
}
