// vsmc_cuda.hpp -- C++ interface of the B200 SMC step, shaped like vSMC's.
//
// Header-only, C++11, no CUDA toolkit needed: everything goes through the
// C ABI of include/vsmc_cuda.h (link libvsmc_cuda.so).  Status codes become
// vsmc_b200::RuntimeError exceptions, the way vSMC's runtime assertions
// throw (include/vsmc/internal/assert.hpp:60-99).
//
// What replaces what (reference paths relative to the vSMC project root):
//
//   vsmc::Seed                     -> vsmc_b200::Seed (rng/seed.hpp:86-207)
//   vsmc::Philox4x32, Threefry4x64 -> vsmc_b200::Philox4x32, Threefry4x64
//                                     (include/vsmc_b200/rng.hpp)
//   vsmc::ResampleScheme           -> vsmc_b200::ResampleScheme (same values)
//   ResampleType<S>::type          -> vsmc_b200::Resample<S>: the same
//                                     (M, N, rng, weight, replication)
//                                     call, computed on the device
//   vsmc::WeightSet                -> vsmc_b200::WeightSetCUDA (device)
//   StateMatrix<ColMajor, Dim, double> with StateOMP
//                                  -> vsmc_b200::StateCUDA<Dim> (device SoA)
//   vsmc::Particle<T>              -> vsmc_b200::ParticleCUDA<Dim>
//   vsmc::Sampler<cv_state> of example/pf
//                                  -> vsmc_b200::CVSampler (the fused filter)
//   vsmc::Sampler<gmm_state> of example/gmm (tempered SMC)
//                                  -> vsmc_b200::GmmSampler
//   (no counterpart)               -> vsmc_b200::CVBatch, CVServer
#ifndef VSMC_B200_VSMC_CUDA_HPP
#define VSMC_B200_VSMC_CUDA_HPP

#include <vsmc_cuda.h>
#include <vsmc_b200/rng.hpp>

#include <cstddef>
#include <cstdint>
#include <limits>
#include <ostream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace vsmc_b200 {

// vsmc::ResampleScheme (include/vsmc/resample/common.hpp:124-131)
enum ResampleScheme {
    Multinomial = VSMC_CUDA_MULTINOMIAL,
    Residual = VSMC_CUDA_RESIDUAL,
    Stratified = VSMC_CUDA_STRATIFIED,
    Systematic = VSMC_CUDA_SYSTEMATIC,
    ResidualStratified = VSMC_CUDA_RESIDUAL_STRATIFIED,
    ResidualSystematic = VSMC_CUDA_RESIDUAL_SYSTEMATIC
};

// Precision form of the fused filter.
enum Form { FP64 = VSMC_CUDA_FP64, Mixed = VSMC_CUDA_MIXED };

class RuntimeError : public std::runtime_error
{
  public:
    RuntimeError(int status, const std::string &what)
        : std::runtime_error(what), status_(status)
    {
    }
    int status() const { return status_; }

  private:
    int status_;
};

inline void check(int status, const char *where)
{
    if (status != VSMC_CUDA_OK)
        throw RuntimeError(status, std::string(where) + ": " +
                                       vsmc_cuda_status_string(status) +
                                       " (" + vsmc_cuda_last_error() + ")");
}

// vsmc::Seed: set(s), then get() returns s+1, s+2, ... (skipping 0 after
// the maximum), shared by every object seeded from it.
class Seed
{
  public:
    static Seed &instance()
    {
        static Seed s;
        return s;
    }
    void set(std::uint64_t s) { seed_ = static_cast<std::uint32_t>(s % max_); }
    std::uint32_t get()
    {
        seed_ = seed_ == max_ ? 1u : seed_ + 1u;
        return seed_;
    }
    std::uint32_t seed() const { return seed_; }

  private:
    Seed() : seed_(0) {}
    static const std::uint32_t max_ = 0xFFFFFFFFu;
    std::uint32_t seed_;
};

// Owning device array (cudaMalloc through the C ABI), move-only.
template <typename T>
class DeviceVector
{
  public:
    DeviceVector() : ptr_(nullptr), size_(0) {}
    explicit DeviceVector(std::size_t n) : ptr_(nullptr), size_(n)
    {
        void *p = nullptr;
        check(vsmc_cuda_device_alloc(n * sizeof(T), &p), "DeviceVector");
        ptr_ = static_cast<T *>(p);
    }
    DeviceVector(const DeviceVector &) = delete;
    DeviceVector &operator=(const DeviceVector &) = delete;
    DeviceVector(DeviceVector &&o) noexcept : ptr_(o.ptr_), size_(o.size_)
    {
        o.ptr_ = nullptr;
        o.size_ = 0;
    }
    DeviceVector &operator=(DeviceVector &&o) noexcept
    {
        std::swap(ptr_, o.ptr_);
        std::swap(size_, o.size_);
        return *this;
    }
    ~DeviceVector() { vsmc_cuda_device_free(ptr_); }

    std::size_t size() const { return size_; }
    T *data() { return ptr_; }
    const T *data() const { return ptr_; }

    void upload(const T *host, std::size_t n, void *stream = nullptr)
    {
        check(vsmc_cuda_memcpy(ptr_, host, n * sizeof(T),
                               VSMC_CUDA_HOST_TO_DEVICE, stream),
              "DeviceVector::upload");
    }
    void download(T *host, std::size_t n, void *stream = nullptr) const
    {
        check(vsmc_cuda_memcpy(host, ptr_, n * sizeof(T),
                               VSMC_CUDA_DEVICE_TO_HOST, stream),
              "DeviceVector::download");
    }

  private:
    T *ptr_;
    std::size_t size_;
};

// Position of a host Threefry4x64 engine in the ABI's terms.  The engine
// must have been seeded (key set, counter 0) and only drawn from.
inline vsmc_cuda_threefry_state threefry_position(const Threefry4x64 &eng)
{
    vsmc_cuda_threefry_state st;
    const Threefry4x64::key_type k = eng.key();
    for (int i = 0; i < 4; ++i) {
        st.key[i] = k[i];
        st.ctr[i] = 0;
    }
    st.offset = eng.words_used();
    return st;
}

// Resample<Scheme>: vSMC's resample_type call (particle.hpp:61-62;
// resample/*.hpp) on host arrays, computed on the device.  The engine
// advances by exactly the words the reference would draw.  M == N.
template <ResampleScheme Scheme>
class Resample
{
  public:
    template <typename IntType>
    void operator()(std::size_t M, std::size_t N, Threefry4x64 &rng,
                    const double *weight, IntType *replication) const
    {
        if (M != N)
            throw RuntimeError(VSMC_CUDA_EINVAL,
                               "Resample: only M == N is supported");
        DeviceVector<double> w(N);
        DeviceVector<std::int32_t> rep(N);
        DeviceVector<unsigned char> ws(vsmc_cuda_resample_workspace_size(N));
        w.upload(weight, N);
        vsmc_cuda_threefry_state st = threefry_position(rng);
        const std::uint64_t before = st.offset;
        check(vsmc_cuda_resample(Scheme, N, w.data(), nullptr, 0, &st,
                                 rep.data(), nullptr, ws.data(), ws.size(),
                                 nullptr),
              "vsmc_cuda_resample");
        std::vector<std::int32_t> r(N);
        rep.download(r.data(), N);
        for (std::size_t i = 0; i != N; ++i)
            replication[i] = static_cast<IntType>(r[i]);
        rng.discard(st.offset - before);
    }
};

// vsmc::WeightSet with the weights resident on the device
// (core/weight_set.hpp).  Log-weights are stored max-normalised, weights
// normalised, and ess() is the ESS of the last update.
class WeightSetCUDA
{
  public:
    typedef std::size_t size_type;

    explicit WeightSetCUDA(size_type N, void *stream = nullptr)
        : size_(N), stream_(stream), lw_(N), w_(N), buf_(N), ess_(0)
    {
        set_equal_weight();
    }

    size_type size() const { return size_; }
    size_type resample_size() const { return size_; }
    double ess() const { return ess_; }

    void set_equal_weight()
    {
        std::vector<double> v(size_, 0.0);
        lw_.upload(v.data(), size_, stream_);
        v.assign(size_, 1.0 / static_cast<double>(size_));
        w_.upload(v.data(), size_, stream_);
        ess_ = static_cast<double>(size_);
    }

    template <typename InputIter>
    void set_log_weight(InputIter first)
    {
        std::vector<double> v(first, first + static_cast<long>(size_));
        lw_.upload(v.data(), size_, stream_);
        update(nullptr);
    }

    template <typename InputIter>
    void add_log_weight(InputIter first)
    {
        std::vector<double> v(first, first + static_cast<long>(size_));
        buf_.upload(v.data(), size_, stream_);
        update(buf_.data());
    }

    // device arrays of size() values
    void set_log_weight_device(const double *lw)
    {
        check(vsmc_cuda_memcpy(lw_.data(), lw, size_ * sizeof(double),
                               VSMC_CUDA_DEVICE_TO_DEVICE, stream_),
              "WeightSetCUDA::set_log_weight_device");
        update(nullptr);
    }
    void add_log_weight_device(const double *inc) { update(inc); }

    template <typename OutputIter>
    void read_weight(OutputIter first) const
    {
        read(w_, first);
    }
    template <typename OutputIter>
    void read_log_weight(OutputIter first) const
    {
        read(lw_, first);
    }

    // device data
    const double *resample_weight_data() const { return w_.data(); }
    const double *weight_data() const { return w_.data(); }
    double *mutable_log_weight_data() { return lw_.data(); }
    void *stream() const { return stream_; }

  private:
    size_type size_;
    void *stream_;
    DeviceVector<double> lw_, w_, buf_;
    double ess_;

    void update(const double *inc)
    {
        check(vsmc_cuda_weight_add_log(size_, lw_.data(), w_.data(), inc,
                                       &ess_, stream_),
              "vsmc_cuda_weight_add_log");
    }

    template <typename OutputIter>
    void read(const DeviceVector<double> &d, OutputIter first) const
    {
        std::vector<double> v(size_);
        d.download(v.data(), size_, stream_);
        for (size_type i = 0; i != size_; ++i)
            *first++ = v[i];
    }
};

// StateMatrix<ColMajor, Dim, double> on the device: column d is a device
// array of size() values.  copy() is StateMatrix::copy
// (core/state_matrix.hpp:378-394) as a device gather.
template <std::size_t Dim>
class StateCUDA
{
  public:
    typedef std::size_t size_type;

    explicit StateCUDA(size_type N, void *stream = nullptr)
        : size_(N), stream_(stream), data_(Dim * N), tmp_(Dim * N), cf_(N)
    {
    }

    size_type size() const { return size_; }
    static constexpr std::size_t dim() { return Dim; }
    double *data(std::size_t d) { return data_.data() + d * size_; }
    const double *data(std::size_t d) const
    {
        return data_.data() + d * size_;
    }

    template <typename IntType>
    void copy(size_type N, const IntType *copy_from)
    {
        if (N != size_)
            throw RuntimeError(VSMC_CUDA_EINVAL, "StateCUDA::copy: N");
        std::vector<std::int32_t> c(copy_from, copy_from + N);
        cf_.upload(c.data(), N, stream_);
        copy_device(cf_.data());
    }

    // copy_from: N int32 on the device
    void copy_device(const std::int32_t *copy_from)
    {
        check(vsmc_cuda_copy_f64(size_, Dim, data_.data(), tmp_.data(),
                                 copy_from, stream_),
              "vsmc_cuda_copy_f64");
        std::swap(data_, tmp_);
    }

    template <typename OutputIter>
    void read_state(std::size_t d, OutputIter first) const
    {
        std::vector<double> v(size_);
        check(vsmc_cuda_memcpy(v.data(), data(d), size_ * sizeof(double),
                               VSMC_CUDA_DEVICE_TO_HOST, stream_),
              "StateCUDA::read_state");
        for (size_type i = 0; i != size_; ++i)
            *first++ = v[i];
    }

    template <typename InputIter>
    void write_state(std::size_t d, InputIter first)
    {
        std::vector<double> v(first, first + static_cast<long>(size_));
        check(vsmc_cuda_memcpy(data(d), v.data(), size_ * sizeof(double),
                               VSMC_CUDA_HOST_TO_DEVICE, stream_),
              "StateCUDA::write_state");
    }

  private:
    size_type size_;
    void *stream_;
    DeviceVector<double> data_, tmp_;
    DeviceVector<std::int32_t> cf_;
};

// vsmc::Particle<T> for a StateCUDA value: value, weight set, the key of
// the per-particle RNG streams and the resample engine (seeded from Seed in
// that order, particle.hpp:64-70, 254-258), and
// resample() as Particle::resample (particle.hpp:230-250), all on the
// device.
template <std::size_t Dim>
class ParticleCUDA
{
  public:
    typedef std::size_t size_type;

    explicit ParticleCUDA(size_type N, void *stream = nullptr)
        : size_(N), value_(N, stream), weight_set_(N, stream),
          rng_set_key_(Seed::instance().get()),
          resample_rng_(Seed::instance().get()), rep_(N), cf_(N),
          ws_(vsmc_cuda_resample_workspace_size(N)), stream_(stream)
    {
    }

    size_type size() const { return size_; }
    StateCUDA<Dim> &value() { return value_; }
    const StateCUDA<Dim> &value() const { return value_; }
    WeightSetCUDA &weight_set() { return weight_set_; }
    const WeightSetCUDA &weight_set() const { return weight_set_; }
    Threefry4x64 &resample_rng() { return resample_rng_; }
    // key word 0 of the per-particle Philox4x32 streams (vsmc::RngSet,
    // rng/rng_set.hpp:69-135), for device moves
    std::uint32_t rng_set_key() const { return rng_set_key_; }

    bool resample(ResampleScheme scheme, double threshold)
    {
        const bool resampled =
            weight_set_.ess() < threshold * static_cast<double>(size_);
        if (resampled) {
            vsmc_cuda_threefry_state st = threefry_position(resample_rng_);
            const std::uint64_t before = st.offset;
            check(vsmc_cuda_resample(scheme, size_,
                                     weight_set_.resample_weight_data(),
                                     nullptr, 0, &st, rep_.data(), cf_.data(),
                                     ws_.data(), ws_.size(), stream_),
                  "vsmc_cuda_resample");
            resample_rng_.discard(st.offset - before);
            value_.copy_device(cf_.data());
            weight_set_.set_equal_weight();
        }
        return resampled;
    }

    // the last copy_from (host), valid after a resampling
    std::vector<std::int32_t> copy_from() const
    {
        std::vector<std::int32_t> c(size_);
        cf_.download(c.data(), size_, stream_);
        return c;
    }

  private:
    size_type size_;
    StateCUDA<Dim> value_;
    WeightSetCUDA weight_set_;
    std::uint32_t rng_set_key_;
    Threefry4x64 resample_rng_;
    DeviceVector<std::int32_t> rep_, cf_;
    DeviceVector<unsigned char> ws_;
    void *stream_;
};

// The constant-velocity Student-t filter of example/pf as a Sampler
// (core/sampler.hpp): Sampler<cv_state>(N, scheme, threshold) with cv_init,
// cv_move and the "pos" monitor, fused on the device.  Seeded from Seed
// like the reference (the model's RngSet takes the first get(), the
// resample engine the second).
class CVSampler
{
  public:
    typedef std::size_t size_type;

    CVSampler(size_type N, ResampleScheme scheme = Multinomial,
              double threshold = 0.5, size_type T_max = 1024,
              Form form = FP64, void *stream = nullptr)
        : f_(nullptr), N_(N), iter_(0), cached_(false)
    {
        vsmc_cuda_cv_config cfg;
        vsmc_cuda_cv_config_default(&cfg);
        cfg.N = N;
        cfg.T_max = T_max;
        cfg.scheme = scheme;
        cfg.form = form;
        cfg.threshold = threshold;
        // the library applies Seed::get() twice from the set seed
        Seed &s = Seed::instance();
        cfg.seed = s.seed();
        s.get();
        s.get();
        check(vsmc_cuda_cv_create(&cfg, stream, &f_), "vsmc_cuda_cv_create");
        names_[0] = "pos.0";
        names_[1] = "pos.1";
    }
    CVSampler(const CVSampler &) = delete;
    CVSampler &operator=(const CVSampler &) = delete;
    ~CVSampler() { vsmc_cuda_cv_destroy(f_); }

    size_type size() const { return N_; }
    std::size_t iter_size() const { return iter_; }

    // Sampler::initialize(param) with the observations as the parameter
    // (cv_init::initialize_param reads the data file, pf_smp.hpp:176-177).
    CVSampler &initialize(const double *obs_x, const double *obs_y,
                          std::size_t T)
    {
        check(vsmc_cuda_cv_set_observations(f_, obs_x, obs_y, T, 0),
              "vsmc_cuda_cv_set_observations");
        check(vsmc_cuda_cv_synchronize(f_), "vsmc_cuda_cv_synchronize");
        check(vsmc_cuda_cv_initialize(f_), "vsmc_cuda_cv_initialize");
        iter_ = 1;
        cached_ = false;
        return *this;
    }

    CVSampler &iterate(std::size_t num = 1)
    {
        check(vsmc_cuda_cv_iterate(f_, num), "vsmc_cuda_cv_iterate");
        iter_ += num;
        cached_ = false;
        return *this;
    }

    double ess_history(std::size_t iter) const { return hist().ess[iter]; }
    bool resampled_history(std::size_t iter) const
    {
        return hist().resampled[iter] != 0;
    }
    std::size_t size_history(std::size_t) const { return N_; }
    // cv_init / cv_move count every particle as accepted
    std::size_t accept_history(std::size_t, std::size_t) const { return N_; }
    template <typename OutputIter>
    void read_ess_history(OutputIter first) const
    {
        for (double v : hist().ess)
            *first++ = v;
    }
    template <typename OutputIter>
    void read_resampled_history(OutputIter first) const
    {
        for (std::int32_t v : hist().resampled)
            *first++ = v != 0;
    }

    // Monitor "pos": record(d, iter) is the importance-sampling estimate of
    // the position (x for d = 0, y for d = 1) after step iter.
    double monitor_record(std::size_t d, std::size_t iter) const
    {
        return d == 0 ? hist().mean_x[iter] : hist().mean_y[iter];
    }
    std::string &monitor_name(std::size_t d) { return names_[d]; }

    // the running log-evidence and its per-step increments
    double log_evidence() const
    {
        double z = 0;
        check(vsmc_cuda_cv_log_evidence(f_, &z), "vsmc_cuda_cv_log_evidence");
        return z;
    }
    double log_evidence_increment(std::size_t iter) const
    {
        return hist().logz_inc[iter];
    }

    // Sampler::print (core/sampler.hpp:684-721): the same table.
    template <typename CharT, typename Traits>
    std::basic_ostream<CharT, Traits> &print(
        std::basic_ostream<CharT, Traits> &os, char sepchar = '\t') const
    {
        if (iter_ == 0 || !os.good())
            return os;
        const History &h = hist();
        os << "Size" << sepchar << "Resampled" << sepchar << "Accept.0"
           << sepchar << "ESS" << sepchar << names_[0] << sepchar
           << names_[1] << sepchar << '\n';
        for (std::size_t t = 0; t != iter_; ++t) {
            os << N_ << sepchar << (h.resampled[t] != 0 ? 1 : 0) << sepchar
               << N_ << sepchar << h.ess[t] << sepchar << h.mean_x[t]
               << sepchar << h.mean_y[t] << sepchar << '\n';
        }
        return os;
    }

    vsmc_cuda_cv_filter *handle() { return f_; }

  private:
    struct History {
        std::vector<double> ess, logz_inc, mean_x, mean_y;
        std::vector<std::int32_t> resampled;
    };

    vsmc_cuda_cv_filter *f_;
    size_type N_;
    std::size_t iter_;
    std::string names_[2];
    mutable bool cached_;
    mutable History h_;

    const History &hist() const
    {
        if (!cached_) {
            h_.ess.resize(iter_);
            h_.logz_inc.resize(iter_);
            h_.mean_x.resize(iter_);
            h_.mean_y.resize(iter_);
            h_.resampled.resize(iter_);
            if (iter_ > 0)
                check(vsmc_cuda_cv_history(f_, h_.ess.data(),
                                           h_.resampled.data(),
                                           h_.logz_inc.data(),
                                           h_.mean_x.data(), h_.mean_y.data()),
                      "vsmc_cuda_cv_history");
            cached_ = true;
        }
        return h_;
    }
};

template <typename CharT, typename Traits>
inline std::basic_ostream<CharT, Traits> &operator<<(
    std::basic_ostream<CharT, Traits> &os, const CVSampler &s)
{
    return s.print(os);
}

// The tempered SMC sampler of example/gmm (gmm_smc.cpp with alpha_prior,
// move_smc, the three MH block moves and path sampling), on the device.
// Seeded like the reference from Seed: the N particle engines take the
// next N Seed::get() values and the resample engine the one after.
class GmmSampler
{
  public:
    typedef std::size_t size_type;

    GmmSampler(const double *data, std::size_t n, size_type N,
               std::size_t iters = 100, int power = 4, int sweeps = 5,
               double sd = 0.1, ResampleScheme scheme = Systematic,
               double threshold = 0.5, Form form = FP64,
               void *stream = nullptr)
        : g_(nullptr), N_(N), sweeps_(sweeps), iter_(0), cached_(false)
    {
        vsmc_cuda_gmm_config cfg;
        vsmc_cuda_gmm_config_default(&cfg);
        cfg.N = N;
        cfg.iters = iters;
        cfg.power = power;
        cfg.sweeps = sweeps;
        cfg.sd = sd;
        cfg.scheme = scheme;
        cfg.threshold = threshold;
        cfg.form = form;
        Seed &s = Seed::instance();
        cfg.seed = s.seed();
        for (size_type i = 0; i != N + 1; ++i)
            s.get();
        check(vsmc_cuda_gmm_create(&cfg, data, n, stream, &g_),
              "vsmc_cuda_gmm_create");
    }
    GmmSampler(const GmmSampler &) = delete;
    GmmSampler &operator=(const GmmSampler &) = delete;
    ~GmmSampler() { vsmc_cuda_gmm_destroy(g_); }

    size_type size() const { return N_; }
    std::size_t iter_size() const { return iter_; }

    GmmSampler &initialize()
    {
        check(vsmc_cuda_gmm_initialize(g_), "vsmc_cuda_gmm_initialize");
        iter_ = 1;
        cached_ = false;
        return *this;
    }

    GmmSampler &iterate(std::size_t num = 1)
    {
        check(vsmc_cuda_gmm_iterate(g_, num), "vsmc_cuda_gmm_iterate");
        iter_ += num;
        cached_ = false;
        return *this;
    }

    double ess_history(std::size_t iter) const { return hist().ess[iter]; }
    bool resampled_history(std::size_t iter) const
    {
        return hist().resampled[iter] != 0;
    }
    // Sampler::accept_history(id, iter): id 0 is move_smc, then the MH
    // moves in queue order
    std::size_t accept_history(std::size_t id, std::size_t iter) const
    {
        return static_cast<std::size_t>(
            hist().accept[iter * (1 + 3 * sweeps_) + id]);
    }

    // zconst + log_likelihood_const (example/include/smc_do.hpp)
    double log_evidence() const
    {
        double smc = 0, path = 0;
        check(vsmc_cuda_gmm_log_evidence(g_, &smc, &path),
              "vsmc_cuda_gmm_log_evidence");
        return smc;
    }
    double path_log_evidence() const
    {
        double smc = 0, path = 0;
        check(vsmc_cuda_gmm_log_evidence(g_, &smc, &path),
              "vsmc_cuda_gmm_log_evidence");
        return path;
    }

    // Sampler::print: Size, Resampled, Accept.k, ESS, Path.Integrand,
    // Path.Grid (core/sampler.hpp:566-721).
    template <typename CharT, typename Traits>
    std::basic_ostream<CharT, Traits> &print(
        std::basic_ostream<CharT, Traits> &os, char sepchar = '\t') const
    {
        if (iter_ == 0 || !os.good())
            return os;
        const History &h = hist();
        const std::size_t nacc = 1 + 3 * static_cast<std::size_t>(sweeps_);
        os << "Size" << sepchar << "Resampled" << sepchar;
        for (std::size_t k = 0; k != nacc; ++k)
            os << "Accept." << k << sepchar;
        os << "ESS" << sepchar << "Path.Integrand" << sepchar << "Path.Grid"
           << sepchar << '\n';
        for (std::size_t t = 0; t != iter_; ++t) {
            os << N_ << sepchar << (h.resampled[t] != 0 ? 1 : 0) << sepchar;
            for (std::size_t k = 0; k != nacc; ++k)
                os << h.accept[t * nacc + k] << sepchar;
            os << h.ess[t] << sepchar << h.integrand[t] << sepchar
               << h.grid[t] << sepchar << '\n';
        }
        return os;
    }

    vsmc_cuda_gmm *handle() { return g_; }

  private:
    struct History {
        std::vector<double> ess, zinc, integrand, grid;
        std::vector<std::int32_t> resampled;
        std::vector<std::int64_t> accept;
    };

    vsmc_cuda_gmm *g_;
    size_type N_;
    int sweeps_;
    std::size_t iter_;
    mutable bool cached_;
    mutable History h_;

    const History &hist() const
    {
        if (!cached_) {
            const std::size_t T = iter_;
            h_.ess.resize(T);
            h_.zinc.resize(T);
            h_.integrand.resize(T);
            h_.grid.resize(T);
            h_.resampled.resize(T);
            h_.accept.resize(T * (1 + 3 * static_cast<std::size_t>(sweeps_)));
            if (T > 0)
                check(vsmc_cuda_gmm_history(g_, h_.ess.data(),
                                            h_.resampled.data(),
                                            h_.zinc.data(),
                                            h_.integrand.data(),
                                            h_.grid.data(), h_.accept.data()),
                      "vsmc_cuda_gmm_history");
            cached_ = true;
        }
        return h_;
    }
};

template <typename CharT, typename Traits>
inline std::basic_ostream<CharT, Traits> &operator<<(
    std::basic_ostream<CharT, Traits> &os, const GmmSampler &s)
{
    return s.print(os);
}

// Many CV filters on one device (vsmc_cuda_cv_batch), RAII.
class CVBatch
{
  public:
    CVBatch(std::uint32_t capacity, ResampleScheme scheme = Multinomial,
            Form form = FP64, double threshold = 0.5,
            std::uint64_t hbm_budget = 0, void *stream = nullptr)
        : b_(nullptr)
    {
        vsmc_cuda_cv_config m;
        vsmc_cuda_cv_config_default(&m);
        m.scheme = scheme;
        m.form = form;
        m.threshold = threshold;
        check(vsmc_cuda_cv_batch_create(&m, capacity, hbm_budget, stream, &b_),
              "vsmc_cuda_cv_batch_create");
    }
    CVBatch(const CVBatch &) = delete;
    CVBatch &operator=(const CVBatch &) = delete;
    ~CVBatch() { vsmc_cuda_cv_batch_destroy(b_); }

    std::uint32_t admit(std::uint64_t N, std::uint64_t T_max,
                        std::uint32_t seed, std::uint32_t stream_id)
    {
        std::uint32_t s = 0;
        check(vsmc_cuda_cv_batch_admit(b_, N, T_max, seed, stream_id, &s),
              "vsmc_cuda_cv_batch_admit");
        return s;
    }
    void release(std::uint32_t slot)
    {
        check(vsmc_cuda_cv_batch_release(b_, slot),
              "vsmc_cuda_cv_batch_release");
    }
    void set_observations(const std::vector<std::uint32_t> &slots,
                          const std::vector<std::uint64_t> &T,
                          const double *ox, const double *oy)
    {
        check(vsmc_cuda_cv_batch_set_observations(
                  b_, static_cast<std::uint32_t>(slots.size()), slots.data(),
                  T.data(), ox, oy, 0),
              "vsmc_cuda_cv_batch_set_observations");
    }
    void step(const std::vector<std::uint32_t> &slots)
    {
        check(vsmc_cuda_cv_batch_step(
                  b_, static_cast<std::uint32_t>(slots.size()), slots.data()),
              "vsmc_cuda_cv_batch_step");
    }
    void run(const std::vector<std::uint32_t> &slots)
    {
        check(vsmc_cuda_cv_batch_run(
                  b_, static_cast<std::uint32_t>(slots.size()), slots.data()),
              "vsmc_cuda_cv_batch_run");
    }
    std::vector<double> log_evidence(const std::vector<std::uint32_t> &slots)
    {
        std::vector<double> z(slots.size());
        check(vsmc_cuda_cv_batch_read_last(
                  b_, static_cast<std::uint32_t>(slots.size()), slots.data(),
                  nullptr, nullptr, nullptr, z.data(), nullptr),
              "vsmc_cuda_cv_batch_read_last");
        return z;
    }
    // Appends one observation to each listed slot.
    void append(const std::vector<std::uint32_t> &slots,
                const std::vector<double> &x, const std::vector<double> &y)
    {
        check(vsmc_cuda_cv_batch_append_observations(
                  b_, static_cast<std::uint32_t>(slots.size()), slots.data(),
                  x.data(), y.data()),
              "vsmc_cuda_cv_batch_append_observations");
    }
    // The last counts[k] steps of each slot, packed in list order.
    struct Steps {
        std::vector<double> ess, logz_inc;
        std::vector<std::int32_t> resampled, status;
    };
    Steps read_steps(const std::vector<std::uint32_t> &slots,
                     const std::vector<std::uint32_t> &counts)
    {
        std::size_t total = 0;
        for (std::uint32_t c : counts)
            total += c;
        Steps r;
        r.ess.resize(total);
        r.logz_inc.resize(total);
        r.resampled.resize(total);
        r.status.resize(slots.size());
        const int st = vsmc_cuda_cv_batch_read_steps(
            b_, static_cast<std::uint32_t>(slots.size()), slots.data(),
            counts.data(), r.ess.data(), r.logz_inc.data(),
            r.resampled.data(), r.status.data());
        if (st != VSMC_CUDA_EDEGENERATE) // reported per slot in r.status
            check(st, "vsmc_cuda_cv_batch_read_steps");
        return r;
    }
    // Times the launch shapes on a trial copy of (a sample of) the slots and
    // keeps the fastest; no result changes.
    void autotune(const std::vector<std::uint32_t> &slots)
    {
        check(vsmc_cuda_cv_batch_autotune(
                  b_, static_cast<std::uint32_t>(slots.size()), slots.data(),
                  nullptr, nullptr),
              "vsmc_cuda_cv_batch_autotune");
    }
    vsmc_cuda_cv_batch *handle() { return b_; }

  private:
    vsmc_cuda_cv_batch *b_;
};

// The serving loop (vsmc_cuda_cv_server), RAII.
class CVServer
{
  public:
    CVServer(std::uint32_t max_filters, std::uint64_t hbm_budget,
             ResampleScheme scheme = Multinomial, Form form = FP64,
             double threshold = 0.5)
        : s_(nullptr)
    {
        vsmc_cuda_cv_config m;
        vsmc_cuda_cv_config_default(&m);
        m.scheme = scheme;
        m.form = form;
        m.threshold = threshold;
        check(vsmc_cuda_cv_server_create(&m, max_filters, hbm_budget, &s_),
              "vsmc_cuda_cv_server_create");
    }
    CVServer(const CVServer &) = delete;
    CVServer &operator=(const CVServer &) = delete;
    ~CVServer() { vsmc_cuda_cv_server_destroy(s_); }

    std::uint64_t open(std::uint64_t N, std::uint64_t T_max,
                       std::uint32_t seed, std::uint32_t stream_id)
    {
        std::uint64_t r = 0;
        check(vsmc_cuda_cv_server_open(s_, N, T_max, seed, stream_id, &r),
              "vsmc_cuda_cv_server_open");
        return r;
    }
    void observe(std::uint64_t request, double x, double y)
    {
        check(vsmc_cuda_cv_server_observe(s_, 1, &request, &x, &y, nullptr),
              "vsmc_cuda_cv_server_observe");
    }
    void close(std::uint64_t request)
    {
        check(vsmc_cuda_cv_server_close(s_, request),
              "vsmc_cuda_cv_server_close");
    }
    std::vector<vsmc_cuda_cv_result> poll(std::uint32_t max = 4096,
                                          int wait_ms = 0)
    {
        std::vector<vsmc_cuda_cv_result> r(max);
        std::uint32_t n = 0;
        check(vsmc_cuda_cv_server_poll(s_, r.data(), max, &n, wait_ms),
              "vsmc_cuda_cv_server_poll");
        r.resize(n);
        return r;
    }
    void drain(int timeout_ms = 60000)
    {
        check(vsmc_cuda_cv_server_drain(s_, timeout_ms),
              "vsmc_cuda_cv_server_drain");
    }

  private:
    vsmc_cuda_cv_server *s_;
};

} // namespace vsmc_b200

#endif // VSMC_B200_VSMC_CUDA_HPP
