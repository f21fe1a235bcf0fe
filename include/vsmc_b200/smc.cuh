// smc.cuh -- vSMC's Sampler<T> with the particle code compiled for B200.
//
// For programs compiled with nvcc (-gencode arch=compute_100a,code=sm_100a)
// and linked against libvsmc_cuda.  The user writes the reference's
// per-particle functions -- initialize_state(SingleParticle<T>),
// move_state(iter, SingleParticle<T>), monitor_state(iter, dim,
// ConstSingleParticle<T>, double *) -- as __device__ member functions of
// InitializeCUDA / MoveCUDA / MonitorEvalCUDA functors (CRTP, like
// InitializeOMP / MoveOMP / MonitorEvalOMP, include/vsmc/smp/
// backend_base.hpp:77-532 and backend_omp.hpp:99-149).  Sampler<T> launches
// one fused kernel per functor and step: every particle is gathered from its
// parent of the last resampling, moved by the user's code, and its
// log-weight updated, while each tile's log-sum-exp statistics are reduced
// on chip; the library (vsmc_cuda_smc_*) then normalises, computes ESS and
// the log-evidence increment, decides and resamples, all on the device.
//
// Names follow the reference (include/vsmc/core/sampler.hpp, particle.hpp,
// weight_set.hpp, resample/common.hpp) inside namespace vsmc, plus the later
// vSMC spellings as aliases (Weight::set_log / add_log / ess, MoveSMP,
// MonitorEvalSMP, ResampleMultinomial, ...).
//
// Differences a user of the reference sees:
// * per-particle code is __device__ and the functor is copied into the
//   kernel, so it carries its data as device pointers and plain values;
// * a move passes its log-weight increment with sp.add_log_weight(inc) (or
//   sp.set_log_weight(v) in initialize_state), which replaces the
//   post_processor's WeightSet::add_log_weight call of the examples;
// * accept counts are summed on the device, so the functors' operator()
//   returns 0 and Sampler::accept_history reads the device sums;
// * the history capacity (steps) is a constructor argument.
#ifndef VSMC_B200_SMC_CUH
#define VSMC_B200_SMC_CUH

#include <vsmc_cuda.h>
#include <vsmc_b200/smc_device.cuh>
#include <vsmc_b200/vsmc_cuda.hpp>

#include <cstddef>
#include <cstdint>
#include <functional>
#include <limits>
#include <map>
#include <memory>
#include <ostream>
#include <sstream>
#include <string>
#include <vector>

namespace vsmc {

// ------------------------------------------------------------ reference names
typedef vsmc_b200::ResampleScheme ResampleScheme;
using vsmc_b200::Multinomial;
using vsmc_b200::Residual;
using vsmc_b200::Stratified;
using vsmc_b200::Systematic;
using vsmc_b200::ResidualStratified;
using vsmc_b200::ResidualSystematic;
using vsmc_b200::RuntimeError;
using vsmc_b200::Seed;
using vsmc_b200::Philox4x32;
using vsmc_b200::Threefry4x64;

// ResampleType<Scheme>::type (resample/common.hpp:139-141): the host-callable
// (M, N, rng, weight, replication) functor, computed on the device.
template <ResampleScheme Scheme>
struct ResampleType {
    typedef vsmc_b200::Resample<Scheme> type;
};
typedef ResampleType<Multinomial>::type ResampleMultinomial;
typedef ResampleType<Residual>::type ResampleResidual;
typedef ResampleType<Stratified>::type ResampleStratified;
typedef ResampleType<Systematic>::type ResampleSystematic;
typedef ResampleType<ResidualStratified>::type ResampleResidualStratified;
typedef ResampleType<ResidualSystematic>::type ResampleResidualSystematic;

// RngSet kinds (rng/rng_set.hpp:69-135): Vector gives every particle slot
// its own engine seeded from Seed (the reference's default), Scalar one
// engine whose counter the per-particle code positions itself.
struct Scalar {};
struct Vector {};
template <typename RngType = Threefry4x64, typename Kind = Vector>
struct RngSet {
    typedef RngType rng_type;
    typedef Kind kind;
};

// --------------------------------------------------------- device engines
// PhiloxEngine<uint32_t,4,10> on the device (rng/philox.hpp:305-524): the
// counter is incremented before each block; ctr(c) sets the counter and
// empties the buffer, as the reference's does.
class PhiloxEngineCUDA
{
  public:
    typedef std::uint32_t result_type;

    __device__ PhiloxEngineCUDA(std::uint32_t k0, std::uint32_t k1)
        : c_(make_uint4(0u, 0u, 0u, 0u)), k0_(k0), k1_(k1), index_(4)
    {
    }

    __device__ void ctr(uint4 c)
    {
        c_ = c;
        index_ = 4;
    }
    __device__ uint4 ctr() const { return c_; }

    __device__ result_type operator()()
    {
        if (index_ == 4) {
            if (++c_.x == 0)
                if (++c_.y == 0)
                    if (++c_.z == 0)
                        ++c_.w;
            buf_ = vsmc_b200::philox4x32_10(c_, k0_, k1_);
            index_ = 0;
        }
        const int k = index_++;
        return k == 0 ? buf_.x : k == 1 ? buf_.y : k == 2 ? buf_.z : buf_.w;
    }

    static constexpr int result_bits = 32;

  private:
    uint4 c_;
    std::uint32_t k0_, k1_;
    uint4 buf_;
    int index_;
};

// ThreefryEngine<uint64_t,4,20> on the device (rng/threefry.hpp:263-507),
// positioned by the number of words drawn since its counter was zero.
class ThreefryEngineCUDA
{
  public:
    typedef std::uint64_t result_type;

    __device__ ThreefryEngineCUDA(std::uint64_t key0, std::uint64_t words)
        : words_(words)
    {
        for (int i = 0; i < 4; ++i) {
            key_.v[i] = 0;
            zero_.v[i] = 0;
        }
        key_.v[0] = key0;
        if (words_ % 4 != 0)
            buf_ = vsmc_b200::threefry4x64_20(
                vsmc_b200::ctr64_add(zero_, words_ / 4 + 1), key_);
    }

    __device__ result_type operator()()
    {
        const int k = (int)(words_ % 4);
        if (k == 0)
            buf_ = vsmc_b200::threefry4x64_20(
                vsmc_b200::ctr64_add(zero_, words_ / 4 + 1), key_);
        ++words_;
        return buf_.v[k];
    }

    __device__ std::uint64_t words() const { return words_; }

    static constexpr int result_bits = 64;

  private:
    vsmc_b200::u64x4 key_, zero_, buf_;
    std::uint64_t words_;
};

// libstdc++'s generate_canonical<double, 53> over the engine: one 64-bit
// word, or two 32-bit words (low first).
template <typename Eng>
__device__ __forceinline__ double canonical(Eng &eng)
{
    if (Eng::result_bits == 64)
        return vsmc_b200::canonical_u64(eng());
    const std::uint32_t a = static_cast<std::uint32_t>(eng());
    const std::uint32_t b = static_cast<std::uint32_t>(eng());
    return vsmc_b200::canonical_u32x2(a, b);
}

// std::normal_distribution<double> (libstdc++'s Marsaglia polar method with
// the cached second variate), the distribution of the reference's moves.
class NormalDistribution
{
  public:
    __device__ NormalDistribution(double mean = 0.0, double stddev = 1.0)
        : mean_(mean), sd_(stddev), saved_(0.0), have_(false)
    {
    }

    template <typename Eng>
    __device__ double operator()(Eng &eng)
    {
        double ret;
        if (have_) {
            have_ = false;
            ret = saved_;
        } else {
            double x, y, r2;
            do {
                x = __dadd_rn(__dmul_rn(2.0, canonical(eng)), -1.0);
                y = __dadd_rn(__dmul_rn(2.0, canonical(eng)), -1.0);
                r2 = __dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y));
            } while (r2 > 1.0 || r2 == 0.0);
            const double mult =
                __dsqrt_rn(__ddiv_rn(__dmul_rn(-2.0, log(r2)), r2));
            saved_ = __dmul_rn(x, mult);
            have_ = true;
            ret = __dmul_rn(y, mult);
        }
        return __dadd_rn(__dmul_rn(ret, sd_), mean_);
    }

  private:
    double mean_, sd_, saved_;
    bool have_;
};

namespace detail {

template <typename T, typename = void>
struct RngSetOf {
    typedef RngSet<Threefry4x64, Vector> type;
};
template <typename T>
struct RngSetOf<T, decltype(void(sizeof(typename T::rng_set_type)))> {
    typedef typename T::rng_set_type type;
};

template <typename Set>
struct DeviceEngine;
template <>
struct DeviceEngine<RngSet<Threefry4x64, Vector> > {
    typedef ThreefryEngineCUDA type;
    static const bool per_slot = true;
};
template <>
struct DeviceEngine<RngSet<Philox4x32, Scalar> > {
    typedef PhiloxEngineCUDA type;
    static const bool per_slot = false;
};

} // namespace detail

// ------------------------------------------------------------ value type
// StateMatrix<ColMajor, Dim, StateType> on the device: column d of the
// current state is data(d); two buffers, because every step's kernel
// reads one and writes the other (the gather of a resampling is fused
// into that read).
template <std::size_t Dim, typename StateType = double>
class StateCUDA
{
  public:
    typedef std::size_t size_type;
    typedef StateType state_type;
    static constexpr std::size_t dim_value = Dim;

    explicit StateCUDA(size_type N) : size_(N), cur_(0)
    {
        buf_[0] = vsmc_b200::DeviceVector<StateType>(Dim * N);
        buf_[1] = vsmc_b200::DeviceVector<StateType>(Dim * N);
    }

    size_type size() const { return size_; }
    static constexpr std::size_t dim() { return Dim; }

    // the current state (device), column-major
    StateType *data() { return buf_[cur_].data(); }
    const StateType *data() const { return buf_[cur_].data(); }
    StateType *other() { return buf_[1 - cur_].data(); }
    void flip() { cur_ = 1 - cur_; }

    template <typename OutputIter>
    void read_state(std::size_t d, OutputIter first) const
    {
        std::vector<StateType> v(size_);
        vsmc_b200::check(vsmc_cuda_memcpy(v.data(), data() + d * size_,
                                          size_ * sizeof(StateType),
                                          VSMC_CUDA_DEVICE_TO_HOST, nullptr),
                         "StateCUDA::read_state");
        for (size_type i = 0; i != size_; ++i)
            *first++ = v[i];
    }

  private:
    size_type size_;
    int cur_;
    vsmc_b200::DeviceVector<StateType> buf_[2];
};

template <typename T>
class Particle;

// ------------------------------------------------- per-particle handles
// SingleParticle<T> (core/single_particle.hpp): the particle's state in
// registers, its id, its engine, and its log-weight increment.
template <typename T>
class SingleParticle
{
  public:
    typedef typename T::state_type state_type;
    typedef typename detail::DeviceEngine<
        typename detail::RngSetOf<T>::type>::type rng_type;

    __device__ SingleParticle(std::size_t id, state_type *s, rng_type *rng,
                              double *inc, bool *set)
        : id_(id), s_(s), rng_(rng), inc_(inc), set_(set)
    {
    }

    __device__ std::size_t id() const { return id_; }
    __device__ state_type &state(std::size_t d) const { return s_[d]; }
    __device__ rng_type &rng() const { return *rng_; }
    // WeightSet::add_log_weight for this particle, on the device
    __device__ void add_log_weight(double inc) const { *inc_ += inc; }
    // WeightSet::set_log_weight for this particle (initialize_state)
    __device__ void set_log_weight(double v) const
    {
        *set_ = true;
        *inc_ = v;
    }

  private:
    std::size_t id_;
    state_type *s_;
    rng_type *rng_;
    double *inc_;
    bool *set_;
};

template <typename T>
class ConstSingleParticle
{
  public:
    typedef typename T::state_type state_type;

    __device__ ConstSingleParticle(std::size_t id, const state_type *s)
        : id_(id), s_(s)
    {
    }

    __device__ std::size_t id() const { return id_; }
    __device__ const state_type &state(std::size_t d) const { return s_[d]; }

  private:
    std::size_t id_;
    const state_type *s_;
};

// ------------------------------------------------------------ kernels
namespace detail {

enum Stage { StageInit = 0, StageMove = 1, StageMCMC = 2 };

constexpr int kStepThreads = 256;
constexpr int kStepItems = VSMC_CUDA_SMC_TILE / kStepThreads;
constexpr int kMonitorBlocks = 1184;
constexpr int kMaxMonitorDim = 16;

template <typename T>
struct StepLaunch {
    typedef typename T::state_type state_type;
    const state_type *in;
    state_type *out;
    long long N;
    std::uint64_t iter;
    double *lw;
    const double *lw_max;
    const std::int32_t *resampled;
    const std::int32_t *copy_from;
    vsmc_b200::TileStats *tile_stats;
    unsigned long long *accept;
    int gather;     // the first state read since a finished step
    int first_move; // the step's first move (normalises the log-weights)
    std::uint32_t key;            // Scalar engine key / unused
    const std::uint32_t *keys;    // Vector: per-slot engine keys
    std::uint64_t *words;         // Vector: per-slot words drawn
};

template <typename Engine>
struct EngineMaker;
template <>
struct EngineMaker<ThreefryEngineCUDA> {
    template <typename A>
    __device__ static ThreefryEngineCUDA make(const A &a, long long i)
    {
        return ThreefryEngineCUDA(a.keys[i], a.words[i]);
    }
    template <typename A>
    __device__ static void save(const A &a, long long i,
                                const ThreefryEngineCUDA &e)
    {
        a.words[i] = e.words();
    }
};
template <>
struct EngineMaker<PhiloxEngineCUDA> {
    template <typename A>
    __device__ static PhiloxEngineCUDA make(const A &a, long long)
    {
        return PhiloxEngineCUDA(a.key, 0u);
    }
    template <typename A>
    __device__ static void save(const A &, long long, const PhiloxEngineCUDA &)
    {
    }
};

// One tile of VSMC_CUDA_SMC_TILE particles per CTA: gather, the user's
// initialize_state / move_state, the log-weight update, the tile's
// log-sum-exp statistics and the accept count.
template <typename T, typename D, int S>
__global__ void __launch_bounds__(kStepThreads)
k_sampler_step(D d, StepLaunch<T> a)
{
    typedef typename T::state_type state_type;
    typedef typename SingleParticle<T>::rng_type rng_type;
    constexpr std::size_t Dim = T::dim_value;
    __shared__ double sh_w[7 * (kStepThreads / 32)];
    const long long N = a.N;
    const long long base = (long long)blockIdx.x * VSMC_CUDA_SMC_TILE;
    const int res = S == StageInit ? 0 : *a.resampled;
    const bool gather = a.gather && res;
    const double mprev = (S == StageMove && a.first_move && !res)
                             ? *a.lw_max
                             : 0.0;
    vsmc_b200::LseRef acc;
    acc.init();
    unsigned long long accept = 0;
#pragma unroll 1
    for (int j = 0; j < kStepItems; ++j) {
        const long long i = base + (long long)j * kStepThreads + threadIdx.x;
        if (i >= N)
            continue;
        long long src = i;
        if (gather) { // clamped: never leaves [0, N)
            src = a.copy_from[i];
            src = src < 0 ? 0 : (src >= N ? N - 1 : src);
        }
        state_type s[Dim];
#pragma unroll
        for (std::size_t k = 0; k < Dim; ++k)
            s[k] = a.in[(long long)k * N + src];
        rng_type eng = EngineMaker<rng_type>::make(a, i);
        double inc = 0.0;
        bool set = false;
        SingleParticle<T> sp(static_cast<std::size_t>(i), s, &eng, &inc,
                             &set);
        if constexpr (S == StageInit)
            accept += d.initialize_state(sp);
        else
            accept += d.move_state(static_cast<std::size_t>(a.iter), sp);
#pragma unroll
        for (std::size_t k = 0; k < Dim; ++k)
            a.out[(long long)k * N + i] = s[k];
        EngineMaker<rng_type>::save(a, i, eng);
        if constexpr (S != StageMCMC) {
            double lwn;
            if (S == StageInit || set) {
                lwn = inc;
            } else {
                const double prev =
                    !a.first_move ? a.lw[i]
                                  : (res ? 0.0 : __dadd_rn(a.lw[i], -mprev));
                lwn = __dadd_rn(prev, inc);
            }
            a.lw[i] = lwn;
            vsmc_b200::lse_add<double>(acc, lwn, 0.0, 0.0);
        }
    }
    if constexpr (S != StageMCMC)
        vsmc_b200::tile_stats_reduce<kStepThreads / 32>(
            acc, 0.0, 0.0, sh_w, a.tile_stats + blockIdx.x);
    // integer sums are exact in any order
    for (int o = 16; o > 0; o >>= 1)
        accept += __shfl_xor_sync(0xffffffffu, accept, o);
    if ((threadIdx.x & 31) == 0 && accept != 0)
        atomicAdd(a.accept, accept);
}

template <typename T>
struct MonitorLaunch {
    typedef typename T::state_type state_type;
    const state_type *state;
    long long N;
    std::uint64_t iter;
    int dim;
    int gather;
    const double *lw;
    const double *lw_max;
    const double *s1;
    const std::int32_t *resampled;
    const std::int32_t *copy_from;
    double *part; // kMonitorBlocks x dim
};

// Monitor::eval with ISIntegrate (core/monitor.hpp:274-302,
// integrate/is_integrate.hpp:56-80): sum_i W_i h(X_i) with the step's
// normalised weights (1/N after a resampling, whose parents are read
// through copy_from), per-block partial sums in a fixed order.
template <typename T, typename D>
__global__ void __launch_bounds__(256) k_sampler_monitor(D d, MonitorLaunch<T> a)
{
    typedef typename T::state_type state_type;
    constexpr std::size_t Dim = T::dim_value;
    __shared__ double sh[kMaxMonitorDim][8];
    const int res = *a.resampled;
    const bool gather = a.gather && res;
    const double M = *a.lw_max;
    const double coeff = __ddiv_rn(1.0, *a.s1);
    const double eq = 1.0 / (double)a.N;
    double sum[kMaxMonitorDim];
    for (int k = 0; k < kMaxMonitorDim; ++k)
        sum[k] = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
         i < a.N; i += (long long)gridDim.x * blockDim.x) {
        long long src = i;
        if (gather) {
            src = a.copy_from[i];
            src = src < 0 ? 0 : (src >= a.N ? a.N - 1 : src);
        }
        state_type s[Dim];
#pragma unroll
        for (std::size_t k = 0; k < Dim; ++k)
            s[k] = a.state[(long long)k * a.N + src];
        double r[kMaxMonitorDim];
        d.monitor_state(static_cast<std::size_t>(a.iter),
                        static_cast<std::size_t>(a.dim),
                        ConstSingleParticle<T>(static_cast<std::size_t>(i), s),
                        r);
        const double w =
            res ? eq : __dmul_rn(exp(__dadd_rn(a.lw[i], -M)), coeff);
        for (int k = 0; k < a.dim; ++k)
            sum[k] = __dadd_rn(sum[k], __dmul_rn(w, r[k]));
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int k = 0; k < a.dim; ++k) {
        double v = sum[k];
        for (int o = 16; o > 0; o >>= 1)
            v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0)
            sh[k][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < a.dim) {
        double t = 0.0;
        for (int w = 0; w < 8; ++w)
            t += sh[threadIdx.x][w];
        a.part[blockIdx.x * a.dim + threadIdx.x] = t;
    }
}

static __global__ void k_sampler_monitor_finish(const double *part,
                                                int nparts, int dim,
                                                double *record)
{
    if (threadIdx.x >= (unsigned)dim)
        return;
    double t = 0.0;
    for (int b = 0; b < nparts; ++b)
        t += part[b * dim + threadIdx.x];
    record[threadIdx.x] = t;
}

// The move of a step whose move queue is empty: weights unchanged.
template <typename T>
struct IdentityMove {
    __device__ std::size_t move_state(std::size_t, SingleParticle<T>) const
    {
        return 0;
    }
};

// Seeds of an RngSet<Threefry4x64, Vector> (one Seed::get() per slot) and
// zero words drawn.
inline void seed_vector_engines(std::size_t N,
                                vsmc_b200::DeviceVector<std::uint32_t> &keys,
                                vsmc_b200::DeviceVector<std::uint64_t> &words)
{
    std::vector<std::uint32_t> k(N);
    for (std::size_t i = 0; i != N; ++i)
        k[i] = Seed::instance().get();
    keys.upload(k.data(), N);
    std::vector<std::uint64_t> z(N, 0);
    words.upload(z.data(), N);
}

} // namespace detail

// ------------------------------------------------------------ Particle<T>
// Particle<T> (core/particle.hpp): the value, the weight set, the RngSet and
// the resample engine, seeded from Seed in the reference's member order
// (value, weight_set, rng_set, resample_rng; particle.hpp:64-70, 254-258).
template <typename T>
class Particle
{
  public:
    typedef std::size_t size_type;
    typedef T value_type;
    typedef typename detail::RngSetOf<T>::type rng_set_type;
    typedef detail::DeviceEngine<rng_set_type> engine_traits;

    Particle(size_type N, ResampleScheme scheme, double threshold,
             size_type T_max, void *stream)
        : size_(N), value_(N), key_(0), core_(nullptr), stream_(stream)
    {
        if (engine_traits::per_slot) {
            keys_ = vsmc_b200::DeviceVector<std::uint32_t>(N);
            words_ = vsmc_b200::DeviceVector<std::uint64_t>(N);
            detail::seed_vector_engines(N, keys_, words_);
        } else {
            key_ = Seed::instance().get();
        }
        resample_seed_ = Seed::instance().get();
        vsmc_b200::check(vsmc_cuda_smc_create(N, T_max, scheme, threshold,
                                              resample_seed_, stream, &core_),
                         "vsmc_cuda_smc_create");
    }
    Particle(const Particle &) = delete;
    Particle &operator=(const Particle &) = delete;
    ~Particle() { vsmc_cuda_smc_destroy(core_); }

    size_type size() const { return size_; }
    T &value() { return value_; }
    const T &value() const { return value_; }
    void *stream() const { return stream_; }
    vsmc_cuda_smc *core() { return core_; }
    // key of a Scalar RngSet's engine (its counter is set per particle)
    std::uint32_t rng_key() const { return key_; }
    std::uint32_t resample_seed() const { return resample_seed_; }

    // WeightSet::read_weight / read_log_weight (host iterators)
    template <typename OutputIter>
    void read_weight(OutputIter first) const
    {
        std::vector<double> w(size_);
        vsmc_b200::check(vsmc_cuda_smc_read_weights(core_, w.data(), nullptr),
                         "vsmc_cuda_smc_read_weights");
        for (double v : w)
            *first++ = v;
    }
    template <typename OutputIter>
    void read_log_weight(OutputIter first) const
    {
        std::vector<double> w(size_);
        vsmc_b200::check(vsmc_cuda_smc_read_weights(core_, nullptr, w.data()),
                         "vsmc_cuda_smc_read_weights");
        for (double v : w)
            *first++ = v;
    }
    // the running log-evidence (sum of the increments of move_smc.hpp)
    double log_evidence() const
    {
        double z = 0;
        vsmc_b200::check(vsmc_cuda_smc_log_evidence(core_, &z),
                         "vsmc_cuda_smc_log_evidence");
        return z;
    }

    // ---- driven by Sampler<T> ---------------------------------------
    // Launches the fused kernel of one functor at the current stage.
    template <typename D, int S>
    void launch(const D &d)
    {
        vsmc_cuda_smc_step st;
        vsmc_b200::check(vsmc_cuda_smc_step_args(core_, &st),
                         "vsmc_cuda_smc_step_args");
        detail::StepLaunch<T> a;
        a.in = value_.data();
        a.out = value_.other();
        a.N = static_cast<long long>(size_);
        a.iter = st.iter;
        a.lw = st.log_weight;
        a.lw_max = st.lw_max;
        a.resampled = st.resampled;
        a.copy_from = st.copy_from;
        a.tile_stats = static_cast<vsmc_b200::TileStats *>(st.tile_stats);
        a.accept = reinterpret_cast<unsigned long long *>(
            st.accept + st.iter * VSMC_CUDA_SMC_MAX_QUEUE + queue_pos_);
        a.gather = gather_pending_ ? 1 : 0;
        a.first_move = first_move_ ? 1 : 0;
        a.key = key_;
        a.keys = engine_traits::per_slot ? keys_.data() : nullptr;
        a.words = engine_traits::per_slot ? words_.data() : nullptr;
        detail::k_sampler_step<T, D, S>
            <<<static_cast<unsigned>(st.ntiles), detail::kStepThreads, 0,
               static_cast<cudaStream_t>(st.stream)>>>(d, a);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess)
            throw RuntimeError(VSMC_CUDA_ECUDA,
                               std::string("Sampler step kernel: ") +
                                   cudaGetErrorString(e));
        value_.flip();
        gather_pending_ = false;
        if (S == detail::StageMove)
            first_move_ = false;
    }

    template <typename D>
    void launch_monitor(const D &d, std::size_t dim, double *part,
                        double *record)
    {
        vsmc_cuda_smc_step st;
        vsmc_b200::check(vsmc_cuda_smc_step_args(core_, &st),
                         "vsmc_cuda_smc_step_args");
        detail::MonitorLaunch<T> a;
        a.state = value_.data();
        a.N = static_cast<long long>(size_);
        a.iter = st.iter - 1;
        a.dim = static_cast<int>(dim);
        a.gather = gather_pending_ ? 1 : 0;
        a.lw = st.log_weight;
        a.lw_max = st.lw_max;
        a.s1 = st.weight_s1;
        a.resampled = st.resampled;
        a.copy_from = st.copy_from;
        a.part = part;
        cudaStream_t s = static_cast<cudaStream_t>(st.stream);
        detail::k_sampler_monitor<T, D>
            <<<detail::kMonitorBlocks, 256, 0, s>>>(d, a);
        detail::k_sampler_monitor_finish<<<1, 32, 0, s>>>(
            part, detail::kMonitorBlocks, static_cast<int>(dim), record);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess)
            throw RuntimeError(VSMC_CUDA_ECUDA,
                               std::string("Monitor kernel: ") +
                                   cudaGetErrorString(e));
    }

    void begin_init()
    {
        queue_pos_ = 0;
        first_move_ = true;
        gather_pending_ = false;
    }
    void begin_step()
    {
        queue_pos_ = 0;
        first_move_ = true;
    }
    void step_finished() { gather_pending_ = true; }
    void set_queue_pos(int k) { queue_pos_ = k; }

  private:
    size_type size_;
    T value_;
    std::uint32_t key_;
    std::uint32_t resample_seed_;
    vsmc_b200::DeviceVector<std::uint32_t> keys_;
    vsmc_b200::DeviceVector<std::uint64_t> words_;
    vsmc_cuda_smc *core_;
    void *stream_;
    int queue_pos_ = 0;
    bool first_move_ = true;
    bool gather_pending_ = false;
};

// ------------------------------------------------------- functor bases
// InitializeCUDA<T, Derived>: Derived defines
//   __device__ std::size_t initialize_state(SingleParticle<T> sp)
// and may define the host hooks initialize_param(Particle<T>&, void *),
// pre_processor(Particle<T>&), post_processor(Particle<T>&).
template <typename T, typename Derived>
class InitializeCUDA
{
  public:
    std::size_t operator()(Particle<T> &particle, void *param)
    {
        Derived &d = static_cast<Derived &>(*this);
        d.initialize_param(particle, param);
        d.pre_processor(particle);
        particle.template launch<Derived, detail::StageInit>(d);
        d.post_processor(particle);
        return 0;
    }
    void initialize_param(Particle<T> &, void *) {}
    void pre_processor(Particle<T> &) {}
    void post_processor(Particle<T> &) {}
};

// MoveCUDA<T, Derived>: Derived defines
//   __device__ std::size_t move_state(std::size_t iter, SingleParticle<T> sp)
// and may define pre_processor(iter, Particle<T>&) / post_processor.  In
// the move queue it updates weights; in the MCMC queue it must not.
template <typename T, typename Derived>
class MoveCUDA
{
  public:
    std::size_t operator()(std::size_t iter, Particle<T> &particle)
    {
        Derived &d = static_cast<Derived &>(*this);
        d.pre_processor(iter, particle);
        if (mcmc_)
            particle.template launch<Derived, detail::StageMCMC>(d);
        else
            particle.template launch<Derived, detail::StageMove>(d);
        d.post_processor(iter, particle);
        return 0;
    }
    void pre_processor(std::size_t, Particle<T> &) {}
    void post_processor(std::size_t, Particle<T> &) {}
    // set by Sampler::mcmc for functors placed in the MCMC queue
    void as_mcmc(bool m) { mcmc_ = m; }

  private:
    bool mcmc_ = false;
};

// MonitorEvalCUDA<T, Derived>: Derived defines
//   __device__ void monitor_state(std::size_t iter, std::size_t dim,
//                                 ConstSingleParticle<T> csp, double *res)
template <typename T, typename Derived>
class MonitorEvalCUDA
{
};

// The later vSMC spellings of the backend-generic names.
template <typename T, typename Derived>
using InitializeSMP = InitializeCUDA<T, Derived>;
template <typename T, typename Derived>
using MoveSMP = MoveCUDA<T, Derived>;
template <typename T, typename Derived>
using MonitorEvalSMP = MonitorEvalCUDA<T, Derived>;

// ------------------------------------------------------------ Monitor
// Monitor<T> (core/monitor.hpp): records of dim importance-sampling
// estimates per step, named like the reference's (name(i), record(i, iter)).
class Monitor
{
  public:
    Monitor(std::size_t dim, std::size_t T_max)
        : dim_(dim), T_max_(T_max), names_(dim), part_(detail::kMonitorBlocks * dim),
          rec_(T_max * dim), iter_(0), cached_(false)
    {
    }
    std::size_t dim() const { return dim_; }
    std::size_t iter_size() const { return iter_; }
    std::string &name(std::size_t i) { return names_[i]; }
    const std::string &name(std::size_t i) const { return names_[i]; }
    double record(std::size_t id, std::size_t iter) const
    {
        fetch();
        return host_[iter * dim_ + id];
    }
    void clear()
    {
        iter_ = 0;
        cached_ = false;
    }
    // device slots for the next evaluation
    double *part() { return part_.data(); }
    double *next_record()
    {
        if (iter_ >= T_max_)
            throw RuntimeError(VSMC_CUDA_EINVAL, "Monitor: more steps than T_max");
        cached_ = false;
        return rec_.data() + (iter_++) * dim_;
    }

  private:
    std::size_t dim_, T_max_;
    std::vector<std::string> names_;
    vsmc_b200::DeviceVector<double> part_, rec_;
    std::size_t iter_;
    mutable bool cached_;
    mutable std::vector<double> host_;

    void fetch() const
    {
        if (cached_)
            return;
        host_.assign(iter_ * dim_, 0.0);
        if (!host_.empty())
            rec_.download(host_.data(), host_.size());
        cached_ = true;
    }
};

// ------------------------------------------------------------ Sampler<T>
template <typename T>
class Sampler
{
  public:
    typedef std::size_t size_type;
    typedef T value_type;
    typedef std::function<std::size_t(Particle<T> &, void *)> init_type;
    typedef std::function<std::size_t(std::size_t, Particle<T> &)> move_type;
    typedef std::function<std::size_t(std::size_t, Particle<T> &)> mcmc_type;

    // Sampler(N): no resampling; Sampler(N, scheme): resample at every
    // step; Sampler(N, scheme, threshold): when ESS < threshold * N
    // (core/sampler.hpp:80-104).  T_max: steps of history on the device.
    explicit Sampler(size_type N, size_type T_max = 1024,
                     void *stream = nullptr)
        : particle_(N, Multinomial, 0.0, T_max, stream), T_max_(T_max)
    {
    }
    Sampler(size_type N, ResampleScheme scheme, size_type T_max = 1024,
            void *stream = nullptr)
        : particle_(N, scheme, std::numeric_limits<double>::max(), T_max,
                    stream),
          T_max_(T_max)
    {
    }
    Sampler(size_type N, ResampleScheme scheme, double threshold,
            size_type T_max = 1024, void *stream = nullptr)
        : particle_(N, scheme, threshold, T_max, stream), T_max_(T_max)
    {
    }

    size_type size() const { return particle_.size(); }
    std::size_t iter_size() const { return iter_; }
    Particle<T> &particle() { return particle_; }
    const Particle<T> &particle() const { return particle_; }

    Sampler &init(const init_type &f)
    {
        init_ = f;
        return *this;
    }
    Sampler &move(const move_type &f, bool append)
    {
        if (!append)
            move_queue_.clear();
        move_queue_.push_back(f);
        return *this;
    }
    // an MCMC move (MoveCUDA-derived): state only, after the resampling
    template <typename M>
    Sampler &mcmc(M f, bool append)
    {
        if (!append)
            mcmc_queue_.clear();
        f.as_mcmc(true);
        mcmc_queue_.push_back(move_type(f));
        return *this;
    }
    Sampler &move_queue_clear()
    {
        move_queue_.clear();
        return *this;
    }
    Sampler &mcmc_queue_clear()
    {
        mcmc_queue_.clear();
        return *this;
    }

    // Sampler::monitor(name, dim, eval): eval derives from MonitorEvalCUDA
    template <typename Eval>
    Sampler &monitor(const std::string &name, std::size_t dim,
                     const Eval &eval)
    {
        if (dim == 0 || dim > (std::size_t)detail::kMaxMonitorDim)
            throw RuntimeError(VSMC_CUDA_EINVAL,
                               "Sampler::monitor: dim must be 1..16");
        MonitorEntry m;
        m.mon = std::make_shared<Monitor>(dim, T_max_);
        Monitor *mp = m.mon.get();
        m.eval = [eval, mp, dim](Particle<T> &p) {
            p.launch_monitor(eval, dim, mp->part(), mp->next_record());
        };
        monitors_[name] = m;
        return *this;
    }
    Monitor &monitor(const std::string &name)
    {
        return *monitors_.at(name).mon;
    }
    const Monitor &monitor(const std::string &name) const
    {
        return *monitors_.at(name).mon;
    }

    // Sampler::initialize (core/sampler.hpp:450-463)
    Sampler &initialize(void *param = nullptr)
    {
        if (!init_)
            throw RuntimeError(VSMC_CUDA_EINVAL,
                               "Sampler::initialize: no init functor");
        vsmc_b200::check(vsmc_cuda_smc_reset(particle_.core()),
                         "vsmc_cuda_smc_reset");
        for (auto &m : monitors_)
            m.second.mon->clear();
        iter_ = 0;
        particle_.begin_init();
        init_(particle_, param);
        finish();
        return *this;
    }

    // Sampler::iterate (core/sampler.hpp:471-483): moves, resampling,
    // MCMC moves, monitors
    Sampler &iterate(std::size_t num = 1)
    {
        for (std::size_t n = 0; n != num; ++n) {
            if (iter_ >= T_max_)
                throw RuntimeError(VSMC_CUDA_EINVAL,
                                   "Sampler::iterate: more steps than T_max");
            particle_.begin_step();
            if (move_queue_.empty()) {
                detail::IdentityMove<T> id;
                particle_.template launch<detail::IdentityMove<T>,
                                          detail::StageMove>(id);
            }
            int k = 0;
            for (auto &m : move_queue_) {
                particle_.set_queue_pos(k++);
                m(iter_, particle_);
            }
            finish_resample();
            for (auto &m : mcmc_queue_) {
                particle_.set_queue_pos(k++);
                m(iter_, particle_);
            }
            do_monitor();
            ++iter_;
        }
        cached_ = false;
        return *this;
    }

    double ess_history(std::size_t i) const { return hist().ess[i]; }
    bool resampled_history(std::size_t i) const
    {
        return hist().resampled[i] != 0;
    }
    std::size_t size_history(std::size_t) const { return size(); }
    std::size_t accept_history(std::size_t id, std::size_t i) const
    {
        return static_cast<std::size_t>(
            hist().accept[i * VSMC_CUDA_SMC_MAX_QUEUE + id]);
    }
    double log_evidence_increment(std::size_t i) const
    {
        return hist().logz_inc[i];
    }
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

    // Sampler::print (core/sampler.hpp:684-721)
    template <typename CharT, typename Traits>
    std::basic_ostream<CharT, Traits> &print(
        std::basic_ostream<CharT, Traits> &os, char sepchar = '\t') const
    {
        if (iter_ == 0 || !os.good())
            return os;
        const History &h = hist();
        const std::size_t nacc =
            std::max<std::size_t>(1, move_queue_.size() + mcmc_queue_.size());
        os << "Size" << sepchar << "Resampled" << sepchar;
        for (std::size_t k = 0; k != nacc; ++k)
            os << "Accept." << k << sepchar;
        os << "ESS" << sepchar;
        for (const auto &m : monitors_) {
            const Monitor &mon = *m.second.mon;
            if (mon.iter_size() == 0)
                continue;
            for (std::size_t d = 0; d != mon.dim(); ++d) {
                if (!mon.name(d).empty())
                    os << mon.name(d) << sepchar;
                else
                    os << m.first << '.' << d << sepchar;
            }
        }
        os << '\n';
        for (std::size_t t = 0; t != iter_; ++t) {
            os << size() << sepchar << (h.resampled[t] != 0 ? 1 : 0)
               << sepchar;
            for (std::size_t k = 0; k != nacc; ++k)
                os << h.accept[t * VSMC_CUDA_SMC_MAX_QUEUE + k] << sepchar;
            os << h.ess[t] << sepchar;
            for (const auto &m : monitors_) {
                const Monitor &mon = *m.second.mon;
                if (mon.iter_size() == 0)
                    continue;
                for (std::size_t d = 0; d != mon.dim(); ++d)
                    os << mon.record(d, t) << sepchar;
            }
            os << '\n';
        }
        return os;
    }

  private:
    struct MonitorEntry {
        std::shared_ptr<Monitor> mon;
        std::function<void(Particle<T> &)> eval;
    };
    struct History {
        std::vector<double> ess, logz_inc;
        std::vector<std::int32_t> resampled;
        std::vector<std::uint64_t> accept;
    };

    Particle<T> particle_;
    std::size_t T_max_;
    std::size_t iter_ = 0;
    init_type init_;
    std::vector<move_type> move_queue_, mcmc_queue_;
    std::map<std::string, MonitorEntry> monitors_;
    mutable bool cached_ = false;
    mutable History h_;

    void finish_resample()
    {
        vsmc_b200::check(vsmc_cuda_smc_finish_step(particle_.core()),
                         "vsmc_cuda_smc_finish_step");
        particle_.step_finished();
    }
    void do_monitor()
    {
        for (auto &m : monitors_)
            m.second.eval(particle_);
    }
    void finish()
    {
        finish_resample();
        do_monitor();
        iter_ = 1;
        cached_ = false;
    }
    const History &hist() const
    {
        if (!cached_) {
            h_.ess.assign(iter_, 0.0);
            h_.logz_inc.assign(iter_, 0.0);
            h_.resampled.assign(iter_, 0);
            h_.accept.assign(iter_ * VSMC_CUDA_SMC_MAX_QUEUE, 0);
            vsmc_cuda_smc *c =
                const_cast<Particle<T> &>(particle_).core();
            if (iter_ > 0)
                vsmc_b200::check(
                    vsmc_cuda_smc_history(c, h_.ess.data(),
                                          h_.resampled.data(),
                                          h_.logz_inc.data(),
                                          h_.accept.data()),
                    "vsmc_cuda_smc_history");
            cached_ = true;
        }
        return h_;
    }
};

template <typename CharT, typename Traits, typename T>
inline std::basic_ostream<CharT, Traits> &operator<<(
    std::basic_ostream<CharT, Traits> &os, const Sampler<T> &s)
{
    return s.print(os);
}

// BASELINE's WeightSet spelling: Weight::set_log / add_log / ess on the
// device-resident weight set of the C++ interface.
class Weight : public vsmc_b200::WeightSetCUDA
{
  public:
    using vsmc_b200::WeightSetCUDA::WeightSetCUDA;
    template <typename InputIter>
    void set_log(InputIter first)
    {
        set_log_weight(first);
    }
    template <typename InputIter>
    void add_log(InputIter first)
    {
        add_log_weight(first);
    }
};
typedef vsmc_b200::WeightSetCUDA WeightSet;

} // namespace vsmc

#endif // VSMC_B200_SMC_CUH
