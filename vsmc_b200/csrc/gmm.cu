// gmm.cu -- tempered SMC sampler for a 1-D Gaussian mixture on the device.
//
// The sampler of the reference's example/gmm (gmm_smc.cpp) with the
// alpha_prior schedule: Sampler<gmm_state>(N, scheme, threshold); init
// gmm_init; move move_smc (tempering step: alpha_t = (t / T)^power,
// incremental weight loglik * (alpha_t - alpha_{t-1}), log-evidence
// increment); resampling when ESS < threshold N; then `sweeps` sweeps of the
// three Metropolis-Hastings block moves gmm_move_mu, gmm_move_lambda and
// gmm_move_weight; path sampling over (alpha_t, sum_i W_i loglik_i).
//
// Reference: example/gmm/include/gmm_param.hpp, gmm_state.hpp:61-168,
// gmm_init.hpp:51-76, gmm_move.hpp:35-117, example/include/move_smc.hpp:
// 51-75, move_alpha.hpp:120-140, smc_path.hpp, core/path.hpp:170-239,
// core/sampler.hpp:450-483, 758-834; the draws are libstdc++'s normal,
// lognormal, gamma and uniform distributions over each particle's own
// Threefry4x64 engine (RngSet<Threefry4x64, Vector>, rng/rng_set.hpp).
//
// Kernels of a step (t >= 1):
//   k_gmm_reweight   lw += loglik * alpha_inc, per-tile log-sum-exp stats
//   k_cv_finalize    normalising constant, ESS, log-evidence increment,
//                    resampling decision, weight spine (shared with the
//                    CV filter)
//   resample.cuh     the scheme's kernels (return at once if no resampling)
//   k_gmm_mcmc       gather through copy_from + sweeps x 3 MH moves; one
//                    particle per group of G lanes, the likelihood's data
//                    loop split over the group; per-CTA acceptance counts
//   k_gmm_path       acceptance totals, path integrand, trapezoid rule
//
// Forms: FP64 evaluates the likelihood in double throughout (the reference
// arithmetic, one rounding per operation in the reference's order); MIXED
// evaluates each data point's mixture density in float (exp2 / log2 on the
// special-function units, one log2 per pair of points) and accumulates the
// log terms of a particle in double.  Everything else is double in both.
#include "cv_kernels.cuh"

#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

namespace vsmc_b200 {

void set_last_error(const std::string &msg);
int cuda_status(cudaError_t e, const char *what);

constexpr int kGmmK = 4;              // mixture components
constexpr int kGmmThreads = 256;      // threads per MCMC CTA
constexpr int kGmmMaxSweeps = 16;
constexpr int kGmmMaxAcc = 3 * kGmmMaxSweeps;
constexpr int kGmmMaxData = 16384;    // data points held in shared memory
constexpr int kGmmParamArrays = 14;   // mu[4], lambda[4], weight[4], lp, ll

// CTAs per SM the MCMC and init kernels are compiled for (register cap).
#ifndef VSMC_GMM_MIN_BLOCKS
#define VSMC_GMM_MIN_BLOCKS 2
#endif

// SoA parameter buffer: array a of particle i at base[a * N + i].
struct GmmBuf {
    double *base;
};

struct GmmArgs {
    GmmBuf src, dst;
    const int32_t *copy_from;
    const FilterCtl *ctl;
    uint64_t *words;
    const void *data; // n doubles (FP64) or floats (MIXED)
    int n;
    long long N;
    double mu0, sd0, shape0, scale0;
    double alpha, sd;
    int sweeps;
    uint32_t seed_base; // Seed after Seed::set(seed), before any get()
    long long *tile_acc; // per CTA: 3 * sweeps acceptance counts
};

struct GmmState {
    double mu[kGmmK], lam[kGmmK], loglam[kGmmK], w[kGmmK];
    double lp, ll, lt;
};

// One out-of-line copy of the double log / exp / sqrt for the proposal and
// acceptance code: inlined at every call site they made the kernel too large
// for the instruction cache (warps stalled waiting for instructions).
static __device__ __noinline__ double mh_log(double x) { return log(x); }
static __device__ __noinline__ double mh_exp(double x) { return exp(x); }
static __device__ __noinline__ double mh_sqrt(double x) { return sqrt(x); }

// One Threefry4x64-20 block, out of line for the same reason.
static __device__ __noinline__ u64x4 mh_threefry(uint64_t ctr0, u64x4 key)
{
    u64x4 c;
    c.v[0] = ctr0;
    c.v[1] = c.v[2] = c.v[3] = 0;
    return threefry4x64_20(c, key);
}

// One particle's Threefry4x64 engine: key {seed_i, 0, 0, 0}; the word at
// position `off` is lane off % 4 of block ctr = off / 4 + 1 (the counter is
// incremented before each block, utility/counter.hpp).
struct ParticleRng {
    u64x4 key;
    uint64_t off;
    uint64_t blk; // block held in b0..b3 (~0 = none)
    uint64_t b0, b1, b2, b3;

    __device__ __forceinline__ void init(uint32_t k0, uint64_t offset)
    {
        key.v[0] = k0;
        key.v[1] = key.v[2] = key.v[3] = 0;
        off = offset;
        blk = ~0ull;
    }

    __device__ __forceinline__ uint64_t next()
    {
        const uint64_t b = off >> 2;
        if (b != blk) {
            const u64x4 w = mh_threefry(b + 1, key);
            b0 = w.v[0];
            b1 = w.v[1];
            b2 = w.v[2];
            b3 = w.v[3];
            blk = b;
        }
        const unsigned l = (unsigned)(off & 3);
        ++off;
        return l == 0 ? b0 : (l == 1 ? b1 : (l == 2 ? b2 : b3));
    }

    __device__ __forceinline__ double canonical()
    {
        return canonical_u64(next());
    }
};

// libstdc++ normal_distribution: Marsaglia polar method, the second value
// of a pair cached in the distribution object.
struct NormalDist {
    double saved;
    bool avail;

    __device__ __forceinline__ void reset()
    {
        avail = false;
        saved = 0.0;
    }

    __device__ __forceinline__ double operator()(ParticleRng &r, double mean,
                                                 double sd)
    {
        double ret;
        if (avail) {
            avail = false;
            ret = saved;
        } else {
            double x, y, r2;
            do {
                x = 2.0 * r.canonical() - 1.0;
                y = 2.0 * r.canonical() - 1.0;
                r2 = __dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y));
            } while (r2 > 1.0 || r2 == 0.0);
            const double mult = mh_sqrt(__ddiv_rn(-2.0 * mh_log(r2), r2));
            saved = __dmul_rn(x, mult);
            avail = true;
            ret = __dmul_rn(y, mult);
        }
        return __dadd_rn(__dmul_rn(ret, sd), mean);
    }
};

// libstdc++ gamma_distribution (Marsaglia and Tsang) with its own normal.
__device__ __forceinline__ double gamma_draw(NormalDist &nd, ParticleRng &r,
                                             double alpha, double beta)
{
    const double malpha = alpha < 1.0 ? alpha + 1.0 : alpha;
    const double a1 = malpha - 1.0 / 3.0;
    const double a2 = 1.0 / sqrt(9.0 * a1);
    double u, v, n;
    for (;;) {
        do {
            n = nd(r, 0.0, 1.0);
            v = __dadd_rn(1.0, __dmul_rn(a2, n));
        } while (v <= 0.0);
        v = __dmul_rn(__dmul_rn(v, v), v);
        u = r.canonical();
        const double n4 =
            __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(0.0331, n), n), n), n);
        if (!(u > __dadd_rn(1.0, -n4)))
            break;
        const double rhs = __dadd_rn(
            __dmul_rn(__dmul_rn(0.5, n), n),
            __dmul_rn(a1, __dadd_rn(__dadd_rn(1.0, -v), mh_log(v))));
        if (!(mh_log(u) > rhs))
            break;
    }
    if (alpha == malpha)
        return __dmul_rn(__dmul_rn(a1, v), beta);
    do
        u = r.canonical();
    while (u == 0.0);
    return pow(u, 1.0 / alpha) * a1 * v * beta;
}

// Special-function unit instructions (PTX ex2.approx.ftz.f32 and
// lg2.approx.ftz.f32): 2^x and log2 x in float, subnormals flushed to 0.
__device__ __forceinline__ float sfu_ex2(float x)
{
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ float sfu_lg2(float x)
{
    float y;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// MIXED form: the mixture density of one point plus the reference's 1e-13
// floor, in float.
__device__ __forceinline__ float mix_density(float x, const float *m,
                                             const float *A, const float *B)
{
    float lli = 0.0f;
#pragma unroll
    for (int d = 0; d < kGmmK; ++d) {
        const float r = __fsub_rn(x, m[d]);
        lli = __fadd_rn(lli, sfu_ex2(__fmaf_rn(-B[d], __fmul_rn(r, r), A[d])));
    }
    return __fadd_rn(lli, 1e-13f);
}

// The likelihood's sum over the data points has one fixed order whatever
// the lanes per particle G: point i goes to class i mod 16, each class sums
// its points in increasing order, and the 16 class sums are added in a
// balanced binary tree.  Lane g of a group holds classes g, g + G, ...; an
// xor butterfly over the group forms the subtrees of G consecutive classes
// (IEEE addition is commutative, so every lane gets the same bits) and the
// lane adds those subtrees pairwise.  G only changes the speed.
constexpr int kLlClasses = 16;

template <int G, bool F32>
__device__ __forceinline__ double gmm_loglik(const GmmState &s,
                                             const void *data, int n, int g,
                                             unsigned mask)
{
    constexpr int J = kLlClasses / G;
    double acc[J];
#pragma unroll
    for (int j = 0; j < J; ++j)
        acc[j] = 0.0;
    if (F32) {
        // w_d exp(0.5 log lambda_d - 0.5 lambda_d r^2) = exp2(A_d - B_d r^2)
        constexpr double kLog2e = 1.4426950408889634074;
        float m[kGmmK], A[kGmmK], B[kGmmK];
#pragma unroll
        for (int d = 0; d < kGmmK; ++d) {
            m[d] = (float)s.mu[d];
            A[d] = (float)(log2(s.w[d]) + 0.5 * s.loglam[d] * kLog2e);
            B[d] = (float)(0.5 * s.lam[d] * kLog2e);
        }
        // Points i and i + 16 of a class share one log: log2 of the
        // product of their densities (each >= 1e-13, so the product stays
        // a normal float); the class adds these pair terms in double.
        const float *x = static_cast<const float *>(data);
        for (int base = 0; base < n; base += 2 * kLlClasses) {
#pragma unroll
            for (int j = 0; j < J; ++j) {
                const int i = base + g + j * G;
                if (i < n) {
                    float p = mix_density(x[i], m, A, B);
                    if (i + kLlClasses < n)
                        p = __fmul_rn(p, mix_density(x[i + kLlClasses], m, A, B));
                    acc[j] = __dadd_rn(acc[j], (double)sfu_lg2(p));
                }
            }
        }
    } else {
        const double *x = static_cast<const double *>(data);
        double c[kGmmK], h[kGmmK];
#pragma unroll
        for (int d = 0; d < kGmmK; ++d) {
            c[d] = __dmul_rn(0.5, s.loglam[d]);
            h[d] = __dmul_rn(0.5, s.lam[d]);
        }
        for (int base = 0; base < n; base += kLlClasses) {
#pragma unroll
            for (int j = 0; j < J; ++j) {
                const int i = base + g + j * G;
                if (i < n) {
                    // lli += w_d exp(0.5 log lambda_d - 0.5 lambda_d r r)
                    double lli = 0.0;
#pragma unroll
                    for (int d = 0; d < kGmmK; ++d) {
                        const double r = __dsub_rn(x[i], s.mu[d]);
                        const double t = __dmul_rn(__dmul_rn(h[d], r), r);
                        const double e = exp(__dsub_rn(c[d], t));
                        lli = __dadd_rn(lli, __dmul_rn(s.w[d], e));
                    }
                    acc[j] = __dadd_rn(acc[j], log(__dadd_rn(lli, 1e-13)));
                }
            }
        }
    }
#pragma unroll
    for (int j = 0; j < J; ++j)
#pragma unroll
        for (int o = 1; o < G; o <<= 1)
            acc[j] = __dadd_rn(acc[j], __shfl_xor_sync(mask, acc[j], o));
#pragma unroll
    for (int w = 1; w < J; w <<= 1)
#pragma unroll
        for (int j = 0; j + w < J; j += 2 * w)
            acc[j] = __dadd_rn(acc[j], acc[j + w]);
    return F32 ? __dmul_rn(acc[0], 0.69314718055994530942) : acc[0];
}

// gmm_state::log_prior (gmm_state.hpp:67-80)
__device__ __forceinline__ double gmm_log_prior(const GmmState &s,
                                                const GmmArgs &a)
{
    double lp = 0.0;
    const double sd02 = __dmul_rn(a.sd0, a.sd0);
#pragma unroll
    for (int d = 0; d < kGmmK; ++d) {
        const double resid = __dsub_rn(s.mu[d], a.mu0);
        lp = __dadd_rn(lp, __ddiv_rn(__dmul_rn(-0.5, __dmul_rn(resid, resid)),
                                     sd02));
        lp = __dadd_rn(lp, __dsub_rn(__dmul_rn(a.shape0 - 1, s.loglam[d]),
                                     __ddiv_rn(s.lam[d], a.scale0)));
    }
    return lp;
}

// gmm_state::log_target: log prior + alpha * log likelihood (the likelihood
// refreshes log lambda).
template <int G, bool F32>
__device__ __forceinline__ void gmm_log_target(GmmState &s, const GmmArgs &a,
                                               const void *data, int g,
                                               unsigned mask)
{
#pragma unroll
    for (int d = 0; d < kGmmK; ++d)
        s.loglam[d] = mh_log(s.lam[d]);
    s.lp = gmm_log_prior(s, a); // its log(lambda_d) is loglam[d]
    s.ll = gmm_loglik<G, F32>(s, data, a.n, g, mask);
    s.lt = __dadd_rn(s.lp, __dmul_rn(a.alpha, s.ll));
}

// logit_weight_diff's per-vector term (gmm_param.hpp:221-248)
__device__ __forceinline__ double logit_term(const double *w)
{
    double sum_lw = 1.0, sum_llw = 0.0;
#pragma unroll
    for (int d = 0; d < kGmmK - 1; ++d) {
        const double r = __ddiv_rn(w[d], w[kGmmK - 1]);
        sum_lw = __dadd_rn(sum_lw, r);
        sum_llw = __dadd_rn(sum_llw, mh_log(r));
    }
    return __dsub_rn(sum_llw, __dmul_rn((double)kGmmK, mh_log(sum_lw)));
}

// The three block moves (gmm_move.hpp:35-117); each returns 1 if accepted.
template <int G, bool F32>
__device__ __forceinline__ int gmm_move_block(int block, GmmState &s,
                                              ParticleRng &rng,
                                              const GmmArgs &a,
                                              const void *data, int g,
                                              unsigned mask)
{
    const GmmState o = s; // save_old
    const double lt_old = __dadd_rn(s.lp, __dmul_rn(a.alpha, s.ll));
    NormalDist nd;
    nd.reset();
    double extra = 0.0;
    if (block == 0) {
#pragma unroll
        for (int d = 0; d < kGmmK; ++d)
            s.mu[d] = __dadd_rn(s.mu[d], nd(rng, 0.0, a.sd));
    } else if (block == 1) {
        // lognormal_distribution(0, sd): exp(sd * n + 0)
#pragma unroll
        for (int d = 0; d < kGmmK; ++d)
            s.lam[d] = __dmul_rn(
                s.lam[d],
                mh_exp(__dadd_rn(__dmul_rn(a.sd, nd(rng, 0.0, 1.0)), 0.0)));
    } else {
        double sum_weight = 1.0;
#pragma unroll
        for (int d = 0; d < kGmmK - 1; ++d) {
            double v = mh_log(__ddiv_rn(s.w[d], s.w[kGmmK - 1]));
            v = __dadd_rn(v, nd(rng, 0.0, a.sd));
            v = mh_exp(v);
            s.w[d] = v;
            sum_weight = __dadd_rn(sum_weight, v);
        }
        s.w[kGmmK - 1] = 1.0;
#pragma unroll
        for (int d = 0; d < kGmmK; ++d)
            s.w[d] = __ddiv_rn(s.w[d], sum_weight);
    }
    gmm_log_target<G, F32>(s, a, data, g, mask);
    if (block == 1) {
        double lld = 0.0;
#pragma unroll
        for (int d = 0; d < kGmmK; ++d)
            lld = __dadd_rn(lld, __dsub_rn(s.loglam[d], o.loglam[d]));
        extra = lld;
    } else if (block == 2) {
        extra = __dsub_rn(logit_term(s.w), logit_term(o.w));
    }
    const double p = block == 0 ? __dsub_rn(s.lt, lt_old)
                                : __dadd_rn(__dsub_rn(s.lt, lt_old), extra);
    const double u = mh_log(rng.canonical());
    if (p < u) {
        s = o;
        s.lt = lt_old;
        return 0;
    }
    return 1;
}

template <int G>
__device__ __forceinline__ unsigned group_mask()
{
    if (G >= 32)
        return 0xffffffffu;
    const unsigned lane = threadIdx.x & 31;
    return ((1u << G) - 1u) << (lane & ~(unsigned)(G - 1));
}

__device__ __forceinline__ uint32_t particle_key(uint32_t base, long long i)
{
    // the (i+1)-th Seed::get() after Seed::set: ((base + i) mod (2^32 - 1)) + 1
    return (uint32_t)(((uint64_t)base + (uint64_t)i) % 0xFFFFFFFFull) + 1u;
}

__device__ __forceinline__ void load_state(GmmState &s, const GmmBuf &b,
                                           long long N, long long i)
{
#pragma unroll
    for (int d = 0; d < kGmmK; ++d) {
        s.mu[d] = b.base[d * N + i];
        s.lam[d] = b.base[(4 + d) * N + i];
        s.w[d] = b.base[(8 + d) * N + i];
        s.loglam[d] = mh_log(s.lam[d]);
    }
    s.lp = b.base[12 * N + i];
    s.ll = b.base[13 * N + i];
    s.lt = s.lp; // recomputed by save_old before use
}

__device__ __forceinline__ void store_state(const GmmState &s, GmmBuf &b,
                                            long long N, long long i)
{
#pragma unroll
    for (int d = 0; d < kGmmK; ++d) {
        b.base[d * N + i] = s.mu[d];
        b.base[(4 + d) * N + i] = s.lam[d];
        b.base[(8 + d) * N + i] = s.w[d];
    }
    b.base[12 * N + i] = s.lp;
    b.base[13 * N + i] = s.ll;
}

// Stage the data in shared memory.
template <bool F32>
__device__ __forceinline__ const void *stage_data(const GmmArgs &a,
                                                  unsigned char *smem)
{
    if (F32) {
        float *x = reinterpret_cast<float *>(smem);
        const float *src = static_cast<const float *>(a.data);
        for (int i = threadIdx.x; i < a.n; i += blockDim.x)
            x[i] = src[i];
    } else {
        double *x = reinterpret_cast<double *>(smem);
        const double *src = static_cast<const double *>(a.data);
        for (int i = threadIdx.x; i < a.n; i += blockDim.x)
            x[i] = src[i];
    }
    __syncthreads();
    return smem;
}

// Per-CTA acceptance counts (integer sums: any order gives the same).  Bit
// m of `acc` is 1 if this thread's particle accepted move m.
__device__ __forceinline__ void cta_reduce_acc(uint64_t acc, int nacc,
                                               long long *tile_acc)
{
    __shared__ long long sh_acc[kGmmThreads / 32][kGmmMaxAcc];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int k = 0; k < nacc; ++k) {
        const unsigned votes =
            __ballot_sync(0xffffffffu, (unsigned)((acc >> k) & 1u));
        if (lane == 0)
            sh_acc[wid][k] = __popc(votes);
    }
    __syncthreads();
    if (threadIdx.x < nacc) {
        long long t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
            t += sh_acc[w][threadIdx.x];
        tile_acc[(long long)blockIdx.x * kGmmMaxAcc + threadIdx.x] = t;
    }
}

// Initialisation (gmm_init::initialize_state): prior draws, log target at
// alpha 0, log-weight 0.  Each engine continues from its stored position
// (the RngSet outlives Sampler::initialize).
template <int G, bool F32>
__global__ void __launch_bounds__(kGmmThreads, VSMC_GMM_MIN_BLOCKS)
k_gmm_init(GmmArgs a, double *lw)
{
    extern __shared__ __align__(16) unsigned char gmm_smem[];
    const void *data = stage_data<F32>(a, gmm_smem);
    const long long gt = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long i0 = gt / G;
    const int g = (int)(gt % G);
    const bool active = i0 < a.N;
    const long long i = active ? i0 : a.N - 1;
    const unsigned mask = group_mask<G>();
    ParticleRng rng;
    rng.init(particle_key(a.seed_base, i), a.words[i]);
    GmmState s;
    NormalDist nmu, nlam, nw;
    nmu.reset();
    nlam.reset();
    nw.reset();
    double sum_weight = 0.0;
#pragma unroll
    for (int d = 0; d < kGmmK; ++d) {
        s.mu[d] = nmu(rng, a.mu0, a.sd0);
        s.lam[d] = gamma_draw(nlam, rng, a.shape0, a.scale0);
        s.w[d] = gamma_draw(nw, rng, 1.0, 1.0);
        sum_weight = __dadd_rn(sum_weight, s.w[d]);
    }
#pragma unroll
    for (int d = 0; d < kGmmK; ++d)
        s.w[d] = __ddiv_rn(s.w[d], sum_weight);
    gmm_log_target<G, F32>(s, a, data, g, mask);
    // every lane of the group has read words[i] before the leader writes
    __syncwarp();
    if (active && g == 0) {
        store_state(s, a.dst, a.N, i);
        a.words[i] = rng.off;
        lw[i] = 0.0;
    }
    cta_reduce_acc(0, 3 * a.sweeps, a.tile_acc);
}

// One MCMC stage: gather (if this step resampled), sweeps x 3 MH moves.
template <int G, bool F32>
__global__ void __launch_bounds__(kGmmThreads, VSMC_GMM_MIN_BLOCKS)
k_gmm_mcmc(GmmArgs a)
{
    extern __shared__ __align__(16) unsigned char gmm_smem[];
    const void *data = stage_data<F32>(a, gmm_smem);
    const long long gt = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long i0 = gt / G;
    const int g = (int)(gt % G);
    const bool active = i0 < a.N;
    const long long i = active ? i0 : a.N - 1;
    const unsigned mask = group_mask<G>();
    const int resampled = a.ctl->resampled;
    long long src = i;
    if (resampled) {
        src = a.copy_from[i];
        src = src < 0 ? 0 : (src >= a.N ? a.N - 1 : src);
    }
    GmmState s;
    load_state(s, a.src, a.N, src);
    ParticleRng rng;
    rng.init(particle_key(a.seed_base, i), a.words[i]);
    uint64_t acc = 0; // bit 3k + b: sweep k's move b accepted
#pragma unroll 1
    for (int k = 0; k < a.sweeps; ++k)
#pragma unroll 1
        for (int b = 0; b < 3; ++b)
            acc |= (uint64_t)gmm_move_block<G, F32>(b, s, rng, a, data, g,
                                                    mask)
                   << (3 * k + b);
    __syncwarp();
    const bool leader = active && g == 0;
    if (leader) {
        store_state(s, a.dst, a.N, i);
        a.words[i] = rng.off;
    } else {
        acc = 0;
    }
    cta_reduce_acc(acc, 3 * a.sweeps, a.tile_acc);
}

// Likelihood only (autotuning and precision checks): ll of every particle
// of `src` into out[i].
template <int G, bool F32>
__global__ void __launch_bounds__(kGmmThreads)
k_gmm_loglik(GmmArgs a, double *out)
{
    extern __shared__ __align__(16) unsigned char gmm_smem[];
    const void *data = stage_data<F32>(a, gmm_smem);
    const long long gt = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long i0 = gt / G;
    const int g = (int)(gt % G);
    const long long i = i0 < a.N ? i0 : a.N - 1;
    GmmState s;
    load_state(s, a.src, a.N, i);
    const double ll = gmm_loglik<G, F32>(s, data, a.n, g, group_mask<G>());
    if (i0 < a.N && g == 0)
        out[i] = ll;
}

// move_smc: lw += loglik * alpha_inc (after resampling lw restarts at 0),
// with the online log-sum-exp statistics of each tile of kTile particles.
static __global__ void __launch_bounds__(kThreads)
k_gmm_reweight(const double *ll, double *lw, const FilterCtl *ctl,
               long long N, double alpha_inc, TileStats *ts)
{
    __shared__ double sh[3][kThreads / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int gather = ctl->resampled;
    const double mprev = gather ? 0.0 : ctl->lw_max;
    const long long base = (long long)blockIdx.x * kTile;
    LseRef acc;
    acc.init();
#pragma unroll 4
    for (int k = 0; k < kItems; ++k) {
        const long long i = base + (long long)k * kThreads + threadIdx.x;
        if (i < N) {
            const double v = __dadd_rn(gather ? 0.0 : __dsub_rn(lw[i], mprev),
                                       __dmul_rn(ll[i], alpha_inc));
            lw[i] = v;
            lse_add<double>(acc, v, 0.0, 0.0);
        }
    }
    const double wm = warp_max_nan(acc.mx, 32);
    lse_rescale(acc, wm);
    double gx = 0.0, gy = 0.0;
    warp_sum_stats(acc, gx, gy, 32);
    if (lane == 0) {
        sh[0][wid] = wm;
        sh[1][wid] = acc.s1;
        sh[2][wid] = acc.s2;
    }
    __syncthreads();
    if (wid == 0) {
        constexpr int NW = kThreads / 32;
        LseRef r;
        r.init();
        if (lane < NW) {
            r.ref = sh[0][lane];
            r.mx = r.ref;
            r.s1 = sh[1][lane];
            r.s2 = sh[2][lane];
        }
        const double tm = warp_max_nan(r.mx, NW);
        lse_rescale(r, tm);
        double hx = 0.0, hy = 0.0;
        warp_sum_stats(r, hx, hy, NW);
        if (lane == 0) {
            TileStats t;
            t.m = tm;
            t.s1 = r.s1;
            t.s2 = r.s2;
            t.sx = t.sy = t.gx = t.gy = t.pad = 0.0;
            ts[blockIdx.x] = t;
        }
    }
}

struct GmmCtl {
    double prev_integrand;
    double prev_grid;
    double path_logz;
};

// Acceptance totals and path sampling of step t (Path::eval + push_back):
// integrand = sum_i w_i loglik_i / sum_i w_i with w_i = 1 after resampling
// and exp(lw_i - M) otherwise, grid = alpha_t, trapezoid rule.  The sums
// run over the particles in one fixed order (thread k of 1024 takes
// i = k, k + 1024, ...).
static __global__ void __launch_bounds__(1024)
k_gmm_path(const long long *tile_acc, int ntiles, int nacc,
           const double *ll, const double *lw, const FilterCtl *ctl,
           long long N, long long t, double grid, GmmCtl *gc,
           int64_t *hist_accept, double *hist_integrand, double *hist_grid)
{
    __shared__ double sh[2][32];
    __shared__ long long sha[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int resampled = ctl->resampled;
    const double M = ctl->lw_max;
    double p0 = 0.0, p1 = 0.0;
    for (long long i = threadIdx.x; i < N; i += blockDim.x) {
        const double w = resampled ? 1.0 : exp(lw[i] - M);
        p0 = __dadd_rn(p0, __dmul_rn(w, ll[i]));
        p1 = __dadd_rn(p1, w);
    }
    p0 = warp_sum(p0);
    p1 = warp_sum(p1);
    if (lane == 0) {
        sh[0][wid] = p0;
        sh[1][wid] = p1;
    }
    for (int m = 0; m < nacc; ++m) {
        __syncthreads();
        long long v = 0;
        for (int k = threadIdx.x; k < ntiles; k += blockDim.x)
            v += tile_acc[(long long)k * kGmmMaxAcc + m];
        for (int o = 16; o > 0; o >>= 1)
            v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0)
            sha[wid] = v;
        __syncthreads();
        if (threadIdx.x == 0) {
            long long tot = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
                tot += sha[w];
            hist_accept[t * (1 + nacc) + 1 + m] = tot;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s0 = 0.0, s1 = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            s0 += sh[0][w];
            s1 += sh[1][w];
        }
        const double integrand = s0 / s1;
        hist_accept[t * (1 + nacc)] = 0;
        hist_integrand[t] = integrand;
        hist_grid[t] = grid;
        if (t > 0)
            gc->path_logz += 0.5 * (grid - gc->prev_grid) *
                             (integrand + gc->prev_integrand);
        else
            gc->path_logz = 0.0;
        gc->prev_grid = grid;
        gc->prev_integrand = integrand;
    }
}

} // namespace vsmc_b200

using namespace vsmc_b200;

struct vsmc_cuda_gmm {
    vsmc_cuda_gmm_config cfg;
    cudaStream_t stream;
    char *mem;
    size_t bytes;
    GmmBuf buf[2];
    int cur;
    double *lw;
    uint64_t *words;
    int32_t *copy_from;
    FilterCtl *ctl;
    GmmCtl *gctl;
    TileStats *tile_stats;
    long long *tile_acc;
    double *scratch; // N doubles (loglik checks)
    double *data64;  // the data in double
    float *data32;   // and in float (MIXED form)
    int n;
    double mu0, sd0, shape0, scale0;
    double *hist_ess, *hist_zinc, *hist_integrand, *hist_grid;
    double *hist_mx, *hist_my; // finalize's monitor slots (unused)
    int32_t *hist_resampled;
    int64_t *hist_accept;
    ResampleWorkspace rws;
    EngineRef eng;
    long long ntiles;      // kTile tiles (weights)
    int group;             // lanes per particle
    uint64_t iter;         // steps done (initialize = 1)
    double alpha;
    uint32_t seed_base;
    // timing of the MCMC kernels (vsmc_cuda_gmm_set_timing)
    bool timing;
    std::vector<cudaEvent_t> ev;
    size_t ev_used;
    uint64_t launches;
};

namespace {

constexpr double kLnPi2 = 1.8378770664093454835606594728112;

int gmm_ntiles_mcmc(long long N, int G)
{
    return (int)((N * G + kGmmThreads - 1) / kGmmThreads);
}

bool gmm_f32(const vsmc_cuda_gmm *g) { return g->cfg.form == VSMC_CUDA_MIXED; }

GmmArgs gmm_args(vsmc_cuda_gmm *g, int src, int dst)
{
    GmmArgs a;
    a.src = g->buf[src];
    a.dst = g->buf[dst];
    a.copy_from = g->copy_from;
    a.ctl = g->ctl;
    a.words = g->words;
    a.data = gmm_f32(g) ? (const void *)g->data32 : (const void *)g->data64;
    a.n = g->n;
    a.N = (long long)g->cfg.N;
    a.mu0 = g->mu0;
    a.sd0 = g->sd0;
    a.shape0 = g->shape0;
    a.scale0 = g->scale0;
    a.alpha = g->alpha;
    a.sd = g->cfg.sd;
    a.sweeps = g->cfg.sweeps;
    a.seed_base = g->seed_base;
    a.tile_acc = g->tile_acc;
    return a;
}

#define VSMC_GMM_SWITCH(G, CALL)                                              \
    switch (G) {                                                              \
    case 1:                                                                   \
        CALL(1);                                                              \
        break;                                                                \
    case 2:                                                                   \
        CALL(2);                                                              \
        break;                                                                \
    case 4:                                                                   \
        CALL(4);                                                              \
        break;                                                                \
    case 8:                                                                   \
        CALL(8);                                                              \
        break;                                                                \
    default:                                                                  \
        CALL(16);                                                             \
        break;                                                                \
    }

template <bool F32>
void launch_init_t(vsmc_cuda_gmm *g, const GmmArgs &a, int G, unsigned grid)
{
    const size_t smem = (size_t)a.n * (F32 ? 4 : 8);
#define VSMC_CALL(K)                                                          \
    k_gmm_init<K, F32><<<grid, kGmmThreads, smem, g->stream>>>(a, g->lw)
    VSMC_GMM_SWITCH(G, VSMC_CALL)
#undef VSMC_CALL
}

template <bool F32>
void launch_mcmc_t(vsmc_cuda_gmm *g, const GmmArgs &a, int G, unsigned grid)
{
    const size_t smem = (size_t)a.n * (F32 ? 4 : 8);
#define VSMC_CALL(K)                                                          \
    k_gmm_mcmc<K, F32><<<grid, kGmmThreads, smem, g->stream>>>(a)
    VSMC_GMM_SWITCH(G, VSMC_CALL)
#undef VSMC_CALL
}

template <bool F32>
void launch_loglik_t(vsmc_cuda_gmm *g, const GmmArgs &a, int G, double *out)
{
    const unsigned grid = (unsigned)gmm_ntiles_mcmc(a.N, G);
    const size_t smem = (size_t)a.n * (F32 ? 4 : 8);
#define VSMC_CALL(K)                                                          \
    k_gmm_loglik<K, F32><<<grid, kGmmThreads, smem, g->stream>>>(a, out)
    VSMC_GMM_SWITCH(G, VSMC_CALL)
#undef VSMC_CALL
}

template <bool F32>
void set_smem_attrs(size_t smem)
{
    const int b = (int)smem;
#define VSMC_GMM_ATTR(G)                                                      \
    cudaFuncSetAttribute(k_gmm_init<G, F32>,                                  \
                         cudaFuncAttributeMaxDynamicSharedMemorySize, b);     \
    cudaFuncSetAttribute(k_gmm_mcmc<G, F32>,                                  \
                         cudaFuncAttributeMaxDynamicSharedMemorySize, b);     \
    cudaFuncSetAttribute(k_gmm_loglik<G, F32>,                                \
                         cudaFuncAttributeMaxDynamicSharedMemorySize, b)
    VSMC_GMM_ATTR(1);
    VSMC_GMM_ATTR(2);
    VSMC_GMM_ATTR(4);
    VSMC_GMM_ATTR(8);
    VSMC_GMM_ATTR(16);
#undef VSMC_GMM_ATTR
}

bool is_residual(int s)
{
    return s == VSMC_CUDA_RESIDUAL || s == VSMC_CUDA_RESIDUAL_STRATIFIED ||
           s == VSMC_CUDA_RESIDUAL_SYSTEMATIC;
}

bool is_sys(int s)
{
    return s == VSMC_CUDA_SYSTEMATIC || s == VSMC_CUDA_RESIDUAL_SYSTEMATIC;
}

// alpha_prior<Power>::alpha_iter + gmm_state::alpha (move_alpha.hpp:
// 124-140, gmm_state.hpp:159-168)
double alpha_at(uint64_t t, uint64_t iters, int power)
{
    const double b = (double)t / (double)iters;
    double a = 1;
    for (int p = 0; p != power; ++p)
        a *= b;
    a = a < 1 ? a : 1;
    a = a > 0 ? a : 0;
    return a;
}

// Picks the lanes per particle with the fastest MCMC sweep on the current
// particles (CUDA events, best of 3 per candidate).  The trial sweeps write
// into the spare parameter buffer and a copy of the engine positions, so
// the sampler's state is untouched; and the choice changes no result, the
// likelihood's summation order not depending on it.  The proposal and
// acceptance work is repeated in every lane of a group, so the fastest G
// balances it against the split data loop.
int autotune_group(vsmc_cuda_gmm *g)
{
    GmmArgs a = gmm_args(g, g->cur, 1 - g->cur);
    a.words = reinterpret_cast<uint64_t *>(g->scratch);
    a.sweeps = 1;
    cudaMemcpyAsync(a.words, g->words, g->cfg.N * 8, cudaMemcpyDeviceToDevice,
                    g->stream);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int cand[5] = {1, 2, 4, 8, 16};
    int best = 4;
    float best_ms = 1e30f;
    for (int c = 0; c < 5; ++c) {
        const unsigned grid = (unsigned)gmm_ntiles_mcmc(a.N, cand[c]);
        float ms_min = 1e30f;
        for (int r = 0; r < 3; ++r) {
            cudaEventRecord(e0, g->stream);
            if (gmm_f32(g))
                launch_mcmc_t<true>(g, a, cand[c], grid);
            else
                launch_mcmc_t<false>(g, a, cand[c], grid);
            cudaEventRecord(e1, g->stream);
            cudaEventSynchronize(e1);
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, e0, e1);
            ms_min = ms < ms_min ? ms : ms_min;
            g->launches++;
        }
        if (ms_min < best_ms) {
            best_ms = ms_min;
            best = cand[c];
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return best;
}

} // namespace

extern "C" {

void vsmc_cuda_gmm_config_default(vsmc_cuda_gmm_config *c)
{
    if (c == nullptr)
        return;
    std::memset(c, 0, sizeof(*c));
    c->N = 1 << 16;
    c->iters = 100;
    c->power = 4;
    c->sweeps = 5;
    c->sd = 0.1;
    c->scheme = VSMC_CUDA_SYSTEMATIC;
    c->threshold = 0.5;
    c->seed = 101;
    c->form = VSMC_CUDA_FP64;
    c->group = 0;
}

int vsmc_cuda_gmm_create(const vsmc_cuda_gmm_config *cfg, const double *data,
                         uint64_t n, void *stream, vsmc_cuda_gmm **out)
{
    if (out == nullptr || cfg == nullptr || data == nullptr || n < 1 ||
        n > (uint64_t)kGmmMaxData || cfg->N < 2 || cfg->N > (1ull << 28) ||
        cfg->iters < 1 || cfg->iters > (1ull << 24) || cfg->power < 1 ||
        cfg->power > 16 || cfg->sweeps < 0 || cfg->sweeps > kGmmMaxSweeps ||
        !(cfg->sd > 0.0) || cfg->scheme < 0 || cfg->scheme > 5 ||
        !(cfg->threshold >= 0.0) ||
        (cfg->form != VSMC_CUDA_FP64 && cfg->form != VSMC_CUDA_MIXED) ||
        !(cfg->group == 0 || cfg->group == 1 || cfg->group == 2 ||
          cfg->group == 4 || cfg->group == 8 || cfg->group == 16)) {
        set_last_error("vsmc_cuda_gmm_create: invalid configuration");
        return VSMC_CUDA_EINVAL;
    }
    *out = nullptr;
    vsmc_cuda_gmm *g = new (std::nothrow) vsmc_cuda_gmm();
    if (g == nullptr)
        return VSMC_CUDA_ENOMEM;
    g->cfg = *cfg;
    g->stream = static_cast<cudaStream_t>(stream);
    g->n = (int)n;
    const size_t N = cfg->N, T = cfg->iters + 1;
    const size_t nt = (N + kTile - 1) / kTile;
    const size_t ntm = (size_t)gmm_ntiles_mcmc((long long)N, 16);
    const size_t nacc = 1 + 3 * (size_t)cfg->sweeps;
    size_t b = 0;
    b += 2 * align256(N * 8 * kGmmParamArrays);
    b += 3 * align256(N * 8) + align256(N * 4);
    b += align256(sizeof(FilterCtl)) + align256(sizeof(GmmCtl));
    b += align256(nt * sizeof(TileStats));
    b += align256(ntm * kGmmMaxAcc * 8);
    b += align256(n * 8) + align256(n * 4);
    b += 6 * align256(T * 8) + align256(T * 4) + align256(T * nacc * 8);
    b += resample_workspace_bytes((long long)N);
    g->bytes = b;
    cudaError_t e = cudaMalloc(&g->mem, b);
    if (e != cudaSuccess) {
        cudaGetLastError();
        delete g;
        set_last_error("vsmc_cuda_gmm_create: cudaMalloc failed");
        return VSMC_CUDA_ENOMEM;
    }
    char *p = g->mem;
    for (int k = 0; k < 2; ++k) {
        g->buf[k].base = reinterpret_cast<double *>(p);
        p += align256(N * 8 * kGmmParamArrays);
    }
    g->lw = reinterpret_cast<double *>(p);
    p += align256(N * 8);
    g->scratch = reinterpret_cast<double *>(p);
    p += align256(N * 8);
    g->words = reinterpret_cast<uint64_t *>(p);
    p += align256(N * 8);
    g->copy_from = reinterpret_cast<int32_t *>(p);
    p += align256(N * 4);
    g->ctl = reinterpret_cast<FilterCtl *>(p);
    p += align256(sizeof(FilterCtl));
    g->gctl = reinterpret_cast<GmmCtl *>(p);
    p += align256(sizeof(GmmCtl));
    g->tile_stats = reinterpret_cast<TileStats *>(p);
    p += align256(nt * sizeof(TileStats));
    g->tile_acc = reinterpret_cast<long long *>(p);
    p += align256(ntm * kGmmMaxAcc * 8);
    g->data64 = reinterpret_cast<double *>(p);
    p += align256(n * 8);
    g->data32 = reinterpret_cast<float *>(p);
    p += align256(n * 4);
    g->hist_ess = reinterpret_cast<double *>(p);
    p += align256(T * 8);
    g->hist_zinc = reinterpret_cast<double *>(p);
    p += align256(T * 8);
    g->hist_integrand = reinterpret_cast<double *>(p);
    p += align256(T * 8);
    g->hist_grid = reinterpret_cast<double *>(p);
    p += align256(T * 8);
    g->hist_mx = reinterpret_cast<double *>(p);
    p += align256(T * 8);
    g->hist_my = reinterpret_cast<double *>(p);
    p += align256(T * 8);
    g->hist_resampled = reinterpret_cast<int32_t *>(p);
    p += align256(T * 4);
    g->hist_accept = reinterpret_cast<int64_t *>(p);
    p += align256(T * nacc * 8);
    g->rws = carve_workspace(p, (long long)N);
    g->ntiles = (long long)nt;
    g->cur = 0;
    g->iter = 0;
    g->alpha = 0.0;
    g->timing = false;
    g->ev_used = 0;
    g->launches = 0;
    g->group = cfg->group == 0 ? 4 : cfg->group;
    // gmm_state::read_data (gmm_state.hpp:118-157)
    double xmax = data[0], xmin = data[0];
    for (uint64_t i = 0; i != n; ++i) {
        if (data[i] > xmax)
            xmax = data[i];
        if (data[i] < xmin)
            xmin = data[i];
    }
    const double kappa = 1 / ((xmax - xmin) * (xmax - xmin));
    g->mu0 = 0.5 * (xmin + xmax);
    g->sd0 = 1 / std::sqrt(kappa);
    g->shape0 = 2;
    g->scale0 = 50 * kappa;
    // Seed::set(seed); the RngSet takes N gets, the resample engine one more
    g->seed_base = (uint32_t)(cfg->seed % 0xFFFFFFFFu);
    std::memset(&g->eng, 0, sizeof(g->eng));
    g->eng.key.v[0] =
        (uint32_t)(((uint64_t)g->seed_base + N) % 0xFFFFFFFFull) + 1u;
    std::vector<float> f(data, data + n);
    e = cudaMemsetAsync(g->mem, 0, b, g->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(g->data64, data, n * 8, cudaMemcpyHostToDevice,
                            g->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(g->data32, f.data(), n * 4,
                            cudaMemcpyHostToDevice, g->stream);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(g->stream);
    if (e != cudaSuccess) {
        cudaFree(g->mem);
        delete g;
        return cuda_status(e, "vsmc_cuda_gmm_create");
    }
    set_smem_attrs<true>((size_t)n * 4);
    set_smem_attrs<false>((size_t)n * 8);
    cudaFuncSetAttribute(k_cv_finalize,
                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                         kFinalSmemTiles * (int)sizeof(double));
    *out = g;
    return VSMC_CUDA_OK;
}

int vsmc_cuda_gmm_destroy(vsmc_cuda_gmm *g)
{
    if (g == nullptr)
        return VSMC_CUDA_OK;
    cudaStreamSynchronize(g->stream);
    for (cudaEvent_t ev : g->ev)
        cudaEventDestroy(ev);
    cudaError_t e = cudaFree(g->mem);
    delete g;
    return e == cudaSuccess ? VSMC_CUDA_OK
                            : cuda_status(e, "vsmc_cuda_gmm_destroy");
}

int vsmc_cuda_gmm_initialize(vsmc_cuda_gmm *g)
{
    if (g == nullptr)
        return VSMC_CUDA_EINVAL;
    const long long N = (long long)g->cfg.N;
    // do_reset: equal weights (the resample engine and the particles'
    // engines keep their positions, as the reference's Particle does)
    FilterCtl h;
    std::memset(&h, 0, sizeof(h));
    h.lw_max = 0.0;
    h.s1 = (double)N;
    h.s2 = (double)N;
    h.ess = (double)N;
    h.monitor_done = -1;
    const double ess = (double)N, dz = 0.0;
    const int32_t zero = 0;
    cudaError_t e = cudaMemcpyAsync(g->ctl, &h, sizeof(h),
                                    cudaMemcpyHostToDevice, g->stream);
    // t = 0: ESS N, no resampling (weights equal), no evidence increment
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(g->hist_ess, &ess, 8, cudaMemcpyHostToDevice,
                            g->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(g->hist_zinc, &dz, 8, cudaMemcpyHostToDevice,
                            g->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(g->hist_resampled, &zero, 4,
                            cudaMemcpyHostToDevice, g->stream);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(g->stream); // the host values above
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_gmm_initialize");
    g->cur = 0;
    g->alpha = 0.0;
    g->group = g->cfg.group == 0 ? 4 : g->cfg.group;
    GmmArgs a = gmm_args(g, 0, 0);
    const unsigned grid = (unsigned)gmm_ntiles_mcmc(N, g->group);
    if (gmm_f32(g))
        launch_init_t<true>(g, a, g->group, grid);
    else
        launch_init_t<false>(g, a, g->group, grid);
    k_gmm_path<<<1, 1024, 0, g->stream>>>(
        g->tile_acc, grid, 3 * g->cfg.sweeps, g->buf[0].base + 13 * N, g->lw,
        g->ctl, N, 0, 0.0, g->gctl, g->hist_accept, g->hist_integrand,
        g->hist_grid);
    g->launches += 2;
    e = cudaGetLastError();
    if (e == cudaSuccess && g->cfg.group == 0)
        g->group = autotune_group(g);
    g->iter = 1;
    if (e == cudaSuccess)
        e = cudaGetLastError();
    return e == cudaSuccess ? VSMC_CUDA_OK
                            : cuda_status(e, "vsmc_cuda_gmm_initialize");
}

int vsmc_cuda_gmm_iterate(vsmc_cuda_gmm *g, uint64_t num)
{
    if (g == nullptr || g->iter == 0) {
        set_last_error("vsmc_cuda_gmm_iterate: initialize first");
        return VSMC_CUDA_EINVAL;
    }
    if (g->iter + num > g->cfg.iters + 1) {
        set_last_error("vsmc_cuda_gmm_iterate: beyond the schedule");
        return VSMC_CUDA_EINVAL;
    }
    const long long N = (long long)g->cfg.N;
    cudaStream_t s = g->stream;
    const int scheme = g->cfg.scheme;
    for (uint64_t k = 0; k < num; ++k) {
        const uint64_t t = g->iter;
        const double a = alpha_at(t, g->cfg.iters, g->cfg.power);
        const double a_inc = a > 0 ? a - g->alpha : 0;
        g->alpha = a;
        k_gmm_reweight<<<(unsigned)g->ntiles, kThreads, 0, s>>>(
            g->buf[g->cur].base + 13 * N, g->lw, g->ctl, N, a_inc,
            g->tile_stats);
        FinalizeArgs fa;
        fa.ctl = g->ctl;
        fa.ts = g->tile_stats;
        fa.ntiles = (int)g->ntiles;
        fa.N = N;
        fa.threshold = g->cfg.threshold;
        fa.t = (long long)t;
        fa.init = 0;
        fa.anchored = 0;
        fa.obs_x = g->hist_mx; // not read (anchored is 0)
        fa.obs_y = g->hist_my;
        fa.hist_ess = g->hist_ess;
        fa.hist_resampled = g->hist_resampled;
        fa.hist_logz_inc = g->hist_zinc;
        fa.hist_mean_x = g->hist_mx;
        fa.hist_mean_y = g->hist_my;
        fa.rctl = g->rws.ctl;
        fa.tile_excl = g->rws.tile_excl;
        fa.residual = is_residual(scheme);
        fa.sys = is_sys(scheme);
        fa.eng = g->eng;
        fa.replay_flags = nullptr;
        fa.compare = 0;
        const size_t fin_smem = g->ntiles <= kFinalSmemTiles
                                    ? (size_t)g->ntiles * sizeof(double)
                                    : 0;
        k_cv_finalize<<<1, kFinalThreads, fin_smem, s>>>(fa);
        WeightsFromLog<double> w;
        w.lw = g->lw;
        w.stats = &g->ctl->lw_max;
        launch_resample_core(scheme, w, N, g->eng, g->rws, nullptr, 0,
                             /*spine_done=*/true, nullptr, g->copy_from, s);
        cudaEvent_t *ev = nullptr;
        if (g->timing) {
            if (g->ev_used + 2 > g->ev.size())
                for (int q = 0; q < 128; ++q) {
                    cudaEvent_t x;
                    cudaEventCreate(&x);
                    g->ev.push_back(x);
                }
            ev = &g->ev[g->ev_used];
            g->ev_used += 2;
            cudaEventRecord(ev[0], s);
        }
        GmmArgs ga = gmm_args(g, g->cur, 1 - g->cur);
        const unsigned grid = (unsigned)gmm_ntiles_mcmc(N, g->group);
        if (gmm_f32(g))
            launch_mcmc_t<true>(g, ga, g->group, grid);
        else
            launch_mcmc_t<false>(g, ga, g->group, grid);
        if (ev)
            cudaEventRecord(ev[1], s);
        k_gmm_path<<<1, 1024, 0, s>>>(
            g->tile_acc, grid, 3 * g->cfg.sweeps,
            g->buf[1 - g->cur].base + 13 * N, g->lw, g->ctl, N, (long long)t,
            a, g->gctl, g->hist_accept, g->hist_integrand, g->hist_grid);
        g->cur = 1 - g->cur;
        g->launches += 4 + resample_launches(scheme, false, true);
        ++g->iter;
    }
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? VSMC_CUDA_OK
                            : cuda_status(e, "vsmc_cuda_gmm_iterate");
}

int vsmc_cuda_gmm_iter_size(vsmc_cuda_gmm *g, uint64_t *n)
{
    if (g == nullptr || n == nullptr)
        return VSMC_CUDA_EINVAL;
    *n = g->iter;
    return VSMC_CUDA_OK;
}

int vsmc_cuda_gmm_history(vsmc_cuda_gmm *g, double *ess, int32_t *resampled,
                          double *zinc, double *integrand, double *grid,
                          int64_t *accept)
{
    if (g == nullptr)
        return VSMC_CUDA_EINVAL;
    const uint64_t T = g->iter;
    const size_t nacc = 1 + 3 * (size_t)g->cfg.sweeps;
    cudaError_t e = cudaStreamSynchronize(g->stream);
    auto get = [&](void *dst, const void *src, size_t bytes) {
        if (dst != nullptr && e == cudaSuccess && bytes > 0)
            e = cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost);
    };
    get(ess, g->hist_ess, T * 8);
    get(resampled, g->hist_resampled, T * 4);
    get(zinc, g->hist_zinc, T * 8);
    get(integrand, g->hist_integrand, T * 8);
    get(grid, g->hist_grid, T * 8);
    get(accept, g->hist_accept, T * nacc * 8);
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_gmm_history");
    FilterCtl h;
    e = cudaMemcpy(&h, g->ctl, sizeof(h), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_gmm_history");
    if (h.error != 0) {
        set_last_error("vsmc_cuda_gmm: degenerate weights");
        return h.error;
    }
    return VSMC_CUDA_OK;
}

int vsmc_cuda_gmm_log_evidence(vsmc_cuda_gmm *g, double *smc, double *path)
{
    if (g == nullptr)
        return VSMC_CUDA_EINVAL;
    cudaError_t e = cudaStreamSynchronize(g->stream);
    FilterCtl h;
    GmmCtl gc;
    if (e == cudaSuccess)
        e = cudaMemcpy(&h, g->ctl, sizeof(h), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess)
        e = cudaMemcpy(&gc, g->gctl, sizeof(gc), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_gmm_log_evidence");
    const double llc = -0.5 * (double)g->n * kLnPi2;
    if (smc)
        *smc = h.logz + llc;
    if (path)
        *path = gc.path_logz + llc;
    return VSMC_CUDA_OK;
}

int vsmc_cuda_gmm_read_params(vsmc_cuda_gmm *g, double *params, double *lw,
                              uint64_t *words)
{
    if (g == nullptr)
        return VSMC_CUDA_EINVAL;
    const size_t N = g->cfg.N;
    cudaError_t e = cudaStreamSynchronize(g->stream);
    if (params != nullptr && e == cudaSuccess) {
        std::vector<double> soa(N * kGmmParamArrays);
        e = cudaMemcpy(soa.data(), g->buf[g->cur].base, soa.size() * 8,
                       cudaMemcpyDeviceToHost);
        for (size_t i = 0; i < N && e == cudaSuccess; ++i)
            for (int k = 0; k < kGmmParamArrays; ++k)
                params[i * kGmmParamArrays + k] = soa[k * N + i];
    }
    if (lw != nullptr && e == cudaSuccess) {
        // the reference stores max-normalised log-weights (0 after
        // resampling)
        FilterCtl h;
        e = cudaMemcpy(&h, g->ctl, sizeof(h), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess)
            e = cudaMemcpy(lw, g->lw, N * 8, cudaMemcpyDeviceToHost);
        for (size_t i = 0; i < N && e == cudaSuccess; ++i)
            lw[i] = h.resampled ? 0.0 : lw[i] - h.lw_max;
    }
    if (words != nullptr && e == cudaSuccess)
        e = cudaMemcpy(words, g->words, N * 8, cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? VSMC_CUDA_OK
                            : cuda_status(e, "vsmc_cuda_gmm_read_params");
}

int vsmc_cuda_gmm_loglik(vsmc_cuda_gmm *g, int form, double *out)
{
    if (g == nullptr || out == nullptr ||
        (form != VSMC_CUDA_FP64 && form != VSMC_CUDA_MIXED))
        return VSMC_CUDA_EINVAL;
    // the likelihood of the current particles in `form`, whatever the
    // sampler's own form
    GmmArgs a = gmm_args(g, g->cur, g->cur);
    if (form == VSMC_CUDA_MIXED) {
        a.data = g->data32;
        launch_loglik_t<true>(g, a, g->group, g->scratch);
    } else {
        a.data = g->data64;
        launch_loglik_t<false>(g, a, g->group, g->scratch);
    }
    cudaError_t e = cudaMemcpyAsync(out, g->scratch, g->cfg.N * 8,
                                    cudaMemcpyDeviceToHost, g->stream);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(g->stream);
    g->launches++;
    return e == cudaSuccess ? VSMC_CUDA_OK
                            : cuda_status(e, "vsmc_cuda_gmm_loglik");
}

int vsmc_cuda_gmm_group(vsmc_cuda_gmm *g, int *group)
{
    if (g == nullptr || group == nullptr)
        return VSMC_CUDA_EINVAL;
    *group = g->group;
    return VSMC_CUDA_OK;
}

int vsmc_cuda_gmm_set_timing(vsmc_cuda_gmm *g, int enable)
{
    if (g == nullptr)
        return VSMC_CUDA_EINVAL;
    g->timing = enable != 0;
    g->ev_used = 0;
    return VSMC_CUDA_OK;
}

int vsmc_cuda_gmm_timing(vsmc_cuda_gmm *g, double *mcmc_ms, uint64_t *steps,
                         uint64_t *launches)
{
    if (g == nullptr)
        return VSMC_CUDA_EINVAL;
    cudaError_t e = cudaStreamSynchronize(g->stream);
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_gmm_timing");
    double tot = 0.0;
    for (size_t k = 0; k + 1 < g->ev_used; k += 2) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, g->ev[k], g->ev[k + 1]);
        tot += ms;
    }
    if (mcmc_ms)
        *mcmc_ms = tot;
    if (steps)
        *steps = g->ev_used / 2;
    if (launches)
        *launches = g->launches;
    return VSMC_CUDA_OK;
}

} // extern "C"
