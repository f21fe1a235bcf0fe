// resample.cuh -- the six vSMC resampling schemes on the device.
//
// Reference: include/vsmc/resample/{multinomial,residual,stratified,
// systematic,residual_stratified,residual_systematic}.hpp, internal::inversion
// and internal::cfrp_trans (resample/common.hpp:57-118), the U01 sequences of
// include/vsmc/rng/u01.hpp:165-287 and Particle::resample
// (core/particle.hpp:230-250).
//
// Pipeline for N particles in tiles of kTile:
//   (residual only) tile sums of r = modf(N w) and of floor(N w)
//   spine      one CTA: deterministic exclusive prefix of the tile sums
//   uniforms   U01 sequence u_0..u_{NN-1} (not for Systematic: closed form)
//   invert     per tile: FP64 scan of the weights anchored on the spine,
//              count of uniforms <= C_i, replication, zero-slot ranks by an
//              integer decoupled look-back, copy_from for survivors and the
//              inclusive surplus-children count
//   fill       zero slots find their parent by a galloping search
// Every FP64 sum is formed in a fixed order (no float atomics, no look-back
// on floats), so results are reproducible run to run.
#pragma once

#include "smc_common.cuh"
#include "exact_scan.cuh"

namespace vsmc_b200 {

// Device-side control block of one resampling call.
struct ResampleCtl {
    int active;           // 0: every resample kernel returns at once
    int error;            // sticky vsmc_cuda_status
    long long NN;         // length of the U01 sequence fed to inversion
    double coeff_r;       // 1 / sum of residuals (exact once the residuals'
                          // sequential sum is known)
    double coeff_r_apx;   // 1 / the spine's sum of residuals
    double coeff_w;       // 1 / the weights' sequential sum (filters)
    double delta;         // 1 / NN
    double u0;            // systematic start
    long long n_final;    // uniforms consumed by particles 0..N-2
    unsigned long long words;   // engine words drawn by this call
    unsigned long long offset;  // engine offset before the call
    int kbits;            // bin index: K = 2^kbits bins over [0, 1)
    unsigned long long spec_offset; // engine offset the held speculative
                                    // sorted sequence was drawn at (~0: none)
    long long Nout; // children in total when it differs from the number of
                    // weights (Resample(M, N) with M != N); 0: the same
};

// The number of children of a resampling of N weights (ctl->Nout when the
// caller asked for M != N).
__device__ __forceinline__ long long resample_children(const ResampleCtl *ctl,
                                                      long long N)
{
    return ctl->Nout > 0 ? ctl->Nout : N;
}

struct EngineRef {
    u64x4 key;
    u64x4 ctr;
};

// Bin index of a non-decreasing U01 sequence u_0..u_{NN-1}:
// L[k] = #{n : u_n < k/K} for k = 0..K (K = 2^kbits, about NN/8), so the
// count of u_n <= C for C in [k/K, (k+1)/K) lies in [L[k], L[k+1]].  Each
// n writes the bins k with u_{n-1} < k/K <= u_n (k/K and u*K are exact), so
// every bin is written exactly once; the owner of the last n also closes the
// bins above u_{NN-1}.
__device__ __forceinline__ int bin_kbits(long long NN)
{
    int kb = 0;
    while (kb < 40 && (2ll << kb) <= NN / 8)
        ++kb;
    return kb;
}

__device__ __forceinline__ long long bin_floor(double u, int kb)
{
    // floor(u * K) clamped to [-1, K]; K = 2^kb, so u * K is exact
    const double K = (double)(1ll << kb);
    const double v = __dmul_rn(u, K);
    if (!(v >= 0.0))
        return -1;
    return v >= K ? (1ll << kb) : (long long)v;
}

// Bins (klo - 1, khi] start at u_n: klo - 1 = bin_floor(u_{n-1}) (0 for
// n = 0), khi = bin_floor(u_n); callers carry khi on to the next n.
__device__ __forceinline__ void bin_fill(int32_t *L, int kb, long long klo,
                                         long long khi, long long n,
                                         long long NN)
{
    const long long K = 1ll << kb;
    // k/K <= u  <=>  k <= floor(u K)
    for (long long k = klo; k <= khi && k <= K; ++k)
        L[k] = (int32_t)n;
    if (n == NN - 1)
        for (long long k = max(khi + 1, 0ll); k <= K; ++k)
            L[k] = (int32_t)NN;
}

// Window of the count of u_n <= C from the bin index.
__device__ __forceinline__ void bin_window(const int32_t *L, int kb,
                                           long long NN, double C,
                                           long long &lo, long long &hi)
{
    const long long K = 1ll << kb;
    long long k = bin_floor(C, kb);
    if (k < 0) {
        lo = 0;
        hi = L[0];
        return;
    }
    if (k >= K) {
        lo = L[K];
        hi = NN;
        return;
    }
    lo = L[k];
    hi = L[k + 1];
}

constexpr int resample_ntiles(long long N)
{
    return (int)((N + kTile - 1) / kTile);
}

// Weight sources --------------------------------------------------------
// Normalised weights given in memory (generic C ABI).
struct WeightsGiven {
    static constexpr bool kExactNorm = false;
    static constexpr bool kApprox = false;
    typedef double stage_t; // the per-element value a kernel stages
    const double *w;
    __device__ __forceinline__ const double *stage_src() const { return w; }
    __device__ __forceinline__ double from_stage(double x) const { return x; }
    __device__ __forceinline__ double unnorm_stage(double x) const
    {
        return x;
    }
    __device__ __forceinline__ void prepare() {}
    __device__ __forceinline__ double operator()(long long i) const
    {
        return w[i];
    }
    __device__ __forceinline__ double unnorm(long long i) const
    {
        return w[i];
    }
    // the approximate spine's scale relative to these weights'
    __device__ __forceinline__ double spine_ratio() const { return 1.0; }
    __device__ __forceinline__ double spine_unnorm() const { return 1.0; }
    // whether the resampling runs, and the scanned length
    __device__ __forceinline__ bool active(const ResampleCtl *ctl) const
    {
        return ctl->active != 0;
    }
    __device__ __forceinline__ long long length(const ResampleCtl *,
                                                long long N) const
    {
        return N;
    }
};

// Weights of a filter: w_i = exp(lw_i - M) * coeff, i.e. the reference's
// normalize_log_weight, vExp and normalize_weight (core/weight_set.hpp:
// 108-125) evaluated on the fly from raw log-weights.  coeff is 1 / S1 from
// the tile statistics, or (FP64, `coeff_exact` set) 1 / the sequential sum
// of exp(lw_i - M) in index order, the reference's `1 / math::asum`
// (weight_set.hpp:121, math/cblas.hpp:54-63), so that the weights are the
// reference's bit for bit where exp agrees.
template <typename Real>
struct WeightsFromLog {
    static constexpr bool kExactNorm = sizeof(Real) == sizeof(double);
    // The mixed form's weights are not the reference's bit for bit (float
    // log-weights), so the reference's sequential cumulative sum has nothing
    // to reproduce there: its cumulative weight is a plain FP64 scan
    // (approx_tile_compute / approx_spine).
    static constexpr bool kApprox = sizeof(Real) == sizeof(float);
    typedef Real stage_t; // lw, or (FP64, raw set) the kept exp(lw - M)
    const Real *lw;
    const double *stats;       // [0] = M (max log-weight), [1] = S1
    const double *coeff_exact = nullptr; // the sequential sum's reciprocal
    const double *raw = nullptr; // exp(lw_i - M), kept by that pass
    double M, coeff, coeff_apx;
    __device__ __forceinline__ void prepare()
    {
        M = stats[0];
        coeff_apx = __ddiv_rn(1.0, stats[1]);
        coeff = coeff_exact != nullptr ? *coeff_exact : coeff_apx;
    }
    __device__ __forceinline__ double operator()(long long i) const;
    __device__ __forceinline__ double unnorm(long long i) const;
    __device__ __forceinline__ const Real *stage_src() const;
    __device__ __forceinline__ double unnorm_stage(Real x) const;
    __device__ __forceinline__ double from_stage(Real x) const
    {
        return __dmul_rn(unnorm_stage(x), coeff);
    }
    // the approximate spine (tile statistics scaled by coeff_apx) relative
    // to these weights' scale, and to the unnormalised weights'
    __device__ __forceinline__ double spine_ratio() const
    {
        return coeff_exact != nullptr ? __ddiv_rn(coeff, coeff_apx) : 1.0;
    }
    __device__ __forceinline__ double spine_unnorm() const
    {
        return stats[1];
    }
    __device__ __forceinline__ bool active(const ResampleCtl *ctl) const
    {
        return ctl->active != 0;
    }
    __device__ __forceinline__ long long length(const ResampleCtl *,
                                                long long N) const
    {
        return N;
    }
};

template <>
__device__ __forceinline__ double
WeightsFromLog<double>::unnorm(long long i) const
{
    return raw != nullptr ? raw[i] : fm::fm_exp(__dadd_rn(lw[i], -M));
}

template <>
__device__ __forceinline__ double
WeightsFromLog<double>::operator()(long long i) const
{
    return __dmul_rn(unnorm(i), coeff);
}

template <>
__device__ __forceinline__ const double *
WeightsFromLog<double>::stage_src() const
{
    return raw != nullptr ? raw : lw;
}

template <>
__device__ __forceinline__ double
WeightsFromLog<double>::unnorm_stage(double x) const
{
    return raw != nullptr ? x : fm::fm_exp(__dadd_rn(x, -M));
}

template <>
__device__ __forceinline__ const float *
WeightsFromLog<float>::stage_src() const
{
    return lw;
}

template <>
__device__ __forceinline__ double
WeightsFromLog<float>::unnorm_stage(float x) const
{
    return static_cast<double>(expf(x - static_cast<float>(M)));
}

template <>
__device__ __forceinline__ double
WeightsFromLog<float>::unnorm(long long i) const
{
    return static_cast<double>(expf(lw[i] - static_cast<float>(M)));
}

// The sorted U01 sequence's negated terms -log(1 - U_n) / (NN - n) >= 0,
// which pass 1 stores in u[]: their exact sequential sum is the reference's
// -lmax_n (u01.hpp:185-186).  spec_N > 0: the speculative Multinomial
// sequence of spec_N uniforms (sorted_run).
struct TermsNeg {
    static constexpr bool kExactNorm = false;
    static constexpr bool kApprox = false;
    typedef double stage_t;
    const double *u;
    long long spec_N;
    __device__ __forceinline__ const double *stage_src() const { return u; }
    __device__ __forceinline__ double from_stage(double x) const { return -x; }
    __device__ __forceinline__ double unnorm_stage(double x) const
    {
        return -x;
    }
    __device__ __forceinline__ void prepare() {}
    __device__ __forceinline__ double operator()(long long i) const
    {
        return -u[i];
    }
    __device__ __forceinline__ double unnorm(long long i) const
    {
        return -u[i];
    }
    // the spine of the sorted sequence sums the terms themselves
    __device__ __forceinline__ double spine_ratio() const { return -1.0; }
    __device__ __forceinline__ double spine_unnorm() const { return -1.0; }
    __device__ __forceinline__ bool active(const ResampleCtl *ctl) const
    {
        return spec_N > 0 ? ctl->spec_offset != ctl->offset
                          : ctl->active != 0;
    }
    __device__ __forceinline__ long long length(const ResampleCtl *ctl,
                                                long long) const
    {
        return spec_N > 0 ? spec_N : ctl->NN;
    }
};

// The weight source with the exact normalisation coefficient (held in the
// control block once the normalisation pass has run) and the unnormalised
// weights that pass kept, where it has them.
template <typename W>
__host__ __device__ inline W with_exact_coeff(W w, const double *,
                                              const double *)
{
    return w;
}
template <>
__host__ __device__ inline WeightsFromLog<double>
with_exact_coeff(WeightsFromLog<double> w, const double *c, const double *raw)
{
    w.coeff_exact = c;
    w.raw = raw;
    return w;
}

template <>
__device__ __forceinline__ double
WeightsFromLog<float>::operator()(long long i) const
{
    return __dmul_rn(static_cast<double>(expf(lw[i] - static_cast<float>(M))),
                     coeff);
}

// Relative error margin of the approximate cumulative weights the exact
// scan classifies with (its spine comes from the weights' tile sums): FP64
// weights carry a few ulps.
template <typename W>
struct ExactMargin {
    static constexpr double rel = 0x1p-44;
};

// Residual split of a weight: r = modf(N w, &k) (residual.hpp:61-62).
__device__ __forceinline__ double residual_split(double w, double Nd,
                                                 double &k)
{
    return modf(__dmul_rn(Nd, w), &k);
}

// The latency-bound per-tile kernels of the sorted sequence and the cfrp
// fill are compiled for eight CTAs per SM (32 registers): more warps in
// flight hide their dependent loads.
#ifndef VSMC_SCAN_MIN_BLOCKS
#define VSMC_SCAN_MIN_BLOCKS 8
#endif
#define VSMC_SCAN_BOUNDS kThreads, VSMC_SCAN_MIN_BLOCKS

// Shared memory of each per-tile body (the __global__ wrappers declare one;
// a caller that runs several bodies in one CTA can overlay them).
struct SmemTileSums {
    double shd[kThreads / 32];
    long long shk[kThreads / 32];
};
struct SmemSpine {
    double shd[kSpineThreads / 32];
    long long shk[kSpineThreads / 32];
    double coeff;
};
struct SmemNone {
    int unused;
};
struct SmemSortedSums {
    double sh[kThreads / 32];
};
struct SmemSortedUniforms {
    double sh[kThreads / 32];
    double shm[kThreads];
    int shi[kThreads / 32];
    double sv[kExactCap]; // exact -lmax at the tile's specials
};
// Uniforms staged in shared memory per tile: twice the expected count, so
// that only a tile holding more than twice its share searches global memory.
constexpr int kUStage = 2 * kTile;

// Asynchronous 8-byte global-to-shared copies (cp.async): the tile's
// uniforms travel while the threads work on their records.
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa),
                 "l"(gmem)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit()
{
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all()
{
    asm volatile("cp.async.wait_all;\n" ::: "memory");
}

template <bool Residual>
struct SmemInvert {
    double sw[kUStage];               // uniforms, then the outputs
    long long shl[kThreads / 32];
    long long bound[2];
    long long last[kThreads / 32];
    // the exact S at the tile's specials (exact_scan.cuh)
    double sv[kExactCap];
};

// ---------------------------------------------------------------------------
// Tile sums of the weights (or, residual, of r and k).
template <typename W, bool Residual>
__device__ __forceinline__ void
k_tile_sums_body(W wsrc, long long N, const ResampleCtl *ctl, double *tile_sum,
                 long long *tile_k, int bid, SmemTileSums &sm)
{
    if (!ctl->active)
        return;
    double *shd = sm.shd;
    long long *shk = sm.shk;
    wsrc.prepare();
    const long long base = (long long)bid * kTile;
    const double Nd = (double)resample_children(ctl, N);
    double s = 0.0;
    long long ks = 0;
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const long long i = base + (long long)j * kThreads + threadIdx.x;
        if (i < N) {
            const double w = wsrc(i);
            if (Residual) {
                double k;
                s += fabs(residual_split(w, Nd, k));
                ks += (long long)k;
            } else {
                s += w;
            }
        }
    }
    s = warp_sum(s);
    ks = warp_sum_ll(ks);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        shd[wid] = s;
        shk[wid] = ks;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        long long kt = 0;
        for (int w = 0; w < kThreads / 32; ++w) {
            t += shd[w];
            kt += shk[w];
        }
        tile_sum[bid] = t;
        if (Residual)
            tile_k[bid] = kt;
    }
}

template <typename W, bool Residual>
__global__ void __launch_bounds__(kThreads)
k_tile_sums(W wsrc, long long N, const ResampleCtl *ctl, double *tile_sum,
            long long *tile_k)
{
    __shared__ SmemTileSums sm;
    k_tile_sums_body<W, Residual>(wsrc, N, ctl, tile_sum, tile_k, blockIdx.x,
        sm);
}

// One CTA: exclusive prefix of `ntiles` doubles in a fixed association
// (contiguous runs per thread, then a block scan).  excl has ntiles + 1
// entries; excl[ntiles] is the total.  `scale` multiplies every input.
__device__ __forceinline__ void spine_scan_f64(const double *in, double *excl,
                                               int ntiles, double scale,
                                               double *sh)
{
    const int per = (ntiles + blockDim.x - 1) / blockDim.x;
    const int b = threadIdx.x * per;
    const int e = min(b + per, ntiles);
    double run = 0.0;
    double total;
    if (per <= 8) {
        // the run's loads issued together, then summed in order
        double x[8];
#pragma unroll
        for (int k = 0; k < 8; ++k)
            x[k] = b + k < e ? __dmul_rn(in[b + k], scale) : 0.0;
#pragma unroll
        for (int k = 0; k < 8; ++k)
            if (b + k < e)
                run += x[k];
        run = block_excl_scan(run, sh, total);
#pragma unroll
        for (int k = 0; k < 8; ++k)
            if (b + k < e) {
                excl[b + k] = run;
                run += x[k];
            }
    } else {
        for (int t = b; t < e; ++t)
            run += __dmul_rn(in[t], scale);
        const double off = block_excl_scan(run, sh, total);
        run = off;
        for (int t = b; t < e; ++t) {
            excl[t] = run;
            run += __dmul_rn(in[t], scale);
        }
    }
    if (threadIdx.x == blockDim.x - 1)
        excl[ntiles] = total;
}

__device__ __forceinline__ void spine_scan_ll(const long long *in,
                                              long long *excl, int ntiles,
                                              long long *sh)
{
    const int per = (ntiles + blockDim.x - 1) / blockDim.x;
    const int b = threadIdx.x * per;
    const int e = min(b + per, ntiles);
    long long run = 0;
    for (int t = b; t < e; ++t)
        run += in[t];
    long long total;
    const long long off = block_excl_scan(run, sh, total);
    run = off;
    for (int t = b; t < e; ++t) {
        excl[t] = run;
        run += in[t];
    }
    if (threadIdx.x == blockDim.x - 1)
        excl[ntiles] = total;
}

// Spine of the resampling weights plus the scheme set-up: NN, coeff_r, the
// systematic start u0 (one engine word, U01SequenceSystematic's constructor,
// u01.hpp:253-263) and the words drawn when they do not depend on the data.
template <bool Residual, bool Sys>
__device__ __forceinline__ void
k_spine_weights_body(const double *tile_sum, const long long *tile_k,
                     double *tile_excl, long long *tile_kexcl, int ntiles,
                     long long N, EngineRef eng, ResampleCtl *ctl, int bid,
                     SmemSpine &sm)
{
    if (!ctl->active)
        return;
    double *shd = sm.shd;
    long long *shk = sm.shk;
    double &coeff_sh = sm.coeff;
    long long NN = resample_children(ctl, N);
    double coeff = 1.0;
    if (Residual) {
        spine_scan_ll(tile_k, tile_kexcl, ntiles, shk);
        __syncthreads();
        // asum of the residuals in the spine's fixed order
        const int per = (ntiles + blockDim.x - 1) / blockDim.x;
        double run = 0.0;
        const int e = min((int)(threadIdx.x + 1) * per, ntiles);
        for (int t = threadIdx.x * per; t < e; ++t)
            run += tile_sum[t];
        double total;
        block_excl_scan(run, shd, total);
        if (threadIdx.x == 0)
            coeff_sh = __ddiv_rn(1.0, total);
        __syncthreads();
        coeff = coeff_sh;
        NN = resample_children(ctl, N) - tile_kexcl[ntiles];
    }
    spine_scan_f64(tile_sum, tile_excl, ntiles, coeff, shd);
    if (threadIdx.x == 0) {
        ctl->NN = NN;
        ctl->coeff_r = coeff;
        ctl->coeff_r_apx = coeff;
        ctl->delta = __ddiv_rn(1.0, (double)NN);
        ctl->kbits = bin_kbits(NN);
        ctl->n_final = 0;
        if (Sys) {
            const uint64_t w = threefry_word(eng.key, eng.ctr, ctl->offset);
            ctl->u0 = __dmul_rn(canonical_u64(w), ctl->delta);
            ctl->words = 1;
        } else {
            ctl->words = 0;
        }
    }
}

template <bool Residual, bool Sys>
__global__ void __launch_bounds__(kSpineThreads)
k_spine_weights(const double *tile_sum, const long long *tile_k,
                double *tile_excl, long long *tile_kexcl, int ntiles,
                long long N, EngineRef eng, ResampleCtl *ctl)
{
    __shared__ SmemSpine sm;
    k_spine_weights_body<Residual, Sys>(tile_sum, tile_k, tile_excl, tile_kexcl,
        ntiles, N, eng, ctl, blockIdx.x, sm);
}

// Words at stream positions pos0 .. pos0+7 of a Threefry4x64 engine (two or
// three block evaluations).
__device__ __forceinline__ void threefry_words8(const EngineRef &eng,
                                                unsigned long long pos0,
                                                uint64_t w[8])
{
    const unsigned long long b0 = pos0 / 4;
    const int s = (int)(pos0 % 4);
    const u64x4 x = threefry4x64_20(ctr64_add(eng.ctr, b0 + 1), eng.key);
    const u64x4 y = threefry4x64_20(ctr64_add(eng.ctr, b0 + 2), eng.key);
    u64x4 z;
    z.v[0] = z.v[1] = z.v[2] = z.v[3] = 0;
    if (s > 0)
        z = threefry4x64_20(ctr64_add(eng.ctr, b0 + 3), eng.key);
    const uint64_t q[12] = {x.v[0], x.v[1], x.v[2], x.v[3], y.v[0], y.v[1],
                            y.v[2], y.v[3], z.v[0], z.v[1], z.v[2], z.v[3]};
    // w[j] = q[s + j] with constant indices only (register selects)
#pragma unroll
    for (int j = 0; j < 8; ++j)
        w[j] = s == 0 ? q[j] : s == 1 ? q[j + 1] : s == 2 ? q[j + 2] : q[j + 3];
}

// Stratified U01 sequence (U01SequenceStratified, u01.hpp:212-243):
// u_n = U_n * delta + n * delta, U_n from engine word offset + n.  One
// Threefry block per thread gives four consecutive u_n.  Adjacent values can
// cross by rounding only between neighbours, so the running maximum is
// max(u_n, u_{n-1}); the neighbour of a thread's first value comes from the
// previous lane (lane 0 recomputes it).
__device__ __forceinline__ double strat_u(uint64_t w, long long n, double delta)
{
    return __dadd_rn(__dmul_rn(canonical_u64(w), delta),
                     __dmul_rn((double)n, delta));
}

__device__ __forceinline__ void
k_uniforms_stratified_body(EngineRef eng, const ResampleCtl *ctl, double *u,
                           int32_t *L, unsigned long long gid, SmemNone &sm)
{
    if (!ctl->active)
        return;
    const long long NN = ctl->NN;
    const double delta = ctl->delta;
    const int kb = ctl->kbits;
    const unsigned long long off = ctl->offset;
    const unsigned long long b =
        off / 4 + (unsigned long long)gid;
    const bool live = b * 4 < off + (unsigned long long)NN;
    double raw[4] = {-INFINITY, -INFINITY, -INFINITY, -INFINITY};
    if (live) {
        const u64x4 w = threefry4x64_20(ctr64_add(eng.ctr, b + 1), eng.key);
#pragma unroll
        for (int l = 0; l < 4; ++l) {
            const long long n = (long long)(b * 4 + l) - (long long)off;
            if (n >= 0 && n < NN)
                raw[l] = strat_u(w.v[l], n, delta);
        }
    }
    // raw values of n-1 and n-2 for the thread's first n
    double p1 = __shfl_up_sync(0xffffffffu, raw[3], 1);
    double p2 = __shfl_up_sync(0xffffffffu, raw[2], 1);
    if ((threadIdx.x & 31) == 0) {
        p1 = p2 = -INFINITY;
        const long long n = (long long)(b * 4) - (long long)off;
        if (live && n - 1 >= 0 && n - 1 < NN)
            p1 = strat_u(threefry_word(eng.key, eng.ctr, off + n - 1), n - 1,
                         delta);
        if (live && n - 2 >= 0 && n - 2 < NN)
            p2 = strat_u(threefry_word(eng.key, eng.ctr, off + n - 2), n - 2,
                         delta);
    }
    if (!live)
        return;
    // monotone sequence v_n = max(u_n, u_{n-1}); kprev = bin of v_{n-1}
    long long kprev = bin_floor(fmax(p1, p2), kb);
    double rprev = p1;
#pragma unroll
    for (int l = 0; l < 4; ++l) {
        const long long n = (long long)(b * 4 + l) - (long long)off;
        if (n >= 0 && n < NN) {
            const double v = fmax(raw[l], rprev);
            u[n] = v;
            const long long khi = bin_floor(v, kb);
            bin_fill(L, kb, n == 0 ? 0 : kprev + 1, khi, n, NN);
            kprev = khi;
        }
        rprev = raw[l];
    }
}

static __global__ void __launch_bounds__(kThreads)
k_uniforms_stratified(EngineRef eng, const ResampleCtl *ctl, double *u,
                      int32_t *L)
{
    __shared__ SmemNone sm;
    k_uniforms_stratified_body(eng, ctl, u, L,
        (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x, sm);
}

// Sorted U01 sequence (U01SequenceSorted, u01.hpp:165-202): lmax_n =
// sum_{k<=n} log(1 - U_k) / (NN - k); u_n = 1 - exp(lmax_n).  Two passes
// over tiles of kTile uniforms around a deterministic spine; each thread owns
// 8 consecutive n.
__device__ __forceinline__ void sorted_terms8(const EngineRef &eng,
                                              unsigned long long off,
                                              long long n0, long long NN,
                                              double t[8])
{
    uint64_t w[8];
    threefry_words8(eng, off + (unsigned long long)n0, w);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const long long n = n0 + j;
        const double U = canonical_u64(w[j]);
        t[j] = n < NN ? __ddiv_rn(fm::fm_log(__dadd_rn(1.0, -U)),
                                  (double)(NN - n))
                      : 0.0;
    }
}

// Which sorted sequence a launch builds: the step's (ctl->active, NN,
// kbits), or with spec_N > 0 a speculative Multinomial sequence of spec_N
// uniforms at the engine's current position, drawn before the step decides
// to resample (NN = N does not depend on the weights) and skipped when the
// held sequence was drawn at that position already.
struct SortedRun {
    bool run;
    long long NN;
    int kbits;
};

__device__ __forceinline__ SortedRun sorted_run(const ResampleCtl *ctl,
                                                long long spec_N)
{
    SortedRun r;
    if (spec_N > 0) {
        r.run = ctl->spec_offset != ctl->offset;
        r.NN = spec_N;
        r.kbits = bin_kbits(spec_N);
    } else {
        r.run = ctl->active != 0;
        r.NN = ctl->NN;
        r.kbits = ctl->kbits;
    }
    return r;
}

// Pass 1: the terms log(1 - U_n) / (NN - n), stored in u[] for pass 2,
// and their tile sums.
__device__ __forceinline__ void
k_sorted_tile_sums_body(EngineRef eng, const ResampleCtl *ctl, double *tile_sum,
                        double *u, int bid, SmemSortedSums &sm,
                        long long spec_N = 0)
{
    const SortedRun q = sorted_run(ctl, spec_N);
    if (!q.run)
        return;
    double *sh = sm.sh;
    const long long NN = q.NN;
    const long long base = (long long)bid * kTile;
    if (base >= NN)
        return;
    double t[kItems];
    const long long n0 = base + (long long)threadIdx.x * kItems;
    sorted_terms8(eng, ctl->offset, n0, NN, t);
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        s += t[j];
        if (n0 + j < NN)
            u[n0 + j] = t[j];
    }
    double total;
    block_excl_scan(s, sh, total);
    if (threadIdx.x == 0)
        tile_sum[bid] = total;
}

static __global__ void __launch_bounds__(VSMC_SCAN_BOUNDS)
k_sorted_tile_sums(EngineRef eng, const ResampleCtl *ctl, double *tile_sum,
                   double *u)
{
    __shared__ SmemSortedSums sm;
    k_sorted_tile_sums_body(eng, ctl, tile_sum, u, blockIdx.x, sm);
}

__device__ __forceinline__ void
k_sorted_spine_body(const double *tile_sum, double *tile_excl,
                    const ResampleCtl *ctl, int bid, SmemSpine &sm,
                    long long spec_N = 0)
{
    const SortedRun q = sorted_run(ctl, spec_N);
    if (!q.run)
        return;
    double *sh = sm.shd;
    const int ntiles = (int)((q.NN + kTile - 1) / kTile);
    spine_scan_f64(tile_sum, tile_excl, ntiles, 1.0, sh);
}

static __global__ void __launch_bounds__(kSpineThreads)
k_sorted_spine(const double *tile_sum, double *tile_excl,
               const ResampleCtl *ctl)
{
    __shared__ SmemSpine sm;
    k_sorted_spine_body(tile_sum, tile_excl, ctl, blockIdx.x, sm);
}

// Pass 2: u_n = 1 - exp(lmax_n) with lmax_n the reference's sequential sum
// exactly, from the exact scan of the negated terms (its records replaced
// the terms in u[]), then the running maximum and the bin index.
__device__ __forceinline__ void
k_sorted_uniforms_body(const ResampleCtl *ctl, const ExactScan exu,
                       double *u, int32_t *L, int bid, SmemSortedUniforms &sm,
                       long long spec_N = 0)
{
    const SortedRun q = sorted_run(ctl, spec_N);
    if (!q.run)
        return;
    double *shm = sm.shm;
    const long long NN = q.NN;
    const long long base = (long long)bid * kTile;
    if (base >= NN)
        return;
    const long long n0 = base + (long long)threadIdx.x * kItems;
    // the thread's records (vector loads; u is padded past NN)
    double rv[kItems];
#pragma unroll
    for (int j = 0; j < kItems; ++j)
        rv[j] = 0.0;
    if (n0 < NN) {
        const double2 *r2 = reinterpret_cast<const double2 *>(u + n0);
#pragma unroll
        for (int j = 0; j < kItems / 2; ++j) {
            const double2 v = r2[j];
            rv[2 * j] = n0 + 2 * j < NN ? v.x : 0.0;
            rv[2 * j + 1] = n0 + 2 * j + 1 < NN ? v.y : 0.0;
        }
    }
    const int nsp_tile = exu.tiles[bid].nspec;
    if (nsp_tile <= kExactCap && (int)threadIdx.x < nsp_tile)
        sm.sv[threadIdx.x] = exu.s_spec[(size_t)bid * kExactCap + threadIdx.x];
    int nsp = 0;
#pragma unroll
    for (int j = 0; j < kItems; ++j)
        nsp += rv[j] < 0.0;
    int nspec;
    const int rank0 = block_excl_scan(nsp, sm.shi, nspec); // ends with a barrier
    const double a = exu.start[bid]; // -lmax before the tile
    double S[kItems];
    exact_values(rv, rank0, a, sm.sv, nsp_tile > kExactCap, S);
    // carry: the previous tile ends exactly at lmax = -a
    const double umax = bid > 0 ? __dadd_rn(1.0, -fm::fm_exp(-a)) : -INFINITY;
    double uv[kItems];
    double tmax = -INFINITY;
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        uv[j] = __dadd_rn(1.0, -fm::fm_exp(-S[j]));
        tmax = fmax(tmax, uv[j]);
    }
    // block exclusive max-scan (max is exact, so any order gives the same
    // values): inclusive warp scan, then the maxima of the earlier warps
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    double inc = tmax;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double v = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o)
            inc = fmax(inc, v);
    }
    if (lane == 31)
        shm[wid] = inc;
    double exc = __shfl_up_sync(0xffffffffu, inc, 1);
    if (lane == 0)
        exc = -INFINITY;
    __syncthreads();
    for (int w = 0; w < wid; ++w)
        exc = fmax(exc, shm[w]);
    double m = fmax(umax, exc);
    const int kb = q.kbits;
    long long kprev = bin_floor(m, kb); // bin of u_{n-1}
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        m = fmax(m, uv[j]);
        const long long n = n0 + j;
        if (n < NN) {
            u[n] = m;
            const long long khi = bin_floor(m, kb);
            bin_fill(L, kb, n == 0 ? 0 : kprev + 1, khi, n, NN);
            kprev = khi;
        }
    }
}

static __global__ void __launch_bounds__(VSMC_SCAN_BOUNDS)
k_sorted_uniforms(const ResampleCtl *ctl, ExactScan exu, double *u,
                  int32_t *L)
{
    __shared__ SmemSortedUniforms sm;
    k_sorted_uniforms_body(ctl, exu, u, L, blockIdx.x, sm);
}

// The speculative Multinomial sequence (N uniforms at the engine's current
// position), on a stream of its own while the step's move and weights run.
static __global__ void __launch_bounds__(VSMC_SCAN_BOUNDS)
k_spec_tile_sums(EngineRef eng, const ResampleCtl *ctl, long long N,
                 double *tile_sum, double *u)
{
    __shared__ SmemSortedSums sm;
    k_sorted_tile_sums_body(eng, ctl, tile_sum, u, blockIdx.x, sm, N);
}

static __global__ void __launch_bounds__(kSpineThreads)
k_spec_spine(const double *tile_sum, double *tile_excl,
             const ResampleCtl *ctl, long long N)
{
    __shared__ SmemSpine sm;
    k_sorted_spine_body(tile_sum, tile_excl, ctl, blockIdx.x, sm, N);
}

static __global__ void __launch_bounds__(VSMC_SCAN_BOUNDS)
k_spec_uniforms(const ResampleCtl *ctl, long long N, ExactScan exu, double *u,
                int32_t *L)
{
    __shared__ SmemSortedUniforms sm;
    k_sorted_uniforms_body(ctl, exu, u, L, blockIdx.x, sm, N);
}

// The held sequence is now the one for the current position (launched
// after the three kernels above, which all test the same condition).
static __global__ void k_spec_commit(ResampleCtl *ctl)
{
    ctl->spec_offset = ctl->offset;
}

// No sequence held (a fresh workspace).
static __global__ void k_spec_invalidate(ResampleCtl *ctl)
{
    ctl->spec_offset = ~0ull;
}

// ---------------------------------------------------------------------------
// Count of the U01 sequence values <= C ("first n with u_n > C", which for a
// non-decreasing sequence is the upper bound).
__device__ __forceinline__ int ub_shared(const double *u, int lo, int hi,
                                         double C)
{
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (u[mid] <= C)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// First index with s[index] > r in a non-decreasing int array of length n
// (n - 1 when none is; callers check s[n - 1] > r first).
__device__ __forceinline__ int first_above_shared(const int32_t *s, int n,
                                                  long long r)
{
    int l = 0, h = n - 1;
    while (l < h) {
        const int m = (l + h) >> 1;
        if (s[m] > r)
            h = m;
        else
            l = m + 1;
    }
    return l;
}

// The same count for a query C >= the previous query of this thread, whose
// count was `c`: gallop from c (probes c, c+1, c+3, c+7, ...) and finish
// with a binary search inside the last gap, so a query that passes k values
// costs about 2 log2(k + 1) probes instead of log2(n).
__device__ __forceinline__ int ub_gallop(const double *u, int c, int n,
                                         double C)
{
    int lo = c, step = 1;
    while (lo < n) {
        const int p = min(lo + step - 1, n - 1);
        if (u[p] > C)
            return ub_shared(u, lo, p, C);
        lo = p + 1;
        step <<= 1;
    }
    return n;
}

__device__ __forceinline__ long long ub_global(const double *u, long long lo,
                                               long long hi, double C)
{
    while (lo < hi) {
        const long long mid = lo + ((hi - lo) >> 1);
        if (u[mid] <= C)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// ub_gallop over global memory: the count from a known count c <= it.
__device__ __forceinline__ long long ub_gallop_global(const double *u,
                                                      long long c,
                                                      long long n, double C)
{
    long long lo = c, step = 1;
    while (lo < n) {
        const long long p = min(lo + step - 1, n - 1);
        if (u[p] > C)
            return ub_global(u, lo, p, C);
        lo = p + 1;
        step <<= 1;
    }
    return n;
}

// Warp-cooperative upper bound over a non-decreasing sequence f(0..n-1):
// each round the 32 lanes probe 32 evenly spaced points, so a range of n
// shrinks by 33x per global-memory round trip.  Every lane returns the
// count of indices with f(i) <= C.
template <typename F>
__device__ __forceinline__ long long warp_upper_bound(F f, long long lo,
                                                      long long hi, double C)
{
    const int lane = threadIdx.x & 31;
    while (hi - lo > 32) {
        const long long span = hi - lo;
        const long long p = lo + (span * (lane + 1)) / 33;
        const unsigned le = __ballot_sync(0xffffffffu, f(p) <= C);
        const int k = __popc(le); // probes are increasing: a prefix is true
        const long long nlo =
            k > 0 ? lo + (span * k) / 33 + 1 : lo;
        const long long nhi = k < 32 ? lo + (span * (k + 1)) / 33 : hi;
        lo = nlo;
        hi = nhi;
    }
    const long long p = lo + lane;
    const bool le = p < hi && f(p) <= C;
    return lo + __popc(__ballot_sync(0xffffffffu, le));
}

// Systematic (U01SequenceSystematic, u01.hpp:253-287): u_n = u0 + n delta,
// non-decreasing in n; the count is found from a closed-form guess and
// corrected by evaluating the exact rounded sequence.
__device__ __forceinline__ double sys_u(double u0, double delta, long long n)
{
    return __dadd_rn(u0, __dmul_rn((double)n, delta));
}

__device__ __forceinline__ long long sys_count(double C, double u0,
                                               double delta, long long NN)
{
    if (NN <= 0)
        return 0;
    const double g = (C - u0) * (double)NN;
    long long n;
    if (!(g > 0.0))
        n = 0;
    else if (g >= (double)NN)
        n = NN;
    else
        n = (long long)g;
    while (n > 0 && sys_u(u0, delta, n - 1) > C)
        --n;
    while (n < NN && sys_u(u0, delta, n) <= C)
        ++n;
    return n;
}



// The weight the inversion scans for element i: w_i, or for the residual
// schemes its residual r_i * coeff_r (residual.hpp:59-66).  Raw: the
// unnormalised weight exp(lw_i - M) (the normalisation pass), or the
// residual r_i unscaled (the residuals' sum).
template <typename W, bool Residual, bool Raw = false>
__device__ __forceinline__ double scan_weight(const W &wsrc, long long i,
                                              double Nd, double coeff_r,
                                              double *kint)
{
    double w, k = 0.0;
    if (Raw && !Residual) {
        w = wsrc.unnorm(i);
    } else {
        w = wsrc(i);
        if (Residual)
            w = __dmul_rn(residual_split(w, Nd, k), coeff_r);
    }
    if (kint)
        *kint = k;
    return w;
}

// A tile's values in shared memory are padded by one slot per 8, so that a
// thread reading its kItems consecutive values meets no bank conflict.
constexpr int kTilePad = kTile + kTile / 8;
__device__ __forceinline__ int pad8(int l) { return l + (l >> 3); }

struct SmemExactCore {
    double shd[kThreads / 32];
    SmemExactThread et;
};

template <bool Residual>
struct SmemExactTiles {
    double sw[kTilePad];
    int32_t sk[Residual ? kTilePad : 1]; // floor(N w)
    SmemExactCore core;
};

// The weight scanned for a value staged from the source's array.
template <typename W, bool Residual, bool Raw>
__device__ __forceinline__ double
scan_weight_staged(const W &wsrc, typename W::stage_t x, double Nd,
                   double coeff_r, double &kint)
{
    double w, k = 0.0;
    if (Raw && !Residual) {
        w = wsrc.unnorm_stage(x);
    } else {
        w = wsrc.from_stage(x);
        if (Residual)
            w = __dmul_rn(residual_split(w, Nd, k), coeff_r);
    }
    kint = k;
    return w;
}

// Eight values of a thread to global memory (vector stores when all are
// below N).
template <typename T>
__device__ __forceinline__ void store8(T *dst, long long i0, long long N,
                                       const T (&v)[kItems])
{
    if (i0 + kItems <= N) {
        if (sizeof(T) == 8) {
            double2 *d = reinterpret_cast<double2 *>(dst + i0);
#pragma unroll
            for (int j = 0; j < kItems / 2; ++j) {
                double2 q;
                q.x = *reinterpret_cast<const double *>(&v[2 * j]);
                q.y = *reinterpret_cast<const double *>(&v[2 * j + 1]);
                d[j] = q;
            }
        } else {
            int4 *d = reinterpret_cast<int4 *>(dst + i0);
#pragma unroll
            for (int j = 0; j < kItems / 4; ++j) {
                int4 q;
                q.x = *reinterpret_cast<const int *>(&v[4 * j]);
                q.y = *reinterpret_cast<const int *>(&v[4 * j + 1]);
                q.z = *reinterpret_cast<const int *>(&v[4 * j + 2]);
                q.w = *reinterpret_cast<const int *>(&v[4 * j + 3]);
                d[j] = q;
            }
        }
    } else {
#pragma unroll
        for (int j = 0; j < kItems; ++j)
            if (i0 + j < N)
                dst[i0 + j] = v[j];
    }
}

// The mixed form's cumulative weight: a plain FP64 scan.  Each element's
// record is its inclusive prefix within the tile (a block scan of the
// thread's sequential run); the tile's total goes to the spine as an
// unsigned 2^-60 fixed-point integer, so that the tile starts are an exact
// integer scan (non-decreasing whatever the association, hence the same in
// every launch shape) rounded once to double.  The weights are normalised
// (total about 1); totals are clamped to [0, 8] and NaN counts as 0.  The
// inversion gives each tile's last particle the uniforms up to the next
// tile's start, so the records' rounding cannot lose or repeat a child.
constexpr double kApproxScale = 0x1p60;

__device__ __forceinline__ unsigned long long approx_fixed(double x)
{
    if (!(x > 0.0))
        return 0ull;
    return __double2ull_rn(__dmul_rn(fmin(x, 8.0), kApproxScale));
}

template <bool Residual>
__device__ __forceinline__ void
approx_tile_record(const double (&w)[kItems], const int32_t (&kk)[kItems],
                   double pre, double total, long long N, long long i0,
                   int tile, const ExactScan &ex)
{
    double rec[kItems];
    double s = pre;
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        s += w[j];
        rec[j] = s;
    }
    if (i0 < N) {
        store8(ex.rec, i0, N, rec);
        if (Residual)
            store8(ex.kint, i0, N, kk);
    }
    if (threadIdx.x == 0) {
        ExactTile et;
        et.k_total = 0;
        et.nspec = 0;
        et.e_last = kNoBinade;
        ex.tiles[tile] = et;
        ex.pk[tile] = approx_fixed(total);
    }
}

// The tile starts of the plain scan (one CTA): the exclusive integer scan
// of the tiles' fixed-point totals, each rounded once to double.
__device__ __forceinline__ void approx_spine(const ExactScan &ex, int nt,
                                             unsigned long long *sh)
{
    const int per = (nt + (int)blockDim.x - 1) / (int)blockDim.x;
    const int b = (int)threadIdx.x * per, e = min(b + per, nt);
    unsigned long long run = 0;
    for (int t = b; t < e; ++t)
        run += ex.pk[t];
    unsigned long long total;
    unsigned long long off = block_excl_scan(run, sh, total);
    for (int t = b; t < e; ++t) {
        ex.start[t] = __dmul_rn(__ull2double_rn(off), 1.0 / kApproxScale);
        off += ex.pk[t];
    }
    if (threadIdx.x == blockDim.x - 1)
        ex.start[nt] = __dmul_rn(__ull2double_rn(total), 1.0 / kApproxScale);
}

// Phase A of the exact cumulative weight (exact_scan.cuh) for one tile,
// given the thread's kItems weights w (and, residual, integer parts kk).
// Raw: the weights' or the residuals' sequential sum only (for their
// coefficient); the normalisation pass also keeps the unnormalised
// weights in ex.rec.  Otherwise also the element records (and, residual,
// the integer parts floor(N w)) for the inversion; a tile with more
// specials than kept keeps its values for the spine, which writes S itself
// there.  The approximate spine tile_excl is of the weights (or residuals)
// scaled by the spine's coefficient: it is rescaled to the weights scanned
// here.
template <typename W, bool Residual, bool Raw>
__device__ __forceinline__ void
exact_tile_compute(const W &wsrc, long long N, const ResampleCtl *ctl,
                   const double *tile_excl, const ExactScan &ex, int tile,
                   double coeff_r, const double (&w)[kItems],
                   const int32_t (&kk)[kItems], SmemExactCore &sm)
{
    const long long base = (long long)tile * kTile;
    double run = 0.0;
#pragma unroll
    for (int j = 0; j < kItems; ++j)
        run += w[j];
    double total;
    const double pre = block_excl_scan(run, sm.shd, total);
    const long long i0 = base + (long long)threadIdx.x * kItems;
    if (W::kApprox) {
        if (!Raw)
            approx_tile_record<Residual>(w, kk, pre, total, N, i0, tile, ex);
        return;
    }
    double a_apx;
    if (Residual)
        a_apx = Raw ? __ddiv_rn(tile_excl[tile], ctl->coeff_r_apx)
                    : __dmul_rn(tile_excl[tile],
                                __ddiv_rn(coeff_r, ctl->coeff_r_apx));
    else
        a_apx = Raw ? __dmul_rn(tile_excl[tile], wsrc.spine_unnorm())
                    : __dmul_rn(tile_excl[tile], wsrc.spine_ratio());
    ExactThread x;
    exact_thread(i0, N, w, a_apx, pre, ExactMargin<W>::rel, x, sm.et);
    double rec[kItems];
    exact_tile_record(x, w, base, i0, N, tile, ex, rec);
    if (i0 < N) {
        if (Raw && !Residual && W::kExactNorm)
            store8(ex.rec, i0, N, w);
        if (!Raw && x.nspec <= kExactCap)
            store8(ex.rec, i0, N, rec);
        if (!Raw && Residual)
            store8(ex.kint, i0, N, kk);
    }
}

// Phase A for one tile, reading the source in global memory (the batched
// kernels' tile loops).
template <typename W, bool Residual, bool Raw = false>
__device__ __forceinline__ void
k_exact_tiles_body(W wsrc, long long N, const ResampleCtl *ctl,
                   const double *tile_excl, ExactScan ex, int tile,
                   SmemExactTiles<Residual> &sm)
{
    if (!wsrc.active(ctl))
        return;
    N = wsrc.length(ctl, N);
    if ((long long)tile * kTile >= N)
        return;
    // residual schemes without residual children scan nothing (the
    // inversion still takes the integer parts)
    const bool none = Residual && ctl->NN <= 0;
    if (none && Raw)
        return;
    wsrc.prepare();
    const long long base = (long long)tile * kTile;
    const double Nd = (double)resample_children(ctl, N);
    const double coeff_r = Residual && !Raw ? ctl->coeff_r : 1.0;
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const int l = j * kThreads + threadIdx.x;
        const long long i = base + l;
        double k = 0.0;
        const double w = i < N ? scan_weight<W, Residual, Raw>(
                                     wsrc, i, Nd, coeff_r,
                                     Residual && !Raw ? &k : nullptr)
                               : 0.0;
        if (none) {
            if (i < N)
                ex.kint[i] = (int32_t)k;
            continue;
        }
        sm.sw[pad8(l)] = w;
        if (Residual && !Raw)
            sm.sk[pad8(l)] = (int32_t)k;
    }
    if (none)
        return;
    __syncthreads();
    double w[kItems];
    int32_t kk[kItems];
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const int l = pad8(threadIdx.x * kItems + j);
        w[j] = sm.sw[l];
        kk[j] = Residual && !Raw ? sm.sk[l] : 0;
    }
    exact_tile_compute<W, Residual, Raw>(wsrc, N, ctl, tile_excl, ex, tile,
                                         coeff_r, w, kk, sm.core);
}

// Four CTAs per SM (64 registers, a few spilled) hide the exact scan's
// load latency better than three without the bound (measured: the
// resampling chain of a 2^24-particle step 0.18 ms shorter).
#ifndef VSMC_EXACT_MIN_BLOCKS
#define VSMC_EXACT_MIN_BLOCKS 4
#endif

template <int Bytes>
__device__ __forceinline__ void cp_async_n(void *smem, const void *gmem)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    if (Bytes == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa),
                     "l"(gmem)
                     : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa),
                     "l"(gmem)
                     : "memory");
}
__device__ __forceinline__ void cp_async_wait_one()
{
    asm volatile("cp.async.wait_group 1;\n" ::: "memory");
}

// CTAs per SM of the staging k_exact_tiles: the prefetch hides the load
// latency, so three CTAs (85 registers) do without four's spills.
#ifndef VSMC_EXACT_STAGE_MIN_BLOCKS
#define VSMC_EXACT_STAGE_MIN_BLOCKS 3
#endif

// The persistent grid of k_exact_tiles for nt tiles: the SMs times the
// CTAs that fit on one, or fewer for small filters.
inline int exact_grid(int nt)
{
    static int sms = 0;
    if (sms == 0) {
        int dev = 0, v = 0;
        if (cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) ==
                cudaSuccess &&
            v > 0)
            sms = v;
        else
            sms = 148;
    }
    const int g = sms * VSMC_EXACT_STAGE_MIN_BLOCKS;
    return nt < 1 ? 1 : (nt < g ? nt : g);
}

struct SmemExactStage {
    double stage[2][kTilePad]; // the source's values of two tiles
    SmemExactCore core;
};

// Phase A over every tile: a persistent grid (the SMs times the CTAs that
// fit on one) whose CTAs stage the next tile's source values with cp.async
// while they classify the current one, so the loads' latency is hidden.
template <typename W, bool Residual, bool Raw = false>
__global__ void __launch_bounds__(kThreads, VSMC_EXACT_STAGE_MIN_BLOCKS)
k_exact_tiles(W wsrc, long long N, const ResampleCtl *ctl,
              const double *tile_excl, ExactScan ex)
{
    typedef typename W::stage_t S;
    __shared__ SmemExactStage sm;
    if (!wsrc.active(ctl))
        return;
    N = wsrc.length(ctl, N);
    const bool none = Residual && ctl->NN <= 0;
    if (none && Raw)
        return;
    wsrc.prepare();
    const int nt = resample_ntiles(N);
    const double Nd = (double)resample_children(ctl, N);
    const double coeff_r = Residual && !Raw ? ctl->coeff_r : 1.0;
    const S *src = wsrc.stage_src();
    const auto issue = [&](int t, int b) {
        S *dst = reinterpret_cast<S *>(sm.stage[b]);
        const long long base = (long long)t * kTile;
#pragma unroll
        for (int j = 0; j < kItems; ++j) {
            const int l = j * kThreads + threadIdx.x;
            if (base + l < N)
                cp_async_n<sizeof(S)>(&dst[pad8(l)], &src[base + l]);
        }
        cp_async_commit();
    };
    int buf = 0;
    if ((int)blockIdx.x < nt)
        issue(blockIdx.x, 0);
    for (int tile = blockIdx.x; tile < nt; tile += gridDim.x) {
        const int next = tile + gridDim.x;
        if (next < nt) {
            issue(next, buf ^ 1);
            cp_async_wait_one();
        } else {
            cp_async_wait_all();
        }
        __syncthreads();
        const S *st = reinterpret_cast<const S *>(sm.stage[buf]);
        const long long i0 =
            (long long)tile * kTile + (long long)threadIdx.x * kItems;
        double w[kItems];
        int32_t kk[kItems];
#pragma unroll
        for (int j = 0; j < kItems; ++j) {
            double k = 0.0;
            w[j] = i0 + j < N ? scan_weight_staged<W, Residual, Raw>(
                                    wsrc, st[pad8(threadIdx.x * kItems + j)],
                                    Nd, coeff_r, k)
                              : 0.0;
            kk[j] = (int32_t)k;
        }
        if (none) {
            if (i0 < N)
                store8(ex.kint, i0, N, kk);
        } else {
            exact_tile_compute<W, Residual, Raw>(wsrc, N, ctl, tile_excl, ex,
                                                 tile, coeff_r, w, kk,
                                                 sm.core);
        }
        __syncthreads(); // every read of stage[buf] before it is refilled
        buf ^= 1;
    }
}

constexpr int kExactDirtyStage = 256; // tiles with specials the spine stages

// Per tile with specials (its rank q among them, in order): the tile d, its
// record, the clean k before it (pk: tiles with specials count 0), the
// binade of the clean tiles after it and the exact S after it.  Ranks below
// kExactDirtyStage live in shared memory, the others in the ExactScan
// arrays dirty / pk / eaft / s_out (indexed by q).
struct SmemExactSpine {
    unsigned long long wk[32]; // per warp: clean k before its tiles
    int wd[32];                // per warp: tiles with specials before
    unsigned long long ktot;
    int ndt;
    int shi[kSpineThreads / 32];
    int dq[kExactDirtyStage];
    ExactTile tq[kExactDirtyStage];
    unsigned long long pkq[kExactDirtyStage];
    int eaft[kExactDirtyStage];
    double sout[kExactDirtyStage];
    // the specials of the staged tiles, when they fit: tile q's at
    // st[st_off[q]...]
    ExactSpecial st[kExactStage];
    int st_off[kExactDirtyStage];
};

// Phase B (one CTA): the exact S before every tile and at every special.
// Each warp owns a contiguous range of tiles and reads it 32 tiles at a
// time (coalesced), with warp scans for the clean k and the ranks of the
// tiles with specials; only thread 0's walk over the specials is
// sequential, and it reads shared memory.  Raw: the sequential sum sets
// the coefficient -- of the residuals, coeff_r = 1 / sum as the
// reference's `1 / math::asum(M, rptr)` (residual.hpp:63); of the
// unnormalised weights, coeff_w (weight_set.hpp:121).
template <typename W, bool Residual, bool Raw = false>
__device__ __forceinline__ void
k_exact_spine_body(W wsrc, long long N, ResampleCtl *ctl, int nt,
                   ExactScan ex, SmemExactSpine &sm)
{
    if (!wsrc.active(ctl) || (Residual && ctl->NN <= 0))
        return;
    wsrc.prepare();
    N = wsrc.length(ctl, N);
    nt = min(nt, resample_ntiles(N));
    if (W::kApprox) {
        // the plain scan's tile starts (the coefficients stay the tile
        // sums' approximate ones)
        if (!Raw)
            approx_spine(ex, nt, sm.wk);
        return;
    }
    const int bd = (int)blockDim.x;
    const int lane = threadIdx.x & 31, wq = threadIdx.x >> 5, nw = bd >> 5;
    const int perw = (nt + nw - 1) / nw;
    const int wb = min(wq * perw, nt), we = min(wb + perw, nt);
    // a tile record, or an empty clean one past the warp's range
    const auto tile_at = [&](int t) {
        ExactTile et;
        et.k_total = 0;
        et.nspec = 0;
        et.e_last = kNoBinade;
        if (t < we)
            et = ex.tiles[t];
        return et;
    };
    // 1a. per warp: clean k and tiles with specials (tile 0 always has one:
    // its first element); their exclusive prefixes over the warps
    {
        unsigned long long k = 0;
        int d = 0;
        for (int t = wb + lane; t < we; t += 32) {
            const ExactTile et = ex.tiles[t];
            k += et.nspec == 0 ? et.k_total : 0ull;
            d += et.nspec != 0;
        }
        k = __shfl_sync(0xffffffffu, warp_incl_scan(k), 31);
        d = __shfl_sync(0xffffffffu, warp_incl_scan(d), 31);
        if (lane == 0) {
            sm.wk[wq] = k;
            sm.wd[wq] = d;
        }
    }
    __syncthreads();
    if (wq == 0) {
        const unsigned long long k = lane < nw ? sm.wk[lane] : 0ull;
        const int d = lane < nw ? sm.wd[lane] : 0;
        const unsigned long long ki = warp_incl_scan(k);
        const int di = warp_incl_scan(d);
        if (lane < nw) {
            sm.wk[lane] = ki - k;
            sm.wd[lane] = di - d;
        }
        if (lane == 31) {
            sm.ktot = ki;
            sm.ndt = di;
        }
    }
    __syncthreads();
    const int ndt = sm.ndt;
    // 1b. the tiles with specials, by rank: the tile, its record, the clean
    // k before it and the binade of the clean tiles after it
    {
        unsigned long long off = sm.wk[wq];
        int q = sm.wd[wq];
        for (int t0 = wb; t0 < we; t0 += 32) {
            const int t = t0 + lane;
            const ExactTile et = tile_at(t);
            const int dc = et.nspec != 0;
            const unsigned long long kc = dc ? 0ull : et.k_total;
            const unsigned long long ki = warp_incl_scan(kc);
            const int di = warp_incl_scan(dc);
            if (dc) {
                const int qq = q + di - 1;
                const unsigned long long pkd = off + ki;
                int ea = kNoBinade;
                if (t + 1 < nt) {
                    const ExactTile nx = ex.tiles[t + 1];
                    if (nx.nspec == 0)
                        ea = nx.e_last;
                }
                if (qq < kExactDirtyStage) {
                    sm.dq[qq] = t;
                    sm.tq[qq] = et;
                    sm.pkq[qq] = pkd;
                    sm.eaft[qq] = ea;
                } else {
                    ex.dirty[qq] = t;
                    ex.pk[qq] = pkd;
                    ex.eaft[qq] = ea;
                }
            }
            off += __shfl_sync(0xffffffffu, ki, 31);
            q += __shfl_sync(0xffffffffu, di, 31);
        }
    }
    __syncthreads();
    const bool staged_all = ndt <= kExactDirtyStage;
    // 2. stage the staged tiles' specials when they all fit
    int nsq = 0;
    if ((int)threadIdx.x < min(ndt, kExactDirtyStage)) {
        const ExactTile et = sm.tq[threadIdx.x];
        nsq = et.nspec <= kExactCap ? et.nspec : 0;
    }
    int nst;
    const int soff = block_excl_scan(nsq, sm.shi, nst); // ends with a barrier
    const bool fits = staged_all && nst <= kExactStage;
    if (fits && (int)threadIdx.x < ndt)
        sm.st_off[threadIdx.x] = soff;
    __syncthreads();
    if (fits) { // a warp per tile with specials
        for (int q = wq; q < ndt; q += nw) {
            const int ns = sm.tq[q].nspec;
            if (ns > kExactCap)
                continue;
            for (int r = lane; r < ns; r += 32)
                sm.st[sm.st_off[q] + r] =
                    ex.spec[(size_t)sm.dq[q] * kExactCap + r];
        }
    }
    __syncthreads();
    // 3. the walk over the tiles with specials
    if (threadIdx.x == 0) {
        const double Nd = (double)resample_children(ctl, N);
        const double coeff_r = Residual && !Raw ? ctl->coeff_r : 1.0;
        double S = 0.0;
        unsigned long long pk_prev = 0;
        int ea_prev = kNoBinade;
        for (int q = 0; q < ndt; ++q) {
            const bool sq = q < kExactDirtyStage;
            const int d = sq ? sm.dq[q] : ex.dirty[q];
            const ExactTile et = sq ? sm.tq[q] : ex.tiles[d];
            const unsigned long long pkd = sq ? sm.pkq[q] : ex.pk[q];
            const unsigned long long K = pkd - pk_prev;
            if (K != 0) // the clean tiles between the previous and d
                S = __dadd_rn(S, __dmul_rn((double)K, exact_pow2(ea_prev - 52)));
            ex.start[d] = S;
            if (et.nspec <= kExactCap) {
                unsigned long long kb = 0;
                for (int r = 0; r < et.nspec; ++r) {
                    const ExactSpecial sp =
                        fits ? sm.st[sm.st_off[q] + r]
                             : ex.spec[(size_t)d * kExactCap + r];
                    const unsigned long long seg = sp.k_before - kb;
                    if (seg != 0)
                        S = __dadd_rn(S, __dmul_rn((double)seg,
                                                   exact_pow2(sp.e_seg - 52)));
                    S = __dadd_rn(S, sp.w);
                    ex.s_spec[(size_t)d * kExactCap + r] = S;
                    kb = sp.k_before;
                }
                const unsigned long long tail = et.k_total - kb;
                if (tail != 0)
                    S = __dadd_rn(S, __dmul_rn((double)tail,
                                               exact_pow2(et.e_last - 52)));
            } else {
                // more specials than kept: the reference's loop itself
                const long long b0 = (long long)d * kTile;
                const long long b1 = min(b0 + (long long)kTile, N);
                for (long long i = b0; i < b1; ++i) {
                    S = __dadd_rn(S, scan_weight<W, Residual, Raw>(
                                         wsrc, i, Nd, coeff_r, nullptr));
                    if (!Raw)
                        ex.rec[i] = S;
                }
            }
            if (sq)
                sm.sout[q] = S;
            else
                ex.s_out[q] = S;
            pk_prev = pkd;
            ea_prev = sq ? sm.eaft[q] : ex.eaft[q];
        }
    }
    __syncthreads();
    // 4. every clean tile (and the end): the exact S after the last tile
    // with specials before it plus the clean k since, in that binade
    const auto after = [&](int qq, unsigned long long k) {
        if (qq < 0) // (tile 0 always has a special)
            return 0.0;
        const bool sq = qq < kExactDirtyStage;
        double S = sq ? sm.sout[qq] : ex.s_out[qq];
        const unsigned long long K = k - (sq ? sm.pkq[qq] : ex.pk[qq]);
        if (K != 0) {
            const int ea = sq ? sm.eaft[qq] : ex.eaft[qq];
            S = __dadd_rn(S, __dmul_rn((double)K, exact_pow2(ea - 52)));
        }
        return S;
    };
    {
        unsigned long long off = sm.wk[wq];
        int q = sm.wd[wq];
        for (int t0 = wb; t0 < we; t0 += 32) {
            const int t = t0 + lane;
            const ExactTile et = tile_at(t);
            const int dc = et.nspec != 0;
            const unsigned long long kc = dc ? 0ull : et.k_total;
            const unsigned long long ki = warp_incl_scan(kc);
            const int di = warp_incl_scan(dc);
            if (t < we && !dc)
                ex.start[t] = after(q + di - 1, off + ki - kc);
            off += __shfl_sync(0xffffffffu, ki, 31);
            q += __shfl_sync(0xffffffffu, di, 31);
        }
    }
    if (threadIdx.x == 0) {
        const double S = after(ndt - 1, sm.ktot);
        ex.start[nt] = S;
        if (Raw && Residual)
            ctl->coeff_r = __ddiv_rn(1.0, S);
        else if (Raw)
            ctl->coeff_w = __ddiv_rn(1.0, S);
    }
}

template <typename W, bool Residual, bool Raw = false>
__global__ void __launch_bounds__(kSpineThreads)
k_exact_spine(W wsrc, long long N, ResampleCtl *ctl, int nt, ExactScan ex)
{
    __shared__ SmemExactSpine sm;
    k_exact_spine_body<W, Residual, Raw>(wsrc, N, ctl, nt, ex, sm);
}

// The inversion kernel (internal::inversion, common.hpp:57-84, on the FP64
// scan of the weights) and the first half of internal::cfrp_trans.
// Residual: weights are r * coeff_r and k = floor(N w) is added back
// (residual.hpp:59-76).  Sys: closed-form count.  Outputs: replication
// (optional), copy_from (self for survivors, -(r+1) for the tile's r-th
// slot without offspring), sinc_local (surplus children of particles <= i
// minus the zero slots of earlier tiles) and the tile's zero-slot count.
template <typename W, bool Residual, bool Sys>
__device__ __forceinline__ void
k_invert_body(W wsrc, long long N, ResampleCtl *ctl, const double *tile_excl,
              const long long *tile_kexcl, const double *u, long long n_u,
              const int32_t *L, int32_t *rep_out, int32_t *copy_from,
              int32_t *sinc_local, int32_t *tile_zeros, int32_t *tile_sinc_last,
              ExactScan ex, int tile_bid, SmemInvert<Residual> &sm)
{
    if (!ctl->active)
        return;
    double *sw = sm.sw; // uniforms, then the outputs
    long long *shl = sm.shl;
    long long *sh_bound = sm.bound;
    long long *sh_last = sm.last;
    (void)wsrc; // the weights enter through the exact scan's records

    const int tile = tile_bid;
    const long long base = (long long)tile * kTile;
    const long long NN = ctl->NN;
    const long long Nout = resample_children(ctl, N);
    const double u0 = Sys ? ctl->u0 : 0.0;
    const double delta = ctl->delta;
    const long long nu = Sys ? NN : min(NN, n_u);
    // the reference's cumulative weight before and at the end of the tile,
    // exactly (exact_scan.cuh).  Residual schemes without residual children
    // draw no uniform and scan nothing.
    const bool exact = !(Residual && NN <= 0);
    const double a = exact ? ex.start[tile] : 0.0;
    const double b = exact ? ex.start[tile + 1] : 0.0;
    const int nsp_tile = exact ? ex.tiles[tile].nspec : 0;

    // uniforms that can fall in this tile: (ub(a), ub(b)], each found in a
    // bin window of about 8 values by one warp while the others load weights
    const int wid = threadIdx.x >> 5;
    if (wid < 2) {
        const double C = wid == 0 ? a : b;
        long long r;
        if ((wid == 0 && tile == 0) || nu <= 0) {
            r = 0; // (no uniform: the bin index L is not written)
        } else if (Sys) {
            r = sys_count(C, u0, delta, NN);
        } else {
            long long wl, wh;
            bin_window(L, ctl->kbits, nu, C, wl, wh);
            wl = max(min(wl, nu), 0ll);
            wh = min(max(wh, wl), nu);
            r = warp_upper_bound([u](long long i) { return u[i]; }, wl, wh, C);
        }
        if ((threadIdx.x & 31) == 0)
            sh_bound[wid] = r;
    }
    // the thread's records and integer parts, straight into registers
    // (kItems consecutive values: vector loads; the arrays are padded past
    // N to a multiple of 32 elements)
    const long long i0l = base + (long long)threadIdx.x * kItems;
    double rv[kItems];
    int k_int[kItems];
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        rv[j] = 0.0;
        k_int[j] = 0;
    }
    if (exact && i0l < N) {
        const double2 *r2 = reinterpret_cast<const double2 *>(ex.rec + i0l);
#pragma unroll
        for (int j = 0; j < kItems / 2; ++j) {
            const double2 v = r2[j];
            rv[2 * j] = i0l + 2 * j < N ? v.x : 0.0;
            rv[2 * j + 1] = i0l + 2 * j + 1 < N ? v.y : 0.0;
        }
    }
    if (Residual && i0l < N) {
        const int4 *k4 = reinterpret_cast<const int4 *>(ex.kint + i0l);
#pragma unroll
        for (int j = 0; j < kItems / 4; ++j) {
            const int4 v = k4[j];
            const int q[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int m = 0; m < 4; ++m)
                k_int[4 * j + m] = i0l + 4 * j + m < N ? q[m] : 0;
        }
    }
    if (nsp_tile <= kExactCap && (int)threadIdx.x < nsp_tile)
        sm.sv[threadIdx.x] = ex.s_spec[(size_t)tile * kExactCap + threadIdx.x];
    __syncthreads();
    // the tile's uniforms into shared memory, asynchronously
    const long long lo = sh_bound[0];
    const long long hi = max(sh_bound[1], lo);
    const bool staged = !Sys && (hi - lo) <= kUStage;
    if (staged) {
        for (int k = threadIdx.x; k < (int)(hi - lo); k += kThreads)
            cp_async8(&sw[k], &u[lo + k]);
        cp_async_commit();
    }
    // each particle's cumulative weight, exactly the reference's
    double Cx[kItems];
#pragma unroll
    for (int j = 0; j < kItems; ++j)
        Cx[j] = 0.0;
    if (exact) {
        int nsp = 0;
#pragma unroll
        for (int j = 0; j < kItems; ++j)
            nsp += rv[j] < 0.0;
        int nspec;
        const int rank0 = block_excl_scan(nsp, reinterpret_cast<int *>(shl),
                                          nspec);
        exact_values(rv, rank0, a, sm.sv, nsp_tile > kExactCap, Cx);
    }
    if (staged)
        cp_async_wait_all();
    __syncthreads();

    // counts c_i = #{n: u_n <= C_i} for this thread's particles; C_i is
    // non-decreasing along the thread's particles, so after the first
    // search each count gallops on from the previous one.  Counts, indices
    // and prefixes are 32-bit: N <= 2^30.
    const int ilo = (int)lo, ihi = (int)hi, iNN = (int)NN, iN = (int)N;
    const int i0 = (int)base + (int)threadIdx.x * kItems;
    int cnt[kItems];
    int pos = -1;
    long long gpos = -1;
    const int tile_last = (int)min(base + (long long)kTile, N) - 1;
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const int i = i0 + j;
        const double C = Cx[j];
        int c;
        if (i >= iN - 1) {
            c = iNN; // the last particle takes every remaining uniform
        } else if (W::kApprox && i == tile_last) {
            // the plain scan: the tile closes at the next tile's start
            c = ihi;
        } else if (Sys) {
            c = (int)sys_count(C, u0, delta, NN);
        } else if (staged) {
            pos = pos < 0 ? ub_shared(sw, 0, ihi - ilo, C)
                          : ub_gallop(sw, pos, ihi - ilo, C);
            c = ilo + pos;
        } else {
            gpos = gpos < 0 ? ub_global(u, lo, hi, C)
                            : ub_gallop_global(u, gpos, hi, C);
            c = (int)gpos;
        }
        cnt[j] = min(max(c, ilo), i >= iN - 1 ? iNN : ihi);
    }
#pragma unroll
    for (int j = 1; j < kItems; ++j)
        cnt[j] = max(cnt[j], cnt[j - 1]);
    int prev = __shfl_up_sync(0xffffffffu, cnt[kItems - 1], 1);
    if ((threadIdx.x & 31) == 31)
        sh_last[wid] = cnt[kItems - 1];
    __syncthreads();
    if ((threadIdx.x & 31) == 0)
        prev = (threadIdx.x == 0) ? (tile > 0 ? ilo : 0)
                                  : (int)sh_last[wid - 1];
    int rep[kItems];
    int zeros = 0;
    int ksum = 0;
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const int i = i0 + j;
        const int c = max(cnt[j], prev);
        rep[j] = (i < iN) ? (c - prev) + k_int[j] : 0;
        prev = c;
        cnt[j] = c;
        zeros += (i < iN && rep[j] == 0) ? 1 : 0;
        ksum += k_int[j];
    }
    // the last queried uniform fixes the words drawn (inversion queries
    // u_0..u_{n_final}, common.hpp:76-81)
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        if (i0 + j == iN - 2) {
            ctl->n_final = cnt[j];
            if (!Sys)
                ctl->words = (NN > 0) ? (unsigned long long)min(iNN, cnt[j] + 1)
                                      : 0ull;
        }
    }
    int *shi = reinterpret_cast<int *>(shl);
    int ztot;
    int zloc = block_excl_scan(zeros, shi, ztot);
    int ktot;
    const int kex = Residual ? block_excl_scan(ksum, shi, ktot) : 0;
    if (threadIdx.x == 0)
        tile_zeros[tile] = ztot;
    int kprefix = Residual ? (int)tile_kexcl[tile] + kex : 0;
    int32_t cf[kItems], sc[kItems], rp[kItems];
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const int i = i0 + j;
        kprefix += k_int[j];
        // R_{<=i} = count_i + K_{<=i}; the last particle closes at the
        // number of children
        const int R = (i >= iN - 1) ? (int)Nout : cnt[j] + kprefix;
        if (rep[j] == 0) {
            cf[j] = -(zloc + 1);
            ++zloc;
        } else {
            cf[j] = i;
        }
        sc[j] = R - (i + 1) + zloc;
        rp[j] = rep[j];
        if (i == tile_last)
            tile_sinc_last[tile] = sc[j];
    }
    // stage the outputs through shared memory for coalesced stores
    __syncthreads();
    int32_t *s32 = reinterpret_cast<int32_t *>(sw);
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        s32[threadIdx.x * kItems + j] = cf[j];
        s32[kTile + threadIdx.x * kItems + j] = sc[j];
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const long long i = base + (long long)j * kThreads + threadIdx.x;
        if (i < N) {
            copy_from[i] = s32[j * kThreads + threadIdx.x];
            sinc_local[i] = s32[kTile + j * kThreads + threadIdx.x];
        }
    }
    if (rep_out != nullptr) {
        __syncthreads();
#pragma unroll
        for (int j = 0; j < kItems; ++j)
            s32[threadIdx.x * kItems + j] = rp[j];
        __syncthreads();
#pragma unroll
        for (int j = 0; j < kItems; ++j) {
            const long long i = base + (long long)j * kThreads + threadIdx.x;
            if (i < N)
                rep_out[i] = s32[j * kThreads + threadIdx.x];
        }
    }
}

// Five CTAs per SM: 48 registers without spills.
#ifndef VSMC_INVERT_MIN_BLOCKS
#define VSMC_INVERT_MIN_BLOCKS 5
#endif

template <typename W, bool Residual, bool Sys>
__global__ void __launch_bounds__(kThreads, VSMC_INVERT_MIN_BLOCKS)
k_invert(W wsrc, long long N, ResampleCtl *ctl, const double *tile_excl,
         const long long *tile_kexcl, const double *u, long long n_u,
         const int32_t *L, int32_t *rep_out, int32_t *copy_from,
         int32_t *sinc_local, int32_t *tile_zeros, int32_t *tile_sinc_last,
         ExactScan ex)
{
    __shared__ SmemInvert<Residual> sm;
    k_invert_body<W, Residual, Sys>(wsrc, N, ctl, tile_excl, tile_kexcl, u, n_u,
        L, rep_out, copy_from, sinc_local, tile_zeros, tile_sinc_last, ex,
        blockIdx.x, sm);
}

// Exclusive prefix of the per-tile zero-slot counts (one CTA) and, per
// tile, the range of tiles holding the parents of its zero slots.  The
// surplus count at the end of tile t is E[t] = tile_sinc_last[t] + zexcl[t]
// (non-decreasing); the parent of rank k is in the first tile with
// E > k, found by a binary search over E staged in shared memory.
constexpr int kSpineStage = 8192; // tiles whose E fits in shared memory

struct SmemZeroSpine {
    long long sh[kSpineThreads / 32];
    int32_t S[kSpineStage]; // zero counts, then surplus ends E
};
struct SmemFill {
    int32_t ss[kTile];  // sinc of one parent tile
    int32_t tab[kTile]; // parent of each zero-slot rank of this tile
};

__device__ __forceinline__ void
k_zero_spine_body(const int32_t *tile_zeros, const int32_t *tile_sinc_last,
                  int32_t *zexcl, int32_t *tfirst, int32_t *tlast, int ntiles,
                  const ResampleCtl *ctl, int bid, SmemZeroSpine &sm)
{
    if (!ctl->active)
        return;
    long long *sh = sm.sh;
    int32_t *S = sm.S; // zero counts, then surplus ends E
    const bool staged = ntiles <= kSpineStage;
    // phase 1: exclusive prefix of the zero counts (striped load, ordered
    // contiguous runs from shared memory)
    if (staged) {
#pragma unroll 8
        for (int t = threadIdx.x; t < ntiles; t += blockDim.x)
            S[t] = tile_zeros[t];
        __syncthreads();
    }
    const int32_t *Z = staged ? S : tile_zeros;
    const int per = (ntiles + blockDim.x - 1) / blockDim.x;
    const int b = threadIdx.x * per;
    const int e = min(b + per, ntiles);
    long long run = 0;
    for (int t = b; t < e; ++t)
        run += Z[t];
    long long total;
    run = block_excl_scan(run, sh, total);
    for (int t = b; t < e; ++t) {
        const int32_t z = Z[t];
        zexcl[t] = (int32_t)run;
        run += z;
    }
    if (threadIdx.x == blockDim.x - 1)
        zexcl[ntiles] = (int32_t)total;
    __syncthreads();
    // phase 2: E[t] = surplus count at the end of tile t (non-decreasing)
    if (staged) {
#pragma unroll 8
        for (int t = threadIdx.x; t < ntiles; t += blockDim.x)
            S[t] = tile_sinc_last[t] + zexcl[t];
        __syncthreads();
    }
    auto Eat = [&](int t) {
        return staged ? (long long)S[t]
                      : (long long)tile_sinc_last[t] + zexcl[t];
    };
    auto first_tile_above = [&](long long k) {
        int lo = 0, hi = ntiles - 1;
        while (lo < hi) {
            const int m = (lo + hi) >> 1;
            if (Eat(m) > k)
                hi = m;
            else
                lo = m + 1;
        }
        return lo;
    };
    // phase 3: the parent tiles of each tile's zero slots
    for (int t = threadIdx.x; t < ntiles; t += blockDim.x) {
        const long long z0 = zexcl[t];
        const long long z1 = zexcl[t + 1];
        if (z0 == z1) {
            tfirst[t] = 0;
            tlast[t] = -1;
        } else {
            tfirst[t] = first_tile_above(z0);
            tlast[t] = first_tile_above(z1 - 1);
        }
    }
}

// The zero-slot spine, then the engine position (the words the inversion
// counted are final here; nothing after this kernel reads the offset).
static __global__ void __launch_bounds__(kSpineThreads)
k_zero_spine(const int32_t *tile_zeros, const int32_t *tile_sinc_last,
             int32_t *zexcl, int32_t *tfirst, int32_t *tlast, int ntiles,
             ResampleCtl *ctl)
{
    __shared__ SmemZeroSpine sm;
    k_zero_spine_body(tile_zeros, tile_sinc_last, zexcl, tfirst, tlast, ntiles,
        ctl, blockIdx.x, sm);
    if (threadIdx.x == 0 && ctl->active)
        ctl->offset += ctl->words;
}

// internal::cfrp_trans for the slots without offspring (common.hpp:94-106):
// the k-th such slot takes the k-th surplus child in parent order, i.e. the
// first parent p with sinc(p) > k, sinc(p) = sinc_local[p] + zexcl[tile(p)].
// The zero slots of tile t hold the consecutive ranks [zexcl[t],
// zexcl[t + 1]).  The CTA of tile t stages the parent tiles tfirst[t]..
// tlast[t] one at a time in shared memory; parent p owns the ranks
// [sinc(p - 1), sinc(p)) and writes itself into a rank -> parent table for
// those that fall in the tile's window, so no slot searches.
__device__ __forceinline__ void
k_cfrp_fill_body(long long N, ResampleCtl *ctl, const int32_t *sinc_local,
                 const int32_t *zexcl, const int32_t *tfirst,
                 const int32_t *tlast, int32_t *copy_from, int tile_bid,
                 SmemFill &sm)
{
    if (!ctl->active)
        return;
    int32_t *ss = sm.ss;
    int32_t *tab = sm.tab;
    const int tile = tile_bid;
    const int t0 = tfirst[tile], t1 = tlast[tile];
    if (t1 < t0)
        return; // every particle of the tile has offspring
    const int Z0 = zexcl[tile];
    const int z = min(zexcl[tile + 1] - Z0, kTile); // zero slots of the tile
    const long long base = (long long)tile * kTile;
    int32_t cf[kItems];
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const long long i = base + (long long)j * kThreads + threadIdx.x;
        cf[j] = i < N ? copy_from[i] : 0;
    }
    for (int k = threadIdx.x; k < z; k += kThreads)
        tab[k] = -1;
    int prev_top = INT_MIN; // ranks below the first staged tile map to it
    for (int pt = t0; pt <= t1; ++pt) {
        const long long pb = (long long)pt * kTile;
        const int len = (int)min((long long)kTile, N - pb);
        const int32_t zoff = zexcl[pt];
        for (int j = threadIdx.x; j < len; j += kThreads)
            ss[j] = sinc_local[pb + j] + zoff;
        __syncthreads();
        for (int j = threadIdx.x; j < len; j += kThreads) {
            const int lo = max(j > 0 ? ss[j - 1] : prev_top, Z0);
            const int hi = min(ss[j], Z0 + z);
            for (int r = lo; r < hi; ++r)
                tab[r - Z0] = (int32_t)(pb + j);
        }
        prev_top = max(prev_top, ss[len - 1]);
        __syncthreads();
    }
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const long long i = base + (long long)j * kThreads + threadIdx.x;
        if (i < N && cf[j] < 0) {
            const int k = -cf[j] - 1; // rank - Z0
            const int32_t p = k < z ? tab[k] : -1;
            if (p >= 0) {
                copy_from[i] = p;
            } else { // no parent found: replication != N
                atomicExch(&ctl->error, (int)VSMC_CUDA_EDEGENERATE);
                copy_from[i] = (int32_t)i;
            }
        }
    }
}

static __global__ void __launch_bounds__(VSMC_SCAN_BOUNDS)
k_cfrp_fill(long long N, ResampleCtl *ctl, const int32_t *sinc_local,
            const int32_t *zexcl, const int32_t *tfirst, const int32_t *tlast,
            int32_t *copy_from)
{
    __shared__ SmemFill sm;
    k_cfrp_fill_body(N, ctl, sinc_local, zexcl, tfirst, tlast, copy_from,
        blockIdx.x, sm);
}

// Finalise the engine position.
static __global__ void k_resample_done(ResampleCtl *ctl)
{
    if (!ctl->active)
        return;
    ctl->offset += ctl->words;
}

// Running maximum of caller-supplied uniforms (parity mode): tile maxima,
// then each tile folds the maxima before it.
static __global__ void __launch_bounds__(kThreads)
k_tile_max(const double *u, long long n, double *tile_max)
{
    __shared__ double sh[kThreads / 32];
    const long long base = (long long)blockIdx.x * kTile;
    double m = -INFINITY;
    for (int j = 0; j < kItems; ++j) {
        const long long i = base + (long long)j * kThreads + threadIdx.x;
        if (i < n)
            m = fmax(m, u[i]);
    }
    m = warp_max(m);
    if ((threadIdx.x & 31) == 0)
        sh[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = -INFINITY;
        for (int w = 0; w < kThreads / 32; ++w)
            r = fmax(r, sh[w]);
        tile_max[blockIdx.x] = r;
    }
}

static __global__ void __launch_bounds__(kThreads)
k_apply_max(const double *u, long long n, const double *tile_max, double *out,
            const ResampleCtl *ctl, int32_t *L)
{
    __shared__ double carry_sh;
    __shared__ double shm[kThreads];
    if (threadIdx.x == 0) {
        double c = -INFINITY;
        for (unsigned t = 0; t < blockIdx.x; ++t)
            c = fmax(c, tile_max[t]);
        carry_sh = c;
    }
    const long long base = (long long)blockIdx.x * kTile;
    double v[kItems];
    double tm = -INFINITY;
    for (int j = 0; j < kItems; ++j) {
        const long long i = base + (long long)threadIdx.x * kItems + j;
        v[j] = i < n ? u[i] : -INFINITY;
        tm = fmax(tm, v[j]);
    }
    shm[threadIdx.x] = tm;
    __syncthreads();
    for (int o = 1; o < kThreads; o <<= 1) {
        const double x = threadIdx.x >= (unsigned)o ? shm[threadIdx.x - o]
                                                    : -INFINITY;
        __syncthreads();
        shm[threadIdx.x] = fmax(shm[threadIdx.x], x);
        __syncthreads();
    }
    double m = fmax(carry_sh, threadIdx.x > 0 ? shm[threadIdx.x - 1]
                                              : -INFINITY);
    const int kb = ctl->kbits;
    long long kprev = bin_floor(m, kb);
    for (int j = 0; j < kItems; ++j) {
        const long long i = base + (long long)threadIdx.x * kItems + j;
        m = fmax(m, v[j]);
        if (i < n) {
            out[i] = m;
            const long long khi = bin_floor(m, kb);
            bin_fill(L, kb, i == 0 ? 0 : kprev + 1, khi, i, n);
            kprev = khi;
        }
    }
}

// ------------------------------------------------------------ host side --
struct ResampleWorkspace {
    ResampleCtl *ctl;
    double *tile_sum;      // ntiles + 1
    double *tile_excl;     // ntiles + 1
    long long *tile_k;     // ntiles + 1
    long long *tile_kexcl; // ntiles + 1
    double *u_tile_sum;    // ntiles + 1
    double *u_tile_excl;   // ntiles + 1
    int32_t *tile_zeros;   // ntiles + 1
    int32_t *zexcl;        // ntiles + 1
    int32_t *tile_sinc_last; // ntiles + 1
    int32_t *tfirst;       // ntiles + 1
    int32_t *tlast;        // ntiles + 1
    int32_t *bins;         // N / 8 + 2 (bin index of the U01 sequence)
    double *u;             // N
    int32_t *sinc;         // N (tile-local surplus counts)
    ExactScan ex;          // the exact cumulative weight (exact_scan.cuh)
    ExactScan exu;         // the exact lmax of the sorted U01 sequence
                           // (its records live in u)
};


constexpr size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// Bytes carve_workspace lays out for N particles (constexpr so that a static
// scratch array can be sized from it at compile time).
// Bytes of the exact scan's arrays for N particles.
constexpr size_t exact_scan_bytes(long long N)
{
    const size_t nt = (size_t)resample_ntiles(N) + 1;
    return align256(nt * sizeof(ExactTile)) +
           align256(nt * kExactCap * sizeof(ExactSpecial)) +
           align256(nt * kExactCap * 8) + 3 * align256(nt * 8) +
           align256((size_t)N * 8) + align256((size_t)N * 4) +
           2 * align256(nt * 4);
}

// The per-tile arrays of an exact scan whose records live elsewhere.
constexpr size_t exact_scan_tile_bytes(long long N)
{
    const size_t nt = (size_t)resample_ntiles(N) + 1;
    return align256(nt * sizeof(ExactTile)) +
           align256(nt * kExactCap * sizeof(ExactSpecial)) +
           align256(nt * kExactCap * 8) + 3 * align256(nt * 8) +
           2 * align256(nt * 4);
}

constexpr size_t resample_workspace_bytes(long long N)
{
    const size_t nt = (size_t)resample_ntiles(N) + 1;
    return align256(sizeof(ResampleCtl)) + 6 * align256(nt * 8) +
           5 * align256(nt * 4) + align256(((size_t)N / 8 + 2) * 4) +
           align256((size_t)N * 8) + align256((size_t)N * 4) +
           exact_scan_bytes(N) + exact_scan_tile_bytes(N);
}

inline ResampleWorkspace carve_workspace(void *base, long long N)
{
    char *p = static_cast<char *>(base);
    const size_t nt = (size_t)resample_ntiles(N) + 1;
    ResampleWorkspace w;
    w.ctl = reinterpret_cast<ResampleCtl *>(p);
    p += align256(sizeof(ResampleCtl));
    w.tile_sum = reinterpret_cast<double *>(p);
    p += align256(nt * 8);
    w.tile_excl = reinterpret_cast<double *>(p);
    p += align256(nt * 8);
    w.tile_k = reinterpret_cast<long long *>(p);
    p += align256(nt * 8);
    w.tile_kexcl = reinterpret_cast<long long *>(p);
    p += align256(nt * 8);
    w.u_tile_sum = reinterpret_cast<double *>(p);
    p += align256(nt * 8);
    w.u_tile_excl = reinterpret_cast<double *>(p);
    p += align256(nt * 8);
    w.tile_zeros = reinterpret_cast<int32_t *>(p);
    p += align256(nt * 4);
    w.zexcl = reinterpret_cast<int32_t *>(p);
    p += align256(nt * 4);
    w.tile_sinc_last = reinterpret_cast<int32_t *>(p);
    p += align256(nt * 4);
    w.tfirst = reinterpret_cast<int32_t *>(p);
    p += align256(nt * 4);
    w.tlast = reinterpret_cast<int32_t *>(p);
    p += align256(nt * 4);
    w.bins = reinterpret_cast<int32_t *>(p);
    p += align256(((size_t)N / 8 + 2) * 4);
    w.u = reinterpret_cast<double *>(p);
    p += align256((size_t)N * 8);
    w.sinc = reinterpret_cast<int32_t *>(p);
    p += align256((size_t)N * 4);
    w.ex.tiles = reinterpret_cast<ExactTile *>(p);
    p += align256(nt * sizeof(ExactTile));
    w.ex.spec = reinterpret_cast<ExactSpecial *>(p);
    p += align256(nt * kExactCap * sizeof(ExactSpecial));
    w.ex.s_spec = reinterpret_cast<double *>(p);
    p += align256(nt * kExactCap * 8);
    w.ex.start = reinterpret_cast<double *>(p);
    p += align256(nt * 8);
    w.ex.s_out = reinterpret_cast<double *>(p);
    p += align256(nt * 8);
    w.ex.pk = reinterpret_cast<unsigned long long *>(p);
    p += align256(nt * 8);
    w.ex.rec = reinterpret_cast<double *>(p);
    p += align256((size_t)N * 8);
    w.ex.kint = reinterpret_cast<int32_t *>(p);
    p += align256((size_t)N * 4);
    w.ex.dirty = reinterpret_cast<int32_t *>(p);
    p += align256(nt * 4);
    w.ex.eaft = reinterpret_cast<int32_t *>(p);
    p += align256(nt * 4);
    w.exu.tiles = reinterpret_cast<ExactTile *>(p);
    p += align256(nt * sizeof(ExactTile));
    w.exu.spec = reinterpret_cast<ExactSpecial *>(p);
    p += align256(nt * kExactCap * sizeof(ExactSpecial));
    w.exu.s_spec = reinterpret_cast<double *>(p);
    p += align256(nt * kExactCap * 8);
    w.exu.start = reinterpret_cast<double *>(p);
    p += align256(nt * 8);
    w.exu.s_out = reinterpret_cast<double *>(p);
    p += align256(nt * 8);
    w.exu.pk = reinterpret_cast<unsigned long long *>(p);
    p += align256(nt * 8);
    w.exu.dirty = reinterpret_cast<int32_t *>(p);
    p += align256(nt * 4);
    w.exu.eaft = reinterpret_cast<int32_t *>(p);
    w.exu.rec = w.u;
    w.exu.kint = nullptr;
    return w;
}

// Kernels launch_resample_core issues (for the launch counters); the
// filters' FP64 weights add the normalisation pass (exact_norm), the mixed
// form's plain scan drops the residuals' exact sum (approx).
inline int resample_launches(int scheme, bool parity, bool exact_norm = false,
                             bool approx = false)
{
    const bool residual = scheme == VSMC_CUDA_RESIDUAL ||
                          scheme == VSMC_CUDA_RESIDUAL_STRATIFIED ||
                          scheme == VSMC_CUDA_RESIDUAL_SYSTEMATIC;
    const bool sys = scheme == VSMC_CUDA_SYSTEMATIC ||
                     scheme == VSMC_CUDA_RESIDUAL_SYSTEMATIC;
    const bool strat = scheme == VSMC_CUDA_STRATIFIED ||
                       scheme == VSMC_CUDA_RESIDUAL_STRATIFIED;
    int n = 5; // exact tiles and spine, invert, zero spine (and engine
               // position), cfrp fill
    if (residual)
        n += approx ? 2 : 4; // tile sums, spine, the residuals' exact sum
    if (exact_norm)
        n += 2;
    if (parity)
        n += 2;
    else if (strat)
        n += 1;
    else if (!sys)
        n += 5; // sorted sequence: terms, spine, exact scan, uniforms
    return n;
}

// Launch the scheme-specific part of a resampling (everything after the
// weight tile sums and spine when `spine_done`).  `u_given` (parity mode)
// replaces the device-drawn U01 sequence.
template <typename W>
inline void launch_resample_core(int scheme, W wsrc, long long N,
                                 const EngineRef &eng, ResampleWorkspace &ws,
                                 const double *u_given, long long n_given,
                                 bool spine_done, int32_t *rep_out,
                                 int32_t *copy_from, cudaStream_t s,
                                 bool sorted_ready = false, bool cfrp = true,
                                 long long Nout = 0)
{
    const int nt = resample_ntiles(N);
    // uniforms: up to the number of children (Nout when it is not N)
    const long long Nu = Nout > N ? Nout : N;
    const int ntu_dev = resample_ntiles(Nu);
    // spines of at most 256 tiles on 256 threads: each thread holds at most
    // one tile either way, so the sums are the same, with a quarter of the
    // CTA to synchronise
    const int spt = nt <= 256 ? 256 : kSpineThreads;
    const int sptu = ntu_dev <= 256 ? 256 : kSpineThreads;
    const bool residual = scheme == VSMC_CUDA_RESIDUAL ||
                          scheme == VSMC_CUDA_RESIDUAL_STRATIFIED ||
                          scheme == VSMC_CUDA_RESIDUAL_SYSTEMATIC;
    const bool sys = scheme == VSMC_CUDA_SYSTEMATIC ||
                     scheme == VSMC_CUDA_RESIDUAL_SYSTEMATIC;
    const bool strat = scheme == VSMC_CUDA_STRATIFIED ||
                       scheme == VSMC_CUDA_RESIDUAL_STRATIFIED;
    // the filters' FP64 weights: first the sequential sum of exp(lw - M),
    // whose reciprocal normalises them (on the approximate spine of the
    // weights, drawn here when the caller has none)
    W wx = wsrc;
    if (W::kExactNorm) {
        if (!spine_done) {
            k_tile_sums<W, false><<<nt, kThreads, 0, s>>>(
                wsrc, N, ws.ctl, ws.tile_sum, nullptr);
            if (sys)
                k_spine_weights<false, true><<<1, spt, 0, s>>>(
                    ws.tile_sum, nullptr, ws.tile_excl, nullptr, nt, N, eng,
                    ws.ctl);
            else
                k_spine_weights<false, false><<<1, spt, 0, s>>>(
                    ws.tile_sum, nullptr, ws.tile_excl, nullptr, nt, N, eng,
                    ws.ctl);
        }
        k_exact_tiles<W, false, true><<<exact_grid(nt), kThreads, 0, s>>>(
            wsrc, N, ws.ctl, ws.tile_excl, ws.ex);
        k_exact_spine<W, false, true><<<1, spt, 0, s>>>(
            wsrc, N, ws.ctl, nt, ws.ex);
        wx = with_exact_coeff(wsrc, &ws.ctl->coeff_w, ws.ex.rec);
    }
    if (residual) {
        k_tile_sums<W, true><<<nt, kThreads, 0, s>>>(wx, N, ws.ctl,
                                                    ws.tile_sum, ws.tile_k);
        if (sys)
            k_spine_weights<true, true><<<1, spt, 0, s>>>(
                ws.tile_sum, ws.tile_k, ws.tile_excl, ws.tile_kexcl, nt, N,
                eng, ws.ctl);
        else
            k_spine_weights<true, false><<<1, spt, 0, s>>>(
                ws.tile_sum, ws.tile_k, ws.tile_excl, ws.tile_kexcl, nt, N,
                eng, ws.ctl);
    } else if (!spine_done && !W::kExactNorm) {
        k_tile_sums<W, false><<<nt, kThreads, 0, s>>>(wx, N, ws.ctl,
                                                     ws.tile_sum, nullptr);
        if (sys)
            k_spine_weights<false, true><<<1, spt, 0, s>>>(
                ws.tile_sum, nullptr, ws.tile_excl, nullptr, nt, N, eng,
                ws.ctl);
        else
            k_spine_weights<false, false><<<1, spt, 0, s>>>(
                ws.tile_sum, nullptr, ws.tile_excl, nullptr, nt, N, eng,
                ws.ctl);
    }
    const double *u = ws.u;
    long long n_u = Nu;
    if (u_given != nullptr) {
        const int ntu = (int)((n_given + kTile - 1) / kTile);
        if (n_given > 0) {
            k_tile_max<<<ntu, kThreads, 0, s>>>(u_given, n_given,
                                                ws.u_tile_sum);
            k_apply_max<<<ntu, kThreads, 0, s>>>(u_given, n_given,
                                                 ws.u_tile_sum, ws.u, ws.ctl,
                                                 ws.bins);
        }
        n_u = n_given;
    } else if (strat) {
        const long long blocks = Nu / 4 + 2;
        k_uniforms_stratified<<<(unsigned)((blocks + kThreads - 1) / kThreads),
                                kThreads, 0, s>>>(eng, ws.ctl, ws.u,
                                                  ws.bins);
    } else if (!sys && !sorted_ready) {
        k_sorted_tile_sums<<<ntu_dev, kThreads, 0, s>>>(eng, ws.ctl,
                                                        ws.u_tile_sum, ws.u);
        k_sorted_spine<<<1, sptu, 0, s>>>(ws.u_tile_sum,
                                                   ws.u_tile_excl, ws.ctl);
        // lmax exactly: the exact scan of the negated terms
        const TermsNeg tn{ws.u, 0};
        k_exact_tiles<TermsNeg, false><<<exact_grid(ntu_dev), kThreads, 0, s>>>(
            tn, Nu, ws.ctl, ws.u_tile_excl, ws.exu);
        k_exact_spine<TermsNeg, false><<<1, sptu, 0, s>>>(
            tn, Nu, ws.ctl, ntu_dev, ws.exu);
        k_sorted_uniforms<<<ntu_dev, kThreads, 0, s>>>(ws.ctl, ws.exu, ws.u,
                                                       ws.bins);
    }
    const long long *kex = residual ? ws.tile_kexcl : nullptr;
    // the reference's sequential cumulative weight, exactly (for the
    // residual schemes first the sum of the residuals, whose reciprocal
    // scales them)
    if (residual) {
        if (!W::kApprox) {
            k_exact_tiles<W, true, true><<<exact_grid(nt), kThreads, 0, s>>>(
                wx, N, ws.ctl, ws.tile_excl, ws.ex);
            k_exact_spine<W, true, true><<<1, spt, 0, s>>>(
                wx, N, ws.ctl, nt, ws.ex);
        }
        k_exact_tiles<W, true><<<exact_grid(nt), kThreads, 0, s>>>(wx, N, ws.ctl,
                                                       ws.tile_excl, ws.ex);
        k_exact_spine<W, true><<<1, spt, 0, s>>>(wx, N, ws.ctl,
                                                           nt, ws.ex);
    } else {
        k_exact_tiles<W, false><<<exact_grid(nt), kThreads, 0, s>>>(wx, N, ws.ctl,
                                                        ws.tile_excl, ws.ex);
        k_exact_spine<W, false><<<1, spt, 0, s>>>(wx, N, ws.ctl,
                                                            nt, ws.ex);
    }
#define VSMC_INVERT(R, S)                                                     \
    k_invert<W, R, S><<<nt, kThreads, 0, s>>>(                                \
        wx, N, ws.ctl, ws.tile_excl, kex, u, n_u, ws.bins, rep_out,        \
        copy_from, ws.sinc, ws.tile_zeros, ws.tile_sinc_last, ws.ex)
    if (residual && sys)
        VSMC_INVERT(true, true);
    else if (residual)
        VSMC_INVERT(true, false);
    else if (sys)
        VSMC_INVERT(false, true);
    else
        VSMC_INVERT(false, false);
#undef VSMC_INVERT
    if (cfrp) {
        // the spine kernel also advances the engine position
        k_zero_spine<<<1, spt, 0, s>>>(
            ws.tile_zeros, ws.tile_sinc_last, ws.zexcl, ws.tfirst, ws.tlast,
            nt, ws.ctl);
        k_cfrp_fill<<<nt, kThreads, 0, s>>>(N, ws.ctl, ws.sinc, ws.zexcl,
                                            ws.tfirst, ws.tlast, copy_from);
    } else {
        k_resample_done<<<1, 1, 0, s>>>(ws.ctl);
    }
}

// internal::cfrp_trans for M != N (resample/common.hpp:110-117): parent i
// fills the next rep[i] slots, so copy_from is the parents in order, each
// repeated rep[i] times.  Per-tile sums of rep, their exclusive spine, the
// inclusive prefix P of rep, then slot j takes the first parent with
// P > j (a binary search per slot keeps a parent with many children from
// serialising its tile).
static __global__ void __launch_bounds__(kThreads)
k_rep_tile_sums(const int32_t *rep, long long M, long long *tile_sum)
{
    __shared__ long long sh[kThreads / 32];
    const long long base = (long long)blockIdx.x * kTile;
    long long v = 0;
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const long long i = base + (long long)j * kThreads + threadIdx.x;
        if (i < M)
            v += rep[i];
    }
    long long total;
    block_excl_scan(v, sh, total);
    if (threadIdx.x == 0)
        tile_sum[blockIdx.x] = total;
}

static __global__ void __launch_bounds__(kSpineThreads)
k_rep_spine(const long long *tile_sum, long long *tile_excl, int ntiles)
{
    __shared__ long long sh[kSpineThreads / 32];
    spine_scan_ll(tile_sum, tile_excl, ntiles, sh);
}

static __global__ void __launch_bounds__(kThreads)
k_rep_prefix(const int32_t *rep, long long M, const long long *tile_excl,
             int32_t *incl)
{
    __shared__ long long sh[kThreads / 32];
    const long long base = (long long)blockIdx.x * kTile;
    const long long i0 = base + (long long)threadIdx.x * kItems;
    long long r[kItems];
    long long run = 0;
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        r[j] = i0 + j < M ? rep[i0 + j] : 0;
        run += r[j];
    }
    long long total;
    long long off = block_excl_scan(run, sh, total) + tile_excl[blockIdx.x];
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        off += r[j];
        if (i0 + j < M)
            incl[i0 + j] = (int32_t)off;
    }
}

static __global__ void k_expand_fill(const int32_t *incl, long long M,
                                     long long N, int32_t *copy_from)
{
    const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= N)
        return;
    long long lo = 0, hi = M - 1; // incl[M - 1] == N > j
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        if (incl[mid] > j)
            hi = mid;
        else
            lo = mid + 1;
    }
    copy_from[j] = (int32_t)lo;
}

// The launches of the M != N copy_from (4 kernels).
inline void launch_expand(const int32_t *rep, long long M, long long N,
                          ResampleWorkspace &ws, int32_t *copy_from,
                          cudaStream_t s)
{
    const int nt = resample_ntiles(M);
    k_rep_tile_sums<<<nt, kThreads, 0, s>>>(rep, M, ws.tile_k);
    k_rep_spine<<<1, kSpineThreads, 0, s>>>(ws.tile_k, ws.tile_kexcl, nt);
    k_rep_prefix<<<nt, kThreads, 0, s>>>(rep, M, ws.tile_kexcl, ws.sinc);
    k_expand_fill<<<(unsigned)((N + 255) / 256), 256, 0, s>>>(ws.sinc, M, N,
                                                               copy_from);
}

// The speculative Multinomial sequence for the next resampling (see
// sorted_run); 6 launches on `s`.
inline void launch_spec_sorted(long long N, const EngineRef &eng,
                               ResampleWorkspace &ws, cudaStream_t s)
{
    const int nt = resample_ntiles(N);
    k_spec_tile_sums<<<nt, kThreads, 0, s>>>(eng, ws.ctl, N, ws.u_tile_sum,
                                             ws.u);
    k_spec_spine<<<1, kSpineThreads, 0, s>>>(ws.u_tile_sum, ws.u_tile_excl,
                                             ws.ctl, N);
    const TermsNeg tn{ws.u, N};
    k_exact_tiles<TermsNeg, false><<<exact_grid(nt), kThreads, 0, s>>>(
        tn, N, ws.ctl, ws.u_tile_excl, ws.exu);
    k_exact_spine<TermsNeg, false><<<1, kSpineThreads, 0, s>>>(
        tn, N, ws.ctl, nt, ws.exu);
    k_spec_uniforms<<<nt, kThreads, 0, s>>>(ws.ctl, N, ws.exu, ws.u,
                                            ws.bins);
    k_spec_commit<<<1, 1, 0, s>>>(ws.ctl);
}

} // namespace vsmc_b200
