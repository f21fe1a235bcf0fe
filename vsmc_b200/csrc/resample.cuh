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

namespace vsmc_b200 {

// Device-side control block of one resampling call.
struct ResampleCtl {
    int active;           // 0: every resample kernel returns at once
    int error;            // sticky vsmc_cuda_status
    long long NN;         // length of the U01 sequence fed to inversion
    double coeff_r;       // 1 / sum of residuals
    double delta;         // 1 / NN
    double u0;            // systematic start
    long long n_final;    // uniforms consumed by particles 0..N-2
    unsigned long long words;   // engine words drawn by this call
    unsigned long long offset;  // engine offset before the call
    unsigned long long ticket;  // dynamic tile counter of the invert kernel
};

struct EngineRef {
    u64x4 key;
    u64x4 ctr;
};

// Weight sources --------------------------------------------------------
// Normalised weights given in memory (generic C ABI).
struct WeightsGiven {
    const double *w;
    __device__ __forceinline__ void prepare() {}
    __device__ __forceinline__ double operator()(long long i) const
    {
        return w[i];
    }
};

// Weights of a filter: w_i = exp(lw_i - M) * (1 / S1), i.e. the reference's
// normalize_log_weight, vExp and normalize_weight (core/weight_set.hpp:
// 108-125) evaluated on the fly from raw log-weights.
template <typename Real>
struct WeightsFromLog {
    const Real *lw;
    const double *stats; // [0] = M (max log-weight), [1] = S1
    double M, coeff;
    __device__ __forceinline__ void prepare()
    {
        M = stats[0];
        coeff = __ddiv_rn(1.0, stats[1]);
    }
    __device__ __forceinline__ double operator()(long long i) const;
};

template <>
__device__ __forceinline__ double
WeightsFromLog<double>::operator()(long long i) const
{
    return __dmul_rn(exp(__dadd_rn(lw[i], -M)), coeff);
}

template <>
__device__ __forceinline__ double
WeightsFromLog<float>::operator()(long long i) const
{
    return __dmul_rn(static_cast<double>(expf(lw[i] - static_cast<float>(M))),
                     coeff);
}

// Residual split of a weight: r = modf(N w, &k) (residual.hpp:61-62).
__device__ __forceinline__ double residual_split(double w, double Nd,
                                                 double &k)
{
    return modf(__dmul_rn(Nd, w), &k);
}

// ---------------------------------------------------------------------------
// Tile sums of the weights (or, residual, of r and k).
template <typename W, bool Residual>
__global__ void __launch_bounds__(kThreads)
k_tile_sums(W wsrc, long long N, const ResampleCtl *ctl, double *tile_sum,
            long long *tile_k)
{
    if (!ctl->active)
        return;
    __shared__ double shd[kThreads / 32];
    __shared__ long long shk[kThreads / 32];
    wsrc.prepare();
    const long long base = (long long)blockIdx.x * kTile;
    const double Nd = (double)N;
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
        tile_sum[blockIdx.x] = t;
        if (Residual)
            tile_k[blockIdx.x] = kt;
    }
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
    for (int t = b; t < e; ++t)
        run += __dmul_rn(in[t], scale);
    double total;
    const double off = block_excl_scan(run, sh, total);
    run = off;
    for (int t = b; t < e; ++t) {
        excl[t] = run;
        run += __dmul_rn(in[t], scale);
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
__global__ void __launch_bounds__(kSpineThreads)
k_spine_weights(const double *tile_sum, const long long *tile_k,
                double *tile_excl, long long *tile_kexcl, int ntiles,
                long long N, EngineRef eng, ResampleCtl *ctl)
{
    if (!ctl->active)
        return;
    __shared__ double shd[kSpineThreads / 32];
    __shared__ long long shk[kSpineThreads / 32];
    __shared__ double coeff_sh;
    long long NN = N;
    double coeff = 1.0;
    if (Residual) {
        spine_scan_ll(tile_k, tile_kexcl, ntiles, shk);
        __syncthreads();
        // asum of the residuals in the spine's fixed order
        const int per = (ntiles + blockDim.x - 1) / blockDim.x;
        double run = 0.0;
        for (int t = threadIdx.x * per; t < min((int)(threadIdx.x + 1) * per, ntiles); ++t)
            run += tile_sum[t];
        double total;
        block_excl_scan(run, shd, total);
        if (threadIdx.x == 0)
            coeff_sh = __ddiv_rn(1.0, total);
        __syncthreads();
        coeff = coeff_sh;
        NN = N - tile_kexcl[ntiles];
    }
    spine_scan_f64(tile_sum, tile_excl, ntiles, coeff, shd);
    if (threadIdx.x == 0) {
        ctl->NN = NN;
        ctl->coeff_r = coeff;
        ctl->delta = __ddiv_rn(1.0, (double)NN);
        ctl->n_final = 0;
        ctl->ticket = 0;
        if (Sys) {
            const uint64_t w = threefry_word(eng.key, eng.ctr, ctl->offset);
            ctl->u0 = __dmul_rn(canonical_u64(w), ctl->delta);
            ctl->words = 1;
        } else {
            ctl->words = 0;
        }
    }
}

// Stratified U01 sequence (U01SequenceStratified, u01.hpp:212-243):
// u_n = U_n * delta + n * delta, U_n from engine word offset + n.  Adjacent
// values can cross by rounding only between neighbours, so the running
// maximum is max(u_n, u_{n-1}).
static __global__ void __launch_bounds__(kThreads)
k_uniforms_stratified(EngineRef eng, const ResampleCtl *ctl, double *u)
{
    if (!ctl->active)
        return;
    const long long NN = ctl->NN;
    const double delta = ctl->delta;
    const unsigned long long off = ctl->offset;
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= NN)
        return;
    const double a = __dadd_rn(
        __dmul_rn(canonical_u64(threefry_word(eng.key, eng.ctr, off + n)),
                  delta),
        __dmul_rn((double)n, delta));
    double v = a;
    if (n > 0) {
        const double p = __dadd_rn(
            __dmul_rn(canonical_u64(threefry_word(eng.key, eng.ctr,
                                                  off + n - 1)),
                      delta),
            __dmul_rn((double)(n - 1), delta));
        v = fmax(a, p);
    }
    u[n] = v;
}

// Sorted U01 sequence (U01SequenceSorted, u01.hpp:165-202): lmax_n =
// sum_{k<=n} log(1 - U_k) / (NN - k); u_n = 1 - exp(lmax_n).  Two passes
// over tiles of kTile uniforms around a deterministic spine.
__device__ __forceinline__ double sorted_term(const EngineRef &eng,
                                              unsigned long long off,
                                              long long n, long long NN)
{
    const double U = canonical_u64(threefry_word(eng.key, eng.ctr, off + n));
    return __ddiv_rn(log(__dadd_rn(1.0, -U)), (double)(NN - n));
}

static __global__ void __launch_bounds__(kThreads)
k_sorted_tile_sums(EngineRef eng, const ResampleCtl *ctl, double *tile_sum)
{
    if (!ctl->active)
        return;
    __shared__ double sh[kThreads / 32];
    const long long NN = ctl->NN;
    const long long base = (long long)blockIdx.x * kTile;
    if (base >= NN)
        return;
    double s = 0.0;
    for (int j = 0; j < kItems; ++j) {
        const long long n = base + (long long)threadIdx.x * kItems + j;
        if (n < NN)
            s += sorted_term(eng, ctl->offset, n, NN);
    }
    double total;
    block_excl_scan(s, sh, total);
    if (threadIdx.x == 0)
        tile_sum[blockIdx.x] = total;
}

static __global__ void __launch_bounds__(kSpineThreads)
k_sorted_spine(const double *tile_sum, double *tile_excl,
               const ResampleCtl *ctl)
{
    if (!ctl->active)
        return;
    __shared__ double sh[kSpineThreads / 32];
    const int ntiles = (int)((ctl->NN + kTile - 1) / kTile);
    spine_scan_f64(tile_sum, tile_excl, ntiles, 1.0, sh);
}

static __global__ void __launch_bounds__(kThreads)
k_sorted_uniforms(EngineRef eng, const ResampleCtl *ctl,
                  const double *tile_excl, double *u)
{
    if (!ctl->active)
        return;
    __shared__ double sh[kThreads / 32];
    const long long NN = ctl->NN;
    const long long base = (long long)blockIdx.x * kTile;
    if (base >= NN)
        return;
    const long long last = min(base + (long long)kTile, NN) - 1;
    double t[kItems];
    double run = 0.0;
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const long long n = base + (long long)threadIdx.x * kItems + j;
        t[j] = n < NN ? sorted_term(eng, ctl->offset, n, NN) : 0.0;
        run += t[j];
    }
    double total;
    double pre = block_excl_scan(run, sh, total);
    const double a = tile_excl[blockIdx.x];
    const double b = tile_excl[blockIdx.x + 1];
    // carry: the previous tile ends exactly at lmax = a
    double umax = blockIdx.x > 0 ? __dadd_rn(1.0, -exp(a)) : -INFINITY;
    double uv[kItems];
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const long long n = base + (long long)threadIdx.x * kItems + j;
        pre += t[j];
        double lmax = fmax(__dadd_rn(a, pre), b); // lmax is non-increasing
        if (n == last)
            lmax = b;
        uv[j] = __dadd_rn(1.0, -exp(lmax));
    }
    // running max within the thread, then across the block
    double tmax = -INFINITY;
#pragma unroll
    for (int j = 0; j < kItems; ++j)
        tmax = fmax(tmax, uv[j]);
    // block exclusive max-scan via shared memory
    __shared__ double shm[kThreads];
    shm[threadIdx.x] = tmax;
    __syncthreads();
    for (int o = 1; o < kThreads; o <<= 1) {
        const double v = threadIdx.x >= (unsigned)o ? shm[threadIdx.x - o]
                                                    : -INFINITY;
        __syncthreads();
        shm[threadIdx.x] = fmax(shm[threadIdx.x], v);
        __syncthreads();
    }
    double m = threadIdx.x > 0 ? fmax(umax, shm[threadIdx.x - 1]) : umax;
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const long long n = base + (long long)threadIdx.x * kItems + j;
        m = fmax(m, uv[j]);
        if (n < NN)
            u[n] = m;
    }
}

// ---------------------------------------------------------------------------
// Count of the U01 sequence values <= C ("first n with u_n > C", which for a
// non-decreasing sequence is the upper bound).
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

constexpr int kUStage = kTile; // uniforms staged in shared memory per tile (the
                                // weight buffer is reused, kTile doubles)
constexpr unsigned long long kSpinLimit = 1ull << 22;

// Look-back status word: bits 62-63 flag (1 aggregate, 2 inclusive prefix),
// low 32 bits the zero-slot count.
__device__ __forceinline__ void lb_publish(unsigned long long *st, int flag,
                                           unsigned count)
{
    const unsigned long long v =
        ((unsigned long long)flag << 62) | (unsigned long long)count;
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(st), "l"(v)
                 : "memory");
}

__device__ __forceinline__ unsigned long long lb_load(
    const unsigned long long *st)
{
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];"
                 : "=l"(v)
                 : "l"(st)
                 : "memory");
    return v;
}

// The inversion + cfrp ranks kernel.  Residual: weights are r * coeff_r and
// k = floor(N w) is added back (residual.hpp:59-76).  Sys: closed-form
// count.  Outputs: replication (optional), copy_from (self for survivors,
// -(rank+1) for the rank-th zero slot) and sinc (inclusive count of surplus
// children, sum_{j<=i} max(rep_j - 1, 0)).
template <typename W, bool Residual, bool Sys>
__global__ void __launch_bounds__(kThreads)
k_invert(W wsrc, long long N, ResampleCtl *ctl, const double *tile_excl,
         const long long *tile_kexcl, const double *u, long long n_u,
         unsigned long long *lb_status, int32_t *rep_out, int32_t *copy_from,
         int32_t *sinc)
{
    if (!ctl->active)
        return;
    __shared__ double sw[kTile];         // weights, then staged uniforms
    __shared__ double sk[Residual ? kTile : 1]; // floor(N w) (residual)
    __shared__ long long shl[kThreads / 32];
    __shared__ double shd[kThreads / 32];
    __shared__ long long sh_bound[2];
    __shared__ unsigned sh_zexcl;
    __shared__ unsigned sh_tile;
    wsrc.prepare();

    if (threadIdx.x == 0)
        sh_tile = (unsigned)atomicAdd(&ctl->ticket, 1ull);
    __syncthreads();
    const int tile = (int)sh_tile;
    const long long base = (long long)tile * kTile;
    const long long NN = ctl->NN;
    const double Nd = (double)N;
    const double coeff_r = Residual ? ctl->coeff_r : 1.0;
    const double u0 = Sys ? ctl->u0 : 0.0;
    const double delta = ctl->delta;
    const long long nu = Sys ? NN : min(NN, n_u);

    // striped (coalesced) load of the tile's weights into shared memory
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const int l = j * kThreads + threadIdx.x;
        const long long i = base + l;
        double w = 0.0, k = 0.0;
        if (i < N) {
            w = wsrc(i);
            if (Residual)
                w = __dmul_rn(residual_split(w, Nd, k), coeff_r);
        }
        sw[l] = w;
        if (Residual)
            sk[l] = k;
    }
    __syncthreads();
    double wv[kItems];
    double run = 0.0;
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        wv[j] = sw[threadIdx.x * kItems + j];
        run += wv[j];
    }
    double total;
    double pre = block_excl_scan(run, shd, total);
    const double a = tile_excl[tile];
    const double b = tile_excl[tile + 1];

    // uniforms that can fall in this tile: (ub(a), ub(b)]
    if (threadIdx.x == 0) {
        if (Sys) {
            sh_bound[0] = tile > 0 ? sys_count(a, u0, delta, NN) : 0;
            sh_bound[1] = sys_count(b, u0, delta, NN);
        } else {
            sh_bound[0] = tile > 0 ? ub_global(u, 0, nu, a) : 0;
            sh_bound[1] = ub_global(u, sh_bound[0], nu, b);
        }
    }
    __syncthreads(); // also: every thread has read sw
    const long long lo = sh_bound[0];
    const long long hi = max(sh_bound[1], lo);
    const bool staged = !Sys && (hi - lo) <= kUStage;
    if (staged) {
        for (long long n = lo + threadIdx.x; n < hi; n += kThreads)
            sw[n - lo] = u[n];
    }
    __syncthreads();

    // counts c_i = #{n: u_n <= C_i} for this thread's particles
    long long cnt[kItems];
    long long k_int[kItems];
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const long long i = base + (long long)threadIdx.x * kItems + j;
        pre += wv[j];
        double C = fmin(__dadd_rn(a, pre), b);
        if (i == base + kTile - 1 || i == N - 1)
            C = b;
        long long c;
        if (i >= N - 1) {
            c = NN; // the last particle takes every remaining uniform
        } else if (Sys) {
            c = sys_count(C, u0, delta, NN);
        } else if (staged) {
            c = lo + ub_shared(sw, 0, (int)(hi - lo), C);
        } else {
            c = ub_global(u, lo, hi, C);
        }
        cnt[j] = min(max(c, lo), i >= N - 1 ? NN : hi);
        k_int[j] = Residual ? (long long)sk[threadIdx.x * kItems + j] : 0;
    }
    // non-decreasing counts within the thread; neighbour's last count
#pragma unroll
    for (int j = 1; j < kItems; ++j)
        cnt[j] = max(cnt[j], cnt[j - 1]);
    long long prev = __shfl_up_sync(0xffffffffu, cnt[kItems - 1], 1);
    __shared__ long long sh_last[kThreads / 32];
    if ((threadIdx.x & 31) == 31)
        sh_last[threadIdx.x >> 5] = cnt[kItems - 1];
    __syncthreads();
    if ((threadIdx.x & 31) == 0)
        prev = (threadIdx.x == 0) ? (tile > 0 ? lo : 0)
                                  : sh_last[(threadIdx.x >> 5) - 1];
    // warp-level running max of prev across threads is implied by the
    // per-thread clamps to [lo, hi] and the monotone C_i.
    long long rep[kItems];
    unsigned zeros = 0;
    long long ksum = 0;
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const long long i = base + (long long)threadIdx.x * kItems + j;
        const long long c = max(cnt[j], prev);
        rep[j] = (i < N) ? (c - prev) + k_int[j] : 0;
        prev = c;
        cnt[j] = c;
        zeros += (i < N && rep[j] == 0) ? 1u : 0u;
        ksum += k_int[j];
    }
    // the last queried uniform fixes the words drawn (inversion queries
    // u_0..u_{n_final}, common.hpp:76-81)
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const long long i = base + (long long)threadIdx.x * kItems + j;
        if (i == N - 2) {
            ctl->n_final = cnt[j];
            if (!Sys)
                ctl->words = (NN > 0) ? (unsigned long long)min(NN, cnt[j] + 1)
                                      : 0ull;
        }
    }

    // zero-slot counts: block scan, then the tile look-back
    long long ztot;
    const long long zex_thread = block_excl_scan((long long)zeros, shl, ztot);
    long long ktot;
    const long long kex_thread = Residual ? block_excl_scan(ksum, shl, ktot)
                                          : 0;
    if (threadIdx.x == 0) {
        unsigned long long *st = lb_status + tile;
        if (tile == 0) {
            lb_publish(st, 2, (unsigned)ztot);
            sh_zexcl = 0;
        } else {
            lb_publish(st, 1, (unsigned)ztot);
            unsigned excl = 0;
            int p = tile - 1;
            unsigned long long spins = 0;
            while (p >= 0) {
                const unsigned long long v = lb_load(lb_status + p);
                const int flag = (int)(v >> 62);
                if (flag == 0) {
                    if (++spins > kSpinLimit) {
                        atomicExch(&ctl->error, (int)VSMC_CUDA_ETIMEOUT);
                        break;
                    }
                    __nanosleep(32);
                    continue;
                }
                excl += (unsigned)(v & 0xffffffffull);
                if (flag == 2)
                    break;
                --p;
            }
            lb_publish(st, 2, excl + (unsigned)ztot);
            sh_zexcl = excl;
        }
    }
    __syncthreads();
    long long zeros_before = (long long)sh_zexcl + zex_thread;
    const long long kbase = Residual ? tile_kexcl[tile] + kex_thread : 0;
    long long kprefix = kbase;
    int32_t cf[kItems], sc[kItems], rp[kItems];
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const long long i = base + (long long)threadIdx.x * kItems + j;
        kprefix += k_int[j];
        // R_{<=i} = count_i + K_{<=i}; the last particle closes at N
        const long long R = (i >= N - 1) ? N : cnt[j] + kprefix;
        if (rep[j] == 0) {
            cf[j] = (int32_t)(-(zeros_before + 1));
            ++zeros_before;
        } else {
            cf[j] = (int32_t)i;
        }
        sc[j] = (int32_t)(R - (i + 1) + zeros_before);
        rp[j] = (int32_t)rep[j];
    }
    // stage the three outputs through shared memory for coalesced stores
    __syncthreads();
    int32_t *s32 = reinterpret_cast<int32_t *>(sw);
#pragma unroll
    for (int j = 0; j < kItems; ++j)
        s32[threadIdx.x * kItems + j] = cf[j];
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const long long i = base + (long long)j * kThreads + threadIdx.x;
        if (i < N)
            copy_from[i] = s32[j * kThreads + threadIdx.x];
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kItems; ++j)
        s32[threadIdx.x * kItems + j] = sc[j];
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const long long i = base + (long long)j * kThreads + threadIdx.x;
        if (i < N)
            sinc[i] = s32[j * kThreads + threadIdx.x];
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

// Parent of the rank-th surplus child: the first p with sinc[p] > rank,
// found by galloping outwards from the zero slot's own index.
__device__ __forceinline__ int32_t cfrp_parent(const int32_t *sinc,
                                               long long N, long long i,
                                               long long rank)
{
    long long lo, hi; // invariant: sinc[lo] <= rank < sinc[hi] (virtual ends)
    if (sinc[i] > rank) {
        hi = i;
        long long step = 1;
        lo = i - 1;
        while (lo >= 0 && sinc[lo] > rank) {
            hi = lo;
            lo = i - (step <<= 1);
        }
        if (lo < -1)
            lo = -1;
    } else {
        lo = i;
        long long step = 1;
        hi = i + 1;
        while (hi < N && sinc[hi] <= rank) {
            lo = hi;
            hi = i + (step <<= 1);
        }
        if (hi > N)
            hi = N;
    }
    while (hi - lo > 1) {
        const long long mid = lo + ((hi - lo) >> 1);
        if (sinc[mid] > rank)
            hi = mid;
        else
            lo = mid;
    }
    return (int32_t)hi; // N when no parent exists (caller checks)
}

// internal::cfrp_trans for the zero slots (common.hpp:94-106): the k-th
// slot without offspring takes the k-th surplus child in parent order.
static __global__ void __launch_bounds__(kThreads)
k_cfrp_fill(long long N, const ResampleCtl *ctl, const int32_t *sinc,
            int32_t *copy_from)
{
    if (!ctl->active)
        return;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N)
        return;
    const int32_t c = copy_from[i];
    if (c >= 0)
        return;
    const int32_t p = cfrp_parent(sinc, N, i, (long long)(-c) - 1);
    if (p >= N) { // replication did not sum to N: never index past the end
        atomicExch(const_cast<int *>(&ctl->error), (int)VSMC_CUDA_EDEGENERATE);
        copy_from[i] = (int32_t)i;
        return;
    }
    copy_from[i] = p;
}

// Finalise the engine position.
static __global__ void k_resample_done(ResampleCtl *ctl)
{
    if (!ctl->active)
        return;
    ctl->offset += ctl->words;
}

// Running maximum of caller-supplied uniforms (parity mode): tile maxima,
// spine, apply.
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
k_apply_max(const double *u, long long n, const double *tile_max, double *out)
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
    for (int j = 0; j < kItems; ++j) {
        const long long i = base + (long long)threadIdx.x * kItems + j;
        m = fmax(m, v[j]);
        if (i < n)
            out[i] = m;
    }
}

// ------------------------------------------------------------ host side --
struct ResampleWorkspace {
    ResampleCtl *ctl;
    double *tile_sum;     // ntiles + 1
    double *tile_excl;    // ntiles + 1
    long long *tile_k;    // ntiles + 1
    long long *tile_kexcl; // ntiles + 1
    double *u;            // N
    double *u_tile_sum;   // ntiles + 1
    double *u_tile_excl;  // ntiles + 1
    unsigned long long *lb_status; // ntiles
    int32_t *sinc;        // N
};

inline int resample_ntiles(long long N)
{
    return (int)((N + kTile - 1) / kTile);
}

inline size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

inline size_t resample_workspace_bytes(long long N)
{
    const size_t nt = (size_t)resample_ntiles(N) + 1;
    return align256(sizeof(ResampleCtl)) + 6 * align256(nt * 8) +
           align256(nt * 8) /* lb */ + align256((size_t)N * 8) +
           align256((size_t)N * 4);
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
    w.lb_status = reinterpret_cast<unsigned long long *>(p);
    p += align256(nt * 8);
    w.u = reinterpret_cast<double *>(p);
    p += align256((size_t)N * 8);
    w.sinc = reinterpret_cast<int32_t *>(p);
    return w;
}

// Kernels launch_resample_core issues (for the launch counters).
inline int resample_launches(int scheme, bool parity)
{
    const bool residual = scheme == VSMC_CUDA_RESIDUAL ||
                          scheme == VSMC_CUDA_RESIDUAL_STRATIFIED ||
                          scheme == VSMC_CUDA_RESIDUAL_SYSTEMATIC;
    const bool sys = scheme == VSMC_CUDA_SYSTEMATIC ||
                     scheme == VSMC_CUDA_RESIDUAL_SYSTEMATIC;
    const bool strat = scheme == VSMC_CUDA_STRATIFIED ||
                       scheme == VSMC_CUDA_RESIDUAL_STRATIFIED;
    int n = 3; // invert, cfrp fill, done
    if (residual)
        n += 2;
    if (parity)
        n += 2;
    else if (strat)
        n += 1;
    else if (!sys)
        n += 3;
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
                                 int32_t *copy_from, cudaStream_t s)
{
    const int nt = resample_ntiles(N);
    const bool residual = scheme == VSMC_CUDA_RESIDUAL ||
                          scheme == VSMC_CUDA_RESIDUAL_STRATIFIED ||
                          scheme == VSMC_CUDA_RESIDUAL_SYSTEMATIC;
    const bool sys = scheme == VSMC_CUDA_SYSTEMATIC ||
                     scheme == VSMC_CUDA_RESIDUAL_SYSTEMATIC;
    const bool strat = scheme == VSMC_CUDA_STRATIFIED ||
                       scheme == VSMC_CUDA_RESIDUAL_STRATIFIED;
    if (residual) {
        k_tile_sums<W, true><<<nt, kThreads, 0, s>>>(wsrc, N, ws.ctl,
                                                    ws.tile_sum, ws.tile_k);
        if (sys)
            k_spine_weights<true, true><<<1, kSpineThreads, 0, s>>>(
                ws.tile_sum, ws.tile_k, ws.tile_excl, ws.tile_kexcl, nt, N,
                eng, ws.ctl);
        else
            k_spine_weights<true, false><<<1, kSpineThreads, 0, s>>>(
                ws.tile_sum, ws.tile_k, ws.tile_excl, ws.tile_kexcl, nt, N,
                eng, ws.ctl);
    } else if (!spine_done) {
        k_tile_sums<W, false><<<nt, kThreads, 0, s>>>(wsrc, N, ws.ctl,
                                                     ws.tile_sum, nullptr);
        if (sys)
            k_spine_weights<false, true><<<1, kSpineThreads, 0, s>>>(
                ws.tile_sum, nullptr, ws.tile_excl, nullptr, nt, N, eng,
                ws.ctl);
        else
            k_spine_weights<false, false><<<1, kSpineThreads, 0, s>>>(
                ws.tile_sum, nullptr, ws.tile_excl, nullptr, nt, N, eng,
                ws.ctl);
    }
    const double *u = ws.u;
    long long n_u = N;
    if (u_given != nullptr) {
        const int ntu = (int)((n_given + kTile - 1) / kTile);
        if (n_given > 0) {
            k_tile_max<<<ntu, kThreads, 0, s>>>(u_given, n_given,
                                                ws.u_tile_sum);
            k_apply_max<<<ntu, kThreads, 0, s>>>(u_given, n_given,
                                                 ws.u_tile_sum, ws.u);
        }
        n_u = n_given;
    } else if (strat) {
        k_uniforms_stratified<<<(unsigned)((N + kThreads - 1) / kThreads),
                                kThreads, 0, s>>>(eng, ws.ctl, ws.u);
    } else if (!sys) {
        k_sorted_tile_sums<<<nt, kThreads, 0, s>>>(eng, ws.ctl,
                                                   ws.u_tile_sum);
        k_sorted_spine<<<1, kSpineThreads, 0, s>>>(ws.u_tile_sum,
                                                   ws.u_tile_excl, ws.ctl);
        k_sorted_uniforms<<<nt, kThreads, 0, s>>>(eng, ws.ctl,
                                                  ws.u_tile_excl, ws.u);
    }
    cudaMemsetAsync(ws.lb_status, 0, sizeof(unsigned long long) * nt, s);
    const long long *kex = residual ? ws.tile_kexcl : nullptr;
#define VSMC_INVERT(R, S)                                                     \
    k_invert<W, R, S><<<nt, kThreads, 0, s>>>(wsrc, N, ws.ctl, ws.tile_excl,  \
                                              kex, u, n_u, ws.lb_status,     \
                                              rep_out, copy_from, ws.sinc)
    if (residual && sys)
        VSMC_INVERT(true, true);
    else if (residual)
        VSMC_INVERT(true, false);
    else if (sys)
        VSMC_INVERT(false, true);
    else
        VSMC_INVERT(false, false);
#undef VSMC_INVERT
    k_cfrp_fill<<<(unsigned)((N + kThreads - 1) / kThreads), kThreads, 0,
                  s>>>(N, ws.ctl, ws.sinc, copy_from);
    k_resample_done<<<1, 1, 0, s>>>(ws.ctl);
}

} // namespace vsmc_b200
