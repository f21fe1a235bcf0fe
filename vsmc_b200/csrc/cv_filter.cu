// cv_filter.cu -- the constant-velocity Student-t bootstrap filter as one
// device-resident Sampler (FP64 and mixed FP32/FP64 forms).
//
// Reference: example/pf/include/pf_smp.hpp:73-258 (model), core/sampler.hpp:
// 450-483 and 758-834 (initialize / iterate / do_resample / do_monitor),
// core/weight_set.hpp:108-125, 441-446 (normalisation and ESS), example/
// include/move_smc.hpp:63-71 (log-evidence increment), core/monitor.hpp:
// 274-302 with integrate/is_integrate.hpp:56-80 (posterior mean).
//
// One step = k_cv_move (gather of the previous resampling fused into the
// load, move, likelihood, log-weight update, per-tile online log-sum-exp
// statistics) + k_cv_finalize (one CTA: max, sum, ESS, log-evidence,
// monitor, resampling decision and the weight spine) + the resampling
// kernels of resample.cuh, which return at once when the step does not
// resample.  No host round trip happens inside a step.
#include "resample.cuh"

#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

namespace vsmc_b200 {

void set_last_error(const std::string &msg);
int cuda_status(cudaError_t e, const char *what);

struct FilterCtl {
    double lw_max;  // M: raw log-weights minus M are the reference's lw
    double s1;      // sum exp(lw - M)
    double s2;
    double ess;
    double logz;
    int resampled;  // the last finished step resampled
    int error;
    long long monitor_done; // step whose gathered monitor is already written
};

// Per-tile statistics of the new log-weights: online log-sum-exp (m, s1, s2),
// the weighted position sums (sx, sy) and the sums of the gathered previous
// positions (gx, gy) for the monitor of a resampled step.
struct TileStats {
    double m, s1, s2, sx, sy, gx, gy, pad;
};

struct CVParam {
    double dt, sd_pos, sd_vel, sd_pos0, sd_vel0, scale, nu;
    double inv_nu; // 1 / nu
    double coef;   // -(nu + 1) / 2
};

template <typename Real>
struct MoveArgs {
    const Real *in[4];
    Real *out[4];
    Real *lw;
    const int32_t *copy_from;
    const FilterCtl *ctl;
    const double *obs_x;
    const double *obs_y;
    TileStats *tile_stats;
    long long N;
    int ntiles;
    uint32_t iter, k0, k1, stream;
    CVParam p;
};

template <typename Real>
struct Vec;
template <>
struct Vec<double> {
    static constexpr int n = 2;
    typedef double2 type;
};
template <>
struct Vec<float> {
    static constexpr int n = 4;
    typedef float4 type;
};

__device__ __forceinline__ double plus0(double v) { return __dadd_rn(v, 0.0); }

__device__ __forceinline__ PhiloxStream particle_stream(uint32_t iter,
                                                        uint32_t id,
                                                        uint32_t stream,
                                                        uint32_t k0,
                                                        uint32_t k1)
{
    PhiloxStream s;
    s.ctr = make_uint4(0u, iter, id, stream);
    s.k0 = k0;
    s.k1 = k1;
    return s;
}

// FP64 form: cv_move::move_state / cv_init::initialize_state
// (pf_smp.hpp:150-173, 207-238).  The two polar points are drawn first and
// their transforms evaluated together (independent chains for the FP64
// pipe); the state update keeps the reference's evaluation order.
template <bool Init>
__device__ __forceinline__ void cv_particle(const CVParam &p, uint32_t iter,
                                            uint32_t id, uint32_t stream,
                                            uint32_t k0, uint32_t k1,
                                            double &x, double &y, double &vx,
                                            double &vy, double, double)
{
    double x1, y1, q1, x2, y2, q2;
    polar_two(iter, id, stream, k0, k1, x1, y1, q1, x2, y2, q2);
    const double m1 = polar_mult_f64(q1);
    const double m2 = polar_mult_f64(q2);
    const double a = __dmul_rn(y1, m1), b = __dmul_rn(x1, m1);
    const double c = __dmul_rn(y2, m2), d = __dmul_rn(x2, m2);
    if (Init) {
        x = plus0(__dmul_rn(a, p.sd_pos0));
        y = plus0(__dmul_rn(b, p.sd_pos0));
        vx = plus0(__dmul_rn(c, p.sd_vel0));
        vy = plus0(__dmul_rn(d, p.sd_vel0));
    } else {
        const double n1 = plus0(__dmul_rn(a, p.sd_pos));
        const double n2 = plus0(__dmul_rn(b, p.sd_pos));
        const double n3 = plus0(__dmul_rn(c, p.sd_vel));
        const double n4 = plus0(__dmul_rn(d, p.sd_vel));
        x = __dadd_rn(x, __dadd_rn(n1, __dmul_rn(p.dt, vx)));
        y = __dadd_rn(y, __dadd_rn(n2, __dmul_rn(p.dt, vy)));
        vx = __dadd_rn(vx, n3);
        vy = __dadd_rn(vy, n4);
    }
}

// cv_state::log_likelihood (pf_smp.hpp:96-112): the two Student-t terms
// share one log, log(1 + a) + log(1 + b) = log((1 + a)(1 + b)).
__device__ __forceinline__ double cv_loglik(const CVParam &p, double x,
                                            double y, double ox, double oy)
{
    const double lx = p.scale * (x - ox);
    const double ly = p.scale * (y - oy);
    const double a = lx * lx * p.inv_nu, b = ly * ly * p.inv_nu;
    return p.coef * log((1.0 + a) * (1.0 + b));
}

// Mixed form: the same stream consumption; float transforms and state.  The
// stored positions are offsets from the step's observation (x - ox, y - oy)
// so that float keeps its precision where the likelihood looks (the
// residual); (shx, shy) = previous observation minus this one, in double
// rounded once, re-anchors the loaded offsets.
template <bool Init>
__device__ __forceinline__ void cv_particle(const CVParam &p, uint32_t iter,
                                            uint32_t id, uint32_t stream,
                                            uint32_t k0, uint32_t k1, float &x,
                                            float &y, float &vx, float &vy,
                                            double shx, double shy)
{
    double x1, y1, q1, x2, y2, q2;
    polar_two(iter, id, stream, k0, k1, x1, y1, q1, x2, y2, q2);
    if (Init) {
        // once per run: the prior in double, then stored as float offsets
        const double m1 = polar_mult_f64(q1), m2 = polar_mult_f64(q2);
        x = (float)(y1 * m1 * p.sd_pos0 + shx);
        y = (float)(x1 * m1 * p.sd_pos0 + shy);
        vx = (float)(y2 * m2 * p.sd_vel0);
        vy = (float)(x2 * m2 * p.sd_vel0);
    } else {
        const float m1 = polar_mult_f32(q1), m2 = polar_mult_f32(q2);
        const float dt = (float)p.dt;
        x = (x + (float)shx) + ((float)y1 * m1 * (float)p.sd_pos + dt * vx);
        y = (y + (float)shy) + ((float)x1 * m1 * (float)p.sd_pos + dt * vy);
        vx = vx + (float)y2 * m2 * (float)p.sd_vel;
        vy = vy + (float)x2 * m2 * (float)p.sd_vel;
    }
}

// Mixed form likelihood on the anchored offsets (x, y are x - ox, y - oy).
__device__ __forceinline__ float cv_loglik(const CVParam &p, float x, float y,
                                           double, double)
{
    const float s = (float)p.scale, inv = (float)p.inv_nu;
    const float lx = s * x, ly = s * y;
    const float a = lx * lx * inv, b = ly * ly * inv;
    return (float)p.coef * log1pf(a + b + a * b);
}

__device__ __forceinline__ double lse_exp(double v) { return exp(v); }
__device__ __forceinline__ double lse_exp(float v) { return (double)expf(v); }

// Per-thread weight statistics against a lazy reference: the first finite
// log-weight becomes the reference and later values are accumulated as
// exp(lw - ref) even above it (double has the range), so the exponential is
// evaluated once per particle; the reference moves only when a value
// exceeds it by more than kLazy (then exp^2 could overflow).  mx tracks the
// true maximum.
struct LseRef {
    double ref, mx, s1, s2, sx, sy;

    __device__ __forceinline__ void init()
    {
        ref = -INFINITY;
        mx = -INFINITY;
        s1 = s2 = sx = sy = 0.0;
    }
};

template <typename Real>
struct LazyBound;
template <>
struct LazyBound<double> {
    static constexpr double v = 300.0;
};
template <>
struct LazyBound<float> {
    static constexpr double v = 40.0;
};

template <typename Real>
__device__ __forceinline__ void lse_add(LseRef &a, Real lw, Real x, Real y)
{
    const double l = (double)lw;
    if (l != l) {
        a.s1 = l; // NaN propagates to the degenerate check
        return;
    }
    if (l == -INFINITY)
        return;
    a.mx = fmax(a.mx, l);
    if (a.ref == -INFINITY) {
        a.ref = l;
    } else if (l - a.ref > LazyBound<Real>::v) {
        const double f = exp(a.ref - l);
        a.s1 *= f;
        a.s2 *= f * f;
        a.sx *= f;
        a.sy *= f;
        a.ref = l;
    }
    const double e = lse_exp((Real)(lw - (Real)a.ref));
    a.s1 += e;
    a.s2 += e * e;
    a.sx += e * (double)x;
    a.sy += e * (double)y;
}

// Rescale a thread's sums to the common maximum M: exp(ref - M) <= 1.
__device__ __forceinline__ void lse_rescale(LseRef &a, double M)
{
    const double f = a.ref == -INFINITY ? 0.0 : exp(a.ref - M);
    a.s1 *= f;
    a.s2 *= f * f;
    a.sx *= f;
    a.sy *= f;
    a.ref = M;
}

__device__ __forceinline__ double warp_max_nan(double v, unsigned width)
{
    for (unsigned o = width / 2; o > 0; o >>= 1)
        v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Sum of the rescaled statistics over `width` lanes.
__device__ __forceinline__ void warp_sum_stats(LseRef &a, double &gx,
                                               double &gy, unsigned width)
{
    for (unsigned o = width / 2; o > 0; o >>= 1) {
        a.s1 += __shfl_xor_sync(0xffffffffu, a.s1, o);
        a.s2 += __shfl_xor_sync(0xffffffffu, a.s2, o);
        a.sx += __shfl_xor_sync(0xffffffffu, a.sx, o);
        a.sy += __shfl_xor_sync(0xffffffffu, a.sy, o);
        gx += __shfl_xor_sync(0xffffffffu, gx, o);
        gy += __shfl_xor_sync(0xffffffffu, gy, o);
    }
}

#ifndef VSMC_MOVE_MIN_BLOCKS
#define VSMC_MOVE_MIN_BLOCKS 3
#endif

template <typename Real, bool Init>
__global__ void __launch_bounds__(kThreads, VSMC_MOVE_MIN_BLOCKS)
k_cv_move(MoveArgs<Real> a)
{
    constexpr int V = Vec<Real>::n;
    constexpr int NV = kItems / V;
    constexpr bool Anchored = sizeof(Real) == 4;
    typedef typename Vec<Real>::type VT;
    constexpr int NW = kThreads / 32;
    // double-buffered warp partials: one barrier per tile
    __shared__ double sh_w[2][7][NW];

    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int gather = Init ? 0 : a.ctl->resampled;
    const Real mprev = Init || gather ? Real(0) : (Real)a.ctl->lw_max;
    const double ox = a.obs_x[a.iter], oy = a.obs_y[a.iter];
    // re-anchoring of the mixed form's offsets
    double shx = 0.0, shy = 0.0;
    if (Anchored) {
        shx = Init ? -ox : a.obs_x[a.iter - 1] - ox;
        shy = Init ? -oy : a.obs_y[a.iter - 1] - oy;
    }
    const long long N = a.N;
    int buf = 0;

    for (int tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
        const long long base = (long long)tile * kTile;
        LseRef acc;
        acc.init();
        double gx = 0.0, gy = 0.0;
#pragma unroll 1
        for (int v = 0; v < NV; ++v) {
            const long long p0 =
                base + ((long long)v * kThreads + threadIdx.x) * V;
            Real s[4][V];
            Real lwv[V];
            const bool full = p0 + V <= N;
            if (Init) {
                // prior: no state is read
            } else if (!gather && full) {
#pragma unroll
                for (int d = 0; d < 4; ++d) {
                    const VT t = *reinterpret_cast<const VT *>(a.in[d] + p0);
                    const Real *tp = reinterpret_cast<const Real *>(&t);
#pragma unroll
                    for (int e = 0; e < V; ++e)
                        s[d][e] = tp[e];
                }
                const VT t = *reinterpret_cast<const VT *>(a.lw + p0);
                const Real *tp = reinterpret_cast<const Real *>(&t);
#pragma unroll
                for (int e = 0; e < V; ++e)
                    lwv[e] = tp[e];
            } else {
#pragma unroll
                for (int e = 0; e < V; ++e) {
                    const long long i = p0 + e;
                    if (i < N) {
                        long long src = i;
                        if (gather) { // clamped: never leaves [0, N)
                            src = a.copy_from[i];
                            src = src < 0 ? 0 : (src >= N ? N - 1 : src);
                        }
#pragma unroll
                        for (int d = 0; d < 4; ++d)
                            s[d][e] = a.in[d][src];
                        lwv[e] = gather ? Real(0) : a.lw[i];
                        if (gather) {
                            gx += (double)s[0][e];
                            gy += (double)s[1][e];
                        }
                    }
                }
            }
            Real lwn[V];
#pragma unroll
            for (int e = 0; e < V; ++e) {
                const long long i = p0 + e;
                if (i < N) {
                    cv_particle<Init>(a.p, a.iter, (uint32_t)i, a.stream, a.k0,
                                      a.k1, s[0][e], s[1][e], s[2][e],
                                      s[3][e], shx, shy);
                    const Real inc = cv_loglik(a.p, s[0][e], s[1][e], ox, oy);
                    // lw += -max (normalize_log_weight), then += inc
                    lwn[e] = Init ? inc : (lwv[e] - mprev) + inc;
                    lse_add<Real>(acc, lwn[e], s[0][e], s[1][e]);
                }
            }
            if (full) {
#pragma unroll
                for (int d = 0; d < 4; ++d) {
                    VT t;
                    Real *tp = reinterpret_cast<Real *>(&t);
#pragma unroll
                    for (int e = 0; e < V; ++e)
                        tp[e] = s[d][e];
                    *reinterpret_cast<VT *>(a.out[d] + p0) = t;
                }
                VT t;
                Real *tp = reinterpret_cast<Real *>(&t);
#pragma unroll
                for (int e = 0; e < V; ++e)
                    tp[e] = lwn[e];
                *reinterpret_cast<VT *>(a.lw + p0) = t;
            } else {
#pragma unroll
                for (int e = 0; e < V; ++e) {
                    const long long i = p0 + e;
                    if (i < N) {
#pragma unroll
                        for (int d = 0; d < 4; ++d)
                            a.out[d][i] = s[d][e];
                        a.lw[i] = lwn[e];
                    }
                }
            }
        }
        // warp: common maximum, one rescale per lane, plain sums
        const double wm = warp_max_nan(acc.mx, 32);
        lse_rescale(acc, wm);
        warp_sum_stats(acc, gx, gy, 32);
        if (lane == 0) {
            double *w = &sh_w[buf][0][0];
            w[0 * NW + wid] = wm;
            w[1 * NW + wid] = acc.s1;
            w[2 * NW + wid] = acc.s2;
            w[3 * NW + wid] = acc.sx;
            w[4 * NW + wid] = acc.sy;
            w[5 * NW + wid] = gx;
            w[6 * NW + wid] = gy;
        }
        __syncthreads();
        if (wid == 0) {
            const double *w = &sh_w[buf][0][0];
            LseRef r;
            double tx = 0.0, ty = 0.0;
            r.init();
            if (lane < NW) {
                r.ref = w[0 * NW + lane];
                r.mx = r.ref;
                r.s1 = w[1 * NW + lane];
                r.s2 = w[2 * NW + lane];
                r.sx = w[3 * NW + lane];
                r.sy = w[4 * NW + lane];
                tx = w[5 * NW + lane];
                ty = w[6 * NW + lane];
            }
            const double tm = warp_max_nan(r.mx, NW);
            lse_rescale(r, tm);
            warp_sum_stats(r, tx, ty, NW);
            if (lane == 0) {
                TileStats ts;
                ts.m = tm;
                ts.s1 = r.s1;
                ts.s2 = r.s2;
                ts.sx = r.sx;
                ts.sy = r.sy;
                ts.gx = tx;
                ts.gy = ty;
                ts.pad = 0.0;
                a.tile_stats[tile] = ts;
            }
        }
        buf ^= 1;
    }
}

struct FinalizeArgs {
    FilterCtl *ctl;
    const TileStats *ts;
    int ntiles;
    long long N;
    double threshold;
    long long t;
    int init;
    int anchored;
    const double *obs_x;
    const double *obs_y;
    double *hist_ess;
    int32_t *hist_resampled;
    double *hist_logz_inc;
    double *hist_mean_x;
    double *hist_mean_y;
    ResampleCtl *rctl;
    double *tile_excl;
    int residual;
    int sys;
    EngineRef eng;
    const int32_t *replay_flags; // replay: resampling decisions to follow
};

constexpr int kFinalThreads = 1024;
constexpr int kFinalSmemTiles = 16384; // spine staged in shared memory

// One CTA, deterministic.  Pass 1 (striped, coalesced loads): the global
// maximum M.  Pass 2 (striped): the rescaled sums s1_t exp(m_t - M) etc.
// with independent exponentials, and each tile's share of the normalised
// weight mass stored for the spine.  Then the decisions of
// Sampler::do_resample and the ordered exclusive spine over the stored
// shares (contiguous runs per thread, read from shared memory).
__global__ void __launch_bounds__(kFinalThreads) k_cv_finalize(FinalizeArgs a)
{
    constexpr int NW = kFinalThreads / 32;
    extern __shared__ double agg[]; // ntiles shares (when staged)
    __shared__ double sh[6][NW];
    __shared__ double sh_spine[NW];
    __shared__ int sh_res;
    __shared__ double sh_M, sh_coeff;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nt = a.ntiles;
    const bool staged = nt <= kFinalSmemTiles;
    double *share = staged ? agg : a.tile_excl; // scratch when not staged
    // pass 1: maximum (NaN propagates)
    double m = -INFINITY;
    for (int t = threadIdx.x; t < nt; t += blockDim.x) {
        const double mt = a.ts[t].m, st = a.ts[t].s1;
        m = (mt != mt || st != st) ? NAN : (m != m ? m : fmax(m, mt));
    }
    for (int o = 16; o > 0; o >>= 1) {
        const double q = __shfl_xor_sync(0xffffffffu, m, o);
        m = (q != q || m != m) ? NAN : fmax(m, q);
    }
    if (lane == 0)
        sh[0][wid] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = -INFINITY;
        for (int w = 0; w < NW; ++w)
            r = (sh[0][w] != sh[0][w] || r != r) ? NAN : fmax(r, sh[0][w]);
        sh_M = r;
    }
    __syncthreads();
    const double M = sh_M;
    // pass 2: sums rescaled to M; shares exp(m_t - M) s1_t (unnormalised)
    double v[6] = {0, 0, 0, 0, 0, 0};
    for (int t = threadIdx.x; t < nt; t += blockDim.x) {
        const TileStats ts = a.ts[t];
        const double f = ts.m == -INFINITY ? 0.0 : exp(ts.m - M);
        const double s1 = ts.s1 * f;
        share[t] = s1;
        v[0] += s1;
        v[1] += ts.s2 * f * f;
        v[2] += ts.sx * f;
        v[3] += ts.sy * f;
        v[4] += ts.gx;
        v[5] += ts.gy;
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        v[k] = warp_sum(v[k]);
        if (lane == 0)
            sh[k][wid] = v[k];
    }
    __syncthreads();
    FilterCtl *c = a.ctl;
    const double Nd = (double)a.N;
    if (threadIdx.x == 0) {
        double r[6] = {0, 0, 0, 0, 0, 0};
        for (int w = 0; w < NW; ++w)
            for (int k = 0; k < 6; ++k)
                r[k] += sh[k][w];
        const double S1 = r[0], S2 = r[1];
        // monitor of the previous step, gathered by this move
        if (!a.init && c->resampled && c->monitor_done != a.t - 1) {
            const double ax = a.anchored ? a.obs_x[a.t - 1] : 0.0;
            const double ay = a.anchored ? a.obs_y[a.t - 1] : 0.0;
            a.hist_mean_x[a.t - 1] = ax + r[4] / Nd;
            a.hist_mean_y[a.t - 1] = ay + r[5] / Nd;
            c->monitor_done = a.t - 1;
        }
        const double s1prev = (a.init || c->resampled) ? Nd : c->s1;
        int res = 0;
        double ess = S1 * S1 / S2;
        double dz = M + log(S1) - log(s1prev);
        if (!(M > -INFINITY && M < INFINITY && S1 > 0.0 && S1 < INFINITY &&
              S2 > 0.0 && S2 < INFINITY)) {
            c->error = VSMC_CUDA_EDEGENERATE;
            ess = NAN;
            dz = NAN;
        } else {
            res = ess < a.threshold * Nd;
        }
        if (a.replay_flags != nullptr)
            res = a.replay_flags[a.t] != 0;
        a.hist_ess[a.t] = ess;
        a.hist_resampled[a.t] = res;
        a.hist_logz_inc[a.t] = dz;
        c->logz += dz;
        c->lw_max = M;
        c->s1 = S1;
        c->s2 = S2;
        c->ess = ess;
        c->resampled = res;
        if (!res) {
            const double ax = a.anchored ? a.obs_x[a.t] : 0.0;
            const double ay = a.anchored ? a.obs_y[a.t] : 0.0;
            a.hist_mean_x[a.t] = ax + r[2] / S1;
            a.hist_mean_y[a.t] = ay + r[3] / S1;
        }
        a.rctl->active = a.replay_flags != nullptr ? 0 : res;
        sh_res = a.replay_flags != nullptr ? 0 : res;
        sh_coeff = __ddiv_rn(1.0, S1);
    }
    __syncthreads();
    if (!sh_res || a.residual)
        return;
    // ordered exclusive spine of the normalised shares
    const double coeff = sh_coeff;
    const int per = (nt + blockDim.x - 1) / blockDim.x;
    const int b = threadIdx.x * per, e = min(b + per, nt);
    double run = 0.0;
    for (int t = b; t < e; ++t)
        run += share[t] * coeff;
    double total;
    double off = block_excl_scan(run, sh_spine, total);
    // in place when the shares live in tile_excl: read before write per t
    for (int t = b; t < e; ++t) {
        const double x = share[t] * coeff;
        a.tile_excl[t] = off;
        off += x;
    }
    if (threadIdx.x == blockDim.x - 1)
        a.tile_excl[nt] = total;
    if (threadIdx.x == 0) {
        ResampleCtl *rc = a.rctl;
        rc->NN = a.N;
        rc->coeff_r = 1.0;
        rc->delta = __ddiv_rn(1.0, Nd);
        rc->kbits = bin_kbits(a.N);
        rc->n_final = 0;
        if (a.sys) {
            const uint64_t w = threefry_word(a.eng.key, a.eng.ctr, rc->offset);
            rc->u0 = __dmul_rn(canonical_u64(w), rc->delta);
            rc->words = 1;
        } else {
            rc->words = 0;
        }
    }
}

// Monitor of a step that resampled and has no following move yet:
// (1/N) sum_i x[copy_from[i]] (set_equal_weight then ISIntegrate), plus the
// anchor of the mixed form.
template <typename Real>
__global__ void __launch_bounds__(kThreads)
k_cv_monitor_gather(const Real *x, const Real *y, const int32_t *copy_from,
                    long long N, double *part)
{
    __shared__ double sh[2][kThreads / 32];
    double gx = 0.0, gy = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
         i += (long long)gridDim.x * blockDim.x) {
        const int32_t c = copy_from[i];
        gx += (double)x[c];
        gy += (double)y[c];
    }
    gx = warp_sum(gx);
    gy = warp_sum(gy);
    if ((threadIdx.x & 31) == 0) {
        sh[0][threadIdx.x >> 5] = gx;
        sh[1][threadIdx.x >> 5] = gy;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double tx = 0.0, ty = 0.0;
        for (int w = 0; w < kThreads / 32; ++w) {
            tx += sh[0][w];
            ty += sh[1][w];
        }
        part[2 * blockIdx.x] = tx;
        part[2 * blockIdx.x + 1] = ty;
    }
}

__global__ void k_cv_monitor_finish(const double *part, int nparts,
                                    long long N, long long t, FilterCtl *ctl,
                                    const double *anchor_x,
                                    const double *anchor_y,
                                    double *hist_mean_x, double *hist_mean_y)
{
    if (threadIdx.x != 0)
        return;
    double tx = 0.0, ty = 0.0;
    for (int i = 0; i < nparts; ++i) {
        tx += part[2 * i];
        ty += part[2 * i + 1];
    }
    hist_mean_x[t] = (anchor_x ? anchor_x[t] : 0.0) + tx / (double)N;
    hist_mean_y[t] = (anchor_y ? anchor_y[t] : 0.0) + ty / (double)N;
    ctl->monitor_done = t;
}

// Gather of the final resampling into the other buffer (read_state).
template <typename Real>
__global__ void k_gather_state(const Real *in, Real *out,
                               const int32_t *copy_from, long long N)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N)
        out[i] = in[copy_from[i]];
}

} // namespace vsmc_b200

using namespace vsmc_b200;

struct vsmc_cuda_cv_filter {
    vsmc_cuda_cv_config cfg;
    cudaStream_t stream;
    char *mem;
    size_t bytes;
    void *state[2][4];
    int cur;
    void *lw;
    int32_t *copy_from;
    FilterCtl *ctl;
    TileStats *tile_stats;
    double *obs_x, *obs_y;
    double *hist_ess, *hist_logz_inc, *hist_mean_x, *hist_mean_y;
    int32_t *hist_resampled;
    double *mon_part;
    ResampleWorkspace rws;
    long long ntiles;
    int move_grid;
    uint64_t iter;   // steps launched so far
    uint64_t T_obs;
    EngineRef eng;
    // CUDA-event timing (vsmc_cuda_cv_set_timing)
    bool timing;
    std::vector<cudaEvent_t> ev;  // 3 per timed step: move begin/end, step end
    size_t ev_used;
    uint64_t launches;
    // ancestry record / replay (fixed-ancestry comparisons)
    int32_t *rec_cf;            // T_max x N, device, caller-owned
    const int32_t *rep_cf;      // T_max x N, device, caller-owned
    const int32_t *rep_flags;   // T_max, device, caller-owned
};

namespace {

constexpr int kMonParts = 1184;

size_t filter_bytes(const vsmc_cuda_cv_config &c)
{
    const size_t N = c.N, T = c.T_max ? c.T_max : 1;
    const size_t real = c.form == VSMC_CUDA_MIXED ? 4 : 8;
    const size_t nt = (N + kTile - 1) / kTile;
    size_t b = 0;
    b += 8 * align256(N * real);           // two state buffers
    b += align256(N * real);               // log-weights
    b += align256(N * 4);                  // copy_from
    b += align256(sizeof(FilterCtl));
    b += align256(nt * sizeof(TileStats));
    b += 2 * align256(T * 8);              // observations
    b += 4 * align256(T * 8) + align256(T * 4); // histories
    b += align256(kMonParts * 16);
    b += resample_workspace_bytes((long long)N);
    return b;
}

int check_config(const vsmc_cuda_cv_config *c)
{
    if (c == nullptr)
        return VSMC_CUDA_EINVAL;
    if (c->N < 2 || c->N > (1ull << 30) || c->T_max < 1 ||
        c->T_max > (1ull << 31) || c->scheme < 0 || c->scheme > 5 ||
        (c->form != VSMC_CUDA_FP64 && c->form != VSMC_CUDA_MIXED) ||
        !(c->threshold >= 0.0))
        return VSMC_CUDA_EINVAL;
    return VSMC_CUDA_OK;
}

template <typename Real>
void launch_step(vsmc_cuda_cv_filter *f, bool init)
{
    const vsmc_cuda_cv_config &c = f->cfg;
    cudaStream_t s = f->stream;
    const long long N = (long long)c.N;
    MoveArgs<Real> a;
    const int src = f->cur, dst = init ? f->cur : 1 - f->cur;
    for (int d = 0; d < 4; ++d) {
        a.in[d] = static_cast<const Real *>(f->state[src][d]);
        a.out[d] = static_cast<Real *>(f->state[dst][d]);
    }
    a.lw = static_cast<Real *>(f->lw);
    a.copy_from = f->copy_from;
    a.ctl = f->ctl;
    a.obs_x = f->obs_x;
    a.obs_y = f->obs_y;
    a.tile_stats = f->tile_stats;
    a.N = N;
    a.ntiles = (int)f->ntiles;
    a.iter = (uint32_t)f->iter;
    const uint32_t model_seed = (c.seed % 0xFFFFFFFFu) == 0xFFFFFFFFu
                                    ? 1u
                                    : (c.seed % 0xFFFFFFFFu) + 1u;
    a.k0 = model_seed;
    a.k1 = 0;
    a.stream = c.stream_id;
    a.p = CVParam{c.dt,     c.sd_pos,     c.sd_vel,
                  c.sd_pos0, c.sd_vel0,  c.scale,
                  c.nu,     1.0 / c.nu, -0.5 * (c.nu + 1.0)};
    cudaEvent_t *ev = nullptr;
    if (f->timing) {
        if (f->ev_used + 3 > f->ev.size()) {
            for (int k = 0; k < 3 * 64; ++k) {
                cudaEvent_t e;
                cudaEventCreate(&e);
                f->ev.push_back(e);
            }
        }
        ev = &f->ev[f->ev_used];
        f->ev_used += 3;
        cudaEventRecord(ev[0], s);
    }
    if (init)
        k_cv_move<Real, true><<<f->move_grid, kThreads, 0, s>>>(a);
    else
        k_cv_move<Real, false><<<f->move_grid, kThreads, 0, s>>>(a);
    if (ev)
        cudaEventRecord(ev[1], s);
    f->cur = dst;

    const bool residual = c.scheme == VSMC_CUDA_RESIDUAL ||
                          c.scheme == VSMC_CUDA_RESIDUAL_STRATIFIED ||
                          c.scheme == VSMC_CUDA_RESIDUAL_SYSTEMATIC;
    const bool sys = c.scheme == VSMC_CUDA_SYSTEMATIC ||
                     c.scheme == VSMC_CUDA_RESIDUAL_SYSTEMATIC;
    FinalizeArgs fa;
    fa.ctl = f->ctl;
    fa.ts = f->tile_stats;
    fa.ntiles = (int)f->ntiles;
    fa.N = N;
    fa.threshold = c.threshold;
    fa.t = (long long)f->iter;
    fa.init = init ? 1 : 0;
    fa.anchored = c.form == VSMC_CUDA_MIXED;
    fa.obs_x = f->obs_x;
    fa.obs_y = f->obs_y;
    fa.hist_ess = f->hist_ess;
    fa.hist_resampled = f->hist_resampled;
    fa.hist_logz_inc = f->hist_logz_inc;
    fa.hist_mean_x = f->hist_mean_x;
    fa.hist_mean_y = f->hist_mean_y;
    fa.rctl = f->rws.ctl;
    fa.tile_excl = f->rws.tile_excl;
    fa.residual = residual;
    fa.sys = sys;
    fa.eng = f->eng;
    fa.replay_flags = f->rep_flags;
    const size_t fin_smem = f->ntiles <= kFinalSmemTiles
                                ? (size_t)f->ntiles * sizeof(double)
                                : 0;
    k_cv_finalize<<<1, kFinalThreads, fin_smem, s>>>(fa);

    WeightsFromLog<Real> w;
    w.lw = static_cast<const Real *>(f->lw);
    w.stats = &f->ctl->lw_max;
    if (f->rep_cf != nullptr) {
        // replay: the recorded ancestry of this step (used only if the
        // recorded decision was to resample)
        cudaMemcpyAsync(f->copy_from, f->rep_cf + (size_t)f->iter * c.N,
                        c.N * 4, cudaMemcpyDeviceToDevice, s);
    } else {
        launch_resample_core(c.scheme, w, N, f->eng, f->rws, nullptr, 0,
                             /*spine_done=*/true, nullptr, f->copy_from, s);
    }
    if (f->rec_cf != nullptr)
        cudaMemcpyAsync(f->rec_cf + (size_t)f->iter * c.N, f->copy_from,
                        c.N * 4, cudaMemcpyDeviceToDevice, s);
    if (ev)
        cudaEventRecord(ev[2], s);
    f->launches += 2 + resample_launches(c.scheme, false);
    ++f->iter;
}

template <typename Real>
void launch_monitor_flush(vsmc_cuda_cv_filter *f)
{
    const long long N = (long long)f->cfg.N;
    k_cv_monitor_gather<Real><<<kMonParts, kThreads, 0, f->stream>>>(
        static_cast<const Real *>(f->state[f->cur][0]),
        static_cast<const Real *>(f->state[f->cur][1]), f->copy_from, N,
        f->mon_part);
    const bool anch = f->cfg.form == VSMC_CUDA_MIXED;
    k_cv_monitor_finish<<<1, 32, 0, f->stream>>>(
        f->mon_part, kMonParts, N, (long long)f->iter - 1, f->ctl,
        anch ? f->obs_x : nullptr, anch ? f->obs_y : nullptr,
        f->hist_mean_x, f->hist_mean_y);
}

int sync_and_check(vsmc_cuda_cv_filter *f)
{
    cudaError_t e = cudaStreamSynchronize(f->stream);
    if (e != cudaSuccess)
        return cuda_status(e, "cudaStreamSynchronize");
    FilterCtl h;
    ResampleCtl r;
    e = cudaMemcpy(&h, f->ctl, sizeof(h), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess)
        e = cudaMemcpy(&r, f->rws.ctl, sizeof(r), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
        return cuda_status(e, "cudaMemcpy(ctl)");
    if (h.error != 0) {
        set_last_error(h.error == VSMC_CUDA_EDEGENERATE
                           ? "degenerate weights: every log-weight is -inf "
                             "or a log-weight/likelihood is NaN or +inf"
                           : "device error");
        return h.error;
    }
    if (r.error != 0) {
        set_last_error("resampling look-back wait gave up (timeout)");
        return r.error;
    }
    return VSMC_CUDA_OK;
}

// Gathered monitor of a final resampled step, if not yet written.
int flush_monitor(vsmc_cuda_cv_filter *f)
{
    if (f->iter == 0)
        return VSMC_CUDA_OK;
    FilterCtl h;
    cudaError_t e = cudaMemcpyAsync(&h, f->ctl, sizeof(h),
                                    cudaMemcpyDeviceToHost, f->stream);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(f->stream);
    if (e != cudaSuccess)
        return cuda_status(e, "monitor flush");
    if (h.resampled && h.monitor_done != (long long)f->iter - 1) {
        if (f->cfg.form == VSMC_CUDA_MIXED)
            launch_monitor_flush<float>(f);
        else
            launch_monitor_flush<double>(f);
    }
    return VSMC_CUDA_OK;
}

} // namespace

extern "C" {

void vsmc_cuda_cv_config_default(vsmc_cuda_cv_config *c)
{
    if (c == nullptr)
        return;
    std::memset(c, 0, sizeof(*c));
    c->scheme = VSMC_CUDA_MULTINOMIAL;
    c->form = VSMC_CUDA_FP64;
    c->threshold = 0.5;
    c->seed = 101;
    c->stream_id = 0;
    c->dt = 0.1;
    c->sd_pos = 0.02;
    c->sd_vel = 0.5;
    c->sd_pos0 = 2.0;
    c->sd_vel0 = 1.0;
    c->scale = 10.0;
    c->nu = 10.0;
}

size_t vsmc_cuda_cv_device_bytes(const vsmc_cuda_cv_config *cfg)
{
    if (check_config(cfg) != VSMC_CUDA_OK)
        return 0;
    return filter_bytes(*cfg);
}

int vsmc_cuda_cv_create(const vsmc_cuda_cv_config *cfg, void *stream,
                        vsmc_cuda_cv_filter **out)
{
    if (out == nullptr || check_config(cfg) != VSMC_CUDA_OK) {
        set_last_error("vsmc_cuda_cv_create: invalid configuration");
        return VSMC_CUDA_EINVAL;
    }
    *out = nullptr;
    vsmc_cuda_cv_filter *f = new (std::nothrow) vsmc_cuda_cv_filter();
    if (f == nullptr)
        return VSMC_CUDA_ENOMEM;
    f->cfg = *cfg;
    f->stream = static_cast<cudaStream_t>(stream);
    f->bytes = filter_bytes(*cfg);
    cudaError_t e = cudaMalloc(&f->mem, f->bytes);
    if (e != cudaSuccess) {
        delete f;
        cudaGetLastError();
        set_last_error("vsmc_cuda_cv_create: cudaMalloc of " +
                       std::to_string(cfg->N) + " particles failed");
        return VSMC_CUDA_ENOMEM;
    }
    const size_t N = cfg->N, T = cfg->T_max;
    const size_t real = cfg->form == VSMC_CUDA_MIXED ? 4 : 8;
    const size_t nt = (N + kTile - 1) / kTile;
    char *p = f->mem;
    for (int b = 0; b < 2; ++b)
        for (int d = 0; d < 4; ++d) {
            f->state[b][d] = p;
            p += align256(N * real);
        }
    f->lw = p;
    p += align256(N * real);
    f->copy_from = reinterpret_cast<int32_t *>(p);
    p += align256(N * 4);
    f->ctl = reinterpret_cast<FilterCtl *>(p);
    p += align256(sizeof(FilterCtl));
    f->tile_stats = reinterpret_cast<TileStats *>(p);
    p += align256(nt * sizeof(TileStats));
    f->obs_x = reinterpret_cast<double *>(p);
    p += align256(T * 8);
    f->obs_y = reinterpret_cast<double *>(p);
    p += align256(T * 8);
    f->hist_ess = reinterpret_cast<double *>(p);
    p += align256(T * 8);
    f->hist_logz_inc = reinterpret_cast<double *>(p);
    p += align256(T * 8);
    f->hist_mean_x = reinterpret_cast<double *>(p);
    p += align256(T * 8);
    f->hist_mean_y = reinterpret_cast<double *>(p);
    p += align256(T * 8);
    f->hist_resampled = reinterpret_cast<int32_t *>(p);
    p += align256(T * 4);
    f->mon_part = reinterpret_cast<double *>(p);
    p += align256(kMonParts * 16);
    f->rws = carve_workspace(p, (long long)N);
    f->ntiles = (long long)nt;
    f->cur = 0;
    f->iter = 0;
    f->T_obs = 0;
    f->timing = false;
    f->ev_used = 0;
    f->launches = 0;
    f->rec_cf = nullptr;
    f->rep_cf = nullptr;
    f->rep_flags = nullptr;
    // resample engine: Threefry4x64 seeded seed+2 (Seed::get twice)
    uint32_t sg = cfg->seed % 0xFFFFFFFFu;
    sg = sg == 0xFFFFFFFFu ? 1u : sg + 1u;
    sg = sg == 0xFFFFFFFFu ? 1u : sg + 1u;
    std::memset(&f->eng, 0, sizeof(f->eng));
    f->eng.key.v[0] = sg;
    int dev = 0, sms = 148, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cfg->form == VSMC_CUDA_MIXED)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per, k_cv_move<float, false>, kThreads, 0);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per, k_cv_move<double, false>, kThreads, 0);
    if (per < 1)
        per = 1;
    const long long g = (long long)sms * per;
    cudaFuncSetAttribute(k_cv_finalize,
                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                         kFinalSmemTiles * (int)sizeof(double));
    f->move_grid = (int)(f->ntiles < g ? f->ntiles : g);
    e = cudaMemsetAsync(f->mem, 0, f->bytes, f->stream);
    if (e != cudaSuccess) {
        cudaFree(f->mem);
        delete f;
        return cuda_status(e, "vsmc_cuda_cv_create: memset");
    }
    *out = f;
    return VSMC_CUDA_OK;
}

int vsmc_cuda_cv_destroy(vsmc_cuda_cv_filter *f)
{
    if (f == nullptr)
        return VSMC_CUDA_OK;
    cudaStreamSynchronize(f->stream);
    for (cudaEvent_t ev : f->ev)
        cudaEventDestroy(ev);
    cudaError_t e = cudaFree(f->mem);
    delete f;
    return e == cudaSuccess ? VSMC_CUDA_OK : cuda_status(e, "cudaFree");
}

int vsmc_cuda_cv_set_observations(vsmc_cuda_cv_filter *f, const double *ox,
                                  const double *oy, uint64_t T, int on_device)
{
    if (f == nullptr || ox == nullptr || oy == nullptr || T == 0 ||
        T > f->cfg.T_max) {
        set_last_error("vsmc_cuda_cv_set_observations: invalid arguments");
        return VSMC_CUDA_EINVAL;
    }
    const cudaMemcpyKind k =
        on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    cudaError_t e = cudaMemcpyAsync(f->obs_x, ox, T * 8, k, f->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(f->obs_y, oy, T * 8, k, f->stream);
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_cv_set_observations");
    f->T_obs = T;
    return VSMC_CUDA_OK;
}

int vsmc_cuda_cv_initialize(vsmc_cuda_cv_filter *f)
{
    if (f == nullptr || f->T_obs < 1) {
        set_last_error("vsmc_cuda_cv_initialize: no observations");
        return VSMC_CUDA_EINVAL;
    }
    // do_reset: histories cleared, equal weights, engine offset kept
    FilterCtl h;
    std::memset(&h, 0, sizeof(h));
    h.monitor_done = -1;
    cudaError_t e = cudaMemcpyAsync(f->ctl, &h, sizeof(h),
                                    cudaMemcpyHostToDevice, f->stream);
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_cv_initialize");
    // the host struct must outlive the copy
    e = cudaStreamSynchronize(f->stream);
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_cv_initialize");
    f->iter = 0;
    f->cur = 0;
    if (f->cfg.form == VSMC_CUDA_MIXED)
        launch_step<float>(f, true);
    else
        launch_step<double>(f, true);
    e = cudaGetLastError();
    return e == cudaSuccess ? VSMC_CUDA_OK
                            : cuda_status(e, "vsmc_cuda_cv_initialize");
}

int vsmc_cuda_cv_iterate(vsmc_cuda_cv_filter *f, uint64_t num)
{
    if (f == nullptr || f->iter == 0) {
        set_last_error("vsmc_cuda_cv_iterate: initialize first");
        return VSMC_CUDA_EINVAL;
    }
    if (f->iter + num > f->T_obs) {
        set_last_error("vsmc_cuda_cv_iterate: not enough observations");
        return VSMC_CUDA_EINVAL;
    }
    for (uint64_t k = 0; k < num; ++k) {
        if (f->cfg.form == VSMC_CUDA_MIXED)
            launch_step<float>(f, false);
        else
            launch_step<double>(f, false);
    }
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? VSMC_CUDA_OK
                            : cuda_status(e, "vsmc_cuda_cv_iterate");
}

int vsmc_cuda_cv_synchronize(vsmc_cuda_cv_filter *f)
{
    if (f == nullptr)
        return VSMC_CUDA_EINVAL;
    return sync_and_check(f);
}

int vsmc_cuda_cv_iter_size(vsmc_cuda_cv_filter *f, uint64_t *n)
{
    if (f == nullptr || n == nullptr)
        return VSMC_CUDA_EINVAL;
    *n = f->iter;
    return VSMC_CUDA_OK;
}

int vsmc_cuda_cv_history(vsmc_cuda_cv_filter *f, double *ess,
                         int32_t *resampled, double *logz_inc, double *mean_x,
                         double *mean_y)
{
    if (f == nullptr)
        return VSMC_CUDA_EINVAL;
    int st = flush_monitor(f);
    if (st != VSMC_CUDA_OK)
        return st;
    const size_t T = f->iter;
    cudaError_t e = cudaSuccess;
    if (ess && e == cudaSuccess)
        e = cudaMemcpyAsync(ess, f->hist_ess, T * 8, cudaMemcpyDeviceToHost,
                            f->stream);
    if (resampled && e == cudaSuccess)
        e = cudaMemcpyAsync(resampled, f->hist_resampled, T * 4,
                            cudaMemcpyDeviceToHost, f->stream);
    if (logz_inc && e == cudaSuccess)
        e = cudaMemcpyAsync(logz_inc, f->hist_logz_inc, T * 8,
                            cudaMemcpyDeviceToHost, f->stream);
    if (mean_x && e == cudaSuccess)
        e = cudaMemcpyAsync(mean_x, f->hist_mean_x, T * 8,
                            cudaMemcpyDeviceToHost, f->stream);
    if (mean_y && e == cudaSuccess)
        e = cudaMemcpyAsync(mean_y, f->hist_mean_y, T * 8,
                            cudaMemcpyDeviceToHost, f->stream);
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_cv_history");
    return sync_and_check(f);
}

int vsmc_cuda_cv_log_evidence(vsmc_cuda_cv_filter *f, double *logz)
{
    if (f == nullptr || logz == nullptr)
        return VSMC_CUDA_EINVAL;
    cudaError_t e = cudaMemcpyAsync(logz, &f->ctl->logz, 8,
                                    cudaMemcpyDeviceToHost, f->stream);
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_cv_log_evidence");
    return sync_and_check(f);
}

int vsmc_cuda_cv_read_state(vsmc_cuda_cv_filter *f, double *x, double *y,
                            double *vx, double *vy, double *lwout)
{
    if (f == nullptr)
        return VSMC_CUDA_EINVAL;
    int st = sync_and_check(f);
    if (st != VSMC_CUDA_OK)
        return st;
    const size_t N = f->cfg.N;
    const bool mixed = f->cfg.form == VSMC_CUDA_MIXED;
    FilterCtl h;
    cudaError_t e = cudaMemcpy(&h, f->ctl, sizeof(h), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
        return cuda_status(e, "read_state");
    double *outs[4] = {x, y, vx, vy};
    // the mixed form stores positions as offsets from the last observation
    double anchor[2] = {0.0, 0.0};
    if (mixed && f->iter > 0) {
        e = cudaMemcpy(&anchor[0], f->obs_x + (f->iter - 1), 8,
                       cudaMemcpyDeviceToHost);
        if (e == cudaSuccess)
            e = cudaMemcpy(&anchor[1], f->obs_y + (f->iter - 1), 8,
                           cudaMemcpyDeviceToHost);
        if (e != cudaSuccess)
            return cuda_status(e, "read_state");
    }
    // after a resampling the particles are the gathered previous ones
    const int src = f->cur, tmp = 1 - f->cur;
    for (int d = 0; d < 4; ++d) {
        if (outs[d] == nullptr)
            continue;
        const void *from = f->state[src][d];
        if (h.resampled) {
            const unsigned g = (unsigned)((N + 255) / 256);
            if (mixed)
                k_gather_state<float><<<g, 256, 0, f->stream>>>(
                    static_cast<const float *>(f->state[src][d]),
                    static_cast<float *>(f->state[tmp][d]), f->copy_from,
                    (long long)N);
            else
                k_gather_state<double><<<g, 256, 0, f->stream>>>(
                    static_cast<const double *>(f->state[src][d]),
                    static_cast<double *>(f->state[tmp][d]), f->copy_from,
                    (long long)N);
            from = f->state[tmp][d];
        }
        if (mixed) {
            std::string buf(N * 4, '\0');
            e = cudaMemcpyAsync(&buf[0], from, N * 4, cudaMemcpyDeviceToHost,
                                f->stream);
            if (e == cudaSuccess)
                e = cudaStreamSynchronize(f->stream);
            const float *fp = reinterpret_cast<const float *>(buf.data());
            const double an = d < 2 ? anchor[d] : 0.0;
            for (size_t i = 0; i < N; ++i)
                outs[d][i] = an + (double)fp[i];
        } else {
            e = cudaMemcpyAsync(outs[d], from, N * 8, cudaMemcpyDeviceToHost,
                                f->stream);
            if (e == cudaSuccess)
                e = cudaStreamSynchronize(f->stream);
        }
        if (e != cudaSuccess)
            return cuda_status(e, "read_state");
    }
    if (lwout != nullptr) {
        if (h.resampled) {
            for (size_t i = 0; i < N; ++i)
                lwout[i] = 0.0;
        } else {
            if (mixed) {
                std::string buf(N * 4, '\0');
                e = cudaMemcpy(&buf[0], f->lw, N * 4, cudaMemcpyDeviceToHost);
                const float *fp = reinterpret_cast<const float *>(buf.data());
                for (size_t i = 0; i < N; ++i)
                    lwout[i] = (double)(fp[i] - (float)h.lw_max);
            } else {
                e = cudaMemcpy(lwout, f->lw, N * 8, cudaMemcpyDeviceToHost);
                for (size_t i = 0; i < N; ++i)
                    lwout[i] = lwout[i] + -h.lw_max;
            }
            if (e != cudaSuccess)
                return cuda_status(e, "read_state");
        }
    }
    return VSMC_CUDA_OK;
}

int vsmc_cuda_cv_append_observations(vsmc_cuda_cv_filter *f,
                                     const double *ox, const double *oy,
                                     uint64_t n, int on_device)
{
    if (f == nullptr || ox == nullptr || oy == nullptr || n == 0 ||
        f->T_obs + n > f->cfg.T_max) {
        set_last_error("vsmc_cuda_cv_append_observations: invalid arguments "
                       "or T_max exceeded");
        return VSMC_CUDA_EINVAL;
    }
    const cudaMemcpyKind k =
        on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    cudaError_t e = cudaMemcpyAsync(f->obs_x + f->T_obs, ox, n * 8, k,
                                    f->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(f->obs_y + f->T_obs, oy, n * 8, k, f->stream);
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_cv_append_observations");
    f->T_obs += n;
    return VSMC_CUDA_OK;
}

int vsmc_cuda_cv_read_step(vsmc_cuda_cv_filter *f, uint64_t t, double *ess,
                           double *logz_inc, int32_t *resampled,
                           int synchronize)
{
    if (f == nullptr || t >= f->iter) {
        set_last_error("vsmc_cuda_cv_read_step: step not run yet");
        return VSMC_CUDA_EINVAL;
    }
    cudaError_t e = cudaSuccess;
    if (ess)
        e = cudaMemcpyAsync(ess, f->hist_ess + t, 8, cudaMemcpyDeviceToHost,
                            f->stream);
    if (logz_inc && e == cudaSuccess)
        e = cudaMemcpyAsync(logz_inc, f->hist_logz_inc + t, 8,
                            cudaMemcpyDeviceToHost, f->stream);
    if (resampled && e == cudaSuccess)
        e = cudaMemcpyAsync(resampled, f->hist_resampled + t, 4,
                            cudaMemcpyDeviceToHost, f->stream);
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_cv_read_step");
    return synchronize ? sync_and_check(f) : VSMC_CUDA_OK;
}

int vsmc_cuda_cv_set_ancestry(vsmc_cuda_cv_filter *f, int32_t *record,
                              const int32_t *replay,
                              const int32_t *replay_resampled)
{
    if (f == nullptr || (replay == nullptr) != (replay_resampled == nullptr)) {
        set_last_error("vsmc_cuda_cv_set_ancestry: replay needs both the "
                       "ancestry and the decisions");
        return VSMC_CUDA_EINVAL;
    }
    f->rec_cf = record;
    f->rep_cf = replay;
    f->rep_flags = replay_resampled;
    return VSMC_CUDA_OK;
}

int vsmc_cuda_cv_set_timing(vsmc_cuda_cv_filter *f, int enable)
{
    if (f == nullptr)
        return VSMC_CUDA_EINVAL;
    f->timing = enable != 0;
    f->ev_used = 0;
    f->launches = 0;
    return VSMC_CUDA_OK;
}

int vsmc_cuda_cv_timing(vsmc_cuda_cv_filter *f, double *move_ms,
                        double *step_ms, uint64_t *steps, uint64_t *launches)
{
    if (f == nullptr)
        return VSMC_CUDA_EINVAL;
    cudaError_t e = cudaStreamSynchronize(f->stream);
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_cv_timing");
    double mv = 0.0, st = 0.0;
    for (size_t k = 0; k + 3 <= f->ev_used; k += 3) {
        float a = 0.0f, b = 0.0f;
        e = cudaEventElapsedTime(&a, f->ev[k], f->ev[k + 1]);
        if (e == cudaSuccess)
            e = cudaEventElapsedTime(&b, f->ev[k], f->ev[k + 2]);
        if (e != cudaSuccess)
            return cuda_status(e, "vsmc_cuda_cv_timing");
        mv += a;
        st += b;
    }
    if (move_ms)
        *move_ms = mv;
    if (step_ms)
        *step_ms = st;
    if (steps)
        *steps = f->ev_used / 3;
    if (launches)
        *launches = f->launches;
    return VSMC_CUDA_OK;
}

int vsmc_cuda_cv_resample_words(vsmc_cuda_cv_filter *f, uint64_t *words)
{
    if (f == nullptr || words == nullptr)
        return VSMC_CUDA_EINVAL;
    int st = sync_and_check(f);
    if (st != VSMC_CUDA_OK)
        return st;
    ResampleCtl r;
    cudaError_t e = cudaMemcpy(&r, f->rws.ctl, sizeof(r),
                               cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
        return cuda_status(e, "resample_words");
    *words = r.offset;
    return VSMC_CUDA_OK;
}

int vsmc_cuda_cv_copy_from(vsmc_cuda_cv_filter *f, int32_t *copy_from,
                           int32_t *resampled)
{
    if (f == nullptr)
        return VSMC_CUDA_EINVAL;
    int st = sync_and_check(f);
    if (st != VSMC_CUDA_OK)
        return st;
    FilterCtl h;
    cudaError_t e = cudaMemcpy(&h, f->ctl, sizeof(h), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && copy_from != nullptr)
        e = cudaMemcpy(copy_from, f->copy_from, f->cfg.N * 4,
                       cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
        return cuda_status(e, "copy_from");
    if (resampled)
        *resampled = h.resampled;
    return VSMC_CUDA_OK;
}

} // extern "C"
