// cv_kernels.cuh -- device code of the constant-velocity Student-t
// bootstrap filter: the fused move / likelihood / log-weight tile, the
// per-step finalisation (normalising constant, ESS, log-evidence, monitor,
// resampling decision, weight spine) and the monitor gathers.  Each kernel
// is a __device__ body plus a one-filter __global__ wrapper; cv_filter.cu
// launches the wrappers for one filter, cv_batch.cu runs the same bodies
// over many filters in one launch, so both give identical results.
//
// Reference: example/pf/include/pf_smp.hpp:73-258 (model), core/sampler.hpp:
// 450-483 and 758-834 (initialize / iterate / do_resample / do_monitor),
// core/weight_set.hpp:108-125, 441-446 (normalisation and ESS), example/
// include/move_smc.hpp:63-71 (log-evidence increment), core/monitor.hpp:
// 274-302 with integrate/is_integrate.hpp:56-80 (posterior mean).
#pragma once

#include "resample.cuh"

namespace vsmc_b200 {

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
// Particles per thread per pass: FP64 one (scalar loads keep the move at
// 64 registers without spills), float two (float2); both measured faster
// than double2 / float4.
template <>
struct Vec<double> {
    static constexpr int n = 1;
    typedef double type;
};
template <>
struct Vec<float> {
    static constexpr int n = 2;
    typedef float2 type;
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

// The two accepted polar points of one particle's step (libstdc++'s two
// calls of the polar loop), from the particle's own Philox stream
// (polar_two).  r2 = x^2 + y^2 is recomputed with the same two products and
// sum, so it is the value the acceptance test saw.
struct PolarPair {
    double x1, y1, x2, y2;
};

__device__ __forceinline__ PolarPair polar_pair_draw(uint32_t iter,
                                                     uint32_t id,
                                                     uint32_t stream,
                                                     uint32_t k0, uint32_t k1)
{
    PolarPair pp;
    double q1, q2;
    polar_two(iter, id, stream, k0, k1, pp.x1, pp.y1, q1, pp.x2, pp.y2, q2);
    return pp;
}

__device__ __forceinline__ double polar_r2(double x, double y)
{
    return __dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y));
}

// FP64 form: cv_move::move_state / cv_init::initialize_state
// (pf_smp.hpp:150-173, 207-238).  The two polar transforms are evaluated
// together (independent chains for the FP64 pipe); the state update keeps
// the reference's evaluation order.
template <bool Init>
__device__ __forceinline__ void cv_particle(const CVParam &p,
                                            const PolarPair &pp, double &x,
                                            double &y, double &vx,
                                            double &vy, double, double)
{
    const double x1 = pp.x1, y1 = pp.y1, x2 = pp.x2, y2 = pp.y2;
    const double q1 = polar_r2(x1, y1), q2 = polar_r2(x2, y2);
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
    return p.coef * fm::fm_log((1.0 + a) * (1.0 + b));
}

// Mixed form: the same stream consumption; float transforms and state.  The
// stored positions are offsets from the step's observation (x - ox, y - oy)
// so that float keeps its precision where the likelihood looks (the
// residual); (shx, shy) = previous observation minus this one, in double
// rounded once, re-anchors the loaded offsets.
template <bool Init>
__device__ __forceinline__ void cv_particle(const CVParam &p,
                                            const PolarPair &pp, float &x,
                                            float &y, float &vx, float &vy,
                                            double shx, double shy)
{
    const double x1 = pp.x1, y1 = pp.y1, x2 = pp.x2, y2 = pp.y2;
    const double q1 = polar_r2(x1, y1), q2 = polar_r2(x2, y2);
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

// Four move CTAs per SM (64 registers, no spills in the steady-state move):
// 32 resident warps instead of 24 at 80 registers: the FP64 move 0.75 ->
// 0.70 ms at 2^24 particles.
#ifndef VSMC_MOVE_MIN_BLOCKS
#define VSMC_MOVE_MIN_BLOCKS 4
#endif

// Per-step values every tile of one filter's move shares.
template <typename Real>
struct MoveStep {
    int gather;   // the previous step resampled: gather through copy_from
    Real mprev;   // the previous maximum, subtracted from every lw
    double ox, oy;
    double shx, shy; // re-anchoring of the mixed form's offsets
};

template <typename Real, bool Init>
__device__ __forceinline__ MoveStep<Real> move_step(const MoveArgs<Real> &a)
{
    constexpr bool Anchored = sizeof(Real) == 4;
    MoveStep<Real> m;
    m.gather = Init ? 0 : a.ctl->resampled;
    m.mprev = Init || m.gather ? Real(0) : (Real)a.ctl->lw_max;
    m.ox = a.obs_x[a.iter];
    m.oy = a.obs_y[a.iter];
    m.shx = 0.0;
    m.shy = 0.0;
    if (Anchored) {
        m.shx = Init ? -m.ox : a.obs_x[a.iter - 1] - m.ox;
        m.shy = Init ? -m.oy : a.obs_y[a.iter - 1] - m.oy;
    }
    return m;
}

// A move CTA of 8 warps (8 particles per thread per tile).  4-warp CTAs
// measured 1.3% faster at 2^24 particles but 20% slower at 2^16, where 32
// tiles leave most SMs idle and a tile's latency is the step's.
constexpr int kMoveThreads = 256;                 // threads of a move CTA
constexpr int kMoveItems = kTile / kMoveThreads; // particles per thread
constexpr int kMoveWarps = kMoveThreads / 32;

// One tile of kTile particles: load (gather), move, likelihood, log-weight
// update and the tile's online log-sum-exp statistics.  `sh_w` holds
// 7 x kMoveWarps warp partials; a CTA alternates two such buffers so that
// one barrier per tile suffices.
template <typename Real, bool Init>
__device__ __forceinline__ void cv_move_tile(const MoveArgs<Real> &a,
                                             const MoveStep<Real> &ms,
                                             int tile, double *sh_w)
{
    constexpr int V = Vec<Real>::n;
    constexpr int NV = kMoveItems / V;
    typedef typename Vec<Real>::type VT;
    constexpr int NW = kMoveWarps;
    const int gather = ms.gather;
    const Real mprev = ms.mprev;
    const double ox = ms.ox, oy = ms.oy, shx = ms.shx, shy = ms.shy;
    const long long N = a.N;
    {
        const long long base = (long long)tile * kTile;
        LseRef acc;
        acc.init();
        double gx = 0.0, gy = 0.0;
#pragma unroll 1
        for (int v = 0; v < NV; ++v) {
            const long long p0 =
                base + ((long long)v * kMoveThreads + threadIdx.x) * V;
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
                    cv_particle<Init>(
                        a.p,
                        polar_pair_draw(a.iter, (uint32_t)i, a.stream, a.k0,
                                        a.k1),
                        s[0][e], s[1][e], s[2][e], s[3][e], shx, shy);
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
        tile_stats_reduce<NW>(acc, gx, gy, sh_w, a.tile_stats + tile);
    }
}

template <typename Real, bool Init>
__global__ void __launch_bounds__(kMoveThreads,
                                  VSMC_MOVE_MIN_BLOCKS * 256 / kMoveThreads)
k_cv_move(MoveArgs<Real> a)
{
    // double-buffered warp partials: one barrier per tile
    __shared__ double sh_w[2][7 * kMoveWarps];
    const MoveStep<Real> ms = move_step<Real, Init>(a);
    int buf = 0;
    for (int tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
        cv_move_tile<Real, Init>(a, ms, tile, sh_w[buf]);
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
    int compare; // replay, and still resample on this step's own decision
};

constexpr int kFinalThreads = 1024;
constexpr int kFinalSmemTiles = 16384; // spine staged in shared memory

// One CTA, deterministic.  Pass 1 (striped, coalesced loads): the global
// maximum M.  Pass 2 (striped): the rescaled sums s1_t exp(m_t - M) etc.
// with independent exponentials, and each tile's share of the normalised
// weight mass stored for the spine.  Then the decisions of
// Sampler::do_resample and the ordered exclusive spine over the stored
// shares (contiguous runs per thread, read from shared memory).
struct SmemFinal {
    double sh[6][kFinalThreads / 32];
    double spine[kFinalThreads / 32];
    int res;
    double M, coeff;
};

// `agg` stages up to `agg_cap` tile shares in shared memory; larger filters
// keep them in tile_excl.
__device__ __forceinline__ void k_cv_finalize_body(const FinalizeArgs &a,
                                                   double *agg, int agg_cap,
                                                   SmemFinal &sm)
{
    constexpr int NW = kFinalThreads / 32;
    double(&sh)[6][NW] = sm.sh;
    double *sh_spine = sm.spine;
    int &sh_res = sm.res;
    double &sh_M = sm.M;
    double &sh_coeff = sm.coeff;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nt = a.ntiles;
    const bool staged = nt <= agg_cap;
    double *share = staged ? agg : a.tile_excl; // scratch when not staged
    // thread 0's reads of the control block and observations, issued
    // before the passes so that its serial section does not wait on them
    FilterCtl *c = a.ctl;
    int c_res = 0, rflag = 0;
    long long c_mdone = 0;
    double c_s1 = 0.0, c_logz = 0.0;
    double ax0 = 0.0, ay0 = 0.0, ax1 = 0.0, ay1 = 0.0;
    if (threadIdx.x == 0) {
        c_res = c->resampled;
        c_mdone = c->monitor_done;
        c_s1 = c->s1;
        c_logz = c->logz;
        if (a.anchored) {
            if (!a.init) {
                ax0 = a.obs_x[a.t - 1];
                ay0 = a.obs_y[a.t - 1];
            }
            ax1 = a.obs_x[a.t];
            ay1 = a.obs_y[a.t];
        }
        if (a.replay_flags != nullptr)
            rflag = a.replay_flags[a.t];
    }
    // pass 1: maximum (NaN propagates); a thread's tiles t, t + blockDim,
    // ... are loaded four at a time so that their latencies overlap
    const int bd = (int)blockDim.x;
    double m = -INFINITY;
    for (int t0 = threadIdx.x; t0 < nt; t0 += 4 * bd) {
        double mt[4], st[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int t = t0 + k * bd;
            mt[k] = t < nt ? a.ts[t].m : -INFINITY; // -inf: no effect
            st[k] = t < nt ? a.ts[t].s1 : 0.0;
        }
#pragma unroll
        for (int k = 0; k < 4; ++k)
            m = (mt[k] != mt[k] || st[k] != st[k])
                    ? NAN
                    : (m != m ? m : fmax(m, mt[k]));
    }
    for (int o = 16; o > 0; o >>= 1) {
        const double q = __shfl_xor_sync(0xffffffffu, m, o);
        m = (q != q || m != m) ? NAN : fmax(m, q);
    }
    if (lane == 0)
        sh[0][wid] = m;
    __syncthreads();
    // the warps of this launch (at most NW; a batch may launch fewer)
    const int nwa = (int)(blockDim.x >> 5);
    if (threadIdx.x == 0) {
        double r = -INFINITY;
        for (int w = 0; w < nwa; ++w)
            r = (sh[0][w] != sh[0][w] || r != r) ? NAN : fmax(r, sh[0][w]);
        sh_M = r;
    }
    __syncthreads();
    const double M = sh_M;
    // pass 2: sums rescaled to M; shares exp(m_t - M) s1_t (unnormalised)
    double v[6] = {0, 0, 0, 0, 0, 0};
    for (int t0 = threadIdx.x; t0 < nt; t0 += 2 * bd) {
        TileStats tb[2];
#pragma unroll
        for (int k = 0; k < 2; ++k)
            if (t0 + k * bd < nt)
                tb[k] = a.ts[t0 + k * bd];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const int t = t0 + k * bd;
            if (t < nt) {
                const TileStats &ts = tb[k];
                const double f = ts.m == -INFINITY ? 0.0 : fm::fm_exp(ts.m - M);
                const double s1 = ts.s1 * f;
                share[t] = s1;
                v[0] += s1;
                v[1] += ts.s2 * f * f;
                v[2] += ts.sx * f;
                v[3] += ts.sy * f;
                v[4] += ts.gx;
                v[5] += ts.gy;
            }
        }
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        v[k] = warp_sum(v[k]);
        if (lane == 0)
            sh[k][wid] = v[k];
    }
    __syncthreads();
    const double Nd = (double)a.N;
    if (threadIdx.x == 0) {
        double r[6] = {0, 0, 0, 0, 0, 0};
        for (int w = 0; w < nwa; ++w)
            for (int k = 0; k < 6; ++k)
                r[k] += sh[k][w];
        const double S1 = r[0], S2 = r[1];
        // monitor of the previous step, gathered by this move
        if (!a.init && c_res && c_mdone != a.t - 1) {
            a.hist_mean_x[a.t - 1] = ax0 + r[4] / Nd;
            a.hist_mean_y[a.t - 1] = ay0 + r[5] / Nd;
            c->monitor_done = a.t - 1;
        }
        const double s1prev = (a.init || c_res) ? Nd : c_s1;
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
        // the step's own decision runs the resampling kernels unless the
        // step follows a recorded ancestry without comparing
        const int own = res;
        const int run = a.replay_flags == nullptr || a.compare ? own : 0;
        if (a.replay_flags != nullptr)
            res = rflag != 0;
        a.hist_ess[a.t] = ess;
        a.hist_resampled[a.t] = res;
        a.hist_logz_inc[a.t] = dz;
        c->logz = c_logz + dz;
        c->lw_max = M;
        c->s1 = S1;
        c->s2 = S2;
        c->ess = ess;
        c->resampled = res;
        if (!res) {
            a.hist_mean_x[a.t] = ax1 + r[2] / S1;
            a.hist_mean_y[a.t] = ay1 + r[3] / S1;
        }
        a.rctl->active = run;
        sh_res = run;
        sh_coeff = __ddiv_rn(1.0, S1);
    }
    __syncthreads();
    if (!sh_res)
        return;
    // ordered exclusive spine of the normalised shares (the residual
    // schemes' normalisation pass classifies on it too)
    const double coeff = sh_coeff;
    const int per = (nt + blockDim.x - 1) / blockDim.x;
    const int b = threadIdx.x * per, e = min(b + per, nt);
    double run = 0.0;
    for (int t = b; t < e; ++t)
        run += share[t] * coeff;
    double total;
    double off = block_excl_scan(run, sh_spine, total);
    // in place in `share` (read before write per t); staged shares are then
    // copied out with coalesced stores
    for (int t = b; t < e; ++t) {
        const double x = share[t] * coeff;
        share[t] = off;
        off += x;
    }
    if (threadIdx.x == blockDim.x - 1)
        a.tile_excl[nt] = total;
    if (staged) {
        __syncthreads();
        for (int t = threadIdx.x; t < nt; t += bd)
            a.tile_excl[t] = share[t];
    }
    if (threadIdx.x == 0 && !a.residual) {
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

static __global__ void __launch_bounds__(kFinalThreads)
k_cv_finalize(FinalizeArgs a)
{
    extern __shared__ double agg[]; // ntiles shares (when staged)
    __shared__ SmemFinal sm;
    k_cv_finalize_body(a, agg, kFinalSmemTiles, sm);
}

// Monitor of a step that resampled and has no following move yet:
// (1/N) sum_i x[copy_from[i]] (set_equal_weight then ISIntegrate), plus the
// anchor of the mixed form.
// Both kernels return at once unless step t resampled and its gathered
// monitor is not yet written (the decision is read on the device, so the
// host enqueues them without a round trip).
__device__ __forceinline__ bool monitor_pending(const FilterCtl *ctl,
                                                long long t)
{
    return ctl->resampled && ctl->monitor_done != t;
}

template <typename Real>
__global__ void __launch_bounds__(kThreads)
k_cv_monitor_gather(const Real *x, const Real *y, const int32_t *copy_from,
                    long long N, double *part, const FilterCtl *ctl,
                    long long t)
{
    __shared__ double sh[2][kThreads / 32];
    if (!monitor_pending(ctl, t))
        return;
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

static __global__ void k_cv_monitor_finish(const double *part, int nparts,
                                    long long N, long long t, FilterCtl *ctl,
                                    const double *anchor_x,
                                    const double *anchor_y,
                                    double *hist_mean_x, double *hist_mean_y)
{
    if (threadIdx.x != 0 || !monitor_pending(ctl, t))
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


// Seed::get() (rng/seed.hpp:102,149): a seed s gives s+1, s+2, ... modulo
// the seed range of a 32-bit key, skipping 0.
inline uint32_t seed_next(uint32_t s)
{
    return s == 0xFFFFFFFFu ? 1u : s + 1u;
}

// Philox4x32 key word 0 of the model's RngSet (first Seed::get after
// Seed::set(seed)).
inline uint32_t cv_model_key(uint64_t seed)
{
    return seed_next((uint32_t)(seed % 0xFFFFFFFFu));
}

// Threefry4x64 resample engine (second Seed::get).
inline EngineRef cv_resample_engine(uint64_t seed)
{
    EngineRef e;
    for (int i = 0; i < 4; ++i) {
        e.key.v[i] = 0;
        e.ctr.v[i] = 0;
    }
    e.key.v[0] = seed_next(seed_next((uint32_t)(seed % 0xFFFFFFFFu)));
    return e;
}

inline CVParam cv_param(const vsmc_cuda_cv_config &c)
{
    return CVParam{c.dt,       c.sd_pos,   c.sd_vel,
                   c.sd_pos0,  c.sd_vel0,  c.scale,
                   c.nu,       1.0 / c.nu, -0.5 * (c.nu + 1.0)};
}

} // namespace vsmc_b200
