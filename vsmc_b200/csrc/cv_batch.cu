// cv_batch.cu -- many independent constant-velocity Student-t filters held
// on the device at once and stepped together.
//
// vSMC runs one Sampler per filter (core/sampler.hpp:450-483); a program
// with many filters loops over them.  Here every filter lives in a slot of
// one vsmc_cuda_cv_batch: its particles, weights, RNG counters, resampling
// workspace, observations and histories stay resident in device memory
// (one allocation per slot from the batch's own memory pool, admitted
// against a byte budget).  A step over a list of slots is one launch per
// kernel of the single-filter step (cv_kernels.cuh, resample.cuh) with
// the grid flattened over all (slot, tile) pairs: each CTA looks up its
// slot and tile in a map, reads the slot's record and runs the same
// per-tile body as the single-filter kernel.  Results therefore do not
// depend on which other filters share a launch, and equal those of a
// single filter with the same configuration bit for bit.
//
// Each slot keeps its own step count on the device, so one launch can mix
// filters at different steps (serving: each filter advances when its next
// observation arrives) and filters that start (step 0 runs the prior).
#include "cv_kernels.cuh"

#include <algorithm>
#include <cstring>
#include <new>
#include <string>
#include <vector>

namespace vsmc_b200 {

void set_last_error(const std::string &msg);
int cuda_status(cudaError_t e, const char *what);

// Device record of one filter slot.
struct BatchSlot {
    void *state[2][4]; // step t writes state[t & 1]
    void *lw;
    int32_t *copy_from;
    FilterCtl *ctl;
    TileStats *tile_stats;
    double *obs_x, *obs_y;
    double *hist_ess, *hist_logz_inc, *hist_mean_x, *hist_mean_y;
    int32_t *hist_resampled;
    ResampleWorkspace rws;
    EngineRef eng;
    long long N;
    long long T_max;
    long long t; // steps done; advanced by the last kernel of each step
    int ntiles;
    uint32_t k0, stream_id;
};

// Flattened grid: CTA b of a tile kernel works on tile `tile` of `slot`.
struct TileRef {
    int32_t slot;
    int32_t tile;
};

// Settings shared by every filter of a batch.
struct BatchConst {
    CVParam p;
    double threshold;
    int residual, sys, anchored;
};

template <typename Real>
__device__ __forceinline__ MoveArgs<Real> batch_move_args(const BatchSlot &b,
                                                          const CVParam &p)
{
    MoveArgs<Real> a;
    const int out = (int)(b.t & 1), in = (int)((b.t + 1) & 1);
    for (int d = 0; d < 4; ++d) {
        a.in[d] = static_cast<const Real *>(b.state[in][d]);
        a.out[d] = static_cast<Real *>(b.state[out][d]);
    }
    a.lw = static_cast<Real *>(b.lw);
    a.copy_from = b.copy_from;
    a.ctl = b.ctl;
    a.obs_x = b.obs_x;
    a.obs_y = b.obs_y;
    a.tile_stats = b.tile_stats;
    a.N = b.N;
    a.ntiles = b.ntiles;
    a.iter = (uint32_t)b.t;
    a.k0 = b.k0;
    a.k1 = 0;
    a.stream = b.stream_id;
    a.p = p;
    return a;
}

// A slot's weights; `normed`: with the exact normalisation coefficient of
// the FP64 form and the unnormalised weights its normalisation pass kept
// (after that pass).
template <typename Real>
__device__ __forceinline__ WeightsFromLog<Real> batch_weights(
    const BatchSlot &b, bool normed = true)
{
    WeightsFromLog<Real> w;
    w.lw = static_cast<const Real *>(b.lw);
    w.stats = &b.ctl->lw_max;
    if (normed)
        w = with_exact_coeff(w, &b.rws.ctl->coeff_w, b.rws.ex.rec);
    return w;
}

// CTA per work item: the map entries of its slot's tiles.
static __global__ void kb_expand(const BatchSlot *slots, const int32_t *work,
                                 const int32_t *tile0, int n, TileRef *map)
{
    const int w = blockIdx.x;
    if (w >= n)
        return;
    const int slot = work[w];
    const int nt = slots[slot].ntiles;
    for (int k = threadIdx.x; k < nt; k += blockDim.x)
        map[tile0[w] + k] = TileRef{slot, k};
}

// MinBlocks: 256-thread groups per SM the move is compiled for (a tuning choice of
// vsmc_cuda_cv_batch_autotune; every variant computes the same values).
template <typename Real, int MinBlocks>
__global__ void __launch_bounds__(kMoveThreads, MinBlocks * 256 / kMoveThreads)
kb_move(const BatchSlot *slots, const TileRef *map, CVParam p)
{
    __shared__ double sh_w[7 * kMoveWarps];
    const TileRef r = map[blockIdx.x];
    const BatchSlot &b = slots[r.slot];
    const MoveArgs<Real> a = batch_move_args<Real>(b, p);
    if (a.iter == 0) {
        const MoveStep<Real> ms = move_step<Real, true>(a);
        cv_move_tile<Real, true>(a, ms, r.tile, sh_w);
    } else {
        const MoveStep<Real> ms = move_step<Real, false>(a);
        cv_move_tile<Real, false>(a, ms, r.tile, sh_w);
    }
}

constexpr int kBatchAgg = 2048; // tile shares staged in shared memory

static __global__ void __launch_bounds__(kFinalThreads)
kb_finalize(const BatchSlot *slots, const int32_t *work, BatchConst c)
{
    __shared__ SmemFinal sm;
    __shared__ double agg[kBatchAgg];
    const BatchSlot &b = slots[work[blockIdx.x]];
    FinalizeArgs a;
    a.ctl = b.ctl;
    a.ts = b.tile_stats;
    a.ntiles = b.ntiles;
    a.N = b.N;
    a.threshold = c.threshold;
    a.t = b.t;
    a.init = b.t == 0;
    a.anchored = c.anchored;
    a.obs_x = b.obs_x;
    a.obs_y = b.obs_y;
    a.hist_ess = b.hist_ess;
    a.hist_resampled = b.hist_resampled;
    a.hist_logz_inc = b.hist_logz_inc;
    a.hist_mean_x = b.hist_mean_x;
    a.hist_mean_y = b.hist_mean_y;
    a.rctl = b.rws.ctl;
    a.tile_excl = b.rws.tile_excl;
    a.residual = c.residual;
    a.sys = c.sys;
    a.eng = b.eng;
    a.replay_flags = nullptr;
    a.compare = 0;
    k_cv_finalize_body(a, agg, kBatchAgg, sm);
}

template <typename Real, bool Residual>
__global__ void __launch_bounds__(kThreads)
kb_tile_sums(const BatchSlot *slots, const TileRef *map)
{
    __shared__ SmemTileSums sm;
    const TileRef r = map[blockIdx.x];
    const BatchSlot &b = slots[r.slot];
    k_tile_sums_body<WeightsFromLog<Real>, Residual>(
        batch_weights<Real>(b), b.N, b.rws.ctl, b.rws.tile_sum,
        Residual ? b.rws.tile_k : nullptr, r.tile, sm);
}

template <bool Residual, bool Sys>
__global__ void __launch_bounds__(kSpineThreads)
kb_spine_weights(const BatchSlot *slots, const int32_t *work)
{
    __shared__ SmemSpine sm;
    const BatchSlot &b = slots[work[blockIdx.x]];
    k_spine_weights_body<Residual, Sys>(
        b.rws.tile_sum, Residual ? b.rws.tile_k : nullptr, b.rws.tile_excl,
        Residual ? b.rws.tile_kexcl : nullptr, b.ntiles, b.N, b.eng,
        b.rws.ctl, 0, sm);
}

// Stratified uniforms: the single-filter kernel runs one thread per block
// of 4 uniforms over N / 4 + 2 blocks; here the CTA of tile k covers blocks
// [512 k, 512 (k + 1)) and the last tile the remainder, every warp whole.
static __global__ void __launch_bounds__(kThreads)
kb_uniforms_stratified(const BatchSlot *slots, const TileRef *map)
{
    __shared__ SmemNone sm;
    const TileRef r = map[blockIdx.x];
    const BatchSlot &b = slots[r.slot];
    constexpr long long per = kTile / 4;
    const long long lo = (long long)r.tile * per;
    const long long hi =
        r.tile == b.ntiles - 1 ? b.N / 4 + 2 : lo + per;
    for (long long g = lo; g < hi; g += kThreads)
        k_uniforms_stratified_body(b.eng, b.rws.ctl, b.rws.u, b.rws.bins,
                                   (unsigned long long)(g + threadIdx.x), sm);
}

static __global__ void __launch_bounds__(kThreads)
kb_sorted_tile_sums(const BatchSlot *slots, const TileRef *map)
{
    __shared__ SmemSortedSums sm;
    const TileRef r = map[blockIdx.x];
    const BatchSlot &b = slots[r.slot];
    k_sorted_tile_sums_body(b.eng, b.rws.ctl, b.rws.u_tile_sum, b.rws.u,
                            r.tile, sm);
}

static __global__ void __launch_bounds__(kSpineThreads)
kb_sorted_spine(const BatchSlot *slots, const int32_t *work)
{
    __shared__ SmemSpine sm;
    const BatchSlot &b = slots[work[blockIdx.x]];
    k_sorted_spine_body(b.rws.u_tile_sum, b.rws.u_tile_excl, b.rws.ctl, 0,
                        sm);
}

static __global__ void __launch_bounds__(kThreads)
kb_sorted_uniforms(const BatchSlot *slots, const TileRef *map)
{
    __shared__ SmemSortedUniforms sm;
    const TileRef r = map[blockIdx.x];
    const BatchSlot &b = slots[r.slot];
    k_sorted_uniforms_body(b.rws.ctl, b.rws.exu, b.rws.u, b.rws.bins, r.tile,
                           sm);
}

// The exact lmax of a slot's sorted sequence (exact_scan.cuh over the
// negated terms): per slot (its tiles run in kb_exact_tiles_staged).
static __global__ void __launch_bounds__(kSpineThreads)
kb_exact_terms_spine(const BatchSlot *slots, const int32_t *work)
{
    __shared__ SmemExactSpine sm;
    const BatchSlot &b = slots[work[blockIdx.x]];
    k_exact_spine_body<TermsNeg, false>(TermsNeg{b.rws.u, 0}, b.N, b.rws.ctl,
                                        b.ntiles, b.rws.exu, sm);
}

template <typename Real, bool Residual, bool Sys>
__global__ void __launch_bounds__(kThreads, VSMC_INVERT_MIN_BLOCKS)
kb_invert(const BatchSlot *slots, const TileRef *map)
{
    __shared__ SmemInvert<Residual> sm;
    const TileRef r = map[blockIdx.x];
    const BatchSlot &b = slots[r.slot];
    k_invert_body<WeightsFromLog<Real>, Residual, Sys>(
        batch_weights<Real>(b), b.N, b.rws.ctl, b.rws.tile_excl,
        Residual ? b.rws.tile_kexcl : nullptr, b.rws.u, b.N, b.rws.bins,
        nullptr, b.copy_from, b.rws.sinc, b.rws.tile_zeros,
        b.rws.tile_sinc_last, b.rws.ex, r.tile, sm);
}

// The sources a batched exact scan runs over: a slot's weights (with the
// normalisation pass's coefficient, or unnormalised for that pass) and its
// sorted sequence's negated terms, with the approximate spine and the
// ExactScan arrays that go with each.
template <typename Real, bool Normed>
struct SlotWeights {
    typedef WeightsFromLog<Real> W;
    __device__ static W get(const BatchSlot &b)
    {
        return batch_weights<Real>(b, Normed);
    }
    __device__ static const double *excl(const BatchSlot &b)
    {
        return b.rws.tile_excl;
    }
    __device__ static ExactScan scan(const BatchSlot &b) { return b.rws.ex; }
};

struct SlotTerms {
    typedef TermsNeg W;
    __device__ static W get(const BatchSlot &b) { return TermsNeg{b.rws.u, 0}; }
    __device__ static const double *excl(const BatchSlot &b)
    {
        return b.rws.u_tile_excl;
    }
    __device__ static ExactScan scan(const BatchSlot &b) { return b.rws.exu; }
};

// Phase A of the exact scan over every (slot, tile) entry of the map: a
// persistent grid whose CTAs stage the next entry's source values with
// cp.async while they classify the current one (the single filter's
// k_exact_tiles, over many filters).  Each entry computes what
// k_exact_tiles_body computes for it, so the results are the same.
template <typename Src, bool Residual, bool Raw>
__global__ void __launch_bounds__(kThreads, VSMC_EXACT_STAGE_MIN_BLOCKS)
kb_exact_tiles_staged(const BatchSlot *slots, const TileRef *map, int nmap)
{
    typedef typename Src::W W;
    typedef typename W::stage_t S;
    __shared__ SmemExactStage sm;
    // the scanned length of an entry's slot, or -1 when the entry's tile
    // is not scanned (no resampling, past the length, or residual children
    // none: then only the integer parts are stored)
    const auto length = [&](const BatchSlot &b, const W &w, int tile,
                            bool &none) -> long long {
        const ResampleCtl *ctl = b.rws.ctl;
        none = false;
        if (!w.active(ctl))
            return -1;
        const long long N = w.length(ctl, b.N);
        if ((long long)tile * kTile >= N)
            return -1;
        none = Residual && ctl->NN <= 0;
        if (none && Raw)
            return -1;
        return N;
    };
    const auto issue = [&](int m, int buf) {
        const TileRef r = map[m];
        const BatchSlot &b = slots[r.slot];
        const W w = Src::get(b);
        bool none;
        const long long N = length(b, w, r.tile, none);
        if (N > 0) {
            S *dst = reinterpret_cast<S *>(sm.stage[buf]);
            const S *src = w.stage_src();
            const long long base = (long long)r.tile * kTile;
#pragma unroll
            for (int j = 0; j < kItems; ++j) {
                const int l = j * kThreads + threadIdx.x;
                if (base + l < N)
                    cp_async_n<sizeof(S)>(&dst[pad8(l)], &src[base + l]);
            }
        }
        cp_async_commit(); // (an empty group keeps the counting uniform)
    };
    int buf = 0;
    if ((int)blockIdx.x < nmap)
        issue(blockIdx.x, 0);
    for (int m = blockIdx.x; m < nmap; m += gridDim.x) {
        const int next = m + gridDim.x;
        if (next < nmap) {
            issue(next, buf ^ 1);
            cp_async_wait_one();
        } else {
            cp_async_wait_all();
        }
        __syncthreads();
        const TileRef r = map[m];
        const BatchSlot &b = slots[r.slot];
        W w = Src::get(b);
        bool none;
        const long long N = length(b, w, r.tile, none);
        if (N > 0) {
            const ResampleCtl *ctl = b.rws.ctl;
            const ExactScan ex = Src::scan(b);
            w.prepare();
            const double Nd = (double)resample_children(ctl, N);
            const double coeff_r = Residual && !Raw ? ctl->coeff_r : 1.0;
            const S *st = reinterpret_cast<const S *>(sm.stage[buf]);
            const long long i0 =
                (long long)r.tile * kTile + (long long)threadIdx.x * kItems;
            double wv[kItems];
            int32_t kk[kItems];
#pragma unroll
            for (int j = 0; j < kItems; ++j) {
                double k = 0.0;
                wv[j] = i0 + j < N
                            ? scan_weight_staged<W, Residual, Raw>(
                                  w, st[pad8(threadIdx.x * kItems + j)], Nd,
                                  coeff_r, k)
                            : 0.0;
                kk[j] = (int32_t)k;
            }
            if (none) {
                if (i0 < N)
                    store8(ex.kint, i0, N, kk);
            } else {
                exact_tile_compute<W, Residual, Raw>(w, N, ctl, Src::excl(b),
                                                     ex, r.tile, coeff_r, wv,
                                                     kk, sm.core);
            }
        }
        __syncthreads(); // every read of stage[buf] before it is refilled
        buf ^= 1;
    }
}

template <typename Real, bool Residual, bool Raw = false>
__global__ void __launch_bounds__(kSpineThreads)
kb_exact_spine(const BatchSlot *slots, const int32_t *work)
{
    __shared__ SmemExactSpine sm;
    const BatchSlot &b = slots[work[blockIdx.x]];
    k_exact_spine_body<WeightsFromLog<Real>, Residual, Raw>(
        batch_weights<Real>(b, Residual || !Raw), b.N, b.rws.ctl, b.ntiles,
        b.rws.ex, sm);
}

static __global__ void __launch_bounds__(kSpineThreads)
kb_zero_spine(const BatchSlot *slots, const int32_t *work)
{
    __shared__ SmemZeroSpine sm;
    const BatchSlot &b = slots[work[blockIdx.x]];
    k_zero_spine_body(b.rws.tile_zeros, b.rws.tile_sinc_last, b.rws.zexcl,
                      b.rws.tfirst, b.rws.tlast, b.ntiles, b.rws.ctl, 0, sm);
}

static __global__ void __launch_bounds__(kThreads)
kb_cfrp_fill(const BatchSlot *slots, const TileRef *map)
{
    __shared__ SmemFill sm;
    const TileRef r = map[blockIdx.x];
    const BatchSlot &b = slots[r.slot];
    k_cfrp_fill_body(b.N, b.rws.ctl, b.rws.sinc, b.rws.zexcl, b.rws.tfirst,
                     b.rws.tlast, b.copy_from, r.tile, sm);
}

// End of a step: the resample engine position (k_resample_done) and the
// slot's step count.
static __global__ void kb_step_done(BatchSlot *slots, const int32_t *work,
                                    int n)
{
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= n)
        return;
    BatchSlot &b = slots[work[w]];
    ResampleCtl *c = b.rws.ctl;
    if (c->active)
        c->offset += c->words;
    b.t += 1;
}

// ---- block per filter ----------------------------------------------------
// Small filters (a few tiles) spend most of a grid-per-filter step waiting
// at kernel boundaries: each of the step's 9 launches has one or two CTAs
// of work per filter.  kb_block_run gives each such filter one CTA that
// runs all of the filter's remaining steps with block barriers only: the
// same per-tile bodies in the same order (tile by tile where the grid runs
// tiles in parallel), so every filter's results equal those of a lone
// filter bit for bit.  The spines and the finalize run on the CTA's 256
// threads, which gives the same sums as 1024 while a filter has at most
// 256 tiles.  Persistent CTAs take filters from a queue, largest work
// first.
constexpr int kBlockMaxTiles = 64; // largest filter kb_block_run takes

struct BlockItem {
    int32_t slot;
    int32_t steps;
};

template <bool Residual>
union SmemBlockPhase {
    SmemFinal fin;
    SmemTileSums ts;
    SmemSpine sp;
    SmemNone none;
    SmemSortedSums ss;
    SmemSortedUniforms su;
    SmemInvert<Residual> inv;
    SmemZeroSpine zsp;
    SmemFill fill;
    SmemExactTiles<Residual> ext;
    SmemExactTiles<false> ext0;
    SmemExactSpine exs;
};

template <bool Residual>
struct SmemBlock {
    SmemBlockPhase<Residual> ph;
    double agg[kBlockMaxTiles];
    double sh_w[2][7 * kMoveWarps];
    int item;
};

template <bool Residual>
constexpr size_t block_smem_bytes()
{
    return sizeof(SmemBlock<Residual>);
}

// Two CTAs per SM: the whole step in one kernel needs more registers than
// the move alone (three CTAs spilled).
constexpr int kBlockCtasPerSm = 2;

template <typename Real, bool Residual, bool Sys, bool Strat>
__global__ void __launch_bounds__(kThreads, kBlockCtasPerSm)
kb_block_run(BatchSlot *slots, const BlockItem *items, int n, int *queue,
             BatchConst c)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SmemBlock<Residual> &sm = *reinterpret_cast<SmemBlock<Residual> *>(smem_raw);
    for (;;) {
        if (threadIdx.x == 0)
            sm.item = atomicAdd(queue, 1);
        __syncthreads();
        const int it = sm.item;
        __syncthreads();
        if (it >= n)
            return;
        BatchSlot &b = slots[items[it].slot];
        const int steps = items[it].steps;
        const int nt = b.ntiles;
        for (int st = 0; st < steps; ++st) {
            // move: kb_move's body, tile by tile
            {
                const MoveArgs<Real> a = batch_move_args<Real>(b, c.p);
                int buf = 0;
                if (a.iter == 0) {
                    const MoveStep<Real> ms = move_step<Real, true>(a);
                    for (int tile = 0; tile < nt; ++tile, buf ^= 1)
                        cv_move_tile<Real, true>(a, ms, tile, sm.sh_w[buf]);
                } else {
                    const MoveStep<Real> ms = move_step<Real, false>(a);
                    for (int tile = 0; tile < nt; ++tile, buf ^= 1)
                        cv_move_tile<Real, false>(a, ms, tile,
                                                  sm.sh_w[buf]);
                }
            }
            __syncthreads();
            // finalize: kb_finalize's body
            {
                FinalizeArgs a;
                a.ctl = b.ctl;
                a.ts = b.tile_stats;
                a.ntiles = nt;
                a.N = b.N;
                a.threshold = c.threshold;
                a.t = b.t;
                a.init = b.t == 0;
                a.anchored = c.anchored;
                a.obs_x = b.obs_x;
                a.obs_y = b.obs_y;
                a.hist_ess = b.hist_ess;
                a.hist_resampled = b.hist_resampled;
                a.hist_logz_inc = b.hist_logz_inc;
                a.hist_mean_x = b.hist_mean_x;
                a.hist_mean_y = b.hist_mean_y;
                a.rctl = b.rws.ctl;
                a.tile_excl = b.rws.tile_excl;
                a.residual = c.residual;
                a.sys = c.sys;
                a.eng = b.eng;
                a.replay_flags = nullptr;
                a.compare = 0;
                k_cv_finalize_body(a, sm.agg, kBlockMaxTiles, sm.ph.fin);
            }
            __syncthreads();
            if (WeightsFromLog<Real>::kExactNorm) {
                // the weights' sequential sum and coefficient
                const WeightsFromLog<Real> w0 = batch_weights<Real>(b, false);
                for (int tile = 0; tile < nt; ++tile) {
                    k_exact_tiles_body<WeightsFromLog<Real>, false, true>(
                        w0, b.N, b.rws.ctl, b.rws.tile_excl, b.rws.ex, tile,
                        sm.ph.ext0);
                    __syncthreads();
                }
                k_exact_spine_body<WeightsFromLog<Real>, false, true>(
                    w0, b.N, b.rws.ctl, nt, b.rws.ex, sm.ph.exs);
                __syncthreads();
            }
            const WeightsFromLog<Real> w = batch_weights<Real>(b);
            if (Residual) {
                for (int tile = 0; tile < nt; ++tile) {
                    k_tile_sums_body<WeightsFromLog<Real>, true>(
                        w, b.N, b.rws.ctl, b.rws.tile_sum, b.rws.tile_k,
                        tile, sm.ph.ts);
                    __syncthreads();
                }
                k_spine_weights_body<true, Sys>(
                    b.rws.tile_sum, b.rws.tile_k, b.rws.tile_excl,
                    b.rws.tile_kexcl, nt, b.N, b.eng, b.rws.ctl, 0, sm.ph.sp);
                __syncthreads();
            }
            if (Strat) {
                const long long blocks = b.N / 4 + 2;
                for (long long g = 0; g < blocks; g += kThreads)
                    k_uniforms_stratified_body(
                        b.eng, b.rws.ctl, b.rws.u, b.rws.bins,
                        (unsigned long long)(g + threadIdx.x), sm.ph.none);
                __syncthreads();
            } else if (!Sys) {
                for (int tile = 0; tile < nt; ++tile) {
                    k_sorted_tile_sums_body(b.eng, b.rws.ctl,
                                            b.rws.u_tile_sum, b.rws.u, tile,
                                            sm.ph.ss);
                    __syncthreads();
                }
                k_sorted_spine_body(b.rws.u_tile_sum, b.rws.u_tile_excl,
                                    b.rws.ctl, 0, sm.ph.sp);
                __syncthreads();
                const TermsNeg tn{b.rws.u, 0};
                for (int tile = 0; tile < nt; ++tile) {
                    k_exact_tiles_body<TermsNeg, false>(
                        tn, b.N, b.rws.ctl, b.rws.u_tile_excl, b.rws.exu,
                        tile, sm.ph.ext0);
                    __syncthreads();
                }
                k_exact_spine_body<TermsNeg, false>(tn, b.N, b.rws.ctl, nt,
                                                    b.rws.exu, sm.ph.exs);
                __syncthreads();
                for (int tile = 0; tile < nt; ++tile) {
                    k_sorted_uniforms_body(b.rws.ctl, b.rws.exu, b.rws.u,
                                           b.rws.bins, tile, sm.ph.su);
                    __syncthreads();
                }
            }
            if constexpr (Residual && !WeightsFromLog<Real>::kApprox) {
                // the residuals' exact sum
                for (int tile = 0; tile < nt; ++tile) {
                    k_exact_tiles_body<WeightsFromLog<Real>, true, true>(
                        w, b.N, b.rws.ctl, b.rws.tile_excl, b.rws.ex, tile,
                        sm.ph.ext);
                    __syncthreads();
                }
                k_exact_spine_body<WeightsFromLog<Real>, true, true>(
                    w, b.N, b.rws.ctl, nt, b.rws.ex, sm.ph.exs);
                __syncthreads();
            }
            for (int tile = 0; tile < nt; ++tile) {
                k_exact_tiles_body<WeightsFromLog<Real>, Residual>(
                    w, b.N, b.rws.ctl, b.rws.tile_excl, b.rws.ex, tile,
                    sm.ph.ext);
                __syncthreads();
            }
            k_exact_spine_body<WeightsFromLog<Real>, Residual>(
                w, b.N, b.rws.ctl, nt, b.rws.ex, sm.ph.exs);
            __syncthreads();
            for (int tile = 0; tile < nt; ++tile) {
                k_invert_body<WeightsFromLog<Real>, Residual, Sys>(
                    w, b.N, b.rws.ctl, b.rws.tile_excl,
                    Residual ? b.rws.tile_kexcl : nullptr, b.rws.u, b.N,
                    b.rws.bins, nullptr, b.copy_from, b.rws.sinc,
                    b.rws.tile_zeros, b.rws.tile_sinc_last, b.rws.ex, tile,
                    sm.ph.inv);
                __syncthreads();
            }
            k_zero_spine_body(b.rws.tile_zeros, b.rws.tile_sinc_last,
                              b.rws.zexcl, b.rws.tfirst, b.rws.tlast, nt,
                              b.rws.ctl, 0, sm.ph.zsp);
            __syncthreads();
            for (int tile = 0; tile < nt; ++tile) {
                k_cfrp_fill_body(b.N, b.rws.ctl, b.rws.sinc, b.rws.zexcl,
                                 b.rws.tfirst, b.rws.tlast, b.copy_from, tile,
                                 sm.ph.fill);
                __syncthreads();
            }
            // kb_step_done
            if (threadIdx.x == 0) {
                ResampleCtl *rc = b.rws.ctl;
                if (rc->active)
                    rc->offset += rc->words;
                b.t += 1;
            }
            __syncthreads();
        }
    }
}

// The kb_block_run instance of a scheme and form: dynamic shared memory
// above the default (set once at batch creation) and its launch.
template <typename Real, bool R, bool Sy, bool St>
cudaError_t block_smem_one()
{
    return cudaFuncSetAttribute(kb_block_run<Real, R, Sy, St>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)block_smem_bytes<R>());
}

template <typename Real>
cudaError_t block_smem_real(int scheme)
{
    switch (scheme) {
    case VSMC_CUDA_MULTINOMIAL:
        return block_smem_one<Real, false, false, false>();
    case VSMC_CUDA_RESIDUAL:
        return block_smem_one<Real, true, false, false>();
    case VSMC_CUDA_STRATIFIED:
        return block_smem_one<Real, false, false, true>();
    case VSMC_CUDA_SYSTEMATIC:
        return block_smem_one<Real, false, true, false>();
    case VSMC_CUDA_RESIDUAL_STRATIFIED:
        return block_smem_one<Real, true, false, true>();
    default:
        return block_smem_one<Real, true, true, false>();
    }
}

inline cudaError_t set_block_smem(int scheme, int form)
{
    return form == VSMC_CUDA_MIXED ? block_smem_real<float>(scheme)
                                   : block_smem_real<double>(scheme);
}

template <typename Real>
void launch_block_real(int scheme, BatchSlot *slots, const BlockItem *items,
                       int n, int *queue, const BatchConst &c, int grid,
                       cudaStream_t s)
{
    const size_t sm_res = block_smem_bytes<true>();
    const size_t sm_plain = block_smem_bytes<false>();
    switch (scheme) {
    case VSMC_CUDA_MULTINOMIAL:
        kb_block_run<Real, false, false, false>
            <<<grid, kThreads, sm_plain, s>>>(slots, items, n, queue, c);
        break;
    case VSMC_CUDA_RESIDUAL:
        kb_block_run<Real, true, false, false>
            <<<grid, kThreads, sm_res, s>>>(slots, items, n, queue, c);
        break;
    case VSMC_CUDA_STRATIFIED:
        kb_block_run<Real, false, false, true>
            <<<grid, kThreads, sm_plain, s>>>(slots, items, n, queue, c);
        break;
    case VSMC_CUDA_SYSTEMATIC:
        kb_block_run<Real, false, true, false>
            <<<grid, kThreads, sm_plain, s>>>(slots, items, n, queue, c);
        break;
    case VSMC_CUDA_RESIDUAL_STRATIFIED:
        kb_block_run<Real, true, false, true>
            <<<grid, kThreads, sm_res, s>>>(slots, items, n, queue, c);
        break;
    default:
        kb_block_run<Real, true, true, false>
            <<<grid, kThreads, sm_res, s>>>(slots, items, n, queue, c);
        break;
    }
}

// Fresh filter state (Sampler::initialize's reset): step count 0, cleared
// control block; the resample engine position is kept.
__device__ __forceinline__ void reset_slot(BatchSlot &b)
{
    FilterCtl h;
    h.lw_max = 0.0;
    h.s1 = 0.0;
    h.s2 = 0.0;
    h.ess = 0.0;
    h.logz = 0.0;
    h.resampled = 0;
    h.error = 0;
    h.monitor_done = -1;
    *b.ctl = h;
    b.t = 0;
}

static __global__ void kb_reset(BatchSlot *slots, const int32_t *work, int n)
{
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w < n)
        reset_slot(slots[work[w]]);
}

static __global__ void kb_reset_slot(BatchSlot *slots, int slot)
{
    if (threadIdx.x == 0)
        reset_slot(slots[slot]);
}

// Observations: record k writes obs[index] of `slot`.
struct ObsRecord {
    int32_t slot;
    int32_t count;  // values to copy from `src` (set) or 1 (append)
    long long index; // first index written
    long long src;   // offset in the packed source arrays
};

static __global__ void kb_scatter_obs(const BatchSlot *slots,
                                      const ObsRecord *rec, const double *sx,
                                      const double *sy)
{
    const ObsRecord r = rec[blockIdx.x];
    const BatchSlot &b = slots[r.slot];
    for (int k = threadIdx.x; k < r.count; k += blockDim.x) {
        b.obs_x[r.index + k] = sx[r.src + k];
        b.obs_y[r.index + k] = sy[r.src + k];
    }
}

// The last `count` steps of each record's slot (index = first step): ess,
// log-evidence increment, resampled flag packed at `src`; the slot's error
// code per record.
static __global__ void kb_read_steps(const BatchSlot *slots,
                                     const ObsRecord *rec, double *out,
                                     double *err)
{
    const ObsRecord r = rec[blockIdx.x];
    const BatchSlot &b = slots[r.slot];
    for (int k = threadIdx.x; k < r.count; k += blockDim.x) {
        double *o = out + 3 * (r.src + k);
        o[0] = b.hist_ess[r.index + k];
        o[1] = b.hist_logz_inc[r.index + k];
        o[2] = (double)b.hist_resampled[r.index + k];
    }
    if (threadIdx.x == 0)
        err[blockIdx.x] =
            (double)(b.ctl->error != 0 ? b.ctl->error : b.rws.ctl->error);
}

// Summary of each work item's last step: ess, log-evidence increment,
// resampled flag, running log-evidence, error code.
static __global__ void kb_read_last(const BatchSlot *slots,
                                    const int32_t *work, int n, double *out)
{
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= n)
        return;
    const BatchSlot &b = slots[work[w]];
    const long long t = b.t - 1;
    double *o = out + 5 * (long long)w;
    if (t < 0) {
        o[0] = o[1] = o[2] = o[3] = 0.0;
    } else {
        o[0] = b.hist_ess[t];
        o[1] = b.hist_logz_inc[t];
        o[2] = (double)b.hist_resampled[t];
        o[3] = b.ctl->logz;
    }
    const int e = b.ctl->error != 0 ? b.ctl->error : b.rws.ctl->error;
    o[4] = (double)e;
}

// Monitor of a slot's last step when it resampled and no later move has
// gathered it.  Same association as k_cv_monitor_gather over kMonParts
// CTAs of kThreads followed by k_cv_monitor_finish.
constexpr int kMonParts = 1184;

template <typename Real>
__global__ void __launch_bounds__(kThreads)
kb_monitor_flush(const BatchSlot *slots, const int32_t *work, int anchored)
{
    __shared__ double sh[2][kThreads / 32];
    const BatchSlot &b = slots[work[blockIdx.x]];
    const long long t = b.t - 1;
    if (t < 0 || !b.ctl->resampled || b.ctl->monitor_done == t)
        return;
    const long long N = b.N;
    const long long stride = (long long)kMonParts * kThreads;
    const Real *x = static_cast<const Real *>(b.state[t & 1][0]);
    const Real *y = static_cast<const Real *>(b.state[t & 1][1]);
    double tx = 0.0, ty = 0.0;
    const long long need = (N + kThreads - 1) / kThreads;
    const long long parts = need < kMonParts ? need : kMonParts;
    for (long long p = 0; p < parts; ++p) {
        double gx = 0.0, gy = 0.0;
        for (long long i = p * kThreads + threadIdx.x; i < N; i += stride) {
            const int32_t c = b.copy_from[i];
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
            double px = 0.0, py = 0.0;
            for (int w = 0; w < kThreads / 32; ++w) {
                px += sh[0][w];
                py += sh[1][w];
            }
            tx += px;
            ty += py;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        b.hist_mean_x[t] = (anchored ? b.obs_x[t] : 0.0) + tx / (double)N;
        b.hist_mean_y[t] = (anchored ? b.obs_y[t] : 0.0) + ty / (double)N;
        b.ctl->monitor_done = t;
    }
}

} // namespace vsmc_b200

using namespace vsmc_b200;

struct vsmc_cuda_cv_batch {
    vsmc_cuda_cv_config model;
    BatchConst bc;
    cudaStream_t stream;
    cudaMemPool_t pool;
    uint32_t capacity;
    uint64_t budget;
    uint64_t in_use;
    BatchSlot *d_slots;
    std::vector<BatchSlot> slots; // host copies of the records
    std::vector<char *> mem;      // per slot; nullptr = free
    std::vector<uint64_t> bytes;
    std::vector<uint64_t> t;      // steps enqueued
    std::vector<uint64_t> T_obs;  // observations held
    // work list: slot indices, tile offsets; pinned staging for both
    int32_t *d_work;
    int32_t *d_tile0;
    int32_t *h_work;
    TileRef *d_map;
    size_t map_cap;
    cudaEvent_t staged; // the last copy out of the pinned staging is done
    // observations staging
    ObsRecord *d_rec;
    ObsRecord *h_rec;
    double *d_obs;
    size_t obs_cap;
    double *h_obs; // pinned, 2 x capacity (append)
    BatchSlot *h_slot; // pinned staging of one slot record
    double *d_out;
    double *h_out;
    // per-step read-back (vsmc_cuda_cv_batch_read_steps), grown on demand
    double *d_steps;
    double *h_steps;
    size_t steps_cap; // steps, 3 doubles each
    uint64_t launches;
    // graph of the last run (vsmc_cuda_cv_batch_run)
    bool use_graphs;
    cudaStream_t cap_stream; // capture only; graphs launch on `stream`
    cudaGraphExec_t run_exec;
    std::vector<uint64_t> run_key;
    const TileRef *run_map;
    uint64_t run_launches;
    // launch shapes (vsmc_cuda_cv_batch_autotune); no result depends on them
    int tune_move;        // x 256 threads per SM the move is compiled for: 2, 3, 4
    int tune_final;       // finalize CTA size: 256 or 1024
    int max_ntiles;       // largest slot admitted, in tiles
    // tiling (vsmc_cuda_cv_batch_autotune): filters of at most tune_block
    // tiles run block-per-filter in kb_block_run (0: every filter runs
    // grid-per-filter); no result depends on it
    int tune_block;
    int sms;                  // multiprocessors of the device
    BlockItem *d_items;       // capacity block-per-filter work items
    BlockItem *h_items;       // pinned staging
    int *d_queue;             // kb_block_run's work counter
    cudaEvent_t items_staged; // the last copy out of h_items is done
    cudaStream_t block_stream;     // block-per-filter launches
    cudaStream_t block_cap_stream; // their capture twin
    cudaEvent_t ev_fork, ev_join;
};

namespace {

bool is_residual(int s)
{
    return s == VSMC_CUDA_RESIDUAL || s == VSMC_CUDA_RESIDUAL_STRATIFIED ||
           s == VSMC_CUDA_RESIDUAL_SYSTEMATIC;
}

bool is_sys(int s)
{
    return s == VSMC_CUDA_SYSTEMATIC || s == VSMC_CUDA_RESIDUAL_SYSTEMATIC;
}

bool is_strat(int s)
{
    return s == VSMC_CUDA_STRATIFIED || s == VSMC_CUDA_RESIDUAL_STRATIFIED;
}

size_t slot_bytes(const vsmc_cuda_cv_config &m, uint64_t N, uint64_t T)
{
    const size_t real = m.form == VSMC_CUDA_MIXED ? 4 : 8;
    const size_t nt = (N + kTile - 1) / kTile;
    size_t b = 0;
    b += 8 * align256(N * real);                 // two state buffers
    b += align256(N * real);                     // log-weights
    b += align256(N * 4);                        // copy_from
    b += align256(sizeof(FilterCtl));
    b += align256(nt * sizeof(TileStats));
    b += 2 * align256(T * 8);                    // observations
    b += 4 * align256(T * 8) + align256(T * 4);  // histories
    b += resample_workspace_bytes((long long)N);
    return b;
}

void carve_slot(BatchSlot &s, char *p, const vsmc_cuda_cv_config &m,
                uint64_t N, uint64_t T)
{
    const size_t real = m.form == VSMC_CUDA_MIXED ? 4 : 8;
    const size_t nt = (N + kTile - 1) / kTile;
    for (int b = 0; b < 2; ++b)
        for (int d = 0; d < 4; ++d) {
            s.state[b][d] = p;
            p += align256(N * real);
        }
    s.lw = p;
    p += align256(N * real);
    s.copy_from = reinterpret_cast<int32_t *>(p);
    p += align256(N * 4);
    s.ctl = reinterpret_cast<FilterCtl *>(p);
    p += align256(sizeof(FilterCtl));
    s.tile_stats = reinterpret_cast<TileStats *>(p);
    p += align256(nt * sizeof(TileStats));
    s.obs_x = reinterpret_cast<double *>(p);
    p += align256(T * 8);
    s.obs_y = reinterpret_cast<double *>(p);
    p += align256(T * 8);
    s.hist_ess = reinterpret_cast<double *>(p);
    p += align256(T * 8);
    s.hist_logz_inc = reinterpret_cast<double *>(p);
    p += align256(T * 8);
    s.hist_mean_x = reinterpret_cast<double *>(p);
    p += align256(T * 8);
    s.hist_mean_y = reinterpret_cast<double *>(p);
    p += align256(T * 8);
    s.hist_resampled = reinterpret_cast<int32_t *>(p);
    p += align256(T * 4);
    s.rws = carve_workspace(p, (long long)N);
    s.N = (long long)N;
    s.T_max = (long long)T;
    s.t = 0;
    s.ntiles = (int)nt;
}

bool valid_slot(const vsmc_cuda_cv_batch *b, uint32_t s)
{
    return s < b->capacity && b->mem[s] != nullptr;
}

// Copies the work list into the device arrays: slots in the given order,
// tile offsets as their exclusive prefix.  Returns the tile total.
int stage_work(vsmc_cuda_cv_batch *b, const std::vector<uint32_t> &w,
               long long *tiles)
{
    const int n = (int)w.size();
    cudaError_t e = cudaEventSynchronize(b->staged);
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_cv_batch: staging");
    long long acc = 0;
    int32_t *hw = b->h_work;
    int32_t *ht = b->h_work + b->capacity;
    for (int k = 0; k < n; ++k) {
        hw[k] = (int32_t)w[k];
        ht[k] = (int32_t)acc;
        acc += b->slots[w[k]].ntiles;
    }
    ht[n] = (int32_t)acc;
    if (acc > 0x7FFFFFFFLL) {
        set_last_error("vsmc_cuda_cv_batch: more than 2^31 tiles in a step");
        return VSMC_CUDA_EINVAL;
    }
    if ((size_t)acc > b->map_cap) {
        if (b->d_map != nullptr)
            cudaFreeAsync(b->d_map, b->stream);
        b->d_map = nullptr;
        size_t cap = std::max<size_t>((size_t)acc, 2 * b->map_cap);
        e = cudaMallocFromPoolAsync(reinterpret_cast<void **>(&b->d_map),
                                    cap * sizeof(TileRef), b->pool,
                                    b->stream);
        if (e != cudaSuccess) {
            b->map_cap = 0;
            return cuda_status(e, "vsmc_cuda_cv_batch: tile map");
        }
        b->map_cap = cap;
    }
    e = cudaMemcpyAsync(b->d_work, hw, (size_t)n * 4, cudaMemcpyHostToDevice,
                        b->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->d_tile0, ht, (size_t)(n + 1) * 4,
                            cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess)
        e = cudaEventRecord(b->staged, b->stream);
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_cv_batch: work list");
    if (n > 0) {
        kb_expand<<<n, 256, 0, b->stream>>>(b->d_slots, b->d_work,
                                            b->d_tile0, n, b->d_map);
        ++b->launches;
    }
    *tiles = acc;
    return VSMC_CUDA_OK;
}

// One step of the first n work items (whose tiles are the first `tiles`
// map entries).
template <typename Real>
void launch_batch_step(vsmc_cuda_cv_batch *b, int n, long long tiles,
                       cudaStream_t s)
{
    const int scheme = b->model.scheme;
    const bool residual = is_residual(scheme), sys = is_sys(scheme),
               strat = is_strat(scheme);
    const unsigned nt = (unsigned)tiles;
    const BatchSlot *sl = b->d_slots;
    const TileRef *map = b->d_map;
    const int32_t *work = b->d_work;
    switch (b->tune_move) {
    case 2:
        kb_move<Real, 2><<<nt, kMoveThreads, 0, s>>>(
            sl, map, b->bc.p);
        break;
    case 4:
        kb_move<Real, 4><<<nt, kMoveThreads, 0, s>>>(
            sl, map, b->bc.p);
        break;
    default:
        kb_move<Real, 3><<<nt, kMoveThreads, 0, s>>>(
            sl, map, b->bc.p);
        break;
    }
    // a finalize CTA narrower than 1024 threads gives the same sums only
    // while every slot has at most 256 tiles
    kb_finalize<<<n, b->max_ntiles <= 256 ? b->tune_final : kFinalThreads, 0,
                  s>>>(sl, work, b->bc);
    // the per-filter spines on 256 threads while every slot has at most 256
    // tiles (each thread then holds at most one tile, so the sums are those
    // of 1024 threads): four times the spine CTAs fit on an SM
    const int spt = b->max_ntiles <= 256 ? 256 : kSpineThreads;
    int launches = 2;
    if (WeightsFromLog<Real>::kExactNorm) {
        // the weights' sequential sum, whose reciprocal normalises them
        kb_exact_tiles_staged<SlotWeights<Real, false>, false, true>
            <<<exact_grid((int)nt), kThreads, 0, s>>>(sl, map, (int)nt);
        kb_exact_spine<Real, false, true><<<n, spt, 0, s>>>(sl,
                                                                     work);
        launches += 2;
    }
    if (residual) {
        kb_tile_sums<Real, true><<<nt, kThreads, 0, s>>>(sl, map);
        if (sys)
            kb_spine_weights<true, true><<<n, spt, 0, s>>>(sl,
                                                                    work);
        else
            kb_spine_weights<true, false><<<n, spt, 0, s>>>(sl,
                                                                     work);
        launches += 2;
    }
    if (strat) {
        kb_uniforms_stratified<<<nt, kThreads, 0, s>>>(sl, map);
        launches += 1;
    } else if (!sys) {
        kb_sorted_tile_sums<<<nt, kThreads, 0, s>>>(sl, map);
        kb_sorted_spine<<<n, spt, 0, s>>>(sl, work);
        kb_exact_tiles_staged<SlotTerms, false, false>
            <<<exact_grid((int)nt), kThreads, 0, s>>>(sl, map, (int)nt);
        kb_exact_terms_spine<<<n, spt, 0, s>>>(sl, work);
        kb_sorted_uniforms<<<nt, kThreads, 0, s>>>(sl, map);
        launches += 5;
    }
    if (residual) {
        if (!WeightsFromLog<Real>::kApprox) { // the residuals' exact sum
            kb_exact_tiles_staged<SlotWeights<Real, true>, true, true>
                <<<exact_grid((int)nt), kThreads, 0, s>>>(sl, map, (int)nt);
            kb_exact_spine<Real, true, true><<<n, spt, 0, s>>>(
                sl, work);
            launches += 2;
        }
        kb_exact_tiles_staged<SlotWeights<Real, true>, true, false>
            <<<exact_grid((int)nt), kThreads, 0, s>>>(sl, map, (int)nt);
        kb_exact_spine<Real, true><<<n, spt, 0, s>>>(sl, work);
    } else {
        kb_exact_tiles_staged<SlotWeights<Real, true>, false, false>
            <<<exact_grid((int)nt), kThreads, 0, s>>>(sl, map, (int)nt);
        kb_exact_spine<Real, false><<<n, spt, 0, s>>>(sl, work);
    }
    launches += 2;
    if (residual && sys)
        kb_invert<Real, true, true><<<nt, kThreads, 0, s>>>(sl, map);
    else if (residual)
        kb_invert<Real, true, false><<<nt, kThreads, 0, s>>>(sl, map);
    else if (sys)
        kb_invert<Real, false, true><<<nt, kThreads, 0, s>>>(sl, map);
    else
        kb_invert<Real, false, false><<<nt, kThreads, 0, s>>>(sl, map);
    kb_zero_spine<<<n, spt, 0, s>>>(sl, work);
    kb_cfrp_fill<<<nt, kThreads, 0, s>>>(sl, map);
    kb_step_done<<<(n + 255) / 256, 256, 0, s>>>(b->d_slots, b->d_work, n);
    launches += 4;
    b->launches += launches;
}

void launch_step_any(vsmc_cuda_cv_batch *b, int n, long long tiles,
                     cudaStream_t s)
{
    if (b->model.form == VSMC_CUDA_MIXED)
        launch_batch_step<float>(b, n, tiles, s);
    else
        launch_batch_step<double>(b, n, tiles, s);
}

void drop_run_graph(vsmc_cuda_cv_batch *b)
{
    if (b->run_exec != nullptr) {
        cudaStreamSynchronize(b->stream); // the last launch has finished
        cudaGraphExecDestroy(b->run_exec);
    }
    b->run_exec = nullptr;
    b->run_key.clear();
}

// The steps of a run: step k runs the first active(k) work items.
void launch_run_steps(vsmc_cuda_cv_batch *b, const std::vector<int> &active,
                      const std::vector<long long> &tile0, cudaStream_t s)
{
    for (int a : active)
        launch_step_any(b, a, tile0[a], s);
}

// The block-per-filter part of a run: `bs` forks from `s`, resets the work
// counter and runs one persistent kb_block_run over the staged items; the
// grid-per-filter steps go on `s` meanwhile; join_block_part joins them.
void launch_block_part(vsmc_cuda_cv_batch *b, int nitems, cudaStream_t s,
                       cudaStream_t bs)
{
    cudaEventRecord(b->ev_fork, s);
    cudaStreamWaitEvent(bs, b->ev_fork, 0);
    cudaMemsetAsync(b->d_queue, 0, sizeof(int), bs);
    const int grid = std::min(nitems, kBlockCtasPerSm * b->sms);
    if (b->model.form == VSMC_CUDA_MIXED)
        launch_block_real<float>(b->model.scheme, b->d_slots, b->d_items,
                                 nitems, b->d_queue, b->bc, grid, bs);
    else
        launch_block_real<double>(b->model.scheme, b->d_slots, b->d_items,
                                  nitems, b->d_queue, b->bc, grid, bs);
    b->launches += 1;
}

void join_block_part(vsmc_cuda_cv_batch *b, cudaStream_t s, cudaStream_t bs)
{
    cudaEventRecord(b->ev_join, bs);
    cudaStreamWaitEvent(s, b->ev_join, 0);
}

// Items of the block-per-filter part (slot, remaining steps), the largest
// work first, copied to the device on the batch's stream.
int stage_block_items(vsmc_cuda_cv_batch *b, const std::vector<uint32_t> &sm)
{
    cudaError_t e = cudaEventSynchronize(b->items_staged);
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_cv_batch: block staging");
    std::vector<uint32_t> o(sm);
    std::stable_sort(o.begin(), o.end(), [b](uint32_t a, uint32_t c) {
        const double wa = (double)b->slots[a].N * (double)(b->T_obs[a] - b->t[a]);
        const double wc = (double)b->slots[c].N * (double)(b->T_obs[c] - b->t[c]);
        return wa > wc;
    });
    for (size_t k = 0; k < o.size(); ++k)
        b->h_items[k] = BlockItem{(int32_t)o[k],
                                  (int32_t)(b->T_obs[o[k]] - b->t[o[k]])};
    e = cudaMemcpyAsync(b->d_items, b->h_items, o.size() * sizeof(BlockItem),
                        cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess)
        e = cudaEventRecord(b->items_staged, b->stream);
    return e == cudaSuccess ? VSMC_CUDA_OK
                            : cuda_status(e, "vsmc_cuda_cv_batch: block items");
}

int check_slots(const vsmc_cuda_cv_batch *b, uint32_t n,
                const uint32_t *slots, const char *what)
{
    if (b == nullptr || (n > 0 && slots == nullptr) || n > b->capacity) {
        set_last_error(std::string(what) + ": invalid arguments");
        return VSMC_CUDA_EINVAL;
    }
    std::vector<char> seen(b->capacity, 0);
    for (uint32_t k = 0; k < n; ++k) {
        if (!valid_slot(b, slots[k])) {
            set_last_error(std::string(what) + ": slot " +
                           std::to_string(slots[k]) + " is not admitted");
            return VSMC_CUDA_EINVAL;
        }
        if (seen[slots[k]]) {
            set_last_error(std::string(what) + ": slot " +
                           std::to_string(slots[k]) + " listed twice");
            return VSMC_CUDA_EINVAL;
        }
        seen[slots[k]] = 1;
    }
    return VSMC_CUDA_OK;
}

int grow_obs(vsmc_cuda_cv_batch *b, size_t values)
{
    if (values <= b->obs_cap)
        return VSMC_CUDA_OK;
    if (b->d_obs != nullptr)
        cudaFreeAsync(b->d_obs, b->stream);
    b->d_obs = nullptr;
    const size_t cap = std::max(values, 2 * b->obs_cap);
    cudaError_t e = cudaMallocFromPoolAsync(
        reinterpret_cast<void **>(&b->d_obs), 2 * cap * sizeof(double),
        b->pool, b->stream);
    if (e != cudaSuccess) {
        b->obs_cap = 0;
        return cuda_status(e, "vsmc_cuda_cv_batch: observation staging");
    }
    b->obs_cap = cap;
    return VSMC_CUDA_OK;
}

} // namespace

extern "C" {

uint64_t vsmc_cuda_cv_batch_slot_bytes(const vsmc_cuda_cv_config *model,
                                       uint64_t N, uint64_t T_max)
{
    if (model == nullptr || N < 2 || N > (1ull << 30) || T_max < 1 ||
        T_max > (1ull << 31))
        return 0;
    return slot_bytes(*model, N, T_max);
}

int vsmc_cuda_cv_batch_create(const vsmc_cuda_cv_config *model,
                              uint32_t capacity, uint64_t hbm_budget,
                              void *stream, vsmc_cuda_cv_batch **out)
{
    if (out == nullptr || model == nullptr || capacity == 0 ||
        capacity > (1u << 24) || model->scheme < 0 || model->scheme > 5 ||
        (model->form != VSMC_CUDA_FP64 && model->form != VSMC_CUDA_MIXED) ||
        !(model->threshold >= 0.0)) {
        set_last_error("vsmc_cuda_cv_batch_create: invalid arguments");
        return VSMC_CUDA_EINVAL;
    }
    *out = nullptr;
    vsmc_cuda_cv_batch *b = new (std::nothrow) vsmc_cuda_cv_batch();
    if (b == nullptr)
        return VSMC_CUDA_ENOMEM;
    b->model = *model;
    b->bc.p = cv_param(*model);
    b->bc.threshold = model->threshold;
    b->bc.residual = is_residual(model->scheme);
    b->bc.sys = is_sys(model->scheme);
    b->bc.anchored = model->form == VSMC_CUDA_MIXED;
    b->stream = static_cast<cudaStream_t>(stream);
    b->capacity = capacity;
    b->budget = hbm_budget;
    b->in_use = 0;
    b->slots.resize(capacity);
    b->mem.assign(capacity, nullptr);
    b->bytes.assign(capacity, 0);
    b->t.assign(capacity, 0);
    b->T_obs.assign(capacity, 0);
    b->d_map = nullptr;
    b->map_cap = 0;
    b->d_obs = nullptr;
    b->obs_cap = 0;
    b->launches = 0;
    b->d_steps = nullptr;
    b->h_steps = nullptr;
    b->steps_cap = 0;
    b->use_graphs = true;
    // the autotuner's usual pick on mixed workloads; 256-thread finalize
    // applies only while every filter has at most 256 tiles
    b->tune_move = 4;
    b->tune_final = 256;
    b->max_ntiles = 0;
    b->tune_block = 0;
    b->sms = 148;
    b->d_items = nullptr;
    b->h_items = nullptr;
    b->d_queue = nullptr;
    b->items_staged = nullptr;
    b->block_stream = nullptr;
    b->block_cap_stream = nullptr;
    b->ev_fork = nullptr;
    b->ev_join = nullptr;
    b->run_exec = nullptr;
    b->run_map = nullptr;
    b->run_launches = 0;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    if (e == cudaSuccess)
        e = cudaMemPoolCreate(&b->pool, &props);
    if (e != cudaSuccess) {
        delete b;
        return cuda_status(e, "vsmc_cuda_cv_batch_create: memory pool");
    }
    // keep freed slots' memory in the pool for the next admissions
    uint64_t keep = ~0ull;
    cudaMemPoolSetAttribute(b->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    if (hbm_budget > 0) {
        // hold the budget from the start: admissions then carve slots out
        // of memory the pool already has instead of growing it one slot at
        // a time (which stalled a busy serving loop); best effort
        void *r = nullptr;
        if (cudaMallocFromPoolAsync(&r, hbm_budget, b->pool, b->stream) ==
            cudaSuccess) {
            cudaFreeAsync(r, b->stream);
            cudaStreamSynchronize(b->stream);
        } else {
            cudaGetLastError();
        }
    }
    const size_t n = capacity;
    e = cudaMalloc(&b->d_slots, n * sizeof(BatchSlot));
    if (e == cudaSuccess)
        e = cudaMalloc(&b->d_work, (2 * n + 1) * 4);
    if (e == cudaSuccess)
        e = cudaMalloc(&b->d_rec, n * sizeof(ObsRecord));
    if (e == cudaSuccess)
        e = cudaMalloc(&b->d_out, n * 5 * sizeof(double));
    if (e == cudaSuccess)
        e = cudaMallocHost(&b->h_work, (2 * n + 1) * 4);
    if (e == cudaSuccess)
        e = cudaMallocHost(&b->h_rec, n * sizeof(ObsRecord));
    if (e == cudaSuccess)
        e = cudaMallocHost(&b->h_obs, 2 * n * sizeof(double));
    if (e == cudaSuccess)
        e = cudaMallocHost(&b->h_out, n * 5 * sizeof(double));
    if (e == cudaSuccess)
        e = cudaMallocHost(&b->h_slot, sizeof(BatchSlot));
    if (e == cudaSuccess)
        e = cudaEventCreateWithFlags(&b->staged, cudaEventDisableTiming);
    if (e == cudaSuccess)
        e = cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess)
        e = cudaMalloc(&b->d_items, n * sizeof(BlockItem) + 256);
    if (e == cudaSuccess) {
        b->d_queue = reinterpret_cast<int *>(b->d_items + n); // after items
        e = cudaMallocHost(&b->h_items, n * sizeof(BlockItem));
    }
    if (e == cudaSuccess)
        e = cudaEventCreateWithFlags(&b->items_staged, cudaEventDisableTiming);
    if (e == cudaSuccess)
        e = cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess)
        e = cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming);
    if (e == cudaSuccess)
        e = cudaStreamCreateWithFlags(&b->block_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess)
        e = cudaStreamCreateWithFlags(&b->block_cap_stream,
                                      cudaStreamNonBlocking);
    if (e == cudaSuccess)
        e = cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount,
                                   dev);
    if (e == cudaSuccess)
        e = set_block_smem(model->scheme, model->form);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_last_error("vsmc_cuda_cv_batch_create: allocation failed");
        // partial allocations are released by destroy
        vsmc_cuda_cv_batch_destroy(b);
        return VSMC_CUDA_ENOMEM;
    }
    b->d_tile0 = b->d_work + n;
    e = cudaMemsetAsync(b->d_slots, 0, n * sizeof(BatchSlot), b->stream);
    if (e == cudaSuccess)
        e = cudaEventRecord(b->staged, b->stream);
    if (e == cudaSuccess)
        e = cudaEventRecord(b->items_staged, b->stream);
    if (e != cudaSuccess) {
        vsmc_cuda_cv_batch_destroy(b);
        return cuda_status(e, "vsmc_cuda_cv_batch_create");
    }
    *out = b;
    return VSMC_CUDA_OK;
}

int vsmc_cuda_cv_batch_destroy(vsmc_cuda_cv_batch *b)
{
    if (b == nullptr)
        return VSMC_CUDA_OK;
    cudaStreamSynchronize(b->stream);
    for (char *m : b->mem)
        if (m != nullptr)
            cudaFreeAsync(m, b->stream);
    if (b->d_map != nullptr)
        cudaFreeAsync(b->d_map, b->stream);
    if (b->d_obs != nullptr)
        cudaFreeAsync(b->d_obs, b->stream);
    cudaStreamSynchronize(b->stream);
    cudaFree(b->d_slots);
    cudaFree(b->d_work);
    cudaFree(b->d_rec);
    cudaFree(b->d_out);
    cudaFree(b->d_steps);
    cudaFreeHost(b->h_steps);
    cudaFreeHost(b->h_work);
    cudaFreeHost(b->h_rec);
    cudaFreeHost(b->h_obs);
    cudaFreeHost(b->h_out);
    cudaFreeHost(b->h_slot);
    cudaEventDestroy(b->staged);
    drop_run_graph(b);
    if (b->cap_stream != nullptr)
        cudaStreamDestroy(b->cap_stream);
    if (b->block_stream != nullptr) {
        cudaStreamSynchronize(b->block_stream);
        cudaStreamDestroy(b->block_stream);
    }
    if (b->block_cap_stream != nullptr)
        cudaStreamDestroy(b->block_cap_stream);
    cudaFree(b->d_items);
    cudaFreeHost(b->h_items);
    if (b->items_staged != nullptr)
        cudaEventDestroy(b->items_staged);
    if (b->ev_fork != nullptr)
        cudaEventDestroy(b->ev_fork);
    if (b->ev_join != nullptr)
        cudaEventDestroy(b->ev_join);
    cudaMemPoolDestroy(b->pool);
    cudaError_t e = cudaGetLastError();
    delete b;
    return e == cudaSuccess ? VSMC_CUDA_OK
                            : cuda_status(e, "vsmc_cuda_cv_batch_destroy");
}

int vsmc_cuda_cv_batch_admit(vsmc_cuda_cv_batch *b, uint64_t N,
                             uint64_t T_max, uint32_t seed,
                             uint32_t stream_id, uint32_t *slot)
{
    if (b == nullptr || slot == nullptr || N < 2 || N > (1ull << 30) ||
        T_max < 1 || T_max > (1ull << 31)) {
        set_last_error("vsmc_cuda_cv_batch_admit: invalid arguments");
        return VSMC_CUDA_EINVAL;
    }
    uint32_t s = 0;
    while (s < b->capacity && b->mem[s] != nullptr)
        ++s;
    if (s == b->capacity) {
        set_last_error("vsmc_cuda_cv_batch_admit: every slot is in use");
        return VSMC_CUDA_ENOMEM;
    }
    const uint64_t bytes = slot_bytes(b->model, N, T_max);
    if (b->budget != 0 && b->in_use + bytes > b->budget) {
        set_last_error("vsmc_cuda_cv_batch_admit: " + std::to_string(bytes) +
                       " bytes exceed the remaining budget of " +
                       std::to_string(b->budget - b->in_use));
        return VSMC_CUDA_ENOMEM;
    }
    char *m = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(reinterpret_cast<void **>(&m),
                                            bytes, b->pool, b->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_last_error("vsmc_cuda_cv_batch_admit: device allocation of " +
                       std::to_string(bytes) + " bytes failed");
        return VSMC_CUDA_ENOMEM;
    }
    BatchSlot &r = b->slots[s];
    std::memset(&r, 0, sizeof(r));
    carve_slot(r, m, b->model, N, T_max);
    r.eng = cv_resample_engine(seed);
    r.k0 = cv_model_key(seed);
    r.stream_id = stream_id;
    e = cudaMemsetAsync(m, 0, bytes, b->stream);
    if (e == cudaSuccess)
        e = cudaEventSynchronize(b->staged);
    if (e == cudaSuccess) {
        // the record travels through the pinned staging
        *b->h_slot = r;
        e = cudaMemcpyAsync(b->d_slots + s, b->h_slot, sizeof(r),
                            cudaMemcpyHostToDevice, b->stream);
    }
    if (e == cudaSuccess)
        e = cudaEventRecord(b->staged, b->stream);
    if (e != cudaSuccess) {
        cudaFreeAsync(m, b->stream);
        return cuda_status(e, "vsmc_cuda_cv_batch_admit");
    }
    kb_reset_slot<<<1, 32, 0, b->stream>>>(b->d_slots, (int)s);
    ++b->launches;
    b->mem[s] = m;
    if (r.ntiles > b->max_ntiles)
        b->max_ntiles = r.ntiles;
    b->bytes[s] = bytes;
    b->in_use += bytes;
    b->t[s] = 0;
    b->T_obs[s] = 0;
    *slot = s;
    return VSMC_CUDA_OK;
}

int vsmc_cuda_cv_batch_release(vsmc_cuda_cv_batch *b, uint32_t slot)
{
    if (b == nullptr || !valid_slot(b, slot)) {
        set_last_error("vsmc_cuda_cv_batch_release: slot not admitted");
        return VSMC_CUDA_EINVAL;
    }
    cudaError_t e = cudaFreeAsync(b->mem[slot], b->stream);
    b->mem[slot] = nullptr;
    b->in_use -= b->bytes[slot];
    b->bytes[slot] = 0;
    return e == cudaSuccess ? VSMC_CUDA_OK
                            : cuda_status(e, "vsmc_cuda_cv_batch_release");
}

int vsmc_cuda_cv_batch_bytes_in_use(vsmc_cuda_cv_batch *b, uint64_t *bytes)
{
    if (b == nullptr || bytes == nullptr)
        return VSMC_CUDA_EINVAL;
    *bytes = b->in_use;
    return VSMC_CUDA_OK;
}

int vsmc_cuda_cv_batch_set_observations(vsmc_cuda_cv_batch *b, uint32_t n,
                                        const uint32_t *slots,
                                        const uint64_t *T, const double *ox,
                                        const double *oy, int on_device)
{
    int st = check_slots(b, n, slots, "vsmc_cuda_cv_batch_set_observations");
    if (st != VSMC_CUDA_OK)
        return st;
    if (n > 0 && (T == nullptr || ox == nullptr || oy == nullptr)) {
        set_last_error("vsmc_cuda_cv_batch_set_observations: null array");
        return VSMC_CUDA_EINVAL;
    }
    size_t total = 0;
    for (uint32_t k = 0; k < n; ++k) {
        const uint32_t s = slots[k];
        if (T[k] == 0 || T[k] > (uint64_t)b->slots[s].T_max ||
            T[k] > 0x7FFFFFFFull) {
            set_last_error("vsmc_cuda_cv_batch_set_observations: slot " +
                           std::to_string(s) + " series length invalid");
            return VSMC_CUDA_EINVAL;
        }
        total += T[k];
    }
    if (n == 0)
        return VSMC_CUDA_OK;
    st = grow_obs(b, total);
    if (st != VSMC_CUDA_OK)
        return st;
    cudaError_t e = cudaEventSynchronize(b->staged);
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_cv_batch_set_observations");
    size_t off = 0;
    for (uint32_t k = 0; k < n; ++k) {
        ObsRecord r;
        r.slot = (int32_t)slots[k];
        r.count = (int32_t)T[k];
        r.index = 0;
        r.src = (long long)off;
        b->h_rec[k] = r;
        off += T[k];
    }
    const cudaMemcpyKind kind =
        on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    e = cudaMemcpyAsync(b->d_obs, ox, total * 8, kind, b->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->d_obs + b->obs_cap, oy, total * 8, kind,
                            b->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->d_rec, b->h_rec, n * sizeof(ObsRecord),
                            cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess)
        e = cudaEventRecord(b->staged, b->stream);
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_cv_batch_set_observations");
    kb_scatter_obs<<<n, 256, 0, b->stream>>>(b->d_slots, b->d_rec, b->d_obs,
                                             b->d_obs + b->obs_cap);
    ++b->launches;
    for (uint32_t k = 0; k < n; ++k)
        b->T_obs[slots[k]] = T[k];
    e = cudaGetLastError();
    return e == cudaSuccess
               ? VSMC_CUDA_OK
               : cuda_status(e, "vsmc_cuda_cv_batch_set_observations");
}

int vsmc_cuda_cv_batch_append_observations(vsmc_cuda_cv_batch *b,
                                           uint32_t n, const uint32_t *slots,
                                           const double *x, const double *y)
{
    int st =
        check_slots(b, n, slots, "vsmc_cuda_cv_batch_append_observations");
    if (st != VSMC_CUDA_OK)
        return st;
    if (n == 0)
        return VSMC_CUDA_OK;
    if (x == nullptr || y == nullptr) {
        set_last_error("vsmc_cuda_cv_batch_append_observations: null array");
        return VSMC_CUDA_EINVAL;
    }
    for (uint32_t k = 0; k < n; ++k)
        if (b->T_obs[slots[k]] >= (uint64_t)b->slots[slots[k]].T_max) {
            set_last_error("vsmc_cuda_cv_batch_append_observations: slot " +
                           std::to_string(slots[k]) + " is full");
            return VSMC_CUDA_EINVAL;
        }
    cudaError_t e = cudaEventSynchronize(b->staged);
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_cv_batch_append_observations");
    // pinned staging: records, then x values, then y values (in h_obs)
    for (uint32_t k = 0; k < n; ++k) {
        ObsRecord r;
        r.slot = (int32_t)slots[k];
        r.count = 1;
        r.index = (long long)b->T_obs[slots[k]];
        r.src = (long long)k;
        b->h_rec[k] = r;
        b->h_obs[k] = x[k];
        b->h_obs[b->capacity + k] = y[k];
    }
    st = grow_obs(b, b->capacity);
    if (st != VSMC_CUDA_OK)
        return st;
    e = cudaMemcpyAsync(b->d_rec, b->h_rec, n * sizeof(ObsRecord),
                        cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->d_obs, b->h_obs, n * 8,
                            cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->d_obs + b->obs_cap, b->h_obs + b->capacity,
                            n * 8, cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess)
        e = cudaEventRecord(b->staged, b->stream);
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_cv_batch_append_observations");
    kb_scatter_obs<<<n, 32, 0, b->stream>>>(b->d_slots, b->d_rec, b->d_obs,
                                            b->d_obs + b->obs_cap);
    ++b->launches;
    for (uint32_t k = 0; k < n; ++k)
        ++b->T_obs[slots[k]];
    e = cudaGetLastError();
    return e == cudaSuccess
               ? VSMC_CUDA_OK
               : cuda_status(e, "vsmc_cuda_cv_batch_append_observations");
}

int vsmc_cuda_cv_batch_initialize(vsmc_cuda_cv_batch *b, uint32_t n,
                                  const uint32_t *slots)
{
    int st = check_slots(b, n, slots, "vsmc_cuda_cv_batch_initialize");
    if (st != VSMC_CUDA_OK)
        return st;
    if (n == 0)
        return VSMC_CUDA_OK;
    std::vector<uint32_t> w(slots, slots + n);
    long long tiles = 0;
    st = stage_work(b, w, &tiles);
    if (st != VSMC_CUDA_OK)
        return st;
    kb_reset<<<(n + 255) / 256, 256, 0, b->stream>>>(b->d_slots, b->d_work,
                                                    (int)n);
    ++b->launches;
    for (uint32_t k = 0; k < n; ++k)
        b->t[slots[k]] = 0;
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? VSMC_CUDA_OK
                            : cuda_status(e, "vsmc_cuda_cv_batch_initialize");
}

int vsmc_cuda_cv_batch_step(vsmc_cuda_cv_batch *b, uint32_t n,
                            const uint32_t *slots)
{
    int st = check_slots(b, n, slots, "vsmc_cuda_cv_batch_step");
    if (st != VSMC_CUDA_OK)
        return st;
    for (uint32_t k = 0; k < n; ++k)
        if (b->t[slots[k]] >= b->T_obs[slots[k]]) {
            set_last_error("vsmc_cuda_cv_batch_step: slot " +
                           std::to_string(slots[k]) +
                           " has no observation for its next step");
            return VSMC_CUDA_EINVAL;
        }
    if (n == 0)
        return VSMC_CUDA_OK;
    std::vector<uint32_t> w(slots, slots + n);
    long long tiles = 0;
    st = stage_work(b, w, &tiles);
    if (st != VSMC_CUDA_OK)
        return st;
    launch_step_any(b, (int)n, tiles, b->stream);
    for (uint32_t k = 0; k < n; ++k)
        ++b->t[slots[k]];
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? VSMC_CUDA_OK
                            : cuda_status(e, "vsmc_cuda_cv_batch_step");
}

int vsmc_cuda_cv_batch_run(vsmc_cuda_cv_batch *b, uint32_t n,
                           const uint32_t *slots)
{
    int st = check_slots(b, n, slots, "vsmc_cuda_cv_batch_run");
    if (st != VSMC_CUDA_OK)
        return st;
    if (n == 0)
        return VSMC_CUDA_OK;
    // small filters (at most tune_block tiles) run block-per-filter, the
    // rest grid-per-filter, longest remaining series first: the slots still
    // running at step k are a prefix of the list, and so are their tiles
    std::vector<uint32_t> all(slots, slots + n), w, small;
    for (uint32_t x : all) {
        if (b->tune_block > 0 && b->slots[x].ntiles <= b->tune_block &&
            b->T_obs[x] > b->t[x])
            small.push_back(x);
        else
            w.push_back(x);
    }
    std::stable_sort(w.begin(), w.end(), [b](uint32_t a, uint32_t c) {
        return b->T_obs[a] - b->t[a] > b->T_obs[c] - b->t[c];
    });
    const uint32_t nw = (uint32_t)w.size();
    if (!small.empty()) {
        st = stage_block_items(b, small);
        if (st != VSMC_CUDA_OK)
            return st;
    }
    long long tiles = 0;
    st = stage_work(b, w, &tiles);
    if (st != VSMC_CUDA_OK)
        return st;
    std::vector<long long> tile0(nw + 1, 0);
    for (uint32_t k = 0; k < nw; ++k)
        tile0[k + 1] = tile0[k] + b->slots[w[k]].ntiles;
    std::vector<int> active;
    int a = (int)nw;
    for (uint64_t step = 0;; ++step) {
        while (a > 0 && b->T_obs[w[a - 1]] - b->t[w[a - 1]] <= step)
            --a;
        if (a == 0)
            break;
        active.push_back(a);
    }
    const int nsmall = (int)small.size();
    cudaError_t e = cudaSuccess;
    if (b->use_graphs && (!active.empty() || nsmall > 0)) {
        // the whole run as one CUDA graph, reused while the work lists and
        // their step counts repeat (kernels read everything else from the
        // slot records and the staged block items)
        std::vector<uint64_t> key;
        key.reserve(2 * n + 2);
        for (uint32_t k = 0; k < nw; ++k) {
            key.push_back(w[k]);
            key.push_back(b->T_obs[w[k]] - b->t[w[k]]);
        }
        key.push_back(~0ull);
        for (uint32_t x : small) {
            key.push_back(x);
            key.push_back(b->T_obs[x] - b->t[x]);
        }
        if (b->run_exec == nullptr || key != b->run_key ||
            b->run_map != b->d_map) {
            drop_run_graph(b);
            cudaGraph_t g = nullptr;
            e = cudaStreamBeginCapture(b->cap_stream,
                                       cudaStreamCaptureModeThreadLocal);
            if (e == cudaSuccess) {
                const uint64_t before = b->launches;
                if (nsmall > 0)
                    launch_block_part(b, nsmall, b->cap_stream,
                                      b->block_cap_stream);
                launch_run_steps(b, active, tile0, b->cap_stream);
                if (nsmall > 0)
                    join_block_part(b, b->cap_stream, b->block_cap_stream);
                b->run_launches = b->launches - before;
                e = cudaStreamEndCapture(b->cap_stream, &g);
            }
            if (e == cudaSuccess)
                e = cudaGraphInstantiate(&b->run_exec, g, 0);
            if (g != nullptr)
                cudaGraphDestroy(g);
            if (e != cudaSuccess) {
                b->run_exec = nullptr;
                return cuda_status(e, "vsmc_cuda_cv_batch_run: graph");
            }
            b->run_key = key;
            b->run_map = b->d_map;
            b->launches -= b->run_launches; // counted when launched
        }
        e = cudaGraphLaunch(b->run_exec, b->stream);
        b->launches += b->run_launches;
    } else {
        if (nsmall > 0)
            launch_block_part(b, nsmall, b->stream, b->block_stream);
        launch_run_steps(b, active, tile0, b->stream);
        if (nsmall > 0)
            join_block_part(b, b->stream, b->block_stream);
    }
    for (uint32_t k = 0; k < n; ++k)
        b->t[slots[k]] = b->T_obs[slots[k]];
    if (e == cudaSuccess)
        e = cudaGetLastError();
    return e == cudaSuccess ? VSMC_CUDA_OK
                            : cuda_status(e, "vsmc_cuda_cv_batch_run");
}

int vsmc_cuda_cv_batch_read_steps(vsmc_cuda_cv_batch *b, uint32_t n,
                                  const uint32_t *slots,
                                  const uint32_t *counts, double *ess,
                                  double *logz_inc, int32_t *resampled,
                                  int32_t *status)
{
    int st = check_slots(b, n, slots, "vsmc_cuda_cv_batch_read_steps");
    if (st != VSMC_CUDA_OK)
        return st;
    if (n == 0)
        return VSMC_CUDA_OK;
    if (counts == nullptr) {
        set_last_error("vsmc_cuda_cv_batch_read_steps: null counts");
        return VSMC_CUDA_EINVAL;
    }
    size_t total = 0;
    for (uint32_t k = 0; k < n; ++k) {
        if (counts[k] == 0 || counts[k] > b->t[slots[k]]) {
            set_last_error("vsmc_cuda_cv_batch_read_steps: slot " +
                           std::to_string(slots[k]) + " has not taken " +
                           std::to_string(counts[k]) + " steps");
            return VSMC_CUDA_EINVAL;
        }
        total += counts[k];
    }
    cudaError_t e = cudaSuccess;
    if (total > b->steps_cap) {
        e = cudaStreamSynchronize(b->stream); // old buffers may be in use
        cudaFree(b->d_steps);
        cudaFreeHost(b->h_steps);
        b->d_steps = nullptr;
        b->h_steps = nullptr;
        b->steps_cap = 0;
        const size_t cap = std::max(total, (size_t)4 * b->capacity);
        if (e == cudaSuccess)
            e = cudaMalloc(&b->d_steps, 3 * cap * sizeof(double));
        if (e == cudaSuccess)
            e = cudaMallocHost(&b->h_steps, 3 * cap * sizeof(double));
        if (e != cudaSuccess)
            return cuda_status(e, "vsmc_cuda_cv_batch_read_steps: buffers");
        b->steps_cap = cap;
    }
    e = cudaEventSynchronize(b->staged);
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_cv_batch_read_steps");
    size_t off = 0;
    for (uint32_t k = 0; k < n; ++k) {
        ObsRecord r;
        r.slot = (int32_t)slots[k];
        r.count = (int32_t)counts[k];
        r.index = (long long)(b->t[slots[k]] - counts[k]);
        r.src = (long long)off;
        b->h_rec[k] = r;
        off += counts[k];
    }
    e = cudaMemcpyAsync(b->d_rec, b->h_rec, n * sizeof(ObsRecord),
                        cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess)
        e = cudaEventRecord(b->staged, b->stream);
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_cv_batch_read_steps");
    kb_read_steps<<<n, 32, 0, b->stream>>>(b->d_slots, b->d_rec, b->d_steps,
                                           b->d_out);
    ++b->launches;
    e = cudaMemcpyAsync(b->h_steps, b->d_steps, 3 * total * sizeof(double),
                        cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->h_out, b->d_out, n * sizeof(double),
                            cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_cv_batch_read_steps");
    int err = VSMC_CUDA_OK;
    for (size_t i = 0; i < total; ++i) {
        const double *o = b->h_steps + 3 * i;
        if (ess)
            ess[i] = o[0];
        if (logz_inc)
            logz_inc[i] = o[1];
        if (resampled)
            resampled[i] = (int32_t)o[2];
    }
    for (uint32_t k = 0; k < n; ++k) {
        const int code = (int)b->h_out[k];
        if (status)
            status[k] = code;
        if (code != VSMC_CUDA_OK && err == VSMC_CUDA_OK)
            err = code;
    }
    if (err != VSMC_CUDA_OK)
        set_last_error("vsmc_cuda_cv_batch_read_steps: a filter's weights "
                       "are degenerate");
    return err;
}

int vsmc_cuda_cv_batch_read_last(vsmc_cuda_cv_batch *b, uint32_t n,
                                 const uint32_t *slots, double *ess,
                                 double *logz_inc, int32_t *resampled,
                                 double *log_evidence, int32_t *status)
{
    int st = check_slots(b, n, slots, "vsmc_cuda_cv_batch_read_last");
    if (st != VSMC_CUDA_OK)
        return st;
    if (n == 0)
        return VSMC_CUDA_OK;
    std::vector<uint32_t> w(slots, slots + n);
    long long tiles = 0;
    st = stage_work(b, w, &tiles);
    if (st != VSMC_CUDA_OK)
        return st;
    kb_read_last<<<(n + 255) / 256, 256, 0, b->stream>>>(
        b->d_slots, b->d_work, (int)n, b->d_out);
    ++b->launches;
    cudaError_t e = cudaMemcpyAsync(b->h_out, b->d_out, n * 5 * 8,
                                    cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_cv_batch_read_last");
    int err = VSMC_CUDA_OK;
    for (uint32_t k = 0; k < n; ++k) {
        const double *o = b->h_out + 5 * k;
        if (ess)
            ess[k] = o[0];
        if (logz_inc)
            logz_inc[k] = o[1];
        if (resampled)
            resampled[k] = (int32_t)o[2];
        if (log_evidence)
            log_evidence[k] = o[3];
        if (status)
            status[k] = (int32_t)o[4];
        if (o[4] != 0.0 && err == VSMC_CUDA_OK)
            err = (int)o[4];
    }
    if (err != VSMC_CUDA_OK)
        set_last_error(err == VSMC_CUDA_EDEGENERATE
                           ? "vsmc_cuda_cv_batch: degenerate weights in a "
                             "listed slot"
                           : "vsmc_cuda_cv_batch: device error in a listed "
                             "slot");
    return err;
}

int vsmc_cuda_cv_batch_iter_size(vsmc_cuda_cv_batch *b, uint32_t slot,
                                 uint64_t *n)
{
    if (b == nullptr || n == nullptr || !valid_slot(b, slot))
        return VSMC_CUDA_EINVAL;
    *n = b->t[slot];
    return VSMC_CUDA_OK;
}

int vsmc_cuda_cv_batch_history(vsmc_cuda_cv_batch *b, uint32_t slot,
                               double *ess, int32_t *resampled,
                               double *logz_inc, double *mean_x,
                               double *mean_y)
{
    if (b == nullptr || !valid_slot(b, slot)) {
        set_last_error("vsmc_cuda_cv_batch_history: slot not admitted");
        return VSMC_CUDA_EINVAL;
    }
    const uint64_t T = b->t[slot];
    if (T == 0)
        return VSMC_CUDA_OK;
    std::vector<uint32_t> w(1, slot);
    long long tiles = 0;
    int st = stage_work(b, w, &tiles);
    if (st != VSMC_CUDA_OK)
        return st;
    if (b->model.form == VSMC_CUDA_MIXED)
        kb_monitor_flush<float><<<1, kThreads, 0, b->stream>>>(
            b->d_slots, b->d_work, 1);
    else
        kb_monitor_flush<double><<<1, kThreads, 0, b->stream>>>(
            b->d_slots, b->d_work, 0);
    ++b->launches;
    const BatchSlot &r = b->slots[slot];
    cudaError_t e = cudaSuccess;
    auto get = [&](void *dst, const void *src, size_t bytes) {
        if (dst != nullptr && e == cudaSuccess)
            e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost,
                                b->stream);
    };
    get(ess, r.hist_ess, T * 8);
    get(resampled, r.hist_resampled, T * 4);
    get(logz_inc, r.hist_logz_inc, T * 8);
    get(mean_x, r.hist_mean_x, T * 8);
    get(mean_y, r.hist_mean_y, T * 8);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(b->stream);
    return e == cudaSuccess ? VSMC_CUDA_OK
                            : cuda_status(e, "vsmc_cuda_cv_batch_history");
}

int vsmc_cuda_cv_batch_synchronize(vsmc_cuda_cv_batch *b)
{
    if (b == nullptr)
        return VSMC_CUDA_EINVAL;
    cudaError_t e = cudaStreamSynchronize(b->stream);
    return e == cudaSuccess ? VSMC_CUDA_OK
                            : cuda_status(e, "vsmc_cuda_cv_batch_synchronize");
}

int vsmc_cuda_cv_batch_set_graphs(vsmc_cuda_cv_batch *b, int enable)
{
    if (b == nullptr)
        return VSMC_CUDA_EINVAL;
    b->use_graphs = enable != 0;
    if (!b->use_graphs) {
        cudaStreamSynchronize(b->stream);
        drop_run_graph(b);
    }
    return VSMC_CUDA_OK;
}

int vsmc_cuda_cv_batch_set_launch_shape(vsmc_cuda_cv_batch *b,
                                        int move_blocks, int final_threads)
{
    if (b == nullptr || move_blocks < 2 || move_blocks > 4 ||
        (final_threads != kFinalThreads && final_threads != 256)) {
        set_last_error("vsmc_cuda_cv_batch_set_launch_shape: invalid "
                       "arguments");
        return VSMC_CUDA_EINVAL;
    }
    if (move_blocks != b->tune_move || final_threads != b->tune_final) {
        drop_run_graph(b); // recorded with the old shapes
        b->tune_move = move_blocks;
        b->tune_final = final_threads;
    }
    return VSMC_CUDA_OK;
}

int vsmc_cuda_cv_batch_set_tiling(vsmc_cuda_cv_batch *b, int block_tiles)
{
    if (b == nullptr || block_tiles < 0 || block_tiles > kBlockMaxTiles) {
        set_last_error("vsmc_cuda_cv_batch_set_tiling: block_tiles must be "
                       "0.." + std::to_string(kBlockMaxTiles));
        return VSMC_CUDA_EINVAL;
    }
    if (block_tiles != b->tune_block) {
        drop_run_graph(b); // recorded with the old tiling
        b->tune_block = block_tiles;
    }
    return VSMC_CUDA_OK;
}

int vsmc_cuda_cv_batch_tiling(vsmc_cuda_cv_batch *b, int *block_tiles)
{
    if (b == nullptr || block_tiles == nullptr)
        return VSMC_CUDA_EINVAL;
    *block_tiles = b->tune_block;
    return VSMC_CUDA_OK;
}

int vsmc_cuda_cv_batch_autotune(vsmc_cuda_cv_batch *b, uint32_t n,
                                const uint32_t *slots, int *move_blocks,
                                int *final_threads)
{
    int st = check_slots(b, n, slots, "vsmc_cuda_cv_batch_autotune");
    if (st != VSMC_CUDA_OK)
        return st;
    if (n == 0)
        return VSMC_CUDA_OK;
    // a sample of the listed filters (every k-th, at most 256 of them and
    // 1 GiB of trial memory) in a trial batch of its own, with zero
    // observations: the trial's steps touch none of this batch's slots
    constexpr uint64_t kTrialT = 8;
    constexpr uint64_t kTrialBytes = 1ull << 30;
    const uint32_t k = (n + 255) / 256;
    std::vector<uint32_t> pick;
    uint64_t trial_bytes = 0;
    for (uint32_t i = 0; i < n; i += k) {
        const uint64_t by = slot_bytes(b->model, b->slots[slots[i]].N, kTrialT);
        if (!pick.empty() && trial_bytes + by > kTrialBytes)
            break;
        pick.push_back(slots[i]);
        trial_bytes += by;
    }
    const uint32_t m = (uint32_t)pick.size();
    vsmc_cuda_cv_batch *t = nullptr;
    st = vsmc_cuda_cv_batch_create(&b->model, m, 0, b->stream, &t);
    if (st != VSMC_CUDA_OK)
        return st;
    t->use_graphs = false;
    std::vector<uint32_t> ts(m);
    std::vector<uint64_t> T(m, kTrialT);
    std::vector<double> zero(m * kTrialT, 0.0);
    for (uint32_t i = 0; i < m && st == VSMC_CUDA_OK; ++i) {
        const BatchSlot &r = b->slots[pick[i]];
        st = vsmc_cuda_cv_batch_admit(t, (uint64_t)r.N, kTrialT, 101 + i,
                                      r.stream_id, &ts[i]);
    }
    if (st == VSMC_CUDA_OK)
        st = vsmc_cuda_cv_batch_set_observations(t, m, ts.data(), T.data(),
                                                 zero.data(), zero.data(), 0);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int best_move = b->tune_move, best_final = b->tune_final;
    float best_ms = 1e30f;
    const int moves[3] = {2, 3, 4};
    const int finals[2] = {kFinalThreads, 256};
    const int nfinal = t->max_ntiles <= 256 ? 2 : 1;
    for (int im = 0; im < 3 && st == VSMC_CUDA_OK; ++im)
        for (int jf = 0; jf < nfinal && st == VSMC_CUDA_OK; ++jf) {
            t->tune_move = moves[im];
            t->tune_final = finals[jf];
            st = vsmc_cuda_cv_batch_initialize(t, m, ts.data());
            if (st == VSMC_CUDA_OK) // the prior step, untimed
                st = vsmc_cuda_cv_batch_step(t, m, ts.data());
            cudaEventRecord(e0, b->stream);
            for (int q = 0; q < 3 && st == VSMC_CUDA_OK; ++q)
                st = vsmc_cuda_cv_batch_step(t, m, ts.data());
            cudaEventRecord(e1, b->stream);
            if (st != VSMC_CUDA_OK)
                break;
            cudaEventSynchronize(e1);
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (ms < best_ms) {
                best_ms = ms;
                best_move = moves[im];
                best_final = finals[jf];
            }
        }
    // tiling: whole trial runs (kTrialT steps) with the filters of at most
    // K tiles block-per-filter, K = 0 (all grid-per-filter) and powers of
    // two up to the largest trial filter
    int best_block = b->tune_block;
    if (st == VSMC_CUDA_OK) {
        t->tune_move = best_move;
        t->tune_final = best_final;
        best_ms = 1e30f;
        for (int K = 0; K <= kBlockMaxTiles && st == VSMC_CUDA_OK;
             K = K == 0 ? 1 : 2 * K) {
            if (K > 1 && K / 2 >= t->max_ntiles)
                break; // every trial filter ran block-per-filter already
            t->tune_block = K;
            float ms = 0.0f;
            for (int rep = 0; rep < 2 && st == VSMC_CUDA_OK; ++rep) {
                st = vsmc_cuda_cv_batch_initialize(t, m, ts.data());
                cudaEventRecord(e0, b->stream);
                if (st == VSMC_CUDA_OK)
                    st = vsmc_cuda_cv_batch_run(t, m, ts.data());
                cudaEventRecord(e1, b->stream);
                cudaEventSynchronize(e1);
                cudaEventElapsedTime(&ms, e0, e1); // the second, warm run
            }
            if (st == VSMC_CUDA_OK && ms < best_ms) {
                best_ms = ms;
                best_block = K;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->launches += t->launches;
    const int dst = vsmc_cuda_cv_batch_destroy(t);
    if (st == VSMC_CUDA_OK)
        st = dst;
    if (st != VSMC_CUDA_OK)
        return st;
    st = vsmc_cuda_cv_batch_set_launch_shape(b, best_move, best_final);
    if (st == VSMC_CUDA_OK)
        st = vsmc_cuda_cv_batch_set_tiling(b, best_block);
    if (st != VSMC_CUDA_OK)
        return st;
    if (move_blocks)
        *move_blocks = b->tune_move;
    if (final_threads)
        *final_threads = b->tune_final;
    return VSMC_CUDA_OK;
}

int vsmc_cuda_cv_batch_launches(vsmc_cuda_cv_batch *b, uint64_t *launches)
{
    if (b == nullptr || launches == nullptr)
        return VSMC_CUDA_EINVAL;
    *launches = b->launches;
    return VSMC_CUDA_OK;
}

} // extern "C"
