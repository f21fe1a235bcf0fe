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
#include "cv_kernels.cuh"

#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

namespace vsmc_b200 {

void set_last_error(const std::string &msg);
int cuda_status(cudaError_t e, const char *what);

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
    // Multinomial: the sorted U01 sequence of the next resampling is drawn
    // on `side` while the step's move and weights run on `stream`
    cudaStream_t side;
    cudaEvent_t ev_pos;  // on stream: the engine position is final
    cudaEvent_t ev_seq;  // on side: the sequence for that position is held
    bool seq_pending;    // a sequence is enqueued after the last ev_pos
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

// Multinomial: enqueue the sorted U01 sequence for the engine position the
// filter's stream has reached, on the side stream (it overlaps the next
// move and weights; the kernels skip when that position's sequence is held).
void enqueue_sequence(vsmc_cuda_cv_filter *f)
{
    cudaEventRecord(f->ev_pos, f->stream);
    cudaStreamWaitEvent(f->side, f->ev_pos, 0);
    launch_spec_sorted((long long)f->cfg.N, f->eng, f->rws, f->side);
    cudaEventRecord(f->ev_seq, f->side);
    f->seq_pending = true;
    f->launches += 6;
}

// The filter's stream waits for the side stream's last sequence (after a
// run of several steps, so that the stream's completion covers the work
// those steps enqueued; single steps leave it running under the next move).
// The side stream writes only the filter's own workspace, which the next
// inversion reads after waiting for it.
void join_sequence(vsmc_cuda_cv_filter *f)
{
    if (f->side != nullptr && f->seq_pending)
        cudaStreamWaitEvent(f->stream, f->ev_seq, 0);
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
    a.k0 = cv_model_key(c.seed);
    a.k1 = 0;
    a.stream = c.stream_id;
    a.p = cv_param(c);
    // the sequence of this step's resampling, drawn while the move runs
    const bool speculate = f->side != nullptr && f->rep_cf == nullptr;
    if (speculate && !f->seq_pending)
        enqueue_sequence(f);
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
        k_cv_move<Real, true><<<f->move_grid, kMoveThreads, 0, s>>>(a);
    else
        k_cv_move<Real, false><<<f->move_grid, kMoveThreads, 0, s>>>(a);
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
    const bool compare = f->rep_cf != nullptr && f->rec_cf != nullptr;
    fa.compare = compare ? 1 : 0;
    const size_t fin_smem = f->ntiles <= kFinalSmemTiles
                                ? (size_t)f->ntiles * sizeof(double)
                                : 0;
    k_cv_finalize<<<1, kFinalThreads, fin_smem, s>>>(fa);

    WeightsFromLog<Real> w;
    w.lw = static_cast<const Real *>(f->lw);
    w.stats = &f->ctl->lw_max;
    if (f->rep_cf != nullptr) {
        if (compare) {
            // the step's own resampling of its own weights, into the
            // record row; the engine advances by the words it drew
            launch_resample_core(c.scheme, w, N, f->eng, f->rws, nullptr, 0,
                                 /*spine_done=*/true, nullptr,
                                 f->rec_cf + (size_t)f->iter * c.N, s);
            f->launches += resample_launches(c.scheme, false,
                                           WeightsFromLog<Real>::kExactNorm,
                                           WeightsFromLog<Real>::kApprox);
        }
        // replay: the recorded ancestry of this step (used only if the
        // recorded decision was to resample)
        cudaMemcpyAsync(f->copy_from, f->rep_cf + (size_t)f->iter * c.N,
                        c.N * 4, cudaMemcpyDeviceToDevice, s);
    } else if (speculate) {
        cudaStreamWaitEvent(s, f->ev_seq, 0);
        launch_resample_core(c.scheme, w, N, f->eng, f->rws, nullptr, 0,
                             /*spine_done=*/true, nullptr, f->copy_from, s,
                             /*sorted_ready=*/true);
        f->launches -= 5; // the sequence's launches are counted on the side
        enqueue_sequence(f); // for the next resampling
    } else {
        launch_resample_core(c.scheme, w, N, f->eng, f->rws, nullptr, 0,
                             /*spine_done=*/true, nullptr, f->copy_from, s);
    }
    if (f->rec_cf != nullptr && !compare)
        cudaMemcpyAsync(f->rec_cf + (size_t)f->iter * c.N, f->copy_from,
                        c.N * 4, cudaMemcpyDeviceToDevice, s);
    if (ev)
        cudaEventRecord(ev[2], s);
    f->launches += 2 + resample_launches(c.scheme, false,
                                           WeightsFromLog<Real>::kExactNorm,
                                           WeightsFromLog<Real>::kApprox);
    ++f->iter;
}

template <typename Real>
void launch_monitor_flush(vsmc_cuda_cv_filter *f)
{
    const long long N = (long long)f->cfg.N;
    const long long t = (long long)f->iter - 1;
    k_cv_monitor_gather<Real><<<kMonParts, kThreads, 0, f->stream>>>(
        static_cast<const Real *>(f->state[f->cur][0]),
        static_cast<const Real *>(f->state[f->cur][1]), f->copy_from, N,
        f->mon_part, f->ctl, t);
    const bool anch = f->cfg.form == VSMC_CUDA_MIXED;
    k_cv_monitor_finish<<<1, 32, 0, f->stream>>>(
        f->mon_part, kMonParts, N, t, f->ctl,
        anch ? f->obs_x : nullptr, anch ? f->obs_y : nullptr,
        f->hist_mean_x, f->hist_mean_y);
}

int sync_and_check(vsmc_cuda_cv_filter *f)
{
    cudaError_t e = cudaStreamSynchronize(f->stream);
    if (e == cudaSuccess && f->side != nullptr)
        e = cudaStreamSynchronize(f->side);
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

// Gathered monitor of a final resampled step, if not yet written; the
// kernels read the decision on the device, so nothing waits here.
int flush_monitor(vsmc_cuda_cv_filter *f)
{
    if (f->iter == 0)
        return VSMC_CUDA_OK;
    if (f->cfg.form == VSMC_CUDA_MIXED)
        launch_monitor_flush<float>(f);
    else
        launch_monitor_flush<double>(f);
    f->launches += 2;
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? VSMC_CUDA_OK : cuda_status(e, "monitor flush");
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
    f->side = nullptr;
    f->ev_pos = nullptr;
    f->ev_seq = nullptr;
    f->seq_pending = false;
    // resample engine: Threefry4x64 seeded seed+2 (Seed::get twice)
    f->eng = cv_resample_engine(cfg->seed);
    cudaFuncSetAttribute(k_cv_finalize,
                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                         kFinalSmemTiles * (int)sizeof(double));
    // one CTA per tile: the block scheduler hands tiles to SMs as they
    // free, which balances the rejection loops' uneven cost better than a
    // persistent grid striding over tiles (measured 5% faster at 2^24)
    f->move_grid = (int)f->ntiles;
    e = cudaMemsetAsync(f->mem, 0, f->bytes, f->stream);
    if (e == cudaSuccess && cfg->scheme == VSMC_CUDA_MULTINOMIAL) {
        // the lowest priority: the sequence fills SMs the step's own
        // kernels leave idle (the one-CTA finalize and spines) instead of
        // competing with the move
        int lo = 0, hi = 0;
        cudaDeviceGetStreamPriorityRange(&lo, &hi);
        e = cudaStreamCreateWithPriority(&f->side, cudaStreamNonBlocking, lo);
        if (e == cudaSuccess)
            e = cudaEventCreateWithFlags(&f->ev_pos, cudaEventDisableTiming);
        if (e == cudaSuccess)
            e = cudaEventCreateWithFlags(&f->ev_seq, cudaEventDisableTiming);
        if (e == cudaSuccess) {
            k_spec_invalidate<<<1, 1, 0, f->stream>>>(f->rws.ctl);
            e = cudaGetLastError();
        }
    }
    if (e != cudaSuccess) {
        if (f->side)
            cudaStreamDestroy(f->side);
        if (f->ev_pos)
            cudaEventDestroy(f->ev_pos);
        if (f->ev_seq)
            cudaEventDestroy(f->ev_seq);
        cudaFree(f->mem);
        delete f;
        return cuda_status(e, "vsmc_cuda_cv_create");
    }
    *out = f;
    return VSMC_CUDA_OK;
}

int vsmc_cuda_cv_destroy(vsmc_cuda_cv_filter *f)
{
    if (f == nullptr)
        return VSMC_CUDA_OK;
    cudaStreamSynchronize(f->stream);
    if (f->side) {
        cudaStreamSynchronize(f->side);
        cudaStreamDestroy(f->side);
        cudaEventDestroy(f->ev_pos);
        cudaEventDestroy(f->ev_seq);
    }
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
    if (num > 1)
        join_sequence(f);
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

int vsmc_cuda_cv_complete_monitor(vsmc_cuda_cv_filter *f)
{
    if (f == nullptr)
        return VSMC_CUDA_EINVAL;
    return flush_monitor(f);
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
    if (f->side != nullptr) {
        // a speculative sequence still running on the side stream must not
        // overlap the non-speculative resampling of a replayed step, and the
        // held one is dropped
        join_sequence(f);
        f->seq_pending = false;
        k_spec_invalidate<<<1, 1, 0, f->stream>>>(f->rws.ctl);
        ++f->launches;
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
