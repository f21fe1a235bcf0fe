// smc_core.cu -- the model-independent part of a device Sampler: weights,
// normalisation, ESS, log-evidence, the resampling decision and the six
// resampling schemes, for moves that the caller compiles itself against
// include/vsmc_b200/smc_device.cuh (the generic Sampler<T> of
// include/vsmc_b200/smc.cuh).
//
// Reference: core/sampler.hpp:450-483 and 758-834 (initialize / iterate /
// do_resample), core/weight_set.hpp:108-125, 296-344, 441-446 (add/set log
// weight, normalisation, ESS), core/particle.hpp:230-250 (resample),
// example/include/move_smc.hpp:63-71 (log-evidence increment).
//
// A step is: the caller's move kernel(s) write raw log-weights and per-tile
// statistics (TileStats, one per kTile particles) and gather through
// copy_from when the previous step resampled; vsmc_cuda_smc_finish_step then
// runs the same finalize and resampling kernels as the built-in filter.
#include "cv_kernels.cuh"

#include <cstring>
#include <new>
#include <string>

namespace vsmc_b200 {

void set_last_error(const std::string &msg);
int cuda_status(cudaError_t e, const char *what);

} // namespace vsmc_b200

using namespace vsmc_b200;

static_assert(VSMC_CUDA_SMC_TILE == kTile, "tile size of the C ABI");

struct vsmc_cuda_smc {
    uint64_t N, T_max;
    int scheme;
    double threshold;
    cudaStream_t stream;
    char *mem;
    size_t bytes;
    double *lw;
    int32_t *copy_from;
    FilterCtl *ctl;
    TileStats *tile_stats;
    double *hist_ess, *hist_logz_inc, *hist_mean_x, *hist_mean_y;
    int32_t *hist_resampled;
    unsigned long long *accept; // T_max x VSMC_CUDA_SMC_MAX_QUEUE
    ResampleWorkspace rws;
    long long ntiles;
    uint64_t iter;
    EngineRef eng;
    uint64_t launches;
};

namespace {

size_t smc_bytes(uint64_t N, uint64_t T)
{
    const size_t nt = (N + kTile - 1) / kTile;
    size_t b = 0;
    b += align256(N * 8);                            // log-weights
    b += align256(N * 4);                            // copy_from
    b += align256(sizeof(FilterCtl));
    b += align256(nt * sizeof(TileStats));
    b += 4 * align256(T * 8) + align256(T * 4);      // histories
    b += align256(T * VSMC_CUDA_SMC_MAX_QUEUE * 8);  // accept counters
    b += resample_workspace_bytes((long long)N);
    return b;
}

// Normalised weights and max-normalised log-weights of the last step, as
// WeightSet::read_weight / read_log_weight would give them after
// Sampler::iterate: equal weights once the step resampled.
__global__ void k_smc_read_weights(const double *lw, const FilterCtl *ctl,
                                   long long N, double *w, double *lwn)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N)
        return;
    if (ctl->resampled) {
        if (w)
            w[i] = 1.0 / (double)N;
        if (lwn)
            lwn[i] = 0.0;
        return;
    }
    const double l = __dadd_rn(lw[i], -ctl->lw_max);
    if (w)
        w[i] = __dmul_rn(exp(l), __ddiv_rn(1.0, ctl->s1));
    if (lwn)
        lwn[i] = l;
}

// Sampler::initialize's reset (do_reset): equal weights, no resampling
// pending, running log-evidence 0.
__global__ void k_smc_reset(FilterCtl *ctl, ResampleCtl *rctl)
{
    ctl->lw_max = 0.0;
    ctl->s1 = 0.0;
    ctl->s2 = 0.0;
    ctl->ess = 0.0;
    ctl->logz = 0.0;
    ctl->resampled = 0;
    ctl->error = 0;
    ctl->monitor_done = -1;
    rctl->active = 0;
    rctl->error = 0;
}

} // namespace

extern "C" {

int vsmc_cuda_smc_create(uint64_t N, uint64_t T_max, int scheme,
                         double threshold, uint32_t resample_seed,
                         void *stream, vsmc_cuda_smc **out)
{
    if (out == nullptr || N < 2 || N > (1ull << 30) || T_max < 1 ||
        T_max > (1ull << 31) || scheme < 0 || scheme > 5 ||
        !(threshold >= 0.0)) {
        set_last_error("vsmc_cuda_smc_create: invalid arguments");
        return VSMC_CUDA_EINVAL;
    }
    *out = nullptr;
    vsmc_cuda_smc *s = new (std::nothrow) vsmc_cuda_smc();
    if (s == nullptr)
        return VSMC_CUDA_ENOMEM;
    s->N = N;
    s->T_max = T_max;
    s->scheme = scheme;
    s->threshold = threshold;
    s->stream = static_cast<cudaStream_t>(stream);
    s->bytes = smc_bytes(N, T_max);
    cudaError_t e = cudaMalloc(&s->mem, s->bytes);
    if (e != cudaSuccess) {
        delete s;
        cudaGetLastError();
        set_last_error("vsmc_cuda_smc_create: cudaMalloc of " +
                       std::to_string(N) + " particles failed");
        return VSMC_CUDA_ENOMEM;
    }
    const size_t nt = (N + kTile - 1) / kTile;
    char *p = s->mem;
    s->lw = reinterpret_cast<double *>(p);
    p += align256(N * 8);
    s->copy_from = reinterpret_cast<int32_t *>(p);
    p += align256(N * 4);
    s->ctl = reinterpret_cast<FilterCtl *>(p);
    p += align256(sizeof(FilterCtl));
    s->tile_stats = reinterpret_cast<TileStats *>(p);
    p += align256(nt * sizeof(TileStats));
    s->hist_ess = reinterpret_cast<double *>(p);
    p += align256(T_max * 8);
    s->hist_logz_inc = reinterpret_cast<double *>(p);
    p += align256(T_max * 8);
    s->hist_mean_x = reinterpret_cast<double *>(p);
    p += align256(T_max * 8);
    s->hist_mean_y = reinterpret_cast<double *>(p);
    p += align256(T_max * 8);
    s->hist_resampled = reinterpret_cast<int32_t *>(p);
    p += align256(T_max * 4);
    s->accept = reinterpret_cast<unsigned long long *>(p);
    p += align256(T_max * VSMC_CUDA_SMC_MAX_QUEUE * 8);
    s->rws = carve_workspace(p, (long long)N);
    s->ntiles = (long long)nt;
    s->iter = 0;
    s->launches = 0;
    for (int i = 0; i < 4; ++i) {
        s->eng.key.v[i] = 0;
        s->eng.ctr.v[i] = 0;
    }
    s->eng.key.v[0] = resample_seed;
    cudaFuncSetAttribute(k_cv_finalize,
                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                         kFinalSmemTiles * (int)sizeof(double));
    e = cudaMemsetAsync(s->mem, 0, s->bytes, s->stream);
    if (e == cudaSuccess) {
        k_smc_reset<<<1, 1, 0, s->stream>>>(s->ctl, s->rws.ctl);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        cudaFree(s->mem);
        delete s;
        return cuda_status(e, "vsmc_cuda_smc_create");
    }
    *out = s;
    return VSMC_CUDA_OK;
}

int vsmc_cuda_smc_destroy(vsmc_cuda_smc *s)
{
    if (s == nullptr)
        return VSMC_CUDA_OK;
    cudaStreamSynchronize(s->stream);
    cudaFree(s->mem);
    delete s;
    return VSMC_CUDA_OK;
}

int vsmc_cuda_smc_reset(vsmc_cuda_smc *s)
{
    if (s == nullptr)
        return VSMC_CUDA_EINVAL;
    s->iter = 0;
    k_smc_reset<<<1, 1, 0, s->stream>>>(s->ctl, s->rws.ctl);
    cudaError_t e = cudaMemsetAsync(
        s->accept, 0, s->T_max * VSMC_CUDA_SMC_MAX_QUEUE * 8, s->stream);
    if (e == cudaSuccess)
        e = cudaGetLastError();
    ++s->launches;
    return e == cudaSuccess ? VSMC_CUDA_OK
                            : cuda_status(e, "vsmc_cuda_smc_reset");
}

int vsmc_cuda_smc_step_args(vsmc_cuda_smc *s, vsmc_cuda_smc_step *out)
{
    if (s == nullptr || out == nullptr)
        return VSMC_CUDA_EINVAL;
    out->N = s->N;
    out->ntiles = (uint64_t)s->ntiles;
    out->iter = s->iter;
    out->log_weight = s->lw;
    out->lw_max = &s->ctl->lw_max;
    out->weight_s1 = &s->ctl->s1;
    out->resampled = &s->ctl->resampled;
    out->copy_from = s->copy_from;
    out->tile_stats = s->tile_stats;
    out->accept = reinterpret_cast<uint64_t *>(s->accept);
    out->stream = s->stream;
    return VSMC_CUDA_OK;
}

int vsmc_cuda_smc_finish_step(vsmc_cuda_smc *s)
{
    if (s == nullptr)
        return VSMC_CUDA_EINVAL;
    if (s->iter >= s->T_max) {
        set_last_error("vsmc_cuda_smc_finish_step: more steps than T_max");
        return VSMC_CUDA_EINVAL;
    }
    const long long N = (long long)s->N;
    const int sch = s->scheme;
    FinalizeArgs fa;
    std::memset(&fa, 0, sizeof(fa));
    fa.ctl = s->ctl;
    fa.ts = s->tile_stats;
    fa.ntiles = (int)s->ntiles;
    fa.N = N;
    fa.threshold = s->threshold;
    fa.t = (long long)s->iter;
    fa.init = s->iter == 0 ? 1 : 0;
    fa.anchored = 0;
    fa.obs_x = nullptr;
    fa.obs_y = nullptr;
    fa.hist_ess = s->hist_ess;
    fa.hist_resampled = s->hist_resampled;
    fa.hist_logz_inc = s->hist_logz_inc;
    fa.hist_mean_x = s->hist_mean_x; // the built-in filter's monitor; unused
    fa.hist_mean_y = s->hist_mean_y;
    fa.rctl = s->rws.ctl;
    fa.tile_excl = s->rws.tile_excl;
    fa.residual = sch == VSMC_CUDA_RESIDUAL ||
                  sch == VSMC_CUDA_RESIDUAL_STRATIFIED ||
                  sch == VSMC_CUDA_RESIDUAL_SYSTEMATIC;
    fa.sys = sch == VSMC_CUDA_SYSTEMATIC ||
             sch == VSMC_CUDA_RESIDUAL_SYSTEMATIC;
    fa.eng = s->eng;
    fa.replay_flags = nullptr;
    fa.compare = 0;
    const size_t fin_smem = s->ntiles <= kFinalSmemTiles
                                ? (size_t)s->ntiles * sizeof(double)
                                : 0;
    k_cv_finalize<<<1, kFinalThreads, fin_smem, s->stream>>>(fa);
    WeightsFromLog<double> w;
    w.lw = s->lw;
    w.stats = &s->ctl->lw_max;
    launch_resample_core(sch, w, N, s->eng, s->rws, nullptr, 0,
                         /*spine_done=*/true, nullptr, s->copy_from,
                         s->stream);
    s->launches += 1 + resample_launches(sch, false, true);
    ++s->iter;
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? VSMC_CUDA_OK
                            : cuda_status(e, "vsmc_cuda_smc_finish_step");
}

int vsmc_cuda_smc_synchronize(vsmc_cuda_smc *s)
{
    if (s == nullptr)
        return VSMC_CUDA_EINVAL;
    cudaError_t e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_smc_synchronize");
    FilterCtl h;
    ResampleCtl r;
    e = cudaMemcpy(&h, s->ctl, sizeof(h), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess)
        e = cudaMemcpy(&r, s->rws.ctl, sizeof(r), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_smc_synchronize");
    if (h.error != 0) {
        set_last_error("degenerate weights: every log-weight is -inf or a "
                       "log-weight is NaN or +inf");
        return h.error;
    }
    if (r.error != 0) {
        set_last_error("resampling: replication did not sum to N");
        return r.error;
    }
    return VSMC_CUDA_OK;
}

int vsmc_cuda_smc_iter_size(vsmc_cuda_smc *s, uint64_t *n)
{
    if (s == nullptr || n == nullptr)
        return VSMC_CUDA_EINVAL;
    *n = s->iter;
    return VSMC_CUDA_OK;
}

int vsmc_cuda_smc_history(vsmc_cuda_smc *s, double *ess, int32_t *resampled,
                          double *logz_inc, uint64_t *accept)
{
    int st = vsmc_cuda_smc_synchronize(s);
    if (st != VSMC_CUDA_OK)
        return st;
    const size_t T = s->iter;
    cudaError_t e = cudaSuccess;
    if (ess && T)
        e = cudaMemcpy(ess, s->hist_ess, T * 8, cudaMemcpyDeviceToHost);
    if (resampled && T && e == cudaSuccess)
        e = cudaMemcpy(resampled, s->hist_resampled, T * 4,
                       cudaMemcpyDeviceToHost);
    if (logz_inc && T && e == cudaSuccess)
        e = cudaMemcpy(logz_inc, s->hist_logz_inc, T * 8,
                       cudaMemcpyDeviceToHost);
    if (accept && T && e == cudaSuccess)
        e = cudaMemcpy(accept, s->accept, T * VSMC_CUDA_SMC_MAX_QUEUE * 8,
                       cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? VSMC_CUDA_OK
                            : cuda_status(e, "vsmc_cuda_smc_history");
}

int vsmc_cuda_smc_log_evidence(vsmc_cuda_smc *s, double *logz)
{
    if (logz == nullptr)
        return VSMC_CUDA_EINVAL;
    int st = vsmc_cuda_smc_synchronize(s);
    if (st != VSMC_CUDA_OK)
        return st;
    FilterCtl h;
    cudaError_t e = cudaMemcpy(&h, s->ctl, sizeof(h), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_smc_log_evidence");
    *logz = h.logz;
    return VSMC_CUDA_OK;
}

int vsmc_cuda_smc_read_weights(vsmc_cuda_smc *s, double *weight,
                               double *log_weight)
{
    if (s == nullptr)
        return VSMC_CUDA_EINVAL;
    const long long N = (long long)s->N;
    // device scratch: the resample workspace's U01 array holds N doubles and
    // is rewritten before the next resampling reads it
    double *wd = s->rws.u;
    const unsigned grid = (unsigned)((N + 255) / 256);
    cudaError_t e = cudaSuccess;
    if (weight != nullptr) {
        k_smc_read_weights<<<grid, 256, 0, s->stream>>>(s->lw, s->ctl, N, wd,
                                                         nullptr);
        e = cudaMemcpyAsync(weight, wd, (size_t)N * 8, cudaMemcpyDeviceToHost,
                            s->stream);
    }
    if (log_weight != nullptr && e == cudaSuccess) {
        k_smc_read_weights<<<grid, 256, 0, s->stream>>>(s->lw, s->ctl, N,
                                                         nullptr, wd);
        e = cudaMemcpyAsync(log_weight, wd, (size_t)N * 8,
                            cudaMemcpyDeviceToHost, s->stream);
    }
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s->stream);
    return e == cudaSuccess ? VSMC_CUDA_OK
                            : cuda_status(e, "vsmc_cuda_smc_read_weights");
}

int vsmc_cuda_smc_resample_words(vsmc_cuda_smc *s, uint64_t *words)
{
    if (words == nullptr)
        return VSMC_CUDA_EINVAL;
    int st = vsmc_cuda_smc_synchronize(s);
    if (st != VSMC_CUDA_OK)
        return st;
    ResampleCtl r;
    cudaError_t e = cudaMemcpy(&r, s->rws.ctl, sizeof(r),
                               cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_smc_resample_words");
    *words = r.offset;
    return VSMC_CUDA_OK;
}

int vsmc_cuda_smc_launches(vsmc_cuda_smc *s, uint64_t *launches)
{
    if (s == nullptr || launches == nullptr)
        return VSMC_CUDA_EINVAL;
    *launches = s->launches;
    return VSMC_CUDA_OK;
}

} // extern "C"
