// capi.cu -- status handling and the generic C entry points of libvsmc_cuda:
// RNG word streams, the device WeightSet update, the device resampler and
// the particle gather.  The CV filter's entry points are in cv_filter.cu.
#include "resample.cuh"

#include <cstdio>
#include <cstring>
#include <string>

namespace vsmc_b200 {

static thread_local std::string g_last_error;

void set_last_error(const std::string &msg) { g_last_error = msg; }

int cuda_status(cudaError_t e, const char *what)
{
    g_last_error = std::string(what) + ": " + cudaGetErrorName(e) + " (" +
                   cudaGetErrorString(e) + ")";
    return e == cudaErrorMemoryAllocation ? VSMC_CUDA_ENOMEM : VSMC_CUDA_ECUDA;
}

// ------------------------------------------------------------ RNG words --
__device__ __forceinline__ uint4 ctr32_add(uint4 c, unsigned long long v)
{
    unsigned long long s = (unsigned long long)c.x + (v & 0xffffffffull);
    c.x = (uint32_t)s;
    unsigned long long carry = (s >> 32) + (v >> 32);
    s = (unsigned long long)c.y + (carry & 0xffffffffull);
    c.y = (uint32_t)s;
    carry = (s >> 32) + (carry >> 32);
    s = (unsigned long long)c.z + carry;
    c.z = (uint32_t)s;
    carry = s >> 32;
    c.w += (uint32_t)carry;
    return c;
}

// Thread b computes block b of the stream (word positions 4b..4b+3 relative
// to skip rounded down) and stores the words that fall in [skip, skip+n).
__global__ void k_philox_words(uint32_t k0, uint32_t k1, uint4 c0,
                               unsigned long long skip,
                               unsigned long long n, uint32_t *out)
{
    const unsigned long long b0 = skip / 4;
    const unsigned long long b =
        b0 + (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned long long wend = skip + n;
    if (b * 4 >= wend)
        return;
    const uint4 r = philox4x32_10(ctr32_add(c0, b + 1), k0, k1);
    const uint32_t w[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
    for (int l = 0; l < 4; ++l) {
        const unsigned long long pos = b * 4 + l;
        if (pos >= skip && pos < wend)
            out[pos - skip] = w[l];
    }
}

__global__ void k_threefry_words(u64x4 key, u64x4 c0, unsigned long long skip,
                                 unsigned long long n, uint64_t *out)
{
    const unsigned long long b0 = skip / 4;
    const unsigned long long b =
        b0 + (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned long long wend = skip + n;
    if (b * 4 >= wend)
        return;
    const u64x4 r = threefry4x64_20(ctr64_add(c0, b + 1), key);
#pragma unroll
    for (int l = 0; l < 4; ++l) {
        const unsigned long long pos = b * 4 + l;
        if (pos >= skip && pos < wend)
            out[pos - skip] = r.v[l];
    }
}

// ------------------------------------------------------------- weights --
struct WeightCtl {
    double M, S1, S2;
    int error;
};

__global__ void __launch_bounds__(kThreads)
k_wadd_tiles(long long N, double *lw, const double *inc, LseAcc *tiles)
{
    __shared__ LseAcc sh[kThreads / 32];
    const long long base = (long long)blockIdx.x * kTile;
    LseAcc acc;
    acc.init();
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const long long i = base + (long long)j * kThreads + threadIdx.x;
        if (i < N) {
            double l = lw[i];
            if (inc != nullptr) {
                l = __dadd_rn(l, inc[i]);
                lw[i] = l;
            }
            acc.add(l, 0.0, 0.0);
        }
    }
    const LseAcc r = block_reduce_lse(acc, sh);
    if (threadIdx.x == 0)
        tiles[blockIdx.x] = r;
}

__global__ void __launch_bounds__(kSpineThreads)
k_wadd_reduce(const LseAcc *tiles, int ntiles, WeightCtl *ctl)
{
    __shared__ LseAcc sh[kSpineThreads / 32];
    const int per = (ntiles + blockDim.x - 1) / blockDim.x;
    const int b = threadIdx.x * per, e = min(b + per, ntiles);
    LseAcc acc;
    acc.init();
    for (int t = b; t < e; ++t) {
        if (tiles[t].s1 != tiles[t].s1)
            acc.s1 = tiles[t].s1;
        else
            acc.merge(tiles[t]);
    }
    const LseAcc r = block_reduce_lse(acc, sh);
    if (threadIdx.x == 0) {
        ctl->M = r.m;
        ctl->S1 = r.s1;
        ctl->S2 = r.s2;
        ctl->error = (r.m > -INFINITY && r.m < INFINITY && r.s1 > 0.0 &&
                      r.s1 < INFINITY)
                         ? 0
                         : (int)VSMC_CUDA_EDEGENERATE;
    }
}

// Sums of prospective weights b_i for WeightSet::ess(first, use_log) and
// cess(first, use_log) (core/weight_set.hpp:132-186, compute_ess :385-409,
// compute_cess :411-431):
//   kind 0 (ESS, use_log):  b = exp(lw + inc - max), online log-sum-exp;
//   kind 1 (ESS, linear):   b = w * inc;           s1 = sum |b|, s2 = sum b^2;
//   kind 2 (CESS, use_log): s1 = sum w e^inc,      s2 = sum w e^inc e^inc;
//   kind 3 (CESS, linear):  s1 = sum w inc,        s2 = sum w inc inc.
// ESS = s1^2 / s2 (the reference's 1 / sum (b / asum b)^2), CESS = s1^2 / s2
// (above^2 / below).
__global__ void __launch_bounds__(kThreads)
k_prospective_tiles(long long N, const double *lw, const double *w,
                    const double *inc, int kind, LseAcc *tiles)
{
    __shared__ LseAcc sh[kThreads / 32];
    const long long base = (long long)blockIdx.x * kTile;
    LseAcc acc;
    acc.init();
    if (kind != 0)
        acc.m = 0.0; // plain sums: every partial has the same reference 0
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const long long i = base + (long long)j * kThreads + threadIdx.x;
        if (i >= N)
            continue;
        if (kind == 0) {
            acc.add(__dadd_rn(lw[i], inc[i]), 0.0, 0.0);
        } else if (kind == 1) {
            // the reference normalises by asum, a sum of |b|
            const double b = __dmul_rn(w[i], inc[i]);
            acc.s1 = __dadd_rn(acc.s1, fabs(b));
            acc.s2 = __dadd_rn(acc.s2, __dmul_rn(b, b));
        } else {
            const double b = kind == 2 ? exp(inc[i]) : inc[i];
            const double wb = __dmul_rn(w[i], b);
            acc.s1 = __dadd_rn(acc.s1, wb);
            acc.s2 = __dadd_rn(acc.s2, __dmul_rn(wb, b));
        }
    }
    const LseAcc r = block_reduce_lse(acc, sh);
    if (threadIdx.x == 0)
        tiles[blockIdx.x] = r;
}

// lw += -max (normalize_log_weight); w = exp(lw) * (1 / sum).
__global__ void k_wadd_apply(long long N, double *lw, double *w,
                             const WeightCtl *ctl)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N)
        return;
    const double l = __dadd_rn(lw[i], -ctl->M);
    lw[i] = l;
    if (w != nullptr)
        w[i] = __dmul_rn(exp(l), __ddiv_rn(1.0, ctl->S1));
}

__global__ void k_copy_f64(long long N, unsigned dim, const double *src,
                           double *dst, const int32_t *copy_from)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N)
        return;
    const long long c = copy_from[i];
    for (unsigned d = 0; d < dim; ++d)
        dst[(long long)d * N + i] = src[(long long)d * N + c];
}

static __global__ void k_math_eval(int fn, long long n, const double *in,
                                   double *out)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = fn == 0 ? fm::fm_log(in[i]) : fm::fm_exp(in[i]);
}

} // namespace vsmc_b200

using namespace vsmc_b200;

namespace {

size_t generic_resample_bytes(long long N)
{
    return resample_workspace_bytes(N) + align256((size_t)N * 4);
}

} // namespace

extern "C" {

const char *vsmc_cuda_status_string(int s)
{
    switch (s) {
    case VSMC_CUDA_OK:
        return "VSMC_CUDA_OK";
    case VSMC_CUDA_EINVAL:
        return "VSMC_CUDA_EINVAL";
    case VSMC_CUDA_ENOMEM:
        return "VSMC_CUDA_ENOMEM";
    case VSMC_CUDA_EDEGENERATE:
        return "VSMC_CUDA_EDEGENERATE";
    case VSMC_CUDA_ETIMEOUT:
        return "VSMC_CUDA_ETIMEOUT";
    case VSMC_CUDA_ECUDA:
        return "VSMC_CUDA_ECUDA";
    default:
        return "unknown status";
    }
}

const char *vsmc_cuda_last_error(void) { return g_last_error.c_str(); }

int vsmc_cuda_abi_version(void) { return VSMC_CUDA_ABI_VERSION; }

int vsmc_cuda_philox4x32_words(const uint32_t key[2], const uint32_t ctr[4],
                               uint64_t skip, uint64_t n, uint32_t *out,
                               void *stream)
{
    if (key == nullptr || ctr == nullptr || (out == nullptr && n > 0)) {
        set_last_error("vsmc_cuda_philox4x32_words: null pointer");
        return VSMC_CUDA_EINVAL;
    }
    if (n == 0)
        return VSMC_CUDA_OK;
    const unsigned long long blocks = (skip + n + 3) / 4 - skip / 4;
    const unsigned g = (unsigned)((blocks + 255) / 256);
    k_philox_words<<<g, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        key[0], key[1], make_uint4(ctr[0], ctr[1], ctr[2], ctr[3]), skip, n,
        out);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? VSMC_CUDA_OK
                            : cuda_status(e, "vsmc_cuda_philox4x32_words");
}

int vsmc_cuda_threefry4x64_words(const uint64_t key[4], const uint64_t ctr[4],
                                 uint64_t skip, uint64_t n, uint64_t *out,
                                 void *stream)
{
    if (key == nullptr || ctr == nullptr || (out == nullptr && n > 0)) {
        set_last_error("vsmc_cuda_threefry4x64_words: null pointer");
        return VSMC_CUDA_EINVAL;
    }
    if (n == 0)
        return VSMC_CUDA_OK;
    u64x4 k, c;
    for (int i = 0; i < 4; ++i) {
        k.v[i] = key[i];
        c.v[i] = ctr[i];
    }
    const unsigned long long blocks = (skip + n + 3) / 4 - skip / 4;
    const unsigned g = (unsigned)((blocks + 255) / 256);
    k_threefry_words<<<g, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        k, c, skip, n, out);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? VSMC_CUDA_OK
                            : cuda_status(e, "vsmc_cuda_threefry4x64_words");
}

int vsmc_cuda_weight_add_log(uint64_t N, double *lw, double *w,
                             const double *inc, double *ess, void *stream)
{
    if (N == 0 || lw == nullptr || ess == nullptr) {
        set_last_error("vsmc_cuda_weight_add_log: invalid arguments");
        return VSMC_CUDA_EINVAL;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int nt = (int)((N + kTile - 1) / kTile);
    void *scratch = nullptr;
    cudaError_t e = cudaMallocAsync(
        &scratch, align256(sizeof(WeightCtl)) + sizeof(LseAcc) * nt, s);
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_weight_add_log: scratch");
    WeightCtl *ctl = static_cast<WeightCtl *>(scratch);
    LseAcc *tiles = reinterpret_cast<LseAcc *>(
        static_cast<char *>(scratch) + align256(sizeof(WeightCtl)));
    k_wadd_tiles<<<nt, kThreads, 0, s>>>((long long)N, lw, inc, tiles);
    k_wadd_reduce<<<1, kSpineThreads, 0, s>>>(tiles, nt, ctl);
    k_wadd_apply<<<(unsigned)((N + 255) / 256), 256, 0, s>>>((long long)N, lw,
                                                             w, ctl);
    WeightCtl h;
    e = cudaMemcpyAsync(&h, ctl, sizeof(h), cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(scratch, s);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_weight_add_log");
    if (h.error) {
        set_last_error("vsmc_cuda_weight_add_log: degenerate log-weights");
        *ess = NAN;
        return h.error;
    }
    *ess = h.S1 * h.S1 / h.S2;
    return VSMC_CUDA_OK;
}

namespace {

int prospective(uint64_t N, const double *lw, const double *w,
                const double *inc, int kind, double *out, void *stream,
                const char *where)
{
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int nt = (int)((N + kTile - 1) / kTile);
    void *scratch = nullptr;
    cudaError_t e = cudaMallocAsync(
        &scratch, align256(sizeof(WeightCtl)) + sizeof(LseAcc) * nt, s);
    if (e != cudaSuccess)
        return cuda_status(e, where);
    WeightCtl *ctl = static_cast<WeightCtl *>(scratch);
    LseAcc *tiles = reinterpret_cast<LseAcc *>(
        static_cast<char *>(scratch) + align256(sizeof(WeightCtl)));
    k_prospective_tiles<<<nt, kThreads, 0, s>>>((long long)N, lw, w, inc,
                                                kind, tiles);
    k_wadd_reduce<<<1, kSpineThreads, 0, s>>>(tiles, nt, ctl);
    WeightCtl h;
    e = cudaMemcpyAsync(&h, ctl, sizeof(h), cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(scratch, s);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
        return cuda_status(e, where);
    *out = h.S1 * h.S1 / h.S2;
    // the log form needs a finite maximum and a positive sum; the plain
    // forms only finite sums (increments may be negative) and S2 > 0
    const bool bad = kind == 0 ? h.error != 0
                               : !(h.S1 == h.S1 && h.S1 > -INFINITY &&
                                   h.S1 < INFINITY && h.S2 < INFINITY);
    if (bad || !(h.S2 > 0.0)) {
        set_last_error(std::string(where) + ": degenerate weights");
        *out = NAN;
        return VSMC_CUDA_EDEGENERATE;
    }
    return VSMC_CUDA_OK;
}

} // namespace

int vsmc_cuda_weight_ess(uint64_t N, const double *log_weight,
                         const double *weight, const double *inc, int use_log,
                         double *ess, void *stream)
{
    if (N == 0 || inc == nullptr || ess == nullptr ||
        (use_log ? log_weight == nullptr : weight == nullptr)) {
        set_last_error("vsmc_cuda_weight_ess: invalid arguments");
        return VSMC_CUDA_EINVAL;
    }
    return prospective(N, log_weight, weight, inc, use_log ? 0 : 1, ess,
                       stream, "vsmc_cuda_weight_ess");
}

int vsmc_cuda_weight_cess(uint64_t N, const double *weight, const double *inc,
                          int use_log, double *cess, void *stream)
{
    if (N == 0 || weight == nullptr || inc == nullptr || cess == nullptr) {
        set_last_error("vsmc_cuda_weight_cess: invalid arguments");
        return VSMC_CUDA_EINVAL;
    }
    return prospective(N, nullptr, weight, inc, use_log ? 2 : 3, cess, stream,
                       "vsmc_cuda_weight_cess");
}

size_t vsmc_cuda_resample_workspace_size(uint64_t N)
{
    if (N == 0 || N > (1ull << 30))
        return 0;
    return generic_resample_bytes((long long)N);
}

int vsmc_cuda_resample(int scheme, uint64_t N, const double *weight,
                       const double *uniforms, uint64_t n_uniforms,
                       vsmc_cuda_threefry_state *rng, int32_t *replication,
                       int32_t *copy_from, void *workspace,
                       size_t workspace_bytes, void *stream)
{
    if (scheme < 0 || scheme > 5 || N == 0 || N > (1ull << 30) ||
        weight == nullptr || rng == nullptr || workspace == nullptr ||
        workspace_bytes < generic_resample_bytes((long long)N) ||
        (uniforms == nullptr && n_uniforms != 0) || n_uniforms > N ||
        (reinterpret_cast<uintptr_t>(workspace) & 255) != 0) {
        set_last_error("vsmc_cuda_resample: invalid arguments (scheme, N, "
                       "null pointer, or workspace too small / not "
                       "256-byte aligned)");
        return VSMC_CUDA_EINVAL;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    ResampleWorkspace ws = carve_workspace(workspace, (long long)N);
    int32_t *cf = copy_from;
    if (cf == nullptr)
        cf = reinterpret_cast<int32_t *>(static_cast<char *>(workspace) +
                                         resample_workspace_bytes((long long)N));
    ResampleCtl h;
    std::memset(&h, 0, sizeof(h));
    h.active = 1;
    h.offset = rng->offset;
    cudaError_t e =
        cudaMemcpyAsync(ws.ctl, &h, sizeof(h), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_resample: control block");
    EngineRef eng;
    for (int i = 0; i < 4; ++i) {
        eng.key.v[i] = rng->key[i];
        eng.ctr.v[i] = rng->ctr[i];
    }
    WeightsGiven w;
    w.w = weight;
    launch_resample_core(scheme, w, (long long)N, eng, ws, uniforms,
                         (long long)n_uniforms, false, replication, cf, s);
    e = cudaGetLastError();
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_resample: launch");
    e = cudaMemcpyAsync(&h, ws.ctl, sizeof(h), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_resample");
    if (h.error != 0) {
        set_last_error("vsmc_cuda_resample: look-back wait gave up");
        return h.error;
    }
    rng->offset = h.offset;
    return VSMC_CUDA_OK;
}

size_t vsmc_cuda_resample_mn_workspace_size(uint64_t M, uint64_t N)
{
    if (M == 0 || M > (1ull << 30) || N > (1ull << 30))
        return 0;
    const long long Nmax = (long long)(M > N ? M : N);
    return resample_workspace_bytes(Nmax) + 2 * align256((size_t)Nmax * 4);
}

int vsmc_cuda_resample_mn(int scheme, uint64_t M, uint64_t N,
                          const double *weight, const double *uniforms,
                          uint64_t n_uniforms, vsmc_cuda_threefry_state *rng,
                          int32_t *replication, int32_t *copy_from,
                          void *workspace, size_t workspace_bytes,
                          void *stream)
{
    const size_t need = vsmc_cuda_resample_mn_workspace_size(M, N);
    if (scheme < 0 || scheme > 5 || need == 0 || weight == nullptr ||
        rng == nullptr || workspace == nullptr || workspace_bytes < need ||
        (uniforms == nullptr && n_uniforms != 0) || n_uniforms > N ||
        (reinterpret_cast<uintptr_t>(workspace) & 255) != 0) {
        set_last_error("vsmc_cuda_resample_mn: invalid arguments (scheme, "
                       "M >= 1, N, null pointer, or workspace too small / "
                       "not 256-byte aligned)");
        return VSMC_CUDA_EINVAL;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const bool sys = scheme == VSMC_CUDA_SYSTEMATIC ||
                     scheme == VSMC_CUDA_RESIDUAL_SYSTEMATIC;
    const long long Nmax = (long long)(M > N ? M : N);
    char *wsp = static_cast<char *>(workspace);
    int32_t *cf_scratch =
        reinterpret_cast<int32_t *>(wsp + resample_workspace_bytes(Nmax));
    int32_t *rep = replication != nullptr
                       ? replication
                       : cf_scratch + align256((size_t)Nmax * 4) / 4;
    cudaError_t e = cudaSuccess;
    if (N == 0) {
        // inversion(M, 0, ...) leaves every count at zero; only the
        // systematic sequence draws its one word, in its constructor
        // (rng/u01.hpp:253-263)
        e = cudaMemsetAsync(rep, 0, M * 4, s);
        if (e == cudaSuccess)
            e = cudaStreamSynchronize(s);
        if (e != cudaSuccess)
            return cuda_status(e, "vsmc_cuda_resample_mn");
        rng->offset += sys ? 1 : 0;
        return VSMC_CUDA_OK;
    }
    if (M == N)
        return vsmc_cuda_resample(scheme, N, weight, uniforms, n_uniforms,
                                  rng, replication, copy_from, workspace,
                                  workspace_bytes, stream);
    ResampleWorkspace ws = carve_workspace(workspace, Nmax);
    ResampleCtl h;
    std::memset(&h, 0, sizeof(h));
    h.active = 1;
    h.offset = rng->offset;
    h.Nout = (long long)N;
    e = cudaMemcpyAsync(ws.ctl, &h, sizeof(h), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_resample_mn: control block");
    EngineRef eng;
    for (int i = 0; i < 4; ++i) {
        eng.key.v[i] = rng->key[i];
        eng.ctr.v[i] = rng->ctr[i];
    }
    WeightsGiven w;
    w.w = weight;
    launch_resample_core(scheme, w, (long long)M, eng, ws, uniforms,
                         (long long)n_uniforms, false, rep, cf_scratch, s,
                         false, /*cfrp=*/false, (long long)N);
    if (copy_from != nullptr)
        launch_expand(rep, (long long)M, (long long)N, ws, copy_from, s);
    e = cudaGetLastError();
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_resample_mn: launch");
    e = cudaMemcpyAsync(&h, ws.ctl, sizeof(h), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_resample_mn");
    if (h.error != 0) {
        set_last_error("vsmc_cuda_resample_mn: replication did not sum to N");
        return h.error;
    }
    rng->offset = h.offset;
    return VSMC_CUDA_OK;
}

int vsmc_cuda_copy_f64(uint64_t N, uint32_t dim, const double *src,
                       double *dst, const int32_t *copy_from, void *stream)
{
    if (N == 0 || src == nullptr || dst == nullptr || copy_from == nullptr ||
        src == dst) {
        set_last_error("vsmc_cuda_copy_f64: invalid arguments");
        return VSMC_CUDA_EINVAL;
    }
    k_copy_f64<<<(unsigned)((N + 255) / 256), 256, 0,
                 static_cast<cudaStream_t>(stream)>>>((long long)N, dim, src,
                                                      dst, copy_from);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? VSMC_CUDA_OK
                            : cuda_status(e, "vsmc_cuda_copy_f64");
}

int vsmc_cuda_math_eval(int fn, uint64_t n, const double *in, double *out,
                        void *stream)
{
    if ((fn != 0 && fn != 1) || n == 0 || in == nullptr || out == nullptr) {
        set_last_error("vsmc_cuda_math_eval: invalid arguments");
        return VSMC_CUDA_EINVAL;
    }
    const long long blocks = ((long long)n + 255) / 256;
    k_math_eval<<<(unsigned)(blocks < 4736 ? blocks : 4736), 256, 0,
                  static_cast<cudaStream_t>(stream)>>>(fn, (long long)n, in,
                                                       out);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? VSMC_CUDA_OK
                            : cuda_status(e, "vsmc_cuda_math_eval");
}

int vsmc_cuda_device_alloc(size_t bytes, void **ptr)
{
    if (ptr == nullptr) {
        set_last_error("vsmc_cuda_device_alloc: null pointer");
        return VSMC_CUDA_EINVAL;
    }
    *ptr = nullptr;
    if (bytes == 0)
        return VSMC_CUDA_OK;
    cudaError_t e = cudaMalloc(ptr, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *ptr = nullptr;
        set_last_error("vsmc_cuda_device_alloc: cudaMalloc of " +
                       std::to_string(bytes) + " bytes failed");
        return VSMC_CUDA_ENOMEM;
    }
    return VSMC_CUDA_OK;
}

int vsmc_cuda_device_free(void *ptr)
{
    if (ptr == nullptr)
        return VSMC_CUDA_OK;
    cudaError_t e = cudaFree(ptr);
    return e == cudaSuccess ? VSMC_CUDA_OK
                            : cuda_status(e, "vsmc_cuda_device_free");
}

int vsmc_cuda_memcpy(void *dst, const void *src, size_t bytes, int kind,
                     void *stream)
{
    cudaMemcpyKind k;
    switch (kind) {
    case VSMC_CUDA_HOST_TO_DEVICE:
        k = cudaMemcpyHostToDevice;
        break;
    case VSMC_CUDA_DEVICE_TO_HOST:
        k = cudaMemcpyDeviceToHost;
        break;
    case VSMC_CUDA_DEVICE_TO_DEVICE:
        k = cudaMemcpyDeviceToDevice;
        break;
    default:
        set_last_error("vsmc_cuda_memcpy: unknown direction");
        return VSMC_CUDA_EINVAL;
    }
    if (bytes == 0)
        return VSMC_CUDA_OK;
    if (dst == nullptr || src == nullptr) {
        set_last_error("vsmc_cuda_memcpy: null pointer");
        return VSMC_CUDA_EINVAL;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, k, s);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? VSMC_CUDA_OK : cuda_status(e, "vsmc_cuda_memcpy");
}

int vsmc_cuda_stream_synchronize(void *stream)
{
    cudaError_t e = cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? VSMC_CUDA_OK
                            : cuda_status(e, "vsmc_cuda_stream_synchronize");
}

} // extern "C"
