// resample_static.cu -- the resampler for callers that cannot allocate.
//
// vsmc_cuda_resample needs a caller-provided device workspace.  Some callers
// cannot provide one: code that runs under a fixed device-memory budget
// reserved up front (a serving process whose HBM is carved out before it
// starts), latency-critical loops where cudaMalloc / cudaFree would
// synchronise the device, and plugins whose host application owns every
// device allocation and offers them no allocator.  For them,
// vsmc_cuda_resample_noalloc runs the same kernels on a scratch array that
// the library itself holds in device memory.
//
// The scratch is one file-scope __device__ array sized for at most
// VSMC_CUDA_NOALLOC_MAX_N particles.  Every GPU that loads the library keeps
// it (about 7.4 MiB) until the process exits.  All calls share it and it
// keeps the previous call's contents: each call rewrites the control block
// from the host and every other array is fully written before it is read,
// so nothing stale is used, but two calls that overlap on the GPU (for
// example on two streams) race on the same memory and must be serialised by
// the caller.
#include "resample.cuh"

#include <cstring>
#include <mutex>
#include <string>

namespace vsmc_b200 {

void set_last_error(const std::string &msg);
int cuda_status(cudaError_t e, const char *what);

namespace {

// The workspace carve_workspace lays out for the largest N, plus the int32
// copy_from scratch used when the caller passes no copy_from array.  Both
// come from the same constexpr size functions the workspace path uses, so a
// change of the workspace layout resizes the array with it.
constexpr long long kNoallocMaxN = VSMC_CUDA_NOALLOC_MAX_N;
constexpr size_t kNoallocCopyFromOffset = resample_workspace_bytes(kNoallocMaxN);
constexpr size_t kNoallocBytes =
    kNoallocCopyFromOffset + align256((size_t)kNoallocMaxN * 4);
// Smaller N needs no more: the layout grows with N.
static_assert(resample_workspace_bytes(1) <= kNoallocCopyFromOffset,
              "workspace layout must grow with N");

// In host code this name is only a stand-in for the symbol; its device
// address comes from cudaGetSymbolAddress on each device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
void *g_noalloc_ptr[kMaxDevices] = {};
void *g_noalloc_ctx[kMaxDevices] = {}; // the context the address belongs to

// cuCtxGetCurrent through the runtime's driver entry point (no link against
// libcuda): the current context identifies the module instance the cached
// address belongs to.  After cudaDeviceReset the device's primary context is
// a new one, the module is loaded again and the symbol may move.
typedef int (*CtxGetCurrentFn)(void **);

void *current_context()
{
    static CtxGetCurrentFn fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault,
                                    &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<CtxGetCurrentFn>(p);
    }();
    void *ctx = nullptr;
    if (fn == nullptr || fn(&ctx) != 0)
        return nullptr;
    return ctx;
}

// Device address of the scratch array on the current device, looked up
// once per device and context (with that device current) and cached.
int noalloc_scratch(void **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_resample_noalloc: cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) {
        set_last_error("vsmc_cuda_resample_noalloc: device index out of range");
        return VSMC_CUDA_EINVAL;
    }
    // (no context is current before the process's first runtime call that
    // needs one; the lookup below creates it, and the next call then finds
    // the context and looks the address up once more)
    void *ctx = current_context();
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (g_noalloc_ptr[dev] == nullptr || ctx == nullptr ||
        ctx != g_noalloc_ctx[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            return cuda_status(e,
                               "vsmc_cuda_resample_noalloc: "
                               "cudaGetSymbolAddress");
        g_noalloc_ptr[dev] = p;
        g_noalloc_ctx[dev] = ctx != nullptr ? ctx : current_context();
    }
    *out = g_noalloc_ptr[dev];
    return VSMC_CUDA_OK;
}

} // namespace

} // namespace vsmc_b200

using namespace vsmc_b200;

extern "C" int vsmc_cuda_resample_noalloc(int scheme, uint64_t N,
                                          const double *weight,
                                          const double *uniforms,
                                          uint64_t n_uniforms,
                                          vsmc_cuda_threefry_state *rng,
                                          int32_t *replication,
                                          int32_t *copy_from, void *stream)
{
    if (N > (uint64_t)kNoallocMaxN) {
        set_last_error("vsmc_cuda_resample_noalloc: N = " + std::to_string(N) +
                       " exceeds the static scratch limit of " +
                       std::to_string(kNoallocMaxN) +
                       " particles (use vsmc_cuda_resample with a workspace)");
        return VSMC_CUDA_EINVAL;
    }
    if (scheme < 0 || scheme > 5 || N == 0 || weight == nullptr ||
        rng == nullptr || (uniforms == nullptr && n_uniforms != 0) ||
        n_uniforms > N) {
        set_last_error("vsmc_cuda_resample_noalloc: invalid arguments");
        return VSMC_CUDA_EINVAL;
    }
    void *scratch = nullptr;
    int st = noalloc_scratch(&scratch);
    if (st != VSMC_CUDA_OK)
        return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    ResampleWorkspace ws = carve_workspace(scratch, (long long)N);
    int32_t *cf = copy_from;
    if (cf == nullptr)
        cf = reinterpret_cast<int32_t *>(static_cast<char *>(scratch) +
                                         kNoallocCopyFromOffset);
    // the control block starts from the host's values on every call
    ResampleCtl h;
    std::memset(&h, 0, sizeof(h));
    h.active = 1;
    h.offset = rng->offset;
    cudaError_t e =
        cudaMemcpyAsync(ws.ctl, &h, sizeof(h), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_resample_noalloc: control block");
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
        return cuda_status(e, "vsmc_cuda_resample_noalloc: launch");
    e = cudaMemcpyAsync(&h, ws.ctl, sizeof(h), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
        return cuda_status(e, "vsmc_cuda_resample_noalloc");
    if (h.error != 0) {
        set_last_error("vsmc_cuda_resample_noalloc: replication did not sum "
                       "to N");
        return h.error;
    }
    rng->offset = h.offset;
    return VSMC_CUDA_OK;
}
