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
// it (about 4.1 MiB) until the process exits.  All calls share it and it
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

// resample_workspace_bytes(N) plus the int32 copy_from scratch used when the
// caller passes no copy_from array.
constexpr long long kNoallocMaxN = VSMC_CUDA_NOALLOC_MAX_N;
constexpr size_t kNoallocNt = (size_t)((kNoallocMaxN + kTile - 1) / kTile) + 1;
constexpr size_t kAlign = 256;
constexpr size_t al(size_t b) { return (b + kAlign - 1) / kAlign * kAlign; }
constexpr size_t kNoallocBytes =
    al(sizeof(ResampleCtl)) + 6 * al(kNoallocNt * 8) + 5 * al(kNoallocNt * 4) +
    al(((size_t)kNoallocMaxN / 8 + 2) * 4) + al((size_t)kNoallocMaxN * 8) +
    al((size_t)kNoallocMaxN * 4) + al((size_t)kNoallocMaxN * 4);

// In host code this name is only a stand-in for the symbol; its device
// address comes from cudaGetSymbolAddress on each device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
void *g_noalloc_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device, looked up
// once per device (with that device current) and cached.
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
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (g_noalloc_ptr[dev] == nullptr) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            return cuda_status(e,
                               "vsmc_cuda_resample_noalloc: "
                               "cudaGetSymbolAddress");
        g_noalloc_ptr[dev] = p;
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
                                         resample_workspace_bytes((long long)N));
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
