// tcv_static.cu -- gridding for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc: an ingest or imaging pipeline that keeps latency-critical
// work running on other streams cannot afford the device-wide synchronisation that cudaMalloc and
// cudaFree imply, and a host framework that owns all device memory through its own pool or
// arena forbids allocations behind its back.  tcv_grid_raw_static serves them: it is
// tcv_grid_raw (binning plan + gridding) with the plan's scratch taken from a fixed array in this
// library's device image instead of a caller workspace.
//
// The array is a file-scope __device__ variable of kStaticScratchBytes (64 MiB).  Every GPU that
// loads the library holds it until the process exits.  Its device address is looked up with
// cudaGetSymbolAddress on the first call made in a CUDA context of the device (the first call on
// the device, and the first call after a cudaDeviceReset made a new context); the host name of
// the array is only a stand-in and is never passed to a kernel.  That first call also loads the
// library's device code on the device, so make it at set-up, before any stream capture.
//
// The entry never compiles or loads a footprint-specialised kernel (tcv_jit.cu): it launches the
// specialised copy only when tcv_jit_prepare (or an earlier plan) built it, and the generic copy
// compiled into this library otherwise.  Both give the same sums.
//
// Every call shares the array and it keeps the previous call's contents: the plan clears
// everything that must start at zero, but calls that overlap on the GPU (different streams, or
// threads calling concurrently) race on the array and must be serialised by the caller.
#include "tcv_internal.cuh"

#include <cuda.h>

#include <mutex>

namespace {

constexpr size_t kStaticScratchBytes = size_t(64) << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

// driver entry points for the identity of the current context (no link against libcuda)
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

std::mutex g_mu;
bool g_entry_tried = false;
CtxGetCurrentFn g_ctx_current = nullptr;
CtxGetIdFn g_ctx_id = nullptr;
struct Cached {
    unsigned long long ctx_id;  // context the address belongs to (0: not looked up)
    void* addr;
};
Cached g_cached[kMaxDevices] = {};

void load_entry_points()
{
    if (g_entry_tried) return;
    g_entry_tried = true;
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
        g_ctx_current = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
        g_ctx_id = reinterpret_cast<CtxGetIdFn>(f);
    cudaGetLastError();
}

// identity of the calling thread's current context (0 if it cannot be told)
unsigned long long current_ctx_id()
{
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (!g_ctx_current || !g_ctx_id || g_ctx_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
    if (g_ctx_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Device address of the array in the current context of the current device.  Looked up once per
// context; without a context identity (an old driver) it is looked up on every call.
tcv_status scratch_address(void** out)
{
    int dev = 0;
    TCV_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return TCV_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_mu);
    load_entry_points();
    unsigned long long id = current_ctx_id();
    if (id != 0 && g_cached[dev].ctx_id == id && g_cached[dev].addr) {
        *out = g_cached[dev].addr;
        return TCV_OK;
    }
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);  // makes the primary context current
    if (e != cudaSuccess) return tcv::cuda_status(e);
    if (!p) return TCV_ERR_CUDA;
    if (id == 0) id = current_ctx_id();
    g_cached[dev] = Cached{id, id ? p : nullptr};
    *out = p;
    return TCV_OK;
}

}  // namespace

extern "C" {

size_t tcv_static_scratch_bytes(void) { return kStaticScratchBytes; }

tcv_status tcv_grid_raw_static(const float* d_data, int64_t n, int support, const void* d_c, int c_type,
                               float c_scale, int64_t c_len, const int32_t* d_coff, const int32_t* d_iu,
                               const int32_t* d_iv, float* d_grid, int g_size, void* stream)
{
    if (n < 0 || support < 0 || g_size < 1 || c_len < 1 || !d_c || !d_grid) return TCV_ERR_ARG;
    if (n > 0 && (!d_data || !d_coff || !d_iu || !d_iv)) return TCV_ERR_ARG;
    if (tcv_ctype_bytes(c_type) == 0) return TCV_ERR_ARG;
    // sizes beyond the fixed array are rejected before anything touches the device
    const size_t need = tcv_plan_workspace_bytes(n, support, g_size, c_len);
    if (need == 0 || need > kStaticScratchBytes) return TCV_ERR_WORKSPACE;
    void* scratch = nullptr;
    tcv_status s = scratch_address(&scratch);
    if (s != TCV_OK) return s;
    tcv_plan plan;  // host-side description on the stack; its arrays live in the static scratch
    s = tcv::plan_init(&plan, d_iu, d_iv, d_coff, n, support, g_size, c_len, scratch, kStaticScratchBytes,
                       static_cast<cudaStream_t>(stream));
    if (s != TCV_OK) return s;
    plan.jit_cached_only = true;  // no NVRTC build or module load inside this call
    return tcv_plan_grid(&plan, d_data, d_c, c_type, c_scale, d_grid, stream);
}

}  // extern "C"
