// tcv_jit.cu -- copies of the tile kernels specialised on the footprint width, built at run time.
//
// The tile kernels (tcv_device.cuh) spend most of their issue slots on per-row index arithmetic
// when sSize is a run-time value.  With sSize a compile-time constant, the row offsets of the 16
// loads a lane issues per sample become immediates of the load instructions and the loop bounds
// constants.  sSize depends on the problem (support = f(cellSize, baseline, frequency),
// attic/tConvolveMPI/Benchmark.cc:212-213), so the specialised copies are compiled with NVRTC the
// first time a (kernel, table form, sSize) combination is launched, loaded with
// cudaLibraryLoadData and cached for the life of the process.  NVRTC is loaded with dlopen; if it
// is missing or a compilation fails, the launch uses the generic copy compiled into this library
// (the same code with sSize at run time) and tcv_jit_info reports why.  The first launch for a new
// footprint width pays the compilation (about a second); call tcv_jit_prepare at set-up to pay it
// there.
#include "tcv_internal.cuh"

#include <dlfcn.h>
#include <nvrtc.h>

#include <cstdio>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "tcv_device_src.inc"  // kDeviceSrc: the text of tcv_device.cuh

namespace tcv {
namespace {

struct NvrtcApi {
    decltype(&nvrtcCreateProgram) create = nullptr;
    decltype(&nvrtcCompileProgram) compile = nullptr;
    decltype(&nvrtcGetProgramLogSize) log_size = nullptr;
    decltype(&nvrtcGetProgramLog) log = nullptr;
    decltype(&nvrtcGetCUBINSize) cubin_size = nullptr;
    decltype(&nvrtcGetCUBIN) cubin = nullptr;
    decltype(&nvrtcAddNameExpression) add_name = nullptr;
    decltype(&nvrtcGetLoweredName) lowered = nullptr;
    decltype(&nvrtcDestroyProgram) destroy = nullptr;
    bool ok = false;
};

std::mutex g_mu;
NvrtcApi g_api;
bool g_api_tried = false;
bool g_enabled = true;
std::string g_info = "no specialised kernel built yet";
std::map<std::tuple<int, int, int, int>, cudaKernel_t> g_cache;  // (kind, c_type, sSize, rows) -> kernel
std::map<std::tuple<int, int, int, int>, bool> g_failed;

bool load_api()
{
    if (g_api_tried) return g_api.ok;
    g_api_tried = true;
    const char* names[] = {"libnvrtc.so.12", "libnvrtc.so"};
    void* h = nullptr;
    for (const char* n : names)
        if ((h = dlopen(n, RTLD_NOW | RTLD_LOCAL))) break;
    if (!h) {
        g_info = "NVRTC not found (libnvrtc.so.12); generic kernels in use";
        return false;
    }
    auto sym = [&](const char* n) { return dlsym(h, n); };
    g_api.create = reinterpret_cast<decltype(g_api.create)>(sym("nvrtcCreateProgram"));
    g_api.compile = reinterpret_cast<decltype(g_api.compile)>(sym("nvrtcCompileProgram"));
    g_api.log_size = reinterpret_cast<decltype(g_api.log_size)>(sym("nvrtcGetProgramLogSize"));
    g_api.log = reinterpret_cast<decltype(g_api.log)>(sym("nvrtcGetProgramLog"));
    g_api.cubin_size = reinterpret_cast<decltype(g_api.cubin_size)>(sym("nvrtcGetCUBINSize"));
    g_api.cubin = reinterpret_cast<decltype(g_api.cubin)>(sym("nvrtcGetCUBIN"));
    g_api.add_name = reinterpret_cast<decltype(g_api.add_name)>(sym("nvrtcAddNameExpression"));
    g_api.lowered = reinterpret_cast<decltype(g_api.lowered)>(sym("nvrtcGetLoweredName"));
    g_api.destroy = reinterpret_cast<decltype(g_api.destroy)>(sym("nvrtcDestroyProgram"));
    g_api.ok = g_api.create && g_api.compile && g_api.log_size && g_api.log && g_api.cubin_size && g_api.cubin &&
               g_api.add_name && g_api.lowered && g_api.destroy;
    if (!g_api.ok) g_info = "NVRTC symbols missing; generic kernels in use";
    return g_api.ok;
}

const char* tab_name(int c_type)
{
    switch (c_type) {
        case TCV_C_C64: return "tcv::TabC64";
        case TCV_C_R32: return "tcv::TabR32";
        case TCV_C_CBF16: return "tcv::TabCBF16";
        case TCV_C_RBF16: return "tcv::TabRBF16";
        default: return nullptr;  // float16 forms need cuda_fp16.h: generic kernels only
    }
}

// Build (or fetch) the specialised kernel; nullptr if unavailable.  Caller holds g_mu.
cudaKernel_t build(int kind, int c_type, int s, int rows)
{
    const auto key = std::make_tuple(kind, c_type, s, rows);
    auto it = g_cache.find(key);
    if (it != g_cache.end()) return it->second;
    if (g_failed.count(key)) return nullptr;
    const char* tab = tab_name(c_type);
    if (!tab || s < 1 || s > 4096 || (rows != 8 && rows != 16 && rows != 32) || !load_api()) {
        g_failed[key] = true;
        return nullptr;
    }
    const std::string expr = std::string(kind == 0 ? "tcv::grid_tile_kernel<" : "tcv::degrid_tile_kernel<") + tab +
                             ", " + std::to_string(s) + ", " + std::to_string(rows) + ">";
    const std::string body = "#include \"tcv_device.cuh\"\n";
    const char* hdr_src[] = {kDeviceSrc};
    const char* hdr_name[] = {"tcv_device.cuh"};
    nvrtcProgram prog = nullptr;
    if (g_api.create(&prog, body.c_str(), "tcv_tile_specialised.cu", 1, hdr_src, hdr_name) != NVRTC_SUCCESS) {
        g_failed[key] = true;
        g_info = "nvrtcCreateProgram failed; generic kernels in use";
        return nullptr;
    }
    g_api.add_name(prog, expr.c_str());
    const char* opts[] = {"--gpu-architecture=sm_100a", "-std=c++17", "-default-device", "--fmad=true"};
    const nvrtcResult cr = g_api.compile(prog, 4, opts);
    cudaKernel_t k = nullptr;
    if (cr == NVRTC_SUCCESS) {
        size_t n = 0;
        g_api.cubin_size(prog, &n);
        std::vector<char> cubin(n);
        const char* lowered = nullptr;
        if (n && g_api.cubin(prog, cubin.data()) == NVRTC_SUCCESS &&
            g_api.lowered(prog, expr.c_str(), &lowered) == NVRTC_SUCCESS && lowered) {
            cudaLibrary_t lib = nullptr;
            if (cudaLibraryLoadData(&lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0) == cudaSuccess &&
                cudaLibraryGetKernel(&k, lib, lowered) == cudaSuccess) {
                g_info = "specialised tile kernels in use (NVRTC, sSize " + std::to_string(s) + ", " +
                         std::to_string(rows) + " rows per warp)";
            } else {
                k = nullptr;
                cudaGetLastError();
                g_info = "loading the specialised kernel failed; generic kernels in use";
            }
        }
    } else {
        size_t ln = 0;
        g_api.log_size(prog, &ln);
        std::string log(ln, '\0');
        if (ln) g_api.log(prog, &log[0]);
        g_info = "NVRTC compilation failed; generic kernels in use: " + log.substr(0, 400);
    }
    g_api.destroy(&prog);
    if (k)
        g_cache[key] = k;
    else
        g_failed[key] = true;
    return k;
}

}  // namespace

const void* jit_tile_kernel(int kind, int c_type, int s, int rows)
{
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_enabled) return nullptr;
    return reinterpret_cast<const void*>(build(kind, c_type, s, rows));
}

const void* jit_tile_kernel_cached(int kind, int c_type, int s, int rows)
{
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_enabled) return nullptr;
    const auto it = g_cache.find(std::make_tuple(kind, c_type, s, rows));
    return it == g_cache.end() ? nullptr : reinterpret_cast<const void*>(it->second);
}

void jit_prepare(int c_type, int s, int rows)
{
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_enabled) return;
    build(0, c_type & 0xff, s, rows);
    build(1, c_type & 0xff, s, rows);
}

}  // namespace tcv

using namespace tcv;

extern "C" {

tcv_status tcv_jit_prepare(int c_type, int support)
{
    if (tcv_ctype_bytes(c_type) == 0 || support < 0) return TCV_ERR_ARG;
    const int s = 2 * support + 1;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_enabled) return TCV_OK;
    build(0, c_type & 0xff, s, 16);
    build(1, c_type & 0xff, s, 16);
    return TCV_OK;
}

void tcv_jit_enable(int enabled)
{
    std::lock_guard<std::mutex> lock(g_mu);
    g_enabled = enabled != 0;
}

const char* tcv_jit_info(void)
{
    std::lock_guard<std::mutex> lock(g_mu);
    static thread_local std::string copy;
    copy = g_enabled ? g_info : std::string("specialisation disabled; generic kernels in use");
    return copy.c_str();
}

}  // extern "C"
