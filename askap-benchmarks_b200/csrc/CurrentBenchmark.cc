// CurrentBenchmark.cc -- current::Benchmark over the tcv_cur_* C ABI.
#include "CurrentBenchmark.h"

#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

namespace current {

namespace {
struct DevBuf {
    void* p = nullptr;
    explicit DevBuf(size_t bytes)
    {
        if (bytes && cudaMalloc(&p, bytes) != cudaSuccess) throw std::runtime_error("cudaMalloc failed");
    }
    ~DevBuf()
    {
        if (p) cudaFree(p);
    }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
};

void cuda_check(cudaError_t e, const char* what)
{
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}
}  // namespace

Benchmark::Benchmark(int device) { check(tcv_cur_create(device, &ctx_), "tcv_cur_create"); }

Benchmark::~Benchmark()
{
    if (ctx_) tcv_cur_destroy(ctx_);
}

void Benchmark::check(tcv_status s, const char* what) const
{
    if (s != TCV_OK) {
        std::string msg = std::string(what) + " failed: " + tcv_status_string(s);
        if (ctx_) msg += std::string(" (") + tcv_cur_last_error(ctx_) + ")";
        throw std::runtime_error(msg);
    }
}

void Benchmark::init() { check(tcv_cur_init(ctx_), "tcv_cur_init"); }
void Benchmark::runGrid() { check(tcv_cur_run_grid(ctx_), "tcv_cur_run_grid"); }
void Benchmark::runDegrid() { check(tcv_cur_run_degrid(ctx_), "tcv_cur_run_degrid"); }
void Benchmark::sync() { check(tcv_cur_sync(ctx_), "tcv_cur_sync"); }
int Benchmark::getSupport() { return tcv_cur_support(ctx_); }
long Benchmark::nVisibilitiesGridded() { return long(tcv_cur_n_visibilities(ctx_)); }
long Benchmark::nPixelsGridded() { return long(tcv_cur_n_pixels(ctx_)); }
void Benchmark::setSort(const int type) { check(tcv_cur_set_sort(ctx_, type), "tcv_cur_set_sort"); }
void Benchmark::setRunType(const int type) { check(tcv_cur_set_run_type(ctx_, type), "tcv_cur_set_run_type"); }
int Benchmark::getRunType() { return tcv_cur_get_run_type(ctx_); }

std::vector<float> Benchmark::requiredRate()
{
    std::vector<float> r(2);
    tcv_cur_required_rate(r.data());
    return r;
}

void Benchmark::tune(int reps)
{
    tcv_tuning t{};
    check(tcv_cur_tune(ctx_, reps, &t, nullptr), "tcv_cur_tune");
    tuning_ = t;
}

void Benchmark::setTuning(const tcv_tuning& t)
{
    check(tcv_cur_set_tuning(ctx_, &t), "tcv_cur_set_tuning");
    tuning_ = t;
}

tcv_cur_geometry Benchmark::geometry()
{
    tcv_cur_geometry g{};
    check(tcv_cur_info(ctx_, &g), "tcv_cur_info");
    return g;
}

std::vector<Value> Benchmark::gridValues()
{
    const tcv_cur_geometry g = geometry();
    std::vector<Value> out(size_t(g.g_size) * g.g_size);
    check(tcv_cur_get_grid(ctx_, reinterpret_cast<float*>(out.data())), "tcv_cur_get_grid");
    return out;
}

std::vector<Value> Benchmark::outdata()
{
    std::vector<Value> out(static_cast<size_t>(nVisibilitiesGridded()));
    check(tcv_cur_get_outdata(ctx_, reinterpret_cast<float*>(out.data()), int64_t(out.size())), "tcv_cur_get_outdata");
    return out;
}

void Benchmark::initC(const Coord uvCellSize, const int wSize, int& support, int& overSample, Coord& wCellSize,
                      std::vector<Value>& C)
{
    const tcv_cur_geometry g = geometry();
    if (wSize != g.w_size || uvCellSize != g.uv_cell_size)
        throw std::runtime_error("initC: uvCellSize and wSize must be the run type's");
    support = g.support;
    overSample = g.over_sample;
    wCellSize = g.w_cell_size;
    C.resize(size_t(g.c_len));
    DevBuf d(size_t(g.c_len) * sizeof(Value));
    check(tcv_cur_init_c_raw(getRunType(), static_cast<float*>(d.p), nullptr), "tcv_cur_init_c_raw");
    cuda_check(cudaMemcpy(C.data(), d.p, C.size() * sizeof(Value), cudaMemcpyDeviceToHost), "copy C");
}

// The object's offsets with a caller's table: a variable-width plan over device copies.
namespace {
struct VarRun {
    DevBuf iu, iv, wp, co, work;
    tcv_plan* plan = nullptr;
    VarRun(size_t n, size_t wbytes) : iu(n * 4), iv(n * 4), wp(n * 4), co(n * 4), work(wbytes) {}
    ~VarRun()
    {
        if (plan) tcv_plan_destroy(plan);
    }
};
}  // namespace

void Benchmark::gridKernel(const std::vector<Value>& C, std::vector<Value>& grid, const int gSize)
{
    const tcv_cur_geometry g = geometry();
    if (gSize != g.g_size || grid.size() != size_t(gSize) * gSize || int64_t(C.size()) < g.c_len)
        throw std::runtime_error("gridKernel: grid or table of the wrong size");
    const size_t n = size_t(nVisibilitiesGridded());
    std::vector<int32_t> iu(n), iv(n), wp(n), co(n), s(size_t(g.w_size)), off0(size_t(g.w_size));
    check(tcv_cur_get_offsets(ctx_, iu.data(), iv.data(), wp.data(), co.data()), "tcv_cur_get_offsets");
    check(tcv_cur_get_planes(ctx_, s.data(), off0.data()), "tcv_cur_get_planes");
    const size_t wb = tcv_plan_workspace_bytes_var(int64_t(n), s.data(), off0.data(), g.w_size, gSize, int64_t(C.size()),
                                                   &tuning_);
    if (wb == 0) throw std::runtime_error("gridKernel: plan geometry");
    VarRun r(n, wb);
    DevBuf dc(C.size() * sizeof(Value)), dg(grid.size() * sizeof(Value)), dd(n * sizeof(Value));
    cuda_check(cudaMemcpy(r.iu.p, iu.data(), n * 4, cudaMemcpyHostToDevice), "copy iu");
    cuda_check(cudaMemcpy(r.iv.p, iv.data(), n * 4, cudaMemcpyHostToDevice), "copy iv");
    cuda_check(cudaMemcpy(r.wp.p, wp.data(), n * 4, cudaMemcpyHostToDevice), "copy wplane");
    cuda_check(cudaMemcpy(r.co.p, co.data(), n * 4, cudaMemcpyHostToDevice), "copy cOffset");
    cuda_check(cudaMemcpy(dc.p, C.data(), C.size() * sizeof(Value), cudaMemcpyHostToDevice), "copy C");
    cuda_check(cudaMemcpy(dg.p, grid.data(), grid.size() * sizeof(Value), cudaMemcpyHostToDevice), "copy grid");
    // the object's visibilities (1 + 0i as the reference's init sets them, or set by the caller)
    std::vector<Value> ones(n, Value(1.0f, 0.0f));
    cuda_check(cudaMemcpy(dd.p, ones.data(), n * sizeof(Value), cudaMemcpyHostToDevice), "copy data");
    check(tcv_plan_build_var(&r.plan, static_cast<int32_t*>(r.iu.p), static_cast<int32_t*>(r.iv.p),
                             static_cast<int32_t*>(r.co.p), static_cast<int32_t*>(r.wp.p), int64_t(n), s.data(),
                             off0.data(), g.w_size, gSize, int64_t(C.size()), &tuning_, r.work.p, wb, nullptr),
          "tcv_plan_build_var");
    check(tcv_plan_grid(r.plan, static_cast<float*>(dd.p), dc.p, TCV_C_C64, 1.f, static_cast<float*>(dg.p), nullptr),
          "tcv_plan_grid");
    cuda_check(cudaMemcpy(grid.data(), dg.p, grid.size() * sizeof(Value), cudaMemcpyDeviceToHost), "copy grid");
}

void Benchmark::degridKernel(const std::vector<Value>& grid, const int gSize, const std::vector<Value>& C,
                             std::vector<Value>& data)
{
    const tcv_cur_geometry g = geometry();
    if (gSize != g.g_size || grid.size() != size_t(gSize) * gSize || int64_t(C.size()) < g.c_len)
        throw std::runtime_error("degridKernel: grid or table of the wrong size");
    const size_t n = size_t(nVisibilitiesGridded());
    data.resize(n);
    std::vector<int32_t> iu(n), iv(n), wp(n), co(n), s(size_t(g.w_size)), off0(size_t(g.w_size));
    check(tcv_cur_get_offsets(ctx_, iu.data(), iv.data(), wp.data(), co.data()), "tcv_cur_get_offsets");
    check(tcv_cur_get_planes(ctx_, s.data(), off0.data()), "tcv_cur_get_planes");
    const size_t wb = tcv_plan_workspace_bytes_var(int64_t(n), s.data(), off0.data(), g.w_size, gSize, int64_t(C.size()),
                                                   &tuning_);
    if (wb == 0) throw std::runtime_error("degridKernel: plan geometry");
    VarRun r(n, wb);
    DevBuf dc(C.size() * sizeof(Value)), dg(grid.size() * sizeof(Value)), dd(n * sizeof(Value));
    cuda_check(cudaMemcpy(r.iu.p, iu.data(), n * 4, cudaMemcpyHostToDevice), "copy iu");
    cuda_check(cudaMemcpy(r.iv.p, iv.data(), n * 4, cudaMemcpyHostToDevice), "copy iv");
    cuda_check(cudaMemcpy(r.wp.p, wp.data(), n * 4, cudaMemcpyHostToDevice), "copy wplane");
    cuda_check(cudaMemcpy(r.co.p, co.data(), n * 4, cudaMemcpyHostToDevice), "copy cOffset");
    cuda_check(cudaMemcpy(dc.p, C.data(), C.size() * sizeof(Value), cudaMemcpyHostToDevice), "copy C");
    cuda_check(cudaMemcpy(dg.p, grid.data(), grid.size() * sizeof(Value), cudaMemcpyHostToDevice), "copy grid");
    check(tcv_plan_build_var(&r.plan, static_cast<int32_t*>(r.iu.p), static_cast<int32_t*>(r.iv.p),
                             static_cast<int32_t*>(r.co.p), static_cast<int32_t*>(r.wp.p), int64_t(n), s.data(),
                             off0.data(), g.w_size, gSize, int64_t(C.size()), &tuning_, r.work.p, wb, nullptr),
          "tcv_plan_build_var");
    check(tcv_plan_degrid(r.plan, static_cast<float*>(dg.p), dc.p, TCV_C_C64, 1.f, static_cast<float*>(dd.p), nullptr),
          "tcv_plan_degrid");
    cuda_check(cudaMemcpy(data.data(), dd.p, n * sizeof(Value), cudaMemcpyDeviceToHost), "copy data");
}

}  // namespace current
