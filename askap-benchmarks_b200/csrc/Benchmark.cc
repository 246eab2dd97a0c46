// Benchmark.cc -- the reference's Benchmark class on libtconvolve (see Benchmark.h).
#include "Benchmark.h"

#include <cmath>
#include <iostream>
#include <limits>
#include <stdexcept>
#include <string>

namespace {
tcv_config defaults()
{
    tcv_config c;
    tcv_config_default(&c);
    return c;
}
}  // namespace

Benchmark::Benchmark() : Benchmark(defaults()) {}

Benchmark::Benchmark(const tcv_config& cfg) : cfg_(cfg), next_(cfg.seed + 1)
{
    check(tcv_create(&cfg_, &ctx_), "tcv_create");
}

Benchmark::~Benchmark() { tcv_destroy(ctx_); }

void Benchmark::check(tcv_status s, const char* what) const
{
    if (s == TCV_OK) return;
    std::string msg = std::string(what) + " failed: " + tcv_status_string(s);
    if (ctx_) msg += std::string(" (") + tcv_last_error(ctx_) + ")";
    throw std::runtime_error(msg);
}

// attic/tConvolveMPI/Benchmark.cc:53-58
int Benchmark::randomInt()
{
    const unsigned int maxint = std::numeric_limits<int>::max();
    next_ = next_ * 1103515245 + 12345;
    return ((unsigned int)(next_ / 65536) % maxint);
}

// Benchmark::init, printing the lines the reference's initC prints (Benchmark.cc:211-234).
void Benchmark::init()
{
    std::cout << "Initializing W projection convolution function" << std::endl;
    const tcv_status s = tcv_init(ctx_);
    const int support = tcv_support(ctx_);
    const int sSize = 2 * support + 1;
    const int os = tcv_over_sample(ctx_);
    std::cout << "Support = " << support << " pixels" << std::endl;
    std::cout << "W cellsize = " << tcv_w_cell_size(ctx_) << " wavelengths" << std::endl;
    std::cout << "Size of convolution function = " << tcv_c_len(ctx_) * int64_t(sizeof(Value)) / (1024 * 1024)
              << " MB" << std::endl;
    std::cout << "Shape of convolution function = [" << sSize << ", " << sSize << ", " << os << ", " << os
              << ", " << cfg_.w_size << "]" << std::endl;
    check(s, "init");
}
void Benchmark::runGrid() { check(tcv_run_grid(ctx_), "runGrid"); }
void Benchmark::runDegrid() { check(tcv_run_degrid(ctx_), "runDegrid"); }
int Benchmark::getSupport() { return tcv_support(ctx_); }
void Benchmark::sync() { check(tcv_sync(ctx_), "sync"); }
double Benchmark::updatesPerPass() const { return tcv_updates_per_pass(ctx_); }

std::vector<Sample> Benchmark::samples()
{
    const int64_t n = tcv_n_data(ctx_);
    std::vector<Value> d(n);
    std::vector<int32_t> iu(n), iv(n), co(n);
    check(tcv_get_data(ctx_, reinterpret_cast<float*>(d.data()), n), "samples");
    check(tcv_get_offsets(ctx_, iu.data(), iv.data(), co.data()), "samples");
    std::vector<Sample> s(n);
    for (int64_t i = 0; i < n; ++i) s[i] = Sample{d[i], iu[i], iv[i], co[i]};
    return s;
}

void Benchmark::setData(const std::vector<Value>& data)
{
    check(tcv_set_data(ctx_, reinterpret_cast<const float*>(data.data()), int64_t(data.size())), "setData");
}

std::vector<Value> Benchmark::gridValues()
{
    std::vector<Value> g(size_t(cfg_.g_size) * cfg_.g_size);
    check(tcv_get_grid(ctx_, reinterpret_cast<float*>(g.data())), "grid");
    return g;
}

std::vector<Value> Benchmark::outdata()
{
    std::vector<Value> d(tcv_n_data(ctx_));
    check(tcv_get_outdata(ctx_, reinterpret_cast<float*>(d.data()), int64_t(d.size())), "outdata");
    return d;
}

// Benchmark::gridKernel with the caller's table and grid (host vectors), on this object's samples.
void Benchmark::gridKernel(const int support, const std::vector<Value>& C, std::vector<Value>& grid,
                           const int gSize)
{
    if (grid.size() != size_t(gSize) * gSize) throw std::runtime_error("gridKernel: grid size mismatch");
    const std::vector<Sample> s = samples();
    const int64_t n = int64_t(s.size());
    std::vector<Value> d(n);
    std::vector<int32_t> iu(n), iv(n), co(n);
    for (int64_t i = 0; i < n; ++i) {
        d[i] = s[i].data;
        iu[i] = s[i].iu;
        iv[i] = s[i].iv;
        co[i] = s[i].cOffset;
    }
    check(tcv_grid_host_raw(reinterpret_cast<const float*>(d.data()), n, support,
                            reinterpret_cast<const float*>(C.data()), int64_t(C.size()), co.data(),
                            iu.data(), iv.data(), reinterpret_cast<float*>(grid.data()), gSize,
                            cfg_.device, nullptr),
          "gridKernel");
}

void Benchmark::degridKernel(const std::vector<Value>& grid, const int gSize, const int support,
                             const std::vector<Value>& C, std::vector<Value>& data)
{
    if (grid.size() != size_t(gSize) * gSize) throw std::runtime_error("degridKernel: grid size mismatch");
    const std::vector<Sample> s = samples();
    const int64_t n = int64_t(s.size());
    data.resize(n);
    std::vector<int32_t> iu(n), iv(n), co(n);
    for (int64_t i = 0; i < n; ++i) {
        iu[i] = s[i].iu;
        iv[i] = s[i].iv;
        co[i] = s[i].cOffset;
    }
    check(tcv_degrid_host_raw(reinterpret_cast<const float*>(grid.data()), gSize, support,
                              reinterpret_cast<const float*>(C.data()), int64_t(C.size()), co.data(),
                              iu.data(), iv.data(), reinterpret_cast<float*>(data.data()), n,
                              cfg_.device, nullptr),
          "degridKernel");
}

void Benchmark::initC(const std::vector<Coord>& freq, const Coord cellSize, const int wSize,
                      int& support, int& overSample, Coord& wCellSize, std::vector<Value>& C)
{
    if (freq.empty()) throw std::runtime_error("initC: empty frequency list");
    int64_t c_len = 0;
    check(tcv_c_geometry(freq[0], cellSize, cfg_.baseline, wSize, &support, &overSample, &wCellSize, &c_len),
          "initC");
    C.resize(size_t(c_len));
    float sum_c = 0.f;
    check(tcv_init_c_host(freq[0], cellSize, cfg_.baseline, wSize, reinterpret_cast<float*>(C.data()), c_len,
                          cfg_.device, &support, &overSample, &wCellSize, &sum_c),
          "initC");
}

// The offsets are computed on the device for this object's samples; the arguments must describe
// this object's problem (the reference passes its own members, Benchmark.cc:94-95).
void Benchmark::initCOffset(const std::vector<Coord>& u, const std::vector<Coord>& v,
                            const std::vector<Coord>& w, const std::vector<Coord>& freq,
                            const Coord cellSize, const Coord wCellSize, const int wSize,
                            const int gSize, const int support, const int overSample)
{
    if (int64_t(u.size()) != cfg_.n_samples || v.size() != u.size() || w.size() != u.size() ||
        int(freq.size()) != cfg_.n_chan || cellSize != cfg_.cell_size || wSize != cfg_.w_size ||
        gSize != cfg_.g_size || support != tcv_support(ctx_) || overSample != tcv_over_sample(ctx_) ||
        wCellSize != tcv_w_cell_size(ctx_))
        throw std::runtime_error("initCOffset: arguments do not match this Benchmark's problem");
    check(tcv_set_uvw(ctx_, u.data(), v.data(), w.data()), "initCOffset");
}
