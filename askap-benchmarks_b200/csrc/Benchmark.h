// Benchmark.h -- the reference's Benchmark class (attic/tConvolveMPI/Benchmark.h:55-99) on the
// B200 library.  Same type names, method names, argument meaning and call order; the problem
// constants (Benchmark.h:39-46 in the reference) become a runtime tcv_config whose defaults are
// the reference's values.  Every buffer lives on the GPU inside a tcv_ctx; the std::vector
// forms of the kernels (gridKernel, degridKernel, initC) copy to and from the device.
//
// Errors are thrown as std::runtime_error, as the reference's helpers throw
// (attic/tConvolveMPI/Stopwatch.cc:47-61).
#ifndef TCONVOLVE_B200_BENCHMARK_H
#define TCONVOLVE_B200_BENCHMARK_H

#include <complex>
#include <vector>

#include "tconvolve.h"

typedef double Coord;
typedef float Real;
typedef std::complex<Real> Value;

struct Sample {
    Value data;
    int iu;
    int iv;
    int cOffset;
};

class Benchmark {
public:
    Benchmark();                              // the reference's constants
    explicit Benchmark(const tcv_config& cfg);
    ~Benchmark();
    Benchmark(const Benchmark&) = delete;
    Benchmark& operator=(const Benchmark&) = delete;

    int randomInt();
    void init();
    void runGrid();
    void runDegrid();

    void gridKernel(const int support, const std::vector<Value>& C, std::vector<Value>& grid,
                    const int gSize);
    void degridKernel(const std::vector<Value>& grid, const int gSize, const int support,
                      const std::vector<Value>& C, std::vector<Value>& data);
    void initC(const std::vector<Coord>& freq, const Coord cellSize, const int wSize, int& support,
               int& overSample, Coord& wCellSize, std::vector<Value>& C);
    void initCOffset(const std::vector<Coord>& u, const std::vector<Coord>& v,
                     const std::vector<Coord>& w, const std::vector<Coord>& freq,
                     const Coord cellSize, const Coord wCellSize, const int wSize,
                     const int gSize, const int support, const int overSample);
    int getSupport();

    // Beyond the reference interface: device synchronisation and result access.
    void sync();
    const tcv_config& config() const { return cfg_; }
    tcv_ctx* context() { return ctx_; }
    double updatesPerPass() const;
    std::vector<Value> gridValues();
    std::vector<Value> outdata();
    std::vector<Sample> samples();
    void setData(const std::vector<Value>& data);

private:
    void check(tcv_status s, const char* what) const;
    tcv_config cfg_;
    tcv_ctx* ctx_ = nullptr;
    unsigned long next_;
};

#endif
