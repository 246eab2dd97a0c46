// CurrentBenchmark.h -- the Benchmark class of current/tConvolveMPI (current/tConvolveMPI/Benchmark.h:38-111)
// on the B200 library, in namespace `current` (the attic Benchmark keeps the global name).  Same
// method names, argument meaning and call order; every buffer lives on the GPU inside a
// tcv_cur_ctx.  The std::vector forms of the kernels and of initC copy to and from the device.
// Errors are thrown as std::runtime_error.
#ifndef TCONVOLVE_B200_CURRENT_BENCHMARK_H
#define TCONVOLVE_B200_CURRENT_BENCHMARK_H

#include <complex>
#include <vector>

#include "tconvolve.h"

namespace current {

typedef double Coord;
typedef float Real;
typedef std::complex<Real> Value;

class Benchmark {
public:
    explicit Benchmark(int device = 0);
    ~Benchmark();
    Benchmark(const Benchmark&) = delete;
    Benchmark& operator=(const Benchmark&) = delete;

    void init();
    void runGrid();
    void runDegrid();

    // the object's samples (with the unit visibilities its init() sets, Benchmark.cc:258-262) and a
    // caller's table and grid (current/tConvolveMPI/Benchmark.cc:373-452)
    void gridKernel(const std::vector<Value>& C, std::vector<Value>& grid, const int gSize);
    void degridKernel(const std::vector<Value>& grid, const int gSize, const std::vector<Value>& C,
                      std::vector<Value>& data);
    // the run type's table (Benchmark.cc:471-586); uvCellSize and wSize must be the run type's
    void initC(const Coord uvCellSize, const int wSize, int& support, int& overSample, Coord& wCellSize,
               std::vector<Value>& C);

    int getSupport();
    long nVisibilitiesGridded();
    long nPixelsGridded();
    std::vector<float> requiredRate();

    void setMPIrank(const int rank) { mpirank_ = rank; }
    void setSort(const int type);
    void setRunType(const int type);
    int getRunType();

    // Beyond the reference interface
    void sync();
    void tune(int reps = 3);  // tcv_cur_tune: picks the plan for this run type (untimed set-up)
    void setTuning(const tcv_tuning& t);
    tcv_tuning tuning() const { return tuning_; }
    tcv_cur_geometry geometry();
    std::vector<Value> gridValues();
    std::vector<Value> outdata();
    tcv_cur_ctx* context() { return ctx_; }

private:
    void check(tcv_status s, const char* what) const;
    tcv_cur_ctx* ctx_ = nullptr;
    int mpirank_ = 0;
    tcv_tuning tuning_{16, 32, 0, 0, 0};
};

}  // namespace current

#endif
