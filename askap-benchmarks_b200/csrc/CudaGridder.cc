// CudaGridder.cc -- libCudaGridder.so: the reference's gridKernelCuda / degridKernelCuda
// (attic/tConvolveCuda/CudaGridder.h:32-50) on the B200 library.
#include "CudaGridder.h"

#include <cstdlib>
#include <iostream>

#include "tconvolve.h"

namespace {
void check(tcv_status s)
{
    if (s == TCV_OK) return;
    std::cout << "CUDA Error: " << tcv_status_string(s) << std::endl;
    std::exit(1);
}

void report_device()
{
    // the reference reports the device in use (CudaGridder.cc:60-66)
    std::cout << "    Using CUDA Device 0: " << tcv_version() << std::endl;
}
}  // namespace

void gridKernelCuda(const std::vector<std::complex<float> >& data, const int support,
                    const std::vector<std::complex<float> >& C, const std::vector<int>& cOffset,
                    const std::vector<int>& iu, const std::vector<int>& iv,
                    std::vector<std::complex<float> >& grid, const int gSize, double& time)
{
    report_device();
    if (cOffset.size() != data.size() || iu.size() != data.size() || iv.size() != data.size() ||
        grid.size() != size_t(gSize) * size_t(gSize))
        check(TCV_ERR_ARG);
    check(tcv_grid_host_raw(reinterpret_cast<const float*>(data.data()), int64_t(data.size()), support,
                            reinterpret_cast<const float*>(C.data()), int64_t(C.size()), cOffset.data(),
                            iu.data(), iv.data(), reinterpret_cast<float*>(grid.data()), gSize, 0, &time));
}

void degridKernelCuda(const std::vector<std::complex<float> >& grid, const int gSize,
                      const int support, const std::vector<std::complex<float> >& C,
                      const std::vector<int>& cOffset, const std::vector<int>& iu,
                      const std::vector<int>& iv, std::vector<std::complex<float> >& data,
                      double& time)
{
    report_device();
    if (cOffset.size() != data.size() || iu.size() != data.size() || iv.size() != data.size() ||
        grid.size() != size_t(gSize) * size_t(gSize))
        check(TCV_ERR_ARG);
    check(tcv_degrid_host_raw(reinterpret_cast<const float*>(grid.data()), gSize, support,
                              reinterpret_cast<const float*>(C.data()), int64_t(C.size()), cOffset.data(),
                              iu.data(), iv.data(), reinterpret_cast<float*>(data.data()),
                              int64_t(data.size()), 0, &time));
}
