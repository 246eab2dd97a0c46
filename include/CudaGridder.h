/*
 * CudaGridder.h -- the reference's host-side CUDA gridder seam, provided by libCudaGridder.so of
 * this project so that programs written against attic/tConvolveCuda/CudaGridder.h:32-50 link
 * unchanged.  C++ symbols (std::vector in the signatures), as in the reference; the
 * implementation forwards to the C ABI of tconvolve.h (tcv_grid_host_raw / tcv_degrid_host_raw).
 *
 *   gridKernelCuda   replaces attic/tConvolveCuda/CudaGridder.cc:54-128
 *   degridKernelCuda replaces attic/tConvolveCuda/CudaGridder.cc:130-207
 *
 * `time` receives the device time (CUDA events) of the binning plan plus the kernel, the region
 * the reference times around its launches.  On error the functions print "CUDA Error: ..." and
 * exit(1), as the reference's checkerror does (CudaGridder.cc:45-52).
 */
#ifndef CUDA_GRIDDER_H
#define CUDA_GRIDDER_H

#include <complex>
#include <vector>

void gridKernelCuda(const std::vector<std::complex<float> >& data, const int support,
                    const std::vector<std::complex<float> >& C, const std::vector<int>& cOffset,
                    const std::vector<int>& iu, const std::vector<int>& iv,
                    std::vector<std::complex<float> >& grid, const int gSize, double& time);

void degridKernelCuda(const std::vector<std::complex<float> >& grid, const int gSize,
                      const int support, const std::vector<std::complex<float> >& C,
                      const std::vector<int>& cOffset, const std::vector<int>& iu,
                      const std::vector<int>& iv, std::vector<std::complex<float> >& data,
                      double& time);

#endif
