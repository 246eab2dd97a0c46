// HogbomB200.cc -- HogbomB200 over tcv_hogbom_deconvolve: the images are copied to the device,
// cleaned there, and the model and residual copied back.
#include "HogbomB200.h"

#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

#include "tconvolve.h"

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

void tcv_check(tcv_status s, const char* what)
{
    if (s != TCV_OK) throw std::runtime_error(std::string(what) + " failed: " + tcv_status_string(s));
}
}  // namespace

HogbomB200::HogbomB200(unsigned int niters, float gain, float threshold)
    : niters_(niters), gain_(gain), threshold_(threshold)
{
}

void HogbomB200::deconvolve(const std::vector<float>& dirty, const size_t dirtyWidth, const std::vector<float>& psf,
                            const size_t psfWidth, std::vector<float>& model, std::vector<float>& residual)
{
    if (dirty.size() != dirtyWidth * dirtyWidth || psf.size() != psfWidth * psfWidth || model.size() != dirty.size())
        throw std::runtime_error("deconvolve: image sizes");
    const size_t nb = dirty.size() * sizeof(float), pb = psf.size() * sizeof(float);
    const size_t wb = tcv_hogbom_workspace_bytes(int(dirtyWidth));
    DevBuf dd(nb), dp(pb), dm(nb), dr(nb), dw(wb);
    cuda_check(cudaMemcpy(dd.p, dirty.data(), nb, cudaMemcpyHostToDevice), "copy dirty");
    cuda_check(cudaMemcpy(dp.p, psf.data(), pb, cudaMemcpyHostToDevice), "copy psf");
    cuda_check(cudaMemcpy(dm.p, model.data(), nb, cudaMemcpyHostToDevice), "copy model");
    cudaEvent_t e0, e1;
    cuda_check(cudaEventCreate(&e0), "event");
    cuda_check(cudaEventCreate(&e1), "event");
    cuda_check(cudaEventRecord(e0, nullptr), "event");
    tcv_check(tcv_hogbom_deconvolve(static_cast<float*>(dd.p), int(dirtyWidth), static_cast<float*>(dp.p),
                                    int(psfWidth), static_cast<float*>(dm.p), static_cast<float*>(dr.p),
                                    int(niters_), gain_, threshold_, nullptr, nullptr, dw.p, wb, nullptr),
              "tcv_hogbom_deconvolve");
    cuda_check(cudaEventRecord(e1, nullptr), "event");
    cuda_check(cudaEventSynchronize(e1), "event");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    seconds_ = ms * 1e-3;
    tcv_check(tcv_hogbom_result(dw.p, &done_, nullptr, nullptr, nullptr, nullptr), "tcv_hogbom_result");
    residual.resize(dirty.size());
    cuda_check(cudaMemcpy(residual.data(), dr.p, nb, cudaMemcpyDeviceToHost), "copy residual");
    cuda_check(cudaMemcpy(model.data(), dm.p, nb, cudaMemcpyDeviceToHost), "copy model");
}
