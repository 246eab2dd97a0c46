// tcv_probe.cu -- a measurement of this GPU's L2-to-SM bandwidth for the tile kernels' table reads.
//
// The gridding and degridding tile kernels keep the grid in registers (or shared memory) and read
// the convolution table from L2: per sample and warp, kR rows of 32 consecutive entries (128 bytes
// for the real float form) at the table's row stride (the footprint width), at a random position
// (the sample's oversampling offset and w-plane).  The HBM copy bandwidth is not their ceiling;
// this probe measures the one that is: warps reading random 128-byte row segments, 16 rows of one
// "kernel" each with a 129-entry stride, from a buffer that fits in L2, 16 loads in flight per lane.
// Built as its own library (libtcvprobe.so): a measurement tool, not part of the gridding ABI.
// No counterpart in the reference.
#include "tcv_internal.cuh"
#include "tcv_probe.h"

namespace tcv {
namespace {

constexpr int kProbeThreads = 256;
constexpr int kProbeRows = 16;

__device__ __forceinline__ unsigned int mix32(unsigned int x)
{
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}

// Each warp reads `samples` random 16-row windows; lane l reads entry l of every row.  The sum
// is written so that the loads are not removed.
__global__ void __launch_bounds__(kProbeThreads) probe_table_kernel(const float* __restrict__ buf,
                                                                    unsigned int n_starts, int stride, int samples,
                                                                    float* __restrict__ out)
{
    const unsigned int warp = (blockIdx.x * kProbeThreads + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    float acc = 0.f;
    for (int j = 0; j < samples; ++j) {
        const unsigned int base = mix32(warp * 2654435761U + unsigned(j)) % n_starts;
        const float* p = buf + base + lane;
        float v[kProbeRows];
#pragma unroll
        for (int r = 0; r < kProbeRows; ++r) v[r] = __ldg(p + r * stride);
#pragma unroll
        for (int r = 0; r < kProbeRows; ++r) acc += v[r];
    }
    out[blockIdx.x * kProbeThreads + threadIdx.x] = acc;
}

}  // namespace
}  // namespace tcv

using namespace tcv;

extern "C" {

int64_t tcv_probe_table_threads(void)
{
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return int64_t(sms) * 8 * kProbeThreads;
}

tcv_status tcv_probe_table_stream(const float* d_buf, int64_t n_floats, int stride, int samples, float* d_out,
                                  int64_t* bytes_out, void* stream)
{
    if (!d_buf || !d_out || stride < 32 || samples < 1) return TCV_ERR_ARG;
    const int64_t span = int64_t(kProbeRows - 1) * stride + 32;
    if (n_floats < span + 1 || n_floats - span > int64_t(0xffffffffll)) return TCV_ERR_ARG;
    const int64_t threads = tcv_probe_table_threads();
    const unsigned blocks = unsigned(threads / kProbeThreads);
    probe_table_kernel<<<blocks, kProbeThreads, 0, static_cast<cudaStream_t>(stream)>>>(
        d_buf, unsigned(n_floats - span), stride, samples, d_out);
    TCV_CUDA(cudaGetLastError());
    if (bytes_out) *bytes_out = (threads / 32) * int64_t(samples) * kProbeRows * 128;
    return TCV_OK;
}

}  // extern "C"
