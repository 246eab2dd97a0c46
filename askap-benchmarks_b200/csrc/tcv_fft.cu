// tcv_fft.cu -- the FFT steps either side of gridding and degridding in the imaging major cycle.
//
// Reference: current/tMajorACC/tMajorACC.cc:487-640.  fftExec / fftExecGPU rotate the grid by half
// its size in both axes (the fftshift, :514-525), run an unnormalised 2-D C2C transform (FFTW or
// cuFFT; FFTW_FORWARD / CUFFT_FORWARD = exp(-i..), BACKWARD / INVERSE = exp(+i..)) and rotate back
// (:530-541); fftFix / fftFixGPU keep the real part times a scale (:620-640).  Odd sizes are
// refused, as there (:496-499).
//
// B200 form: the transform is cuFFT's single-precision C2C (the library the reference's own GPU
// path calls).  The two rotations cost no pass of their own: for an even size N, with S the
// half-size rotation and D the checkerboard sign (-1)^(x+y), F S = D F and S F = F D, so
//     S F S X = S D F X:   Y[k] = (-1)^(kx+ky) Z[k + N/2],  Z = F X      (fftExec in place)
//     S F S X = F D S X:   transform of (-1)^(x+y) X[x + N/2]             (from a real model image)
// Signs are exact, so only the transform rounds.  Image formation fuses the sign, the rotation, the
// real part and the scale into the gather that writes the float image (8 B read + 4 B written per
// pixel); the model-to-grid step fuses them into the pass that builds the complex input.
#include "tcv_internal.cuh"

#include <cufft.h>

#include <mutex>
#include <vector>

namespace tcv {
namespace {

struct FftPlan {
    int device, n;
    cufftHandle h;
};
std::mutex g_fft_mu;
std::vector<FftPlan> g_fft_plans;

tcv_status fft_status(cufftResult r) { return r == CUFFT_SUCCESS ? TCV_OK : TCV_ERR_CUDA; }

// The cached plan for an n x n C2C transform on the current device (g_fft_mu held).
tcv_status plan_for(int n, cufftHandle* out)
{
    int dev = 0;
    TCV_CUDA(cudaGetDevice(&dev));
    for (const FftPlan& p : g_fft_plans)
        if (p.device == dev && p.n == n) {
            *out = p.h;
            return TCV_OK;
        }
    cufftHandle h;
    if (cufftPlan2d(&h, n, n, CUFFT_C2C) != CUFFT_SUCCESS) return TCV_ERR_CUDA;
    g_fft_plans.push_back(FftPlan{dev, n, h});
    *out = h;
    return TCV_OK;
}

tcv_status exec_c2c(float2* d, int n, bool forward, cudaStream_t st)
{
    std::lock_guard<std::mutex> lock(g_fft_mu);
    cufftHandle h;
    const tcv_status s = plan_for(n, &h);
    if (s != TCV_OK) return s;
    if (cufftSetStream(h, st) != CUFFT_SUCCESS) return TCV_ERR_CUDA;
    return fft_status(cufftExecC2C(h, reinterpret_cast<cufftComplex*>(d), reinterpret_cast<cufftComplex*>(d),
                                   forward ? CUFFT_FORWARD : CUFFT_INVERSE));
}

__device__ __forceinline__ float chk(int x, int y) { return ((x + y) & 1) ? -1.f : 1.f; }

// In place: z[k] <- s(k) z[k + h], z[k + h] <- s(k) z[k] (h = (n/2, n/2)); one thread per pair.
__global__ void swap_sign_kernel(float2* __restrict__ z, int n)
{
    const int h = n >> 1;
    const long long pairs = (long long)h * n;  // rows 0 .. h-1, every column
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < pairs; i += (long long)gridDim.x * blockDim.x) {
        const int y = int(i / n), x = int(i - (long long)y * n);
        const int x2 = x < h ? x + h : x - h, y2 = y + h;
        const long long a = (long long)y * n + x, b = (long long)y2 * n + x2;
        const float s = chk(x, y);
        const float2 za = z[a], zb = z[b];
        z[a] = make_float2(s * zb.x, s * zb.y);
        z[b] = make_float2(s * za.x, s * za.y);
    }
}

// image[k] = Re(s(k) z[k + h]) * scale  (fftExec backward + fftFix, real part kept as float)
__global__ void image_fix_kernel(const float2* __restrict__ z, int n, float scale, float* __restrict__ image,
                                 float2* __restrict__ image_c)
{
    const int h = n >> 1;
    const long long np = (long long)n * n;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < np; i += (long long)gridDim.x * blockDim.x) {
        const int y = int(i / n), x = int(i - (long long)y * n);
        const int xs = x < h ? x + h : x - h, ys = y < h ? y + h : y - h;
        const float v = __fmul_rn(chk(x, y) * z[(long long)ys * n + xs].x, scale);
        if (image) image[i] = v;
        if (image_c) image_c[i] = make_float2(v, 0.f);
    }
}

// x[k] = s(k) * (image[k + h], 0): the input whose plain transform is fftExec(image) forward
__global__ void model_input_kernel(const float* __restrict__ image, int n, float2* __restrict__ x_out)
{
    const int h = n >> 1;
    const long long np = (long long)n * n;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < np; i += (long long)gridDim.x * blockDim.x) {
        const int y = int(i / n), x = int(i - (long long)y * n);
        const int xs = x < h ? x + h : x - h, ys = y < h ? y + h : y - h;
        x_out[i] = make_float2(chk(x, y) * image[(long long)ys * n + xs], 0.f);
    }
}

// grid[i] = (Re grid[i] * scale, 0)   (fftFix)
__global__ void fix_kernel(float2* __restrict__ g, long long n, float scale)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        g[i] = make_float2(__fmul_rn(g[i].x, scale), 0.f);
}

unsigned grid_blocks(long long work)
{
    const long long b = (work + 255) / 256;
    return unsigned(b < 148LL * 16 ? (b < 1 ? 1 : b) : 148LL * 16);
}

}  // namespace

tcv_status fft_exec(float2* d_grid, int n, bool forward, cudaStream_t st)
{
    TCV_CHECK(exec_c2c(d_grid, n, forward, st));
    swap_sign_kernel<<<grid_blocks((long long)(n / 2) * n), 256, 0, st>>>(d_grid, n);
    TCV_CUDA(cudaGetLastError());
    return TCV_OK;
}

tcv_status image_from_grid(float2* d_grid, int n, float scale, float* d_image, float2* d_image_c, cudaStream_t st)
{
    TCV_CHECK(exec_c2c(d_grid, n, false, st));
    image_fix_kernel<<<grid_blocks((long long)n * n), 256, 0, st>>>(d_grid, n, scale, d_image, d_image_c);
    TCV_CUDA(cudaGetLastError());
    return TCV_OK;
}

tcv_status grid_from_image(const float* d_image, int n, float2* d_grid, cudaStream_t st)
{
    model_input_kernel<<<grid_blocks((long long)n * n), 256, 0, st>>>(d_image, n, d_grid);
    TCV_CUDA(cudaGetLastError());
    return exec_c2c(d_grid, n, true, st);
}

}  // namespace tcv

using namespace tcv;

extern "C" {

tcv_status tcv_fft_exec(float* d_grid, int g_size, int forward, void* stream)
{
    if (!d_grid || g_size < 2) return TCV_ERR_ARG;
    if (g_size % 2) return TCV_ERR_UNSUPPORTED;  // as the reference (tMajorACC.cc:496-499)
    return fft_exec(reinterpret_cast<float2*>(d_grid), g_size, forward != 0, static_cast<cudaStream_t>(stream));
}

tcv_status tcv_fft_fix(float* d_grid, int64_t n, float scale, void* stream)
{
    if (!d_grid || n < 0) return TCV_ERR_ARG;
    if (n == 0) return TCV_OK;
    fix_kernel<<<grid_blocks(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(reinterpret_cast<float2*>(d_grid), n, scale);
    TCV_CUDA(cudaGetLastError());
    return TCV_OK;
}

tcv_status tcv_image_from_grid(float* d_grid, int g_size, float scale, float* d_image, void* stream)
{
    if (!d_grid || !d_image || g_size < 2) return TCV_ERR_ARG;
    if (g_size % 2) return TCV_ERR_UNSUPPORTED;
    return image_from_grid(reinterpret_cast<float2*>(d_grid), g_size, scale, d_image, nullptr,
                           static_cast<cudaStream_t>(stream));
}

tcv_status tcv_grid_from_image(const float* d_image, int g_size, float* d_grid, void* stream)
{
    if (!d_grid || !d_image || g_size < 2) return TCV_ERR_ARG;
    if (g_size % 2) return TCV_ERR_UNSUPPORTED;
    return grid_from_image(d_image, g_size, reinterpret_cast<float2*>(d_grid), static_cast<cudaStream_t>(stream));
}

}  // extern "C"
