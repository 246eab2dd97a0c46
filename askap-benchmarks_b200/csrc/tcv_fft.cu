// tcv_fft.cu -- the FFT steps either side of gridding and degridding in the imaging major cycle.
//
// Reference: current/tMajorACC/tMajorACC.cc:487-640.  fftExec / fftExecGPU rotate the grid by half
// its size in both axes (the fftshift, :514-525), run an unnormalised 2-D C2C transform (FFTW or
// cuFFT; FFTW_FORWARD / CUFFT_FORWARD = exp(-i..), BACKWARD / INVERSE = exp(+i..)) and rotate back
// (:530-541); fftFix / fftFixGPU keep the real part times a scale (:620-640).  Odd sizes are
// refused, as there (:496-499).
//
// B200 form.  The two rotations cost no pass of their own: for an even size N, with S the
// half-size rotation and D the checkerboard sign (-1)^(x+y), F S = D F and S F = F D, so
//     S F S X = S D F X:   Y[k] = (-1)^(kx+ky) Z[k + N/2],  Z = F X      (fftExec in place)
//     S F S X = F D S X:   transform of (-1)^(x+y) X[x + N/2]             (from a real model image)
// Signs are exact, so only the transform rounds.
//
// Power-of-two sizes 128 .. 8192 use this file's own transform: two passes over the grid, each a
// set of 1-D transforms held in shared memory (4096 complex values and 256 threads per CTA, four
// CTAs per SM; 8192 and 512 for the 8192 size): first
// the rows, then the columns.  Each 1-D transform is the Stockham autosort form of the radix-4
// (and one radix-2) decimation (Govindaraju et al., "High performance discrete Fourier transforms
// on graphics processors", SC 2008): every stage reads R values per butterfly, multiplies by the
// twiddles exp(-+2 pi i r (j mod Ns) / (Ns R)), takes the R-point DFT and writes the results
// Ns apart, so the output comes out in natural order; each stage reads all its values before a
// barrier and writes after it, so one buffer serves in place.  Twiddles come from a table of
// exp(-2 pi i k / N) computed in double precision and rounded once.  The rotation and sign
// separate by axis, so each pass applies its own axis's half (a line's values only move within
// the line); the model step builds the complex rows from the float image in the row pass, and
// image formation writes the float image from the column pass (no complex write-back).  Other
// even sizes use cuFFT's single-precision C2C (the library the reference's own GPU path calls)
// with the fused passes below.
#include "tcv_internal.cuh"

#include <cufft.h>

#include <cmath>
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

// ------------------------------------------------------------------------------------------
// Hand-written transform (power-of-two sizes)
// ------------------------------------------------------------------------------------------
constexpr int kFftMinN = 128, kFftMaxN = 8192;
__host__ __device__ constexpr int fft_pad(int p) { return p + (p >> 4); }  // one slot in 16: fewer bank conflicts

// how a pass reads its lines and what it does with the transformed values
enum { kFftInGrid = 0, kFftInImage = 1 };                          // input: the grid, or the rotated signed image
enum { kFftOutGrid = 0, kFftOutRotated = 1, kFftOutImage = 2 };    // output: as is, rotated and signed, or the float image

// A CTA holds 2^kLog complex values (whole lines, twice: the stages go from one buffer to the
// other) and runs kThreads threads; kMinBlocks CTAs fit an SM, so that one CTA's loads and stores
// overlap another's transforms.
template <int kLog, int kThreads>
struct FftShape {
    static constexpr int kElems = 1 << kLog;
    static constexpr int kPer = kElems / kThreads;  // values a thread loads and stores
    static constexpr int kBatch = kPer < 8 ? kPer : 8;  // loads in flight per thread
    static constexpr int kMinBlocks = kThreads <= 256 ? 3 : 1;
    static constexpr size_t kSmem = 2 * size_t(fft_pad(kElems)) * sizeof(float2);  // two buffers
};

__device__ __forceinline__ float2 cmul(const float2 a, const float2 w)
{
    return make_float2(a.x * w.x - a.y * w.y, a.x * w.y + a.y * w.x);
}

// One radix-R Stockham stage over the CTA's values (lines of n, natural order), from src into dst
// (two shared-memory buffers: a butterfly writes as soon as it has read, so it holds only its own
// R values in registers, and a stage costs one barrier).
template <int R, bool kInverse, int kElems, int kThreads>
__device__ __forceinline__ void fft_stage(const float2* src, float2* dst, int log2n, int log_ns,
                                          const float2* __restrict__ tw)
{
    constexpr int kLogR = R == 4 ? 2 : 1;
    constexpr int kPer = kElems / R / kThreads;  // butterflies per thread
    const int ns = 1 << log_ns;
    const int lq = log2n - kLogR;                 // log2 of butterflies per line
#pragma unroll 2
    for (int k = 0; k < kPer; ++k) {
        const int b = int(threadIdx.x) + k * kThreads;
        const int l = b >> lq, j = b & ((1 << lq) - 1);
        const int base = l << log2n;
        const int kk = j & (ns - 1);
        const int step = kk << (log2n - log_ns - kLogR);  // twiddle index r * kk * n / (ns R)
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            float2 x = src[fft_pad(base + j + (r << lq))];
            if (r > 0) {
                float2 w = __ldg(tw + r * step);
                if (kInverse) w.y = -w.y;
                x = cmul(x, w);
            }
            v[r] = x;
        }
        if (R == 2) {
            const float2 a = v[0], c = v[1];
            v[0] = make_float2(a.x + c.x, a.y + c.y);
            v[1] = make_float2(a.x - c.x, a.y - c.y);
        } else {
            const float2 a0 = make_float2(v[0].x + v[2].x, v[0].y + v[2].y);
            const float2 a1 = make_float2(v[0].x - v[2].x, v[0].y - v[2].y);
            const float2 a2 = make_float2(v[1].x + v[3].x, v[1].y + v[3].y);
            const float2 d = make_float2(v[1].x - v[3].x, v[1].y - v[3].y);
            // (v1 - v3) * -i (forward) or * +i (inverse)
            const float2 a3 = kInverse ? make_float2(-d.y, d.x) : make_float2(d.y, -d.x);
            v[0] = make_float2(a0.x + a2.x, a0.y + a2.y);
            v[1] = make_float2(a1.x + a3.x, a1.y + a3.y);
            v[2] = make_float2(a0.x - a2.x, a0.y - a2.y);
            v[3] = make_float2(a1.x - a3.x, a1.y - a3.y);
        }
        const int o = base + ((j >> log_ns) << (log_ns + kLogR)) + kk;
#pragma unroll
        for (int r = 0; r < R; ++r) dst[fft_pad(o + r * ns)] = v[r];
    }
    __syncthreads();
}

// All stages of the CTA's lines; the values start in buf[0] and the function returns the buffer
// that holds the transform.
template <bool kInverse, int kElems, int kThreads>
__device__ __forceinline__ float2* fft_lines(float2* buf0, float2* buf1, int log2n, const float2* __restrict__ tw)
{
    float2 *a = buf0, *b = buf1;
    int log_ns = 0;
    if (log2n & 1) {
        fft_stage<2, kInverse, kElems, kThreads>(a, b, log2n, 0, tw);
        float2* t = a;
        a = b;
        b = t;
        log_ns = 1;
    }
    for (; log_ns < log2n; log_ns += 2) {
        fft_stage<4, kInverse, kElems, kThreads>(a, b, log2n, log_ns, tw);
        float2* t = a;
        a = b;
        b = t;
    }
    return a;
}

// One pass of 1-D transforms over all lines of the grid, 2^kLog / n lines per CTA: the rows
// (kCols false; CTA b holds rows b L .. b L + L - 1) or the columns (CTA b holds columns
// b L .. b L + L - 1).  The fftshift and checkerboard sign separate by axis,
// (-1)^(x+y) Z[y+h][x+h] = S_y D_y F_y S_x D_x F_x X, so a pass whose output is rotated writes
// value k of a line as (-1)^k times value k + n/2 of its transform: only the line's own values
// move, and the pass works in place.  Loads and stores go through registers, kBatch in flight.
template <int kLog, int kThreads, bool kCols, bool kInverse, int kIn, int kOut>
__global__ void __launch_bounds__(kThreads, FftShape<kLog, kThreads>::kMinBlocks)
fft_pass_kernel(float2* __restrict__ grid, const float* __restrict__ image, float* __restrict__ image_out,
                float2* __restrict__ image_c, float scale, int log2n, const float2* __restrict__ tw)
{
    using S = FftShape<kLog, kThreads>;
    extern __shared__ float2 fsm[];
    const int n = 1 << log2n, h = n >> 1, mask = n - 1;
    const int log_l = kLog - log2n;  // lines per CTA = 2^log_l
    const int lmask = (1 << log_l) - 1;
    const int first = int(blockIdx.x) << log_l;
    auto line_of = [&](int idx) { return kCols ? (idx & lmask) : (idx >> log2n); };
    auto pos_of = [&](int idx) { return kCols ? (idx >> log_l) : (idx & mask); };
    auto gaddr = [&](int line, int pos) {
        return kCols ? (size_t)pos * n + (first + line) : (size_t)(first + line) * n + pos;
    };
#pragma unroll
    for (int b0 = 0; b0 < S::kPer; b0 += S::kBatch) {
        float2 v[S::kBatch];
#pragma unroll
        for (int e = 0; e < S::kBatch; ++e) {
            const int idx = int(threadIdx.x) + (b0 + e) * kThreads;
            const int line = line_of(idx), pos = pos_of(idx);
            if (kIn == kFftInImage) {  // rows only: (-1)^(x+y) image[y + h][x + h], as complex
                const int y = first + line;
                v[e] = make_float2(chk(pos, y) * image[(size_t)((y + h) & mask) * n + ((pos + h) & mask)], 0.f);
            } else {
                v[e] = grid[gaddr(line, pos)];
            }
        }
#pragma unroll
        for (int e = 0; e < S::kBatch; ++e) {
            const int idx = int(threadIdx.x) + (b0 + e) * kThreads;
            fsm[fft_pad((line_of(idx) << log2n) + pos_of(idx))] = v[e];
        }
    }
    __syncthreads();
    const float2* res = fft_lines<kInverse, S::kElems, kThreads>(fsm, fsm + fft_pad(S::kElems), log2n, tw);
#pragma unroll
    for (int b0 = 0; b0 < S::kPer; b0 += S::kBatch) {
        float2 v[S::kBatch];
#pragma unroll
        for (int e = 0; e < S::kBatch; ++e) {
            const int idx = int(threadIdx.x) + (b0 + e) * kThreads;
            const int line = line_of(idx), pos = pos_of(idx);
            if (kOut == kFftOutGrid) {
                v[e] = res[fft_pad((line << log2n) + pos)];
            } else {
                const float2 z = res[fft_pad((line << log2n) + ((pos + h) & mask))];
                const float sg = (pos & 1) ? -1.f : 1.f;
                v[e] = make_float2(sg * z.x, sg * z.y);
            }
        }
#pragma unroll
        for (int e = 0; e < S::kBatch; ++e) {
            const int idx = int(threadIdx.x) + (b0 + e) * kThreads;
            const size_t o = gaddr(line_of(idx), pos_of(idx));
            if (kOut == kFftOutImage) {
                const float r = __fmul_rn(v[e].x, scale);
                if (image_out) image_out[o] = r;
                if (image_c) image_c[o] = make_float2(r, 0.f);
            } else {
                grid[o] = v[e];
            }
        }
    }
}

struct Twiddles {
    int device, n;
    float2* d;
};
std::vector<Twiddles> g_twiddles;  // guarded by g_fft_mu

bool own_fft(int n) { return n >= kFftMinN && n <= kFftMaxN && (n & (n - 1)) == 0; }

int ilog2(int n)
{
    int l = 0;
    while ((1 << l) < n) ++l;
    return l;
}

// exp(-2 pi i k / n), k < n, on the current device: computed in double, rounded once, made at the
// first use of the size on the device (set-up: allocates and copies synchronously)
tcv_status twiddles_for(int n, const float2** out)
{
    std::lock_guard<std::mutex> lock(g_fft_mu);
    int dev = 0;
    TCV_CUDA(cudaGetDevice(&dev));
    for (const Twiddles& t : g_twiddles)
        if (t.device == dev && t.n == n) {
            *out = t.d;
            return TCV_OK;
        }
    std::vector<float2> h(static_cast<size_t>(n));
    const double pi = 3.14159265358979323846;
    for (int k = 0; k < n; ++k) {
        const double a = 2.0 * pi * double(k) / double(n);
        h[size_t(k)] = make_float2(float(std::cos(a)), float(-std::sin(a)));
    }
    float2* d = nullptr;
    TCV_CUDA(cudaMalloc(&d, size_t(n) * sizeof(float2)));
    const cudaError_t e = cudaMemcpy(d, h.data(), size_t(n) * sizeof(float2), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(d);
        return cuda_status(e);
    }
    g_twiddles.push_back(Twiddles{dev, n, d});
    *out = d;
    return TCV_OK;
}

template <typename K>
tcv_status launch_fft_kernel(K kernel, unsigned ctas, int threads, size_t smem, void** args, cudaStream_t st)
{
    const void* f = reinterpret_cast<const void*>(kernel);
    TCV_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    TCV_CUDA(cudaLaunchKernel(f, dim3(ctas), dim3(threads), args, smem, st));
    return TCV_OK;
}

// Both passes of the own transform with CTAs of 2^kLog values and kThreads threads: rows (from the
// grid, or from the float image rotated and signed), then columns (into the grid, or the float
// image).  fftExec's rotation and sign are applied per axis by each pass (kFftOutRotated); image
// formation's column pass writes the float image (Re times scale) after its rotation.
template <int kLog, int kThreads>
tcv_status own_passes(float2* grid, const float* image_in, float* image_out, float2* image_c, float scale, int n,
                      const float2* tw, bool forward, int in_kind, int out_kind, cudaStream_t st)
{
    using S = FftShape<kLog, kThreads>;
    int log2n = ilog2(n);
    const unsigned ctas = unsigned(size_t(n) * size_t(n) / S::kElems);
    void* args[] = {&grid, const_cast<const float**>(&image_in), &image_out, &image_c, &scale, &log2n,
                    const_cast<const float2**>(&tw)};
    auto go = [&](auto kernel) { return launch_fft_kernel(kernel, ctas, kThreads, S::kSmem, args, st); };
    const bool rot = out_kind != kFftOutGrid;  // rows rotate exactly when the output does
    if (!forward)
        TCV_CHECK(rot ? go(&fft_pass_kernel<kLog, kThreads, false, true, kFftInGrid, kFftOutRotated>)
                      : go(&fft_pass_kernel<kLog, kThreads, false, true, kFftInGrid, kFftOutGrid>));
    else if (in_kind == kFftInImage)
        TCV_CHECK(go(&fft_pass_kernel<kLog, kThreads, false, false, kFftInImage, kFftOutGrid>));
    else
        TCV_CHECK(rot ? go(&fft_pass_kernel<kLog, kThreads, false, false, kFftInGrid, kFftOutRotated>)
                      : go(&fft_pass_kernel<kLog, kThreads, false, false, kFftInGrid, kFftOutGrid>));
    if (out_kind == kFftOutImage)
        return forward ? go(&fft_pass_kernel<kLog, kThreads, true, false, kFftInGrid, kFftOutImage>)
                       : go(&fft_pass_kernel<kLog, kThreads, true, true, kFftInGrid, kFftOutImage>);
    if (out_kind == kFftOutRotated)
        return forward ? go(&fft_pass_kernel<kLog, kThreads, true, false, kFftInGrid, kFftOutRotated>)
                       : go(&fft_pass_kernel<kLog, kThreads, true, true, kFftInGrid, kFftOutRotated>);
    return forward ? go(&fft_pass_kernel<kLog, kThreads, true, false, kFftInGrid, kFftOutGrid>)
                   : go(&fft_pass_kernel<kLog, kThreads, true, true, kFftInGrid, kFftOutGrid>);
}

#ifndef TCV_FFT_SHAPE
#define TCV_FFT_SHAPE 0
#endif

tcv_status own_transform(float2* grid, const float* image_in, float* image_out, float2* image_c, float scale, int n,
                         bool forward, int in_kind, int out_kind, cudaStream_t st)
{
    const float2* tw = nullptr;
    TCV_CHECK(twiddles_for(n, &tw));
    // CTAs of 4096 values and 256 threads (four per SM) up to n = 4096; a line of 8192 needs 8192
#if TCV_FFT_SHAPE == 1
    return own_passes<13, 512>(grid, image_in, image_out, image_c, scale, n, tw, forward, in_kind, out_kind, st);
#elif TCV_FFT_SHAPE == 2
    if (n <= 4096)
        return own_passes<12, 512>(grid, image_in, image_out, image_c, scale, n, tw, forward, in_kind, out_kind, st);
    return own_passes<13, 512>(grid, image_in, image_out, image_c, scale, n, tw, forward, in_kind, out_kind, st);
#else
    if (n <= 4096)
        return own_passes<12, 256>(grid, image_in, image_out, image_c, scale, n, tw, forward, in_kind, out_kind, st);
    return own_passes<13, 512>(grid, image_in, image_out, image_c, scale, n, tw, forward, in_kind, out_kind, st);
#endif
}


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

tcv_status fft_prepare(int n)
{
    if (!own_fft(n)) return TCV_OK;
    const float2* tw = nullptr;
    return twiddles_for(n, &tw);
}

tcv_status fft_exec(float2* d_grid, int n, bool forward, cudaStream_t st)
{
    if (own_fft(n)) return own_transform(d_grid, nullptr, nullptr, nullptr, 1.f, n, forward, kFftInGrid, kFftOutRotated, st);
    TCV_CHECK(exec_c2c(d_grid, n, forward, st));
    swap_sign_kernel<<<grid_blocks((long long)(n / 2) * n), 256, 0, st>>>(d_grid, n);
    TCV_CUDA(cudaGetLastError());
    return TCV_OK;
}

tcv_status image_from_grid(float2* d_grid, int n, float scale, float* d_image, float2* d_image_c, cudaStream_t st)
{
    if (own_fft(n)) return own_transform(d_grid, nullptr, d_image, d_image_c, scale, n, false, kFftInGrid, kFftOutImage, st);
    TCV_CHECK(exec_c2c(d_grid, n, false, st));
    image_fix_kernel<<<grid_blocks((long long)n * n), 256, 0, st>>>(d_grid, n, scale, d_image, d_image_c);
    TCV_CUDA(cudaGetLastError());
    return TCV_OK;
}

tcv_status grid_from_image(const float* d_image, int n, float2* d_grid, cudaStream_t st)
{
    if (own_fft(n)) return own_transform(d_grid, d_image, nullptr, nullptr, 1.f, n, true, kFftInImage, kFftOutGrid, st);
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
