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
// Power-of-two sizes 128 .. 8192 use this file's own transform, in three passes over the grid:
//   rows:    each CTA holds whole rows (4096 values, 256 threads; one row of 8192 with 512),
//            transforms them in shared memory and writes them to a scratch grid;
//   columns: the four-step split of a column of n = N1 N2 (y = N2 y1 + y2, k = k1 + N1 k2): a
//            CTA holds 16 adjacent columns (128-byte row segments) of the N1 rows of one y2,
//            takes their DFT_N1, multiplies by exp(-+2 pi i y2 k1 / n) and writes them back in
//            place; then a CTA holds the N2 contiguous rows of one k1 and writes DFT_N2 to rows
//            k1 + N1 k2 of the output.
// Each 1-D transform is the Stockham autosort form (Govindaraju et al., "High performance discrete
// Fourier transforms on graphics processors", SC 2008) with radix-16 stages (a 16-point DFT in
// registers as 4 x 4) and one radix-2, -4 or -8 stage for the rest of the exponent: a butterfly
// reads R values, multiplies value r by exp(-+2 pi i r (j mod Ns) / (Ns R)), takes the R-point
// DFT and writes the results Ns apart, so the output comes out in natural order.  The twiddles
// come from a table of exp(-2 pi i k / n) computed in double precision and rounded once: w, w^2,
// w^4, w^8 are read and the other powers formed as products.  The rotation and sign separate by
// axis, so the row pass applies the row's half (value p = (-1)^p Z[p + n/2]) and the last column
// pass the column's; the model step builds the complex rows from the float image in the row pass,
// and image formation writes the float image from the last column pass.  Other even sizes use
// cuFFT's single-precision C2C (the library the reference's own GPU path calls) with the fused
// passes below.
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
constexpr int kColW = 16;  // columns per column-pass CTA: 128-byte row segments
__host__ __device__ constexpr int fft_pad(int p) { return p + (p >> 4); }  // one slot in 16: fewer bank conflicts

__device__ __forceinline__ float2 cadd(const float2 a, const float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(const float2 a, const float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
// One fixed rounding sequence (explicit fused multiply-adds): every kernel that multiplies the same
// values gets the same bits, whatever the compiler would contract in its context.
__device__ __forceinline__ float2 cmul(const float2 a, const float2 w)
{
    return make_float2(__fmaf_rn(a.x, w.x, -__fmul_rn(a.y, w.y)), __fmaf_rn(a.x, w.y, __fmul_rn(a.y, w.x)));
}
// a * (-i) forward, a * (+i) inverse: exact
template <bool kInverse>
__device__ __forceinline__ float2 mul_mi(const float2 a) { return kInverse ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x); }
template <bool kInverse>
__device__ __forceinline__ float2 conj_if(const float2 w) { return kInverse ? make_float2(w.x, -w.y) : w; }

// 4-point DFT in place (natural order in and out)
template <bool kInverse>
__device__ __forceinline__ void dft4(float2& a, float2& b, float2& c, float2& d)
{
    const float2 t0 = cadd(a, c), t1 = csub(a, c), t2 = cadd(b, d), t3 = mul_mi<kInverse>(csub(b, d));
    a = cadd(t0, t2);
    b = cadd(t1, t3);
    c = csub(t0, t2);
    d = csub(t1, t3);
}

// exp(-+2 pi i m / 16) for the products i * k1 of the 4 x 4 split (m in 1, 2, 3, 6, 9)
__device__ __forceinline__ float2 w16(int m, bool inv)
{
    const float c1 = 0.92387953251128676f, s1 = 0.38268343236508977f, r = 0.70710678118654752f;
    float2 w;
    switch (m) {
        case 1: w = make_float2(c1, -s1); break;
        case 2: w = make_float2(r, -r); break;
        case 3: w = make_float2(s1, -c1); break;
        case 6: w = make_float2(-r, -r); break;
        default: w = make_float2(-c1, s1); break;  // 9
    }
    return inv ? make_float2(w.x, -w.y) : w;
}

// R-point DFT (R = 2, 4, 8, 16) of v[0..R-1] in place, natural order in and out.  R = 8 and 16
// split as 2 x 4 and 4 x 4 (x[i + S n1]: DFT4 over n1, twiddle, DFT over i, outputs transposed).
template <int R, bool kInverse>
__device__ __forceinline__ void dft(float2 (&v)[R])
{
    if constexpr (R == 2) {
        const float2 a = v[0];
        v[0] = cadd(a, v[1]);
        v[1] = csub(a, v[1]);
    } else if constexpr (R == 4) {
        dft4<kInverse>(v[0], v[1], v[2], v[3]);
    } else if constexpr (R == 8) {
        dft4<kInverse>(v[0], v[2], v[4], v[6]);  // i = 0: u[0][k1] at v[2 k1]
        dft4<kInverse>(v[1], v[3], v[5], v[7]);  // i = 1: u[1][k1] at v[2 k1 + 1]
        const float r = 0.70710678118654752f;
        v[3] = cmul(v[3], kInverse ? make_float2(r, r) : make_float2(r, -r));    // * w8^1
        v[5] = mul_mi<kInverse>(v[5]);                                           // * w8^2
        v[7] = cmul(v[7], kInverse ? make_float2(-r, r) : make_float2(-r, -r));  // * w8^3
        float2 o[8];
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1) {  // X[k1] = u0 + u1, X[k1 + 4] = u0 - u1
            o[k1] = cadd(v[2 * k1], v[2 * k1 + 1]);
            o[k1 + 4] = csub(v[2 * k1], v[2 * k1 + 1]);
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] = o[k];
    } else {
#pragma unroll
        for (int i = 0; i < 4; ++i) dft4<kInverse>(v[i], v[i + 4], v[i + 8], v[i + 12]);  // u[i][k1] at v[i + 4 k1]
#pragma unroll
        for (int i = 1; i < 4; ++i)
#pragma unroll
            for (int k1 = 1; k1 < 4; ++k1) {
                const int m = i * k1;
                v[i + 4 * k1] = m == 4 ? mul_mi<kInverse>(v[i + 4 * k1]) : cmul(v[i + 4 * k1], w16(m, kInverse));
            }
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1) dft4<kInverse>(v[4 * k1], v[4 * k1 + 1], v[4 * k1 + 2], v[4 * k1 + 3]);
        float2 o[16];
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1)
#pragma unroll
            for (int k2 = 0; k2 < 4; ++k2) o[k1 + 4 * k2] = v[4 * k1 + k2];
#pragma unroll
        for (int k = 0; k < 16; ++k) v[k] = o[k];
    }
}

// One radix-R Stockham stage over `lines` lines of length 2^log2n held in shared memory (line
// l at l << log2n, padded), in place: every butterfly reads R values Nl/R apart, multiplies
// value r by exp(-+2 pi i r (j mod Ns) / (Ns R)), takes the R-point DFT and writes the results
// Ns apart (Govindaraju et al., SC 2008); reads finish before a barrier, writes after it.
// Butterfly b of the CTA: line b / (N / R), index j = b mod (N / R); this thread takes b = tid +
// k * nthreads.  tw: exp(-2 pi i m / Ntab) for m < Ntab, read at m * (Ntab / N).
// Shared-memory place of value i of line l: kLines == 0, lines one after another (padded: the row
// pass); kLines > 0, kLines lines interleaved value by value ([i][l], the column passes: a
// half-warp's 16 lines of one position are one 128-byte row).
template <int kLines>
__device__ __forceinline__ int fft_at(int l, int i, int log2n)
{
    return kLines ? i * kLines + l : fft_pad((l << log2n) + i);
}

template <int R, bool kInverse, int kPer, int kLines, bool kSrcSm, bool kDstSm, class Load, class Store>
__device__ __forceinline__ void stage(float2* sm, int log2n, int log_ns, const float2* __restrict__ tw, int log_tab,
                                      Load load, Store store)
{
    constexpr int kLogR = R == 2 ? 1 : R == 4 ? 2 : R == 8 ? 3 : 4;
    const int lq = log2n - kLogR;  // log2 butterflies per line
    const int ns = 1 << log_ns;
    const int tscale = log_tab - log2n;  // table index = m << tscale
    float2 v[kPer][R];
    int dst[kPer], dl[kPer];
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        const int b = int(threadIdx.x) + k * int(blockDim.x);
        // butterfly b: line and index in line (interleaved lines: the line varies fastest)
        const int l = kLines ? b % kLines : b >> lq, j = kLines ? b / kLines : b & ((1 << lq) - 1);
        const int kk = j & (ns - 1);
#pragma unroll
        for (int r = 0; r < R; ++r)
            v[k][r] = kSrcSm ? sm[fft_at<kLines>(l, j + (r << lq), log2n)] : load(l, j + (r << lq));
        if (log_ns > 0) {
            // twiddles w^r, w = exp(-+2 pi i kk / (Ns R)): r = 1, 2, 4, 8 from the table, the rest as products
            const int t = kk << (log2n - log_ns - kLogR + tscale);
            float2 w[R];
            w[1] = conj_if<kInverse>(__ldg(tw + t));
            if (R > 2) {
                w[2] = conj_if<kInverse>(__ldg(tw + 2 * t));
                w[3] = cmul(w[1], w[2]);
            }
            if (R > 4) {
                w[4] = conj_if<kInverse>(__ldg(tw + 4 * t));
                w[5] = cmul(w[1], w[4]);
                w[6] = cmul(w[2], w[4]);
                w[7] = cmul(w[3], w[4]);
            }
            if (R > 8) {
                w[8] = conj_if<kInverse>(__ldg(tw + 8 * t));
#pragma unroll
                for (int r = 9; r < R; ++r) w[r] = cmul(w[r - 8], w[8]);
            }
#pragma unroll
            for (int r = 1; r < R; ++r) v[k][r] = cmul(v[k][r], w[r]);
        }
        dft<R, kInverse>(v[k]);
        dst[k] = ((j >> log_ns) << (log_ns + kLogR)) + kk;
        dl[k] = l;
    }
    // in place (shared memory, or a lone stage reading and writing the same grid rows): every value
    // of the stage is read before any is written
    if (kSrcSm == kDstSm) __syncthreads();
#pragma unroll
    for (int k = 0; k < kPer; ++k)
#pragma unroll
        for (int r = 0; r < R; ++r) {
            if (kDstSm)
                sm[fft_at<kLines>(dl[k], dst[k] + r * ns, log2n)] = v[k][r];
            else
                store(dl[k], dst[k] + r * ns, v[k][r]);
        }
    if (kDstSm) __syncthreads();
}

// All stages for the CTA's lines of 2^kLog (blockDim.x = lines * 2^kLog / 16 threads): radix-16
// stages, then one radix-2, -4 or -8 stage for the rest of the exponent, scheduled at compile time.
// The first stage reads its values with load(line, index) straight from global memory and the last
// writes them with store(line, index, value) (natural order): shared memory holds the values
// between stages only.
template <bool kInverse, int kLines, int kLog, int kStage = 0, class Load, class Store>
__device__ __forceinline__ void fft_lines(float2* sm, const float2* __restrict__ tw, int log_tab, Load& load,
                                          Store& store)
{
    constexpr int kA = kLog / 4, kRem = kLog % 4, kStages = kA + (kRem ? 1 : 0);
    if constexpr (kStage < kStages) {
        constexpr int R = kStage < kA ? 16 : (1 << kRem);
        constexpr bool kFirst = kStage == 0, kLast = kStage == kStages - 1;
        stage<R, kInverse, 16 / R, kLines, !kFirst, !kLast>(sm, kLog, 4 * kStage, tw, log_tab, load, store);
        fft_lines<kInverse, kLines, kLog, kStage + 1>(sm, tw, log_tab, load, store);
    }
}

// how the passes read and write
enum { kFftInGrid = 0, kFftInImage = 1 };                          // row pass input
enum { kFftOutGrid = 0, kFftOutRotated = 1, kFftOutImage = 2 };    // last pass output

// Row pass: CTA b holds rows b L .. b L + L - 1 (L = max(1, 4096 / n); n / 16 threads per row)
// and writes their transforms to dst.  Input: src (the grid) or the float image rotated by n/2 in
// both axes and signed, (-1)^(x+y) image[y + n/2][x + n/2].  With kRot the row's half of the
// fftshift and sign is applied on the way out: value p = (-1)^p Z[p + n/2].
template <bool kInverse, int kIn, bool kRot, int kThreads, int kLog>
__global__ void __launch_bounds__(kThreads, kThreads <= 256 ? 4 : 1)
fft_rows_kernel(const float2* __restrict__ src, const float* __restrict__ image, float2* __restrict__ dst,
                const float2* __restrict__ tw)
{
    extern __shared__ float2 fsm[];
    constexpr int log2n = kLog, n = 1 << log2n, h = n >> 1, mask = n - 1;
    const int total = int(blockDim.x) * 16;  // values held by the CTA: 16 per thread
    const int y0 = int(blockIdx.x) * (total >> log2n);
    const size_t row0 = (size_t)y0 * n;     // the CTA's rows are contiguous: value (l, i) at row0 + (l << log2n) + i
    auto load = [&](int l, int i) -> float2 {
        if (kIn == kFftInImage) {
            const int y = y0 + l;
            return make_float2(chk(i, y) * image[(size_t)((y + h) & mask) * n + ((i + h) & mask)], 0.f);
        }
        return src[row0 + ((size_t)l << log2n) + i];
    };
    auto store = [&](int l, int i, float2 v) {
        if (kRot) {  // Z[i] lands at p = i - n/2, signed (-1)^p = (-1)^i
            if (i & 1) v = make_float2(-v.x, -v.y);
            i = (i + h) & mask;
        }
        dst[row0 + ((size_t)l << log2n) + i] = v;
    };
    fft_lines<kInverse, 0, kLog>(fsm, tw, log2n, load, store);
}

// Column transforms of length n = N1 N2 in two passes (the four-step split, y = N2 y1 + y2,
// k = k1 + N1 k2), each CTA holding kColW adjacent columns (128-byte row segments):
//   first:  for one y2, the rows N2 y1 + y2: A[k1] = exp(-+2 pi i y2 k1 / n) * DFT_N1 over y1,
//           written back over the same rows (row N2 k1 + y2), in place in buf;
//   second: for one k1, the rows N2 k1 + y2 (contiguous): X[k1 + N1 k2] = DFT_N2 over y2, written
//           to row k1 + N1 k2 of the output -- as is, or with the column's half of the fftshift
//           and sign (row p = (-1)^p X[p + n/2]), or as the float image Re(.) * scale.
template <bool kInverse, int kLogL>
__global__ void __launch_bounds__(128, 4)
fft_cols1_kernel(float2* __restrict__ buf, int log2n, const float2* __restrict__ tw)
{
    constexpr int log_n1 = kLogL;
    extern __shared__ float2 fsm[];
    const int n = 1 << log2n, n2 = n >> log_n1;
    const int x0 = int(blockIdx.x) * kColW, y2 = int(blockIdx.y);
    // line l = column x0 + l; value i = row n2 i + y2; every read precedes the first write (stage 1)
    auto load = [&](int l, int i) -> float2 { return buf[(size_t)(n2 * i + y2) * n + x0 + l]; };
    auto store = [&](int l, int k1, float2 v) {
        const float2 w = conj_if<kInverse>(__ldg(tw + ((y2 * k1) & (n - 1))));
        buf[(size_t)(n2 * k1 + y2) * n + x0 + l] = cmul(v, w);
    };
    fft_lines<kInverse, kColW, kLogL>(fsm, tw, log2n, load, store);
}

template <bool kInverse, int kOut, int kLogL>
__global__ void __launch_bounds__(128, 4)
fft_cols2_kernel(const float2* __restrict__ buf, float2* __restrict__ out, float* __restrict__ image,
                 float2* __restrict__ image_c, float scale, int log2n, const float2* __restrict__ tw)
{
    extern __shared__ float2 fsm[];
    const int log_n1 = log2n - kLogL;
    const int n = 1 << log2n, n1 = 1 << log_n1, n2 = n >> log_n1, h = n >> 1, mask = n - 1;
    const int x0 = int(blockIdx.x) * kColW, k1 = int(blockIdx.y);
    auto load = [&](int l, int i) -> float2 { return buf[(size_t)(n2 * k1 + i) * n + x0 + l]; };
    auto store = [&](int l, int k2, float2 z) {
        const int k = k1 + n1 * k2, x = x0 + l;
        if (kOut == kFftOutGrid) {
            out[(size_t)k * n + x] = z;
        } else {
            const int p = (k - h) & mask;  // X[k] lands at row p, signed (-1)^p = (-1)^k
            const float sg = (k & 1) ? -1.f : 1.f;
            const size_t o = (size_t)p * n + x;
            if (kOut == kFftOutRotated) {
                out[o] = make_float2(sg * z.x, sg * z.y);
            } else {
                const float v = __fmul_rn(sg * z.x, scale);
                if (image) image[o] = v;
                if (image_c) image_c[o] = make_float2(v, 0.f);
            }
        }
    };
    fft_lines<kInverse, kColW, kLogL>(fsm, tw, log2n, load, store);
}

struct FftRes {
    int device, n;
    float2* tw;       // exp(-2 pi i k / n), k < n
    float2* scratch;  // n x n complex: the row pass's output, transformed in place by the first column pass
};
std::vector<FftRes> g_fft_res;  // guarded by g_fft_mu

bool own_fft(int n) { return n >= kFftMinN && n <= kFftMaxN && (n & (n - 1)) == 0; }

int ilog2(int n)
{
    int l = 0;
    while ((1 << l) < n) ++l;
    return l;
}

// The twiddle table and scratch grid of size n on the current device: the twiddles computed in
// double precision and rounded once; made at the first use of the size on the device (set-up:
// allocates and copies synchronously).
tcv_status fft_resources(int n, FftRes* out)
{
    std::lock_guard<std::mutex> lock(g_fft_mu);
    int dev = 0;
    TCV_CUDA(cudaGetDevice(&dev));
    for (const FftRes& r : g_fft_res)
        if (r.device == dev && r.n == n) {
            *out = r;
            return TCV_OK;
        }
    std::vector<float2> h(static_cast<size_t>(n));
    const double pi = 3.14159265358979323846;
    for (int k = 0; k < n; ++k) {
        const double a = 2.0 * pi * double(k) / double(n);
        h[size_t(k)] = make_float2(float(std::cos(a)), float(-std::sin(a)));
    }
    FftRes r{dev, n, nullptr, nullptr};
    TCV_CUDA(cudaMalloc(&r.tw, size_t(n) * sizeof(float2)));
    cudaError_t e = cudaMalloc(&r.scratch, size_t(n) * size_t(n) * sizeof(float2));
    if (e == cudaSuccess) e = cudaMemcpy(r.tw, h.data(), size_t(n) * sizeof(float2), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(r.tw);
        if (r.scratch) cudaFree(r.scratch);
        return cuda_status(e);
    }
    g_fft_res.push_back(r);
    *out = r;
    return TCV_OK;
}

template <typename K>
tcv_status launch_fft(K kernel, dim3 grid, int threads, size_t smem, void** args, cudaStream_t st)
{
    const void* f = reinterpret_cast<const void*>(kernel);
    if (smem > 48 * 1024) TCV_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    TCV_CUDA(cudaLaunchKernel(f, grid, dim3(threads), args, smem, st));
    return TCV_OK;
}

// Row pass of size 2^kLog: the kernel for the direction, input and output kinds.
template <int kLog>
tcv_status launch_rows(bool forward, int in_kind, bool rot, const float2* grid, const float* image_in, float2* sc,
                       const float2* tw, cudaStream_t st)
{
    constexpr int n = 1 << kLog, kThreads = n >= 4096 ? n / 16 : 256;
    const unsigned ctas = unsigned(size_t(n) * size_t(n) / (size_t(kThreads) * 16));
    const size_t smem = size_t(fft_pad(kThreads * 16)) * sizeof(float2);
    void* args[] = {const_cast<const float2**>(&grid), const_cast<const float**>(&image_in), &sc,
                    const_cast<const float2**>(&tw)};
    const dim3 g(ctas);
    if (!forward)
        return rot ? launch_fft(&fft_rows_kernel<true, kFftInGrid, true, kThreads, kLog>, g, kThreads, smem, args, st)
                   : launch_fft(&fft_rows_kernel<true, kFftInGrid, false, kThreads, kLog>, g, kThreads, smem, args, st);
    if (in_kind == kFftInImage)
        return launch_fft(&fft_rows_kernel<false, kFftInImage, false, kThreads, kLog>, g, kThreads, smem, args, st);
    return rot ? launch_fft(&fft_rows_kernel<false, kFftInGrid, true, kThreads, kLog>, g, kThreads, smem, args, st)
               : launch_fft(&fft_rows_kernel<false, kFftInGrid, false, kThreads, kLog>, g, kThreads, smem, args, st);
}

// The two column passes of size 2^kLog: N1 = 2^(kLog / 2), N2 = 2^kLog / N1.
template <int kLog>
tcv_status launch_cols(bool forward, int out_kind, float2* sc, float2* grid, float* image_out, float2* image_c,
                       float scale, const float2* tw, cudaStream_t st)
{
    constexpr int n = 1 << kLog, kL1 = kLog / 2, kL2 = kLog - kL1;
    int log2n = kLog;
    {
        constexpr int threads = kColW * (1 << kL1) / 16;
        const size_t smem = size_t(kColW << kL1) * sizeof(float2);
        void* args[] = {&sc, &log2n, const_cast<const float2**>(&tw)};
        const dim3 g(unsigned(n / kColW), unsigned(1 << kL2));
        TCV_CHECK(forward ? launch_fft(&fft_cols1_kernel<false, kL1>, g, threads, smem, args, st)
                          : launch_fft(&fft_cols1_kernel<true, kL1>, g, threads, smem, args, st));
    }
    constexpr int threads = kColW * (1 << kL2) / 16;
    const size_t smem = size_t(kColW << kL2) * sizeof(float2);
    const float2* csc = sc;
    void* args[] = {const_cast<const float2**>(&csc), &grid, &image_out, &image_c, &scale, &log2n,
                    const_cast<const float2**>(&tw)};
    const dim3 g(unsigned(n / kColW), unsigned(1 << kL1));
    if (out_kind == kFftOutImage)
        return forward ? launch_fft(&fft_cols2_kernel<false, kFftOutImage, kL2>, g, threads, smem, args, st)
                       : launch_fft(&fft_cols2_kernel<true, kFftOutImage, kL2>, g, threads, smem, args, st);
    if (out_kind == kFftOutRotated)
        return forward ? launch_fft(&fft_cols2_kernel<false, kFftOutRotated, kL2>, g, threads, smem, args, st)
                       : launch_fft(&fft_cols2_kernel<true, kFftOutRotated, kL2>, g, threads, smem, args, st);
    return forward ? launch_fft(&fft_cols2_kernel<false, kFftOutGrid, kL2>, g, threads, smem, args, st)
                   : launch_fft(&fft_cols2_kernel<true, kFftOutGrid, kL2>, g, threads, smem, args, st);
}

template <int kLog>
tcv_status own_passes(float2* grid, const float* image_in, float* image_out, float2* image_c, float scale,
                      bool forward, int in_kind, int out_kind, const FftRes& res, cudaStream_t st)
{
    TCV_CHECK(launch_rows<kLog>(forward, in_kind, out_kind != kFftOutGrid, grid, image_in, res.scratch, res.tw, st));
    return launch_cols<kLog>(forward, out_kind, res.scratch, grid, image_out, image_c, scale, res.tw, st);
}

// The three passes of the own transform: rows (grid or rotated signed image -> scratch, with the
// row half of the rotation when the output is rotated or an image), columns in place in the
// scratch, columns from the scratch into the grid (as is, rotated and signed) or the float image.
tcv_status own_transform(float2* grid, const float* image_in, float* image_out, float2* image_c, float scale, int n,
                         bool forward, int in_kind, int out_kind, cudaStream_t st)
{
    FftRes res{};
    TCV_CHECK(fft_resources(n, &res));
    switch (ilog2(n)) {
        case 7: return own_passes<7>(grid, image_in, image_out, image_c, scale, forward, in_kind, out_kind, res, st);
        case 8: return own_passes<8>(grid, image_in, image_out, image_c, scale, forward, in_kind, out_kind, res, st);
        case 9: return own_passes<9>(grid, image_in, image_out, image_c, scale, forward, in_kind, out_kind, res, st);
        case 10: return own_passes<10>(grid, image_in, image_out, image_c, scale, forward, in_kind, out_kind, res, st);
        case 11: return own_passes<11>(grid, image_in, image_out, image_c, scale, forward, in_kind, out_kind, res, st);
        case 12: return own_passes<12>(grid, image_in, image_out, image_c, scale, forward, in_kind, out_kind, res, st);
        case 13: return own_passes<13>(grid, image_in, image_out, image_c, scale, forward, in_kind, out_kind, res, st);
        default: return TCV_ERR_UNSUPPORTED;
    }
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
    FftRes res{};
    return fft_resources(n, &res);
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
