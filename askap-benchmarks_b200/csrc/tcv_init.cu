// tcv_init.cu -- device set-up of the tConvolve problem: sample coordinates, the W-projection
// table C, and per-sample grid/table offsets.  These are the untimed parts of Benchmark::init
// (attic/tConvolveMPI/Benchmark.cc:60-96, 206-324); every floating-point step uses the same
// IEEE operations in the same order as the reference so that the results agree with its CPU
// output (offsets bit for bit; the table up to the last-bit behaviour of the FP64 cos/exp).
#include "tcv_internal.cuh"

#include <cmath>
#include <climits>
#include <vector>

namespace tcv {
namespace {

constexpr double kMaxInt = 2147483647.0;

__device__ __forceinline__ double lcg_coord(uint64_t& state, double baseline, double half)
{
    // Benchmark::randomInt (Benchmark.cc:53-58), then baseline * r / maxint - baseline/2 (:72-74)
    state = state * kLcgA + kLcgC;
    const unsigned int r = (unsigned int)(state / 65536ull) % 2147483647u;
    return __dsub_rn(__ddiv_rn(__dmul_rn(baseline, (double)(int)r), kMaxInt), half);
}

__global__ void uvw_kernel(int64_t n, int baseline, uint64_t state0, double* u, double* v, double* w)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint64_t A, C;
    lcg_jump(3ull * (uint64_t)i, A, C);
    uint64_t s = A * state0 + C;
    const double b = (double)baseline, h = (double)(baseline / 2);
    u[i] = lcg_coord(s, b, h);
    v[i] = lcg_coord(s, b, h);
    w[i] = lcg_coord(s, b, h);
}

struct CParams {
    int s, os, w_size, c_center;
    double w_cell_size, freq0, cell_size;
    int64_t n;
};

// One thread per table entry: Benchmark.cc:236-258 in FP64, stored as float (imaginary part 0).
__global__ void init_c_kernel(CParams p, float2* c)
{
    const int64_t cind = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (cind >= p.n) return;
    int64_t t = cind;
    const int i = int(t % p.s); t /= p.s;
    const int j = int(t % p.s); t /= p.s;
    const int osi = int(t % p.os); t /= p.os;
    const int osj = int(t % p.os); t /= p.os;
    const int k = int(t);
    const double w = (double)(k - p.w_size / 2);
    const double f_scale = __ddiv_rn(sqrt(__dmul_rn(__dmul_rn(fabs(w), p.w_cell_size), p.freq0)), p.cell_size);
    const double os = (double)p.os;
    const double dj = __dadd_rn((double)(j - p.c_center), __ddiv_rn((double)osj, os));
    const double di = __dadd_rn((double)(i - p.c_center), __ddiv_rn((double)osi, os));
    const double r2 = __dadd_rn(__dmul_rn(dj, dj), __dmul_rn(di, di));
    double val;
    if (w != 0.0)
        val = cos(__ddiv_rn(r2, __dmul_rn(w, f_scale)));
    else
        val = exp(-r2);
    c[cind] = make_float2((float)val, 0.0f);
}

__device__ __forceinline__ float cabs_ref(float2 z)
{
    // std::abs(std::complex<float>) is hypotf(re, im); exact |re| when im == 0
    return z.y == 0.0f ? fabsf(z.x) : hypotf(z.x, z.y);
}

// The reference normalises with a sequential float sum of |C| over the flat table
// (Benchmark.cc:261-265).  The order of a float sum decides its value (it saturates at 2^24
// for the default 35 M entry table), so one thread adds the values in index order while the
// rest of the block stages the next chunk in shared memory.
constexpr int kSumChunk = 4096;
__global__ void __launch_bounds__(1024) sum_abs_seq_kernel(const float2* c, int64_t n, float* out)
{
    __shared__ float buf[2][kSumChunk];
    const int64_t nchunks = (n + kSumChunk - 1) / kSumChunk;
    for (int i = threadIdx.x; i < kSumChunk && i < n; i += blockDim.x) buf[0][i] = cabs_ref(c[i]);
    __syncthreads();
    float sum = 0.0f;
    for (int64_t ch = 0; ch < nchunks; ++ch) {
        const int cur = int(ch & 1);
        if (threadIdx.x >= 32) {
            const int64_t base = (ch + 1) * kSumChunk;
            for (int i = threadIdx.x - 32; i < kSumChunk && base + i < n; i += blockDim.x - 32)
                buf[cur ^ 1][i] = cabs_ref(c[base + i]);
        } else if (threadIdx.x == 0) {
            const int64_t base = ch * kSumChunk;
            const int len = int(n - base < kSumChunk ? n - base : kSumChunk);
            const float* b = buf[cur];
            for (int i = 0; i < len; ++i) sum = __fadd_rn(sum, b[i]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = sum;
}

// C *= float(wSize*os*os) / sumC, as a complex multiply by (scale, 0) (Benchmark.cc:267-269).
__global__ void scale_c_kernel(float2* c, int64_t n, float numer, const float* sum_c)
{
    const float scale = __fdiv_rn(numer, sum_c[0]);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float2 z = c[i];
        z.x = __fmul_rn(z.x, scale);
        z.y = __fmul_rn(z.y, scale);
        c[i] = z;
    }
}

struct OffParams {
    int64_t n_samples;
    int n_chan, w_size, g_size, s, os;
    double cell_size, w_cell_size;
};

// Benchmark.cc:293-323, one thread per (sample, channel).
__global__ void offsets_kernel(OffParams p, const double* u, const double* v, const double* w,
                               const double* freq, int32_t* iu_out, int32_t* iv_out, int32_t* co_out)
{
    const int64_t d = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (d >= p.n_samples * p.n_chan) return;
    const int64_t i = d / p.n_chan;
    const int chan = int(d % p.n_chan);
    const double f = freq[chan];
    const double os = (double)p.os;
    const double us = __ddiv_rn(__dmul_rn(f, u[i]), p.cell_size);
    int iu = (int)us;
    if (us < (double)iu) iu -= 1;
    const int fracu = (int)__dmul_rn(os, __dsub_rn(us, (double)iu));
    iu += p.g_size / 2;
    const double vs = __ddiv_rn(__dmul_rn(f, v[i]), p.cell_size);
    int iv = (int)vs;
    if (vs < (double)iv) iv -= 1;
    const int fracv = (int)__dmul_rn(os, __dsub_rn(vs, (double)iv));
    iv += p.g_size / 2;
    const double ws = __ddiv_rn(__dmul_rn(f, w[i]), p.w_cell_size);
    const int woff = p.w_size / 2 + (int)ws;
    iu_out[d] = iu;
    iv_out[d] = iv;
    co_out[d] = p.s * p.s * (fracu + p.os * (fracv + p.os * woff));
}

// ---- table storage conversions ----
__global__ void absmax_imag_kernel(const float2* c, int64_t n, unsigned int* absmax_bits,
                                   unsigned long long* imag_nonzero)
{
    float m = 0.f;
    unsigned long long nz = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float2 z = c[i];
        m = fmaxf(m, fmaxf(fabsf(z.x), fabsf(z.y)));
        nz += (z.y != 0.f);
    }
    for (int o = 16; o; o >>= 1) {
        m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
        nz += __shfl_xor_sync(0xffffffffu, nz, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(absmax_bits, __float_as_uint(m));  // non-negative floats order like their bits
        if (nz) atomicAdd(imag_nonzero, nz);
    }
}

__global__ void convert_kernel(const float2* c, int64_t n, int c_type, float pre_scale, void* out)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float2 z = c[i];
        switch (c_type) {
            case TCV_C_R32: static_cast<float*>(out)[i] = z.x; break;
            case TCV_C_CBF16: {
                const __nv_bfloat16 re = __float2bfloat16_rn(z.x), im = __float2bfloat16_rn(z.y);
                const uint32_t u = (uint32_t)__bfloat16_as_ushort(re) | ((uint32_t)__bfloat16_as_ushort(im) << 16);
                static_cast<uint32_t*>(out)[i] = u;
                break;
            }
            case TCV_C_RBF16: static_cast<__nv_bfloat16*>(out)[i] = __float2bfloat16_rn(z.x); break;
            case TCV_C_CF16:
                static_cast<__half2*>(out)[i] = __halves2half2(__float2half_rn(z.x * pre_scale), __float2half_rn(z.y * pre_scale));
                break;
            case TCV_C_RF16: static_cast<__half*>(out)[i] = __float2half_rn(z.x * pre_scale); break;
            default: break;
        }
    }
}

inline int grid_blocks(int64_t n, int threads)
{
    int64_t b = (n + threads - 1) / threads;
    return int(b > 148 * 64 ? 148 * 64 : (b < 1 ? 1 : b));
}

}  // namespace
}  // namespace tcv

using namespace tcv;

extern "C" {

tcv_status tcv_c_geometry(double freq0, double cell_size, int baseline, int w_size, int* support,
                          int* over_sample, double* w_cell_size, int64_t* c_len)
{
    if (!(cell_size > 0.0) || !(freq0 > 0.0) || w_size < 1) return TCV_ERR_ARG;
    // Benchmark.cc:212-217
    const int sup = static_cast<int>(1.5 * std::sqrt(double(std::abs(baseline)) * cell_size * freq0) / cell_size);
    const int os = 8;
    const double wcs = double(2 * baseline) * freq0 / double(w_size);
    const int64_t s = 2 * int64_t(sup) + 1;
    if (support) *support = sup;
    if (over_sample) *over_sample = os;
    if (w_cell_size) *w_cell_size = wcs;
    if (c_len) *c_len = s * s * os * os * w_size;
    return TCV_OK;
}

size_t tcv_init_c_scratch_bytes(void) { return 256; }

tcv_status tcv_init_c_raw(double freq0, double cell_size, int baseline, int w_size, float* d_c,
                          void* d_scratch, float* sum_c_out, void* stream)
{
    if (!d_c || !d_scratch) return TCV_ERR_ARG;
    int support, os;
    double wcs;
    int64_t n;
    tcv_status st = tcv_c_geometry(freq0, cell_size, baseline, w_size, &support, &os, &wcs, &n);
    if (st != TCV_OK) return st;
    if (n > INT_MAX) return TCV_ERR_UNSUPPORTED;  // cOffset is a 32-bit int in the reference
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    CParams p{2 * support + 1, os, w_size, support, wcs, freq0, cell_size, n};
    init_c_kernel<<<unsigned((n + 255) / 256), 256, 0, s>>>(p, reinterpret_cast<float2*>(d_c));
    TCV_CUDA(cudaGetLastError());
    float* d_sum = static_cast<float*>(d_scratch);
    sum_abs_seq_kernel<<<1, 1024, 0, s>>>(reinterpret_cast<const float2*>(d_c), n, d_sum);
    TCV_CUDA(cudaGetLastError());
    scale_c_kernel<<<grid_blocks(n, 256), 256, 0, s>>>(reinterpret_cast<float2*>(d_c), n,
                                                       float(w_size * os * os), d_sum);
    TCV_CUDA(cudaGetLastError());
    if (sum_c_out) {
        TCV_CUDA(cudaMemcpyAsync(sum_c_out, d_sum, sizeof(float), cudaMemcpyDeviceToHost, s));
        TCV_CUDA(cudaStreamSynchronize(s));
    }
    return TCV_OK;
}

size_t tcv_ctype_bytes(int c_type)
{
    switch (c_type & 0xff) {
        case TCV_C_C64: return 8;
        case TCV_C_R32: return 4;
        case TCV_C_CBF16: return 4;
        case TCV_C_RBF16: return 2;
        case TCV_C_CF16: return 4;
        case TCV_C_RF16: return 2;
        default: return 0;
    }
}

tcv_status tcv_convert_c(const float* d_c64, int64_t c_len, int c_type, void* d_out,
                         float* c_scale_out, int64_t* imag_nonzero_out, void* stream)
{
    if (!d_c64 || c_len <= 0 || tcv_ctype_bytes(c_type) == 0 || (c_type & TCV_C_PADDED)) return TCV_ERR_ARG;
    if (c_type == TCV_C_C64) {
        if (!d_out) return TCV_ERR_ARG;
        if (d_out != d_c64)
            TCV_CUDA(cudaMemcpyAsync(d_out, d_c64, size_t(c_len) * 8, cudaMemcpyDeviceToDevice,
                                     static_cast<cudaStream_t>(stream)));
        if (c_scale_out) *c_scale_out = 1.0f;
        if (imag_nonzero_out) *imag_nonzero_out = 0;
        return TCV_OK;
    }
    if (!d_out) return TCV_ERR_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const float2* c = reinterpret_cast<const float2*>(d_c64);
    // set-up path: a 16-byte device scratch for the max-abs and imaginary-part counters
    void* scratch = nullptr;
    TCV_CUDA(cudaMalloc(&scratch, 16));
    unsigned int* d_max = static_cast<unsigned int*>(scratch);
    unsigned long long* d_nz = reinterpret_cast<unsigned long long*>(static_cast<char*>(scratch) + 8);
    cudaError_t e = cudaMemsetAsync(scratch, 0, 16, s);
    if (e == cudaSuccess) {
        absmax_imag_kernel<<<grid_blocks(c_len, 256), 256, 0, s>>>(c, c_len, d_max, d_nz);
        e = cudaGetLastError();
    }
    unsigned int hmax = 0;
    unsigned long long hnz = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&hmax, d_max, 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&hnz, d_nz, 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(scratch);
    TCV_CUDA(e);
    float pre = 1.0f, post = 1.0f;
    if (c_type == TCV_C_CF16 || c_type == TCV_C_RF16) {
        // power-of-two scale putting max |C| in [2^14, 2^15): the table keeps FP16's full
        // precision without approaching its 65504 limit; kernels undo it exactly with c_scale.
        const float amax = __builtin_bit_cast(float, hmax);
        int ex = 0;
        if (amax > 0.f) {
            std::frexp(amax, &ex);  // amax = m * 2^ex, m in [0.5, 1)
            const int shift = 15 - ex;
            pre = std::ldexp(1.0f, shift);
            post = std::ldexp(1.0f, -shift);
        }
    }
    convert_kernel<<<grid_blocks(c_len, 256), 256, 0, s>>>(c, c_len, c_type, pre, d_out);
    TCV_CUDA(cudaGetLastError());
    if (c_scale_out) *c_scale_out = post;
    if (imag_nonzero_out) *imag_nonzero_out = int64_t(hnz);
    return TCV_OK;
}

tcv_status tcv_init_uvw_raw(int64_t n_samples, int baseline, uint64_t state0, double* d_u,
                            double* d_v, double* d_w, void* stream)
{
    if (n_samples < 0 || (n_samples > 0 && (!d_u || !d_v || !d_w))) return TCV_ERR_ARG;
    if (n_samples == 0) return TCV_OK;
    uvw_kernel<<<unsigned((n_samples + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        n_samples, baseline, state0, d_u, d_v, d_w);
    TCV_CUDA(cudaGetLastError());
    return TCV_OK;
}

tcv_status tcv_init_offsets_raw(const double* d_u, const double* d_v, const double* d_w,
                                int64_t n_samples, const double* d_freq, int n_chan,
                                double cell_size, double w_cell_size, int w_size, int g_size,
                                int support, int over_sample, int32_t* d_iu, int32_t* d_iv,
                                int32_t* d_coff, void* stream)
{
    if (n_samples < 0 || n_chan < 1 || support < 0 || over_sample < 1 || g_size < 1 || w_size < 1)
        return TCV_ERR_ARG;
    if (n_samples == 0) return TCV_OK;
    if (!d_u || !d_v || !d_w || !d_freq || !d_iu || !d_iv || !d_coff) return TCV_ERR_ARG;
    OffParams p{n_samples, n_chan, w_size, g_size, 2 * support + 1, over_sample, cell_size, w_cell_size};
    const int64_t n = n_samples * n_chan;
    offsets_kernel<<<unsigned((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        p, d_u, d_v, d_w, d_freq, d_iu, d_iv, d_coff);
    TCV_CUDA(cudaGetLastError());
    return TCV_OK;
}

}  // extern "C"
