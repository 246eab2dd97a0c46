// tcv_bands.cu -- the device steps of a row-band split of one gridding job over several GPUs.
//
// The reference scales only by independent replicas (attic/tConvolveMPI/tConvolveMPI.cc:78-119:
// every MPI rank grids its own copy of the problem); one grid shared by several GPUs has no
// counterpart there.  Here rank b owns the grid rows [rows[b], rows[b+1]).  A sample belongs to
// the band of its footprint's centre row iv + support: the footprint covers rows iv .. iv +
// 2*support (attic/tConvolveMPI/Benchmark.cc:137-150, gind = iu + gSize*iv - support, one row of
// sSize points per suppv), so it reaches at most `support` rows past either edge of its band, and
// every band is at least `support` rows high, so that halo lies in the neighbouring band only.
//
//   tcv_band_histogram  centre-row histogram of the samples (the band bounds balance it)
//   tcv_band_bounds     the bounds themselves (host arithmetic)
//   tcv_band_bucket     stable partition of the samples by band into packed 20-byte records (the
//                       all-to-all payload: data, iu, iv, cOffset) and the permutation back to
//                       the input order
//   tcv_band_unpack     records -> data, iu, iv, cOffset arrays
//   tcv_band_scatter    dst[perm[i]] = src[i] (degridded samples back to their input order)
//   tcv_rows_add        dst += src (a neighbour's halo rows added into the owner's rows)
//
// The exchanges between the steps are NCCL calls of the host (one all-to-all of the records, one
// send/receive of `support` rows per band edge after gridding and before degridding).
#include "tcv_internal.cuh"

#include <algorithm>

namespace tcv {
namespace {

constexpr int kBandMax = 64;                       // most bands of one split
constexpr int kBkThreads = 256;                    // bucketing block
constexpr int kBkWarps = kBkThreads / 32;
constexpr int kBkChunks = 16;                      // chunks of kBkThreads samples per block
constexpr int64_t kBkTile = int64_t(kBkThreads) * kBkChunks;
constexpr int kScanThreads = 1024;

struct BandRows {
    int32_t r[kBandMax + 1];
};

// Band of a sample: its centre row, clamped to the grid (samples outside the grid are rejected
// by whichever rank's plan receives them), against the ascending bounds.
__device__ __forceinline__ int band_of(int32_t iv, int support, int g_size, const BandRows& rows, int n_bands)
{
    int64_t c = int64_t(iv) + support;
    c = c < 0 ? 0 : (c >= g_size ? g_size - 1 : c);
    int b = 0;
    for (int k = 1; k < n_bands; ++k) b += c >= rows.r[k] ? 1 : 0;
    return b;
}

__global__ void band_hist_kernel(const int32_t* __restrict__ iv, int64_t n, int support, int g_size,
                                 unsigned long long* __restrict__ hist)
{
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        int64_t c = int64_t(iv[i]) + support;
        c = c < 0 ? 0 : (c >= g_size ? g_size - 1 : c);
        atomicAdd(hist + c, 1ull);
    }
}

// Per block of kBkTile samples: how many fall in each band, stored band-major
// (cnt[band * nblocks + block]) so that one exclusive scan gives every (band, block) its first
// output position.
__global__ void __launch_bounds__(kBkThreads) band_count_kernel(const int32_t* __restrict__ iv, int64_t n, int support,
                                                                int g_size, BandRows rows, int n_bands,
                                                                uint32_t* __restrict__ cnt)
{
    __shared__ uint32_t c[kBandMax];
    for (int k = threadIdx.x; k < n_bands; k += kBkThreads) c[k] = 0;
    __syncthreads();
    const int64_t t0 = int64_t(blockIdx.x) * kBkTile;
    for (int j = 0; j < kBkChunks; ++j) {
        const int64_t i = t0 + int64_t(j) * kBkThreads + threadIdx.x;
        if (i < n) atomicAdd(&c[band_of(iv[i], support, g_size, rows, n_bands)], 1u);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < n_bands; k += kBkThreads) cnt[int64_t(k) * gridDim.x + blockIdx.x] = c[k];
}

// Exclusive scan of the m per-(band, block) counts (one block), and each band's total.
__global__ void __launch_bounds__(kScanThreads) band_scan_kernel(const uint32_t* __restrict__ cnt, int64_t m,
                                                                  int nblocks, int n_bands,
                                                                  uint32_t* __restrict__ offs,
                                                                  int64_t* __restrict__ band_counts)
{
    __shared__ uint32_t wsum[kScanThreads / 32];
    __shared__ uint32_t carry_s;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) carry_s = 0;
    __syncthreads();
    for (int64_t base = 0; base < m; base += kScanThreads) {
        const int64_t i = base + threadIdx.x;
        const uint32_t v = i < m ? cnt[i] : 0u;
        uint32_t x = v;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
            if (lane >= d) x += y;
        }
        if (lane == 31) wsum[warp] = x;
        __syncthreads();
        if (warp == 0) {
            uint32_t s = wsum[lane];
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, s, d);
                if (lane >= d) s += y;
            }
            wsum[lane] = s;
        }
        __syncthreads();
        const uint32_t excl = carry_s + (warp ? wsum[warp - 1] : 0u) + x - v;
        if (i < m) offs[i] = excl;
        __syncthreads();  // carry_s and wsum are read by every thread before they change
        if (threadIdx.x == kScanThreads - 1) carry_s = excl + v;
        __syncthreads();
    }
    for (int k = threadIdx.x; k < n_bands; k += kScanThreads) {
        const uint32_t s = offs[int64_t(k) * nblocks];
        const uint32_t e = k + 1 < n_bands ? offs[int64_t(k + 1) * nblocks] : carry_s;
        band_counts[k] = int64_t(e - s);
    }
}

// Stable partition: a block walks its tile in chunks of kBkThreads samples in input order; within
// a chunk a sample's position in its band is (block's running count) + (same-band samples of the
// lower warps) + (same-band lanes below it), so the output keeps the input order inside every band.
__global__ void __launch_bounds__(kBkThreads) band_scatter_kernel(
    const float2* __restrict__ data, const int32_t* __restrict__ iu, const int32_t* __restrict__ iv,
    const int32_t* __restrict__ coff, int64_t n, int support, int g_size, BandRows rows, int n_bands,
    const uint32_t* __restrict__ offs, int32_t* __restrict__ rec, int32_t* __restrict__ perm)
{
    __shared__ uint32_t run[kBandMax];
    __shared__ uint32_t wcnt[kBkWarps][kBandMax];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int k = threadIdx.x; k < n_bands; k += kBkThreads) run[k] = offs[int64_t(k) * gridDim.x + blockIdx.x];
    const int64_t t0 = int64_t(blockIdx.x) * kBkTile;
    for (int j = 0; j < kBkChunks; ++j) {
        for (int e = threadIdx.x; e < kBkWarps * kBandMax; e += kBkThreads) (&wcnt[0][0])[e] = 0u;
        const int64_t i = t0 + int64_t(j) * kBkThreads + threadIdx.x;
        const bool valid = i < n;
        const int b = valid ? band_of(iv[i], support, g_size, rows, n_bands) : kBandMax;
        const unsigned same = __match_any_sync(0xffffffffu, b);
        const unsigned below = __popc(same & ((1u << lane) - 1u));
        __syncthreads();  // S1: counts zeroed; the previous chunk's run[] update is visible
        if (valid && below == 0) wcnt[warp][b] = __popc(same);
        __syncthreads();  // S2: every warp's counts are in
        uint32_t pos = 0;
        if (valid) {
            uint32_t before = 0;
            for (int w = 0; w < warp; ++w) before += wcnt[w][b];
            pos = run[b] + before + below;
        }
        uint32_t tot = 0;
        if (int(threadIdx.x) < n_bands) {
            for (int w = 0; w < kBkWarps; ++w) tot += wcnt[w][threadIdx.x];
        }
        __syncthreads();  // S3: run[] and wcnt are read before they change
        if (int(threadIdx.x) < n_bands) run[threadIdx.x] += tot;
        if (valid) {
            const float2 d = data[i];
            int32_t* r = rec + 5 * int64_t(pos);
            r[0] = __float_as_int(d.x);
            r[1] = __float_as_int(d.y);
            r[2] = iu[i];
            r[3] = iv[i];
            r[4] = coff[i];
            perm[pos] = int32_t(i);
        }
    }
}

__global__ void band_unpack_kernel(const int32_t* __restrict__ rec, int64_t n, float2* __restrict__ data,
                                   int32_t* __restrict__ iu, int32_t* __restrict__ iv, int32_t* __restrict__ coff)
{
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const int32_t* r = rec + 5 * i;
        data[i] = make_float2(__int_as_float(r[0]), __int_as_float(r[1]));
        iu[i] = r[2];
        iv[i] = r[3];
        coff[i] = r[4];
    }
}

__global__ void band_perm_scatter_kernel(const float2* __restrict__ src, const int32_t* __restrict__ perm, int64_t n,
                                         float2* __restrict__ dst)
{
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) dst[perm[i]] = src[i];
}

__global__ void rows_add4_kernel(float4* __restrict__ dst, const float4* __restrict__ src, int64_t n4)
{
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n4; i += stride) {
        float4 a = dst[i];
        const float4 b = src[i];
        a.x += b.x;
        a.y += b.y;
        a.z += b.z;
        a.w += b.w;
        dst[i] = a;
    }
}

__global__ void rows_add_kernel(float* __restrict__ dst, const float* __restrict__ src, int64_t n)
{
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) dst[i] += src[i];
}

int sm_count()
{
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

// Grid of a grid-stride elementwise launch: enough blocks for n items, at most 8 per SM.
unsigned stride_blocks(int64_t n, int threads)
{
    const int64_t want = (n + threads - 1) / threads;
    return unsigned(std::max<int64_t>(1, std::min<int64_t>(want, int64_t(sm_count()) * 8)));
}

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

int64_t bucket_blocks(int64_t n) { return (n + kBkTile - 1) / kBkTile; }

bool rows_valid(const int32_t* rows, int n_bands, int g_size)
{
    if (!rows || n_bands < 1 || n_bands > kBandMax) return false;
    if (rows[0] != 0 || rows[n_bands] != g_size) return false;
    for (int b = 0; b < n_bands; ++b)
        if (rows[b + 1] <= rows[b]) return false;
    return true;
}

}  // namespace
}  // namespace tcv

using namespace tcv;

extern "C" {

tcv_status tcv_band_histogram(const int32_t* d_iv, int64_t n, int support, int g_size, int64_t* d_hist, void* stream)
{
    if (n < 0 || g_size < 1 || support < 0 || !d_hist || (n > 0 && !d_iv)) return TCV_ERR_ARG;
    if (n == 0) return TCV_OK;
    band_hist_kernel<<<stride_blocks(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        d_iv, n, support, g_size, reinterpret_cast<unsigned long long*>(d_hist));
    TCV_CUDA(cudaGetLastError());
    return TCV_OK;
}

tcv_status tcv_band_bounds(const int64_t* hist, int g_size, int support, int n_bands, int32_t* rows_out)
{
    if (!hist || !rows_out || g_size < 1 || support < 0 || n_bands < 1 || n_bands > kBandMax) return TCV_ERR_ARG;
    const int h = std::max(support, 1);  // every band at least `support` rows (and one row) high
    if (int64_t(n_bands) * h > g_size) return TCV_ERR_ARG;
    int64_t total = 0;
    for (int r = 0; r < g_size; ++r) {
        if (hist[r] < 0) return TCV_ERR_ARG;
        total += hist[r];
    }
    // bound b: the first row at which the samples of the rows below reach b/n_bands of the total
    rows_out[0] = 0;
    rows_out[n_bands] = g_size;
    int64_t cum = 0;
    int r = 0;
    for (int b = 1; b < n_bands; ++b) {
        const int64_t target = (total * b + n_bands - 1) / n_bands;
        while (r < g_size && cum < target) cum += hist[r++];
        rows_out[b] = r;
    }
    // heights of at least h: push bounds up from the bottom, then down from the top
    for (int b = 1; b < n_bands; ++b) rows_out[b] = std::max(rows_out[b], rows_out[b - 1] + h);
    for (int b = n_bands - 1; b >= 1; --b) rows_out[b] = std::min(rows_out[b], rows_out[b + 1] - h);
    return TCV_OK;
}

size_t tcv_band_workspace_bytes(int64_t n, int n_bands)
{
    if (n < 0 || n_bands < 1 || n_bands > kBandMax) return 0;
    const size_t m = size_t(bucket_blocks(n)) * size_t(n_bands);
    return 2 * align256(std::max<size_t>(m, 1) * sizeof(uint32_t));
}

tcv_status tcv_band_bucket(const float* d_data, const int32_t* d_iu, const int32_t* d_iv, const int32_t* d_coff,
                           int64_t n, int support, int g_size, const int32_t* rows, int n_bands, int32_t* d_records,
                           int32_t* d_perm, int64_t* d_counts, void* d_work, size_t work_bytes, void* stream)
{
    if (n < 0 || n > int64_t(INT32_MAX) || support < 0 || g_size < 1 || !d_counts) return TCV_ERR_ARG;
    if (!rows_valid(rows, n_bands, g_size)) return TCV_ERR_ARG;
    if (n > 0 && (!d_data || !d_iu || !d_iv || !d_coff || !d_records || !d_perm || !d_work)) return TCV_ERR_ARG;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (n == 0) {
        TCV_CUDA(cudaMemsetAsync(d_counts, 0, size_t(n_bands) * sizeof(int64_t), s));
        return TCV_OK;
    }
    if (work_bytes < tcv_band_workspace_bytes(n, n_bands)) return TCV_ERR_WORKSPACE;
    BandRows br{};
    for (int b = 0; b <= n_bands; ++b) br.r[b] = rows[b];
    const int64_t nblocks = bucket_blocks(n);
    const int64_t m = nblocks * n_bands;
    uint32_t* cnt = static_cast<uint32_t*>(d_work);
    uint32_t* offs = reinterpret_cast<uint32_t*>(static_cast<char*>(d_work) + align256(size_t(m) * sizeof(uint32_t)));
    band_count_kernel<<<unsigned(nblocks), kBkThreads, 0, s>>>(d_iv, n, support, g_size, br, n_bands, cnt);
    TCV_CUDA(cudaGetLastError());
    band_scan_kernel<<<1, kScanThreads, 0, s>>>(cnt, m, int(nblocks), n_bands, offs, d_counts);
    TCV_CUDA(cudaGetLastError());
    band_scatter_kernel<<<unsigned(nblocks), kBkThreads, 0, s>>>(reinterpret_cast<const float2*>(d_data), d_iu, d_iv,
                                                                 d_coff, n, support, g_size, br, n_bands, offs,
                                                                 d_records, d_perm);
    TCV_CUDA(cudaGetLastError());
    return TCV_OK;
}

tcv_status tcv_band_unpack(const int32_t* d_records, int64_t n, float* d_data, int32_t* d_iu, int32_t* d_iv,
                           int32_t* d_coff, void* stream)
{
    if (n < 0) return TCV_ERR_ARG;
    if (n == 0) return TCV_OK;
    if (!d_records || !d_data || !d_iu || !d_iv || !d_coff) return TCV_ERR_ARG;
    band_unpack_kernel<<<stride_blocks(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        d_records, n, reinterpret_cast<float2*>(d_data), d_iu, d_iv, d_coff);
    TCV_CUDA(cudaGetLastError());
    return TCV_OK;
}

tcv_status tcv_band_scatter(const float* d_src, const int32_t* d_perm, int64_t n, float* d_dst, void* stream)
{
    if (n < 0) return TCV_ERR_ARG;
    if (n == 0) return TCV_OK;
    if (!d_src || !d_perm || !d_dst) return TCV_ERR_ARG;
    band_perm_scatter_kernel<<<stride_blocks(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const float2*>(d_src), d_perm, n, reinterpret_cast<float2*>(d_dst));
    TCV_CUDA(cudaGetLastError());
    return TCV_OK;
}

tcv_status tcv_rows_add(float* d_dst, const float* d_src, int64_t n_complex, void* stream)
{
    if (n_complex < 0) return TCV_ERR_ARG;
    if (n_complex == 0) return TCV_OK;
    if (!d_dst || !d_src) return TCV_ERR_ARG;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int64_t nf = 2 * n_complex;
    const bool vec = (reinterpret_cast<uintptr_t>(d_dst) % 16 == 0) && (reinterpret_cast<uintptr_t>(d_src) % 16 == 0) &&
                     nf % 4 == 0;
    if (vec) {
        rows_add4_kernel<<<stride_blocks(nf / 4, 256), 256, 0, s>>>(reinterpret_cast<float4*>(d_dst),
                                                                   reinterpret_cast<const float4*>(d_src), nf / 4);
    } else {
        rows_add_kernel<<<stride_blocks(nf, 256), 256, 0, s>>>(d_dst, d_src, nf);
    }
    TCV_CUDA(cudaGetLastError());
    return TCV_OK;
}

}  // extern "C"
