// tcv_hogbom.cu -- Hogbom CLEAN (the minor cycle) on the device.
//
// Reference: current/tHogbomCleanOMP/HogbomGolden.cc:47-141 (HogbomGolden::deconvolve, findPeak,
// subtractPSF) and the same steps inside current/tMajorACC/tMajorACC.cc:689-877 (deconvolve).  Each
// iteration takes the pixel of largest |residual| (the first such index, as the reference's strict
// '>' scan in index order does), adds gain * peak to the model there, and subtracts
// (gain * peak) * psf, shifted so that the PSF's own peak lands on that pixel, over the overlap of
// the two images.  The arithmetic is the reference's, rounding by rounding: t = gain * peak,
// u = t * psf, r = r - u, each rounded to float (no contraction into fused multiply-adds), so the
// model and the residual are bit-identical to the reference's.
//
// The reference computes the PSF row as y - (ry - px) (its diffy uses the PSF peak's x,
// HogbomGolden.cc:108); that is kept.  Where it points outside the PSF (only when the PSF peak is
// off the diagonal) the reference reads out of bounds; here those rows are skipped and counted.
//
// B200 layout: one launch per iteration, no host round trip.  A launch subtracts the PSF over its
// blocks' slices of the image and scans the updated values for the next peak in the same pass, so
// an iteration reads the residual once, reads the PSF's overlap once and writes the overlap once.
// Each block leaves one candidate, a 64-bit key (|value| bits << 32 | ~index: the largest key is
// the largest magnitude at the smallest index) with its signed value; the last block to finish
// (an atomic ticket, no waiting) reduces the candidates to the winner that the next launch reads.
// The stop test (|peak| < threshold) is taken on the device: later launches see the flag and return.
#include "tcv_internal.cuh"

#include <algorithm>
#include <cstdint>

namespace tcv {
namespace {

constexpr int kHogThreads = 256;
constexpr int kHogMaxBlocks = 592;  // 4 x 148: one wave of four 256-thread CTAs per SM

// device state of one deconvolution (start of the caller's workspace; zeroed by the host)
struct HogState {
    unsigned long long win_key[3];  // winners: [0], [1] by iteration parity, [2] the PSF's
    float win_val[3];
    unsigned int arrived;           // blocks finished in the current launch (persistent loop: in all
                                    // iterations so far)
    int stopped;                    // 1 + the iteration whose |peak| fell below the threshold; 0 = running
    int done;                       // iterations carried out
    unsigned int psf_pos;           // PSF peak index
    unsigned long long skipped_rows;  // PSF rows outside the PSF (reference out-of-bounds reads)
    int error;                        // persistent kernel: a barrier wait gave up
};

struct HogArgs {
    const float* psf;
    float* residual;
    float* model;
    unsigned long long* keys;  // one candidate per block
    float* vals;
    unsigned long long* keys2;  // persistent loop: the candidates of odd iterations
    float* vals2;
    HogState* state;
    float* hist_val;         // per iteration: peak value (may be null)
    unsigned int* hist_pos;  // per iteration: peak index (may be null)
    int width, psf_width, nblocks;
    long long n;  // width * width
    float gain, threshold;
    unsigned long long wait_ns;  // persistent loop: limit of one grid-barrier wait
    unsigned int withheld;       // persistent loop: arrivals the barrier counts that never come (test hook)
};

__device__ __forceinline__ unsigned int key_index(unsigned long long k) { return ~static_cast<unsigned int>(k); }

// Block-wide maximum of (key, value); the winner is returned to every thread.
__device__ unsigned long long block_max(unsigned long long k, float& v)
{
    __shared__ unsigned long long sk[kHogThreads / 32];
    __shared__ float sv[kHogThreads / 32];
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long ko = __shfl_down_sync(0xffffffffu, k, o);
        const float vo = __shfl_down_sync(0xffffffffu, v, o);
        if (ko > k) {
            k = ko;
            v = vo;
        }
    }
    const int w = threadIdx.x >> 5;
    __syncthreads();  // earlier readers of sk/sv are done
    if ((threadIdx.x & 31) == 0) {
        sk[w] = k;
        sv[w] = v;
    }
    __syncthreads();
    k = sk[0];
    v = sv[0];
    for (int i = 1; i < kHogThreads / 32; ++i)
        if (sk[i] > k) {
            k = sk[i];
            v = sv[i];
        }
    return k;
}

// Leave this block's candidate; the last block of the launch reduces all of them into
// state->win_key/win_val[slot] (and for the PSF slot, the PSF peak position).
__device__ void finish_scan(unsigned long long best, float bv, unsigned long long* keys, float* vals, int nblocks,
                            HogState* st, int slot)
{
    best = block_max(best, bv);
    __shared__ bool last;
    if (threadIdx.x == 0) {
        keys[blockIdx.x] = best;
        vals[blockIdx.x] = bv;
        __threadfence();
        last = atomicAdd(&st->arrived, 1u) == unsigned(nblocks - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    unsigned long long k = 0;
    float v = 0.f;
    for (int i = threadIdx.x; i < nblocks; i += kHogThreads) {
        const unsigned long long ki = __ldcg(keys + i);
        if (ki > k) {
            k = ki;
            v = __ldcg(vals + i);
        }
    }
    k = block_max(k, v);
    if (threadIdx.x == 0) {
        const bool zero = (k >> 32) == 0;  // an all-zero image: the reference keeps maxPos = 0, maxVal = 0
        st->win_key[slot] = zero ? static_cast<unsigned long long>(~0u) : k;
        st->win_val[slot] = zero ? 0.f : v;
        if (slot == 2) st->psf_pos = zero ? 0u : key_index(k);
        st->arrived = 0;
    }
}

// Scan an image (copying it to copy_to when given) for its peak.
__global__ void __launch_bounds__(kHogThreads) hog_scan_kernel(const float* __restrict__ img, float* __restrict__ copy_to,
                                                               long long n, int nblocks, unsigned long long* keys,
                                                               float* vals, HogState* st, int slot)
{
    const long long per = (n + nblocks - 1) / nblocks;
    const long long lo = per * blockIdx.x, hi = min(n, lo + per);
    float best_abs = -1.f, bv = 0.f;
    unsigned int bi = 0;
    for (long long i = lo + threadIdx.x; i < hi; i += kHogThreads) {
        const float v = img[i];
        if (copy_to) copy_to[i] = v;
        if (fabsf(v) > best_abs) {  // strict '>' in index order keeps the first index
            best_abs = fabsf(v);
            bv = v;
            bi = static_cast<unsigned int>(i);
        }
    }
    const unsigned long long best =
        best_abs < 0.f ? 0ull : (static_cast<unsigned long long>(__float_as_uint(best_abs)) << 32) | (~bi & 0xffffffffu);
    finish_scan(best, bv, keys, vals, nblocks, st, slot);
}

// subtractPSF (HogbomGolden.cc:99-124) over this CTA's share of the image, and the scan of the
// updated values: returns the CTA-thread's candidate key (0 if it saw no pixel) and value.
// kVec: width a multiple of 4 and the residual 16-byte aligned (float4 residual I/O).
template <bool kVec>
__device__ __forceinline__ unsigned long long iter_body(const HogArgs& a, unsigned int ppos, float peak,
                                                        unsigned int psf_pos, float& bv_out,
                                                        unsigned long long& skipped_out)
{
    const int W = a.width, P = a.psf_width;
    const int rx = int(ppos % unsigned(W)), ry = int(ppos / unsigned(W));
    const int px = int(psf_pos % unsigned(P)), py = int(psf_pos / unsigned(P));
    const int diffx = rx - px, diffy = ry - px;  // diffy uses px, as the reference does
    const int startx = max(0, rx - px), starty = max(0, ry - py);
    const int stopx = min(W - 1, rx + (P - px - 1)), stopy = min(W - 1, ry + (P - py - 1));
    const float t = __fmul_rn(a.gain, peak);

    // running maximum of |value| in index order: strict '>' keeps the first index (findPeak's rule)
    float best_abs = -1.f, bv = 0.f;
    unsigned int bi = 0;
    unsigned long long skipped = 0;
    auto track = [&](float v, unsigned int idx) {
        const float av = fabsf(v);
        if (av > best_abs) {
            best_abs = av;
            bv = v;
            bi = idx;
        }
    };
    if (kVec) {
        // whole rows per block, walked as items (row, column chunk of 256 float4) in index order;
        // every thread loads the float4s of U items (of one or several rows) before any store
        constexpr int U = 4;
        const int rows_per = (W + a.nblocks - 1) / a.nblocks;
        const int r0 = int(blockIdx.x) * rows_per, r1 = min(W, r0 + rows_per);
        const int nch = (W / 4 + kHogThreads - 1) / kHogThreads;  // chunks per row
        if (threadIdx.x == 0)
            for (int y = r0; y < r1; ++y)
                if (y >= starty && y <= stopy && !(y - diffy >= 0 && y - diffy < P)) ++skipped;
        int y = r0, c = 0;
        while (y < r1) {
            float4 r[U];
            float pv[U][4];
            bool sub[U], val[U];
            int xs[U], ys[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                ys[u] = y;
                xs[u] = 4 * (int(threadIdx.x) + kHogThreads * c);
                val[u] = y < r1 && xs[u] < W;
                if (++c == nch) {
                    c = 0;
                    ++y;
                }
                sub[u] = false;
                r[u] = make_float4(0.f, 0.f, 0.f, 0.f);
                if (val[u]) {
                    r[u] = __ldcg(reinterpret_cast<const float4*>(a.residual + ((long long)ys[u] * W + xs[u])));
                    const int prow = ys[u] - diffy;
                    sub[u] = ys[u] >= starty && ys[u] <= stopy && prow >= 0 && prow < P && xs[u] + 3 >= startx &&
                             xs[u] <= stopx;
                    const long long pbase = (long long)prow * P - diffx;  // + x: inside the PSF row for x in range
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const int x = xs[u] + j;
                        pv[u][j] = (sub[u] && x >= startx && x <= stopx) ? __ldg(a.psf + (pbase + x)) : 0.f;
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                if (!val[u]) continue;
                if (sub[u]) {
                    float* rv = reinterpret_cast<float*>(&r[u]);
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const int x = xs[u] + j;
                        if (x >= startx && x <= stopx) rv[j] = __fsub_rn(rv[j], __fmul_rn(t, pv[u][j]));
                    }
                    __stcg(reinterpret_cast<float4*>(a.residual + ((long long)ys[u] * W + xs[u])), r[u]);
                }
                const unsigned int i0 = unsigned(ys[u]) * unsigned(W) + unsigned(xs[u]);
                track(r[u].x, i0);
                track(r[u].y, i0 + 1);
                track(r[u].z, i0 + 2);
                track(r[u].w, i0 + 3);
            }
        }
    } else {
        const long long per = (a.n + a.nblocks - 1) / a.nblocks;
        const long long lo = per * blockIdx.x, hi = min(a.n, lo + per);
        for (long long i = lo + threadIdx.x; i < hi; i += kHogThreads) {
            const unsigned ui = unsigned(i);  // n < 2^32
            const int y = int(ui / unsigned(W)), x = int(ui - unsigned(y) * unsigned(W));
            float r = a.residual[i];
            const int prow = y - diffy;
            if (y >= starty && y <= stopy && x >= startx && x <= stopx) {
                if (prow >= 0 && prow < P) {
                    r = __fsub_rn(r, __fmul_rn(t, a.psf[(long long)prow * P + (x - diffx)]));
                    a.residual[i] = r;
                } else if (x == startx) {
                    ++skipped;
                }
            }
            track(r, ui);
        }
    }
    const unsigned long long best =
        best_abs < 0.f ? 0ull : (static_cast<unsigned long long>(__float_as_uint(best_abs)) << 32) | (~bi & 0xffffffffu);
    bv_out = bv;
    skipped_out = skipped;
    return best;
}

// model[absPeakPos] += absPeakVal * g_gain (HogbomGolden.cc:93), by one thread
__device__ __forceinline__ void model_update(const HogArgs& a, int it, unsigned int ppos, float peak)
{
    a.model[ppos] = __fadd_rn(a.model[ppos], __fmul_rn(peak, a.gain));
    if (a.hist_val) a.hist_val[it] = peak;
    if (a.hist_pos) a.hist_pos[it] = ppos;
}

// One launch per iteration: the previous scan's winner, the model update, the PSF subtraction and
// the scan of this CTA's rows.
template <bool kVec>
__global__ void __launch_bounds__(kHogThreads, 4) hog_iter_kernel(HogArgs a, int it)
{
    HogState* st = a.state;
    if (st->stopped) return;  // an earlier launch stopped the loop
    const int par = it & 1;
    const unsigned int ppos = key_index(st->win_key[par]);
    const float peak = st->win_val[par];
    if (fabsf(peak) < a.threshold) {  // HogbomGolden.cc:86-89
        if (blockIdx.x == 0 && threadIdx.x == 0) st->stopped = it + 1;
        return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        model_update(a, it, ppos, peak);
        st->done = it + 1;
    }
    if (kVec && it > 0) {
        // rows wholly outside this iteration's PSF overlap do not change: the CTA's candidate from
        // an earlier iteration (same row partition; iteration 0 always scans, after the image
        // scan's pixel partition) still holds, so it is left as it is without reading the rows
        const int W = a.width, P = a.psf_width;
        const int ry = int(ppos / unsigned(W)), py = int(st->psf_pos / unsigned(P));
        const int starty = max(0, ry - py), stopy = min(W - 1, ry + (P - py - 1));
        const int rows_per = (W + a.nblocks - 1) / a.nblocks;
        const int r0 = int(blockIdx.x) * rows_per, r1 = min(W, r0 + rows_per);
        if (r1 <= starty || r0 > stopy) {
            const unsigned long long old = __ldcg(a.keys + blockIdx.x);
            const float oldv = __ldcg(a.vals + blockIdx.x);
            finish_scan(old, oldv, a.keys, a.vals, a.nblocks, st, par ^ 1);
            return;
        }
    }
    float bv;
    unsigned long long skipped;
    const unsigned long long best = iter_body<kVec>(a, ppos, peak, st->psf_pos, bv, skipped);
    if (skipped) atomicAdd(&st->skipped_rows, skipped);
    finish_scan(best, bv, a.keys, a.vals, a.nblocks, st, par ^ 1);
}

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// All iterations in one cooperative launch (every CTA resident).  Per iteration each CTA leaves its
// candidate in the buffer of the iteration's parity and adds one to a monotonic arrival count;
// once the count reaches the iteration's target every CTA reads all candidates itself and reduces
// them in the same order (so every CTA holds the same winner), with no second round trip through a
// published winner.  Waits are bounded by an iteration count and 2 s of %globaltimer, after which
// the CTA flags the error and returns (the host reports TCV_ERR_TIMEOUT).  Two candidate buffers
// suffice: a CTA cannot write iteration it + 1's candidates before every CTA has arrived at barrier
// it, i.e. has read iteration it - 1's.
template <bool kVec>
__global__ void __launch_bounds__(kHogThreads, 2) hog_persist_kernel(HogArgs a, int niters)
{
    HogState* st = a.state;
    const unsigned int psf_pos = st->psf_pos;
    __shared__ int ok;
    unsigned int ppos = key_index(__ldcg(&st->win_key[0]));  // the dirty image's scan
    float peak = __ldcg(&st->win_val[0]);
    for (int it = 0; it < niters; ++it) {
        if (fabsf(peak) < a.threshold) {  // every CTA holds the same winner: all stop here
            if (blockIdx.x == 0 && threadIdx.x == 0) st->stopped = it + 1;
            return;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            model_update(a, it, ppos, peak);
            st->done = it + 1;
        }
        float bv;
        unsigned long long skipped;
        unsigned long long best = iter_body<kVec>(a, ppos, peak, psf_pos, bv, skipped);
        if (skipped) atomicAdd(&st->skipped_rows, skipped);
        best = block_max(best, bv);
        unsigned long long* keys = (it & 1) ? a.keys2 : a.keys;
        float* vals = (it & 1) ? a.vals2 : a.vals;
        if (threadIdx.x == 0) {
            keys[blockIdx.x] = best;
            vals[blockIdx.x] = bv;
            __threadfence();
            atomicAdd(&st->arrived, 1u);
            const unsigned int target = unsigned(it + 1) * unsigned(a.nblocks) + a.withheld;
            ok = 0;
            const unsigned long long t0 = global_ns();
            for (unsigned int spin = 0; spin < (1u << 24); ++spin) {
                if (*reinterpret_cast<volatile unsigned int*>(&st->arrived) >= target) {
                    ok = 1;
                    break;
                }
                if (*reinterpret_cast<volatile int*>(&st->error)) break;
                __nanosleep(32);
                if ((spin & 63u) == 63u && global_ns() - t0 >= a.wait_ns) break;
            }
            if (!ok) st->error = 1;
            __threadfence();
        }
        __syncthreads();
        if (!ok) return;
        // every CTA: the winner of this iteration's candidates, in the same order everywhere
        unsigned long long k = 0;
        float v = 0.f;
        for (int i = threadIdx.x; i < a.nblocks; i += kHogThreads) {
            const unsigned long long ki = __ldcg(keys + i);
            if (ki > k) {
                k = ki;
                v = __ldcg(vals + i);
            }
        }
        k = block_max(k, v);
        const bool zero = (k >> 32) == 0;  // an all-zero residual: the reference keeps maxPos = 0, maxVal = 0
        ppos = zero ? 0u : key_index(k);
        peak = zero ? 0.f : v;
    }
}

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// residual + PSF bytes up to which the persistent kernel is chosen (they stay in the 126 MB L2)
constexpr size_t kPersistBytes = size_t(48) << 20;
int g_hog_strategy = TCV_HOGBOM_AUTO;
constexpr unsigned long long kDefaultWaitNs = 2000000000ull;  // 2 s
unsigned long long g_wait_ns = kDefaultWaitNs;
unsigned int g_withheld = 0;

int hog_blocks(long long n)
{
    const long long want = (n + 4095) / 4096;  // at least ~4096 pixels per block
    return int(std::max<long long>(1, std::min<long long>(kHogMaxBlocks, want)));
}

}  // namespace
}  // namespace tcv

using namespace tcv;

extern "C" {

size_t tcv_hogbom_workspace_bytes(int width)
{
    if (width < 1) return 0;
    return align256(sizeof(HogState)) + 2 * align256(size_t(kHogMaxBlocks) * 8) + 2 * align256(size_t(kHogMaxBlocks) * 4);
}

tcv_status tcv_hogbom_deconvolve(const float* d_dirty, int width, const float* d_psf, int psf_width, float* d_model,
                                 float* d_residual, int niters, float gain, float threshold, float* d_hist_val,
                                 uint32_t* d_hist_pos, void* d_work, size_t work_bytes, void* stream)
{
    if (!d_dirty || !d_psf || !d_model || !d_residual || !d_work || width < 1 || psf_width < 1 || niters < 0)
        return TCV_ERR_ARG;
    if (uint64_t(width) * uint64_t(width) >= 0xffffffffull || uint64_t(psf_width) * uint64_t(psf_width) >= 0xffffffffull)
        return TCV_ERR_UNSUPPORTED;
    if (work_bytes < tcv_hogbom_workspace_bytes(width)) return TCV_ERR_WORKSPACE;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    char* w = static_cast<char*>(d_work);
    HogArgs a{};
    a.state = reinterpret_cast<HogState*>(w);
    {
        char* q = w + align256(sizeof(HogState));
        a.keys = reinterpret_cast<unsigned long long*>(q);
        a.keys2 = reinterpret_cast<unsigned long long*>(q + align256(size_t(kHogMaxBlocks) * 8));
        q += 2 * align256(size_t(kHogMaxBlocks) * 8);
        a.vals = reinterpret_cast<float*>(q);
        a.vals2 = reinterpret_cast<float*>(q + align256(size_t(kHogMaxBlocks) * 4));
    }
    a.psf = d_psf;
    a.residual = d_residual;
    a.model = d_model;
    a.hist_val = d_hist_val;
    a.hist_pos = d_hist_pos;
    a.width = width;
    a.psf_width = psf_width;
    a.n = (long long)width * width;
    a.nblocks = hog_blocks(a.n);
    a.gain = gain;
    a.threshold = threshold;
    a.wait_ns = g_wait_ns;
    a.withheld = g_withheld;
    TCV_CUDA(cudaMemsetAsync(a.state, 0, sizeof(HogState), st));
    // the PSF's peak (HogbomGolden.cc:73-76), then residual = dirty with the first scan (:70)
    const long long np = (long long)psf_width * psf_width;
    const int pb = hog_blocks(np);
    hog_scan_kernel<<<pb, kHogThreads, 0, st>>>(d_psf, nullptr, np, pb, a.keys, a.vals, a.state, 2);
    TCV_CUDA(cudaGetLastError());
    hog_scan_kernel<<<a.nblocks, kHogThreads, 0, st>>>(d_dirty, d_residual, a.n, a.nblocks, a.keys, a.vals, a.state, 0);
    TCV_CUDA(cudaGetLastError());
    const bool vec = width % 4 == 0 && reinterpret_cast<uintptr_t>(d_residual) % 16 == 0;
    // images whose residual and PSF sit in L2 run every iteration in one cooperative launch
    const size_t resident = size_t(a.n) * 4 + size_t(np) * 4;
    bool persist = g_hog_strategy == TCV_HOGBOM_PERSISTENT ||
                   (g_hog_strategy == TCV_HOGBOM_AUTO && resident <= kPersistBytes);
    int dev = 0, coop = 0, sms = 0, per_sm = 0;
    if (persist) {
        TCV_CUDA(cudaGetDevice(&dev));
        TCV_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
        TCV_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        if (vec)
            TCV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, hog_persist_kernel<true>, kHogThreads, 0));
        else
            TCV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, hog_persist_kernel<false>, kHogThreads, 0));
        persist = coop && per_sm > 0;
    }
    // the persistent loop's arrival count reaches niters x CTAs: keep it within 32 bits
    if (persist && uint64_t(niters) * uint64_t(std::max(1, sms * 2)) >= (1ull << 32)) persist = false;
    if (persist && niters > 0) {
        // two CTAs per SM at most (fewer candidates per barrier), never more than resident
        a.nblocks = std::max(1, std::min({sms * std::min(per_sm, 2), hog_blocks(a.n), width}));
        int n_it = niters;
        void* args[] = {&a, &n_it};
        TCV_CUDA(cudaLaunchCooperativeKernel(vec ? reinterpret_cast<const void*>(hog_persist_kernel<true>)
                                                 : reinterpret_cast<const void*>(hog_persist_kernel<false>),
                                             dim3(unsigned(a.nblocks)), dim3(kHogThreads), args, 0, st));
        return TCV_OK;
    }
    for (int it = 0; it < niters; ++it) {
        if (vec)
            hog_iter_kernel<true><<<a.nblocks, kHogThreads, 0, st>>>(a, it);
        else
            hog_iter_kernel<false><<<a.nblocks, kHogThreads, 0, st>>>(a, it);
    }
    TCV_CUDA(cudaGetLastError());
    return TCV_OK;
}

void tcv_hogbom_set_strategy(int strategy)
{
    if (strategy >= TCV_HOGBOM_AUTO && strategy <= TCV_HOGBOM_PERSISTENT) g_hog_strategy = strategy;
}

tcv_status tcv_hogbom_set_wait(uint64_t limit_ns, uint32_t withheld_arrivals)
{
    if (limit_ns > kDefaultWaitNs || withheld_arrivals > 1024u) return TCV_ERR_ARG;
    g_wait_ns = limit_ns;
    g_withheld = withheld_arrivals;
    return TCV_OK;
}

tcv_status tcv_hogbom_result(const void* d_work, int* iters_done, int* stopped_at, int64_t* skipped_rows,
                             int64_t* psf_peak_pos, void* stream)
{
    if (!d_work) return TCV_ERR_ARG;
    HogState h{};
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    TCV_CUDA(cudaMemcpyAsync(&h, d_work, sizeof(h), cudaMemcpyDeviceToHost, st));
    TCV_CUDA(cudaStreamSynchronize(st));
    if (iters_done) *iters_done = h.done;
    if (stopped_at) *stopped_at = h.stopped - 1;
    if (skipped_rows) *skipped_rows = int64_t(h.skipped_rows);
    if (psf_peak_pos) *psf_peak_pos = int64_t(h.psf_pos);
    return h.error ? TCV_ERR_TIMEOUT : TCV_OK;
}

tcv_status tcv_find_peak(const float* d_image, int64_t n, float* val_out, int64_t* pos_out, void* d_work,
                         size_t work_bytes, void* stream)
{
    if (!d_image || n < 1 || !d_work || n >= int64_t(0xffffffffll)) return TCV_ERR_ARG;
    if (work_bytes < tcv_hogbom_workspace_bytes(1)) return TCV_ERR_WORKSPACE;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    char* w = static_cast<char*>(d_work);
    HogState* state = reinterpret_cast<HogState*>(w);
    unsigned long long* keys = reinterpret_cast<unsigned long long*>(w + align256(sizeof(HogState)));
    float* vals = reinterpret_cast<float*>(w + align256(sizeof(HogState)) + 2 * align256(size_t(kHogMaxBlocks) * 8));
    TCV_CUDA(cudaMemsetAsync(state, 0, sizeof(HogState), st));
    const int nb = hog_blocks(n);
    hog_scan_kernel<<<nb, kHogThreads, 0, st>>>(d_image, nullptr, n, nb, keys, vals, state, 0);
    TCV_CUDA(cudaGetLastError());
    HogState h{};
    TCV_CUDA(cudaMemcpyAsync(&h, state, sizeof(h), cudaMemcpyDeviceToHost, st));
    TCV_CUDA(cudaStreamSynchronize(st));
    if (val_out) *val_out = h.win_val[0];
    if (pos_out) *pos_out = int64_t(~static_cast<unsigned int>(h.win_key[0]));
    return TCV_OK;
}

}  // extern "C"
