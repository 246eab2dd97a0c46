// tcv_degrid.cu -- degridding (Benchmark::degridKernel, attic/tConvolveMPI/Benchmark.cc:158-195).
//
// Staged kernel (default).  One CTA per anchor tile of ta x ta grid points.  The samples binned
// to the tile have their footprint's top-left corner inside it, so every footprint lies inside
// the region [x0, x0 + ta + sSize - 1) x [y0, y0 + ta + sSize - 1), which one TMA tensor load
// (cp.async.bulk.tensor.2d, completion on an mbarrier) brings into shared memory.  A sample's
// table entries are contiguous (sSize rows of sSize entries, rows adjacent), so warps walk the
// footprint as one flat range: each lane takes every 32nd entry, the table read is a fully
// coalesced stream, the grid value comes from shared memory, and products accumulate in FP32
// registers; a shuffle reduction finishes each warp's share.  To keep 16 warps busy on tiles
// with few samples, each footprint is split into `parts` flat ranges handled by different
// warps; partial sums are combined in a fixed order, so results do not depend on scheduling.
//
// Direct kernel (fallback for supports too wide to stage, or odd grid sizes): one warp per
// sample, grid values read from global memory (L2), otherwise the same walk.
//
// Every wait on the mbarrier is bounded by a timer; on timeout the kernel sets bit 0 of the
// plan's status word, waits once more (bounded) for its copy to land, and returns.
#include "tcv_internal.cuh"

#include <cuda.h>
#include <mutex>

namespace tcv {
namespace {

constexpr int kWarps = 16;
constexpr int kThreads = kWarps * 32;
constexpr int kChunk = 64;       // samples per round of partial sums
constexpr int kMaxParts = 8;
constexpr int kUnroll = 8;
constexpr unsigned long long kWaitNs = 2000000000ull;  // 2 s: a tile load takes microseconds

struct DegridArgs {
    int support, s, g_size;
    int ta, natx, natiles, box_w, box_h, parts;
    float c_scale;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t phase)
{
    const uint64_t t0 = global_ns();
    while (!mbar_try_wait(bar, phase))
        if (global_ns() - t0 > kWaitNs) return false;
    return true;
}

// Advance a flat footprint position by 32 entries: column, and the matching index into a
// row-major region whose rows are `pitch` entries long.
__device__ __forceinline__ void advance32(int& col, int& idx, int s, int wrap)
{
    col += 32;
    idx += 32;
    if (col >= s) {
        col -= s;
        idx += wrap;
        if (col >= s) {  // only for footprints narrower than 32
            const int q = col / s;
            col -= q * s;
            idx += q * wrap;
        }
    }
}

// Sum over flat footprint positions [f_lo, f_hi) of region[idx(f)] * C[f]; lane-partial result.
template <class Tab, class Src>
__device__ __forceinline__ float2 walk(const typename Tab::elem* __restrict__ cbase, Src region,
                                       int f_lo, int f_hi, int s, int pitch, int fx, int fy, int lane)
{
    int f = f_lo + lane;
    const int row = f / s;
    int col = f - row * s;
    int idx = (fy + row) * pitch + fx + col;
    const int wrap = pitch - s;
    float2 acc0 = make_float2(0.f, 0.f), acc1 = make_float2(0.f, 0.f);
    for (int f0 = f_lo; f0 < f_hi; f0 += 32 * kUnroll) {
        int sidx[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            sidx[u] = idx;
            advance32(col, idx, s, wrap);
        }
        float2 cv[kUnroll], gv[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            if (f + 32 * u < f_hi) {
                cv[u] = Tab::load(cbase + f + 32 * u);
                gv[u] = region(sidx[u]);
            } else {
                cv[u] = make_float2(0.f, 0.f);
                gv[u] = make_float2(0.f, 0.f);
            }
        }
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) cmac<Tab::kReal>((u & 1) ? acc1 : acc0, gv[u], cv[u]);
        f += 32 * kUnroll;
    }
    return make_float2(acc0.x + acc1.x, acc0.y + acc1.y);
}

__device__ __forceinline__ float2 warp_sum(float2 v)
{
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    return v;
}

struct SmemRegion {
    const float2* p;
    __device__ __forceinline__ float2 operator()(int i) const { return p[i]; }
};
struct GlobalRegion {
    const float2* __restrict__ p;
    __device__ __forceinline__ float2 operator()(int i) const { return __ldg(p + i); }
};

template <class Tab>
__global__ void __launch_bounds__(kThreads, 1)
degrid_staged_kernel(const __grid_constant__ CUtensorMap tmap,
                     const typename Tab::elem* __restrict__ ctab, const int32_t* __restrict__ iu,
                     const int32_t* __restrict__ iv, const int32_t* __restrict__ coff,
                     const uint32_t* __restrict__ order, const uint32_t* __restrict__ atile_start,
                     const uint32_t* __restrict__ atile_count, const uint32_t* __restrict__ aitems,
                     const uint32_t* __restrict__ n_aitems, float2* __restrict__ out,
                     unsigned int* status, DegridArgs a)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    const uint32_t box_bytes = uint32_t(a.box_w) * a.box_h * 8u;
    float2* box = reinterpret_cast<float2*>(smem);
    float2* part = reinterpret_cast<float2*>(smem + box_bytes);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + box_bytes + kChunk * kMaxParts * 8);
    volatile int& give_up = *reinterpret_cast<volatile int*>(bar + 1);  // inside the dynamic region

    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        give_up = 0;
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s = a.s, s2 = s * s, P = a.parts;
    const int per = (s2 + P - 1) / P;
    const SmemRegion region{box};
    const uint32_t n_items = *n_aitems;
    uint32_t phase = 0;
    // persistent: cells in group-major order, so all SMs work on one slice of the table at a time
    for (uint32_t it = blockIdx.x; it < n_items; it += gridDim.x, phase ^= 1u) {
        const uint32_t cell = aitems[it];
        const uint32_t cnt = atile_count[cell];
        const uint32_t start = atile_start[cell];
        const int at = int(cell % uint32_t(a.natiles));
        const int x0 = (at % a.natx) * a.ta;
        const int y0 = (at / a.natx) * a.ta;
        if (threadIdx.x == 0) {
            // the box was last read through the generic proxy; order that before the TMA write
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(box_bytes)
                         : "memory");
            asm volatile(
                "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(box)),
                "l"(reinterpret_cast<uint64_t>(&tmap)), "r"(x0), "r"(y0), "r"(smem_u32(bar))
                : "memory");
        }
        if (!mbar_wait_bounded(bar, phase)) give_up = 1;
        __syncthreads();
        if (give_up) {
            if (threadIdx.x == 0) {
                atomicOr(status, 1u);
                mbar_wait_bounded(bar, phase);  // let the copy land before shared memory is released
            }
            return;
        }
        for (uint32_t c0 = 0; c0 < cnt; c0 += kChunk) {
            const int m = int(cnt - c0 < uint32_t(kChunk) ? cnt - c0 : uint32_t(kChunk));
            const int items = m * P;
            for (int w = warp; w < items; w += kWarps) {
                const int j = w / P, p = w - j * P;
                const uint32_t k = order[start + c0 + j];
                const int fx = iu[k] - a.support - x0;
                const int fy = iv[k] - y0;
                const int f_lo = p * per;
                const int f_hi = min(s2, f_lo + per);
                float2 v = walk<Tab>(ctab + coff[k], region, f_lo, f_hi, s, a.box_w, fx, fy, lane);
                v = warp_sum(v);
                if (lane == 0) part[j * kMaxParts + p] = v;
            }
            __syncthreads();
            for (int j = threadIdx.x; j < m; j += kThreads) {
                float2 v = part[j * kMaxParts];
                for (int p = 1; p < P; ++p) {
                    v.x += part[j * kMaxParts + p].x;
                    v.y += part[j * kMaxParts + p].y;
                }
                out[order[start + c0 + j]] = make_float2(v.x * a.c_scale, v.y * a.c_scale);
            }
            __syncthreads();  // the box and the partial sums are free again
        }
    }
}

template <class Tab>
__global__ void __launch_bounds__(256)
degrid_direct_kernel(const float2* __restrict__ grid, const typename Tab::elem* __restrict__ ctab,
                     const int32_t* __restrict__ iu, const int32_t* __restrict__ iv,
                     const int32_t* __restrict__ coff, const uint32_t* __restrict__ order,
                     const unsigned long long n_valid_max, const uint32_t* __restrict__ atile_start,
                     const uint32_t* __restrict__ atile_count, int n_atiles,
                     float2* __restrict__ out, DegridArgs a)
{
    // samples in anchor-sorted order; the valid ones are the first atile_start[last]+count[last]
    const uint32_t n_valid = atile_start[n_atiles - 1] + atile_count[n_atiles - 1];
    const uint64_t w = (blockIdx.x * uint64_t(blockDim.x) + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= n_valid || w >= n_valid_max) return;
    const uint32_t k = order[w];
    const int s = a.s;
    const GlobalRegion region{grid};
    float2 v = walk<Tab>(ctab + coff[k], region, 0, s * s, s, a.g_size, iu[k] - a.support, iv[k], lane);
    v = warp_sum(v);
    if (lane == 0) out[k] = make_float2(v.x * a.c_scale, v.y * a.c_scale);
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link against libcuda).
using EncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                              const cuuint64_t*, const cuuint32_t*, const cuuint32_t*,
                              CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                              CUtensorMapFloatOOBfill);

EncodeFn get_encode()
{
    static EncodeFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeFn>(p);
    });
    return fn;
}

template <class Tab>
tcv_status launch_staged(const tcv_plan* p, const float2* grid, const void* c, float c_scale,
                         float2* out, cudaStream_t st)
{
    const PlanGeom& g = p->g;
    EncodeFn enc = get_encode();
    if (!enc) return TCV_ERR_CUDA;
    // the checks cuTensorMapEncodeTiled and the TMA unit require, made explicitly
    if ((reinterpret_cast<uintptr_t>(grid) & 15) || (g.g_size & 1) || (g.box_w & 1) || g.box_w > 256 ||
        g.box_h > 256 || (g.ta & 1))
        return TCV_ERR_UNSUPPORTED;
    CUtensorMap map;
    const cuuint64_t dims[2] = {cuuint64_t(g.g_size), cuuint64_t(g.g_size)};
    const cuuint64_t strides[1] = {cuuint64_t(g.g_size) * 8};
    const cuuint32_t box[2] = {cuuint32_t(g.box_w), cuuint32_t(g.box_h)};
    const cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(&map, CU_TENSOR_MAP_DATA_TYPE_UINT64, 2, const_cast<float2*>(grid), dims, strides,
                     box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return TCV_ERR_CUDA;
    const size_t smem = size_t(g.box_w) * g.box_h * 8 + kChunk * kMaxParts * 8 + 16;
    static std::once_flag attr_once;
    static cudaError_t attr_err = cudaSuccess;
    std::call_once(attr_once, [] {
        attr_err = cudaFuncSetAttribute(degrid_staged_kernel<Tab>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        227 * 1024);
    });
    TCV_CUDA(attr_err);
    const int parts = g.degrid_parts < 1 ? 1 : (g.degrid_parts > kMaxParts ? kMaxParts : g.degrid_parts);
    DegridArgs a{g.support, g.s, g.g_size, g.ta, g.natx, g.natx * g.naty, g.box_w, g.box_h, parts, c_scale};
    int sms = 148, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    degrid_staged_kernel<Tab><<<sms, kThreads, smem, st>>>(
        map, static_cast<const typename Tab::elem*>(c), p->iu, p->iv, p->coff, p->avals[p->asel],
        p->atile_start, p->atile_count, p->aitems, p->n_aitems, out, p->status, a);
    TCV_CUDA(cudaGetLastError());
    return TCV_OK;
}

template <class Tab>
tcv_status launch_direct(const tcv_plan* p, const float2* grid, const void* c, float c_scale,
                         float2* out, cudaStream_t st)
{
    const PlanGeom& g = p->g;
    if (int64_t(g.g_size) * g.g_size >= (int64_t(1) << 31)) return TCV_ERR_UNSUPPORTED;
    DegridArgs a{g.support, g.s, g.g_size, g.ta, g.natx, g.natx * g.naty, g.box_w, g.box_h, 1, c_scale};
    const uint64_t threads = uint64_t(g.n) * 32;
    degrid_direct_kernel<Tab><<<unsigned((threads + 255) / 256), 256, 0, st>>>(
        grid, static_cast<const typename Tab::elem*>(c), p->iu, p->iv, p->coff, p->avals[p->asel],
        (unsigned long long)g.n, p->atile_start, p->atile_count, g.n_groups * g.natx * g.naty, out, a);
    TCV_CUDA(cudaGetLastError());
    return TCV_OK;
}

template <class Tab>
tcv_status launch(const tcv_plan* p, const float2* grid, const void* c, float c_scale, float2* out,
                  cudaStream_t st)
{
    if (p->g.n == 0) return TCV_OK;
    // samples rejected by the plan are not visited; their output is defined as zero
    TCV_CUDA(cudaMemsetAsync(out, 0, size_t(p->g.n) * sizeof(float2), st));
    if (p->g.degrid_mode == 0) {
        const tcv_status s = launch_staged<Tab>(p, grid, c, c_scale, out, st);
        if (s != TCV_ERR_UNSUPPORTED) return s;
    }
    return launch_direct<Tab>(p, grid, c, c_scale, out, st);
}

}  // namespace

tcv_status launch_degrid(const tcv_plan* p, const float2* grid, const void* c, int c_type,
                         float c_scale, float2* out, cudaStream_t st)
{
    switch (c_type) {
        case TCV_C_C64: return launch<TabC64>(p, grid, c, c_scale, out, st);
        case TCV_C_R32: return launch<TabR32>(p, grid, c, c_scale, out, st);
        case TCV_C_CBF16: return launch<TabCBF16>(p, grid, c, c_scale, out, st);
        case TCV_C_RBF16: return launch<TabRBF16>(p, grid, c, c_scale, out, st);
        case TCV_C_CF16: return launch<TabCF16>(p, grid, c, c_scale, out, st);
        case TCV_C_RF16: return launch<TabRF16>(p, grid, c, c_scale, out, st);
        default: return TCV_ERR_ARG;
    }
}

}  // namespace tcv
