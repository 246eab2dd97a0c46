// tcv_pipe.cu -- the TMA pipeline kernels for gridding and degridding (prepared tables).
//
// Same binning plan and tiles as tcv_grid.cu: one CTA per 64 x 64 grid tile walks the samples
// whose footprint overlaps the tile, in (w-plane, oversampling kernel) order.  What changes is
// how the table reaches the SMs.  The table is prepared once in a padded layout
// [kernel][row][col] with rows padded to a 16-byte pitch, which makes it a 3-D TMA tensor
// (x = column, y = row, z = kernel).  A producer warp issues, for each sample, one
// cp.async.bulk.tensor.3d load of the 64-row x (64 + A)-column window of that sample's kernel that
// lies over the tile, into a ring of shared-memory stages with full/empty mbarriers.  The TMA
// unit zero-fills the parts of the window outside the footprint (negative or >= sSize rows and
// columns), so the eight consumer warps need no bounds tests: each lane reads its 16 table
// values from shared memory and issues packed FP32x2 FMAs.  A = 16 / entry size: the window's x
// origin is rounded down to a 16-byte boundary (the TMA alignment rule) and each lane indexes
// `shift` entries further on.
//
// Gridding: accumulators in registers (one grid point x 16 rows per lane), added into the grid
// once at the end (every point has one owner: no atomics, deterministic).
// Degridding (the adjoint): the lane holds its 16 grid points in registers and forms partial
// dot products; each warp reduces its partial with shuffles, the producer sums the eight warp
// partials of a (tile, sample) in fixed order into a per-sample slot, and a final kernel adds a
// sample's slots in fixed tile order.  Results do not depend on scheduling.
//
// Every mbarrier wait is bounded by a timer; on timeout the kernel sets the plan's status word,
// stops issuing, waits (bounded) for its own copies in flight and returns.
#include "tcv_internal.cuh"

#include <cuda.h>
#include <mutex>

namespace tcv {
namespace {

constexpr int kTileW = 64;
constexpr int kTileH = 64;
constexpr int kRows = 16;                                    // rows per consumer lane
constexpr int kConsumerWarps = (kTileW / 32) * (kTileH / kRows);  // 8
constexpr int kThreads = (kConsumerWarps + 1) * 32;           // + 1 producer warp
constexpr unsigned long long kWaitNs = 2000000000ull;

struct PipeArgs {
    int support, s, g_size, ntx, ntiles, group, max_tiles;
    int bx;            // window width in entries (64 + A)
    int align;         // A: entries per 16 bytes
    int stages;
    uint32_t stage_bytes;
    float c_scale;
};

struct StageMeta {
    float dr, di;      // sample value (gridding)
    int dx0, dy0;      // footprint column / row of the tile's first column / row
    int shift;         // dx0 - (TMA x origin)
    uint32_t k;        // sample index
    int slot;          // slot of this tile among the sample's tiles (degridding)
    int pad;
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

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait; false if the timer ran out or another thread already gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag)
{
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    while (!mbar_try_wait(bar, parity)) {
        if (*abort_flag) return false;
        if (global_ns() - t0 > kWaitNs) {
            *abort_flag = 1;
            return false;
        }
    }
    return true;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

template <class Form>
struct Pipe;

// Per-form consumer arithmetic.  `Entry` is the shared-memory element type.
struct PipeC64 {
    using Entry = float2;
    static constexpr int kAlign = 2;
    static constexpr CUtensorMapDataType kTmaType = CU_TENSOR_MAP_DATA_TYPE_UINT64;
    __device__ __forceinline__ static float2 get(const Entry* p) { return *p; }
};
struct PipeR32 {
    using Entry = float;
    static constexpr int kAlign = 4;
    static constexpr CUtensorMapDataType kTmaType = CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    __device__ __forceinline__ static float get(const Entry* p) { return *p; }
};
struct PipeCBF16 {
    using Entry = uint32_t;
    static constexpr int kAlign = 4;
    static constexpr CUtensorMapDataType kTmaType = CU_TENSOR_MAP_DATA_TYPE_UINT32;
    __device__ __forceinline__ static float2 get(const Entry* p)
    {
        const uint32_t u = *p;
        return make_float2(__uint_as_float(u << 16), __uint_as_float(u & 0xffff0000u));
    }
};
struct PipeRBF16 {
    using Entry = uint16_t;
    static constexpr int kAlign = 8;
    static constexpr CUtensorMapDataType kTmaType = CU_TENSOR_MAP_DATA_TYPE_UINT16;
    __device__ __forceinline__ static float get(const Entry* p) { return __uint_as_float(uint32_t(*p) << 16); }
};
struct PipeCF16 {
    using Entry = __half2;
    static constexpr int kAlign = 4;
    static constexpr CUtensorMapDataType kTmaType = CU_TENSOR_MAP_DATA_TYPE_UINT32;
    __device__ __forceinline__ static float2 get(const Entry* p) { return __half22float2(*p); }
};
struct PipeRF16 {
    using Entry = __half;
    static constexpr int kAlign = 8;
    static constexpr CUtensorMapDataType kTmaType = CU_TENSOR_MAP_DATA_TYPE_UINT16;
    __device__ __forceinline__ static float get(const Entry* p) { return __half2float(*p); }
};

// complex table: split accumulators a1 += (x.re, x.re) * c, a2 += (x.im, x.im) * c, so every
// product is one packed FMA on the table value as loaded; combined at the end as
// re = a1.x - a2.y, im = a1.y + a2.x.
__device__ __forceinline__ void mac_split(float2& a1, float2& a2, const float2 xr, const float2 xi, const float2 c)
{
    a1 = __ffma2_rn(xr, c, a1);
    a2 = __ffma2_rn(xi, c, a2);
}

template <class F, bool kDegrid>
__global__ void __launch_bounds__(kThreads, 2)
pipe_kernel(const __grid_constant__ CUtensorMap cmap, const float2* __restrict__ data,
            const int32_t* __restrict__ iu, const int32_t* __restrict__ iv,
            const int32_t* __restrict__ coff, const uint32_t* __restrict__ order,
            const uint32_t* __restrict__ tile_start, const uint32_t* __restrict__ tile_count,
            const uint32_t* __restrict__ items, const uint32_t* __restrict__ group_start,
            float2* __restrict__ grid, float2* __restrict__ slots, unsigned int* status, PipeArgs a)
{
    using Entry = typename F::Entry;
    constexpr bool kComplex = sizeof(decltype(F::get(nullptr))) == 8;
    extern __shared__ __align__(1024) unsigned char smem[];
    const uint32_t i0 = group_start[a.group] + blockIdx.x, i1 = group_start[a.group + 1];
    if (i0 >= i1) return;
    const int NS = a.stages;

    unsigned char* p = smem + size_t(NS) * a.stage_bytes;
    StageMeta* meta = reinterpret_cast<StageMeta*>(p);
    p += NS * sizeof(StageMeta);
    float2* part = reinterpret_cast<float2*>(p);  // [NS][kConsumerWarps]
    p += NS * kConsumerWarps * sizeof(float2);
    uint64_t* full = reinterpret_cast<uint64_t*>(p);
    uint64_t* empty = full + NS;
    volatile int* abort_flag = reinterpret_cast<volatile int*>(empty + NS);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int i = 0; i < NS; ++i) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&full[i])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&empty[i])), "r"(kConsumerWarps)
                         : "memory");
        }
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    const int s = a.s;
    if (warp == kConsumerWarps) {
        // ---------------- producer warp ----------------
        // the stage ring runs on across this CTA's cells: sample jj of the CTA uses stage jj % NS
        uint32_t issued = 0;
        bool ok = true;
        for (uint32_t it = i0; it < i1 && ok; it += gridDim.x) {
          const uint32_t cell = items[it];
          const uint32_t cnt = tile_count[cell];
          const uint32_t start = tile_start[cell];
          const int tile = int(cell % uint32_t(a.ntiles));
          const int tx = tile % a.ntx, ty = tile / a.ntx;
          const int tx0g = tx * kTileW, ty0g = ty * kTileH;
          for (uint32_t base = 0; base < cnt && ok; base += 32) {
            const uint32_t j = base + lane;
            uint32_t k = 0;
            int fx = 0, fy = 0, co = 0;
            float2 d = make_float2(0.f, 0.f);
            if (j < cnt) {
                k = order[start + j];
                fx = iu[k] - a.support;
                fy = iv[k];
                co = coff[k];
                if (!kDegrid) d = data[k];
            }
            const int m = int(cnt - base < 32u ? cnt - base : 32u);
            for (int i = 0; i < m; ++i) {
                const uint32_t kk = __shfl_sync(0xffffffffu, k, i);
                const int ffx = __shfl_sync(0xffffffffu, fx, i);
                const int ffy = __shfl_sync(0xffffffffu, fy, i);
                const int cco = __shfl_sync(0xffffffffu, co, i);
                const float ddr = __shfl_sync(0xffffffffu, d.x, i);
                const float ddi = __shfl_sync(0xffffffffu, d.y, i);
                if (lane == 0) {
                    const uint32_t jj = issued;  // samples are issued strictly in order
                    const int st = int(jj % NS);
                    const uint32_t round = jj / NS;
                    if (!mbar_wait(&empty[st], (round & 1) ^ 1, abort_flag)) {
                        ok = false;
                    } else {
                        if (kDegrid && jj >= uint32_t(NS)) {
                            // the stage's previous sample is done by every consumer warp
                            float2 v = part[st * kConsumerWarps];
#pragma unroll
                            for (int w = 1; w < kConsumerWarps; ++w) {
                                v.x += part[st * kConsumerWarps + w].x;
                                v.y += part[st * kConsumerWarps + w].y;
                            }
                            slots[size_t(meta[st].k) * a.max_tiles + meta[st].slot] = v;
                        }
                        const int dx0 = tx0g - ffx, dy0 = ty0g - ffy;
                        const int x0 = dx0 >= 0 ? dx0 - dx0 % F::kAlign : -((-dx0 + F::kAlign - 1) / F::kAlign) * F::kAlign;
                        StageMeta mt;
                        mt.dr = ddr * a.c_scale;
                        mt.di = ddi * a.c_scale;
                        mt.dx0 = dx0;
                        mt.dy0 = dy0;
                        mt.shift = dx0 - x0;
                        mt.k = kk;
                        const int sx0 = ffx / kTileW, sx1 = (ffx + s - 1) / kTileW, sy0 = ffy / kTileH;
                        mt.slot = (ty - sy0) * (sx1 - sx0 + 1) + (tx - sx0);
                        mt.pad = 0;
                        meta[st] = mt;
                        const int kid = cco / (s * s);
                        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(&full[st])),
                                     "r"(a.stage_bytes)
                                     : "memory");
                        asm volatile(
                            "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                            " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(smem + size_t(st) * a.stage_bytes)),
                            "l"(reinterpret_cast<uint64_t>(&cmap)), "r"(x0), "r"(dy0), "r"(kid),
                            "r"(smem_u32(&full[st]))
                            : "memory");
                        ++issued;
                    }
                }
                ok = __shfl_sync(0xffffffffu, ok, 0);
                if (!ok) break;
            }
          }
        }
        if (lane == 0) {
            if (ok && kDegrid) {
                // finish the last samples once every consumer warp is done with them
                const uint32_t first = issued > uint32_t(NS) ? issued - NS : 0;
                for (uint32_t jj = first; jj < issued && ok; ++jj) {
                    const int st = int(jj % NS);
                    if (!mbar_wait(&empty[st], (jj / NS) & 1, abort_flag)) {
                        ok = false;
                        break;
                    }
                    float2 v = part[st * kConsumerWarps];
#pragma unroll
                    for (int w = 1; w < kConsumerWarps; ++w) {
                        v.x += part[st * kConsumerWarps + w].x;
                        v.y += part[st * kConsumerWarps + w].y;
                    }
                    slots[size_t(meta[st].k) * a.max_tiles + meta[st].slot] = v;
                }
            }
            if (!ok) {
                atomicOr(status, 1u);
                // let copies already issued land before the CTA's shared memory is released
                for (uint32_t jj = (issued > uint32_t(NS) ? issued - NS : 0); jj < issued; ++jj) {
                    const uint64_t t0 = global_ns();
                    while (!mbar_try_wait(&full[jj % NS], (jj / NS) & 1) && global_ns() - t0 < kWaitNs) {
                    }
                }
            }
        }
        return;
    }

    // ---------------- consumer warps ----------------
    const int band = warp % (kTileW / 32), rg = warp / (kTileW / 32);
    const int col = band * 32 + lane;           // tile column of this lane
    const int row0 = rg * kRows;                // first tile row of this warp
    uint32_t jg = 0;                            // this CTA's running sample index
    for (uint32_t it = i0; it < i1; it += gridDim.x) {
        const uint32_t cell = items[it];
        const uint32_t cnt = tile_count[cell];
        const int tile = int(cell % uint32_t(a.ntiles));
        const int tx = tile % a.ntx, ty = tile / a.ntx;
        const int gx = tx * kTileW + col;
        const int gy0 = ty * kTileH + row0;

        // gridding: accumulators; degridding: the grid values (as needed by the packed FMAs)
        float2 acc1[kRows], acc2[kRows];
        if (!kDegrid) {
#pragma unroll
            for (int r = 0; r < kRows; ++r) acc1[r] = acc2[r] = make_float2(0.f, 0.f);
        } else {
#pragma unroll
            for (int r = 0; r < kRows; ++r) {
                float2 g = make_float2(0.f, 0.f);
                if (gx < a.g_size && gy0 + r < a.g_size) g = grid[size_t(gy0 + r) * a.g_size + gx];
                if constexpr (kComplex) {
                    acc1[r] = make_float2(g.x, g.x);  // (g.re, g.re)
                    acc2[r] = make_float2(g.y, g.y);  // (g.im, g.im)
                } else {
                    acc1[r] = g;
                }
            }
        }

        for (uint32_t j = 0; j < cnt; ++j, ++jg) {
            const int st = int(jg % NS);
            if (!mbar_wait(&full[st], (jg / NS) & 1, abort_flag)) return;
            const StageMeta mt = meta[st];
            const bool rows_hit = mt.dy0 + row0 < s && mt.dy0 + row0 + kRows > 0;
            const bool cols_hit = mt.dx0 + band * 32 < s && mt.dx0 + band * 32 + 32 > 0;
            const Entry* sp = reinterpret_cast<const Entry*>(smem + size_t(st) * a.stage_bytes) + row0 * a.bx + col + mt.shift;
            if (!kDegrid) {
                if (rows_hit && cols_hit) {
                    const float2 dr2 = make_float2(mt.dr, mt.dr), di2 = make_float2(mt.di, mt.di);
                    const float2 dv = make_float2(mt.dr, mt.di);
#pragma unroll
                    for (int r = 0; r < kRows; ++r) {
                        if constexpr (kComplex) {
                            mac_split(acc1[r], acc2[r], dr2, di2, F::get(sp + r * a.bx));
                        } else {
                            const float c = F::get(sp + r * a.bx);
                            acc1[r] = __ffma2_rn(dv, make_float2(c, c), acc1[r]);
                        }
                    }
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(&empty[st]);
            } else {
                float2 p1 = make_float2(0.f, 0.f), p2 = make_float2(0.f, 0.f);
                if (rows_hit && cols_hit) {
#pragma unroll
                    for (int r = 0; r < kRows; ++r) {
                        if constexpr (kComplex) {
                            mac_split(p1, p2, acc1[r], acc2[r], F::get(sp + r * a.bx));
                        } else {
                            const float c = F::get(sp + r * a.bx);
                            p1 = __ffma2_rn(acc1[r], make_float2(c, c), p1);
                        }
                    }
                }
                float2 v = kComplex ? make_float2(p1.x - p2.y, p1.y + p2.x) : p1;
#pragma unroll
                for (int o = 16; o; o >>= 1) {
                    v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
                    v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
                }
                if (lane == 0) {
                    part[st * kConsumerWarps + warp] = v;
                    mbar_arrive(&empty[st]);
                }
            }
        }

        if (!kDegrid && gx < a.g_size) {
#pragma unroll
            for (int r = 0; r < kRows; ++r) {
                const int gy = gy0 + r;
                if (gy < a.g_size) {
                    float2* gp = grid + size_t(gy) * a.g_size + gx;
                    float2 v = *gp;
                    if constexpr (kComplex) {
                        v.x += acc1[r].x - acc2[r].y;
                        v.y += acc1[r].y + acc2[r].x;
                    } else {
                        v.x += acc1[r].x;
                        v.y += acc1[r].y;
                    }
                    *gp = v;
                }
            }
        }
    }
}

// out[k] = c_scale x the sum of the sample's tile slots in tile order (0 for rejected samples).
__global__ void slot_reduce_kernel(const float2* __restrict__ slots, const uint16_t* __restrict__ ntl, int64_t n,
                                   int max_tiles, float c_scale, float2* __restrict__ out)
{
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int nt = ntl[k];  // tiles of the sample's footprint, in the plan's order; 0 = left out
    float2 v = make_float2(0.f, 0.f);
    const float2* sl = slots + k * max_tiles;
    for (int t = 0; t < nt; ++t) {
        v.x += sl[t].x;
        v.y += sl[t].y;
    }
    out[k] = make_float2(v.x * c_scale, v.y * c_scale);
}

// reference layout -> padded layout [kernel][row][pitch], converting the storage type
template <typename T>
__global__ void pad_kernel(const T* __restrict__ in, T* __restrict__ out, int64_t nk, int s, int pitch)
{
    const int64_t total = nk * s * int64_t(pitch);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int c = int(i % pitch);
        const int64_t kr = i / pitch;  // kernel * s + row
        out[i] = c < s ? in[kr * s + c] : T{};
    }
}

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

template <class F, bool kDegrid>
cudaError_t set_smem_attr(size_t bytes)
{
    static std::once_flag once;
    static cudaError_t err = cudaSuccess;
    std::call_once(once, [] {
        err = cudaFuncSetAttribute(pipe_kernel<F, kDegrid>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    });
    (void)bytes;
    return err;
}

template <class F, bool kDegrid>
tcv_status launch_pipe(const tcv_plan* p, const float2* data, const void* table, float c_scale, float2* grid,
                       float2* out, cudaStream_t st)
{
    const PlanGeom& g = p->g;
    if (g.n == 0) return TCV_OK;
    if (g.tw != kTileW || g.th != kTileH) return TCV_ERR_UNSUPPORTED;
    const int64_t s2 = int64_t(g.s) * g.s;
    if (g.c_len % s2) return TCV_ERR_UNSUPPORTED;
    const int64_t nk = g.c_len / s2;
    constexpr int esize = int(sizeof(typename F::Entry));
    const int pitch = (g.s + F::kAlign - 1) / F::kAlign * F::kAlign;
    if ((reinterpret_cast<uintptr_t>(table) & 15)) return TCV_ERR_UNSUPPORTED;
    EncodeFn enc = get_encode();
    if (!enc) return TCV_ERR_CUDA;
    PipeArgs a{};
    a.support = g.support;
    a.s = g.s;
    a.g_size = g.g_size;
    a.ntx = g.ntx;
    a.ntiles = g.ntx * g.nty;
    a.max_tiles = g.max_tiles;
    a.align = F::kAlign;
    a.bx = kTileW + F::kAlign;
    a.stage_bytes = uint32_t(a.bx) * kTileH * esize;
    a.c_scale = c_scale;
    // two CTAs per SM: as many stages as fit in half of the 228 KB of shared memory
    const size_t extra_per_stage = sizeof(StageMeta) + kConsumerWarps * sizeof(float2) + 16;
    int stages = int((113 * 1024 - 64) / (a.stage_bytes + extra_per_stage));
    stages = stages < 2 ? 2 : (stages > 8 ? 8 : stages);
    a.stages = stages;
    const size_t smem = size_t(stages) * (a.stage_bytes + extra_per_stage) + 64;

    CUtensorMap map;
    const cuuint64_t dims[3] = {cuuint64_t(g.s), cuuint64_t(g.s), cuuint64_t(nk)};
    const cuuint64_t strides[2] = {cuuint64_t(pitch) * esize, cuuint64_t(pitch) * esize * g.s};
    const cuuint32_t box[3] = {cuuint32_t(a.bx), cuuint32_t(kTileH), 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = enc(&map, F::kTmaType, 3, const_cast<void*>(table), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return TCV_ERR_CUDA;
    TCV_CUDA((set_smem_attr<F, kDegrid>(smem)));
    int sms = 148, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // one persistent launch per plane group (two CTAs per SM), in group order
    for (int grp = 0; grp < g.n_groups; ++grp) {
        a.group = grp;
        pipe_kernel<F, kDegrid><<<2 * sms, kThreads, smem, st>>>(
            map, data, p->iu, p->iv, p->coff, p->vals[p->sel], p->tile_start, p->tile_count, p->items,
            p->group_start, grid, p->slots, p->status, a);
        TCV_CUDA(cudaGetLastError());
    }
    if (kDegrid) return slot_reduce(p, c_scale, out, st);
    return TCV_OK;
}

template <bool kDegrid>
tcv_status dispatch(const tcv_plan* p, const float2* data, const void* table, int c_type, float c_scale,
                    float2* grid, float2* out, cudaStream_t st)
{
    switch (c_type) {
        case TCV_C_C64: return launch_pipe<PipeC64, kDegrid>(p, data, table, c_scale, grid, out, st);
        case TCV_C_R32: return launch_pipe<PipeR32, kDegrid>(p, data, table, c_scale, grid, out, st);
        case TCV_C_CBF16: return launch_pipe<PipeCBF16, kDegrid>(p, data, table, c_scale, grid, out, st);
        case TCV_C_RBF16: return launch_pipe<PipeRBF16, kDegrid>(p, data, table, c_scale, grid, out, st);
        case TCV_C_CF16: return launch_pipe<PipeCF16, kDegrid>(p, data, table, c_scale, grid, out, st);
        case TCV_C_RF16: return launch_pipe<PipeRF16, kDegrid>(p, data, table, c_scale, grid, out, st);
        default: return TCV_ERR_ARG;
    }
}

}  // namespace

tcv_status slot_reduce(const tcv_plan* p, float c_scale, float2* out, cudaStream_t st)
{
    const PlanGeom& g = p->g;
    if (g.n == 0) return TCV_OK;
    slot_reduce_kernel<<<unsigned((g.n + 255) / 256), 256, 0, st>>>(p->slots, p->ntl, g.n, g.max_tiles, c_scale, out);
    TCV_CUDA(cudaGetLastError());
    return TCV_OK;
}

tcv_status launch_grid_pipe(const tcv_plan* p, const float2* data, const void* table, int c_type, float c_scale,
                            float2* grid, cudaStream_t st)
{
    return dispatch<false>(p, data, table, c_type, c_scale, grid, nullptr, st);
}

tcv_status launch_degrid_pipe(const tcv_plan* p, const float2* grid, const void* table, int c_type,
                              float c_scale, float2* out, cudaStream_t st)
{
    // the degridding kernel reads the grid; c_scale (FP16 forms) is applied to each sample's sum
    return dispatch<true>(p, nullptr, table, c_type, c_scale, const_cast<float2*>(grid), out, st);
}

size_t padded_table_bytes(int64_t c_len, int s, int c_type)
{
    const size_t es = tcv_ctype_bytes(c_type);
    if (!es || s < 1) return 0;
    const int64_t s2 = int64_t(s) * s;
    if (c_len % s2) return 0;
    const int align = int(16 / es);
    const int64_t pitch = (s + align - 1) / align * align;
    return size_t(c_len / s2) * size_t(s) * size_t(pitch) * es;
}

tcv_status pad_table(const void* in, int64_t c_len, int s, int c_type, void* out, cudaStream_t st)
{
    const size_t es = tcv_ctype_bytes(c_type);
    const int64_t s2 = int64_t(s) * s;
    if (!es || c_len % s2) return TCV_ERR_ARG;
    const int align = int(16 / es);
    const int pitch = (s + align - 1) / align * align;
    const int64_t nk = c_len / s2;
    const int blocks = 148 * 32;
    switch (es) {
        case 8: pad_kernel<uint64_t><<<blocks, 256, 0, st>>>(static_cast<const uint64_t*>(in), static_cast<uint64_t*>(out), nk, s, pitch); break;
        case 4: pad_kernel<uint32_t><<<blocks, 256, 0, st>>>(static_cast<const uint32_t*>(in), static_cast<uint32_t*>(out), nk, s, pitch); break;
        case 2: pad_kernel<uint16_t><<<blocks, 256, 0, st>>>(static_cast<const uint16_t*>(in), static_cast<uint16_t*>(out), nk, s, pitch); break;
        default: return TCV_ERR_ARG;
    }
    TCV_CUDA(cudaGetLastError());
    return TCV_OK;
}

}  // namespace tcv

using namespace tcv;

extern "C" {

size_t tcv_table_bytes(int64_t c_len, int support, int c_type)
{
    const size_t es = tcv_ctype_bytes(c_type);
    if (!es || c_len < 0 || support < 0 || (c_type & TCV_C_PADDED && c_type & TCV_C_PAIRED)) return 0;
    if (c_type & TCV_C_PADDED) return padded_table_bytes(c_len, 2 * support + 1, c_type & 0xff);
    if (c_type & TCV_C_PAIRED) return paired_table_bytes(c_len, 2 * support + 1, c_type & 0xff);
    return size_t(c_len) * es;
}

tcv_status tcv_prepare_table(const float* d_c64, int64_t c_len, int support, int c_type, void* d_out,
                             float* c_scale_out, int64_t* imag_nonzero_out, void* stream)
{
    const int base = c_type & 0xff;
    const bool paired = (c_type & TCV_C_PAIRED) != 0;
    if (!d_c64 || !d_out || c_len <= 0 || support < 0 || tcv_ctype_bytes(base) == 0) return TCV_ERR_ARG;
    if (paired == ((c_type & TCV_C_PADDED) != 0) && (c_type & (TCV_C_PADDED | TCV_C_PAIRED))) return TCV_ERR_ARG;
    const int s = 2 * support + 1;
    if ((paired ? paired_table_bytes(c_len, s, base) : padded_table_bytes(c_len, s, base)) == 0) return TCV_ERR_ARG;
    if ((reinterpret_cast<uintptr_t>(d_out) & 15)) return TCV_ERR_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    auto layout = [&](const void* in) {
        return paired ? pair_table(in, c_len, s, base, d_out, st) : pad_table(in, c_len, s, base, d_out, st);
    };
    if (base == TCV_C_C64) {
        if (c_scale_out) *c_scale_out = 1.0f;
        if (imag_nonzero_out) *imag_nonzero_out = 0;
        return layout(d_c64);
    }
    void* tmp = nullptr;
    TCV_CUDA(cudaMalloc(&tmp, size_t(c_len) * tcv_ctype_bytes(base) + 16));
    tcv_status r = tcv_convert_c(d_c64, c_len, base, tmp, c_scale_out, imag_nonzero_out, stream);
    if (r == TCV_OK) r = layout(tmp);
    const cudaError_t e = cudaStreamSynchronize(st);
    cudaFree(tmp);
    if (r != TCV_OK) return r;
    TCV_CUDA(e);
    return TCV_OK;
}

}  // extern "C"
