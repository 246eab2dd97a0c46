// tcv_grid.cu -- gridding (Benchmark::gridKernel, attic/tConvolveMPI/Benchmark.cc:125-155).
//
// Output-stationary tiles.  One CTA owns a 64 x 64 tile of the grid; each of its 8 warps owns a
// 32-column x RH-row block with one accumulator per point held in registers (lane = column).
// The CTA walks the tile's sample list (from the plan, ordered by w-plane/oversampling kernel),
// staging sample records in shared memory; for each sample a warp whose block meets the
// footprint reads the table rows it needs (32 consecutive entries per row: one coalesced
// 256-byte load for the complex64 table) and accumulates data * C into its registers.  When the
// list is done the tile is added into the grid with coalesced read-modify-writes.
//
// Every grid point has exactly one owner thread, so there are no atomics and the result is the
// same on every run.  HBM traffic is the table entries each sample needs plus one read and one
// write of each touched tile, instead of a read and a write of the grid per update.
#include "tcv_internal.cuh"

namespace tcv {
namespace {

constexpr int kTileW = 64;
constexpr int kTileH = 64;
constexpr int kRowsPerWarp = 16;
constexpr int kWarps = (kTileW / 32) * (kTileH / kRowsPerWarp);
constexpr int kThreads = kWarps * 32;
constexpr int kChunk = kThreads;  // samples staged per round

struct GridArgs {
    int support, s, g_size, ntx, ntiles, group;
    float c_scale;
};

template <class Tab>
__global__ void __launch_bounds__(kThreads, 3)
grid_tile_kernel(const float2* __restrict__ data, const typename Tab::elem* __restrict__ ctab,
                 const int32_t* __restrict__ iu, const int32_t* __restrict__ iv,
                 const int32_t* __restrict__ coff, const uint32_t* __restrict__ order,
                 const uint32_t* __restrict__ tile_start, const uint32_t* __restrict__ tile_count,
                 const uint32_t* __restrict__ items, const uint32_t* __restrict__ group_start,
                 float2* __restrict__ grid, GridArgs a)
{
    __shared__ float4 sm_rec[kChunk];  // (data.re, data.im, first column, first row)
    __shared__ int sm_coff[kChunk];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s = a.s;
    // persistent: this CTA takes every gridDim.x-th non-empty cell of the group
    const uint32_t i1 = group_start[a.group + 1];
    for (uint32_t it = group_start[a.group] + blockIdx.x; it < i1; it += gridDim.x) {
        const uint32_t cell = items[it];
        const uint32_t cnt = tile_count[cell];
        const uint32_t start = tile_start[cell];
        const int tile = int(cell % uint32_t(a.ntiles));
        const int tx = tile % a.ntx, ty = tile / a.ntx;
        const int bx0 = tx * kTileW + (warp % (kTileW / 32)) * 32;  // first column of this warp
        const int gx = bx0 + lane;
        const int gy0 = ty * kTileH + (warp / (kTileW / 32)) * kRowsPerWarp;

        float2 acc[kRowsPerWarp];
#pragma unroll
        for (int r = 0; r < kRowsPerWarp; ++r) acc[r] = make_float2(0.f, 0.f);

        for (uint32_t base = 0; base < cnt; base += kChunk) {
            const int m = int(cnt - base < uint32_t(kChunk) ? cnt - base : uint32_t(kChunk));
            __syncthreads();
            if (threadIdx.x < m) {
                const uint32_t k = order[start + base + threadIdx.x];
                const float2 d = data[k];
                sm_rec[threadIdx.x] = make_float4(d.x * a.c_scale, d.y * a.c_scale,
                                                  __int_as_float(iu[k] - a.support), __int_as_float(iv[k]));
                sm_coff[threadIdx.x] = coff[k];
            }
            __syncthreads();
            for (int j = 0; j < m; ++j) {
                const float4 q = sm_rec[j];
                const int fx = __float_as_int(q.z), fy = __float_as_int(q.w);
                const int dy0 = gy0 - fy;  // footprint row of this warp's first row
                if (dy0 >= s || dy0 + kRowsPerWarp <= 0) continue;   // warp-uniform
                if (fx > bx0 + 31 || fx + s <= bx0) continue;          // warp-uniform
                const int dx = gx - fx;
                const bool colok = unsigned(dx) < unsigned(s);
                const float2 dv = make_float2(q.x, q.y);
                const typename Tab::elem* cp = ctab + (sm_coff[j] + dy0 * s + dx);
                if (dy0 >= 0 && dy0 + kRowsPerWarp <= s) {
                    // every row of the block is inside the footprint: only the column test remains
                    if (colok) {
#pragma unroll
                        for (int r = 0; r < kRowsPerWarp; ++r) cmac<Tab::kReal>(acc[r], dv, Tab::load(cp + r * s));
                    }
                } else {
#pragma unroll
                    for (int r = 0; r < kRowsPerWarp; ++r) {
                        if (colok && unsigned(dy0 + r) < unsigned(s)) {
                            const float2 c = Tab::load(cp + r * s);
                            cmac<Tab::kReal>(acc[r], dv, c);
                        }
                    }
                }
            }
        }
        if (gx < a.g_size) {
#pragma unroll
            for (int r = 0; r < kRowsPerWarp; ++r) {
                const int gy = gy0 + r;
                if (gy < a.g_size) {
                    float2* gp = grid + (size_t(gy) * a.g_size + gx);
                    float2 v = *gp;
                    v.x += acc[r].x;
                    v.y += acc[r].y;
                    *gp = v;
                }
            }
        }
    }
}

// Degridding on the gridding plan (the adjoint of grid_tile_kernel).  A lane holds its 16 grid
// points in registers; for each sample of the cell a warp whose block meets the footprint forms
// the partial dot product of its block with the table, reduces it with shuffles, and the CTA
// adds its 8 warp partials in warp order into the sample's slot for this tile.  A final pass
// (slot_reduce_kernel) adds each sample's tile slots in tile order: no atomics, deterministic.
template <class Tab>
__global__ void __launch_bounds__(kThreads, 3)
degrid_tile_kernel(const float2* __restrict__ grid, const typename Tab::elem* __restrict__ ctab,
                   const int32_t* __restrict__ iu, const int32_t* __restrict__ iv,
                   const int32_t* __restrict__ coff, const uint32_t* __restrict__ order,
                   const uint32_t* __restrict__ tile_start, const uint32_t* __restrict__ tile_count,
                   const uint32_t* __restrict__ items, const uint32_t* __restrict__ group_start,
                   float2* __restrict__ slots, int max_tiles, GridArgs a)
{
    __shared__ int4 sm_rec[kChunk];              // (sample, first column, first row, cOffset)
    __shared__ float2 sm_part[kChunk][kWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s = a.s;
    const uint32_t i1 = group_start[a.group + 1];
    for (uint32_t it = group_start[a.group] + blockIdx.x; it < i1; it += gridDim.x) {
        const uint32_t cell = items[it];
        const uint32_t cnt = tile_count[cell];
        const uint32_t start = tile_start[cell];
        const int tile = int(cell % uint32_t(a.ntiles));
        const int tx = tile % a.ntx, ty = tile / a.ntx;
        const int bx0 = tx * kTileW + (warp % (kTileW / 32)) * 32;
        const int gx = bx0 + lane;
        const int gy0 = ty * kTileH + (warp / (kTileW / 32)) * kRowsPerWarp;
        float2 gv[kRowsPerWarp];
#pragma unroll
        for (int r = 0; r < kRowsPerWarp; ++r)
            gv[r] = (gx < a.g_size && gy0 + r < a.g_size) ? grid[size_t(gy0 + r) * a.g_size + gx] : make_float2(0.f, 0.f);

        for (uint32_t base = 0; base < cnt; base += kChunk) {
            const int m = int(cnt - base < uint32_t(kChunk) ? cnt - base : uint32_t(kChunk));
            __syncthreads();
            if (threadIdx.x < m) {
                const uint32_t k = order[start + base + threadIdx.x];
                sm_rec[threadIdx.x] = make_int4(int(k), iu[k] - a.support, iv[k], coff[k]);
            }
            __syncthreads();
            for (int j = 0; j < m; ++j) {
                const int4 q = sm_rec[j];
                const int fx = q.y, fy = q.z;
                const int dy0 = gy0 - fy;
                float2 v = make_float2(0.f, 0.f);
                if (!(dy0 >= s || dy0 + kRowsPerWarp <= 0) && !(fx > bx0 + 31 || fx + s <= bx0)) {  // warp-uniform
                    const int dx = gx - fx;
                    const bool colok = unsigned(dx) < unsigned(s);
                    const typename Tab::elem* cp = ctab + (q.w + dy0 * s + dx);
                    // four independent partial sums keep the FMA chains short
                    float2 pv[4] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f),
                                    make_float2(0.f, 0.f)};
                    if (dy0 >= 0 && dy0 + kRowsPerWarp <= s) {
                        if (colok) {
#pragma unroll
                            for (int r = 0; r < kRowsPerWarp; ++r) cmac<Tab::kReal>(pv[r & 3], gv[r], Tab::load(cp + r * s));
                        }
                    } else {
#pragma unroll
                        for (int r = 0; r < kRowsPerWarp; ++r) {
                            if (colok && unsigned(dy0 + r) < unsigned(s)) {
                                const float2 c = Tab::load(cp + r * s);
                                cmac<Tab::kReal>(pv[r & 3], gv[r], c);
                            }
                        }
                    }
                    v = make_float2((pv[0].x + pv[1].x) + (pv[2].x + pv[3].x), (pv[0].y + pv[1].y) + (pv[2].y + pv[3].y));
#pragma unroll
                    for (int o = 16; o; o >>= 1) {
                        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
                        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
                    }
                }
                if (lane == 0) sm_part[j][warp] = v;
            }
            __syncthreads();
            if (threadIdx.x < m) {
                const int4 q = sm_rec[threadIdx.x];
                float2 v = sm_part[threadIdx.x][0];
#pragma unroll
                for (int w = 1; w < kWarps; ++w) {
                    v.x += sm_part[threadIdx.x][w].x;
                    v.y += sm_part[threadIdx.x][w].y;
                }
                const int sx0 = q.y / kTileW, sx1 = (q.y + s - 1) / kTileW, sy0 = q.z / kTileH;
                const int slot = (ty - sy0) * (sx1 - sx0 + 1) + (tx - sx0);
                slots[size_t(uint32_t(q.x)) * max_tiles + slot] = v;
            }
        }
    }
}

template <class Tab>
int resident_ctas()
{
    static int per_sm = 0;
    static int sms = 0;
    if (!per_sm) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, grid_tile_kernel<Tab>, kThreads, 0);
        if (per_sm < 1) per_sm = 1;
    }
    return per_sm * sms;
}

// One persistent launch per plane group, in group order on the stream: launches of one stream
// run one after another, so a tile's read-modify-write never races with another group's.
template <class Tab>
tcv_status launch(const tcv_plan* p, const float2* data, const void* c, float c_scale, float2* grid,
                  cudaStream_t st)
{
    const PlanGeom& g = p->g;
    if (g.tw != kTileW || g.th != kTileH) return TCV_ERR_UNSUPPORTED;
    if (g.n == 0) return TCV_OK;
    const int ctas = resident_ctas<Tab>();
    for (int grp = 0; grp < g.n_groups; ++grp) {
        GridArgs a{g.support, g.s, g.g_size, g.ntx, g.ntx * g.nty, grp, c_scale};
        grid_tile_kernel<Tab><<<ctas, kThreads, 0, st>>>(
            data, static_cast<const typename Tab::elem*>(c), p->iu, p->iv, p->coff, p->vals[p->sel],
            p->tile_start, p->tile_count, p->items, p->group_start, grid, a);
        TCV_CUDA(cudaGetLastError());
    }
    return TCV_OK;
}

template <class Tab>
int resident_degrid_ctas()
{
    static int per_sm = 0;
    static int sms = 0;
    if (!per_sm) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, degrid_tile_kernel<Tab>, kThreads, 0);
        if (per_sm < 1) per_sm = 1;
    }
    return per_sm * sms;
}

template <class Tab>
tcv_status launch_adjoint(const tcv_plan* p, const float2* grid, const void* c, float c_scale, float2* out,
                          cudaStream_t st)
{
    const PlanGeom& g = p->g;
    if (g.tw != kTileW || g.th != kTileH) return TCV_ERR_UNSUPPORTED;
    if (g.n == 0) return TCV_OK;
    const int ctas = resident_degrid_ctas<Tab>();
    for (int grp = 0; grp < g.n_groups; ++grp) {
        GridArgs a{g.support, g.s, g.g_size, g.ntx, g.ntx * g.nty, grp, c_scale};
        degrid_tile_kernel<Tab><<<ctas, kThreads, 0, st>>>(
            grid, static_cast<const typename Tab::elem*>(c), p->iu, p->iv, p->coff, p->vals[p->sel],
            p->tile_start, p->tile_count, p->items, p->group_start, p->slots, g.max_tiles, a);
        TCV_CUDA(cudaGetLastError());
    }
    return slot_reduce(p, c_scale, out, st);
}

}  // namespace

tcv_status launch_degrid_tiles(const tcv_plan* p, const float2* grid, const void* c, int c_type,
                               float c_scale, float2* out, cudaStream_t st)
{
    switch (c_type) {
        case TCV_C_C64: return launch_adjoint<TabC64>(p, grid, c, c_scale, out, st);
        case TCV_C_R32: return launch_adjoint<TabR32>(p, grid, c, c_scale, out, st);
        case TCV_C_CBF16: return launch_adjoint<TabCBF16>(p, grid, c, c_scale, out, st);
        case TCV_C_RBF16: return launch_adjoint<TabRBF16>(p, grid, c, c_scale, out, st);
        case TCV_C_CF16: return launch_adjoint<TabCF16>(p, grid, c, c_scale, out, st);
        case TCV_C_RF16: return launch_adjoint<TabRF16>(p, grid, c, c_scale, out, st);
        default: return TCV_ERR_ARG;
    }
}

tcv_status launch_grid(const tcv_plan* p, const float2* data, const void* c, int c_type,
                       float c_scale, float2* grid, cudaStream_t st)
{
    switch (c_type) {
        case TCV_C_C64: return launch<TabC64>(p, data, c, c_scale, grid, st);
        case TCV_C_R32: return launch<TabR32>(p, data, c, c_scale, grid, st);
        case TCV_C_CBF16: return launch<TabCBF16>(p, data, c, c_scale, grid, st);
        case TCV_C_RBF16: return launch<TabRBF16>(p, data, c, c_scale, grid, st);
        case TCV_C_CF16: return launch<TabCF16>(p, data, c, c_scale, grid, st);
        case TCV_C_RF16: return launch<TabRF16>(p, data, c, c_scale, grid, st);
        default: return TCV_ERR_ARG;
    }
}

}  // namespace tcv
