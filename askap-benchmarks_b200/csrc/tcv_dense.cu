// tcv_dense.cu -- sample-parallel tile kernels for variable-width plans with small footprints
// (the current/tConvolveMPI path: kernels 7..121 wide, most under 20).
//
// The output-stationary tile kernels (tcv_device.cuh) give every lane a fixed grid column and
// make all eight warps test every sample of the tile; with a 9-wide footprint a warp then works
// with 9 of its 32 lanes and most warps only test and skip.  Here each sample of a work unit is
// handled by one warp (sample j by warp j mod kWarps), whose lanes cover the intersection of the
// footprint with the 64 x 32 tile densely: a rectangle w x h is walked as floor(32 / w) rows of w
// lanes per step (w <= 32) or as 32-column strips (w > 32).
//
// Gridding accumulates into a warp-private copy of the tile in shared memory (no two warps write
// one copy, so no atomics); at the end of the unit the copies are added in warp order into the
// grid, or into the unit's partial tile for a split cell (fold_kernel then adds those in unit
// order, as for the tile kernels).  Degridding stages the grid tile in shared memory once per unit
// and reduces each sample's products across its warp into the sample's slot for the tile
// (slot_reduce_kernel adds the slots in tile order).  Every sum is taken in a fixed order, so
// results are deterministic; they group the reference's per-point sums differently (by warp),
// which moves them by FP32 rounding only.
//
// Tiles are the plans' 64 x 32 tiles (tile rows 8), so the plans are those of the tile kernels.
#include "tcv_internal.cuh"

namespace tcv {
namespace {

constexpr int kDTW = kTileW;              // 64 columns
constexpr int kDTH = 32;                  // rows (tile_height(8))
constexpr int kDPts = kDTW * kDTH;        // 2048 points
constexpr int kGWarps = 4;                // gridding: warps per CTA (private tile copies)
constexpr int kGThreads = kGWarps * 32;
constexpr int kDWarps = 8;                // degridding: warps per CTA
constexpr int kDThreads = kDWarps * 32;
static_assert(tile_height(8) == kDTH, "dense kernels use the 64 x 32 tiles of 8-row plans");

// lane -> (row in step, column) of a w-wide rectangle walked floor(32 / w) rows at a time
struct DenseLut {
    unsigned char q[33][32], r[33][32], k[33];
};

__device__ __forceinline__ void build_lut(DenseLut& L, int tid, int nthreads)
{
    for (int i = tid; i < 33 * 32; i += nthreads) {
        const int w = i / 32, lane = i % 32;
        const int ww = w < 1 ? 1 : w;
        L.q[w][lane] = (unsigned char)(lane / ww);
        L.r[w][lane] = (unsigned char)(lane % ww);
        if (lane == 0) L.k[w] = (unsigned char)(32 / ww);
    }
}

// The intersection of sample footprint (fx, fy, s) with the tile at (tx0, ty0), in footprint
// coordinates: columns [c0, c1), rows [r0, r1).
struct Rect {
    int c0, c1, r0, r1;
};
__device__ __forceinline__ Rect clip(int fx, int fy, int s, int tx0, int ty0)
{
    Rect R;
    R.c0 = max(0, tx0 - fx);
    R.c1 = min(s, tx0 + kDTW - fx);
    R.r0 = max(0, ty0 - fy);
    R.r1 = min(s, ty0 + kDTH - fy);
    return R;
}

// A staged sample, prepared once by the staging thread so that the warp that takes it only
// walks its rectangle: the table index and tile point of the rectangle's first element, the table
// row stride (the kernel width), and the rectangle's width, height and rows per step.
struct DenseRec {
    int c0;      // table index of the rectangle's first element (cOffset + r0 * s + c0)
    int p0;      // tile point of that element
    int s;       // table row stride
    int shape;   // w | h << 8 | rows per step << 16 (h = 0: nothing to do)
};

__device__ __forceinline__ DenseRec prepare(int coffk, int s, int fx, int fy, int tx0, int ty0, const DenseLut& L)
{
    const Rect R = clip(fx, fy, s, tx0, ty0);
    const int w = R.c1 - R.c0, h = R.r1 - R.r0;
    DenseRec d;
    d.s = s;
    if (w <= 0 || h <= 0) {  // no overlap (a binned sample always has one)
        d.c0 = d.p0 = 0;
        d.shape = 0;
        return d;
    }
    d.c0 = coffk + R.r0 * s + R.c0;
    d.p0 = (fy + R.r0 - ty0) * kDTW + (fx + R.c0 - tx0);
    d.shape = w | (h << 8) | ((w <= 32 ? int(L.k[w]) : 0) << 16);
    return d;
}

template <class Tab>
__global__ void __launch_bounds__(kGThreads)
dense_grid_kernel(const float2* __restrict__ data, const typename Tab::elem* __restrict__ ctab,
                  const int* __restrict__ iu, const int* __restrict__ iv, const int* __restrict__ coff,
                  const u32* __restrict__ order, const uint4* __restrict__ units,
                  const u32* __restrict__ group_ustart, GridArgs a)
{
    extern __shared__ float2 dsm[];
    float2* acc_all = dsm;                                                // [kGWarps][kDPts]
    DenseRec* rec = reinterpret_cast<DenseRec*>(dsm + kGWarps * kDPts);  // [kGThreads]
    float2* rdv = reinterpret_cast<float2*>(rec + kGThreads);             // scaled data
    __shared__ DenseLut L;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    build_lut(L, threadIdx.x, kGThreads);
    float2* acc = acc_all + warp * kDPts;
    for (int i = lane; i < kDPts; i += 32) acc[i] = make_float2(0.f, 0.f);
    __syncthreads();  // the lane table is complete
    const u32 i1 = group_ustart[a.group + 1];
    for (u32 it = group_ustart[a.group] + blockIdx.x; it < i1; it += gridDim.x) {
        const uint4 u = units[it];
        const u32 start = u.y, cnt = u.z, pslot = u.w;
        const u32 ti = a.tinfo[u.x - u32(a.group) * u32(a.ntiles)];
        const int tx0 = rec_tx(ti) * kDTW, ty0 = rec_ty(ti) * kDTH;
        for (u32 base = 0; base < cnt; base += kGThreads) {
            const int m = int(cnt - base < u32(kGThreads) ? cnt - base : u32(kGThreads));
            __syncthreads();  // the previous chunk's records are consumed
            if (int(threadIdx.x) < m) {
                const u32 k = order[start + base + threadIdx.x];
                const float2 d = data[k];
                const int sk = int(a.ssz[k]);
                rec[threadIdx.x] = prepare(coff[k], sk, iu[k] - sk / 2, iv[k], tx0, ty0, L);
                rdv[threadIdx.x] = make_float2(d.x * a.c_scale, d.y * a.c_scale);
            }
            __syncthreads();
            // U steps per iteration: every table load of the iteration is issued before any update
            // of the warp's tile copy (memory in flight at 12 warps per SM)
            constexpr int U = 4;
            for (int j = warp; j < m; j += kGWarps) {
                const DenseRec d = rec[j];
                const float2 dv = rdv[j];
                const int w = d.shape & 255, h = (d.shape >> 8) & 255, kk = d.shape >> 16;
                if (h == 0) continue;  // warp-uniform
                if (w <= 32) {
                    const int qq = L.q[w][lane], rr = L.r[w][lane];
                    const bool lane_ok = qq < kk;
                    const int cbase = d.c0 + qq * d.s + rr, pbase = d.p0 + qq * kDTW + rr;
                    for (int row0 = 0; row0 < h; row0 += U * kk) {
                        float2 cv[U];
                        bool ok[U];
#pragma unroll
                        for (int e = 0; e < U; ++e) {
                            const int ro = row0 + e * kk;  // this step's first row; the lane's is ro + qq
                            ok[e] = lane_ok && ro + qq < h;
                            cv[e] = ok[e] ? Tab::load(ctab + (cbase + ro * d.s)) : make_float2(0.f, 0.f);
                        }
#pragma unroll
                        for (int e = 0; e < U; ++e) {
                            if (ok[e]) {
                                float2& g = acc[pbase + (row0 + e * kk) * kDTW];
                                float2 t = g;
                                cmac<Tab::kReal>(t, dv, cv[e]);
                                g = t;
                            }
                        }
                    }
                } else {
                    const bool oka = lane < w, okb = lane + 32 < w;
                    for (int row0 = 0; row0 < h; row0 += U / 2) {
                        float2 cv[U];
                        bool ok[U];
#pragma unroll
                        for (int e = 0; e < U; ++e) {
                            const int row = row0 + e / 2;
                            ok[e] = row < h && ((e & 1) ? okb : oka);
                            cv[e] = ok[e] ? Tab::load(ctab + (d.c0 + row * d.s + lane + (e & 1) * 32))
                                          : make_float2(0.f, 0.f);
                        }
#pragma unroll
                        for (int e = 0; e < U; ++e) {
                            if (ok[e]) {
                                float2& g = acc[d.p0 + (row0 + e / 2) * kDTW + lane + (e & 1) * 32];
                                float2 t = g;
                                cmac<Tab::kReal>(t, dv, cv[e]);
                                g = t;
                            }
                        }
                    }
                }
                __syncwarp();  // this sample's updates land before another lane reads them for the next
            }
        }
        __syncthreads();  // every warp's copy is complete
        // the copies in warp order, into the grid (a whole cell) or the unit's partial tile
        const JobDesc& jd = a.jobs[rec_job(ti)];
        const int gs = jd.g_size;
        float2* grid = a.grid ? a.grid : jd.grid;
        for (int p = threadIdx.x; p < kDPts; p += kGThreads) {
            float2 v = acc_all[p];
#pragma unroll
            for (int w = 1; w < kGWarps; ++w) {
                const float2 o = acc_all[w * kDPts + p];
                v.x += o.x;
                v.y += o.y;
            }
#pragma unroll
            for (int w = 0; w < kGWarps; ++w) acc_all[w * kDPts + p] = make_float2(0.f, 0.f);
            if (pslot != kDirect) {
                a.partial[(unsigned long long)(pslot) * kDPts + p] = v;
            } else {
                const int gx = tx0 + (p % kDTW), gy = ty0 + (p / kDTW);
                if (gx < gs && gy < gs) {
                    float2* gp = grid + ((unsigned long long)(gy) * gs + gx);
                    float2 o = *gp;
                    o.x += v.x;
                    o.y += v.y;
                    *gp = o;
                }
            }
        }
        // the zeroed copies are rewritten only after the next unit's first barrier
    }
}

template <class Tab>
__global__ void __launch_bounds__(kDThreads)
dense_degrid_kernel(const typename Tab::elem* __restrict__ ctab, const int* __restrict__ iu,
                    const int* __restrict__ iv, const int* __restrict__ coff, const u32* __restrict__ order,
                    const uint4* __restrict__ units, const u32* __restrict__ group_ustart,
                    float2* __restrict__ slots, int max_tiles, GridArgs a)
{
    __shared__ float2 gt[kDPts];           // the grid tile
    __shared__ DenseRec rec[kDThreads];
    __shared__ unsigned long long rslot[kDThreads];  // slot index of (sample, this tile)
    __shared__ DenseLut L;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    build_lut(L, threadIdx.x, kDThreads);
    const u32 i1 = group_ustart[a.group + 1];
    for (u32 it = group_ustart[a.group] + blockIdx.x; it < i1; it += gridDim.x) {
        const uint4 u = units[it];
        const u32 start = u.y, cnt = u.z;
        const u32 ti = a.tinfo[u.x - u32(a.group) * u32(a.ntiles)];
        const int tx = rec_tx(ti), ty = rec_ty(ti);
        const int tx0 = tx * kDTW, ty0 = ty * kDTH;
        const JobDesc& jd = a.jobs[rec_job(ti)];
        const int gs = jd.g_size;
        const float2* grid = a.grid ? a.grid : jd.grid;
        __syncthreads();  // the previous unit is done with gt and the records
        for (int p = threadIdx.x; p < kDPts; p += kDThreads) {
            const int gx = tx0 + (p % kDTW), gy = ty0 + (p / kDTW);
            gt[p] = (gx < gs && gy < gs) ? grid[(unsigned long long)(gy) * gs + gx] : make_float2(0.f, 0.f);
        }
        for (u32 base = 0; base < cnt; base += kDThreads) {
            const int m = int(cnt - base < u32(kDThreads) ? cnt - base : u32(kDThreads));
            __syncthreads();
            if (int(threadIdx.x) < m) {
                const u32 k = order[start + base + threadIdx.x];
                const int sk = int(a.ssz[k]);
                const int fx = iu[k] - sk / 2, fy = iv[k];
                rec[threadIdx.x] = prepare(coff[k], sk, fx, fy, tx0, ty0, L);
                const int sx0 = fx / kDTW, sx1 = (fx + sk - 1) / kDTW, sy0 = fy / kDTH;
                rslot[threadIdx.x] = (unsigned long long)(k) * max_tiles + (ty - sy0) * (sx1 - sx0 + 1) + (tx - sx0);
            }
            __syncthreads();
            for (int j = warp; j < m; j += kDWarps) {
                const DenseRec d = rec[j];
                const int w = d.shape & 255, h = (d.shape >> 8) & 255, kk = d.shape >> 16;
                float2 p0 = make_float2(0.f, 0.f), p1 = make_float2(0.f, 0.f);  // two FMA chains
                if (h > 0 && w <= 32) {
                    const int qq = L.q[w][lane], rr = L.r[w][lane];
                    const bool lane_ok = qq < kk;
                    const int cbase = d.c0 + qq * d.s + rr, pbase = d.p0 + qq * kDTW + rr;
                    for (int row0 = 0; row0 < h; row0 += 2 * kk) {
                        const bool oka = lane_ok && row0 + qq < h, okb = lane_ok && row0 + kk + qq < h;
                        if (oka) cmac<Tab::kReal>(p0, gt[pbase + row0 * kDTW], Tab::load(ctab + (cbase + row0 * d.s)));
                        if (okb)
                            cmac<Tab::kReal>(p1, gt[pbase + (row0 + kk) * kDTW],
                                             Tab::load(ctab + (cbase + (row0 + kk) * d.s)));
                    }
                } else if (h > 0) {
                    const bool oka = lane < w, okb = lane + 32 < w;
                    for (int row = 0; row < h; ++row) {
                        if (oka) cmac<Tab::kReal>(p0, gt[d.p0 + row * kDTW + lane], Tab::load(ctab + (d.c0 + row * d.s + lane)));
                        if (okb)
                            cmac<Tab::kReal>(p1, gt[d.p0 + row * kDTW + lane + 32],
                                             Tab::load(ctab + (d.c0 + row * d.s + lane + 32)));
                    }
                }
                float2 v = make_float2(p0.x + p1.x, p0.y + p1.y);
#pragma unroll
                for (int o = 16; o; o >>= 1) {
                    v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
                    v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
                }
                if (lane == 0) slots[rslot[j]] = v;  // an empty overlap writes its empty slot
            }
        }
    }
}

int resident(const void* kernel, int threads, size_t smem)
{
    int dev = 0, sms = 148, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    return per_sm * sms;
}

constexpr size_t kGridSmem = size_t(kGWarps) * kDPts * sizeof(float2) + size_t(kGThreads) * (sizeof(DenseRec) + sizeof(float2));

GridArgs dense_args(const tcv_plan* p, int grp, float c_scale, float2* grid)
{
    const PlanGeom& g = p->g;
    GridArgs a{};
    a.support = g.support;
    a.s = g.s;
    a.ntiles = int(g.ntiles);
    a.group = grp;
    a.c_scale = c_scale;
    a.grid = grid;
    a.jobs = p->jobs;
    a.tinfo = p->tinfo;
    a.partial = p->partial;
    a.ssz = p->ssz;
    return a;
}

}  // namespace

template <class Tab>
tcv_status launch_dense_grid(const tcv_plan* p, const float2* data, const void* c, float c_scale, float2* grid,
                             cudaStream_t st)
{
    const PlanGeom& g = p->g;
    if (g.n == 0) return TCV_OK;
    if (!g.var || g.tw != kDTW || g.th != kDTH) return TCV_ERR_UNSUPPORTED;
    const void* kernel = reinterpret_cast<const void*>(&dense_grid_kernel<Tab>);
    TCV_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kGridSmem)));
    const int ctas = resident(kernel, kGThreads, kGridSmem);
    const typename Tab::elem* tab = static_cast<const typename Tab::elem*>(c);
    const unsigned int* order = p->vals[p->sel];
    for (int grp = 0; grp < g.n_groups; ++grp) {
        GridArgs a = dense_args(p, grp, c_scale, grid);
        void* args[] = {&data, &tab, const_cast<const int32_t**>(&p->iu), const_cast<const int32_t**>(&p->iv),
                        const_cast<const int32_t**>(&p->coff), &order, const_cast<uint4**>(&p->units),
                        const_cast<uint32_t**>(&p->group_ustart), &a};
        TCV_CUDA(cudaLaunchKernel(kernel, dim3(ctas), dim3(kGThreads), args, kGridSmem, st));
        if (g.split) TCV_CHECK(launch_fold8(p, a, st));
    }
    return TCV_OK;
}

template <class Tab>
tcv_status launch_dense_degrid(const tcv_plan* p, const float2* grid, const void* c, float c_scale, float2* out,
                               cudaStream_t st)
{
    const PlanGeom& g = p->g;
    if (g.n == 0) return TCV_OK;
    if (!g.var || g.tw != kDTW || g.th != kDTH) return TCV_ERR_UNSUPPORTED;
    const void* kernel = reinterpret_cast<const void*>(&dense_degrid_kernel<Tab>);
    const int ctas = resident(kernel, kDThreads, 0);
    const typename Tab::elem* tab = static_cast<const typename Tab::elem*>(c);
    const unsigned int* order = p->vals[p->sel];
    int max_tiles = g.max_tiles;
    float2* gridp = const_cast<float2*>(grid);
    for (int grp = 0; grp < g.n_groups; ++grp) {
        GridArgs a = dense_args(p, grp, c_scale, gridp);
        void* args[] = {&tab, const_cast<const int32_t**>(&p->iu), const_cast<const int32_t**>(&p->iv),
                        const_cast<const int32_t**>(&p->coff), &order, const_cast<uint4**>(&p->d_units),
                        const_cast<uint32_t**>(&p->d_group_ustart), const_cast<float2**>(&p->slots), &max_tiles, &a};
        TCV_CUDA(cudaLaunchKernel(kernel, dim3(ctas), dim3(kDThreads), args, 0, st));
    }
    return slot_reduce(p, c_scale, out, st);
}

template tcv_status launch_dense_grid<TabC64>(const tcv_plan*, const float2*, const void*, float, float2*, cudaStream_t);
template tcv_status launch_dense_grid<TabCBF16>(const tcv_plan*, const float2*, const void*, float, float2*, cudaStream_t);
template tcv_status launch_dense_grid<TabCF16>(const tcv_plan*, const float2*, const void*, float, float2*, cudaStream_t);
template tcv_status launch_dense_degrid<TabC64>(const tcv_plan*, const float2*, const void*, float, float2*, cudaStream_t);
template tcv_status launch_dense_degrid<TabCBF16>(const tcv_plan*, const float2*, const void*, float, float2*, cudaStream_t);
template tcv_status launch_dense_degrid<TabCF16>(const tcv_plan*, const float2*, const void*, float, float2*, cudaStream_t);

}  // namespace tcv
