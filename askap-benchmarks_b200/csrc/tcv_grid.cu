// tcv_grid.cu -- launchers of the output-stationary tile kernels (tcv_device.cuh): gridding
// (Benchmark::gridKernel, attic/tConvolveMPI/Benchmark.cc:125-155) and its adjoint degridding
// (Benchmark::degridKernel, :158-195), one persistent launch per plane group.  Each launch uses
// the copy of the kernel specialised on the footprint width when one is available (tcv_jit.cu)
// and the generic copy otherwise.
#include "tcv_internal.cuh"

namespace tcv {
namespace {

// CTAs of a persistent launch: every SM filled to the kernel's occupancy
int resident_of(const void* kernel)
{
    int dev = 0, sms = 148, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kTileThreads, 0) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    return per_sm * sms;
}

// CTAs of a fold launch: a few per SM, each walking the group's cells
int fold_ctas()
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return 4 * sms;
}

GridArgs make_args(const tcv_plan* p, int grp, float c_scale, float2* grid)
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
    a.sched = p->status + kSchedWord;
    return a;
}

// One persistent launch per plane group, in group order on the stream: launches of one stream
// run one after another, so a tile's read-modify-write never races with another group's.
template <class Tab, int kR, bool kVar = false>
tcv_status launch(const tcv_plan* p, const float2* data, const void* c, float c_scale, float2* grid,
                  cudaStream_t st, int c_type)
{
    const PlanGeom& g = p->g;
    if (g.n == 0) return TCV_OK;
    const void* spec = kVar ? nullptr
                       : p->jit_cached_only ? jit_tile_kernel_cached(0, c_type, g.s, kR)
                                            : jit_tile_kernel(0, c_type, g.s, kR);
    const void* generic = reinterpret_cast<const void*>(&grid_tile_kernel<Tab, 0, kR, kVar>);
    const void* kernel = spec ? spec : generic;
    const int ctas = resident_of(kernel);
    const typename Tab::elem* tab = static_cast<const typename Tab::elem*>(c);
    const unsigned int* order = p->vals[p->sel];
    for (int grp = 0; grp < g.n_groups; ++grp) {
        GridArgs a = make_args(p, grp, c_scale, grid);
        void* args[] = {&data, &tab, const_cast<const int32_t**>(&p->iu), const_cast<const int32_t**>(&p->iv),
                        const_cast<const int32_t**>(&p->coff), &order, const_cast<uint4**>(&p->units),
                        const_cast<uint32_t**>(&p->group_ustart), &a};
        TCV_CUDA(cudaLaunchKernel(kernel, dim3(ctas), dim3(kTileThreads), args, 0, st));
        if (g.split) {
            // the split cells' partial tiles into the grid, before the next group touches it
            fold_kernel<kR><<<fold_ctas(), kTileThreads, 0, st>>>(p->items, p->group_start, p->nunits, p->pstart, a);
            TCV_CUDA(cudaGetLastError());
        }
    }
    return TCV_OK;
}

template <class Tab, int kR, bool kVar = false>
tcv_status launch_adjoint(const tcv_plan* p, const float2* grid, const void* c, float c_scale, float2* out,
                          cudaStream_t st, int c_type)
{
    const PlanGeom& g = p->g;
    if (g.n == 0) return TCV_OK;
    const void* spec = kVar ? nullptr
                       : p->jit_cached_only ? jit_tile_kernel_cached(1, c_type, g.s, kR)
                                            : jit_tile_kernel(1, c_type, g.s, kR);
    const void* generic = reinterpret_cast<const void*>(&degrid_tile_kernel<Tab, 0, kR, kVar>);
    const void* kernel = spec ? spec : generic;
    const int ctas = resident_of(kernel);
    const typename Tab::elem* tab = static_cast<const typename Tab::elem*>(c);
    const unsigned int* order = p->vals[p->sel];
    int max_tiles = g.max_tiles;
    float2* gridp = const_cast<float2*>(grid);
    for (int grp = 0; grp < g.n_groups; ++grp) {
        GridArgs a = make_args(p, grp, c_scale, gridp);
        void* args[] = {&tab, const_cast<const int32_t**>(&p->iu), const_cast<const int32_t**>(&p->iv),
                        const_cast<const int32_t**>(&p->coff), &order, const_cast<uint4**>(&p->d_units),
                        const_cast<uint32_t**>(&p->d_group_ustart), const_cast<float2**>(&p->slots), &max_tiles, &a};
        TCV_CUDA(cudaLaunchKernel(kernel, dim3(ctas), dim3(kTileThreads), args, 0, st));
    }
    return slot_reduce(p, c_scale, out, st);
}

}  // namespace

tcv_status launch_fold8(const tcv_plan* p, const GridArgs& a, cudaStream_t st)
{
    fold_kernel<8><<<fold_ctas(), kTileThreads, 0, st>>>(p->items, p->group_start, p->nunits, p->pstart, a);
    TCV_CUDA(cudaGetLastError());
    return TCV_OK;
}

namespace {

template <class Tab>
tcv_status grid_rows(const tcv_plan* p, const float2* data, const void* c, float c_scale, float2* grid,
                     cudaStream_t st, int c_type)
{
    if (p->g.var) {  // per-sample widths: complex tables (the w-term is complex), 64 x 64 or 64 x 32 tiles
        if constexpr (!Tab::kReal) {
            if (p->g.dense) return launch_dense_grid<Tab>(p, data, c, c_scale, grid, st);
            if (p->g.rows == 16) return launch<Tab, 16, true>(p, data, c, c_scale, grid, st, c_type);
            if (p->g.rows == 8) return launch<Tab, 8, true>(p, data, c, c_scale, grid, st, c_type);
        }
        return TCV_ERR_UNSUPPORTED;
    }
    if (p->g.dense) return launch_dense_grid<Tab>(p, data, c, c_scale, grid, st);
    switch (p->g.rows) {
        case 8: return launch<Tab, 8>(p, data, c, c_scale, grid, st, c_type);
        case 16: return launch<Tab, 16>(p, data, c, c_scale, grid, st, c_type);
        case 32: return launch<Tab, 32>(p, data, c, c_scale, grid, st, c_type);
        default: return TCV_ERR_UNSUPPORTED;
    }
}

template <class Tab>
tcv_status degrid_rows(const tcv_plan* p, const float2* grid, const void* c, float c_scale, float2* out,
                       cudaStream_t st, int c_type)
{
    if (p->g.var) {
        if constexpr (!Tab::kReal) {
            if (p->g.ddense) return launch_dense_degrid<Tab>(p, grid, c, c_scale, out, st);
            if (p->g.rows == 16) return launch_adjoint<Tab, 16, true>(p, grid, c, c_scale, out, st, c_type);
            if (p->g.rows == 8) return launch_adjoint<Tab, 8, true>(p, grid, c, c_scale, out, st, c_type);
        }
        return TCV_ERR_UNSUPPORTED;
    }
    if (p->g.ddense) return launch_dense_degrid<Tab>(p, grid, c, c_scale, out, st);
    switch (p->g.rows) {
        case 8: return launch_adjoint<Tab, 8>(p, grid, c, c_scale, out, st, c_type);
        case 16: return launch_adjoint<Tab, 16>(p, grid, c, c_scale, out, st, c_type);
        case 32: return launch_adjoint<Tab, 32>(p, grid, c, c_scale, out, st, c_type);
        default: return TCV_ERR_UNSUPPORTED;
    }
}

}  // namespace

tcv_status launch_degrid_tiles(const tcv_plan* p, const float2* grid, const void* c, int c_type,
                               float c_scale, float2* out, cudaStream_t st)
{
    switch (c_type) {
        case TCV_C_C64: return degrid_rows<TabC64>(p, grid, c, c_scale, out, st, c_type);
        case TCV_C_R32: return degrid_rows<TabR32>(p, grid, c, c_scale, out, st, c_type);
        case TCV_C_CBF16: return degrid_rows<TabCBF16>(p, grid, c, c_scale, out, st, c_type);
        case TCV_C_RBF16: return degrid_rows<TabRBF16>(p, grid, c, c_scale, out, st, c_type);
        case TCV_C_CF16: return degrid_rows<TabCF16>(p, grid, c, c_scale, out, st, c_type);
        case TCV_C_RF16: return degrid_rows<TabRF16>(p, grid, c, c_scale, out, st, c_type);
        default: return TCV_ERR_ARG;
    }
}

tcv_status launch_grid(const tcv_plan* p, const float2* data, const void* c, int c_type,
                       float c_scale, float2* grid, cudaStream_t st)
{
    switch (c_type) {
        case TCV_C_C64: return grid_rows<TabC64>(p, data, c, c_scale, grid, st, c_type);
        case TCV_C_R32: return grid_rows<TabR32>(p, data, c, c_scale, grid, st, c_type);
        case TCV_C_CBF16: return grid_rows<TabCBF16>(p, data, c, c_scale, grid, st, c_type);
        case TCV_C_RBF16: return grid_rows<TabRBF16>(p, data, c, c_scale, grid, st, c_type);
        case TCV_C_CF16: return grid_rows<TabCF16>(p, data, c, c_scale, grid, st, c_type);
        case TCV_C_RF16: return grid_rows<TabRF16>(p, data, c, c_scale, grid, st, c_type);
        default: return TCV_ERR_ARG;
    }
}

}  // namespace tcv
