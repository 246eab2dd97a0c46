// tcv_grid.cu -- launchers of the output-stationary tile kernels (tcv_device.cuh): gridding
// (Benchmark::gridKernel, attic/tConvolveMPI/Benchmark.cc:125-155) and its adjoint degridding
// (Benchmark::degridKernel, :158-195), one persistent launch per plane group.  Each launch uses
// the copy of the kernel specialised on the footprint width when one is available (tcv_jit.cu)
// and the generic copy otherwise.
#include "tcv_internal.cuh"

namespace tcv {
namespace {

template <class Tab>
int resident_ctas()
{
    static int per_sm = 0;
    static int sms = 0;
    if (!per_sm) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, grid_tile_kernel<Tab, 0>, kTileThreads, 0);
        if (per_sm < 1) per_sm = 1;
    }
    return per_sm * sms;
}

// One persistent launch per plane group, in group order on the stream: launches of one stream
// run one after another, so a tile's read-modify-write never races with another group's.
int resident_of(const void* kernel)
{
    int dev = 0, sms = 148, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kTileThreads, 0) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    return per_sm * sms;
}

template <class Tab>
tcv_status launch(const tcv_plan* p, const float2* data, const void* c, float c_scale, float2* grid,
                  cudaStream_t st, int c_type)
{
    const PlanGeom& g = p->g;
    if (g.tw != kTileW || g.th != kTileH) return TCV_ERR_UNSUPPORTED;
    if (g.n == 0) return TCV_OK;
    const void* spec = jit_tile_kernel(0, c_type, g.s);
    const int ctas = spec ? resident_of(spec) : resident_ctas<Tab>();
    const typename Tab::elem* tab = static_cast<const typename Tab::elem*>(c);
    const unsigned int* order = p->vals[p->sel];
    for (int grp = 0; grp < g.n_groups; ++grp) {
        GridArgs a{g.support, g.s, g.g_size, g.ntx, g.ntx * g.nty, grp, c_scale};
        if (spec) {
            void* args[] = {&data, &tab, const_cast<const int32_t**>(&p->iu), const_cast<const int32_t**>(&p->iv),
                            const_cast<const int32_t**>(&p->coff), &order,
                            const_cast<uint32_t**>(&p->tile_start), const_cast<uint32_t**>(&p->tile_count),
                            const_cast<uint32_t**>(&p->items), const_cast<uint32_t**>(&p->group_start), &grid, &a};
            TCV_CUDA(cudaLaunchKernel(spec, dim3(ctas), dim3(kTileThreads), args, 0, st));
        } else {
            grid_tile_kernel<Tab, 0><<<ctas, kTileThreads, 0, st>>>(data, tab, p->iu, p->iv, p->coff, order,
                                                                     p->tile_start, p->tile_count, p->items,
                                                                     p->group_start, grid, a);
            TCV_CUDA(cudaGetLastError());
        }
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
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, degrid_tile_kernel<Tab, 0>, kTileThreads, 0);
        if (per_sm < 1) per_sm = 1;
    }
    return per_sm * sms;
}

template <class Tab>
tcv_status launch_adjoint(const tcv_plan* p, const float2* grid, const void* c, float c_scale, float2* out,
                          cudaStream_t st, int c_type)
{
    const PlanGeom& g = p->g;
    if (g.tw != kTileW || g.th != kTileH) return TCV_ERR_UNSUPPORTED;
    if (g.n == 0) return TCV_OK;
    const void* spec = jit_tile_kernel(1, c_type, g.s);
    const int ctas = spec ? resident_of(spec) : resident_degrid_ctas<Tab>();
    const typename Tab::elem* tab = static_cast<const typename Tab::elem*>(c);
    const unsigned int* order = p->vals[p->sel];
    int max_tiles = g.max_tiles;
    for (int grp = 0; grp < g.n_groups; ++grp) {
        GridArgs a{g.support, g.s, g.g_size, g.ntx, g.ntx * g.nty, grp, c_scale};
        if (spec) {
            void* args[] = {&grid, &tab, const_cast<const int32_t**>(&p->iu), const_cast<const int32_t**>(&p->iv),
                            const_cast<const int32_t**>(&p->coff), &order,
                            const_cast<uint32_t**>(&p->tile_start), const_cast<uint32_t**>(&p->tile_count),
                            const_cast<uint32_t**>(&p->items), const_cast<uint32_t**>(&p->group_start),
                            const_cast<float2**>(&p->slots), &max_tiles, &a};
            TCV_CUDA(cudaLaunchKernel(spec, dim3(ctas), dim3(kTileThreads), args, 0, st));
        } else {
            degrid_tile_kernel<Tab, 0><<<ctas, kTileThreads, 0, st>>>(grid, tab, p->iu, p->iv, p->coff, order,
                                                                       p->tile_start, p->tile_count, p->items,
                                                                       p->group_start, p->slots, max_tiles, a);
            TCV_CUDA(cudaGetLastError());
        }
    }
    return slot_reduce(p, c_scale, out, st);
}

}  // namespace

tcv_status launch_degrid_tiles(const tcv_plan* p, const float2* grid, const void* c, int c_type,
                               float c_scale, float2* out, cudaStream_t st)
{
    switch (c_type) {
        case TCV_C_C64: return launch_adjoint<TabC64>(p, grid, c, c_scale, out, st, c_type);
        case TCV_C_R32: return launch_adjoint<TabR32>(p, grid, c, c_scale, out, st, c_type);
        case TCV_C_CBF16: return launch_adjoint<TabCBF16>(p, grid, c, c_scale, out, st, c_type);
        case TCV_C_RBF16: return launch_adjoint<TabRBF16>(p, grid, c, c_scale, out, st, c_type);
        case TCV_C_CF16: return launch_adjoint<TabCF16>(p, grid, c, c_scale, out, st, c_type);
        case TCV_C_RF16: return launch_adjoint<TabRF16>(p, grid, c, c_scale, out, st, c_type);
        default: return TCV_ERR_ARG;
    }
}

tcv_status launch_grid(const tcv_plan* p, const float2* data, const void* c, int c_type,
                       float c_scale, float2* grid, cudaStream_t st)
{
    switch (c_type) {
        case TCV_C_C64: return launch<TabC64>(p, data, c, c_scale, grid, st, c_type);
        case TCV_C_R32: return launch<TabR32>(p, data, c, c_scale, grid, st, c_type);
        case TCV_C_CBF16: return launch<TabCBF16>(p, data, c, c_scale, grid, st, c_type);
        case TCV_C_RBF16: return launch<TabRBF16>(p, data, c, c_scale, grid, st, c_type);
        case TCV_C_CF16: return launch<TabCF16>(p, data, c, c_scale, grid, st, c_type);
        case TCV_C_RF16: return launch<TabRF16>(p, data, c, c_scale, grid, st, c_type);
        default: return TCV_ERR_ARG;
    }
}

}  // namespace tcv
