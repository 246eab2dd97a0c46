// tcv_plan.cu -- binning of samples for the tile kernels.
//
// The reference grids samples in index order, straight into HBM-sized memory
// (attic/tConvolveMPI/Benchmark.cc:131-154; "some presorting might be advantageous", :113-114).
// Here a plan sorts (sample, tile) pairs with a device radix sort:
//   gridding  : every output tile of tw x th points gets the list of samples whose footprint
//               overlaps it (a footprint of sSize^2 touches up to max_tiles tiles);
//   degridding: every anchor tile of ta x ta gets the samples whose footprint's top-left corner
//               lies in it (each sample exactly once).
// Kernel indices kid = cOffset / sSize^2 (w-plane major, then the oversampling offsets) are
// grouped into runs of whole w-planes whose slice of the table fits in L2 with room to spare.
// The sort key is the work cell (group, tile), ordered group-major, so all SMs work through the
// table one group at a time and the slice in use stays resident in L2; within a cell the stable
// sort keeps samples in index order (the reference's order).  The non-empty cells are compacted
// into work lists (with per-group ranges) that persistent kernels walk.
// Samples whose footprint or table range falls outside the grid or the table are counted and
// left out (sentinel key, sorted past the end).
#include "tcv_internal.cuh"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/iterator/transform_iterator.h>

#include <algorithm>
#include <new>

namespace tcv {
namespace {

int bits_for(uint64_t v)  // bits needed to represent values 0..v
{
    int b = 0;
    while (v) {
        ++b;
        v >>= 1;
    }
    return b < 1 ? 1 : b;
}

template <typename K>
__global__ void plan_keys_kernel(const int32_t* __restrict__ iu, const int32_t* __restrict__ iv,
                                 const int32_t* __restrict__ coff, PlanGeom g, K* keys,
                                 uint32_t* vals, K* akeys, uint32_t* avals, uint32_t* tile_count,
                                 uint32_t* atile_count, unsigned long long* rejected)
{
    const int64_t d = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (d >= g.n) return;
    const int64_t fx = (int64_t)iu[d] - g.support;
    const int64_t fy = iv[d];
    const int64_t co = coff[d];
    const int64_t s = g.s;
    const bool ok = fx >= 0 && fx + s <= g.g_size && fy >= 0 && fy + s <= g.g_size && co >= 0 &&
                    co + s * s <= g.c_len;
    K* kp = keys + d * g.max_tiles;
    uint32_t* vp = vals + d * g.max_tiles;
    const K sentinel = K(1) << (g.key_bits - 1);
    const K asentinel = K(1) << (g.akey_bits - 1);
    if (!ok) {
        atomicAdd(rejected, 1ull);
        for (int t = 0; t < g.max_tiles; ++t) {
            kp[t] = sentinel;
            vp[t] = uint32_t(d);
        }
        akeys[d] = asentinel;
        avals[d] = uint32_t(d);
        return;
    }
    const uint32_t grp = uint32_t(co / (s * s) / g.kid_group);
    const uint32_t cell0 = grp * uint32_t(g.ntx * g.nty);
    const int tx0 = int(fx / g.tw), tx1 = int((fx + s - 1) / g.tw);
    const int ty0 = int(fy / g.th), ty1 = int((fy + s - 1) / g.th);
    int t = 0;
    for (int ty = ty0; ty <= ty1; ++ty)
        for (int tx = tx0; tx <= tx1; ++tx) {
            const uint32_t cell = cell0 + uint32_t(ty) * g.ntx + tx;
            kp[t] = K(cell);
            vp[t] = uint32_t(d);
            atomicAdd(&tile_count[cell], 1u);
            ++t;
        }
    for (; t < g.max_tiles; ++t) {
        kp[t] = sentinel;
        vp[t] = uint32_t(d);
    }
    const uint32_t at = grp * uint32_t(g.natx * g.naty) + uint32_t(fy / g.ta) * g.natx + uint32_t(fx / g.ta);
    akeys[d] = K(at);
    avals[d] = uint32_t(d);
    atomicAdd(&atile_count[at], 1u);
}

struct NonZero {
    __host__ __device__ __forceinline__ bool operator()(const uint32_t& v) const { return v != 0; }
};

// group_start[g] = first item whose cell belongs to group g or later (items are sorted)
__global__ void group_ranges_kernel(const uint32_t* items, const uint32_t* n_items, int n_groups,
                                    uint32_t cells_per_group, uint32_t* group_start)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g > n_groups) return;
    const uint32_t key = uint32_t(g) * cells_per_group;
    uint32_t lo = 0, hi = *n_items;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (items[mid] < key)
            lo = mid + 1;
        else
            hi = mid;
    }
    group_start[g] = lo;
}

inline size_t align_up(size_t x, size_t a = 256) { return (x + a - 1) / a * a; }

template <typename K>
size_t cub_temp_bytes(const PlanGeom& g)
{
    size_t a = 0, b = 0, c = 0, d = 0, e = 0, f = 0;
    const int64_t np = g.n * g.max_tiles;
    const int cells = g.n_groups * g.ntx * g.nty, acells = g.n_groups * g.natx * g.naty;
    cub::DoubleBuffer<K> kb(nullptr, nullptr);
    cub::DoubleBuffer<uint32_t> vb(nullptr, nullptr);
    cub::DeviceRadixSort::SortPairs(nullptr, a, kb, vb, np, 0, g.key_bits);
    cub::DeviceRadixSort::SortPairs(nullptr, b, kb, vb, g.n, 0, g.akey_bits);
    cub::DeviceScan::ExclusiveSum(nullptr, c, (uint32_t*)nullptr, (uint32_t*)nullptr, cells);
    cub::DeviceScan::ExclusiveSum(nullptr, d, (uint32_t*)nullptr, (uint32_t*)nullptr, acells);
    thrust::counting_iterator<uint32_t> it(0);
    thrust::transform_iterator<NonZero, const uint32_t*> fl((const uint32_t*)nullptr, NonZero());
    cub::DeviceSelect::Flagged(nullptr, e, it, fl, (uint32_t*)nullptr, (uint32_t*)nullptr, cells);
    cub::DeviceSelect::Flagged(nullptr, f, it, fl, (uint32_t*)nullptr, (uint32_t*)nullptr, acells);
    return std::max(std::max(std::max(a, b), std::max(c, d)), std::max(e, f));
}

template <typename K>
tcv_status build(tcv_plan* p, const int32_t* iu, const int32_t* iv, const int32_t* coff,
                 cudaStream_t st)
{
    const PlanGeom& g = p->g;
    const int64_t np = g.n * g.max_tiles;
    const int cells = g.n_groups * g.ntx * g.nty, acells = g.n_groups * g.natx * g.naty;
    TCV_CUDA(cudaMemsetAsync(p->tile_count, 0, sizeof(uint32_t) * size_t(cells), st));
    TCV_CUDA(cudaMemsetAsync(p->atile_count, 0, sizeof(uint32_t) * size_t(acells), st));
    TCV_CUDA(cudaMemsetAsync(p->rejected, 0, sizeof(unsigned long long), st));
    TCV_CUDA(cudaMemsetAsync(p->status, 0, sizeof(unsigned int), st));
    if (g.n > 0) {
        plan_keys_kernel<K><<<unsigned((g.n + 255) / 256), 256, 0, st>>>(
            iu, iv, coff, g, static_cast<K*>(p->keys[0]), p->vals[0], static_cast<K*>(p->akeys[0]),
            p->avals[0], p->tile_count, p->atile_count, p->rejected);
        TCV_CUDA(cudaGetLastError());
        cub::DoubleBuffer<K> kb(static_cast<K*>(p->keys[0]), static_cast<K*>(p->keys[1]));
        cub::DoubleBuffer<uint32_t> vb(p->vals[0], p->vals[1]);
        size_t tb = p->cub_bytes;
        TCV_CUDA(cub::DeviceRadixSort::SortPairs(p->cub_temp, tb, kb, vb, np, 0, g.key_bits, st));
        p->sel = vb.selector;
        cub::DoubleBuffer<K> akb(static_cast<K*>(p->akeys[0]), static_cast<K*>(p->akeys[1]));
        cub::DoubleBuffer<uint32_t> avb(p->avals[0], p->avals[1]);
        tb = p->cub_bytes;
        TCV_CUDA(cub::DeviceRadixSort::SortPairs(p->cub_temp, tb, akb, avb, g.n, 0, g.akey_bits, st));
        p->asel = avb.selector;
    } else {
        p->sel = 0;
        p->asel = 0;
    }
    size_t tb = p->cub_bytes;
    TCV_CUDA(cub::DeviceScan::ExclusiveSum(p->cub_temp, tb, p->tile_count, p->tile_start, cells, st));
    tb = p->cub_bytes;
    TCV_CUDA(cub::DeviceScan::ExclusiveSum(p->cub_temp, tb, p->atile_count, p->atile_start, acells, st));
    thrust::counting_iterator<uint32_t> it(0);
    thrust::transform_iterator<NonZero, const uint32_t*> fl(p->tile_count, NonZero());
    tb = p->cub_bytes;
    TCV_CUDA(cub::DeviceSelect::Flagged(p->cub_temp, tb, it, fl, p->items, p->n_items, cells, st));
    thrust::transform_iterator<NonZero, const uint32_t*> afl(p->atile_count, NonZero());
    tb = p->cub_bytes;
    TCV_CUDA(cub::DeviceSelect::Flagged(p->cub_temp, tb, it, afl, p->aitems, p->n_aitems, acells, st));
    group_ranges_kernel<<<(g.n_groups + 1 + 127) / 128, 128, 0, st>>>(p->items, p->n_items, g.n_groups,
                                                                       uint32_t(g.ntx * g.nty), p->group_start);
    TCV_CUDA(cudaGetLastError());
    return TCV_OK;
}

}  // namespace

// Tile geometry.  Gridding tiles are 64 x 64 points (8 warps of 32 columns x 16 rows).
// Degridding anchor tiles are the largest ta whose staged region (ta + sSize - 1)^2 complex
// points fits in shared memory next to the partial sums; beyond that the direct kernel reads
// the grid from global memory.
PlanGeom make_geom(int64_t n, int support, int g_size, int64_t c_len)
{
    PlanGeom g{};
    g.n = n;
    g.support = support;
    g.s = 2 * support + 1;
    g.g_size = g_size;
    g.c_len = c_len;
    const int64_t s2 = int64_t(g.s) * g.s;
    const int64_t nk = (c_len + s2 - 1) / s2;
    g.kid_bits = bits_for(uint64_t(nk));
    // kernels per group: whole planes of 64 (8 x 8 oversampling) whose complex64 slice is about
    // 32 MiB, a quarter of the 126 MB L2
    const int64_t per_kernel = s2 * 8;
    int64_t kg = ((int64_t(32) << 20) / per_kernel) / 64 * 64;
    if (kg < 64) kg = 64;
    if (kg > nk) kg = nk < 1 ? 1 : nk;
    g.kid_group = int(kg);
    g.n_groups = int((nk + kg - 1) / kg);
    if (g.n_groups < 1) g.n_groups = 1;
    g.group_bits = bits_for(uint64_t(g.n_groups - 1));
    g.tw = 64;
    g.th = 64;
    g.ntx = (g_size + g.tw - 1) / g.tw;
    g.nty = (g_size + g.th - 1) / g.th;
    g.max_tiles = ((g.s + g.tw - 2) / g.tw + 1) * ((g.s + g.th - 2) / g.th + 1);
    g.tile_bits = bits_for(uint64_t(g.n_groups) * g.ntx * g.nty - 1);
    g.key_bits = g.tile_bits + 1;  // cell, plus the sentinel bit

    constexpr size_t kSmemBudget = 220 * 1024;  // of 227 KB per CTA; the rest holds partial sums
    const int cand[] = {128, 96, 64, 48, 32, 16, 8};
    g.degrid_mode = 1;
    g.ta = 32;
    for (int ta : cand) {
        const int w = ((ta + g.s - 1) + 1) & ~1;
        const int h = ta + g.s - 1;
        if (w <= 256 && h <= 256 && size_t(w) * h * 8 <= kSmemBudget && ta <= g_size) {
            g.ta = ta;
            g.box_w = w;
            g.box_h = h;
            g.degrid_mode = (g_size % 2 == 0) ? 0 : 1;  // TMA row stride must be a multiple of 16 B
            break;
        }
    }
    g.natx = (g_size + g.ta - 1) / g.ta;
    g.naty = (g_size + g.ta - 1) / g.ta;
    g.atile_bits = bits_for(uint64_t(g.n_groups) * g.natx * g.naty - 1);
    g.akey_bits = g.atile_bits + 1;
    g.key64 = g.key_bits > 32 || g.akey_bits > 32;
    g.degrid_parts = 4;
    return g;
}

size_t plan_bytes(const PlanGeom& g, size_t* cub_bytes_out)
{
    const size_t ks = g.key64 ? 8 : 4;
    const size_t np = size_t(g.n) * g.max_tiles;
    const size_t cb = g.key64 ? cub_temp_bytes<uint64_t>(g) : cub_temp_bytes<uint32_t>(g);
    if (cub_bytes_out) *cub_bytes_out = cb;
    size_t b = 0;
    b += 2 * align_up(np * ks) + 2 * align_up(np * 4);
    b += 2 * align_up(size_t(g.n) * ks) + 2 * align_up(size_t(g.n) * 4);
    const size_t cells = size_t(g.n_groups) * g.ntx * g.nty, acells = size_t(g.n_groups) * g.natx * g.naty;
    b += 3 * align_up(cells * 4) + align_up(4) + align_up(size_t(g.n_groups + 1) * 4);
    b += 3 * align_up(acells * 4) + align_up(4);
    b += align_up(sizeof(unsigned long long)) + align_up(sizeof(unsigned int));
    b += align_up(np * sizeof(float2));
    b += align_up(cb);
    return b;
}

}  // namespace tcv

using namespace tcv;

extern "C" {

size_t tcv_plan_workspace_bytes(int64_t n, int support, int g_size, int64_t c_len)
{
    if (n < 0 || support < 0 || g_size < 1 || c_len < 1) return 0;
    PlanGeom g = make_geom(n, support, g_size, c_len);
    return plan_bytes(g, nullptr);
}

}  // extern "C"

namespace tcv {

// Fill *p (a caller-owned object) with a plan built in d_work.
tcv_status plan_init(tcv_plan* p, const int32_t* d_iu, const int32_t* d_iv, const int32_t* d_coff, int64_t n,
                     int support, int g_size, int64_t c_len, void* d_work, size_t work_bytes, cudaStream_t st)
{
    if (!p || n < 0 || support < 0 || g_size < 1 || c_len < 1) return TCV_ERR_ARG;
    if (n > 0 && (!d_iu || !d_iv || !d_coff)) return TCV_ERR_ARG;
    if (n >= (int64_t(1) << 32) / 16) return TCV_ERR_UNSUPPORTED;  // 32-bit sample indices
    if (!d_work) return TCV_ERR_ARG;
    *p = tcv_plan{};
    p->g = make_geom(n, support, g_size, c_len);
    size_t cb = 0;
    const size_t need = plan_bytes(p->g, &cb);
    if (work_bytes < need) return TCV_ERR_WORKSPACE;
    const PlanGeom& g = p->g;
    const size_t ks = g.key64 ? 8 : 4;
    const size_t np = size_t(g.n) * g.max_tiles;
    char* w = static_cast<char*>(d_work);
    auto take = [&](size_t bytes) {
        char* r = w;
        w += align_up(bytes);
        return static_cast<void*>(r);
    };
    p->keys[0] = take(np * ks);
    p->keys[1] = take(np * ks);
    p->vals[0] = static_cast<uint32_t*>(take(np * 4));
    p->vals[1] = static_cast<uint32_t*>(take(np * 4));
    p->akeys[0] = take(size_t(g.n) * ks);
    p->akeys[1] = take(size_t(g.n) * ks);
    p->avals[0] = static_cast<uint32_t*>(take(size_t(g.n) * 4));
    p->avals[1] = static_cast<uint32_t*>(take(size_t(g.n) * 4));
    const size_t cells = size_t(g.n_groups) * g.ntx * g.nty, acells = size_t(g.n_groups) * g.natx * g.naty;
    p->tile_count = static_cast<uint32_t*>(take(cells * 4));
    p->tile_start = static_cast<uint32_t*>(take(cells * 4));
    p->items = static_cast<uint32_t*>(take(cells * 4));
    p->n_items = static_cast<uint32_t*>(take(4));
    p->group_start = static_cast<uint32_t*>(take(size_t(g.n_groups + 1) * 4));
    p->atile_count = static_cast<uint32_t*>(take(acells * 4));
    p->atile_start = static_cast<uint32_t*>(take(acells * 4));
    p->aitems = static_cast<uint32_t*>(take(acells * 4));
    p->n_aitems = static_cast<uint32_t*>(take(4));
    p->rejected = static_cast<unsigned long long*>(take(sizeof(unsigned long long)));
    p->status = static_cast<unsigned int*>(take(sizeof(unsigned int)));
    p->slots = static_cast<float2*>(take(np * sizeof(float2)));
    p->cub_temp = take(cb);
    p->cub_bytes = cb;
    p->iu = d_iu;
    p->iv = d_iv;
    p->coff = d_coff;
    p->degrid_variant = TCV_DEGRID_TILES;
    return g.key64 ? build<uint64_t>(p, d_iu, d_iv, d_coff, st) : build<uint32_t>(p, d_iu, d_iv, d_coff, st);
}

}  // namespace tcv

extern "C" {

tcv_status tcv_plan_build(tcv_plan** plan_out, const int32_t* d_iu, const int32_t* d_iv,
                          const int32_t* d_coff, int64_t n, int support, int g_size,
                          int64_t c_len, void* d_work, size_t work_bytes, void* stream)
{
    if (!plan_out) return TCV_ERR_ARG;
    tcv_plan* p = new (std::nothrow) tcv_plan{};
    if (!p) return TCV_ERR_OOM;
    const tcv_status s = plan_init(p, d_iu, d_iv, d_coff, n, support, g_size, c_len, d_work, work_bytes,
                                   static_cast<cudaStream_t>(stream));
    if (s != TCV_OK) {
        delete p;
        return s;
    }
    *plan_out = p;
    return TCV_OK;
}

tcv_status tcv_plan_rejected(const tcv_plan* plan, int64_t* rejected_out, void* stream)
{
    if (!plan || !rejected_out) return TCV_ERR_ARG;
    unsigned long long h = 0;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    TCV_CUDA(cudaMemcpyAsync(&h, plan->rejected, sizeof(h), cudaMemcpyDeviceToHost, st));
    TCV_CUDA(cudaStreamSynchronize(st));
    *rejected_out = int64_t(h);
    return TCV_OK;
}

tcv_status tcv_plan_status(const tcv_plan* plan, void* stream)
{
    if (!plan) return TCV_ERR_ARG;
    unsigned int h = 0;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    TCV_CUDA(cudaMemcpyAsync(&h, plan->status, sizeof(h), cudaMemcpyDeviceToHost, st));
    TCV_CUDA(cudaStreamSynchronize(st));
    return (h & 1u) ? TCV_ERR_TIMEOUT : TCV_OK;
}

tcv_status tcv_plan_info(const tcv_plan* plan, int* tile_w, int* tile_h, int* anchor,
                         int* degrid_mode, int* n_tiles)
{
    if (!plan) return TCV_ERR_ARG;
    if (tile_w) *tile_w = plan->g.tw;
    if (tile_h) *tile_h = plan->g.th;
    if (anchor) *anchor = plan->g.ta;
    if (degrid_mode) *degrid_mode = plan->g.degrid_mode;
    if (n_tiles) *n_tiles = plan->g.ntx * plan->g.nty * plan->g.n_groups;
    return TCV_OK;
}

void tcv_plan_destroy(tcv_plan* plan) { delete plan; }

tcv_status tcv_plan_grid(const tcv_plan* plan, const float* d_data, const void* d_c, int c_type,
                         float c_scale, float* d_grid, void* stream)
{
    if (!plan || !d_c || !d_grid || (plan->g.n > 0 && !d_data)) return TCV_ERR_ARG;
    if (tcv_ctype_bytes(c_type) == 0) return TCV_ERR_ARG;
    if (c_type & TCV_C_PADDED)
        return launch_grid_pipe(plan, reinterpret_cast<const float2*>(d_data), d_c, c_type & 0xff, c_scale,
                                reinterpret_cast<float2*>(d_grid), static_cast<cudaStream_t>(stream));
    if (c_type & TCV_C_PAIRED)
        return launch_grid_pair(plan, reinterpret_cast<const float2*>(d_data), d_c, c_type & 0xff, c_scale,
                                reinterpret_cast<float2*>(d_grid), static_cast<cudaStream_t>(stream));
    return launch_grid(plan, reinterpret_cast<const float2*>(d_data), d_c, c_type, c_scale,
                       reinterpret_cast<float2*>(d_grid), static_cast<cudaStream_t>(stream));
}

tcv_status tcv_plan_degrid(const tcv_plan* plan, const float* d_grid, const void* d_c, int c_type,
                           float c_scale, float* d_data, void* stream)
{
    if (!plan || !d_c || !d_grid || (plan->g.n > 0 && !d_data)) return TCV_ERR_ARG;
    if (tcv_ctype_bytes(c_type) == 0) return TCV_ERR_ARG;
    if (c_type & TCV_C_PADDED) {
        if (plan->g.n == 0) return TCV_OK;
        return launch_degrid_pipe(plan, reinterpret_cast<const float2*>(d_grid), d_c, c_type & 0xff, c_scale,
                                  reinterpret_cast<float2*>(d_data), static_cast<cudaStream_t>(stream));
    }
    if (c_type & TCV_C_PAIRED) {
        if (plan->g.n == 0) return TCV_OK;
        return launch_degrid_pair(plan, reinterpret_cast<const float2*>(d_grid), d_c, c_type & 0xff, c_scale,
                                  reinterpret_cast<float2*>(d_data), static_cast<cudaStream_t>(stream));
    }
    if (plan->degrid_variant == TCV_DEGRID_TILES) {
        if (plan->g.n == 0) return TCV_OK;
        return launch_degrid_tiles(plan, reinterpret_cast<const float2*>(d_grid), d_c, c_type, c_scale,
                                   reinterpret_cast<float2*>(d_data), static_cast<cudaStream_t>(stream));
    }
    return launch_degrid(plan, reinterpret_cast<const float2*>(d_grid), d_c, c_type, c_scale,
                         reinterpret_cast<float2*>(d_data), static_cast<cudaStream_t>(stream));
}

tcv_status tcv_plan_set_degrid_variant(tcv_plan* plan, int variant)
{
    if (!plan || (variant != TCV_DEGRID_TILES && variant != TCV_DEGRID_ANCHOR)) return TCV_ERR_ARG;
    plan->degrid_variant = variant;
    return TCV_OK;
}

tcv_status tcv_grid_raw(const float* d_data, int64_t n, int support, const void* d_c, int c_type,
                        float c_scale, int64_t c_len, const int32_t* d_coff, const int32_t* d_iu,
                        const int32_t* d_iv, float* d_grid, int g_size, void* d_work,
                        size_t work_bytes, void* stream)
{
    tcv_plan* p = nullptr;
    tcv_status s = tcv_plan_build(&p, d_iu, d_iv, d_coff, n, support, g_size, c_len, d_work,
                                  work_bytes, stream);
    if (s != TCV_OK) return s;
    s = tcv_plan_grid(p, d_data, d_c, c_type, c_scale, d_grid, stream);
    tcv_plan_destroy(p);
    return s;
}

tcv_status tcv_degrid_raw(const float* d_grid, int g_size, int support, const void* d_c,
                          int c_type, float c_scale, int64_t c_len, const int32_t* d_coff,
                          const int32_t* d_iu, const int32_t* d_iv, float* d_data, int64_t n,
                          void* d_work, size_t work_bytes, void* stream)
{
    tcv_plan* p = nullptr;
    tcv_status s = tcv_plan_build(&p, d_iu, d_iv, d_coff, n, support, g_size, c_len, d_work,
                                  work_bytes, stream);
    if (s != TCV_OK) return s;
    s = tcv_plan_degrid(p, d_grid, d_c, c_type, c_scale, d_data, stream);
    tcv_plan_destroy(p);
    return s;
}

}  // extern "C"
