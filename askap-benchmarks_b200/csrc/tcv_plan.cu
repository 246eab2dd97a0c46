// tcv_plan.cu -- binning of samples for the tile kernels.
//
// The reference grids samples in index order, straight into HBM-sized memory
// (attic/tConvolveMPI/Benchmark.cc:131-154; "some presorting might be advantageous", :113-114).
// Here a plan sorts (sample, tile) pairs with a device radix sort:
//   gridding  : every output tile of tw x th points gets the list of samples whose footprint
//               overlaps it (a footprint of sSize^2 touches up to max_tiles tiles);
//   degridding: every anchor tile of ta x ta gets the samples whose footprint's top-left corner
//               lies in it (each sample exactly once; one-job plans only; made with the plan's
//               binning only while the plan degrids by anchor tiles, else at that variant's first
//               use).
// Each cell's pair range comes from the run bounds of the sorted keys (no per-pair atomics), and
// the per-cell bookkeeping (tile offsets, the non-empty cells, per-group ranges, the work-unit
// lists) takes three launches over the cells.
// Kernel indices kid = cOffset / sSize^2 (w-plane major, then the oversampling offsets) are
// grouped into runs of whole w-planes whose slice of the table fits in L2 with room to spare.
// The sort key is the work cell (group, tile), ordered group-major, so all SMs work through the
// table one group at a time and the slice in use stays resident in L2; within a cell the stable
// sort keeps samples in index order (the reference's order).  The non-empty cells are compacted
// into work lists (with per-group ranges) that persistent kernels walk.
// A plan may hold several jobs sharing the table (a batch): their tiles are numbered in one
// space, job after job, so one sort and one sequence of launches covers all of them.
// Cells with many samples are split into work units of about `split` samples for gridding (the
// units of a cell write partial tiles that a fold adds into the grid in unit order) and of about
// `dsplit` samples for degridding (units are independent there), so that a plan with few busy
// tiles still spreads over every SM.
// Samples whose footprint or table range falls outside their grid or the table are counted and
// left out (sentinel key, sorted past the end).
#include "tcv_internal.cuh"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/iterator/transform_iterator.h>

#include <algorithm>
#include <climits>
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

// job of sample d: the last job whose first sample is <= d (empty jobs share their start with
// the next job, which is then the one holding d)
__device__ __forceinline__ int job_of(const uint32_t* __restrict__ job_start, int n_jobs, uint32_t d)
{
    int lo = 0, hi = n_jobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (job_start[mid] <= d)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// Variable-width plans: the sample's w-plane gives its footprint width (plane_s) and its plane
// group (plane_grp); the width is recorded per sample (ssz) for the tile kernels.
struct VarPlanes {
    const int32_t* __restrict__ wplane;
    const int32_t* __restrict__ plane_s;
    const int32_t* __restrict__ plane_grp;
    uint16_t* ssz;
};

// anchor tile of a footprint's top-left corner (fx, fy) in plane group grp
__device__ __forceinline__ uint32_t anchor_cell(const PlanGeom& g, uint32_t grp, uint32_t fx, uint32_t fy)
{
    return grp * uint32_t(g.natx * g.naty) + (fy / uint32_t(g.ta)) * uint32_t(g.natx) + fx / uint32_t(g.ta);
}

// The pairs of sample d (its footprint's tiles, then sentinels up to max_tiles) into kp/vp.
template <typename K>
__device__ __forceinline__ void sample_keys(const int32_t* __restrict__ iu, const int32_t* __restrict__ iv,
                                            const int32_t* __restrict__ coff, const PlanGeom& g,
                                            const JobDesc* __restrict__ jobs, const uint32_t* __restrict__ job_start,
                                            int64_t d, K* kp, uint32_t* vp, K* akeys, uint32_t* avals,
                                            uint32_t* atile_count, uint16_t* ntl, unsigned long long* rejected,
                                            const VarPlanes& var, bool with_anchors)
{
    const int job = g.n_jobs > 1 ? job_of(job_start, g.n_jobs, uint32_t(d)) : 0;
    const JobDesc jd = jobs[job];
    int64_t s = g.s, support = g.support;
    int plane = 0;
    bool plane_ok = true;
    if (g.var) {
        plane = var.wplane[d];
        plane_ok = plane >= 0 && plane < g.n_planes;
        s = plane_ok ? var.plane_s[plane] : 1;
        support = s / 2;
        var.ssz[d] = uint16_t(s);
    }
    const int64_t fx = (int64_t)iu[d] - support;
    const int64_t fy = iv[d];
    const int64_t co = coff[d];
    const bool ok = plane_ok && fx >= 0 && fx + s <= jd.g_size && fy >= 0 && fy + s <= jd.g_size && co >= 0 &&
                    co + s * s <= g.c_len;
    const K sentinel = K(1) << (g.key_bits - 1);
    if (!ok) {
        atomicAdd(rejected, 1ull);
        for (int t = 0; t < g.max_tiles; ++t) {
            kp[t] = sentinel;
            vp[t] = uint32_t(d);
        }
        ntl[d] = 0;
        if (with_anchors) {
            akeys[d] = K(1) << (g.akey_bits - 1);
            avals[d] = uint32_t(d);
        }
        return;
    }
    // in bounds, every operand below fits 32 bits (fx + s <= g_size, s*s <= c_len): 32-bit
    // divisions (a 64-bit one is a long software sequence, several per sample)
    const uint32_t ufx = uint32_t(fx), ufy = uint32_t(fy), us = uint32_t(s);
    const uint32_t grp = g.var ? uint32_t(var.plane_grp[plane])
                               : (co <= int64_t(0xffffffffll) ? uint32_t(co) / (us * us) : uint32_t(co / (s * s))) /
                                     uint32_t(g.kid_group);
    const uint32_t cell0 = grp * uint32_t(g.ntiles) + jd.tile_base;
    const uint32_t utw = uint32_t(g.tw), uth = uint32_t(g.th);
    const int tx0 = int(ufx / utw), tx1 = int((ufx + us - 1) / utw);
    const int ty0 = int(ufy / uth), ty1 = int((ufy + us - 1) / uth);
    int t = 0;
    for (int ty = ty0; ty <= ty1; ++ty)
        for (int tx = tx0; tx <= tx1; ++tx) {
            kp[t] = K(cell0 + uint32_t(ty) * uint32_t(jd.ntx) + uint32_t(tx));
            vp[t] = uint32_t(d);
            ++t;
        }
    ntl[d] = uint16_t(t);
    for (; t < g.max_tiles; ++t) {
        kp[t] = sentinel;
        vp[t] = uint32_t(d);
    }
    if (with_anchors) {
        const uint32_t at = anchor_cell(g, grp, ufx, ufy);
        akeys[d] = K(at);
        avals[d] = uint32_t(d);
        atomicAdd(&atile_count[at], 1u);
    }
}

// (sample, tile) pairs, max_tiles per sample in sample order.  kStaged: a block's pairs are built
// in shared memory and written out in one coalesced sweep (a sample's pairs are max_tiles apart
// across a warp otherwise).  The cells' sample counts come later from the sorted keys.
template <typename K, bool kStaged>
__global__ void plan_keys_kernel(const int32_t* __restrict__ iu, const int32_t* __restrict__ iv,
                                 const int32_t* __restrict__ coff, PlanGeom g, const JobDesc* __restrict__ jobs,
                                 const uint32_t* __restrict__ job_start, K* keys, uint32_t* vals, K* akeys,
                                 uint32_t* avals, uint32_t* atile_count, uint16_t* ntl, unsigned long long* rejected,
                                 VarPlanes var, bool with_anchors)
{
    extern __shared__ __align__(16) unsigned char pk_smem[];
    const int64_t d0 = int64_t(blockIdx.x) * blockDim.x;
    const int64_t d = d0 + threadIdx.x;
    K* sk = reinterpret_cast<K*>(pk_smem);
    uint32_t* sv = reinterpret_cast<uint32_t*>(sk + size_t(blockDim.x) * g.max_tiles);
    K* kp = kStaged ? sk + size_t(threadIdx.x) * g.max_tiles : keys + d * g.max_tiles;
    uint32_t* vp = kStaged ? sv + size_t(threadIdx.x) * g.max_tiles : vals + d * g.max_tiles;
    if (d < g.n)
        sample_keys<K>(iu, iv, coff, g, jobs, job_start, d, kp, vp, akeys, avals, atile_count, ntl, rejected, var,
                       with_anchors);
    if (kStaged) {
        __syncthreads();
        const int64_t rows = g.n - d0 < int64_t(blockDim.x) ? g.n - d0 : int64_t(blockDim.x);
        const int64_t m = rows * g.max_tiles;
        K* gk = keys + d0 * g.max_tiles;
        uint32_t* gv = vals + d0 * g.max_tiles;
        for (int64_t i = threadIdx.x; i < m; i += blockDim.x) {
            gk[i] = sk[i];
            gv[i] = sv[i];
        }
    }
}

// Cell bounds from the sorted keys: run_start[c] = first pair of cell c, run_end[c] = one past its
// last (both stay 0 for an empty cell); sentinel pairs (left-out samples) sort last and count for
// no cell.
template <typename K>
__global__ void run_bounds_kernel(const K* __restrict__ keys, int64_t np, int key_bits, uint32_t* run_start,
                                  uint32_t* run_end)
{
    const K sentinel = K(1) << (key_bits - 1);
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < np; i += stride) {
        const K k = keys[i];
        if (k >= sentinel) continue;
        if (i == 0 || keys[i - 1] != k) run_start[k] = uint32_t(i);
        if (i + 1 == np || keys[i + 1] != k) run_end[k] = uint32_t(i + 1);
    }
}

// The anchor keys alone (one-job plans of one footprint width), for an anchor binning made after
// the plan's own: the same bounds and cells as plan_keys_kernel.
template <typename K>
__global__ void anchor_keys_kernel(const int32_t* __restrict__ iu, const int32_t* __restrict__ iv,
                                   const int32_t* __restrict__ coff, PlanGeom g, K* akeys, uint32_t* avals,
                                   uint32_t* atile_count)
{
    const int64_t d = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (d >= g.n) return;
    const int64_t s = g.s;
    const int64_t fx = (int64_t)iu[d] - g.support, fy = iv[d], co = coff[d];
    const bool ok = fx >= 0 && fx + s <= g.g_size && fy >= 0 && fy + s <= g.g_size && co >= 0 && co + s * s <= g.c_len;
    avals[d] = uint32_t(d);
    if (!ok) {
        akeys[d] = K(1) << (g.akey_bits - 1);
        return;
    }
    const uint32_t us = uint32_t(s);
    const uint32_t grp =
        (co <= int64_t(0xffffffffll) ? uint32_t(co) / (us * us) : uint32_t(co / (s * s))) / uint32_t(g.kid_group);
    const uint32_t at = anchor_cell(g, grp, uint32_t(fx), uint32_t(fy));
    akeys[d] = K(at);
    atomicAdd(&atile_count[at], 1u);
}

// the job table of a one-job plan (written on the device, so building such a plan is device
// work only)
__global__ void one_job_kernel(JobDesc* jobs, uint32_t* job_start, int g_size, int ntx, uint32_t ntiles, uint32_t n)
{
    jobs[0] = JobDesc{nullptr, g_size, ntx, 0u, ntiles};
    job_start[0] = 0;
    job_start[1] = n;
}

// the job table of a batch of up to kParamJobs jobs, passed by value: no host-memory copy, so
// creating such a plan neither waits for the stream nor keeps a host buffer alive
constexpr int kParamJobs = 128;
struct JobTableParam {
    JobDesc jobs[kParamJobs];
    uint32_t start[kParamJobs + 1];
};
static_assert(sizeof(JobTableParam) <= 4000, "kernel parameter space");

__global__ void job_table_kernel(const JobTableParam t, int n_jobs, JobDesc* jobs, uint32_t* job_start)
{
    const int j = threadIdx.x;
    if (j < n_jobs) jobs[j] = t.jobs[j];
    if (j <= n_jobs) job_start[j] = t.start[j];
}

// per tile of all jobs: its record (job, column, row)
__global__ void tile_info_kernel(const JobDesc* __restrict__ jobs, int n_jobs, uint32_t ntiles, uint32_t* tinfo)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntiles) return;
    int lo = 0, hi = n_jobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (jobs[mid].tile_base <= t)
            lo = mid;
        else
            hi = mid - 1;
    }
    const uint32_t local = t - jobs[lo].tile_base;
    const uint32_t ntx = uint32_t(jobs[lo].ntx);
    tinfo[t] = tile_record(uint32_t(lo), local % ntx, local / ntx);
}

struct NonZero {
    __host__ __device__ __forceinline__ bool operator()(const uint32_t& v) const { return v != 0; }
};

// ------------------------------------------------------------------------------------------
// Cell bookkeeping after the sort, in three launches over the cells (c = group * ntiles + tile):
// per-block sums, one scan of those sums, then every cell's outputs.
//   tile_start[c]     first sorted pair of cell c (exclusive sum of tile_count)
//   items, n_items    the non-empty cells in order; group_start[g] = non-empty cells before
//                     cell g*ntiles (group g's first item)
//   per unit list (the gridding split, and the degridding split when it differs): per item its
//   units (a cell of cnt >= 2*split samples makes cnt/split units, any other non-empty cell one),
//   first unit and first partial tile (split cells only); the units themselves, unit q of a cell
//   taking its samples [q*cnt/nu, (q+1)*cnt/nu); group_ustart[g] = units of the cells before
//   cell g*ntiles
// Item-indexed entries past n_items hold 0 units and the totals, as exclusive sums would.
// ------------------------------------------------------------------------------------------
constexpr int kCellThreads = 256;
constexpr int kCellPer = 1;  // consecutive cells per thread
constexpr uint32_t kCellBlock = uint32_t(kCellThreads) * kCellPer;
constexpr int kCellVals = 6;  // pairs, non-empty, units, partials (gridding), units, partials (degridding)

struct CellArgs {
    uint32_t* tile_count;  // run ends on entry (run_bounds_kernel), the cells' pair counts on exit
    uint32_t cells, ntiles, split, dsplit;
    int n_groups;
    bool own_d;
    uint32_t* part;  // [kCellVals][blocks] block sums, scanned in place, then the kCellVals totals
    uint32_t *tile_start, *items, *n_items, *group_start;
    uint32_t *nunits, *ustart, *pstart, *group_ustart;
    uint4* units;
    uint32_t *d_nunits, *d_ustart, *d_pstart, *d_group_ustart;
    uint4* d_units;
};

__device__ __forceinline__ uint32_t units_of(uint32_t cnt, uint32_t split)
{
    return cnt == 0 ? 0u : ((split && cnt >= 2u * split) ? cnt / split : 1u);
}

__device__ __forceinline__ void cell_vals(uint32_t cnt, uint32_t split, uint32_t dsplit, uint32_t* v)
{
    const uint32_t nu = units_of(cnt, split), dnu = units_of(cnt, dsplit);
    v[0] = cnt;
    v[1] = cnt ? 1u : 0u;
    v[2] = nu;
    v[3] = nu > 1 ? nu : 0u;
    v[4] = dnu;
    v[5] = dnu > 1 ? dnu : 0u;
}

// pairs of each cell: run end - run start (tile_start holds the run starts until cell_out_kernel)
__device__ __forceinline__ void load_counts(const CellArgs& a, uint32_t c0, uint32_t* cnt)
{
#pragma unroll
    for (int e = 0; e < kCellPer; ++e) cnt[e] = c0 + e < a.cells ? a.tile_count[c0 + e] - a.tile_start[c0 + e] : 0u;
}

__global__ void __launch_bounds__(kCellThreads) cell_sums_kernel(CellArgs a)
{
    __shared__ uint32_t ws[kCellVals][kCellThreads / 32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t cnt[kCellPer], s[kCellVals] = {};
    load_counts(a, blockIdx.x * kCellBlock + threadIdx.x * kCellPer, cnt);
#pragma unroll
    for (int e = 0; e < kCellPer; ++e) {
        uint32_t v[kCellVals];
        cell_vals(cnt[e], a.split, a.dsplit, v);
#pragma unroll
        for (int j = 0; j < kCellVals; ++j) s[j] += v[j];
    }
#pragma unroll
    for (int j = 0; j < kCellVals; ++j) {
#pragma unroll
        for (int o = 16; o; o >>= 1) s[j] += __shfl_xor_sync(0xffffffffu, s[j], o);
        if (lane == 0) ws[j][warp] = s[j];
    }
    __syncthreads();
    if (threadIdx.x < kCellVals) {
        uint32_t t = 0;
        for (int w = 0; w < kCellThreads / 32; ++w) t += ws[threadIdx.x][w];
        a.part[threadIdx.x * gridDim.x + blockIdx.x] = t;
    }
}

// one block: exclusive sums of every row of part, the totals after them, and the totals'
// entries of n_items, group_start and group_ustart
__global__ void __launch_bounds__(1024) cell_scan_kernel(CellArgs a, uint32_t blocks)
{
    __shared__ uint32_t wsum[32];
    __shared__ uint32_t carry_s;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int j = 0; j < kCellVals; ++j) {
        uint32_t* row = a.part + size_t(j) * blocks;
        if (threadIdx.x == 0) carry_s = 0;
        __syncthreads();
        for (uint32_t base = 0; base < blocks; base += 1024) {
            const uint32_t i = base + threadIdx.x;
            const uint32_t v = i < blocks ? row[i] : 0u;
            uint32_t x = v;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
                if (lane >= d) x += y;
            }
            if (lane == 31) wsum[warp] = x;
            __syncthreads();
            if (warp == 0) {
                uint32_t t = wsum[lane];
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    const uint32_t y = __shfl_up_sync(0xffffffffu, t, d);
                    if (lane >= d) t += y;
                }
                wsum[lane] = t;
            }
            __syncthreads();
            const uint32_t excl = carry_s + (warp ? wsum[warp - 1] : 0u) + x - v;
            if (i < blocks) row[i] = excl;
            __syncthreads();  // carry_s and wsum are read before they change
            if (threadIdx.x == 1023) carry_s = excl + v;
            __syncthreads();
        }
        if (threadIdx.x == 0) a.part[size_t(kCellVals) * blocks + j] = carry_s;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const uint32_t* tot = a.part + size_t(kCellVals) * blocks;
        *a.n_items = tot[1];
        a.group_start[a.n_groups] = tot[1];
        a.group_ustart[a.n_groups] = tot[2];
        if (a.own_d) a.d_group_ustart[a.n_groups] = tot[4];
    }
}

// unit q takes the cell's pairs [floor(q*cnt/nu), floor((q+1)*cnt/nu)), stepped without a division
// per unit: floor((q+1)*cnt/nu) = floor(q*cnt/nu) + cnt/nu + (carry of the remainders)
__device__ __forceinline__ void write_units(uint4* units, uint32_t cell, uint32_t cnt, uint32_t first, uint32_t nu,
                                            uint32_t u0, uint32_t p0)
{
    const uint32_t base = cnt / nu, rem = cnt % nu;
    uint32_t b0 = 0, r = 0;
    for (uint32_t q = 0; q < nu; ++q) {
        uint32_t b1 = b0 + base;
        r += rem;
        if (r >= nu) {
            r -= nu;
            ++b1;
        }
        units[u0 + q] = make_uint4(cell, first + b0, b1 - b0, nu > 1 ? p0 + q : kDirect);
        b0 = b1;
    }
}

__global__ void __launch_bounds__(kCellThreads) cell_out_kernel(CellArgs a)
{
    __shared__ uint32_t ws[kCellVals][kCellThreads / 32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t blocks = gridDim.x;
    const uint32_t* tot = a.part + size_t(kCellVals) * blocks;
    const uint32_t c0 = blockIdx.x * kCellBlock + threadIdx.x * kCellPer;
    uint32_t cnt[kCellPer], s[kCellVals] = {};
    load_counts(a, c0, cnt);
#pragma unroll
    for (int e = 0; e < kCellPer; ++e) {
        uint32_t v[kCellVals];
        cell_vals(cnt[e], a.split, a.dsplit, v);
#pragma unroll
        for (int j = 0; j < kCellVals; ++j) s[j] += v[j];
    }
    // the thread's first cell: block offset + the lower warps' sums + the lower lanes' sums
    uint32_t x[kCellVals];
#pragma unroll
    for (int j = 0; j < kCellVals; ++j) {
        x[j] = s[j];
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x[j], d);
            if (lane >= d) x[j] += y;
        }
        if (lane == 31) ws[j][warp] = x[j];
    }
    __syncthreads();
    uint32_t pre[kCellVals];
#pragma unroll
    for (int j = 0; j < kCellVals; ++j) {
        uint32_t w = 0;
        for (int k = 0; k < warp; ++k) w += ws[j][k];
        pre[j] = a.part[size_t(j) * blocks + blockIdx.x] + w + x[j] - s[j];
    }
#pragma unroll
    for (int e = 0; e < kCellPer; ++e) {
        const uint32_t c = c0 + e;
        if (c >= a.cells) break;
        uint32_t v[kCellVals];
        cell_vals(cnt[e], a.split, a.dsplit, v);
        a.tile_start[c] = pre[0];
        a.tile_count[c] = cnt[e];
        if (c % a.ntiles == 0) {
            const uint32_t gi = c / a.ntiles;
            a.group_start[gi] = pre[1];
            a.group_ustart[gi] = pre[2];
            if (a.own_d) a.d_group_ustart[gi] = pre[4];
        }
        if (cnt[e]) {
            const uint32_t k = pre[1];
            a.items[k] = c;
            a.nunits[k] = v[2];
            a.ustart[k] = pre[2];
            a.pstart[k] = pre[3];
            write_units(a.units, c, cnt[e], pre[0], v[2], pre[2], pre[3]);
            if (a.own_d) {
                a.d_nunits[k] = v[4];
                a.d_ustart[k] = pre[4];
                a.d_pstart[k] = pre[5];
                write_units(a.d_units, c, cnt[e], pre[0], v[4], pre[4], pre[5]);
            }
        }
        if (c >= tot[1]) {  // item-indexed entries past the last item
            a.nunits[c] = 0;
            a.ustart[c] = tot[2];
            a.pstart[c] = tot[3];
            if (a.own_d) {
                a.d_nunits[c] = 0;
                a.d_ustart[c] = tot[4];
                a.d_pstart[c] = tot[5];
            }
        }
#pragma unroll
        for (int j = 0; j < kCellVals; ++j) pre[j] += v[j];
    }
}

inline size_t align_up(size_t x, size_t a = 256) { return (x + a - 1) / a * a; }

inline size_t grid_cells(const PlanGeom& g) { return size_t(g.n_groups) * size_t(g.ntiles); }
// a split cell of cnt >= 2*split samples makes floor(cnt/split) units, so the units of split cells
// number at most pairs/split, and every other non-empty cell makes one
inline size_t max_partials(const PlanGeom& g, int split) { return split ? size_t(g.n) * g.max_tiles / size_t(split) : 0; }
inline size_t max_units(const PlanGeom& g, int split) { return grid_cells(g) + max_partials(g, split); }
inline bool own_degrid_units(const PlanGeom& g) { return g.dsplit != g.split; }
inline size_t anchor_cells(const PlanGeom& g) { return g.anchors ? size_t(g.n_groups) * g.natx * g.naty : 0; }

inline uint32_t cell_blocks(const PlanGeom& g) { return uint32_t((grid_cells(g) + kCellBlock - 1) / kCellBlock); }
inline size_t cell_scratch_bytes(const PlanGeom& g) { return (size_t(cell_blocks(g)) + 1) * kCellVals * 4; }

template <typename K>
size_t cub_temp_bytes(const PlanGeom& g)
{
    size_t a = 0, b = 0, c = 0, d = 0, f = 0;
    const int64_t np = g.n * g.max_tiles;
    const int acells = int(anchor_cells(g));
    cub::DoubleBuffer<K> kb(nullptr, nullptr);
    cub::DoubleBuffer<uint32_t> vb(nullptr, nullptr);
    thrust::counting_iterator<uint32_t> it(0);
    thrust::transform_iterator<NonZero, const uint32_t*> fl((const uint32_t*)nullptr, NonZero());
    cub::DeviceRadixSort::SortPairs(nullptr, a, kb, vb, np, 0, g.key_bits);
    c = cell_scratch_bytes(g);  // the cell sums use this space after the sort
    if (g.anchors) {
        cub::DeviceRadixSort::SortPairs(nullptr, b, kb, vb, g.n, 0, g.akey_bits);
        cub::DeviceScan::ExclusiveSum(nullptr, d, (uint32_t*)nullptr, (uint32_t*)nullptr, acells);
        cub::DeviceSelect::Flagged(nullptr, f, it, fl, (uint32_t*)nullptr, (uint32_t*)nullptr, acells);
    }
    return std::max(std::max(std::max(a, b), std::max(c, d)), f);
}

// sort, scan and compact the anchor keys (written by plan_keys_kernel or anchor_keys_kernel)
template <typename K>
tcv_status sort_anchors(tcv_plan* p, cudaStream_t st)
{
    const PlanGeom& g = p->g;
    const int acells = int(anchor_cells(g));
    if (g.n > 0) {
        cub::DoubleBuffer<K> akb(static_cast<K*>(p->akeys[0]), static_cast<K*>(p->akeys[1]));
        cub::DoubleBuffer<uint32_t> avb(p->avals[0], p->avals[1]);
        size_t tb = p->cub_bytes;
        TCV_CUDA(cub::DeviceRadixSort::SortPairs(p->cub_temp, tb, akb, avb, g.n, 0, g.akey_bits, st));
        p->asel = avb.selector;
    } else {
        p->asel = 0;
    }
    thrust::counting_iterator<uint32_t> it(0);
    size_t tb = p->cub_bytes;
    TCV_CUDA(cub::DeviceScan::ExclusiveSum(p->cub_temp, tb, p->atile_count, p->atile_start, acells, st));
    thrust::transform_iterator<NonZero, const uint32_t*> afl(p->atile_count, NonZero());
    tb = p->cub_bytes;
    TCV_CUDA(cub::DeviceSelect::Flagged(p->cub_temp, tb, it, afl, p->aitems, p->n_aitems, acells, st));
    return TCV_OK;
}

template <typename K>
tcv_status bin_anchors_now(tcv_plan* p, cudaStream_t st)
{
    const PlanGeom& g = p->g;
    TCV_CUDA(cudaMemsetAsync(p->atile_count, 0, sizeof(uint32_t) * anchor_cells(g), st));
    if (g.n > 0) {
        anchor_keys_kernel<K><<<unsigned((g.n + 255) / 256), 256, 0, st>>>(
            p->iu, p->iv, p->coff, g, static_cast<K*>(p->akeys[0]), p->avals[0], p->atile_count);
        TCV_CUDA(cudaGetLastError());
    }
    return sort_anchors<K>(p, st);
}

bool stream_capturing(cudaStream_t st)
{
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    return cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone;
}

// The anchor binning of a plan's samples, made now unless the last binning made it (a cache of
// the plan's samples, so a const plan may fill it).
tcv_status plan_anchors_ready(const tcv_plan* cp, cudaStream_t st)
{
    tcv_plan* p = const_cast<tcv_plan*>(cp);
    if (p->anchors_ready && !p->anchors_stale) return TCV_OK;
    const tcv_status s = p->g.key64 ? bin_anchors_now<uint64_t>(p, st) : bin_anchors_now<uint32_t>(p, st);
    if (s == TCV_OK && !stream_capturing(st)) p->anchors_ready = true;  // a captured one runs at each replay
    return s;
}

// The anchor binning is made with the plan's only when the plan degrids by anchor tiles at that
// time; otherwise the first anchor degridding makes it (plan_anchors_ready).
template <typename K>
tcv_status build(tcv_plan* p, const int32_t* iu, const int32_t* iv, const int32_t* coff, cudaStream_t st)
{
    const PlanGeom& g = p->g;
    const int64_t np = g.n * g.max_tiles;
    const int cells = int(grid_cells(g)), acells = int(anchor_cells(g));
    const bool with_anchors = g.anchors && p->degrid_variant == TCV_DEGRID_ANCHOR;
    TCV_CUDA(cudaMemsetAsync(p->tile_count, 0, sizeof(uint32_t) * size_t(cells), st));  // run ends
    TCV_CUDA(cudaMemsetAsync(p->tile_start, 0, sizeof(uint32_t) * size_t(cells), st));  // run starts
    if (with_anchors) TCV_CUDA(cudaMemsetAsync(p->atile_count, 0, sizeof(uint32_t) * size_t(acells), st));
    TCV_CUDA(cudaMemsetAsync(p->rejected, 0, sizeof(unsigned long long), st));
    TCV_CUDA(cudaMemsetAsync(p->status, 0, kStatusWords * sizeof(unsigned int), st));
    if (g.n > 0) {
        const VarPlanes var{p->wplane, p->plane_s, p->plane_grp, p->ssz};
        // staged key writes while a block's pairs fit the default 48 KB of shared memory
        const size_t per = size_t(g.max_tiles) * (sizeof(K) + 4);
        int threads = 256;
        while (threads > 64 && size_t(threads) * per > (48u << 10)) threads /= 2;
        const bool staged = size_t(threads) * per <= (48u << 10);
        if (!staged) threads = 256;
        const unsigned blocks = unsigned((g.n + threads - 1) / threads);
        K* k0 = static_cast<K*>(p->keys[0]);
        K* ak0 = static_cast<K*>(p->akeys[0]);
        if (staged)
            plan_keys_kernel<K, true><<<blocks, threads, size_t(threads) * per, st>>>(
                iu, iv, coff, g, p->jobs, p->job_start, k0, p->vals[0], ak0, p->avals[0], p->atile_count, p->ntl,
                p->rejected, var, with_anchors);
        else
            plan_keys_kernel<K, false><<<blocks, threads, 0, st>>>(iu, iv, coff, g, p->jobs, p->job_start, k0,
                                                                   p->vals[0], ak0, p->avals[0], p->atile_count,
                                                                   p->ntl, p->rejected, var, with_anchors);
        TCV_CUDA(cudaGetLastError());
        cub::DoubleBuffer<K> kb(static_cast<K*>(p->keys[0]), static_cast<K*>(p->keys[1]));
        cub::DoubleBuffer<uint32_t> vb(p->vals[0], p->vals[1]);
        size_t tb = p->cub_bytes;
        TCV_CUDA(cub::DeviceRadixSort::SortPairs(p->cub_temp, tb, kb, vb, np, 0, g.key_bits, st));
        p->sel = vb.selector;
        int sms = 148, dev = 0;
        if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const int64_t rb = std::min<int64_t>((np + 255) / 256, int64_t(sms) * 8);
        run_bounds_kernel<K><<<unsigned(rb), 256, 0, st>>>(kb.Current(), np, g.key_bits, p->tile_start, p->tile_count);
        TCV_CUDA(cudaGetLastError());
    } else {
        p->sel = 0;
    }
    const bool own_d = own_degrid_units(g);
    const CellArgs ca{p->tile_count, uint32_t(cells), uint32_t(g.ntiles), uint32_t(g.split), uint32_t(g.dsplit),
                      g.n_groups, own_d, static_cast<uint32_t*>(p->cub_temp), p->tile_start, p->items, p->n_items,
                      p->group_start, p->nunits, p->ustart, p->pstart, p->group_ustart, p->units,
                      own_d ? p->d_nunits : nullptr, own_d ? p->d_ustart : nullptr, own_d ? p->d_pstart : nullptr,
                      own_d ? p->d_group_ustart : nullptr, own_d ? p->d_units : nullptr};
    const uint32_t cb = cell_blocks(g);
    cell_sums_kernel<<<cb, kCellThreads, 0, st>>>(ca);
    TCV_CUDA(cudaGetLastError());
    cell_scan_kernel<<<1, 1024, 0, st>>>(ca, cb);
    TCV_CUDA(cudaGetLastError());
    cell_out_kernel<<<cb, kCellThreads, 0, st>>>(ca);
    TCV_CUDA(cudaGetLastError());
    if (with_anchors) TCV_CHECK(sort_anchors<K>(p, st));
    p->anchors_ready = with_anchors;
    // a captured binning without anchors may be replayed on new samples behind the host's back:
    // from then on an anchor degridding always bins the anchors itself
    if (g.anchors && !with_anchors && stream_capturing(st)) p->anchors_stale = true;
    return TCV_OK;
}

bool valid_tuning(const tcv_tuning* t)
{
    if (!t) return true;
    const bool rows_ok = t->tile_rows == 0 || t->tile_rows == 8 || t->tile_rows == 16 || t->tile_rows == 32;
    const bool kernel_ok = t->kernel == 0 || (t->kernel >= 1 && t->kernel <= 3 && t->tile_rows == 8);
    return rows_ok && kernel_ok && t->group_mib >= -1 && t->split >= 0 && t->split <= (1 << 24) &&
           t->degrid_split >= 0 && t->degrid_split <= (1 << 24);
}

// Lay the plan's arrays out in d_work and write the job table: from host memory for a batch,
// by a one-thread kernel for a one-job plan (so that plan_init is device work only).
tcv_status plan_create(tcv_plan* p, void* d_work, size_t work_bytes, cudaStream_t st)
{
    const PlanGeom& g = p->g;
    size_t cb = 0;
    const size_t need = plan_bytes(g, &cb);
    if (work_bytes < need) return TCV_ERR_WORKSPACE;
    const size_t ks = g.key64 ? 8 : 4;
    const size_t np = size_t(g.n) * g.max_tiles;
    const size_t an = g.anchors ? size_t(g.n) : 0;
    char* w = static_cast<char*>(d_work);
    auto take = [&](size_t bytes) {
        char* r = w;
        w += align_up(bytes);
        return static_cast<void*>(r);
    };
    p->jobs = static_cast<JobDesc*>(take(size_t(g.n_jobs) * sizeof(JobDesc)));
    p->job_start = static_cast<uint32_t*>(take(size_t(g.n_jobs + 1) * 4));
    p->tinfo = static_cast<uint32_t*>(take(size_t(g.ntiles) * 4));
    p->ntl = static_cast<uint16_t*>(take(size_t(g.n) * 2));
    if (g.var) {
        p->ssz = static_cast<uint16_t*>(take(size_t(g.n) * 2));
        p->plane_s = static_cast<int32_t*>(take(size_t(g.n_planes) * 4));
        p->plane_grp = static_cast<int32_t*>(take(size_t(g.n_planes) * 4));
    }
    p->keys[0] = take(np * ks);
    p->keys[1] = take(np * ks);
    p->vals[0] = static_cast<uint32_t*>(take(np * 4));
    p->vals[1] = static_cast<uint32_t*>(take(np * 4));
    p->akeys[0] = take(an * ks);
    p->akeys[1] = take(an * ks);
    p->avals[0] = static_cast<uint32_t*>(take(an * 4));
    p->avals[1] = static_cast<uint32_t*>(take(an * 4));
    const size_t cells = grid_cells(g), acells = anchor_cells(g);
    p->tile_count = static_cast<uint32_t*>(take(cells * 4));
    p->tile_start = static_cast<uint32_t*>(take(cells * 4));
    p->items = static_cast<uint32_t*>(take(cells * 4));
    p->n_items = static_cast<uint32_t*>(take(4));
    p->group_start = static_cast<uint32_t*>(take(size_t(g.n_groups + 1) * 4));
    p->group_ustart = static_cast<uint32_t*>(take(size_t(g.n_groups + 1) * 4));
    p->nunits = static_cast<uint32_t*>(take(cells * 4));
    p->ustart = static_cast<uint32_t*>(take(cells * 4));
    p->pstart = static_cast<uint32_t*>(take(cells * 4));
    p->units = static_cast<uint4*>(take(max_units(g, g.split) * sizeof(uint4)));
    p->partial = static_cast<float2*>(take(max_partials(g, g.split) * size_t(g.tw) * g.th * sizeof(float2)));
    if (own_degrid_units(g)) {
        p->d_group_ustart = static_cast<uint32_t*>(take(size_t(g.n_groups + 1) * 4));
        p->d_nunits = static_cast<uint32_t*>(take(cells * 4));
        p->d_ustart = static_cast<uint32_t*>(take(cells * 4));
        p->d_pstart = static_cast<uint32_t*>(take(cells * 4));
        p->d_units = static_cast<uint4*>(take(max_units(g, g.dsplit) * sizeof(uint4)));
    } else {
        p->d_group_ustart = p->group_ustart;
        p->d_units = p->units;
    }
    p->atile_count = static_cast<uint32_t*>(take(acells * 4));
    p->atile_start = static_cast<uint32_t*>(take(acells * 4));
    p->aitems = static_cast<uint32_t*>(take(acells * 4));
    p->n_aitems = static_cast<uint32_t*>(take(4));
    p->rejected = static_cast<unsigned long long*>(take(sizeof(unsigned long long)));
    p->status = static_cast<unsigned int*>(take(kStatusWords * sizeof(unsigned int)));
    p->slots = static_cast<float2*>(take(np * sizeof(float2)));
    p->grec = (g.dense || g.ddense) ? static_cast<int4*>(take(np * sizeof(int4))) : nullptr;
    p->cub_temp = take(cb);
    p->cub_bytes = cb;
    p->degrid_variant = TCV_DEGRID_TILES;
    if (p->batch && g.n_jobs <= kParamJobs) {
        JobTableParam t{};
        for (int j = 0; j < g.n_jobs; ++j) t.jobs[j] = p->host_jobs[size_t(j)];
        for (int j = 0; j <= g.n_jobs; ++j) t.start[j] = p->host_job_start[size_t(j)];
        job_table_kernel<<<1, kParamJobs + 1, 0, st>>>(t, g.n_jobs, p->jobs, p->job_start);
        TCV_CUDA(cudaGetLastError());
    } else if (p->batch) {
        TCV_CUDA(cudaMemcpyAsync(p->jobs, p->host_jobs.data(), p->host_jobs.size() * sizeof(JobDesc),
                                 cudaMemcpyHostToDevice, st));
        TCV_CUDA(cudaMemcpyAsync(p->job_start, p->host_job_start.data(), p->host_job_start.size() * 4,
                                 cudaMemcpyHostToDevice, st));
    } else {
        one_job_kernel<<<1, 1, 0, st>>>(p->jobs, p->job_start, g.g_size, g.ntx, uint32_t(g.ntiles), uint32_t(g.n));
        TCV_CUDA(cudaGetLastError());
    }
    tile_info_kernel<<<unsigned((g.ntiles + 255) / 256), 256, 0, st>>>(p->jobs, g.n_jobs, uint32_t(g.ntiles), p->tinfo);
    TCV_CUDA(cudaGetLastError());
    if (g.var) {  // the plane widths and groups (host vectors owned by the plan)
        TCV_CUDA(cudaMemcpyAsync(p->plane_s, p->host_plane_s.data(), size_t(g.n_planes) * 4, cudaMemcpyHostToDevice, st));
        TCV_CUDA(cudaMemcpyAsync(p->plane_grp, p->host_plane_grp.data(), size_t(g.n_planes) * 4,
                                 cudaMemcpyHostToDevice, st));
    }
    return TCV_OK;
}

// limits of the plan's index types: 32-bit sample indices in the sort (16 tile pairs per sample
// at most within 2^32), 32-bit cells, and the fields of the tile record (jobs, tile columns and
// rows per job; g_max is the largest grid side)
bool geom_supported(const PlanGeom& g)
{
    if (g.n_jobs > kMaxJobs) return false;
    if ((g.g_size + g.tw - 1) / g.tw > kMaxTilesPerSide || (g.g_size + g.th - 1) / g.th > kMaxTilesPerSide) return false;
    if (g.n >= (int64_t(1) << 32) / 16) return false;
    if (g.n * g.max_tiles >= (int64_t(1) << 31)) return false;
    if (int64_t(g.n_groups) * g.ntiles >= (int64_t(1) << 31)) return false;
    if (g.max_tiles > 65535) return false;
    if (max_units(g, g.split) >= (size_t(1) << 31) || max_units(g, g.dsplit) >= (size_t(1) << 31)) return false;
    return true;
}

}  // namespace

// Tile geometry.  Gridding tiles are 64 x 4*rows points (8 warps of 32 columns x rows rows).
// Degridding anchor tiles are the largest ta whose staged region (ta + sSize - 1)^2 complex
// points fits in shared memory next to the partial sums; beyond that the direct kernel reads
// the grid from global memory.
PlanGeom make_geom(int64_t n, int support, const int* g_sizes, int n_jobs, int64_t c_len, const tcv_tuning* t,
                   bool anchors)
{
    PlanGeom g{};
    g.n = n;
    g.support = support;
    g.s = 2 * support + 1;
    g.c_len = c_len;
    g.n_jobs = n_jobs;
    g.g_size = 0;
    for (int j = 0; j < n_jobs; ++j) g.g_size = std::max(g.g_size, g_sizes[j]);
    const int64_t s2 = int64_t(g.s) * g.s;
    const int64_t nk = (c_len + s2 - 1) / s2;
    g.kid_bits = bits_for(uint64_t(nk));
    // kernels per group: whole planes of 64 (8 x 8 oversampling) whose complex64 slice is about
    // group_mib MiB (32 by default, a quarter of the 126 MB L2)
    g.group_mib = (t && t->group_mib) ? t->group_mib : 32;
    int64_t kg = nk;
    if (g.group_mib > 0) {
        const int64_t per_kernel = s2 * 8;
        kg = ((int64_t(g.group_mib) << 20) / per_kernel) / 64 * 64;
        if (kg < 64) kg = 64;
    }
    if (kg > nk) kg = nk < 1 ? 1 : nk;
    g.kid_group = int(kg);
    g.n_groups = int((nk + kg - 1) / kg);
    if (g.n_groups < 1) g.n_groups = 1;
    g.group_bits = bits_for(uint64_t(g.n_groups - 1));
    g.rows = (t && t->tile_rows) ? t->tile_rows : 16;
    g.split = t ? t->split : 0;
    g.dsplit = t ? t->degrid_split : 0;
    g.dense = t && (t->kernel & 1);
    g.ddense = t && (t->kernel & 2);
    g.tw = kTileW;
    g.th = tile_height(g.rows);
    g.ntiles = 0;
    for (int j = 0; j < n_jobs; ++j)
        g.ntiles += int64_t((g_sizes[j] + g.tw - 1) / g.tw) * ((g_sizes[j] + g.th - 1) / g.th);
    g.ntx = n_jobs == 1 ? (g.g_size + g.tw - 1) / g.tw : 0;
    g.nty = n_jobs == 1 ? (g.g_size + g.th - 1) / g.th : 0;
    g.max_tiles = ((g.s + g.tw - 2) / g.tw + 1) * ((g.s + g.th - 2) / g.th + 1);
    g.tile_bits = bits_for(uint64_t(g.n_groups) * uint64_t(g.ntiles) - 1);
    g.key_bits = g.tile_bits + 1;  // cell, plus the sentinel bit

    g.anchors = anchors && n_jobs == 1;
    g.degrid_mode = 1;
    g.ta = 32;
    g.degrid_parts = 4;
    if (g.anchors) {
        constexpr size_t kSmemBudget = 220 * 1024;  // of 227 KB per CTA; the rest holds partial sums
        const int cand[] = {128, 96, 64, 48, 32, 16, 8};
        for (int ta : cand) {
            const int w = ((ta + g.s - 1) + 1) & ~1;
            const int h = ta + g.s - 1;
            if (w <= 256 && h <= 256 && size_t(w) * h * 8 <= kSmemBudget && ta <= g.g_size) {
                g.ta = ta;
                g.box_w = w;
                g.box_h = h;
                g.degrid_mode = (g.g_size % 2 == 0) ? 0 : 1;  // TMA row stride must be a multiple of 16 B
                break;
            }
        }
        g.natx = (g.g_size + g.ta - 1) / g.ta;
        g.naty = (g.g_size + g.ta - 1) / g.ta;
        g.atile_bits = bits_for(uint64_t(g.n_groups) * g.natx * g.naty - 1);
        g.akey_bits = g.atile_bits + 1;
    }
    g.key64 = g.key_bits > 32 || (g.anchors && g.akey_bits > 32);
    return g;
}

size_t plan_bytes(const PlanGeom& g, size_t* cub_bytes_out)
{
    const size_t ks = g.key64 ? 8 : 4;
    const size_t np = size_t(g.n) * g.max_tiles;
    const size_t an = g.anchors ? size_t(g.n) : 0;
    const size_t cb = g.key64 ? cub_temp_bytes<uint64_t>(g) : cub_temp_bytes<uint32_t>(g);
    if (cub_bytes_out) *cub_bytes_out = cb;
    size_t b = 0;
    b += align_up(size_t(g.n_jobs) * sizeof(JobDesc)) + align_up(size_t(g.n_jobs + 1) * 4);
    b += align_up(size_t(g.ntiles) * 4) + align_up(size_t(g.n) * 2);
    if (g.var) b += align_up(size_t(g.n) * 2) + 2 * align_up(size_t(g.n_planes) * 4);
    b += 2 * align_up(np * ks) + 2 * align_up(np * 4);
    b += 2 * align_up(an * ks) + 2 * align_up(an * 4);
    const size_t cells = grid_cells(g), acells = anchor_cells(g);
    b += 3 * align_up(cells * 4) + align_up(4) + align_up(size_t(g.n_groups + 1) * 4);
    b += align_up(size_t(g.n_groups + 1) * 4) + 3 * align_up(cells * 4) + align_up(max_units(g, g.split) * sizeof(uint4));
    b += align_up(max_partials(g, g.split) * size_t(g.tw) * g.th * sizeof(float2));
    if (own_degrid_units(g))
        b += align_up(size_t(g.n_groups + 1) * 4) + 3 * align_up(cells * 4) +
             align_up(max_units(g, g.dsplit) * sizeof(uint4));
    b += 3 * align_up(acells * 4) + align_up(4);
    b += align_up(sizeof(unsigned long long)) + align_up(kStatusWords * sizeof(unsigned int));
    b += align_up(np * sizeof(float2));
    if (g.dense || g.ddense) b += align_up(np * sizeof(int4));  // pair records (tcv_dense.cu)
    b += align_up(cb);
    return b;
}

// Geometry of a variable-width plan: the widest plane sets the tile reach; whole planes are
// grouped in order until a group's slice of the table passes group_mib (complex64).
PlanGeom make_geom_var(int64_t n, const int32_t* s_size, const int32_t* c_off0, int n_planes, int g_size,
                       int64_t c_len, const tcv_tuning* t, std::vector<int32_t>& plane_grp)
{
    int s_max = 1;
    for (int k = 0; k < n_planes; ++k) s_max = std::max(s_max, int(s_size[k]));
    PlanGeom g = make_geom(n, s_max / 2, &g_size, 1, c_len, t, false);
    g.var = true;
    g.n_planes = n_planes;
    plane_grp.assign(size_t(n_planes), 0);
    const int64_t budget = g.group_mib > 0 ? (int64_t(g.group_mib) << 20) : INT64_MAX;
    int grp = 0;
    int64_t used = 0;
    for (int k = 0; k < n_planes; ++k) {
        const int64_t end = k + 1 < n_planes ? c_off0[k + 1] : c_len;
        const int64_t bytes = (end - c_off0[k]) * 8;
        if (used > 0 && used + bytes > budget) {
            ++grp;
            used = 0;
        }
        used += bytes;
        plane_grp[size_t(k)] = grp;
    }
    g.n_groups = grp + 1;
    g.kid_group = 0;
    g.group_bits = bits_for(uint64_t(g.n_groups - 1));
    g.tile_bits = bits_for(uint64_t(g.n_groups) * uint64_t(g.ntiles) - 1);
    g.key_bits = g.tile_bits + 1;
    g.key64 = g.key_bits > 32;
    return g;
}

tcv_status plan_bin(tcv_plan* p, const int32_t* d_iu, const int32_t* d_iv, const int32_t* d_coff, cudaStream_t st)
{
    if (!p) return TCV_ERR_ARG;
    if (p->g.n > 0 && (!d_iu || !d_iv || !d_coff)) return TCV_ERR_ARG;
    p->iu = d_iu;
    p->iv = d_iv;
    p->coff = d_coff;
    tcv_status s = p->g.key64 ? build<uint64_t>(p, d_iu, d_iv, d_coff, st) : build<uint32_t>(p, d_iu, d_iv, d_coff, st);
    if (s == TCV_OK && p->grec) s = gather_pair_records(p, st);
    p->binned = s == TCV_OK;
    return s;
}

// Fill *p (a caller-owned object) with a one-job plan built in d_work.
tcv_status plan_init(tcv_plan* p, const int32_t* d_iu, const int32_t* d_iv, const int32_t* d_coff, int64_t n,
                     int support, int g_size, int64_t c_len, void* d_work, size_t work_bytes, cudaStream_t st,
                     const tcv_tuning* t)
{
    if (!p || n < 0 || support < 0 || g_size < 1 || c_len < 1 || !valid_tuning(t)) return TCV_ERR_ARG;
    if (n > 0 && (!d_iu || !d_iv || !d_coff)) return TCV_ERR_ARG;
    if (!d_work) return TCV_ERR_ARG;
    *p = tcv_plan{};
    p->g = make_geom(n, support, &g_size, 1, c_len, t, true);
    if (!geom_supported(p->g)) return TCV_ERR_UNSUPPORTED;
    const tcv_status s = plan_create(p, d_work, work_bytes, st);
    if (s != TCV_OK) return s;
    return plan_bin(p, d_iu, d_iv, d_coff, st);
}

// Fill *p with a variable-width one-job plan (per-sample widths from the w-planes) built in d_work.
tcv_status plan_init_var(tcv_plan* p, const int32_t* d_iu, const int32_t* d_iv, const int32_t* d_coff,
                         const int32_t* d_wplane, int64_t n, const int32_t* s_size, const int32_t* c_off0,
                         int n_planes, int g_size, int64_t c_len, void* d_work, size_t work_bytes, cudaStream_t st,
                         const tcv_tuning* t)
{
    if (!p || n < 0 || g_size < 1 || c_len < 1 || n_planes < 1 || !s_size || !c_off0 || !valid_tuning(t))
        return TCV_ERR_ARG;
    if (n > 0 && (!d_iu || !d_iv || !d_coff || !d_wplane)) return TCV_ERR_ARG;
    for (int k = 0; k < n_planes; ++k)
        if (s_size[k] < 1 || s_size[k] % 2 == 0 || s_size[k] > 4095 || c_off0[k] < 0 || c_off0[k] > c_len)
            return TCV_ERR_ARG;
    if (!d_work) return TCV_ERR_ARG;
    *p = tcv_plan{};
    p->g = make_geom_var(n, s_size, c_off0, n_planes, g_size, c_len, t, p->host_plane_grp);
    if (!geom_supported(p->g)) return TCV_ERR_UNSUPPORTED;
    p->host_plane_s.assign(s_size, s_size + n_planes);
    p->wplane = d_wplane;
    const tcv_status s = plan_create(p, d_work, work_bytes, st);
    if (s != TCV_OK) return s;
    return plan_bin(p, d_iu, d_iv, d_coff, st);
}

}  // namespace tcv

using namespace tcv;

namespace {

// checks shared by the batch entry points; fills the per-job grid sides and the sample total
tcv_status batch_args(const tcv_job* jobs, int n_jobs, int support, int64_t c_len, const tcv_tuning* t,
                      std::vector<int>& sides, int64_t& n_total)
{
    if (!jobs || n_jobs < 1 || support < 0 || c_len < 1 || !valid_tuning(t)) return TCV_ERR_ARG;
    sides.resize(size_t(n_jobs));
    n_total = 0;
    for (int j = 0; j < n_jobs; ++j) {
        if (jobs[j].n < 0 || jobs[j].g_size < 1 || !jobs[j].d_grid) return TCV_ERR_ARG;
        sides[size_t(j)] = jobs[j].g_size;
        n_total += jobs[j].n;
    }
    return TCV_OK;
}

}  // namespace

extern "C" {

size_t tcv_plan_workspace_bytes(int64_t n, int support, int g_size, int64_t c_len)
{
    if (n < 0 || support < 0 || g_size < 1 || c_len < 1) return 0;
    PlanGeom g = make_geom(n, support, &g_size, 1, c_len, nullptr, true);
    return plan_bytes(g, nullptr);
}

size_t tcv_batch_workspace_bytes(const tcv_job* jobs, int n_jobs, int support, int64_t c_len, const tcv_tuning* tuning)
{
    std::vector<int> sides;
    int64_t n = 0;
    if (batch_args(jobs, n_jobs, support, c_len, tuning, sides, n) != TCV_OK) return 0;
    PlanGeom g = make_geom(n, support, sides.data(), n_jobs, c_len, tuning, false);
    return plan_bytes(g, nullptr);
}

tcv_status tcv_batch_plan_create(tcv_plan** plan_out, const tcv_job* jobs, int n_jobs, int support, int64_t c_len,
                                 const tcv_tuning* tuning, void* d_work, size_t work_bytes, void* stream)
{
    if (!plan_out || !d_work) return TCV_ERR_ARG;
    std::vector<int> sides;
    int64_t n = 0;
    tcv_status s = batch_args(jobs, n_jobs, support, c_len, tuning, sides, n);
    if (s != TCV_OK) return s;
    tcv_plan* p = new (std::nothrow) tcv_plan{};
    if (!p) return TCV_ERR_OOM;
    p->g = make_geom(n, support, sides.data(), n_jobs, c_len, tuning, false);
    if (!geom_supported(p->g)) {
        delete p;
        return TCV_ERR_UNSUPPORTED;
    }
    p->batch = true;
    p->host_jobs.resize(size_t(n_jobs));
    p->host_job_start.resize(size_t(n_jobs) + 1);
    uint32_t tile_base = 0, first = 0;
    for (int j = 0; j < n_jobs; ++j) {
        const int ntx = (jobs[j].g_size + p->g.tw - 1) / p->g.tw, nty = (jobs[j].g_size + p->g.th - 1) / p->g.th;
        p->host_jobs[size_t(j)] = JobDesc{reinterpret_cast<float2*>(jobs[j].d_grid), jobs[j].g_size, ntx, tile_base,
                                          uint32_t(ntx) * uint32_t(nty)};
        p->host_job_start[size_t(j)] = first;
        tile_base += uint32_t(ntx) * uint32_t(nty);
        first += uint32_t(jobs[j].n);
    }
    p->host_job_start[size_t(n_jobs)] = first;
    s = plan_create(p, d_work, work_bytes, static_cast<cudaStream_t>(stream));
    if (s != TCV_OK) {
        delete p;
        return s;
    }
    *plan_out = p;
    return TCV_OK;
}

size_t tcv_plan_workspace_bytes_var(int64_t n, const int32_t* s_size, const int32_t* c_off0, int n_planes,
                                    int g_size, int64_t c_len, const tcv_tuning* tuning)
{
    if (n < 0 || !s_size || !c_off0 || n_planes < 1 || g_size < 1 || c_len < 1 || !valid_tuning(tuning)) return 0;
    std::vector<int32_t> grp;
    PlanGeom g = make_geom_var(n, s_size, c_off0, n_planes, g_size, c_len, tuning, grp);
    return plan_bytes(g, nullptr);
}

tcv_status tcv_plan_build_var(tcv_plan** plan_out, const int32_t* d_iu, const int32_t* d_iv, const int32_t* d_coff,
                              const int32_t* d_wplane, int64_t n, const int32_t* s_size, const int32_t* c_off0,
                              int n_planes, int g_size, int64_t c_len, const tcv_tuning* tuning, void* d_work,
                              size_t work_bytes, void* stream)
{
    if (!plan_out) return TCV_ERR_ARG;
    tcv_plan* p = new (std::nothrow) tcv_plan{};
    if (!p) return TCV_ERR_OOM;
    const tcv_status s = plan_init_var(p, d_iu, d_iv, d_coff, d_wplane, n, s_size, c_off0, n_planes, g_size, c_len,
                                       d_work, work_bytes, static_cast<cudaStream_t>(stream), tuning);
    if (s != TCV_OK) {
        delete p;
        return s;
    }
    *plan_out = p;
    return TCV_OK;
}

tcv_status tcv_plan_bin(tcv_plan* plan, const int32_t* d_iu, const int32_t* d_iv, const int32_t* d_coff, void* stream)
{
    return plan_bin(plan, d_iu, d_iv, d_coff, static_cast<cudaStream_t>(stream));
}

tcv_status tcv_plan_tuning(const tcv_plan* plan, tcv_tuning* tuning_out)
{
    if (!plan || !tuning_out) return TCV_ERR_ARG;
    tuning_out->tile_rows = plan->g.rows;
    tuning_out->group_mib = plan->g.group_mib;
    tuning_out->split = plan->g.split;
    tuning_out->degrid_split = plan->g.dsplit;
    tuning_out->kernel = (plan->g.dense ? 1 : 0) | (plan->g.ddense ? 2 : 0);
    return TCV_OK;
}

size_t tcv_plan_workspace_bytes_tuned(int64_t n, int support, int g_size, int64_t c_len, const tcv_tuning* tuning)
{
    if (n < 0 || support < 0 || g_size < 1 || c_len < 1 || !valid_tuning(tuning)) return 0;
    PlanGeom g = make_geom(n, support, &g_size, 1, c_len, tuning, true);
    return plan_bytes(g, nullptr);
}

tcv_status tcv_plan_build(tcv_plan** plan_out, const int32_t* d_iu, const int32_t* d_iv,
                          const int32_t* d_coff, int64_t n, int support, int g_size,
                          int64_t c_len, void* d_work, size_t work_bytes, void* stream)
{
    return tcv_plan_build_tuned(plan_out, d_iu, d_iv, d_coff, n, support, g_size, c_len, nullptr, d_work,
                                work_bytes, stream);
}

tcv_status tcv_plan_build_tuned(tcv_plan** plan_out, const int32_t* d_iu, const int32_t* d_iv,
                                const int32_t* d_coff, int64_t n, int support, int g_size, int64_t c_len,
                                const tcv_tuning* tuning, void* d_work, size_t work_bytes, void* stream)
{
    if (!plan_out) return TCV_ERR_ARG;
    tcv_plan* p = new (std::nothrow) tcv_plan{};
    if (!p) return TCV_ERR_OOM;
    const tcv_status s = plan_init(p, d_iu, d_iv, d_coff, n, support, g_size, c_len, d_work, work_bytes,
                                   static_cast<cudaStream_t>(stream), tuning);
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
    if (n_tiles) *n_tiles = int(plan->g.ntiles * plan->g.n_groups);
    return TCV_OK;
}

void tcv_plan_destroy(tcv_plan* plan) { delete plan; }

tcv_status tcv_plan_grid(const tcv_plan* plan, const float* d_data, const void* d_c, int c_type,
                         float c_scale, float* d_grid, void* stream)
{
    if (!plan || !d_c || (plan->g.n > 0 && !d_data)) return TCV_ERR_ARG;
    if (plan->batch ? d_grid != nullptr : d_grid == nullptr) return TCV_ERR_ARG;
    if (tcv_ctype_bytes(c_type) == 0) return TCV_ERR_ARG;
    if (!plan->binned) return TCV_ERR_STATE;
    const bool plain_tiles = !plan->batch && !plan->g.var && plan->g.rows == 16;  // what the other families need
    if (c_type & TCV_C_PADDED) {
        if (!plain_tiles) return TCV_ERR_UNSUPPORTED;
        return launch_grid_pipe(plan, reinterpret_cast<const float2*>(d_data), d_c, c_type & 0xff, c_scale,
                                reinterpret_cast<float2*>(d_grid), static_cast<cudaStream_t>(stream));
    }
    if (c_type & TCV_C_PAIRED) {
        if (!plain_tiles) return TCV_ERR_UNSUPPORTED;
        return launch_grid_pair(plan, reinterpret_cast<const float2*>(d_data), d_c, c_type & 0xff, c_scale,
                                reinterpret_cast<float2*>(d_grid), static_cast<cudaStream_t>(stream));
    }
    return launch_grid(plan, reinterpret_cast<const float2*>(d_data), d_c, c_type, c_scale,
                       reinterpret_cast<float2*>(d_grid), static_cast<cudaStream_t>(stream));
}

tcv_status tcv_plan_degrid(const tcv_plan* plan, const float* d_grid, const void* d_c, int c_type,
                           float c_scale, float* d_data, void* stream)
{
    if (!plan || !d_c || (plan->g.n > 0 && !d_data)) return TCV_ERR_ARG;
    if (plan->batch ? d_grid != nullptr : d_grid == nullptr) return TCV_ERR_ARG;
    if (tcv_ctype_bytes(c_type) == 0) return TCV_ERR_ARG;
    if (!plan->binned) return TCV_ERR_STATE;
    const bool plain_tiles = !plan->batch && !plan->g.var && plan->g.rows == 16;
    if (c_type & TCV_C_PADDED) {
        if (!plain_tiles) return TCV_ERR_UNSUPPORTED;
        if (plan->g.n == 0) return TCV_OK;
        return launch_degrid_pipe(plan, reinterpret_cast<const float2*>(d_grid), d_c, c_type & 0xff, c_scale,
                                  reinterpret_cast<float2*>(d_data), static_cast<cudaStream_t>(stream));
    }
    if (c_type & TCV_C_PAIRED) {
        if (!plain_tiles) return TCV_ERR_UNSUPPORTED;
        if (plan->g.n == 0) return TCV_OK;
        return launch_degrid_pair(plan, reinterpret_cast<const float2*>(d_grid), d_c, c_type & 0xff, c_scale,
                                  reinterpret_cast<float2*>(d_data), static_cast<cudaStream_t>(stream));
    }
    if (plan->degrid_variant == TCV_DEGRID_TILES || plan->batch || plan->g.var) {
        if (plan->g.n == 0) return TCV_OK;
        return launch_degrid_tiles(plan, reinterpret_cast<const float2*>(d_grid), d_c, c_type, c_scale,
                                   reinterpret_cast<float2*>(d_data), static_cast<cudaStream_t>(stream));
    }
    TCV_CHECK(plan_anchors_ready(plan, static_cast<cudaStream_t>(stream)));
    return launch_degrid(plan, reinterpret_cast<const float2*>(d_grid), d_c, c_type, c_scale,
                         reinterpret_cast<float2*>(d_data), static_cast<cudaStream_t>(stream));
}

tcv_status tcv_plan_set_degrid_variant(tcv_plan* plan, int variant)
{
    if (!plan || (variant != TCV_DEGRID_TILES && variant != TCV_DEGRID_ANCHOR)) return TCV_ERR_ARG;
    if (variant == TCV_DEGRID_ANCHOR && !plan->g.anchors) return TCV_ERR_UNSUPPORTED;
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
