// tcv_dense.cu -- sample-parallel tile kernels for variable-width plans with small footprints
// (the current/tConvolveMPI path: kernels 7..121 wide, most under 20).
//
// The output-stationary tile kernels (tcv_device.cuh) give every lane a fixed grid column and
// make all eight warps test every sample of the tile; with a 9-wide footprint a warp then works
// with 9 of its 32 lanes and most warps only test and skip.  Here each sample is handled by one
// warp per region of the tile it meets, whose lanes cover the intersection densely: a w-wide
// rectangle is walked floor(32 / w) rows of w lanes per step (w <= 32) or in 32-column strips.
// The staging thread of each sample prepares its rectangle once (tile coordinates, table index
// of its first element, rows per step), so a warp only walks it.
//
// Gridding: a work item is one 32-column half of a unit's 64 x 32 tile; groups of four warps
// take items from a counter as they finish their last (no fixed share per CTA, so no CTA is left
// with a long tail), and each warp adds into a private copy of the half in shared memory (8 KB
// each, no two warps write one copy: no atomics).  The warps of a group work independently: each
// takes every fourth group of 32 samples of the unit, stages them as jobs for the half (one per
// sample that meets the half) and adds them into its copy, keeping the next job's first table
// loads in flight while it adds the current one (a two-stage software pipeline).  At the end of
// the item the four warps meet (a named barrier) and add their copies in warp order into the
// grid, or into the unit's partial tile for a split cell (fold_kernel then adds those in unit
// order, as for the tile kernels).
// Degridding: the grid tile is staged in shared memory once per unit; a warp takes four samples
// at a time and reduces their products across the warp together (one transposing reduction) into
// the samples' slots for the tile (slot_reduce_kernel adds the slots in tile order).
//
// Every sum is taken in a fixed order, so results are deterministic; they group the reference's
// per-point sums differently (by warp), which moves them by FP32 rounding only.  Tiles are the
// plans' 64 x 32 tiles (tile rows 8), so the plans are those of the tile kernels.
#include "tcv_internal.cuh"

namespace tcv {
namespace {

constexpr int kDTW = kTileW;              // 64 columns
constexpr int kDTH = 32;                  // rows (tile_height(8))
constexpr int kDPts = kDTW * kDTH;        // 2048 points
constexpr int kGWarps = 8;                // gridding: warps per CTA, four per 32-column half
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

// Gridding lane table: for a rectangle width w (1 .. 32) and a lane, the lane's row in the step
// (lane / w), its column (lane % w) and the rows per step (floor(32 / w)), as
// row | column << 5 | rows << 10.
__device__ __forceinline__ void build_grid_lut(unsigned short (&gl)[33][32], int tid, int nthreads)
{
    for (int i = tid; i < 33 * 32; i += nthreads) {
        const int w = i / 32 < 1 ? 1 : i / 32, lane = i % 32;
        gl[i / 32][lane] = (unsigned short)((lane / w) | (lane % w) << 5 | (32 / w) << 10);
    }
}

// A kernel's position in its work: unit list position, first sample of the chunk in that unit, the
// unit's sample range, tile record and partial tile, and the chunk's sample count (0: no more
// work).  Chunks are kChunk samples.
struct DChunk {
    u32 it, base, cnt, start, ti, pslot;
    int m;
};
template <int kChunk>
__device__ __forceinline__ void dchunk_load(DChunk& c, u32 it, u32 i1, const uint4* __restrict__ units,
                                            const GridArgs& a)
{
    c.it = it;
    c.base = 0;
    c.m = 0;
    if (it < i1) {
        const uint4 u = units[it];
        c.start = u.y;
        c.cnt = u.z;
        c.pslot = u.w;
        c.ti = a.tinfo[u.x - u32(a.group) * u32(a.ntiles)];
        c.m = int(c.cnt < u32(kChunk) ? c.cnt : u32(kChunk));
    }
}

// the named barrier of one tile half's four gridding warps (barrier 0 is the CTA's)
__device__ __forceinline__ void half_barrier(int half)
{
    if (half == 0)
        asm volatile("bar.sync 1, 128;" ::: "memory");
    else
        asm volatile("bar.sync 2, 128;" ::: "memory");
}

// Gridding.  The CTA's two groups of kGWarps / 2 warps each take one (unit, 32-column tile half)
// work item at a time, handed out by a counter, and their warps hold private copies of a half.
// The warps work independently: warp j of a group takes samples 32 j + 128 i + [0, 32) of the
// unit (i = 0, 1, ...), stages them as jobs for the item's half (one per sample that meets it: the
// table index of the first element of the sample's rectangle in the half, and first point |
// (width - 1) << 10 | (height - 1) << 15 | table row stride << 20, and the scaled data value),
// packed in sample order by ballot into its own 32-entry list, and adds them into its copy,
// keeping the next job's first table loads in flight while it adds the current one.  Only the
// four warps of a group meet, at the end of each item (a named barrier per group), to add their
// copies in warp order into the grid or the unit's partial tile.
template <class Tab>
__global__ void __launch_bounds__(kGThreads, 3)
dense_grid_kernel(const float2* __restrict__ data, const u32* __restrict__ order,
                  const typename Tab::elem* __restrict__ ctab,
                  const int4* __restrict__ grec, const uint4* __restrict__ units,
                  const u32* __restrict__ group_ustart, GridArgs a)
{
    using E = typename Tab::elem;
    constexpr int kHalf = kDTW / 2;            // 32 columns
    constexpr int kHPts = kHalf * kDTH;        // 1024 points per half
    constexpr int kPerHalf = kGWarps / 2;      // warps per half
    constexpr int U = 3;                       // table loads of a job issued together
    static_assert(kPerHalf * 32 == 128, "a half's warps meet at a 128-thread named barrier");
    extern __shared__ __align__(16) float2 dsm[];
    float2* acc_all = dsm;                                                    // [kGWarps][kHPts]
    int4* jobs_all = reinterpret_cast<int4*>(dsm + kGWarps * kHPts);         // [kGWarps][32]
    __shared__ unsigned short gl[33][32];
    __shared__ u32 sm_item[2][2];  // per warp group: its current and next work item
    __shared__ u32 sm_range[2];    // the group's first unit and its number of work items
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int half = warp / kPerHalf, sub = warp % kPerHalf;  // warp group (copies, barrier), warp in it
    // Work items are (unit, tile half) pairs, 2 i and 2 i + 1 the halves of the group's unit i,
    // handed out to the warp groups in turn by a counter (a.sched[0]) as each group finishes its
    // last; the group that finds the list exhausted last (a.sched[1] counts them) sets both counters
    // to zero again for the next launch.  Which group takes an item does not change any sum.
    // (the unit range is read back from shared memory where it is used, so that it holds no
    // registers through the job loop)
    if (threadIdx.x == 0) {
        const u32 i0 = group_ustart[a.group];
        sm_range[0] = i0;
        sm_range[1] = 2u * (group_ustart[a.group + 1] - i0);
    }
    auto fetch = [&](int slot) {  // the group's first lane only
        const u32 v = atomicAdd(a.sched, 1u);
        if (v >= sm_range[1] && atomicAdd(a.sched + 1, 1u) == 2u * gridDim.x - 1u) {
            atomicExch(a.sched, 0u);
            atomicExch(a.sched + 1, 0u);
        }
        sm_item[half][slot] = v;
    };
    build_grid_lut(gl, threadIdx.x, kGThreads);
    float2* acc = acc_all + warp * kHPts;
    int4* jl = jobs_all + warp * 32;
    for (int i = lane; i < kHPts; i += 32) acc[i] = make_float2(0.f, 0.f);
    __syncthreads();  // the lane table and the unit range are set
    if (sub == 0 && lane == 0) fetch(0);
    half_barrier(half);  // the group's first item is in sm_item

    struct Job {
        const E* tp;   // the lane's first table entry
        int ap;        // the lane's first point in the copy
        int rem, h;    // rows of the lane (from its first, in steps of kk) and of the rectangle
        int kk, kks;   // rows per step, and table entries per step
        float2 dv;
    };
    auto setup = [&](int i, Job& J) {
        const int4 jb = jl[i];
        const u32 meta = u32(jb.y);
        const int wc = int((meta >> 10) & 31u) + 1, s = int(meta >> 20);
        const u32 lu = gl[wc][lane];
        const int q = int(lu & 31u), r = int((lu >> 5) & 31u);
        J.h = int((meta >> 15) & 31u) + 1;
        J.kk = int(lu >> 10);
        J.rem = q < J.kk ? J.h - q : 0;
        J.tp = ctab + (jb.x + q * s + r);
        J.ap = int(meta & 1023u) + q * kHalf + r;
        J.kks = J.kk * s;
        J.dv = make_float2(__int_as_float(jb.z), __int_as_float(jb.w));
    };
    auto load = [&](const Job& J, int e0, float2 (&cv)[U]) {
#pragma unroll
        for (int e = 0; e < U; ++e) {
            const int ro = (e0 + e) * J.kk;
            cv[e] = ro < J.rem ? Tab::load(J.tp + (e0 + e) * J.kks) : make_float2(0.f, 0.f);
        }
    };
    auto apply = [&](const Job& J, int e0, const float2 (&cv)[U]) {
        // the steps' points are distinct: all their reads first, then the adds and writes
        float2 t[U];
#pragma unroll
        for (int e = 0; e < U; ++e) {
            const int ro = (e0 + e) * J.kk;
            if (ro < J.rem) t[e] = acc[J.ap + ro * kHalf];
        }
#pragma unroll
        for (int e = 0; e < U; ++e) {
            const int ro = (e0 + e) * J.kk;
            if (ro < J.rem) {
                cmac<Tab::kReal>(t[e], J.dv, cv[e]);
                acc[J.ap + ro * kHalf] = t[e];
            }
        }
    };

    for (int par = 0;; par ^= 1) {
        const u32 item = sm_item[half][par];  // written before the last barrier of the group
        if (item >= sm_range[1]) break;       // the group's four warps read the same item
        const int hx0 = int(item & 1u) * kHalf;
        const uint4 u = units[sm_range[0] + (item >> 1)];
        const u32 start = u.y, cnt = u.z, pslot = u.w;
        const u32 ti = a.tinfo[u.x - u32(a.group) * u32(a.ntiles)];
        const int tx0 = rec_tx(ti) * kDTW, ty0 = rec_ty(ti) * kDTH;
        for (u32 base = u32(sub) * 32u; base < cnt; base += u32(kPerHalf) * 32u) {
            bool has = false;
            int4 jb = make_int4(0, 0, 0, 0);
            if (base + u32(lane) < cnt) {
                const int4 pr = grec[start + base + u32(lane)];  // (first column, first row, cOffset, width)
                const float2 d = data[order[start + base + u32(lane)]];  // in flight during the clip below
                const int fx = pr.x, fy = pr.y, sk = pr.w;
                const Rect R = clip(fx, fy, sk, tx0, ty0);
                const int tc = fx + R.c0 - tx0, h = R.r1 - R.r0;
                const int lo = max(tc, hx0), hi = min(fx + R.c1 - tx0, hx0 + kHalf);
                has = h > 0 && lo < hi;
                if (has) {
                    jb.x = pr.z + R.r0 * sk + R.c0 + (lo - tc);
                    jb.y = int(u32((fy + R.r0 - ty0) * kHalf + lo - hx0) | u32(hi - lo - 1) << 10 |
                               u32(h - 1) << 15 | u32(sk) << 20);
                    jb.z = __float_as_int(d.x * a.c_scale);
                    jb.w = __float_as_int(d.y * a.c_scale);
                }
            }
            const u32 b = __ballot_sync(0xffffffffu, has);
            if (has) jl[__popc(b & ((1u << lane) - 1u))] = jb;
            __syncwarp();
            const int n = __popc(b);
            if (n > 0) {
                Job cur;
                float2 cv[U];
                setup(0, cur);
                load(cur, 0, cv);
                for (int i = 0;; ++i) {
                    const bool more = i + 1 < n;
                    Job nx;
                    float2 nv[U];
                    if (more) {  // in flight during the updates below
                        setup(i + 1, nx);
                        load(nx, 0, nv);
                    }
                    apply(cur, 0, cv);
                    for (int e0 = U; e0 * cur.kk < cur.h; e0 += U) {  // tall rectangles (warp-uniform)
                        float2 t[U];
                        load(cur, e0, t);
                        apply(cur, e0, t);
                    }
                    __syncwarp();  // this job's updates land before another lane reads them for the next
                    if (!more) break;
                    cur = nx;
#pragma unroll
                    for (int e = 0; e < U; ++e) cv[e] = nv[e];
                }
            }
            __syncwarp();  // the list is read before the next samples are packed into it
        }
        // the unit is done in this half: its copies in warp order into the grid or the partial tile
        if (sub == 0 && lane == 0) fetch(par ^ 1);  // read by the group after the barrier below
        half_barrier(half);
        const JobDesc& jd = a.jobs[rec_job(ti)];
        const int gs = jd.g_size;
        float2* grid = a.grid ? a.grid : jd.grid;
        for (int p = int(threadIdx.x) & 127; p < kHPts; p += 128) {
            float2* c = acc_all + half * kPerHalf * kHPts + p;
            float2 v = c[0];
#pragma unroll
            for (int w = 1; w < kPerHalf; ++w) {
                const float2 o = c[w * kHPts];
                v.x += o.x;
                v.y += o.y;
            }
#pragma unroll
            for (int w = 0; w < kPerHalf; ++w) c[w * kHPts] = make_float2(0.f, 0.f);
            const int px = hx0 + p % kHalf, py = p / kHalf;  // point in the tile
            if (pslot != kDirect) {
                a.partial[(unsigned long long)(pslot) * kDPts + py * kDTW + px] = v;
            } else {
                const int gx = tx0 + px, gy = ty0 + py;
                if (gx < gs && gy < gs) {
                    float2* gp = grid + ((unsigned long long)(gy) * gs + gx);
                    float2 o = *gp;
                    o.x += v.x;
                    o.y += v.y;
                    *gp = o;
                }
            }
        }
        half_barrier(half);  // the copies are zero again before the next unit's adds
    }
}

// Degridding.  The unit's grid tile is staged in shared memory; a chunk of kDThreads samples is
// staged as rectangles (prepare) with their slot indices, the next chunk while this one is read
// (two buffers, one barrier per chunk).  Warp w takes samples 4g .. 4g + 3 for g = w, w + 8, ...:
// each lane's partial products of the four, then one transposing warp reduction for all four
// (6 complex shuffles instead of 20), which sums each sample over the lanes in the same tree as a
// plain butterfly.
template <class Tab>
__global__ void __launch_bounds__(kDThreads)
dense_degrid_kernel(const typename Tab::elem* __restrict__ ctab, const int4* __restrict__ grec,
                    const u32* __restrict__ order, const uint4* __restrict__ units,
                    const u32* __restrict__ group_ustart, float2* __restrict__ slots, int max_tiles, GridArgs a)
{
    __shared__ float2 gt[kDPts];           // the grid tile
    __shared__ DenseRec rec[2][kDThreads];
    __shared__ unsigned long long rslot[2][kDThreads];  // slot index of (sample, this tile)
    __shared__ DenseLut L;
    // Work units are handed out by a counter (a.sched[0]) as CTAs finish their last, one unit
    // ahead: sm_unit[q] is the CTA's next unit, drawn by thread 0 when the unit before it
    // started (the units' work differs by the footprint widths, up to 121² against 7² updates per
    // sample, which a fixed share per CTA left as a tail).  The CTA that draws past the end last
    // (a.sched[1] counts them) sets both counters to zero again.  Which CTA takes a unit changes
    // no sum: every unit writes its own samples' slots.
    __shared__ u32 sm_unit[3];  // two unit slots, and the group's first unit
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const u32 i1 = group_ustart[a.group + 1];
    auto fetch = [&]() -> u32 {  // thread 0 only
        const u32 v = sm_unit[2] + atomicAdd(a.sched, 1u);
        if (v >= i1 && atomicAdd(a.sched + 1, 1u) == gridDim.x - 1u) {
            atomicExch(a.sched, 0u);
            atomicExch(a.sched + 1, 0u);
        }
        return v;
    };
    if (threadIdx.x == 0) {
        sm_unit[2] = group_ustart[a.group];
        const u32 v = fetch();
        sm_unit[0] = v;
        sm_unit[1] = v < i1 ? fetch() : v;  // no draw after the first past the end
    }
    build_lut(L, threadIdx.x, kDThreads);
    __syncthreads();  // the lane table is built (the staging reads it); the first units are drawn
    int q = 1;        // slot of the next unit (uniform)
    auto next_chunk = [&](DChunk& c) {
        if (c.base + u32(kDThreads) < c.cnt) {
            c.base += u32(kDThreads);
            const u32 left = c.cnt - c.base;
            c.m = int(left < u32(kDThreads) ? left : u32(kDThreads));
        } else {
            // the slot was written before the last barrier; the other slot was last read before it
            const u32 v = sm_unit[q];
            if (threadIdx.x == 0 && v < i1) sm_unit[q ^ 1] = fetch();
            q ^= 1;
            dchunk_load<kDThreads>(c, v, i1, units, a);
        }
    };
    auto stage = [&](const DChunk& c, int buf) {
        if (int(threadIdx.x) < c.m) {
            const u32 pos = c.start + c.base + threadIdx.x;
            const u32 k = order[pos];
            const int4 pr = grec[pos];  // (first column, first row, cOffset, width)
            const int fx = pr.x, fy = pr.y, sk = pr.w;
            const int tx = rec_tx(c.ti), ty = rec_ty(c.ti);
            rec[buf][threadIdx.x] = prepare(pr.z, sk, fx, fy, tx * kDTW, ty * kDTH, L);
            const int sx0 = fx / kDTW, sx1 = (fx + sk - 1) / kDTW, sy0 = fy / kDTH;
            rslot[buf][threadIdx.x] = (unsigned long long)(k) * max_tiles + (ty - sy0) * (sx1 - sx0 + 1) + (tx - sx0);
        }
    };
    auto load_tile = [&](u32 ti) {
        const JobDesc& jd = a.jobs[rec_job(ti)];
        const int gs = jd.g_size;
        const float2* grid = a.grid ? a.grid : jd.grid;
        const int tx0 = rec_tx(ti) * kDTW, ty0 = rec_ty(ti) * kDTH;
        for (int p = threadIdx.x; p < kDPts; p += kDThreads) {
            const int gx = tx0 + (p % kDTW), gy = ty0 + (p / kDTW);
            gt[p] = (gx < gs && gy < gs) ? grid[(unsigned long long)(gy) * gs + gx] : make_float2(0.f, 0.f);
        }
    };
    // the partial dot product of this lane with sample j's rectangle
    auto partial = [&](int buf, int j) -> float2 {
        const DenseRec d = rec[buf][j];
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
                    cmac<Tab::kReal>(p1, gt[pbase + (row0 + kk) * kDTW], Tab::load(ctab + (cbase + (row0 + kk) * d.s)));
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
        return make_float2(p0.x + p1.x, p0.y + p1.y);
    };
    DChunk cur;
    dchunk_load<kDThreads>(cur, sm_unit[0], i1, units, a);
    stage(cur, 0);
    if (cur.m > 0) load_tile(cur.ti);
    __syncthreads();  // slot 0 is read before thread 0 can draw into it again
    int buf = 0;
    while (cur.m > 0) {
        DChunk nxt = cur;
        next_chunk(nxt);
        stage(nxt, buf ^ 1);  // the next chunk, while this one is read
        for (int g0 = warp * 4; g0 < cur.m; g0 += kDWarps * 4) {
            float2 v[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) v[e] = g0 + e < cur.m ? partial(buf, g0 + e) : make_float2(0.f, 0.f);  // warp-uniform
            // exchange over lane bit 4 (lanes keep samples 0,1 or 2,3) and bit 3 (one sample each):
            // lane holds sample (lane >> 3) & 3 summed over 4 lanes; butterflies over bits 2..0 finish
            const bool h16 = (lane & 16) != 0, h8 = (lane & 8) != 0;
            const float2 s0 = h16 ? v[0] : v[2], k0 = h16 ? v[2] : v[0];
            const float2 s1 = h16 ? v[1] : v[3], k1 = h16 ? v[3] : v[1];
            const float2 w0 = make_float2(k0.x + __shfl_xor_sync(0xffffffffu, s0.x, 16),
                                          k0.y + __shfl_xor_sync(0xffffffffu, s0.y, 16));
            const float2 w1 = make_float2(k1.x + __shfl_xor_sync(0xffffffffu, s1.x, 16),
                                          k1.y + __shfl_xor_sync(0xffffffffu, s1.y, 16));
            const float2 sd = h8 ? w0 : w1, kp = h8 ? w1 : w0;
            float2 y = make_float2(kp.x + __shfl_xor_sync(0xffffffffu, sd.x, 8),
                                   kp.y + __shfl_xor_sync(0xffffffffu, sd.y, 8));
#pragma unroll
            for (int o = 4; o; o >>= 1) {
                y.x += __shfl_xor_sync(0xffffffffu, y.x, o);
                y.y += __shfl_xor_sync(0xffffffffu, y.y, o);
            }
            const int js = g0 + (lane >> 3);
            if ((lane & 7) == 0 && js < cur.m) slots[rslot[buf][js]] = y;  // an empty overlap writes its empty slot
        }
        if (nxt.m > 0 && nxt.it != cur.it) {  // a new unit: its grid tile (block-uniform)
            __syncthreads();  // every warp is done with this tile
            load_tile(nxt.ti);
        }
        __syncthreads();  // the next chunk (and tile) is staged; this chunk's records are free
        cur = nxt;
        buf ^= 1;
    }
}

// The footprint of every sorted (sample, tile) pair, in pair order, so that the sample-parallel
// kernels stage a sample with one coalesced load instead of gathering its fields by sample index
// (ssz: per-sample widths of a variable-width plan; nullptr: every sample is s_all wide).
// Blocks stride over the work units, which cover every pair of every non-empty cell.
__global__ void pair_records_kernel(const uint4* __restrict__ units, const u32* __restrict__ group_ustart,
                                    int n_groups, const u32* __restrict__ order, const int* __restrict__ iu,
                                    const int* __restrict__ iv, const int* __restrict__ coff,
                                    const unsigned short* __restrict__ ssz, int s_all, int4* __restrict__ grec)
{
    const u32 nu = group_ustart[n_groups];
    for (u32 it = blockIdx.x; it < nu; it += gridDim.x) {
        const uint4 u = units[it];
        for (u32 r = threadIdx.x; r < u.z; r += blockDim.x) {
            const u32 pos = u.y + r, k = order[pos];
            const int sk = ssz ? int(ssz[k]) : s_all;  // the plane's width, or the plan's one width
            grec[pos] = make_int4(iu[k] - sk / 2, iv[k], coff[k], sk);
        }
    }
}

int sm_count()
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
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

constexpr size_t kGridSmem = size_t(kGWarps) * (kDPts / 2) * sizeof(float2) + size_t(kGWarps * 32) * sizeof(int4);

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
    a.sched = p->status + kSchedWord;
    return a;
}

}  // namespace

template <class Tab>
tcv_status launch_dense_grid(const tcv_plan* p, const float2* data, const void* c, float c_scale, float2* grid,
                             cudaStream_t st)
{
    const PlanGeom& g = p->g;
    if (g.n == 0) return TCV_OK;
    if (g.tw != kDTW || g.th != kDTH || g.s > 4095) return TCV_ERR_UNSUPPORTED;  // widths: 12 bits of a job
    const void* kernel = reinterpret_cast<const void*>(&dense_grid_kernel<Tab>);
    TCV_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kGridSmem)));
    const int ctas = resident(kernel, kGThreads, kGridSmem);
    if (!p->grec) return TCV_ERR_UNSUPPORTED;
    const typename Tab::elem* tab = static_cast<const typename Tab::elem*>(c);
    const unsigned int* order = p->vals[p->sel];
    const int4* grec = p->grec;
    for (int grp = 0; grp < g.n_groups; ++grp) {
        GridArgs a = dense_args(p, grp, c_scale, grid);
        void* args[] = {const_cast<float2**>(&data), const_cast<unsigned int**>(&order), &tab, &grec,
                        const_cast<uint4**>(&p->units), const_cast<uint32_t**>(&p->group_ustart), &a};
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
    if (g.tw != kDTW || g.th != kDTH) return TCV_ERR_UNSUPPORTED;
    const void* kernel = reinterpret_cast<const void*>(&dense_degrid_kernel<Tab>);
    if (!p->grec) return TCV_ERR_UNSUPPORTED;
    const int ctas = resident(kernel, kDThreads, 0);
    const typename Tab::elem* tab = static_cast<const typename Tab::elem*>(c);
    const unsigned int* order = p->vals[p->sel];
    const int4* grec = p->grec;
    int max_tiles = g.max_tiles;
    float2* gridp = const_cast<float2*>(grid);
    for (int grp = 0; grp < g.n_groups; ++grp) {
        GridArgs a = dense_args(p, grp, c_scale, gridp);
        void* args[] = {&tab, &grec, &order, const_cast<uint4**>(&p->d_units),
                        const_cast<uint32_t**>(&p->d_group_ustart), const_cast<float2**>(&p->slots), &max_tiles, &a};
        TCV_CUDA(cudaLaunchKernel(kernel, dim3(ctas), dim3(kDThreads), args, 0, st));
    }
    return slot_reduce(p, c_scale, out, st);
}

tcv_status gather_pair_records(const tcv_plan* p, cudaStream_t st)
{
    const PlanGeom& g = p->g;
    if (!p->grec || g.n == 0) return TCV_OK;
    pair_records_kernel<<<unsigned(8 * sm_count()), 256, 0, st>>>(p->units, p->group_ustart, g.n_groups, p->vals[p->sel],
                                                                  p->iu, p->iv, p->coff, g.var ? p->ssz : nullptr, g.s,
                                                                  p->grec);
    TCV_CUDA(cudaGetLastError());
    return TCV_OK;
}

template tcv_status launch_dense_grid<TabC64>(const tcv_plan*, const float2*, const void*, float, float2*, cudaStream_t);
template tcv_status launch_dense_grid<TabR32>(const tcv_plan*, const float2*, const void*, float, float2*, cudaStream_t);
template tcv_status launch_dense_grid<TabCBF16>(const tcv_plan*, const float2*, const void*, float, float2*, cudaStream_t);
template tcv_status launch_dense_grid<TabRBF16>(const tcv_plan*, const float2*, const void*, float, float2*, cudaStream_t);
template tcv_status launch_dense_grid<TabCF16>(const tcv_plan*, const float2*, const void*, float, float2*, cudaStream_t);
template tcv_status launch_dense_grid<TabRF16>(const tcv_plan*, const float2*, const void*, float, float2*, cudaStream_t);
template tcv_status launch_dense_degrid<TabC64>(const tcv_plan*, const float2*, const void*, float, float2*, cudaStream_t);
template tcv_status launch_dense_degrid<TabR32>(const tcv_plan*, const float2*, const void*, float, float2*, cudaStream_t);
template tcv_status launch_dense_degrid<TabCBF16>(const tcv_plan*, const float2*, const void*, float, float2*, cudaStream_t);
template tcv_status launch_dense_degrid<TabRBF16>(const tcv_plan*, const float2*, const void*, float, float2*, cudaStream_t);
template tcv_status launch_dense_degrid<TabCF16>(const tcv_plan*, const float2*, const void*, float, float2*, cudaStream_t);
template tcv_status launch_dense_degrid<TabRF16>(const tcv_plan*, const float2*, const void*, float, float2*, cudaStream_t);

}  // namespace tcv
