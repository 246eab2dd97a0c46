// tcv_device.cuh -- device code of the output-stationary tile kernels (gridding and its adjoint).
//
// Self-contained device code: compiled into libtconvolve for every table form with the footprint
// width sSize as a runtime value (kS = 0), and handed to NVRTC at plan time to build copies with
// sSize a compile-time constant (kS = sSize), where row offsets become load immediates and loop
// bounds constants.  Nothing here includes a host header, so both compilers accept it.
//
// Output-stationary tiles.  One CTA owns a tile of 64 x 4*kR grid points (kR = rows per warp, 8,
// 16 or 32: the tile shape an autotuner chooses between); each of its 8 warps owns a 32-column x
// kR-row block with one accumulator per point held in registers (lane = column).
// The CTA walks the tile's sample list (from the plan), staging sample records in shared memory;
// for each sample a warp whose block meets the footprint reads the table rows it needs (32
// consecutive entries per row: one coalesced load per row) and accumulates data * C into its
// registers.  When the list is done the tile is added into the grid with coalesced
// read-modify-writes.  Every grid point has exactly one owner thread: no atomics, and the result
// is the same on every run.  Gridding follows attic/tConvolveMPI/Benchmark.cc:125-155.
//
// Degridding (Benchmark.cc:158-195) is the adjoint on the same plan: a lane holds its kR grid
// points in registers; for each sample a warp whose block meets the footprint forms the partial
// dot product of its block with the table, reduces it with shuffles, and the CTA adds its 8 warp
// partials in warp order into the sample's slot for this tile; a final pass adds each sample's
// tile slots in tile order.
//
// A plan may hold several jobs (channels, Taylor terms) that share the table but have their own
// samples, grid and grid size.  Tiles of all jobs are numbered in one space; a 32-bit per-tile
// record gives the job and the tile's column and row, and the job table gives the job's grid.
#pragma once

namespace tcv {

using u32 = unsigned int;

constexpr int kTileW = 64;         // tile width: two warps of 32 columns
constexpr int kTileWarps = 8;      // four rows of two warps
constexpr int kTileThreads = kTileWarps * 32;
constexpr int kTileChunk = kTileThreads;  // samples staged per round
__host__ __device__ constexpr int tile_height(int rows_per_warp) { return rows_per_warp * (kTileWarps * 32 / kTileW); }

// One job of a plan: its grid (nullptr: the grid is passed at launch), side, tiles per row and
// first tile number.
struct JobDesc {
    float2* grid;
    int g_size, ntx;
    u32 tile_base, n_tiles;
};

struct GridArgs {
    int support, s, ntiles, group;  // ntiles: tiles of all jobs (cells per plane group)
    float c_scale;
    float2* grid;                   // grid of a one-job plan given at launch, else nullptr
    const JobDesc* __restrict__ jobs;
    const u32* __restrict__ tinfo;  // per tile: column | row << 11 | job << 22
    float2* partial;                // partial tiles of split cells (gridding), tile after tile
    const unsigned short* __restrict__ ssz;  // per-sample footprint width (variable-width plans)
    // two work-item counters of the plan, zero at every launch (the sample-parallel gridding
    // kernel hands out its work items with them and sets them to zero again when it finishes)
    u32* sched;
};

// A work unit: a cell's samples [first, first + count) of the sorted order, and the partial tile
// it writes when its cell is split among several units (kDirect: the unit owns the whole cell
// and adds its tile into the grid itself).
constexpr u32 kDirect = 0xffffffffu;

// per-tile record: tile column (11 bits), tile row (11 bits), job (10 bits)
__host__ __device__ constexpr u32 tile_record(u32 job, u32 tx, u32 ty) { return tx | (ty << 11) | (job << 22); }
__host__ __device__ constexpr int rec_tx(u32 r) { return int(r & 0x7ffu); }
__host__ __device__ constexpr int rec_ty(u32 r) { return int((r >> 11) & 0x7ffu); }
__host__ __device__ constexpr int rec_job(u32 r) { return int(r >> 22); }
constexpr int kMaxJobs = 1 << 10;
constexpr int kMaxTilesPerSide = 1 << 11;

// ------------------------------------------------------------------------------------------
// Table loaders.  Every storage form returns the entry as (re, im) floats; the real forms
// return im = 0 and tell the multiply-accumulate to skip the imaginary products, which gives
// exactly the same result as the complex form on a table whose imaginary parts are zero
// (fma(-d.im, 0, acc) == acc).
// ------------------------------------------------------------------------------------------
struct TabC64 {
    static constexpr int kMinBlocks = 3;  // CTAs per SM the register budget is sized for
    static constexpr bool kReal = false;
    using elem = float2;
    __device__ __forceinline__ static float2 load(const elem* p) { return __ldg(p); }
};
struct TabR32 {
    static constexpr int kMinBlocks = 4;
    static constexpr bool kReal = true;
    using elem = float;
    __device__ __forceinline__ static float2 load(const elem* p) { return make_float2(__ldg(p), 0.f); }
};
struct TabCBF16 {
    static constexpr int kMinBlocks = 3;
    static constexpr bool kReal = false;
    using elem = u32;  // (re, im) bfloat16 pair, re in the low half
    __device__ __forceinline__ static float2 load(const elem* p)
    {
        const u32 u = __ldg(p);
        return make_float2(__uint_as_float(u << 16), __uint_as_float(u & 0xffff0000u));
    }
};
struct TabRBF16 {
    static constexpr int kMinBlocks = 4;
    static constexpr bool kReal = true;
    using elem = unsigned short;
    __device__ __forceinline__ static float2 load(const elem* p)
    {
        const u32 u = __ldg(p);
        return make_float2(__uint_as_float(u << 16), 0.f);
    }
};

// acc += a * b (complex), FP32 fused multiply-adds issued as paired FMAs (one instruction for the
// real and imaginary lanes; each lane rounds as a separate fmaf).  With a real table (b.y == 0
// by construction) only the real-by-complex pair is issued.
template <bool kReal>
__device__ __forceinline__ void cmac(float2& acc, const float2 a, const float2 b)
{
    acc = __ffma2_rn(a, make_float2(b.x, b.x), acc);                        // (re, im) += a * b.re
    if (!kReal) acc = __ffma2_rn(make_float2(-a.y, a.x), make_float2(b.y, b.y), acc);  // += i * a * b.im
}

// The same multiply-add for the degridding tile kernel, where a is the lane's grid value of the
// row (a register, different for every row): with a complex table the packed form needs the
// swapped, negated copy of a and duplicated halves of b for every row, so it is written as four
// scalar fused multiply-adds instead (the negation an operand modifier), which are the same
// operations with the same roundings, component by component, as cmac.
template <bool kReal>
__device__ __forceinline__ void cmac_grid(float2& acc, const float2 a, const float2 b)
{
    if (kReal) {
        cmac<true>(acc, a, b);
    } else {
        acc.x = fmaf(a.x, b.x, acc.x);
        acc.y = fmaf(a.y, b.x, acc.y);
        acc.x = fmaf(-a.y, b.y, acc.x);
        acc.y = fmaf(a.x, b.y, acc.y);
    }
}

// CTAs per SM the register budget of a tile kernel is sized for: kR accumulators (gridding) or
// grid values (degridding) per lane, two floats each.
template <class Tab, int kR>
__host__ __device__ constexpr int grid_min_blocks() { return kR >= 32 ? 2 : Tab::kMinBlocks; }
template <class Tab, int kR>
__host__ __device__ constexpr int degrid_min_blocks() { return kR >= 32 ? 2 : Tab::kMinBlocks; }

// The CTA's work is the sequence of chunks (up to kTileChunk samples) of the work units it owns
// (every gridDim.x-th unit of the plane group).  Chunk i is staged in shared memory while chunk
// i-1 is processed, so each chunk costs one barrier and the next unit's samples arrive early.
struct ChunkCursor {
    u32 it, base;  // unit list position, first sample of the chunk in that unit
    u32 cnt, start;
    u32 ti;        // the unit's tile record (tile_record)
    u32 pslot;     // partial tile of a split cell, or kDirect
    int m;         // samples in the chunk (0: no more work)
};

__device__ __forceinline__ void cursor_load(ChunkCursor& c, u32 it, u32 i1, const uint4* __restrict__ units,
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
        c.m = int(c.cnt < u32(kTileChunk) ? c.cnt : u32(kTileChunk));
    }
}

__device__ __forceinline__ void cursor_next(ChunkCursor& c, u32 i1, const uint4* __restrict__ units, const GridArgs& a)
{
    if (c.base + u32(kTileChunk) < c.cnt) {
        c.base += u32(kTileChunk);
        const u32 left = c.cnt - c.base;
        c.m = int(left < u32(kTileChunk) ? left : u32(kTileChunk));
    } else {
        cursor_load(c, c.it + gridDim.x, i1, units, a);
    }
}

// kVar: every sample has its own footprint width (its w-plane's, a.ssz) instead of one width
// for the plan (variable-support tables, current/tConvolveMPI/Benchmark.cc:373-411).
template <class Tab, int kS, int kR, bool kVar = false>
__global__ void __launch_bounds__(kTileThreads, grid_min_blocks<Tab, kR>())
grid_tile_kernel(const float2* __restrict__ data, const typename Tab::elem* __restrict__ ctab,
                 const int* __restrict__ iu, const int* __restrict__ iv,
                 const int* __restrict__ coff, const u32* __restrict__ order,
                 const uint4* __restrict__ units, const u32* __restrict__ group_ustart, GridArgs a)
{
    constexpr int kTH = tile_height(kR);
    __shared__ float4 sm_rec[2][kTileChunk];  // (data.re, data.im, first column, first row)
    __shared__ int sm_coff[2][kTileChunk];
    __shared__ int sm_w[kVar ? 2 : 1][kVar ? kTileChunk : 1];  // per-sample widths
    __shared__ unsigned char sm_mask[2][kTileChunk];  // per sample: the warps whose blocks it meets
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s0 = kS > 0 ? kS : a.s;  // compile-time footprint width when specialised
    const u32 i1 = group_ustart[a.group + 1];
    auto stage = [&](const ChunkCursor& c, int buf) {
        if (int(threadIdx.x) < c.m) {
            const u32 k = order[c.start + c.base + threadIdx.x];
            const float2 d = data[k];
            const int sk = kVar ? int(a.ssz[k]) : s0;
            const int fx = iu[k] - (kVar ? sk / 2 : a.support), fy = iv[k];
            sm_rec[buf][threadIdx.x] = make_float4(d.x * a.c_scale, d.y * a.c_scale, __int_as_float(fx),
                                                   __int_as_float(fy));
            sm_coff[buf][threadIdx.x] = coff[k];
            if (kVar) sm_w[kVar ? buf : 0][kVar ? threadIdx.x : 0] = sk;
            // warp w's block: columns tx*64 + (w % 2)*32 + [0, 32), rows ty*kTH + (w / 2)*kR + [0, kR)
            const int bx = rec_tx(c.ti) * kTileW - fx, by = rec_ty(c.ti) * kTH - fy;
            u32 cols = 0, rows = 0;
#pragma unroll
            for (int h = 0; h < kTileW / 32; ++h)
                cols |= u32(bx + h * 32 < sk && bx + h * 32 + 32 > 0) << h;
#pragma unroll
            for (int r = 0; r < kTileWarps / (kTileW / 32); ++r)
                rows |= u32(by + r * kR < sk && by + r * kR + kR > 0) << r;
            u32 m = 0;
#pragma unroll
            for (int w = 0; w < kTileWarps; ++w)
                m |= (((cols >> (w % (kTileW / 32))) & (rows >> (w / (kTileW / 32)))) & 1u) << w;
            sm_mask[buf][threadIdx.x] = (unsigned char)m;
        }
    };
    ChunkCursor cur;
    cursor_load(cur, group_ustart[a.group] + blockIdx.x, i1, units, a);
    stage(cur, 0);
    __syncthreads();
    float2 acc[kR];
#pragma unroll
    for (int r = 0; r < kR; ++r) acc[r] = make_float2(0.f, 0.f);
    int buf = 0;
    while (cur.m > 0) {
        ChunkCursor nxt = cur;
        cursor_next(nxt, i1, units, a);
        stage(nxt, buf ^ 1);  // overlaps with the work below

        const int tx = rec_tx(cur.ti), ty = rec_ty(cur.ti);
        const int bx0 = tx * kTileW + (warp % (kTileW / 32)) * 32;  // first column of this warp
        const int gx = bx0 + lane;
        const int gy0 = ty * kTH + (warp / (kTileW / 32)) * kR;
        // the chunk's samples that meet this warp's block, in order: one ballot per 32 samples
        for (int e = 0; e < cur.m; e += 32) {
            u32 bits = __ballot_sync(0xffffffffu, e + lane < cur.m && ((sm_mask[buf][e + lane] >> warp) & 1u));
            while (bits) {
            const int j = e + __ffs(bits) - 1;
            bits &= bits - 1;
            const float4 q = sm_rec[buf][j];
            const int s = kVar ? sm_w[kVar ? buf : 0][kVar ? j : 0] : s0;
            const int fx = __float_as_int(q.z), fy = __float_as_int(q.w);
            const int dy0 = gy0 - fy;  // footprint row of this warp's first row (the block meets the footprint)
            const int dx = gx - fx;
            const bool colok = unsigned(dx) < unsigned(s);
            const float2 dv = make_float2(q.x, q.y);
            // 32-bit element index off the kernel-wide table base (tables hold < 2^31 entries)
            const int ci = sm_coff[buf][j] + dy0 * s + dx;
            if (dy0 >= 0 && dy0 + kR <= s) {
                // every row of the block is inside the footprint: only the column test remains
                if (colok) {
#pragma unroll
                    for (int r = 0; r < kR; ++r) cmac<Tab::kReal>(acc[r], dv, Tab::load(ctab + (ci + r * s)));
                }
            } else {
#pragma unroll
                for (int r = 0; r < kR; ++r) {
                    if (colok && unsigned(dy0 + r) < unsigned(s)) {
                        const float2 c = Tab::load(ctab + (ci + r * s));
                        cmac<Tab::kReal>(acc[r], dv, c);
                    }
                }
            }
            }
        }
        if ((nxt.it != cur.it || nxt.m == 0) && cur.pslot != kDirect) {
            // a unit of a split cell: its partial tile, summed into the grid by fold_kernel
            float2* pt = a.partial + (unsigned long long)(cur.pslot) * (kTileW * kTH) +
                         ((warp / (kTileW / 32)) * kR) * kTileW + (warp % (kTileW / 32)) * 32 + lane;
#pragma unroll
            for (int r = 0; r < kR; ++r) {
                pt[r * kTileW] = acc[r];
                acc[r] = make_float2(0.f, 0.f);
            }
        } else if (nxt.it != cur.it || nxt.m == 0) {
            // the cell is complete: add its tile into the job's grid (each point has this one owner)
            const JobDesc& jd = a.jobs[rec_job(cur.ti)];
            const int gs = jd.g_size;
            float2* grid = a.grid ? a.grid : jd.grid;
            if (gx < gs) {
#pragma unroll
                for (int r = 0; r < kR; ++r) {
                    const int gy = gy0 + r;
                    if (gy < gs) {
                        float2* gp = grid + ((unsigned long long)(gy) * gs + gx);
                        float2 v = *gp;
                        v.x += acc[r].x;
                        v.y += acc[r].y;
                        *gp = v;
                    }
                }
            }
#pragma unroll
            for (int r = 0; r < kR; ++r) acc[r] = make_float2(0.f, 0.f);
        }
        __syncthreads();  // the next chunk is staged; this chunk's records are free
        cur = nxt;
        buf ^= 1;
    }
}

// Degridding on the gridding plan (the adjoint of grid_tile_kernel).  A lane holds its kR grid
// points in registers; for each sample of the cell a warp whose block meets the footprint forms
// the partial dot product of its block with the table, four samples at a time reduced together
// with shuffles, and the CTA adds its 8 warp partials in warp order into the sample's slot for
// this tile.  The sample's staging thread marks the warps whose blocks meet the footprint and
// those whose rows lie wholly inside it, so a warp tests one bit per sample.  A final pass
// (slot_reduce_kernel) adds each sample's tile slots in tile order: no atomics, deterministic.
template <class Tab, int kS, int kR, bool kVar = false>
__global__ void __launch_bounds__(kTileThreads, degrid_min_blocks<Tab, kR>())
degrid_tile_kernel(const typename Tab::elem* __restrict__ ctab,
                   const int* __restrict__ iu, const int* __restrict__ iv,
                   const int* __restrict__ coff, const u32* __restrict__ order,
                   const uint4* __restrict__ units, const u32* __restrict__ group_ustart,
                   float2* __restrict__ slots, int max_tiles, GridArgs a)
{
    constexpr int kTH = tile_height(kR);
    __shared__ int4 sm_rec[kTileChunk];              // (sample, first column, first row, cOffset)
    __shared__ float2 sm_part[kTileChunk][kTileWarps];
    __shared__ int sm_w[kVar ? kTileChunk : 1];      // per-sample widths
    // per sample: the warps whose blocks it meets (bits 0..7) and those whose rows all lie
    // inside its footprint (bits 8..15)
    __shared__ unsigned short sm_mk[kTileChunk];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s0 = kS > 0 ? kS : a.s;  // compile-time footprint width when specialised
    const u32 i1 = group_ustart[a.group + 1];
    for (u32 it = group_ustart[a.group] + blockIdx.x; it < i1; it += gridDim.x) {
        const uint4 u = units[it];  // the units of a split cell each read the tile; no partials
        const u32 start = u.y, cnt = u.z;
        const u32 ti = a.tinfo[u.x - u32(a.group) * u32(a.ntiles)];
        const JobDesc& jd = a.jobs[rec_job(ti)];
        const int gs = jd.g_size;
        const float2* grid = a.grid ? a.grid : jd.grid;
        const int tx = rec_tx(ti), ty = rec_ty(ti);
        const int bx0 = tx * kTileW + (warp % (kTileW / 32)) * 32;
        const int gx = bx0 + lane;
        const int gy0 = ty * kTH + (warp / (kTileW / 32)) * kR;
        float2 gv[kR];
#pragma unroll
        for (int r = 0; r < kR; ++r)
            gv[r] = (gx < gs && gy0 + r < gs) ? grid[(unsigned long long)(gy0 + r) * gs + gx] : make_float2(0.f, 0.f);

        for (u32 base = 0; base < cnt; base += kTileChunk) {
            const int m = int(cnt - base < u32(kTileChunk) ? cnt - base : u32(kTileChunk));
            __syncthreads();
            if (threadIdx.x < m) {
                const u32 k = order[start + base + threadIdx.x];
                const int sk = kVar ? int(a.ssz[k]) : s0;
                const int fx = iu[k] - (kVar ? sk / 2 : a.support), fy = iv[k];
                sm_rec[threadIdx.x] = make_int4(int(k), fx, fy, coff[k]);
                if (kVar) sm_w[kVar ? threadIdx.x : 0] = sk;
                // warp w's block: columns tx*64 + (w % 2)*32 + [0, 32), rows ty*kTH + (w / 2)*kR + [0, kR)
                const int bx = tx * kTileW - fx, by = ty * kTH - fy;
                u32 cols = 0, rows = 0, full = 0;
#pragma unroll
                for (int h = 0; h < kTileW / 32; ++h) cols |= u32(bx + h * 32 < sk && bx + h * 32 + 32 > 0) << h;
#pragma unroll
                for (int r = 0; r < kTileWarps / (kTileW / 32); ++r) {
                    rows |= u32(by + r * kR < sk && by + r * kR + kR > 0) << r;
                    full |= u32(by + r * kR >= 0 && by + r * kR + kR <= sk) << r;
                }
                u32 mk = 0;
#pragma unroll
                for (int w = 0; w < kTileWarps; ++w) {
                    mk |= (((cols >> (w % (kTileW / 32))) & (rows >> (w / (kTileW / 32)))) & 1u) << w;
                    mk |= ((full >> (w / (kTileW / 32))) & 1u) << (8 + w);
                }
                sm_mk[threadIdx.x] = (unsigned short)mk;
            }
            __syncthreads();
            // four samples at a time: each lane's partial dot products of the four, then one
            // transposing warp reduction for all of them (6 complex shuffles instead of 20)
            for (int jg = 0; jg < m; jg += 4) {
                float2 v[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    v[e] = make_float2(0.f, 0.f);
                    const int j = jg + e;
                    if (j >= m) continue;  // warp-uniform
                    const u32 mk = sm_mk[j];
                    if (!((mk >> warp) & 1u)) continue;  // warp-uniform: the block misses the footprint
                    const int4 q = sm_rec[j];
                    const int s = kVar ? sm_w[kVar ? j : 0] : s0;
                    const int fx = q.y, fy = q.z;
                    const int dy0 = gy0 - fy;
                    const int dx = gx - fx;
                    const bool colok = unsigned(dx) < unsigned(s);
                    const int ci = q.w + dy0 * s + dx;
                    float2 p0 = make_float2(0.f, 0.f), p1 = make_float2(0.f, 0.f);  // two FMA chains
                    if ((mk >> (8 + warp)) & 1u) {  // every row of the block is inside the footprint
                        if (colok) {
#pragma unroll
                            for (int r = 0; r < kR; r += 2) {
                                cmac_grid<Tab::kReal>(p0, gv[r], Tab::load(ctab + (ci + r * s)));
                                cmac_grid<Tab::kReal>(p1, gv[r + 1], Tab::load(ctab + (ci + (r + 1) * s)));
                            }
                        }
                    } else {
#pragma unroll
                        for (int r = 0; r < kR; ++r) {
                            if (colok && unsigned(dy0 + r) < unsigned(s))
                                cmac_grid<Tab::kReal>((r & 1) ? p1 : p0, gv[r], Tab::load(ctab + (ci + r * s)));
                        }
                    }
                    v[e] = __fadd2_rn(p0, p1);
                }
                // exchange over lane bit 4 (lanes keep samples 0,1 or 2,3) and bit 3 (one sample
                // each): lane holds sample (lane >> 3) & 3 summed over 4 lanes; butterflies over
                // bits 2..0 finish the sum
                const bool h16 = (lane & 16) != 0, h8 = (lane & 8) != 0;
                const float2 s0 = h16 ? v[0] : v[2], k0 = h16 ? v[2] : v[0];
                const float2 s1 = h16 ? v[1] : v[3], k1 = h16 ? v[3] : v[1];
                // (paired adds: one instruction for the real and imaginary lanes, each rounded as fadd)
                const float2 w0 = __fadd2_rn(k0, make_float2(__shfl_xor_sync(0xffffffffu, s0.x, 16),
                                                             __shfl_xor_sync(0xffffffffu, s0.y, 16)));
                const float2 w1 = __fadd2_rn(k1, make_float2(__shfl_xor_sync(0xffffffffu, s1.x, 16),
                                                             __shfl_xor_sync(0xffffffffu, s1.y, 16)));
                const float2 sd = h8 ? w0 : w1, kp = h8 ? w1 : w0;
                float2 y = __fadd2_rn(kp, make_float2(__shfl_xor_sync(0xffffffffu, sd.x, 8),
                                                      __shfl_xor_sync(0xffffffffu, sd.y, 8)));
#pragma unroll
                for (int o = 4; o; o >>= 1)
                    y = __fadd2_rn(y, make_float2(__shfl_xor_sync(0xffffffffu, y.x, o), __shfl_xor_sync(0xffffffffu, y.y, o)));
                const int js = jg + (lane >> 3);
                if ((lane & 7) == 0 && js < m) sm_part[js][warp] = y;
            }
            __syncthreads();
            if (threadIdx.x < m) {
                const int4 q = sm_rec[threadIdx.x];
                float2 v = sm_part[threadIdx.x][0];
#pragma unroll
                for (int w = 1; w < kTileWarps; ++w) v = __fadd2_rn(v, sm_part[threadIdx.x][w]);
                const int s = kVar ? sm_w[kVar ? threadIdx.x : 0] : s0;
                const int sx0 = q.y / kTileW, sx1 = (q.y + s - 1) / kTileW, sy0 = q.z / kTH;
                const int slot = (ty - sy0) * (sx1 - sx0 + 1) + (tx - sx0);
                slots[(unsigned long long)(u32(q.x)) * max_tiles + slot] = v;
            }
        }
    }
}

// Fold the partial tiles of the split cells of one plane group into the grid: for every point,
// the units' partial sums in unit order, then one add into the grid (deterministic).  Work items
// are (cell, 256-point slice of its tile), block-stride over the group's non-empty cells; cells
// that were not split are skipped.
template <int kR>
__global__ void __launch_bounds__(kTileThreads)
fold_kernel(const u32* __restrict__ items, const u32* __restrict__ group_start, const u32* __restrict__ nunits,
            const u32* __restrict__ pstart, GridArgs a)
{
    constexpr int kTH = tile_height(kR);
    constexpr int kPoints = kTileW * kTH;
    constexpr u32 kSlices = kPoints / kTileThreads;
    const u32 i0 = group_start[a.group], i1 = group_start[a.group + 1];
    for (u32 w = blockIdx.x; w < (i1 - i0) * kSlices; w += gridDim.x) {
        const u32 k = i0 + w / kSlices;
        const u32 nu = nunits[k];
        if (nu < 2) continue;  // block-uniform
        const u32 ti = a.tinfo[items[k] - u32(a.group) * u32(a.ntiles)];
        const JobDesc& jd = a.jobs[rec_job(ti)];
        const int gs = jd.g_size;
        float2* grid = a.grid ? a.grid : jd.grid;
        const float2* pt = a.partial + (unsigned long long)(pstart[k]) * kPoints;
        {
            const int p = int(w % kSlices) * kTileThreads + threadIdx.x;
            const int gx = rec_tx(ti) * kTileW + (p % kTileW), gy = rec_ty(ti) * kTH + (p / kTileW);
            const bool inside = gx < gs && gy < gs;
            float2* gp = grid + (inside ? (unsigned long long)(gy) * gs + gx : 0ull);
            const float2 g0 = inside ? *gp : make_float2(0.f, 0.f);  // in flight with the partials
            float2 v = pt[p];
            u32 q = 1;
            for (; q + 8 <= nu; q += 8) {  // eight loads in flight, added in unit order
                float2 w8[8];
#pragma unroll
                for (int e = 0; e < 8; ++e) w8[e] = pt[(unsigned long long)(q + e) * kPoints + p];
#pragma unroll
                for (int e = 0; e < 8; ++e) {
                    v.x += w8[e].x;
                    v.y += w8[e].y;
                }
            }
            for (; q + 4 <= nu; q += 4) {  // four loads in flight, added in unit order
                float2 w4[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) w4[e] = pt[(unsigned long long)(q + e) * kPoints + p];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    v.x += w4[e].x;
                    v.y += w4[e].y;
                }
            }
            for (; q < nu; ++q) {
                const float2 w1 = pt[(unsigned long long)(q) * kPoints + p];
                v.x += w1.x;
                v.y += w1.y;
            }
            if (inside) {
                float2 o = g0;
                o.x += v.x;
                o.y += v.y;
                *gp = o;
            }
        }
    }
}

}  // namespace tcv
