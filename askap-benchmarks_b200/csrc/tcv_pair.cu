// tcv_pair.cu -- tile kernels on the paired table layout (two columns per lane).
//
// Same plan and tiles as tcv_grid.cu (64 x 64 output tiles, plane-group cells), but each lane
// owns two adjacent grid columns, so one warp row covers the whole tile width with one 8-byte
// (real table) or 16-byte (complex table) load per lane, and the products are packed FP32x2
// FMAs (__ffma2_rn).  A pair load must be aligned: for a sample whose footprint starts dx0
// columns left of the tile, lane l needs table columns (dx0 + 2l, dx0 + 2l + 1), which start on
// an even column only when dx0 is even.  The paired layout therefore stores every kernel row
// twice, with an even pitch P >= sSize + 1:
//   copy A: A[c] = C[c] for c < sSize, 0 beyond;
//   copy B: B[c] = C[c - 1] for 1 <= c <= sSize, B[0] = 0 (the row shifted right by one);
// an odd dx0 reads copy B from column dx0 + 1 (even).  Pairs that straddle the footprint's
// edge read the zeros at the row ends, so the only column test is whether a pair touches the
// footprint at all.  Copy B's zero first column also makes the one entry read past a row's end
// harmless; a 16-byte guard follows the last row.
//
// 8 warps x 8 rows cover a 64 x 64 tile.  Gridding keeps accumulators in registers and adds the
// tile into the grid once per cell; degridding holds the tile's grid values and reduces partial
// dot products into per-(tile, sample) slots summed in fixed order (slot_reduce_kernel).
#include "tcv_internal.cuh"

namespace tcv {
namespace {

constexpr int kTileW = 64;
constexpr int kTileH = 64;
constexpr int kRows = 8;
constexpr int kWarps = kTileH / kRows;  // 8
constexpr int kThreads = kWarps * 32;
constexpr int kChunk = kThreads;

struct PairArgs {
    int support, s, g_size, ntx, ntiles, group, max_tiles;
    int pitch;            // P, entries per stored row (even)
    int64_t copy_stride;  // entries from copy A to copy B
    float c_scale;
};

// Real table entries as pairs (c0, c1)
struct PairR32 {
    static constexpr bool kComplex = false;
    using pair_t = float2;
    __device__ __forceinline__ static float2 load(const void* base, int64_t i)
    {
        return __ldg(reinterpret_cast<const float2*>(static_cast<const float*>(base) + i));
    }
};
struct PairRBF16 {
    static constexpr bool kComplex = false;
    __device__ __forceinline__ static float2 load(const void* base, int64_t i)
    {
        const uint32_t u = __ldg(reinterpret_cast<const uint32_t*>(static_cast<const uint16_t*>(base) + i));
        return make_float2(__uint_as_float(u << 16), __uint_as_float(u & 0xffff0000u));
    }
};
struct PairRF16 {
    static constexpr bool kComplex = false;
    __device__ __forceinline__ static float2 load(const void* base, int64_t i)
    {
        const __half2 h = __ldg(reinterpret_cast<const __half2*>(static_cast<const __half*>(base) + i));
        return __half22float2(h);
    }
};
// Complex table entries as pairs ((c0.re, c0.im), (c1.re, c1.im)) in a float4
struct PairC64 {
    static constexpr bool kComplex = true;
    __device__ __forceinline__ static float4 load(const void* base, int64_t i)
    {
        return __ldg(reinterpret_cast<const float4*>(static_cast<const float2*>(base) + i));
    }
};
struct PairCBF16 {
    static constexpr bool kComplex = true;
    __device__ __forceinline__ static float4 load(const void* base, int64_t i)
    {
        const uint2 u = __ldg(reinterpret_cast<const uint2*>(static_cast<const uint32_t*>(base) + i));
        return make_float4(__uint_as_float(u.x << 16), __uint_as_float(u.x & 0xffff0000u),
                           __uint_as_float(u.y << 16), __uint_as_float(u.y & 0xffff0000u));
    }
};
struct PairCF16 {
    static constexpr bool kComplex = true;
    __device__ __forceinline__ static float4 load(const void* base, int64_t i)
    {
        const uint2 u = __ldg(reinterpret_cast<const uint2*>(static_cast<const __half2*>(base) + i));
        const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&u.x));
        const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&u.y));
        return make_float4(a.x, a.y, b.x, b.y);
    }
};

struct SampleRec {
    float dr, di;  // sample value x c_scale (gridding)
    int fx, fy;    // footprint's first column and row
    int kid;       // kernel index cOffset / sSize^2
    uint32_t k;    // sample index
};

template <class F, bool kDegrid>
__global__ void __launch_bounds__(kThreads, 2)
pair_tile_kernel(const float2* __restrict__ data, const void* __restrict__ table,
                 const int32_t* __restrict__ iu, const int32_t* __restrict__ iv,
                 const int32_t* __restrict__ coff, const uint32_t* __restrict__ order,
                 const uint32_t* __restrict__ tile_start, const uint32_t* __restrict__ tile_count,
                 const uint32_t* __restrict__ items, const uint32_t* __restrict__ group_start,
                 float2* __restrict__ grid, float2* __restrict__ slots, PairArgs a)
{
    __shared__ SampleRec sm_rec[kChunk];
    __shared__ float2 sm_part[kDegrid ? kChunk : 1][kWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s = a.s;
    const int64_t kid_stride = int64_t(s) * a.pitch;
    const uint32_t i1 = group_start[a.group + 1];
    for (uint32_t it = group_start[a.group] + blockIdx.x; it < i1; it += gridDim.x) {
        const uint32_t cell = items[it];
        const uint32_t cnt = tile_count[cell];
        const uint32_t start = tile_start[cell];
        const int tile = int(cell % uint32_t(a.ntiles));
        const int tx = tile % a.ntx, ty = tile / a.ntx;
        const int tx0 = tx * kTileW;
        const int gx = tx0 + 2 * lane;               // first of this lane's two columns
        const int gy0 = ty * kTileH + warp * kRows;  // first row of this warp

        // gridding: re and im accumulators of the two columns, as packed pairs
        //   real table:    (re0, re1), (im0, im1)
        //   complex table: split form a1 = sum (x.re, x.re) * (c.re, c.im), a2 = sum (x.im, x.im) * (c.re, c.im)
        // degridding: the grid values in the packed order the FMAs need
        float2 r0[kRows], r1[kRows], r2[F::kComplex ? kRows : 1], r3[F::kComplex ? kRows : 1];
#pragma unroll
        for (int r = 0; r < kRows; ++r) {
            if (!kDegrid) {
                r0[r] = r1[r] = make_float2(0.f, 0.f);
                if constexpr (F::kComplex) r2[r] = r3[r] = make_float2(0.f, 0.f);
            } else {
                float2 g0 = make_float2(0.f, 0.f), g1 = g0;
                const int gy = gy0 + r;
                if (gy < a.g_size) {
                    if (gx < a.g_size) g0 = grid[size_t(gy) * a.g_size + gx];
                    if (gx + 1 < a.g_size) g1 = grid[size_t(gy) * a.g_size + gx + 1];
                }
                if constexpr (F::kComplex) {
                    r0[r] = make_float2(g0.x, g0.x);
                    r1[r] = make_float2(g0.y, g0.y);
                    r2[r] = make_float2(g1.x, g1.x);
                    r3[r] = make_float2(g1.y, g1.y);
                } else {
                    r0[r] = make_float2(g0.x, g1.x);
                    r1[r] = make_float2(g0.y, g1.y);
                }
            }
        }

        for (uint32_t base = 0; base < cnt; base += kChunk) {
            const int m = int(cnt - base < uint32_t(kChunk) ? cnt - base : uint32_t(kChunk));
            __syncthreads();
            if (threadIdx.x < m) {
                const uint32_t k = order[start + base + threadIdx.x];
                SampleRec q;
                if (!kDegrid) {
                    const float2 d = data[k];
                    q.dr = d.x * a.c_scale;
                    q.di = d.y * a.c_scale;
                } else {
                    q.dr = q.di = 0.f;
                }
                q.fx = iu[k] - a.support;
                q.fy = iv[k];
                q.kid = coff[k] / (s * s);
                q.k = k;
                sm_rec[threadIdx.x] = q;
            }
            __syncthreads();
            for (int j = 0; j < m; ++j) {
                const SampleRec q = sm_rec[j];
                const int dy0 = gy0 - q.fy;                        // footprint row of this warp's first row
                const bool rows_hit = dy0 < s && dy0 + kRows > 0;  // warp-uniform
                float2 v = make_float2(0.f, 0.f);
                if (rows_hit) {
                    const int dx0 = tx0 - q.fx;                    // footprint column of the tile's column 0
                    const int odd = dx0 & 1;
                    const int c0 = dx0 + 2 * lane;                 // first footprint column of this lane's pair
                    const bool col_hit = c0 + 1 >= 0 && c0 < s;
                    // aligned element index of the pair in copy A (even dx0) or copy B (odd dx0)
                    const int64_t e = (odd ? a.copy_stride : 0) + q.kid * kid_stride + int64_t(dy0) * a.pitch + c0 + odd;
                    const bool all_rows = dy0 >= 0 && dy0 + kRows <= s;
                    if constexpr (!kDegrid) {
                        const float2 d_re = make_float2(q.dr, q.dr), d_im = make_float2(q.di, q.di);
                        if (col_hit) {
#pragma unroll
                            for (int r = 0; r < kRows; ++r) {
                                if (all_rows || unsigned(dy0 + r) < unsigned(s)) {
                                    if constexpr (F::kComplex) {
                                        const float4 c = F::load(table, e + int64_t(r) * a.pitch);
                                        const float2 cA = make_float2(c.x, c.y), cB = make_float2(c.z, c.w);
                                        r0[r] = __ffma2_rn(d_re, cA, r0[r]);
                                        r1[r] = __ffma2_rn(d_im, cA, r1[r]);
                                        r2[r] = __ffma2_rn(d_re, cB, r2[r]);
                                        r3[r] = __ffma2_rn(d_im, cB, r3[r]);
                                    } else {
                                        const float2 c = F::load(table, e + int64_t(r) * a.pitch);
                                        r0[r] = __ffma2_rn(d_re, c, r0[r]);
                                        r1[r] = __ffma2_rn(d_im, c, r1[r]);
                                    }
                                }
                            }
                        }
                    } else {
                        float2 p0 = make_float2(0.f, 0.f), p1 = p0, p2 = p0, p3 = p0;
                        if (col_hit) {
#pragma unroll
                            for (int r = 0; r < kRows; ++r) {
                                if (all_rows || unsigned(dy0 + r) < unsigned(s)) {
                                    if constexpr (F::kComplex) {
                                        const float4 c = F::load(table, e + int64_t(r) * a.pitch);
                                        const float2 cA = make_float2(c.x, c.y), cB = make_float2(c.z, c.w);
                                        // g x c = (g.re c.re - g.im c.im, g.re c.im + g.im c.re)
                                        p0 = __ffma2_rn(r0[r], cA, p0);  // (g0.re c.re, g0.re c.im)
                                        p1 = __ffma2_rn(r1[r], cA, p1);  // (g0.im c.re, g0.im c.im)
                                        p2 = __ffma2_rn(r2[r], cB, p2);
                                        p3 = __ffma2_rn(r3[r], cB, p3);
                                    } else {
                                        // the same per-column sums, in the same row order, as the
                                        // complex path: the real form stays bit-identical to it
                                        const float2 c = F::load(table, e + int64_t(r) * a.pitch);
                                        p0 = __ffma2_rn(r0[r], c, p0);  // (g0.re c0, g1.re c1)
                                        p1 = __ffma2_rn(r1[r], c, p1);  // (g0.im c0, g1.im c1)
                                    }
                                }
                            }
                        }
                        if constexpr (F::kComplex)
                            v = make_float2((p0.x - p1.y) + (p2.x - p3.y), (p0.y + p1.x) + (p2.y + p3.x));
                        else
                            v = make_float2(p0.x + p0.y, p1.x + p1.y);
#pragma unroll
                        for (int o = 16; o; o >>= 1) {
                            v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
                            v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
                        }
                    }
                }
                if constexpr (kDegrid) {
                    if (lane == 0) sm_part[j][warp] = v;
                }
            }
            if constexpr (kDegrid) {
                __syncthreads();
                if (threadIdx.x < m) {
                    const SampleRec q = sm_rec[threadIdx.x];
                    float2 v = sm_part[threadIdx.x][0];
#pragma unroll
                    for (int w = 1; w < kWarps; ++w) {
                        v.x += sm_part[threadIdx.x][w].x;
                        v.y += sm_part[threadIdx.x][w].y;
                    }
                    const int sx0 = q.fx / kTileW, sx1 = (q.fx + s - 1) / kTileW, sy0 = q.fy / kTileH;
                    const int slot = (ty - sy0) * (sx1 - sx0 + 1) + (tx - sx0);
                    slots[size_t(q.k) * a.max_tiles + slot] = v;
                }
            }
        }
        if constexpr (!kDegrid) {
#pragma unroll
            for (int r = 0; r < kRows; ++r) {
                const int gy = gy0 + r;
                if (gy >= a.g_size) continue;
                float2 v0, v1;  // this lane's two grid points
                if constexpr (F::kComplex) {
                    v0 = make_float2(r0[r].x - r1[r].y, r0[r].y + r1[r].x);
                    v1 = make_float2(r2[r].x - r3[r].y, r2[r].y + r3[r].x);
                } else {
                    v0 = make_float2(r0[r].x, r1[r].x);
                    v1 = make_float2(r0[r].y, r1[r].y);
                }
                float2* gp = grid + size_t(gy) * a.g_size + gx;
                if (gx + 1 < a.g_size && (a.g_size % 2 == 0)) {
                    float4 g = *reinterpret_cast<float4*>(gp);
                    g.x += v0.x;
                    g.y += v0.y;
                    g.z += v1.x;
                    g.w += v1.y;
                    *reinterpret_cast<float4*>(gp) = g;
                } else {
                    if (gx < a.g_size) {
                        gp[0].x += v0.x;
                        gp[0].y += v0.y;
                    }
                    if (gx + 1 < a.g_size) {
                        gp[1].x += v1.x;
                        gp[1].y += v1.y;
                    }
                }
            }
        }
    }
}

template <class F, bool kDegrid>
int resident()
{
    static int per_sm = 0;
    static int sms = 0;
    if (!per_sm) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pair_tile_kernel<F, kDegrid>, kThreads, 0);
        if (per_sm < 1) per_sm = 1;
    }
    return per_sm * sms;
}

template <class F, bool kDegrid>
tcv_status launch(const tcv_plan* p, const float2* data, const void* table, float c_scale, float2* grid,
                  float2* out, cudaStream_t st)
{
    const PlanGeom& g = p->g;
    if (g.tw != kTileW || g.th != kTileH) return TCV_ERR_UNSUPPORTED;
    if (g.n == 0) return TCV_OK;
    const int64_t s2 = int64_t(g.s) * g.s;
    if (g.c_len % s2) return TCV_ERR_UNSUPPORTED;
    if (reinterpret_cast<uintptr_t>(table) & 15) return TCV_ERR_ARG;
    PairArgs a{};
    a.support = g.support;
    a.s = g.s;
    a.g_size = g.g_size;
    a.ntx = g.ntx;
    a.ntiles = g.ntx * g.nty;
    a.max_tiles = g.max_tiles;
    a.pitch = paired_pitch(g.s);
    a.copy_stride = paired_copy_stride(g.c_len, g.s);
    a.c_scale = c_scale;
    const int ctas = resident<F, kDegrid>();
    for (int grp = 0; grp < g.n_groups; ++grp) {
        a.group = grp;
        pair_tile_kernel<F, kDegrid><<<ctas, kThreads, 0, st>>>(
            data, table, p->iu, p->iv, p->coff, p->vals[p->sel], p->tile_start, p->tile_count, p->items,
            p->group_start, grid, p->slots, a);
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
        case TCV_C_C64: return launch<PairC64, kDegrid>(p, data, table, c_scale, grid, out, st);
        case TCV_C_R32: return launch<PairR32, kDegrid>(p, data, table, c_scale, grid, out, st);
        case TCV_C_CBF16: return launch<PairCBF16, kDegrid>(p, data, table, c_scale, grid, out, st);
        case TCV_C_RBF16: return launch<PairRBF16, kDegrid>(p, data, table, c_scale, grid, out, st);
        case TCV_C_CF16: return launch<PairCF16, kDegrid>(p, data, table, c_scale, grid, out, st);
        case TCV_C_RF16: return launch<PairRF16, kDegrid>(p, data, table, c_scale, grid, out, st);
        default: return TCV_ERR_ARG;
    }
}

// reference layout -> paired layout (copy A, then copy B at copy_stride), same storage type
template <typename T>
__global__ void pair_layout_kernel(const T* __restrict__ in, T* __restrict__ out, int64_t nk, int s, int pitch,
                                   int64_t copy_stride)
{
    const int64_t per_copy = nk * s * int64_t(pitch);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < per_copy; i += (int64_t)gridDim.x * blockDim.x) {
        const int c = int(i % pitch);
        const int64_t kr = i / pitch;  // kernel * s + row
        out[i] = c < s ? in[kr * s + c] : T{};
        out[copy_stride + i] = (c >= 1 && c <= s) ? in[kr * s + c - 1] : T{};
    }
    // guard after the last row of copy B
    if (blockIdx.x == 0 && threadIdx.x < 16 / sizeof(T)) out[copy_stride + per_copy + threadIdx.x] = T{};
}

}  // namespace

int paired_pitch(int s) { return (s + 2) & ~1; }  // >= s + 1, even

int64_t paired_copy_stride(int64_t c_len, int s)
{
    const int64_t per_copy = c_len / (int64_t(s) * s) * s * paired_pitch(s);
    return (per_copy + 31) / 32 * 32;  // keeps copy B 16-byte aligned for every entry size
}

size_t paired_table_bytes(int64_t c_len, int s, int c_type)
{
    const size_t es = tcv_ctype_bytes(c_type);
    if (!es || s < 1 || c_len % (int64_t(s) * s)) return 0;
    const int64_t per_copy = c_len / (int64_t(s) * s) * s * paired_pitch(s);
    return size_t(paired_copy_stride(c_len, s) + per_copy) * es + 16;
}

tcv_status pair_table(const void* in, int64_t c_len, int s, int c_type, void* out, cudaStream_t st)
{
    const size_t es = tcv_ctype_bytes(c_type);
    const int64_t s2 = int64_t(s) * s;
    if (!es || c_len % s2) return TCV_ERR_ARG;
    const int64_t nk = c_len / s2;
    const int pitch = paired_pitch(s);
    const int64_t cs = paired_copy_stride(c_len, s);
    const int blocks = 148 * 32;
    switch (es) {
        case 8: pair_layout_kernel<uint64_t><<<blocks, 256, 0, st>>>(static_cast<const uint64_t*>(in), static_cast<uint64_t*>(out), nk, s, pitch, cs); break;
        case 4: pair_layout_kernel<uint32_t><<<blocks, 256, 0, st>>>(static_cast<const uint32_t*>(in), static_cast<uint32_t*>(out), nk, s, pitch, cs); break;
        case 2: pair_layout_kernel<uint16_t><<<blocks, 256, 0, st>>>(static_cast<const uint16_t*>(in), static_cast<uint16_t*>(out), nk, s, pitch, cs); break;
        default: return TCV_ERR_ARG;
    }
    TCV_CUDA(cudaGetLastError());
    return TCV_OK;
}

tcv_status launch_grid_pair(const tcv_plan* p, const float2* data, const void* table, int c_type, float c_scale,
                            float2* grid, cudaStream_t st)
{
    return dispatch<false>(p, data, table, c_type, c_scale, grid, nullptr, st);
}

tcv_status launch_degrid_pair(const tcv_plan* p, const float2* grid, const void* table, int c_type, float c_scale,
                              float2* out, cudaStream_t st)
{
    return dispatch<true>(p, nullptr, table, c_type, c_scale, const_cast<float2*>(grid), out, st);
}

}  // namespace tcv
