// tcv_internal.cuh -- shared device helpers and the plan layout of libtconvolve.
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cstdint>
#include <cstddef>
#include <utility>
#include <vector>

#include "tconvolve.h"
#include "tcv_device.cuh"

namespace tcv {

// float16 table forms (need cuda_fp16.h, so they live outside the NVRTC-compiled device header)
struct TabCF16 {
    static constexpr int kMinBlocks = 3;
    static constexpr bool kReal = false;
    using elem = __half2;
    __device__ __forceinline__ static float2 load(const elem* p) { return __half22float2(__ldg(p)); }
};
struct TabRF16 {
    static constexpr int kMinBlocks = 4;
    static constexpr bool kReal = true;
    using elem = __half;
    __device__ __forceinline__ static float2 load(const elem* p) { return make_float2(__half2float(__ldg(p)), 0.f); }
};

// ------------------------------------------------------------------------------------------
// Plan: binning of samples into grid tiles (gridding) and anchor tiles (degridding).
// ------------------------------------------------------------------------------------------
struct PlanGeom {
    int64_t n;          // samples (all jobs)
    int support, s;     // support, sSize = 2*support+1
    int g_size;         // grid side of a one-job plan; the largest job's side in a batch
    int64_t c_len;      // table entries
    int kid_bits;       // bits of the kernel index cOffset / sSize^2
    // kernels are processed in groups of kid_group consecutive indices (whole w-planes), sized
    // so that one group's slice of the table stays resident in L2 while every SM works on it
    int kid_group, n_groups, group_bits, group_mib;
    int n_jobs;
    // gridding: output-stationary tiles of tw x th points (th = 4 * rows); work cells are
    // (group, tile) with the tiles of all jobs numbered in one space
    int rows, tw, th;
    int split;          // samples per gridding work unit of a split cell (0: cells are never split)
    int dsplit;         // the same for degridding
    bool dense;         // sample-parallel gridding kernel (tcv_dense.cu; 64 x 32 tiles)
    bool ddense;        // sample-parallel degridding kernel
    int ntx, nty;       // tiles per row / column of a one-job plan
    int64_t ntiles;     // tiles of all jobs
    int max_tiles;      // tiles one footprint can touch
    int tile_bits, key_bits;
    // degridding anchor tiles (footprint top-left corner; one-job plans only)
    bool anchors;
    int ta, natx, naty, atile_bits, akey_bits;
    int box_w, box_h;   // staged region (elements), box_w even
    int degrid_mode;    // 0 staged (TMA), 1 direct from global
    int degrid_parts;   // warps sharing one sample's footprint in the staged kernel
    bool key64;         // 64-bit sort keys
    // variable-width plans (one footprint width per w-plane; s and support are the widest)
    bool var;
    int n_planes;
};

}  // namespace tcv

struct tcv_plan {
    tcv::PlanGeom g;
    const int32_t *iu, *iv, *coff;  // the sample arrays the plan was binned from (device)
    // device arrays inside the caller's workspace
    tcv::JobDesc* jobs;            // job table, n_jobs
    uint32_t* job_start;           // n_jobs + 1: first sample of each job
    uint32_t* tinfo;               // per tile of all jobs: tile_record(job, column, row)
    uint16_t* ntl;                 // per sample: tiles its footprint touches (0 = left out)
    void* keys[2];                 // grid pair keys (double buffer), n * max_tiles
    uint32_t* vals[2];             // grid pair sample indices
    void* akeys[2];                // anchor keys, n
    uint32_t* avals[2];            // anchor sample indices
    uint32_t* tile_count;          // samples per cell (group, tile): n_groups * ntiles
    uint32_t* tile_start;          // first sorted pair of each cell
    uint32_t* items;               // non-empty gridding cells, group-major
    uint32_t* n_items;             // [0] = number of non-empty gridding cells
    uint32_t* group_start;         // n_groups + 1: items of group g are [group_start[g], group_start[g+1])
    uint32_t* group_ustart;        // n_groups + 1: work units of group g
    uint32_t* nunits;              // per item: work units of its cell
    uint32_t* ustart;              // per item: its first unit
    uint32_t* pstart;              // per item: its first partial tile (split cells)
    uint4* units;                  // work units (cell, first sorted pair, count, partial tile or kDirect)
    float2* partial;               // partial tiles of split cells, tw x th points each
    uint4* d_units;                // degridding work units (the gridding list when the sizes agree)
    uint32_t* d_group_ustart;
    uint32_t *d_nunits, *d_ustart, *d_pstart;
    uint32_t* atile_count;         // samples per anchor cell (group, anchor tile)
    uint32_t* atile_start;
    uint32_t* aitems;              // non-empty anchor cells, group-major
    uint32_t* n_aitems;
    unsigned long long* rejected;  // samples left out as out of bounds
    unsigned int* status;          // device status block (tcv::kStatusWords words): word 0 bit 0 = a
                                   // bounded wait timed out; words kSchedWord, +1: the sample-parallel
                                   // gridding kernel's work-item counters (zero between launches)
    float2* slots;                 // degridding partial sums, n * max_tiles
    void* cub_temp;
    size_t cub_bytes;
    int sel;                       // which buffer holds the sorted grid pairs
    int asel;                      // which buffer holds the sorted anchor pairs
    int degrid_variant;            // TCV_DEGRID_TILES or TCV_DEGRID_ANCHOR (reference-layout tables)
    bool batch;                    // jobs carry their own grids (tcv_batch_plan_create)
    bool binned;
    bool jit_cached_only = false;  // launch specialised tile kernels only if already built (never compile)
    bool anchors_ready = false;    // the anchor binning matches the last binning
    bool anchors_stale = false;    // a captured binning skipped it: anchor degridding re-bins always
    std::vector<tcv::JobDesc> host_jobs;  // the job table (kept alive for its asynchronous copy)
    std::vector<uint32_t> host_job_start;
    // variable-width plans
    const int32_t* wplane;         // per-sample w-plane (device, the caller's)
    int32_t* plane_s;              // footprint width per plane (device)
    int32_t* plane_grp;            // plane group per plane (device)
    uint16_t* ssz;                 // per-sample footprint width (device)
    // sample-parallel kernels: per sorted (sample, tile) pair, the sample's footprint (first column,
    // first row, cOffset, width), gathered once per binning (nullptr unless a pass uses them)
    int4* grec;
    std::vector<int32_t> host_plane_s, host_plane_grp;
};

namespace tcv {

constexpr int kStatusWords = 8;  // the plan's status block, zeroed by every binning
constexpr int kSchedWord = 4;    // first of the two work-item counters in it

// Host helpers implemented in tcv_plan.cu
// Geometry for jobs of the given grid sides (n samples in all); tuning may be nullptr.  anchors:
// also bin for the anchor-tile degridding kernels (one-job plans of tcv_plan_build only).
PlanGeom make_geom(int64_t n, int support, const int* g_sizes, int n_jobs, int64_t c_len, const tcv_tuning* t,
                   bool anchors);
size_t plan_bytes(const PlanGeom& g, size_t* cub_bytes_out);
// one-job plan in d_work, binned (tcv_plan_build)
tcv_status plan_init(tcv_plan* p, const int32_t* d_iu, const int32_t* d_iv, const int32_t* d_coff, int64_t n,
                     int support, int g_size, int64_t c_len, void* d_work, size_t work_bytes, cudaStream_t st,
                     const tcv_tuning* t = nullptr);
tcv_status plan_bin(tcv_plan* p, const int32_t* d_iu, const int32_t* d_iv, const int32_t* d_coff, cudaStream_t st);

// Launchers implemented in tcv_grid.cu / tcv_degrid.cu
tcv_status launch_grid(const tcv_plan* p, const float2* data, const void* c, int c_type,
                       float c_scale, float2* grid, cudaStream_t st);
tcv_status launch_degrid(const tcv_plan* p, const float2* grid, const void* c, int c_type,
                         float c_scale, float2* out, cudaStream_t st);

// tile kernels specialised on the footprint width (tcv_jit.cu): kind 0 gridding, 1 degridding;
// nullptr when no specialised copy is available (the generic copy is used)
// rows: grid rows per warp (the tile shape)
const void* jit_tile_kernel(int kind, int c_type, int s, int rows);
// the same, but only a copy built earlier: never compiles or loads a module (nullptr otherwise)
const void* jit_tile_kernel_cached(int kind, int c_type, int s, int rows);
// build both specialised tile kernels of (form, sSize, rows) ahead of a capture or a timing
void jit_prepare(int c_type, int s, int rows);
// FFT steps (tcv_fft.cu): fftExec in place; the inverse transform of a grid fused with fftFix into
// a float image (and/or a complex one); the forward transform of a real image into a grid.
tcv_status fft_exec(float2* d_grid, int n, bool forward, cudaStream_t st);
// the set-up of the transforms of size n (twiddle table; allocates): before any capture
tcv_status fft_prepare(int n);
tcv_status image_from_grid(float2* d_grid, int n, float scale, float* d_image, float2* d_image_c, cudaStream_t st);
tcv_status grid_from_image(const float* d_image, int n, float2* d_grid, cudaStream_t st);
// Sample-parallel kernels on 64 x 32 tiles (tcv_dense.cu), for any plan of 8-row tiles.
template <class Tab>
tcv_status launch_dense_grid(const tcv_plan* p, const float2* data, const void* c, float c_scale, float2* grid,
                             cudaStream_t st);
template <class Tab>
tcv_status launch_dense_degrid(const tcv_plan* p, const float2* grid, const void* c, float c_scale, float2* out,
                               cudaStream_t st);
// fill p->grec from the sorted pairs (after each binning of a plan that has it)
tcv_status gather_pair_records(const tcv_plan* p, cudaStream_t st);
// fold_kernel<8> over one plane group of a plan (the partial tiles of its split cells)
tcv_status launch_fold8(const tcv_plan* p, const GridArgs& a, cudaStream_t st);
// Record the candidates and median times of the last tuning run (read by tcv_autotune_report).
void tune_report_set(const std::vector<std::pair<tcv_tuning, float>>& report);

// degridding on the gridding plan (tcv_grid.cu), and the per-sample slot sum it ends with
tcv_status launch_degrid_tiles(const tcv_plan* p, const float2* grid, const void* c, int c_type,
                               float c_scale, float2* out, cudaStream_t st);
tcv_status slot_reduce(const tcv_plan* p, float c_scale, float2* out, cudaStream_t st);

// TMA pipeline kernels on prepared (padded) tables, tcv_pipe.cu
tcv_status launch_grid_pipe(const tcv_plan* p, const float2* data, const void* table, int c_type,
                            float c_scale, float2* grid, cudaStream_t st);
tcv_status launch_degrid_pipe(const tcv_plan* p, const float2* grid, const void* table, int c_type,
                              float c_scale, float2* out, cudaStream_t st);
size_t padded_table_bytes(int64_t c_len, int s, int c_type);

// two-columns-per-lane tile kernels on paired tables, tcv_pair.cu
tcv_status launch_grid_pair(const tcv_plan* p, const float2* data, const void* table, int c_type,
                            float c_scale, float2* grid, cudaStream_t st);
tcv_status launch_degrid_pair(const tcv_plan* p, const float2* grid, const void* table, int c_type,
                              float c_scale, float2* out, cudaStream_t st);
int paired_pitch(int s);
int64_t paired_copy_stride(int64_t c_len, int s);
size_t paired_table_bytes(int64_t c_len, int s, int c_type);
tcv_status pair_table(const void* in, int64_t c_len, int s, int c_type, void* out, cudaStream_t st);
tcv_status pad_table(const void* in, int64_t c_len, int s, int c_type, void* out, cudaStream_t st);

// The reference's K&R generator x -> a x + c (mod 2^64) (attic/tConvolveMPI/Benchmark.cc:53-58,
// current/tConvolveMPI/Benchmark.cc:53-58): A, C of the map after m steps, by binary powering
// of the affine map, so that sample i's draws start from A * state0 + C.
constexpr uint64_t kLcgA = 1103515245ull;
constexpr uint64_t kLcgC = 12345ull;
__host__ __device__ inline void lcg_jump(uint64_t m, uint64_t& A, uint64_t& C)
{
    uint64_t a = kLcgA, c = kLcgC;
    A = 1;
    C = 0;
    while (m) {
        if (m & 1) {
            C = a * C + c;
            A = a * A;
        }
        c = a * c + c;
        a = a * a;
        m >>= 1;
    }
}

inline tcv_status cuda_status(cudaError_t e)
{
    if (e == cudaSuccess) return TCV_OK;
    if (e == cudaErrorMemoryAllocation) return TCV_ERR_OOM;
    return TCV_ERR_CUDA;
}

}  // namespace tcv

#define TCV_CHECK(call)                    \
    do {                                   \
        const tcv_status _s = (call);      \
        if (_s != TCV_OK) return _s;       \
    } while (0)

#define TCV_CUDA(call)                                         \
    do {                                                       \
        cudaError_t _e = (call);                               \
        if (_e != cudaSuccess) return ::tcv::cuda_status(_e);  \
    } while (0)
