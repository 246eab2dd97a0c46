// tcv_major.cu -- the imaging major cycle of current/tMajorACC on one GPU.
//
// Reference: current/tMajorACC/tMajorACC.cc:889-1635 (main).  Set-up (:930-1010): u, v, w from the
// K&R generator (three draws per sample, as attic/tConvolveMPI), the inverse wavelengths, initC
// (:349-434, which in this program leaves every kernel a single 1 at its (0, 0) corner: the
// w-projection expressions are commented out; normalised by the float sum of |C|, a factor of
// exactly 1), initCOffset (:436-485, the attic formula), a sky of 100 point sources drawn from the
// same generator (:1013-1020), its forward FFT (:1023) and the degridded visibilities (:1032).
// A major cycle (:1096-1452, the OpenACC path): grid the PSF (unit visibilities, first cycle only)
// and the data; inverse FFT with the half-size rotations and keep Re * 1/nVis (fftExecGPU +
// fftFixGPU); Hogbom CLEAN of the dirty image with the PSF (nMinor iterations, gain 0.1, no
// threshold) into a model image; forward FFT of the model; degrid the model visibilities; subtract
// them from the data.  The stage timers follow the reference's (gridding PSF, gridding data,
// inverse FFTs, Hogbom, forward FFT, degridding).
//
// The reference's OpenACC findPeakACC (:703-721) returns |peak| and an arbitrary index among
// equal magnitudes; its verification (:1471-1558) compares against the CPU path, whose signed
// findPeak picks the first index (:689-701).  The CPU path's definition is the one kept here.
//
// B200 form: every buffer resident; one binning plan for all passes (the samples never move); the
// delta table in the real float form (exact: its imaginary parts are zero); the FFT steps of
// tcv_fft.cu (cuFFT with the rotations and the fix fused into one pass each); the Hogbom loop of
// tcv_hogbom.cu on float images; no host round trip inside a cycle.
#include "tcv_internal.cuh"

#include <cmath>
#include <cstring>
#include <limits>
#include <new>
#include <string>
#include <vector>

namespace tcv {
namespace {

// r32 delta table: C[cind] = 1 where i == 0 && j == 0 (tMajorACC.cc:412), every other entry 0
__global__ void delta_table_kernel(float* __restrict__ c, int64_t c_len, int64_t s2)
{
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < c_len; i += int64_t(gridDim.x) * blockDim.x)
        c[i] = (i % s2) == 0 ? 1.f : 0.f;
}

__global__ void fill_kernel(float2* __restrict__ p, int64_t n, float2 v)
{
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        p[i] = v;
}

// the sources in draw order, added one after another (duplicates accumulate as the reference's +=)
__global__ void sky_kernel(float2* __restrict__ grid, const int64_t* __restrict__ idx, const float* __restrict__ val,
                           int n)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    for (int i = 0; i < n; ++i) {
        float2 g = grid[idx[i]];
        g.x = __fadd_rn(g.x, val[i]);
        grid[idx[i]] = g;
    }
}

// data -= model (tMajorACC.cc:1593-1596)
__global__ void subtract_kernel(float2* __restrict__ data, const float2* __restrict__ model, int64_t n)
{
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const float2 d = data[i], m = model[i];
        data[i] = make_float2(__fsub_rn(d.x, m.x), __fsub_rn(d.y, m.y));
    }
}

unsigned nblk(int64_t n) { return unsigned(std::min<int64_t>((n + 255) / 256 < 1 ? 1 : (n + 255) / 256, 148 * 16)); }

}  // namespace
}  // namespace tcv

using namespace tcv;

struct tcv_major_ctx {
    tcv_major_config cfg{};
    cudaStream_t stream = nullptr;
    int support = 0, over_sample = 0;
    double w_cell_size = 0.0;
    int64_t c_len = 0, n = 0;
    float scale = 0.f;  // 1 / nVis as the reference rounds it
    double *u = nullptr, *v = nullptr, *w = nullptr, *freq = nullptr;
    int32_t *iu = nullptr, *iv = nullptr, *coff = nullptr;
    float* table = nullptr;
    float2 *data = nullptr, *model_vis = nullptr, *ones = nullptr, *grid = nullptr;
    float2 *uv_psf = nullptr, *uv_data = nullptr;  // kept copies (keep_stages)
    float *psf = nullptr, *dirty = nullptr, *residual = nullptr, *model = nullptr;
    void* plan_work = nullptr;
    size_t plan_bytes = 0;
    tcv_plan* plan = nullptr;
    void* hog_work = nullptr;
    size_t hog_bytes = 0;
    uint64_t next = 1;  // generator state after the set-up draws
    int cycles = 0;
    bool initialized = false;
    std::vector<cudaEvent_t> events;  // TCV_MAJOR_STAGES + 1 per cycle
    std::vector<int> stage_used;      // per cycle: bit mask of stages recorded
    std::string err;
};

namespace {

tcv_status mfail(tcv_major_ctx* c, tcv_status s, const std::string& what)
{
    if (c) c->err = what + ": " + tcv_status_string(s);
    return s;
}

#define MAJ_TRY(c, call)                                  \
    do {                                                  \
        const tcv_status _s = (call);                     \
        if (_s != TCV_OK) return mfail(c, _s, #call);     \
    } while (0)
#define MAJ_CUDA(c, call) MAJ_TRY(c, ::tcv::cuda_status(call))

void release(tcv_major_ctx* c)
{
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->plan) tcv_plan_destroy(c->plan);
    c->plan = nullptr;
    void* bufs[] = {c->u, c->v, c->w, c->freq, c->iu, c->iv, c->coff, c->table, c->data, c->model_vis, c->ones,
                    c->grid, c->uv_psf, c->uv_data, c->psf, c->dirty, c->residual, c->model, c->plan_work,
                    c->hog_work};
    for (void* b : bufs)
        if (b) cudaFree(b);
    c->u = c->v = c->w = c->freq = nullptr;
    c->iu = c->iv = c->coff = nullptr;
    c->table = nullptr;
    c->data = c->model_vis = c->ones = c->grid = c->uv_psf = c->uv_data = nullptr;
    c->psf = c->dirty = c->residual = c->model = nullptr;
    c->plan_work = c->hog_work = nullptr;
    for (cudaEvent_t e : c->events) cudaEventDestroy(e);
    c->events.clear();
    c->stage_used.clear();
    c->cycles = 0;
    c->initialized = false;
}

// event pair index of (cycle, stage): start = events[base + stage], end = events[base + stage + 1]
tcv_status stage_event(tcv_major_ctx* c, int cycle, int k, cudaEvent_t* out)
{
    const size_t need = size_t(cycle + 1) * (TCV_MAJOR_STAGES + 1);
    while (c->events.size() < need) {
        cudaEvent_t e;
        TCV_CUDA(cudaEventCreate(&e));
        c->events.push_back(e);
    }
    if (c->stage_used.size() < size_t(cycle + 1)) c->stage_used.resize(size_t(cycle + 1), 0);
    *out = c->events[size_t(cycle) * (TCV_MAJOR_STAGES + 1) + size_t(k)];
    return TCV_OK;
}

}  // namespace

extern "C" {

void tcv_major_config_default(tcv_major_config* cfg)
{
    if (!cfg) return;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->n_samples = 160000;  // tMajorACC.cc:893-896, 923-930
    cfg->w_size = 33;
    cfg->n_chan = 1;
    cfg->cell_size = 5.0;
    cfg->g_size = 4096;
    cfg->baseline = 2000;
    cfg->n_major = 5;
    cfg->n_minor = 100;
    cfg->gain = 0.1f;  // tMajorACC.cc:793
    cfg->n_sources = 100;  // :1012
    cfg->device = 0;
    cfg->keep_stages = 0;
    cfg->tuning = tcv_tuning{16, 64, 0, 64};
}

tcv_status tcv_major_create(const tcv_major_config* cfg, tcv_major_ctx** out)
{
    if (!cfg || !out || cfg->n_samples < 1 || cfg->w_size < 1 || cfg->n_chan < 1 || !(cfg->cell_size > 0.0) ||
        cfg->g_size < 2 || cfg->n_minor < 0 || cfg->n_sources < 0)
        return TCV_ERR_ARG;
    if (cfg->g_size % 2) return TCV_ERR_UNSUPPORTED;  // the FFT steps need an even size (tMajorACC.cc:496)
    tcv_major_ctx* c = new (std::nothrow) tcv_major_ctx{};
    if (!c) return TCV_ERR_OOM;
    c->cfg = *cfg;
    cudaError_t e = cudaSetDevice(cfg->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete c;
        return cuda_status(e);
    }
    *out = c;
    return TCV_OK;
}

void tcv_major_destroy(tcv_major_ctx* c)
{
    if (!c) return;
    cudaSetDevice(c->cfg.device);
    release(c);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

const char* tcv_major_last_error(const tcv_major_ctx* c) { return c ? c->err.c_str() : "null context"; }
void* tcv_major_get_stream(const tcv_major_ctx* c) { return c ? static_cast<void*>(c->stream) : nullptr; }

tcv_status tcv_major_init(tcv_major_ctx* c)
{
    if (!c) return TCV_ERR_ARG;
    MAJ_CUDA(c, cudaSetDevice(c->cfg.device));
    release(c);
    const tcv_major_config& g = c->cfg;
    const int64_t ns = g.n_samples;
    c->n = ns * g.n_chan;
    const int N = g.g_size;
    const size_t g2 = size_t(N) * N;
    // inverse wavelengths (tMajorACC.cc:945-950)
    std::vector<double> freq(size_t(g.n_chan));
    for (int i = 0; i < g.n_chan; ++i) freq[size_t(i)] = (1.4e9 - 2.0e5 * double(i) / double(g.n_chan)) / 2.998e8;
    MAJ_TRY(c, tcv_c_geometry(freq[0], g.cell_size, g.baseline, g.w_size, &c->support, &c->over_sample, &c->w_cell_size,
                              &c->c_len));
    if (c->c_len > INT32_MAX) return mfail(c, TCV_ERR_UNSUPPORTED, "table larger than a 32-bit cOffset");
    // 1 / nVis as fftFix receives it: double 1.0 / float(n), rounded to float (:1188)
    c->scale = float(1.0 / double(float(c->n)));
    MAJ_CUDA(c, cudaMalloc(&c->u, size_t(ns) * 8));
    MAJ_CUDA(c, cudaMalloc(&c->v, size_t(ns) * 8));
    MAJ_CUDA(c, cudaMalloc(&c->w, size_t(ns) * 8));
    MAJ_CUDA(c, cudaMalloc(&c->freq, freq.size() * 8));
    MAJ_CUDA(c, cudaMalloc(&c->iu, size_t(c->n) * 4));
    MAJ_CUDA(c, cudaMalloc(&c->iv, size_t(c->n) * 4));
    MAJ_CUDA(c, cudaMalloc(&c->coff, size_t(c->n) * 4));
    MAJ_CUDA(c, cudaMalloc(&c->table, size_t(c->c_len) * 4));
    MAJ_CUDA(c, cudaMalloc(&c->data, size_t(c->n) * 8));
    MAJ_CUDA(c, cudaMalloc(&c->model_vis, size_t(c->n) * 8));
    MAJ_CUDA(c, cudaMalloc(&c->ones, size_t(c->n) * 8));
    MAJ_CUDA(c, cudaMalloc(&c->grid, g2 * 8));
    MAJ_CUDA(c, cudaMalloc(&c->psf, g2 * 4));
    MAJ_CUDA(c, cudaMalloc(&c->dirty, g2 * 4));
    MAJ_CUDA(c, cudaMalloc(&c->residual, g2 * 4));
    MAJ_CUDA(c, cudaMalloc(&c->model, g2 * 4));
    if (g.keep_stages) {
        MAJ_CUDA(c, cudaMalloc(&c->uv_psf, g2 * 8));
        MAJ_CUDA(c, cudaMalloc(&c->uv_data, g2 * 8));
    }
    cudaStream_t st = c->stream;
    // u, v, w: three draws per sample from state 1 (:933-940)
    MAJ_TRY(c, tcv_init_uvw_raw(ns, g.baseline, 1, c->u, c->v, c->w, st));
    {
        uint64_t A, C;
        lcg_jump(uint64_t(3) * uint64_t(ns), A, C);
        c->next = A * 1 + C;
    }
    MAJ_CUDA(c, cudaMemcpyAsync(c->freq, freq.data(), freq.size() * 8, cudaMemcpyHostToDevice, st));
    const int64_t s = 2 * int64_t(c->support) + 1;
    delta_table_kernel<<<nblk(c->c_len), 256, 0, st>>>(c->table, c->c_len, s * s);
    MAJ_CUDA(c, cudaGetLastError());
    MAJ_TRY(c, tcv_init_offsets_raw(c->u, c->v, c->w, ns, c->freq, g.n_chan, g.cell_size, c->w_cell_size, g.w_size, N,
                                    c->support, c->over_sample, c->iu, c->iv, c->coff, st));
    fill_kernel<<<nblk(c->n), 256, 0, st>>>(c->ones, c->n, make_float2(1.f, 0.f));
    MAJ_CUDA(c, cudaGetLastError());
    MAJ_CUDA(c, cudaMemsetAsync(c->model_vis, 0, size_t(c->n) * 8, st));
    // the plan: one binning for every pass
    c->plan_bytes = tcv_plan_workspace_bytes_tuned(c->n, c->support, N, c->c_len, &g.tuning);
    if (c->plan_bytes == 0) return mfail(c, TCV_ERR_UNSUPPORTED, "plan geometry");
    MAJ_CUDA(c, cudaMalloc(&c->plan_work, c->plan_bytes));
    MAJ_TRY(c, tcv::fft_prepare(N));  // the transforms' twiddle table, made here rather than mid-cycle
    MAJ_TRY(c, tcv_plan_build_tuned(&c->plan, c->iu, c->iv, c->coff, c->n, c->support, N, c->c_len, &g.tuning,
                                    c->plan_work, c->plan_bytes, st));
    int64_t rej = 0;
    MAJ_TRY(c, tcv_plan_rejected(c->plan, &rej, st));
    if (rej > 0) {
        c->err = std::to_string(rej) + " sample(s) fall outside the grid or the table";
        return TCV_ERR_BOUNDS;
    }
    c->hog_bytes = tcv_hogbom_workspace_bytes(N);
    MAJ_CUDA(c, cudaMalloc(&c->hog_work, c->hog_bytes));
    // the true sky (:1012-1020): draws continue after the samples'
    {
        const unsigned int maxint = unsigned(std::numeric_limits<int>::max());
        uint64_t nx = c->next;
        auto draw = [&]() -> int {
            nx = nx * kLcgA + kLcgC;
            return int((unsigned int)(nx / 65536) % maxint);
        };
        std::vector<int64_t> idx(size_t(g.n_sources));
        std::vector<float> val(size_t(g.n_sources));
        for (int i = 0; i < g.n_sources; ++i) {
            const int l = int(N * double(draw()) / double(maxint));
            const int m = int(N * double(draw()) / double(maxint));
            // std::complex<float>(randomInt()) / std::complex<float>(maxint): float(r) / 2^31, exact
            val[size_t(i)] = float(draw()) / float(maxint);
            idx[size_t(i)] = int64_t(m) * N + l;
        }
        c->next = nx;
        MAJ_CUDA(c, cudaMemsetAsync(c->grid, 0, g2 * 8, st));
        if (g.n_sources > 0) {
            int64_t* d_idx = nullptr;
            float* d_val = nullptr;
            cudaError_t e = cudaMalloc(&d_idx, idx.size() * 8);
            if (e == cudaSuccess) e = cudaMalloc(&d_val, val.size() * 4);
            if (e == cudaSuccess) e = cudaMemcpyAsync(d_idx, idx.data(), idx.size() * 8, cudaMemcpyHostToDevice, st);
            if (e == cudaSuccess) e = cudaMemcpyAsync(d_val, val.data(), val.size() * 4, cudaMemcpyHostToDevice, st);
            if (e == cudaSuccess) {
                sky_kernel<<<1, 32, 0, st>>>(c->grid, d_idx, d_val, g.n_sources);
                e = cudaGetLastError();
            }
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            cudaFree(d_idx);
            cudaFree(d_val);
            MAJ_CUDA(c, e);
        }
    }
    // FFT to the true uv grid (:1023) and degrid the true visibilities (:1032)
    MAJ_TRY(c, fft_exec(c->grid, N, true, st));
    MAJ_TRY(c, tcv_plan_degrid(c->plan, reinterpret_cast<const float*>(c->grid), c->table, TCV_C_R32, 1.f,
                               reinterpret_cast<float*>(c->data), st));
    MAJ_CUDA(c, cudaStreamSynchronize(st));
    c->initialized = true;
    return TCV_OK;
}

tcv_status tcv_major_run_cycle(tcv_major_ctx* c)
{
    if (!c) return TCV_ERR_ARG;
    if (!c->initialized) return mfail(c, TCV_ERR_STATE, "run_cycle before init");
    MAJ_CUDA(c, cudaSetDevice(c->cfg.device));
    const int N = c->cfg.g_size;
    const size_t g2 = size_t(N) * N;
    cudaStream_t st = c->stream;
    const int cyc = c->cycles;
    cudaEvent_t ev;
    auto mark = [&](int k) -> tcv_status {
        TCV_CHECK(stage_event(c, cyc, k, &ev));
        TCV_CUDA(cudaEventRecord(ev, st));
        return TCV_OK;
    };
    auto stage = [&](int k) -> tcv_status {  // start of stage k (its end is the next stage's start)
        TCV_CHECK(mark(k));
        c->stage_used[size_t(cyc)] |= 1 << k;
        return TCV_OK;
    };
    if (cyc == 0) {
        // gridding of the PSF (:1238-1253) and its image (:1262-1276)
        MAJ_TRY(c, stage(TCV_MAJOR_PSF_GRID));
        MAJ_CUDA(c, cudaMemsetAsync(c->grid, 0, g2 * 8, st));
        MAJ_TRY(c, tcv_plan_grid(c->plan, reinterpret_cast<const float*>(c->ones), c->table, TCV_C_R32, 1.f,
                                 reinterpret_cast<float*>(c->grid), st));
        MAJ_TRY(c, stage(TCV_MAJOR_PSF_IFFT));
        if (c->uv_psf) MAJ_CUDA(c, cudaMemcpyAsync(c->uv_psf, c->grid, g2 * 8, cudaMemcpyDeviceToDevice, st));
        MAJ_TRY(c, image_from_grid(c->grid, N, c->scale, c->psf, nullptr, st));
    }
    // gridding of the data (:1254-1270)
    MAJ_TRY(c, stage(TCV_MAJOR_GRID));
    MAJ_CUDA(c, cudaMemsetAsync(c->grid, 0, g2 * 8, st));
    MAJ_TRY(c, tcv_plan_grid(c->plan, reinterpret_cast<const float*>(c->data), c->table, TCV_C_R32, 1.f,
                             reinterpret_cast<float*>(c->grid), st));
    // dirty image (:1280-1297)
    MAJ_TRY(c, stage(TCV_MAJOR_IFFT));
    if (c->uv_data) MAJ_CUDA(c, cudaMemcpyAsync(c->uv_data, c->grid, g2 * 8, cudaMemcpyDeviceToDevice, st));
    MAJ_TRY(c, image_from_grid(c->grid, N, c->scale, c->dirty, nullptr, st));
    // Hogbom CLEAN into a fresh model (:1299-1313)
    MAJ_TRY(c, stage(TCV_MAJOR_HOGBOM));
    MAJ_CUDA(c, cudaMemsetAsync(c->model, 0, g2 * 4, st));
    MAJ_TRY(c, tcv_hogbom_deconvolve(c->dirty, N, c->psf, N, c->model, c->residual, c->cfg.n_minor, c->cfg.gain, 0.f,
                                     nullptr, nullptr, c->hog_work, c->hog_bytes, st));
    // forward FFT of the model (:1319-1338)
    MAJ_TRY(c, stage(TCV_MAJOR_FFT));
    MAJ_TRY(c, grid_from_image(c->model, N, c->grid, st));
    // degridding of the model (:1340-1348)
    MAJ_TRY(c, stage(TCV_MAJOR_DEGRID));
    MAJ_TRY(c, tcv_plan_degrid(c->plan, reinterpret_cast<const float*>(c->grid), c->table, TCV_C_R32, 1.f,
                               reinterpret_cast<float*>(c->model_vis), st));
    // data -= model (:1593-1596)
    MAJ_TRY(c, stage(TCV_MAJOR_SUBTRACT));
    subtract_kernel<<<nblk(c->n), 256, 0, st>>>(c->data, c->model_vis, c->n);
    MAJ_CUDA(c, cudaGetLastError());
    MAJ_TRY(c, mark(TCV_MAJOR_STAGES));
    c->cycles = cyc + 1;
    return TCV_OK;
}

tcv_status tcv_major_sync(tcv_major_ctx* c)
{
    if (!c) return TCV_ERR_ARG;
    MAJ_CUDA(c, cudaStreamSynchronize(c->stream));
    return TCV_OK;
}

tcv_status tcv_major_stage_ms(tcv_major_ctx* c, double* ms, int* cycles)
{
    if (!c || !ms) return TCV_ERR_ARG;
    MAJ_CUDA(c, cudaStreamSynchronize(c->stream));
    for (int k = 0; k < TCV_MAJOR_STAGES; ++k) ms[k] = 0.0;
    for (int cyc = 0; cyc < c->cycles; ++cyc) {
        const size_t base = size_t(cyc) * (TCV_MAJOR_STAGES + 1);
        const int used = c->stage_used[size_t(cyc)];
        for (int k = 0; k < TCV_MAJOR_STAGES; ++k) {
            if (!(used & (1 << k))) continue;
            int nxt = k + 1;  // the end of stage k: the next recorded stage's start, or the cycle end
            while (nxt < TCV_MAJOR_STAGES && !(used & (1 << nxt))) ++nxt;
            float m = 0.f;
            MAJ_CUDA(c, cudaEventElapsedTime(&m, c->events[base + size_t(k)], c->events[base + size_t(nxt)]));
            ms[k] += m;
        }
    }
    if (cycles) *cycles = c->cycles;
    return TCV_OK;
}

tcv_status tcv_major_info(const tcv_major_ctx* c, int* support, int64_t* n_vis, int64_t* c_len, float* scale)
{
    if (!c) return TCV_ERR_ARG;
    if (support) *support = c->support;
    if (n_vis) *n_vis = c->n;
    if (c_len) *c_len = c->c_len;
    if (scale) *scale = c->scale;
    return TCV_OK;
}

static tcv_status major_copy(tcv_major_ctx* c, void* dst, const void* src, size_t bytes)
{
    if (!c || !dst) return TCV_ERR_ARG;
    if (!c->initialized) return mfail(c, TCV_ERR_STATE, "copy before init");
    if (!src) return mfail(c, TCV_ERR_STATE, "not kept (keep_stages = 0)");
    MAJ_CUDA(c, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream));
    MAJ_CUDA(c, cudaStreamSynchronize(c->stream));
    return TCV_OK;
}

tcv_status tcv_major_get_image(tcv_major_ctx* c, int which, float* out)
{
    if (!c) return TCV_ERR_ARG;
    const size_t b = size_t(c->cfg.g_size) * c->cfg.g_size * 4;
    const float* src[] = {c->psf, c->dirty, c->residual, c->model};
    if (which < 0 || which > 3) return TCV_ERR_ARG;
    return major_copy(c, out, src[which], b);
}

tcv_status tcv_major_get_grid(tcv_major_ctx* c, int which, float* out)
{
    if (!c) return TCV_ERR_ARG;
    const size_t b = size_t(c->cfg.g_size) * c->cfg.g_size * 8;
    const float2* src[] = {c->uv_psf, c->uv_data, c->grid};
    if (which < 0 || which > 2) return TCV_ERR_ARG;
    return major_copy(c, out, src[which], b);
}

tcv_status tcv_major_get_vis(tcv_major_ctx* c, int which, float* out)
{
    if (!c) return TCV_ERR_ARG;
    const float2* src[] = {c->data, c->model_vis};
    if (which < 0 || which > 1) return TCV_ERR_ARG;
    return major_copy(c, out, src[which], size_t(c->n) * 8);
}

tcv_status tcv_major_get_offsets(tcv_major_ctx* c, int32_t* iu, int32_t* iv, int32_t* coff)
{
    if (!c || !iu || !iv || !coff) return TCV_ERR_ARG;
    MAJ_TRY(c, major_copy(c, iu, c->iu, size_t(c->n) * 4));
    MAJ_TRY(c, major_copy(c, iv, c->iv, size_t(c->n) * 4));
    return major_copy(c, coff, c->coff, size_t(c->n) * 4);
}

}  // extern "C"
