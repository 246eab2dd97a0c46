// tcv_api.cu -- the context API: the reference's Benchmark object (attic/tConvolveMPI/Benchmark.h:55-99)
// with all of its buffers resident on one GPU, built on the raw entry points.
#include "tcv_internal.cuh"

#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

struct tcv_ctx {
    tcv_config cfg{};
    int support = 0, over_sample = 0;
    double w_cell_size = 0.0;
    int64_t c_len = 0, n_data = 0;
    float sum_c = 0.f;
    cudaStream_t own_stream = nullptr, stream = nullptr;
    double *u = nullptr, *v = nullptr, *w = nullptr, *freq = nullptr;
    float2 *data = nullptr, *outdata = nullptr, *grid = nullptr, *c64 = nullptr;
    void* c_alt = nullptr;      // active form, reference layout (when not complex64)
    int c_alt_type = -1;
    float c_alt_scale = 1.f;
    void* c_pad = nullptr;      // active form, prepared layout (padded or paired) for the active path
    int c_pad_type = -1;        // storage type | layout flag of c_pad
    float c_pad_scale = 1.f;
    int c_type = TCV_C_C64;     // active storage form
    int path = TCV_PATH_DIRECT;
    int32_t *iu = nullptr, *iv = nullptr, *coff = nullptr;
    void* work = nullptr;
    size_t work_bytes = 0;
    void* c_scratch = nullptr;
    tcv_plan* plan = nullptr;
    tcv_tuning tuning{16, 32, 0, 0};
    bool initialized = false;
    std::string err;
};

namespace {

tcv_status fail(tcv_ctx* c, tcv_status s, const std::string& what)
{
    if (c) c->err = what + ": " + tcv_status_string(s);
    return s;
}

tcv_status cuda_fail(tcv_ctx* c, cudaError_t e, const char* what)
{
    if (c) c->err = std::string(what) + ": " + cudaGetErrorString(e);
    return tcv::cuda_status(e);
}

#define CTX_CUDA(ctx, call)                                       \
    do {                                                          \
        cudaError_t _e = (call);                                  \
        if (_e != cudaSuccess) return cuda_fail(ctx, _e, #call);  \
    } while (0)

#define CTX_TRY(ctx, call)                                 \
    do {                                                   \
        tcv_status _s = (call);                            \
        if (_s != TCV_OK) return fail(ctx, _s, #call);     \
    } while (0)

__global__ void fill_kernel(float2* p, int64_t n, float2 v)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = v;
}

template <typename T>
cudaError_t dalloc(T** p, size_t count)
{
    return cudaMalloc(reinterpret_cast<void**>(p), count * sizeof(T) + 16);
}

// table, type code (with the layout flag) and scale the kernels are given
int layout_flag(int path) { return path == TCV_PATH_TMA ? TCV_C_PADDED : (path == TCV_PATH_PAIRED ? TCV_C_PAIRED : 0); }
const void* active_table(const tcv_ctx* c)
{
    if (c->path != TCV_PATH_DIRECT) return c->c_pad;
    return c->c_type == TCV_C_C64 ? static_cast<const void*>(c->c64) : c->c_alt;
}
int active_code(const tcv_ctx* c) { return c->c_type | layout_flag(c->path); }
float active_scale(const tcv_ctx* c)
{
    if (c->path != TCV_PATH_DIRECT) return c->c_pad_scale;
    return c->c_type == TCV_C_C64 ? 1.f : c->c_alt_scale;
}

// make sure the table of the active form exists in the layout the active path needs
tcv_status ensure_tables(tcv_ctx* c)
{
    const int t = c->c_type;
    if (c->path != TCV_PATH_DIRECT) {
        const int want = t | layout_flag(c->path);
        if (c->c_pad_type == want) return TCV_OK;
        if (c->c_pad) {
            CTX_CUDA(c, cudaStreamSynchronize(c->stream));
            cudaFree(c->c_pad);
            c->c_pad = nullptr;
            c->c_pad_type = -1;
        }
        const size_t bytes = tcv_table_bytes(c->c_len, c->support, want);
        if (!bytes) return fail(c, TCV_ERR_UNSUPPORTED, "table shape has no prepared layout");
        CTX_CUDA(c, cudaMalloc(&c->c_pad, bytes));
        int64_t nz = 0;
        CTX_TRY(c, tcv_prepare_table(reinterpret_cast<const float*>(c->c64), c->c_len, c->support, want, c->c_pad,
                                     &c->c_pad_scale, &nz, c->stream));
        const bool real_form = t == TCV_C_R32 || t == TCV_C_RBF16 || t == TCV_C_RF16;
        if (real_form && nz > 0) return fail(c, TCV_ERR_ARG, "real table form requested for a table with imaginary parts");
        c->c_pad_type = want;
        return TCV_OK;
    }
    tcv::jit_prepare(t, 2 * c->support + 1, c->tuning.tile_rows);  // the direct path's tile kernels, specialised on sSize
    if (t == TCV_C_C64 || c->c_alt_type == t) return TCV_OK;
    if (c->c_alt) {
        CTX_CUDA(c, cudaStreamSynchronize(c->stream));
        cudaFree(c->c_alt);
        c->c_alt = nullptr;
        c->c_alt_type = -1;
    }
    CTX_CUDA(c, cudaMalloc(&c->c_alt, size_t(c->c_len) * tcv_ctype_bytes(t) + 16));
    int64_t nz = 0;
    CTX_TRY(c, tcv_convert_c(reinterpret_cast<const float*>(c->c64), c->c_len, t, c->c_alt, &c->c_alt_scale, &nz,
                             c->stream));
    const bool real_form = t == TCV_C_R32 || t == TCV_C_RBF16 || t == TCV_C_RF16;
    if (real_form && nz > 0) return fail(c, TCV_ERR_ARG, "real table form requested for a table with imaginary parts");
    c->c_alt_type = t;
    return TCV_OK;
}

tcv_status rebuild_plan(tcv_ctx* c)
{
    if (c->plan) {
        tcv_plan_destroy(c->plan);
        c->plan = nullptr;
    }
    const size_t need = tcv_plan_workspace_bytes_tuned(c->n_data, c->support, c->cfg.g_size, c->c_len, &c->tuning);
    if (need > c->work_bytes) {
        CTX_CUDA(c, cudaStreamSynchronize(c->stream));
        cudaFree(c->work);
        c->work = nullptr;
        c->work_bytes = 0;
        CTX_CUDA(c, cudaMalloc(&c->work, need));
        c->work_bytes = need;
    }
    CTX_TRY(c, tcv_plan_build_tuned(&c->plan, c->iu, c->iv, c->coff, c->n_data, c->support, c->cfg.g_size,
                                    c->c_len, &c->tuning, c->work, c->work_bytes, c->stream));
    int64_t rej = 0;
    CTX_TRY(c, tcv_plan_rejected(c->plan, &rej, c->stream));
    if (rej > 0) {
        c->err = std::to_string(rej) + " sample(s) fall outside the grid or the table and are skipped";
        return TCV_ERR_BOUNDS;
    }
    return TCV_OK;
}

}  // namespace

extern "C" {

const char* tcv_status_string(tcv_status s)
{
    switch (s) {
        case TCV_OK: return "ok";
        case TCV_ERR_ARG: return "invalid argument";
        case TCV_ERR_BOUNDS: return "sample outside grid or table";
        case TCV_ERR_OOM: return "device out of memory";
        case TCV_ERR_CUDA: return "CUDA error";
        case TCV_ERR_TIMEOUT: return "device wait timed out";
        case TCV_ERR_STATE: return "call out of order";
        case TCV_ERR_WORKSPACE: return "workspace too small";
        case TCV_ERR_UNSUPPORTED: return "unsupported shape";
        default: return "unknown status";
    }
}

const char* tcv_version(void) { return "tconvolve-b200 1.0 sm_100a"; }

void tcv_config_default(tcv_config* cfg)
{
    if (!cfg) return;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->n_samples = 160000;  // attic/tConvolveMPI/Benchmark.h:39-46
    cfg->w_size = 33;
    cfg->n_chan = 1;
    cfg->g_size = 4096;
    cfg->baseline = 2000;
    cfg->cell_size = 5.0;
    cfg->seed = 0;
    cfg->c_type = TCV_C_C64;
    cfg->device = 0;
}

void tcv_destroy(tcv_ctx* c)
{
    if (!c) return;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaSetDevice(c->cfg.device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->plan) tcv_plan_destroy(c->plan);
    void* bufs[] = {c->u, c->v, c->w, c->freq, c->data, c->outdata, c->grid, c->c64, c->c_alt,
                    c->c_pad, c->iu, c->iv, c->coff, c->work, c->c_scratch};
    for (void* b : bufs)
        if (b) cudaFree(b);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    cudaSetDevice(dev);
    delete c;
}

tcv_status tcv_create(const tcv_config* cfg, tcv_ctx** out)
{
    if (!cfg || !out) return TCV_ERR_ARG;
    *out = nullptr;
    if (cfg->n_samples < 1 || cfg->n_chan < 1 || cfg->w_size < 1 || cfg->g_size < 2 ||
        cfg->g_size > 32768 || !(cfg->cell_size > 0.0) || tcv_ctype_bytes(cfg->c_type) == 0)
        return TCV_ERR_ARG;
    tcv_ctx* c = new (std::nothrow) tcv_ctx;
    if (!c) return TCV_ERR_OOM;
    c->cfg = *cfg;
    c->n_data = cfg->n_samples * cfg->n_chan;
    const double freq0 = 1.4e9 / 2.998e8;  // Benchmark.cc:89 with chan = 0
    tcv_status st = tcv_c_geometry(freq0, cfg->cell_size, cfg->baseline, cfg->w_size, &c->support,
                                   &c->over_sample, &c->w_cell_size, &c->c_len);
    if (st != TCV_OK || c->c_len > INT32_MAX) {
        delete c;
        return st != TCV_OK ? st : TCV_ERR_UNSUPPORTED;
    }
    cudaError_t e = cudaSetDevice(cfg->device);
    const size_t g2 = size_t(cfg->g_size) * cfg->g_size;
    c->work_bytes = tcv_plan_workspace_bytes(c->n_data, c->support, cfg->g_size, c->c_len);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
    c->stream = c->own_stream;
    if (e == cudaSuccess) e = dalloc(&c->u, cfg->n_samples);
    if (e == cudaSuccess) e = dalloc(&c->v, cfg->n_samples);
    if (e == cudaSuccess) e = dalloc(&c->w, cfg->n_samples);
    if (e == cudaSuccess) e = dalloc(&c->freq, cfg->n_chan);
    if (e == cudaSuccess) e = dalloc(&c->data, c->n_data);
    if (e == cudaSuccess) e = dalloc(&c->outdata, c->n_data);
    if (e == cudaSuccess) e = dalloc(&c->grid, g2);
    if (e == cudaSuccess) e = dalloc(&c->c64, c->c_len);
    if (e == cudaSuccess) e = dalloc(&c->iu, c->n_data);
    if (e == cudaSuccess) e = dalloc(&c->iv, c->n_data);
    if (e == cudaSuccess) e = dalloc(&c->coff, c->n_data);
    if (e == cudaSuccess) e = cudaMalloc(&c->work, c->work_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&c->c_scratch, tcv_init_c_scratch_bytes());
    if (e != cudaSuccess) {
        const tcv_status s = tcv::cuda_status(e);
        tcv_destroy(c);
        return s;
    }
    *out = c;
    return TCV_OK;
}

const char* tcv_last_error(const tcv_ctx* c) { return c ? c->err.c_str() : "null context"; }

tcv_status tcv_set_stream(tcv_ctx* c, void* stream)
{
    if (!c) return TCV_ERR_ARG;
    CTX_CUDA(c, cudaStreamSynchronize(c->stream));
    c->stream = stream ? static_cast<cudaStream_t>(stream) : c->own_stream;
    return TCV_OK;
}

void* tcv_get_stream(const tcv_ctx* c) { return c ? static_cast<void*>(c->stream) : nullptr; }

tcv_status tcv_sync(tcv_ctx* c)
{
    if (!c) return TCV_ERR_ARG;
    CTX_CUDA(c, cudaStreamSynchronize(c->stream));
    if (c->plan) CTX_TRY(c, tcv_plan_status(c->plan, c->stream));
    return TCV_OK;
}

tcv_status tcv_init(tcv_ctx* c)
{
    if (!c) return TCV_ERR_ARG;
    CTX_CUDA(c, cudaSetDevice(c->cfg.device));
    const tcv_config& cfg = c->cfg;
    // Benchmark::init (attic/tConvolveMPI/Benchmark.cc:60-96)
    CTX_TRY(c, tcv_init_uvw_raw(cfg.n_samples, cfg.baseline, cfg.seed + 1, c->u, c->v, c->w, c->stream));
    fill_kernel<<<256, 256, 0, c->stream>>>(c->data, c->n_data, make_float2(1.f, 0.f));
    CTX_CUDA(c, cudaGetLastError());
    CTX_CUDA(c, cudaMemsetAsync(c->outdata, 0, size_t(c->n_data) * sizeof(float2), c->stream));
    CTX_CUDA(c, cudaMemsetAsync(c->grid, 0, size_t(cfg.g_size) * cfg.g_size * sizeof(float2), c->stream));
    std::vector<double> freq(cfg.n_chan);
    for (int i = 0; i < cfg.n_chan; ++i) freq[i] = (1.4e9 - 2.0e5 * double(i) / double(cfg.n_chan)) / 2.998e8;
    CTX_CUDA(c, cudaMemcpyAsync(c->freq, freq.data(), freq.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CTX_TRY(c, tcv_init_c_raw(freq[0], cfg.cell_size, cfg.baseline, cfg.w_size, reinterpret_cast<float*>(c->c64),
                              c->c_scratch, &c->sum_c, c->stream));
    CTX_TRY(c, tcv_init_offsets_raw(c->u, c->v, c->w, cfg.n_samples, c->freq, cfg.n_chan, cfg.cell_size,
                                    c->w_cell_size, cfg.w_size, cfg.g_size, c->support, c->over_sample,
                                    c->iu, c->iv, c->coff, c->stream));
    c->initialized = true;
    c->c_alt_type = -1;
    c->c_pad_type = -1;
    c->c_type = cfg.c_type & 0xff;
    CTX_TRY(c, ensure_tables(c));
    return rebuild_plan(c);
}

tcv_status tcv_set_ctype(tcv_ctx* c, int c_type)
{
    if (!c || tcv_ctype_bytes(c_type) == 0 || (c_type & TCV_C_PADDED)) return TCV_ERR_ARG;
    if (!c->initialized) return fail(c, TCV_ERR_STATE, "set_ctype before init");
    const int prev = c->c_type;
    c->c_type = c_type;
    const tcv_status s = ensure_tables(c);
    if (s != TCV_OK) c->c_type = prev;
    return s;
}

tcv_status tcv_set_path(tcv_ctx* c, int path)
{
    if (!c || (path != TCV_PATH_TMA && path != TCV_PATH_DIRECT && path != TCV_PATH_PAIRED)) return TCV_ERR_ARG;
    const int prev = c->path;
    c->path = path;
    if (!c->initialized) return TCV_OK;
    const tcv_status s = ensure_tables(c);
    if (s != TCV_OK) c->path = prev;
    return s;
}

int tcv_get_path(const tcv_ctx* c) { return c ? c->path : -1; }

tcv_status tcv_set_tuning(tcv_ctx* c, const tcv_tuning* t)
{
    if (!c || !t) return TCV_ERR_ARG;
    const tcv_tuning nt{t->tile_rows ? t->tile_rows : 16, t->group_mib ? t->group_mib : 32, t->split,
                        t->degrid_split, t->kernel};
    // the sample-parallel kernel bits (1 gridding, 2 degridding) work on the 64 x 32 tiles of 8-row plans
    if ((nt.tile_rows != 8 && nt.tile_rows != 16 && nt.tile_rows != 32) || nt.group_mib < -1 || nt.split < 0 ||
        nt.degrid_split < 0 || nt.kernel < 0 || nt.kernel > 3 || (nt.kernel != 0 && nt.tile_rows != 8))
        return TCV_ERR_ARG;
    const tcv_tuning prev = c->tuning;
    c->tuning = nt;
    if (!c->initialized) return TCV_OK;
    tcv_status s = ensure_tables(c);
    if (s == TCV_OK) s = rebuild_plan(c);
    if (s != TCV_OK && s != TCV_ERR_BOUNDS) {
        c->tuning = prev;
        rebuild_plan(c);
    }
    return s;
}

tcv_status tcv_get_tuning(const tcv_ctx* c, tcv_tuning* out)
{
    if (!c || !out) return TCV_ERR_ARG;
    *out = c->tuning;
    return TCV_OK;
}

tcv_status tcv_tune(tcv_ctx* c, int reps, tcv_tuning* best_out, float* best_ms_out)
{
    if (!c || reps < 1) return TCV_ERR_ARG;
    if (!c->initialized) return fail(c, TCV_ERR_STATE, "tune before init");
    if (c->path != TCV_PATH_DIRECT) return fail(c, TCV_ERR_UNSUPPORTED, "tuning needs the direct path");
    const tcv_job job{c->n_data, c->cfg.g_size, reinterpret_cast<float*>(c->grid)};
    tcv_tuning best{16, 32, 0, 0};
    float ms = 0.f;
    CTX_TRY(c, tcv_autotune(&job, 1, c->iu, c->iv, c->coff, reinterpret_cast<const float*>(c->data), active_table(c),
                            active_code(c), active_scale(c), c->c_len, c->support, reps, &best, &ms, c->stream));
    const tcv_status s = tcv_set_tuning(c, &best);
    if (s != TCV_OK) return s;
    if (best_out) *best_out = best;
    if (best_ms_out) *best_ms_out = ms;
    return TCV_OK;
}

tcv_status tcv_run_grid(tcv_ctx* c)
{
    if (!c) return TCV_ERR_ARG;
    if (!c->initialized || !c->plan) return fail(c, TCV_ERR_STATE, "run_grid before init");
    CTX_TRY(c, tcv_plan_grid(c->plan, reinterpret_cast<const float*>(c->data), active_table(c), active_code(c),
                             active_scale(c), reinterpret_cast<float*>(c->grid), c->stream));
    return TCV_OK;
}

tcv_status tcv_run_degrid(tcv_ctx* c)
{
    if (!c) return TCV_ERR_ARG;
    if (!c->initialized || !c->plan) return fail(c, TCV_ERR_STATE, "run_degrid before init");
    CTX_TRY(c, tcv_plan_degrid(c->plan, reinterpret_cast<const float*>(c->grid), active_table(c), active_code(c),
                               active_scale(c), reinterpret_cast<float*>(c->outdata), c->stream));
    return TCV_OK;
}

int tcv_support(const tcv_ctx* c) { return c ? c->support : -1; }
int tcv_over_sample(const tcv_ctx* c) { return c ? c->over_sample : -1; }
double tcv_w_cell_size(const tcv_ctx* c) { return c ? c->w_cell_size : 0.0; }
float tcv_sum_c(const tcv_ctx* c) { return c ? c->sum_c : 0.f; }
int64_t tcv_c_len(const tcv_ctx* c) { return c ? c->c_len : 0; }
int64_t tcv_n_data(const tcv_ctx* c) { return c ? c->n_data : 0; }
double tcv_updates_per_pass(const tcv_ctx* c)
{
    if (!c) return 0.0;
    const double s = 2.0 * c->support + 1.0;
    return double(c->n_data) * s * s;
}

static tcv_status copy_sync(tcv_ctx* c, void* dst, const void* src, size_t bytes, cudaMemcpyKind k)
{
    if (!c || (bytes && (!dst || !src))) return TCV_ERR_ARG;
    CTX_CUDA(c, cudaMemcpyAsync(dst, src, bytes, k, c->stream));
    CTX_CUDA(c, cudaStreamSynchronize(c->stream));
    return TCV_OK;
}

tcv_status tcv_set_data(tcv_ctx* c, const float* vis, int64_t n)
{
    if (!c || n != c->n_data) return TCV_ERR_ARG;
    return copy_sync(c, c->data, vis, size_t(n) * 8, cudaMemcpyHostToDevice);
}
tcv_status tcv_get_data(tcv_ctx* c, float* vis, int64_t n)
{
    if (!c || n != c->n_data) return TCV_ERR_ARG;
    return copy_sync(c, vis, c->data, size_t(n) * 8, cudaMemcpyDeviceToHost);
}
tcv_status tcv_get_outdata(tcv_ctx* c, float* vis, int64_t n)
{
    if (!c || n != c->n_data) return TCV_ERR_ARG;
    return copy_sync(c, vis, c->outdata, size_t(n) * 8, cudaMemcpyDeviceToHost);
}
tcv_status tcv_set_grid(tcv_ctx* c, const float* grid)
{
    if (!c) return TCV_ERR_ARG;
    return copy_sync(c, c->grid, grid, size_t(c->cfg.g_size) * c->cfg.g_size * 8, cudaMemcpyHostToDevice);
}
tcv_status tcv_get_grid(tcv_ctx* c, float* grid)
{
    if (!c) return TCV_ERR_ARG;
    return copy_sync(c, grid, c->grid, size_t(c->cfg.g_size) * c->cfg.g_size * 8, cudaMemcpyDeviceToHost);
}
tcv_status tcv_zero_grid(tcv_ctx* c)
{
    if (!c) return TCV_ERR_ARG;
    CTX_CUDA(c, cudaMemsetAsync(c->grid, 0, size_t(c->cfg.g_size) * c->cfg.g_size * 8, c->stream));
    return TCV_OK;
}
tcv_status tcv_get_c(tcv_ctx* c, float* out, int64_t n_entries)
{
    if (!c || n_entries != c->c_len) return TCV_ERR_ARG;
    return copy_sync(c, out, c->c64, size_t(n_entries) * 8, cudaMemcpyDeviceToHost);
}
tcv_status tcv_get_offsets(tcv_ctx* c, int32_t* iu, int32_t* iv, int32_t* coff)
{
    if (!c) return TCV_ERR_ARG;
    const size_t b = size_t(c->n_data) * 4;
    tcv_status s = TCV_OK;
    if (iu && s == TCV_OK) s = copy_sync(c, iu, c->iu, b, cudaMemcpyDeviceToHost);
    if (iv && s == TCV_OK) s = copy_sync(c, iv, c->iv, b, cudaMemcpyDeviceToHost);
    if (coff && s == TCV_OK) s = copy_sync(c, coff, c->coff, b, cudaMemcpyDeviceToHost);
    return s;
}
tcv_status tcv_get_uvw(tcv_ctx* c, double* u, double* v, double* w)
{
    if (!c) return TCV_ERR_ARG;
    const size_t b = size_t(c->cfg.n_samples) * 8;
    tcv_status s = TCV_OK;
    if (u && s == TCV_OK) s = copy_sync(c, u, c->u, b, cudaMemcpyDeviceToHost);
    if (v && s == TCV_OK) s = copy_sync(c, v, c->v, b, cudaMemcpyDeviceToHost);
    if (w && s == TCV_OK) s = copy_sync(c, w, c->w, b, cudaMemcpyDeviceToHost);
    return s;
}
tcv_status tcv_set_uvw(tcv_ctx* c, const double* u, const double* v, const double* w)
{
    if (!c || !u || !v || !w) return TCV_ERR_ARG;
    if (!c->initialized) return fail(c, TCV_ERR_STATE, "set_uvw before init");
    const size_t b = size_t(c->cfg.n_samples) * 8;
    CTX_TRY(c, copy_sync(c, c->u, u, b, cudaMemcpyHostToDevice));
    CTX_TRY(c, copy_sync(c, c->v, v, b, cudaMemcpyHostToDevice));
    CTX_TRY(c, copy_sync(c, c->w, w, b, cudaMemcpyHostToDevice));
    const tcv_config& cfg = c->cfg;
    CTX_TRY(c, tcv_init_offsets_raw(c->u, c->v, c->w, cfg.n_samples, c->freq, cfg.n_chan, cfg.cell_size,
                                    c->w_cell_size, cfg.w_size, cfg.g_size, c->support, c->over_sample,
                                    c->iu, c->iv, c->coff, c->stream));
    return rebuild_plan(c);
}

tcv_status tcv_get_device_buffers(tcv_ctx* c, tcv_device_buffers* o)
{
    if (!c || !o) return TCV_ERR_ARG;
    o->data = reinterpret_cast<float*>(c->data);
    o->outdata = reinterpret_cast<float*>(c->outdata);
    o->grid = reinterpret_cast<float*>(c->grid);
    o->c64 = reinterpret_cast<float*>(c->c64);
    o->c_active = active_table(c);
    o->iu = c->iu;
    o->iv = c->iv;
    o->coff = c->coff;
    o->u = c->u;
    o->v = c->v;
    o->w = c->w;
    o->plan = c->plan;
    o->c_scale = active_scale(c);
    o->c_type = active_code(c);
    return TCV_OK;
}

}  // extern "C"
