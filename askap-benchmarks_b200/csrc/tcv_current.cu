// tcv_current.cu -- the variable-support benchmark of current/tConvolveMPI on the device: the run
// types' geometry, samples from the 36-antenna array over a 12 h track, the per-plane complex
// W-projection table, offsets with the w-plane of each sample, and the Benchmark object of that
// benchmark (current/tConvolveMPI/Benchmark.h:38-111) with its buffers resident on one GPU.
//
// Set-up follows current/tConvolveMPI/Benchmark.cc:61-311 and :471-655 operation by operation,
// keeping the reference's float (Real) and double (Coord) types: the geometry and the baselines
// are computed on the host exactly as there; the samples, the table and the offsets on the
// device with explicit IEEE roundings (no fused multiply-adds).  Where the reference calls
// float sinf/cosf on a float phase, the device rounds the double sin/cos of that phase to float
// (the correctly rounded value, which is what the reference's libm returns but for rare last-bit
// cases).  Gridding and degridding use variable-width plans (tcv_plan_build_var).
#include "tcv_internal.cuh"

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

namespace tcv {
namespace {

constexpr double kCurPi = 3.141593;  // the reference's constant
constexpr double kMaxIntD = 2147483647.0;
constexpr int kAntennas = 36;

// antenna positions in metres east and north (current/tConvolveMPI/Benchmark.cc:183-204)
const double kEast[kAntennas] = {
    -42.43847222,  -15.46047222,  -6.48847222,    -51.41747222,   -116.43047222, 93.22152778,
    200.42152778,  -80.24847222,  -286.64847222,  -138.75447222,  225.51252778,  353.48652778,
    396.28152778,  -67.29847222,  -782.13847222,  -678.55347222,  -539.25647222, -149.22347222,
    175.37552778,  463.88152778,  643.72952778,   803.40152778,   -43.14647222,  36.03352778,
    -656.05547222, -435.77447222, -1112.94147222, 207.32652778,   523.49152778,  1186.61752778,
    2178.51052778, 2982.48652778, -17.41247222,   -3017.44747222, -2213.43647222, -19.20647222};
const double kNorth[kAntennas] = {
    -105.22933333, -118.24033333, -97.73933333,   -70.22133333,  -73.72633333,  6.77066667,
    -215.20933333, -343.73933333, 5.32066667,     174.26666667,  235.30966667,  164.24666667,
    -469.23433333, -565.23833333, -263.22233333,  260.21066667,  417.28966667,  270.27966667,
    376.29066667,  209.79766667,  216.77666667,   230.75266667,  -762.23633333, -1083.75233333,
    548.27766667,  562.27366667,  835.74566667,   1093.28166667, 647.98066667,  693.23866667,
    887.75566667,  -2612.27533333, -2916.19433333, -2112.20733333, 887.76166667, 3084.83866667};

struct CurParams {
    float baseline;
    int over_sample, support, w_size, g_size;
    double w_cell, uv_cell;
};

// current/tConvolveMPI/Benchmark.cc:64-158: per run type, in the reference's float arithmetic
bool cur_params(int run_type, CurParams& p)
{
    const int aperture = 12;
    const float max_freq = 1.0e9f;
    const float lambda = float(2.998e8 / double(max_freq));
    float img_os = 0.f, img_ext = 0.f;
    p = CurParams{};
    if (run_type == 0 || run_type == 1) {
        p.baseline = run_type == 0 ? 6440.f : 2000.f;
        img_os = run_type == 0 ? 4.0f : 3.1f;
        img_ext = run_type == 0 ? 3.0f : 2.0f;
        p.over_sample = run_type == 0 ? 4 : 8;
        const float wmax = p.baseline / lambda;
        const float fov = lambda / float(aperture) * img_ext;
        const float w_part = wmax * fov * fov;
        const float a_part = 7.f;
        p.support = int(std::ceil(std::sqrt(a_part * a_part + w_part * w_part))) / 2;
        p.w_size = int(std::ceil(float(p.over_sample) * w_part));
        p.w_size += (p.w_size + 1) % 2;  // odd
        p.w_cell = double(2.f * wmax / float(p.w_size - 1));
    } else if (run_type == 2) {  // nearest neighbour
        p.baseline = 6440.f;
        img_os = 2.0f;
        img_ext = 1.0f;
        p.over_sample = 1;
        p.support = 0;
        p.w_size = 1;
    } else if (run_type == 3 || run_type == 4) {  // 7x7 / 87x87 kernels, no w-projection
        p.baseline = 6440.f;
        img_os = 4.0f;
        img_ext = 1.923f;
        p.over_sample = run_type == 3 ? 128 : 8;
        p.support = run_type == 3 ? 3 : 43;
        p.w_size = 1;
    } else {
        return false;
    }
    p.g_size = int(std::ceil(p.baseline / float(aperture) * img_os * img_ext));
    p.uv_cell = double(p.baseline / lambda * img_os / float(p.g_size));
    return true;
}

// current/tConvolveMPI/Benchmark.cc:164-228: the baselines no longer than the run's baseline
int cur_baselines(float baseline, std::vector<double>& bx, std::vector<double>& by, std::vector<double>& bz)
{
    const double lat = -26.6970 * kCurPi / 180.0;
    double x[kAntennas], y[kAntennas], z[kAntennas];
    for (int i = 0; i < kAntennas; ++i) {
        x[i] = -kNorth[i] * std::sin(lat);
        y[i] = kEast[i];
        z[i] = kNorth[i] * std::cos(lat);
    }
    const double lim = double(baseline * baseline);
    bx.clear();
    by.clear();
    bz.clear();
    for (int i = 0; i < kAntennas - 1; ++i)
        for (int j = i + 1; j < kAntennas; ++j) {
            const double dx = x[i] - x[j], dy = y[i] - y[j], dz = z[i] - z[j];
            if (dx * dx + dy * dy + dz * dz > lim) continue;
            bx.push_back(dx);
            by.push_back(dy);
            bz.push_back(dz);
        }
    return int(bx.size());
}

// per-plane widths and offsets (current/tConvolveMPI/Benchmark.cc:491-515)
int64_t cur_planes(const CurParams& p, std::vector<int32_t>& s_size, std::vector<int32_t>& c_off0)
{
    s_size.assign(size_t(p.w_size), 2 * p.support + 1);
    c_off0.assign(size_t(p.w_size), 0);
    int64_t offset = 0;
    for (int k = 0; k < p.w_size; ++k) {
        if (p.w_size > 1) {
            const int wind = k - p.w_size / 2;
            const double w = wind * p.w_cell;
            const float w_part = float(w / p.uv_cell / p.uv_cell);
            const float a_part = 7.f;
            int s = int(std::ceil(std::sqrt(a_part * a_part + w_part * w_part)));
            s += (s + 1) % 2;
            s_size[size_t(k)] = s;
        }
        c_off0[size_t(k)] = int32_t(offset);
        offset += int64_t(s_size[size_t(k)]) * s_size[size_t(k)] * p.over_sample * p.over_sample;
    }
    return offset;
}

constexpr int kScans = int(12. * 3600. / 5.);  // obslen / scanlen (Benchmark.cc:64-66)

// Benchmark.cc:246-262: draws 2i and 2i+1 give sample i's baseline and hour angle
__global__ void cur_uvw_kernel(int64_t n, int nb, uint64_t state0, const double* __restrict__ bx,
                               const double* __restrict__ by, const double* __restrict__ bz, double cdec,
                               double sdec, double* u, double* v, double* w)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint64_t A, C;
    lcg_jump(2ull * uint64_t(i), A, C);
    uint64_t s = A * state0 + C;
    s = s * kLcgA + kLcgC;
    const unsigned int r1 = (unsigned int)(s / 65536ull) % 2147483647u;
    s = s * kLcgA + kLcgC;
    const unsigned int r2 = (unsigned int)(s / 65536ull) % 2147483647u;
    const int bl = int(__dmul_rn(double(nb), __ddiv_rn(double(int(r1)), kMaxIntD)));
    const double ha = __dmul_rn(__ddiv_rn(__dmul_rn(12., kCurPi), 12.0), __dsub_rn(__ddiv_rn(double(int(r2)), kMaxIntD), 0.5));
    const double cha = cos(ha), sha = sin(ha);
    u[i] = __dadd_rn(__dmul_rn(sha, bx[bl]), __dmul_rn(cha, by[bl]));
    v[i] = __dadd_rn(__dadd_rn(__dmul_rn(__dmul_rn(-sdec, cha), bx[bl]), __dmul_rn(__dmul_rn(sdec, sha), by[bl])),
                     __dmul_rn(cdec, bz[bl]));
    w[i] = __dadd_rn(__dsub_rn(__dmul_rn(__dmul_rn(cdec, cha), bx[bl]), __dmul_rn(__dmul_rn(cdec, sha), by[bl])),
                     __dmul_rn(sdec, bz[bl]));
}

__device__ __forceinline__ int plane_of(const int32_t* __restrict__ c_off0, int w_size, int64_t e)
{
    int lo = 0, hi = w_size - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (c_off0[mid] <= e)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

struct CurCParams {
    int64_t c_len;
    int w_size, os;
    double w_cell, uv_cell;
};

// Benchmark.cc:517-560: one table entry, before the per-plane normalisation
__global__ void cur_c_kernel(CurCParams p, const int32_t* __restrict__ s_size, const int32_t* __restrict__ c_off0,
                             float2* c)
{
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= p.c_len) return;
    const int k = plane_of(c_off0, p.w_size, e);
    const int s = s_size[k];
    int64_t idx = e - c_off0[k];
    const int i = int(idx % s);
    idx /= s;
    const int j = int(idx % s);
    idx /= s;
    const int osi = int(idx % p.os), osj = int(idx / p.os);
    const int wind = k - p.w_size / 2;
    const double w = __dmul_rn(double(wind), p.w_cell);
    const double f_scale = wind != 0 ? __ddiv_rn(__dmul_rn(p.uv_cell, p.uv_cell), w) : 0.0;
    const int center = s / 2;
    const double dj = __dadd_rn(double(j - center), __ddiv_rn(double(osj), double(p.os)));
    const double di = __dadd_rn(double(i - center), __ddiv_rn(double(osi), double(p.os)));
    const double r2 = __dadd_rn(__dmul_rn(dj, dj), __dmul_rn(di, di));
    float cre = float(exp(-r2)), cim = 0.f;
    if (wind != 0 && r2 < double(s / 2)) {
        const float n = float(__dsqrt_rn(__dsub_rn(1., __ddiv_rn(__dmul_rn(r2, f_scale), w))));
        const float phase = float(__dmul_rn(-2. * kCurPi, __dadd_rn(__dmul_rn(r2, f_scale),
                                                                   __dmul_rn(w, __dsub_rn(double(n), 1.)))));
        const float a = float(__ddiv_rn(double(n), w));
        const float sn = float(sin(double(phase))), cs = -float(cos(double(phase)));
        // (a + 0i) * (sn + cs i), then C *= that: the plain 4-multiply complex products in float
        const float xre = __fsub_rn(__fmul_rn(a, sn), __fmul_rn(0.f, cs));
        const float xim = __fadd_rn(__fmul_rn(a, cs), __fmul_rn(0.f, sn));
        const float nre = __fsub_rn(__fmul_rn(cre, xre), __fmul_rn(cim, xim));
        const float nim = __fadd_rn(__fmul_rn(cre, xim), __fmul_rn(cim, xre));
        cre = nre;
        cim = nim;
    }
    c[e] = make_float2(cre, cim);
}

// Benchmark.cc:556-568: per plane, the double sum of float |C| in table order, and the float
// factor os^2 / sum.  One warp per plane: lanes compute 32 magnitudes, lane 0 adds them in order.
__global__ void cur_norm_kernel(int w_size, int os, int64_t c_len, const int32_t* __restrict__ c_off0,
                                const float2* __restrict__ c, float* norm)
{
    const int k = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (k >= w_size) return;
    const int64_t b = c_off0[k], e = k + 1 < w_size ? c_off0[k + 1] : c_len;
    double sum = 0.0;
    for (int64_t base = b; base < e; base += 32) {
        float mag = 0.f;
        if (base + lane < e) {
            const float2 v = c[base + lane];
            // cabsf (hypotf): the square root of the double sum of squares, rounded to float
            mag = float(__dsqrt_rn(__dadd_rn(__dmul_rn(double(v.x), double(v.x)), __dmul_rn(double(v.y), double(v.y)))));
        }
        const int m = int(e - base < 32 ? e - base : 32);
        for (int t = 0; t < m; ++t) {
            const float x = __shfl_sync(0xffffffffu, mag, t);
            if (lane == 0) sum = __dadd_rn(sum, double(x));
        }
    }
    if (lane == 0) norm[k] = float(__ddiv_rn(double(os * os), sum));
}

// Benchmark.cc:565-568: C *= (norm + 0i), the 4-multiply product
__global__ void cur_scale_kernel(int64_t c_len, int w_size, const int32_t* __restrict__ c_off0,
                                 const float* __restrict__ norm, float2* c)
{
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= c_len) return;
    const float nm = norm[plane_of(c_off0, w_size, e)];
    const float2 v = c[e];
    c[e] = make_float2(__fsub_rn(__fmul_rn(v.x, nm), __fmul_rn(v.y, 0.f)), __fadd_rn(__fmul_rn(v.x, 0.f), __fmul_rn(v.y, nm)));
}

struct CurOffParams {
    int64_t n;
    double wavenumber, uv_cell, w_cell;
    int w_size, g_size, os;
};

// Benchmark.cc:599-640: grid position, w-plane and table offset per sample
__global__ void cur_offsets_kernel(CurOffParams p, const double* __restrict__ u, const double* __restrict__ v,
                                   const double* __restrict__ w, const int32_t* __restrict__ s_size,
                                   const int32_t* __restrict__ c_off0, int32_t* iu_out, int32_t* iv_out,
                                   int32_t* wplane_out, int32_t* coff_out)
{
    const int64_t d = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (d >= p.n) return;
    const double us = __ddiv_rn(__dmul_rn(p.wavenumber, u[d]), p.uv_cell);
    int iu = int(us);
    if (us < double(iu)) iu -= 1;
    const int fracu = int(__dmul_rn(double(p.os), __dsub_rn(us, double(iu))));
    iu += p.g_size / 2;
    const double vs = __ddiv_rn(__dmul_rn(p.wavenumber, v[d]), p.uv_cell);
    int iv = int(vs);
    if (vs < double(iv)) iv -= 1;
    const int fracv = int(__dmul_rn(double(p.os), __dsub_rn(vs, double(iv))));
    iv += p.g_size / 2;
    int woff = 0;
    if (p.w_cell > 0.0) woff = p.w_size / 2 + int(__ddiv_rn(__dmul_rn(p.wavenumber, w[d]), p.w_cell));
    if (woff < 0 || woff >= p.w_size) woff = woff < 0 ? 0 : p.w_size - 1;  // never for the reference's samples
    iu_out[d] = iu;
    iv_out[d] = iv;
    wplane_out[d] = woff;
    coff_out[d] = s_size[woff] * s_size[woff] * (fracu + p.os * fracv) + c_off0[woff];
}

__global__ void cur_fill_kernel(float2* p, int64_t n, float2 v)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = v;
}

__global__ void cur_iota_kernel(uint32_t* p, int64_t n)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) p[i] = uint32_t(i);
}

__global__ void cur_gather_kernel(int64_t n, const uint32_t* __restrict__ order, const int32_t* __restrict__ a,
                                  const int32_t* __restrict__ b, const int32_t* __restrict__ c, int32_t* oa,
                                  int32_t* ob, int32_t* oc)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t k = order[i];
    oa[i] = a[k];
    ob[i] = b[k];
    oc[i] = c[k];
}

__global__ void cur_count_kernel(int64_t n, const int32_t* __restrict__ wplane, unsigned long long* counts)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) atomicAdd(&counts[wplane[i]], 1ull);
}

unsigned blocks(int64_t n, int t = 256) { return unsigned((n + t - 1) / t); }

}  // namespace
}  // namespace tcv

using namespace tcv;

struct tcv_cur_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    uint64_t next = 1;  // the reference object's generator state (Benchmark::Benchmark, :47-50)
    int run_type = 0, sort = 0, c_type = TCV_C_C64;
    tcv_tuning tuning{16, 32, 0, 0};
    CurParams p{};
    int nb = 0;
    int64_t n = 0, c_len = 0, n_pixels = 0;
    std::vector<int32_t> s_size, c_off0;
    double *u = nullptr, *v = nullptr, *w = nullptr, *bxyz = nullptr;
    int32_t *iu = nullptr, *iv = nullptr, *wplane = nullptr, *coff = nullptr, *d_s = nullptr, *d_off0 = nullptr;
    float2 *data = nullptr, *outdata = nullptr, *grid = nullptr, *c64 = nullptr;
    void* c_alt = nullptr;
    float c_scale = 1.f;
    void* work = nullptr;
    size_t work_bytes = 0;
    tcv_plan* plan = nullptr;
    bool initialized = false;
    std::string err;
};

namespace {

tcv_status cur_fail(tcv_cur_ctx* c, tcv_status s, const std::string& what)
{
    if (c) c->err = what + ": " + tcv_status_string(s);
    return s;
}

#define CUR_TRY(c, call)                                   \
    do {                                                   \
        const tcv_status _s = (call);                      \
        if (_s != TCV_OK) return cur_fail(c, _s, #call);   \
    } while (0)

#define CUR_CUDA(c, call) CUR_TRY(c, ::tcv::cuda_status(call))

void cur_release(tcv_cur_ctx* c)
{
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->plan) tcv_plan_destroy(c->plan);
    c->plan = nullptr;
    void* bufs[] = {c->u, c->v, c->w, c->bxyz, c->iu, c->iv, c->wplane, c->coff, c->d_s, c->d_off0,
                    c->data, c->outdata, c->grid, c->c64, c->c_alt, c->work};
    for (void* b : bufs)
        if (b) cudaFree(b);
    c->u = c->v = c->w = c->bxyz = nullptr;
    c->iu = c->iv = c->wplane = c->coff = c->d_s = c->d_off0 = nullptr;
    c->data = c->outdata = c->grid = c->c64 = nullptr;
    c->c_alt = nullptr;
    c->work = nullptr;
    c->work_bytes = 0;
    c->initialized = false;
}

const void* cur_table(const tcv_cur_ctx* c) { return c->c_type == TCV_C_C64 ? static_cast<const void*>(c->c64) : c->c_alt; }

tcv_status cur_set_form(tcv_cur_ctx* c)
{
    if (c->c_alt) {
        CUR_CUDA(c, cudaStreamSynchronize(c->stream));
        cudaFree(c->c_alt);
        c->c_alt = nullptr;
    }
    c->c_scale = 1.f;
    if (c->c_type == TCV_C_C64) return TCV_OK;
    CUR_CUDA(c, cudaMalloc(&c->c_alt, size_t(c->c_len) * tcv_ctype_bytes(c->c_type) + 16));
    CUR_TRY(c, tcv_convert_c(reinterpret_cast<const float*>(c->c64), c->c_len, c->c_type, c->c_alt, &c->c_scale,
                             nullptr, c->stream));
    return TCV_OK;
}

tcv_status cur_build_plan(tcv_cur_ctx* c)
{
    if (c->plan) {
        tcv_plan_destroy(c->plan);
        c->plan = nullptr;
    }
    const size_t need = tcv_plan_workspace_bytes_var(c->n, c->s_size.data(), c->c_off0.data(), c->p.w_size,
                                                     c->p.g_size, c->c_len, &c->tuning);
    if (need == 0) return cur_fail(c, TCV_ERR_UNSUPPORTED, "plan geometry");
    if (need > c->work_bytes) {
        CUR_CUDA(c, cudaStreamSynchronize(c->stream));
        if (c->work) cudaFree(c->work);
        c->work = nullptr;
        c->work_bytes = 0;
        CUR_CUDA(c, cudaMalloc(&c->work, need));
        c->work_bytes = need;
    }
    CUR_TRY(c, tcv_plan_build_var(&c->plan, c->iu, c->iv, c->coff, c->wplane, c->n, c->s_size.data(),
                                  c->c_off0.data(), c->p.w_size, c->p.g_size, c->c_len, &c->tuning, c->work,
                                  c->work_bytes, c->stream));
    int64_t rej = 0;
    CUR_TRY(c, tcv_plan_rejected(c->plan, &rej, c->stream));
    if (rej > 0) {
        c->err = std::to_string(rej) + " sample(s) fall outside the grid or the table and are skipped";
        return TCV_ERR_BOUNDS;
    }
    return TCV_OK;
}

tcv_status copy_out(tcv_cur_ctx* c, void* dst, const void* src, size_t bytes)
{
    if (!c || !dst) return TCV_ERR_ARG;
    if (!c->initialized) return cur_fail(c, TCV_ERR_STATE, "copy before init");
    CUR_CUDA(c, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream));
    CUR_CUDA(c, cudaStreamSynchronize(c->stream));
    return TCV_OK;
}

}  // namespace

extern "C" {

tcv_status tcv_cur_geometry_of(int run_type, tcv_cur_geometry* out)
{
    if (!out) return TCV_ERR_ARG;
    CurParams p;
    if (!cur_params(run_type, p)) return TCV_ERR_ARG;
    std::vector<double> bx, by, bz;
    const int nb = cur_baselines(p.baseline, bx, by, bz);
    std::vector<int32_t> s_size, off0;
    const int64_t c_len = cur_planes(p, s_size, off0);
    tcv_cur_geometry g{};
    g.run_type = run_type;
    g.w_size = p.w_size;
    g.over_sample = p.over_sample;
    g.support = p.support;
    g.g_size = p.g_size;
    g.n_baselines = nb;
    g.n_samples = int64_t(kScans) * nb;
    g.c_len = c_len;
    g.s_min = s_size[0];
    g.s_max = s_size[0];
    for (int32_t s : s_size) {
        g.s_min = std::min(g.s_min, s);
        g.s_max = std::max(g.s_max, s);
    }
    g.w_cell_size = p.w_cell;
    g.uv_cell_size = p.uv_cell;
    *out = g;
    return TCV_OK;
}

tcv_status tcv_cur_planes(int run_type, int32_t* s_size, int32_t* c_off0)
{
    if (!s_size || !c_off0) return TCV_ERR_ARG;
    CurParams p;
    if (!cur_params(run_type, p)) return TCV_ERR_ARG;
    std::vector<int32_t> s, o;
    cur_planes(p, s, o);
    std::memcpy(s_size, s.data(), s.size() * 4);
    std::memcpy(c_off0, o.data(), o.size() * 4);
    return TCV_OK;
}

tcv_status tcv_cur_init_uvw_raw(int run_type, uint64_t state0, double* d_u, double* d_v, double* d_w,
                                uint64_t* state_after, void* stream)
{
    CurParams p;
    if (!cur_params(run_type, p) || !d_u || !d_v || !d_w) return TCV_ERR_ARG;
    std::vector<double> bx, by, bz;
    const int nb = cur_baselines(p.baseline, bx, by, bz);
    const int64_t n = int64_t(kScans) * nb;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    double* dev = nullptr;
    TCV_CUDA(cudaMalloc(&dev, size_t(3 * nb) * sizeof(double)));
    std::vector<double> all(bx);
    all.insert(all.end(), by.begin(), by.end());
    all.insert(all.end(), bz.begin(), bz.end());
    cudaError_t e = cudaMemcpyAsync(dev, all.data(), all.size() * sizeof(double), cudaMemcpyHostToDevice, st);
    const double lat = -26.6970 * kCurPi / 180.0;
    if (e == cudaSuccess) {
        cur_uvw_kernel<<<blocks(n), 256, 0, st>>>(n, nb, state0, dev, dev + nb, dev + 2 * nb, std::cos(lat),
                                                  std::sin(lat), d_u, d_v, d_w);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(dev);
    if (e != cudaSuccess) return cuda_status(e);
    if (state_after) {
        uint64_t A, C;
        lcg_jump(2ull * uint64_t(n), A, C);
        *state_after = A * state0 + C;
    }
    return TCV_OK;
}

tcv_status tcv_cur_init_c_raw(int run_type, float* d_c, void* stream)
{
    CurParams p;
    if (!cur_params(run_type, p) || !d_c) return TCV_ERR_ARG;
    std::vector<int32_t> s_size, off0;
    const int64_t c_len = cur_planes(p, s_size, off0);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    void* dev = nullptr;
    const size_t wb = size_t(p.w_size) * 4;
    TCV_CUDA(cudaMalloc(&dev, 3 * wb + 64));
    int32_t* d_s = static_cast<int32_t*>(dev);
    int32_t* d_o = d_s + p.w_size;
    float* d_norm = reinterpret_cast<float*>(d_o + p.w_size);
    cudaError_t e = cudaMemcpyAsync(d_s, s_size.data(), wb, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_o, off0.data(), wb, cudaMemcpyHostToDevice, st);
    float2* c = reinterpret_cast<float2*>(d_c);
    if (e == cudaSuccess) {
        cur_c_kernel<<<blocks(c_len), 256, 0, st>>>(CurCParams{c_len, p.w_size, p.over_sample, p.w_cell, p.uv_cell},
                                                    d_s, d_o, c);
        cur_norm_kernel<<<blocks(int64_t(p.w_size) * 32), 256, 0, st>>>(p.w_size, p.over_sample, c_len, d_o, c, d_norm);
        cur_scale_kernel<<<blocks(c_len), 256, 0, st>>>(c_len, p.w_size, d_o, d_norm, c);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(dev);
    return cuda_status(e);
}

tcv_status tcv_cur_init_offsets_raw(int run_type, const double* d_u, const double* d_v, const double* d_w, int64_t n,
                                    const int32_t* d_s_size, const int32_t* d_c_off0, int32_t* d_iu, int32_t* d_iv,
                                    int32_t* d_wplane, int32_t* d_coff, void* stream)
{
    CurParams p;
    if (!cur_params(run_type, p) || n < 0) return TCV_ERR_ARG;
    if (n > 0 && (!d_u || !d_v || !d_w || !d_s_size || !d_c_off0 || !d_iu || !d_iv || !d_wplane || !d_coff))
        return TCV_ERR_ARG;
    if (n == 0) return TCV_OK;
    const double wavenumber = (double(1.0e9f) - 2.0e5 * 0.0 / 1.0) / 2.998e8;  // Benchmark.cc:269-272, channel 0
    const CurOffParams op{n, wavenumber, p.uv_cell, p.w_cell, p.w_size, p.g_size, p.over_sample};
    cur_offsets_kernel<<<blocks(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(op, d_u, d_v, d_w, d_s_size, d_c_off0,
                                                                                  d_iu, d_iv, d_wplane, d_coff);
    TCV_CUDA(cudaGetLastError());
    return TCV_OK;
}

void tcv_cur_required_rate(float* rates)
{
    if (!rates) return;
    // current/tConvolveMPI/Benchmark.cc:697-739 (continuum, then spectral line)
    long n_vis = long((36 * 35) / 2 * 12 * 3600. / 5.);
    rates[0] = float(double(10L * n_vis * 10L * 3L * 3L * 1L * 1L * 400L) / 5250.);
    n_vis = long((30 * 29) / 2 * 12 * 3600. / 5.);
    rates[1] = float(double(10L * n_vis * 4L * 3L * 1L * 1L * 78L * 100L) / 5500.);
}

tcv_status tcv_cur_create(int device, tcv_cur_ctx** out)
{
    if (!out) return TCV_ERR_ARG;
    *out = nullptr;
    tcv_cur_ctx* c = new (std::nothrow) tcv_cur_ctx;
    if (!c) return TCV_ERR_OOM;
    c->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete c;
        return cuda_status(e);
    }
    *out = c;
    return TCV_OK;
}

void tcv_cur_destroy(tcv_cur_ctx* c)
{
    if (!c) return;
    cudaSetDevice(c->device);
    cur_release(c);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

const char* tcv_cur_last_error(const tcv_cur_ctx* c) { return c ? c->err.c_str() : "null context"; }

tcv_status tcv_cur_set_sort(tcv_cur_ctx* c, int sort)
{
    if (!c || (sort != 0 && sort != 1)) return TCV_ERR_ARG;
    c->sort = sort;
    return TCV_OK;
}

tcv_status tcv_cur_set_run_type(tcv_cur_ctx* c, int run_type)
{
    CurParams p;
    if (!c || !cur_params(run_type, p)) return TCV_ERR_ARG;
    c->run_type = run_type;
    return TCV_OK;
}

int tcv_cur_get_run_type(const tcv_cur_ctx* c) { return c ? c->run_type : -1; }

tcv_status tcv_cur_set_ctype(tcv_cur_ctx* c, int c_type)
{
    if (!c || (c_type != TCV_C_C64 && c_type != TCV_C_CBF16 && c_type != TCV_C_CF16)) return TCV_ERR_ARG;
    c->c_type = c_type;
    return c->initialized ? cur_set_form(c) : TCV_OK;
}

tcv_status tcv_cur_set_tuning(tcv_cur_ctx* c, const tcv_tuning* t)
{
    if (!c || !t || (t->tile_rows != 0 && t->tile_rows != 8 && t->tile_rows != 16) || t->group_mib < -1 ||
        t->split < 0 || t->degrid_split < 0 || (t->kernel != 0 && !(t->kernel >= 1 && t->kernel <= 3 && t->tile_rows == 8)))
        return TCV_ERR_ARG;
    c->tuning = tcv_tuning{t->tile_rows ? t->tile_rows : 16, t->group_mib ? t->group_mib : 32, t->split, t->degrid_split,
                           t->kernel};
    return c->initialized ? cur_build_plan(c) : TCV_OK;
}

tcv_status tcv_cur_tune(tcv_cur_ctx* c, int reps, tcv_tuning* best_out, float* best_ms_out)
{
    if (!c || reps < 1) return TCV_ERR_ARG;
    if (!c->initialized) return cur_fail(c, TCV_ERR_STATE, "tune before init");
    reps = std::min(reps, 50);
    const size_t g2 = size_t(c->p.g_size) * c->p.g_size;
    float2 *grid = nullptr, *out = nullptr;
    cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
    cudaError_t e = cudaMalloc(&grid, g2 * 8);
    if (e == cudaSuccess) e = cudaMalloc(&out, size_t(std::max<int64_t>(c->n, 1)) * 8);
    for (int k = 0; k < 3 && e == cudaSuccess; ++k) e = cudaEventCreate(&ev[k]);
    std::vector<std::pair<tcv_tuning, float>> report;
    tcv_tuning best = c->tuning;
    float best_ms = -1.f;
    tcv_status s = cuda_status(e);
    // one candidate: build its plan, then (reps + 1) x (grid pass, degrid pass), the first untimed
    auto time_one = [&](const tcv_tuning& t) -> tcv_status {
        c->tuning = t;
        tcv_status r = cur_build_plan(c);
        if (r != TCV_OK) return r;
        std::vector<float> ms;
        for (int k = 0; k <= reps && r == TCV_OK; ++k) {
            r = cuda_status(cudaMemsetAsync(grid, 0, g2 * 8, c->stream));
            if (r == TCV_OK) r = cuda_status(cudaEventRecord(ev[0], c->stream));
            if (r == TCV_OK)
                r = tcv_plan_grid(c->plan, reinterpret_cast<const float*>(c->data), cur_table(c), c->c_type,
                                  c->c_scale, reinterpret_cast<float*>(grid), c->stream);
            if (r == TCV_OK)
                r = tcv_plan_degrid(c->plan, reinterpret_cast<const float*>(grid), cur_table(c), c->c_type,
                                    c->c_scale, reinterpret_cast<float*>(out), c->stream);
            if (r == TCV_OK) r = cuda_status(cudaEventRecord(ev[1], c->stream));
            if (r == TCV_OK) r = cuda_status(cudaEventSynchronize(ev[1]));
            float m = 0.f;
            if (r == TCV_OK) r = cuda_status(cudaEventElapsedTime(&m, ev[0], ev[1]));
            if (k > 0) ms.push_back(m);
        }
        if (r != TCV_OK) return r;
        std::sort(ms.begin(), ms.end());
        const float med = ms[ms.size() / 2];
        report.emplace_back(t, med);
        if (best_ms < 0.f || med < best_ms) {
            best_ms = med;
            best = t;
        }
        return TCV_OK;
    };
    // stage 1: kernel families and tile height x plane-group slice (slices that give the same
    // grouping timed once), with typical work units (256 gridding, 128 degridding samples: these
    // problems' busy cells need them, and the families rank differently without).  Variants:
    // 64 x 64 and 64 x 32 tile kernels; on 64 x 32 tiles the sample-parallel degridding, and both
    // passes sample-parallel (kernel bits 2 and 3).
    if (s == TCV_OK) {
        std::vector<std::pair<int, int>> seen;  // (variant, number of plane groups)
        for (int variant : {16, 8, -2, -3})
            for (int mib : {32, 128, -1}) {
                const int rows = variant < 0 ? 8 : variant;
                const tcv_tuning t{rows, mib, 256, 128, variant < 0 ? -variant : 0};
                int groups = 1;
                const int64_t budget = mib > 0 ? (int64_t(mib) << 20) : INT64_MAX;
                int64_t used = 0;
                for (int k = 0; k < c->p.w_size; ++k) {
                    const int64_t end = k + 1 < c->p.w_size ? c->c_off0[size_t(k) + 1] : c->c_len;
                    const int64_t bytes = (end - c->c_off0[size_t(k)]) * 8;
                    if (used > 0 && used + bytes > budget) {
                        ++groups;
                        used = 0;
                    }
                    used += bytes;
                }
                const std::pair<int, int> id(variant, groups);
                if (std::find(seen.begin(), seen.end(), id) != seen.end()) continue;
                seen.push_back(id);
                if ((s = time_one(t)) != TCV_OK) break;
            }
    }
    if (s == TCV_OK) {  // stage 2: gridding work units
        const tcv_tuning base = best;
        for (int split : {1024, 512, 128, 64})  // the partial-tile bound grows as 1 / split
            if ((s = time_one(tcv_tuning{base.tile_rows, base.group_mib, split, base.degrid_split, base.kernel})) !=
                TCV_OK)
                break;
    }
    if (s == TCV_OK) {  // stage 3: degridding work units
        const tcv_tuning base = best;
        for (int split : {256, 64, 32, 16})
            if ((s = time_one(tcv_tuning{base.tile_rows, base.group_mib, base.split, split, base.kernel})) != TCV_OK)
                break;
    }
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (cudaEvent_t x : ev)
        if (x) cudaEventDestroy(x);
    if (grid) cudaFree(grid);
    if (out) cudaFree(out);
    if (s != TCV_OK) return cur_fail(c, s, "tuning candidate");
    tune_report_set(report);
    c->tuning = best;
    CUR_TRY(c, cur_build_plan(c));
    if (best_out) *best_out = best;
    if (best_ms_out) *best_ms_out = best_ms;
    return TCV_OK;
}

tcv_status tcv_cur_init(tcv_cur_ctx* c)
{
    if (!c) return TCV_ERR_ARG;
    CUR_CUDA(c, cudaSetDevice(c->device));
    cur_release(c);
    if (!cur_params(c->run_type, c->p)) return cur_fail(c, TCV_ERR_ARG, "run type");
    std::vector<double> bx, by, bz;
    c->nb = cur_baselines(c->p.baseline, bx, by, bz);
    c->n = int64_t(kScans) * c->nb;
    c->c_len = cur_planes(c->p, c->s_size, c->c_off0);
    const int64_t n = c->n;
    const size_t g2 = size_t(c->p.g_size) * c->p.g_size;
    const size_t wb = size_t(c->p.w_size) * 4;
    CUR_CUDA(c, cudaMalloc(&c->u, size_t(n) * 8));
    CUR_CUDA(c, cudaMalloc(&c->v, size_t(n) * 8));
    CUR_CUDA(c, cudaMalloc(&c->w, size_t(n) * 8));
    CUR_CUDA(c, cudaMalloc(&c->iu, size_t(n) * 4));
    CUR_CUDA(c, cudaMalloc(&c->iv, size_t(n) * 4));
    CUR_CUDA(c, cudaMalloc(&c->wplane, size_t(n) * 4));
    CUR_CUDA(c, cudaMalloc(&c->coff, size_t(n) * 4));
    CUR_CUDA(c, cudaMalloc(&c->data, size_t(n) * 8));
    CUR_CUDA(c, cudaMalloc(&c->outdata, size_t(n) * 8));
    CUR_CUDA(c, cudaMalloc(&c->grid, g2 * 8));
    CUR_CUDA(c, cudaMalloc(&c->c64, size_t(c->c_len) * 8));
    CUR_CUDA(c, cudaMalloc(&c->d_s, wb));
    CUR_CUDA(c, cudaMalloc(&c->d_off0, wb));
    CUR_CUDA(c, cudaMemcpyAsync(c->d_s, c->s_size.data(), wb, cudaMemcpyHostToDevice, c->stream));
    CUR_CUDA(c, cudaMemcpyAsync(c->d_off0, c->c_off0.data(), wb, cudaMemcpyHostToDevice, c->stream));
    // Benchmark::init (Benchmark.cc:61-311): samples, data = 1 + 0i, zero grid, table, offsets
    uint64_t after = 0;
    CUR_TRY(c, tcv_cur_init_uvw_raw(c->run_type, c->next, c->u, c->v, c->w, &after, c->stream));
    c->next = after;
    cur_fill_kernel<<<1024, 256, 0, c->stream>>>(c->data, n, make_float2(1.f, 0.f));
    CUR_CUDA(c, cudaGetLastError());
    CUR_CUDA(c, cudaMemsetAsync(c->outdata, 0, size_t(n) * 8, c->stream));
    CUR_CUDA(c, cudaMemsetAsync(c->grid, 0, g2 * 8, c->stream));
    CUR_TRY(c, tcv_cur_init_c_raw(c->run_type, reinterpret_cast<float*>(c->c64), c->stream));
    CUR_TRY(c, tcv_cur_init_offsets_raw(c->run_type, c->u, c->v, c->w, n, c->d_s, c->d_off0, c->iu, c->iv, c->wplane,
                                        c->coff, c->stream));
    // numPerPlane and nPixelsGridded (Benchmark.cc:637, 679-694)
    {
        unsigned long long* counts = nullptr;
        CUR_CUDA(c, cudaMalloc(&counts, size_t(c->p.w_size) * 8));
        cudaError_t e = cudaMemsetAsync(counts, 0, size_t(c->p.w_size) * 8, c->stream);
        if (e == cudaSuccess) {
            cur_count_kernel<<<blocks(n), 256, 0, c->stream>>>(n, c->wplane, counts);
            e = cudaGetLastError();
        }
        std::vector<unsigned long long> h(size_t(c->p.w_size));
        if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), counts, size_t(c->p.w_size) * 8, cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        cudaFree(counts);
        CUR_CUDA(c, e);
        c->n_pixels = 0;
        for (int k = 0; k < c->p.w_size; ++k)
            c->n_pixels += int64_t(h[size_t(k)]) * c->s_size[size_t(k)] * c->s_size[size_t(k)];
    }
    // setSort(1) (Benchmark.cc:287-306): offsets stably ordered by w-plane; the data stay put
    if (c->sort == 1 && c->p.w_size > 1 && n > 0) {
        int bits = 1;
        while ((1 << bits) < c->p.w_size) ++bits;
        uint32_t *idx = nullptr, *idx2 = nullptr;
        int32_t *keys2 = nullptr, *t = nullptr;
        size_t tb = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, tb, (const int32_t*)nullptr, (int32_t*)nullptr,
                                        (const uint32_t*)nullptr, (uint32_t*)nullptr, n, 0, bits);
        void* tmp = nullptr;
        cudaError_t e = cudaMalloc(&idx, size_t(n) * 4);
        if (e == cudaSuccess) e = cudaMalloc(&idx2, size_t(n) * 4);
        if (e == cudaSuccess) e = cudaMalloc(&keys2, size_t(n) * 4);
        if (e == cudaSuccess) e = cudaMalloc(&t, size_t(n) * 12);
        if (e == cudaSuccess) e = cudaMalloc(&tmp, tb);
        if (e == cudaSuccess) {
            cur_iota_kernel<<<blocks(n), 256, 0, c->stream>>>(idx, n);
            e = cub::DeviceRadixSort::SortPairs(tmp, tb, c->wplane, keys2, idx, idx2, n, 0, bits, c->stream);
        }
        if (e == cudaSuccess) {
            cur_gather_kernel<<<blocks(n), 256, 0, c->stream>>>(n, idx2, c->iu, c->iv, c->coff, t, t + n, t + 2 * n);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(c->iu, t, size_t(n) * 4, cudaMemcpyDeviceToDevice, c->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(c->iv, t + n, size_t(n) * 4, cudaMemcpyDeviceToDevice, c->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(c->coff, t + 2 * n, size_t(n) * 4, cudaMemcpyDeviceToDevice, c->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(c->wplane, keys2, size_t(n) * 4, cudaMemcpyDeviceToDevice, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        void* fr[] = {idx, idx2, keys2, t, tmp};
        for (void* f : fr)
            if (f) cudaFree(f);
        CUR_CUDA(c, e);
    }
    c->initialized = true;
    CUR_TRY(c, cur_set_form(c));
    return cur_build_plan(c);
}

tcv_status tcv_cur_run_grid(tcv_cur_ctx* c)
{
    if (!c) return TCV_ERR_ARG;
    if (!c->initialized || !c->plan) return cur_fail(c, TCV_ERR_STATE, "run_grid before init");
    CUR_TRY(c, tcv_plan_grid(c->plan, reinterpret_cast<const float*>(c->data), cur_table(c), c->c_type, c->c_scale,
                             reinterpret_cast<float*>(c->grid), c->stream));
    return TCV_OK;
}

tcv_status tcv_cur_run_degrid(tcv_cur_ctx* c)
{
    if (!c) return TCV_ERR_ARG;
    if (!c->initialized || !c->plan) return cur_fail(c, TCV_ERR_STATE, "run_degrid before init");
    CUR_TRY(c, tcv_plan_degrid(c->plan, reinterpret_cast<const float*>(c->grid), cur_table(c), c->c_type,
                               c->c_scale, reinterpret_cast<float*>(c->outdata), c->stream));
    return TCV_OK;
}

tcv_status tcv_cur_sync(tcv_cur_ctx* c)
{
    if (!c) return TCV_ERR_ARG;
    CUR_CUDA(c, cudaStreamSynchronize(c->stream));
    return TCV_OK;
}

void* tcv_cur_get_stream(const tcv_cur_ctx* c) { return c ? static_cast<void*>(c->stream) : nullptr; }
int tcv_cur_support(const tcv_cur_ctx* c) { return c ? c->p.support : -1; }
int64_t tcv_cur_n_visibilities(const tcv_cur_ctx* c) { return c ? c->n : 0; }
int64_t tcv_cur_n_pixels(const tcv_cur_ctx* c) { return c ? c->n_pixels : 0; }
uint64_t tcv_cur_generator_state(const tcv_cur_ctx* c) { return c ? c->next : 0; }

tcv_status tcv_cur_info(const tcv_cur_ctx* c, tcv_cur_geometry* g)
{
    if (!c || !g) return TCV_ERR_ARG;
    return tcv_cur_geometry_of(c->run_type, g);
}

tcv_status tcv_cur_set_data(tcv_cur_ctx* c, const float* vis, int64_t n)
{
    if (!c || !vis || !c->initialized || n != c->n) return TCV_ERR_ARG;
    CUR_CUDA(c, cudaMemcpyAsync(c->data, vis, size_t(n) * 8, cudaMemcpyHostToDevice, c->stream));
    CUR_CUDA(c, cudaStreamSynchronize(c->stream));
    return TCV_OK;
}

tcv_status tcv_cur_zero_grid(tcv_cur_ctx* c)
{
    if (!c || !c->initialized) return TCV_ERR_ARG;
    CUR_CUDA(c, cudaMemsetAsync(c->grid, 0, size_t(c->p.g_size) * c->p.g_size * 8, c->stream));
    return TCV_OK;
}

tcv_status tcv_cur_get_grid(tcv_cur_ctx* c, float* grid)
{
    return copy_out(c, grid, c ? c->grid : nullptr, c ? size_t(c->p.g_size) * c->p.g_size * 8 : 0);
}
tcv_status tcv_cur_get_outdata(tcv_cur_ctx* c, float* vis, int64_t n)
{
    if (!c || n != c->n) return TCV_ERR_ARG;
    return copy_out(c, vis, c->outdata, size_t(n) * 8);
}
tcv_status tcv_cur_get_c(tcv_cur_ctx* c, float* out, int64_t n)
{
    if (!c || n != c->c_len) return TCV_ERR_ARG;
    return copy_out(c, out, c->c64, size_t(n) * 8);
}
tcv_status tcv_cur_get_uvw(tcv_cur_ctx* c, double* u, double* v, double* w)
{
    if (!c) return TCV_ERR_ARG;
    tcv_status s = copy_out(c, u, c->u, size_t(c->n) * 8);
    if (s == TCV_OK) s = copy_out(c, v, c->v, size_t(c->n) * 8);
    if (s == TCV_OK) s = copy_out(c, w, c->w, size_t(c->n) * 8);
    return s;
}
tcv_status tcv_cur_get_offsets(tcv_cur_ctx* c, int32_t* iu, int32_t* iv, int32_t* wplane, int32_t* coff)
{
    if (!c) return TCV_ERR_ARG;
    const size_t b = size_t(c->n) * 4;
    tcv_status s = copy_out(c, iu, c->iu, b);
    if (s == TCV_OK) s = copy_out(c, iv, c->iv, b);
    if (s == TCV_OK) s = copy_out(c, wplane, c->wplane, b);
    if (s == TCV_OK) s = copy_out(c, coff, c->coff, b);
    return s;
}
tcv_status tcv_cur_get_planes(const tcv_cur_ctx* c, int32_t* s_size, int32_t* c_off0)
{
    if (!c || !s_size || !c_off0 || !c->initialized) return TCV_ERR_ARG;
    std::memcpy(s_size, c->s_size.data(), c->s_size.size() * 4);
    std::memcpy(c_off0, c->c_off0.data(), c->c_off0.size() * 4);
    return TCV_OK;
}

}  // extern "C"
