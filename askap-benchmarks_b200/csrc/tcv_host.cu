// tcv_host.cu -- host-buffer one-call entry points.
//
// These follow the reference's libCudaGridder seam (attic/tConvolveCuda/CudaGridder.cc:54-207):
// allocate device buffers, upload, run, download, free, and report the device time of the work
// itself (the reference times the kernel launches and the synchronisation, :108-115, 188-195;
// here CUDA events bracket the binning plan plus the kernel).
#include "tcv_internal.cuh"

#include <vector>

namespace {

struct DevBufs {
    std::vector<void*> ptrs;
    ~DevBufs()
    {
        for (void* p : ptrs)
            if (p) cudaFree(p);
    }
    cudaError_t alloc(void** p, size_t bytes)
    {
        *p = nullptr;
        cudaError_t e = cudaMalloc(p, bytes ? bytes : 16);
        if (e == cudaSuccess) ptrs.push_back(*p);
        return e;
    }
};

struct Events {
    cudaEvent_t a = nullptr, b = nullptr;
    ~Events()
    {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
    }
};

struct Stream {
    cudaStream_t s = nullptr;
    ~Stream()
    {
        if (s) cudaStreamDestroy(s);
    }
};

tcv_status run_host(bool gridding, const float* data_in, float* data_out, int64_t n, int support,
                    const float* c, int64_t c_len, const int32_t* coff, const int32_t* iu,
                    const int32_t* iv, const float* grid_in, float* grid_out, int g_size, int device,
                    double* device_seconds)
{
    if (n < 0 || support < 0 || g_size < 1 || c_len < 1 || !c || !coff || !iu || !iv) return TCV_ERR_ARG;
    if (gridding ? (!data_in || !grid_out) : (!grid_in || !data_out)) return TCV_ERR_ARG;
    TCV_CUDA(cudaSetDevice(device));
    Stream st;
    TCV_CUDA(cudaStreamCreateWithFlags(&st.s, cudaStreamNonBlocking));
    DevBufs b;
    void *d_data, *d_c, *d_co, *d_iu, *d_iv, *d_grid, *d_work;
    const size_t gbytes = size_t(g_size) * g_size * 8;
    const size_t wbytes = tcv_plan_workspace_bytes(n, support, g_size, c_len);
    TCV_CUDA(b.alloc(&d_data, size_t(n) * 8));
    TCV_CUDA(b.alloc(&d_c, size_t(c_len) * 8));
    TCV_CUDA(b.alloc(&d_co, size_t(n) * 4));
    TCV_CUDA(b.alloc(&d_iu, size_t(n) * 4));
    TCV_CUDA(b.alloc(&d_iv, size_t(n) * 4));
    TCV_CUDA(b.alloc(&d_grid, gbytes));
    TCV_CUDA(b.alloc(&d_work, wbytes));
    TCV_CUDA(cudaMemcpyAsync(d_c, c, size_t(c_len) * 8, cudaMemcpyHostToDevice, st.s));
    TCV_CUDA(cudaMemcpyAsync(d_co, coff, size_t(n) * 4, cudaMemcpyHostToDevice, st.s));
    TCV_CUDA(cudaMemcpyAsync(d_iu, iu, size_t(n) * 4, cudaMemcpyHostToDevice, st.s));
    TCV_CUDA(cudaMemcpyAsync(d_iv, iv, size_t(n) * 4, cudaMemcpyHostToDevice, st.s));
    if (gridding) {
        TCV_CUDA(cudaMemcpyAsync(d_data, data_in, size_t(n) * 8, cudaMemcpyHostToDevice, st.s));
        TCV_CUDA(cudaMemcpyAsync(d_grid, grid_out, gbytes, cudaMemcpyHostToDevice, st.s));  // accumulate
    } else {
        TCV_CUDA(cudaMemcpyAsync(d_grid, grid_in, gbytes, cudaMemcpyHostToDevice, st.s));
    }
    Events ev;
    TCV_CUDA(cudaEventCreate(&ev.a));
    TCV_CUDA(cudaEventCreate(&ev.b));
    TCV_CUDA(cudaEventRecord(ev.a, st.s));
    tcv_plan* plan = nullptr;
    tcv_status s = tcv_plan_build(&plan, static_cast<const int32_t*>(d_iu), static_cast<const int32_t*>(d_iv),
                                  static_cast<const int32_t*>(d_co), n, support, g_size, c_len, d_work,
                                  wbytes, st.s);
    if (s != TCV_OK) return s;
    s = gridding ? tcv_plan_grid(plan, static_cast<const float*>(d_data), d_c, TCV_C_C64, 1.0f,
                                 static_cast<float*>(d_grid), st.s)
                 : tcv_plan_degrid(plan, static_cast<const float*>(d_grid), d_c, TCV_C_C64, 1.0f,
                                   static_cast<float*>(d_data), st.s);
    if (s != TCV_OK) {
        tcv_plan_destroy(plan);
        return s;
    }
    cudaError_t e = cudaEventRecord(ev.b, st.s);
    if (e == cudaSuccess)
        e = gridding ? cudaMemcpyAsync(grid_out, d_grid, gbytes, cudaMemcpyDeviceToHost, st.s)
                     : cudaMemcpyAsync(data_out, d_data, size_t(n) * 8, cudaMemcpyDeviceToHost, st.s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st.s);
    int64_t rejected = 0;
    if (e == cudaSuccess) s = tcv_plan_rejected(plan, &rejected, st.s);
    if (e == cudaSuccess && s == TCV_OK) s = tcv_plan_status(plan, st.s);
    tcv_plan_destroy(plan);
    TCV_CUDA(e);
    if (s != TCV_OK) return s;
    float ms = 0.f;
    TCV_CUDA(cudaEventElapsedTime(&ms, ev.a, ev.b));
    if (device_seconds) *device_seconds = ms * 1e-3;
    if (rejected > 0) return TCV_ERR_BOUNDS;
    return TCV_OK;
}

}  // namespace

extern "C" {

tcv_status tcv_grid_host_raw(const float* data, int64_t n, int support, const float* c, int64_t c_len,
                             const int32_t* coff, const int32_t* iu, const int32_t* iv, float* grid,
                             int g_size, int device, double* device_seconds)
{
    return run_host(true, data, nullptr, n, support, c, c_len, coff, iu, iv, nullptr, grid, g_size,
                    device, device_seconds);
}

tcv_status tcv_degrid_host_raw(const float* grid, int g_size, int support, const float* c, int64_t c_len,
                               const int32_t* coff, const int32_t* iu, const int32_t* iv, float* data,
                               int64_t n, int device, double* device_seconds)
{
    return run_host(false, nullptr, data, n, support, c, c_len, coff, iu, iv, grid, nullptr, g_size,
                    device, device_seconds);
}

tcv_status tcv_init_c_host(double freq0, double cell_size, int baseline, int w_size, float* c,
                           int64_t c_len, int device, int* support, int* over_sample,
                           double* w_cell_size, float* sum_c)
{
    int64_t need = 0;
    tcv_status s = tcv_c_geometry(freq0, cell_size, baseline, w_size, support, over_sample, w_cell_size, &need);
    if (s != TCV_OK) return s;
    if (!c || c_len != need) return TCV_ERR_ARG;
    TCV_CUDA(cudaSetDevice(device));
    Stream st;
    TCV_CUDA(cudaStreamCreateWithFlags(&st.s, cudaStreamNonBlocking));
    DevBufs b;
    void *d_c, *d_scratch;
    TCV_CUDA(b.alloc(&d_c, size_t(c_len) * 8));
    TCV_CUDA(b.alloc(&d_scratch, tcv_init_c_scratch_bytes()));
    s = tcv_init_c_raw(freq0, cell_size, baseline, w_size, static_cast<float*>(d_c), d_scratch, sum_c, st.s);
    if (s != TCV_OK) return s;
    TCV_CUDA(cudaMemcpyAsync(c, d_c, size_t(c_len) * 8, cudaMemcpyDeviceToHost, st.s));
    TCV_CUDA(cudaStreamSynchronize(st.s));
    return TCV_OK;
}

}  // extern "C"
