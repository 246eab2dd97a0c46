// tcv_serve.cu -- request loop with continuous batching over resident grids and table.
//
// Threads: callers submit requests (host pointers) into a FIFO; one scheduler thread forms a
// batch whenever a batch slot is free and launches it on that slot's stream (host staging copy,
// H2D, offsets, a batched gridding plan and pass, a batched degridding plan and pass, D2H, an
// event); one completion thread per slot waits for the slot's event, copies degridded samples
// to the callers' buffers and marks the requests done.  So while one batch runs on the GPU the
// scheduler stages and launches the next on another slot, and requests that arrive meanwhile
// join the next batch that forms.
//
// Ordering: a batch holds at most one request per grid, and a request is taken only when no
// earlier request on its grid is pending or in flight, so the requests on one grid are applied
// in submission order.  Results do not depend on the rest of the batch (see tcv_plan.cu: a
// job's cells hold only its own samples, summed in index order).
//
// The computations are the reference's: u, v, w -> offsets (Benchmark::initCOffset,
// attic/tConvolveMPI/Benchmark.cc:281-324), gridding (:125-155), degridding (:158-195).
#include "tcv_internal.cuh"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

namespace {

using Clock = std::chrono::steady_clock;

struct ServeReq {
    tcv_request r;
    uint64_t id = 0;
    double t_submit = 0, t_start = 0, t_done = 0;
    int status = TCV_OK;
    int batch_requests = 0;
    int64_t rejected = 0;
    bool done = false;
};
using ReqPtr = std::shared_ptr<ServeReq>;

struct Slot {
    cudaStream_t st = nullptr;
    cudaEvent_t done = nullptr;
    unsigned char* din = nullptr;         // one batch's inputs, packed: u, v, w, then the gridding data
    unsigned char* hin = nullptr;         // their pinned host staging copy (one H2D copy per batch)
    double *du = nullptr, *dv = nullptr, *dw = nullptr;  // the current batch's arrays inside din
    float2 *dvis = nullptr, *dout = nullptr;
    int32_t *diu = nullptr, *div = nullptr, *dco = nullptr;
    void* work = nullptr;
    size_t work_bytes = 0;
    float2* hout = nullptr;
    unsigned long long* hrej = nullptr;  // rejected counts of the grid and degrid plans
    std::vector<ReqPtr> reqs;           // the batch in flight (grid requests first)
    int64_t n_grid = 0;                 // samples of its grid requests
    int launch_status = TCV_OK;
    // executable graphs of earlier batches, by shape (gridding and degridding request counts),
    // updated in place by the next batch of the same shape
    std::vector<std::pair<uint64_t, cudaGraphExec_t>> execs;
    bool busy = false, launched = false;
    std::condition_variable cv;
    std::thread waiter;
};

}  // namespace

struct tcv_server {
    tcv_server_config cfg{};
    Clock::time_point t0;
    int support = 0, over_sample = 0;
    double w_cell = 0;
    int64_t c_len = 0;
    float c_scale = 1.f;
    float2* c64 = nullptr;
    void* c_alt = nullptr;
    double* dfreq = nullptr;
    void* scratch = nullptr;
    cudaStream_t io = nullptr;
    size_t held = 0;
    std::vector<float2*> grids;
    std::vector<int> grid_busy, pending_on;
    std::vector<std::unique_ptr<Slot>> slots;
    std::mutex mu;
    std::condition_variable cv_sched, cv_done;
    std::deque<ReqPtr> pending;
    std::unordered_map<uint64_t, ReqPtr> tickets;
    uint64_t next_id = 1, generation = 0;
    int64_t completed = 0, batches = 0;
    bool stop_sched = false, stop_waiters = false;
    std::thread scheduler;

    double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
    const void* table() const { return cfg.c_type == TCV_C_C64 ? static_cast<const void*>(c64) : c_alt; }
    size_t grid_bytes() const { return size_t(cfg.g_size) * cfg.g_size * sizeof(float2); }
};

namespace {

size_t slot_bytes(const tcv_server_config& c, size_t work)
{
    return size_t(c.batch_samples) * (3 * 8 + 8 + 3 * 4 + 8) + work;
}

// workspace of a batch plan over at most max_batch jobs and batch_samples samples
size_t slot_work_bytes(const tcv_server* s)
{
    std::vector<tcv_job> jobs(size_t(s->cfg.max_batch), tcv_job{0, s->cfg.g_size, reinterpret_cast<float*>(256)});
    jobs[0].n = s->cfg.batch_samples;
    return tcv_batch_workspace_bytes(jobs.data(), int(jobs.size()), s->support, s->c_len, &s->cfg.tuning);
}

tcv_status run_plan(tcv_server* s, Slot& sl, const std::vector<ReqPtr>& reqs, size_t from, size_t to, int64_t at,
                    bool degrid, unsigned long long* rej)
{
    std::vector<tcv_job> jobs;
    for (size_t i = from; i < to; ++i)
        jobs.push_back(tcv_job{reqs[i]->r.n, s->cfg.g_size, reinterpret_cast<float*>(s->grids[size_t(reqs[i]->r.grid)])});
    if (jobs.empty()) return TCV_OK;
    tcv_plan* p = nullptr;
    tcv_status st = tcv_batch_plan_create(&p, jobs.data(), int(jobs.size()), s->support, s->c_len, &s->cfg.tuning,
                                          sl.work, sl.work_bytes, sl.st);
    if (st != TCV_OK) return st;
    st = tcv_plan_bin(p, sl.diu + at, sl.div + at, sl.dco + at, sl.st);
    if (st == TCV_OK && !degrid)
        st = tcv_plan_grid(p, reinterpret_cast<const float*>(sl.dvis + at), s->table(), s->cfg.c_type, s->c_scale,
                           nullptr, sl.st);
    if (st == TCV_OK && degrid)
        st = tcv_plan_degrid(p, nullptr, s->table(), s->cfg.c_type, s->c_scale, reinterpret_cast<float*>(sl.dout + at),
                             sl.st);
    if (st == TCV_OK) st = tcv::cuda_status(cudaMemcpyAsync(rej, p->rejected, sizeof(*rej), cudaMemcpyDeviceToHost, sl.st));
    tcv_plan_destroy(p);  // host object only; its device arrays live in the slot's workspace
    return st;
}

// batches of at most this many requests are replayed as CUDA graphs (tcv_server_config.graphs)
constexpr int kGraphRequests = 4;

// stage and enqueue one batch on its slot (no lock held)
tcv_status launch(tcv_server* s, Slot& sl)
{
    const std::vector<ReqPtr>& reqs = sl.reqs;
    int64_t total = 0, n_grid = 0;
    size_t n_gr = 0;
    for (const ReqPtr& r : reqs) {
        if (r->r.kind == TCV_REQ_GRID) {
            n_grid += r->r.n;
            ++n_gr;
        }
        total += r->r.n;
    }
    sl.n_grid = n_grid;
    // pack the batch's inputs (u, v, w of every request, then the gridding requests' data) so that
    // one copy moves them
    double* hu = reinterpret_cast<double*>(sl.hin);
    double *hv = hu + total, *hw = hv + total;
    float2* hvis = reinterpret_cast<float2*>(hw + total);
    sl.du = reinterpret_cast<double*>(sl.din);
    sl.dv = sl.du + total;
    sl.dw = sl.dv + total;
    sl.dvis = reinterpret_cast<float2*>(sl.dw + total);
    int64_t at = 0;
    for (const ReqPtr& r : reqs) {
        const size_t b = size_t(r->r.n) * 8;
        if (r->r.n) {
            std::memcpy(hu + at, r->r.u, b);
            std::memcpy(hv + at, r->r.v, b);
            std::memcpy(hw + at, r->r.w, b);
            if (r->r.kind == TCV_REQ_GRID) std::memcpy(hvis + at, r->r.vis, b);
        }
        at += r->r.n;
    }
    sl.hrej[0] = sl.hrej[1] = 0;
    if (total <= 0) return TCV_OK;
    // the batch's device work: one H2D copy, offsets, the gridding plan and pass, the degridding
    // plan and pass, the D2H copies of the degridded samples and the rejected counts
    auto enqueue = [&]() -> tcv_status {
        TCV_CUDA(cudaMemcpyAsync(sl.din, sl.hin, size_t(3 * total + n_grid) * 8, cudaMemcpyHostToDevice, sl.st));
        tcv_status st = tcv_init_offsets_raw(sl.du, sl.dv, sl.dw, total, s->dfreq, 1, s->cfg.cell_size, s->w_cell,
                                             s->cfg.w_size, s->cfg.g_size, s->support, s->over_sample, sl.diu, sl.div,
                                             sl.dco, sl.st);
        if (st != TCV_OK) return st;
        st = run_plan(s, sl, reqs, 0, n_gr, 0, false, &sl.hrej[0]);
        if (st != TCV_OK) return st;
        st = run_plan(s, sl, reqs, n_gr, reqs.size(), n_grid, true, &sl.hrej[1]);
        if (st != TCV_OK) return st;
        if (total > n_grid)
            TCV_CUDA(cudaMemcpyAsync(sl.hout + n_grid, sl.dout + n_grid, size_t(total - n_grid) * 8,
                                     cudaMemcpyDeviceToHost, sl.st));
        return TCV_OK;
    };
    if (s->cfg.graphs && reqs.size() <= size_t(kGraphRequests)) {
        // Captured (this thread only) into a graph and launched once: the slot's executable graph
        // for this batch shape takes the new node parameters, or is built for a new shape.
        // Nothing runs while capturing, so a capture that fails falls back to launching the same
        // work one call at a time.  Only small batches go this way: they are the ones whose
        // latency the launches set, and under load the shapes vary too much for the graphs to be
        // reused (building one costs more host time than launching the work).
        if (cudaStreamBeginCapture(sl.st, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            const tcv_status st = enqueue();
            cudaGraph_t g = nullptr;
            const cudaError_t ec = cudaStreamEndCapture(sl.st, &g);
            if (st == TCV_OK && ec == cudaSuccess && g) {
                const uint64_t shape = (uint64_t(n_gr) << 32) | uint64_t(reqs.size() - n_gr);
                cudaGraphExec_t* ex = nullptr;
                for (auto& e : sl.execs)
                    if (e.first == shape) ex = &e.second;
                if (ex) {
                    cudaGraphExecUpdateResultInfo info{};
                    if (cudaGraphExecUpdate(*ex, g, &info) != cudaSuccess) {
                        cudaGetLastError();
                        cudaGraphExecDestroy(*ex);
                        *ex = nullptr;
                    }
                } else {
                    if (sl.execs.size() >= 16) {  // keep the 16 most recent shapes
                        cudaGraphExecDestroy(sl.execs.front().second);
                        sl.execs.erase(sl.execs.begin());
                    }
                    sl.execs.emplace_back(shape, nullptr);
                    ex = &sl.execs.back().second;
                }
                cudaError_t e = cudaSuccess;
                if (!*ex) e = cudaGraphInstantiate(ex, g, 0);
                cudaGraphDestroy(g);
                if (e == cudaSuccess) e = cudaGraphLaunch(*ex, sl.st);
                return tcv::cuda_status(e);
            }
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();  // the capture's error, if any: launch directly below
        } else {
            cudaGetLastError();
        }
    }
    return enqueue();
}

void scheduler_loop(tcv_server* s)
{
    cudaSetDevice(s->cfg.device);
    std::unique_lock<std::mutex> lk(s->mu);
    uint64_t seen = ~uint64_t(0);
    for (;;) {
        if (s->stop_sched) return;
        Slot* free_slot = nullptr;
        for (auto& sl : s->slots)
            if (!sl->busy) {
                free_slot = sl.get();
                break;
            }
        if (!free_slot || s->pending.empty() || seen == s->generation) {
            seen = s->generation;
            s->cv_sched.wait(lk, [&] { return s->stop_sched || s->generation != seen; });
            continue;
        }
        seen = s->generation;
        // form the batch: arrival order, one request per grid, none on a grid with work in flight
        std::vector<ReqPtr> grid_reqs, degrid_reqs;
        std::vector<char> blocked(s->grids.size(), 0);
        for (size_t g = 0; g < s->grids.size(); ++g) blocked[g] = s->grid_busy[g] > 0;
        int64_t total = 0;
        int count = 0;
        for (const ReqPtr& r : s->pending) {
            if (count >= s->cfg.max_batch) break;
            const size_t g = size_t(r->r.grid);
            if (blocked[g]) continue;
            blocked[g] = 1;
            if (total + r->r.n > s->cfg.batch_samples) continue;
            (r->r.kind == TCV_REQ_GRID ? grid_reqs : degrid_reqs).push_back(r);
            total += r->r.n;
            ++count;
        }
        if (count == 0) continue;  // everything waits on grids in flight: sleep until a change
        std::vector<ReqPtr> batch = grid_reqs;
        batch.insert(batch.end(), degrid_reqs.begin(), degrid_reqs.end());
        const double t = s->now();
        for (const ReqPtr& r : batch) {
            s->pending.erase(std::find(s->pending.begin(), s->pending.end(), r));
            --s->pending_on[size_t(r->r.grid)];
            ++s->grid_busy[size_t(r->r.grid)];
            r->t_start = t;
        }
        free_slot->busy = true;
        free_slot->reqs = batch;
        ++s->batches;
        lk.unlock();
        tcv_status st = launch(s, *free_slot);
        const cudaError_t e = cudaEventRecord(free_slot->done, free_slot->st);
        if (st == TCV_OK && e != cudaSuccess) st = tcv::cuda_status(e);
        lk.lock();
        free_slot->launch_status = st;
        free_slot->launched = true;
        free_slot->cv.notify_one();
        seen = ~uint64_t(0);  // look again at once: more requests may fit another free slot
    }
}

void waiter_loop(tcv_server* s, Slot* sl)
{
    cudaSetDevice(s->cfg.device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        sl->cv.wait(lk, [&] { return sl->launched || s->stop_waiters; });
        if (!sl->launched) return;
        const std::vector<ReqPtr> reqs = sl->reqs;
        int st = sl->launch_status;
        lk.unlock();
        const cudaError_t e = cudaEventSynchronize(sl->done);
        if (st == TCV_OK && e != cudaSuccess) st = tcv::cuda_status(e);
        int64_t at = sl->n_grid;
        for (const ReqPtr& r : reqs)
            if (r->r.kind == TCV_REQ_DEGRID) {
                if (st == TCV_OK && r->r.n) std::memcpy(r->r.vis_out, sl->hout + at, size_t(r->r.n) * 8);
                at += r->r.n;
            }
        const double t = s->now();
        const int64_t rej = int64_t(sl->hrej[0] + sl->hrej[1]);
        lk.lock();
        for (const ReqPtr& r : reqs) {
            r->t_done = t;
            r->status = st;
            r->rejected = rej;
            r->batch_requests = int(reqs.size());
            r->done = true;
            --s->grid_busy[size_t(r->r.grid)];
        }
        s->completed += int64_t(reqs.size());
        sl->reqs.clear();
        sl->launched = false;
        sl->busy = false;
        ++s->generation;
        s->cv_sched.notify_one();
        s->cv_done.notify_all();
    }
}

template <typename T>
cudaError_t dmalloc(T** p, size_t count, size_t& held)
{
    const size_t b = count * sizeof(T) + 256;
    const cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), b);
    if (e == cudaSuccess) held += b;
    return e;
}

template <typename T>
cudaError_t hmalloc(T** p, size_t count)
{
    return cudaMallocHost(reinterpret_cast<void**>(p), count * sizeof(T) + 256);
}

void free_server(tcv_server* s)
{
    for (auto& sl : s->slots) {
        if (sl->st) cudaStreamSynchronize(sl->st);
        void* d[] = {sl->din, sl->dout, sl->diu, sl->div, sl->dco, sl->work};
        for (void* p : d)
            if (p) cudaFree(p);
        void* h[] = {sl->hin, sl->hout, sl->hrej};
        for (void* p : h)
            if (p) cudaFreeHost(p);
        for (auto& e : sl->execs) cudaGraphExecDestroy(e.second);
        if (sl->done) cudaEventDestroy(sl->done);
        if (sl->st) cudaStreamDestroy(sl->st);
    }
    for (float2* g : s->grids)
        if (g) cudaFree(g);
    void* d[] = {s->c64, s->c_alt, s->dfreq, s->scratch};
    for (void* p : d)
        if (p) cudaFree(p);
    if (s->io) cudaStreamDestroy(s->io);
    delete s;
}

bool valid_grid(const tcv_server* s, int32_t g) { return g >= 0 && size_t(g) < s->grids.size() && s->grids[size_t(g)]; }

}  // namespace

extern "C" {

void tcv_server_config_default(tcv_server_config* c)
{
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->g_size = 1024;  // the CPU-sized problem: 1024^2 grid, 9 w-planes, 5 arcsec cells
    c->w_size = 9;
    c->cell_size = 1.0 / (1024 * 5.0 * 3.14159265358979323846 / 648000.0);
    c->baseline = 2000;
    c->c_type = TCV_C_R32;
    c->streams = 2;
    c->max_batch = 32;
    c->batch_samples = 262144;
    c->hbm_budget = size_t(150e9);
    // 8-row tiles: gridding on the tile kernels in 32-sample work units (a request's busy tiles
    // spread over the SMs), degridding on the sample-parallel kernel in 128-sample units
    c->tuning = tcv_tuning{8, 32, 32, 128, 2};
    c->device = 0;
    c->graphs = 1;
}

tcv_status tcv_server_create(const tcv_server_config* cfg, tcv_server** out)
{
    if (!cfg || !out) return TCV_ERR_ARG;
    *out = nullptr;
    tcv_server_config c = *cfg;
    if (c.streams == 0) c.streams = 2;
    if (c.max_batch == 0) c.max_batch = 32;
    if (c.batch_samples == 0) c.batch_samples = 262144;
    if (c.hbm_budget == 0) c.hbm_budget = size_t(150e9);
    if (c.tuning.tile_rows == 0) c.tuning.tile_rows = 16;
    if (c.tuning.group_mib == 0) c.tuning.group_mib = 32;
    const int ct = c.c_type;
    if (c.g_size < 2 || c.g_size > 32768 || c.w_size < 1 || !(c.cell_size > 0.0) || c.streams < 1 || c.streams > 8 ||
        c.max_batch < 1 || c.max_batch > 128 || c.batch_samples < 1 || c.batch_samples > (int64_t(1) << 26) ||
        tcv_ctype_bytes(ct) == 0 || (ct & (TCV_C_PADDED | TCV_C_PAIRED)) ||
        (c.tuning.tile_rows != 8 && c.tuning.tile_rows != 16 && c.tuning.tile_rows != 32) || c.tuning.group_mib < -1 ||
        c.tuning.split < 0 || c.tuning.degrid_split < 0)
        return TCV_ERR_ARG;
    tcv_server* s = new (std::nothrow) tcv_server;
    if (!s) return TCV_ERR_OOM;
    s->cfg = c;
    s->t0 = Clock::now();
    const double freq0 = 1.4e9 / 2.998e8;  // Benchmark.cc:89, channel 0
    tcv_status st = tcv_c_geometry(freq0, c.cell_size, c.baseline, c.w_size, &s->support, &s->over_sample, &s->w_cell,
                                   &s->c_len);
    if (st != TCV_OK) {
        delete s;
        return st;
    }
    cudaError_t e = cudaSetDevice(c.device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->io, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = dmalloc(&s->c64, size_t(s->c_len), s->held);
    if (e == cudaSuccess && ct != TCV_C_C64) {
        const size_t b = size_t(s->c_len) * tcv_ctype_bytes(ct) + 256;
        e = cudaMalloc(&s->c_alt, b);
        if (e == cudaSuccess) s->held += b;
    }
    if (e == cudaSuccess) e = dmalloc(&s->dfreq, 1, s->held);
    if (e == cudaSuccess) e = cudaMalloc(&s->scratch, tcv_init_c_scratch_bytes());
    if (e != cudaSuccess) {
        free_server(s);
        return tcv::cuda_status(e);
    }
    // the resident table (Benchmark::initC) in the served form
    float sum_c = 0.f;
    st = tcv_init_c_raw(freq0, c.cell_size, c.baseline, c.w_size, reinterpret_cast<float*>(s->c64), s->scratch,
                        &sum_c, s->io);
    if (st == TCV_OK && ct != TCV_C_C64)
        st = tcv_convert_c(reinterpret_cast<const float*>(s->c64), s->c_len, ct, s->c_alt, &s->c_scale, nullptr, s->io);
    if (st == TCV_OK) st = tcv::cuda_status(cudaMemcpyAsync(s->dfreq, &freq0, 8, cudaMemcpyHostToDevice, s->io));
    if (st == TCV_OK) st = tcv::cuda_status(cudaStreamSynchronize(s->io));
    cudaFree(s->scratch);
    s->scratch = nullptr;
    if (st != TCV_OK) {
        free_server(s);
        return st;
    }
    tcv::jit_prepare(ct, 2 * s->support + 1, c.tuning.tile_rows);
    // batch slots, admitted against the budget
    const size_t work = slot_work_bytes(s);
    if (work == 0 || s->held + size_t(c.streams) * slot_bytes(c, work) > c.hbm_budget) {
        free_server(s);
        return work == 0 ? TCV_ERR_UNSUPPORTED : TCV_ERR_OOM;
    }
    const size_t cap = size_t(c.batch_samples);
    for (int i = 0; i < c.streams && e == cudaSuccess; ++i) {
        s->slots.emplace_back(new Slot);
        Slot& sl = *s->slots.back();
        e = cudaStreamCreateWithFlags(&sl.st, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming);
        if (e == cudaSuccess) e = dmalloc(&sl.din, 32 * cap, s->held);
        if (e == cudaSuccess) e = dmalloc(&sl.dout, cap, s->held);
        if (e == cudaSuccess) e = dmalloc(&sl.diu, cap, s->held);
        if (e == cudaSuccess) e = dmalloc(&sl.div, cap, s->held);
        if (e == cudaSuccess) e = dmalloc(&sl.dco, cap, s->held);
        if (e == cudaSuccess) {
            e = cudaMalloc(&sl.work, work);
            if (e == cudaSuccess) {
                sl.work_bytes = work;
                s->held += work;
            }
        }
        if (e == cudaSuccess) e = hmalloc(&sl.hin, 32 * cap);
        if (e == cudaSuccess) e = hmalloc(&sl.hout, cap);
        if (e == cudaSuccess) e = hmalloc(&sl.hrej, 2);
    }
    if (e != cudaSuccess) {
        free_server(s);
        return tcv::cuda_status(e);
    }
    for (auto& sl : s->slots) sl->waiter = std::thread(waiter_loop, s, sl.get());
    s->scheduler = std::thread(scheduler_loop, s);
    *out = s;
    return TCV_OK;
}

void tcv_server_destroy(tcv_server* s)
{
    if (!s) return;
    {
        std::unique_lock<std::mutex> lk(s->mu);
        s->cv_done.wait(lk, [&] {
            if (!s->pending.empty()) return false;
            for (auto& sl : s->slots)
                if (sl->busy) return false;
            return true;
        });
        s->stop_sched = true;
        s->cv_sched.notify_all();
    }
    s->scheduler.join();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop_waiters = true;
        for (auto& sl : s->slots) sl->cv.notify_all();
    }
    for (auto& sl : s->slots) sl->waiter.join();
    cudaSetDevice(s->cfg.device);
    free_server(s);
}

tcv_status tcv_server_grid_alloc(tcv_server* s, int32_t* out)
{
    if (!s || !out) return TCV_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    const size_t b = s->grid_bytes();
    if (s->held + b > s->cfg.hbm_budget) return TCV_ERR_OOM;
    cudaSetDevice(s->cfg.device);
    float2* g = nullptr;
    TCV_CUDA(cudaMalloc(&g, b));
    const cudaError_t e = cudaMemsetAsync(g, 0, b, s->io);
    const cudaError_t e2 = cudaStreamSynchronize(s->io);
    if (e != cudaSuccess || e2 != cudaSuccess) {
        cudaFree(g);
        return tcv::cuda_status(e != cudaSuccess ? e : e2);
    }
    s->held += b;
    size_t id = 0;
    while (id < s->grids.size() && s->grids[id]) ++id;
    if (id == s->grids.size()) {
        s->grids.push_back(nullptr);
        s->grid_busy.push_back(0);
        s->pending_on.push_back(0);
    }
    s->grids[id] = g;
    *out = int32_t(id);
    return TCV_OK;
}

namespace {

// wait (lock held) until nothing is pending or in flight on grid g, then hold it busy
void hold_grid(tcv_server* s, std::unique_lock<std::mutex>& lk, int32_t g)
{
    s->cv_done.wait(lk, [&] { return s->grid_busy[size_t(g)] == 0 && s->pending_on[size_t(g)] == 0; });
    ++s->grid_busy[size_t(g)];
}

void release_grid(tcv_server* s, int32_t g)
{
    --s->grid_busy[size_t(g)];
    ++s->generation;
    s->cv_sched.notify_one();
    s->cv_done.notify_all();
}

}  // namespace

tcv_status tcv_server_grid_free(tcv_server* s, int32_t g)
{
    if (!s) return TCV_ERR_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    if (!valid_grid(s, g)) return TCV_ERR_ARG;
    hold_grid(s, lk, g);
    cudaSetDevice(s->cfg.device);
    cudaFree(s->grids[size_t(g)]);
    s->grids[size_t(g)] = nullptr;
    s->held -= s->grid_bytes();
    release_grid(s, g);
    return TCV_OK;
}

tcv_status tcv_server_grid_read(tcv_server* s, int32_t g, float* host)
{
    if (!s || !host) return TCV_ERR_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    if (!valid_grid(s, g)) return TCV_ERR_ARG;
    hold_grid(s, lk, g);
    float2* src = s->grids[size_t(g)];
    lk.unlock();
    cudaSetDevice(s->cfg.device);
    cudaError_t e = cudaMemcpyAsync(host, src, s->grid_bytes(), cudaMemcpyDeviceToHost, s->io);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->io);
    lk.lock();
    release_grid(s, g);
    return tcv::cuda_status(e);
}

tcv_status tcv_server_grid_write(tcv_server* s, int32_t g, const float* host)
{
    if (!s || !host) return TCV_ERR_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    if (!valid_grid(s, g)) return TCV_ERR_ARG;
    hold_grid(s, lk, g);
    float2* dst = s->grids[size_t(g)];
    lk.unlock();
    cudaSetDevice(s->cfg.device);
    cudaError_t e = cudaMemcpyAsync(dst, host, s->grid_bytes(), cudaMemcpyHostToDevice, s->io);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->io);
    lk.lock();
    release_grid(s, g);
    return tcv::cuda_status(e);
}

tcv_status tcv_server_submit(tcv_server* s, const tcv_request* req, uint64_t* ticket)
{
    if (!s || !req || !ticket) return TCV_ERR_ARG;
    const tcv_request& r = *req;
    if ((r.kind != TCV_REQ_GRID && r.kind != TCV_REQ_DEGRID) || r.n < 0) return TCV_ERR_ARG;
    if (r.n > 0 && (!r.u || !r.v || !r.w || (r.kind == TCV_REQ_GRID ? !r.vis : !r.vis_out))) return TCV_ERR_ARG;
    if (r.n > s->cfg.batch_samples) return TCV_ERR_UNSUPPORTED;
    auto q = std::make_shared<ServeReq>();
    q->r = r;
    std::lock_guard<std::mutex> lk(s->mu);
    if (!valid_grid(s, r.grid)) return TCV_ERR_ARG;
    q->t_submit = s->now();
    q->id = s->next_id++;
    s->pending.push_back(q);
    ++s->pending_on[size_t(r.grid)];
    s->tickets[q->id] = q;
    ++s->generation;
    s->cv_sched.notify_one();
    *ticket = q->id;
    return TCV_OK;
}

tcv_status tcv_server_wait(tcv_server* s, uint64_t ticket, double timeout_s, tcv_request_info* info)
{
    if (!s) return TCV_ERR_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->tickets.find(ticket);
    if (it == s->tickets.end()) return TCV_ERR_ARG;
    ReqPtr q = it->second;
    if (timeout_s < 0)
        s->cv_done.wait(lk, [&] { return q->done; });
    else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] { return q->done; }))
        return TCV_ERR_TIMEOUT;
    if (info) {
        info->status = q->status;
        info->batch_requests = q->batch_requests;
        info->rejected = q->rejected;
        info->t_submit = q->t_submit;
        info->t_start = q->t_start;
        info->t_done = q->t_done;
    }
    s->tickets.erase(it);
    return tcv_status(q->status);
}

tcv_status tcv_server_stats(const tcv_server* cs, size_t* bytes_held, int64_t* completed, int64_t* batches,
                            int64_t* pending)
{
    if (!cs) return TCV_ERR_ARG;
    tcv_server* s = const_cast<tcv_server*>(cs);
    std::lock_guard<std::mutex> lk(s->mu);
    if (bytes_held) *bytes_held = s->held;
    if (completed) *completed = s->completed;
    if (batches) *batches = s->batches;
    if (pending) *pending = int64_t(s->pending.size());
    return TCV_OK;
}

}  // extern "C"
