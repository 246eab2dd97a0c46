// tcv_batch.cu -- CUDA graphs of a plan's passes and the autotuner of the tile shape and the
// sort granularity.
//
// A batched step (bin + one persistent launch per plane group for gridding + the same for
// degridding + the slot sum) is a few dozen launches; captured once into a CUDA graph it is
// replayed with one launch and no host work.  The autotuner times the candidate tunings
// (rows per warp 8/16/32, i.e. tiles of 64 x 32/64/128 points, and plane-group slices of
// 8/16/32/64 MiB or the whole table; then gridding and degridding work units of 512/256/128/64
// samples for busy cells; then the sample-parallel degridding kernel on 8-row tiles in 256- and
// 128-sample units) on the caller's own batch, into scratch grids, and keeps the fastest.  Neither has a
// counterpart in the reference, whose kernels run one job per call
// (attic/tConvolveMPI/Benchmark.cc:98-106).
#include "tcv_internal.cuh"

#include <algorithm>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <vector>

struct tcv_graph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

using namespace tcv;

namespace {

std::mutex g_tune_mu;
std::map<std::string, std::pair<tcv_tuning, float>> g_tune_cache;
std::vector<std::pair<tcv_tuning, float>> g_report;

constexpr size_t kTuneGridBudget = size_t(8) << 30;  // scratch grids of the timed subset

// the passes in order on one stream (captured or not)
tcv_status run_passes(tcv_plan* plan, int passes, const int32_t* d_iu, const int32_t* d_iv, const int32_t* d_coff,
                      const float* d_data, const void* d_c, int c_type, float c_scale, float* d_grid, float* d_vis,
                      cudaStream_t st)
{
    tcv_status s = TCV_OK;
    if (passes & TCV_PASS_BIN) s = plan_bin(plan, d_iu, d_iv, d_coff, st);
    if (s == TCV_OK && (passes & TCV_PASS_GRID)) s = tcv_plan_grid(plan, d_data, d_c, c_type, c_scale, d_grid, st);
    if (s == TCV_OK && (passes & TCV_PASS_DEGRID)) s = tcv_plan_degrid(plan, d_grid, d_c, c_type, c_scale, d_vis, st);
    return s;
}

std::string tune_key(const tcv_job* jobs, int n_jobs, int support, int c_type, int64_t c_len)
{
    std::string k = std::to_string(support) + "/" + std::to_string(c_type) + "/" + std::to_string(c_len);
    for (int j = 0; j < n_jobs; ++j) k += "/" + std::to_string(jobs[j].n) + "x" + std::to_string(jobs[j].g_size);
    return k;
}

// RAII holder of the tuner's device allocations
struct DevBuf {
    void* p = nullptr;
    ~DevBuf()
    {
        if (p) cudaFree(p);
    }
    tcv_status alloc(size_t bytes)
    {
        if (bytes == 0) bytes = 256;
        return cuda_status(cudaMalloc(&p, bytes));
    }
};

}  // namespace

void tcv::tune_report_set(const std::vector<std::pair<tcv_tuning, float>>& report)
{
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_report = report;
}

extern "C" {

tcv_status tcv_graph_capture(tcv_graph** graph_out, tcv_plan* plan, int passes, const int32_t* d_iu,
                             const int32_t* d_iv, const int32_t* d_coff, const float* d_data, const void* d_c,
                             int c_type, float c_scale, float* d_grid, float* d_vis)
{
    if (!graph_out || !plan || passes <= 0 || (passes & ~7)) return TCV_ERR_ARG;
    if (tcv_ctype_bytes(c_type) == 0) return TCV_ERR_ARG;
    if (!(passes & TCV_PASS_BIN) && !plan->binned) return TCV_ERR_STATE;
    if (plan->batch ? d_grid != nullptr : d_grid == nullptr) return TCV_ERR_ARG;
    if ((passes & TCV_PASS_DEGRID) && plan->g.n > 0 && !d_vis) return TCV_ERR_ARG;
    if (!(c_type & (TCV_C_PADDED | TCV_C_PAIRED))) jit_prepare(c_type, plan->g.s, plan->g.rows);
    tcv_graph* g = new (std::nothrow) tcv_graph{};
    if (!g) return TCV_ERR_OOM;
    cudaStream_t cs = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete g;
        return cuda_status(e);
    }
    e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    tcv_status s = cuda_status(e);
    if (s == TCV_OK) {
        s = run_passes(plan, passes, d_iu, d_iv, d_coff, d_data, d_c, c_type, c_scale, d_grid, d_vis, cs);
        const cudaError_t ee = cudaStreamEndCapture(cs, &g->graph);  // ends the capture on every path
        if (s == TCV_OK) s = cuda_status(ee);
    }
    if (s == TCV_OK) s = cuda_status(cudaGraphInstantiate(&g->exec, g->graph, 0));
    cudaStreamDestroy(cs);
    if (s != TCV_OK) {
        cudaGetLastError();
        tcv_graph_destroy(g);
        return s;
    }
    *graph_out = g;
    return TCV_OK;
}

tcv_status tcv_graph_launch(const tcv_graph* graph, void* stream)
{
    if (!graph || !graph->exec) return TCV_ERR_ARG;
    return cuda_status(cudaGraphLaunch(graph->exec, static_cast<cudaStream_t>(stream)));
}

void tcv_graph_destroy(tcv_graph* graph)
{
    if (!graph) return;
    if (graph->exec) cudaGraphExecDestroy(graph->exec);
    if (graph->graph) cudaGraphDestroy(graph->graph);
    delete graph;
}

tcv_status tcv_autotune(const tcv_job* jobs, int n_jobs, const int32_t* d_iu, const int32_t* d_iv,
                        const int32_t* d_coff, const float* d_data, const void* d_c, int c_type, float c_scale,
                        int64_t c_len, int support, int reps, tcv_tuning* best_out, float* best_ms_out, void* stream)
{
    if (!jobs || n_jobs < 1 || !d_c || !best_out || support < 0 || c_len < 1 || reps < 1) return TCV_ERR_ARG;
    if (tcv_ctype_bytes(c_type) == 0 || (c_type & (TCV_C_PADDED | TCV_C_PAIRED))) return TCV_ERR_ARG;
    int64_t n_all = 0;
    for (int j = 0; j < n_jobs; ++j) {
        if (jobs[j].n < 0 || jobs[j].g_size < 1) return TCV_ERR_ARG;
        n_all += jobs[j].n;
    }
    if (n_all > 0 && (!d_iu || !d_iv || !d_coff || !d_data)) return TCV_ERR_ARG;
    reps = std::min(reps, 50);
    std::lock_guard<std::mutex> lock(g_tune_mu);
    const std::string key = tune_key(jobs, n_jobs, support, c_type, c_len);
    auto hit = g_tune_cache.find(key);
    if (hit != g_tune_cache.end()) {
        *best_out = hit->second.first;
        if (best_ms_out) *best_ms_out = hit->second.second;
        return TCV_OK;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    // the timed subset: every job when their grids fit the budget, else evenly spread jobs
    std::vector<int> pick;
    size_t grid_bytes = 0;
    for (int j = 0; j < n_jobs; ++j) grid_bytes += size_t(jobs[j].g_size) * jobs[j].g_size * 8;
    const int stride = int(std::max<size_t>(1, (grid_bytes + kTuneGridBudget - 1) / kTuneGridBudget));
    for (int j = 0; j < n_jobs; j += stride) pick.push_back(j);
    std::vector<int64_t> first(size_t(n_jobs) + 1, 0);
    for (int j = 0; j < n_jobs; ++j) first[size_t(j) + 1] = first[size_t(j)] + jobs[j].n;
    int64_t n_sub = 0;
    size_t sub_grid = 0;
    for (int j : pick) {
        n_sub += jobs[j].n;
        sub_grid += size_t(jobs[j].g_size) * jobs[j].g_size * 8;
    }
    DevBuf grids, samples, vis, work;
    TCV_CUDA(cudaStreamSynchronize(st));
    tcv_status s = grids.alloc(sub_grid);
    if (s == TCV_OK) s = samples.alloc(size_t(n_sub) * 20 + 1024);
    if (s == TCV_OK) s = vis.alloc(size_t(n_sub) * 8);
    if (s != TCV_OK) return s;
    TCV_CUDA(cudaMemsetAsync(grids.p, 0, sub_grid, st));
    // gather the subset's samples (job ranges are contiguous in the caller's arrays)
    int32_t* s_iu = static_cast<int32_t*>(samples.p);
    int32_t* s_iv = s_iu + n_sub;
    int32_t* s_co = s_iv + n_sub;
    float* s_data = reinterpret_cast<float*>(reinterpret_cast<char*>(samples.p) +
                                             ((size_t(n_sub) * 12 + 255) / 256) * 256);
    std::vector<tcv_job> sub;
    int64_t at = 0;
    size_t goff = 0;
    for (int j : pick) {
        const int64_t n = jobs[j].n, f = first[size_t(j)];
        if (n > 0) {
            TCV_CUDA(cudaMemcpyAsync(s_iu + at, d_iu + f, size_t(n) * 4, cudaMemcpyDeviceToDevice, st));
            TCV_CUDA(cudaMemcpyAsync(s_iv + at, d_iv + f, size_t(n) * 4, cudaMemcpyDeviceToDevice, st));
            TCV_CUDA(cudaMemcpyAsync(s_co + at, d_coff + f, size_t(n) * 4, cudaMemcpyDeviceToDevice, st));
            TCV_CUDA(cudaMemcpyAsync(s_data + 2 * at, d_data + 2 * f, size_t(n) * 8, cudaMemcpyDeviceToDevice, st));
        }
        sub.push_back(tcv_job{n, jobs[j].g_size,
                              reinterpret_cast<float*>(static_cast<char*>(grids.p) + goff)});
        at += n;
        goff += size_t(jobs[j].g_size) * jobs[j].g_size * 8;
    }

    // stage 1: tile shape x plane groups, cells whole; slices that give the same grouping are
    // timed once.  Stage 2: work-unit sizes on the stage-1 winner.
    std::vector<tcv_tuning> cands;
    std::vector<std::pair<int, int>> seen;  // (rows, kid_group)
    const int gs_max = [&] {
        int m = 1;
        for (const tcv_job& jb : sub) m = std::max(m, jb.g_size);
        return m;
    }();
    for (int rows : {16, 8, 32})
        for (int mib : {32, 16, 64, 8, -1}) {
            const tcv_tuning t{rows, mib, 0, 0};
            const PlanGeom g = make_geom(n_sub, support, &gs_max, 1, c_len, &t, false);
            const std::pair<int, int> id(rows, g.kid_group);
            if (std::find(seen.begin(), seen.end(), id) != seen.end()) continue;
            seen.push_back(id);
            cands.push_back(t);
        }

    cudaEvent_t e0 = nullptr, e1 = nullptr;
    TCV_CUDA(cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return TCV_ERR_CUDA;
    }
    std::vector<std::pair<tcv_tuning, float>> report;
    tcv_tuning best{16, 32, 0, 0};
    float best_ms = -1.f;
    size_t have = 0;
    auto time_one = [&](const tcv_tuning& t) -> tcv_status {
        const size_t need = tcv_batch_workspace_bytes(sub.data(), int(sub.size()), support, c_len, &t);
        if (need == 0) return TCV_ERR_UNSUPPORTED;
        if (need > have) {
            TCV_CUDA(cudaStreamSynchronize(st));
            if (work.p) cudaFree(work.p);
            work.p = nullptr;
            have = 0;
            const tcv_status a = work.alloc(need);
            if (a != TCV_OK) return a;
            have = need;
        }
        jit_prepare(c_type, 2 * support + 1, t.tile_rows);
        tcv_plan* plan = nullptr;
        tcv_status r = tcv_batch_plan_create(&plan, sub.data(), int(sub.size()), support, c_len, &t, work.p, have, st);
        if (r != TCV_OK) return r;
        std::vector<float> ms;
        for (int k = 0; k <= reps && r == TCV_OK; ++k) {  // pass 0 warms up
            cudaEventRecord(e0, st);
            r = run_passes(plan, TCV_PASS_BIN | TCV_PASS_GRID | TCV_PASS_DEGRID, s_iu, s_iv, s_co, s_data, d_c,
                           c_type, c_scale, nullptr, static_cast<float*>(vis.p), st);
            cudaEventRecord(e1, st);
            if (r == TCV_OK) r = cuda_status(cudaEventSynchronize(e1));
            float m = 0.f;
            if (r == TCV_OK) cudaEventElapsedTime(&m, e0, e1);
            if (k > 0) ms.push_back(m);
        }
        tcv_plan_destroy(plan);
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
    for (const tcv_tuning& t : cands)
        if ((s = time_one(t)) != TCV_OK) break;
    if (s == TCV_OK) {  // stage 2: gridding units
        const tcv_tuning base = best;
        for (int split : {512, 256, 128, 64})
            if ((s = time_one(tcv_tuning{base.tile_rows, base.group_mib, split, 0})) != TCV_OK) break;
    }
    if (s == TCV_OK) {  // stage 3: degridding units
        const tcv_tuning base = best;
        for (int split : {512, 256, 128, 64})
            if ((s = time_one(tcv_tuning{base.tile_rows, base.group_mib, base.split, split})) != TCV_OK) break;
    }
    if (s == TCV_OK) {  // stage 4: the sample-parallel degridding kernel (8-row tiles), for narrow footprints
        const tcv_tuning base = best;
        for (int split : {256, 128})
            if ((s = time_one(tcv_tuning{8, base.group_mib, base.split, split, 2})) != TCV_OK) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (s != TCV_OK) return s;
    g_report = report;
    g_tune_cache[key] = std::make_pair(best, best_ms);
    *best_out = best;
    if (best_ms_out) *best_ms_out = best_ms;
    return TCV_OK;
}

tcv_status tcv_autotune_report(tcv_tuning* cands, float* ms, int max, int* n_out)
{
    if (!n_out || max < 0 || (max > 0 && (!cands || !ms))) return TCV_ERR_ARG;
    std::lock_guard<std::mutex> lock(g_tune_mu);
    const int n = std::min(max, int(g_report.size()));
    for (int i = 0; i < n; ++i) {
        cands[i] = g_report[size_t(i)].first;
        ms[i] = g_report[size_t(i)].second;
    }
    *n_out = int(g_report.size());
    return TCV_OK;
}

}  // extern "C"
