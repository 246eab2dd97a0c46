/*
 * tconvolve.h -- C ABI of the B200 (sm_100a) W-projection convolutional resampling library
 * (libtconvolve.so).  Plain pointers, sizes and status codes only: no C++ or torch types.
 *
 * Reference interfaces replaced (paths relative to the reference project root):
 *   - class Benchmark                       attic/tConvolveMPI/Benchmark.h:55-99
 *       Benchmark(), init(), runGrid(), runDegrid(), getSupport()  -> tcv_create, tcv_init,
 *       tcv_run_grid, tcv_run_degrid, tcv_support (context API below)
 *   - Benchmark::gridKernel / degridKernel  attic/tConvolveMPI/Benchmark.cc:125-195
 *   - cuda_gridKernel / cuda_degridKernel   attic/tConvolveCuda/CudaGridKernel.h:33-42
 *       (raw device-pointer kernels)       -> tcv_grid_raw, tcv_degrid_raw, tcv_plan_*
 *   - Benchmark::initC                      attic/tConvolveMPI/Benchmark.cc:206-270 -> tcv_c_geometry, tcv_init_c_raw
 *   - Benchmark::initCOffset                attic/tConvolveMPI/Benchmark.cc:281-324 -> tcv_init_offsets_raw
 *   - Benchmark::randomInt + init's u,v,w   attic/tConvolveMPI/Benchmark.cc:46-80   -> tcv_init_uvw_raw
 *
 * Data layout (identical to the reference's memory layout):
 *   complex values are interleaved float pairs (std::complex<float>, cuComplex);
 *   the grid is row-major [v][u], gSize x gSize;
 *   the table C is [k][osj][osi][j][i] flattened, entry index i + sSize*(j + sSize*(osi + os*(osj + os*k)));
 *   per-sample arrays (data, iu, iv, cOffset) are indexed dind = sample * nChan + chan.
 *   A sample grids onto columns iu-support .. iu+support and rows iv .. iv+2*support (the
 *   reference's footprint, Benchmark.cc:133).
 *
 * Errors: every call returns a tcv_status.  Calls taking a `stream` are asynchronous on that
 * stream (NULL = the legacy default stream) and validate host-visible arguments before launching;
 * samples whose footprint or table range falls outside the grid or table are counted as rejected
 * on the device and skipped (the reference has no checks and would write out of bounds).
 * tcv_plan_rejected reads that count; the context API turns it into TCV_ERR_BOUNDS.
 */
#ifndef TCONVOLVE_H
#define TCONVOLVE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum tcv_status {
    TCV_OK = 0,
    TCV_ERR_ARG = 1,        /* invalid argument: null pointer, bad size or type code */
    TCV_ERR_BOUNDS = 2,     /* one or more samples fell outside the grid or the table */
    TCV_ERR_OOM = 3,        /* device memory allocation failed */
    TCV_ERR_CUDA = 4,       /* a CUDA runtime or driver call failed */
    TCV_ERR_TIMEOUT = 5,    /* a bounded device-side wait gave up (status word set by a kernel) */
    TCV_ERR_STATE = 6,      /* call out of order, e.g. run_grid before init */
    TCV_ERR_WORKSPACE = 7,  /* caller-provided workspace smaller than required */
    TCV_ERR_UNSUPPORTED = 8 /* shape outside what the kernels handle (reported, never faked) */
} tcv_status;

/* Storage type of the convolution table C on the device. */
typedef enum tcv_ctype {
    TCV_C_C64 = 0,  /* complex64, the reference's std::complex<float> (8 B/entry): the plain form */
    TCV_C_R32 = 1,  /* real float (4 B/entry); exact when every imaginary part is zero (attic table) */
    TCV_C_CBF16 = 2,/* complex bfloat16 (4 B/entry) */
    TCV_C_RBF16 = 3,/* real bfloat16 (2 B/entry) */
    TCV_C_CF16 = 4, /* complex float16 x 2^e (4 B/entry), power-of-two scale passed as c_scale */
    TCV_C_RF16 = 5, /* real float16 x 2^e (2 B/entry) */
    /* Flag: the table is in the prepared (padded) layout made by tcv_prepare_table, rows of
     * sSize entries padded to a 16-byte pitch; the kernels then stream it with TMA. */
    TCV_C_PADDED = 0x100,
    /* Flag: the table is in the paired layout made by tcv_prepare_table: every kernel row stored
     * twice (as is, and shifted right by one column) with an even pitch, so that the tile
     * kernels read two columns per lane with one aligned load. */
    TCV_C_PAIRED = 0x200
} tcv_ctype;

const char *tcv_status_string(tcv_status s);
/* Bytes per table entry of a tcv_ctype (the TCV_C_PADDED flag is ignored), 0 for an unknown code. */
size_t tcv_ctype_bytes(int c_type);
/* Library version string and the compute capability it was built for ("sm_100a"). */
const char *tcv_version(void);

/* ------------------------------------------------------------------------------------------
 * Set-up functions (the untimed part of Benchmark::init)
 * ---------------------------------------------------------------------------------------- */

/* support, overSample, wCellSize and table length exactly as Benchmark::initC derives them
 * (attic/tConvolveMPI/Benchmark.cc:212-217, 226-230).  Host only. */
tcv_status tcv_c_geometry(double freq0, double cell_size, int baseline, int w_size,
                          int *support, int *over_sample, double *w_cell_size, int64_t *c_len);

/* Fill the table on the device: FP64 arithmetic for r^2 and the cos/exp w-term, float store,
 * then the reference's normalisation by a *sequential float* sum of |C| (Benchmark.cc:260-269),
 * so that the table matches the reference's.  d_c receives c_len complex64 entries.
 * d_scratch: device buffer of at least tcv_init_c_scratch_bytes() bytes.  *sum_c_out (host,
 * may be NULL) receives sumC after a stream synchronisation. */
size_t tcv_init_c_scratch_bytes(void);
tcv_status tcv_init_c_raw(double freq0, double cell_size, int baseline, int w_size, float *d_c,
                          void *d_scratch, float *sum_c_out, void *stream);

/* Convert the complex64 table into another storage type (TCV_C_R32 and the reduced forms).
 * *c_scale_out receives the factor the kernels must be given as c_scale (2^-e for the FP16
 * forms, 1 otherwise).  For the real forms the imaginary parts must be zero; *imag_nonzero_out
 * (may be NULL) receives the number of entries that were not (synchronises the stream). */
tcv_status tcv_convert_c(const float *d_c64, int64_t c_len, int c_type, void *d_out,
                         float *c_scale_out, int64_t *imag_nonzero_out, void *stream);

/* Bytes of a table of c_len entries in storage type c_type; with TCV_C_PADDED or TCV_C_PAIRED
 * set, in that prepared layout for footprints of sSize = 2*support+1 (0 if c_len is not a
 * multiple of sSize^2). */
size_t tcv_table_bytes(int64_t c_len, int support, int c_type);
/* Prepare a table for the faster kernels: convert the complex64 reference-layout table to storage
 * type c_type & 0xff (as tcv_convert_c) and write it to d_out in the layout the flag selects,
 * TCV_C_PADDED (TMA pipeline kernels) or TCV_C_PAIRED (two-columns-per-lane tile kernels);
 * tcv_table_bytes(c_len, support, c_type) bytes.  Set-up path: allocates a temporary for the
 * reduced forms and synchronises the stream.  Pass the result to the kernels with the same
 * c_type (flag included). */
tcv_status tcv_prepare_table(const float *d_c64, int64_t c_len, int support, int c_type,
                             void *d_out, float *c_scale_out, int64_t *imag_nonzero_out,
                             void *stream);

/* u, v, w for n_samples samples from the reference's K&R generator (Benchmark.cc:46-80), state0 =
 * generator state before the first draw (1 in the reference), computed in parallel by jump-ahead. */
tcv_status tcv_init_uvw_raw(int64_t n_samples, int baseline, uint64_t state0, double *d_u,
                            double *d_v, double *d_w, void *stream);

/* iu, iv, cOffset for n_samples x n_chan samples (Benchmark.cc:281-324), FP64 with the
 * reference's truncations.  d_freq: device array of n_chan inverse wavelengths. */
tcv_status tcv_init_offsets_raw(const double *d_u, const double *d_v, const double *d_w,
                                int64_t n_samples, const double *d_freq, int n_chan,
                                double cell_size, double w_cell_size, int w_size, int g_size,
                                int support, int over_sample, int32_t *d_iu, int32_t *d_iv,
                                int32_t *d_coff, void *stream);

/* ------------------------------------------------------------------------------------------
 * Raw device-pointer kernels (replace cuda_gridKernel / cuda_degridKernel)
 *
 * A plan bins samples into grid tiles (gridding) and anchor tiles (degridding) with a device
 * radix sort on (tile, w-plane/oversample kernel); it depends only on iu, iv, cOffset, so one
 * plan serves any number of grid and degrid passes over the same samples.  The plan lives in a
 * caller-provided device workspace of tcv_plan_workspace_bytes() bytes.
 * ---------------------------------------------------------------------------------------- */
typedef struct tcv_plan tcv_plan;

size_t tcv_plan_workspace_bytes(int64_t n, int support, int g_size, int64_t c_len);
/* Build (asynchronously) a plan for n samples.  *plan_out is a small host object; free it with
 * tcv_plan_destroy.  c_len: number of entries in the table (bounds for cOffset). */
tcv_status tcv_plan_build(tcv_plan **plan_out, const int32_t *d_iu, const int32_t *d_iv,
                          const int32_t *d_coff, int64_t n, int support, int g_size,
                          int64_t c_len, void *d_work, size_t work_bytes, void *stream);
/* grid += gridding of d_data (n complex64) with table d_c of type c_type (Benchmark.cc:125-155).
 * d_grid is NULL for a batched plan (each job's own grid). */
tcv_status tcv_plan_grid(const tcv_plan *plan, const float *d_data, const void *d_c, int c_type,
                         float c_scale, float *d_grid, void *stream);
/* d_data[n] = degridding of d_grid (Benchmark.cc:158-195); overwrites d_data.  d_grid is NULL
 * for a batched plan. */
tcv_status tcv_plan_degrid(const tcv_plan *plan, const float *d_grid, const void *d_c, int c_type,
                           float c_scale, float *d_data, void *stream);
/* Number of samples the plan rejected as out of bounds (synchronises the stream). */
tcv_status tcv_plan_rejected(const tcv_plan *plan, int64_t *rejected_out, void *stream);
/* TCV_ERR_TIMEOUT if a kernel run with this plan gave up a bounded wait, else TCV_OK
 * (synchronises the stream). */
tcv_status tcv_plan_status(const tcv_plan *plan, void *stream);
/* Degridding kernel for reference-layout tables: TCV_DEGRID_TILES (default; the adjoint of the
 * gridding tiles, grid values in registers) or TCV_DEGRID_ANCHOR (anchor tiles with the grid
 * region staged in shared memory by TMA).  Prepared (TCV_C_PADDED) tables always use the TMA
 * pipeline kernels. */
enum { TCV_DEGRID_TILES = 0, TCV_DEGRID_ANCHOR = 1 };
tcv_status tcv_plan_set_degrid_variant(tcv_plan *plan, int variant);
/* Tile geometry chosen for the plan: grid tile width/height, anchor tile, degrid mode
 * (0 = TMA-staged tiles, 1 = direct), number of grid tiles, max samples in one grid tile. */
tcv_status tcv_plan_info(const tcv_plan *plan, int *tile_w, int *tile_h, int *anchor,
                         int *degrid_mode, int *n_tiles);
void tcv_plan_destroy(tcv_plan *plan);

/* ------------------------------------------------------------------------------------------
 * Batched plans: many jobs (channels, Taylor terms) of uneven sample counts and grid sizes that
 * share one table, binned together so that a gridding or degridding pass over all of them is
 * one sequence of persistent launches.  No counterpart in the reference, which runs one job per
 * process (attic/tConvolveMPI/tConvolveMPI.cc:78-119) or per thread (attic/tConvolveMT).
 * ---------------------------------------------------------------------------------------- */
typedef struct tcv_job {
    int64_t n;     /* samples of the job; the jobs' samples are consecutive in the sample
                      arrays, job 0 first */
    int g_size;    /* side of the job's grid */
    float *d_grid; /* the job's grid, g_size^2 complex64 (device): gridding adds into it,
                      degridding reads it */
} tcv_job;

/* Tile shape and sort granularity of a plan (tcv_autotune chooses them by timing). */
typedef struct tcv_tuning {
    int tile_rows; /* grid rows per warp of the tile kernels: 8, 16 or 32, i.e. tiles of
                      64 x 4*tile_rows points; 0 = 16 */
    int group_mib; /* table slice per plane group, MiB of complex64 (whole w-planes, at least
                      one); 0 = 32; -1 = the whole table in one group */
    int split;     /* gridding: cells of at least 2*split samples are split into work units of
                      about split samples, so that a plan with few busy tiles still fills the GPU
                      (the units write partial tiles that are folded into the grid in unit
                      order); 0 = cells are never split */
    int degrid_split; /* the same for degridding (units need no fold there) */
    int kernel;    /* bit mask of the passes that use the sample-parallel kernels (one warp per
                      sample and tile region, lanes spread densely over the footprint; they win
                      for footprints up to a few tens wide; tile rows must be 8): 1 gridding,
                      2 degridding; 0 = the tile kernels (every lane owns grid columns).  Plans
                      with a bit set keep a 16-byte record per (sample, tile) pair. */
} tcv_tuning;

/* Workspace of a batched plan (0 for invalid arguments).  tuning may be NULL (defaults). */
size_t tcv_batch_workspace_bytes(const tcv_job *jobs, int n_jobs, int support, int64_t c_len,
                                 const tcv_tuning *tuning);
/* Create a batched plan in d_work: writes the job table to the device and numbers the jobs'
 * tiles.  Up to 128 jobs the table travels as a kernel argument (device work only, capturable);
 * beyond that it is copied from host memory (set-up path, not capturable).  Bin the samples with
 * tcv_plan_bin.  Gridding and degridding take d_grid = NULL and use the jobs' grids. */
tcv_status tcv_batch_plan_create(tcv_plan **plan_out, const tcv_job *jobs, int n_jobs, int support,
                                 int64_t c_len, const tcv_tuning *tuning, void *d_work,
                                 size_t work_bytes, void *stream);
/* Bin (or re-bin) the samples of a plan: device work only, safe to capture in a CUDA graph.
 * tcv_plan_build does this for a one-job plan. */
tcv_status tcv_plan_bin(tcv_plan *plan, const int32_t *d_iu, const int32_t *d_iv,
                        const int32_t *d_coff, void *stream);
/* The tuning a plan was made with. */
tcv_status tcv_plan_tuning(const tcv_plan *plan, tcv_tuning *tuning_out);

/* Autotuner: time every candidate tuning (tile_rows 8/16/32 x plane-group slices) on this batch,
 * each as one bin + grid + degrid pass into scratch grids the tuner allocates (the jobs' grids
 * are not touched), the median of reps passes after a warm-up, and return the fastest.  When the
 * jobs' grids exceed 2 GiB the passes run on an evenly spread subset of jobs.  Set-up path:
 * allocates, builds the specialised kernels it needs and synchronises.  The result is cached
 * for the process per (support, c_type, table size, job sizes). */
tcv_status tcv_autotune(const tcv_job *jobs, int n_jobs, const int32_t *d_iu, const int32_t *d_iv,
                        const int32_t *d_coff, const float *d_data, const void *d_c, int c_type,
                        float c_scale, int64_t c_len, int support, int reps,
                        tcv_tuning *best_out, float *best_ms_out, void *stream);
/* Candidates and median times (ms) of the last tcv_autotune run that timed (not a cache hit). */
tcv_status tcv_autotune_report(tcv_tuning *cands, float *ms, int max, int *n_out);

/* CUDA graph of the passes of one plan: bin (TCV_PASS_BIN), gridding (TCV_PASS_GRID) and
 * degridding into d_vis (TCV_PASS_DEGRID), in that order, captured once and replayed with one
 * launch.  d_grid: the grid of a one-job plan (NULL for a batched plan, whose jobs carry their
 * grids).  The pointers are baked into the graph.  Builds the specialised kernels before
 * capturing; a plan captured without TCV_PASS_BIN must be binned already. */
enum { TCV_PASS_BIN = 1, TCV_PASS_GRID = 2, TCV_PASS_DEGRID = 4 };
typedef struct tcv_graph tcv_graph;
tcv_status tcv_graph_capture(tcv_graph **graph_out, tcv_plan *plan, int passes,
                             const int32_t *d_iu, const int32_t *d_iv, const int32_t *d_coff,
                             const float *d_data, const void *d_c, int c_type, float c_scale,
                             float *d_grid, float *d_vis);
tcv_status tcv_graph_launch(const tcv_graph *graph, void *stream);
void tcv_graph_destroy(tcv_graph *graph);

/* ------------------------------------------------------------------------------------------
 * Serving: a request loop with continuous batching.  The server keeps the table and the grids
 * resident on one GPU; gridding and degridding requests (u, v, w in metres and visibilities in
 * host memory, one channel at the reference's first frequency, Benchmark.cc:89) queue on
 * submission, and a scheduler thread forms a batch whenever one of `streams` batch slots is
 * free: pending requests in arrival order, up to max_batch requests and batch_samples samples,
 * at most one request per grid per batch, requests on one grid in submission order (a grid with
 * a request in flight waits).  Each batch runs as batched plans (above) on its slot's stream, so
 * requests that arrive while others are on the GPU are admitted as slots free up and their work
 * overlaps.  Device memory is admitted against hbm_budget: the table, every batch slot's
 * buffers and every grid; a grid allocation that would exceed it fails with TCV_ERR_OOM.
 * A request's result is the same alone and in any mix (bit-identical: a job's sums do not
 * depend on the other jobs of its batch).  No counterpart in the reference, whose benchmark runs
 * one fixed problem per process (attic/tConvolveMPI/tConvolveMPI.cc:78-119).
 * ---------------------------------------------------------------------------------------- */
typedef struct tcv_server_config {
    int32_t g_size;        /* side of the served grids */
    int32_t w_size;        /* w-planes of the table (Benchmark::initC) */
    double cell_size;      /* cellSize in wavelengths */
    int32_t baseline;      /* metres */
    int32_t c_type;        /* table form the requests run with (TCV_C_R32 / TCV_C_C64 / ...) */
    int32_t streams;       /* batch slots in flight (default 2) */
    int32_t max_batch;     /* requests per batch (default 32, at most 128) */
    int64_t batch_samples; /* samples per batch; also the largest request (default 262144) */
    size_t hbm_budget;     /* device bytes the server may hold (default 150e9) */
    tcv_tuning tuning;     /* tile shape, plane groups, work units, sample-parallel passes
                              (default {8, 32, 32, 128, 2}) */
    int32_t device;
    int32_t graphs;        /* 1 (default): the copies and launches of a batch of up to 4
                              requests are captured and replayed as one CUDA graph launch (the
                              slot's executable graph for that batch shape is updated in place);
                              larger batches, and every batch when 0, are launched one by one */
} tcv_server_config;

enum { TCV_REQ_GRID = 0, TCV_REQ_DEGRID = 1 };
typedef struct tcv_request {
    int32_t kind;          /* TCV_REQ_GRID: grid += gridding of vis; TCV_REQ_DEGRID: vis_out = degridding */
    int32_t grid;          /* a grid id from tcv_server_grid_alloc */
    int64_t n;             /* samples (<= batch_samples) */
    const double *u, *v, *w; /* n positions in metres (host); must stay valid until the request completes */
    const float *vis;      /* TCV_REQ_GRID: n complex64 (host), valid until completion */
    float *vis_out;        /* TCV_REQ_DEGRID: n complex64 (host), written when the request completes */
} tcv_request;

typedef struct tcv_request_info {
    int32_t status;        /* tcv_status of the request */
    int32_t batch_requests;/* requests in the batch it ran in */
    int64_t rejected;      /* samples of its batch (all requests) left out as out of bounds */
    double t_submit, t_start, t_done; /* seconds since the server started: submission, batch
                                         launch, result ready (outputs on the host) */
} tcv_request_info;

typedef struct tcv_server tcv_server;
void tcv_server_config_default(tcv_server_config *cfg);
/* Allocates the table and the batch slots, starts the scheduler. */
tcv_status tcv_server_create(const tcv_server_config *cfg, tcv_server **out);
/* Drains the queue (every submitted request completes), stops the threads, frees everything. */
void tcv_server_destroy(tcv_server *srv);
tcv_status tcv_server_grid_alloc(tcv_server *srv, int32_t *grid_out);   /* a zeroed resident grid */
tcv_status tcv_server_grid_free(tcv_server *srv, int32_t grid);         /* after its requests */
tcv_status tcv_server_grid_read(tcv_server *srv, int32_t grid, float *host); /* waits for its requests */
tcv_status tcv_server_grid_write(tcv_server *srv, int32_t grid, const float *host);
/* Queue a request; *ticket_out identifies it.  TCV_ERR_UNSUPPORTED if n > batch_samples. */
tcv_status tcv_server_submit(tcv_server *srv, const tcv_request *req, uint64_t *ticket_out);
/* Wait up to timeout_s (< 0: no limit) for a request; TCV_ERR_TIMEOUT if it has not completed.
 * A completed request's info is returned (info may be NULL) and the ticket is released. */
tcv_status tcv_server_wait(tcv_server *srv, uint64_t ticket, double timeout_s, tcv_request_info *info);
/* Device bytes held (table + slots + grids), and counters. */
tcv_status tcv_server_stats(const tcv_server *srv, size_t *bytes_held, int64_t *completed,
                            int64_t *batches, int64_t *pending);

/* A one-job plan with a chosen tile shape and sort granularity (tcv_tuning, above; NULL for the
 * defaults, which tcv_plan_workspace_bytes / tcv_plan_build use).  The TMA pipeline and paired
 * kernel families need the default tile shape (TCV_ERR_UNSUPPORTED otherwise). */
size_t tcv_plan_workspace_bytes_tuned(int64_t n, int support, int g_size, int64_t c_len,
                                      const tcv_tuning *tuning);
tcv_status tcv_plan_build_tuned(tcv_plan **plan_out, const int32_t *d_iu, const int32_t *d_iv,
                                const int32_t *d_coff, int64_t n, int support, int g_size,
                                int64_t c_len, const tcv_tuning *tuning, void *d_work,
                                size_t work_bytes, void *stream);

/* Variable-width plans (the current/tConvolveMPI path, current/tConvolveMPI/Benchmark.cc:373-452):
 * every sample grids with the footprint width of its w-plane, s_size[d_wplane[k]] (odd), at
 * columns iu-s/2 .. and rows iv .. iv+s-1; the table holds the planes back to back from
 * c_off0[plane].  s_size and c_off0 are host arrays of n_planes.  Complex table forms only
 * (c64, cbf16, cf16: the w-term is complex); tuning as above, tile rows 8 or 16.  The plan
 * keeps d_wplane for re-binning with tcv_plan_bin. */
size_t tcv_plan_workspace_bytes_var(int64_t n, const int32_t *s_size, const int32_t *c_off0,
                                    int n_planes, int g_size, int64_t c_len,
                                    const tcv_tuning *tuning);
tcv_status tcv_plan_build_var(tcv_plan **plan_out, const int32_t *d_iu, const int32_t *d_iv,
                              const int32_t *d_coff, const int32_t *d_wplane, int64_t n,
                              const int32_t *s_size, const int32_t *c_off0, int n_planes,
                              int g_size, int64_t c_len, const tcv_tuning *tuning, void *d_work,
                              size_t work_bytes, void *stream);

/* Tile kernels specialised on the footprint width.  The first launch of the tile kernels for a
 * (table form, support) builds copies with sSize = 2*support+1 a compile-time constant (NVRTC,
 * about a second, cached for the process); tcv_jit_prepare builds them ahead of time (set-up;
 * call it before any stream capture).  If NVRTC is unavailable or a build fails, the generic
 * copies compiled into the library run instead.  tcv_jit_enable(0) forces the generic copies;
 * tcv_jit_info describes the current state. */
tcv_status tcv_jit_prepare(int c_type, int support);
void tcv_jit_enable(int enabled);
const char *tcv_jit_info(void);

/* One-call forms: plan_build + grid (or degrid) in the given workspace. */
tcv_status tcv_grid_raw(const float *d_data, int64_t n, int support, const void *d_c, int c_type,
                        float c_scale, int64_t c_len, const int32_t *d_coff, const int32_t *d_iu,
                        const int32_t *d_iv, float *d_grid, int g_size, void *d_work,
                        size_t work_bytes, void *stream);
tcv_status tcv_degrid_raw(const float *d_grid, int g_size, int support, const void *d_c,
                          int c_type, float c_scale, int64_t c_len, const int32_t *d_coff,
                          const int32_t *d_iu, const int32_t *d_iv, float *d_data, int64_t n,
                          void *d_work, size_t work_bytes, void *stream);

/* Gridding with no device allocation and no caller workspace, for callers that cannot
 * allocate: a pipeline running latency-critical work on other streams cannot accept the
 * device-wide synchronisation of cudaMalloc/cudaFree, and a host framework that manages all
 * device memory in its own pool forbids allocations it does not make.  No counterpart in the
 * reference (its gridders allocate per call, attic/tConvolveCuda/CudaGridder.cc:80-95).
 * Same arguments and result as tcv_grid_raw (grid += gridding of d_data), with the plan's
 * scratch in a fixed device array of tcv_static_scratch_bytes() (64 MiB) that every GPU loading
 * the library holds until exit.  A problem fits when tcv_plan_workspace_bytes(n, support,
 * g_size, c_len) <= tcv_static_scratch_bytes() (for a 129 x 129 footprint on a 4096 grid with
 * the 33-plane table: n <= 269,745); larger ones return TCV_ERR_WORKSPACE before any device
 * work.  The first call in a context of a device (the first on the device, and the first after
 * a cudaDeviceReset) looks up the array's device address (cudaGetSymbolAddress) and loads the
 * library's device code there: make it at set-up, before any stream capture.  The call never
 * compiles or loads a footprint-specialised kernel: it uses one only if tcv_jit_prepare built it
 * earlier, and the library's generic kernel otherwise (same sums).  All calls share the array:
 * calls that overlap on the GPU race and must be serialised by the caller. */
size_t tcv_static_scratch_bytes(void);
tcv_status tcv_grid_raw_static(const float *d_data, int64_t n, int support, const void *d_c,
                               int c_type, float c_scale, int64_t c_len, const int32_t *d_coff,
                               const int32_t *d_iu, const int32_t *d_iv, float *d_grid,
                               int g_size, void *stream);

/* ------------------------------------------------------------------------------------------
 * Host-buffer one-call forms (the reference's libCudaGridder seam,
 * attic/tConvolveCuda/CudaGridder.cc:54-207 behind CudaGridder.h:32-50): allocate, upload,
 * plan, run, download, free.  *device_seconds (may be NULL) receives the CUDA-event time of the
 * plan plus the kernel.  Returns TCV_ERR_BOUNDS (after computing the in-bounds samples) when
 * samples were skipped.
 * ---------------------------------------------------------------------------------------- */
tcv_status tcv_grid_host_raw(const float *data, int64_t n, int support, const float *c,
                             int64_t c_len, const int32_t *coff, const int32_t *iu,
                             const int32_t *iv, float *grid, int g_size, int device,
                             double *device_seconds);
tcv_status tcv_degrid_host_raw(const float *grid, int g_size, int support, const float *c,
                               int64_t c_len, const int32_t *coff, const int32_t *iu,
                               const int32_t *iv, float *data, int64_t n, int device,
                               double *device_seconds);
/* Benchmark::initC into host memory (computed on the device). */
tcv_status tcv_init_c_host(double freq0, double cell_size, int baseline, int w_size, float *c,
                           int64_t c_len, int device, int *support, int *over_sample,
                           double *w_cell_size, float *sum_c);

/* ------------------------------------------------------------------------------------------
 * Context API: the Benchmark object (attic/tConvolveMPI/Benchmark.h:55-99) with every buffer
 * resident on one GPU.  One context per host thread; calls on one context are serialised on
 * its stream.
 * ---------------------------------------------------------------------------------------- */
typedef struct tcv_config {
    int64_t n_samples;  /* nSamples (Benchmark.h:39) */
    int32_t w_size;     /* wSize (Benchmark.h:40) */
    int32_t n_chan;     /* nChan (Benchmark.h:41) */
    int32_t g_size;     /* gSize (Benchmark.h:44) */
    int32_t baseline;   /* baseline in metres (Benchmark.h:46) */
    double cell_size;   /* cellSize in wavelengths (Benchmark.h:45) */
    uint64_t seed;      /* generator start state = seed + 1; seed 0 reproduces the reference */
    int32_t c_type;     /* tcv_ctype used by run_grid / run_degrid (TCV_C_C64 = plain form) */
    int32_t device;     /* CUDA device ordinal */
} tcv_config;

typedef struct tcv_ctx tcv_ctx;

/* Fill *cfg with the reference defaults (attic/tConvolveMPI/Benchmark.h:39-46). */
void tcv_config_default(tcv_config *cfg);
tcv_status tcv_create(const tcv_config *cfg, tcv_ctx **ctx_out);
void tcv_destroy(tcv_ctx *ctx);
const char *tcv_last_error(const tcv_ctx *ctx);
/* Use an external stream (e.g. the caller's); NULL restores the context's own stream. */
tcv_status tcv_set_stream(tcv_ctx *ctx, void *stream);
void *tcv_get_stream(const tcv_ctx *ctx);
tcv_status tcv_sync(tcv_ctx *ctx);

/* Benchmark::init: u,v,w from the generator, data = 1+0i, grid = 0, freq, initC, initCOffset,
 * then the binning plan. */
tcv_status tcv_init(tcv_ctx *ctx);
/* Benchmark::runGrid: grid += gridding of the samples. */
tcv_status tcv_run_grid(tcv_ctx *ctx);
/* Benchmark::runDegrid: outdata = degridding of the grid. */
tcv_status tcv_run_degrid(tcv_ctx *ctx);
int tcv_support(const tcv_ctx *ctx);
int tcv_over_sample(const tcv_ctx *ctx);
double tcv_w_cell_size(const tcv_ctx *ctx);
float tcv_sum_c(const tcv_ctx *ctx);
int64_t tcv_c_len(const tcv_ctx *ctx);
int64_t tcv_n_data(const tcv_ctx *ctx);        /* nSamples * nChan */
double tcv_updates_per_pass(const tcv_ctx *ctx); /* nSamples * nChan * sSize^2 */
/* Switch the table storage type used by run_grid / run_degrid (converts once, keeps the C64 table). */
tcv_status tcv_set_ctype(tcv_ctx *ctx, int c_type);
/* Kernel family used by run_grid / run_degrid: the TMA pipeline kernels on the padded table,
 * the tile kernels that read the reference-layout table directly (default), or the
 * two-columns-per-lane tile kernels on the paired table. */
enum { TCV_PATH_TMA = 0, TCV_PATH_DIRECT = 1, TCV_PATH_PAIRED = 2 };
tcv_status tcv_set_path(tcv_ctx *ctx, int path);
int tcv_get_path(const tcv_ctx *ctx);
/* Tile shape and sort granularity of the context's plan (rebuilds the plan; the default is
 * {16, 32}).  tcv_tune times the candidates on the context's own samples, table form and grid
 * size (tcv_autotune, reps timed passes each) and keeps the fastest; *best_out and *best_ms_out
 * may be NULL.  Tile shapes other than the default need the direct path. */
tcv_status tcv_set_tuning(tcv_ctx *ctx, const tcv_tuning *tuning);
tcv_status tcv_get_tuning(const tcv_ctx *ctx, tcv_tuning *tuning_out);
tcv_status tcv_tune(tcv_ctx *ctx, int reps, tcv_tuning *best_out, float *best_ms_out);

/* Host <-> device transfers of the context's buffers (synchronous; host pointers). */
tcv_status tcv_set_data(tcv_ctx *ctx, const float *vis, int64_t n);          /* n complex */
tcv_status tcv_get_data(tcv_ctx *ctx, float *vis, int64_t n);                /* samples' data */
tcv_status tcv_get_outdata(tcv_ctx *ctx, float *vis, int64_t n);             /* degridded */
tcv_status tcv_set_grid(tcv_ctx *ctx, const float *grid);                    /* gSize^2 complex */
tcv_status tcv_get_grid(tcv_ctx *ctx, float *grid);
tcv_status tcv_zero_grid(tcv_ctx *ctx);
tcv_status tcv_get_c(tcv_ctx *ctx, float *c, int64_t n_entries);             /* complex64 table */
tcv_status tcv_get_offsets(tcv_ctx *ctx, int32_t *iu, int32_t *iv, int32_t *coff);
tcv_status tcv_get_uvw(tcv_ctx *ctx, double *u, double *v, double *w);
/* Replace u, v, w (host arrays of nSamples) and recompute offsets and plan. */
tcv_status tcv_set_uvw(tcv_ctx *ctx, const double *u, const double *v, const double *w);

/* Device pointers of the context's buffers, for callers that drive the raw API themselves. */
typedef struct tcv_device_buffers {
    float *data;      /* nSamples*nChan complex64 */
    float *outdata;   /* nSamples*nChan complex64 */
    float *grid;      /* gSize^2 complex64 */
    float *c64;       /* c_len complex64 */
    const void *c_active; /* table in the active c_type */
    int32_t *iu, *iv, *coff;
    double *u, *v, *w;
    const tcv_plan *plan;
    float c_scale;    /* c_scale to pass with c_active */
    int32_t c_type;   /* type code of c_active, TCV_C_PADDED set on the TMA path */
} tcv_device_buffers;
tcv_status tcv_get_device_buffers(tcv_ctx *ctx, tcv_device_buffers *out);

/* ------------------------------------------------------------------------------------------
 * The variable-support benchmark of current/tConvolveMPI: samples of a 12 h track of the
 * 36-antenna array (two generator draws each: baseline, hour angle), per-plane kernel widths and
 * complex W-projection kernels.  Run types (current/tConvolveMPI/Benchmark.cc:64-158): 0 continuum
 * (483 planes, widths 7..121, 6440^2 grid), 1 spectral line (135 planes, widths 7..19, 1034^2),
 * 2 nearest neighbour (1 x 1), 3 7 x 7 kernels, 4 87 x 87 kernels (4129^2, no w-projection).
 * ---------------------------------------------------------------------------------------- */
typedef struct tcv_cur_geometry {
    int32_t run_type, w_size, over_sample, support, g_size, n_baselines;
    int64_t n_samples, c_len; /* samples (one channel), table entries */
    int32_t s_min, s_max;     /* narrowest and widest plane */
    double w_cell_size, uv_cell_size;
} tcv_cur_geometry;
/* Host: the run type's constants, as the reference derives them. */
tcv_status tcv_cur_geometry_of(int run_type, tcv_cur_geometry *out);
/* Host: sSize and cOffset0 per plane (arrays of w_size). */
tcv_status tcv_cur_planes(int run_type, int32_t *s_size, int32_t *c_off0);
/* u, v, w of every sample from generator state state0 (1 for a fresh reference object);
 * *state_after (may be NULL) receives the state after the 2 * n_samples draws.  Synchronises. */
tcv_status tcv_cur_init_uvw_raw(int run_type, uint64_t state0, double *d_u, double *d_v, double *d_w,
                                uint64_t *state_after, void *stream);
/* The normalised complex64 table (c_len entries).  Synchronises. */
tcv_status tcv_cur_init_c_raw(int run_type, float *d_c, void *stream);
/* iu, iv, w-plane and cOffset per sample (d_s_size, d_c_off0: device copies of tcv_cur_planes). */
tcv_status tcv_cur_init_offsets_raw(int run_type, const double *d_u, const double *d_v,
                                    const double *d_w, int64_t n, const int32_t *d_s_size,
                                    const int32_t *d_c_off0, int32_t *d_iu, int32_t *d_iv,
                                    int32_t *d_wplane, int32_t *d_coff, void *stream);
/* Benchmark::requiredRate (current/tConvolveMPI/Benchmark.cc:697-739): rates[0] continuum,
 * rates[1] spectral line, pixels per second per process. */
void tcv_cur_required_rate(float *rates);

/* The Benchmark object of current/tConvolveMPI (current/tConvolveMPI/Benchmark.h:38-111) with its
 * buffers on one GPU.  As in the reference, init() may be called again after setRunType on the
 * same object, and the generator continues where the previous init() left it. */
typedef struct tcv_cur_ctx tcv_cur_ctx;
tcv_status tcv_cur_create(int device, tcv_cur_ctx **out);
void tcv_cur_destroy(tcv_cur_ctx *ctx);
const char *tcv_cur_last_error(const tcv_cur_ctx *ctx);
tcv_status tcv_cur_set_sort(tcv_cur_ctx *ctx, int sort);           /* setSort: 1 = by w-plane */
tcv_status tcv_cur_set_run_type(tcv_cur_ctx *ctx, int run_type);   /* setRunType */
int tcv_cur_get_run_type(const tcv_cur_ctx *ctx);
/* Table form of the passes: TCV_C_C64 (plain), TCV_C_CBF16 or TCV_C_CF16. */
tcv_status tcv_cur_set_ctype(tcv_cur_ctx *ctx, int c_type);
/* Tile height, plane-group slice and work units of the plan (tile_rows 0 = 16, or 8). */
tcv_status tcv_cur_set_tuning(tcv_cur_ctx *ctx, const tcv_tuning *tuning);
/* Time one gridding and one degridding pass of the initialised problem per candidate tuning
 * (median of reps, into scratch buffers: the context's grid and samples are left untouched) and
 * keep the fastest: kernel family x tile height x plane groups (with 256 / 128-sample work
 * units), then gridding work units, then degridding work units.  The candidates and their times are readable with tcv_autotune_report.  Set-up path:
 * allocates and synchronises. */
tcv_status tcv_cur_tune(tcv_cur_ctx *ctx, int reps, tcv_tuning *best_out, float *best_ms_out);
tcv_status tcv_cur_init(tcv_cur_ctx *ctx);       /* Benchmark::init */
tcv_status tcv_cur_run_grid(tcv_cur_ctx *ctx);   /* Benchmark::runGrid: grid += ... */
tcv_status tcv_cur_run_degrid(tcv_cur_ctx *ctx); /* Benchmark::runDegrid: outdata = ... */
tcv_status tcv_cur_sync(tcv_cur_ctx *ctx);
void *tcv_cur_get_stream(const tcv_cur_ctx *ctx);
int tcv_cur_support(const tcv_cur_ctx *ctx);                /* getSupport */
int64_t tcv_cur_n_visibilities(const tcv_cur_ctx *ctx);     /* nVisibilitiesGridded */
int64_t tcv_cur_n_pixels(const tcv_cur_ctx *ctx);           /* nPixelsGridded */
uint64_t tcv_cur_generator_state(const tcv_cur_ctx *ctx);
tcv_status tcv_cur_info(const tcv_cur_ctx *ctx, tcv_cur_geometry *g);
tcv_status tcv_cur_set_data(tcv_cur_ctx *ctx, const float *vis, int64_t n);
tcv_status tcv_cur_zero_grid(tcv_cur_ctx *ctx);
tcv_status tcv_cur_get_grid(tcv_cur_ctx *ctx, float *grid);
tcv_status tcv_cur_get_outdata(tcv_cur_ctx *ctx, float *vis, int64_t n);
tcv_status tcv_cur_get_c(tcv_cur_ctx *ctx, float *c, int64_t n_entries);
tcv_status tcv_cur_get_uvw(tcv_cur_ctx *ctx, double *u, double *v, double *w);
tcv_status tcv_cur_get_offsets(tcv_cur_ctx *ctx, int32_t *iu, int32_t *iv, int32_t *wplane,
                               int32_t *coff);
tcv_status tcv_cur_get_planes(const tcv_cur_ctx *ctx, int32_t *s_size, int32_t *c_off0);

/* ------------------------------------------------------------------------------------------
 * Hogbom CLEAN, the minor cycle (current/tHogbomCleanOMP/HogbomGolden.cc:47-141,
 * attic/tHogbomCleanCuda/HogbomCuda.cu:81-202; the same steps in current/tMajorACC/tMajorACC.cc:689-877).
 * Images are float, row-major, square: the dirty image and the residual width x width, the PSF
 * psf_width x psf_width.  Results are bit-identical to the reference's (its float roundings, no
 * fused multiply-adds).  The reference's PSF row index y - (ry - px) is kept; where it falls outside
 * the PSF (PSF peak off the diagonal) the reference reads out of bounds, here the row is skipped
 * and counted (tcv_hogbom_result).
 * ---------------------------------------------------------------------------------------- */
size_t tcv_hogbom_workspace_bytes(int width);
/* residual = dirty, then niters iterations (fewer once |peak| < threshold, HogbomGolden.cc:86-89;
 * threshold 0 never stops, as tMajorACC's loop): model[peak] += peak * gain; residual -= (gain *
 * peak) * shifted psf.  The model is accumulated into (the reference zeroes it first).  d_hist_val /
 * d_hist_pos (device, niters entries, may be NULL) receive each iteration's peak value and index.
 * Asynchronous on the stream: all iterations are issued without waiting; d_work must stay
 * allocated until they finish. */
tcv_status tcv_hogbom_deconvolve(const float *d_dirty, int width, const float *d_psf, int psf_width,
                                 float *d_model, float *d_residual, int niters, float gain,
                                 float threshold, float *d_hist_val, uint32_t *d_hist_pos,
                                 void *d_work, size_t work_bytes, void *stream);
/* How tcv_hogbom_deconvolve issues the iterations (process-wide): AUTO (default) runs images
 * whose residual and PSF fit in 48 MiB as one cooperative launch of all iterations (CTAs meet at a
 * bounded grid barrier per iteration) and larger ones as one launch per iteration; the other two
 * force either form.  Results are identical. */
enum { TCV_HOGBOM_AUTO = 0, TCV_HOGBOM_PER_LAUNCH = 1, TCV_HOGBOM_PERSISTENT = 2 };
void tcv_hogbom_set_strategy(int strategy);
/* The bounded waits of the cooperative form (process-wide, for launches made after the call):
 * limit_ns caps one grid-barrier wait (default and maximum 2e9 ns); withheld_arrivals (default 0)
 * raises every barrier's arrival target by that many CTAs that never arrive, so that every wait
 * runs out: a host-side hook that exercises the timeout path (the loop stops, every CTA returns,
 * tcv_hogbom_result reports TCV_ERR_TIMEOUT) without faulting or hanging the GPU.  Restore (2e9, 0)
 * afterwards.  The device-side counterpart of the reference's error accounting, which counts
 * disagreeing values instead of failing (attic/tConvolveBurnIn/tConvolveBurnIn.cc:94-107). */
tcv_status tcv_hogbom_set_wait(uint64_t limit_ns, uint32_t withheld_arrivals);
/* After tcv_hogbom_deconvolve (synchronises): iterations done, the iteration that met the
 * threshold (-1 if none), PSF rows skipped, the PSF peak index.  Any output may be NULL.
 * TCV_ERR_TIMEOUT if a grid-barrier wait of the persistent form gave up (the loop stopped). */
tcv_status tcv_hogbom_result(const void *d_work, int *iters_done, int *stopped_at,
                             int64_t *skipped_rows, int64_t *psf_peak_pos, void *stream);
/* findPeak (HogbomGolden.cc:127-139): the value of largest magnitude and its first index
 * (0 and 0 for an all-zero image).  Synchronises; d_work as for tcv_hogbom_deconvolve. */
tcv_status tcv_find_peak(const float *d_image, int64_t n, float *val_out, int64_t *pos_out,
                         void *d_work, size_t work_bytes, void *stream);

/* ------------------------------------------------------------------------------------------
 * FFT steps either side of gridding (current/tMajorACC/tMajorACC.cc:487-640).  Grids are square
 * complex64 of even size g_size (odd sizes: TCV_ERR_UNSUPPORTED, as the reference refuses them).
 * ---------------------------------------------------------------------------------------- */
/* fftExec / fftExecGPU: in place, rotate by half the size in both axes, unnormalised 2-D C2C
 * transform (forward: exp(-i..), else exp(+i..)), rotate back.  Single precision: this library's
 * own three-pass transform for power-of-two sizes 128 .. 8192 (the first call of a size on a device
 * makes its twiddle table and a g_size^2 complex scratch grid: set-up, allocates), cuFFT for other
 * even sizes. */
tcv_status tcv_fft_exec(float *d_grid, int g_size, int forward, void *stream);
/* fftFix / fftFixGPU: grid[i] = (Re grid[i] * scale, 0) for n complex values. */
tcv_status tcv_fft_fix(float *d_grid, int64_t n, float scale, void *stream);
/* The dirty-image step fused: d_image (float, g_size^2) = Re(fftExec(d_grid, backward)) * scale;
 * d_grid is used as scratch (overwritten). */
tcv_status tcv_image_from_grid(float *d_grid, int g_size, float scale, float *d_image, void *stream);
/* The model-to-grid step fused: d_grid = fftExec(complex(d_image), forward). */
tcv_status tcv_grid_from_image(const float *d_image, int g_size, float *d_grid, void *stream);

/* ------------------------------------------------------------------------------------------
 * The imaging major cycle of current/tMajorACC (tMajorACC.cc:889-1635) on one GPU: set-up as
 * there (samples, the delta convolution table of its initC, offsets, a 100-source sky and its
 * degridded visibilities), then per cycle: grid the PSF (first cycle), grid the data, inverse FFT
 * to the dirty image, Hogbom CLEAN (n_minor iterations, gain, no threshold), forward FFT of the
 * model, degrid, subtract the model visibilities from the data.
 * ---------------------------------------------------------------------------------------- */
typedef struct tcv_major_config {
    int64_t n_samples; /* 160000 */
    int w_size;        /* 33 */
    int n_chan;        /* 1 */
    double cell_size;  /* 5 wavelengths */
    int g_size;        /* 4096 (even) */
    int baseline;      /* 2000 m */
    int n_major;       /* 5 (the driver's loop count; tcv_major_run_cycle runs one) */
    int n_minor;       /* 100 */
    float gain;        /* 0.1 */
    int n_sources;     /* 100 */
    int device;
    int keep_stages;   /* 1: keep copies of the PSF and data uv grids (tcv_major_get_grid 0, 1) */
    tcv_tuning tuning; /* of the binning plan */
} tcv_major_config;
enum {
    TCV_MAJOR_PSF_GRID = 0, TCV_MAJOR_PSF_IFFT = 1, TCV_MAJOR_GRID = 2, TCV_MAJOR_IFFT = 3,
    TCV_MAJOR_HOGBOM = 4, TCV_MAJOR_FFT = 5, TCV_MAJOR_DEGRID = 6, TCV_MAJOR_SUBTRACT = 7,
    TCV_MAJOR_STAGES = 8
};
enum { TCV_IMG_PSF = 0, TCV_IMG_DIRTY = 1, TCV_IMG_RESIDUAL = 2, TCV_IMG_MODEL = 3 };
typedef struct tcv_major_ctx tcv_major_ctx;
void tcv_major_config_default(tcv_major_config *cfg);
tcv_status tcv_major_create(const tcv_major_config *cfg, tcv_major_ctx **out);
void tcv_major_destroy(tcv_major_ctx *ctx);
const char *tcv_major_last_error(const tcv_major_ctx *ctx);
void *tcv_major_get_stream(const tcv_major_ctx *ctx);
tcv_status tcv_major_init(tcv_major_ctx *ctx);      /* set-up; synchronises */
tcv_status tcv_major_run_cycle(tcv_major_ctx *ctx); /* one major cycle, asynchronous */
tcv_status tcv_major_sync(tcv_major_ctx *ctx);
/* Device time per stage summed over the cycles run (ms[TCV_MAJOR_STAGES]); synchronises. */
tcv_status tcv_major_stage_ms(tcv_major_ctx *ctx, double *ms, int *cycles);
tcv_status tcv_major_info(const tcv_major_ctx *ctx, int *support, int64_t *n_vis, int64_t *c_len,
                          float *scale);
/* Copies to host: images (TCV_IMG_*, float g_size^2), grids (0 PSF uv grid, 1 data uv grid, both
 * with keep_stages; 2 the model grid of the last cycle; complex64 g_size^2), visibilities
 * (0 the data, 1 the last model visibilities; complex64), offsets. */
tcv_status tcv_major_get_image(tcv_major_ctx *ctx, int which, float *out);
tcv_status tcv_major_get_grid(tcv_major_ctx *ctx, int which, float *out);
tcv_status tcv_major_get_vis(tcv_major_ctx *ctx, int which, float *out);
tcv_status tcv_major_get_offsets(tcv_major_ctx *ctx, int32_t *iu, int32_t *iv, int32_t *coff);

/* ------------------------------------------------------------------------------------------
 * Row-band split of one job over several GPUs (one process per GPU): rank b owns grid rows
 * [rows[b], rows[b+1]); a sample goes to the band of its footprint's centre row iv + support
 * (the footprint covers rows iv .. iv + 2*support, attic/tConvolveMPI/Benchmark.cc:137-150), so
 * its updates reach at most `support` rows past its band's edges, into the neighbouring band
 * (every band is at least `support` rows high).  These are the device steps; the host exchanges
 * the records (one all-to-all) and the halo rows (one send/receive per band edge) with NCCL.
 * No counterpart in the reference, whose ranks are independent replicas
 * (attic/tConvolveMPI/tConvolveMPI.cc:78-119).
 * ---------------------------------------------------------------------------------------- */
/* d_hist[r] += samples whose centre row (iv + support, clamped to the grid) is r; d_hist holds
 * g_size int64 counts, zeroed by the caller (then summed over the ranks). */
tcv_status tcv_band_histogram(const int32_t *d_iv, int64_t n, int support, int g_size, int64_t *d_hist,
                              void *stream);
/* Host arithmetic: rows_out[0..n_bands] with rows_out[0] = 0, rows_out[n_bands] = g_size, bound b
 * the first row where the histogram's samples below reach b/n_bands of the total, then moved
 * (up from the bottom, down from the top) so that every band is at least max(support, 1) rows
 * high.  TCV_ERR_ARG if n_bands is outside 1..64 or n_bands * max(support, 1) > g_size. */
tcv_status tcv_band_bounds(const int64_t *hist, int g_size, int support, int n_bands, int32_t *rows_out);
/* Workspace of tcv_band_bucket (0 for invalid arguments). */
size_t tcv_band_workspace_bytes(int64_t n, int n_bands);
/* Stable partition of n samples by band (rows: host array of n_bands + 1 bounds): records band
 * by band in input order, 5 int32 per sample (data re and im bits, iu, iv, cOffset), perm[j] =
 * the input index of record j, d_counts[b] (int64, device) = samples of band b.  n < 2^31. */
tcv_status tcv_band_bucket(const float *d_data, const int32_t *d_iu, const int32_t *d_iv,
                           const int32_t *d_coff, int64_t n, int support, int g_size,
                           const int32_t *rows, int n_bands, int32_t *d_records, int32_t *d_perm,
                           int64_t *d_counts, void *d_work, size_t work_bytes, void *stream);
/* Records -> complex64 data and the iu, iv, cOffset arrays. */
tcv_status tcv_band_unpack(const int32_t *d_records, int64_t n, float *d_data, int32_t *d_iu,
                           int32_t *d_iv, int32_t *d_coff, void *stream);
/* d_dst[perm[i]] = d_src[i] for n complex64 values. */
tcv_status tcv_band_scatter(const float *d_src, const int32_t *d_perm, int64_t n, float *d_dst,
                            void *stream);
/* d_dst += d_src over n_complex complex64 values (a received halo into the owner's rows). */
tcv_status tcv_rows_add(float *d_dst, const float *d_src, int64_t n_complex, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* TCONVOLVE_H */
