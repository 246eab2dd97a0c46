/*
 * tconvolve_oracle.c -- CPU restatement of the tConvolve W-projection resampling path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker: only tests/, the smoke check of
 * __graft_entry__ and the cpu_baseline leg of bench.py may load it.  The product (the CUDA
 * library under askap-benchmarks_b200/) never links, calls or falls back to it.
 *
 * Parity status: pinned.  The FP32 functions reproduce the reference's arithmetic operation by
 * operation (same double expressions, same float rounding points, same sequential float sums),
 * and tests/test_oracle.py checks them bit for bit against outputs of the reference's own
 * attic/tConvolveMPI/Benchmark.cc, compiled from source by oracle/Makefile into oracle/_ref/
 * (fixtures in tests/golden/, generator tests/golden/make_golden.py).
 *
 * Every function cites the reference lines it restates (paths relative to the reference
 * project root).  Complex values are interleaved float (re, im) pairs, exactly the memory
 * layout of std::complex<float>.
 *
 * Build: gcc -O3 -fstrict-aliasing -fcx-limited-range -ffp-contract=off -fPIC -shared
 * (-ffp-contract=off keeps x*y+z as two roundings, as the reference's x86-64 build does).
 */
#include <stdint.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <limits.h>
#include <pthread.h>

#define ORC_MAXINT 2147483647u

/* ---------------------------------------------------------------------------------------------
 * Random sample coordinates.
 * attic/tConvolveMPI/Benchmark.cc:46-58 (K&R linear congruential generator on an unsigned long
 * state that starts at 1) and :69-80 (u, v, w drawn in that order per sample).
 * `state` is the generator state before the first draw (1 for the reference).
 * ------------------------------------------------------------------------------------------- */
int orc_random_int(uint64_t *state)
{
    *state = *state * 1103515245ull + 12345ull;
    return (int)((unsigned int)(*state / 65536ull) % ORC_MAXINT);
}

void orc_init_uvw(int64_t n_samples, int baseline, uint64_t state,
                  double *u, double *v, double *w)
{
    const double maxint = (double)ORC_MAXINT;
    const double half = (double)(baseline / 2); /* integer division, as in the reference */
    for (int64_t i = 0; i < n_samples; ++i) {
        u[i] = (double)baseline * (double)orc_random_int(&state) / maxint - half;
        v[i] = (double)baseline * (double)orc_random_int(&state) / maxint - half;
        w[i] = (double)baseline * (double)orc_random_int(&state) / maxint - half;
    }
}

/* freq[c] = (1.4e9 - 2e5 * c / nChan) / 2.998e8 : attic/tConvolveMPI/Benchmark.cc:86-90 */
void orc_init_freq(int n_chan, double *freq)
{
    for (int i = 0; i < n_chan; ++i)
        freq[i] = (1.4e9 - 2.0e5 * (double)i / (double)n_chan) / 2.998e8;
}

/* ---------------------------------------------------------------------------------------------
 * Geometry of the convolution table.  attic/tConvolveMPI/Benchmark.cc:212-217.
 * ------------------------------------------------------------------------------------------- */
void orc_c_geometry(double freq0, double cell_size, int baseline, int w_size,
                    int *support, int *over_sample, double *w_cell_size)
{
    *support = (int)(1.5 * sqrt((double)abs(baseline) * cell_size * freq0) / cell_size);
    *over_sample = 8;
    *w_cell_size = (double)(2 * baseline) * freq0 / (double)w_size;
}

/* ---------------------------------------------------------------------------------------------
 * Unnormalised table value for one entry, in double.  attic/tConvolveMPI/Benchmark.cc:236-258:
 * w is the plane index k - wSize/2 (not wavelengths); r2 uses the oversampled offsets; the
 * table is cos(r2 / (w * fScale)) off the w = 0 plane and exp(-r2) on it.
 * ------------------------------------------------------------------------------------------- */
static double orc_c_raw(int k, int osj, int osi, int j, int i, int w_size, int over_sample,
                        int s_size, double w_cell_size, double freq0, double cell_size)
{
    const int c_center = (s_size - 1) / 2;
    const double w = (double)(k - w_size / 2);
    const double f_scale = sqrt(fabs(w) * w_cell_size * freq0) / cell_size;
    const double dj = (double)(j - c_center) + (double)osj / (double)over_sample;
    const double di = (double)(i - c_center) + (double)osi / (double)over_sample;
    const double r2 = dj * dj + di * di; /* pow(x, 2) == x*x exactly for these multiples of 1/8 */
    if (w != 0.0)
        return cos(r2 / (w * f_scale));
    return exp(-r2);
}

/*
 * Build the FP32 table C (interleaved complex64, layout [k][osj][osi][j][i], index
 * i + sSize*(j + sSize*(osi + os*(osj + os*k))), Benchmark.cc:247) and normalise it the way
 * Benchmark.cc:260-269 does: a sequential *float* sum of |C| (which saturates at 2^24 for the
 * 35 M entry default table), then C *= float(wSize*os*os) / sumC in float.
 * If c64 is non-NULL it receives the same table in double (real parts only; imaginary parts are
 * zero in this form), normalised by the same reference constant computed in double:
 * c64 = raw * (wSize*os*os / (double)sumC).  Returns sumC.
 */
float orc_init_c(double freq0, double cell_size, int baseline, int w_size,
                 float *c, double *c64, int *support_out, int *over_sample_out,
                 double *w_cell_size_out)
{
    int support, os;
    double wcs;
    orc_c_geometry(freq0, cell_size, baseline, w_size, &support, &os, &wcs);
    const int s = 2 * support + 1;
    const int64_t n = (int64_t)s * s * os * os * w_size;
    for (int k = 0; k < w_size; ++k)
        for (int osj = 0; osj < os; ++osj)
            for (int osi = 0; osi < os; ++osi)
                for (int j = 0; j < s; ++j)
                    for (int i = 0; i < s; ++i) {
                        const int64_t cind = i + (int64_t)s * (j + (int64_t)s * (osi + os * (osj + (int64_t)os * k)));
                        const double raw = orc_c_raw(k, osj, osi, j, i, w_size, os, s, wcs, freq0, cell_size);
                        c[2 * cind] = (float)raw;
                        c[2 * cind + 1] = 0.0f;
                        if (c64) c64[cind] = raw;
                    }
    float sum_c = 0.0f;
    for (int64_t i = 0; i < n; ++i)
        sum_c += hypotf(c[2 * i], c[2 * i + 1]);
    const float scale = (float)(w_size * os * os) / sum_c;
    for (int64_t i = 0; i < n; ++i) {
        c[2 * i] = c[2 * i] * scale;
        c[2 * i + 1] = c[2 * i + 1] * scale;
    }
    if (c64) {
        const double scale64 = (double)(w_size * os * os) / (double)sum_c;
        for (int64_t i = 0; i < n; ++i) c64[i] *= scale64;
    }
    *support_out = support;
    *over_sample_out = os;
    *w_cell_size_out = wcs;
    return sum_c;
}

/* ---------------------------------------------------------------------------------------------
 * Per-sample grid position and table offset.  attic/tConvolveMPI/Benchmark.cc:281-324:
 * iu = floor(freq*u/cellSize) (int truncation, minus one if that overshot), fracu the
 * oversampled fraction (truncated), iu += gSize/2; the same for v; woff = wSize/2 +
 * int(freq*w/wCellSize) (truncation toward zero); cOffset = sSize^2 * (fracu + os*(fracv + os*woff)).
 * Output index dind = i * nChan + chan.
 * ------------------------------------------------------------------------------------------- */
void orc_init_offsets(int64_t n_samples, int n_chan, const double *u, const double *v,
                      const double *w, const double *freq, double cell_size,
                      double w_cell_size, int w_size, int g_size, int support, int over_sample,
                      int32_t *iu_out, int32_t *iv_out, int32_t *coff_out)
{
    const int s = 2 * support + 1;
    for (int64_t i = 0; i < n_samples; ++i)
        for (int chan = 0; chan < n_chan; ++chan) {
            const int64_t d = i * n_chan + chan;
            const double us = freq[chan] * u[i] / cell_size;
            int iu = (int)us;
            if (us < (double)iu) iu -= 1;
            const int fracu = (int)((double)over_sample * (us - (double)iu));
            iu += g_size / 2;
            const double vs = freq[chan] * v[i] / cell_size;
            int iv = (int)vs;
            if (vs < (double)iv) iv -= 1;
            const int fracv = (int)((double)over_sample * (vs - (double)iv));
            iv += g_size / 2;
            const double ws = freq[chan] * w[i] / w_cell_size;
            const int woff = w_size / 2 + (int)ws;
            iu_out[d] = iu;
            iv_out[d] = iv;
            coff_out[d] = s * s * (fracu + over_sample * (fracv + over_sample * woff));
        }
}

/* ---------------------------------------------------------------------------------------------
 * Gridding, FP32, reference order.  attic/tConvolveMPI/Benchmark.cc:125-155: for each sample in
 * index order, rows iv .. iv+2*support, columns iu-support .. iu+support,
 * grid[gind + x] += data * C[cind + x] with the 4-multiply complex product (-fcx-limited-range).
 * The grid is accumulated into, not cleared.
 *
 * The threaded form splits the grid into row bands; each thread visits every sample in index
 * order and updates only its rows, so every grid point sees the same additions in the same
 * order as the sequential loop: the result is bit-identical for any thread count.
 * ------------------------------------------------------------------------------------------- */
typedef struct {
    const float *data, *c;
    const int32_t *iu, *iv, *coff;
    int64_t n;
    int support, g_size;
    float *grid;
    int row_lo, row_hi;
} orc_grid_job;

static void orc_grid_rows(const orc_grid_job *jb)
{
    const int s = 2 * jb->support + 1;
    const int64_t g = jb->g_size;
    for (int64_t d = 0; d < jb->n; ++d) {
        const float dr = jb->data[2 * d], di = jb->data[2 * d + 1];
        const int iv = jb->iv[d];
        int r0 = iv > jb->row_lo ? iv : jb->row_lo;
        int r1 = iv + s < jb->row_hi ? iv + s : jb->row_hi;
        for (int row = r0; row < r1; ++row) {
            float *gp = jb->grid + 2 * ((int64_t)row * g + jb->iu[d] - jb->support);
            const float *cp = jb->c + 2 * ((int64_t)jb->coff[d] + (int64_t)(row - iv) * s);
            for (int x = 0; x < s; ++x) {
                const float cr = cp[2 * x], ci = cp[2 * x + 1];
                const float pr = dr * cr - di * ci;
                const float pi = dr * ci + di * cr;
                gp[2 * x] += pr;
                gp[2 * x + 1] += pi;
            }
        }
    }
}

static void *orc_grid_thread(void *arg)
{
    orc_grid_rows((const orc_grid_job *)arg);
    return NULL;
}

void orc_grid_f32(const float *data, int64_t n, int support, const float *c,
                  const int32_t *coff, const int32_t *iu, const int32_t *iv,
                  float *grid, int g_size, int n_threads)
{
    if (n_threads < 1) n_threads = 1;
    orc_grid_job *jobs = (orc_grid_job *)calloc((size_t)n_threads, sizeof(orc_grid_job));
    pthread_t *th = (pthread_t *)calloc((size_t)n_threads, sizeof(pthread_t));
    for (int t = 0; t < n_threads; ++t) {
        orc_grid_job jb = {data, c, iu, iv, coff, n, support, g_size, grid,
                           (int)((int64_t)g_size * t / n_threads),
                           (int)((int64_t)g_size * (t + 1) / n_threads)};
        jobs[t] = jb;
    }
    if (n_threads == 1) {
        orc_grid_rows(&jobs[0]);
    } else {
        for (int t = 0; t < n_threads; ++t) pthread_create(&th[t], NULL, orc_grid_thread, &jobs[t]);
        for (int t = 0; t < n_threads; ++t) pthread_join(th[t], NULL);
    }
    free(jobs);
    free(th);
}

/* ---------------------------------------------------------------------------------------------
 * Degridding, FP32, reference order.  attic/tConvolveMPI/Benchmark.cc:158-195: data[d] = 0, then
 * data[d] += grid[gind + x] * C[cind + x] row by row (product with grid as the left operand).
 * Samples are independent, so the threaded form splits them into contiguous ranges.
 * ------------------------------------------------------------------------------------------- */
typedef struct {
    const float *grid, *c;
    const int32_t *iu, *iv, *coff;
    int64_t lo, hi;
    int support, g_size;
    float *out;
} orc_degrid_job;

static void orc_degrid_range(const orc_degrid_job *jb)
{
    const int s = 2 * jb->support + 1;
    const int64_t g = jb->g_size;
    for (int64_t d = jb->lo; d < jb->hi; ++d) {
        float ar = 0.0f, ai = 0.0f;
        int64_t gind = jb->iu[d] + g * jb->iv[d] - jb->support;
        int64_t cind = jb->coff[d];
        for (int sv = 0; sv < s; ++sv) {
            const float *gp = jb->grid + 2 * gind;
            const float *cp = jb->c + 2 * cind;
            for (int x = 0; x < s; ++x) {
                const float gr = gp[2 * x], gi = gp[2 * x + 1];
                const float cr = cp[2 * x], ci = cp[2 * x + 1];
                const float pr = gr * cr - gi * ci;
                const float pi = gr * ci + gi * cr;
                ar += pr;
                ai += pi;
            }
            gind += g;
            cind += s;
        }
        jb->out[2 * d] = ar;
        jb->out[2 * d + 1] = ai;
    }
}

static void *orc_degrid_thread(void *arg)
{
    orc_degrid_range((const orc_degrid_job *)arg);
    return NULL;
}

void orc_degrid_f32(const float *grid, int g_size, int support, const float *c,
                    const int32_t *coff, const int32_t *iu, const int32_t *iv,
                    float *out, int64_t n, int n_threads)
{
    if (n_threads < 1) n_threads = 1;
    orc_degrid_job *jobs = (orc_degrid_job *)calloc((size_t)n_threads, sizeof(orc_degrid_job));
    pthread_t *th = (pthread_t *)calloc((size_t)n_threads, sizeof(pthread_t));
    for (int t = 0; t < n_threads; ++t) {
        orc_degrid_job jb = {grid, c, iu, iv, coff, n * t / n_threads, n * (t + 1) / n_threads,
                             support, g_size, out};
        jobs[t] = jb;
    }
    if (n_threads == 1) {
        orc_degrid_range(&jobs[0]);
    } else {
        for (int t = 0; t < n_threads; ++t) pthread_create(&th[t], NULL, orc_degrid_thread, &jobs[t]);
        for (int t = 0; t < n_threads; ++t) pthread_join(th[t], NULL);
    }
    free(jobs);
    free(th);
}

/* ---------------------------------------------------------------------------------------------
 * FP64 forms of the two kernels (the precision oracle).  Same loops and footprint geometry as
 * Benchmark.cc:125-195, with a real double table (the attic table has zero imaginary part),
 * complex double data and a complex double grid (interleaved).
 * ------------------------------------------------------------------------------------------- */
typedef struct {
    const double *data, *c_real;
    const int32_t *iu, *iv, *coff;
    int64_t n;
    int support, g_size;
    double *grid;
    int row_lo, row_hi;
} orc_grid64_job;

/* Rows [row_lo, row_hi) of the grid, every sample in input order (as orc_grid_rows): each point
 * sees the same additions in the same order for any thread count. */
static void *orc_grid64_rows(void *arg)
{
    const orc_grid64_job *jb = (const orc_grid64_job *)arg;
    const int s = 2 * jb->support + 1;
    const int64_t g = jb->g_size;
    for (int64_t d = 0; d < jb->n; ++d) {
        const double dr = jb->data[2 * d], di = jb->data[2 * d + 1];
        const int iv = jb->iv[d];
        int r0 = iv > jb->row_lo ? iv : jb->row_lo;
        int r1 = iv + s < jb->row_hi ? iv + s : jb->row_hi;
        for (int row = r0; row < r1; ++row) {
            double *gp = jb->grid + 2 * ((int64_t)row * g + jb->iu[d] - jb->support);
            const double *cp = jb->c_real + (int64_t)jb->coff[d] + (int64_t)(row - iv) * s;
            for (int x = 0; x < s; ++x) {
                gp[2 * x] += dr * cp[x];
                gp[2 * x + 1] += di * cp[x];
            }
        }
    }
    return NULL;
}

void orc_grid_f64(const double *data, int64_t n, int support, const double *c_real,
                  const int32_t *coff, const int32_t *iu, const int32_t *iv,
                  double *grid, int g_size, int n_threads)
{
    if (n_threads < 1) n_threads = 1;
    orc_grid64_job *jobs = (orc_grid64_job *)calloc((size_t)n_threads, sizeof(orc_grid64_job));
    pthread_t *th = (pthread_t *)calloc((size_t)n_threads, sizeof(pthread_t));
    for (int t = 0; t < n_threads; ++t) {
        orc_grid64_job jb = {data, c_real, iu, iv, coff, n, support, g_size, grid,
                             (int)((int64_t)g_size * t / n_threads),
                             (int)((int64_t)g_size * (t + 1) / n_threads)};
        jobs[t] = jb;
    }
    if (n_threads == 1) {
        orc_grid64_rows(&jobs[0]);
    } else {
        for (int t = 0; t < n_threads; ++t) pthread_create(&th[t], NULL, orc_grid64_rows, &jobs[t]);
        for (int t = 0; t < n_threads; ++t) pthread_join(th[t], NULL);
    }
    free(jobs);
    free(th);
}

typedef struct {
    const double *grid, *c_real;
    const int32_t *iu, *iv, *coff;
    int64_t lo, hi;
    int support, g_size;
    double *out;
} orc_degrid64_job;

static void *orc_degrid64_range(void *arg)
{
    const orc_degrid64_job *jb = (const orc_degrid64_job *)arg;
    const int s = 2 * jb->support + 1;
    const int64_t g = jb->g_size;
    for (int64_t d = jb->lo; d < jb->hi; ++d) {
        double ar = 0.0, ai = 0.0;
        int64_t gind = jb->iu[d] + g * jb->iv[d] - jb->support;
        int64_t cind = jb->coff[d];
        for (int sv = 0; sv < s; ++sv) {
            const double *gp = jb->grid + 2 * gind;
            const double *cp = jb->c_real + cind;
            for (int x = 0; x < s; ++x) {
                ar += gp[2 * x] * cp[x];
                ai += gp[2 * x + 1] * cp[x];
            }
            gind += g;
            cind += s;
        }
        jb->out[2 * d] = ar;
        jb->out[2 * d + 1] = ai;
    }
    return NULL;
}

void orc_degrid_f64(const double *grid, int g_size, int support, const double *c_real,
                    const int32_t *coff, const int32_t *iu, const int32_t *iv,
                    double *out, int64_t n, int n_threads)
{
    if (n_threads < 1) n_threads = 1;
    orc_degrid64_job *jobs = (orc_degrid64_job *)calloc((size_t)n_threads, sizeof(orc_degrid64_job));
    pthread_t *th = (pthread_t *)calloc((size_t)n_threads, sizeof(pthread_t));
    for (int t = 0; t < n_threads; ++t) {
        orc_degrid64_job jb = {grid, c_real, iu, iv, coff, n * t / n_threads, n * (t + 1) / n_threads,
                               support, g_size, out};
        jobs[t] = jb;
    }
    if (n_threads == 1) {
        orc_degrid64_range(&jobs[0]);
    } else {
        for (int t = 0; t < n_threads; ++t) pthread_create(&th[t], NULL, orc_degrid64_range, &jobs[t]);
        for (int t = 0; t < n_threads; ++t) pthread_join(th[t], NULL);
    }
    free(jobs);
    free(th);
}
