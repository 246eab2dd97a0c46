/*
 * tconvolve_oracle_current.c -- CPU restatement of the variable-support W-projection path of
 * current/tConvolveMPI (Benchmark::init, initC, initCOffset, gridKernel, degridKernel).
 *
 * TEST INFRASTRUCTURE ONLY (the parity checker; the product never links or calls it).
 *
 * Parity status: pinned.  tests/test_oracle.py checks these functions bit for bit against the
 * reference's own current/tConvolveMPI/Benchmark.cc compiled from source by oracle/Makefile
 * (target `ref`, driver oracle/ref_driver_current.cc; fixtures in tests/golden/).
 *
 * The reference mixes float (`Real`) and double (`Coord`) arithmetic; every expression below
 * keeps the reference's types and order of operations (paths relative to the reference root).
 * Compiled with -ffp-contract=off, as the reference's x86-64 build has no fused multiply-adds.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>

#define CUR_MAXINT 2147483647u
#define CUR_PI 3.141593 /* the reference's constant */
#define CUR_NANT 36

/* current/tConvolveMPI/Benchmark.cc:183-204: antenna positions (metres east, north) */
static const double cur_east[CUR_NANT] = {
    -42.43847222,  -15.46047222,  -6.48847222,    -51.41747222,   -116.43047222, 93.22152778,
    200.42152778,  -80.24847222,  -286.64847222,  -138.75447222,  225.51252778,  353.48652778,
    396.28152778,  -67.29847222,  -782.13847222,  -678.55347222,  -539.25647222, -149.22347222,
    175.37552778,  463.88152778,  643.72952778,   803.40152778,   -43.14647222,  36.03352778,
    -656.05547222, -435.77447222, -1112.94147222, 207.32652778,   523.49152778,  1186.61752778,
    2178.51052778, 2982.48652778, -17.41247222,   -3017.44747222, -2213.43647222, -19.20647222};
static const double cur_north[CUR_NANT] = {
    -105.22933333, -118.24033333, -97.73933333,   -70.22133333,  -73.72633333,  6.77066667,
    -215.20933333, -343.73933333, 5.32066667,     174.26666667,  235.30966667,  164.24666667,
    -469.23433333, -565.23833333, -263.22233333,  260.21066667,  417.28966667,  270.27966667,
    376.29066667,  209.79766667,  216.77666667,   230.75266667,  -762.23633333, -1083.75233333,
    548.27766667,  562.27366667,  835.74566667,   1093.28166667, 647.98066667,  693.23866667,
    887.75566667,  -2612.27533333, -2916.19433333, -2112.20733333, 887.76166667, 3084.83866667};

typedef struct {
    float baseline;
    int over_sample, support, w_size, g_size;
    double w_cell_size, uv_cell_size;
} cur_params;

/* current/tConvolveMPI/Benchmark.cc:64-158: the run type's constants, in the reference's float
 * arithmetic (Real = float; lambda, wmax, fov, wPart and the grid geometry are float). */
static int cur_params_of(int run_type, cur_params *p)
{
    const int aperture = 12;
    const float max_freq = 1.0e9f;
    const float lambda = (float)(2.998e8 / (double)max_freq);
    float img_os, img_ext;
    memset(p, 0, sizeof(*p));
    if (run_type == 0 || run_type == 1) {
        p->baseline = run_type == 0 ? 6440.f : 2000.f;
        img_os = run_type == 0 ? 4.0f : 3.1f;
        img_ext = run_type == 0 ? 3.0f : 2.0f;
        p->over_sample = run_type == 0 ? 4 : 8;
        const float wmax = p->baseline / lambda;
        const float fov = lambda / (float)aperture * img_ext;
        const float w_part = wmax * fov * fov;
        const float a_part = 7.f;
        p->support = (int)ceilf(sqrtf(a_part * a_part + w_part * w_part)) / 2;
        p->w_size = (int)ceilf((float)p->over_sample * w_part);
        p->w_size += (p->w_size + 1) % 2;
        p->w_cell_size = (double)(2.f * wmax / (float)(p->w_size - 1));
    } else if (run_type == 2) {
        p->baseline = 6440.f;
        img_os = 2.0f;
        img_ext = 1.0f;
        p->over_sample = 1;
        p->support = 0;
        p->w_size = 1;
    } else if (run_type == 3 || run_type == 4) {
        p->baseline = 6440.f;
        img_os = 4.0f;
        img_ext = 1.923f;
        p->over_sample = run_type == 3 ? 128 : 8;
        p->support = run_type == 3 ? 3 : 43;
        p->w_size = 1;
    } else {
        return -1;
    }
    p->g_size = (int)ceilf(p->baseline / (float)aperture * img_os * img_ext);
    p->uv_cell_size = (double)(p->baseline / lambda * img_os / (float)p->g_size);
    return 0;
}

/* current/tConvolveMPI/Benchmark.cc:164-228: baselines no longer than `baseline` between the 36
 * antennas (X, Y, Z from east/north at the observatory latitude); returns their number. */
static int cur_baselines(float baseline, double *bx, double *by, double *bz)
{
    const double lat = -26.6970 * CUR_PI / 180.0;
    double x[CUR_NANT], y[CUR_NANT], z[CUR_NANT];
    for (int i = 0; i < CUR_NANT; ++i) {
        x[i] = -cur_north[i] * sin(lat);
        y[i] = cur_east[i];
        z[i] = cur_north[i] * cos(lat);
    }
    const double lim = (double)(baseline * baseline);
    int bl = 0;
    for (int i = 0; i < CUR_NANT - 1; ++i)
        for (int j = i + 1; j < CUR_NANT; ++j) {
            const double dx = x[i] - x[j], dy = y[i] - y[j], dz = z[i] - z[j];
            if (dx * dx + dy * dy + dz * dz > lim) continue;
            bx[bl] = dx;
            by[bl] = dy;
            bz[bl] = dz;
            ++bl;
        }
    return bl;
}

/* Geometry of a run type: out[0..9] = w_size, over_sample, support, g_size, n_baselines,
 * n_samples, w_cell_size, uv_cell_size, c_len, max sSize.  Returns -1 for an unknown type. */
int orc_cur_geometry(int run_type, double *out)
{
    cur_params p;
    if (cur_params_of(run_type, &p)) return -1;
    double bx[CUR_NANT * CUR_NANT], by[CUR_NANT * CUR_NANT], bz[CUR_NANT * CUR_NANT];
    const int nb = cur_baselines(p.baseline, bx, by, bz);
    const int n_scans = (int)(12. * 3600. / 5.);
    out[0] = p.w_size;
    out[1] = p.over_sample;
    out[2] = p.support;
    out[3] = p.g_size;
    out[4] = nb;
    out[5] = (double)n_scans * nb;
    out[6] = p.w_cell_size;
    out[7] = p.uv_cell_size;
    /* c_len and the widest kernel from the per-plane widths (initC below) */
    int64_t len = 0;
    int smax = 0;
    for (int k = 0; k < p.w_size; ++k) {
        int s = 2 * p.support + 1;
        if (p.w_size > 1) {
            const int wind = k - p.w_size / 2;
            const double w = wind * p.w_cell_size;
            const float w_part = (float)(w / p.uv_cell_size / p.uv_cell_size);
            const float a_part = 7.f;
            s = (int)ceilf(sqrtf(a_part * a_part + w_part * w_part));
            s += (s + 1) % 2;
        }
        if (s > smax) smax = s;
        len += (int64_t)s * s * p.over_sample * p.over_sample;
    }
    out[8] = (double)len;
    out[9] = smax;
    return 0;
}

static int cur_random_int(uint64_t *state)
{
    *state = *state * 1103515245ull + 12345ull;
    return (int)((unsigned int)(*state / 65536ull) % CUR_MAXINT);
}

/* current/tConvolveMPI/Benchmark.cc:246-262: per sample a baseline and an hour angle from two
 * draws, then u, v, w.  *state: generator state before the first draw (advanced on return). */
int orc_cur_init_uvw(int run_type, uint64_t *state, double *u, double *v, double *w)
{
    cur_params p;
    if (cur_params_of(run_type, &p)) return -1;
    double bx[CUR_NANT * CUR_NANT], by[CUR_NANT * CUR_NANT], bz[CUR_NANT * CUR_NANT];
    const int nb = cur_baselines(p.baseline, bx, by, bz);
    const int64_t n = (int64_t)(int)(12. * 3600. / 5.) * nb;
    const double lat = -26.6970 * CUR_PI / 180.0;
    const double cdec = cos(lat), sdec = sin(lat);
    const double maxint = (double)CUR_MAXINT;
    for (int64_t i = 0; i < n; ++i) {
        const int bl = (int)(nb * ((double)cur_random_int(state) / maxint));
        const double ha = 12. * CUR_PI / 12.0 * (((double)cur_random_int(state) / maxint) - 0.5);
        const double cha = cos(ha), sha = sin(ha);
        u[i] = sha * bx[bl] + cha * by[bl];
        v[i] = -sdec * cha * bx[bl] + sdec * sha * by[bl] + cdec * bz[bl];
        w[i] = cdec * cha * bx[bl] - cdec * sha * by[bl] + sdec * bz[bl];
    }
    return 0;
}

/* current/tConvolveMPI/Benchmark.cc:487-583: per-plane widths sSize[k] (odd, from the w term;
 * 2*support+1 with one plane), plane offsets cOffset0[k], and the table: exp(-r2) times, off the
 * w = 0 plane and inside r2 < sSize/2, the complex Fresnel factor (n/w)(sin phase, -cos phase)
 * in float, each plane normalised by os^2 / (double sum of float |C|).  c: interleaved
 * complex64, c_len entries.  The complex products are the plain 4-multiply formula in float
 * (-fcx-limited-range); |C| is cabsf (hypotf), as std::abs(std::complex<float>) in libstdc++. */
int orc_cur_init_c(int run_type, int32_t *s_size, int32_t *c_off0, float *c)
{
    cur_params p;
    if (cur_params_of(run_type, &p)) return -1;
    const int os = p.over_sample, w_size = p.w_size;
    const double uvc = p.uv_cell_size, wcs = p.w_cell_size;
    int64_t offset = 0;
    for (int k = 0; k < w_size; ++k) {
        const int wind = k - w_size / 2;
        const double w = wind * wcs;
        double f_scale = 0.0;
        if (wind != 0) f_scale = uvc * uvc / w;
        c_off0[k] = (int32_t)offset;
        int s = 2 * p.support + 1;
        if (w_size > 1) {
            const float w_part = (float)(w / uvc / uvc);
            const float a_part = 7.f;
            s = (int)ceilf(sqrtf(a_part * a_part + w_part * w_part));
            s += (s + 1) % 2;
        }
        s_size[k] = s;
        const int center = s / 2;
        double sum_c = 0.0;
        for (int osj = 0; osj < os; ++osj)
            for (int osi = 0; osi < os; ++osi) {
                const int64_t os_off = (int64_t)s * s * (osi + os * osj) + offset;
                for (int j = 0; j < s; ++j) {
                    const double dj = (double)(j - center) + (double)osj / (double)os;
                    const double j2 = dj * dj; /* pow(x, 2): the correctly rounded square */
                    for (int i = 0; i < s; ++i) {
                        const int64_t cind = i + (int64_t)s * j + os_off;
                        const double di = (double)(i - center) + (double)osi / (double)os;
                        const double r2 = j2 + di * di;
                        float cre = (float)exp(-r2), cim = 0.f;
                        if (wind != 0 && r2 < (double)(s / 2)) {
                            const float n = (float)sqrt(1. - r2 * f_scale / w);
                            const float phase = (float)(-2. * CUR_PI * (r2 * f_scale + w * ((double)n - 1.)));
                            const float a = (float)((double)n / w);  /* static_cast<Value>(n/w) */
                            const float sn = sinf(phase), cs = -cosf(phase);
                            /* (a + 0i) * (sn + cs i), then C *= that, 4-multiply formulas */
                            const float xre = a * sn - 0.f * cs, xim = a * cs + 0.f * sn;
                            const float nre = cre * xre - cim * xim, nim = cre * xim + cim * xre;
                            cre = nre;
                            cim = nim;
                        }
                        c[2 * cind] = cre;
                        c[2 * cind + 1] = cim;
                        sum_c += (double)hypotf(cre, cim);
                    }
                }
            }
        const float norm = (float)((double)(os * os) / sum_c);
        const int64_t m = (int64_t)s * s * os * os;
        for (int64_t i = 0; i < m; ++i) {
            const float re = c[2 * (offset + i)], im = c[2 * (offset + i) + 1];
            c[2 * (offset + i)] = re * norm - im * 0.f;
            c[2 * (offset + i) + 1] = re * 0.f + im * norm;
        }
        offset += m;
    }
    return 0;
}

/* current/tConvolveMPI/Benchmark.cc:599-650: grid position, w-plane and table offset per sample
 * (one channel at the wavenumber maxFreq/c, Benchmark.cc:269-272). */
int orc_cur_init_offsets(int run_type, int64_t n, const double *u, const double *v, const double *w,
                         const int32_t *s_size, const int32_t *c_off0, int32_t *iu_out, int32_t *iv_out,
                         int32_t *wplane_out, int32_t *coff_out)
{
    cur_params p;
    if (cur_params_of(run_type, &p)) return -1;
    const double wn = ((double)1.0e9f - 2.0e5 * 0.0 / 1.0) / 2.998e8;
    const int os = p.over_sample;
    for (int64_t d = 0; d < n; ++d) {
        const double us = wn * u[d] / p.uv_cell_size;
        int iu = (int)us;
        if (us < (double)iu) iu -= 1;
        const int fracu = (int)(os * (us - (double)iu));
        iu += p.g_size / 2;
        const double vs = wn * v[d] / p.uv_cell_size;
        int iv = (int)vs;
        if (vs < (double)iv) iv -= 1;
        const int fracv = (int)(os * (vs - (double)iv));
        iv += p.g_size / 2;
        int woff = 0;
        if (p.w_cell_size > 0.0) {
            const double ws = wn * w[d] / p.w_cell_size;
            woff = p.w_size / 2 + (int)ws;
        }
        iu_out[d] = iu;
        iv_out[d] = iv;
        wplane_out[d] = woff;
        coff_out[d] = s_size[woff] * s_size[woff] * (fracu + os * fracv) + c_off0[woff];
    }
    return 0;
}

/* current/tConvolveMPI/Benchmark.cc:287-306 with setSort(1): the offsets (not the data) stably
 * ordered by w-plane. */
void orc_cur_sort_by_plane(int64_t n, int w_size, int32_t *iu, int32_t *iv, int32_t *wplane, int32_t *coff)
{
    int64_t *start = calloc((size_t)w_size + 1, sizeof(int64_t));
    int32_t *t = malloc((size_t)n * 4 * sizeof(int32_t));
    for (int64_t d = 0; d < n; ++d) start[wplane[d] + 1]++;
    for (int k = 0; k < w_size; ++k) start[k + 1] += start[k];
    memcpy(t, iu, (size_t)n * 4);
    memcpy(t + n, iv, (size_t)n * 4);
    memcpy(t + 2 * n, wplane, (size_t)n * 4);
    memcpy(t + 3 * n, coff, (size_t)n * 4);
    for (int64_t d = 0; d < n; ++d) {
        const int64_t j = start[t[2 * n + d]]++;
        iu[j] = t[d];
        iv[j] = t[n + d];
        wplane[j] = t[2 * n + d];
        coff[j] = t[3 * n + d];
    }
    free(t);
    free(start);
}

typedef struct {
    const float *data, *c, *grid_in;
    const int32_t *iu, *iv, *wplane, *coff, *s_size;
    float *grid, *out;
    int64_t n, d0, d1;
    int g_size, row0, row1;
} cur_job;

/* current/tConvolveMPI/Benchmark.cc:373-411: for each sample in index order, its sSize[plane]^2
 * footprint (rows iv.., columns iu-support..), g.re += dre*cre - dim*cim, g.im += dim*cre +
 * dre*cim.  Threads own row bands and visit every sample, so each point's additions keep the
 * reference's order. */
static void *cur_grid_rows(void *arg)
{
    const cur_job *jb = (const cur_job *)arg;
    for (int64_t d = 0; d < jb->n; ++d) {
        const int s = jb->s_size[jb->wplane[d]];
        const int support = s / 2;
        const int64_t gind0 = (int64_t)jb->iu[d] + (int64_t)jb->g_size * jb->iv[d] - support;
        const int r0 = jb->iv[d];
        const float dre = jb->data[2 * d], dim = jb->data[2 * d + 1];
        for (int sv = 0; sv < s; ++sv) {
            const int row = r0 + sv;
            if (row < jb->row0 || row >= jb->row1) continue;
            float *g = jb->grid + 2 * (gind0 + (int64_t)jb->g_size * sv);
            const float *cp = jb->c + 2 * ((int64_t)jb->coff[d] + (int64_t)s * sv);
            for (int su = 0; su < s; ++su) {
                g[2 * su] += dre * cp[2 * su] - dim * cp[2 * su + 1];
                g[2 * su + 1] += dim * cp[2 * su] + dre * cp[2 * su + 1];
            }
        }
    }
    return NULL;
}

void orc_cur_grid_f32(const float *data, int64_t n, const int32_t *iu, const int32_t *iv, const int32_t *wplane,
                      const int32_t *coff, const int32_t *s_size, const float *c, float *grid, int g_size,
                      int threads)
{
    if (threads < 1) threads = 1;
    pthread_t th[64];
    cur_job jobs[64];
    if (threads > 64) threads = 64;
    for (int t = 0; t < threads; ++t) {
        cur_job jb = {data, c, NULL, iu, iv, wplane, coff, s_size, grid, NULL, n, 0, 0, g_size,
                      (int)((int64_t)g_size * t / threads), (int)((int64_t)g_size * (t + 1) / threads)};
        jobs[t] = jb;
        pthread_create(&th[t], NULL, cur_grid_rows, &jobs[t]);
    }
    for (int t = 0; t < threads; ++t) pthread_join(th[t], NULL);
}

/* current/tConvolveMPI/Benchmark.cc:414-452: re += gre*cre - gim*cim, im += gim*cre + gre*cim
 * over the footprint in row order; data[d] = (re, im). */
static void *cur_degrid_range(void *arg)
{
    const cur_job *jb = (const cur_job *)arg;
    for (int64_t d = jb->d0; d < jb->d1; ++d) {
        const int s = jb->s_size[jb->wplane[d]];
        const int support = s / 2;
        const int64_t gind0 = (int64_t)jb->iu[d] + (int64_t)jb->g_size * jb->iv[d] - support;
        float re = 0.f, im = 0.f;
        for (int sv = 0; sv < s; ++sv) {
            const float *g = jb->grid_in + 2 * (gind0 + (int64_t)jb->g_size * sv);
            const float *cp = jb->c + 2 * ((int64_t)jb->coff[d] + (int64_t)s * sv);
            for (int su = 0; su < s; ++su) {
                re += g[2 * su] * cp[2 * su] - g[2 * su + 1] * cp[2 * su + 1];
                im += g[2 * su + 1] * cp[2 * su] + g[2 * su] * cp[2 * su + 1];
            }
        }
        jb->out[2 * d] = re;
        jb->out[2 * d + 1] = im;
    }
    return NULL;
}

void orc_cur_degrid_f32(const float *grid, int g_size, int64_t n, const int32_t *iu, const int32_t *iv,
                        const int32_t *wplane, const int32_t *coff, const int32_t *s_size, const float *c,
                        float *out, int threads)
{
    if (threads < 1) threads = 1;
    if (threads > 64) threads = 64;
    pthread_t th[64];
    cur_job jobs[64];
    for (int t = 0; t < threads; ++t) {
        cur_job jb = {NULL, c, grid, iu, iv, wplane, coff, s_size, NULL, out, n, n * t / threads,
                      n * (t + 1) / threads, g_size, 0, 0};
        jobs[t] = jb;
        pthread_create(&th[t], NULL, cur_degrid_range, &jobs[t]);
    }
    for (int t = 0; t < threads; ++t) pthread_join(th[t], NULL);
}

/* Degridding with double accumulation of the same float grid and table (the exact answer the
 * FP32 sums of current/tConvolveMPI/Benchmark.cc:414-452 approximate); out: interleaved doubles. */
static void *cur_degrid64_range(void *arg)
{
    const cur_job *jb = (const cur_job *)arg;
    double *out = (double *)(void *)jb->out;
    for (int64_t d = jb->d0; d < jb->d1; ++d) {
        const int s = jb->s_size[jb->wplane[d]];
        const int64_t gind0 = (int64_t)jb->iu[d] + (int64_t)jb->g_size * jb->iv[d] - s / 2;
        double re = 0.0, im = 0.0;
        for (int sv = 0; sv < s; ++sv) {
            const float *g = jb->grid_in + 2 * (gind0 + (int64_t)jb->g_size * sv);
            const float *cp = jb->c + 2 * ((int64_t)jb->coff[d] + (int64_t)s * sv);
            for (int su = 0; su < s; ++su) {
                re += (double)g[2 * su] * cp[2 * su] - (double)g[2 * su + 1] * cp[2 * su + 1];
                im += (double)g[2 * su + 1] * cp[2 * su] + (double)g[2 * su] * cp[2 * su + 1];
            }
        }
        out[2 * d] = re;
        out[2 * d + 1] = im;
    }
    return NULL;
}

void orc_cur_degrid_f64(const float *grid, int g_size, int64_t n, const int32_t *iu, const int32_t *iv,
                        const int32_t *wplane, const int32_t *coff, const int32_t *s_size, const float *c,
                        double *out, int threads)
{
    if (threads < 1) threads = 1;
    if (threads > 64) threads = 64;
    pthread_t th[64];
    cur_job jobs[64];
    for (int t = 0; t < threads; ++t) {
        cur_job jb = {NULL, c, grid, iu, iv, wplane, coff, s_size, NULL, (float *)(void *)out, n, n * t / threads,
                      n * (t + 1) / threads, g_size, 0, 0};
        jobs[t] = jb;
        pthread_create(&th[t], NULL, cur_degrid64_range, &jobs[t]);
    }
    for (int t = 0; t < threads; ++t) pthread_join(th[t], NULL);
}

/* Gridding with double accumulation (grid: interleaved doubles) of the float data and table: the
 * exact answer the FP32 sums of current/tConvolveMPI/Benchmark.cc:373-411 approximate.  Row
 * bands per thread, as orc_cur_grid_f32. */
typedef struct {
    const float *data, *c;
    const int32_t *iu, *iv, *wplane, *coff, *s_size;
    double *grid;
    int64_t n;
    int g_size, row0, row1;
} cur_job64;

static void *cur_grid64_rows(void *arg)
{
    const cur_job64 *jb = (const cur_job64 *)arg;
    for (int64_t d = 0; d < jb->n; ++d) {
        const int s = jb->s_size[jb->wplane[d]];
        const int64_t gind0 = (int64_t)jb->iu[d] + (int64_t)jb->g_size * jb->iv[d] - s / 2;
        const double dre = jb->data[2 * d], dim = jb->data[2 * d + 1];
        for (int sv = 0; sv < s; ++sv) {
            const int row = jb->iv[d] + sv;
            if (row < jb->row0 || row >= jb->row1) continue;
            double *g = jb->grid + 2 * (gind0 + (int64_t)jb->g_size * sv);
            const float *cp = jb->c + 2 * ((int64_t)jb->coff[d] + (int64_t)s * sv);
            for (int su = 0; su < s; ++su) {
                g[2 * su] += dre * cp[2 * su] - dim * cp[2 * su + 1];
                g[2 * su + 1] += dim * cp[2 * su] + dre * cp[2 * su + 1];
            }
        }
    }
    return NULL;
}

void orc_cur_grid_f64(const float *data, int64_t n, const int32_t *iu, const int32_t *iv, const int32_t *wplane,
                      const int32_t *coff, const int32_t *s_size, const float *c, double *grid, int g_size,
                      int threads)
{
    if (threads < 1) threads = 1;
    if (threads > 64) threads = 64;
    pthread_t th[64];
    cur_job64 jobs[64];
    for (int t = 0; t < threads; ++t) {
        cur_job64 jb = {data, c, iu, iv, wplane, coff, s_size, grid, n, g_size,
                        (int)((int64_t)g_size * t / threads), (int)((int64_t)g_size * (t + 1) / threads)};
        jobs[t] = jb;
        pthread_create(&th[t], NULL, cur_grid64_rows, &jobs[t]);
    }
    for (int t = 0; t < threads; ++t) pthread_join(th[t], NULL);
}
