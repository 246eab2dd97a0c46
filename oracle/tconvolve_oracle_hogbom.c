/*
 * tconvolve_oracle_hogbom.c -- TEST INFRASTRUCTURE ONLY (the parity checker; the product never
 * links it): a plain-C restatement of Hogbom CLEAN as the reference computes it, in float with
 * the reference's roundings (compiled with -ffp-contract=off).
 *
 *   orc_find_peak       current/tHogbomCleanOMP/HogbomGolden.cc:127-139 (findPeak): strict '>'
 *                       on |value| in index order, starting from (0, 0)
 *   orc_subtract_psf    HogbomGolden.cc:99-124 (subtractPSF), including diffy = ry - px (:108);
 *                       PSF rows that index outside the PSF (the reference reads out of bounds
 *                       there) are skipped and counted
 *   orc_hogbom          HogbomGolden.cc:62-97 (deconvolve): residual = dirty, PSF peak, then
 *                       niters iterations with the |peak| < threshold stop (:86-89); the model is
 *                       accumulated into; tMajorACC's loop (current/tMajorACC/tMajorACC.cc:786-827)
 *                       is the same with no threshold (threshold 0)
 *
 * Parity status: pinned bit for bit against the reference's own HogbomGolden.cc, compiled
 * unmodified by `make ref-hogbom` (tests/golden/hogbom.json, tests/test_oracle_hogbom.py).
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

void orc_find_peak(const float *image, int64_t size, float *max_val, int64_t *max_pos)
{
    float mv = 0.0f;
    int64_t mp = 0;
    for (int64_t i = 0; i < size; ++i) {
        if (fabsf(image[i]) > fabsf(mv)) {
            mv = image[i];
            mp = i;
        }
    }
    *max_val = mv;
    *max_pos = mp;
}

int64_t orc_subtract_psf(const float *psf, int psf_width, float *residual, int residual_width, int64_t peak_pos,
                         int64_t psf_peak_pos, float abs_peak_val, float gain)
{
    const int rx = (int)(peak_pos % residual_width), ry = (int)(peak_pos / residual_width);
    const int px = (int)(psf_peak_pos % psf_width), py = (int)(psf_peak_pos / psf_width);
    const int diffx = rx - px;
    const int diffy = ry - px; /* as the reference (HogbomGolden.cc:108) */
    const int startx = rx - px > 0 ? rx - px : 0;
    const int starty = ry - py > 0 ? ry - py : 0;
    const int stopx = residual_width - 1 < rx + (psf_width - px - 1) ? residual_width - 1 : rx + (psf_width - px - 1);
    const int stopy = residual_width - 1 < ry + (psf_width - py - 1) ? residual_width - 1 : ry + (psf_width - py - 1);
    int64_t skipped = 0;
    for (int y = starty; y <= stopy; ++y) {
        const int prow = y - diffy;
        if (prow < 0 || prow >= psf_width) {
            ++skipped;
            continue;
        }
        for (int x = startx; x <= stopx; ++x) {
            const float t = gain * abs_peak_val;
            const float u = t * psf[(int64_t)prow * psf_width + (x - diffx)];
            float *r = &residual[(int64_t)y * residual_width + x];
            *r = *r - u;
        }
    }
    return skipped;
}

/* Returns the number of iterations carried out; *stopped_at = iteration that met the threshold
 * or -1; hist_val / hist_pos (may be NULL) receive each iteration's peak. */
int orc_hogbom(const float *dirty, int width, const float *psf, int psf_width, float *model, float *residual,
               int niters, float gain, float threshold, float *hist_val, int64_t *hist_pos, int *stopped_at,
               int64_t *skipped_rows, int64_t *psf_peak_pos)
{
    const int64_t n = (int64_t)width * width;
    memcpy(residual, dirty, (size_t)n * sizeof(float));
    float psf_val;
    int64_t psf_pos;
    orc_find_peak(psf, (int64_t)psf_width * psf_width, &psf_val, &psf_pos);
    if (psf_peak_pos) *psf_peak_pos = psf_pos;
    int64_t skipped = 0;
    int done = 0;
    if (stopped_at) *stopped_at = -1;
    for (int i = 0; i < niters; ++i) {
        float peak;
        int64_t pos;
        orc_find_peak(residual, n, &peak, &pos);
        if (fabsf(peak) < threshold) {
            if (stopped_at) *stopped_at = i;
            break;
        }
        model[pos] += peak * gain;
        if (hist_val) hist_val[i] = peak;
        if (hist_pos) hist_pos[i] = pos;
        skipped += orc_subtract_psf(psf, psf_width, residual, width, pos, psf_pos, peak, gain);
        done = i + 1;
    }
    if (skipped_rows) *skipped_rows = skipped;
    return done;
}
