/*
 * tcv_probe.h -- C ABI of libtcvprobe.so, a measurement tool beside the gridding library (not part
 * of the gridding path or of libtconvolve.so).  It measures this GPU's L2-to-SM bandwidth for the
 * access shape of the tile kernels' table reads: random 128-byte row segments, 16 rows at a row
 * stride, from an L2-resident buffer -- the ceiling those kernels are bound by.  No counterpart in
 * the reference.
 */
#ifndef TCV_PROBE_H
#define TCV_PROBE_H

#include <stdint.h>

#include "tconvolve.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Threads of one probe launch (d_out must hold as many floats). */
int64_t tcv_probe_table_threads(void);
/* One launch over d_buf (n_floats, ideally a few tens of MB so that it stays in L2), each warp
 * reading `samples` random 16-row windows of `stride` floats; *bytes_out receives the bytes the
 * warps read (128 per row segment).  Asynchronous on the stream: time it with events. */
tcv_status tcv_probe_table_stream(const float *d_buf, int64_t n_floats, int stride, int samples,
                                  float *d_out, int64_t *bytes_out, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* TCV_PROBE_H */
