/*
 * psbx_probe.h -- measurement entry points of libpsbx.so (not part of the
 * reference's interface; used to state the bound an SpMV is measured
 * against).
 */
#ifndef PSBX_PROBE_H
#define PSBX_PROBE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Times the reads of x at n column indices (device int32, index base
 * `base`, 8-byte aligned; an odd last index is skipped) -- the gathers of an
 * SpMV with no values and no row sums -- on the library stream: best of
 * `reps` launches after two untimed ones, in milliseconds.  d_out receives
 * one double per 8 indices (ceil(n / 8) of them).  With random columns over
 * a vector larger than L1 this is the L2 sector-request floor of the SpMV. */
int psbx_probe_gather(const int *d_idx, long long n, int base, const double *d_x, double *d_out, int reps,
                      double *best_ms);

#ifdef __cplusplus
}
#endif
#endif
