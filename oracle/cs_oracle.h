/*
 * Test infrastructure (oracle).  Not product code; only tests/, smoke() and
 * bench.py's CPU-baseline leg may load it.
 *
 * CPU restatement of the coherent-search hot path of CoherentSearch_C,
 * written from the reference's algorithm (citations in cs_oracle.c) without
 * sharing code with the product.  It evaluates the per-trial metric of every
 * decimation slot, which the reference only exposes as above-threshold
 * candidates, so tests can compare the GPU kernel trial by trial.
 *
 * Pinned by tests/test_oracle.py against the reference itself compiled here
 * (oracle/_ref, built by oracle/Makefile from the reference sources): same
 * candidate set and S/N as the reference CPU path on seeded inputs.
 */
#ifndef CS_ORACLE_H
#define CS_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Metrics of trials [t_begin, t_begin + count) for the chunk table cstarts.
 * metrics[s * count + i] is the boxcar metric of slot s (0 = base profile,
 * then each decimation factor > 1 of decims[] in order) or NaN where the
 * decimated trial lies beyond the Nyquist frequency.  prec64 != 0 evaluates
 * the profile stage in FP64 (the reference's --precision f64 oracle).
 * Returns the number of slots, or -1 on invalid input. */
int cso_trial_metrics(const float *amps, long long namps, long long N,
                      int nharms, int m, double hidr, int ndecim, const int *decims,
                      double fsp, double maxfrac, double r_lo,
                      const long long *cstarts, long long nchunks, long long total,
                      long long t_begin, int count, int prec64, double *metrics);

/* Unnormalised c2r of the interpolated harmonic stack of one trial (FP64),
 * for direct profile comparisons: prof[0 .. 2*nharms-1]. */
int cso_trial_profile(const float *amps, long long namps, long long N, int nharms,
                      int m, double hidr, double r_lo, const long long *cstarts,
                      long long nchunks, long long total, long long t, double *prof);

#ifdef __cplusplus
}
#endif

#endif
