/*
 * Test infrastructure (oracle), not product code.
 *
 * Drives the reference's vendored PRESTO dedispersion routines
 * (third_party/presto/src/dispersion.c: subband_search_delays,
 * subband_delays, dedisp_subbands, float_dedisp), compiled from the
 * reference sources into the same library, exactly as the reference's
 * prepsubband path does for 8-bit SIGPROC filterbank input with no
 * barycentring, clipping, masking or downsampling:
 *
 *   delay tables     src/prep_dedisp.c:318-331 (DM list, average DM),
 *                    :362-367 (blocks per read), :444-466 (idispdt,
 *                    offsets; NEAREST_LONG at :37)
 *   raw conversion   third_party/presto/src/sigproc_fb.c:656-664 (8-bit,
 *                    unsigned: channel order reversed)
 *   block reader     third_party/presto/src/sigproc_fb.c:549-620 (a partial
 *                    final block is dropped), backend_common.c:936-1066 and
 *                    :1684-1738 (prep_subbands / read_subbands: transpose to
 *                    channel-major, one block of latency)
 *   chunk driver     src/prep_dedisp.c:1104-1275 (get_data: blocks per read
 *                    per chunk, one chunk of latency, zero-filled failed
 *                    reads) and :484-522 (write while full chunks, at most
 *                    numout points)
 *
 * Compiled with -Ofast like the reference's PREP sources (src/Makefile:152-161).
 *
 * odd_run_clip adds PRESTO's time-domain clipping (clipping.c clip_times,
 * with median.c and misc_utils.c's avg_var, compiled into the same library)
 * at its place in prep_subbands (backend_common.c:976-986): on each raw block
 * in time-major PRESTO channel order, before the transpose.  clip_times keeps
 * its running averages in static variables, so a clipped run needs a fresh
 * copy of this library.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

double *subband_search_delays(int numchan, int numsubbands, double dm, double lofreq,
                              double chanwidth, double voverc);
double *subband_delays(int numchan, int numsubbands, double dm, double lofreq,
                       double chanwidth, double voverc);
double delay_from_dm(double dm, double freq_emitted);
void dedisp_subbands(float *data, float *lastdata, int numpts, int numchan, int *delays,
                     int numsubbands, float *result, int blockN, int thisblock);
void float_dedisp(float *data, float *lastdata, int numpts, int numchan, int *delays,
                  float approx_mean, float *result, int transpose);
void vect_free(void *vect);
int clip_times(float *rawdata, int ptsperblk, int numchan, float clip_sigma,
               float *good_chan_levels, int thread);

/* Two functions the linked PRESTO files reference outside the clipping path:
 * misc_utils.c's date helpers call SLALIB's slaDjcl, and clip_times opens a
 * bin file only when CLIPBINSFILE is set (neither is reached here). */
#include <stdio.h>
void slaDjcl(double djm, int *iy, int *im, int *id, double *fd, int *j)
{
    (void)djm; *iy = *im = *id = 0; *fd = 0.0; *j = 1;
}
FILE *chkfopen(char *path, const char *mode)
{
    FILE *f = fopen(path, mode);
    if (!f) { perror(path); exit(1); }
    return f;
}

#define NEAREST_LONG(x) (long) (x < 0 ? ceil(x - 0.5) : floor(x + 0.5))

/* dispersion.c's delay helpers call doppler(), which lives in PRESTO's
 * barycenter.c beside the TEMPO driver; restated here
 * (third_party/presto/src/barycenter.c:3-10): the emitted frequency for an
 * observed one at radial velocity voverc (v/c). */
double doppler(double freq_observed, double voverc)
{
    return freq_observed * (1.0 + voverc);
}

/* Tables of src/prep_dedisp.c for -lodm/-dmstep/-numdms/-nsub and an
 * observation with the centre frequency of its lowest channel `lofreq`
 * (idata.freq), channel width `chanwid` (MHz) and sample time `dt`. */
int odd_tables(int nchan, int nsub, int ndm, double lodm, double dmstep, double lofreq,
               double chanwid, double dt, int downsamp, int spectra_per_subint,
               int *idispdt, int *offsets, int *blocksperread, double *avgdm_out)
{
    int ii, jj;
    double avgdm = 0.0, maxdm;
    double *dms = (double *)malloc(sizeof(double) * ndm);
    for (ii = 0; ii < ndm; ii++) {
        dms[ii] = lodm + ii * dmstep;
        avgdm += dms[ii];
    }
    avgdm /= ndm;
    maxdm = dms[ndm - 1];
    const double dsdt = downsamp * dt;
    const double bw_ddelay = delay_from_dm(maxdm, lofreq) -
                             delay_from_dm(maxdm, lofreq + (nchan - 1) * chanwid);
    *blocksperread = ((int)(bw_ddelay / dt) / spectra_per_subint + 1);

    double *dispdt = subband_search_delays(nchan, nsub, avgdm, lofreq, chanwid, 0.0);
    for (ii = 0; ii < nchan; ii++) idispdt[ii] = NEAREST_LONG(dispdt[ii] / dt);
    vect_free(dispdt);
    for (ii = 0; ii < ndm; ii++) {
        double *subdispdt = subband_delays(nchan, nsub, dms[ii], lofreq, chanwid, 0.0);
        const double dtmp = subdispdt[nsub - 1];
        for (jj = 0; jj < nsub; jj++)
            offsets[ii * nsub + jj] = NEAREST_LONG((subdispdt[jj] - dtmp) / dsdt);
        vect_free(subdispdt);
    }
    free(dms);
    if (avgdm_out) *avgdm_out = avgdm;
    return 0;
}

/* Blocks of `L` spectra in the raw file of `nspec` spectra. */
typedef struct {
    const unsigned char *raw;
    long long nspec;
    int nchan, L;
    long long next;          /* next block to read */
} Reader;

/* One block converted to PRESTO order, clipped when clip_sigma > 0, and
 * transposed channel-major; 0 when no full block is left. */
static float g_clip_sigma;
static float *g_timemajor, *g_padvals;
static long long g_nclipped;
static float *g_levels;             /* optional: clip_times' channel levels per block */
static long long g_levels_nblocks;

static int read_block(Reader *r, float *chanmajor)
{
    if ((r->next + 1) * (long long)r->L > r->nspec) return 0;
    const unsigned char *b = r->raw + r->next * (long long)r->L * r->nchan;
    if (g_clip_sigma > 0.0f) {
        for (int t = 0; t < r->L; t++)
            for (int c = 0; c < r->nchan; c++)
                g_timemajor[(long long)t * r->nchan + c] =
                    (float)b[(long long)t * r->nchan + (r->nchan - 1 - c)];
        g_nclipped += clip_times(g_timemajor, r->L, r->nchan, g_clip_sigma, g_padvals, 1);
        if (g_levels && r->next < g_levels_nblocks)
            memcpy(g_levels + r->next * r->nchan, g_padvals, sizeof(float) * r->nchan);
        for (int t = 0; t < r->L; t++)
            for (int c = 0; c < r->nchan; c++)
                chanmajor[(long long)c * r->L + t] = g_timemajor[(long long)t * r->nchan + c];
    } else {
        for (int t = 0; t < r->L; t++)
            for (int c = 0; c < r->nchan; c++)
                chanmajor[(long long)c * r->L + t] =
                    (float)b[(long long)t * r->nchan + (r->nchan - 1 - c)];
    }
    r->next++;
    return 1;
}

/* The prepsubband output of every DM: out[d*out_stride + t] for
 * t < *nout_written (at most numout).  raw is [nspec][nchan], 8-bit,
 * SIGPROC order (highest frequency first). */
int odd_run(const unsigned char *raw, long long nspec, int nchan, int nsub, int ndm,
            int L, int bpr, const int *idispdt, const int *offsets_in, long long numout,
            float *out, long long out_stride, long long *nout_written)
{
    const int worklen = L * bpr;
    float *raw1 = calloc((size_t)L * nchan, sizeof(float));
    float *raw2 = calloc((size_t)L * nchan, sizeof(float));
    float *cur = calloc((size_t)nsub * worklen, sizeof(float));
    float *last = calloc((size_t)nsub * worklen, sizeof(float));
    float *tmp = calloc((size_t)worklen, sizeof(float));
    int *idisp = malloc(sizeof(int) * nchan);
    int *offs = malloc(sizeof(int) * nsub);
    memcpy(idisp, idispdt, sizeof(int) * nchan);
    Reader rd = {raw, nspec, nchan, L, 0};
    float *rcur = raw1, *rlast = raw2, *sw;
    int primed = 0, first_chunk = 1;
    long long totwrote = 0;
    *nout_written = 0;

    /* read_subbands: one subband block per call, one raw block of latency */
    #define READ_SUBBANDS(dst_chunk, blk) ({                                   \
        int ok_ = 0;                                                           \
        if (!primed) { primed = 1; if (read_block(&rd, rcur)) {                \
            sw = rcur; rcur = rlast; rlast = sw; } }                           \
        if (read_block(&rd, rcur)) {                                           \
            dedisp_subbands(rcur, rlast, L, nchan, idisp, nsub, (dst_chunk),   \
                            bpr, (blk) + 1);                                   \
            sw = rcur; rcur = rlast; rlast = sw; ok_ = 1; }                    \
        ok_; })

    for (;;) {
        long long totnumread = 0;
        for (int pass = 0; pass < (first_chunk ? 2 : 1); pass++) {
            for (int ii = 0; ii < bpr; ii++) {
                int ok = READ_SUBBANDS(cur, ii);
                if (!ok)
                    for (int jj = 0; jj < nsub; jj++)
                        memset(cur + (long long)jj * worklen + (long long)ii * L, 0,
                               sizeof(float) * L);
                if (!(first_chunk && pass == 0)) totnumread += ok ? L : 0;
            }
            if (first_chunk && pass == 0) { sw = cur; cur = last; last = sw; }
        }
        first_chunk = 0;
        /* float_dedisp over the subband chunks, per DM */
        long long towrite = totnumread == worklen ? worklen : 0;
        if (totwrote + towrite > numout) towrite = numout - totwrote;
        for (int d = 0; d < ndm && towrite > 0; d++) {
            memcpy(offs, offsets_in + (long long)d * nsub, sizeof(int) * nsub);
            float_dedisp(cur, last, worklen, nsub, offs, 0.0f, tmp, 1);
            memcpy(out + (long long)d * out_stride + totwrote, tmp, sizeof(float) * towrite);
        }
        sw = cur; cur = last; last = sw;
        totwrote += towrite;
        if (totnumread != worklen || totwrote == numout) break;
    }
    #undef READ_SUBBANDS
    *nout_written = totwrote;
    free(raw1); free(raw2); free(cur); free(last); free(tmp); free(idisp); free(offs);
    return 0;
}

/* odd_run with prepsubband's -clip clip_sigma; *nclipped = spectra replaced. */
/* Record, for the next odd_run_clip, the good_chan_levels that clip_times
 * leaves after each raw block (PRESTO channel order, ascending frequency):
 * levels[b * nchan + c] for blocks b < nblocks; NULL stops recording. */
void odd_clip_levels_to(float *levels, long long nblocks)
{
    g_levels = levels;
    g_levels_nblocks = levels ? nblocks : 0;
}

int odd_run_clip(const unsigned char *raw, long long nspec, int nchan, int nsub, int ndm,
                 int L, int bpr, const int *idispdt, const int *offsets_in, long long numout,
                 float *out, long long out_stride, long long *nout_written, float clip_sigma,
                 long long *nclipped)
{
    g_clip_sigma = clip_sigma;
    g_nclipped = 0;
    g_timemajor = calloc((size_t)L * nchan, sizeof(float));
    g_padvals = calloc((size_t)nchan, sizeof(float));
    const int rc = odd_run(raw, nspec, nchan, nsub, ndm, L, bpr, idispdt, offsets_in, numout,
                           out, out_stride, nout_written);
    free(g_timemajor); free(g_padvals);
    g_timemajor = g_padvals = NULL;
    g_clip_sigma = 0.0f;
    *nclipped = g_nclipped;
    return rc;
}
