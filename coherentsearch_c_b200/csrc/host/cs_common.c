/*
 * Host-side planning shared by the search driver and the GPU backend.
 *
 * Everything here is integer or FP64 bookkeeping that fixes the trial grid,
 * the interpolation tables, the chunk table and the boxcar normalisation.  It
 * must reproduce the reference bit for bit (same operation order, compiled
 * with -ffp-contract=off like src/Makefile:43), because candidate frequencies
 * and S/N scales are derived from it.  Each function names the reference
 * lines whose arithmetic it restates.
 *
 * This file is compiled into libcoherent_search.so (exported) and into
 * libcsgpu.so (hidden), so the GPU backend is self-contained when it is
 * linked into a reference program in place of src/cuda.cu.
 */
#include "coherent_search.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.141592653589793238462643383279502884
#endif

#ifdef CS_HIDDEN
#define CS_API __attribute__((visibility("hidden")))
#else
#define CS_API
#endif

/* ------------------------------------------------------------------ */
/* Julia-compatible trigonometry, src/interp.c:17-43                  */
/* ------------------------------------------------------------------ */
CS_API double cs_sinpi(double x)
{
    if (!isfinite(x)) return x - x;
    double r = fmod(x, 2.0);
    if (r < 0) r += 2.0;
    if (r == 0.0 || r == 1.0) return 0.0 * r;
    if (r == 0.5) return 1.0;
    if (r == 1.5) return -1.0;
    return sin(M_PI * r);
}

CS_API double cs_cospi(double x)
{
    if (!isfinite(x)) return x - x;
    double r = fmod(x, 2.0);
    if (r < 0) r += 2.0;
    if (r == 0.0) return 1.0;
    if (r == 0.5 || r == 1.5) return 0.0;
    if (r == 1.0) return -1.0;
    return cos(M_PI * r);
}

CS_API double cs_eps(double x)
{
    x = fabs(x);
    if (x == 0.0) return 4.9406564584124654e-324;
    return nextafter(x, INFINITY) - x;
}

/* ------------------------------------------------------------------ */
/* Parameters, src/interp.c:48-75                                     */
/* ------------------------------------------------------------------ */
CS_API int decimation_set(int nharms, int maxdecim, int *out, int outcap)
{
    int n = 0, k;
    if (maxdecim < 1) maxdecim = 1;
    for (k = 1; k <= maxdecim; k++) {
        if (nharms / k < 2) continue;
        if (n < outcap) out[n] = k;
        n++;
    }
    return n < outcap ? n : outcap;
}

CS_API void params_defaults(SearchParams *p)
{
    memset(p, 0, sizeof(*p));
    p->nharms = 60;
    p->m = 16;
    p->numbetween = 16;
    p->hidr = 0.5;
    p->threshold = 8.0;
    p->boxcar_fsp = 1.5;
    p->boxcar_maxfrac = 0.3;
    p->boxcar_gatemargin = 0.01;
    p->precision = CS_PREC_F32;
    p->sigma = CS_SIGMA_ANALYTIC;
    p->ndecim = decimation_set(p->nharms, 6, p->decimations, 64);
}

/* ------------------------------------------------------------------ */
/* Rational trial step, src/interp.c:80-118                           */
/* Continued-fraction convergents of lodr until one is within 1e-13,  */
/* with denominator at most CS_DIRECT_QMAX.                           */
/* ------------------------------------------------------------------ */
CS_API int trial_grid_rational(double lodr, int *pnum_out, int *q_out)
{
    const double tol = 1e-13;
    if (!(lodr > 0.0)) return 0;
    long long hm2 = 0, km2 = 1;      /* convergent n-2 */
    long long hm1 = 1, km1 = 0;      /* convergent n-1 */
    long long p = 0, q = 1;
    double y = lodr;
    int hit = 0, iter;
    for (iter = 0; iter < 200; iter++) {
        double a_f = floor(y);
        if (a_f > 2.0e9) break;
        long long a = (long long)a_f;
        __int128 hn = (__int128)a * hm1 + hm2;
        __int128 kn = (__int128)a * km1 + km2;
        if (hn > (__int128)1e18 || kn > (__int128)1e18) break;
        p = (long long)hn;
        q = (long long)kn;
        hm2 = hm1; km2 = km1; hm1 = p; km1 = q;
        if (q > CS_DIRECT_QMAX) break;
        if (fabs((double)p / (double)q - lodr) <= tol) { hit = 1; break; }
        double frac = y - a_f;
        if (frac <= 0.0) break;
        y = 1.0 / frac;
        if (!isfinite(y)) break;
    }
    if (!hit && q > 0 && q <= CS_DIRECT_QMAX && p >= 1 &&
        fabs((double)p / (double)q - lodr) <= tol)
        hit = 1;
    if (!hit || q <= 0 || q > CS_DIRECT_QMAX || p < 1) return 0;
    if (fabs((double)p / (double)q - lodr) > 8.0 * cs_eps(lodr)) return 0;
    *pnum_out = (int)p;
    *q_out = (int)q;
    return 1;
}

/* ------------------------------------------------------------------ */
/* Per-harmonic interpolation tables, src/interp.c:219-303            */
/* ------------------------------------------------------------------ */
static long long gcd_ll(long long a, long long b)
{
    if (a < 0) a = -a;
    if (b < 0) b = -b;
    while (b) { long long t = a % b; a = b; b = t; }
    return a;
}

static void plan_release(DirectPlan *dp)
{
    free(dp->row); free(dp->W); free(dp->A_re); free(dp->A_im); free(dp->carry);
    free(dp->grow); free(dp->goff); free(dp->gnj); free(dp->gW);
    free(dp->gA_re); free(dp->gA_im);
    memset(dp, 0, sizeof(*dp));
}

/* Phase cycle of harmonic h on the rational grid: trial t has Fourier
 * position h*r_lo + t*h*pnum/q, i.e. residue (t*s) mod q of the fractional
 * step, so only P = q/gcd(h*pnum, q) distinct fractional offsets occur.
 * For each offset: the carry into the next integer bin, the m sinc weights
 * W[i] = 1/(dr - (i+1-m/2)) and the phase factor conj-rotation A. */
static int plan_one(DirectPlan *dp, int h, const SearchParams *sp, double r_lo,
                    int rational, int pnum, int q)
{
    const int m = sp->m, m2 = m / 2;
    memset(dp, 0, sizeof(*dp));
    dp->h = h;
    dp->m = m;
    dp->pnum = pnum;
    dp->q = q;
    const double hr = (double)h * r_lo;
    dp->rfloor0 = (int)floor(hr);
    dp->dr0 = hr - (double)dp->rfloor0;
    if (!rational) return 0;           /* P = 0: no tabulated kernel */

    const long long step = (long long)h * pnum;
    dp->s = (int)(step % q);
    dp->base_adv = (int)(step / q);
    dp->P = (int)(q / gcd_ll(step, q));
    const int P = dp->P;
    dp->row = (int32_t *)calloc((size_t)q, sizeof(int32_t));
    dp->W = (float *)malloc((size_t)m * P * sizeof(float));
    dp->A_re = (float *)malloc((size_t)P * sizeof(float));
    dp->A_im = (float *)malloc((size_t)P * sizeof(float));
    dp->carry = (uint8_t *)malloc((size_t)P);
    if (!dp->row || !dp->W || !dp->A_re || !dp->A_im || !dp->carry) return -1;

    int res = 0, ph;
    for (ph = 0; ph < P; ph++) {
        dp->row[res] = ph + 1;
        const double u = dp->dr0 + (double)res / (double)q;
        const int carry = (u >= 1.0);
        const double dr = carry ? u - 1.0 : u;
        float *w = dp->W + (size_t)ph * m;
        dp->carry[ph] = (uint8_t)carry;
        if (dr == 0.0) {
            int i;
            dp->A_re[ph] = 1.0f;
            dp->A_im[ph] = 0.0f;
            for (i = 0; i < m; i++) w[i] = (i == m2 - 1) ? 1.0f : 0.0f;
        } else {
            const double sn = cs_sinpi(dr), cs = cs_cospi(dr);
            int i;
            dp->A_re[ph] = (float)(sn * cs / M_PI);
            dp->A_im[ph] = (float)(-sn * sn / M_PI);
            for (i = 0; i < m; i++)
                w[i] = (float)(1.0 / (dr - (double)(i + 1 - m2)));
        }
        res += dp->s;
        if (res >= q) res -= q;
    }
    return 0;
}

CS_API int direct_plans_build(DirectPlanSet *set, const SearchParams *p, double r_lo)
{
    memset(set, 0, sizeof(*set));
    if (p->m <= 0 || (p->m & 1)) {
        fprintf(stderr, "Error: m must be a positive even integer\n");
        return -1;
    }
    const double lodr = p->hidr / (double)p->nharms;
    int pnum = 0, q = 0;
    const int rational = trial_grid_rational(lodr, &pnum, &q);
    set->n = p->nharms;
    set->plans = (DirectPlan *)calloc((size_t)set->n, sizeof(DirectPlan));
    if (!set->plans) return -1;
    int h;
    for (h = 1; h <= p->nharms; h++) {
        if (plan_one(&set->plans[h - 1], h, p, r_lo, rational, pnum, q) != 0) {
            direct_plans_free(set);
            return -1;
        }
    }
    return 0;
}

CS_API void direct_plans_free(DirectPlanSet *set)
{
    int i;
    if (!set) return;
    for (i = 0; i < set->n; i++) plan_release(&set->plans[i]);
    free(set->plans);
    set->plans = NULL;
    set->n = 0;
}

/* ------------------------------------------------------------------ */
/* Harmonic availability, src/interp.c:349-416                        */
/* ------------------------------------------------------------------ */
CS_API void cs_chunk_state(const DirectPlan *dp, long long t, int *res, long long *qint)
{
    const __int128 prod = (__int128)t * (long long)(dp->h * dp->pnum);
    const long long q = dp->q;
    long long rem = (long long)(prod % q);
    if (rem < 0) rem += q;
    *res = (int)rem;
    *qint = (long long)(prod / q);
}

/* Fourier position of harmonic h at trial t for the non-rational grid. */
static double slow_position(const DirectPlan *dp, const SearchParams *p, long long t)
{
    return (double)(dp->rfloor0 + dp->dr0) +
           (double)t * ((double)dp->h * (p->hidr / (double)p->nharms));
}

/* Window base bin and integer part of the position, both 0-based. */
static void position_at(const DirectPlan *dp, const SearchParams *p, long long t,
                        long long *base, long long *nyqbin)
{
    if (dp->P == 0) {
        const double r = slow_position(dp, p, t);
        *base = (long long)floor(r + 1e-15);
        *nyqbin = (long long)floor(r);
        return;
    }
    int res;
    long long qint;
    cs_chunk_state(dp, t, &res, &qint);
    const int ph = dp->row[res] - 1;
    *base = (long long)dp->rfloor0 + qint + (dp->carry[ph] ? 1 : 0);
    *nyqbin = (long long)dp->rfloor0 + qint;
}

CS_API int cs_harmonic_fits(const DirectPlan *dp, const FFTFile *ft,
                            const SearchParams *p, long long t)
{
    const int m2 = dp->m / 2;
    long long base, nyqbin;
    position_at(dp, p, t, &base, &nyqbin);
    return (base + 2 - m2) >= 1 && (base + 1 + m2) <= ft->namps &&
           nyqbin < ft->N / 2;
}

/* ------------------------------------------------------------------ */
/* Chunk table, src/interp.c:866-966                                  */
/* ------------------------------------------------------------------ */
typedef struct { int m2; long long namps, nhalf; } FitBounds;

static int fits_low(const DirectPlan *dp, const SearchParams *p, long long t,
                    const FitBounds *fb)
{
    long long base, nyqbin;
    position_at(dp, p, t, &base, &nyqbin);
    /* src/interp.c:360-372 returns the base as int before comparing */
    return (int)base + 2 - fb->m2 >= 1;
}

static int fits_high(const DirectPlan *dp, const SearchParams *p, long long t,
                     const FitBounds *fb)
{
    long long base, nyqbin;
    position_at(dp, p, t, &base, &nyqbin);
    return (long long)((int)base + 1 + fb->m2) <= fb->namps &&
           (long long)(int)nyqbin < fb->nhalf;
}

/* First trial in [0,total) where a monotone predicate turns true (or false). */
static long long first_switch(int (*pred)(const DirectPlan *, const SearchParams *,
                                          long long, const FitBounds *),
                              int want, const DirectPlan *dp, const SearchParams *p,
                              long long total, const FitBounds *fb)
{
    if (total < 1) return total;
    if ((pred(dp, p, 0, fb) != 0) == want) return 0;
    if ((pred(dp, p, total - 1, fb) != 0) != want) return total;
    long long lo = 0, hi = total - 1;
    while (hi - lo > 1) {
        const long long mid = (lo + hi) >> 1;
        if ((pred(dp, p, mid, fb) != 0) == want) hi = mid; else lo = mid;
    }
    return hi;
}

static int cmp_ll(const void *a, const void *b)
{
    const long long x = *(const long long *)a, y = *(const long long *)b;
    return (x > y) - (x < y);
}

static long long sort_unique_ll(long long *v, long long n)
{
    long long i, m = 0;
    qsort(v, (size_t)n, sizeof(long long), cmp_ll);
    for (i = 0; i < n; i++)
        if (m == 0 || v[i] != v[m - 1]) v[m++] = v[i];
    return m;
}

CS_API int harmonic_change_trials(const DirectPlanSet *set, const FFTFile *ft,
                                  const SearchParams *p, long long total,
                                  long long **out_bnds)
{
    *out_bnds = NULL;
    if (total <= 1) return 0;
    long long *b = (long long *)malloc((size_t)(2 * set->n + 1) * sizeof(long long));
    if (!b) return 0;
    long long n = 0;
    FitBounds fb;
    fb.namps = ft->namps;
    fb.nhalf = ft->N / 2;
    int i;
    for (i = 0; i < set->n; i++) {
        const DirectPlan *dp = &set->plans[i];
        fb.m2 = dp->m / 2;
        /* the reference stores these as int (src/interp.c:930-931) */
        const int on = (int)first_switch(fits_low, 1, dp, p, total, &fb);
        const int off = (int)first_switch(fits_high, 0, dp, p, total, &fb);
        if (on > 0 && on < total) b[n++] = on;
        if (off > 0 && off < total) b[n++] = off;
    }
    *out_bnds = b;
    return (int)sort_unique_ll(b, n);
}

CS_API int chunk_starts(const DirectPlanSet *set, const FFTFile *ft, const SearchParams *p,
                        long long total, int Nprof, long long **out, long long *nout)
{
    *out = NULL;
    *nout = 0;
    if (total < 1) return 0;
    long long *bnds = NULL;
    const int nb = harmonic_change_trials(set, ft, p, total, &bnds);
    const long long nreg = (total + Nprof - 1) / Nprof;
    long long *s = (long long *)malloc((size_t)(nreg + nb + 1) * sizeof(long long));
    if (!s) { free(bnds); return -1; }
    long long n = 0, t;
    int i;
    for (t = 0; t < total; t += Nprof) s[n++] = t;
    for (i = 0; i < nb; i++) s[n++] = bnds[i];
    free(bnds);
    *nout = sort_unique_ll(s, n);
    *out = s;
    return 0;
}

/* ------------------------------------------------------------------ */
/* Boxcar width banks and noise scales, src/boxcar.c:78-198           */
/* ------------------------------------------------------------------ */
CS_API int boxcar_widths(int nbins, double fsp, double maxfrac, int *out, int cap)
{
    if (nbins < 2) return 0;
    int wmax = (int)floor(maxfrac * (double)nbins);
    if (wmax < 1) wmax = 1;
    if (wmax > nbins - 1) wmax = nbins - 1;
    int n = 0, w = 1;
    while (w <= wmax) {
        if (n < cap) out[n] = w;
        n++;
        const int grown = (int)floor(fsp * (double)w);
        w = grown > w + 1 ? grown : w + 1;
    }
    return n < cap ? n : cap;
}

static int cmp_int(const void *a, const void *b)
{
    const int x = *(const int *)a, y = *(const int *)b;
    return (x > y) - (x < y);
}

/* Ladder pruning: with a decimation ladder whose factors grow by at most
 * LADDER_WMAX/2 per step, width 1 is kept only at the smallest factor and
 * widths above LADDER_WMAX only at the largest (longer pulses are seen at
 * the next factor up). */
CS_API int ladder_boxcar_widths(int nbins, int k, const SearchParams *p, int *out, int cap)
{
    int full[256];
    const int nf = boxcar_widths(nbins, p->boxcar_fsp, p->boxcar_maxfrac, full, 256);
    const int nfull = nf < cap ? nf : cap;
    if (p->ndecim <= 1) {
        memcpy(out, full, (size_t)nfull * sizeof(int));
        return nfull;
    }
    int ks[64], i;
    const int nk = p->ndecim < 64 ? p->ndecim : 64;
    memcpy(ks, p->decimations, (size_t)nk * sizeof(int));
    qsort(ks, (size_t)nk, sizeof(int), cmp_int);
    for (i = 0; i + 1 < nk; i++) {
        if (ks[i + 1] > (CS_LADDER_WMAX / 2) * ks[i]) {
            memcpy(out, full, (size_t)nfull * sizeof(int));
            return nfull;
        }
    }
    const int kmin = ks[0], kmax = ks[nk - 1];
    int n = 0;
    for (i = 0; i < nf; i++) {
        const int w = full[i];
        const int keep_lo = (w >= 2) || (k == kmin);
        const int keep_hi = (w <= CS_LADDER_WMAX) || (k == kmax);
        if (keep_lo && keep_hi) {
            if (n < cap) out[n] = w;
            n++;
        }
    }
    if (n == 0) {
        memcpy(out, full, (size_t)nfull * sizeof(int));
        return nfull;
    }
    return n < cap ? n : cap;
}

/* Noise scale of the unnormalised c2r profile of the decimated stack
 * {k, 2k, ..., Hk*k}: each filled non-Nyquist harmonic contributes variance
 * 2 (unit-power complex noise, counted twice), the Nyquist 0.5. */
CS_API double analytic_sigma(const uint8_t *filled, int k, int Hk)
{
    int nlow = 0, j;
    for (j = 1; j <= Hk - 1; j++)
        if (filled[j * k - 1]) nlow++;
    const int nnyq = filled[Hk * k - 1] ? 1 : 0;
    if (nlow + nnyq < 1) return 0.0;
    return sqrt(2.0 * nlow + 0.5 * nnyq);
}

/* Exact noise std of a width-w boxcar over that profile, relative to sigma:
 * shape[w] = sigma / std(boxcar_w). */
CS_API void boxcar_shape(double *shape, int nbins, const int *widths, int nw,
                         const uint8_t *filled, int k, int Hk)
{
    const double sigma = analytic_sigma(filled, k, Hk);
    int i;
    for (i = 0; i < nw; i++) {
        const int w = widths[i];
        double v = 0.0;
        int j;
        for (j = 1; j <= Hk - 1; j++) {
            if (!filled[j * k - 1]) continue;
            const double d = cs_sinpi((double)(j * w) / (double)nbins) /
                             cs_sinpi((double)j / (double)nbins);
            v += 2.0 * d * d;
        }
        if (filled[Hk * k - 1]) {
            const double d = cs_sinpi(0.5 * (double)w);
            v += 0.5 * d * d;
        }
        shape[i] = (sigma > 0.0 && v > 0.0) ? sigma / sqrt(v) : 0.0;
    }
}

/* ------------------------------------------------------------------ */
/* Candidate lists, src/candidate.c:11-93                             */
/* ------------------------------------------------------------------ */
CS_API void candlist_init(CandidateList *l) { l->v = NULL; l->n = 0; l->cap = 0; }

CS_API void candlist_free(CandidateList *l)
{
    free(l->v);
    l->v = NULL;
    l->n = 0;
    l->cap = 0;
}

CS_API void candlist_push(CandidateList *l, Candidate c)
{
    if (l->n == l->cap) {
        const size_t nc = l->cap ? 2 * l->cap : 256;
        Candidate *v = (Candidate *)realloc(l->v, nc * sizeof(Candidate));
        if (!v) return;
        l->v = v;
        l->cap = nc;
    }
    l->v[l->n++] = c;
}

CS_API void candlist_append(CandidateList *dst, const CandidateList *src)
{
    size_t i;
    for (i = 0; i < src->n; i++) candlist_push(dst, src->v[i]);
}

typedef int (*cand_cmp)(const Candidate *, const Candidate *);

static int by_metric_desc(const Candidate *a, const Candidate *b)
{
    return (b->metric > a->metric) - (b->metric < a->metric);
}
static int by_freq(const Candidate *a, const Candidate *b)
{
    return (a->freq > b->freq) - (a->freq < b->freq);
}
static int by_r(const Candidate *a, const Candidate *b)
{
    return (a->r > b->r) - (a->r < b->r);
}

/* Stable top-down merge sort (any stable sort yields the same order). */
static void msort(Candidate *v, Candidate *tmp, size_t n, cand_cmp cmp)
{
    if (n < 2) return;
    const size_t h = n / 2;
    msort(v, tmp, h, cmp);
    msort(v + h, tmp, n - h, cmp);
    size_t a = 0, b = h, k = 0;
    while (a < h && b < n) {
        if (cmp(&v[b], &v[a]) < 0) tmp[k++] = v[b++];
        else tmp[k++] = v[a++];
    }
    while (a < h) tmp[k++] = v[a++];
    while (b < n) tmp[k++] = v[b++];
    memcpy(v, tmp, n * sizeof(Candidate));
}

static void stable_sort(CandidateList *l, cand_cmp cmp)
{
    if (l->n < 2) return;
    Candidate *tmp = (Candidate *)malloc(l->n * sizeof(Candidate));
    if (!tmp) return;
    msort(l->v, tmp, l->n, cmp);
    free(tmp);
}

CS_API void candlist_sort_metric_desc(CandidateList *l) { stable_sort(l, by_metric_desc); }
CS_API void candlist_sort_freq(CandidateList *l) { stable_sort(l, by_freq); }
CS_API void candlist_sort_r(CandidateList *l) { stable_sort(l, by_r); }
CS_API void candlist_sort_metric_desc_stable(CandidateList *l) { stable_sort(l, by_metric_desc); }
CS_API void candlist_sort_freq_stable(CandidateList *l) { stable_sort(l, by_freq); }
CS_API void candlist_sort_r_stable(CandidateList *l) { stable_sort(l, by_r); }
