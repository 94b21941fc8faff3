/*
 * Test infrastructure (oracle).  Not product code.
 *
 * CPU restatement of the CoherentSearch_C hot path, one trial at a time:
 *   trial grid       src/interp.c:80-118 (continued fractions, tol 1e-13)
 *   interpolation    src/interp.c:219-281 (weights and phase factor of the
 *                    phase offset), src/cuda.cu:86-140 (FP32 FMA chain over
 *                    the m-bin window, then the unfused complex rotation)
 *   availability     src/interp.c:386-405 (harmonic fits), chunk filled set
 *                    at both chunk ends (src/cuda.cu:899-913)
 *   c2r profile      FFTW c2r definition (src/search.c:288-292), evaluated
 *                    directly in FP64 (rounded to FP32 in the f32 mode)
 *   folds            src/search.c:294-331 (FP32 sum, times 1/k)
 *   decimated c2r    src/search.c:402-407 (strided stack, Hk*k as Nyquist)
 *   boxcar metric    src/boxcar.c:203-252 (cyclic prefix, widths scan)
 *   noise scales     src/boxcar.c:78-198 (ladder widths, analytic sigma,
 *                    boxcar shape)
 *   Nyquist limit    src/search.c:616-629
 * Straightforward loops, no tables: slow, exact, and independent of the
 * product code it checks.
 */
#include "cs_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define PI_D 3.141592653589793238462643383279502884

static double sinpi_j(double x)
{
    if (!isfinite(x)) return x - x;
    double r = fmod(x, 2.0);
    if (r < 0) r += 2.0;
    if (r == 0.0 || r == 1.0) return 0.0 * r;
    if (r == 0.5) return 1.0;
    if (r == 1.5) return -1.0;
    return sin(PI_D * r);
}

static double cospi_j(double x)
{
    if (!isfinite(x)) return x - x;
    double r = fmod(x, 2.0);
    if (r < 0) r += 2.0;
    if (r == 0.0) return 1.0;
    if (r == 0.5 || r == 1.5) return 0.0;
    if (r == 1.0) return -1.0;
    return cos(PI_D * r);
}

static int rational(double x, long long *pn, long long *qn)
{
    const double tol = 1e-13;
    long long a0 = 0, b0 = 1, a1 = 1, b1 = 0, p = 0, q = 1;
    double y = x;
    int k;
    if (!(x > 0.0)) return 0;
    for (k = 0; k < 200; k++) {
        double f = floor(y);
        if (f > 2.0e9) break;
        long long a = (long long)f;
        p = a * a1 + a0;
        q = a * b1 + b0;
        a0 = a1; b0 = b1; a1 = p; b1 = q;
        if (q > 65536) break;
        if (fabs((double)p / (double)q - x) <= tol) break;
        double fr = y - f;
        if (fr <= 0.0) break;
        y = 1.0 / fr;
    }
    if (q < 1 || q > 65536 || p < 1) return 0;
    if (fabs((double)p / (double)q - x) > tol) return 0;
    *pn = p;
    *qn = q;
    return 1;
}

typedef struct {
    const float *amps;
    long long namps, N;
    int nh, m;
    double r_lo;
    long long pnum, q;
} Geo;

/* Position of harmonic h at trial t: window base bin, fractional offset,
 * and the integer bin used by the Nyquist test. */
static void position(const Geo *g, int h, long long t, long long *base, double *dr,
                     long long *nyqbin)
{
    const double hr = (double)h * g->r_lo;
    const int rf0 = (int)floor(hr);
    const double dr0 = hr - (double)rf0;
    const __int128 prod = (__int128)t * (__int128)(h * g->pnum);
    const long long res = (long long)(prod % g->q);
    const long long qint = (long long)(prod / g->q);
    const double u = dr0 + (double)res / (double)g->q;
    const int carry = u >= 1.0;
    *dr = carry ? u - 1.0 : u;
    *base = (long long)rf0 + qint + carry;
    *nyqbin = (long long)rf0 + qint;
}

static int fits(const Geo *g, int h, long long t)
{
    long long base, nyq;
    double dr;
    position(g, h, t, &base, &dr, &nyq);
    const int m2 = g->m / 2;
    return base + 2 - m2 >= 1 && base + 1 + m2 <= g->namps && nyq < g->N / 2;
}

static void interpolate(const Geo *g, int h, long long t, float *xr, float *xi)
{
    long long base, nyq;
    double dr;
    position(g, h, t, &base, &dr, &nyq);
    const int m = g->m, m2 = m / 2;
    float are, aim;
    float w[64];
    int i;
    if (dr == 0.0) {
        are = 1.0f; aim = 0.0f;
        for (i = 0; i < m; i++) w[i] = (i == m2 - 1) ? 1.0f : 0.0f;
    } else {
        const double s = sinpi_j(dr), c = cospi_j(dr);
        are = (float)(s * c / PI_D);
        aim = (float)(-s * s / PI_D);
        for (i = 0; i < m; i++) w[i] = (float)(1.0 / (dr - (double)(i + 1 - m2)));
    }
    float ar = 0.0f, ai = 0.0f;
    const long long b0 = base + 1 - m2;
    for (i = 0; i < m; i++) {
        const long long idx = b0 + i;
        float vr = 0.0f, vi = 0.0f;
        if (idx >= 0 && idx < g->namps) { vr = g->amps[2 * idx]; vi = g->amps[2 * idx + 1]; }
        ar = fmaf(w[i], vr, ar);
        ai = fmaf(w[i], vi, ai);
    }
    const float p1 = are * ar, p2 = aim * ai, p3 = are * ai, p4 = aim * ar;
    *xr = p1 - p2;
    *xi = p3 + p4;
}

/* Unnormalised c2r of the stack X[j] = (re, im) of harmonics j*k, j=1..H. */
static double tw_cos[512], tw_sin[512];
static int tw_n = 0;

static void c2r(const double *Xr, const double *Xi, int H, double *y)
{
    const int n = 2 * H;
    int j, t;
    if (tw_n != n) {
        for (t = 0; t < n; t++) {
            const double a = 2.0 * PI_D * (double)t / (double)n;
            tw_cos[t] = cos(a);
            tw_sin[t] = sin(a);
        }
        tw_n = n;
    }
    for (t = 0; t < n; t++) {
        double acc = 0.0;
        for (j = 1; j < H; j++) {
            const int ph = (int)(((long long)j * t) % n);
            acc += 2.0 * (Xr[j] * tw_cos[ph] - Xi[j] * tw_sin[ph]);
        }
        acc += (t & 1) ? -Xr[H] : Xr[H];
        y[t] = acc;
    }
}

static int widths_full(int nb, double fsp, double maxfrac, int *out)
{
    if (nb < 2) return 0;
    int wmax = (int)floor(maxfrac * (double)nb);
    if (wmax < 1) wmax = 1;
    if (wmax > nb - 1) wmax = nb - 1;
    int n = 0, w = 1;
    while (w <= wmax && n < 64) {
        out[n++] = w;
        int nw = (int)floor(fsp * (double)w);
        w = nw > w + 1 ? nw : w + 1;
    }
    return n;
}

static int widths_ladder(int nb, int k, int ndecim, const int *decims, double fsp,
                         double maxfrac, int *out)
{
    int full[64];
    const int nf = widths_full(nb, fsp, maxfrac, full);
    int i, j;
    if (ndecim <= 1) { memcpy(out, full, nf * sizeof(int)); return nf; }
    int ks[64];
    const int nk = ndecim < 64 ? ndecim : 64;
    memcpy(ks, decims, nk * sizeof(int));
    for (i = 1; i < nk; i++)            /* insertion sort */
        for (j = i; j > 0 && ks[j - 1] > ks[j]; j--) { int t = ks[j]; ks[j] = ks[j - 1]; ks[j - 1] = t; }
    for (i = 0; i + 1 < nk; i++)
        if (ks[i + 1] > 3 * ks[i]) { memcpy(out, full, nf * sizeof(int)); return nf; }
    int n = 0;
    for (i = 0; i < nf; i++) {
        const int w = full[i];
        if ((w >= 2 || k == ks[0]) && (w <= 6 || k == ks[nk - 1])) out[n++] = w;
    }
    if (n == 0) { memcpy(out, full, nf * sizeof(int)); return nf; }
    return n;
}

static double sigma_of(const uint8_t *filled, int k, int Hk)
{
    int nlow = 0, j;
    for (j = 1; j <= Hk - 1; j++) nlow += filled[j * k - 1] ? 1 : 0;
    const int nnyq = filled[Hk * k - 1] ? 1 : 0;
    if (nlow + nnyq < 1) return 0.0;
    return sqrt(2.0 * nlow + 0.5 * nnyq);
}

static double shape_of(const uint8_t *filled, int k, int Hk, int nb, int w)
{
    const double sigma = sigma_of(filled, k, Hk);
    double v = 0.0;
    int j;
    for (j = 1; j <= Hk - 1; j++) {
        if (!filled[j * k - 1]) continue;
        const double d = sinpi_j((double)(j * w) / (double)nb) / sinpi_j((double)j / (double)nb);
        v += 2.0 * d * d;
    }
    if (filled[Hk * k - 1]) {
        const double d = sinpi_j(0.5 * (double)w);
        v += 0.5 * d * d;
    }
    return (sigma > 0.0 && v > 0.0) ? sigma / sqrt(v) : 0.0;
}

static double metric_f32(const float *x, int nb, const int *ws, int nw, const float *invsw)
{
    float ps[512];
    const int wmax = ws[nw - 1];
    int i, p;
    ps[0] = 0.0f;
    for (i = 1; i <= nb + wmax; i++) ps[i] = ps[i - 1] + x[(i > nb ? i - nb : i) - 1];
    const float tot = ps[nb] - ps[0];
    float best = -INFINITY;
    for (i = 0; i < nw; i++) {
        const int w = ws[i];
        const float duty = (float)w / (float)nb;
        float mx = ps[w] - ps[0];
        for (p = 2; p <= nb; p++) {
            const float d = ps[p + w - 1] - ps[p - 1];
            if (d > mx) mx = d;
        }
        const float dt = duty * tot;
        const float c = (mx - dt) * invsw[i];
        if (c > best) best = c;
    }
    return (double)best;
}

static double metric_f64(const double *x, int nb, const int *ws, int nw, const double *invsw)
{
    double ps[512];
    const int wmax = ws[nw - 1];
    int i, p;
    ps[0] = 0.0;
    for (i = 1; i <= nb + wmax; i++) ps[i] = ps[i - 1] + x[(i > nb ? i - nb : i) - 1];
    const double tot = ps[nb] - ps[0];
    double best = -INFINITY;
    for (i = 0; i < nw; i++) {
        const int w = ws[i];
        const double duty = (double)w / (double)nb;
        double mx = ps[w] - ps[0];
        for (p = 2; p <= nb; p++) {
            const double d = ps[p + w - 1] - ps[p - 1];
            if (d > mx) mx = d;
        }
        const double dt = duty * tot;
        const double c = (mx - dt) * invsw[i];
        if (c > best) best = c;
    }
    return best;
}

static long long chunk_of(const long long *cs, long long nchunks, long long t)
{
    long long lo = 0, hi = nchunks - 1;
    while (lo < hi) {
        const long long mid = (lo + hi + 1) >> 1;
        if (cs[mid] <= t) lo = mid; else hi = mid - 1;
    }
    return lo;
}

static int setup(Geo *g, const float *amps, long long namps, long long N, int nharms, int m,
                 double hidr, double r_lo)
{
    if (nharms < 1 || nharms > 256 || m < 2 || (m & 1) || m > 64) return -1;
    g->amps = amps; g->namps = namps; g->N = N; g->nh = nharms; g->m = m; g->r_lo = r_lo;
    return rational(hidr / (double)nharms, &g->pnum, &g->q) ? 0 : -1;
}

static void chunk_filled(const Geo *g, const long long *cs, long long nchunks, long long total,
                         long long c, uint8_t *filled, long long *i0, int *n)
{
    *i0 = cs[c];
    *n = (int)((c + 1 < nchunks ? cs[c + 1] : total) - *i0);
    int h;
    for (h = 1; h <= g->nh; h++)
        filled[h - 1] = (uint8_t)(*n > 0 && fits(g, h, *i0) && fits(g, h, *i0 + *n - 1));
}

int cso_trial_metrics(const float *amps, long long namps, long long N,
                      int nharms, int m, double hidr, int ndecim, const int *decims,
                      double fsp, double maxfrac, double r_lo,
                      const long long *cstarts, long long nchunks, long long total,
                      long long t_begin, int count, int prec64, double *metrics)
{
    Geo g;
    if (setup(&g, amps, namps, N, nharms, m, hidr, r_lo) != 0) return -1;
    const int nh = nharms, nb = 2 * nh;
    int ks[64], nslot = 0, i;
    ks[nslot++] = 1;
    for (i = 0; i < ndecim && nslot < 64; i++) if (decims[i] > 1) ks[nslot++] = decims[i];
    const double lodr = hidr / (double)nharms;
    const double nyq = (double)N / 2.0;

    uint8_t filled[256];
    long long cur = -1, i0 = 0;
    int n = 0;
    int ws[64][64], nws[64];
    float invf[64][64];
    double invd[64][64];
    int nvalid[64];
    double Xr[257], Xi[257], y[512], sr[257], si[257];
    float x32[512], f32[512];
    double xd[512];
    int it;
    for (it = 0; it < count; it++) {
        const long long t = t_begin + it;
        const long long c = chunk_of(cstarts, nchunks, t);
        if (c != cur) {
            cur = c;
            chunk_filled(&g, cstarts, nchunks, total, c, filled, &i0, &n);
            const double rstart = r_lo + (double)i0 * lodr;
            int s;
            for (s = 0; s < nslot; s++) {
                const int k = ks[s], Hk = nh / k, nk = 2 * Hk;
                nws[s] = widths_ladder(nk, k, ndecim, decims, fsp, maxfrac, ws[s]);
                const double sig = sigma_of(filled, k, Hk);
                const float sigf = (float)sig;
                const float isf = sigf > 0.0f ? 1.0f / sigf : 0.0f;
                const double isd = sig > 0.0 ? 1.0 / sig : 0.0;
                int w;
                for (w = 0; w < nws[s]; w++) {
                    const double sh = shape_of(filled, k, Hk, nk, ws[s][w]);
                    invf[s][w] = (float)((double)isf * sh);
                    invd[s][w] = isd * sh;
                }
                if (s == 0) { nvalid[s] = n; continue; }
                int lo = 0, hi = n;
                while (lo < hi) {
                    const int mid = lo + ((hi - lo) >> 1);
                    if ((double)k * (rstart + (double)mid * lodr) < nyq) lo = mid + 1;
                    else hi = mid;
                }
                nvalid[s] = lo;
            }
        }
        const int j = (int)(t - i0);
        int h, s;
        Xr[0] = Xi[0] = 0.0;
        for (h = 1; h <= nh; h++) {
            float a = 0.0f, b = 0.0f;
            if (filled[h - 1]) interpolate(&g, h, t, &a, &b);
            Xr[h] = (double)a;
            Xi[h] = (double)b;
        }
        c2r(Xr, Xi, nh, y);
        for (i = 0; i < nb; i++) { x32[i] = (float)y[i]; xd[i] = y[i]; }
        for (s = 0; s < nslot; s++) {
            const int k = ks[s], Hk = nh / k, nk = 2 * Hk;
            double mval;
            if (j >= nvalid[s]) { metrics[(long long)s * count + it] = NAN; continue; }
            if (s == 0) {
                mval = prec64 ? metric_f64(xd, nb, ws[s], nws[s], invd[s])
                              : metric_f32(x32, nb, ws[s], nws[s], invf[s]);
            } else if (nh % k == 0 && nk * k == nb) {
                int q, jj;
                if (prec64) {
                    const double ik = 1.0 / (double)k;
                    for (jj = 0; jj < nk; jj++) {
                        double a = xd[jj];
                        for (q = 1; q < k; q++) a += xd[jj + q * nk];
                        y[jj] = a * ik;
                    }
                    mval = metric_f64(y, nk, ws[s], nws[s], invd[s]);
                } else {
                    const float ik = 1.0f / (float)k;
                    for (jj = 0; jj < nk; jj++) {
                        float a = x32[jj];
                        for (q = 1; q < k; q++) a += x32[jj + q * nk];
                        f32[jj] = a * ik;
                    }
                    mval = metric_f32(f32, nk, ws[s], nws[s], invf[s]);
                }
            } else {
                int jj;
                sr[0] = si[0] = 0.0;
                for (jj = 1; jj <= Hk; jj++) { sr[jj] = Xr[jj * k]; si[jj] = Xi[jj * k]; }
                c2r(sr, si, Hk, y);
                if (prec64) {
                    mval = metric_f64(y, nk, ws[s], nws[s], invd[s]);
                } else {
                    for (jj = 0; jj < nk; jj++) f32[jj] = (float)y[jj];
                    mval = metric_f32(f32, nk, ws[s], nws[s], invf[s]);
                }
            }
            metrics[(long long)s * count + it] = mval;
        }
    }
    return nslot;
}

int cso_trial_profile(const float *amps, long long namps, long long N, int nharms,
                      int m, double hidr, double r_lo, const long long *cstarts,
                      long long nchunks, long long total, long long t, double *prof)
{
    Geo g;
    if (setup(&g, amps, namps, N, nharms, m, hidr, r_lo) != 0) return -1;
    uint8_t filled[256];
    long long i0;
    int n, h;
    chunk_filled(&g, cstarts, nchunks, total, chunk_of(cstarts, nchunks, t), filled, &i0, &n);
    double Xr[257], Xi[257];
    Xr[0] = Xi[0] = 0.0;
    for (h = 1; h <= nharms; h++) {
        float a = 0.0f, b = 0.0f;
        if (filled[h - 1]) interpolate(&g, h, t, &a, &b);
        Xr[h] = a;
        Xi[h] = b;
    }
    c2r(Xr, Xi, nharms, prof);
    return 2 * nharms;
}
