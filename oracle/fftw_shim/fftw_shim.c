/*
 * Test infrastructure (oracle).  Not product code.
 *
 * Restatement of the transforms of FFTW 3.3.10 (the version the reference
 * was validated with, README.md:475-483) that the reference CPU path calls,
 * from their published definitions:
 *   complex DFT   Y[k] = sum_j X[j] exp(sign * 2 pi i j k / n)   (unnormalised)
 *   c2r           y[j] = sum_{k=0}^{n-1} X[k] exp(+2 pi i j k / n) with
 *                 X[n-k] = conj(X[k]); the imaginary parts of X[0] and, for
 *                 even n, X[n/2] are ignored (FFTW's documented convention).
 * Engine: recursive mixed-radix decimation in time (radix 4, 2, 3 and a
 * direct small-prime butterfly), Bluestein's chirp-z convolution for sizes
 * with a prime factor above 31, and the standard half-length packing for the
 * even-length c2r.  Single precision plans compute in float with twiddles
 * rounded from double, like FFTW's fftwf_* plans; double plans in double.
 * The last bits therefore differ from FFTW's own codelets; every parity
 * tolerance in tests/ is set well above that (S/N to 1e-3 relative).
 */
#include "fftw3.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define SHIM_PI 3.14159265358979323846264338327950288

void *fftw_malloc(size_t n)
{
    void *p = NULL;
    if (posix_memalign(&p, 64, n ? n : 64) != 0) return NULL;
    return p;
}
void fftw_free(void *p) { free(p); }
void *fftwf_malloc(size_t n) { return fftw_malloc(n); }
void fftwf_free(void *p) { free(p); }

int fftw_import_wisdom_from_filename(const char *f) { (void)f; return 0; }
int fftwf_import_wisdom_from_filename(const char *f) { (void)f; return 0; }
int fftw_export_wisdom_to_filename(const char *f) { (void)f; return 1; }
int fftwf_export_wisdom_to_filename(const char *f) { (void)f; return 1; }

/* ------------------------------------------------------------------ */
/* Complex FFT engine, instantiated for float (S=f) and double (S=d)   */
/* ------------------------------------------------------------------ */
#define DEFINE_ENGINE(R, S)                                                      \
typedef struct { R re, im; } cx_##S;                                             \
typedef struct eng_##S eng_##S;                                                  \
struct eng_##S {                                                                 \
    int n, sign;                                                                 \
    int nf, fac[64];                                                             \
    cx_##S *tw;          /* exp(sign 2 pi i j / n), j < n */                     \
    int blue;            /* Bluestein */                                         \
    int M;                                                                       \
    cx_##S *chirp;       /* exp(sign pi i j^2 / n), j < n */                     \
    cx_##S *bspec;       /* FFT_M of the conjugate chirp kernel */               \
    eng_##S *fwd, *bwd;  /* power-of-two engines of size M */                    \
    cx_##S *scratch;     /* n (recursion) or 2*M (Bluestein) */                  \
};                                                                               \
                                                                                 \
static eng_##S *eng_new_##S(int n, int sign);                                    \
static void eng_free_##S(eng_##S *e)                                             \
{                                                                                \
    if (!e) return;                                                              \
    free(e->tw); free(e->chirp); free(e->bspec); free(e->scratch);               \
    eng_free_##S(e->fwd); eng_free_##S(e->bwd);                                  \
    free(e);                                                                     \
}                                                                                \
                                                                                 \
static void rec_##S(const eng_##S *e, int n, int tws, const cx_##S *in, long is, \
                    cx_##S *out, int depth)                                      \
{                                                                                \
    if (n == 1) { out[0] = in[0]; return; }                                      \
    const int p = e->fac[depth];                                                 \
    const int m = n / p;                                                         \
    { int r; for (r = 0; r < p; r++)                                             \
        rec_##S(e, m, tws * p, in + (long)r * is, is * p, out + (long)r * m,     \
                depth + 1); }                                                    \
    const int N = e->n;                                                          \
    const cx_##S *tw = e->tw;                                                    \
    int k;                                                                       \
    for (k = 0; k < m; k++) {                                                    \
        cx_##S t[64];                                                            \
        int r;                                                                   \
        t[0] = out[k];                                                           \
        for (r = 1; r < p; r++) {                                                \
            cx_##S a = out[(long)r * m + k];                                     \
            cx_##S w = tw[(long)r * k * tws];                                    \
            t[r].re = a.re * w.re - a.im * w.im;                                 \
            t[r].im = a.re * w.im + a.im * w.re;                                 \
        }                                                                        \
        if (p == 2) {                                                            \
            out[k].re = t[0].re + t[1].re; out[k].im = t[0].im + t[1].im;        \
            out[m + k].re = t[0].re - t[1].re;                                   \
            out[m + k].im = t[0].im - t[1].im;                                   \
        } else if (p == 4) {                                                     \
            const R s = (R)e->sign;                                              \
            R a0r = t[0].re + t[2].re, a0i = t[0].im + t[2].im;                  \
            R a1r = t[0].re - t[2].re, a1i = t[0].im - t[2].im;                  \
            R b0r = t[1].re + t[3].re, b0i = t[1].im + t[3].im;                  \
            R b1r = t[1].re - t[3].re, b1i = t[1].im - t[3].im;                  \
            /* (s i) * b1 = (-s b1i, s b1r) */                                   \
            out[k].re = a0r + b0r; out[k].im = a0i + b0i;                        \
            out[2 * m + k].re = a0r - b0r; out[2 * m + k].im = a0i - b0i;        \
            out[m + k].re = a1r - s * b1i; out[m + k].im = a1i + s * b1r;        \
            out[3 * m + k].re = a1r + s * b1i; out[3 * m + k].im = a1i - s * b1r;\
        } else if (p == 3) {                                                     \
            const R c3 = (R)(0.86602540378443864676372317075293618 * e->sign);   \
            R ar = t[1].re + t[2].re, ai = t[1].im + t[2].im;                    \
            R br = t[1].re - t[2].re, bi = t[1].im - t[2].im;                    \
            R mr = t[0].re - (R)0.5 * ar, mi = t[0].im - (R)0.5 * ai;            \
            out[k].re = t[0].re + ar; out[k].im = t[0].im + ai;                  \
            out[m + k].re = mr - c3 * bi; out[m + k].im = mi + c3 * br;          \
            out[2 * m + k].re = mr + c3 * bi; out[2 * m + k].im = mi - c3 * br;  \
        } else {                                                                 \
            int q;                                                               \
            for (q = 0; q < p; q++) {                                            \
                R sr = 0, si = 0;                                                \
                for (r = 0; r < p; r++) {                                        \
                    long idx = ((long)r * q % p) * (long)m * tws;                \
                    cx_##S w = tw[idx % N];                                      \
                    sr += t[r].re * w.re - t[r].im * w.im;                       \
                    si += t[r].re * w.im + t[r].im * w.re;                       \
                }                                                                \
                out[(long)q * m + k].re = sr;                                    \
                out[(long)q * m + k].im = si;                                    \
            }                                                                    \
        }                                                                        \
    }                                                                            \
}                                                                                \
                                                                                 \
/* out may not alias in; in is read with stride is */                          \
static void eng_run_##S(eng_##S *e, const cx_##S *in, long is, cx_##S *out)     \
{                                                                                \
    const int n = e->n;                                                          \
    if (!e->blue) { rec_##S(e, n, 1, in, is, out, 0); return; }                  \
    const int M = e->M;                                                          \
    cx_##S *a = e->scratch, *A = e->scratch + M;                                 \
    int j;                                                                       \
    for (j = 0; j < n; j++) {                                                    \
        cx_##S x = in[(long)j * is], c = e->chirp[j];                            \
        a[j].re = x.re * c.re - x.im * c.im;                                     \
        a[j].im = x.re * c.im + x.im * c.re;                                     \
    }                                                                            \
    for (; j < M; j++) { a[j].re = 0; a[j].im = 0; }                             \
    rec_##S(e->fwd, M, 1, a, 1, A, 0);                                           \
    for (j = 0; j < M; j++) {                                                    \
        cx_##S u = A[j], v = e->bspec[j];                                        \
        A[j].re = u.re * v.re - u.im * v.im;                                     \
        A[j].im = u.re * v.im + u.im * v.re;                                     \
    }                                                                            \
    rec_##S(e->bwd, M, 1, A, 1, a, 0);                                           \
    const R inv = (R)(1.0 / (double)M);                                          \
    for (j = 0; j < n; j++) {                                                    \
        cx_##S y = a[j], c = e->chirp[j];                                        \
        y.re *= inv; y.im *= inv;                                                \
        out[j].re = y.re * c.re - y.im * c.im;                                   \
        out[j].im = y.re * c.im + y.im * c.re;                                   \
    }                                                                            \
}                                                                                \
                                                                                 \
static eng_##S *eng_new_##S(int n, int sign)                                     \
{                                                                                \
    eng_##S *e = (eng_##S *)calloc(1, sizeof(eng_##S));                          \
    if (!e) return NULL;                                                         \
    e->n = n; e->sign = sign;                                                    \
    int rem = n, ok = 1;                                                         \
    while (rem % 4 == 0 && e->nf < 60) { e->fac[e->nf++] = 4; rem /= 4; }        \
    while (rem % 2 == 0 && e->nf < 60) { e->fac[e->nf++] = 2; rem /= 2; }        \
    { int f; for (f = 3; f <= 31 && rem > 1; f += 2)                             \
        while (rem % f == 0 && e->nf < 60) { e->fac[e->nf++] = f; rem /= f; } }  \
    if (rem > 1) ok = 0;                                                         \
    if (ok) {                                                                    \
        e->tw = (cx_##S *)malloc((size_t)n * sizeof(cx_##S));                    \
        if (!e->tw) { eng_free_##S(e); return NULL; }                            \
        { int j; for (j = 0; j < n; j++) {                                       \
            double ang = sign * 2.0 * SHIM_PI * (double)j / (double)n;           \
            e->tw[j].re = (R)cos(ang); e->tw[j].im = (R)sin(ang);                \
        } }                                                                      \
        return e;                                                                \
    }                                                                            \
    e->blue = 1;                                                                 \
    int M = 1;                                                                   \
    while (M < 2 * n - 1) M <<= 1;                                               \
    e->M = M;                                                                    \
    e->fwd = eng_new_##S(M, -1);                                                 \
    e->bwd = eng_new_##S(M, +1);                                                 \
    e->chirp = (cx_##S *)malloc((size_t)n * sizeof(cx_##S));                     \
    e->bspec = (cx_##S *)malloc((size_t)M * sizeof(cx_##S));                     \
    e->scratch = (cx_##S *)malloc((size_t)2 * M * sizeof(cx_##S));              \
    if (!e->fwd || !e->bwd || !e->chirp || !e->bspec || !e->scratch) {           \
        eng_free_##S(e); return NULL;                                            \
    }                                                                            \
    { int j; for (j = 0; j < n; j++) {                                           \
        long long jj = ((long long)j * j) % (2LL * n);                           \
        double ang = sign * SHIM_PI * (double)jj / (double)n;                    \
        e->chirp[j].re = (R)cos(ang); e->chirp[j].im = (R)sin(ang);              \
    } }                                                                          \
    cx_##S *b = e->scratch;                                                      \
    { int j; for (j = 0; j < M; j++) { b[j].re = 0; b[j].im = 0; } }             \
    { int d; for (d = 0; d < n; d++) {                                           \
        cx_##S c = e->chirp[d]; c.im = -c.im;                                    \
        b[d] = c;                                                                \
        if (d > 0) b[M - d] = c;                                                 \
    } }                                                                          \
    rec_##S(e->fwd, M, 1, b, 1, e->bspec, 0);                                    \
    return e;                                                                    \
}

DEFINE_ENGINE(float, f)
DEFINE_ENGINE(double, d)


/* ------------------------------------------------------------------ */
/* Batch-vectorised engine: 16 independent float transforms per vector */
/* (the batch index is contiguous in the reference's c2r plans,        */
/* src/search.c:180-187: istride = Nprof, idist = 1).                  */
/* ------------------------------------------------------------------ */
typedef float v16 __attribute__((vector_size(64)));
typedef struct { v16 re, im; } cxv;

static void recv(const eng_f *e, int n, int tws, const cxv *in, long is, cxv *out, int depth)
{
    if (n == 1) { out[0] = in[0]; return; }
    const int p = e->fac[depth];
    const int m = n / p;
    int r, k;
    for (r = 0; r < p; r++)
        recv(e, m, tws * p, in + (long)r * is, is * p, out + (long)r * m, depth + 1);
    const int N = e->n;
    const cx_f *tw = e->tw;
    for (k = 0; k < m; k++) {
        cxv t[64];
        t[0] = out[k];
        for (r = 1; r < p; r++) {
            const cxv a = out[(long)r * m + k];
            const cx_f w = tw[(long)r * k * tws];
            t[r].re = a.re * w.re - a.im * w.im;
            t[r].im = a.re * w.im + a.im * w.re;
        }
        if (p == 2) {
            out[k].re = t[0].re + t[1].re; out[k].im = t[0].im + t[1].im;
            out[m + k].re = t[0].re - t[1].re; out[m + k].im = t[0].im - t[1].im;
        } else if (p == 4) {
            const float s = (float)e->sign;
            const v16 a0r = t[0].re + t[2].re, a0i = t[0].im + t[2].im;
            const v16 a1r = t[0].re - t[2].re, a1i = t[0].im - t[2].im;
            const v16 b0r = t[1].re + t[3].re, b0i = t[1].im + t[3].im;
            const v16 b1r = t[1].re - t[3].re, b1i = t[1].im - t[3].im;
            out[k].re = a0r + b0r; out[k].im = a0i + b0i;
            out[2 * m + k].re = a0r - b0r; out[2 * m + k].im = a0i - b0i;
            out[m + k].re = a1r - s * b1i; out[m + k].im = a1i + s * b1r;
            out[3 * m + k].re = a1r + s * b1i; out[3 * m + k].im = a1i - s * b1r;
        } else if (p == 3) {
            const float c3 = (float)(0.86602540378443864676372317075293618 * e->sign);
            const v16 ar = t[1].re + t[2].re, ai = t[1].im + t[2].im;
            const v16 br = t[1].re - t[2].re, bi = t[1].im - t[2].im;
            const v16 mr = t[0].re - 0.5f * ar, mi = t[0].im - 0.5f * ai;
            out[k].re = t[0].re + ar; out[k].im = t[0].im + ai;
            out[m + k].re = mr - c3 * bi; out[m + k].im = mi + c3 * br;
            out[2 * m + k].re = mr + c3 * bi; out[2 * m + k].im = mi - c3 * br;
        } else {
            int q;
            for (q = 0; q < p; q++) {
                v16 sr = t[0].re, si = t[0].im;
                for (r = 1; r < p; r++) {
                    const long idx = ((long)r * q % p) * (long)m * tws;
                    const cx_f w = tw[idx % N];
                    sr += t[r].re * w.re - t[r].im * w.im;
                    si += t[r].re * w.im + t[r].im * w.re;
                }
                out[(long)q * m + k].re = sr;
                out[(long)q * m + k].im = si;
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* Plans                                                               */
/* ------------------------------------------------------------------ */
enum { SHIM_C2R = 1, SHIM_DFT = 2 };

struct cs_shim_plan {
    int kind, is_f64;
    int n, howmany;
    long istride, idist, ostride, odist;
    void *in, *out;
    int sign;
    eng_f *ef;
    eng_d *ed;
    void *tw_half;    /* exp(+2 pi i k / n), k < n/2 (c2r packing) */
    void *zbuf, *ybuf;
};

static struct cs_shim_plan *plan_c2r(int n, int howmany, void *in, long istride,
                                     long idist, void *out, long ostride,
                                     long odist, int is_f64)
{
    if (n < 1 || howmany < 0) return NULL;
    struct cs_shim_plan *p = (struct cs_shim_plan *)calloc(1, sizeof(*p));
    if (!p) return NULL;
    p->kind = SHIM_C2R; p->is_f64 = is_f64;
    p->n = n; p->howmany = howmany;
    p->istride = istride; p->idist = idist;
    p->ostride = ostride; p->odist = odist;
    p->in = in; p->out = out;
    if (n % 2 == 0) {
        int N = n / 2;
        if (is_f64) {
            p->ed = eng_new_d(N, +1);
            cx_d *t = (cx_d *)malloc((size_t)N * sizeof(cx_d));
            if (!p->ed || !t) { free(t); free(p); return NULL; }
            { int k; for (k = 0; k < N; k++) {
                double a = 2.0 * SHIM_PI * (double)k / (double)n;
                t[k].re = cos(a); t[k].im = sin(a);
            } }
            p->tw_half = t;
            p->zbuf = malloc((size_t)2 * N * sizeof(cx_d));
        } else {
            p->ef = eng_new_f(N, +1);
            cx_f *t = (cx_f *)malloc((size_t)N * sizeof(cx_f));
            if (!p->ef || !t) { free(t); free(p); return NULL; }
            { int k; for (k = 0; k < N; k++) {
                double a = 2.0 * SHIM_PI * (double)k / (double)n;
                t[k].re = (float)cos(a); t[k].im = (float)sin(a);
            } }
            p->tw_half = t;
            p->zbuf = malloc((size_t)2 * N * sizeof(cx_f));
        }
        if (!p->zbuf) { free(p->tw_half); free(p); return NULL; }
    }
    return p;
}

fftw_plan fftw_plan_many_dft_c2r(int rank, const int *n, int howmany,
                                 fftw_complex *in, const int *inembed,
                                 int istride, int idist,
                                 double *out, const int *onembed,
                                 int ostride, int odist, unsigned flags)
{
    (void)inembed; (void)onembed; (void)flags;
    if (rank != 1) return NULL;
    return plan_c2r(n[0], howmany, in, istride, idist, out, ostride, odist, 1);
}

fftwf_plan fftwf_plan_many_dft_c2r(int rank, const int *n, int howmany,
                                   fftwf_complex *in, const int *inembed,
                                   int istride, int idist,
                                   float *out, const int *onembed,
                                   int ostride, int odist, unsigned flags)
{
    (void)inembed; (void)onembed; (void)flags;
    if (rank != 1) return NULL;
    return plan_c2r(n[0], howmany, in, istride, idist, out, ostride, odist, 0);
}

fftw_plan fftw_plan_dft_c2r_1d(int n, fftw_complex *in, double *out, unsigned flags)
{
    (void)flags;
    return plan_c2r(n, 1, in, 1, n / 2 + 1, out, 1, n, 1);
}

fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex *in, fftwf_complex *out,
                             int sign, unsigned flags)
{
    (void)flags;
    if (n < 1) return NULL;
    struct cs_shim_plan *p = (struct cs_shim_plan *)calloc(1, sizeof(*p));
    if (!p) return NULL;
    p->kind = SHIM_DFT; p->is_f64 = 0;
    p->n = n; p->howmany = 1;
    p->in = in; p->out = out; p->sign = sign;
    p->ef = eng_new_f(n, sign);
    p->zbuf = malloc((size_t)n * sizeof(cx_f));
    if (!p->ef || !p->zbuf) { eng_free_f(p->ef); free(p->zbuf); free(p); return NULL; }
    return p;
}


/* Float c2r of 16 transforms at a time through the vector engine; returns
 * how many transforms it handled (a multiple of 16, or 0). */
static int c2r_batch16_f(struct cs_shim_plan *p)
{
    const int n = p->n, N = n / 2;
    if (p->idist != 1 || p->howmany < 16 || p->ef->blue || N > 256 || N < 1) return 0;
    const float *in = (const float *)p->in;
    float *out = (float *)p->out;
    const cx_f *tw = (const cx_f *)p->tw_half;
    cxv Z[256], z[256];
    int b0, k, j, l;
    const int nb = p->howmany / 16 * 16;
    for (b0 = 0; b0 < nb; b0 += 16) {
        for (k = 0; k < N; k++) {
            const float *xa = in + 2 * ((long)k * p->istride + b0);
            const float *xb = in + 2 * ((long)(N - k) * p->istride + b0);
            float g[4][16];
            for (l = 0; l < 16; l++) {
                g[0][l] = xa[2 * l];
                g[1][l] = k ? xa[2 * l + 1] : 0.0f;
                g[2][l] = xb[2 * l];
                g[3][l] = k ? -xb[2 * l + 1] : 0.0f;
            }
            v16 ar, ai, br, bi;
            memcpy(&ar, g[0], sizeof(ar));
            memcpy(&ai, g[1], sizeof(ai));
            memcpy(&br, g[2], sizeof(br));
            memcpy(&bi, g[3], sizeof(bi));
            const v16 er = ar + br, ei = ai + bi;
            const v16 dr = ar - br, di = ai - bi;
            const v16 orr = dr * tw[k].re - di * tw[k].im;
            const v16 oi = dr * tw[k].im + di * tw[k].re;
            Z[k].re = er - oi;
            Z[k].im = ei + orr;
        }
        recv(p->ef, N, 1, Z, 1, z, 0);
        for (l = 0; l < 16; l++) {
            float *y = out + (long)(b0 + l) * p->odist;
            for (j = 0; j < N; j++) {
                y[(long)(2 * j) * p->ostride] = z[j].re[l];
                y[(long)(2 * j + 1) * p->ostride] = z[j].im[l];
            }
        }
    }
    return nb;
}
static int c2r_batch16_d(struct cs_shim_plan *p) { (void)p; return 0; }

/* Even-length c2r through one complex FFT of length n/2:
 *   E[k] = X[k] + conj(X[N-k]),  O[k] = (X[k] - conj(X[N-k])) exp(2 pi i k/n)
 *   z = backward DFT_N(E + i O);  y[2j] = Re z[j], y[2j+1] = Im z[j]. */
#define DEFINE_C2R_EXEC(R, S)                                                    \
static void c2r_exec_##S(struct cs_shim_plan *p)                                 \
{                                                                                \
    const int n = p->n;                                                          \
    const R *in = (const R *)p->in;                                              \
    R *out = (R *)p->out;                                                        \
    int b;                                                                       \
    if (n % 2) {                                                                 \
        /* odd length: direct evaluation in double */                            \
        for (b = 0; b < p->howmany; b++) {                                       \
            const R *x = in + 2 * (long)b * p->idist;                            \
            int j;                                                               \
            for (j = 0; j < n; j++) {                                            \
                double acc = (double)x[0];                                       \
                int k;                                                           \
                for (k = 1; k <= n / 2; k++) {                                   \
                    double a = 2.0 * SHIM_PI * (double)((long long)j * k % n) / n; \
                    const R *xk = x + 2 * (long)k * p->istride;                  \
                    acc += 2.0 * ((double)xk[0] * cos(a) - (double)xk[1] * sin(a)); \
                }                                                                \
                out[(long)b * p->odist + (long)j * p->ostride] = (R)acc;         \
            }                                                                    \
        }                                                                        \
        return;                                                                  \
    }                                                                            \
    const int N = n / 2;                                                         \
    cx_##S *Z = (cx_##S *)p->zbuf, *z = Z + N;                                   \
    const cx_##S *tw = (const cx_##S *)p->tw_half;                               \
    b = c2r_batch16_##S(p);                                                      \
    for (; b < p->howmany; b++) {                                                \
        const R *x = in + 2 * (long)b * p->idist;                                \
        int k;                                                                   \
        for (k = 0; k < N; k++) {                                                \
            const R *xa = x + 2 * (long)k * p->istride;                          \
            const R *xb = x + 2 * (long)(N - k) * p->istride;                    \
            R ar = xa[0], ai = (k == 0) ? (R)0 : xa[1];                          \
            R br = xb[0], bi = (k == 0) ? (R)0 : -xb[1];                         \
            R er = ar + br, ei = ai + bi;                                        \
            R dr = ar - br, di = ai - bi;                                        \
            R orr = dr * tw[k].re - di * tw[k].im;                               \
            R oi = dr * tw[k].im + di * tw[k].re;                                \
            Z[k].re = er - oi;                                                   \
            Z[k].im = ei + orr;                                                  \
        }                                                                        \
        eng_run_##S(p->e##S, Z, 1, z);                                           \
        R *y = out + (long)b * p->odist;                                         \
        int j;                                                                   \
        for (j = 0; j < N; j++) {                                                \
            y[(long)(2 * j) * p->ostride] = z[j].re;                             \
            y[(long)(2 * j + 1) * p->ostride] = z[j].im;                         \
        }                                                                        \
    }                                                                            \
}

DEFINE_C2R_EXEC(float, f)
DEFINE_C2R_EXEC(double, d)

static void shim_execute(struct cs_shim_plan *p)
{
    if (!p) return;
    if (p->kind == SHIM_C2R) {
        if (p->is_f64) c2r_exec_d(p); else c2r_exec_f(p);
        return;
    }
    /* complex DFT (possibly in place): run out of place into zbuf, copy */
    cx_f *tmp = (cx_f *)p->zbuf;
    eng_run_f(p->ef, (const cx_f *)p->in, 1, tmp);
    memcpy(p->out, tmp, (size_t)p->n * sizeof(cx_f));
}

#ifdef CS_SHIM_TIMING
/* Time spent in the transforms, for the CPU baseline's phase split: built
 * only into libcsref_timed.so.  Thread CPU time summed over the calls of the
 * calling thread's process; meaningful with one OpenMP thread. */
#include <time.h>
static double g_fft_seconds;
static long long g_fft_calls;

static double thread_seconds(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_THREAD_CPUTIME_ID, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static void shim_execute_timed(struct cs_shim_plan *p)
{
    const double t0 = thread_seconds();
    shim_execute(p);
    const double dt = thread_seconds() - t0;
#pragma omp atomic
    g_fft_seconds += dt;
#pragma omp atomic
    g_fft_calls += 1;
}

/* Seconds spent in fftw(f)_execute so far (and the number of calls);
 * reset != 0 clears both after reading. */
double cs_shim_fft_seconds(long long *calls, int reset)
{
    const double s = g_fft_seconds;
    if (calls) *calls = g_fft_calls;
    if (reset) {
        g_fft_seconds = 0.0;
        g_fft_calls = 0;
    }
    return s;
}

void fftw_execute(const fftw_plan p) { shim_execute_timed(p); }
void fftwf_execute(const fftwf_plan p) { shim_execute_timed(p); }
#else
void fftw_execute(const fftw_plan p) { shim_execute(p); }
void fftwf_execute(const fftwf_plan p) { shim_execute(p); }
#endif

static void shim_destroy(struct cs_shim_plan *p)
{
    if (!p) return;
    eng_free_f(p->ef);
    eng_free_d(p->ed);
    free(p->tw_half);
    free(p->zbuf);
    free(p->ybuf);
    free(p);
}
void fftw_destroy_plan(fftw_plan p) { shim_destroy(p); }
void fftwf_destroy_plan(fftwf_plan p) { shim_destroy(p); }
