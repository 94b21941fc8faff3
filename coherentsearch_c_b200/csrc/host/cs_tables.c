/*
 * Session tables for the B200 search kernel, built on the host once per
 * observation geometry.  Compiled with -ffp-contract=off: the FP64
 * expressions below (chunk start frequencies, Nyquist limits, noise scales)
 * must round exactly like the reference's, which is built the same way
 * (src/Makefile:43).
 */
#include "../cs_internal.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.141592653589793238462643383279502884
#endif

#define CS_HIDDEN_API __attribute__((visibility("hidden")))

static int round_up(int x, int a) { return (x + a - 1) / a * a; }

/* IEEE binary16 round-to-nearest-even of a double. */
static uint16_t half_bits(double v)
{
    uint16_t sign = 0;
    if (v < 0) { sign = 0x8000; v = -v; }
    if (!(v == v)) return 0x7E00;
    if (v >= 65520.0) return (uint16_t)(sign | 0x7C00);
    if (v <= 0x1p-25) return sign;               /* ties to even: zero */
    int E;
    frexp(v, &E);                                  /* v = f 2^E, f in [0.5,1) */
    int e = E - 1;                                 /* v in [2^e, 2^(e+1)) */
    if (e < -14) {
        double mant = nearbyint(v * 0x1p24);       /* subnormal: units of 2^-24 */
        return (uint16_t)(sign | (uint16_t)mant); /* 1024 encodes the min normal */
    }
    double mant = nearbyint((ldexp(v, -e) - 1.0) * 1024.0);
    if (mant >= 1024.0) { mant = 0.0; e += 1; }
    if (e > 15) return (uint16_t)(sign | 0x7C00);
    return (uint16_t)(sign | (uint16_t)((e + 15) << 10) | (uint16_t)mant);
}

static double half_value(uint16_t h)
{
    const int e = (h >> 10) & 0x1F, m = h & 0x3FF;
    double v;
    if (e == 0) v = ldexp((double)m, -24);
    else if (e == 31) v = m ? NAN : INFINITY;
    else v = ldexp(1.0 + m / 1024.0, e - 15);
    return (h & 0x8000) ? -v : v;
}

/* Byte offset of element (row, k) in a canonical K-major no-swizzle UMMA
 * operand with `rows` rows: 8x16-byte core matrices, row groups 128 B apart,
 * K groups of 8 elements rows*16 B apart. */
static size_t umma_offset(int rows, int row, int k)
{
    return (size_t)(k >> 3) * (size_t)rows * 16u + (size_t)(row >> 3) * 128u +
           (size_t)(row & 7) * 16u + (size_t)(k & 7) * 2u;
}

CS_HIDDEN_API void cs_tables_free(CsTables *t)
{
    if (!t) return;
    free(t->chunks);
    free(t->tiles);
    free(t->W);
    free(t->A);
    free(t->carry);
    free(t->rowtab);
    free(t->Wt);
    free(t->AC);
    free(t->invsw64);
    memset(t, 0, sizeof(*t));
}

CS_HIDDEN_API int cs_tables_build(CsTables *t, const FFTFile *ft, const SearchParams *p,
                                  const DirectPlanSet *dplans, const long long *cstarts,
                                  long long total, long long nchunks, double r_lo,
                                  double lodr, char *err, size_t errlen)
{
    memset(t, 0, sizeof(*t));
    const int nh = p->nharms;
    if (nh < 1 || nh > CS_MAX_NH) {
        snprintf(err, errlen, "nharms=%d is outside the range 1..%d handled by the "
                 "B200 kernel", nh, CS_MAX_NH);
        return -1;
    }
    if (p->m < 2 || (p->m & 1) || p->m > 64) {
        snprintf(err, errlen, "m=%d must be even and in 2..64", p->m);
        return -1;
    }
    if (!dplans || dplans->n != nh) {
        snprintf(err, errlen, "plan set has %d harmonics, expected %d",
                 dplans ? dplans->n : -1, nh);
        return -1;
    }
    int h;
    for (h = 1; h <= nh; h++) {
        if (dplans->plans[h - 1].P <= 0) {
            snprintf(err, errlen, "hidr=%g is not a simple rational: the tabulated "
                     "interpolation kernel is required", p->hidr);
            return -1;
        }
    }
    t->nh = nh;
    t->m = p->m;
    t->q = dplans->plans[0].q;
    t->pnum = dplans->plans[0].pnum;

    /* decimation slots, in the order of p->decimations (src/cuda.cu:638-662) */
    int ncol = 2 * nh;
    t->nslot = 0;
    {
        CsSlot *s = &t->slot[t->nslot++];
        memset(s, 0, sizeof(*s));
        s->k = 1; s->Hk = nh; s->nk = 2 * nh; s->fold = 0; s->col0 = 0;
    }
    int i;
    for (i = 0; i < p->ndecim; i++) {
        const int k = p->decimations[i];
        if (k <= 1) continue;
        if (t->nslot >= CS_MAX_SLOT) {
            snprintf(err, errlen, "more than %d decimations", CS_MAX_SLOT - 1);
            return -1;
        }
        CsSlot *s = &t->slot[t->nslot++];
        memset(s, 0, sizeof(*s));
        s->k = k;
        s->Hk = nh / k;
        s->nk = 2 * s->Hk;
        s->fold = (nh % k == 0) && (s->nk * k == 2 * nh);
        s->col0 = -1;
        if (!s->fold) { s->col0 = ncol; ncol += s->nk; }
    }
    for (i = 0; i < t->nslot; i++) {
        CsSlot *s = &t->slot[i];
        int wbuf[256];
        const int nw = ladder_boxcar_widths(s->nk, s->k, p, wbuf, 256);
        if (nw < 1 || nw > CS_NWMAX) {
            snprintf(err, errlen, "decimation k=%d has %d boxcar widths (1..%d "
                     "supported)", s->k, nw, CS_NWMAX);
            return -1;
        }
        s->nw = nw;
        s->wmax = wbuf[nw - 1];
        int w;
        for (w = 0; w < nw; w++) {
            s->widths[w] = wbuf[w];
            s->duty[w] = (float)wbuf[w] / (float)s->nk;
        }
    }
    t->ncol = ncol;
    t->npad = round_up(ncol, 16);
    t->kpad = round_up(2 * nh, 16);
    if (t->npad > CS_MAX_NCOL) {
        snprintf(err, errlen, "%d profile columns exceed one MMA (N <= %d)",
                 ncol, CS_MAX_NCOL);
        return -1;
    }

    /* chunk table, filled harmonics and per-region noise scales */
    t->nchunks = nchunks;
    t->chunks = (CsChunk *)calloc((size_t)(nchunks ? nchunks : 1), sizeof(CsChunk));
    if (!t->chunks) { snprintf(err, errlen, "out of host memory"); return -1; }
    t->prec64 = p->precision == CS_PREC_F64;
    if (t->prec64) {
        t->invsw64 = (double *)calloc((size_t)(nchunks ? nchunks : 1) * CS_F64_SCALES,
                                      sizeof(double));
        if (!t->invsw64) { snprintf(err, errlen, "out of host memory"); return -1; }
    }
    const double nyq = (double)ft->N / 2.0;
    uint8_t filled[CS_MAX_NH];
    long long c;
    int ntiles = 0;
    for (c = 0; c < nchunks; c++) {
        CsChunk *ch = &t->chunks[c];
        ch->i0 = cstarts[c];
        ch->n = (int)((c + 1 < nchunks ? cstarts[c + 1] : total) - ch->i0);
        ch->tile0 = ntiles;
        ntiles += (ch->n + CS_TILE_M - 1) / CS_TILE_M;
        ch->filled = 0;
        for (h = 1; h <= nh; h++) {
            const DirectPlan *dp = &dplans->plans[h - 1];
            const int fits = ch->n > 0 &&
                             cs_harmonic_fits(dp, ft, p, ch->i0) &&
                             cs_harmonic_fits(dp, ft, p, ch->i0 + ch->n - 1);
            filled[h - 1] = (uint8_t)fits;
            if (fits) ch->filled |= 1ULL << (h - 1);
        }
        const double rstart = r_lo + (double)ch->i0 * lodr;
        /* the noise scales depend on the filled set and the slot only, and
         * consecutive chunks mostly share it (it changes at the harmonic
         * change points): reuse the previous chunk's, bit for bit */
        const int same = c > 0 && t->chunks[c - 1].filled == ch->filled;
        for (i = 0; i < t->nslot; i++) {
            const CsSlot *s = &t->slot[i];
            /* src/cuda.cu:1079-1086 / src/search.c:622-629 */
            if (i == 0) {
                ch->nvalid[i] = ch->n;
            } else {
                int lo = 0, hi = ch->n;
                while (lo < hi) {
                    const int mid = lo + ((hi - lo) >> 1);
                    if ((double)s->k * (rstart + (double)mid * lodr) < nyq) lo = mid + 1;
                    else hi = mid;
                }
                ch->nvalid[i] = lo;
            }
            if (same) {
                memcpy(ch->invsw[i], t->chunks[c - 1].invsw[i], sizeof(ch->invsw[i]));
                if (t->prec64)
                    memcpy(t->invsw64 + (size_t)c * CS_F64_SCALES + i * (CS_NWMAX + 1),
                           t->invsw64 + (size_t)(c - 1) * CS_F64_SCALES + i * (CS_NWMAX + 1),
                           (CS_NWMAX + 1) * sizeof(double));
                continue;
            }
            /* src/search.c:851-858, 657-664 */
            const double sig = analytic_sigma(filled, s->k, s->Hk);
            const float sigf = (float)sig;
            const float invsigma = sigf > 0.0f ? 1.0f / sigf : 0.0f;
            double shape[CS_NWMAX];
            boxcar_shape(shape, s->nk, s->widths, s->nw, filled, s->k, s->Hk);
            int w;
            for (w = 0; w < s->nw; w++)
                ch->invsw[i][w] = (float)((double)invsigma * shape[w]);
            if (t->prec64) {
                /* the FP64 path keeps sigma in double (src/search.c:649-651) */
                double *d = t->invsw64 + (size_t)c * CS_F64_SCALES + i * (CS_NWMAX + 1);
                const double inv64 = sig > 0.0 ? 1.0 / sig : 0.0;
                d[0] = inv64;
                for (w = 0; w < s->nw; w++) d[1 + w] = inv64 * shape[w];
            }
        }
    }
    t->ntiles = ntiles;
    t->tiles = (int *)malloc((size_t)(ntiles ? ntiles : 1) * 3 * sizeof(int));
    if (!t->tiles) { snprintf(err, errlen, "out of host memory"); return -1; }
    {
        int ti = 0;
        for (c = 0; c < nchunks; c++) {
            const CsChunk *ch = &t->chunks[c];
            int j0;
            for (j0 = 0; j0 < ch->n; j0 += CS_TILE_M) {
                t->tiles[3 * ti + 0] = (int)c;
                t->tiles[3 * ti + 1] = j0;
                t->tiles[3 * ti + 2] = ch->n - j0 < CS_TILE_M ? ch->n - j0 : CS_TILE_M;
                ti++;
            }
        }
    }

    /* packed interpolation tables */
    int nrows = 0;
    for (h = 1; h <= nh; h++) {
        t->harm[h - 1].rfloor0 = dplans->plans[h - 1].rfloor0;
        t->harm[h - 1].P = dplans->plans[h - 1].P;
        t->harm[h - 1].woff = nrows;
        nrows += dplans->plans[h - 1].P;
    }
    t->nrows = nrows;
    t->W = (float *)malloc((size_t)nrows * t->m * sizeof(float));
    t->A = (float *)malloc((size_t)nrows * 2 * sizeof(float));
    t->carry = (uint8_t *)malloc((size_t)nrows);
    t->rowtab = (uint16_t *)malloc((size_t)nh * t->q * sizeof(uint16_t));
    if (!t->W || !t->A || !t->carry || !t->rowtab) {
        snprintf(err, errlen, "out of host memory");
        return -1;
    }
    double gmax = 0.0;
    for (h = 1; h <= nh; h++) {
        const DirectPlan *dp = &dplans->plans[h - 1];
        const int off = t->harm[h - 1].woff;
        int ph, r;
        for (ph = 0; ph < dp->P; ph++) {
            double sw = 0.0;
            int k;
            for (k = 0; k < t->m; k++) {
                const float wv = dp->W[(size_t)ph * t->m + k];
                t->W[(size_t)(off + ph) * t->m + k] = wv;
                sw += fabs((double)wv);
            }
            t->A[2 * (off + ph) + 0] = dp->A_re[ph];
            t->A[2 * (off + ph) + 1] = dp->A_im[ph];
            t->carry[off + ph] = dp->carry[ph];
            const double g = (fabs((double)dp->A_re[ph]) + fabs((double)dp->A_im[ph])) * sw;
            if (g > gmax) gmax = g;
        }
        for (r = 0; r < t->q; r++) {
            const int row = dp->row[r];
            t->rowtab[(size_t)(h - 1) * t->q + r] = (uint16_t)(row > 0 ? row - 1 : 0xFFFF);
        }
    }
    /* pad the bound by 1% for the FP32 rounding of the accumulation */
    t->gbound = (float)(gmax * 1.01 + 1e-30);

    /* carry thresholds, with the reference's expression for the offset */
    for (h = 1; h <= nh; h++) {
        const DirectPlan *dp = &dplans->plans[h - 1];
        int res = 0;
        while (res < t->q && !(dp->dr0 + (double)res / (double)t->q >= 1.0)) res++;
        t->carry_res[h - 1] = res;
        /* cross-check against the tabulated carries */
        int rr;
        for (rr = 0; rr < t->q; rr++) {
            const int row = dp->row[rr];
            if (row > 0 && (int)dp->carry[row - 1] != (rr >= res)) {
                snprintf(err, errlen, "carry of harmonic %d is not monotone in the residue", h);
                return -1;
            }
        }
    }

    /* transposed weights and packed phase factor + carry */
    t->Wt = (float *)malloc((size_t)nrows * t->m * sizeof(float));
    t->AC = (float *)malloc((size_t)nrows * 4 * sizeof(float));
    if (!t->Wt || !t->AC) {
        snprintf(err, errlen, "out of host memory");
        return -1;
    }
    {
        int f4 = 0;
        const int m4 = (t->m + 3) / 4;
        for (h = 1; h <= nh; h++) {
            const int P = t->harm[h - 1].P, off = t->harm[h - 1].woff;
            t->wt_off[h - 1] = f4;
            int ph, i4, e;
            for (i4 = 0; i4 < m4; i4++)
                for (ph = 0; ph < P; ph++)
                    for (e = 0; e < 4; e++) {
                        const int tap = 4 * i4 + e;
                        t->Wt[4 * (size_t)(f4 + i4 * P + ph) + e] =
                            tap < t->m ? t->W[(size_t)(off + ph) * t->m + tap] : 0.0f;
                    }
            for (ph = 0; ph < P; ph++) {
                int32_t cbits = t->carry[off + ph];
                float cf;
                memcpy(&cf, &cbits, sizeof(cf));
                t->AC[4 * (off + ph) + 0] = t->A[2 * (off + ph) + 0];
                t->AC[4 * (off + ph) + 1] = t->A[2 * (off + ph) + 1];
                t->AC[4 * (off + ph) + 2] = cf;
                t->AC[4 * (off + ph) + 3] = 0.0f;
            }
            f4 += m4 * P;
        }
    }
    return 0;
}

/* Coefficient of (Re X_h, Im X_h) in bin n of the unnormalised c2r of
 * length 2H (src/search.c:288-292, FFTW c2r convention: Nyquist imaginary
 * part ignored, interior harmonics counted twice). */
static void c2r_coeff(int j, int H, int n, double *cre, double *cim)
{
    const int nb = 2 * H;
    if (j == H) {
        *cre = (n & 1) ? -1.0 : 1.0;
        *cim = 0.0;
        return;
    }
    const long long ph = ((long long)j * n) % nb;
    const double a = 2.0 * M_PI * (double)ph / (double)nb;
    *cre = 2.0 * cos(a);
    *cim = -2.0 * sin(a);
}

CS_HIDDEN_API void cs_tables_dft_images(const CsTables *t, uint16_t *bhi, uint16_t *blo)
{
    const int rows = t->npad, kpad = t->kpad, nh = t->nh;
    memset(bhi, 0, (size_t)rows * kpad * sizeof(uint16_t));
    memset(blo, 0, (size_t)rows * kpad * sizeof(uint16_t));
    int s, n, h;
    for (s = 0; s < t->nslot; s++) {
        const CsSlot *sl = &t->slot[s];
        if (sl->col0 < 0) continue;           /* folded from the base profile */
        const int k = sl->k, Hk = sl->Hk;
        for (n = 0; n < sl->nk; n++) {
            const int col = sl->col0 + n;
            for (h = 1; h <= nh; h++) {
                if (h % k) continue;
                const int j = h / k;
                if (j > Hk) continue;
                double v[2];
                c2r_coeff(j, Hk, n, &v[0], &v[1]);
                int c;
                for (c = 0; c < 2; c++) {
                    const int kk = 2 * (h - 1) + c;
                    const uint16_t hb = half_bits(v[c]);
                    const uint16_t lb = half_bits(v[c] - half_value(hb));
                    const size_t o = umma_offset(rows, col, kk) / 2;
                    bhi[o] = hb;
                    blo[o] = lb;
                }
            }
        }
    }
}

CS_HIDDEN_API int cs_tables_f64_units(const CsTables *t)
{
    int s, u = 0;
    for (s = 0; s < t->nslot; s++)
        if (t->slot[s].col0 >= 0) u += t->slot[s].Hk + 1;
    return u;
}

CS_HIDDEN_API int cs_tables_dft_f64(const CsTables *t, double *bc, double *bs, int ucols,
                                    int unit0[CS_MAX_SLOT])
{
    const int nh = t->nh;
    memset(bc, 0, (size_t)nh * ucols * sizeof(double));
    memset(bs, 0, (size_t)nh * ucols * sizeof(double));
    int s, n, h, u = 0;
    for (s = 0; s < CS_MAX_SLOT; s++) unit0[s] = -1;
    for (s = 0; s < t->nslot; s++) {
        const CsSlot *sl = &t->slot[s];
        if (sl->col0 < 0) continue;           /* folded from the base profile */
        const int k = sl->k, Hk = sl->Hk;
        unit0[s] = u;
        for (n = 0; n <= Hk; n++, u++) {
            for (h = 1; h <= nh; h++) {
                if (h % k) continue;
                const int j = h / k;
                if (j > Hk) continue;
                double cre, cim;
                c2r_coeff(j, Hk, n, &cre, &cim);
                bc[(size_t)(h - 1) * ucols + u] = cre;
                /* x[n] = C - S: S carries +2 sin, the negation of cim */
                bs[(size_t)(h - 1) * ucols + u] = (n == 0 || n == Hk || j == Hk) ? 0.0 : -cim;
            }
        }
    }
    return u;
}

static int rec_cmp(const void *a, const void *b)
{
    const CsRec *x = (const CsRec *)a, *y = (const CsRec *)b;
    if (x->chunk != y->chunk) return (x->chunk > y->chunk) - (x->chunk < y->chunk);
    if (x->slot != y->slot) return (x->slot > y->slot) - (x->slot < y->slot);
    return (x->j > y->j) - (x->j < y->j);
}

static int bit_length(unsigned v)
{
    int b = 0;
    while (v) { b++; v >>= 1; }
    return b;
}

/* Records into (chunk, slot, j) order.  Each (chunk, slot, j) is written at
 * most once, so the order is total and any correct sort gives the same
 * sequence; this one is an LSD radix sort on the packed key (11-bit digits,
 * usually three passes), linear in n where a comparison sort of the tens of
 * thousands of records a strong source gives would dominate the search. */
CS_HIDDEN_API void cs_sort_records(CsRec *recs, long long n)
{
    if (n < 2) return;
    unsigned mc = 0, ms = 0, mj = 0;
    long long i;
    for (i = 0; i < n; i++) {
        if (recs[i].chunk < 0 || recs[i].slot < 0 || recs[i].j < 0) {
            qsort(recs, (size_t)n, sizeof(CsRec), rec_cmp);
            return;
        }
        if ((unsigned)recs[i].chunk > mc) mc = (unsigned)recs[i].chunk;
        if ((unsigned)recs[i].slot > ms) ms = (unsigned)recs[i].slot;
        if ((unsigned)recs[i].j > mj) mj = (unsigned)recs[i].j;
    }
    const int bj = bit_length(mj), bs = bit_length(ms), bc = bit_length(mc);
    const int bits = bj + bs + bc;
    if (n < 256 || bits > 63) {
        qsort(recs, (size_t)n, sizeof(CsRec), rec_cmp);
        return;
    }
    uint64_t *key = (uint64_t *)malloc((size_t)n * 2 * sizeof(uint64_t));
    CsRec *tmp = (CsRec *)malloc((size_t)n * sizeof(CsRec));
    if (!key || !tmp) {
        free(key); free(tmp);
        qsort(recs, (size_t)n, sizeof(CsRec), rec_cmp);
        return;
    }
    uint64_t *key2 = key + n;
    for (i = 0; i < n; i++)
        key[i] = ((uint64_t)(unsigned)recs[i].chunk << (bj + bs)) |
                 ((uint64_t)(unsigned)recs[i].slot << bj) | (uint64_t)(unsigned)recs[i].j;
    enum { DIG = 11, NB = 1 << DIG };
    long long cnt[NB];
    CsRec *src = recs, *dst = tmp;
    uint64_t *ks = key, *kd = key2;
    int shift;
    for (shift = 0; shift < bits; shift += DIG) {
        memset(cnt, 0, sizeof(cnt));
        for (i = 0; i < n; i++) cnt[(ks[i] >> shift) & (NB - 1)]++;
        long long sum = 0;
        int d;
        for (d = 0; d < NB; d++) { const long long c = cnt[d]; cnt[d] = sum; sum += c; }
        for (i = 0; i < n; i++) {
            const long long o = cnt[(ks[i] >> shift) & (NB - 1)]++;
            dst[o] = src[i];
            kd[o] = ks[i];
        }
        CsRec *tr = src; src = dst; dst = tr;
        uint64_t *tk = ks; ks = kd; kd = tk;
    }
    if (src != recs) memcpy(recs, src, (size_t)n * sizeof(CsRec));
    free(key);
    free(tmp);
}

/* One record -> Candidate (src/cuda.cu:837-881 arithmetic); false when it
 * is not reported (below the threshold, or a decimated trial at or past the
 * Nyquist frequency). */
static int harvest_one(const CsTables *t, int chunk, int slot, int j, double metric,
                       double r_lo, double lodr, double nyq, double T, double threshold,
                       Candidate *cd)
{
    if (!(metric > threshold)) return 0;
    const CsSlot *s = &t->slot[slot];
    const double rstart = r_lo + (double)t->chunks[chunk].i0 * lodr;
    const double rfreq = rstart + (double)j * lodr;
    const double kmul = (double)s->k;
    const double rsel = kmul != 1.0 ? kmul * rfreq : rfreq;
    if (slot != 0 && !(rsel < nyq)) return 0;
    cd->freq = rsel / T;
    cd->metric = metric;
    cd->r = rsel;
    cd->nharm = s->Hk;
    cd->ducy = NAN;
    return 1;
}

CS_HIDDEN_API void cs_harvest(const CsTables *t, const CsRec *recs, long long n,
                              double r_lo, double lodr, double N, double T,
                              double threshold, CandidateList *out)
{
    long long i;
    Candidate cd;
    for (i = 0; i < n; i++)
        if (harvest_one(t, recs[i].chunk, recs[i].slot, recs[i].j, (double)recs[i].metric,
                        r_lo, lodr, N / 2.0, T, threshold, &cd))
            candlist_push(out, cd);
}

static int rec64_cmp(const void *a, const void *b)
{
    const CsRec64 *x = (const CsRec64 *)a, *y = (const CsRec64 *)b;
    if (x->chunk != y->chunk) return (x->chunk > y->chunk) - (x->chunk < y->chunk);
    if (x->slot != y->slot) return (x->slot > y->slot) - (x->slot < y->slot);
    return (x->j > y->j) - (x->j < y->j);
}

/* FP64 searches are rare and their record lists short: a comparison sort
 * (each (chunk, slot, j) appears once, so the order is total). */
CS_HIDDEN_API void cs_sort_records64(CsRec64 *recs, long long n)
{
    if (n > 1) qsort(recs, (size_t)n, sizeof(CsRec64), rec64_cmp);
}

CS_HIDDEN_API void cs_harvest64(const CsTables *t, const CsRec64 *recs, long long n,
                                double r_lo, double lodr, double N, double T,
                                double threshold, CandidateList *out)
{
    long long i;
    Candidate cd;
    for (i = 0; i < n; i++)
        if (harvest_one(t, recs[i].chunk, recs[i].slot, recs[i].j, recs[i].metric,
                        r_lo, lodr, N / 2.0, T, threshold, &cd))
            candlist_push(out, cd);
}
