/*
 * Internal layout shared by the host table builder (host/cs_tables.c, plain
 * C compiled with -ffp-contract=off so its FP64 arithmetic matches the
 * reference's) and the CUDA backend (cs_gpu.cu).  Not a public interface.
 */
#ifndef CS_INTERNAL_H
#define CS_INTERNAL_H

#include <stdint.h>
#include "coherent_search.h"

#ifdef __cplusplus
extern "C" {
#endif

#define CS_TILE_M 128          /* trials per tile = tcgen05 M */
#define CS_MAX_NH 60           /* harmonics supported by the fused kernel */
#define CS_MAX_SLOT 8          /* base + decimations */
#define CS_NWMAX 12            /* boxcar widths per decimation */
#define CS_MAX_NCOL 256        /* DFT output columns (one MMA, N <= 256) */

/* One decimation slot: slot 0 is the full-resolution profile (k = 1). */
typedef struct {
    int k, Hk, nk;             /* factor, harmonics, profile bins (2*Hk) */
    int fold;                  /* k | nharms: folded from the base profile */
    int col0;                  /* first DFT column (non-fold slots and base) */
    int nw, wmax;
    int widths[CS_NWMAX];
    float duty[CS_NWMAX];      /* (float)w / (float)nk, src/boxcar.c:220 */
} CsSlot;

/* One chunk of the reference chunk table (src/interp.c:944-966). */
typedef struct {
    long long i0;              /* first trial */
    int n;                     /* trials */
    int tile0;                 /* first tile of this chunk */
    unsigned long long filled; /* bit h-1: harmonic h interpolated */
    int nvalid[CS_MAX_SLOT];   /* trials below the decimated Nyquist */
    float invsw[CS_MAX_SLOT][CS_NWMAX];  /* (float)(invsigma * shape[w]) */
} CsChunk;

/* Device-side per-harmonic table header. */
typedef struct {
    long long rfloor0;
    int P;                     /* phase-cycle length */
    int woff;                  /* first row in the packed W/A/carry tables */
} CsHarm;

/* Candidate record written by the kernel. */
typedef struct {
    int chunk;
    int slot;
    int j;                     /* trial offset inside the chunk */
    float metric;
} CsRec;

/* Candidate record of the FP64 search (--precision f64). */
typedef struct {
    int chunk;
    int slot;
    int j;
    int pad;
    double metric;
} CsRec64;

/* Per chunk, per slot of the FP64 search: invsigma = 1/sigma in double,
 * then invsigma * shape[w] for each width (src/search.c:649-656). */
#define CS_F64_SCALES (CS_MAX_SLOT * (CS_NWMAX + 1))

/* Everything the host builds once per session geometry. */
typedef struct {
    int nh, m, q, pnum;
    int nslot;
    CsSlot slot[CS_MAX_SLOT];
    int ncol;                  /* DFT columns used */
    int npad;                  /* MMA N (multiple of 16) */
    int kpad;                  /* MMA K (multiple of 16) = 2*nh rounded up */
    long long nchunks;
    CsChunk *chunks;           /* nchunks */
    int ntiles;
    int *tiles;                /* 3 ints per tile: chunk, j0, count */
    /* packed interpolation tables */
    CsHarm harm[CS_MAX_NH];
    int nrows;                 /* sum of P over harmonics */
    float *W;                  /* nrows * m */
    float *A;                  /* nrows * 2 (re, im) */
    uint8_t *carry;            /* nrows */
    uint16_t *rowtab;          /* nh * q: residue -> phase index */
    float gbound;              /* max over rows of (|A_re|+|A_im|) * sum|W| */
    /* layout for the warp-specialised kernel (m % 4 == 0):
     *   Wt: per harmonic, [m/4][P] float4 -- lanes on consecutive phases
     *       read consecutive 16-byte words;
     *   AC: per row float4 {A_re, A_im, carry (int bits), 0} */
    float *Wt;                 /* nrows * m */
    float *AC;                 /* nrows * 4 */
    int wt_off[CS_MAX_NH];     /* first float4 of harmonic h in Wt */
    /* carry into the next bin as a residue threshold: for the trial residue
     * res = (t*h*pnum) mod q the phase offset dr0 + res/q reaches 1 exactly
     * when res >= carry_res[h] (monotone in res; src/interp.c:260-262) */
    int carry_res[CS_MAX_NH];
    /* FP64 search only (p->precision == CS_PREC_F64): CS_F64_SCALES doubles
     * per chunk, [slot][0] = invsigma, [slot][1 + w] = invsw of width w */
    int prec64;
    double *invsw64;
} CsTables;

/* Build / free the tables.  Returns 0 or -1 with a message in err. */
int  cs_tables_build(CsTables *t, const FFTFile *ft, const SearchParams *p,
                     const DirectPlanSet *dplans, const long long *cstarts,
                     long long total, long long nchunks, double r_lo,
                     double lodr, char *err, size_t errlen);
void cs_tables_free(CsTables *t);

/* Fill the B operand images (fp16 hi and lo parts of the c2r matrix) in the
 * canonical no-swizzle K-major UMMA layout: npad rows (output columns) by
 * kpad (interleaved Re/Im of harmonics 1..nh).  Each image holds
 * npad*kpad halves, returned as raw 16-bit patterns. */
void cs_tables_dft_images(const CsTables *t, uint16_t *bhi, uint16_t *blo);

/* The half-spectrum DFT of the FP64 search.  Each profile-producing slot
 * (the base and every decimation that does not fold) owns Hk+1 units, one per
 * output bin n = 0..Hk; for harmonic h (row h-1) and unit u,
 *   bc[(h-1)*ucols + u] = c2r cosine weight of bin n  (2 cos, or cos(pi n) at
 *                         the sub-stack's Nyquist harmonic),
 *   bs[(h-1)*ucols + u] = 2 sin(2 pi j n / 2Hk), zero at n = 0, Hk and for the
 *                         Nyquist harmonic,
 * so that with C = sum_h Re X_h bc and S = sum_h Im X_h bs the profile is
 * x[n] = C - S and x[2Hk - n] = C + S (0 < n < Hk).  unit0[s] is the slot's
 * first unit, or -1 for a folded slot.  Returns the unit count; bc and bs
 * hold nh * ucols doubles each (ucols = units rounded up to 4). */
int  cs_tables_dft_f64(const CsTables *t, double *bc, double *bs, int ucols,
                       int unit0[CS_MAX_SLOT]);
int  cs_tables_f64_units(const CsTables *t);

/* Turn sorted records into the reference's Candidate list
 * (src/cuda.cu:837-881 arithmetic). */
void cs_harvest(const CsTables *t, const CsRec *recs, long long n,
                double r_lo, double lodr, double N, double T,
                double threshold, CandidateList *out);

/* Sort records by (chunk, slot, j). */
void cs_sort_records(CsRec *recs, long long n);

/* The same for FP64 records. */
void cs_sort_records64(CsRec64 *recs, long long n);
void cs_harvest64(const CsTables *t, const CsRec64 *recs, long long n,
                  double r_lo, double lodr, double N, double T,
                  double threshold, CandidateList *out);

#ifdef __cplusplus
}
#endif

#endif
