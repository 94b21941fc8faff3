/*
 * coherent_search.h -- public interface of the B200 coherent harmonic-sum
 * search.
 *
 * The types and entry points keep the layout and meaning of the reference
 * interface (CoherentSearch_C include/coherent_search.h), so programs written
 * against it (src/search.c, src/cli.c, src/prep_search.c) link against this
 * implementation unchanged:
 *   - FFTFile / SimpleInf      include/coherent_search.h:48-76
 *   - SearchParams             include/coherent_search.h:118-131
 *   - Candidate / CandidateList include/coherent_search.h:139-151
 *   - DirectPlan / DirectPlanSet include/coherent_search.h:170-195
 *   - GPU backend ABI          include/coherent_search.h:436-460
 * The host implementation (planning, candidates, search driver, CLI) is C in
 * coherentsearch_c_b200/csrc/host; the GPU backend is libcsgpu.so
 * (coherentsearch_c_b200/csrc/cs_gpu.cu), which exports exactly the
 * cs_gpu_* symbols below plus the additions declared in cs_b200.h.
 *
 * Unlike the reference, nothing here depends on FFTW: the CPU transform path
 * does not exist in this implementation (no CPU fallback).
 */
#ifndef COHERENT_SEARCH_H
#define COHERENT_SEARCH_H

#include <stddef.h>
#include <stdint.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Tunables with the reference's values (include/coherent_search.h:34-43). */
#define CS_DIRECT_GROUP_V 32
#define CS_DIRECT_QMAX (1 << 16)
#define CS_LADDER_WMAX 6
#define CS_CPU_DEFAULT_BLOCKSIZE 2048
#define CS_GPU_DEFAULT_BLOCKSIZE 65536

/* ------------------------------------------------------------------ */
/* PRESTO .inf / .fft                                                 */
/* ------------------------------------------------------------------ */
typedef struct {
    char *path;
    char *object;
    int has_epoch;
    double epoch;
    long long N;
    int has_N;
    double dt;
    int has_dt;
    double DM;
    int has_DM;
} SimpleInf;

typedef struct {
    char *path;
    SimpleInf inf;
    long long N;        /* time-series length */
    double T;           /* N * dt */
    double df;          /* 1 / T */
    int dereddened;
    int detrended;
    float DC;
    float Nyquist;
    float *amps;        /* 2*namps interleaved floats (re, im) */
    long long namps;
    void *map;
    size_t mapsize;
    int owns_amps;
} FFTFile;

int  inf_read(const char *path, SimpleInf *inf);
void inf_free(SimpleInf *inf);
int  fftfile_open(FFTFile *ft, const char *path);
void fftfile_close(FFTFile *ft);
/* Wrap a caller-owned spectrum (not copied) as an FFTFile. */
void fftfile_from_memory(FFTFile *ft, const float *amps, long long namps,
                         long long N, double dt);

/* ------------------------------------------------------------------ */
/* Search parameters                                                  */
/* ------------------------------------------------------------------ */
typedef enum { CS_PREC_F32 = 0, CS_PREC_F64 = 1 } cs_precision;
typedef enum { CS_SIGMA_ANALYTIC = 0, CS_SIGMA_MEASURED = 1 } cs_sigma;

typedef struct {
    int nharms;
    int m;
    int numbetween;
    double hidr;
    double threshold;
    double boxcar_fsp;
    double boxcar_maxfrac;
    double boxcar_gatemargin;
    int ndecim;
    int decimations[64];
    cs_precision precision;
    cs_sigma sigma;
} SearchParams;

void params_defaults(SearchParams *p);
int  decimation_set(int nharms, int maxdecim, int *out, int outcap);

/* ------------------------------------------------------------------ */
/* Candidates                                                         */
/* ------------------------------------------------------------------ */
typedef struct {
    double freq;
    double metric;
    double r;
    int nharm;
    double ducy;
} Candidate;

typedef struct {
    Candidate *v;
    size_t n;
    size_t cap;
} CandidateList;

void candlist_init(CandidateList *l);
void candlist_free(CandidateList *l);
void candlist_push(CandidateList *l, Candidate c);
void candlist_append(CandidateList *dst, const CandidateList *src);
void candlist_sort_metric_desc(CandidateList *l);
void candlist_sort_freq(CandidateList *l);
void candlist_sort_r(CandidateList *l);
void candlist_sort_metric_desc_stable(CandidateList *l);
void candlist_sort_freq_stable(CandidateList *l);
void candlist_sort_r_stable(CandidateList *l);
CandidateList remove_duplicates(const CandidateList *in, double dr_tol);
CandidateList remove_harmonics(const CandidateList *in, int numharm, double tol);
int harmonically_related(double r1, double r2, int numharm, double tol);

/* ------------------------------------------------------------------ */
/* Direct interpolation plans                                         */
/* ------------------------------------------------------------------ */
typedef struct {
    int h;
    int m;
    int q;
    int s;
    int base_adv;
    int pnum;
    int rfloor0;
    double dr0;
    int P;
    int32_t *row;          /* q entries, 1-based phase index or 0 */
    float *W;              /* (m, P): W[p*m + i] */
    float *A_re, *A_im;    /* (P,) conj(A(dr)) */
    uint8_t *carry;        /* (P,) */
    int ngrp;              /* CPU group tables: not built here (0 / NULL) */
    int32_t *grow;
    int32_t *goff;
    int32_t *gnj;
    float *gW;
    float *gA_re, *gA_im;
} DirectPlan;

typedef struct {
    DirectPlan *plans;
    int n;
} DirectPlanSet;

int  direct_plans_build(DirectPlanSet *set, const SearchParams *p, double r_lo);
void direct_plans_free(DirectPlanSet *set);
int  trial_grid_rational(double lodr, int *pnum, int *q);
int  harmonic_change_trials(const DirectPlanSet *set, const FFTFile *ft,
                            const SearchParams *p, long long total,
                            long long **out_bnds);
void cs_chunk_state(const DirectPlan *dp, long long t, int *res, long long *qint);
int  cs_harmonic_fits(const DirectPlan *dp, const FFTFile *ft,
                      const SearchParams *p, long long t);
int  chunk_starts(const DirectPlanSet *set, const FFTFile *ft, const SearchParams *p,
                  long long total, int Nprof, long long **out, long long *nout);

/* ------------------------------------------------------------------ */
/* Boxcar matched filter (host tables)                                */
/* ------------------------------------------------------------------ */
int    boxcar_widths(int nbins, double fsp, double maxfrac, int *out, int cap);
int    ladder_boxcar_widths(int nbins, int k, const SearchParams *p, int *out, int cap);
double analytic_sigma(const uint8_t *filled, int k, int Hk);
void   boxcar_shape(double *shape, int nbins, const int *widths, int nw,
                    const uint8_t *filled, int k, int Hk);
int    boxcar_best_width(const double *prof, int nbins, double fsp, double maxfrac,
                         int *out_w, double *out_ducy);
double cs_sinpi(double x);
double cs_cospi(double x);
double cs_eps(double x);

/* ------------------------------------------------------------------ */
/* Search driver / output                                             */
/* ------------------------------------------------------------------ */
/* Field layout of include/coherent_search.h:350-373; the CPU workspace
 * pointer (ws) is kept as an opaque slot and is never set here. */
typedef struct {
    int Nprof;
    int nthreads;
    void *ws;
    SearchParams *params;
    int plan_valid;
    double plan_T;
    long long plan_N, plan_namps;
    double plan_lofreq, plan_hifreq;
    int plan_lobin, plan_Nprof;
    long long plan_total;
    DirectPlanSet dplans;
    long long *cstarts;
    long long nchunks;
    void *gpu_session;   /* GpuSession* */
    int wisdom_done;
    int sigma_warned;
    double sigma_warn_T;
    long long sigma_warn_namps;
} SearchCache;

void search_cache_free(SearchCache *cache);

/* Same argument list as the reference (include/coherent_search.h:427-434).
 * metricstats / normalize / wisdom are CPU-path features the reference
 * refuses on its GPU path (src/cli.c:905-915); they are accepted and must be
 * NULL / 0 here.  gpu_device < 0 is an error: there is no CPU path. */
CandidateList search_file(const FFTFile *ft, const SearchParams *p,
                          double lofreq, double hifreq, int lobin, int blocksize,
                          double threshold, int remove, double dr_tol,
                          int harm_remove, int numharm,
                          void *metricstats, int normalize, int verbose,
                          int wisdom, const char *wisdom_file,
                          SearchCache *cache, double harm_tol,
                          int gpu_device);

int  cs_main(int argc, char **argv);
int  cs_main_list(int argc, char **argv);
int  write_candidates(const CandidateList *cands, const char *outfile, double threshold);
void cs_format_double(char *buf, size_t n, double x);
CandidateList measure_ducy(const FFTFile *ft, const CandidateList *in,
                           const SearchParams *p);
CandidateList read_candidates_file(const char *path, double T);
double *candidate_profile(const FFTFile *ft, double r, int nharm, int m, int *out_n);
void fourier_interp_complex(double r, const float *amps, long long namps, int m,
                            double *out_re, double *out_im);

/* ------------------------------------------------------------------ */
/* GPU backend (libcsgpu.so) -- the reference's ABI, unchanged         */
/* ------------------------------------------------------------------ */
/* Replaces src/cuda.cu:488-528.  1 = device usable (errbuf receives
 * "name (device d, cc X.Y)"), -1 = runtime/device error.  This build always
 * has CUDA, so 0 ("no CUDA support", src/gpu_stub.c) is never returned. */
int cs_gpu_available(int device, char *errbuf, size_t errlen);

typedef struct GpuSession GpuSession;

/* Replaces src/cuda.cu:554-792.  dplans is borrowed for the session's
 * lifetime (as in the reference, the plan cache owns it); cstarts is copied.
 * Returns NULL on failure (message on stderr) -- never exits. */
GpuSession *cs_gpu_session_create(const FFTFile *ft, const SearchParams *p,
                                  const DirectPlanSet *dplans,
                                  const long long *cstarts, long long total,
                                  int Nprof, long long nchunks,
                                  double r_lo, double lodr, int device);
/* Replaces src/cuda.cu:1257-1266 (identity of p is part of the match). */
int cs_gpu_session_matches(const GpuSession *s, const FFTFile *ft,
                           const SearchParams *p, int Nprof, long long total,
                           double r_lo, double lodr, int device);
/* Replaces src/cuda.cu:793-1176: uploads ft->amps, searches every chunk and
 * decimation, returns the above-threshold candidates unsorted in the
 * reference's (chunk, decimation slot, trial) order with ducy = NaN. */
CandidateList cs_gpu_session_run(GpuSession *s, const FFTFile *ft,
                                 double threshold);
/* Replaces src/cuda.cu:1178-1235. */
void cs_gpu_session_free(GpuSession *s);
/* Replaces src/cuda.cu:1238-1255 (create + run + free). */
CandidateList cs_gpu_search_region(const FFTFile *ft, const SearchParams *p,
                                   const DirectPlanSet *dplans,
                                   const long long *cstarts, long long total,
                                   int Nprof, long long nchunks,
                                   double r_lo, double r_hi, double lodr,
                                   double threshold,
                                   int device);

#ifdef __cplusplus
}
#endif

#endif /* COHERENT_SEARCH_H */
