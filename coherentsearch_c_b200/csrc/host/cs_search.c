/*
 * Search driver, candidate post-processing, output and file I/O for the B200
 * build (host side of the drop-in for src/search.c, src/candidate.c and
 * src/fileio.c).  The search itself always runs on the GPU backend: there is
 * no CPU transform path here.  Compiled with -ffp-contract=off so the FP64
 * candidate arithmetic rounds like the reference's.
 */
#include "coherent_search.h"
#include "cs_b200.h"

#include <errno.h>
#include <fcntl.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#ifndef M_PI
#define M_PI 3.141592653589793238462643383279502884
#endif

/* ------------------------------------------------------------------ */
/* Candidate collapsing, src/candidate.c:98-161                       */
/* ------------------------------------------------------------------ */
static CandidateList clone_list(const CandidateList *in)
{
    CandidateList c;
    candlist_init(&c);
    c.v = (Candidate *)malloc((in->n ? in->n : 1) * sizeof(Candidate));
    if (!c.v) return c;
    memcpy(c.v, in->v, in->n * sizeof(Candidate));
    c.n = in->n;
    c.cap = in->n ? in->n : 1;
    return c;
}

/* Runs of candidates within dr_tol bins of their predecessor (in r order)
 * collapse onto their highest-metric member. */
CandidateList remove_duplicates(const CandidateList *in, double dr_tol)
{
    CandidateList out;
    candlist_init(&out);
    if (in->n == 0) return out;
    CandidateList s = clone_list(in);
    candlist_sort_r_stable(&s);
    Candidate keep = s.v[0];
    double last_r = keep.r;
    size_t i;
    for (i = 1; i < s.n; i++) {
        const Candidate c = s.v[i];
        if (c.r - last_r <= dr_tol) {
            if (c.metric > keep.metric) keep = c;
        } else {
            candlist_push(&out, keep);
            keep = c;
        }
        last_r = c.r;
    }
    candlist_push(&out, keep);
    candlist_free(&s);
    candlist_sort_freq_stable(&out);
    return out;
}

int harmonically_related(double r1, double r2, int numharm, double tol)
{
    const double lo = r1 < r2 ? r1 : r2;
    const double hi = r1 < r2 ? r2 : r1;
    if (!(lo > 0.0)) return 0;
    int m;
    for (m = 1; m <= numharm; m++) {
        const int n = (int)nearbyint((double)m * hi / lo);
        if (n < 1 || n > numharm) continue;
        if (fabs((double)m * hi - (double)n * lo) <= tol * (double)m) return 1;
    }
    return 0;
}

/* Greedy in descending metric: a candidate is dropped when it is
 * harmonically related to one already kept. */
CandidateList remove_harmonics(const CandidateList *in, int numharm, double tol)
{
    CandidateList out;
    candlist_init(&out);
    if (in->n == 0) return out;
    CandidateList s = clone_list(in);
    candlist_sort_metric_desc_stable(&s);
    size_t i, j;
    for (i = 0; i < s.n; i++) {
        int related = 0;
        for (j = 0; j < out.n && !related; j++)
            related = harmonically_related(s.v[i].r, out.v[j].r, numharm, tol);
        if (!related) candlist_push(&out, s.v[i]);
    }
    candlist_free(&s);
    candlist_sort_freq_stable(&out);
    return out;
}

/* ------------------------------------------------------------------ */
/* Duty cycle of a candidate, src/candidate.c:208-329, src/boxcar.c:736-785 */
/* ------------------------------------------------------------------ */
void fourier_interp_complex(double r, const float *amps, long long namps, int m,
                            double *out_re, double *out_im)
{
    const int m2 = m / 2;
    double dr = fmod(r, 1.0);
    if (dr < 0) dr += 1.0;
    const long long first = (long long)floor(r + 1e-15) + 1 - m2;
    double sre = 0.0, sim = 0.0;
    int j;
    for (j = 0; j < m; j++) {
        const double off = dr - (double)(-m2 + 1 + j);
        const double sinc = off == 0.0 ? 1.0 : sin(M_PI * off) / (M_PI * off);
        const double c = cos(M_PI * off), s = sin(M_PI * off);
        const double cr = sinc * c, ci = -sinc * s;
        const long long idx = first + j;
        double br = 0.0, bi = 0.0;
        if (idx >= 0 && idx < namps) {
            br = (double)amps[2 * idx];
            bi = (double)amps[2 * idx + 1];
        }
        sre += cr * br - ci * bi;
        sim += cr * bi + ci * br;
    }
    *out_re = sre;
    *out_im = sim;
}

/* Unnormalised c2r of H+1 complex harmonics (index 0 = DC) to n = 2H bins,
 * evaluated directly in FP64. */
static void c2r_direct(const double *X, int H, double *y)
{
    const int n = 2 * H;
    int j, k;
    for (j = 0; j < n; j++) {
        double acc = X[0];
        for (k = 1; k < H; k++) {
            const double a = 2.0 * M_PI * (double)(((long long)j * k) % n) / (double)n;
            acc += 2.0 * (X[2 * k] * cos(a) - X[2 * k + 1] * sin(a));
        }
        acc += (j & 1) ? -X[2 * H] : X[2 * H];
        y[j] = acc;
    }
}

double *candidate_profile(const FFTFile *ft, double r, int nharm, int m, int *out_n)
{
    *out_n = 0;
    if (nharm < 1) return NULL;
    const int m2 = m / 2;
    double *X = (double *)calloc((size_t)(nharm + 1) * 2, sizeof(double));
    if (!X) return NULL;
    int H = 0, h;
    for (h = 1; h <= nharm; h++) {
        const double rh = r * (double)h;
        const long long rint0 = (long long)floor(rh + 1e-15) + 1;
        if (!(rint0 - m2 >= 0 && rint0 + m2 <= ft->namps && rh < (double)(ft->N / 2))) break;
        fourier_interp_complex(rh, ft->amps, ft->namps, m, &X[2 * h], &X[2 * h + 1]);
        H++;
    }
    if (H < 1) {
        free(X);
        *out_n = 2;
        return (double *)calloc(2, sizeof(double));
    }
    const int n = 2 * H;
    double *out = (double *)malloc((size_t)n * sizeof(double));
    if (!out) { free(X); return NULL; }
    c2r_direct(X, H, out);
    const double inv = 1.0 / (double)n;
    int i;
    for (i = 0; i < n; i++) out[i] *= inv;
    free(X);
    *out_n = n;
    return out;
}

int boxcar_best_width(const double *prof, int nbins, double fsp, double maxfrac,
                      int *out_w, double *out_ducy)
{
    if (nbins < 1) return -1;
    int widths[256];
    const int nw = boxcar_widths(nbins, fsp, maxfrac, widths, 256);
    if (nw <= 0) { *out_w = 1; *out_ducy = 1.0 / nbins; return 0; }
    const int wmax = widths[nw - 1];
    double *ps = (double *)malloc((size_t)(nbins + wmax + 1) * sizeof(double));
    double *shape = (double *)malloc((size_t)nw * sizeof(double));
    const int Hk = nbins / 2;
    uint8_t *filled = (uint8_t *)malloc((size_t)(Hk > 0 ? Hk : 1));
    if (!ps || !shape || !filled) { free(ps); free(shape); free(filled); return -1; }
    double sum = 0.0;
    int i;
    for (i = 0; i < nbins; i++) sum += prof[i];
    const double mean = sum / (double)nbins;
    ps[0] = 0.0;
    for (i = 1; i <= nbins + wmax; i++) {
        const int idx = i > nbins ? i - nbins : i;
        ps[i] = ps[i - 1] + (prof[idx - 1] - mean);
    }
    const double stot = ps[nbins] - ps[0];
    for (i = 0; i < Hk; i++) filled[i] = 1;
    if (Hk >= 1) boxcar_shape(shape, nbins, widths, nw, filled, 1, Hk);
    else for (i = 0; i < nw; i++) shape[i] = 0.0;
    double best = -INFINITY;
    int bestw = widths[0];
    for (i = 0; i < nw; i++) {
        const int w = widths[i];
        const double duty = (double)w / (double)nbins;
        double mx = ps[w] - ps[0];
        int q;
        for (q = 2; q <= nbins; q++) {
            const double d = ps[q + w - 1] - ps[q - 1];
            if (d > mx) mx = d;
        }
        const double cand = (mx - duty * stot) * shape[i];
        if (cand > best) { best = cand; bestw = w; }
    }
    *out_w = bestw;
    *out_ducy = (double)bestw / (double)nbins;
    free(ps); free(shape); free(filled);
    return 0;
}

CandidateList measure_ducy(const FFTFile *ft, const CandidateList *in, const SearchParams *p)
{
    CandidateList out;
    candlist_init(&out);
    size_t i;
    for (i = 0; i < in->n; i++) {
        Candidate c = in->v[i];
        c.ducy = NAN;
        if (c.nharm >= 1 && c.r > 0.0) {
            int n = 0;
            double *prof = candidate_profile(ft, c.r, c.nharm, 64, &n);
            if (prof && n >= 2) {
                int w = 1;
                double ducy = NAN;
                if (boxcar_best_width(prof, n, p->boxcar_fsp, p->boxcar_maxfrac, &w, &ducy) == 0)
                    c.ducy = ducy;
            }
            free(prof);
        }
        candlist_push(&out, c);
    }
    return out;
}

/* ------------------------------------------------------------------ */
/* .cohout output, src/candidate.c:336-379                            */
/* ------------------------------------------------------------------ */
void cs_format_double(char *buf, size_t n, double x)
{
    if (isnan(x)) { snprintf(buf, n, "NaN"); return; }
    if (isinf(x)) { snprintf(buf, n, x > 0 ? "Inf" : "-Inf"); return; }
    int prec;
    for (prec = 1; prec <= 17; prec++) {
        char *end = NULL;
        snprintf(buf, n, "%.*g", prec, x);
        if (strtod(buf, &end) == x && end && *end == '\0') break;
    }
    if (!strpbrk(buf, ".eE") && !strstr(buf, "inf") && !strstr(buf, "nan")) {
        const size_t l = strlen(buf);
        if (l + 3 < n) { buf[l] = '.'; buf[l + 1] = '0'; buf[l + 2] = '\0'; }
    }
}

int write_candidates(const CandidateList *cands, const char *outfile, double threshold)
{
    (void)threshold;
    const int to_stdout = (outfile == NULL || *outfile == '\0');
    FILE *f = to_stdout ? stdout : fopen(outfile, "w");
    if (!f) {
        fprintf(stderr, "Error: cannot write candidates to '%s'\n", outfile);
        return -1;
    }
    fprintf(f, "#Num    'S/N'      Frequency (Hz)        Period (ms)    #Harm  Ducy(%%)\n");
    size_t i;
    for (i = 0; i < cands->n; i++) {
        const Candidate *c = &cands->v[i];
        char dstr[32];
        if (isnan(c->ducy)) snprintf(dstr, sizeof(dstr), "-");
        else snprintf(dstr, sizeof(dstr), "%.2f", 100.0 * c->ducy);
        fprintf(f, "%-4zu  %8.2f  %18.12f  %18.12f   %3d   %6s\n", i + 1, c->metric,
                c->freq, 1000.0 / c->freq, c->nharm, dstr);
    }
    if (to_stdout) fflush(stdout);
    else fclose(f);
    return 0;
}

CandidateList read_candidates_file(const char *path, double T)
{
    CandidateList out;
    candlist_init(&out);
    FILE *f = fopen(path, "r");
    if (!f) {
        fprintf(stderr, "Error: cannot open candidate file '%s'\n", path);
        return out;
    }
    char line[4096];
    while (fgets(line, sizeof(line), f)) {
        const char *q = line;
        while (*q == ' ' || *q == '\t') q++;
        if (*q == '#' || *q == '\n' || *q == '\r' || *q == '\0') continue;
        int rank = 0, nharm = 0;
        double snr = 0, freq = 0, period = 0;
        if (sscanf(q, "%d %lf %lf %lf %d", &rank, &snr, &freq, &period, &nharm) >= 5 &&
            freq > 0.0) {
            Candidate c;
            c.freq = freq;
            c.metric = snr;
            c.r = freq * T;
            c.nharm = nharm;
            c.ducy = NAN;
            candlist_push(&out, c);
        }
    }
    fclose(f);
    return out;
}

/* ------------------------------------------------------------------ */
/* .inf / .fft input, src/fileio.c:38-164                             */
/* ------------------------------------------------------------------ */
static char *dupstr(const char *s)
{
    if (!s) return NULL;
    const size_t n = strlen(s) + 1;
    char *d = (char *)malloc(n);
    if (d) memcpy(d, s, n);
    return d;
}

static char *strip(char *s)
{
    while (*s == ' ' || *s == '\t' || *s == '\r' || *s == '\n') s++;
    char *e = s + strlen(s);
    while (e > s && (e[-1] == ' ' || e[-1] == '\t' || e[-1] == '\r' || e[-1] == '\n')) *--e = '\0';
    return s;
}

static char *value_after_eq(char *line)
{
    char *eq = strrchr(line, '=');
    return strip(eq ? eq + 1 : line);
}

int inf_read(const char *path, SimpleInf *inf)
{
    memset(inf, 0, sizeof(*inf));
    inf->path = dupstr(path);
    FILE *f = fopen(path, "r");
    if (!f) return -1;
    char *line = NULL;
    size_t cap = 0;
    while (getline(&line, &cap, f) >= 0) {
        if (strncmp(line, " Object being observed", 22) == 0) {
            free(inf->object);
            inf->object = dupstr(value_after_eq(line));
        } else if (strncmp(line, " Epoch", 6) == 0) {
            inf->epoch = strtod(value_after_eq(line), NULL);
            inf->has_epoch = 1;
        } else if (strncmp(line, " Number of bins", 15) == 0) {
            inf->N = strtoll(value_after_eq(line), NULL, 10);
            inf->has_N = 1;
        } else if (strncmp(line, " Width of each time series bin", 30) == 0) {
            inf->dt = strtod(value_after_eq(line), NULL);
            inf->has_dt = 1;
        } else if (strncmp(line, " Dispersion measure", 19) == 0) {
            inf->DM = strtod(value_after_eq(line), NULL);
            inf->has_DM = 1;
        }
    }
    free(line);
    fclose(f);
    return 0;
}

void inf_free(SimpleInf *inf)
{
    if (!inf) return;
    free(inf->path);
    free(inf->object);
    memset(inf, 0, sizeof(*inf));
}

static char *sibling_inf(const char *path)
{
    const size_t n = strlen(path);
    const size_t keep = n > 4 ? n - 4 : 0;
    char *s = (char *)malloc(keep + 5);
    if (!s) return NULL;
    memcpy(s, path, keep);
    memcpy(s + keep, ".inf", 5);
    return s;
}

int fftfile_open(FFTFile *ft, const char *path)
{
    memset(ft, 0, sizeof(*ft));
    ft->path = dupstr(path);
    char *infpath = sibling_inf(path);
    if (!infpath) return -1;
    if (inf_read(infpath, &ft->inf) != 0) {
        fprintf(stderr, "Error: The .inf file '%s' was not found.\n", infpath);
        free(infpath);
        return -1;
    }
    free(infpath);
    if (!ft->inf.has_N) {
        fprintf(stderr, "Error: Missing 'Number of bins' in %s\n", ft->inf.path);
        return -1;
    }
    if (!ft->inf.has_dt) {
        fprintf(stderr, "Error: Missing 'Width of each time series bin' in %s\n", ft->inf.path);
        return -1;
    }
    const int fd = open(path, O_RDONLY);
    if (fd < 0) {
        fprintf(stderr, "Error: cannot open '%s': %s\n", path, strerror(errno));
        return -1;
    }
    struct stat st;
    if (fstat(fd, &st) != 0) {
        fprintf(stderr, "Error: cannot stat '%s': %s\n", path, strerror(errno));
        close(fd);
        return -1;
    }
    ft->mapsize = (size_t)st.st_size;
    if (ft->mapsize > 0) {
        void *m = mmap(NULL, ft->mapsize, PROT_READ | PROT_WRITE, MAP_PRIVATE, fd, 0);
        if (m == MAP_FAILED) {
            fprintf(stderr, "Error: cannot mmap '%s': %s\n", path, strerror(errno));
            close(fd);
            return -1;
        }
        ft->map = m;
        ft->amps = (float *)m;
        ft->namps = (long long)(ft->mapsize / (2 * sizeof(float)));
    }
    close(fd);
    ft->N = ft->inf.N;
    ft->T = (double)ft->N * ft->inf.dt;
    ft->df = 1.0 / ft->T;
    ft->dereddened = strstr(path, "_red.fft") != NULL;
    ft->detrended = ft->dereddened;
    if (ft->namps > 0) {
        ft->DC = ft->amps[0];
        ft->Nyquist = ft->amps[1];
    }
    return 0;
}

void fftfile_from_memory(FFTFile *ft, const float *amps, long long namps,
                         long long N, double dt)
{
    memset(ft, 0, sizeof(*ft));
    ft->amps = (float *)amps;
    ft->namps = namps;
    ft->N = N;
    ft->inf.N = N;
    ft->inf.has_N = 1;
    ft->inf.dt = dt;
    ft->inf.has_dt = 1;
    ft->T = (double)N * dt;
    ft->df = 1.0 / ft->T;
    if (namps > 0) {
        ft->DC = amps[0];
        ft->Nyquist = amps[1];
    }
}

void fftfile_close(FFTFile *ft)
{
    if (!ft) return;
    if (ft->map && ft->mapsize) munmap(ft->map, ft->mapsize);
    else if (ft->owns_amps) free(ft->amps);
    inf_free(&ft->inf);
    free(ft->path);
    memset(ft, 0, sizeof(*ft));
}

/* ------------------------------------------------------------------ */
/* Search driver, src/search.c:1247-1506                              */
/* ------------------------------------------------------------------ */
void search_cache_free(SearchCache *cache)
{
    if (!cache) return;
    if (cache->gpu_session) {
        cs_gpu_session_free((GpuSession *)cache->gpu_session);
        cache->gpu_session = NULL;
    }
    if (cache->plan_valid) {
        direct_plans_free(&cache->dplans);
        free(cache->cstarts);
        cache->cstarts = NULL;
        cache->plan_valid = 0;
    }
    cache->params = NULL;
}

CandidateList search_file(const FFTFile *ft, const SearchParams *p,
                          double lofreq, double hifreq, int lobin, int blocksize,
                          double threshold, int remove, double dr_tol,
                          int harm_remove, int numharm,
                          void *metricstats, int normalize, int verbose,
                          int wisdom, const char *wisdom_file,
                          SearchCache *cache, double harm_tol,
                          int gpu_device)
{
    (void)wisdom; (void)wisdom_file;
    CandidateList empty;
    candlist_init(&empty);
    if (gpu_device < 0) {
        fprintf(stderr, "Error: this build searches on a B200 GPU only (gpu_device >= 0)\n");
        return empty;
    }
    if (metricstats || normalize) {
        fprintf(stderr, "Error: --metricstats / --normalize are CPU-path features and are "
                        "not available on the GPU path\n");
        return empty;
    }
    const double lodr = p->hidr / (double)p->nharms;
    double r_lo = lofreq * ft->T;
    if (lobin != 100) r_lo = (double)lobin;
    const double r_hi = hifreq * ft->T;
    long long total = (long long)floor((r_hi - r_lo) / lodr) + 1;
    if (total < 0) total = 0;
    if (total == 0) return empty;
    int Nprof = blocksize == 0 ? CS_CPU_DEFAULT_BLOCKSIZE : blocksize;
    if (Nprof < 1) Nprof = 1;

    DirectPlanSet local;
    memset(&local, 0, sizeof(local));
    DirectPlanSet *plans = NULL;
    long long *cstarts = NULL, nchunks = 0;
    int own_plans = 0;
    const int hit = cache && cache->plan_valid && cache->params == p &&
                    cache->plan_T == ft->T && cache->plan_N == ft->N &&
                    cache->plan_namps == ft->namps && cache->plan_lofreq == lofreq &&
                    cache->plan_hifreq == hifreq && cache->plan_lobin == lobin &&
                    cache->plan_Nprof == Nprof && cache->plan_total == total;
    if (hit) {
        plans = &cache->dplans;
        cstarts = cache->cstarts;
        nchunks = cache->nchunks;
    } else {
        DirectPlanSet *target = &local;
        if (cache) {
            if (cache->plan_valid) {
                /* the session borrows the old plans: drop it first */
                if (cache->gpu_session) {
                    cs_gpu_session_free((GpuSession *)cache->gpu_session);
                    cache->gpu_session = NULL;
                }
                direct_plans_free(&cache->dplans);
                free(cache->cstarts);
                cache->cstarts = NULL;
                cache->plan_valid = 0;
            }
            target = &cache->dplans;
        } else {
            own_plans = 1;
        }
        if (direct_plans_build(target, p, r_lo) != 0) return empty;
        if (chunk_starts(target, ft, p, total, Nprof, &cstarts, &nchunks) != 0) {
            direct_plans_free(target);
            return empty;
        }
        plans = target;
        if (cache) {
            cache->cstarts = cstarts;
            cache->nchunks = nchunks;
            cache->params = (SearchParams *)p;
            cache->plan_T = ft->T;
            cache->plan_N = ft->N;
            cache->plan_namps = ft->namps;
            cache->plan_lofreq = lofreq;
            cache->plan_hifreq = hifreq;
            cache->plan_lobin = lobin;
            cache->plan_Nprof = Nprof;
            cache->plan_total = total;
            cache->plan_valid = 1;
        }
    }
    if (verbose) {
        int pmin = 0, pmax = 0, i;
        for (i = 0; i < plans->n; i++) {
            const int P = plans->plans[i].P;
            if (pmin == 0 || P < pmin) pmin = P;
            if (P > pmax) pmax = P;
        }
        fprintf(stderr, "Search: %lld trials in %lld chunks of %d over r = %.1f ... %.1f bins "
                        "(%.4f ... %.4f Hz), GPU\n", total, nchunks, Nprof, r_lo, r_hi,
                r_lo / ft->T, r_hi / ft->T);
        fprintf(stderr, "  phase-cycle lengths P: min %d, max %d (of q = %d)\n", pmin, pmax,
                plans->plans[0].q);
    }

    CandidateList cands;
    candlist_init(&cands);
    GpuSession *gs = cache ? (GpuSession *)cache->gpu_session : NULL;
    int own_session = 0;
    if (!gs || !cs_gpu_session_matches(gs, ft, p, Nprof, total, r_lo, lodr, gpu_device)) {
        if (gs) cs_gpu_session_free(gs);
        if (cache) cache->gpu_session = NULL;
        gs = cs_gpu_session_create(ft, p, plans, cstarts, total, Nprof, nchunks, r_lo, lodr,
                                   gpu_device);
        if (!gs) {
            fprintf(stderr, "Error: failed to create the CUDA session\n");
            if (own_plans) { free(cstarts); direct_plans_free(plans); }
            return empty;
        }
        if (cache) cache->gpu_session = gs;
        else own_session = 1;
    }
    cands = cs_gpu_session_run(gs, ft, threshold);
    if (own_session) cs_gpu_session_free(gs);

    if (remove) {
        CandidateList kept = remove_duplicates(&cands, dr_tol);
        candlist_free(&cands);
        cands = kept;
    } else {
        candlist_sort_freq_stable(&cands);
    }
    if (harm_remove) {
        CandidateList kept = remove_harmonics(&cands, numharm, harm_tol);
        candlist_free(&cands);
        cands = kept;
    }
    if (own_plans) {
        free(cstarts);
        direct_plans_free(plans);
    }
    return cands;
}

/* ------------------------------------------------------------------ */
/* prepsubband padding value                                          */
/* ------------------------------------------------------------------ */
/* The running mean of PRESTO's update_stats
 * (third_party/presto/include/misc_utils.h:114-127) over n samples: each
 * sample as a float, the mean in double, one step at a time.  prepsubband
 * pads every DM series with it, taken over DM 0's samples
 * (src/prep_dedisp.c:505-511, 774-790). */
double cs_prep_pad_value(const float *x, long long n)
{
    double avg = 0.0;
    long long i;
    for (i = 0; i < n; i++) {
        const float xbk = x[i];
        const double dev = xbk - avg;
        avg += dev / ((double)(int)i + 1.0);
    }
    return avg;
}

/* ------------------------------------------------------------------ */
/* SIGPROC filterbank header, third_party/presto/src/sigproc_fb.c      */
/* ------------------------------------------------------------------ */
/* one length-prefixed string (sigproc_fb.c get_string); -1 at end of file or
 * on a length outside 1..79 */
static int sp_string(FILE *f, char *out)
{
    int n;
    if (fread(&n, sizeof(int), 1, f) != 1 || n < 1 || n > 79) return -1;
    if (fread(out, 1, (size_t)n, f) != (size_t)n) return -1;
    out[n] = '\0';
    return 0;
}

/* The keywords read_filterbank_header (sigproc_fb.c:240-345) accepts, with
 * the derived band edges of its spectra_info setup (:435-441).  Only what the
 * device front end takes is accepted: 8-bit unsigned samples, one IF,
 * channels stored highest frequency first (foff < 0).  The data offset is the
 * position after HEADER_END.  Returns 0, or -1 with a message on stderr. */
int cs_sigproc_read_header(const char *path, CsSigproc *h)
{
    char key[80];
    memset(h, 0, sizeof(*h));
    h->nifs = 1;
    h->ibeam = 1;
    FILE *f = fopen(path, "rb");
    if (!f) {
        fprintf(stderr, "Error: cannot open '%s': %s\n", path, strerror(errno));
        return -1;
    }
    int ok = sp_string(f, key) == 0 && strcmp(key, "HEADER_START") == 0;
    if (!ok) fprintf(stderr, "Error: %s: not a SIGPROC filterbank header\n", path);
    int want_name = 0, want_raw = 0, done = 0;
    while (ok && !done) {
        if (sp_string(f, key) != 0) {
            fprintf(stderr, "Error: %s: malformed SIGPROC header\n", path);
            ok = 0;
            break;
        }
        int iv = 0;
        double dv = 0.0;
#define RD(dst) (fread(&(dst), sizeof(dst), 1, f) == 1)
        if (!strcmp(key, "HEADER_END")) done = 1;
        else if (!strcmp(key, "source_name")) want_name = 1;
        else if (!strcmp(key, "rawdatafile")) want_raw = 1;
        else if (!strcmp(key, "tstart")) ok = RD(h->tstart);
        else if (!strcmp(key, "tsamp")) ok = RD(h->tsamp);
        else if (!strcmp(key, "fch1")) ok = RD(h->fch1);
        else if (!strcmp(key, "foff")) ok = RD(h->foff);
        else if (!strcmp(key, "src_raj")) ok = RD(h->src_raj);
        else if (!strcmp(key, "src_dej")) ok = RD(h->src_dej);
        else if (!strcmp(key, "az_start") || !strcmp(key, "za_start")) ok = RD(dv);
        else if (!strcmp(key, "nchans")) ok = RD(h->nchans);
        else if (!strcmp(key, "nbits")) ok = RD(h->nbits);
        else if (!strcmp(key, "nifs")) ok = RD(h->nifs);
        else if (!strcmp(key, "ibeam")) ok = RD(h->ibeam);
        else if (!strcmp(key, "telescope_id")) ok = RD(h->telescope_id);
        else if (!strcmp(key, "machine_id")) ok = RD(h->machine_id);
        else if (!strcmp(key, "data_type") || !strcmp(key, "barycentric") ||
                 !strcmp(key, "pulsarcentric") || !strcmp(key, "nsamples") ||
                 !strcmp(key, "nbeams")) ok = RD(iv);
        else if (!strcmp(key, "signed")) {
            char c;
            ok = fread(&c, 1, 1, f) == 1;
            h->signedints = c;
        }
        else if (want_name) { snprintf(h->source_name, sizeof(h->source_name), "%s", key); want_name = 0; }
        else if (want_raw) { snprintf(h->rawdatafile, sizeof(h->rawdatafile), "%s", key); want_raw = 0; }
        else {
            fprintf(stderr, "Error: %s: unknown SIGPROC header keyword '%s'\n", path, key);
            ok = 0;
        }
#undef RD
    }
    if (!ok || !done) {
        fclose(f);
        return -1;
    }
    h->header_bytes = (long long)ftell(f);
    struct stat stt;
    const int sr = fstat(fileno(f), &stt);
    fclose(f);
    if (sr != 0) return -1;
    if (h->nbits != 8 || h->nifs != 1 || h->nchans < 1 || !(h->foff < 0.0) ||
        !(h->tsamp > 0.0) || h->signedints) {
        fprintf(stderr, "Error: %s: the device front end takes 8-bit unsigned, one-IF "
                        "filterbanks with descending channels (nbits %d, nifs %d, nchans %d, "
                        "foff %g)\n", path, h->nbits, h->nifs, h->nchans, h->foff);
        return -1;
    }
    h->nspectra = ((long long)stt.st_size - h->header_bytes) / h->nchans;
    h->chanwid = fabs(h->foff);
    h->lofreq = h->fch1 - (double)(h->nchans - 1) * h->chanwid;
    return 0;
}
