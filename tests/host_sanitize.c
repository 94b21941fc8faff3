/*
 * Test harness (CPU only): drives the host library -- planning, tables,
 * record harvest, boxcar tables, candidate post-processing, the .cohout
 * writer and reader, measure_ducy, the .fft/.inf and SIGPROC readers -- so
 * that tests/test_host_sanitizers.py can run it under AddressSanitizer and
 * UndefinedBehaviorSanitizer.  It checks memory and undefined behaviour, not
 * results (the parity tests check those).
 *
 * usage: host_sanitize <tmpdir> <stem.fft> <file.fil>
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "coherent_search.h"
#include "cs_b200.h"
#include "cs_internal.h"

/* The host sources call the GPU ABI from search_file only, which this
 * harness does not reach; these stand in for libcsgpu.so at link time. */
int cs_gpu_available(int device, char *errbuf, size_t errlen)
{
    (void)device;
    if (errbuf && errlen) snprintf(errbuf, errlen, "no GPU in this harness");
    return -1;
}
GpuSession *cs_gpu_session_create(const FFTFile *ft, const SearchParams *p,
                                  const DirectPlanSet *dplans, const long long *cstarts,
                                  long long total, int Nprof, long long nchunks, double r_lo,
                                  double lodr, int device)
{
    (void)ft; (void)p; (void)dplans; (void)cstarts; (void)total; (void)Nprof;
    (void)nchunks; (void)r_lo; (void)lodr; (void)device;
    return NULL;
}
int cs_gpu_session_matches(const GpuSession *s, const FFTFile *ft, const SearchParams *p,
                           int Nprof, long long total, double r_lo, double lodr, int device)
{
    (void)s; (void)ft; (void)p; (void)Nprof; (void)total; (void)r_lo; (void)lodr; (void)device;
    return 0;
}
CandidateList cs_gpu_session_run(GpuSession *s, const FFTFile *ft, double threshold)
{
    (void)s; (void)ft; (void)threshold;
    CandidateList l;
    candlist_init(&l);
    return l;
}
void cs_gpu_session_free(GpuSession *s) { (void)s; }

static uint64_t rng_state = 0x9E3779B97F4A7C15ULL;
static double urand(void)
{
    rng_state ^= rng_state << 13;
    rng_state ^= rng_state >> 7;
    rng_state ^= rng_state << 17;
    return (double)(rng_state >> 11) * (1.0 / 9007199254740992.0);
}
static double nrand(void)
{
    const double u = urand() + 1e-300, v = urand();
    return sqrt(-2.0 * log(u)) * cos(2.0 * M_PI * v);
}

static int fail(const char *what)
{
    fprintf(stderr, "host_sanitize: %s failed\n", what);
    return 1;
}

/* planning, tables, DFT images, record sort and harvest for one geometry */
static int geometry(const float *amps, long long namps, long long N, double dt, int nh,
                    double hidr, int blocksize)
{
    SearchParams p;
    params_defaults(&p);
    p.nharms = nh;
    p.hidr = hidr;
    p.ndecim = decimation_set(nh, 6, p.decimations, 64);
    FFTFile ft;
    fftfile_from_memory(&ft, amps, namps, N, dt);
    const double T = (double)N * dt;
    const double lodr = hidr / (double)nh, r_lo = 0.1 * T, r_hi = 125.0 * T;
    const long long total = (long long)floor((r_hi - r_lo) / lodr) + 1;
    int pnum = 0, q = 0;
    if (!trial_grid_rational(lodr, &pnum, &q)) return fail("trial_grid_rational");
    DirectPlanSet plans;
    memset(&plans, 0, sizeof(plans));
    if (direct_plans_build(&plans, &p, r_lo) != 0) return fail("direct_plans_build");
    long long *bnds = NULL;
    const int nb = harmonic_change_trials(&plans, &ft, &p, total, &bnds);
    if (nb < 0) return fail("harmonic_change_trials");
    free(bnds);
    long long *cstarts = NULL, nchunks = 0;
    if (chunk_starts(&plans, &ft, &p, total, blocksize, &cstarts, &nchunks) != 0)
        return fail("chunk_starts");
    for (int h = 0; h < nh; h++) {
        int res;
        long long qint;
        cs_chunk_state(&plans.plans[h], total / 2, &res, &qint);
        (void)cs_harmonic_fits(&plans.plans[h], &ft, &p, total - 1);
    }
    CsTables t;
    char err[512];
    if (cs_tables_build(&t, &ft, &p, &plans, cstarts, total, nchunks, r_lo, lodr, err,
                        sizeof(err)) != 0) {
        fprintf(stderr, "%s\n", err);
        return fail("cs_tables_build");
    }
    const size_t halves = (size_t)t.npad * t.kpad;
    uint16_t *bhi = malloc(halves * sizeof(uint16_t)), *blo = malloc(halves * sizeof(uint16_t));
    if (!bhi || !blo) return fail("malloc");
    cs_tables_dft_images(&t, bhi, blo);
    free(bhi);
    free(blo);
    /* random records inside the tables, sorted and harvested */
    const long long nrec = 5000;
    CsRec *recs = malloc(sizeof(CsRec) * nrec);
    if (!recs) return fail("malloc");
    for (long long i = 0; i < nrec; i++) {
        const int c = (int)(urand() * (double)t.nchunks) % (int)t.nchunks;
        const int n = t.chunks[c].n > 0 ? t.chunks[c].n : 1;
        recs[i].chunk = c;
        recs[i].slot = (int)(urand() * t.nslot) % t.nslot;
        recs[i].j = (int)(urand() * n) % n;
        recs[i].metric = (float)(6.0 + 10.0 * urand());
    }
    cs_sort_records(recs, nrec);
    for (long long i = 1; i < nrec; i++) {
        const CsRec *a = &recs[i - 1], *b = &recs[i];
        if (a->chunk > b->chunk || (a->chunk == b->chunk && (a->slot > b->slot ||
                                    (a->slot == b->slot && a->j > b->j))))
            return fail("cs_sort_records order");
    }
    CandidateList out;
    candlist_init(&out);
    cs_harvest(&t, recs, nrec, r_lo, lodr, (double)N, T, 8.0, &out);
    candlist_free(&out);
    free(recs);
    cs_tables_free(&t);
    free(cstarts);
    direct_plans_free(&plans);
    return 0;
}

int main(int argc, char **argv)
{
    if (argc < 4) {
        fprintf(stderr, "usage: host_sanitize <tmpdir> <stem.fft> <file.fil>\n");
        return 2;
    }
    const char *tmpdir = argv[1];
    const long long N = 1 << 16;
    const double dt = 64e-6;
    const long long namps = N / 2;
    float *amps = malloc(sizeof(float) * 2 * namps);
    if (!amps) return fail("malloc");
    for (long long i = 0; i < 2 * namps; i++) amps[i] = (float)nrand();

    const struct { int nh; double hidr; int bs; } geo[] = {
        {60, 0.5, 4096}, {32, 0.5, 2048}, {16, 0.5, 65536}, {7, 0.5, 1000}, {60, 0.25, 4096},
    };
    for (size_t g = 0; g < sizeof(geo) / sizeof(geo[0]); g++)
        if (geometry(amps, namps, N, dt, geo[g].nh, geo[g].hidr, geo[g].bs) != 0) {
            free(amps);
            return 1;
        }

    /* boxcar tables */
    {
        SearchParams p;
        params_defaults(&p);
        int w[256];
        uint8_t filled[64];
        double shape[256];
        for (int nb = 4; nb <= 120; nb += 7) {
            const int nw = boxcar_widths(nb, 1.5, 0.3, w, 256);
            for (int k = 1; k <= 6; k++) (void)ladder_boxcar_widths(nb, k, &p, w, 256);
            for (int h = 0; h < 64; h++) filled[h] = (uint8_t)(urand() < 0.8);
            const double s = analytic_sigma(filled, 1, nb / 2 > 60 ? 60 : nb / 2);
            if (nw > 0) boxcar_shape(shape, nb, w, nw, filled, 1, nb / 2 > 60 ? 60 : nb / 2);
            (void)s;
            double prof[256];
            for (int i = 0; i < nb; i++) prof[i] = nrand();
            int bw;
            double ducy;
            (void)boxcar_best_width(prof, nb, 1.5, 0.3, &bw, &ducy);
        }
        (void)cs_sinpi(0.3); (void)cs_cospi(0.3); (void)cs_eps(1.0);
    }

    /* candidates: collapse, sorts, writer and reader, duty cycles */
    {
        const double T = (double)N * dt;
        CandidateList l;
        candlist_init(&l);
        for (int i = 0; i < 3000; i++) {
            Candidate c;
            memset(&c, 0, sizeof(c));
            c.r = 100.0 + 20000.0 * urand();
            if (i % 3 == 0 && i > 0) c.r = l.v[i - 1].r * (double)(1 + i % 4);   /* harmonics */
            c.freq = c.r / T;
            c.metric = 8.0 + 30.0 * urand();
            c.nharm = 1 << (i % 6);
            c.ducy = NAN;
            candlist_push(&l, c);
        }
        CandidateList a = remove_duplicates(&l, 1.0);
        CandidateList b = remove_harmonics(&a, 16, 1.0);
        candlist_sort_metric_desc(&b);
        candlist_sort_freq(&b);
        candlist_sort_r(&b);
        candlist_sort_metric_desc_stable(&b);
        candlist_sort_freq_stable(&b);
        candlist_sort_r_stable(&b);
        CandidateList c2;
        candlist_init(&c2);
        candlist_append(&c2, &b);
        (void)harmonically_related(100.0, 300.0, 16, 1.0);
        char path[4096];
        snprintf(path, sizeof(path), "%s/sanitize.cohout", tmpdir);
        if (write_candidates(&b, path, 8.0) != 0) return fail("write_candidates");
        CandidateList back = read_candidates_file(path, T);
        char buf[64];
        cs_format_double(buf, sizeof(buf), 123.456789012345);
        /* duty cycles of a few candidates against the spectrum */
        SearchParams p;
        params_defaults(&p);
        FFTFile ft;
        fftfile_from_memory(&ft, amps, namps, N, dt);
        CandidateList few;
        candlist_init(&few);
        for (long long i = 0; i < back.n && i < 20; i++) candlist_push(&few, back.v[i]);
        CandidateList d = measure_ducy(&ft, &few, &p);
        int nprof = 0;
        double *prof = candidate_profile(&ft, 1234.5, 8, 64, &nprof);
        free(prof);
        double re, im;
        fourier_interp_complex(2000.25, amps, namps, 16, &re, &im);
        candlist_free(&l); candlist_free(&a); candlist_free(&b); candlist_free(&c2);
        candlist_free(&back); candlist_free(&few); candlist_free(&d);
    }

    /* file readers */
    {
        FFTFile ft;
        if (fftfile_open(&ft, argv[2]) != 0) return fail("fftfile_open");
        fftfile_close(&ft);
        CsSigproc h;
        if (cs_sigproc_read_header(argv[3], &h) != 0) return fail("cs_sigproc_read_header");
        float x[1000];
        for (int i = 0; i < 1000; i++) x[i] = (float)nrand();
        (void)cs_prep_pad_value(x, 1000);
    }
    free(amps);
    printf("host_sanitize: ok\n");
    return 0;
}
