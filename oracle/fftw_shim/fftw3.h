/*
 * Test infrastructure (oracle).  Not product code.
 *
 * A minimal FFTW 3 API surface, written for this repository, so that the
 * reference CPU search path (which is written against FFTW 3.3.10, a
 * third-party library that is not part of the reference tree and is not
 * installed here) compiles unmodified into the oracle binaries under
 * oracle/_ref/.  Only the entry points the reference calls are declared:
 *   src/search.c:77-104,160-187   fftw[f]_plan_many_dft_c2r, execute, destroy
 *   src/candidate.c:196,256       fftw_plan_dft_c2r_1d
 *   src/datpipe.c:313-318         fftwf_plan_dft_1d (complex, both signs)
 *   src/search.c:1169-1245        wisdom import/export (no-ops here)
 * Names, types and flag values follow FFTW's published interface so the
 * reference sources need no edits; the transforms themselves are restated
 * from their mathematical definitions in fftw_shim.c.
 */
#ifndef CS_ORACLE_FFTW3_SHIM_H
#define CS_ORACLE_FFTW3_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef float fftwf_complex[2];

typedef struct cs_shim_plan *fftw_plan;
typedef struct cs_shim_plan *fftwf_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)

#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_UNALIGNED (1U << 1)
#define FFTW_CONSERVE_MEMORY (1U << 2)
#define FFTW_EXHAUSTIVE (1U << 3)
#define FFTW_PRESERVE_INPUT (1U << 4)
#define FFTW_PATIENT (1U << 5)
#define FFTW_ESTIMATE (1U << 6)

void *fftw_malloc(size_t n);
void fftw_free(void *p);
void *fftwf_malloc(size_t n);
void fftwf_free(void *p);

fftw_plan fftw_plan_many_dft_c2r(int rank, const int *n, int howmany,
                                 fftw_complex *in, const int *inembed,
                                 int istride, int idist,
                                 double *out, const int *onembed,
                                 int ostride, int odist, unsigned flags);
fftwf_plan fftwf_plan_many_dft_c2r(int rank, const int *n, int howmany,
                                   fftwf_complex *in, const int *inembed,
                                   int istride, int idist,
                                   float *out, const int *onembed,
                                   int ostride, int odist, unsigned flags);
fftw_plan fftw_plan_dft_c2r_1d(int n, fftw_complex *in, double *out,
                               unsigned flags);
fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex *in, fftwf_complex *out,
                             int sign, unsigned flags);

void fftw_execute(const fftw_plan p);
void fftwf_execute(const fftwf_plan p);
void fftw_destroy_plan(fftw_plan p);
void fftwf_destroy_plan(fftwf_plan p);

int fftw_import_wisdom_from_filename(const char *filename);
int fftwf_import_wisdom_from_filename(const char *filename);
int fftw_export_wisdom_to_filename(const char *filename);
int fftwf_export_wisdom_to_filename(const char *filename);

#ifdef __cplusplus
}
#endif

#endif
