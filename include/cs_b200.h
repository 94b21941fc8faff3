/*
 * cs_b200.h -- entry points of libcsgpu.so beyond the reference ABI.
 *
 * The reference GPU backend (src/cuda.cu) has no counterpart for these: they
 * expose the device-resident path (spectrum already in HBM, enqueue without a
 * host round trip), session introspection, and the dedispersion kernel.  The
 * reference-compatible ABI is in coherent_search.h.
 */
#ifndef CS_B200_H
#define CS_B200_H

#include <stddef.h>
#include <stdint.h>
#include "coherent_search.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int ntiles;          /* 128-trial tiles (never straddling a chunk) */
    long long nchunks;   /* reference chunk table entries */
    int nslot;           /* base profile + decimations */
    int npad;            /* tensor-core N (profile columns, padded) */
    int kpad;            /* tensor-core K (2*nharms, padded) */
    int smem_bytes;      /* dynamic shared memory per CTA */
    int grid;            /* persistent CTAs launched */
    long long total;     /* trials */
    unsigned rec_capacity;
    int kernel;          /* 0: generic fused kernel, 1: warp-specialised
                            kernel for the default nharms = 60 ladder */
} CsB200Info;

int cs_b200_session_info(const GpuSession *s, CsB200Info *info);

/* Device address of the session's spectrum buffer (namps float2). */
float *cs_b200_session_device_amps(GpuSession *s);

/* Enqueue one search of a device-resident spectrum (NULL: the session's own
 * buffer) on the session stream without synchronising.  The kernel is
 * bracketed by CUDA events; cs_b200_session_collect reports its time. */
int cs_b200_session_enqueue_device(GpuSession *s, const float *d_amps,
                                   double threshold, void *stream);

/* Wait for the enqueued search, read back and order the candidates exactly
 * as cs_gpu_session_run does.  Returns 0, 1 if the record buffer overflowed
 * (it has been grown; enqueue again), or -1 on error. */
int cs_b200_session_collect(GpuSession *s, double threshold, CandidateList *out,
                            float *kernel_ms);

int cs_b200_session_sync(GpuSession *s);

#ifdef __cplusplus
}
#endif

#endif
