/* Candidate harvest and collapse on the GPU (cs_collapse.cu), used by the
 * session's collect path in cs_gpu.cu.  Internal to libcsgpu.so. */
#ifndef CS_COLLAPSE_H
#define CS_COLLAPSE_H

#include <cuda_runtime.h>
#include "cs_internal.h"

typedef struct CsCollapse CsCollapse;

CsCollapse *cs_collapse_new(void);
void cs_collapse_free(CsCollapse *w);

/* Enqueue, on `st` and without synchronising, the collapse of the n records
 * at device address recs into the candidate list search_file returns after
 * its post-processing (src/search.c:1467-1478).  0 or -1. */
int cs_collapse_enqueue(CsCollapse *w, const CsRec *recs, unsigned n, const CsChunk *chunks,
                        long long nchunks, const int *slot_k, const int *slot_Hk, int nslot,
                        int nprof, double r_lo, double lodr, double N, double T,
                        double threshold, int remove, double dr_tol, int harm_remove,
                        int numharm, double harm_tol, cudaStream_t st);

/* Wait for the enqueued collapse and copy its list to host memory (out;
 * the caller frees it with candlist_free).  0 or -1. */
int cs_collapse_finish(CsCollapse *w, cudaStream_t st, CandidateList *out);

#endif
