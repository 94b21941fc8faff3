/* Candidate harvest and collapse on the GPU (cs_collapse.cu), used by the
 * session's collect path in cs_gpu.cu.  Internal to libcsgpu.so. */
#ifndef CS_COLLAPSE_H
#define CS_COLLAPSE_H

#include <cuda_runtime.h>
#include "cs_internal.h"

typedef struct CsCollapse CsCollapse;

CsCollapse *cs_collapse_new(void);
void cs_collapse_free(CsCollapse *w);

/* The n records at device address recs -> the candidate list search_file
 * returns after its post-processing (src/search.c:1467-1478), in out (host
 * memory, caller frees with candlist_free).  Synchronises `st`.  0 or -1. */
int cs_collapse_run(CsCollapse *w, const CsRec *recs, unsigned n, const CsChunk *chunks,
                    long long nchunks, const int *slot_k, const int *slot_Hk, int nslot,
                    int nprof, double r_lo, double lodr, double N, double T, double threshold,
                    int remove, double dr_tol, int harm_remove, int numharm, double harm_tol,
                    cudaStream_t st, CandidateList *out);

#endif
