/*
 * Candidate harvest and collapse on the GPU: the post-processing of the
 * reference's search_file (src/search.c:1467-1478) applied to a session's
 * raw candidate records without sending them to the host.
 *
 *   harvest          record (chunk, slot, j, metric) -> (r, freq, nharm)
 *                    exactly as the host harvest (src/cuda.cu:837-881):
 *                    metric > threshold, r = k * (r_lo + i0*lodr + j*lodr),
 *                    decimated slots only below the Nyquist bin;
 *   base order       records sorted by (chunk, slot, j): the order
 *                    cs_gpu_session_run returns;
 *   remove           remove_duplicates (src/candidate.c:98-128): a stable
 *                    sort by r, runs whose consecutive r differ by at most
 *                    dr_tol, the first member of largest metric of each run
 *                    (a segmented argmax by 64-bit atomicMax);
 *                    the result is in r order, which is also its frequency
 *                    order (freq = r / T, and two members of one list never
 *                    tie in freq without falling into one run);
 *   no remove        a stable sort by frequency (src/search.c:1472);
 *   harm_remove      remove_harmonics (src/candidate.c:130-161): a stable
 *                    sort by descending metric, then greedily each candidate
 *                    not harmonically related to one already kept is kept;
 *                    the kept ones come out in the input (frequency) order,
 *                    which is what the reference's final stable frequency
 *                    sort gives (kept candidates never tie in frequency:
 *                    equal frequencies are related with m = n = 1).
 *
 * Ordering without a sort on r: within one decimation slot, r (and freq)
 * rises strictly with the trial index, so a CUB radix sort on (slot, chunk,
 * j) lines every slot up in r order, and a merge places each candidate at
 * its own position in its slot plus, for every other slot, the number of
 * candidates there that come before it in (r, chunk, slot, j) order (a
 * binary search): the stable r order of the (chunk, slot, j) base order.
 * The metrics are FP32 values, so the metric sort uses 32-bit float keys.  The greedy pass runs in one
 * CTA: for each kept candidate, in metric order, the threads mark every later
 * candidate it is related to; a candidate is kept when no earlier kept one
 * marked it, as in the host loop.  The FP64 expressions are the host's.
 */
#include <cuda_runtime.h>

#include <atomic>
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "cs_internal.h"
#include "cs_collapse.h"

namespace cl {

constexpr int NT = 256;

struct SlotInfo {
    int k[CS_MAX_SLOT];
    int Hk[CS_MAX_SLOT];
};

__global__ void harvest_kernel(const CsRec *recs, unsigned n, const CsChunk *chunks,
                               long long nchunks, SlotInfo si, int nslot, int nprof,
                               double r_lo, double lodr, double nyq, double T, double thr,
                               uint64_t *key, uint64_t *bkey, int *slot_of, unsigned *idx,
                               double *r, double *freq, double *metric, int *nharm,
                               unsigned *nvalid, unsigned *slot_cnt)
{
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const CsRec rc = recs[i];
    const double m = (double)rc.metric;
    bool ok = m > thr && rc.slot >= 0 && rc.slot < nslot;
    double rsel = INFINITY;
    if (ok) {
        const double rstart = r_lo + (double)chunks[rc.chunk].i0 * lodr;
        const double rfreq = rstart + (double)rc.j * lodr;
        const double kmul = (double)si.k[rc.slot];
        rsel = kmul != 1.0 ? kmul * rfreq : rfreq;
        if (rc.slot != 0 && !(rsel < nyq)) ok = false;
    }
    idx[i] = i;
    if (ok) {
        /* sort key (slot, chunk, j); tie-break key (chunk, slot, j), the base order */
        key[i] = ((uint64_t)rc.slot * (uint64_t)nchunks + (uint64_t)rc.chunk) * (uint64_t)nprof +
                 (uint64_t)rc.j;
        bkey[i] = ((uint64_t)rc.chunk * (uint64_t)nslot + (uint64_t)rc.slot) * (uint64_t)nprof +
                  (uint64_t)rc.j;
        slot_of[i] = rc.slot;
        atomicAdd(&slot_cnt[rc.slot], 1u);
        r[i] = rsel;
        freq[i] = rsel / T;
        metric[i] = m;
        nharm[i] = si.Hk[rc.slot];
        atomicAdd(nvalid, 1u);
    } else {
        key[i] = ~0ull;                 /* after every valid record */
        bkey[i] = ~0ull;
        slot_of[i] = 0;
        r[i] = INFINITY;
        freq[i] = INFINITY;
        metric[i] = -INFINITY;
        nharm[i] = 0;
    }
}

__global__ void slot_starts_kernel(const unsigned *cnt, int nslot, unsigned *start)
{
    unsigned acc = 0;
    for (int s = 0; s < nslot; s++) { start[s] = acc; acc += cnt[s]; }
}

/* order1 holds the valid records grouped by slot, each group in trial order
 * (so in strictly rising v); out receives them in (v, base key) order */
__global__ void merge_kernel(const unsigned *order1, const unsigned *nv, const int *slot_of,
                             const uint64_t *bkey, const double *v, const unsigned *start,
                             const unsigned *cnt, int nslot, unsigned *out)
{
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= *nv) return;
    const unsigned x = order1[i];
    const int s = slot_of[x];
    const double vx = v[x];
    const uint64_t bx = bkey[x];
    unsigned rank = i - start[s];
    for (int t = 0; t < nslot; t++) {
        if (t == s || cnt[t] == 0) continue;
        unsigned lo = start[t], hi = start[t] + cnt[t], a = lo, b = hi;
        while (a < b) {
            const unsigned mid = (a + b) >> 1;
            if (v[order1[mid]] < vx) a = mid + 1; else b = mid;
        }
        unsigned c = a - lo;
        if (a < hi && v[order1[a]] == vx && bkey[order1[a]] < bx) c++;
        rank += c;
    }
    out[rank] = x;
}

/* run starts of remove_duplicates over the first nv of the r-sorted list
 * (zero past nv, so that a scan over all n entries counts only real runs) */
__global__ void run_flags_kernel(const unsigned *order, const double *r, unsigned n,
                                 const unsigned *nv, double drtol, unsigned *flag)
{
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    flag[i] = i < *nv && (i == 0 || r[order[i]] - r[order[i - 1]] > drtol) ? 1u : 0u;
}

/* the first member of largest metric of each run, as a segmented argmax:
 * every candidate offers (metric, earliest position) to its run with one
 * 64-bit atomicMax.  The metrics are FP32 values, so their float bits (made
 * order-preserving) compare like the doubles the host compares. */
static __device__ __forceinline__ uint32_t ordered_bits(float f)
{
    const uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

__global__ void run_offer_kernel(const unsigned *order, const double *metric,
                                 const unsigned *flag, const unsigned *runid,
                                 const unsigned *nv, unsigned long long *best)
{
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= *nv) return;
    const unsigned run = runid[i] + flag[i] - 1u;
    const unsigned long long key =
        ((unsigned long long)ordered_bits((float)metric[order[i]]) << 32) |
        (unsigned long long)(0xFFFFFFFFu - i);
    atomicMax(&best[run], key);
}

__global__ void run_take_kernel(const unsigned *order, const unsigned long long *best,
                                unsigned n, const unsigned *m, unsigned *out)
{
    const unsigned r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n || r >= *m) return;
    out[r] = order[0xFFFFFFFFu - (unsigned)(best[r] & 0xFFFFFFFFull)];
}

__global__ void count_runs_kernel(const unsigned *flag, const unsigned *runid, unsigned n,
                                  unsigned *m)
{
    *m = runid[n - 1] + flag[n - 1];
}

__global__ void copy_count_kernel(const unsigned *src, unsigned *dst)
{
    *dst = *src;
}

/* descending-sort keys; entries past m sort after every real one */
__global__ void gather_metric_kernel(const unsigned *list, const double *metric, unsigned n,
                                     const unsigned *m, float *key, unsigned *pos)
{
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    key[i] = i < *m ? (float)metric[list[i]] : -INFINITY;     /* FP32 values: exact */
    pos[i] = i;
}

static __device__ bool related(double r1, double r2, int numharm, double tol)
{
    const double lo = r1 < r2 ? r1 : r2;
    const double hi = r1 < r2 ? r2 : r1;
    if (!(lo > 0.0)) return false;
    for (int mm = 1; mm <= numharm; mm++) {
        const int nn = (int)rint((double)mm * hi / lo);
        if (nn < 1 || nn > numharm) continue;
        if (fabs((double)mm * hi - (double)nn * lo) <= tol * (double)mm) return true;
    }
    return false;
}

/* remove_harmonics' greedy loop over the metric-ordered list (one CTA).
 * The walk is serial in the list, so with up to GREEDY_SMEM candidates the
 * positions' r values and the removal marks are staged in shared memory and
 * a step costs a shared read, not two dependent global loads; longer lists
 * walk global memory. */
constexpr unsigned GREEDY_SMEM = 8192;
__global__ void __launch_bounds__(1024) greedy_kernel(const unsigned *list, const unsigned *pos,
                                                      const double *r, const unsigned *mp,
                                                      int numharm, double tol,
                                                      unsigned char *removed,
                                                      unsigned char *keep_by_pos)
{
    extern __shared__ double gsm[];               /* [GREEDY_SMEM] r, then the marks */
    const unsigned m = *mp;
    if (m <= GREEDY_SMEM) {
        double *rs = gsm;
        unsigned char *rm = reinterpret_cast<unsigned char *>(gsm + GREEDY_SMEM);
        for (unsigned j = threadIdx.x; j < m; j += blockDim.x) {
            rs[j] = r[list[pos[j]]];
            rm[j] = 0;
        }
        __syncthreads();
        for (unsigned i = 0; i < m; i++) {
            if (rm[i]) continue;                    /* the same value in every thread */
            const double ri = rs[i];
            for (unsigned j = i + 1 + threadIdx.x; j < m; j += blockDim.x)
                if (!rm[j] && related(rs[j], ri, numharm, tol)) rm[j] = 1;
            __syncthreads();
        }
        for (unsigned q = threadIdx.x; q < m; q += blockDim.x) keep_by_pos[pos[q]] = !rm[q];
        return;
    }
    for (unsigned j = threadIdx.x; j < m; j += blockDim.x) removed[j] = 0;
    __syncthreads();
    for (unsigned i = 0; i < m; i++) {
        if (removed[i]) continue;               /* the same value in every thread */
        const double ri = r[list[pos[i]]];
        for (unsigned j = i + 1 + threadIdx.x; j < m; j += blockDim.x)
            if (!removed[j] && related(r[list[pos[j]]], ri, numharm, tol)) removed[j] = 1;
        __syncthreads();
    }
    for (unsigned q = threadIdx.x; q < m; q += blockDim.x) keep_by_pos[pos[q]] = !removed[q];
}

__global__ void emit_kernel(const unsigned *list, const unsigned char *keep, const unsigned *mp,
                            const double *r, const double *freq, const double *metric,
                            const int *nharm, Candidate *out, unsigned *nout)
{
    const unsigned m = *mp;
    /* one CTA: an ordered compaction (m is a few thousand at most) */
    __shared__ unsigned base;
    __shared__ unsigned warp_tot[32];
    if (threadIdx.x == 0) base = 0;
    __syncthreads();
    const unsigned lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (unsigned s = 0; s < m; s += blockDim.x) {
        const unsigned i = s + threadIdx.x;
        const bool k = i < m && (keep == nullptr || keep[i]);
        const unsigned bal = __ballot_sync(0xffffffffu, k);
        if (lane == 0) warp_tot[w] = __popc(bal);
        __syncthreads();
        unsigned off = base;
        for (unsigned q = 0; q < w; q++) off += warp_tot[q];
        if (k) {
            const unsigned c = list[i];
            Candidate cd;
            cd.freq = freq[c];
            cd.metric = metric[c];
            cd.r = r[c];
            cd.nharm = nharm[c];
            cd.ducy = NAN;
            out[off + __popc(bal & ((1u << lane) - 1u))] = cd;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned t = 0;
            for (unsigned q = 0; q < nw; q++) t += warp_tot[q];
            base += t;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *nout = base;
}

}  // namespace cl

/* The greedy kernel's shared-memory limit, raised once per device (the
 * attribute belongs to the device that is current when it is set). */
static cudaError_t greedy_prepare(size_t gsmem)
{
    static std::atomic<unsigned long long> done{0};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64) return e;
    const unsigned long long bit = 1ULL << dev;
    if (done.load(std::memory_order_acquire) & bit) return cudaSuccess;
    e = cudaFuncSetAttribute((const void *)cl::greedy_kernel,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gsmem);
    if (e == cudaSuccess) done.fetch_or(bit, std::memory_order_acq_rel);
    return e;
}

struct CsCollapse {
    size_t cap;                     /* records */
    uint64_t *key[2];
    unsigned *idx[2];
    uint64_t *bkey;
    int *slot_of;
    unsigned *merged;
    double *r, *freq, *metric;
    int *nharm;
    unsigned *flag, *runid, *list;
    float *mkey[2];
    unsigned *mpos[2];
    unsigned char *removed, *keep;
    Candidate *out;
    unsigned *counters;             /* device: nvalid, runs, kept; then per-slot counts
                                       and starts (CS_MAX_SLOT each) */
    unsigned *h_counters;           /* pinned */
    Candidate *h_out;               /* pinned */
    size_t h_out_cap;
    void *temp;
    size_t temp_bytes;
    unsigned pending_n;             /* records of the enqueued collapse */
};

static void collapse_release_buffers(CsCollapse *w)
{
    for (int b = 0; b < 2; b++) {
        cudaFree(w->key[b]); cudaFree(w->idx[b]); cudaFree(w->mkey[b]); cudaFree(w->mpos[b]);
        w->key[b] = nullptr; w->idx[b] = nullptr; w->mkey[b] = nullptr; w->mpos[b] = nullptr;
    }
    cudaFree(w->bkey); cudaFree(w->slot_of); cudaFree(w->merged);
    w->bkey = nullptr; w->slot_of = nullptr; w->merged = nullptr;
    cudaFree(w->r); cudaFree(w->freq); cudaFree(w->metric); cudaFree(w->nharm);
    cudaFree(w->flag); cudaFree(w->runid); cudaFree(w->list);
    cudaFree(w->removed); cudaFree(w->keep); cudaFree(w->out); cudaFree(w->temp);
    w->r = w->freq = w->metric = nullptr;
    w->nharm = nullptr;
    w->flag = w->runid = w->list = nullptr;
    w->removed = w->keep = nullptr;
    w->out = nullptr;
    w->temp = nullptr;
    w->temp_bytes = 0;
    w->cap = 0;
}

static cudaError_t collapse_reserve(CsCollapse *w, size_t n)
{
    if (n <= w->cap) return cudaSuccess;
    collapse_release_buffers(w);
    const size_t c = n + n / 4 + 1024;
    cudaError_t e = cudaSuccess;
#define AL(p, bytes) if (e == cudaSuccess) e = cudaMalloc((void **)&(p), (bytes))
    for (int b = 0; b < 2; b++) {
        AL(w->key[b], c * sizeof(uint64_t));
        AL(w->idx[b], c * sizeof(unsigned));
        AL(w->mkey[b], c * sizeof(float));
        AL(w->mpos[b], c * sizeof(unsigned));
    }
    AL(w->bkey, c * sizeof(uint64_t));
    AL(w->slot_of, c * sizeof(int));
    AL(w->merged, c * sizeof(unsigned));
    AL(w->r, c * sizeof(double));
    AL(w->freq, c * sizeof(double));
    AL(w->metric, c * sizeof(double));
    AL(w->nharm, c * sizeof(int));
    AL(w->flag, c * sizeof(unsigned));
    AL(w->runid, c * sizeof(unsigned));
    AL(w->list, c * sizeof(unsigned));
    AL(w->removed, c);
    AL(w->keep, c);
    AL(w->out, c * sizeof(Candidate));
    if (!w->counters) AL(w->counters, (4 + 2 * CS_MAX_SLOT) * sizeof(unsigned));
#undef AL
    if (e != cudaSuccess) return e;
    /* the largest CUB scratch any step needs at this capacity */
    size_t t1 = 0, t2 = 0, t3 = 0;
    cub::DoubleBuffer<uint64_t> kb(w->key[0], w->key[1]);
    cub::DoubleBuffer<unsigned> ib(w->idx[0], w->idx[1]);
    cub::DoubleBuffer<float> mb(w->mkey[0], w->mkey[1]);
    cub::DoubleBuffer<unsigned> pb(w->mpos[0], w->mpos[1]);
    e = cub::DeviceRadixSort::SortPairs(nullptr, t1, kb, ib, (int)c);
    if (e == cudaSuccess) e = cub::DeviceRadixSort::SortPairsDescending(nullptr, t2, mb, pb, (int)c);
    if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, t3, w->flag, w->runid, (int)c);
    if (e != cudaSuccess) return e;
    w->temp_bytes = std::max(t1, std::max(t2, t3));
    e = cudaMalloc(&w->temp, w->temp_bytes);
    if (e == cudaSuccess) w->cap = c;
    return e;
}

CsCollapse *cs_collapse_new(void)
{
    CsCollapse *w = (CsCollapse *)calloc(1, sizeof(CsCollapse));
    if (!w) return nullptr;
    if (cudaMallocHost((void **)&w->h_counters, 4 * sizeof(unsigned)) != cudaSuccess) {
        free(w);
        return nullptr;
    }
    return w;
}

void cs_collapse_free(CsCollapse *w)
{
    if (!w) return;
    collapse_release_buffers(w);
    cudaFree(w->counters);
    if (w->h_counters) cudaFreeHost(w->h_counters);
    if (w->h_out) cudaFreeHost(w->h_out);
    free(w);
}

static int bit_length_u64(uint64_t v)
{
    int b = 0;
    while (v) { b++; v >>= 1; }
    return b;
}

int cs_collapse_enqueue(CsCollapse *w, const CsRec *recs, unsigned n, const CsChunk *chunks,
                        long long nchunks, const int *slot_k, const int *slot_Hk, int nslot,
                        int nprof, double r_lo, double lodr, double N, double T,
                        double threshold, int remove, double dr_tol, int harm_remove,
                        int numharm, double harm_tol, cudaStream_t st)
{
    if (!w || nslot < 1 || nslot > CS_MAX_SLOT || nprof < 1 || nchunks < 1) return -1;
    w->pending_n = n;
    if (n == 0) return 0;
    cl::SlotInfo si;
    memset(&si, 0, sizeof(si));
    for (int s = 0; s < nslot; s++) { si.k[s] = slot_k[s]; si.Hk[s] = slot_Hk[s]; }
    const unsigned g = (n + cl::NT - 1) / cl::NT;
    const int end_bit = bit_length_u64((uint64_t)nchunks * (uint64_t)nslot * (uint64_t)nprof);
    size_t tb = 0;
    const unsigned *order = nullptr, *listp = nullptr;
    const unsigned char *keep = nullptr;
    cudaError_t e = collapse_reserve(w, n);       /* allocates the counters on first use */
    if (e != cudaSuccess || !w->counters) {
        fprintf(stderr, "Error: candidate collapse on the GPU: %s\n", cudaGetErrorString(e));
        return -1;
    }
    unsigned *nv = w->counters, *m = w->counters + 1, *nout = w->counters + 2;
    e = cudaMemsetAsync(w->counters, 0, (4 + 2 * CS_MAX_SLOT) * sizeof(unsigned), st);
    unsigned *slot_cnt = w->counters + 4, *slot_start = w->counters + 4 + CS_MAX_SLOT;
    if (e == cudaSuccess) {
        cl::harvest_kernel<<<g, cl::NT, 0, st>>>(recs, n, chunks, nchunks, si, nslot, nprof,
                                                 r_lo, lodr, N / 2.0, T, threshold, w->key[0],
                                                 w->bkey, w->slot_of, w->idx[0], w->r, w->freq,
                                                 w->metric, w->nharm, nv, slot_cnt);
        e = cudaGetLastError();
    }
    /* every slot's records in trial order; invalid records (all-ones key) last */
    cub::DoubleBuffer<uint64_t> kb(w->key[0], w->key[1]);
    cub::DoubleBuffer<unsigned> ib(w->idx[0], w->idx[1]);
    if (e == cudaSuccess) {
        tb = w->temp_bytes;
        e = cub::DeviceRadixSort::SortPairs(w->temp, tb, kb, ib, (int)n, 0, end_bit, st);
    }
    /* merged into stable r order (remove) or stable frequency order */
    if (e == cudaSuccess) {
        cl::slot_starts_kernel<<<1, 1, 0, st>>>(slot_cnt, nslot, slot_start);
        cl::merge_kernel<<<g, cl::NT, 0, st>>>(ib.Current(), nv, w->slot_of, w->bkey,
                                               remove ? w->r : w->freq, slot_start, slot_cnt,
                                               nslot, w->merged);
        e = cudaGetLastError();
    }
    order = w->merged;
    if (remove) {
        if (e == cudaSuccess) {
            cl::run_flags_kernel<<<g, cl::NT, 0, st>>>(order, w->r, n, nv, dr_tol, w->flag);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) {
            tb = w->temp_bytes;
            e = cub::DeviceScan::ExclusiveSum(w->temp, tb, w->flag, w->runid, (int)n, st);
        }
        /* the key buffers are free once the merge has run: best-of-run slots */
        unsigned long long *best = reinterpret_cast<unsigned long long *>(w->key[0]);
        if (e == cudaSuccess) e = cudaMemsetAsync(best, 0, (size_t)n * sizeof(uint64_t), st);
        if (e == cudaSuccess) {
            cl::count_runs_kernel<<<1, 1, 0, st>>>(w->flag, w->runid, n, m);
            cl::run_offer_kernel<<<g, cl::NT, 0, st>>>(order, w->metric, w->flag, w->runid, nv,
                                                       best);
            cl::run_take_kernel<<<g, cl::NT, 0, st>>>(order, best, n, m, w->list);
            e = cudaGetLastError();
        }
        listp = w->list;
    } else {
        if (e == cudaSuccess) {
            cl::copy_count_kernel<<<1, 1, 0, st>>>(nv, m);
            e = cudaGetLastError();
        }
        listp = order;
    }
    if (harm_remove) {
        if (e == cudaSuccess) {
            cl::gather_metric_kernel<<<g, cl::NT, 0, st>>>(listp, w->metric, n, m, w->mkey[0],
                                                           w->mpos[0]);
            e = cudaGetLastError();
        }
        cub::DoubleBuffer<float> mb(w->mkey[0], w->mkey[1]);
        cub::DoubleBuffer<unsigned> pb(w->mpos[0], w->mpos[1]);
        if (e == cudaSuccess) {
            tb = w->temp_bytes;
            e = cub::DeviceRadixSort::SortPairsDescending(w->temp, tb, mb, pb, (int)n, 0, 32, st);
        }
        if (e == cudaSuccess) {
            const size_t gsmem = cl::GREEDY_SMEM * (sizeof(double) + 1);
            e = greedy_prepare(gsmem);
            if (e == cudaSuccess) {
                cl::greedy_kernel<<<1, 1024, gsmem, st>>>(listp, pb.Current(), w->r, m, numharm,
                                                          harm_tol, w->removed, w->keep);
                e = cudaGetLastError();
            }
        }
        keep = w->keep;
    }
    if (e == cudaSuccess) {
        cl::emit_kernel<<<1, 1024, 0, st>>>(listp, keep, m, w->r, w->freq, w->metric,
                                            w->nharm, w->out, nout);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(w->h_counters, w->counters, 4 * sizeof(unsigned),
                            cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) {
        fprintf(stderr, "Error: candidate collapse on the GPU: %s\n", cudaGetErrorString(e));
        return -1;
    }
    return 0;
}

int cs_collapse_finish(CsCollapse *w, cudaStream_t st, CandidateList *out)
{
    candlist_init(out);
    if (!w) return -1;
    if (w->pending_n == 0) return 0;
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) goto fail;
    {
        const unsigned nout = w->h_counters[2];
        if (nout > w->h_out_cap) {
            if (w->h_out) cudaFreeHost(w->h_out);
            w->h_out = nullptr;
            w->h_out_cap = 0;
            e = cudaMallocHost((void **)&w->h_out,
                               (size_t)(nout + nout / 4 + 256) * sizeof(Candidate));
            if (e != cudaSuccess) goto fail;
            w->h_out_cap = nout + nout / 4 + 256;
        }
        if (nout) {
            e = cudaMemcpyAsync(w->h_out, w->out, (size_t)nout * sizeof(Candidate),
                                cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) goto fail;
            out->v = (Candidate *)malloc((size_t)nout * sizeof(Candidate));
            if (!out->v) return -1;
            memcpy(out->v, w->h_out, (size_t)nout * sizeof(Candidate));
            out->n = nout;
            out->cap = nout;
        }
    }
    w->pending_n = 0;
    return 0;
fail:
    fprintf(stderr, "Error: candidate collapse on the GPU: %s\n", cudaGetErrorString(e));
    return -1;
}
