/*
 * The decisions of prepsubband's time-domain clipping on the GPU: which
 * spectra PRESTO's clip_times (third_party/presto/src/clipping.c:47-230)
 * replaces when the reference runs its front end with -clip clip_sigma (its
 * default is 6).  clip_times runs on every raw block of L spectra in read
 * order (backend_common.c:976-986), with running statistics carried from
 * block to block:
 *
 *   zero-DM series   the sum of each spectrum over all channels (exact for
 *                    8-bit data: an integer below 2^24 as a float);
 *   block stats      avg_var (misc_utils.c:641-676, AS 52 recurrence in
 *                    double) and the lower median (median.c, element
 *                    (L-1)/2 of the sorted block); the "good" samples lie
 *                    strictly inside median -+ 3 sigma (float cut-offs), and
 *                    their avg_var gives the block's mean and sigma (the
 *                    running values stand in when no sample is good);
 *   running values   floats: mean and sigma of the first block, then
 *                    0.9 * old + 0.1 * new, evaluated in double;
 *   decision         spectrum t is replaced when
 *                    |zdm[t] - running_mean| > clip_sigma * running_sigma
 *                    (the difference in float, the test in double).
 *
 *   replacement      a replaced spectrum takes the block's channel levels:
 *                    per channel the sum over the block's good spectra (an
 *                    integer, exact) over their number, in double, then the
 *                    running level, a float: the first block's value, then
 *                    0.9 * old + 0.1 * new in double (clipping.c:118-160);
 *                    a block without good spectra keeps the old level.
 *
 * cs_clip_count gives the number of replaced spectra (and optionally the
 * flags); cs_clip_levels adds the levels, which the clipped dedispersion
 * (cs_dedisp_run_device_clipped) substitutes.  The arithmetic is the
 * reference's as its build compiles it (-ffp-contract=off, src/Makefile:43):
 * this file is built with -fmad=false.  Its -Ofast may still rewrite a
 * division by the good count as a reciprocal product; that changes the
 * double value by an ulp at most, below what the float level keeps.
 */
#include <cuda_runtime.h>

#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>

#include "cs_b200.h"

#define CS_EXPORT extern "C" __attribute__((visibility("default")))

namespace ck {

constexpr int MAX_L = 8192;
constexpr int NT = 256;

/* zero-DM sum of each spectrum: one warp per spectrum */
__global__ void zdm_kernel(const uint8_t *raw, long long nspec, int nchan, int vec16, int *zdm)
{
    const long long t = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (t >= nspec) return;
    const uint8_t *row = raw + t * (long long)nchan;
    unsigned s = 0;
    if (vec16) {
        const uint4 *r4 = reinterpret_cast<const uint4 *>(row);
        for (int i = lane; i < nchan / 16; i += 32) {
            const uint4 w = __ldg(r4 + i);
            s = __dp4a(w.x, 0x01010101u, s);
            s = __dp4a(w.y, 0x01010101u, s);
            s = __dp4a(w.z, 0x01010101u, s);
            s = __dp4a(w.w, 0x01010101u, s);
        }
    } else {
        for (int c = lane; c < nchan; c += 32) s += row[c];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) zdm[t] = (int)s;
}

/* avg_var (misc_utils.c:641-676) over n floats, in order */
struct AvgVar {
    double mean = 0.0, var_acc = 0.0, an1 = 0.0;
    long n = 0;
    __device__ void push(float x)
    {
        if (n == 0) {
            mean = (double)x;
        } else {
            const double an = (double)(n + 1);
            an1 = (double)n;
            const double dx = ((double)x - mean) / an;
            var_acc += an * an1 * dx * dx;
            mean += dx;
        }
        n++;
    }
    __device__ double var() const { return n > 1 ? var_acc / an1 : var_acc; }
};

struct BlockStats {
    int ngood;
    float med;               /* lower median of the block */
    float lo, hi;            /* good samples lie strictly between */
    double mean, sigma;      /* of the good samples */
};

/* one CTA per block: the lower median, by a shared-memory bitonic sort */
__global__ void __launch_bounds__(NT) median_kernel(const int *zdm, int L, int P2,
                                                    BlockStats *out)
{
    extern __shared__ int srt[];
    const long long b = blockIdx.x;
    for (int i = threadIdx.x; i < P2; i += NT) srt[i] = i < L ? zdm[b * L + i] : INT_MAX;
    __syncthreads();
    for (int k = 2; k <= P2; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < P2; i += NT) {
                const int l = i ^ j;
                if (l > i) {
                    const bool up = (i & k) == 0;
                    const int a = srt[i], c = srt[l];
                    if ((a > c) == up) { srt[i] = c; srt[l] = a; }
                }
            }
            __syncthreads();
        }
    if (threadIdx.x == 0) out[b].med = (float)srt[(L - 1) / 2];
}

/* one thread per block: the two sequential avg_var passes (all samples, then
 * the good ones).  Each is a chain of dependent double divisions; running
 * every block's chain at once keeps the GPU busy where one thread per CTA
 * would leave the CTA idle.  Samples are read eight at a time, ahead of the
 * chain. */
constexpr int ZB = 8;
__global__ void __launch_bounds__(64) stats_kernel(const int *zdm, int L, long long nblocks,
                                                   BlockStats *out)
{
    const long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nblocks) return;
    const int *x = zdm + b * L;
    AvgVar all;
    for (int i0 = 0; i0 < L; i0 += ZB) {
        int v[ZB];
#pragma unroll
        for (int k = 0; k < ZB; k++) v[k] = i0 + k < L ? __ldg(x + i0 + k) : 0;
#pragma unroll
        for (int k = 0; k < ZB; k++)
            if (i0 + k < L) all.push((float)v[k]);
    }
    const double sd = sqrt(all.var());
    const float med = out[b].med;
    const float lo = (float)((double)med - 3.0 * sd);
    const float hi = (float)((double)med + 3.0 * sd);
    AvgVar good;
    for (int i0 = 0; i0 < L; i0 += ZB) {
        int v[ZB];
#pragma unroll
        for (int k = 0; k < ZB; k++) v[k] = i0 + k < L ? __ldg(x + i0 + k) : 0;
#pragma unroll
        for (int k = 0; k < ZB; k++) {
            const float f = (float)v[k];
            if (i0 + k < L && f > lo && f < hi) good.push(f);
        }
    }
    BlockStats &s = out[b];
    s.lo = lo;
    s.hi = hi;
    s.ngood = (int)good.n;
    s.mean = good.mean;
    s.sigma = good.n ? sqrt(good.var()) : 0.0;
}

/* the running mean / sigma from block to block (one thread; the block
 * statistics are read eight blocks ahead of the chain) */
__global__ void running_kernel(const BlockStats *st, long long nblocks, float clip_sigma,
                               float *ravg, float *trig)
{
    float running_avg = 0.0f, running_std = 0.0f;
    for (long long b0 = 0; b0 < nblocks; b0 += ZB) {
        int ng[ZB];
        double mn[ZB], sg[ZB];
#pragma unroll
        for (int k = 0; k < ZB; k++)
            if (b0 + k < nblocks) {
                ng[k] = st[b0 + k].ngood;
                mn[k] = st[b0 + k].mean;
                sg[k] = st[b0 + k].sigma;
            }
#pragma unroll
        for (int k = 0; k < ZB; k++) {
            const long long b = b0 + k;
            if (b >= nblocks) break;
            double cur_avg, cur_std;
            if (ng[k] < 1) {
                cur_avg = (double)running_avg;
                cur_std = (double)running_std;
            } else {
                cur_avg = mn[k];
                cur_std = sg[k];
            }
            if (b) {
                running_avg = (float)(0.9 * (double)running_avg + 0.1 * cur_avg);
                running_std = (float)(0.9 * (double)running_std + 0.1 * cur_std);
            } else {
                running_avg = (float)cur_avg;
                running_std = (float)cur_std;
            }
            ravg[b] = running_avg;
            trig[b] = clip_sigma * running_std;
        }
    }
}

__global__ void decide_kernel(const int *zdm, long long n, int L, const float *ravg,
                              const float *trig, unsigned long long *count, uint8_t *flags)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const long long b = t / L;
    const float d = (float)zdm[t] - ravg[b];
    const bool clip = fabs((double)d) > (double)trig[b];
    if (flags) flags[t] = clip ? 1 : 0;
    if (clip) atomicAdd(count, 1ull);
}

/* per (block, channel column): the sum of the column over the block's good
 * spectra, stored as a float (an integer below 2^24: exact) */
__global__ void chan_sum_kernel(const uint8_t *raw, int L, int nchan, const int *zdm,
                                const BlockStats *st, float *sums)
{
    const long long b = blockIdx.x;
    const int c = blockIdx.y * blockDim.x + threadIdx.x;
    if (c >= nchan) return;
    const float lo = st[b].lo, hi = st[b].hi;
    const uint8_t *col = raw + b * L * (long long)nchan + c;
    unsigned s = 0;
    for (int i = 0; i < L; i++) {
        const float v = (float)zdm[b * L + i];
        if (v > lo && v < hi) s += __ldg(col + (long long)i * nchan);
    }
    sums[b * nchan + c] = (float)s;
}

/* The same sums with 16-byte loads (nchan a multiple of 16, raw 16-byte
 * aligned, nchan / 16 <= NT): one CTA per block; thread (row phase p, group g)
 * adds channels 16g..16g+15 of rows p, p + R, ... and the R row phases are
 * added in shared memory (integers, so the order does not matter). */
__global__ void __launch_bounds__(NT) chan_sum16_kernel(const uint8_t *raw, int L, int nchan,
                                                        const int *zdm, const BlockStats *st,
                                                        float *sums)
{
    extern __shared__ unsigned part[];                /* [R][nchan] */
    const long long b = blockIdx.x;
    const int G = nchan >> 4, R = NT / G;
    const int g = threadIdx.x % G, p = threadIdx.x / G;
    const float lo = st[b].lo, hi = st[b].hi;
    unsigned c[16];
#pragma unroll
    for (int k = 0; k < 16; k++) c[k] = 0;
    if (p < R) {
        const uint4 *rows = reinterpret_cast<const uint4 *>(raw + b * L * (long long)nchan) + g;
        for (int i = p; i < L; i += R) {
            const float v = (float)zdm[b * L + i];
            if (!(v > lo && v < hi)) continue;
            const uint4 w = __ldg(rows + (long long)i * G);
            const unsigned ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
            for (int q = 0; q < 4; q++)
#pragma unroll
                for (int k = 0; k < 4; k++) c[4 * q + k] += (ws[q] >> (8 * k)) & 0xffu;
        }
#pragma unroll
        for (int k = 0; k < 16; k++) part[p * nchan + 16 * g + k] = c[k];
    }
    __syncthreads();
    for (int ch = threadIdx.x; ch < nchan; ch += blockDim.x) {
        unsigned t = 0;
        for (int q = 0; q < R; q++) t += part[q * nchan + ch];
        sums[b * nchan + ch] = (float)t;
    }
}

/* running channel levels from block to block, in place over the sums (one
 * thread per channel column) */
__global__ void levels_kernel(const BlockStats *st, long long nblocks, int nchan, float *lv)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nchan) return;
    float run = 0.0f;
    for (long long b0 = 0; b0 < nblocks; b0 += ZB) {
        int ng[ZB];
        float sum[ZB];
#pragma unroll
        for (int k = 0; k < ZB; k++)
            if (b0 + k < nblocks) {
                ng[k] = st[b0 + k].ngood;
                sum[k] = lv[(b0 + k) * nchan + c];
            }
#pragma unroll
        for (int k = 0; k < ZB; k++) {
            const long long b = b0 + k;
            if (b >= nblocks) break;
            const double cur = ng[k] >= 1 ? (double)sum[k] / (double)ng[k] : (double)run;
            run = b ? (float)(0.9 * (double)run + 0.1 * cur) : (float)cur;
            lv[b * nchan + c] = run;
        }
    }
}

}  // namespace ck

/* scratch layout: zero-DM sums, block statistics, running values, count */
static size_t clip_layout(long long nspec, int L, size_t off[5])
{
    const long long nblocks = nspec / L, n = nblocks * L;
    size_t o = 0;
    auto take = [&](size_t bytes) { const size_t at = o; o = (o + bytes + 255) & ~(size_t)255; return at; };
    off[0] = take((size_t)n * sizeof(int));
    off[1] = take((size_t)nblocks * sizeof(ck::BlockStats));
    off[2] = take((size_t)nblocks * sizeof(float));
    off[3] = take((size_t)nblocks * sizeof(float));
    off[4] = take(sizeof(unsigned long long));
    return o;
}

CS_EXPORT size_t cs_clip_scratch_bytes(long long nspec, int L)
{
    if (nspec < 0 || L < 1) return 0;
    size_t off[5];
    return clip_layout(nspec, L, off);
}

static int clip_run(const uint8_t *d_raw, long long nspec, int nchan, int L, float clip_sigma,
                    long long *nclipped, uint8_t *d_flags, float *d_levels, void *d_scratch,
                    size_t scratch_bytes, void *stream, int device, const char *who)
{
    if (!nclipped || nchan < 1 || L < 1 || L > ck::MAX_L || nspec < 0) return -1;
    *nclipped = 0;
    const long long nblocks = nspec / L;     /* a partial last block is never read */
    if (nblocks == 0 || !(clip_sigma > 0.0f)) return 0;
    if (!d_raw) return -1;
    if (cudaSetDevice(device) != cudaSuccess) return -1;
    cudaStream_t st = (cudaStream_t)stream;
    const long long n = nblocks * L;
    int P2 = 1;
    while (P2 < L) P2 <<= 1;
    const size_t smem = (size_t)P2 * sizeof(int);
    size_t off[5];
    const size_t need = clip_layout(nspec, L, off);
    cudaError_t e = cudaSuccess;
    char *base = (char *)d_scratch;
    const bool own = d_scratch == nullptr;
    if (own) {
        e = cudaMalloc((void **)&base, need);
    } else if (scratch_bytes < need || ((uintptr_t)d_scratch & 255)) {
        fprintf(stderr, "Error: %s: scratch of %zu bytes (256-byte aligned) needed\n", who, need);
        return -1;
    }
    int *zdm = (int *)(base + off[0]);
    ck::BlockStats *bs = (ck::BlockStats *)(base + off[1]);
    float *ravg = (float *)(base + off[2]), *trig = (float *)(base + off[3]);
    unsigned long long *cnt = (unsigned long long *)(base + off[4]), hcnt = 0;
    if (e == cudaSuccess) e = cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), st);
    if (e == cudaSuccess && smem > 48 * 1024)
        e = cudaFuncSetAttribute((const void *)ck::median_kernel,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) {
        const int vec16 = (nchan % 16 == 0) && (((uintptr_t)d_raw & 15) == 0);
        const long long threads = n * 32;
        ck::zdm_kernel<<<(unsigned)((threads + ck::NT - 1) / ck::NT), ck::NT, 0, st>>>(
            d_raw, n, nchan, vec16, zdm);
        ck::median_kernel<<<(unsigned)nblocks, ck::NT, smem, st>>>(zdm, L, P2, bs);
        ck::stats_kernel<<<(unsigned)((nblocks + 63) / 64), 64, 0, st>>>(zdm, L, nblocks, bs);
        ck::running_kernel<<<1, 1, 0, st>>>(bs, nblocks, clip_sigma, ravg, trig);
        ck::decide_kernel<<<(unsigned)((n + ck::NT - 1) / ck::NT), ck::NT, 0, st>>>(
            zdm, n, L, ravg, trig, cnt, d_flags);
        if (d_levels) {
            const dim3 g((unsigned)nblocks, (unsigned)((nchan + ck::NT - 1) / ck::NT));
            const int G = nchan / 16;
            if (vec16 && G <= ck::NT) {
                const size_t psm = (size_t)(ck::NT / G) * nchan * sizeof(unsigned);
                ck::chan_sum16_kernel<<<(unsigned)nblocks, ck::NT, psm, st>>>(d_raw, L, nchan,
                                                                            zdm, bs, d_levels);
            } else {
                ck::chan_sum_kernel<<<g, ck::NT, 0, st>>>(d_raw, L, nchan, zdm, bs, d_levels);
            }
            ck::levels_kernel<<<(nchan + ck::NT - 1) / ck::NT, ck::NT, 0, st>>>(bs, nblocks,
                                                                              nchan, d_levels);
        }
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&hcnt, cnt, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (own) cudaFree(base);
    if (e != cudaSuccess) {
        fprintf(stderr, "Error: %s: %s\n", who, cudaGetErrorString(e));
        return -1;
    }
    *nclipped = (long long)hcnt;
    return 0;
}

CS_EXPORT int cs_clip_count(const uint8_t *d_raw, long long nspec, int nchan, int L,
                            float clip_sigma, long long *nclipped, uint8_t *d_flags,
                            void *d_scratch, size_t scratch_bytes, void *stream, int device)
{
    return clip_run(d_raw, nspec, nchan, L, clip_sigma, nclipped, d_flags, nullptr, d_scratch,
                    scratch_bytes, stream, device, "cs_clip_count");
}

CS_EXPORT int cs_clip_levels(const uint8_t *d_raw, long long nspec, int nchan, int L,
                             float clip_sigma, long long *nclipped, uint8_t *d_flags,
                             float *d_levels, void *d_scratch, size_t scratch_bytes, void *stream,
                             int device)
{
    if (!d_flags || !d_levels) {
        if (nclipped) *nclipped = 0;
        return -1;
    }
    return clip_run(d_raw, nspec, nchan, L, clip_sigma, nclipped, d_flags, d_levels, d_scratch,
                    scratch_bytes, stream, device, "cs_clip_levels");
}
