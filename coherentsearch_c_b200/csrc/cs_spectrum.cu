/*
 * Time series -> normalised spectrum on the GPU: the reference's in-memory
 * `realfft name.dat && rednoise name.fft` (src/datpipe.c:101-253).
 *
 *   realfft   forward real FFT of the N samples, packed PRESTO-style:
 *             N/2 complex bins, bin 0 holding (DC, Nyquist)
 *             (src/datpipe.c:101-138).  The transform is cuFFT's R2C (a plain
 *             library FFT); the packing is a kernel here.
 *   rednoise  the spectrum is normalised by running block medians of the
 *             power (src/datpipe.c:143-253): blocks of startwidth*ln(binnum)
 *             bins below endfreq Hz and endwidth bins above; a block's noise
 *             level is its lower median power / ln 2; from one block centre
 *             to the next the level moves linearly, with the slope (new -
 *             old) / (half the two widths); each bin is scaled by PRESTO's
 *             inverse square root of its level (the 0x5f3759df estimate and
 *             one Newton step, misc_utils.c); bin 0 becomes (1, 0).
 *
 * Block boundaries depend only on N, dt and the widths, not on the data, so
 * the host lays them out once per geometry (cs_spectrum_create) and the GPU
 * works on all blocks at once: one warp per block finds the lower median
 * (the (n-1)/2-th smallest power, by rank counting, which gives the same
 * value as the reference's quickselect); one thread per bin applies its
 * segment's level.  Output segments, in bin order: [1, 1 + mid_0) at level
 * 0; then for each block b >= 1 the bins from block b-1's centre to block
 * b's, at level[b-1] + slope[b] * i; then from the last block's centre to
 * the end with the last slope (1.0 when there is a single block).
 *
 * Parity: the reference's transform is FFTW in single precision followed by
 * a double-precision split whose twiddles come from a recurrence, so no
 * other FFT reproduces its last bits; the tests hold the spectrum to a
 * relative tolerance and the search results to the search's tolerances.
 * Where the reference build contracts a*b + c into a fused multiply-add
 * (src/datpipe.c is built with -ffp-contract=fast), the kernels use one too.
 */
#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "cs_b200.h"

#define CS_EXPORT extern "C" __attribute__((visibility("default")))

namespace sp {

constexpr int MAX_BLOCK = 128;     /* widths above this are refused */

/* PRESTO's inverse square root: estimate, then y * (1.5 - 0.5 x y y). */
static __device__ __forceinline__ float presto_invsqrtf(float x)
{
    const float y = __int_as_float(0x5f3759df - (__float_as_int(x) >> 1));
    const float t = __fmul_rn(__fmul_rn(0.5f, x), y);
    return __fmul_rn(y, __fmaf_rn(-t, y, 1.5f));
}

/* R2C output (N/2 + 1 bins) -> PRESTO packing (N/2 bins, bin 0 = DC, Nyq). */
__global__ void pack_kernel(const float2 *X, float2 *out, long long n2)
{
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n2) return;
    out[k] = k == 0 ? make_float2(X[0].x, X[n2].x) : X[k];
}

/* One warp per block: level = (float)(lower median power / ln 2).  The
 * block's powers (at most MAX_BLOCK, +inf past its end) are sorted by a
 * bitonic network over the warp -- element 32u + lane in register u of lane
 * `lane` -- and the (n-1)/2-th is read out: the reference's quickselect
 * returns the same value. */
__global__ void block_level_kernel(const float2 *amps, const long long *bstart, const int *blen,
                                   int nblk, double ln2, float *level)
{
    constexpr int R = MAX_BLOCK / 32;
    const int b = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (b >= nblk) return;
    const int n = blen[b];
    const float2 *a = amps + bstart[b];
    float p[R];
#pragma unroll
    for (int u = 0; u < R; u++) {
        const int i = lane + 32 * u;
        p[u] = INFINITY;
        if (i < n) {
            const float2 v = a[i];
            p[u] = __fmaf_rn(v.x, v.x, __fmul_rn(v.y, v.y));
        }
    }
#pragma unroll
    for (int k = 2; k <= MAX_BLOCK; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            if (j >= 32) {
                const int ju = j >> 5;            /* partner register */
#pragma unroll
                for (int u = 0; u < R; u++) {
                    if (u & ju) continue;
                    const bool asc = ((32 * u + lane) & k) == 0;
                    const float x = p[u], y = p[u | ju];
                    p[u] = asc ? fminf(x, y) : fmaxf(x, y);
                    p[u | ju] = asc ? fmaxf(x, y) : fminf(x, y);
                }
            } else {
                const bool lower = (lane & j) == 0;
#pragma unroll
                for (int u = 0; u < R; u++) {
                    const bool asc = ((32 * u + lane) & k) == 0;
                    const float x = p[u];
                    const float y = __shfl_xor_sync(0xffffffffu, x, j);
                    p[u] = (lower == asc) ? fminf(x, y) : fmaxf(x, y);
                }
            }
        }
    }
    const int k = (n - 1) / 2;
    float med = p[0];
#pragma unroll
    for (int u = 1; u < R; u++)
        if ((k >> 5) == u) med = p[u];
    med = __shfl_sync(0xffffffffu, med, k & 31);
    if (lane == 0) level[b] = (float)((double)med / ln2);
}

/* slope[b] (b >= 1) = (float)((double)(level[b] - level[b-1]) /
 * (0.5 * (n_{b-1} + n_b))), the difference taken in float as the
 * reference's float means do. */
__global__ void slope_kernel(const float *level, const int *blen, int nblk, float *slope)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < 1 || b >= nblk) return;
    slope[b] = (float)((double)__fsub_rn(level[b], level[b - 1]) /
                       (0.5 * (double)(blen[b - 1] + blen[b])));
}

/* One thread per bin.  Segment s: first bin sstart[s], level index
 * slvl[s]; sslope[s] = -1 for the first half block (no slope), 0 for a
 * slope of 1.0, else the block whose slope applies. */
__global__ void normalise_kernel(const float2 *amps, float2 *out, long long n2,
                                 const long long *sstart, const int *slvl, const int *sslope,
                                 int nseg, const float *level, const float *slope)
{
    /* the segment of the CTA's first bin, found once; a CTA's bins span a
     * few segments, so each thread walks on from there */
    __shared__ int seg0;
    const long long k0 = (long long)blockIdx.x * blockDim.x;
    if (threadIdx.x == 0) {
        int lo = 0, hi = nseg - 1;
        while (lo < hi) {             /* last segment starting at or before k0 */
            const int mid = (lo + hi + 1) >> 1;
            if (sstart[mid] <= k0) lo = mid;
            else hi = mid - 1;
        }
        seg0 = lo;
    }
    __syncthreads();
    const long long k = k0 + threadIdx.x;
    if (k >= n2) return;
    if (k == 0) {
        out[0] = make_float2(1.0f, 0.0f);
        return;
    }
    int lo = seg0;
    while (lo + 1 < nseg && sstart[lo + 1] <= k) lo++;
    const float lv = level[slvl[lo]];
    float norm;
    if (sslope[lo] < 0) {
        norm = presto_invsqrtf(lv);
    } else {
        const float sl = sslope[lo] == 0 ? 1.0f : slope[sslope[lo]];
        norm = presto_invsqrtf(__fmaf_rn(sl, (float)(k - sstart[lo]), lv));
    }
    const float2 v = amps[k];
    out[k] = make_float2(__fmul_rn(v.x, norm), __fmul_rn(v.y, norm));
}

}  // namespace sp

struct CsSpectrum {
    int device;
    long long N, n2;
    double dt;
    cufftHandle plan = 0;
    bool planned = false;
    float *d_series = nullptr;     /* staging for the host entry point */
    float2 *d_X = nullptr;         /* R2C output, N/2 + 1 bins */
    float2 *d_pack = nullptr;      /* packed, before normalisation */
    float2 *d_out = nullptr;       /* staging for the host entry point */
    long long *d_bstart = nullptr, *d_sstart = nullptr;
    int *d_blen = nullptr, *d_slvl = nullptr, *d_sslope = nullptr;
    float *d_level = nullptr, *d_slope = nullptr;
    int nblk = 0, nseg = 0;
    cudaStream_t st = nullptr;
};

static void spec_release(CsSpectrum *S)
{
    if (!S) return;
    if (S->planned) cufftDestroy(S->plan);
    cudaFree(S->d_series);
    cudaFree(S->d_X);
    cudaFree(S->d_pack);
    cudaFree(S->d_out);
    cudaFree(S->d_bstart);
    cudaFree(S->d_sstart);
    cudaFree(S->d_blen);
    cudaFree(S->d_slvl);
    cudaFree(S->d_sslope);
    cudaFree(S->d_level);
    cudaFree(S->d_slope);
    if (S->st) cudaStreamDestroy(S->st);
    delete S;
}

/* The rednoise blocks of src/datpipe.c:143-253 for ncomplex bins: a first
 * block of startwidth bins from bin 1, then blocks of
 * (int)(startwidth * ln(binnum)) bins while (float)binnum / (float)T <
 * endfreq, endwidth bins after, the last one cut to what is left.  Returns
 * -1 (with a message) where the reference stops with an error. */
static int rednoise_blocks(long long ncomplex, long long N, double dt, int startwidth,
                           int endwidth, double endfreq, std::vector<long long> &bstart,
                           std::vector<int> &blen)
{
    const float T = (float)((double)N * dt);
    long long binnum = 1, pos = 1;
    int bufflen = startwidth;
    if (ncomplex - 1 < bufflen) {
        fprintf(stderr, "Error: rednoise: too few Fourier bins (%lld)\n", ncomplex);
        return -1;
    }
    bstart.push_back(pos);
    blen.push_back(bufflen);
    pos += bufflen;
    binnum += bufflen;
    bufflen = (int)(startwidth * log((double)binnum));
    for (;;) {
        const long long avail = ncomplex - pos;
        if (avail <= 0) break;
        const int n = avail < bufflen ? (int)avail : bufflen;
        bstart.push_back(pos);
        blen.push_back(n);
        pos += n;
        binnum += n;
        if ((float)binnum / T < endfreq)
            bufflen = (int)(startwidth * log((double)binnum));
        else
            bufflen = endwidth;
        if (bufflen > endwidth) {
            fprintf(stderr, "Error: rednoise block length %d exceeds %d\n", bufflen, endwidth);
            return -1;
        }
    }
    return 0;
}

CS_EXPORT CsSpectrum *cs_spectrum_create(long long N, double dt, int startwidth, int endwidth,
                                         double endfreq, int device)
{
    if (N < 4 || (N & 1) || dt <= 0.0 || startwidth < 1 || endwidth < startwidth ||
        endwidth > sp::MAX_BLOCK) {
        fprintf(stderr, "Error: cs_spectrum_create: need an even N >= 4, dt > 0 and "
                        "1 <= startwidth <= endwidth <= %d\n", sp::MAX_BLOCK);
        return nullptr;
    }
    std::vector<long long> bstart;
    std::vector<int> blen;
    const long long n2 = N / 2;
    if (rednoise_blocks(n2, N, dt, startwidth, endwidth, endfreq, bstart, blen) != 0)
        return nullptr;
    for (int n : blen)
        if (n > sp::MAX_BLOCK) {
            fprintf(stderr, "Error: cs_spectrum_create: a rednoise block of %d bins\n", n);
            return nullptr;
        }
    const int nblk = (int)blen.size();
    /* output segments in bin order (see the file header) */
    std::vector<long long> sstart;
    std::vector<int> slvl, sslope;
    sstart.push_back(1);
    slvl.push_back(0);
    sslope.push_back(-1);
    for (int b = 1; b < nblk; b++) {
        sstart.push_back(bstart[b - 1] + blen[b - 1] / 2);
        slvl.push_back(b - 1);
        sslope.push_back(b);
    }
    sstart.push_back(bstart[nblk - 1] + blen[nblk - 1] / 2);
    slvl.push_back(nblk - 1);
    sslope.push_back(nblk >= 2 ? nblk - 1 : 0);

    CsSpectrum *S = new CsSpectrum();
    S->device = device;
    S->N = N;
    S->n2 = n2;
    S->dt = dt;
    S->nblk = nblk;
    S->nseg = (int)sstart.size();
#define SPCK(x)                                                                        \
    do {                                                                               \
        cudaError_t e_ = (x);                                                          \
        if (e_ != cudaSuccess) {                                                       \
            fprintf(stderr, "Error: cs_spectrum_create: %s: %s\n", #x, cudaGetErrorString(e_)); \
            spec_release(S);                                                           \
            return nullptr;                                                            \
        }                                                                              \
    } while (0)
    SPCK(cudaSetDevice(device));
    SPCK(cudaStreamCreateWithFlags(&S->st, cudaStreamNonBlocking));
    SPCK(cudaMalloc((void **)&S->d_X, sizeof(float2) * (size_t)(n2 + 1)));
    SPCK(cudaMalloc((void **)&S->d_pack, sizeof(float2) * (size_t)n2));
    SPCK(cudaMalloc((void **)&S->d_bstart, sizeof(long long) * nblk));
    SPCK(cudaMalloc((void **)&S->d_blen, sizeof(int) * nblk));
    SPCK(cudaMalloc((void **)&S->d_level, sizeof(float) * nblk));
    SPCK(cudaMalloc((void **)&S->d_slope, sizeof(float) * nblk));
    SPCK(cudaMalloc((void **)&S->d_sstart, sizeof(long long) * S->nseg));
    SPCK(cudaMalloc((void **)&S->d_slvl, sizeof(int) * S->nseg));
    SPCK(cudaMalloc((void **)&S->d_sslope, sizeof(int) * S->nseg));
    SPCK(cudaMemcpyAsync(S->d_bstart, bstart.data(), sizeof(long long) * nblk,
                         cudaMemcpyHostToDevice, S->st));
    SPCK(cudaMemcpyAsync(S->d_blen, blen.data(), sizeof(int) * nblk, cudaMemcpyHostToDevice,
                         S->st));
    SPCK(cudaMemcpyAsync(S->d_sstart, sstart.data(), sizeof(long long) * S->nseg,
                         cudaMemcpyHostToDevice, S->st));
    SPCK(cudaMemcpyAsync(S->d_slvl, slvl.data(), sizeof(int) * S->nseg, cudaMemcpyHostToDevice,
                         S->st));
    SPCK(cudaMemcpyAsync(S->d_sslope, sslope.data(), sizeof(int) * S->nseg,
                         cudaMemcpyHostToDevice, S->st));
    SPCK(cudaStreamSynchronize(S->st));
#undef SPCK
    if (cufftPlan1d(&S->plan, (int)N, CUFFT_R2C, 1) != CUFFT_SUCCESS) {
        fprintf(stderr, "Error: cs_spectrum_create: cuFFT plan for N = %lld failed\n", N);
        spec_release(S);
        return nullptr;
    }
    S->planned = true;
    return S;
}

static cudaError_t spec_enqueue(CsSpectrum *S, const float *d_series, float2 *d_amps,
                                cudaStream_t st)
{
    if (cufftSetStream(S->plan, st) != CUFFT_SUCCESS ||
        cufftExecR2C(S->plan, (cufftReal *)d_series, (cufftComplex *)S->d_X) != CUFFT_SUCCESS)
        return cudaErrorLaunchFailure;
    const long long n2 = S->n2;
    const unsigned g = (unsigned)((n2 + 255) / 256);
    sp::pack_kernel<<<g, 256, 0, st>>>(S->d_X, S->d_pack, n2);
    sp::block_level_kernel<<<(S->nblk + 7) / 8, 256, 0, st>>>(S->d_pack, S->d_bstart, S->d_blen,
                                                               S->nblk, log(2.0), S->d_level);
    sp::slope_kernel<<<(S->nblk + 255) / 256, 256, 0, st>>>(S->d_level, S->d_blen, S->nblk,
                                                           S->d_slope);
    sp::normalise_kernel<<<g, 256, 0, st>>>(S->d_pack, d_amps, n2, S->d_sstart, S->d_slvl,
                                            S->d_sslope, S->nseg, S->d_level, S->d_slope);
    return cudaGetLastError();
}

CS_EXPORT int cs_spectrum_run_device(CsSpectrum *S, const float *d_series, float *d_amps,
                                     void *stream)
{
    if (!S || !d_series || !d_amps) return -1;
    if (cudaSetDevice(S->device) != cudaSuccess) return -1;
    cudaStream_t st = stream ? (cudaStream_t)stream : S->st;
    const cudaError_t e = spec_enqueue(S, d_series, (float2 *)d_amps, st);
    if (e != cudaSuccess) {
        fprintf(stderr, "Error: cs_spectrum_run: %s\n", cudaGetErrorString(e));
        return -1;
    }
    return 0;
}

CS_EXPORT int cs_spectrum_run(CsSpectrum *S, const float *h_series, float *h_amps)
{
    if (!S || !h_series || !h_amps) return -1;
    if (cudaSetDevice(S->device) != cudaSuccess) return -1;
    cudaError_t e = cudaSuccess;
    if (!S->d_series) e = cudaMalloc((void **)&S->d_series, sizeof(float) * (size_t)S->N);
    if (e == cudaSuccess && !S->d_out) e = cudaMalloc((void **)&S->d_out, sizeof(float2) * (size_t)S->n2);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(S->d_series, h_series, sizeof(float) * (size_t)S->N,
                            cudaMemcpyHostToDevice, S->st);
    if (e == cudaSuccess) e = spec_enqueue(S, S->d_series, S->d_out, S->st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(h_amps, S->d_out, sizeof(float2) * (size_t)S->n2,
                            cudaMemcpyDeviceToHost, S->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(S->st);
    if (e != cudaSuccess) {
        fprintf(stderr, "Error: cs_spectrum_run: %s\n", cudaGetErrorString(e));
        return -1;
    }
    return 0;
}

CS_EXPORT void cs_spectrum_free(CsSpectrum *S)
{
    if (!S) return;
    cudaSetDevice(S->device);
    if (S->st) cudaStreamSynchronize(S->st);
    spec_release(S);
}
