/*
 * Duty cycles of candidates on the GPU: the reference's measure_ducy
 * (src/candidate.c:305-329) over a spectrum that is already in device memory.
 *
 * For each candidate (r, nharm) the reference rebuilds an FP64 pulse profile
 * (candidate_profile, src/candidate.c:208-271):
 *   - harmonics h = 1, 2, ... of r while the m-tap window fits the spectrum
 *     and h*r stays below N/2 (the first one that does not fit ends the
 *     stack), each interpolated with the exact m = 64 sinc kernel
 *     (fourier_interp_complex, src/interp.c:317-344);
 *   - an unnormalised c2r of the stack (DC = 0) to n = 2H bins, times 1/n;
 * then keeps the boxcar width with the best matched-filter metric
 * (boxcar_best_width, src/boxcar.c:736-785) and reports width / n.
 *
 * One CTA per candidate: one thread per harmonic runs the 64 taps in the
 * reference's order; one thread per output bin evaluates the c2r directly in
 * FP64 (the host restatement's c2r_direct, the same terms in the same
 * order); one thread per width scans the cyclic prefix sums.  The width
 * ladders and their shape factors depend only on n, so the host builds them
 * once per plan with the search's own boxcar_widths / boxcar_shape.
 *
 * Parity: the output is a choice among a handful of widths.  The device's
 * FP64 sin and cos may differ from the host's in the last place, which moves
 * the profile by about 1e-16 relative; only an exact tie between two widths'
 * metrics could then change the choice.
 */
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "cs_b200.h"

#define CS_EXPORT extern "C" __attribute__((visibility("default")))

namespace dc {

constexpr int M = 64;          /* interpolation taps (measure_ducy's m) */
constexpr int HMAX = 64;       /* harmonics per candidate profile */
constexpr int NBMAX = 2 * HMAX;
constexpr int WCAP = 32;       /* widths per profile length */
constexpr int NTHREADS = 128;
static_assert(NTHREADS >= NBMAX && NTHREADS >= HMAX && NTHREADS >= WCAP, "one thread per item");

struct Cand {
    double r;
    int nharm;
    int pad;
};

struct Tables {
    int nw[NBMAX + 1];              /* by profile length n */
    int w[NBMAX + 1][WCAP];
    double shape[NBMAX + 1][WCAP];
};

/* fourier_interp_complex (src/interp.c:317-344): the same expressions in the
 * same order, FP64. */
static __device__ void interp64(double r, const float2 *amps, long long namps, double *out_re,
                                double *out_im)
{
    constexpr int m2 = M / 2;
    double dr = fmod(r, 1.0);
    if (dr < 0) dr += 1.0;
    const long long first = (long long)floor(r + 1e-15) + 1 - m2;
    double sre = 0.0, sim = 0.0;
    for (int j = 0; j < M; j++) {
        const double off = dr - (double)(-m2 + 1 + j);
        const double sinc = off == 0.0 ? 1.0 : sin(M_PI * off) / (M_PI * off);
        const double c = cos(M_PI * off), s = sin(M_PI * off);
        const double cr = sinc * c, ci = -sinc * s;
        const long long idx = first + j;
        double br = 0.0, bi = 0.0;
        if (idx >= 0 && idx < namps) {
            const float2 a = amps[idx];
            br = (double)a.x;
            bi = (double)a.y;
        }
        sre += cr * br - ci * bi;
        sim += cr * bi + ci * br;
    }
    *out_re = sre;
    *out_im = sim;
}

__global__ void __launch_bounds__(NTHREADS) ducy_kernel(const float2 *amps, long long namps,
                                                        long long N, const Cand *cands, int ncand,
                                                        const Tables *tab, double *ducy)
{
    __shared__ double X[2 * (HMAX + 1)];
    __shared__ double prof[NBMAX];
    __shared__ double ps[NBMAX + NBMAX + 1];
    __shared__ double cand[WCAP];
    __shared__ int fits[HMAX];
    __shared__ int sH;
    const int c = blockIdx.x, t = threadIdx.x;
    if (c >= ncand) return;
    const double r = cands[c].r;
    const int nharm = cands[c].nharm;
    if (!(nharm >= 1 && r > 0.0) || nharm > HMAX) {
        if (t == 0) ducy[c] = NAN;
        return;
    }
    /* 1. the harmonic stack (src/candidate.c:216-228) */
    if (t < 2 * (HMAX + 1)) X[t] = 0.0;
    __syncthreads();
    if (t < nharm) {
        const int h = t + 1;
        const double rh = r * (double)h;
        const long long rint0 = (long long)floor(rh + 1e-15) + 1;
        const int ok = rint0 - M / 2 >= 0 && rint0 + M / 2 <= namps && rh < (double)(N / 2);
        fits[t] = ok;
        if (ok) interp64(rh, amps, namps, &X[2 * h], &X[2 * h + 1]);
    }
    __syncthreads();
    if (t == 0) {
        int H = 0;
        while (H < nharm && fits[H]) H++;       /* the first misfit ends the stack */
        sH = H;
    }
    __syncthreads();
    const int H = sH;
    int n;
    if (H < 1) {
        n = 2;                                   /* a zero profile of two bins */
        if (t < 2) prof[t] = 0.0;
    } else {
        /* 2. c2r to n = 2H bins, times 1/n (X[2H] is the Nyquist term) */
        n = 2 * H;
        if (t < n) {
            double acc = X[0];
            for (int k = 1; k < H; k++) {
                const double a = 2.0 * M_PI * (double)(((long long)t * k) % n) / (double)n;
                acc += 2.0 * (X[2 * k] * cos(a) - X[2 * k + 1] * sin(a));
            }
            acc += (t & 1) ? -X[2 * H] : X[2 * H];
            prof[t] = acc * (1.0 / (double)n);
        }
    }
    __syncthreads();
    /* 3. boxcar_best_width (src/boxcar.c:736-785) */
    const int nw = tab->nw[n];
    if (nw <= 0) {
        if (t == 0) ducy[c] = 1.0 / (double)n;
        return;
    }
    const int wmax = tab->w[n][nw - 1];
    if (t == 0) {
        double sum = 0.0;
        for (int i = 0; i < n; i++) sum += prof[i];
        const double mean = sum / (double)n;
        ps[0] = 0.0;
        for (int i = 1; i <= n + wmax; i++) {
            const int idx = i > n ? i - n : i;
            ps[i] = ps[i - 1] + (prof[idx - 1] - mean);
        }
    }
    __syncthreads();
    if (t < nw) {
        const int w = tab->w[n][t];
        const double duty = (double)w / (double)n;
        const double stot = ps[n] - ps[0];
        double mx = ps[w] - ps[0];
        for (int q = 2; q <= n; q++) {
            const double d = ps[q + w - 1] - ps[q - 1];
            if (d > mx) mx = d;
        }
        cand[t] = (mx - duty * stot) * tab->shape[n][t];
    }
    __syncthreads();
    if (t == 0) {
        double best = -INFINITY;
        int bestw = tab->w[n][0];
        for (int i = 0; i < nw; i++)
            if (cand[i] > best) { best = cand[i]; bestw = tab->w[n][i]; }
        ducy[c] = (double)bestw / (double)n;
    }
}

}  // namespace dc

struct CsDucy {
    int device;
    cudaStream_t st;
    dc::Tables *d_tab;
    dc::Cand *d_cand;
    double *d_ducy;
    int cap;
    dc::Cand *h_cand;      /* pinned */
    double *h_ducy;        /* pinned */
};

static void ducy_release(CsDucy *D)
{
    if (!D) return;
    cudaFree(D->d_tab);
    cudaFree(D->d_cand);
    cudaFree(D->d_ducy);
    if (D->h_cand) cudaFreeHost(D->h_cand);
    if (D->h_ducy) cudaFreeHost(D->h_ducy);
    if (D->st) cudaStreamDestroy(D->st);
    free(D);
}

CS_EXPORT CsDucy *cs_ducy_create(double fsp, double maxfrac, int device)
{
    if (cudaSetDevice(device) != cudaSuccess) return nullptr;
    CsDucy *D = (CsDucy *)calloc(1, sizeof(CsDucy));
    if (!D) return nullptr;
    D->device = device;
    dc::Tables *tab = (dc::Tables *)calloc(1, sizeof(dc::Tables));
    if (!tab) { free(D); return nullptr; }
    /* the ladder and all-filled shapes of every profile length
     * (boxcar_best_width, src/boxcar.c:741-760) */
    for (int n = 2; n <= dc::NBMAX; n += 2) {
        int widths[256];
        int nw = boxcar_widths(n, fsp, maxfrac, widths, 256);
        if (nw > dc::WCAP) {
            fprintf(stderr, "Error: cs_ducy_create: %d widths at %d bins\n", nw, n);
            free(tab);
            free(D);
            return nullptr;
        }
        if (nw < 0) nw = 0;
        tab->nw[n] = nw;
        if (nw > 0) {
            const int Hk = n / 2;
            std::vector<uint8_t> filled((size_t)Hk, 1);
            double shape[dc::WCAP];
            boxcar_shape(shape, n, widths, nw, filled.data(), 1, Hk);
            for (int i = 0; i < nw; i++) {
                tab->w[n][i] = widths[i];
                tab->shape[n][i] = shape[i];
            }
        }
    }
    cudaError_t e = cudaStreamCreateWithFlags(&D->st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc((void **)&D->d_tab, sizeof(dc::Tables));
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(D->d_tab, tab, sizeof(dc::Tables), cudaMemcpyHostToDevice, D->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(D->st);
    free(tab);
    if (e != cudaSuccess) {
        fprintf(stderr, "Error: cs_ducy_create: %s\n", cudaGetErrorString(e));
        ducy_release(D);
        return nullptr;
    }
    return D;
}

static cudaError_t ducy_reserve(CsDucy *D, int n)
{
    if (n <= D->cap) return cudaSuccess;
    const int cap = n + n / 2 + 64;
    cudaFree(D->d_cand);
    cudaFree(D->d_ducy);
    if (D->h_cand) cudaFreeHost(D->h_cand);
    if (D->h_ducy) cudaFreeHost(D->h_ducy);
    D->d_cand = nullptr; D->d_ducy = nullptr; D->h_cand = nullptr; D->h_ducy = nullptr;
    D->cap = 0;
    cudaError_t e = cudaMalloc((void **)&D->d_cand, sizeof(dc::Cand) * (size_t)cap);
    if (e == cudaSuccess) e = cudaMalloc((void **)&D->d_ducy, sizeof(double) * (size_t)cap);
    if (e == cudaSuccess) e = cudaMallocHost((void **)&D->h_cand, sizeof(dc::Cand) * (size_t)cap);
    if (e == cudaSuccess) e = cudaMallocHost((void **)&D->h_ducy, sizeof(double) * (size_t)cap);
    if (e == cudaSuccess) D->cap = cap;
    return e;
}

CS_EXPORT int cs_ducy_run_device(CsDucy *D, const float *d_amps, long long namps, long long N,
                                 const Candidate *cands, long long ncand, double *ducy_out,
                                 void *stream)
{
    if (!D || (ncand > 0 && (!d_amps || !cands || !ducy_out)) || ncand < 0 ||
        ncand > 0x7fffffffLL)
        return -1;
    if (ncand == 0) return 0;
    if (cudaSetDevice(D->device) != cudaSuccess) return -1;
    cudaStream_t st = stream ? (cudaStream_t)stream : D->st;
    cudaError_t e = ducy_reserve(D, (int)ncand);
    if (e == cudaSuccess) {
        for (long long i = 0; i < ncand; i++) {
            D->h_cand[i].r = cands[i].r;
            D->h_cand[i].nharm = cands[i].nharm;
            D->h_cand[i].pad = 0;
        }
        e = cudaMemcpyAsync(D->d_cand, D->h_cand, sizeof(dc::Cand) * (size_t)ncand,
                            cudaMemcpyHostToDevice, st);
    }
    if (e == cudaSuccess) {
        dc::ducy_kernel<<<(unsigned)ncand, dc::NTHREADS, 0, st>>>(
            (const float2 *)d_amps, namps, N, D->d_cand, (int)ncand, D->d_tab, D->d_ducy);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(D->h_ducy, D->d_ducy, sizeof(double) * (size_t)ncand,
                            cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        fprintf(stderr, "Error: cs_ducy_run: %s\n", cudaGetErrorString(e));
        return -1;
    }
    memcpy(ducy_out, D->h_ducy, sizeof(double) * (size_t)ncand);
    return 0;
}

CS_EXPORT void cs_ducy_free(CsDucy *D)
{
    if (!D) return;
    cudaSetDevice(D->device);
    if (D->st) cudaStreamSynchronize(D->st);
    ducy_release(D);
}
