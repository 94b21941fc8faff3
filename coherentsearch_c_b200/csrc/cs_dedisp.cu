/*
 * Subband dedispersion of 8-bit filterbank data on the B200 -- the
 * prepsubband stage of the reference's raw-data front end
 * (src/prep_dedisp.c:444-466, 1104-1275 over PRESTO's dispersion.c:
 * dedisp_subbands :218-267 and float_dedisp :322-365).
 *
 * In absolute time, with X_c the channel series in ascending frequency
 * (SIGPROC order reversed, third_party/presto/src/sigproc_fb.c:656-664):
 *
 *   S_s[T]   = sum_{c in subband s} X_c[T + idispdt[c]]       (subband stage)
 *   out_d[T] = -0.0f + sum_{s < nsub} S_s[T + offsets[d][s]]  (DM stage)
 *
 * The reference evaluates both in FP32, adding channels and subbands in
 * ascending order.  With 8-bit input every partial sum is an integer below
 * 2^24 (nchan * 255 < 2^24 is checked), so each FP32 addition is exact and
 * integer sums give the identical bits.  S is held as uint16 (cps * 255 <
 * 2^16 is checked), which halves its HBM and shared-memory traffic.
 *
 * Block semantics of the reference driver (spectra_per_subint = L, blocks
 * per read = bpr, worklen W = bpr * L): only whole raw blocks are read
 * (sigproc_fb.c:549-620); subband block b needs raw block b+1; output chunk
 * k needs subband chunk k+1 complete; output stops at the first incomplete
 * chunk or at numout points (prep_dedisp.c:484-522).  With nb raw blocks
 * the output holds min(numout, (floor((nb-1)/bpr) - 1) * W) points and every
 * one of them follows the formula above.
 *
 * Kernels (HBM layout: raw [nspec][nchan] u8 as read; S [nsub][sstride] u16;
 * out [ndm][out_stride] f32):
 *   dd_subband_u8  one CTA per (slab of subbands, 256-sample tile): the
 *                  tile's raw rows plus the delay halo are copied
 *                  asynchronously into shared memory with padded rows (an
 *                  odd number of words: lanes over consecutive samples hit
 *                  consecutive banks), then each warp sums the channels of
 *                  one subband for 32 samples.  HBM-bound: 1 B read per
 *                  channel-sample, 2 B written per subband-sample.
 *   dd_dms_u16     one CTA per (group of up to 32 DMs, 256-sample tile): the
 *                  S windows the group needs (tile + the group's offset
 *                  spread) are staged in shared memory once, with a copy
 *                  shifted by one sample for odd offsets, and serve all the
 *                  group's DMs.  Each thread sums the subbands for 4 sample
 *                  pairs of 4 DMs with packed 16-bit adds (two samples per
 *                  32-bit add, widened before they can carry); lanes read
 *                  consecutive words.  Shared-memory-bound: 2 B of shared
 *                  reads per subband term.
 *   dd_dms_u16_direct  the same sums straight from L1/L2, for geometries
 *                  whose windows do not fit in shared memory.
 *
 * A run with prepsubband's -clip that replaces spectra (cs_clip_levels) has
 * non-integer channel levels in it, so its sums need FP32 in the reference's
 * order; S is float there:
 *   dd_subband_clip  dd_subband_u8's staging plus one clip flag per row;
 *                  channels added in ascending frequency from 0.0f, a
 *                  flagged spectrum contributing its block's level.
 *   dd_dms_f32     one CTA per (1024 samples, 16 DMs); per round of four
 *                  subbands the union windows are copied into shared memory
 *                  with cp.async a round ahead of the sums; subbands added in
 *                  ascending order from -0.0f.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "cs_b200.h"

#define CS_EXPORT extern "C" __attribute__((visibility("default")))

namespace dd {

/* tile shapes (compile-time; DD_* override them for tuning builds) */
#ifndef DD_DM_TT
#define DD_DM_TT 256
#endif
#ifndef DD_DM_GD
#define DD_DM_GD 4
#endif
#ifndef DD_SB_TT
#define DD_SB_TT 256
#endif
constexpr int SB_TT = DD_SB_TT;   /* samples per subband tile */
constexpr int SB_THREADS = 512;
constexpr int DM_TT = DD_DM_TT;   /* samples per DM tile */
constexpr int DM_G = 32;          /* most DMs per group (one CTA) */
constexpr int DM_R = 8;           /* samples (4 pairs) per thread */
constexpr int DM_GD = DD_DM_GD;   /* DMs per thread */
constexpr int DM_THREADS = (DM_TT / DM_R) * (DM_G / DM_GD);
static_assert(DM_THREADS <= 1024 && DM_G % DM_GD == 0, "DM tile shape");

static __device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

/* Asynchronous global -> shared copies (no register round trip, so all of
 * a thread's copies are in flight together); nbytes 0 writes zeros. */
static __device__ __forceinline__ void cp_async4(void *dst, const void *src, int nbytes)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(smem_addr(dst)), "l"(src),
                 "r"(nbytes)
                 : "memory");
}

static __device__ __forceinline__ void cp_async16(void *dst, const void *src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src)
                 : "memory");
}

static __device__ __forceinline__ void cp_async_wait_all()
{
    asm volatile("cp.async.wait_all;" ::: "memory");
}

/* ---------------------------------------------------------------- */
/* Subband stage                                                     */
/* ---------------------------------------------------------------- */
struct SubArgs {
    const uint8_t *raw;
    long long nspec;          /* spectra in raw */
    int nchan, cps, nsub;
    int slab;                 /* subbands per CTA */
    int halo;                 /* max channel delay */
    int rowstride;            /* shared bytes per staged row (multiple of 4) */
    int table_off;            /* shared byte offset of the channel table (16-aligned) */
    const int *idisp;         /* [nchan], ascending frequency */
    long long nvalid;         /* samples with data: (nb - 1) * L */
    long long sfill;          /* samples written per subband */
    uint16_t *sub;
    long long sstride;
    /* clipped runs (dd_subband_clip) */
    const uint8_t *flags;     /* [nflags] 1: spectrum replaced */
    long long nflags;
    const float *levels;      /* [nspec / L][nchan] channel levels, SIGPROC order */
    int L;
    int flag_off;             /* shared byte offset of the staged row flags */
    float *subf;              /* S as float */
};

/* Stage the CTA's raw rows [T0, T0 + SB_TT + halo) of its slab's channel
 * columns in shared memory (padded rows), and the per-channel offsets of the
 * delayed samples (coff).  Ends with a barrier. */
static __device__ __forceinline__ void sb_stage(const SubArgs &a, unsigned char *sm, int s0,
                                                int sc, long long T0)
{
    const int c0 = s0 * a.cps;                            /* first channel */
    const int rows = SB_TT + a.halo;
    /* raw columns [col0, col0 + sc) hold channels c0 + sc - 1 .. c0 */
    const int col0 = a.nchan - c0 - sc;
    /* per staged channel: byte offset of its delayed sample from a row start */
    int *coff = reinterpret_cast<int *>(sm + a.table_off);
    for (int i = threadIdx.x; i < sc; i += blockDim.x)
        coff[i] = a.idisp[c0 + i] * a.rowstride + (sc - 1 - i);

    const bool w4 = ((col0 | sc | a.nchan | (int)((uintptr_t)a.raw & 3)) & 3) == 0;
    if (w4) {
        /* thread -> (row phase, word): a fixed word column, rows step by
         * the number of rows one pass covers */
        const int wpr = sc >> 2;                          /* words per row (<= 65) */
        const int rpp = blockDim.x / wpr;                 /* rows per pass */
        const int w = threadIdx.x % wpr;
        if (threadIdx.x < rpp * wpr) {
            const unsigned char *src = a.raw + T0 * a.nchan + col0 + 4 * w;
            unsigned char *dst = sm + 4 * w;
            for (int r = threadIdx.x / wpr; r < rows; r += rpp) {
                const bool in = T0 + r < a.nspec;
                cp_async4(dst + (size_t)r * a.rowstride, in ? src + (long long)r * a.nchan : a.raw,
                          in ? 4 : 0);
            }
        }
        cp_async_wait_all();
    } else {
        for (int i = threadIdx.x; i < rows * sc; i += blockDim.x) {
            const int r = i / sc, b = i - r * sc;
            const long long T = T0 + r;
            sm[(size_t)r * a.rowstride + b] = T < a.nspec ? __ldg(a.raw + T * a.nchan + col0 + b) : 0;
        }
    }
    __syncthreads();
}

__global__ void __launch_bounds__(SB_THREADS) dd_subband_u8(const SubArgs a)
{
    extern __shared__ __align__(16) unsigned char sm[];
    const int s0 = blockIdx.x * a.slab;                   /* first subband */
    const int nslab = min(a.slab, a.nsub - s0);
    const int sc = nslab * a.cps;                         /* channels staged */
    const long long T0 = (long long)blockIdx.y * SB_TT;
    sb_stage(a, sm, s0, sc, T0);
    const int *coff = reinterpret_cast<const int *>(sm + a.table_off);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nwarps = blockDim.x >> 5;
    /* work items: (subband in slab, 32-sample group) */
    const int ngroups = SB_TT / 32;
    for (int item = warp; item < nslab * ngroups; item += nwarps) {
        const int sl = item / ngroups, g = item - sl * ngroups;
        const int t = g * 32 + lane;
        const long long T = T0 + t;
        if (T >= a.sfill) continue;
        uint32_t acc = 0;
        if (T < a.nvalid) {
            const unsigned char *base = sm + (size_t)t * a.rowstride;
            const int *co = coff + sl * a.cps;
#pragma unroll 8
            for (int k = 0; k < a.cps; k++) acc += base[co[k]];
        }
        a.sub[(long long)(s0 + sl) * a.sstride + T] = (uint16_t)acc;
    }
}

/* The subband stage of a clipped run: spectra flagged by the clip decisions
 * take their block's channel levels (floats), so the sums are evaluated as
 * the reference does (dispersion.c:245-264): in FP32, from 0.0f, adding the
 * channels in ascending frequency.  S is float here. */
__global__ void __launch_bounds__(SB_THREADS) dd_subband_clip(const SubArgs a)
{
    extern __shared__ __align__(16) unsigned char sm[];
    const int s0 = blockIdx.x * a.slab;
    const int nslab = min(a.slab, a.nsub - s0);
    const int sc = nslab * a.cps;
    const long long T0 = (long long)blockIdx.y * SB_TT;
    const int rows = SB_TT + a.halo;
    unsigned char *rflag = sm + a.flag_off;              /* clip flag of each staged row */
    for (int r = threadIdx.x; r < rows; r += blockDim.x)
        rflag[r] = T0 + r < a.nflags ? a.flags[T0 + r] : 0;
    sb_stage(a, sm, s0, sc, T0);
    const int *coff = reinterpret_cast<const int *>(sm + a.table_off);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nwarps = blockDim.x >> 5;
    const int ngroups = SB_TT / 32;
    for (int item = warp; item < nslab * ngroups; item += nwarps) {
        const int sl = item / ngroups, g = item - sl * ngroups;
        const int t = g * 32 + lane;
        const long long T = T0 + t;
        if (T >= a.sfill) continue;
        float acc = 0.0f;
        if (T < a.nvalid) {
            const unsigned char *base = sm + (size_t)t * a.rowstride;
            const int cfirst = (s0 + sl) * a.cps;
            const int *co = coff + sl * a.cps;
            for (int k = 0; k < a.cps; k++) {
                const int c = cfirst + k;
                const int r = t + __ldg(a.idisp + c);
                float x;
                if (rflag[r]) {
                    const long long u = T0 + r;
                    x = __ldg(a.levels + (u / a.L) * a.nchan + (a.nchan - 1 - c));
                } else {
                    x = (float)base[co[k]];
                }
                acc = __fadd_rn(acc, x);
            }
        }
        a.subf[(long long)(s0 + sl) * a.sstride + T] = acc;
    }
}

/* ---------------------------------------------------------------- */
/* DM stage                                                          */
/* ---------------------------------------------------------------- */
struct DmArgs {
    const uint16_t *sub;
    long long sstride;
    int nsub, ndm;
    int G;                    /* DMs per group (<= DM_G) */
    const int *offs;          /* [ndm][nsub] (direct kernel) */
    int flush;                /* subbands per packed-accumulator flush */
    int flush8;               /* flush rounded down to 8 when nsub % 8 == 0, else 0 */
    const long long *chunk;   /* [ngroups][maxch]: S element offset (from T0) of each staged
                                 16-byte chunk */
    const int *nch;           /* [ngroups]: chunks staged */
    int maxch;
    const int *code;          /* [ngroups][G][nsub]: shared word of the window pair
                                 (the shifted copy at +smem_words for odd offsets) */
    int smem_words;           /* staged words per CTA (largest group) */
    long long nout;
    float *out;
    long long ostride;
};

__global__ void __launch_bounds__(DM_THREADS) dd_dms_u16(const DmArgs a)
{
    /* shared: staged words [0, W) | the same rows shifted by one sample
     * [W, 2W): word w there holds samples (2w+1, 2w+2) | (DM, subband) codes */
    extern __shared__ __align__(16) uint32_t smw[];
    const int g = blockIdx.x;                              /* DM group */
    const long long T0 = (long long)blockIdx.y * DM_TT;
    const int W = a.smem_words;
    const int *code = a.code + (size_t)g * a.G * a.nsub;
    int *code_s = reinterpret_cast<int *>(smw + 2 * W);

    for (int i = threadIdx.x; i < a.G * a.nsub; i += blockDim.x) code_s[i] = code[i];
    /* stage the group's windows (subband after subband, each from a multiple
     * of 8 samples): 16-byte chunk i of shared memory comes from
     * S + T0 + chunk[i] */
    const long long *chunk = a.chunk + (size_t)g * a.maxch;
    const int nch = a.nch[g];
    const uint16_t *sub0 = a.sub + T0;
    for (int i = threadIdx.x; i < nch; i += blockDim.x) cp_async16(smw + 4 * i, sub0 + chunk[i]);
    cp_async_wait_all();
    __syncthreads();
    /* the copy shifted by one sample (pairs straddling two windows are never read) */
    for (int i = threadIdx.x; i + 1 < 4 * nch; i += blockDim.x)
        smw[W + i] = __byte_perm(smw[i], smw[i + 1], 0x5432);
    __syncthreads();

    /* thread: sample pairs (2 tt + 2 (DM_TT / DM_R) j, +1), j < 4, of DM_GD
     * DMs; a warp's lanes read consecutive words, so loads are conflict-free */
    constexpr int NP = DM_R / 2;                           /* pairs per thread */
    constexpr int PS = DM_TT / DM_R;                       /* pair stride */
    const int tt = threadIdx.x % PS;
    const int dq = threadIdx.x / PS;
    const uint32_t *wt = smw + tt;
    for (int dd = 0; dd < DM_GD; dd++) {
        const int dl = dq + (DM_G / DM_GD) * dd;           /* DM within group */
        const int d = g * a.G + dl;
        if (dl >= a.G || d >= a.ndm) break;
        uint32_t acc[DM_R];
#pragma unroll
        for (int r = 0; r < DM_R; r++) acc[r] = 0;
        const int *cd = code_s + dl * a.nsub;
        if (a.flush8 > 0) {
            /* 8 subbands per step: two vector loads of codes, then 32
             * independent shared loads */
            for (int sb = 0; sb < a.nsub; sb += a.flush8) {
                uint32_t p[NP];
#pragma unroll
                for (int k = 0; k < NP; k++) p[k] = 0;
                const int se = min(sb + a.flush8, a.nsub);
                for (int s = sb; s < se; s += 8) {
                    const int4 ca = *reinterpret_cast<const int4 *>(cd + s);
                    const int4 cb = *reinterpret_cast<const int4 *>(cd + s + 4);
                    const int cc[8] = {ca.x, ca.y, ca.z, ca.w, cb.x, cb.y, cb.z, cb.w};
#pragma unroll
                    for (int u = 0; u < 8; u++)
#pragma unroll
                        for (int k = 0; k < NP; k++) p[k] += wt[cc[u] + k * PS];
                }
#pragma unroll
                for (int k = 0; k < NP; k++) {
                    acc[2 * k] += p[k] & 0xffffu;
                    acc[2 * k + 1] += p[k] >> 16;
                }
            }
        } else {
            for (int sb = 0; sb < a.nsub; sb += a.flush) {
                uint32_t p[NP];
#pragma unroll
                for (int k = 0; k < NP; k++) p[k] = 0;
                const int se = min(sb + a.flush, a.nsub);
                for (int s = sb; s < se; s++) {
                    const int c = cd[s];
#pragma unroll
                    for (int k = 0; k < NP; k++) p[k] += wt[c + k * PS];
                }
#pragma unroll
                for (int k = 0; k < NP; k++) {
                    acc[2 * k] += p[k] & 0xffffu;
                    acc[2 * k + 1] += p[k] >> 16;
                }
            }
        }
        float *o = a.out + (long long)d * a.ostride + T0 + 2 * tt;
#pragma unroll
        for (int k = 0; k < NP; k++) {
            const long long T = T0 + 2 * tt + 2 * PS * k;
            float *ok = o + 2 * PS * k;
            if (T + 2 <= a.nout) {
                *reinterpret_cast<float2 *>(ok) = make_float2((float)acc[2 * k], (float)acc[2 * k + 1]);
            } else if (T < a.nout) {
                ok[0] = (float)acc[2 * k];
            }
        }
    }
}

/* Any geometry: one thread per (DM, sample), S read through L1/L2.  Used
 * when even a single DM's windows do not fit in shared memory. */
__global__ void __launch_bounds__(256) dd_dms_u16_direct(const DmArgs a)
{
    const long long T = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int d = blockIdx.y;
    if (T >= a.nout) return;
    const int *off = a.offs + (size_t)d * a.nsub;
    uint32_t acc = 0;
    for (int s = 0; s < a.nsub; s++) acc += __ldg(a.sub + (long long)s * a.sstride + T + off[s]);
    a.out[(long long)d * a.ostride + T] = (float)acc;
}

/* The DM stage of a clipped run: S is float, summed as float_dedisp does
 * (dispersion.c:322-365): from -approx_mean = -0.0f, adding the subbands in
 * ascending order in FP32.  One CTA per (tile of FT samples, group of up to
 * FG consecutive DMs), the group index fastest over the grid.  The group's
 * offsets are staged once; then per round of fr subbands the CTA copies, for
 * each, the union of its DMs' windows (fwin[group][s] = lowest offset, width)
 * into shared memory with asynchronous copies, one round ahead of the sums
 * (two buffers).  Each thread adds a subband's term to the FG sums of its FS
 * samples (t, t + 256, ...), so one broadcast read of a DM's offset serves FS
 * sums.  S is filled up to sfill samples (every output below nout reads below
 * it); staged samples from sfill on are zeros and only reach outputs that are
 * not written. */
constexpr int FG = 16;          /* DMs per CTA */
constexpr int FS = 4;           /* samples per thread */
constexpr int FT = 256 * FS;    /* samples per CTA */
constexpr int FR = 4;           /* most subbands per round */
constexpr int FMAXSUB = 256;    /* most subbands (staged offsets) */
/* Three CTAs of 256 threads per SM leave 85 registers a thread (80 after
 * allocation granularity); FG x FS sums take 64 of them.  ptxas reports 80
 * registers with 124 bytes of spill stores at FG 16, FS 4: any larger product
 * would spill the sums themselves, so it needs the two-CTA bound instead. */
static_assert(FG * FS <= 64, "dd_dms_f32: the sums must fit the three-CTA register budget");

static __device__ __forceinline__ void cp_async_commit()
{
    asm volatile("cp.async.commit_group;" ::: "memory");
}

static __device__ __forceinline__ void cp_async_wait_one()
{
    asm volatile("cp.async.wait_group 1;" ::: "memory");
}

__global__ void __launch_bounds__(256, 3) dd_dms_f32(const float *subf, long long sstride, int nsub,
                                                  int ndm, const int *offs, const int2 *fwin,
                                                  int wmax, int fr, long long sfill,
                                                  long long nout, float *out, long long ostride)
{
    extern __shared__ __align__(16) unsigned char fsm[];
    int *soff = reinterpret_cast<int *>(fsm);                  /* [nsub][FG], from the window */
    float *win = reinterpret_cast<float *>(fsm + sizeof(int) * FMAXSUB * FG);  /* [2][fr][wmax] */
    const unsigned ngrp = (unsigned)((ndm + FG - 1) / FG);
    const int grp = (int)(blockIdx.x % ngrp);
    const int d0 = grp * FG;
    const int nd = min(FG, ndm - d0);
    const long long T0 = (long long)(blockIdx.x / ngrp) * FT;
    const int t = threadIdx.x;
    const int2 *fw = fwin + (size_t)grp * nsub;
    for (int i = t; i < nsub * FG; i += blockDim.x) {
        const int sb = i / FG, j = i - sb * FG;
        soff[i] = j < nd ? offs[(size_t)(d0 + j) * nsub + sb] - fw[sb].x : 0;
    }
    /* round r: subbands r*fr .. ; its windows go to buffer r & 1 */
    auto stage = [&](int r) {
        float *buf = win + (size_t)(r & 1) * fr * wmax;
        const int s0 = r * fr, nr = min(fr, nsub - s0);
        for (int q = 0; q < nr; q++) {
            const int2 w = fw[s0 + q];
            const long long first = T0 + w.x;
            const float *src = subf + (long long)(s0 + q) * sstride + first;
            for (int i = t; i < w.y; i += blockDim.x) {
                const bool in = first + i < sfill;
                cp_async4(buf + q * wmax + i, in ? src + i : subf, in ? 4 : 0);
            }
        }
        cp_async_commit();
    };
    float acc[FG][FS];
#pragma unroll
    for (int j = 0; j < FG; j++)
#pragma unroll
        for (int k = 0; k < FS; k++) acc[j][k] = -0.0f;
    const int nround = (nsub + fr - 1) / fr;
    stage(0);
    for (int r = 0; r < nround; r++) {
        if (r + 1 < nround) {
            stage(r + 1);
            cp_async_wait_one();                      /* round r has landed */
        } else {
            cp_async_wait_all();
        }
        __syncthreads();
        const float *buf = win + (size_t)(r & 1) * fr * wmax;
        const int s0 = r * fr, nr = min(fr, nsub - s0);
        for (int q = 0; q < nr; q++) {
            const float *row = buf + q * wmax + t;
            const int *so = soff + (s0 + q) * FG;
#pragma unroll
            for (int j = 0; j < FG; j++) {
                if (j >= nd) break;
                const float *rr = row + so[j];
#pragma unroll
                for (int k = 0; k < FS; k++) acc[j][k] = __fadd_rn(acc[j][k], rr[256 * k]);
            }
        }
        __syncthreads();                              /* buffer r & 1 is free for round r + 2 */
    }
#pragma unroll
    for (int k = 0; k < FS; k++) {
        const long long T = T0 + t + 256 * k;
        if (T >= nout) break;
#pragma unroll
        for (int j = 0; j < FG; j++)
            if (j < nd) out[(long long)(d0 + j) * ostride + T] = acc[j][k];
    }
}

}  // namespace dd

/* ---------------------------------------------------------------- */
/* Host side                                                         */
/* ---------------------------------------------------------------- */
struct CsDedisp {
    int device;
    int nchan, nsub, ndm, cps, L, bpr;
    long long max_spectra;
    int halo, maxoff;
    int flush;
    int G;                         /* DMs per staged group; 0: direct kernel */
    int ngroups;
    int smem_words;
    int maxch = 0;
    int *d_idisp = nullptr;
    int *d_offs = nullptr;
    int *d_code = nullptr, *d_nch = nullptr;
    long long *d_chunk = nullptr;
    uint16_t *d_sub = nullptr;
    float *d_subf = nullptr;       /* S of clipped runs (allocated by the first one) */
    int2 *d_fwin = nullptr;        /* clipped DM stage: per (DM group, subband) window */
    int fwmax = 0;                 /* widest such window (floats) */
    long long sstride = 0;
    uint8_t *d_raw = nullptr;      /* staging for the host-memory entry point */
    float *d_out = nullptr;
    long long out_cap = 0;
    cudaStream_t st = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr;
};

static void dd_release(CsDedisp *D)
{
    if (!D) return;
    cudaFree(D->d_idisp);
    cudaFree(D->d_offs);
    cudaFree(D->d_code);
    cudaFree(D->d_nch);
    cudaFree(D->d_chunk);
    cudaFree(D->d_sub);
    cudaFree(D->d_subf);
    cudaFree(D->d_fwin);
    cudaFree(D->d_raw);
    cudaFree(D->d_out);
    if (D->st) cudaStreamDestroy(D->st);
    if (D->ev0) cudaEventDestroy(D->ev0);
    if (D->ev1) cudaEventDestroy(D->ev1);
    if (D->ev2) cudaEventDestroy(D->ev2);
    delete D;
}

/* PRESTO's delay for a DM at an emitted frequency (MHz), dispersion.c:41-49 */
static double dd_delay_from_dm(double dm, double f)
{
    return f == 0.0 ? 0.0 : dm / (0.000241 * f * f);
}

/* (long)(x < 0 ? ceil(x - 0.5) : floor(x + 0.5)), src/prep_dedisp.c:37 */
static long dd_nearest(double x)
{
    return (long)(x < 0 ? ceil(x - 0.5) : floor(x + 0.5));
}

/* Per-channel delays (subband_search_delays, dispersion.c:164-194, then
 * NEAREST_LONG(delay / dt), prep_dedisp.c:448-452) and per-DM subband
 * offsets (subband_delays :135-152 relative to the highest subband, then
 * NEAREST_LONG(. / dsdt), :456-466), for DMs lodm + i*dmstep whose mean is
 * the subbanding DM (:318-331); blocks per read as :362-367.  FP64 with the
 * reference's operation order; the -Ofast build of the reference may differ
 * only on exact .5 ties of the rounded quotients. */
CS_EXPORT int cs_dedisp_tables(int nchan, int nsub, int ndm, double lodm, double dmstep,
                               double lofreq, double chanwid, double dt,
                               int spectra_per_subint, int *idispdt, int *offsets,
                               int *blocks_per_read, double *avgdm_out)
{
    if (nchan <= 0 || nsub <= 0 || ndm <= 0 || nchan % nsub || dt <= 0.0 ||
        spectra_per_subint <= 0 || !idispdt || !offsets)
        return -1;
    std::vector<double> dms(ndm);
    double avgdm = 0.0;
    for (int i = 0; i < ndm; i++) {
        dms[i] = lodm + i * dmstep;
        avgdm += dms[i];
    }
    avgdm /= ndm;
    const double maxdm = dms[ndm - 1];
    const double bw = dd_delay_from_dm(maxdm, lofreq) -
                      dd_delay_from_dm(maxdm, lofreq + (nchan - 1) * chanwid);
    if (blocks_per_read) *blocks_per_read = (int)(bw / dt) / spectra_per_subint + 1;
    const int cps = nchan / nsub;
    const double subbw = chanwid * cps;
    const double losub_hi = lofreq + subbw - chanwid;
    std::vector<double> subd(nsub);
    for (int s = 0; s < nsub; s++) subd[s] = dd_delay_from_dm(avgdm, losub_hi + s * subbw);
    for (int c = 0; c < nchan; c++) {
        const double d = dd_delay_from_dm(avgdm, lofreq + c * chanwid) - subd[c / cps];
        idispdt[c] = (int)dd_nearest(d / dt);
    }
    for (int i = 0; i < ndm; i++) {
        for (int s = 0; s < nsub; s++) subd[s] = dd_delay_from_dm(dms[i], losub_hi + s * subbw);
        const double top = subd[nsub - 1];
        for (int s = 0; s < nsub; s++) offsets[(size_t)i * nsub + s] = (int)dd_nearest((subd[s] - top) / dt);
    }
    if (avgdm_out) *avgdm_out = avgdm;
    return 0;
}

CS_EXPORT long long cs_dedisp_output_length(const CsDedisp *D, long long nspec, long long numout)
{
    if (!D || nspec < 0) return -1;
    const long long nb = nspec / D->L;
    long long k = nb >= 1 ? (nb - 1) / D->bpr - 1 : -1;
    if (k < 0) k = 0;
    long long n = k * (long long)D->L * D->bpr;
    if (numout >= 0 && n > numout) n = numout;
    return n;
}

/* Shared bytes per staged raw row: the slab's channels rounded up to a
 * word, plus one word, so that consecutive rows start in consecutive banks
 * when the slab is a multiple of 8 words. */
static int sb_rowstride(const CsDedisp *D, int slab)
{
    return (slab * D->cps + 3) / 4 * 4 + 4;
}

static int sb_table_offset(const CsDedisp *D, int slab)
{
    return ((dd::SB_TT + D->halo) * sb_rowstride(D, slab) + 15) / 16 * 16;
}

static int sb_flag_offset(const CsDedisp *D, int slab)
{
    return sb_table_offset(D, slab) + slab * D->cps * 4;
}

/* the clipped kernel also stages one flag byte per row */
static int sb_smem(const CsDedisp *D, int slab, bool clip = false)
{
    return sb_flag_offset(D, slab) + (clip ? dd::SB_TT + D->halo : 0);
}

CS_EXPORT CsDedisp *cs_dedisp_create(int nchan, int nsub, int ndm, const int *idispdt,
                                     const int *offsets, int spectra_per_subint,
                                     int blocks_per_read, long long max_spectra, int device)
{
    if (nchan <= 0 || nsub <= 0 || ndm <= 0 || nchan % nsub || !idispdt || !offsets ||
        spectra_per_subint <= 0 || blocks_per_read <= 0 || max_spectra <= 0) {
        fprintf(stderr, "Error: cs_dedisp_create: invalid geometry\n");
        return nullptr;
    }
    const int cps = nchan / nsub;
    if ((long long)nchan * 255 >= (1LL << 24) || cps * 255 > 65535) {
        fprintf(stderr, "Error: cs_dedisp_create: %d channels (%d per subband) exceed the "
                        "exact 8-bit sums (nchan*255 < 2^24, per subband < 2^16)\n", nchan, cps);
        return nullptr;
    }
    int halo = 0, maxoff = 0;
    for (int c = 0; c < nchan; c++) {
        if (idispdt[c] < 0 || idispdt[c] > spectra_per_subint) {
            fprintf(stderr, "Error: cs_dedisp_create: channel delay %d outside [0, %d]\n",
                    idispdt[c], spectra_per_subint);
            return nullptr;
        }
        halo = std::max(halo, idispdt[c]);
    }
    const long long Wk = (long long)spectra_per_subint * blocks_per_read;
    for (long long i = 0; i < (long long)ndm * nsub; i++) {
        if (offsets[i] < 0 || offsets[i] > Wk) {
            fprintf(stderr, "Error: cs_dedisp_create: subband offset %d outside [0, %lld]\n",
                    offsets[i], Wk);
            return nullptr;
        }
        maxoff = std::max(maxoff, offsets[i]);
    }
    CsDedisp *D = new CsDedisp();
    D->device = device;
    D->nchan = nchan;
    D->nsub = nsub;
    D->ndm = ndm;
    D->cps = cps;
    D->L = spectra_per_subint;
    D->bpr = blocks_per_read;
    D->max_spectra = max_spectra;
    D->halo = halo;
    D->maxoff = maxoff;
    D->flush = std::max(1, 65535 / (cps * 255));
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        fprintf(stderr, "Error: cs_dedisp_create: %s\n", cudaGetErrorString(e));
        dd_release(D);
        return nullptr;
    }
    /* DM-stage tables for groups of G consecutive DMs: per (group, subband)
     * the window start (a multiple of 8 samples), its word base in shared
     * memory and its word count (multiples of 4); per (DM, subband) the word
     * offset and parity.  G is the largest of 32, 16, ..., 1 whose windows fit
     * in shared memory; 0 selects the direct kernel. */
    int max_optin = 0;
    cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    std::vector<int> win, code;
    int G = dd::DM_G, smem_words = 0;
    for (; G >= 1; G /= 2) {
        const int ngroups = (ndm + G - 1) / G;
        win.assign((size_t)ngroups * nsub * 3, 0);
        code.assign((size_t)ngroups * G * nsub, 0);
        smem_words = 0;
        for (int g = 0; g < ngroups; g++) {
            int wb = 0;
            for (int s = 0; s < nsub; s++) {
                int omin = 1 << 30, omax = 0;
                for (int dl = 0; dl < G && g * G + dl < ndm; dl++) {
                    omin = std::min(omin, offsets[(size_t)(g * G + dl) * nsub + s]);
                    omax = std::max(omax, offsets[(size_t)(g * G + dl) * nsub + s]);
                }
                const int start = omin & ~7;
                const int words = ((dd::DM_TT + (omax - start) + 3) / 2 + 3) / 4 * 4;
                win[((size_t)g * nsub + s) * 3] = start;
                win[((size_t)g * nsub + s) * 3 + 1] = wb;
                win[((size_t)g * nsub + s) * 3 + 2] = words;
                for (int dl = 0; dl < G && g * G + dl < ndm; dl++) {
                    const int rel = offsets[(size_t)(g * G + dl) * nsub + s] - start;
                    code[((size_t)g * G + dl) * nsub + s] = ((wb + (rel >> 1)) << 1) | (rel & 1);
                }
                wb += words;
            }
            smem_words = std::max(smem_words, wb);
        }
        if ((long long)smem_words * 8 + (long long)G * nsub * 4 <= max_optin) break;
    }
    /* codes -> absolute shared words: odd offsets read the shifted copy */
    for (int &c : code) c = (c >> 1) + ((c & 1) ? smem_words : 0);
    D->G = G;
    D->ngroups = G > 0 ? (ndm + G - 1) / G : 0;
    D->smem_words = G > 0 ? smem_words : 0;
    const size_t dm_smem = G > 0 ? (size_t)smem_words * 8 + (size_t)G * nsub * 4 : 0;
    if (sb_smem(D, 1) > max_optin) {
        fprintf(stderr, "Error: cs_dedisp_create: channel delays of %d samples need more "
                        "shared memory than a CTA has\n", halo);
        dd_release(D);
        return nullptr;
    }
    /* staging chunks: per group, the windows in subband order; the subband
     * index rides in the high bits until the row stride is known */
    std::vector<long long> chunks;
    std::vector<int> nch;
    if (G > 0) {
        D->maxch = smem_words / 4;
        chunks.assign((size_t)D->ngroups * D->maxch, 0);
        nch.assign(D->ngroups, 0);
        for (int g = 0; g < D->ngroups; g++) {
            int n = 0;
            for (int s = 0; s < nsub; s++) {
                const int start = win[((size_t)g * nsub + s) * 3];
                const int words = win[((size_t)g * nsub + s) * 3 + 2];
                for (int j = 0; j < words / 4; j++)
                    chunks[(size_t)g * D->maxch + n++] = ((long long)s << 40) + start + 8LL * j;
            }
            nch[g] = n;
        }
    }
    /* S is read up to (tiles * DM_TT) + maxoff + a few words beyond */
    const long long ntile = (max_spectra + dd::DM_TT - 1) / dd::DM_TT;
    D->sstride = ((ntile + 1) * dd::DM_TT + maxoff + 64 + 255) / 256 * 256;
    for (long long &c : chunks) c = (c >> 40) * D->sstride + (c & ((1LL << 40) - 1));
#define DDCK(x)                                                                       \
    do {                                                                              \
        cudaError_t e_ = (x);                                                         \
        if (e_ != cudaSuccess) {                                                      \
            fprintf(stderr, "Error: cs_dedisp_create: %s: %s\n", #x, cudaGetErrorString(e_)); \
            dd_release(D);                                                            \
            return nullptr;                                                           \
        }                                                                             \
    } while (0)
    DDCK(cudaMalloc((void **)&D->d_idisp, sizeof(int) * nchan));
    DDCK(cudaMemcpy(D->d_idisp, idispdt, sizeof(int) * nchan, cudaMemcpyHostToDevice));
    DDCK(cudaMalloc((void **)&D->d_offs, sizeof(int) * (size_t)ndm * nsub));
    DDCK(cudaMemcpy(D->d_offs, offsets, sizeof(int) * (size_t)ndm * nsub, cudaMemcpyHostToDevice));
    if (G > 0) {
        DDCK(cudaMalloc((void **)&D->d_code, sizeof(int) * code.size()));
        DDCK(cudaMemcpy(D->d_code, code.data(), sizeof(int) * code.size(), cudaMemcpyHostToDevice));
        DDCK(cudaMalloc((void **)&D->d_chunk, sizeof(long long) * chunks.size()));
        DDCK(cudaMemcpy(D->d_chunk, chunks.data(), sizeof(long long) * chunks.size(),
                        cudaMemcpyHostToDevice));
        DDCK(cudaMalloc((void **)&D->d_nch, sizeof(int) * nch.size()));
        DDCK(cudaMemcpy(D->d_nch, nch.data(), sizeof(int) * nch.size(), cudaMemcpyHostToDevice));
    }
    DDCK(cudaMalloc((void **)&D->d_sub, sizeof(uint16_t) * (size_t)nsub * D->sstride));
    {
        /* clipped DM stage: the union window of each group of FG DMs per subband */
        const int ng = (ndm + dd::FG - 1) / dd::FG;
        std::vector<int2> fw((size_t)ng * nsub);
        int wmax = 0;
        for (int g = 0; g < ng; g++)
            for (int s = 0; s < nsub; s++) {
                int lo = 1 << 30, hi = 0;
                for (int d = g * dd::FG; d < std::min(ndm, (g + 1) * dd::FG); d++) {
                    lo = std::min(lo, offsets[(size_t)d * nsub + s]);
                    hi = std::max(hi, offsets[(size_t)d * nsub + s]);
                }
                fw[(size_t)g * nsub + s] = make_int2(lo, dd::FT + hi - lo);
                wmax = std::max(wmax, dd::FT + hi - lo);
            }
        D->fwmax = wmax;
        DDCK(cudaMalloc((void **)&D->d_fwin, sizeof(int2) * fw.size()));
        DDCK(cudaMemcpy(D->d_fwin, fw.data(), sizeof(int2) * fw.size(), cudaMemcpyHostToDevice));
        DDCK(cudaFuncSetAttribute(dd::dd_dms_f32, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  max_optin));
    }
    DDCK(cudaStreamCreateWithFlags(&D->st, cudaStreamNonBlocking));
    DDCK(cudaEventCreate(&D->ev0));
    DDCK(cudaEventCreate(&D->ev1));
    DDCK(cudaEventCreate(&D->ev2));
    if (G > 0)
        DDCK(cudaFuncSetAttribute(dd::dd_dms_u16, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)dm_smem));
    DDCK(cudaFuncSetAttribute(dd::dd_subband_u8, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              max_optin));
    DDCK(cudaFuncSetAttribute(dd::dd_subband_clip, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              max_optin));
    /* a copy from pageable memory may return before its DMA lands; finish
     * them all before a run on any stream can read the tables */
    DDCK(cudaDeviceSynchronize());
#undef DDCK
    return D;
}

/* Dynamic shared memory of the clipped DM stage: the staged offsets and two
 * rounds of fr windows. */
static size_t dd_clip_smem(int fr, int fwmax)
{
    return sizeof(int) * dd::FMAXSUB * dd::FG + sizeof(float) * 2 * (size_t)fr * fwmax;
}

/* Subbands the clipped DM stage stages per round (FR, fewer when the
 * windows are wide); 0 if not even one fits in shared memory, or there are
 * more subbands than it stages offsets for. */
static int dd_clip_rounds(const CsDedisp *D)
{
    if (D->nsub > dd::FMAXSUB) return 0;
    int max_optin = 0;
    cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, D->device);
    for (int fr = dd::FR; fr >= 1; fr--)
        if (dd_clip_smem(fr, D->fwmax) <= (size_t)max_optin) return fr;
    return 0;
}

static cudaError_t dd_enqueue(CsDedisp *D, const uint8_t *d_raw, long long nspec, long long nout,
                              float *d_out, long long ostride, cudaStream_t st,
                              const uint8_t *d_flags = nullptr, const float *d_levels = nullptr)
{
    const bool clip = d_flags != nullptr;
    if (nout <= 0) return cudaSuccess;
    /* subband stage over every sample the DM stage can read */
    const long long ntile_dm = (nout + dd::DM_TT - 1) / dd::DM_TT;
    const long long sfill = std::min(D->sstride, ntile_dm * dd::DM_TT + D->maxoff + 64);
    int max_optin = 0;
    cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, D->device);
    int slab = std::max(1, std::min(D->nsub, 256 / std::max(1, D->cps)));
    while (slab > 1 && sb_smem(D, slab, clip) > std::min(max_optin, 100 * 1024)) slab /= 2;
    dd::SubArgs sa;
    sa.raw = d_raw;
    sa.nspec = nspec;
    sa.nchan = D->nchan;
    sa.cps = D->cps;
    sa.nsub = D->nsub;
    sa.slab = slab;
    sa.halo = D->halo;
    sa.rowstride = sb_rowstride(D, slab);
    sa.table_off = sb_table_offset(D, slab);
    sa.idisp = D->d_idisp;
    sa.nvalid = nspec / D->L >= 1 ? (nspec / D->L - 1) * D->L : 0;
    sa.sfill = sfill;
    sa.sub = D->d_sub;
    sa.sstride = D->sstride;
    sa.flags = d_flags;
    sa.nflags = nspec / D->L * D->L;
    sa.levels = d_levels;
    sa.L = D->L;
    sa.flag_off = sb_flag_offset(D, slab);
    sa.subf = D->d_subf;
    dim3 gs((D->nsub + slab - 1) / slab, (unsigned)((sfill + dd::SB_TT - 1) / dd::SB_TT));
    cudaEventRecord(D->ev0, st);
    if (clip)
        dd::dd_subband_clip<<<gs, dd::SB_THREADS, sb_smem(D, slab, true), st>>>(sa);
    else
        dd::dd_subband_u8<<<gs, dd::SB_THREADS, sb_smem(D, slab), st>>>(sa);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (clip) {
        const long long ntile = (nout + dd::FT - 1) / dd::FT;
        const long long ngrp = (D->ndm + dd::FG - 1) / dd::FG;
        const int fr = dd_clip_rounds(D);
        cudaEventRecord(D->ev1, st);
        dd::dd_dms_f32<<<(unsigned)(ntile * ngrp), 256, dd_clip_smem(fr, D->fwmax), st>>>(
            D->d_subf, D->sstride, D->nsub, D->ndm, D->d_offs, D->d_fwin, D->fwmax, fr, sfill,
            nout, d_out, ostride);
        cudaEventRecord(D->ev2, st);
        return cudaGetLastError();
    }
    dd::DmArgs da;
    da.sub = D->d_sub;
    da.sstride = D->sstride;
    da.nsub = D->nsub;
    da.ndm = D->ndm;
    da.G = D->G;
    da.offs = D->d_offs;
    da.flush = D->flush;
    da.flush8 = (D->nsub % 8 == 0 && D->flush >= 8) ? D->flush / 8 * 8 : 0;
    da.chunk = D->d_chunk;
    da.nch = D->d_nch;
    da.maxch = D->maxch;
    da.code = D->d_code;
    da.smem_words = D->smem_words;
    da.nout = nout;
    da.out = d_out;
    da.ostride = ostride;
    cudaEventRecord(D->ev1, st);
    if (D->G > 0) {
        const size_t dm_smem = (size_t)D->smem_words * 8 + (size_t)D->G * D->nsub * 4;
        dim3 gd((unsigned)D->ngroups, (unsigned)ntile_dm);
        dd::dd_dms_u16<<<gd, dd::DM_THREADS, dm_smem, st>>>(da);
    } else {
        dim3 gd((unsigned)((nout + 255) / 256), (unsigned)D->ndm);
        dd::dd_dms_u16_direct<<<gd, 256, 0, st>>>(da);
    }
    cudaEventRecord(D->ev2, st);
    return cudaGetLastError();
}

CS_EXPORT int cs_dedisp_run_device(CsDedisp *D, const uint8_t *d_raw, long long nspec,
                                   long long numout, float *d_out, long long out_stride,
                                   void *stream, long long *nout_written)
{
    if (nout_written) *nout_written = 0;
    if (!D || !d_raw || !d_out) return -1;
    if (nspec > D->max_spectra) {
        fprintf(stderr, "Error: cs_dedisp_run: %lld spectra exceed the plan's %lld\n", nspec,
                D->max_spectra);
        return -1;
    }
    const long long nout = cs_dedisp_output_length(D, nspec, numout);
    if (out_stride < nout || (out_stride & 3) || ((uintptr_t)d_out & 15)) {
        fprintf(stderr, "Error: cs_dedisp_run: out_stride must be >= %lld and a multiple of 4, "
                        "the output 16-byte aligned\n", nout);
        return -1;
    }
    if (cudaSetDevice(D->device) != cudaSuccess) return -1;
    cudaStream_t st = stream ? (cudaStream_t)stream : D->st;
    cudaError_t e = dd_enqueue(D, d_raw, nspec, nout, d_out, out_stride, st);
    if (e != cudaSuccess) {
        fprintf(stderr, "Error: cs_dedisp_run: %s\n", cudaGetErrorString(e));
        return -1;
    }
    if (nout_written) *nout_written = nout;
    return 0;
}

CS_EXPORT int cs_dedisp_run_device_clipped(CsDedisp *D, const uint8_t *d_raw, long long nspec,
                                           long long numout, const uint8_t *d_flags,
                                           const float *d_levels, float *d_out,
                                           long long out_stride, void *stream,
                                           long long *nout_written)
{
    if (nout_written) *nout_written = 0;
    if (!D || !d_raw || !d_out || !d_flags || !d_levels) return -1;
    if (nspec > D->max_spectra) {
        fprintf(stderr, "Error: cs_dedisp_run_device_clipped: %lld spectra exceed the plan's "
                        "%lld\n", nspec, D->max_spectra);
        return -1;
    }
    const long long nout = cs_dedisp_output_length(D, nspec, numout);
    if (out_stride < nout || (out_stride & 3) || ((uintptr_t)d_out & 15)) {
        fprintf(stderr, "Error: cs_dedisp_run_device_clipped: out_stride must be >= %lld and a "
                        "multiple of 4, the output 16-byte aligned\n", nout);
        return -1;
    }
    if ((unsigned long long)((nout + dd::FT - 1) / dd::FT) *
            (unsigned long long)((D->ndm + dd::FG - 1) / dd::FG) >= (1ULL << 31)) {
        fprintf(stderr, "Error: cs_dedisp_run_device_clipped: %lld points x %d DMs is too many "
                        "for one launch\n", nout, D->ndm);
        return -1;
    }
    if (dd_clip_rounds(D) < 1) {
        fprintf(stderr, "Error: cs_dedisp_run_device_clipped: subband windows of %d samples "
                        "(%d subbands) need more shared memory than a CTA has\n", D->fwmax,
                D->nsub);
        return -1;
    }
    if (cudaSetDevice(D->device) != cudaSuccess) return -1;
    cudaError_t e = cudaSuccess;
    if (!D->d_subf)
        e = cudaMalloc((void **)&D->d_subf, sizeof(float) * (size_t)D->nsub * D->sstride);
    cudaStream_t st = stream ? (cudaStream_t)stream : D->st;
    if (e == cudaSuccess) e = dd_enqueue(D, d_raw, nspec, nout, d_out, out_stride, st, d_flags,
                                         d_levels);
    if (e != cudaSuccess) {
        fprintf(stderr, "Error: cs_dedisp_run_device_clipped: %s\n", cudaGetErrorString(e));
        return -1;
    }
    if (nout_written) *nout_written = nout;
    return 0;
}

/* Host memory in and out: raw [nspec][nchan] u8, out [ndm][out_stride]. */
CS_EXPORT int cs_dedisp_run(CsDedisp *D, const uint8_t *h_raw, long long nspec, long long numout,
                            float *h_out, long long out_stride, long long *nout_written)
{
    if (nout_written) *nout_written = 0;
    if (!D || !h_raw || !h_out) return -1;
    if (nspec > D->max_spectra) {
        fprintf(stderr, "Error: cs_dedisp_run: %lld spectra exceed the plan's %lld\n", nspec,
                D->max_spectra);
        return -1;
    }
    const long long nout = cs_dedisp_output_length(D, nspec, numout);
    if (out_stride < nout) {
        fprintf(stderr, "Error: cs_dedisp_run: out_stride %lld < %lld\n", out_stride, nout);
        return -1;
    }
    if (cudaSetDevice(D->device) != cudaSuccess) return -1;
    const long long dstride = (nout + 3) / 4 * 4;
    cudaError_t e = cudaSuccess;
    if (!D->d_raw) e = cudaMalloc((void **)&D->d_raw, (size_t)D->max_spectra * D->nchan);
    if (e == cudaSuccess && D->out_cap < dstride * D->ndm) {
        cudaFree(D->d_out);
        D->d_out = nullptr;
        e = cudaMalloc((void **)&D->d_out, sizeof(float) * (size_t)std::max(1LL, dstride * D->ndm));
        D->out_cap = e == cudaSuccess ? dstride * D->ndm : 0;
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(D->d_raw, h_raw, (size_t)nspec * D->nchan, cudaMemcpyHostToDevice, D->st);
    if (e == cudaSuccess) e = dd_enqueue(D, D->d_raw, nspec, nout, D->d_out, dstride, D->st);
    if (e == cudaSuccess && nout > 0)
        e = cudaMemcpy2DAsync(h_out, sizeof(float) * out_stride, D->d_out, sizeof(float) * dstride,
                              sizeof(float) * nout, D->ndm, cudaMemcpyDeviceToHost, D->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(D->st);
    if (e != cudaSuccess) {
        fprintf(stderr, "Error: cs_dedisp_run: %s\n", cudaGetErrorString(e));
        return -1;
    }
    if (nout_written) *nout_written = nout;
    return 0;
}

/* Kernel times of the last run (subband stage, DM stage), from CUDA events
 * recorded around the two launches on the run's stream. */
CS_EXPORT int cs_dedisp_last_times(CsDedisp *D, float *subband_ms, float *dm_ms)
{
    if (!D) return -1;
    if (cudaEventSynchronize(D->ev2) != cudaSuccess) return -1;
    float a = 0.0f, b = 0.0f;
    if (cudaEventElapsedTime(&a, D->ev0, D->ev1) != cudaSuccess ||
        cudaEventElapsedTime(&b, D->ev1, D->ev2) != cudaSuccess) {
        (void)cudaGetLastError();       /* unrecorded events: no stale error left behind */
        return -1;
    }
    if (subband_ms) *subband_ms = a;
    if (dm_ms) *dm_ms = b;
    return 0;
}

CS_EXPORT void cs_dedisp_free(CsDedisp *D)
{
    if (!D) return;
    cudaSetDevice(D->device);
    if (D->st) cudaStreamSynchronize(D->st);
    dd_release(D);
}
