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
 * Kernels (HBM layout: raw [nspec][nchan] u8 as read; S [nsub][sstride]
 * 32-bit words, word w holding samples w (low half) and w + DM_P (high
 * half); out [ndm][out_stride] f32):
 *   dd_subband_u8  one CTA per (slab of subbands, 256-sample tile): the
 *                  tile's raw rows plus the delay halo are copied
 *                  asynchronously into shared memory with padded rows (an
 *                  odd number of words: lanes over consecutive samples hit
 *                  consecutive banks), then each warp sums the channels of
 *                  one subband for 32 samples and writes each sum into the
 *                  two words that hold it.
 *   dd_dms_u16     persistent, warp-specialised: a copy warp bulk-copies
 *                  each work item's S windows (tile + the DM group's offset
 *                  spread) and code block into a ring of shared stages; 16
 *                  summing warps add one word per (DM, subband, column),
 *                  i.e. two samples per 32-bit add (widened before the
 *                  16-bit halves can carry).  Shared-memory-bound: 2 B of
 *                  shared reads per subband term.
 *   dd_dms_u16_direct  the same sums straight from L1/L2, for geometries
 *                  whose windows do not fit in shared memory.
 *
 * A run with prepsubband's -clip that replaces spectra (cs_clip_levels) has
 * non-integer channel levels in it, so its sums need FP32 in the reference's
 * order; S is float there (one sample per element):
 *   dd_subband_clip  dd_subband_u8's staging plus one clip flag per row;
 *                  channels added in ascending frequency from 0.0f, a
 *                  flagged spectrum contributing its block's level.
 *   dd_dms_f32_ws  dd_dms_u16's pipeline over float windows; each summing
 *                  thread adds the subbands in ascending order from -0.0f
 *                  for 2 DMs x 8 samples.
 *   dd_dms_f32     the fallback for geometries whose stages do not fit
 *                  twice: one CTA per (1024 samples, 16 DMs), per round of
 *                  four subbands the union windows copied with cp.async a
 *                  round ahead of the sums.
 *
 * Every wait in the pipelined kernels is bounded; one that gives up sets the
 * plan's error flag (cs_dedisp_run and cs_dedisp_last_times report it).
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
#ifndef DD_SB_TT
#define DD_SB_TT 256
#endif
#ifndef DD_DM_NCW
#define DD_DM_NCW 16
#endif
constexpr int SB_TT = DD_SB_TT;   /* samples per subband tile */
constexpr int SB_THREADS = 512;
/* S word w of a subband holds samples w and w + DM_P (low, high half), so a
 * DM tile of 2 DM_P samples reads one aligned word per (DM, subband, column)
 * whatever the parity of the DM's offset */
constexpr int DM_P = 128;
constexpr int DM_TILE = 2 * DM_P; /* samples per DM tile */
constexpr int DM_G = 32;          /* most DMs per group (one work item) */
constexpr int DM_NCW = DD_DM_NCW; /* summing warps of the DM stage */
constexpr int DM_DPT = DM_G / DM_NCW;   /* most DMs a summing thread */
constexpr int DM_CPT = DM_P / 32;       /* columns a summing thread */
constexpr int DM_THREADS = (DM_NCW + 1) * 32;   /* + one copy warp */
constexpr int DM_MAXST = 4;       /* most pipeline stages */
static_assert(DM_G % DM_NCW == 0 && DM_P % 32 == 0, "DM tile shape");
constexpr unsigned long long DD_WAIT_NS = 2000000000ull;   /* bound on any in-kernel wait */

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

/* mbarriers and bulk copies (one elected thread arms a barrier with the
 * bytes it expects; the copy engine completes them) */
static __device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

static __device__ __forceinline__ void mbar_fence_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

static __device__ __forceinline__ void mbar_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

static __device__ __forceinline__ void mbar_arrive_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}

static __device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
    return ok != 0;
}

/* Bounded wait for the phase of the given parity (false after DD_WAIT_NS). */
static __device__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
    if (mbar_try(bar, parity)) return true;
    unsigned long long t0;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    while (!mbar_try(bar, parity)) {
        unsigned long long t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        if (t - t0 > DD_WAIT_NS) return false;
        __nanosleep(32);
    }
    return true;
}

/* Global -> shared bulk copy (16-byte aligned ends, a multiple of 16 bytes)
 * completing `bytes` on barrier bar. */
static __device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes,
                                                uint32_t bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
                 "[%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
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
    uint32_t *sub;            /* S: [nsub][sstride] words (samples w, w + DM_P) */
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
        /* low half of word T, high half of word T - DM_P */
        uint16_t *row = reinterpret_cast<uint16_t *>(a.sub + (long long)(s0 + sl) * a.sstride);
        row[2 * T] = (uint16_t)acc;
        if (T >= DM_P) row[2 * (T - DM_P) + 1] = (uint16_t)acc;
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
    const uint32_t *sub;      /* S: [nsub][sstride] words */
    long long sstride;        /* words per subband row */
    int nsub, nsub8, ndm;
    int G;                    /* DMs per group (<= DM_G) */
    int ngroups;
    const int *offs;          /* [ndm][nsub] (direct kernel) */
    int flush;                /* subbands per packed-accumulator flush */
    const int4 *win;          /* [ngroups][nsub]: window start (words from the tile
                                 start, a multiple of 4), its shared word, its words */
    const uint16_t *code;     /* [ngroups][G][nsub8]: shared word of each (DM, subband)
                                 row; padding subbands and absent DMs read the zero row */
    const int *gbytes;        /* [ngroups]: bytes of the group's windows */
    int code_bytes;           /* bytes of one group's code block (a multiple of 16) */
    int code_word, zero_word; /* word offsets in a stage */
    int stage_words, nstage;
    long long nitems;         /* tiles x groups */
    long long nout;
    float *out;
    long long ostride;
    int *err;                 /* set when a wait gave up */
};

/* The integer DM stage, warp-specialised over a ring of nstage shared
 * buffers.  Work item = (tile of DM_TILE samples, group of G consecutive
 * DMs), the group index fastest; CTA b takes items b, b + grid, ... so the
 * CTAs sweep the series together and the S rows they read stay in L2.
 *   copy warp:     per item one bulk copy per subband window (the union of
 *                  the group's DM windows, from a multiple of 4 words) and
 *                  one of the group's code block, all completing on the
 *                  stage's full barrier;
 *   summing warps: warp w sums DMs w, w + NCW, ... of the group for the
 *                  columns c = lane + 32 k: one shared word per (DM,
 *                  subband, column) gives samples T0 + c and T0 + c + DM_P,
 *                  added with one 32-bit add (two 16-bit lanes, widened
 *                  every `flush` subbands before they can carry); lanes
 *                  read consecutive words.  The stage is released before
 *                  the float stores.
 * Bound: shared-memory reads, 2 B per subband term. */
__global__ void __launch_bounds__(DM_THREADS, 1) dd_dms_u16(const DmArgs a)
{
    extern __shared__ __align__(128) uint32_t smw[];
    __shared__ __align__(8) unsigned long long bars[2 * DM_MAXST];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t full0 = smem_addr(&bars[0]), empty0 = smem_addr(&bars[DM_MAXST]);
    const int NS = a.nstage;
    if (threadIdx.x == 0) {
        for (int i = 0; i < NS; i++) {
            mbar_init(full0 + 8 * i, 1);
            mbar_init(empty0 + 8 * i, DM_NCW);
        }
        mbar_fence_init();
    }
    for (int st = 0; st < NS; st++)
        for (int i = threadIdx.x; i < DM_P; i += blockDim.x)
            smw[(size_t)st * a.stage_words + a.zero_word + i] = 0;
    __syncthreads();
    const long long grid = gridDim.x;

    if (warp == DM_NCW) {
        /* ------------------------------ copy warp ------------------------------ */
        long long k = 0;
        bool ok = true;
        for (long long item = blockIdx.x; item < a.nitems; item += grid, k++) {
            const int st = (int)(k % NS);
            const uint32_t ph = (uint32_t)(k / NS) & 1u;
            if (k >= NS) ok = __all_sync(0xffffffffu, mbar_wait(empty0 + 8 * st, ph ^ 1u));
            if (!ok) break;
            const long long tile = item / a.ngroups;
            const int g = (int)(item - tile * a.ngroups);
            const uint32_t fb = full0 + 8 * st;
            if (lane == 0) mbar_arrive_tx(fb, (uint32_t)(__ldg(a.gbytes + g) + a.code_bytes));
            __syncwarp();
            uint32_t *stage = smw + (size_t)st * a.stage_words;
            const uint32_t *src0 = a.sub + tile * DM_TILE;
            for (int s = lane; s < a.nsub; s += 32) {
                const int4 w = __ldg(a.win + (size_t)g * a.nsub + s);
                bulk_g2s(stage + w.y, src0 + (long long)s * a.sstride + w.x, (uint32_t)w.z * 4u, fb);
            }
            if (lane == 0)
                bulk_g2s(stage + a.code_word, a.code + (size_t)g * a.G * a.nsub8,
                         (uint32_t)a.code_bytes, fb);
        }
        if (!ok && lane == 0) atomicExch(a.err, 1);
        /* never leave with copies in flight: the last use of each stage landed */
        for (long long j = k > NS ? k - NS : 0; j < k; j++)
            if (!mbar_wait(full0 + 8 * (int)(j % NS), (uint32_t)(j / NS) & 1u) && lane == 0)
                atomicExch(a.err, 1);
        return;
    }

    /* ---------------------------- summing warps ---------------------------- */
    long long k = 0;
    for (long long item = blockIdx.x; item < a.nitems; item += grid, k++) {
        const int st = (int)(k % NS);
        const uint32_t ph = (uint32_t)(k / NS) & 1u;
        if (!__all_sync(0xffffffffu, mbar_wait(full0 + 8 * st, ph))) {
            if (lane == 0) atomicExch(a.err, 1);
            break;
        }
        const long long tile = item / a.ngroups;
        const int g = (int)(item - tile * a.ngroups);
        const uint32_t *stage = smw + (size_t)st * a.stage_words;
        const uint16_t *cb = reinterpret_cast<const uint16_t *>(stage + a.code_word);
        const uint32_t *col = stage + lane;
        uint32_t lo[DM_DPT][DM_CPT], hi[DM_DPT][DM_CPT], p[DM_DPT][DM_CPT];
#pragma unroll
        for (int j = 0; j < DM_DPT; j++)
#pragma unroll
            for (int c = 0; c < DM_CPT; c++) lo[j][c] = hi[j][c] = p[j][c] = 0;
        /* widen the packed sums every `flush` subbands: at 8-subband block
         * boundaries when flush >= 8 (no branch among a block's loads) */
        const int fl8 = a.flush >= 8 ? a.flush / 8 : 0;
        int cnt = 0;
        for (int s8 = 0; s8 < a.nsub8; s8 += 8) {
            uint32_t cw[DM_DPT][4];
#pragma unroll
            for (int j = 0; j < DM_DPT; j++) {
                const int dl = warp + DM_NCW * j;
                if (dl < a.G) {
                    const uint4 v = *reinterpret_cast<const uint4 *>(cb + (size_t)dl * a.nsub8 + s8);
                    cw[j][0] = v.x; cw[j][1] = v.y; cw[j][2] = v.z; cw[j][3] = v.w;
                } else {
                    const uint32_t z = (uint32_t)a.zero_word * 0x10001u;
                    cw[j][0] = cw[j][1] = cw[j][2] = cw[j][3] = z;
                }
            }
            if (fl8) {
#pragma unroll
                for (int u = 0; u < 8; u++)
#pragma unroll
                    for (int j = 0; j < DM_DPT; j++) {
                        const uint32_t off = (u & 1) ? (cw[j][u >> 1] >> 16) : (cw[j][u >> 1] & 0xffffu);
#pragma unroll
                        for (int c = 0; c < DM_CPT; c++) p[j][c] += col[off + 32 * c];
                    }
                if (++cnt == fl8) {
                    cnt = 0;
#pragma unroll
                    for (int j = 0; j < DM_DPT; j++)
#pragma unroll
                        for (int c = 0; c < DM_CPT; c++) {
                            lo[j][c] += p[j][c] & 0xffffu;
                            hi[j][c] += p[j][c] >> 16;
                            p[j][c] = 0;
                        }
                }
            } else {
#pragma unroll
                for (int u = 0; u < 8; u++) {
#pragma unroll
                    for (int j = 0; j < DM_DPT; j++) {
                        const uint32_t off = (u & 1) ? (cw[j][u >> 1] >> 16) : (cw[j][u >> 1] & 0xffffu);
#pragma unroll
                        for (int c = 0; c < DM_CPT; c++) p[j][c] += col[off + 32 * c];
                    }
                    if (++cnt == a.flush) {
                        cnt = 0;
#pragma unroll
                        for (int j = 0; j < DM_DPT; j++)
#pragma unroll
                            for (int c = 0; c < DM_CPT; c++) {
                                lo[j][c] += p[j][c] & 0xffffu;
                                hi[j][c] += p[j][c] >> 16;
                                p[j][c] = 0;
                            }
                    }
                }
            }
        }
#pragma unroll
        for (int j = 0; j < DM_DPT; j++)
#pragma unroll
            for (int c = 0; c < DM_CPT; c++) {
                lo[j][c] += p[j][c] & 0xffffu;
                hi[j][c] += p[j][c] >> 16;
            }
        /* the sums are in registers: release the stage, then store */
        __syncwarp();
        if (lane == 0) mbar_arrive(empty0 + 8 * st);
        const long long T0 = tile * DM_TILE;
#pragma unroll
        for (int j = 0; j < DM_DPT; j++) {
            const int dl = warp + DM_NCW * j;
            const int d = g * a.G + dl;
            if (dl >= a.G || d >= a.ndm) break;
            float *o = a.out + (long long)d * a.ostride + T0 + lane;
#pragma unroll
            for (int c = 0; c < DM_CPT; c++) {
                if (T0 + lane + 32 * c < a.nout) o[32 * c] = (float)lo[j][c];
                if (T0 + DM_P + lane + 32 * c < a.nout) o[DM_P + 32 * c] = (float)hi[j][c];
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
    const uint16_t *s16 = reinterpret_cast<const uint16_t *>(a.sub);
    uint32_t acc = 0;
    /* sample x of a subband row is the low half of its word x */
    for (int s = 0; s < a.nsub; s++) acc += __ldg(s16 + 2 * ((long long)s * a.sstride + T + off[s]));
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

/* The DM stage of a clipped run, warp-specialised like dd_dms_u16: work
 * item = (tile of FD_T samples, group of G consecutive DMs), the group index
 * fastest, CTA b taking items b, b + grid, ...; a copy warp bulk-copies the
 * item's subband windows (floats, from a multiple of 4) and its code block
 * into a ring of stages; summing warp w adds, for DMs w, w + NCW, ... of the
 * group, the subbands in ascending order from -0.0f for the samples
 * lane + 32 k (FP32, the reference's order: dispersion.c:346-362).  S is
 * filled up to sfill samples; every written output reads below it. */
constexpr int FD_T = 256;                 /* samples per tile */
constexpr int FD_NCW = 16;                /* summing warps */
constexpr int FD_SPL = FD_T / 32;         /* samples a lane */
constexpr int FD_DPW = DM_G / FD_NCW;     /* most DMs a summing warp */
constexpr int FD_THREADS = (FD_NCW + 1) * 32;

struct FdArgs {
    const float *sub;         /* S: [nsub][sstride] floats */
    long long sstride;
    int nsub, nsub8, ndm, G, ngroups;
    const int4 *win;          /* [ngroups][nsub]: window start (floats from the tile start,
                                 a multiple of 4), its stage float, its floats */
    const uint16_t *code;     /* [ngroups][G][nsub8]: stage float of each (DM, subband) row */
    const int *gbytes;        /* [ngroups]: bytes of the group's windows */
    int code_bytes, code_word, stage_words, nstage;
    long long nitems;
    long long nout;
    float *out;
    long long ostride;
    int *err;
};

__global__ void __launch_bounds__(FD_THREADS, 1) dd_dms_f32_ws(const FdArgs a)
{
    extern __shared__ __align__(128) float smf[];
    __shared__ __align__(8) unsigned long long bars[2 * DM_MAXST];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t full0 = smem_addr(&bars[0]), empty0 = smem_addr(&bars[DM_MAXST]);
    const int NS = a.nstage;
    if (threadIdx.x == 0) {
        for (int i = 0; i < NS; i++) {
            mbar_init(full0 + 8 * i, 1);
            mbar_init(empty0 + 8 * i, FD_NCW);
        }
        mbar_fence_init();
    }
    __syncthreads();
    const long long grid = gridDim.x;

    if (warp == FD_NCW) {
        /* ------------------------------ copy warp ------------------------------ */
        long long k = 0;
        bool ok = true;
        for (long long item = blockIdx.x; item < a.nitems; item += grid, k++) {
            const int st = (int)(k % NS);
            const uint32_t ph = (uint32_t)(k / NS) & 1u;
            if (k >= NS) ok = __all_sync(0xffffffffu, mbar_wait(empty0 + 8 * st, ph ^ 1u));
            if (!ok) break;
            const long long tile = item / a.ngroups;
            const int g = (int)(item - tile * a.ngroups);
            const uint32_t fb = full0 + 8 * st;
            if (lane == 0) mbar_arrive_tx(fb, (uint32_t)(__ldg(a.gbytes + g) + a.code_bytes));
            __syncwarp();
            float *stage = smf + (size_t)st * a.stage_words;
            const float *src0 = a.sub + tile * FD_T;
            for (int s = lane; s < a.nsub; s += 32) {
                const int4 w = __ldg(a.win + (size_t)g * a.nsub + s);
                bulk_g2s(stage + w.y, src0 + (long long)s * a.sstride + w.x, (uint32_t)w.z * 4u, fb);
            }
            if (lane == 0)
                bulk_g2s(stage + a.code_word, a.code + (size_t)g * a.G * a.nsub8,
                         (uint32_t)a.code_bytes, fb);
        }
        if (!ok && lane == 0) atomicExch(a.err, 1);
        for (long long j = k > NS ? k - NS : 0; j < k; j++)
            if (!mbar_wait(full0 + 8 * (int)(j % NS), (uint32_t)(j / NS) & 1u) && lane == 0)
                atomicExch(a.err, 1);
        return;
    }

    /* ---------------------------- summing warps ---------------------------- */
    long long k = 0;
    for (long long item = blockIdx.x; item < a.nitems; item += grid, k++) {
        const int st = (int)(k % NS);
        const uint32_t ph = (uint32_t)(k / NS) & 1u;
        if (!__all_sync(0xffffffffu, mbar_wait(full0 + 8 * st, ph))) {
            if (lane == 0) atomicExch(a.err, 1);
            break;
        }
        const long long tile = item / a.ngroups;
        const int g = (int)(item - tile * a.ngroups);
        const float *stage = smf + (size_t)st * a.stage_words;
        const uint16_t *cb = reinterpret_cast<const uint16_t *>(stage + a.code_word);
        const float *col = stage + lane;
        float acc[FD_DPW][FD_SPL];
#pragma unroll
        for (int j = 0; j < FD_DPW; j++)
#pragma unroll
            for (int q = 0; q < FD_SPL; q++) acc[j][q] = -0.0f;
        /* this warp's DMs of the group (warp-uniform) */
        int ndw = 0;
#pragma unroll
        for (int j = 0; j < FD_DPW; j++)
            if (warp + FD_NCW * j < a.G) ndw = j + 1;
        for (int s8 = 0; s8 < a.nsub8; s8 += 8) {
            uint32_t cw[FD_DPW][4];
#pragma unroll
            for (int j = 0; j < FD_DPW; j++) {
                const int dl = min(warp + FD_NCW * j, a.G - 1);
                const uint4 v = *reinterpret_cast<const uint4 *>(cb + (size_t)dl * a.nsub8 + s8);
                cw[j][0] = v.x; cw[j][1] = v.y; cw[j][2] = v.z; cw[j][3] = v.w;
            }
            if (s8 + 8 <= a.nsub) {
#pragma unroll
                for (int u = 0; u < 8; u++)
#pragma unroll
                    for (int j = 0; j < FD_DPW; j++) {
                        if (j >= ndw) break;
                        const uint32_t off = (u & 1) ? (cw[j][u >> 1] >> 16) : (cw[j][u >> 1] & 0xffffu);
#pragma unroll
                        for (int q = 0; q < FD_SPL; q++)
                            acc[j][q] = __fadd_rn(acc[j][q], col[off + 32 * q]);
                    }
            } else {
#pragma unroll
                for (int u = 0; u < 8; u++) {
                    if (s8 + u >= a.nsub) break;
#pragma unroll
                    for (int j = 0; j < FD_DPW; j++) {
                        if (j >= ndw) break;
                        const uint32_t off = (u & 1) ? (cw[j][u >> 1] >> 16) : (cw[j][u >> 1] & 0xffffu);
#pragma unroll
                        for (int q = 0; q < FD_SPL; q++)
                            acc[j][q] = __fadd_rn(acc[j][q], col[off + 32 * q]);
                    }
                }
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(empty0 + 8 * st);
        const long long T0 = tile * FD_T;
#pragma unroll
        for (int j = 0; j < FD_DPW; j++) {
            const int d = g * a.G + warp + FD_NCW * j;
            if (j >= ndw || d >= a.ndm) break;
            float *o = a.out + (long long)d * a.ostride + T0 + lane;
#pragma unroll
            for (int q = 0; q < FD_SPL; q++)
                if (T0 + lane + 32 * q < a.nout) o[32 * q] = acc[j][q];
        }
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
    int G;                         /* DMs per group of the DM stage; 0: direct kernel */
    int ngroups;
    int nsub8, code_bytes, code_word, zero_word, stage_words, nstage;
    int *d_idisp = nullptr;
    int *d_offs = nullptr;
    int4 *d_win = nullptr;
    uint16_t *d_code = nullptr;
    int *d_gbytes = nullptr;
    int *d_err = nullptr;          /* set by a DM-stage wait that gave up */
    uint32_t *d_sub = nullptr;
    float *d_subf = nullptr;       /* S of clipped runs (allocated by the first one) */
    int2 *d_fwin = nullptr;        /* clipped DM stage (rounds kernel): per (DM group, subband)
                                      window */
    int fwmax = 0;                 /* widest such window (floats) */
    /* clipped DM stage, warp-specialised kernel (fG 0: the rounds kernel) */
    int fG = 0, fngroups = 0, fcode_bytes = 0, fcode_word = 0, fstage_words = 0, fnstage = 0;
    int4 *d_fwin2 = nullptr;
    uint16_t *d_fcode = nullptr;
    int *d_fgbytes = nullptr;
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
    cudaFree(D->d_win);
    cudaFree(D->d_gbytes);
    cudaFree(D->d_err);
    cudaFree(D->d_sub);
    cudaFree(D->d_subf);
    cudaFree(D->d_fwin);
    cudaFree(D->d_fwin2);
    cudaFree(D->d_fcode);
    cudaFree(D->d_fgbytes);
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
     * the window (from the group's lowest offset rounded down to 4 words, up
     * to its highest offset + DM_P, rounded up to 4 words) and its word in a
     * stage; per (group, DM, subband) the stage word of the DM's row.  A
     * stage holds the windows, the group's code block and a zero row.  G is
     * the largest of 32, 16, ..., 1 whose stages fit twice in shared memory;
     * 0 selects the direct kernel. */
    int max_optin = 0;
    cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    const int nsub8 = (nsub + 7) / 8 * 8;
    std::vector<int4> win;
    std::vector<uint16_t> code;
    std::vector<int> gbytes;
    /* CS_B200_DEDISP_DIRECT=1 selects the direct kernel (its tests) */
    int G = getenv("CS_B200_DEDISP_DIRECT") ? 0 : dd::DM_G;
    for (; G >= 1; G /= 2) {
        const int ngroups = (ndm + G - 1) / G;
        win.assign((size_t)ngroups * nsub, make_int4(0, 0, 0, 0));
        gbytes.assign(ngroups, 0);
        int wmax = 0;
        for (int g = 0; g < ngroups; g++) {
            int wb = 0;
            for (int s = 0; s < nsub; s++) {
                int omin = 1 << 30, omax = 0;
                for (int dl = 0; dl < G && g * G + dl < ndm; dl++) {
                    omin = std::min(omin, offsets[(size_t)(g * G + dl) * nsub + s]);
                    omax = std::max(omax, offsets[(size_t)(g * G + dl) * nsub + s]);
                }
                const int start = omin & ~3;
                const int words = (omax - start + dd::DM_P + 3) / 4 * 4;
                win[(size_t)g * nsub + s] = make_int4(start, wb, words, 0);
                wb += words;
            }
            gbytes[g] = 4 * wb;
            wmax = std::max(wmax, wb);
        }
        D->code_bytes = 2 * G * nsub8;                  /* a multiple of 16 */
        D->code_word = wmax;                            /* a multiple of 4 */
        D->zero_word = wmax + D->code_bytes / 4;
        D->stage_words = (D->zero_word + dd::DM_P + 31) / 32 * 32;
        const long long room = (long long)max_optin - 1024;   /* static barriers */
        D->nstage = (int)std::min<long long>(dd::DM_MAXST, room / (4LL * D->stage_words));
        if (D->nstage >= 2 && D->zero_word < 65536) break;
    }
    D->G = std::max(G, 0);
    D->ngroups = G > 0 ? (ndm + G - 1) / G : 0;
    D->nsub8 = nsub8;
    if (G > 0) {
        code.assign((size_t)D->ngroups * G * nsub8, (uint16_t)D->zero_word);
        for (int g = 0; g < D->ngroups; g++)
            for (int dl = 0; dl < G && g * G + dl < ndm; dl++)
                for (int s = 0; s < nsub; s++) {
                    const int4 w = win[(size_t)g * nsub + s];
                    const int rel = offsets[(size_t)(g * G + dl) * nsub + s] - w.x;
                    code[((size_t)g * G + dl) * nsub8 + s] = (uint16_t)(w.y + rel);
                }
    }
    /* the clipped DM stage's tables: as above with float windows of
     * FD_T + the group's offset spread (the warp-specialised kernel), for
     * the largest G of 32, 16, ..., 1 whose stages fit twice */
    std::vector<int4> fwin2;
    std::vector<uint16_t> fcode;
    std::vector<int> fgbytes;
    {
        int FGs = dd::DM_G;
        for (; FGs >= 1; FGs /= 2) {
            const int ng = (ndm + FGs - 1) / FGs;
            fwin2.assign((size_t)ng * nsub, make_int4(0, 0, 0, 0));
            fgbytes.assign(ng, 0);
            int wmax = 0;
            for (int g = 0; g < ng; g++) {
                int wb = 0;
                for (int s = 0; s < nsub; s++) {
                    int omin = 1 << 30, omax = 0;
                    for (int dl = 0; dl < FGs && g * FGs + dl < ndm; dl++) {
                        omin = std::min(omin, offsets[(size_t)(g * FGs + dl) * nsub + s]);
                        omax = std::max(omax, offsets[(size_t)(g * FGs + dl) * nsub + s]);
                    }
                    const int start = omin & ~3;
                    const int n = (omax - start + dd::FD_T + 3) / 4 * 4;
                    fwin2[(size_t)g * nsub + s] = make_int4(start, wb, n, 0);
                    wb += n;
                }
                fgbytes[g] = 4 * wb;
                wmax = std::max(wmax, wb);
            }
            D->fcode_bytes = 2 * FGs * nsub8;
            D->fcode_word = wmax;
            D->fstage_words = (wmax + D->fcode_bytes / 4 + 31) / 32 * 32;
            const long long room = (long long)max_optin - 1024;
            D->fnstage = (int)std::min<long long>(dd::DM_MAXST, room / (4LL * D->fstage_words));
            if (D->fnstage >= 2 && D->fcode_word < 65536) break;
        }
        D->fG = std::max(FGs, 0);
        D->fngroups = D->fG > 0 ? (ndm + D->fG - 1) / D->fG : 0;
        if (D->fG > 0) {
            fcode.assign((size_t)D->fngroups * D->fG * nsub8, 0);
            for (int g = 0; g < D->fngroups; g++)
                for (int dl = 0; dl < D->fG && g * D->fG + dl < ndm; dl++)
                    for (int s = 0; s < nsub; s++) {
                        const int4 w = fwin2[(size_t)g * nsub + s];
                        const int rel = offsets[(size_t)(g * D->fG + dl) * nsub + s] - w.x;
                        fcode[((size_t)g * D->fG + dl) * nsub8 + s] = (uint16_t)(w.y + rel);
                    }
        }
    }
    if (sb_smem(D, 1) > max_optin) {
        fprintf(stderr, "Error: cs_dedisp_create: channel delays of %d samples need more "
                        "shared memory than a CTA has\n", halo);
        dd_release(D);
        return nullptr;
    }
    /* S is read up to (tiles * DM_TILE) + maxoff + a few words beyond */
    const long long ntile = (max_spectra + dd::DM_TILE - 1) / dd::DM_TILE;
    D->sstride = ((ntile + 1) * dd::DM_TILE + maxoff + 64 + 255) / 256 * 256;
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
        DDCK(cudaMalloc((void **)&D->d_code, sizeof(uint16_t) * code.size()));
        DDCK(cudaMemcpy(D->d_code, code.data(), sizeof(uint16_t) * code.size(),
                        cudaMemcpyHostToDevice));
        DDCK(cudaMalloc((void **)&D->d_win, sizeof(int4) * win.size()));
        DDCK(cudaMemcpy(D->d_win, win.data(), sizeof(int4) * win.size(), cudaMemcpyHostToDevice));
        DDCK(cudaMalloc((void **)&D->d_gbytes, sizeof(int) * gbytes.size()));
        DDCK(cudaMemcpy(D->d_gbytes, gbytes.data(), sizeof(int) * gbytes.size(),
                        cudaMemcpyHostToDevice));
    }
    if (D->fG > 0) {
        DDCK(cudaMalloc((void **)&D->d_fcode, sizeof(uint16_t) * fcode.size()));
        DDCK(cudaMemcpy(D->d_fcode, fcode.data(), sizeof(uint16_t) * fcode.size(),
                        cudaMemcpyHostToDevice));
        DDCK(cudaMalloc((void **)&D->d_fwin2, sizeof(int4) * fwin2.size()));
        DDCK(cudaMemcpy(D->d_fwin2, fwin2.data(), sizeof(int4) * fwin2.size(),
                        cudaMemcpyHostToDevice));
        DDCK(cudaMalloc((void **)&D->d_fgbytes, sizeof(int) * fgbytes.size()));
        DDCK(cudaMemcpy(D->d_fgbytes, fgbytes.data(), sizeof(int) * fgbytes.size(),
                        cudaMemcpyHostToDevice));
        DDCK(cudaFuncSetAttribute(dd::dd_dms_f32_ws, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  4 * D->fnstage * D->fstage_words));
    }
    DDCK(cudaMalloc((void **)&D->d_err, sizeof(int)));
    DDCK(cudaMemset(D->d_err, 0, sizeof(int)));
    /* S: word w of a row holds samples w and w + DM_P; cleared once, so the
     * high halves past the filled samples are zeros rather than stale bytes */
    DDCK(cudaMalloc((void **)&D->d_sub, sizeof(uint32_t) * (size_t)nsub * D->sstride));
    DDCK(cudaMemset(D->d_sub, 0, sizeof(uint32_t) * (size_t)nsub * D->sstride));
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
                                  4 * D->nstage * D->stage_words));
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
    const long long ntile_dm = (nout + dd::DM_TILE - 1) / dd::DM_TILE;
    const long long sfill = std::min(D->sstride, ntile_dm * dd::DM_TILE + D->maxoff + 64);
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
    cudaError_t e = cudaMemsetAsync(D->d_err, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
    cudaEventRecord(D->ev0, st);
    if (clip)
        dd::dd_subband_clip<<<gs, dd::SB_THREADS, sb_smem(D, slab, true), st>>>(sa);
    else
        dd::dd_subband_u8<<<gs, dd::SB_THREADS, sb_smem(D, slab), st>>>(sa);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (clip && D->fG > 0 && !getenv("CS_B200_DEDISP_ROUNDS")) {
        dd::FdArgs fa;
        memset(&fa, 0, sizeof(fa));
        fa.sub = D->d_subf;
        fa.sstride = D->sstride;
        fa.nsub = D->nsub;
        fa.nsub8 = D->nsub8;
        fa.ndm = D->ndm;
        fa.G = D->fG;
        fa.ngroups = D->fngroups;
        fa.win = D->d_fwin2;
        fa.code = D->d_fcode;
        fa.gbytes = D->d_fgbytes;
        fa.code_bytes = D->fcode_bytes;
        fa.code_word = D->fcode_word;
        fa.stage_words = D->fstage_words;
        fa.nstage = D->fnstage;
        fa.nitems = (nout + dd::FD_T - 1) / dd::FD_T * D->fngroups;
        fa.nout = nout;
        fa.out = d_out;
        fa.ostride = ostride;
        fa.err = D->d_err;
        int nsm = 0;
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, D->device);
        const long long grid = std::min<long long>(fa.nitems, nsm);
        cudaEventRecord(D->ev1, st);
        dd::dd_dms_f32_ws<<<(unsigned)grid, dd::FD_THREADS, 4 * D->fnstage * D->fstage_words, st>>>(fa);
        cudaEventRecord(D->ev2, st);
        return cudaGetLastError();
    }
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
    memset(&da, 0, sizeof(da));
    da.sub = D->d_sub;
    da.sstride = D->sstride;
    da.nsub = D->nsub;
    da.nsub8 = D->nsub8;
    da.ndm = D->ndm;
    da.G = D->G;
    da.ngroups = D->ngroups;
    da.offs = D->d_offs;
    da.flush = D->flush;
    da.win = D->d_win;
    da.code = D->d_code;
    da.gbytes = D->d_gbytes;
    da.code_bytes = D->code_bytes;
    da.code_word = D->code_word;
    da.zero_word = D->zero_word;
    da.stage_words = D->stage_words;
    da.nstage = D->nstage;
    da.nitems = ntile_dm * D->ngroups;
    da.nout = nout;
    da.out = d_out;
    da.ostride = ostride;
    da.err = D->d_err;
    cudaEventRecord(D->ev1, st);
    if (D->G > 0) {
        int nsm = 0;
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, D->device);
        const long long grid = std::min<long long>(da.nitems, nsm);
        dd::dd_dms_u16<<<(unsigned)grid, dd::DM_THREADS, 4 * D->nstage * D->stage_words, st>>>(da);
    } else {
        dim3 gd((unsigned)((nout + 255) / 256), (unsigned)D->ndm);
        dd::dd_dms_u16_direct<<<gd, 256, 0, st>>>(da);
    }
    cudaEventRecord(D->ev2, st);
    return cudaGetLastError();
}

/* 0, or -1 (with a message) if a wait of the last DM stage gave up; waits
 * for the stream's work first. */
static int dd_check(CsDedisp *D, cudaStream_t st, const char *who)
{
    int flag = 0;
    if (cudaMemcpyAsync(&flag, D->d_err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        fprintf(stderr, "Error: %s: %s\n", who, cudaGetErrorString(cudaGetLastError()));
        return -1;
    }
    if (flag) {
        fprintf(stderr, "Error: %s: a DM-stage wait gave up (pipeline stalled)\n", who);
        return -1;
    }
    return 0;
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
    /* the rounds kernel (geometries whose windows the warp-specialised one
     * cannot stage twice) has its limits */
    const bool rounds = D->fG == 0 || getenv("CS_B200_DEDISP_ROUNDS");
    if (rounds && (unsigned long long)((nout + dd::FT - 1) / dd::FT) *
                          (unsigned long long)((D->ndm + dd::FG - 1) / dd::FG) >= (1ULL << 31)) {
        fprintf(stderr, "Error: cs_dedisp_run_device_clipped: %lld points x %d DMs is too many "
                        "for one launch\n", nout, D->ndm);
        return -1;
    }
    if (rounds && dd_clip_rounds(D) < 1) {
        fprintf(stderr, "Error: cs_dedisp_run_device_clipped: subband windows of %d samples "
                        "(%d subbands) need more shared memory than a CTA has\n", D->fwmax,
                D->nsub);
        return -1;
    }
    if (cudaSetDevice(D->device) != cudaSuccess) return -1;
    cudaError_t e = cudaSuccess;
    if (!D->d_subf) {
        /* cleared once: staged samples past the filled ones are zeros */
        e = cudaMalloc((void **)&D->d_subf, sizeof(float) * (size_t)D->nsub * D->sstride);
        if (e == cudaSuccess)
            e = cudaMemset(D->d_subf, 0, sizeof(float) * (size_t)D->nsub * D->sstride);
    }
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
    if (dd_check(D, D->st, "cs_dedisp_run") != 0) return -1;
    if (nout_written) *nout_written = nout;
    return 0;
}

/* Kernel times of the last run (subband stage, DM stage), from CUDA events
 * recorded around the two launches on the run's stream. */
CS_EXPORT int cs_dedisp_last_times(CsDedisp *D, float *subband_ms, float *dm_ms)
{
    if (!D) return -1;
    if (cudaEventSynchronize(D->ev2) != cudaSuccess) return -1;
    if (dd_check(D, D->st, "cs_dedisp_last_times") != 0) return -1;
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
