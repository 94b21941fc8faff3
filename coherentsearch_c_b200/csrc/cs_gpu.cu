/*
 * B200 (sm_100a) backend for the coherent harmonic-sum search.
 *
 * Drop-in replacement for the reference GPU backend (src/cuda.cu and the
 * no-CUDA stub src/gpu_stub.c): it exports the same cs_gpu_* C ABI
 * (include/coherent_search.h:436-460) and returns the same candidates.  The
 * reference runs, per chunk of trials, four launches (zero-columns,
 * interpolation, cuFFT c2r, metric) plus cuFFT + metric per non-divisor
 * decimation, with the profiles round-tripping through global memory.  Here a
 * single persistent kernel does all of it per 128-trial tile, on chip:
 *
 *   1. interpolation (src/cuda.cu:86-140, src/interp.c:608-824): each thread
 *      evaluates the m-tap sinc interpolation of 4 consecutive harmonics of
 *      one trial with the reference's exact FP32 FMA chain and rotation, so
 *      the harmonic amplitudes are bit-identical to the reference's;
 *   2. the c2r profile transform (cuFFT C2R in the reference) as a dense
 *      [128 trials x 2*nharms] x [2*nharms x bins] contraction on the
 *      5th-generation tensor cores (tcgen05.mma kind::f16, accumulator in
 *      tensor memory) with a 3-term fp16 split of both operands (hi*hi +
 *      lo*hi + hi*lo) and a per-run power-of-two scale, which keeps ~22
 *      significant bits -- FP32-class accuracy;  non-divisor decimations are
 *      extra output columns of the same MMA;
 *   3. the boxcar matched filter (src/cuda.cu:164-278, src/boxcar.c:203-252)
 *      and the k | nharms folds (src/search.c:294-400) read the accumulator
 *      with tcgen05.ld, in the reference's FP32 expression order;
 *   4. threshold + warp-ballot compaction of candidate records into a
 *      device-resident buffer; the host sorts them into the reference's
 *      (chunk, slot, trial) order and applies its FP64 frequency arithmetic.
 *
 * Every wait in the kernel is bounded (an mbarrier poll with a wall-clock
 * limit); on expiry the kernel records an error, frees its tensor memory and
 * returns, and the host reports the failure instead of hanging.
 */
#include <cuda.h>              /* CUtensorMap and its enums (types only) */
#include <cuda_runtime.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "cs_internal.h"
#include "cs_b200.h"

#define CS_EXPORT extern "C" __attribute__((visibility("default")))

#define CS_NTHREADS 256
#define CS_WAIT_NS 2000000000ull  /* 2 s bound on any in-kernel wait */
#ifndef CS_MBAR_SLEEP_NS
#define CS_MBAR_SLEEP_NS 64       /* back-off between polls of an mbarrier */
#endif

/* ------------------------------------------------------------------ */
/* Kernel arguments                                                   */
/* ------------------------------------------------------------------ */
struct SearchArgs {
    const float2 *amps;
    long long namps;
    const CsHarm *harm;
    const uint16_t *rowtab;
    const float *W;
    const float2 *A;
    const uint8_t *carry;
    const CsChunk *chunks;
    const int *tiles;
    int ntiles;
    const uint4 *bimg;          /* B hi image then B lo image */
    int bbytes;                 /* bytes of one B image */
    int nh, m, q, pnum;
    unsigned qmagic;
    int kpad, npad, ncols_tmem;
    int nslot;
    CsSlot slot[CS_MAX_SLOT];
    float gbound;
    const unsigned *amax;       /* [0]: max |component| bits, [1]: non-finite flag */
    double thresh;
    CsRec *recs;
    unsigned *count;
    unsigned cap;
    int *err;
};

/* ------------------------------------------------------------------ */
/* PTX helpers (tcgen05, mbarrier, proxy fences)                       */
/* ------------------------------------------------------------------ */
static __device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

static __device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(bar), "r"(count));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

static __device__ __forceinline__ uint32_t mbar_try(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
    return ok;
}

static __device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

/* Bounded wait for the phase with the given parity to complete. */
static __device__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
    if (mbar_try(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (!mbar_try(bar, parity)) {
        if (global_ns() - t0 > CS_WAIT_NS) return false;
#if CS_MBAR_SLEEP_NS > 0
        __nanosleep(CS_MBAR_SLEEP_NS);   /* leave the issue slots to the working warps */
#endif
    }
    return true;
}

static __device__ __forceinline__ void fence_proxy_async()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
static __device__ __forceinline__ void tc_fence_before()
{
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
static __device__ __forceinline__ void tc_fence_after()
{
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

static __device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(dst_smem), "r"(ncols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
static __device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                 :: "r"(taddr), "r"(ncols) : "memory");
}

/* D[tmem] (+)= A[smem] * B[smem]^T, 128 x N x 16, fp16 in, fp32 accumulate. */
static __device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t adesc,
                                               uint64_t bdesc, uint32_t idesc,
                                               uint32_t accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                 :: "r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
                 : "memory");
}
static __device__ __forceinline__ void mma_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(bar) : "memory");
}

/* 32 consecutive accumulator columns of this warp's 32 lanes. */
static __device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *v)
{
    uint32_t r[32];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                 "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                 "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                   "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                   "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
                   "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                   "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]),
                   "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

/* 16 consecutive accumulator columns of this warp's 32 lanes. */
static __device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v)
{
    uint32_t r[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                 "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                   "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                   "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

/* Shared-memory matrix descriptor, canonical K-major layout without swizzle:
 * 8-row x 16-byte core matrices; lbo = byte distance between the two K
 * halves of one MMA (adjacent K core matrices), sbo = between 8-row groups. */
static __device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;                 /* descriptor version for sm_100 */
    return d;                                /* base offset 0, no swizzle */
}

/* floor(u / q) and u mod q for q >= 2 with a precomputed 32-bit multiplier
 * floor(2^32/q)+1 (the estimate is exact or one too large). */
static __device__ __forceinline__ void divmod_q(uint32_t u, uint32_t q, uint32_t magic,
                                                uint32_t &quo, uint32_t &rem)
{
    if (q == 1) { quo = u; rem = 0; return; }
    uint32_t e = __umulhi(u, magic);
    uint32_t pr = e * q;
    if (pr > u) { e -= 1; pr -= q; }
    quo = e;
    rem = u - pr;
}

/* ------------------------------------------------------------------ */
/* Spectrum magnitude bound -> fp16 operand scale                      */
/* ------------------------------------------------------------------ */
__global__ void cs_amax_kernel(const float2 *__restrict__ amps, long long namps,
                               unsigned *__restrict__ out)
{
    float mx = 0.0f;
    unsigned bad = 0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < namps;
         i += (long long)gridDim.x * blockDim.x) {
        const float2 a = amps[i];
        const float v = fmaxf(fabsf(a.x), fabsf(a.y));
        if (!(v <= 3.0e38f)) bad = 1;       /* NaN or Inf */
        mx = fmaxf(mx, v);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        bad |= __shfl_xor_sync(0xffffffffu, bad, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&out[0], __float_as_uint(mx));
        if (bad) atomicOr(&out[1], 1u);
    }
}

/* 2^e with e chosen so that gbound * amax * 2^e <= 2^14 (fp16 max 65504). */
static __device__ float operand_scale(const unsigned *amax, float gbound)
{
    const float a = __uint_as_float(amax[0]);
    if (amax[1] != 0u || !(a > 0.0f)) return 1.0f;
    const float bound = a * gbound;
    if (!(bound > 0.0f) || !(bound < 3.0e38f)) return 1.0f;
    int e;
    frexpf(bound, &e);                      /* bound in [2^(e-1), 2^e) */
    int s = 14 - e;
    s = max(-100, min(100, s));
    return ldexpf(1.0f, s);
}

/* ------------------------------------------------------------------ */
/* The fused search kernel                                             */
/* ------------------------------------------------------------------ */
struct SmemLayout {
    int b_off, a_off, ps_off, rk_off, bar_off, tm_off, total;
};

static __host__ __device__ inline int cs_align(int x, int a) { return (x + a - 1) / a * a; }

/* B images | A images (aliased by the epilogue scratch) | barrier | tmem slot */
static __host__ __device__ inline SmemLayout smem_layout(int npad, int kpad, int nbmax, int wmaxmax,
                                                          int nkfold)
{
    SmemLayout L;
    const int bimg = npad * kpad * 2;
    const int aimg = CS_TILE_M * kpad * 2;
    L.b_off = 0;
    L.a_off = cs_align(2 * bimg, 1024);
    const int ps_bytes = (nbmax + wmaxmax + 1) * CS_TILE_M * 4;
    const int rk_bytes = nkfold * CS_TILE_M * 4;
    L.ps_off = L.a_off;
    L.rk_off = L.ps_off + cs_align(ps_bytes, 128);
    const int epi_end = L.rk_off + rk_bytes;
    const int a_end = L.a_off + 2 * aimg;
    L.bar_off = cs_align(epi_end > a_end ? epi_end : a_end, 16);
    L.tm_off = L.bar_off + 16;
    L.total = L.tm_off + 16;
    return L;
}

/* Maximum of the sliding-window sums for every width, then the reference
 * metric max_w (M_w - duty_w * total) * invsw_w (src/boxcar.c:213-231). */
static __device__ __forceinline__ float scan_widths(const float *ps, int row, int nk,
                                                    const CsSlot &s, const float *invsw)
{
    float mx[CS_NWMAX];
#pragma unroll
    for (int w = 0; w < CS_NWMAX; w++) mx[w] = -INFINITY;
    for (int p = 1; p <= nk; p++) {
        const float base = ps[(p - 1) * CS_TILE_M + row];
#pragma unroll
        for (int w = 0; w < CS_NWMAX; w++) {
            if (w < s.nw) {
                const float d = __fsub_rn(ps[(p - 1 + s.widths[w]) * CS_TILE_M + row], base);
                mx[w] = fmaxf(mx[w], d);
            }
        }
    }
    const float tot = __fsub_rn(ps[nk * CS_TILE_M + row], ps[row]);
    float best = -INFINITY;
#pragma unroll
    for (int w = 0; w < CS_NWMAX; w++) {
        if (w < s.nw) {
            const float c = __fmul_rn(__fsub_rn(mx[w], __fmul_rn(s.duty[w], tot)), invsw[w]);
            best = fmaxf(best, c);
        }
    }
    return best;
}

/* The m-tap interpolation of harmonic h of the trial with t*pnum = Q*q + R,
 * rotated by its phase factor (src/cuda.cu:86-140): the reference's FP32 FMA
 * chain in tap order, then the unfused rotation, so the amplitude is
 * bit-identical to the reference's.  Taps outside the spectrum read zero. */
template <int MT>
static __device__ __forceinline__ float2 interp_amp(const SearchArgs &args, const CsHarm &hm,
                                                    int h, int m, long long Q, uint32_t R)
{
    uint32_t qd, res;
    divmod_q((uint32_t)h * R, (uint32_t)args.q, args.qmagic, qd, res);
    const long long qint = (long long)h * Q + qd;
    const int ph = args.rowtab[(size_t)(h - 1) * args.q + res];
    const int row = hm.woff + ph;
    const long long base = hm.rfloor0 + qint + args.carry[row];
    const long long b0 = base + 1 - m / 2;
    const float *wr = args.W + (size_t)row * m;
    float ar = 0.0f, ai = 0.0f;
    if (b0 >= 0 && b0 + m <= args.namps) {
        const float2 *ap = args.amps + b0;
        if (MT) {
#pragma unroll
            for (int i = 0; i < (MT ? MT : 1); i += 4) {
                const float4 w4 = __ldg(reinterpret_cast<const float4 *>(wr + i));
                const float2 a0 = __ldg(ap + i), a1 = __ldg(ap + i + 1);
                const float2 a2 = __ldg(ap + i + 2), a3 = __ldg(ap + i + 3);
                ar = __fmaf_rn(w4.x, a0.x, ar); ai = __fmaf_rn(w4.x, a0.y, ai);
                ar = __fmaf_rn(w4.y, a1.x, ar); ai = __fmaf_rn(w4.y, a1.y, ai);
                ar = __fmaf_rn(w4.z, a2.x, ar); ai = __fmaf_rn(w4.z, a2.y, ai);
                ar = __fmaf_rn(w4.w, a3.x, ar); ai = __fmaf_rn(w4.w, a3.y, ai);
            }
        } else {
            for (int i = 0; i < m; i++) {
                const float w = __ldg(wr + i);
                const float2 a = __ldg(ap + i);
                ar = __fmaf_rn(w, a.x, ar);
                ai = __fmaf_rn(w, a.y, ai);
            }
        }
    } else {
        for (int i = 0; i < m; i++) {
            const long long idx = b0 + i;
            float2 a = make_float2(0.0f, 0.0f);
            if (idx >= 0 && idx < args.namps) a = __ldg(args.amps + idx);
            const float w = __ldg(wr + i);
            ar = __fmaf_rn(w, a.x, ar);
            ai = __fmaf_rn(w, a.y, ai);
        }
    }
    const float2 g = __ldg(args.A + row);
    return make_float2(__fsub_rn(__fmul_rn(g.x, ar), __fmul_rn(g.y, ai)),
                       __fadd_rn(__fmul_rn(g.x, ai), __fmul_rn(g.y, ar)));
}

template <int MT>
__global__ void __launch_bounds__(CS_NTHREADS, 1)
cs_search_kernel(const SearchArgs args)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int lane = tid & 31;
    const int nh = args.nh;
    const int kpad = args.kpad, npad = args.npad;
    const int m = MT ? MT : args.m;

    int nbmax = 2 * nh, wmaxmax = 0, nkfold = 0;
    for (int s = 0; s < args.nslot; s++) {
        nbmax = max(nbmax, args.slot[s].nk);
        wmaxmax = max(wmaxmax, args.slot[s].wmax);
        if (args.slot[s].fold) nkfold = max(nkfold, args.slot[s].nk);
    }
    const SmemLayout L = smem_layout(npad, kpad, nbmax, wmaxmax, nkfold);
    unsigned char *bsm = smem + L.b_off;
    unsigned char *asm_ = smem + L.a_off;
    float *ps = reinterpret_cast<float *>(smem + L.ps_off);
    float *rk = reinterpret_cast<float *>(smem + L.rk_off);
    const uint32_t bar = smem_u32(smem + L.bar_off);
    uint32_t *tm_slot = reinterpret_cast<uint32_t *>(smem + L.tm_off);
    __shared__ CsHarm harm_s[CS_MAX_NH];

    if (warp == 0) tmem_alloc(smem_u32(tm_slot), (uint32_t)args.ncols_tmem);
    if (tid == 0) mbar_init(bar, 1);
    for (int h = tid; h < nh; h += blockDim.x) harm_s[h] = args.harm[h];
    {   /* both B images, verbatim */
        const int n16 = (2 * args.bbytes) / 16;
        uint4 *dst = reinterpret_cast<uint4 *>(bsm);
        for (int i = tid; i < n16; i += blockDim.x) dst[i] = args.bimg[i];
    }
    fence_proxy_async();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tm_slot;
    const float scale = operand_scale(args.amax, args.gbound);
    const float inv_scale = 1.0f / scale;    /* exact: power of two */

    const int bimg = args.bbytes;
    const int aimg = CS_TILE_M * kpad * 2;
    const uint32_t a_hi = smem_u32(asm_), a_lo = a_hi + (uint32_t)aimg;
    const uint32_t b_hi = smem_u32(bsm), b_lo = b_hi + (uint32_t)bimg;
    const uint32_t lbo_a = CS_TILE_M * 16, lbo_b = (uint32_t)npad * 16;
    const uint32_t idesc = (1u << 4) | ((uint32_t)(npad >> 3) << 17) | ((uint32_t)(CS_TILE_M >> 4) << 24);
    const int nhb = (nh + 3) / 4;
    uint32_t phase = 0;
    bool ok = true;

    for (int tile = blockIdx.x; tile < args.ntiles && ok; tile += gridDim.x) {
        const int ci = args.tiles[3 * tile + 0];
        const int j0 = args.tiles[3 * tile + 1];
        const int cnt = args.tiles[3 * tile + 2];
        const CsChunk &ch = args.chunks[ci];
        const unsigned long long filled = ch.filled;

        /* ---- 1. interpolation into the A operand (hi, lo) ---- */
        {
            const int r = tid & (CS_TILE_M - 1);
            const int par = tid >> 7;
            const bool valid = r < cnt;
            const long long t = ch.i0 + j0 + r;
            const long long tp = t * (long long)args.pnum;
            const long long Q = tp / args.q;
            const uint32_t R = (uint32_t)(tp - Q * args.q);
            for (int hb = par; hb < nhb; hb += 2) {
                uint32_t hi_w[4], lo_w[4];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const int h = 4 * hb + u + 1;
                    float xr = 0.0f, xi = 0.0f;
                    if (valid && h <= nh && ((filled >> (h - 1)) & 1ULL)) {
                        const float2 x = interp_amp<MT>(args, harm_s[h - 1], h, m, Q, R);
                        xr = x.x;
                        xi = x.y;
                    }
                    /* split the scaled amplitude into fp16 hi + lo */
                    const float sr = xr * scale, si = xi * scale;
                    const __half hr = __float2half_rn(sr), hi_ = __float2half_rn(si);
                    const __half lr = __float2half_rn(__fsub_rn(sr, __half2float(hr)));
                    const __half li = __float2half_rn(__fsub_rn(si, __half2float(hi_)));
                    hi_w[u] = (uint32_t)__half_as_ushort(hr) | ((uint32_t)__half_as_ushort(hi_) << 16);
                    lo_w[u] = (uint32_t)__half_as_ushort(lr) | ((uint32_t)__half_as_ushort(li) << 16);
                }
                /* K block hb holds harmonics 4hb+1..4hb+4 (Re, Im interleaved) */
                const uint32_t off = (uint32_t)hb * (CS_TILE_M * 16) + (uint32_t)(r >> 3) * 128 + (uint32_t)(r & 7) * 16;
                *reinterpret_cast<uint4 *>(asm_ + off) = make_uint4(hi_w[0], hi_w[1], hi_w[2], hi_w[3]);
                *reinterpret_cast<uint4 *>(asm_ + aimg + off) = make_uint4(lo_w[0], lo_w[1], lo_w[2], lo_w[3]);
            }
            /* zero K blocks past 2*nh (kpad padding) */
            for (int hb = nhb + par; hb < kpad / 8; hb += 2) {
                const uint32_t off = (uint32_t)hb * (CS_TILE_M * 16) + (uint32_t)(r >> 3) * 128 + (uint32_t)(r & 7) * 16;
                *reinterpret_cast<uint4 *>(asm_ + off) = make_uint4(0, 0, 0, 0);
                *reinterpret_cast<uint4 *>(asm_ + aimg + off) = make_uint4(0, 0, 0, 0);
            }
        }
        fence_proxy_async();
        __syncthreads();

        /* ---- 2. tensor-core c2r: D = Ahi*Bhi + Alo*Bhi + Ahi*Blo ---- */
        tc_fence_after();
        if (tid == 0) {
            const int ksteps = kpad / 16;
            uint32_t acc = 0;
            for (int pass = 0; pass < 3; pass++) {
                const uint32_t abase = (pass == 1) ? a_lo : a_hi;
                const uint32_t bbase = (pass == 2) ? b_lo : b_hi;
                for (int s = 0; s < ksteps; s++) {
                    const uint64_t ad = umma_desc(abase + (uint32_t)s * 2 * lbo_a, lbo_a, 128);
                    const uint64_t bd = umma_desc(bbase + (uint32_t)s * 2 * lbo_b, lbo_b, 128);
                    mma_f16(tmem, ad, bd, idesc, acc);
                    acc = 1;
                }
            }
            mma_commit(bar);
        }
        {
            const bool done = mbar_wait(bar, phase);
            if (!done && lane == 0) atomicExch(args.err, 1);
            ok = __syncthreads_and(done) != 0;
        }
        if (!ok) {
            /* give the outstanding MMAs one more bounded wait before the
             * tensor memory they write is released */
            mbar_wait(bar, phase);
            break;
        }
        phase ^= 1u;
        tc_fence_after();

        /* ---- 3. boxcar metrics (warps 0-3 own TMEM lanes 0-127) ---- */
        if (ok && warp < 4) {
            const int r = warp * 32 + lane;
            const bool valid = r < cnt;
            const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
            float best[CS_MAX_SLOT];
            const int nb = 2 * nh;
            float v[32];
            for (int s = 0; s < args.nslot; s++) {
                const CsSlot &sl = args.slot[s];
                const int nk = sl.nk;
                float p = 0.0f;
                ps[r] = 0.0f;
                if (!sl.fold) {
                    /* profile columns col0 .. col0+nk-1, then the wrap */
                    for (int c0 = 0; c0 < nk; c0 += 32) {
                        tmem_ld32(trow + (uint32_t)(sl.col0 + c0), v);
#pragma unroll
                        for (int u = 0; u < 32; u++) {
                            if (c0 + u < nk) {
                                p = __fadd_rn(p, v[u] * inv_scale);
                                ps[(c0 + u + 1) * CS_TILE_M + r] = p;
                            }
                        }
                    }
                    for (int c0 = 0; c0 < sl.wmax; c0 += 32) {
                        tmem_ld32(trow + (uint32_t)(sl.col0 + c0), v);
#pragma unroll
                        for (int u = 0; u < 32; u++) {
                            if (c0 + u < sl.wmax) {
                                p = __fadd_rn(p, v[u] * inv_scale);
                                ps[(nk + c0 + u + 1) * CS_TILE_M + r] = p;
                            }
                        }
                    }
                } else {
                    /* r_k[j] = (x[j] + x[j+nk] + ...) * (1/k), then prefix */
                    int jj = 0;
                    for (int c0 = 0; c0 < nb; c0 += 32) {
                        tmem_ld32(trow + (uint32_t)c0, v);
#pragma unroll
                        for (int u = 0; u < 32; u++) {
                            const int i = c0 + u;
                            if (i < nb) {
                                const float x = v[u] * inv_scale;
                                if (i < nk) rk[jj * CS_TILE_M + r] = x;
                                else rk[jj * CS_TILE_M + r] = __fadd_rn(rk[jj * CS_TILE_M + r], x);
                                jj = (jj + 1 == nk) ? 0 : jj + 1;
                            }
                        }
                    }
                    const float invk = 1.0f / (float)sl.k;
                    for (int j = 0; j < nk; j++) {
                        const float x = __fmul_rn(rk[j * CS_TILE_M + r], invk);
                        p = __fadd_rn(p, x);
                        ps[(j + 1) * CS_TILE_M + r] = p;
                    }
                    for (int u = 0; u < sl.wmax; u++) {
                        const float x = __fmul_rn(rk[u * CS_TILE_M + r], invk);
                        p = __fadd_rn(p, x);
                        ps[(nk + u + 1) * CS_TILE_M + r] = p;
                    }
                }
                best[s] = scan_widths(ps, r, nk, sl, ch.invsw[s]);
            }
            /* ---- 4. threshold + warp-aggregated compaction ---- */
            const int j = j0 + r;
            for (int s = 0; s < args.nslot; s++) {
                const bool hit = valid && j < ch.nvalid[s] && (double)best[s] > args.thresh;
                const unsigned mask = __ballot_sync(0xffffffffu, hit);
                if (mask) {
                    unsigned basei = 0;
                    if (lane == 0) basei = atomicAdd(args.count, (unsigned)__popc(mask));
                    basei = __shfl_sync(0xffffffffu, basei, 0);
                    if (hit) {
                        const unsigned pos = basei + (unsigned)__popc(mask & ((1u << lane) - 1u));
                        if (pos < args.cap) {
                            CsRec rec;
                            rec.chunk = ci;
                            rec.slot = s;
                            rec.j = j;
                            rec.metric = best[s];
                            args.recs[pos] = rec;
                        }
                    }
                }
            }
        }
        tc_fence_before();
        __syncthreads();
    }

    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, (uint32_t)args.ncols_tmem);
    }
}

#include "cs_search_ws.cuh"
#include "cs_interp_tc.cuh"
#include "cs_search_tma.cuh"
#include "cs_search_f64.cuh"
#include "cs_collapse.h"

/* ------------------------------------------------------------------ */
/* Host side                                                          */
/* ------------------------------------------------------------------ */
#define CK(call)                                                               \
    do {                                                                       \
        cudaError_t e_ = (call);                                               \
        if (e_ != cudaSuccess) {                                               \
            fprintf(stderr, "Error: CUDA %s failed: %s (%s:%d)\n", #call,       \
                    cudaGetErrorString(e_), __FILE__, __LINE__);               \
            goto fail;                                                         \
        }                                                                      \
    } while (0)

struct GpuSession {
    const SearchParams *p;
    int device;
    int Nprof;
    long long total, nchunks;
    long long N, namps;
    double T, r_lo, lodr;
    CsTables tab;
    int max_smem;
    int nsm;
    cudaStream_t st;
    cudaEvent_t ev0, ev1;
    cudaEvent_t ev_in;        /* producer hand-off (enqueue_device's stream) */
    /* device buffers */
    float2 *d_amps;
    CsHarm *d_harm;
    uint16_t *d_rowtab;
    float *d_W;
    float2 *d_A;
    uint8_t *d_carry;
    CsChunk *d_chunks;
    int *d_tiles;
    uint4 *d_bimg;
    int bbytes;
    /* what d_bimg holds: the DFT images depend on the harmonic count and the
     * slot layout only, so a reload with the same layout keeps them */
    bool img_ok;
    int img_nh, img_nslot, img_npad, img_kpad;
    CsSlot img_slot[CS_MAX_SLOT];
    unsigned *d_amax;      /* [2] */
    unsigned *d_count;     /* [1] */
    int *d_err;            /* [1] */
    CsRec *d_recs;
    unsigned cap;
    unsigned *h_count;     /* pinned */
    CsRec *h_recs;         /* pinned record staging, grown on demand */
    CsCollapse *coll;      /* device harvest + collapse scratch, on first use */
    size_t h_recs_cap;
    float last_kernel_ms;
    int own_plans;
    /* bumped whenever the tables or the record buffer may move (a reload, a
     * record buffer grown): a captured launch that baked in their addresses
     * checks it before each replay */
    unsigned gen;
    /* warp-specialised kernel (default ladder at nharms = 60) */
    int use_ws;
    float4 *d_Wt;
    float4 *d_AC;
    wsk::Harm *d_harm2;
    wsk::Harm hh[wsk::MAX_NH];
    /* column-tile kernel with TMA-staged windows (search_tma) */
    int use_tma;
    float *d_wtab;         /* weights by trial index */
    int *d_cchunk;         /* chunk of each column tile's first trial */
    CUtensorMap *d_maps;   /* [nh][2] */
    float2 *d_tc[2];       /* zero-padded spectrum copies (second shifted a bin) */
    size_t c_wtab, c_cchunk, c_tc;
    wsk::TArgs tx;
    /* interpolation as tensor-core GEMMs (tci::interp_tc), then search_pre */
    int use_tci;
    tci::Band *d_tci_bands;
    uint4 *d_tci_bimg;
    int *d_tci_hbase;
    float2 *d_X;
    size_t c_tci_bands, c_tci_bimg, c_X;
    int tci_nband;
    float tci_inv_sb;
    long long tci_xstride;
    /* FP64 search (p->precision == CS_PREC_F64) */
    int prec64;
    f64k::Extra fx;
    int f64_smem;
    double *d_bcs, *d_scales;
    CsRec64 *d_recs64;
    unsigned cap64;
    CsRec64 *h_recs64;     /* pinned record staging */
    size_t h_recs64_cap;
    /* capacities (bytes) of the buffers session_load may reuse */
    size_t c_amps, c_rowtab, c_W, c_A, c_carry, c_chunks, c_tiles, c_bimg, c_bcs, c_scales;
};

static cudaError_t select_device(int device)
{
    int cur = -1;
    cudaError_t e = cudaGetDevice(&cur);
    if (e == cudaSuccess && cur == device) return cudaSuccess;
    return cudaSetDevice(device);
}

CS_EXPORT int cs_gpu_available(int device, char *errbuf, size_t errlen)
{
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count <= 0) {
        if (errbuf) snprintf(errbuf, errlen, "no CUDA device available (%s)",
                             e != cudaSuccess ? cudaGetErrorString(e) : "0 devices");
        return -1;
    }
    if (device < 0 || device >= count) {
        if (errbuf) snprintf(errbuf, errlen, "CUDA device %d requested but %d device(s) present",
                             device, count);
        return -1;
    }
    e = select_device(device);
    if (e != cudaSuccess) {
        if (errbuf) snprintf(errbuf, errlen, "cannot select CUDA device %d: %s", device,
                             cudaGetErrorString(e));
        return -1;
    }
    cudaDeviceProp prop;
    e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) {
        if (errbuf) snprintf(errbuf, errlen, "cudaGetDeviceProperties failed: %s",
                             cudaGetErrorString(e));
        return -1;
    }
    if (prop.major != 10) {
        if (errbuf) snprintf(errbuf, errlen, "%s (device %d, cc %d.%d) is not an sm_100 "
                             "(B200-class) device", prop.name, device, prop.major, prop.minor);
        return -1;
    }
    if (errbuf) snprintf(errbuf, errlen, "%s (device %d, cc %d.%d)", prop.name, device,
                         prop.major, prop.minor);
    return 1;
}

static void session_release(GpuSession *S)
{
    if (!S) return;
    cudaFree(S->d_amps);
    cudaFree(S->d_harm);
    cudaFree(S->d_rowtab);
    cudaFree(S->d_W);
    cudaFree(S->d_A);
    cudaFree(S->d_carry);
    cudaFree(S->d_chunks);
    cudaFree(S->d_tiles);
    cudaFree(S->d_bimg);
    cudaFree(S->d_amax);
    cudaFree(S->d_count);
    cudaFree(S->d_err);
    cudaFree(S->d_recs);
    cudaFree(S->d_Wt);
    cudaFree(S->d_AC);
    cudaFree(S->d_harm2);
    cudaFree(S->d_wtab);
    cudaFree(S->d_cchunk);
    cudaFree(S->d_maps);
    cudaFree(S->d_tc[0]);
    cudaFree(S->d_tc[1]);
    cudaFree(S->d_tci_bands);
    cudaFree(S->d_tci_bimg);
    cudaFree(S->d_tci_hbase);
    cudaFree(S->d_X);
    cudaFree(S->d_bcs);
    cudaFree(S->d_scales);
    cudaFree(S->d_recs64);
    if (S->h_recs64) cudaFreeHost(S->h_recs64);
    if (S->h_count) cudaFreeHost(S->h_count);
    if (S->h_recs) cudaFreeHost(S->h_recs);
    cs_collapse_free(S->coll);
    if (S->ev0) cudaEventDestroy(S->ev0);
    if (S->ev1) cudaEventDestroy(S->ev1);
    if (S->ev_in) cudaEventDestroy(S->ev_in);
    if (S->st) cudaStreamDestroy(S->st);
    cs_tables_free(&S->tab);
    free(S);
}

static int smem_bytes(const CsTables &t)
{
    int nbmax = 2 * t.nh, wmaxmax = 0, nkfold = 0;
    for (int s = 0; s < t.nslot; s++) {
        nbmax = std::max(nbmax, t.slot[s].nk);
        wmaxmax = std::max(wmaxmax, t.slot[s].wmax);
        if (t.slot[s].fold) nkfold = std::max(nkfold, t.slot[s].nk);
    }
    return smem_layout(t.npad, t.kpad, nbmax, wmaxmax, nkfold).total;
}

/* Tensor-memory columns: the accumulator plus whole 32-column loads past
 * the start of every profile, rounded to a power of two (>= 32). */
static int tmem_columns(const CsTables &t)
{
    int need = t.npad;
    for (int s = 0; s < t.nslot; s++) {
        const int c0 = t.slot[s].fold ? 0 : t.slot[s].col0;
        const int len = t.slot[s].fold ? 2 * t.nh : t.slot[s].nk;
        need = std::max(need, c0 + (len + 31) / 32 * 32);
    }
    int nc = 32;
    while (nc < need) nc <<= 1;
    return nc;
}

static int grow_records64(GpuSession *S, unsigned cap)
{
    cudaFree(S->d_recs64);
    S->d_recs64 = NULL;
    S->cap64 = 0;
    if (cudaMalloc((void **)&S->d_recs64, (size_t)cap * sizeof(CsRec64)) != cudaSuccess) {
        fprintf(stderr, "Error: cannot allocate %u FP64 candidate records on the GPU\n", cap);
        return -1;
    }
    S->cap64 = cap;
    return 0;
}

static int grow_records(GpuSession *S, unsigned cap)
{
    S->gen++;
    cudaFree(S->d_recs);
    S->d_recs = NULL;
    S->cap = 0;
    if (cudaMalloc((void **)&S->d_recs, (size_t)cap * sizeof(CsRec)) != cudaSuccess) {
        fprintf(stderr, "Error: cannot allocate %u candidate records on the GPU\n", cap);
        return -1;
    }
    S->cap = cap;
    return 0;
}

/* The warp-specialised kernels are compiled for the reference's default
 * search at nharms = 60, 32 and 16: m = 16, decimations 1..6 and the slot
 * layouts and ladder widths of wsk::kCfgDescs, with 32-bit trial positions.
 * Returns the nharms of the matching configuration, or 0. */
static int ws_config(const CsTables &t, long long total)
{
    if (getenv("CS_B200_GENERIC_KERNEL")) return 0;
    if (t.m != wsk::M || t.nslot != 6) return 0;
    const wsk::CfgDesc *cd = NULL;
    for (const wsk::CfgDesc &c : wsk::kCfgDescs)
        if (c.nh == t.nh) cd = &c;
    if (!cd || t.kpad != cd->kpad || t.npad != cd->npad) return 0;
    for (int s = 0; s < 6; s++) {
        const CsSlot &sl = t.slot[s];
        const wsk::SlotDesc &d = cd->slot[s];
        if (sl.k != d.k || sl.nk != d.nk || (sl.fold != 0) != (d.fold != 0) || sl.nw != d.nw)
            return 0;
        if (s > 0 && !d.fold && sl.col0 != d.col0) return 0;
        for (int i = 0; i < d.nw; i++) if (sl.widths[i] != d.w[i]) return 0;
    }
    /* 32-bit positions: t < 2^31 and rfloor0 + floor(t*h*pnum/q) + 1 < 2^31 */
    const double tmax = (double)total + CS_TILE_M;
    if (tmax >= 2147483647.0) return 0;
    double rmax = 0;
    for (int h = 0; h < t.nh; h++) rmax = std::max(rmax, (double)t.harm[h].rfloor0);
    if (rmax + tmax * t.nh * (double)t.pnum / (double)t.q + 64 >= 2147483647.0) return 0;
    if ((double)t.q * 5.0 * t.q >= 4294967295.0) return 0;
    for (int h = 0; h < t.nh; h++) if (t.harm[h].P > wsk::WT_STRIDE) return 0;
    return t.nh;
}

static cudaError_t dev_reserve(void **p, size_t *cap, size_t need);
static uint32_t magic_for(int d);
static int ws_smem(int nh);

/* Tables of the tensor-core interpolation (cs_interp_tc.cuh) for the
 * nharms 60 configuration (pnum 1, q a multiple of tci::NB): per (harmonic,
 * band) the window start R_h(i0) and width, and the band's weight matrix
 * with the rows' gains folded in, scaled by a power of two and split into
 * fp16 hi + lo images in the canonical K-major layout; per harmonic the base
 * bin.  Opt-in with CS_B200_TC_INTERP=1.  Returns false (the session keeps
 * the single-kernel path) when the geometry does not fit. */
static bool tci_load(GpuSession *S, const CsTables &t, long long total)
{
    using namespace tci;
    if (S->use_ws != 60 || !getenv("CS_B200_TC_INTERP")) return false;
    if (t.pnum != 1 || t.q % NB != 0 || t.m != 16) return false;
    const int q = t.q, nh = t.nh, m = t.m, nband = q / NB;
    if (nh * nband > MAXBAND || nh > 64) return false;
    std::vector<Band> bands((size_t)nh * nband);
    std::vector<int> hbase(nh);
    std::vector<double> vals;          /* per band NOUT x kpad, row-major, before the split */
    std::vector<int> voff((size_t)nh * nband);
    double vmax = 0.0;
    for (int h = 1; h <= nh; h++) {
        const CsHarm &hm = t.harm[h - 1];
        const int P = hm.P, woff = hm.woff, cr = t.carry_res[h - 1];
        if (P < 1 || hm.rfloor0 + 1 - m / 2 < -(1LL << 30) || hm.rfloor0 > (1LL << 30)) return false;
        hbase[h - 1] = (int)(hm.rfloor0 + 1 - m / 2);
        auto R = [&](int i) {
            const long long ih = (long long)i * h;
            return (int)(ih / q) + ((ih % q) >= cr ? 1 : 0);
        };
        for (int b = 0; b < nband; b++) {
            const int i0 = b * NB, rel = R(i0);
            const int wb = R(i0 + NB - 1) - rel + m;
            const int kpad = (2 * wb + 15) / 16 * 16;
            if (kpad > KMAX) return false;
            Band &bd = bands[(size_t)(h - 1) * nband + b];
            bd.rel = rel;
            bd.kpad = kpad;
            bd.i0 = i0;
            voff[(size_t)(h - 1) * nband + b] = (int)vals.size();
            vals.resize(vals.size() + (size_t)NOUT * kpad, 0.0);
            double *B = vals.data() + voff[(size_t)(h - 1) * nband + b];
            for (int i = i0; i < i0 + NB; i++) {
                const int ph = i % P;
                const double gr = t.A[2 * (woff + ph)], gi = t.A[2 * (woff + ph) + 1];
                const int nre = 2 * (i - i0);
                for (int k = 0; k < m; k++) {
                    const double w = t.W[(size_t)(woff + ph) * m + k];
                    const int kk = R(i) - rel + k;
                    B[(size_t)nre * kpad + 2 * kk] = gr * w;
                    B[(size_t)nre * kpad + 2 * kk + 1] = -gi * w;
                    B[(size_t)(nre + 1) * kpad + 2 * kk] = gi * w;
                    B[(size_t)(nre + 1) * kpad + 2 * kk + 1] = gr * w;
                }
            }
        }
    }
    for (double v : vals) vmax = std::max(vmax, std::fabs(v));
    if (!(vmax > 0.0) || !(vmax < 1e30)) return false;
    int e;
    std::frexp(vmax, &e);                   /* vmax in [2^(e-1), 2^e) */
    const double sb = std::ldexp(1.0, 14 - e);
    /* images: per band hi then lo, NOUT x kpad halves each */
    std::vector<uint16_t> img;
    for (int j = 0; j < nh * nband; j++) {
        Band &bd = bands[j];
        bd.boff = (int)(img.size() / 8);
        const size_t n = (size_t)NOUT * bd.kpad;
        const size_t base = img.size();
        img.resize(base + 2 * n, 0);
        const double *B = vals.data() + voff[j];
        for (int r = 0; r < NOUT; r++)
            for (int k = 0; k < bd.kpad; k++) {
                const double v = B[(size_t)r * bd.kpad + k] * sb;
                const __half hi = __float2half_rn((float)v);
                const __half lo = __float2half_rn((float)(v - (double)__half2float(hi)));
                const size_t o = b_offset(NOUT, r, k) / 2;
                img[base + o] = __half_as_ushort(hi);
                img[base + n + o] = __half_as_ushort(lo);
            }
    }
    const long long xstride = (total + 1) / 2 * 2;
    if (dev_reserve((void **)&S->d_tci_bands, &S->c_tci_bands, bands.size() * sizeof(Band)) != cudaSuccess ||
        dev_reserve((void **)&S->d_tci_bimg, &S->c_tci_bimg, img.size() * sizeof(uint16_t)) != cudaSuccess ||
        dev_reserve((void **)&S->d_X, &S->c_X, (size_t)nh * xstride * sizeof(float2)) != cudaSuccess)
        return false;
    if (!S->d_tci_hbase && cudaMalloc((void **)&S->d_tci_hbase, sizeof(int) * CS_MAX_NH) != cudaSuccess)
        return false;
    if (cudaMemcpyAsync(S->d_tci_bands, bands.data(), bands.size() * sizeof(Band),
                        cudaMemcpyHostToDevice, S->st) != cudaSuccess ||
        cudaMemcpyAsync(S->d_tci_bimg, img.data(), img.size() * sizeof(uint16_t),
                        cudaMemcpyHostToDevice, S->st) != cudaSuccess ||
        cudaMemcpyAsync(S->d_tci_hbase, hbase.data(), sizeof(int) * nh, cudaMemcpyHostToDevice,
                        S->st) != cudaSuccess)
        return false;
    /* pageable sources: the copies have read them when the stream gets here */
    if (cudaStreamSynchronize(S->st) != cudaSuccess) return false;
    if (cudaFuncSetAttribute((const void *)interp_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             SMEM_BYTES) != cudaSuccess ||
        cudaFuncSetAttribute((const void *)wsk::search_pre<wsk::Cfg60>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, ws_smem(60)) != cudaSuccess)
        return false;
    S->tci_nband = nband;
    S->tci_inv_sb = (float)(1.0 / sb);
    S->tci_xstride = xstride;
    return true;
}

/* The column-tile kernel takes the search_ws configurations when the trial
 * grid has period q = 2*nharms (hidr 0.5, pnum 1): column tiles of q trials,
 * rounds of 8.  Returns the nharms of the configuration, or 0. */
static int tma_config(const CsTables &t, long long total, long long namps, int ws)
{
    if (!ws || getenv("CS_B200_WS_KERNEL") || !getenv("CS_B200_TMA_KERNEL")) return 0;
    if (t.pnum != 1 || t.q != 2 * t.nh || t.q % 8 != 0 || t.q > 128) return 0;
    for (int h = 0; h < t.nh; h++) if (t.harm[h].rfloor0 < 0) return 0;
    /* padded copies and box coordinates (2 floats a bin) in 32-bit ints */
    const double ncol = std::ceil((double)total / t.q / 32.0) * 32.0;
    double xmax = 0;
    for (int h = 0; h < t.nh; h++)
        xmax = std::max(xmax, (double)t.harm[h].rfloor0 + ncol * (h + 1) + t.q);
    if (2.0 * (xmax + wsk::TMA_FRONT + wsk::TMA_BACK) >= 2147483000.0) return 0;
    if (2.0 * ((double)namps + wsk::TMA_FRONT + wsk::TMA_BACK) >= 2147483000.0) return 0;
    return t.nh;
}

static int tma_smem(int nh)
{
    return nh == 60 ? wsk::tma_smem_bytes<wsk::Cfg60>()
         : nh == 32 ? wsk::tma_smem_bytes<wsk::Cfg32>()
                    : wsk::tma_smem_bytes<wsk::Cfg16>();
}

static cudaError_t tma_prepare(int nh)
{
    const void *fn = nh == 60 ? (const void *)wsk::search_tma<wsk::Cfg60>
                   : nh == 32 ? (const void *)wsk::search_tma<wsk::Cfg32>
                              : (const void *)wsk::search_tma<wsk::Cfg16>;
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, tma_smem(nh));
}

static void tma_launch(int nh, int grid, cudaStream_t st, const wsk::Args &w, const wsk::TArgs &x)
{
    if (nh == 60)
        wsk::search_tma<wsk::Cfg60><<<grid, 512, tma_smem(60), st>>>(w, x);
    else if (nh == 32)
        wsk::search_tma<wsk::Cfg32><<<grid, 512, tma_smem(32), st>>>(w, x);
    else
        wsk::search_tma<wsk::Cfg16><<<grid, 512, tma_smem(16), st>>>(w, x);
}

/* cuTensorMapEncodeTiled, reached through the runtime (libcsgpu links no
 * driver library). */
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiledFn encode_tiled()
{
    static const EncodeTiledFn fn = [] {
        void *p = NULL;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
                cudaSuccess || q != cudaDriverEntryPointSuccess)
            p = NULL;
        return (EncodeTiledFn)p;
    }();
    return fn;
}

/* The tables of the column-tile kernel; false (with the session left on
 * search_ws) when any step is refused. */
static bool tma_load(GpuSession *S, const CsTables &t, long long total)
{
    const int nh = t.nh, q = t.q;
    EncodeTiledFn enc = encode_tiled();
    if (!enc) return false;
    /* weights and phase factors by trial index i of a column tile (phase
     * i mod P_h: P_h divides q) */
    std::vector<float> wt((size_t)nh * q * wsk::TMA_WROW, 0.0f);
    for (int h = 0; h < nh; h++) {
        const int P = t.harm[h].P, off = t.harm[h].woff;
        for (int i = 0; i < q; i++) {
            float *d = &wt[((size_t)h * q + i) * wsk::TMA_WROW];
            const int row = off + i % P;
            for (int k = 0; k < wsk::M; k++) d[k] = t.W[(size_t)row * t.m + k];
            d[16] = t.A[2 * (size_t)row];
            d[17] = t.A[2 * (size_t)row + 1];
        }
    }
    /* chunk of the first trial of every column tile (whole super-tiles) */
    const long long ncol = (total + q - 1) / q;
    const long long nsup = (ncol + 31) / 32;
    std::vector<int> cc((size_t)(nsup * 32));
    long long ci = 0;
    for (long long c = 0; c < nsup * 32; c++) {
        const long long t0 = c * q;
        while (ci + 1 < t.nchunks && t.chunks[ci + 1].i0 <= t0) ci++;
        cc[(size_t)c] = (int)ci;
    }
    const size_t nbins = (size_t)S->namps + wsk::TMA_FRONT + wsk::TMA_BACK;
    bool fresh = false;
    for (int k = 0; k < 2; k++) {
        if (!S->d_tc[k] || S->c_tc < nbins * sizeof(float2)) fresh = true;
    }
    if (fresh) {
        for (int k = 0; k < 2; k++) {
            cudaFree(S->d_tc[k]);
            S->d_tc[k] = NULL;
        }
        S->c_tc = 0;
        for (int k = 0; k < 2; k++)
            if (cudaMalloc((void **)&S->d_tc[k], nbins * sizeof(float2)) != cudaSuccess) return false;
        S->c_tc = nbins * sizeof(float2);
    }
    /* the pads are zero; the prep kernel rewrites only the spectrum part */
    for (int k = 0; k < 2; k++)
        if (cudaMemsetAsync(S->d_tc[k], 0, S->c_tc, S->st) != cudaSuccess) return false;
    /* per harmonic and copy: 16 rows of 22 bins, rows 2h bins apart; the
     * inner extent stops 30h bins short of the copy's end, so the last row of
     * a box never reads past the allocation (those bins are zero anyway) */
    std::vector<CUtensorMap> maps((size_t)nh * 2);
    for (int h = 1; h <= nh; h++) {
        for (int k = 0; k < 2; k++) {
            const cuuint64_t gdim[2] = {(cuuint64_t)(2 * (nbins - 30 * (size_t)h)),
                                        (cuuint64_t)wsk::TMA_ROWS};
            const cuuint64_t gstr[1] = {(cuuint64_t)(16 * h)};
            const cuuint32_t box[2] = {2 * wsk::TMA_BOXW, wsk::TMA_ROWS};
            const cuuint32_t est[2] = {1, 1};
            if (enc(&maps[(size_t)(h - 1) * 2 + k], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
                    (void *)S->d_tc[k], gdim, gstr, box, est, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS) {
                fprintf(stderr, "Warning: TMA descriptor for harmonic %d refused; using the "
                                "register-staged kernel\n", h);
                return false;
            }
        }
    }
    if (dev_reserve((void **)&S->d_wtab, &S->c_wtab, wt.size() * sizeof(float)) != cudaSuccess ||
        cudaMemcpyAsync(S->d_wtab, wt.data(), wt.size() * sizeof(float), cudaMemcpyHostToDevice,
                        S->st) != cudaSuccess)
        return false;
    if (dev_reserve((void **)&S->d_cchunk, &S->c_cchunk, cc.size() * sizeof(int)) != cudaSuccess ||
        cudaMemcpyAsync(S->d_cchunk, cc.data(), cc.size() * sizeof(int), cudaMemcpyHostToDevice,
                        S->st) != cudaSuccess)
        return false;
    if (!S->d_maps && cudaMalloc((void **)&S->d_maps, sizeof(CUtensorMap) * 2 * wsk::MAX_NH) !=
                          cudaSuccess)
        return false;
    if (cudaMemcpyAsync(S->d_maps, maps.data(), maps.size() * sizeof(CUtensorMap),
                        cudaMemcpyHostToDevice, S->st) != cudaSuccess)
        return false;
    /* the host vectors go when this returns: finish the copies first */
    if (cudaStreamSynchronize(S->st) != cudaSuccess) return false;
    wsk::TArgs &x = S->tx;
    memset(&x, 0, sizeof(x));
    x.maps = S->d_maps;
    x.wtab = S->d_wtab;
    x.cchunk = S->d_cchunk;
    x.nchunks = (int)t.nchunks;
    x.total = (int)total;
    x.q = q;
    x.qmag = magic_for(q);
    x.rounds_per_super = q / 8;
    x.nitems = (int)(nsup * (q / 8));
    return tma_prepare(nh) == cudaSuccess;
}

static int ws_smem(int nh)
{
    return nh == 60 ? wsk::smem_bytes<wsk::Cfg60>()
         : nh == 32 ? wsk::smem_bytes<wsk::Cfg32>()
                    : wsk::smem_bytes<wsk::Cfg16>();
}

static int ws_smem_multi(int nh)
{
    return nh == 60 ? wsk::smem_bytes_multi<wsk::Cfg60>()
         : nh == 32 ? wsk::smem_bytes_multi<wsk::Cfg32>()
                    : wsk::smem_bytes_multi<wsk::Cfg16>();
}

static cudaError_t ws_prepare_multi(int nh)
{
    const void *fn = nh == 60 ? (const void *)wsk::search_ws_multi<wsk::Cfg60>
                   : nh == 32 ? (const void *)wsk::search_ws_multi<wsk::Cfg32>
                              : (const void *)wsk::search_ws_multi<wsk::Cfg16>;
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                ws_smem_multi(nh));
}

static cudaError_t ws_prepare(int nh)
{
    const cudaError_t e = ws_prepare_multi(nh);
    if (e != cudaSuccess) return e;
    const void *fn = nh == 60 ? (const void *)wsk::search_ws<wsk::Cfg60>
                   : nh == 32 ? (const void *)wsk::search_ws<wsk::Cfg32>
                              : (const void *)wsk::search_ws<wsk::Cfg16>;
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, ws_smem(nh));
}

static void ws_launch(int nh, int grid, cudaStream_t st, const wsk::Args &w)
{
    if (nh == 60)
        wsk::search_ws<wsk::Cfg60><<<grid, wsk::nthreads<wsk::Cfg60>(), ws_smem(60), st>>>(w);
    else if (nh == 32)
        wsk::search_ws<wsk::Cfg32><<<grid, wsk::nthreads<wsk::Cfg32>(), ws_smem(32), st>>>(w);
    else
        wsk::search_ws<wsk::Cfg16><<<grid, wsk::nthreads<wsk::Cfg16>(), ws_smem(16), st>>>(w);
}

static uint32_t magic_for(int d)
{
    return d >= 2 ? (uint32_t)(0x100000000ULL / (unsigned long long)d + 1ULL) : 0u;
}

/* Keep *p at least `need` bytes: reuse it when large enough, else replace it
 * (contents are not kept). */
static cudaError_t dev_reserve(void **p, size_t *cap, size_t need)
{
    if (need == 0) need = 1;
    if (*p && *cap >= need) return cudaSuccess;
    cudaFree(*p);
    *p = NULL;
    *cap = 0;
    const cudaError_t e = cudaMalloc(p, need);
    if (e == cudaSuccess) *cap = need;
    return e;
}

/* Raise a kernel's dynamic shared-memory cap to what the device allows
 * beside the kernel's static shared memory. */
static cudaError_t set_smem_cap(const void *fn, int max_optin)
{
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, fn);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                max_optin - (int)fa.sharedSizeBytes);
}

/* Build the host tables for one geometry and bring the device copies up to
 * date, reusing the session's device buffers where they are large enough.
 * Returns 0, or -1 with a message.  Leaves the session unusable on failure
 * (callers release it). */
static int session_load(GpuSession *S, const FFTFile *ft, const SearchParams *p,
                        const DirectPlanSet *dplans, const long long *cstarts, long long total,
                        int Nprof, long long nchunks, double r_lo, double lodr)
{
    char err[512] = {0};
    std::vector<uint16_t> bhi, blo;
    size_t img_halves = 0;
    int smem = 0;
    S->gen++;
    S->p = p;
    S->Nprof = Nprof;
    S->total = total;
    S->nchunks = nchunks;
    S->N = ft->N;
    S->namps = ft->namps;
    S->T = ft->T;
    S->r_lo = r_lo;
    S->lodr = lodr;
    cs_tables_free(&S->tab);
    if (cs_tables_build(&S->tab, ft, p, dplans, cstarts, total, nchunks, r_lo, lodr,
                        err, sizeof(err)) != 0) {
        fprintf(stderr, "Error: B200 search session: %s\n", err);
        return -1;
    }
    smem = smem_bytes(S->tab);
    if (smem > S->max_smem) {
        fprintf(stderr, "Error: B200 search kernel needs %d bytes of shared memory, device "
                        "%d allows %d\n", smem, S->device, S->max_smem);
        return -1;
    }
    const CsTables &t = S->tab;
    CK(dev_reserve((void **)&S->d_amps, &S->c_amps, (size_t)S->namps * sizeof(float2)));
    CK(cudaMemcpyAsync(S->d_harm, t.harm, sizeof(CsHarm) * CS_MAX_NH, cudaMemcpyHostToDevice, S->st));
    CK(dev_reserve((void **)&S->d_rowtab, &S->c_rowtab, (size_t)t.nh * t.q * sizeof(uint16_t)));
    CK(cudaMemcpyAsync(S->d_rowtab, t.rowtab, (size_t)t.nh * t.q * sizeof(uint16_t), cudaMemcpyHostToDevice, S->st));
    CK(dev_reserve((void **)&S->d_W, &S->c_W, (size_t)t.nrows * t.m * sizeof(float)));
    CK(cudaMemcpyAsync(S->d_W, t.W, (size_t)t.nrows * t.m * sizeof(float), cudaMemcpyHostToDevice, S->st));
    CK(dev_reserve((void **)&S->d_A, &S->c_A, (size_t)t.nrows * sizeof(float2)));
    CK(cudaMemcpyAsync(S->d_A, t.A, (size_t)t.nrows * sizeof(float2), cudaMemcpyHostToDevice, S->st));
    CK(dev_reserve((void **)&S->d_carry, &S->c_carry, (size_t)t.nrows));
    CK(cudaMemcpyAsync(S->d_carry, t.carry, (size_t)t.nrows, cudaMemcpyHostToDevice, S->st));
    CK(dev_reserve((void **)&S->d_chunks, &S->c_chunks, (size_t)nchunks * sizeof(CsChunk)));
    if (nchunks > 0)
        CK(cudaMemcpyAsync(S->d_chunks, t.chunks, (size_t)nchunks * sizeof(CsChunk), cudaMemcpyHostToDevice, S->st));
    CK(dev_reserve((void **)&S->d_tiles, &S->c_tiles, (size_t)t.ntiles * 3 * sizeof(int)));
    if (t.ntiles > 0)
        CK(cudaMemcpyAsync(S->d_tiles, t.tiles, (size_t)t.ntiles * 3 * sizeof(int), cudaMemcpyHostToDevice, S->st));
    img_halves = (size_t)t.npad * t.kpad;
    if (!(S->img_ok && S->img_nh == t.nh && S->img_nslot == t.nslot && S->img_npad == t.npad &&
          S->img_kpad == t.kpad &&
          memcmp(S->img_slot, t.slot, sizeof(CsSlot) * (size_t)t.nslot) == 0)) {
        S->img_ok = false;
        bhi.resize(img_halves);
        blo.resize(img_halves);
        cs_tables_dft_images(&S->tab, bhi.data(), blo.data());
        S->bbytes = (int)(img_halves * 2);
        CK(dev_reserve((void **)&S->d_bimg, &S->c_bimg, (size_t)2 * S->bbytes));
        CK(cudaMemcpyAsync(S->d_bimg, bhi.data(), (size_t)S->bbytes, cudaMemcpyHostToDevice, S->st));
        CK(cudaMemcpyAsync((char *)S->d_bimg + S->bbytes, blo.data(), (size_t)S->bbytes, cudaMemcpyHostToDevice, S->st));
        S->img_ok = true;
        S->img_nh = t.nh;
        S->img_nslot = t.nslot;
        S->img_npad = t.npad;
        S->img_kpad = t.kpad;
        memcpy(S->img_slot, t.slot, sizeof(CsSlot) * (size_t)t.nslot);
    }
    S->prec64 = t.prec64;
    if (S->prec64) {
        /* FP64 profile stage: half-spectrum DFT tables, per-chunk FP64 noise
         * scales, prefix-sum layout (cs_search_f64.cuh) */
        f64k::Extra &x = S->fx;
        memset(&x, 0, sizeof(x));
        x.nunit = cs_tables_f64_units(&t);
        x.ucols = (x.nunit + 3) / 4 * 4;
        std::vector<double> bcs((size_t)2 * t.nh * x.ucols);
        cs_tables_dft_f64(&t, bcs.data(), bcs.data() + (size_t)t.nh * x.ucols, x.ucols, x.unit0);
        x.prs = t.ncol | 1;
        int off = 0;
        for (int q = 0; q < t.nslot; q++) {
            x.ps_off[q] = off;
            off += f64k::TT * (t.slot[q].nk + t.slot[q].wmax + 1);
        }
        x.ps_total = off;
        S->f64_smem = f64k::smem_bytes(t.nh, x.ucols, x.prs, x.ps_total);
        if (S->f64_smem + (int)sizeof(CsHarm) * CS_MAX_NH > S->max_smem) {
            fprintf(stderr, "Error: the FP64 search needs %d bytes of shared memory, device "
                            "%d allows %d\n", S->f64_smem, S->device, S->max_smem);
            return -1;
        }
        CK(dev_reserve((void **)&S->d_bcs, &S->c_bcs, bcs.size() * sizeof(double)));
        CK(cudaMemcpyAsync(S->d_bcs, bcs.data(), bcs.size() * sizeof(double),
                           cudaMemcpyHostToDevice, S->st));
        const size_t nsc = (size_t)(nchunks > 0 ? nchunks : 1) * CS_F64_SCALES;
        CK(dev_reserve((void **)&S->d_scales, &S->c_scales, nsc * sizeof(double)));
        CK(cudaMemcpyAsync(S->d_scales, t.invsw64, nsc * sizeof(double), cudaMemcpyHostToDevice,
                           S->st));
        x.bcs = S->d_bcs;
        x.scales = S->d_scales;
        long long want = (total * t.nslot) / 16 + 4096;
        if (want > (long long)0x7fffffff) want = 0x7fffffff;
        if (!S->d_recs64 || S->cap64 < (unsigned)want)
            if (grow_records64(S, (unsigned)want) != 0) return -1;
        x.recs = S->d_recs64;
        CK(set_smem_cap((const void *)f64k::search_f64<16>, S->max_smem));
        CK(set_smem_cap((const void *)f64k::search_f64<0>, S->max_smem));
    }
    S->use_ws = S->prec64 ? 0 : ws_config(t, total);
    if (S->use_ws && (S->namps >= 2147483000LL || ws_smem(S->use_ws) > S->max_smem))
        S->use_ws = 0;
    if (S->use_ws) {
        /* weights: harmonic h, tap quad i4, phase p at float4
         * h*4*WT_STRIDE + i4*WT_STRIDE + p (room for the largest nharms) */
        const size_t nq = (size_t)wsk::MAX_NH * 4 * wsk::WT_STRIDE;
        std::vector<float> wfix((size_t)t.nh * 4 * wsk::WT_STRIDE * 4, 0.0f);
        for (int h = 0; h < t.nh; h++) {
            S->hh[h].rfloor0 = (int)t.harm[h].rfloor0;
            S->hh[h].P = t.harm[h].P;
            S->hh[h].woff = t.harm[h].woff;
            S->hh[h].wt_off = h * 4 * wsk::WT_STRIDE;
            S->hh[h].pmagic = magic_for(t.harm[h].P);
            S->hh[h].carry_res = t.carry_res[h];
            const int P = t.harm[h].P, off = t.harm[h].woff;
            for (int ph = 0; ph < P; ph++)
                for (int i = 0; i < wsk::M; i++)
                    wfix[4 * ((size_t)h * 4 * wsk::WT_STRIDE + (i / 4) * wsk::WT_STRIDE + ph) + (i & 3)] =
                        t.W[(size_t)(off + ph) * t.m + i];
        }
        if (!S->d_harm2) CK(cudaMalloc((void **)&S->d_harm2, sizeof(wsk::Harm) * wsk::MAX_NH));
        CK(cudaMemcpyAsync(S->d_harm2, S->hh, sizeof(wsk::Harm) * t.nh, cudaMemcpyHostToDevice, S->st));
        if (!S->d_Wt) CK(cudaMalloc((void **)&S->d_Wt, nq * sizeof(float4)));
        CK(cudaMemcpyAsync(S->d_Wt, wfix.data(), wfix.size() * sizeof(float), cudaMemcpyHostToDevice, S->st));
        CK(ws_prepare(S->use_ws));
    }
    S->use_tci = tci_load(S, t, total) ? 1 : 0;
    (void)cudaGetLastError();
    S->use_tma = S->use_tci ? 0 : tma_config(t, total, S->namps, S->use_ws);
    if (S->use_tma && (tma_smem(S->use_tma) > S->max_smem || !tma_load(S, t, total)))
        S->use_tma = 0;
    {
        /* Start with room for 1 in 16 trials per slot; grown on overflow. */
        long long want = (total * t.nslot) / 16 + 4096;
        if (want > (long long)0x7fffffff) want = 0x7fffffff;
        if (!S->d_recs || S->cap < (unsigned)want)
            if (grow_records(S, (unsigned)want) != 0) return -1;
    }
    /* the cap is per kernel, not per session: sessions of other geometries may
     * launch concurrently (batch slots), so it is set to the device limit,
     * never lowered to this geometry's need */
    CK(set_smem_cap((const void *)cs_search_kernel<16>, S->max_smem));
    CK(set_smem_cap((const void *)cs_search_kernel<0>, S->max_smem));
    /* The uploads are ordered on the session stream and finished here: a
     * synchronous copy from pageable memory may return before its DMA lands,
     * and nothing would order that DMA before a kernel on a non-blocking
     * stream -- with reused buffers the kernel could read the previous
     * geometry's tables.  The host tables and vectors may go after this. */
    CK(cudaStreamSynchronize(S->st));
    return 0;
fail:
    return -1;
}

/* Device bytes a session holds for its current geometry. */
static size_t session_bytes(const GpuSession *S)
{
    return S->c_amps + S->c_rowtab + S->c_W + S->c_A + S->c_carry + S->c_chunks + S->c_tiles +
           S->c_bimg + (size_t)S->cap * sizeof(CsRec) + sizeof(CsHarm) * CS_MAX_NH +
           S->c_bcs + S->c_scales + (size_t)S->cap64 * sizeof(CsRec64) + S->c_wtab +
           S->c_cchunk + 2 * S->c_tc + (S->d_maps ? sizeof(CUtensorMap) * 2 * wsk::MAX_NH : 0) +
           (S->d_Wt ? (size_t)wsk::MAX_NH * 4 * wsk::WT_STRIDE * sizeof(float4) : 0);
}

/* A session on `device` with its streams, events and fixed-size buffers,
 * but no geometry yet; NULL on failure. */
static GpuSession *session_new(int device)
{
    GpuSession *S = (GpuSession *)calloc(1, sizeof(GpuSession));
    if (!S) return NULL;
    S->device = device;
    CK(select_device(device));
    {
        cudaDeviceProp prop;
        CK(cudaGetDeviceProperties(&prop, device));
        S->max_smem = (int)prop.sharedMemPerBlockOptin;
        S->nsm = prop.multiProcessorCount;
    }
    CK(cudaStreamCreateWithFlags(&S->st, cudaStreamNonBlocking));
    CK(cudaEventCreate(&S->ev0));
    CK(cudaEventCreate(&S->ev1));
    CK(cudaEventCreateWithFlags(&S->ev_in, cudaEventDisableTiming));
    CK(cudaMalloc((void **)&S->d_harm, sizeof(CsHarm) * CS_MAX_NH));
    CK(cudaMalloc((void **)&S->d_amax, 2 * sizeof(unsigned)));
    CK(cudaMalloc((void **)&S->d_count, sizeof(unsigned)));
    CK(cudaMalloc((void **)&S->d_err, sizeof(int)));
    CK(cudaMallocHost((void **)&S->h_count, 4 * sizeof(unsigned)));
    return S;
fail:
    session_release(S);
    return NULL;
}

/* Freed sessions kept for the next create.  The reference's drivers free
 * their session and build a new one whenever the spectrum length changes
 * (src/search.c:1388-1406): about twenty device and pinned allocations and
 * frees per file, each cudaFree waiting for the whole device.  A parked
 * session keeps its stream, events and grow-only buffers, and the next create
 * on its device reloads it for the new geometry.  CS_B200_SESSION_PARK sets
 * how many are kept (default 2; 0 frees at once, as the reference does);
 * cs_b200_session_park_drain gives their memory back. */
static std::mutex g_park_mu;
static std::vector<GpuSession *> g_park;

static size_t park_limit()
{
    static const size_t lim = [] {
        const char *e = getenv("CS_B200_SESSION_PARK");
        return e ? (size_t)std::max(0, atoi(e)) : (size_t)2;
    }();
    return lim;
}

static GpuSession *park_take(int device)
{
    std::lock_guard<std::mutex> g(g_park_mu);
    for (size_t i = g_park.size(); i-- > 0;) {
        GpuSession *S = g_park[i];
        if (S->device == device) {
            g_park.erase(g_park.begin() + (long)i);
            return S;
        }
    }
    return nullptr;
}

CS_EXPORT int cs_b200_session_park_drain(void)
{
    std::vector<GpuSession *> all;
    {
        std::lock_guard<std::mutex> g(g_park_mu);
        all.swap(g_park);
    }
    for (GpuSession *S : all) {
        select_device(S->device);
        session_release(S);
    }
    return (int)all.size();
}

CS_EXPORT GpuSession *cs_gpu_session_create(const FFTFile *ft, const SearchParams *p,
                                            const DirectPlanSet *dplans,
                                            const long long *cstarts, long long total,
                                            int Nprof, long long nchunks, double r_lo,
                                            double lodr, int device)
{
    GpuSession *S = park_take(device);
    if (S) {
        if (select_device(device) != cudaSuccess) {
            session_release(S);
            return NULL;
        }
    } else {
        S = session_new(device);
    }
    if (!S) return NULL;
    if (session_load(S, ft, p, dplans, cstarts, total, Nprof, nchunks, r_lo, lodr) != 0) {
        session_release(S);
        return NULL;
    }
    return S;
}

CS_EXPORT int cs_gpu_session_matches(const GpuSession *S, const FFTFile *ft,
                                     const SearchParams *p, int Nprof, long long total,
                                     double r_lo, double lodr, int device)
{
    if (!S) return 0;
    return S->p == p && S->device == device && S->Nprof == Nprof && S->total == total &&
           S->T == ft->T && S->N == ft->N && S->namps == ft->namps && S->r_lo == r_lo &&
           S->lodr == lodr;
}

static SearchArgs make_args(GpuSession *S, const float2 *d_amps, double threshold)
{
    SearchArgs a;
    memset(&a, 0, sizeof(a));
    const CsTables &t = S->tab;
    a.amps = d_amps;
    a.namps = S->namps;
    a.harm = S->d_harm;
    a.rowtab = S->d_rowtab;
    a.W = S->d_W;
    a.A = S->d_A;
    a.carry = S->d_carry;
    a.chunks = S->d_chunks;
    a.tiles = S->d_tiles;
    a.ntiles = t.ntiles;
    a.bimg = S->d_bimg;
    a.bbytes = S->bbytes;
    a.nh = t.nh;
    a.m = t.m;
    a.q = t.q;
    a.pnum = t.pnum;
    a.qmagic = t.q >= 2 ? (uint32_t)(0x100000000ULL / (unsigned long long)t.q + 1ULL) : 0u;
    a.kpad = t.kpad;
    a.npad = t.npad;
    a.ncols_tmem = tmem_columns(t);
    a.nslot = t.nslot;
    memcpy(a.slot, t.slot, sizeof(a.slot));
    a.gbound = t.gbound;
    a.amax = S->d_amax;
    a.thresh = threshold;
    a.recs = S->d_recs;
    a.count = S->d_count;
    a.cap = S->cap;
    a.err = S->d_err;
    return a;
}

/* Arguments of the warp-specialised kernels for session S. */
static wsk::Args ws_args(const GpuSession *S, const float2 *d_amps, double threshold)
{
    wsk::Args w;
    memset(&w, 0, sizeof(w));
    w.amps = d_amps;
    w.namps = (int)S->namps;
    w.Wt = S->d_Wt;
    w.A = S->d_A;
    w.harm = S->d_harm2;
    w.chunks = S->d_chunks;
    w.tiles = S->d_tiles;
    w.ntiles = S->tab.ntiles;
    w.bimg = S->d_bimg;
    w.q = S->tab.q;
    w.pnum = S->tab.pnum;
    w.qmagic = magic_for(S->tab.q);
    w.gbound = S->tab.gbound;
    w.amax = S->d_amax;
    w.thresh = threshold;
    w.recs = S->d_recs;
    w.count = S->d_count;
    w.cap = S->cap;
    w.err = S->d_err;
    return w;
}

/* Enqueue the search of the spectrum at d_amps on S->st (no host sync). */
static cudaError_t enqueue_search(GpuSession *S, const float2 *d_amps, double threshold,
                                  bool timed)
{
    cudaError_t e;
    if ((e = cudaMemsetAsync(S->d_amax, 0, 2 * sizeof(unsigned), S->st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(S->d_count, 0, sizeof(unsigned), S->st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(S->d_err, 0, sizeof(int), S->st)) != cudaSuccess) return e;
    if (S->namps > 0) {
        int g = (int)std::min<long long>((S->namps + 255) / 256, (long long)S->nsm * 8);
        if (S->use_tma)
            wsk::tma_prep_kernel<<<g, 256, 0, S->st>>>(d_amps, (int)S->namps, S->d_tc[0],
                                                       S->d_tc[1], S->d_amax);
        else
            cs_amax_kernel<<<g, 256, 0, S->st>>>(d_amps, S->namps, S->d_amax);
    }
    if (S->tab.ntiles <= 0) return cudaGetLastError();
    if (S->prec64) {
        SearchArgs a64 = make_args(S, d_amps, threshold);
        a64.cap = S->cap64;
        f64k::Extra x = S->fx;
        x.recs = S->d_recs64;
        const int nsub = S->tab.ntiles * (CS_TILE_M / f64k::TT);
        const int grid = std::min(nsub, S->nsm);
        if (timed) cudaEventRecord(S->ev0, S->st);
        if (S->tab.m == 16)
            f64k::search_f64<16><<<grid, f64k::NT, S->f64_smem, S->st>>>(a64, x);
        else
            f64k::search_f64<0><<<grid, f64k::NT, S->f64_smem, S->st>>>(a64, x);
        if (timed) cudaEventRecord(S->ev1, S->st);
        return cudaGetLastError();
    }
    if (S->use_ws && S->use_tci) {
        tci::Args ta;
        memset(&ta, 0, sizeof(ta));
        ta.amps = d_amps;
        ta.namps = S->namps;
        ta.amax = S->d_amax;
        ta.bands = S->d_tci_bands;
        ta.bimg = S->d_tci_bimg;
        ta.hbase = S->d_tci_hbase;
        ta.nh = S->tab.nh;
        ta.nband = S->tci_nband;
        ta.q = S->tab.q;
        ta.total = S->total;
        ta.ncol = (S->total + S->tab.q - 1) / S->tab.q;
        ta.nunits = (ta.ncol + tci::ROWS - 1) / tci::ROWS * ta.nh;
        ta.inv_sb = S->tci_inv_sb;
        ta.X = S->d_X;
        ta.xstride = S->tci_xstride;
        ta.err = S->d_err;
        wsk::Args w = ws_args(S, d_amps, threshold);
        w.X = S->d_X;
        w.xstride = S->tci_xstride;
        const int grid1 = (int)std::min<long long>(ta.nunits, S->nsm);
        const int grid = std::min(S->tab.ntiles, S->nsm);
        if (timed) cudaEventRecord(S->ev0, S->st);
        tci::interp_tc<<<grid1, tci::NTHREADS, tci::SMEM_BYTES, S->st>>>(ta);
        wsk::search_pre<wsk::Cfg60><<<grid, 512, ws_smem(60), S->st>>>(w);
        if (timed) cudaEventRecord(S->ev1, S->st);
        return cudaGetLastError();
    }
    if (S->use_ws) {
        const wsk::Args w = ws_args(S, d_amps, threshold);
        if (S->use_tma) {
            const int grid = std::min(S->tx.nitems, S->nsm);
            if (timed) cudaEventRecord(S->ev0, S->st);
            tma_launch(S->use_tma, grid, S->st, w, S->tx);
            if (timed) cudaEventRecord(S->ev1, S->st);
            return cudaGetLastError();
        }
        const int grid = std::min(S->tab.ntiles, S->nsm);
        if (timed) cudaEventRecord(S->ev0, S->st);
        ws_launch(S->use_ws, grid, S->st, w);
        if (timed) cudaEventRecord(S->ev1, S->st);
        return cudaGetLastError();
    }
    const SearchArgs a = make_args(S, d_amps, threshold);
    const int smem = smem_bytes(S->tab);
    const int grid = std::min(S->tab.ntiles, S->nsm);
    if (timed) cudaEventRecord(S->ev0, S->st);
    if (S->tab.m == 16)
        cs_search_kernel<16><<<grid, CS_NTHREADS, smem, S->st>>>(a);
    else
        cs_search_kernel<0><<<grid, CS_NTHREADS, smem, S->st>>>(a);
    if (timed) cudaEventRecord(S->ev1, S->st);
    return cudaGetLastError();
}

/* The FP64 search's records: grow and rerun on overflow, else read back,
 * order and harvest them. */
static int collect64(GpuSession *S, unsigned n, double threshold, CandidateList *out,
                     int *need_rerun)
{
    cudaError_t e;
    if (n > S->cap64) {
        if (grow_records64(S, n + n / 8 + 1024) != 0) return -1;
        *need_rerun = 1;
        return 0;
    }
    if (n == 0) return 0;
    if ((size_t)n > S->h_recs64_cap) {
        const size_t cap = (size_t)n + n / 4 + 1024;
        if (S->h_recs64) cudaFreeHost(S->h_recs64);
        S->h_recs64 = NULL;
        S->h_recs64_cap = 0;
        if ((e = cudaMallocHost((void **)&S->h_recs64, cap * sizeof(CsRec64))) != cudaSuccess) {
            S->h_recs64 = NULL;
            fprintf(stderr, "Error: B200 record staging: %s\n", cudaGetErrorString(e));
            return -1;
        }
        S->h_recs64_cap = cap;
    }
    if ((e = cudaMemcpyAsync(S->h_recs64, S->d_recs64, (size_t)n * sizeof(CsRec64),
                             cudaMemcpyDeviceToHost, S->st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(S->st)) != cudaSuccess) {
        fprintf(stderr, "Error: B200 search readback failed: %s\n", cudaGetErrorString(e));
        return -1;
    }
    cs_sort_records64(S->h_recs64, (long long)n);
    cs_harvest64(&S->tab, S->h_recs64, (long long)n, S->r_lo, S->lodr, (double)S->N, S->T,
                 threshold, out);
    return 0;
}

/* Read back the records and build the candidate list. */
static int collect(GpuSession *S, double threshold, CandidateList *out, int *need_rerun)
{
    *need_rerun = 0;
    cudaError_t e;
    if ((e = cudaMemcpyAsync(S->h_count, S->d_count, sizeof(unsigned), cudaMemcpyDeviceToHost,
                             S->st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(S->h_count + 1, S->d_err, sizeof(int), cudaMemcpyDeviceToHost,
                             S->st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(S->st)) != cudaSuccess) {
        fprintf(stderr, "Error: B200 search failed: %s\n", cudaGetErrorString(e));
        return -1;
    }
    if (S->h_count[1] != 0) {
        fprintf(stderr, "Error: B200 search kernel timed out waiting for the tensor cores\n");
        return -1;
    }
    const unsigned n = S->h_count[0];
    if (S->prec64) return collect64(S, n, threshold, out, need_rerun);
    if (n > S->cap) {
        if (grow_records(S, n + n / 8 + 1024) != 0) return -1;
        *need_rerun = 1;
        return 0;
    }
    if (n == 0) return 0;
    if ((size_t)n > S->h_recs_cap) {
        const size_t cap = (size_t)n + n / 4 + 1024;
        if (S->h_recs) cudaFreeHost(S->h_recs);
        S->h_recs = NULL;
        S->h_recs_cap = 0;
        if ((e = cudaMallocHost((void **)&S->h_recs, cap * sizeof(CsRec))) != cudaSuccess) {
            S->h_recs = NULL;
            fprintf(stderr, "Error: B200 record staging: %s\n", cudaGetErrorString(e));
            return -1;
        }
        S->h_recs_cap = cap;
    }
    if ((e = cudaMemcpyAsync(S->h_recs, S->d_recs, (size_t)n * sizeof(CsRec),
                             cudaMemcpyDeviceToHost, S->st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(S->st)) != cudaSuccess) {
        fprintf(stderr, "Error: B200 search readback failed: %s\n", cudaGetErrorString(e));
        return -1;
    }
    cs_sort_records(S->h_recs, (long long)n);
    cs_harvest(&S->tab, S->h_recs, (long long)n, S->r_lo, S->lodr, (double)S->N, S->T,
               threshold, out);
    return 0;
}

CS_EXPORT CandidateList cs_gpu_session_run(GpuSession *S, const FFTFile *ft, double threshold)
{
    CandidateList cands;
    candlist_init(&cands);
    if (!S) return cands;
    if (ft->namps != S->namps || ft->N != S->N) {
        fprintf(stderr, "Error: GPU session built for N=%lld/%lld amps but the input has "
                        "N=%lld/%lld\n", S->N, S->namps, ft->N, ft->namps);
        return cands;
    }
    if (select_device(S->device) != cudaSuccess) return cands;
    if (S->namps > 0) {
        cudaError_t e = cudaMemcpyAsync(S->d_amps, ft->amps, (size_t)S->namps * sizeof(float2),
                                        cudaMemcpyHostToDevice, S->st);
        if (e != cudaSuccess) {
            fprintf(stderr, "Error: spectrum upload failed: %s\n", cudaGetErrorString(e));
            return cands;
        }
    }
    for (int attempt = 0; attempt < 2; attempt++) {
        cudaError_t e = enqueue_search(S, S->d_amps, threshold, false);
        if (e != cudaSuccess) {
            fprintf(stderr, "Error: B200 search launch failed: %s\n", cudaGetErrorString(e));
            return cands;
        }
        int rerun = 0;
        if (collect(S, threshold, &cands, &rerun) != 0) {
            candlist_free(&cands);
            return cands;
        }
        if (!rerun) break;
    }
    return cands;
}

CS_EXPORT void cs_gpu_session_free(GpuSession *S)
{
    if (!S) return;
    select_device(S->device);
    if (cudaStreamSynchronize(S->st) == cudaSuccess && park_limit() > 0) {
        S->p = NULL;                 /* matches nothing until it is reloaded */
        std::lock_guard<std::mutex> g(g_park_mu);
        if (g_park.size() < park_limit()) {
            g_park.push_back(S);
            return;
        }
    }
    session_release(S);
}

CS_EXPORT CandidateList cs_gpu_search_region(const FFTFile *ft, const SearchParams *p,
                                             const DirectPlanSet *dplans,
                                             const long long *cstarts, long long total,
                                             int Nprof, long long nchunks, double r_lo,
                                             double r_hi, double lodr, double threshold,
                                             int device)
{
    (void)r_hi;
    CandidateList c;
    candlist_init(&c);
    GpuSession *S = cs_gpu_session_create(ft, p, dplans, cstarts, total, Nprof, nchunks,
                                          r_lo, lodr, device);
    if (!S) return c;
    c = cs_gpu_session_run(S, ft, threshold);
    cs_gpu_session_free(S);
    return c;
}

/* ------------------------------------------------------------------ */
/* Additions (cs_b200.h)                                               */
/* ------------------------------------------------------------------ */
CS_EXPORT int cs_b200_session_info(const GpuSession *S, CsB200Info *info)
{
    if (!S || !info) return -1;
    memset(info, 0, sizeof(*info));
    info->ntiles = S->tab.ntiles;
    info->nchunks = S->tab.nchunks;
    info->nslot = S->tab.nslot;
    info->npad = S->tab.npad;
    info->kpad = S->tab.kpad;
    info->smem_bytes = S->prec64 ? S->f64_smem : S->use_tma ? tma_smem(S->use_tma)
                     : S->use_ws ? ws_smem(S->use_ws) : smem_bytes(S->tab);
    info->grid = S->use_tma ? std::min(S->tx.nitems, S->nsm) : std::min(S->tab.ntiles, S->nsm);
    info->kernel = S->prec64 ? 2 : S->use_tci ? 4 : S->use_tma ? 3 : S->use_ws ? 1 : 0;
    info->total = S->total;
    info->rec_capacity = S->cap;
    return 0;
}

CS_EXPORT int cs_b200_session_enqueue_device(GpuSession *S, const float *d_amps,
                                             double threshold, void *stream)
{
    if (!S) return -1;
    if (stream) {
        /* the spectrum is produced on the caller's stream: start after it */
        if (cudaEventRecord(S->ev_in, (cudaStream_t)stream) != cudaSuccess ||
            cudaStreamWaitEvent(S->st, S->ev_in, 0) != cudaSuccess)
            return -1;
    }
    cudaError_t e = enqueue_search(S, d_amps ? (const float2 *)d_amps : S->d_amps, threshold,
                                   true);
    return e == cudaSuccess ? 0 : -1;
}

/* Kernel time of the session's last timed launch, or 0 when its events were
 * not recorded (a search queued without timing, or one that ran inside a
 * multi-spectrum launch timed on another session).  The runtime answers an
 * unrecorded event with an error; it is cleared here so that it does not
 * surface at the next launch check. */
static float last_kernel_ms(const GpuSession *S)
{
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, S->ev0, S->ev1) != cudaSuccess) {
        (void)cudaGetLastError();
        ms = 0.0f;
    }
    return ms;
}

CS_EXPORT int cs_b200_session_collect(GpuSession *S, double threshold, CandidateList *out,
                                      float *kernel_ms)
{
    if (!S || !out) return -1;
    candlist_init(out);
    int rerun = 0;
    if (collect(S, threshold, out, &rerun) != 0) return -1;
    if (kernel_ms) *kernel_ms = last_kernel_ms(S);
    return rerun ? 1 : 0;
}

CS_EXPORT int cs_b200_session_collapse_enqueue(GpuSession *S, double threshold, int remove,
                                               double dr_tol, int harm_remove, int numharm,
                                               double harm_tol)
{
    if (!S) return -1;
    if (S->prec64) {
        fprintf(stderr, "Error: the device collapse takes FP32 sessions; collect an FP64 "
                        "search with cs_b200_session_collect\n");
        return -1;
    }
    cudaError_t e;
    if ((e = cudaMemcpyAsync(S->h_count, S->d_count, sizeof(unsigned), cudaMemcpyDeviceToHost,
                             S->st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(S->h_count + 1, S->d_err, sizeof(int), cudaMemcpyDeviceToHost,
                             S->st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(S->st)) != cudaSuccess) {
        fprintf(stderr, "Error: B200 search failed: %s\n", cudaGetErrorString(e));
        return -1;
    }
    if (S->h_count[1] != 0) {
        fprintf(stderr, "Error: B200 search kernel timed out waiting for the tensor cores\n");
        return -1;
    }
    const unsigned n = S->h_count[0];
    if (n > S->cap) {
        if (grow_records(S, n + n / 8 + 1024) != 0) return -1;
        return 1;
    }
    if (!S->coll && !(S->coll = cs_collapse_new())) return -1;
    int k[CS_MAX_SLOT], Hk[CS_MAX_SLOT];
    for (int i = 0; i < S->tab.nslot; i++) {
        k[i] = S->tab.slot[i].k;
        Hk[i] = S->tab.slot[i].Hk;
    }
    return cs_collapse_enqueue(S->coll, S->d_recs, n, S->d_chunks, S->tab.nchunks, k, Hk,
                               S->tab.nslot, S->Nprof, S->r_lo, S->lodr, (double)S->N, S->T,
                               threshold, remove, dr_tol, harm_remove, numharm, harm_tol,
                               S->st) == 0 ? 0 : -1;
}

CS_EXPORT int cs_b200_session_collapse_wait(GpuSession *S, CandidateList *out, float *kernel_ms)
{
    if (!S || !out) return -1;
    candlist_init(out);
    if (kernel_ms) *kernel_ms = last_kernel_ms(S);
    if (!S->coll) return 0;
    return cs_collapse_finish(S->coll, S->st, out) == 0 ? 0 : -1;
}

CS_EXPORT int cs_b200_session_collect_collapsed(GpuSession *S, double threshold, int remove,
                                                double dr_tol, int harm_remove, int numharm,
                                                double harm_tol, CandidateList *out,
                                                float *kernel_ms)
{
    if (!S || !out) return -1;
    candlist_init(out);
    const int rc = cs_b200_session_collapse_enqueue(S, threshold, remove, dr_tol, harm_remove,
                                                    numharm, harm_tol);
    if (rc != 0) return rc;
    return cs_b200_session_collapse_wait(S, out, kernel_ms);
}

CS_EXPORT float *cs_b200_session_device_amps(GpuSession *S)
{
    return S ? (float *)S->d_amps : NULL;
}

CS_EXPORT int cs_b200_session_sync(GpuSession *S)
{
    if (!S) return -1;
    return cudaStreamSynchronize(S->st) == cudaSuccess ? 0 : -1;
}

/* ------------------------------------------------------------------ */
/* Several spectra in one launch (cs_b200_multi_enqueue)               */
/* ------------------------------------------------------------------ */
/* Per device: an event marking the last launch that read the kernel's
 * constant-memory tables (arguments and tile offsets). */
struct MultiTables {
    cudaEvent_t done;
};
static std::mutex g_multi_mu;
static MultiTables g_multi[64];

static cudaError_t multi_launch(int nh, int grid, cudaStream_t st, const wsk::Args &a0,
                                const wsk::Multi &mu)
{
    const void *fn = nh == 60 ? (const void *)wsk::search_ws_multi<wsk::Cfg60>
                   : nh == 32 ? (const void *)wsk::search_ws_multi<wsk::Cfg32>
                              : (const void *)wsk::search_ws_multi<wsk::Cfg16>;
    const int nthr = nh == 60 ? wsk::nthreads<wsk::Cfg60>()
                   : nh == 32 ? wsk::nthreads<wsk::Cfg32>() : wsk::nthreads<wsk::Cfg16>();
    wsk::Args a = a0;
    wsk::Multi m = mu;
    void *args[2] = {&a, &m};
    return cudaLaunchKernel(fn, dim3(grid), dim3(nthr), args, (size_t)ws_smem_multi(nh), st);
}

/* The sessions of one multi-spectrum launch: FP32, one device, one
 * warp-specialised configuration (nharms and ladder). */
static bool multi_compatible(GpuSession *const *ss, int n)
{
    const GpuSession *S0 = ss[0];
    for (int i = 0; i < n; i++) {
        const GpuSession *S = ss[i];
        if (!S || !S0 || S->device != S0->device || S->prec64 || !S->use_ws ||
            S->use_ws != S0->use_ws || S->tab.nslot != S0->tab.nslot ||
            S->tab.npad != S0->tab.npad || S->tab.kpad != S0->tab.kpad ||
            memcmp(S->tab.slot, S0->tab.slot, sizeof(CsSlot) * (size_t)S0->tab.nslot) != 0) {
            fprintf(stderr, "Error: a multi-spectrum launch takes FP32 sessions of one "
                            "warp-specialised configuration (same nharms and ladder)\n");
            return false;
        }
    }
    return true;
}

CS_EXPORT int cs_b200_multi_enqueue(GpuSession **ss, int n, const float *const *d_amps,
                                    double threshold, void *stream)
{
#define MCK(call)                                                                 \
    do {                                                                          \
        const cudaError_t e_ = (call);                                            \
        if (e_ != cudaSuccess) {                                                  \
            fprintf(stderr, "Error: multi-spectrum launch: %s failed: %s (line %d)\n", \
                    #call, cudaGetErrorString(e_), __LINE__);                     \
            return -1;                                                            \
        }                                                                         \
    } while (0)
    if (!ss || n < 1) return -1;
    if (n > wsk::MULTI_MAX) {
        fprintf(stderr, "Error: a multi-spectrum launch takes at most %d spectra (got %d)\n",
                wsk::MULTI_MAX, n);
        return -1;
    }
    GpuSession *S0 = ss[0];
    if (!multi_compatible(ss, n)) return -1;
    const int dev = S0->device;
    if (dev < 0 || dev >= 64) return -1;
    MCK(select_device(dev));
    cudaStream_t st = stream ? (cudaStream_t)stream : S0->st;
    std::lock_guard<std::mutex> g(g_multi_mu);
    MultiTables &M = g_multi[dev];
    if (!M.done) MCK(cudaEventCreateWithFlags(&M.done, cudaEventDisableTiming));
    std::vector<wsk::Args> files((size_t)n);
    std::vector<int> off((size_t)n + 1, 0);
    for (int i = 0; i < n; i++) {
        GpuSession *S = ss[i];
        /* the launch stream first waits for each session's queued work */
        if (st != S->st) {
            MCK(cudaEventRecord(S->ev_in, S->st));
            MCK(cudaStreamWaitEvent(st, S->ev_in, 0));
        }
        const float2 *amps = d_amps && d_amps[i] ? (const float2 *)d_amps[i] : S->d_amps;
        MCK(cudaMemsetAsync(S->d_amax, 0, 2 * sizeof(unsigned), st));
        MCK(cudaMemsetAsync(S->d_count, 0, sizeof(unsigned), st));
        MCK(cudaMemsetAsync(S->d_err, 0, sizeof(int), st));
        if (S->namps > 0) {
            const int gr = (int)std::min<long long>((S->namps + 255) / 256, (long long)S->nsm * 8);
            cs_amax_kernel<<<gr, 256, 0, st>>>(amps, S->namps, S->d_amax);
            MCK(cudaGetLastError());
        }
        files[(size_t)i] = ws_args(S, amps, threshold);
        off[(size_t)i + 1] = off[(size_t)i] + S->tab.ntiles;
    }
    const int ntiles = off[(size_t)n];
    if (ntiles <= 0) return 0;
    /* the previous launch on this device may still read the tables */
    MCK(cudaStreamWaitEvent(st, M.done, 0));
    /* pageable sources: each copy returns once its data is staged */
    MCK(cudaMemcpyToSymbolAsync(wsk::c_multi_files, files.data(),
                                files.size() * sizeof(wsk::Args), 0, cudaMemcpyHostToDevice, st));
    MCK(cudaMemcpyToSymbolAsync(wsk::c_multi_off, off.data(), off.size() * sizeof(int), 0,
                                cudaMemcpyHostToDevice, st));
    wsk::Multi mu;
    mu.nfiles = n;
    mu.ntiles = ntiles;
    /* tiles per CTA block (the kernel's schedule); CS_B200_MULTI_BLOCK tunes it */
    mu.block = 64;
    if (const char *e = getenv("CS_B200_MULTI_BLOCK")) mu.block = std::max(1, atoi(e));
    const int grid = std::min(ntiles, S0->nsm);
    MCK(cudaEventRecord(S0->ev0, st));
    MCK(multi_launch(S0->use_ws, grid, st, files[0], mu));
    MCK(cudaEventRecord(S0->ev1, st));
    MCK(cudaEventRecord(M.done, st));
    /* each session's later work (its collect) follows the launch */
    for (int i = 0; i < n; i++)
        if (ss[i]->st != st) MCK(cudaStreamWaitEvent(ss[i]->st, M.done, 0));
    return 0;
#undef MCK
}

/* ------------------------------------------------------------------ */
/* A multi-spectrum search captured as a CUDA graph                    */
/* ------------------------------------------------------------------ */
/* The per-spectrum clears and maxima, the copy of the argument table and
 * tile offsets into constant memory, and the persistent launch over all the
 * spectra's tiles, recorded once by stream capture and replayed as one graph
 * launch.  The graph bakes in each session's buffer addresses, so it records
 * each session's generation and refuses to replay after a reload or a grown
 * record buffer.  The table copies read pinned host memory that the graph
 * object owns. */
struct CsMultiGraph {
    int device = -1;
    std::vector<GpuSession *> ss;
    std::vector<unsigned> gen;
    wsk::Args *h_files = nullptr;   /* pinned: constant-table copy source */
    int *h_off = nullptr;           /* pinned */
    cudaGraphExec_t exec = nullptr;
    cudaStream_t cap = nullptr;     /* capture stream */
};

static void multi_graph_release(CsMultiGraph *G)
{
    if (!G) return;
    if (G->exec) cudaGraphExecDestroy(G->exec);
    if (G->cap) cudaStreamDestroy(G->cap);
    if (G->h_files) cudaFreeHost(G->h_files);
    if (G->h_off) cudaFreeHost(G->h_off);
    delete G;
}

/* The captured body: one stream, no events, no host synchronisation. */
static cudaError_t multi_graph_body(CsMultiGraph *G, int nh, int grid, int nsm, int ntiles,
                                    const float *const *d_amps)
{
    cudaError_t e;
    const cudaStream_t st = G->cap;
    const int n = (int)G->ss.size();
    for (int i = 0; i < n; i++) {
        GpuSession *S = G->ss[(size_t)i];
        const float2 *amps = d_amps && d_amps[i] ? (const float2 *)d_amps[i] : S->d_amps;
        if ((e = cudaMemsetAsync(S->d_amax, 0, 2 * sizeof(unsigned), st)) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(S->d_count, 0, sizeof(unsigned), st)) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(S->d_err, 0, sizeof(int), st)) != cudaSuccess) return e;
        if (S->namps > 0) {
            const int gr = (int)std::min<long long>((S->namps + 255) / 256, (long long)nsm * 8);
            cs_amax_kernel<<<gr, 256, 0, st>>>(amps, S->namps, S->d_amax);
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
        }
    }
    if (ntiles <= 0) return cudaSuccess;
    if ((e = cudaMemcpyToSymbolAsync(wsk::c_multi_files, G->h_files, (size_t)n * sizeof(wsk::Args),
                                     0, cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return e;
    if ((e = cudaMemcpyToSymbolAsync(wsk::c_multi_off, G->h_off, (size_t)(n + 1) * sizeof(int), 0,
                                     cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return e;
    wsk::Multi mu;
    mu.nfiles = n;
    mu.ntiles = ntiles;
    mu.block = 64;
    if (const char *v = getenv("CS_B200_MULTI_BLOCK")) mu.block = std::max(1, atoi(v));
    return multi_launch(nh, grid, st, G->h_files[0], mu);
}

CS_EXPORT CsMultiGraph *cs_b200_multi_graph_create(GpuSession **ss, int n,
                                                   const float *const *d_amps, double threshold)
{
    if (!ss || n < 1) return nullptr;
    if (n > wsk::MULTI_MAX) {
        fprintf(stderr, "Error: a multi-spectrum graph takes at most %d spectra (got %d)\n",
                wsk::MULTI_MAX, n);
        return nullptr;
    }
    if (!multi_compatible(ss, n)) return nullptr;
    GpuSession *S0 = ss[0];
    const int dev = S0->device;
    if (dev < 0 || dev >= 64 || select_device(dev) != cudaSuccess) return nullptr;
    CsMultiGraph *G = new CsMultiGraph();
    G->device = dev;
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaSuccess;
    const char *what = "";
#define GCK(call)                                                                 \
    do {                                                                          \
        if ((e = (call)) != cudaSuccess) { what = #call; goto fail; }             \
    } while (0)
    {
        G->ss.assign(ss, ss + n);
        G->gen.resize((size_t)n);
        GCK(cudaMallocHost((void **)&G->h_files, (size_t)n * sizeof(wsk::Args)));
        GCK(cudaMallocHost((void **)&G->h_off, (size_t)(n + 1) * sizeof(int)));
        G->h_off[0] = 0;
        for (int i = 0; i < n; i++) {
            GpuSession *S = ss[i];
            const float2 *amps = d_amps && d_amps[i] ? (const float2 *)d_amps[i] : S->d_amps;
            G->gen[(size_t)i] = S->gen;
            G->h_files[i] = ws_args(S, amps, threshold);
            G->h_off[i + 1] = G->h_off[i] + S->tab.ntiles;
        }
        const int ntiles = G->h_off[n];
        const int grid = std::min(std::max(ntiles, 1), S0->nsm);
        /* attributes are set outside the capture */
        GCK(ws_prepare_multi(S0->use_ws));
        GCK(cudaStreamCreateWithFlags(&G->cap, cudaStreamNonBlocking));
        /* thread-local capture: other threads' calls (batch slots) stay legal */
        GCK(cudaStreamBeginCapture(G->cap, cudaStreamCaptureModeThreadLocal));
        const cudaError_t eb = multi_graph_body(G, S0->use_ws, grid, S0->nsm, ntiles, d_amps);
        const cudaError_t ee = cudaStreamEndCapture(G->cap, &graph);
        GCK(eb);
        GCK(ee);
        GCK(cudaGraphInstantiate(&G->exec, graph, 0ULL));
        cudaGraphDestroy(graph);
        graph = nullptr;
    }
#undef GCK
    return G;
fail:
    fprintf(stderr, "Error: multi-spectrum graph: %s failed: %s\n", what, cudaGetErrorString(e));
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    multi_graph_release(G);
    return nullptr;
}

CS_EXPORT int cs_b200_multi_graph_launch(CsMultiGraph *G, void *stream)
{
#define GLCK(call)                                                                \
    do {                                                                          \
        const cudaError_t e_ = (call);                                            \
        if (e_ != cudaSuccess) {                                                  \
            fprintf(stderr, "Error: multi-spectrum graph launch: %s failed: %s\n", \
                    #call, cudaGetErrorString(e_));                               \
            return -1;                                                            \
        }                                                                         \
    } while (0)
    if (!G || !G->exec) return -1;
    const int n = (int)G->ss.size();
    for (int i = 0; i < n; i++)
        if (G->ss[(size_t)i]->gen != G->gen[(size_t)i]) {
            fprintf(stderr, "Error: multi-spectrum graph: session %d was reloaded or its record "
                            "buffer grew after the capture; create the graph again\n", i);
            return -2;
        }
    GLCK(select_device(G->device));
    GpuSession *S0 = G->ss[0];
    cudaStream_t st = stream ? (cudaStream_t)stream : S0->st;
    std::lock_guard<std::mutex> g(g_multi_mu);
    MultiTables &M = g_multi[G->device];
    if (!M.done) GLCK(cudaEventCreateWithFlags(&M.done, cudaEventDisableTiming));
    for (int i = 0; i < n; i++) {
        GpuSession *S = G->ss[(size_t)i];
        if (st != S->st) {
            GLCK(cudaEventRecord(S->ev_in, S->st));
            GLCK(cudaStreamWaitEvent(st, S->ev_in, 0));
        }
    }
    /* the previous launch on this device may still read the constant tables */
    GLCK(cudaStreamWaitEvent(st, M.done, 0));
    GLCK(cudaEventRecord(S0->ev0, st));
    GLCK(cudaGraphLaunch(G->exec, st));
    GLCK(cudaEventRecord(S0->ev1, st));
    GLCK(cudaEventRecord(M.done, st));
    for (int i = 0; i < n; i++)
        if (G->ss[(size_t)i]->st != st) GLCK(cudaStreamWaitEvent(G->ss[(size_t)i]->st, M.done, 0));
    return 0;
#undef GLCK
}

CS_EXPORT void cs_b200_multi_graph_free(CsMultiGraph *G)
{
    if (!G) return;
    if (select_device(G->device) == cudaSuccess) {
        /* a replay in flight still reads the pinned tables */
        for (GpuSession *S : G->ss) cudaStreamSynchronize(S->st);
        std::lock_guard<std::mutex> g(g_multi_mu);
        if (g_multi[G->device].done) cudaEventSynchronize(g_multi[G->device].done);
    }
    multi_graph_release(G);
}

#ifdef WSK_TMA_PROF
/* timing studies only: read and clear the column-tile kernel's counters */
CS_EXPORT int cs_b200_tma_prof(unsigned long long *out16)
{
    if (cudaMemcpyFromSymbol(out16, wsk::g_tma_prof, 16 * sizeof(unsigned long long)) != cudaSuccess)
        return -1;
    unsigned long long z[16] = {0};
    return cudaMemcpyToSymbol(wsk::g_tma_prof, z, sizeof(z)) == cudaSuccess ? 0 : -1;
}
#endif

/* ------------------------------------------------------------------ */
/* Search without allocation (cs_b200_session_search_noalloc)          */
/* ------------------------------------------------------------------ */
/* Per-call scratch of the search in static device memory: amax[2], the record
 * counter and the error flag in the first 256 bytes, then up to
 * CS_B200_NOALLOC_MAX_RECS records.  One copy per device, so calls on the same
 * device that overlap on the GPU (two streams, two host threads) race on it. */
static_assert(sizeof(CsRec) == 16, "record layout");
static_assert(sizeof(Candidate) >= sizeof(CsRec), "records are expanded in place");
constexpr size_t NOALLOC_HDR = 256;
constexpr size_t NOALLOC_BYTES = NOALLOC_HDR + (size_t)CS_B200_NOALLOC_MAX_RECS * sizeof(CsRec);
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

constexpr int NOALLOC_MAX_DEVICES = 64;

/* The address is cached per device together with the context it belongs to:
 * a cudaDeviceReset (or a new primary context) maps the module again, maybe
 * elsewhere, so a cached address is used only while its context is current.
 * The context comes from the driver's cuCtxGetCurrent, reached through the
 * runtime's entry-point query; where that is unavailable the address is
 * looked up on every call (a symbol lookup, no allocation). */
struct NoallocSlot {
    void *ctx;
    unsigned char *ptr;
};
static NoallocSlot g_noalloc_slot[NOALLOC_MAX_DEVICES];
static std::mutex g_noalloc_mu;

typedef int (*CtxGetCurrentFn)(void **);
static CtxGetCurrentFn ctx_get_current()
{
    static const CtxGetCurrentFn fn = [] {
        void *p = NULL;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) !=
                cudaSuccess || q != cudaDriverEntryPointSuccess)
            p = NULL;
        return (CtxGetCurrentFn)p;
    }();
    return fn;
}

/* Device address of this device's scratch, for the context current on the
 * calling thread (the caller has made `device` current).  Looked up with
 * cudaGetSymbolAddress on the first call in a context; that lookup can load
 * the module, so the first call on a device belongs before any stream
 * capture. */
static unsigned char *noalloc_scratch(int device)
{
    if (device < 0 || device >= NOALLOC_MAX_DEVICES) return NULL;
    void *ctx = NULL;
    const CtxGetCurrentFn get = ctx_get_current();
    const bool have_ctx = get && get(&ctx) == 0 && ctx;
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    NoallocSlot &sl = g_noalloc_slot[device];
    if (have_ctx && sl.ptr && sl.ctx == ctx) return sl.ptr;
    void *addr = NULL;
    const cudaError_t e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
    if (e != cudaSuccess || !addr) {
        fprintf(stderr, "Error: scratch lookup on device %d failed: %s\n", device,
                cudaGetErrorString(e));
        return NULL;
    }
    sl.ctx = have_ctx ? ctx : NULL;
    sl.ptr = have_ctx ? (unsigned char *)addr : NULL;
    return (unsigned char *)addr;
}

/* (chunk, slot, j) order, as cs_sort_records; in place (heapsort), because
 * the library qsort may take heap memory for large arrays. */
static inline bool rec_less(const CsRec &x, const CsRec &y)
{
    if (x.chunk != y.chunk) return x.chunk < y.chunk;
    if (x.slot != y.slot) return x.slot < y.slot;
    return x.j < y.j;
}

static void rec_sift(CsRec *v, long long i, long long n)
{
    for (;;) {
        long long c = 2 * i + 1;
        if (c >= n) return;
        if (c + 1 < n && rec_less(v[c], v[c + 1])) c++;
        if (!rec_less(v[i], v[c])) return;
        std::swap(v[i], v[c]);
        i = c;
    }
}

static void rec_heapsort(CsRec *v, long long n)
{
    for (long long i = n / 2 - 1; i >= 0; i--) rec_sift(v, i, n);
    for (long long e = n - 1; e > 0; e--) {
        std::swap(v[0], v[e]);
        rec_sift(v, 0, e);
    }
}

/* One record to a Candidate with the arithmetic of cs_harvest
 * (src/cuda.cu:837-881); false if the record is not reported. */
static bool rec_to_candidate(const GpuSession *S, const CsRec &r, double threshold,
                             Candidate *cd)
{
    const double metric = (double)r.metric;
    if (!(metric > threshold)) return false;
    const CsSlot *s = &S->tab.slot[r.slot];
    const double rstart = S->r_lo + (double)S->tab.chunks[r.chunk].i0 * S->lodr;
    const double rfreq = rstart + (double)r.j * S->lodr;
    const double kmul = (double)s->k;
    const double rsel = kmul != 1.0 ? kmul * rfreq : rfreq;
    if (r.slot != 0 && !(rsel < (double)S->N / 2.0)) return false;
    cd->freq = rsel / S->T;
    cd->metric = metric;
    cd->r = rsel;
    cd->nharm = s->Hk;
    cd->ducy = NAN;
    return true;
}

CS_EXPORT int cs_b200_session_search_noalloc(GpuSession *S, const float *d_amps,
                                             double threshold, Candidate *out,
                                             long long cap, long long *nout, void *stream)
{
    if (nout) *nout = 0;
    if (!S || !out || !nout || cap < 0) return -1;
    if (S->prec64) {
        fprintf(stderr, "Error: the allocation-free search takes FP32 sessions\n");
        return -1;
    }
    if (select_device(S->device) != cudaSuccess) return -1;
    unsigned char *base = noalloc_scratch(S->device);
    if (!base) return -1;
    unsigned *amax = (unsigned *)base;               /* [2] */
    unsigned *count = amax + 2;
    int *err = (int *)(amax + 3);
    CsRec *recs = (CsRec *)(base + NOALLOC_HDR);
    cudaStream_t st = stream ? (cudaStream_t)stream : S->st;
    const float2 *amps = d_amps ? (const float2 *)d_amps : S->d_amps;

    cudaError_t e = cudaSuccess;
    if (st != S->st) {
        /* the caller's stream first waits for what is queued on the session
         * stream (a spectrum upload into the session buffer, an earlier
         * search): the hand-off event exists since the session was made */
        if ((e = cudaEventRecord(S->ev_in, S->st)) == cudaSuccess)
            e = cudaStreamWaitEvent(st, S->ev_in, 0);
    }
    if (e == cudaSuccess) e = cudaMemsetAsync(base, 0, 4 * sizeof(unsigned), st);
    if (e == cudaSuccess && S->namps > 0) {
        int g = (int)std::min<long long>((S->namps + 255) / 256, (long long)S->nsm * 8);
        cs_amax_kernel<<<g, 256, 0, st>>>(amps, S->namps, amax);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && S->tab.ntiles > 0) {
        const int grid = std::min(S->tab.ntiles, S->nsm);
        if (S->use_ws) {
            wsk::Args w;
            memset(&w, 0, sizeof(w));
            w.amps = amps;
            w.namps = (int)S->namps;
            w.Wt = S->d_Wt;
            w.A = S->d_A;
            w.harm = S->d_harm2;
            w.chunks = S->d_chunks;
            w.tiles = S->d_tiles;
            w.ntiles = S->tab.ntiles;
            w.bimg = S->d_bimg;
            w.q = S->tab.q;
            w.pnum = S->tab.pnum;
            w.qmagic = magic_for(S->tab.q);
            w.gbound = S->tab.gbound;
            w.amax = amax;
            w.thresh = threshold;
            w.recs = recs;
            w.count = count;
            w.cap = CS_B200_NOALLOC_MAX_RECS;
            w.err = err;
            ws_launch(S->use_ws, grid, st, w);
        } else {
            SearchArgs a = make_args(S, amps, threshold);
            a.amax = amax;
            a.recs = recs;
            a.count = count;
            a.cap = CS_B200_NOALLOC_MAX_RECS;
            a.err = err;
            const int smem = smem_bytes(S->tab);
            if (S->tab.m == 16)
                cs_search_kernel<16><<<grid, CS_NTHREADS, smem, st>>>(a);
            else
                cs_search_kernel<0><<<grid, CS_NTHREADS, smem, st>>>(a);
        }
        e = cudaGetLastError();
    }
    unsigned hdr[4] = {0, 0, 0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(hdr, base, sizeof(hdr), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        fprintf(stderr, "Error: B200 search failed: %s\n", cudaGetErrorString(e));
        return -1;
    }
    if (hdr[3] != 0) {
        fprintf(stderr, "Error: B200 search kernel timed out waiting for the tensor cores\n");
        return -1;
    }
    const long long n = hdr[2];
    if (n > CS_B200_NOALLOC_MAX_RECS) {
        fprintf(stderr, "Error: %lld records above threshold %.3f exceed the %d this entry "
                        "point holds; raise the threshold or use cs_gpu_session_run\n",
                n, threshold, CS_B200_NOALLOC_MAX_RECS);
        return -2;
    }
    if (n > cap) {
        fprintf(stderr, "Error: %lld records above threshold need an output array of at "
                        "least %lld candidates (given %lld)\n", n, n, cap);
        return -3;
    }
    if (n == 0) return 0;
    /* records land at the front of the caller's array and are expanded in
     * place: Candidate i (40 B) never overlaps a record j < i (16 B) */
    CsRec *hrec = (CsRec *)out;
    e = cudaMemcpyAsync(hrec, recs, (size_t)n * sizeof(CsRec), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        fprintf(stderr, "Error: B200 search readback failed: %s\n", cudaGetErrorString(e));
        return -1;
    }
    rec_heapsort(hrec, n);
    for (long long i = n - 1; i >= 0; i--) {
        const CsRec r = hrec[i];
        Candidate cd;
        memset(&cd, 0, sizeof(cd));
        if (!rec_to_candidate(S, r, threshold, &cd)) cd.nharm = 0;   /* dropped */
        out[i] = cd;
    }
    long long k = 0;
    for (long long i = 0; i < n; i++)
        if (out[i].nharm != 0) out[k++] = out[i];
    *nout = k;
    return 0;
}

/* ------------------------------------------------------------------ */
/* Batched search of many spectra (cs_gpu_batch_*)                     */
/* ------------------------------------------------------------------ */
/* One request: a spectrum and its search.  The spectrum stays in the
 * caller's memory until the request is waited for. */
struct BatchReq {
    long long id;
    FFTFile ft;
    SearchParams p;
    double lofreq, hifreq, threshold;
    int lobin, blocksize;
    CandidateList out;
    int status;                      /* 0 ok, -1 error */
    bool done;
    bool rekeyed;                    /* the slot's tables were rebuilt for it */
    int only_slot = -1;              /* >= 0: only this slot takes it */
    bool load_only = false;          /* build tables and buffers, no search */
    std::chrono::steady_clock::time_point t_submit, t_start, t_admit, t_loaded, t_end;
};

/* What a slot's session was last loaded for. */
struct BatchKey {
    long long N, namps, total;
    double T, r_lo, lodr;
    int Nprof;
    SearchParams p;
};

struct BatchSlot {
    GpuSession *S = nullptr;
    BatchKey key;
    bool keyed = false;
    bool busy = false;
    size_t bytes = 0;
};

struct CsBatch {
    int device = 0;
    size_t budget = 0;               /* device bytes all slots may hold; 0: no limit */
    std::vector<BatchSlot> slots;
    std::vector<std::thread> workers;
    std::mutex mu;
    std::condition_variable cv_work, cv_done, cv_mem;
    std::deque<BatchReq *> queue;
    std::unordered_map<long long, BatchReq *> reqs;
    long long next_id = 0;
    bool stop = false;
    bool trace = false;              /* CS_B200_BATCH_TRACE: phase times per request */
};

/* Geometry of a request, as search_file derives it (src/search.c:1247-1262). */
static bool batch_geometry(const BatchReq *r, double *r_lo, double *lodr, long long *total,
                           int *Nprof)
{
    *lodr = r->p.hidr / (double)r->p.nharms;
    *r_lo = r->lobin != 100 ? (double)r->lobin : r->lofreq * r->ft.T;
    const double r_hi = r->hifreq * r->ft.T;
    *total = (long long)floor((r_hi - *r_lo) / *lodr) + 1;
    *Nprof = r->blocksize > 0 ? r->blocksize : 65536;
    return *total > 0;
}

/* Device bytes a request's session needs (spectrum, records, tiles, chunk
 * and interpolation tables), before any reuse. */
static size_t batch_footprint(const BatchReq *r, long long total, int Nprof)
{
    const long long recs = (total * (r->p.ndecim + 1)) / 16 + 4096;
    const long long nchunks = total / std::max(1, Nprof) + 2 * r->p.nharms + 2;
    return (size_t)r->ft.namps * sizeof(float2) + (size_t)recs * sizeof(CsRec) +
           (size_t)(total / CS_TILE_M + nchunks + 1) * 3 * sizeof(int) +
           (size_t)nchunks * sizeof(CsChunk) + ((size_t)4 << 20);
}

/* Admit slot k for a request needing `need` bytes: wait (lock held by the
 * caller through `lk`) until the slots' device memory fits the budget,
 * releasing the sessions of idle slots, and this slot's own, when that makes
 * room.  Returns false if the request can never fit. */
static bool batch_admit(CsBatch *B, int k, size_t need, std::unique_lock<std::mutex> &lk)
{
    if (B->budget == 0) return true;
    if (need > B->budget) return false;
    for (;;) {
        size_t others = 0;
        for (size_t j = 0; j < B->slots.size(); j++)
            if ((int)j != k) others += B->slots[j].bytes;
        BatchSlot &me = B->slots[k];
        if (others + std::max(me.bytes, need) <= B->budget) return true;
        /* make room: this slot's own buffers first, then idle slots' */
        bool freed = false;
        if (me.S && me.bytes > need) {
            session_release(me.S);
            me.S = nullptr;
            me.keyed = false;
            me.bytes = 0;
            freed = true;
        }
        for (size_t j = 0; j < B->slots.size() && !freed; j++) {
            BatchSlot &o = B->slots[j];
            if ((int)j != k && !o.busy && o.S) {
                session_release(o.S);
                o.S = nullptr;
                o.keyed = false;
                o.bytes = 0;
                freed = true;
            }
        }
        if (!freed) B->cv_mem.wait(lk);
    }
}

static void batch_run_one(CsBatch *B, int k, BatchReq *r)
{
    BatchSlot &slot = B->slots[k];
    candlist_init(&r->out);
    r->status = -1;
    double r_lo, lodr;
    long long total;
    int Nprof;
    if (!batch_geometry(r, &r_lo, &lodr, &total, &Nprof)) {
        r->status = 0;                               /* empty band: no trials */
        return;
    }
    BatchKey key;
    memset(&key, 0, sizeof(key));
    key.N = r->ft.N;
    key.namps = r->ft.namps;
    key.total = total;
    key.T = r->ft.T;
    key.r_lo = r_lo;
    key.lodr = lodr;
    key.Nprof = Nprof;
    key.p = r->p;
    GpuSession *S = slot.S;
    if (!S) {
        S = session_new(B->device);
        if (!S) return;
        slot.S = S;
        slot.keyed = false;
    }
    r->rekeyed = false;
    if (!slot.keyed || memcmp(&key, &slot.key, sizeof(key)) != 0) {
        r->rekeyed = true;
        DirectPlanSet plans;
        memset(&plans, 0, sizeof(plans));
        long long *cstarts = NULL, nchunks = 0;
        slot.keyed = false;
        if (direct_plans_build(&plans, &r->p, r_lo) != 0) return;
        const int rc = chunk_starts(&plans, &r->ft, &r->p, total, Nprof, &cstarts, &nchunks);
        const int lrc = rc == 0 ? session_load(S, &r->ft, &r->p, &plans, cstarts, total, Nprof,
                                               nchunks, r_lo, lodr)
                                : -1;
        free(cstarts);
        direct_plans_free(&plans);
        if (lrc != 0) return;
        slot.key = key;
        slot.keyed = true;
    }
    if (r->load_only) {
        r->status = 0;
        return;
    }
    S->p = &r->p;
    r->t_loaded = std::chrono::steady_clock::now();
    if (S->namps > 0 &&
        cudaMemcpyAsync(S->d_amps, r->ft.amps, (size_t)S->namps * sizeof(float2),
                        cudaMemcpyHostToDevice, S->st) != cudaSuccess) {
        fprintf(stderr, "Error: batch spectrum upload failed\n");
        return;
    }
    for (int attempt = 0; attempt < 2; attempt++) {
        if (enqueue_search(S, S->d_amps, r->threshold, false) != cudaSuccess) {
            fprintf(stderr, "Error: batch search launch failed\n");
            candlist_free(&r->out);
            return;
        }
        int rerun = 0;
        if (collect(S, r->threshold, &r->out, &rerun) != 0) {
            candlist_free(&r->out);
            return;
        }
        if (!rerun) break;
    }
    r->status = 0;
}

static void batch_worker(CsBatch *B, int k)
{
    select_device(B->device);
    std::unique_lock<std::mutex> lk(B->mu);
    for (;;) {
        auto mine = [&] {
            auto it = B->queue.begin();
            while (it != B->queue.end() && (*it)->only_slot >= 0 && (*it)->only_slot != k) ++it;
            return it;
        };
        B->cv_work.wait(lk, [&] { return B->stop || mine() != B->queue.end(); });
        const auto it = mine();
        if (it == B->queue.end()) break;             /* stopping, nothing left for this slot */
        BatchReq *r = *it;
        B->queue.erase(it);
        double r_lo, lodr;
        long long total;
        int Nprof;
        const size_t need = batch_geometry(r, &r_lo, &lodr, &total, &Nprof)
                                ? batch_footprint(r, total, Nprof) : 0;
        r->t_start = r->t_admit = r->t_loaded = std::chrono::steady_clock::now();
        r->rekeyed = false;
        if (!batch_admit(B, k, need, lk)) {
            fprintf(stderr, "Error: batch request %lld needs about %zu device bytes, more than "
                            "the budget of %zu\n", r->id, need, B->budget);
            candlist_init(&r->out);
            r->status = -1;
        } else {
            B->slots[k].busy = true;
            /* reserve the room while the slot grows into it */
            B->slots[k].bytes = std::max(B->slots[k].bytes, need);
            lk.unlock();
            r->t_admit = r->t_loaded = std::chrono::steady_clock::now();
            batch_run_one(B, k, r);
            lk.lock();
            BatchSlot &slot = B->slots[k];
            slot.busy = false;
            slot.bytes = slot.S ? session_bytes(slot.S) : 0;
        }
        r->t_end = std::chrono::steady_clock::now();
        if (B->trace) {
            using ms = std::chrono::duration<double, std::milli>;
            fprintf(stderr, "batch trace: id %lld slot %d N %lld nharms %d rekeyed %d "
                            "admit %.3f load %.3f search %.3f ms\n", r->id, k, (long long)r->ft.N,
                    r->p.nharms, (int)r->rekeyed, ms(r->t_admit - r->t_start).count(),
                    ms(r->t_loaded - r->t_admit).count(), ms(r->t_end - r->t_loaded).count());
        }
        r->done = true;
        B->cv_done.notify_all();
        B->cv_mem.notify_all();
    }
}

CS_EXPORT CsBatch *cs_gpu_batch_create(int device, int nslots, size_t mem_budget)
{
    if (nslots < 1 || nslots > 16) {
        fprintf(stderr, "Error: cs_gpu_batch_create: 1 to 16 slots\n");
        return NULL;
    }
    char msg[256];
    if (cs_gpu_available(device, msg, sizeof(msg)) != 1) {
        fprintf(stderr, "Error: cs_gpu_batch_create: %s\n", msg);
        return NULL;
    }
    CsBatch *B = new CsBatch();
    B->device = device;
    B->budget = mem_budget;
    B->trace = getenv("CS_B200_BATCH_TRACE") != nullptr;
    B->slots.resize(nslots);
    for (int k = 0; k < nslots; k++) B->workers.emplace_back(batch_worker, B, k);
    return B;
}

CS_EXPORT long long cs_gpu_batch_submit(CsBatch *B, const FFTFile *ft, const SearchParams *p,
                                        double lofreq, double hifreq, int lobin, int blocksize,
                                        double threshold)
{
    if (!B || !ft || !p || (ft->namps > 0 && !ft->amps)) return -1;
    BatchReq *r = new BatchReq();
    r->ft = *ft;
    r->p = *p;
    r->lofreq = lofreq;
    r->hifreq = hifreq;
    r->lobin = lobin;
    r->blocksize = blocksize;
    r->threshold = threshold;
    r->done = false;
    r->status = -1;
    candlist_init(&r->out);
    r->t_submit = std::chrono::steady_clock::now();
    std::lock_guard<std::mutex> g(B->mu);
    r->id = B->next_id++;
    B->reqs[r->id] = r;
    B->queue.push_back(r);
    B->cv_work.notify_one();
    return r->id;
}

CS_EXPORT int cs_gpu_batch_wait(CsBatch *B, long long id, CandidateList *out, double *queued_ms,
                                double *run_ms)
{
    if (out) candlist_init(out);
    if (!B) return -1;
    std::unique_lock<std::mutex> lk(B->mu);
    auto it = B->reqs.find(id);
    if (it == B->reqs.end()) return -1;
    BatchReq *r = it->second;
    B->cv_done.wait(lk, [&] { return r->done; });
    B->reqs.erase(it);
    lk.unlock();
    const int status = r->status;
    if (out) out->v = r->out.v, out->n = r->out.n, out->cap = r->out.cap;
    else candlist_free(&r->out);
    using ms = std::chrono::duration<double, std::milli>;
    if (queued_ms) *queued_ms = ms(r->t_start - r->t_submit).count();
    if (run_ms) *run_ms = ms(r->t_end - r->t_start).count();
    delete r;
    return status;
}

CS_EXPORT long long cs_gpu_batch_device_bytes(CsBatch *B)
{
    if (!B) return -1;
    std::lock_guard<std::mutex> g(B->mu);
    long long total = 0;
    for (const BatchSlot &sl : B->slots) total += (long long)sl.bytes;
    return total;
}

CS_EXPORT int cs_gpu_batch_cancel(CsBatch *B, long long id)
{
    if (!B) return -1;
    std::lock_guard<std::mutex> g(B->mu);
    auto it = B->reqs.find(id);
    if (it == B->reqs.end()) return -1;          /* unknown, or already waited for */
    BatchReq *r = it->second;
    for (auto q = B->queue.begin(); q != B->queue.end(); ++q) {
        if (*q != r) continue;
        B->queue.erase(q);
        r->status = -2;
        r->t_start = r->t_end = std::chrono::steady_clock::now();
        r->done = true;
        B->cv_done.notify_all();
        return 0;
    }
    return 1;                                    /* on a slot or finished */
}

CS_EXPORT int cs_gpu_batch_warm(CsBatch *B, const FFTFile *ft, const SearchParams *p,
                                double lofreq, double hifreq, int lobin, int blocksize)
{
    if (!B || !ft || !p) return -1;
    std::vector<BatchReq *> mine;
    {
        std::lock_guard<std::mutex> g(B->mu);
        for (int k = 0; k < (int)B->slots.size(); k++) {
            BatchReq *r = new BatchReq();
            r->ft = *ft;
            r->ft.amps = NULL;                       /* nothing is uploaded */
            r->p = *p;
            r->lofreq = lofreq;
            r->hifreq = hifreq;
            r->lobin = lobin;
            r->blocksize = blocksize;
            r->threshold = p->threshold;
            r->status = -1;
            r->done = false;
            r->only_slot = k;
            r->load_only = true;
            candlist_init(&r->out);
            r->t_submit = std::chrono::steady_clock::now();
            r->id = B->next_id++;
            B->queue.push_back(r);
            mine.push_back(r);
        }
    }
    B->cv_work.notify_all();
    int rc = 0;
    std::unique_lock<std::mutex> lk(B->mu);
    for (BatchReq *r : mine) {
        B->cv_done.wait(lk, [&] { return r->done; });
        if (r->status != 0) rc = -1;
        candlist_free(&r->out);
        delete r;
    }
    return rc;
}

CS_EXPORT int cs_gpu_batch_pending(CsBatch *B)
{
    if (!B) return -1;
    std::lock_guard<std::mutex> g(B->mu);
    return (int)B->reqs.size();
}

CS_EXPORT void cs_gpu_batch_free(CsBatch *B)
{
    if (!B) return;
    {
        std::lock_guard<std::mutex> g(B->mu);
        B->stop = true;
    }
    B->cv_work.notify_all();
    for (auto &t : B->workers) t.join();
    select_device(B->device);
    for (auto &sl : B->slots)
        if (sl.S) session_release(sl.S);
    for (auto &kv : B->reqs) {
        candlist_free(&kv.second->out);
        delete kv.second;
    }
    delete B;
}
