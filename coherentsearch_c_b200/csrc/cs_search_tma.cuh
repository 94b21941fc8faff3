/*
 * Column-tile search kernels: the default ladder (m = 16, k = 1..6) at
 * nharms 60, 32 and 16 with the spectrum windows staged in shared memory by
 * TMA.  Same configurations, tensor-core DFT and epilogue as search_ws
 * (cs_search_ws.cuh); what changes is how the interpolation gets its data.
 *
 * The trial grid has period q = 1/lodr (120, 64, 32 at hidr 0.5): trials t
 * and t + q sit at the same fractional Fourier position, one bin apart per
 * harmonic number.  Cut the trials into column tiles of q, aligned at
 * multiples of q: every column tile then has the same interpolation phase
 * pattern, and harmonic h of trial i of column tile c starts its window at
 *     X_h(c, i) = rfloor0_h - 7 + c*h + R_h(i),
 *     R_h(i)    = floor(i*h/q) + [ (i*h mod q) >= carry_res_h ],
 * the same bin arithmetic as src/cuda.cu:104-116 restated by column tile.
 * A warp takes 32 column tiles (a super-tile) at the same trial index, so
 * its lanes share the weight row and phase factor of that index (broadcast
 * reads), and each lane interpolates two consecutive trials of its column
 * tile from one window of 18 bins read with float4 loads.
 *
 * Staging: for each (round, harmonic) the window rows of the 32 column
 * tiles are one 2D TMA box per parity class (rows 2h bins apart, 16 rows x
 * 22 bins), plus one bulk copy of the 8 weight rows of the round; an
 * mbarrier with an expected byte count marks the stage full.  The boxes
 * read two zero-padded copies of the spectrum made by cs_tma_prep_kernel,
 * one shifted by a bin, so that every box starts on an even bin (16-byte
 * TMA coordinate).  No multicast; the tensor maps cover this GPU's own
 * buffers only.
 *
 * One round = 8 consecutive trials of the 32 column tiles of a super-tile =
 * two DFT tiles: A0 holds trials i0 + 2r, A1 trials i0 + 2r + 1, where r is
 * the TMEM lane quarter of the warp (a warp may only write its own 32
 * lanes).  Row 32r + l of both is column tile col_of_lane(l).  Warps:
 *   0..7   interpolation: warp 4s + r takes harmonic set s (half the
 *          harmonic blocks) for TMEM quarter r; the set's first lane issues
 *          its TMA stages ahead;
 *   8..15  epilogue (the search_ws one, rows carrying their own chunk) and,
 *          on one thread, the MMAs of a round (A0 -> D0, A1 -> D1).
 * Hand-off by mbarriers: stage full (TMA bytes) / empty (4 warps), a_full (8
 * interpolation warps), a_empty and d_full (tcgen05.commit).  Every wait is
 * bounded; on timeout the kernel records an error, waits for its copies in
 * flight, frees tensor memory and returns.
 *
 * The interpolation arithmetic is the search_ws one (16-tap FP32 FMA chain
 * in tap order with packed f32x2 FMAs, unfused rotation), so the harmonic
 * amplitudes are bit-identical to it and to the reference's.
 */
#pragma once

namespace wsk {

constexpr int TMA_BOXW = 22;                        /* bins per staged row */
constexpr int TMA_ROWS = 16;                        /* rows per box (one parity class) */
constexpr int TMA_BOX_BYTES = TMA_ROWS * TMA_BOXW * 8;     /* 2816 */
constexpr int TMA_BOX1 = 2944;                      /* second box, 128-byte aligned */
constexpr int TMA_WROW = 20;                        /* floats per weight row: 16 taps, A, 2 pad */
constexpr int TMA_WOFF = 5760;                      /* weight rows of the round */
constexpr int TMA_WBYTES = 8 * TMA_WROW * 4;        /* 640 */
constexpr int TMA_STG = 6400;                       /* bytes per stage */
#ifndef WSK_TMA_NSTG
#define WSK_TMA_NSTG 12
#endif
constexpr int TMA_NSTG = WSK_TMA_NSTG;              /* stages per harmonic set */
constexpr int TMA_TX = 2 * TMA_BOX_BYTES + TMA_WBYTES;
constexpr int TMA_FRONT = 64;                       /* zero bins before the staged spectrum */
constexpr int TMA_BACK = 2048;                      /* and after it */
static_assert(TMA_BOX1 >= TMA_BOX_BYTES && TMA_BOX1 % 128 == 0, "box layout");
static_assert(TMA_WOFF >= TMA_BOX1 + TMA_BOX_BYTES && TMA_WOFF % 128 == 0, "stage layout");
static_assert(TMA_WOFF + TMA_WBYTES <= TMA_STG && TMA_STG % 128 == 0, "stage size");
static_assert(TMA_BACK >= 30 * MAX_NH + 2 * TMA_BOXW, "rows of a box stay inside the copy");
/* barriers: full[2][NSTG], empty[2][NSTG], a_full, a_empty, d_full, then the
 * tensor-memory slot */
constexpr int TMA_BAR_BYTES = (8 * 4 * TMA_NSTG + 24 + 4 + 127) / 128 * 128;

/* WSK_TMA_PROF builds (timing studies only) add per-role cycle counters:
 * 0 interp total, 1 stage-full waits, 2 a_empty waits, 3 refill waits,
 * 4 epilogue total, 5 d_full waits + barrier, 6 a_full waits (MMA issuer),
 * 7 epilogue compute. */
#ifdef WSK_TMA_PROF
__device__ unsigned long long g_tma_prof[16];
#define TPROF_T0(v) const long long v = clock64()
#define TPROF_ADD(i, v) do { if (lane == 0) atomicAdd(&g_tma_prof[i], (unsigned long long)(clock64() - (v))); } while (0)
#else
#define TPROF_T0(v)
#define TPROF_ADD(i, v)
#endif

struct TArgs {
    const void *maps;           /* CUtensorMap [nh][2]: copy 0, copy 1 (shifted a bin) */
    const float *wtab;          /* [nh][q][TMA_WROW]: weights, A re, A im by trial index */
    const int *cchunk;          /* chunk of the first trial of every column tile */
    int nchunks;
    int total;                  /* trials */
    int q;                      /* trials per column tile */
    uint32_t qmag;              /* floor(2^32 / q) + 1 */
    int nitems;                 /* rounds = super-tiles x q/8 */
    int rounds_per_super;       /* q/8 */
};

/* Column tile of lane l inside its super-tile: lanes 0..15 the even ones
 * (first box), lanes 16..31 the odd ones (second box), so that a quarter
 * warp's 16-byte reads hit eight different bank groups. */
static __device__ __forceinline__ int col_of_lane(int l)
{
    return l < 16 ? 2 * l : 2 * (l - 16) + 1;
}

/* Bin offset R_h(i) of trial index i inside a column tile (see above). */
static __device__ __forceinline__ int roff(uint32_t i, uint32_t h, uint32_t q, uint32_t qmag,
                                          int carry_res)
{
    uint32_t quo, rem;
    divmod_q(i * h, q, qmag, quo, rem);
    return (int)quo + ((int)rem >= carry_res ? 1 : 0);
}

/* Chunk of trial t, starting from the chunk of its column tile's first trial. */
static __device__ __forceinline__ int chunk_of(const Args &a, const TArgs &x, int c, int t)
{
    int ci = x.cchunk[c];
    while (ci + 1 < x.nchunks && (long long)t >= a.chunks[ci + 1].i0) ci++;
    return ci;
}

static __device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                 :: "r"(bar), "r"(bytes) : "memory");
}

static __device__ __forceinline__ void tma_box(uint32_t dst, const void *map, int x, int y,
                                               uint32_t bar)
{
    asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%2, %3}], [%4];"
                 :: "r"(dst), "l"(map), "r"(x), "r"(y), "r"(bar) : "memory");
}

static __device__ __forceinline__ void bulk_copy(uint32_t dst, const void *src, uint32_t bytes,
                                                 uint32_t bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes"
                 " [%0], [%1], %2, [%3];"
                 :: "r"(dst), "l"(src), "r"(bytes), "r"(bar) : "memory");
}

/* 16-tap FP32 chain (tap order, packed f32x2 FMA: each lane a correctly
 * rounded fma, as two scalar chains) and the unfused rotation.  wrow points
 * at a weight row in shared memory: plain loads, so that the compiler can
 * issue them ahead of the chain (the stage's mbarrier wait, an asm with a
 * memory clobber, keeps them after the data has landed). */
template <int OFF>
static __device__ __forceinline__ float2 chain16(const float2 *v, const float *wrow)
{
    float2 acc = make_float2(0.0f, 0.0f);
#pragma unroll
    for (int i4 = 0; i4 < 4; i4++) {
        const float4 w = reinterpret_cast<const float4 *>(wrow)[i4];
        acc = __ffma2_rn(make_float2(w.x, w.x), v[OFF + 4 * i4 + 0], acc);
        acc = __ffma2_rn(make_float2(w.y, w.y), v[OFF + 4 * i4 + 1], acc);
        acc = __ffma2_rn(make_float2(w.z, w.z), v[OFF + 4 * i4 + 2], acc);
        acc = __ffma2_rn(make_float2(w.w, w.w), v[OFF + 4 * i4 + 3], acc);
    }
    const float2 g = reinterpret_cast<const float2 *>(wrow)[8];
    return make_float2(__fsub_rn(__fmul_rn(g.x, acc.x), __fmul_rn(g.y, acc.y)),
                       __fadd_rn(__fmul_rn(g.x, acc.y), __fmul_rn(g.y, acc.x)));
}

/* fp16 hi/lo split of a scaled amplitude (search_ws's). */
static __device__ __forceinline__ void split_hl(float2 x, float scale, uint32_t &hw, uint32_t &lw)
{
    const float2 sc = make_float2(x.x * scale, x.y * scale);
    const __half2 hi = __float22half2_rn(sc);
    const float2 back = __half22float2(hi);
    const __half2 lo = __float22half2_rn(make_float2(__fsub_rn(sc.x, back.x),
                                                     __fsub_rn(sc.y, back.y)));
    hw = *reinterpret_cast<const uint32_t *>(&hi);
    lw = *reinterpret_cast<const uint32_t *>(&lo);
}

template <class C>
__host__ __device__ constexpr int tma_smem_bytes()
{
    return 2 * C::NPAD * C::KPAD * 2 + 2 * TMA_NSTG * TMA_STG + TMA_BAR_BYTES + C::NH * (int)sizeof(Harm);
}

/* Issue stage n of harmonic set s: the two boxes and the weight rows of
 * (round, harmonic) number n of this CTA's sequence. */
static __device__ __forceinline__ void tma_issue(const Args &a, const TArgs &x, const Harm *hs,
                                                 int item0, int hb0, int nhs, int n,
                                                 uint32_t stg, uint32_t full)
{
    const int item = item0 + n / nhs;
    const int h = 4 * hb0 + 1 + n % nhs;
    const int sup = item / x.rounds_per_super, i0 = 8 * (item % x.rounds_per_super);
    const Harm &hm = hs[h - 1];
    const int r0 = roff((uint32_t)i0, (uint32_t)h, (uint32_t)x.q, x.qmag, hm.carry_res);
    /* first bin of the even-column rows (columns 0, 2, ...) in the padded copy */
    const int xa = hm.rfloor0 - M / 2 + 1 + 32 * sup * h + r0 + TMA_FRONT;
    const char *maps = reinterpret_cast<const char *>(x.maps) + (size_t)(h - 1) * 2 * 128;
    mbar_expect_tx(full, TMA_TX);
#pragma unroll
    for (int cls = 0; cls < 2; cls++) {
        const int xs = xa + cls * h;            /* odd-column rows start one column later */
        const int src = xs & 1;
        tma_box(stg + (cls ? TMA_BOX1 : 0), maps + src * 128, 2 * (xs - src), 0, full);
    }
    bulk_copy(stg + TMA_WOFF, x.wtab + ((size_t)(h - 1) * x.q + i0) * TMA_WROW, TMA_WBYTES, full);
}

template <class C>
__global__ void __launch_bounds__(512, 1)
search_tma(const __grid_constant__ Args a, const __grid_constant__ TArgs x)
{
    constexpr int NH = C::NH, NPAD = C::NPAD, KPAD = C::KPAD, AHALF = KPAD / 2;
    constexpr int NB = NH / 4;                      /* harmonic blocks */
    constexpr int HB1 = (NB + 1) / 2;               /* set 0: blocks 0..HB1-1 */
    constexpr int BIMG = NPAD * KPAD * 2;
    constexpr int SM_B = 0, SM_STG = 2 * BIMG, SM_BAR = SM_STG + 2 * TMA_NSTG * TMA_STG;
    constexpr int SM_HARM = SM_BAR + TMA_BAR_BYTES;
    static_assert(SM_HARM + NH * (int)sizeof(Harm) == tma_smem_bytes<C>(), "layout");
    static_assert(NH % 4 == 0 && 2 * NH <= KPAD && NPAD <= D_STRIDE, "shape");
    extern __shared__ __align__(1024) unsigned char smem[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    /* barriers: full[2][NSTG], empty[2][NSTG], a_full, a_empty, d_full; tmem slot */
    const uint32_t bar0 = smem_u32(smem + SM_BAR);
    const uint32_t bar_full = bar0, bar_empty = bar0 + 8 * 2 * TMA_NSTG;
    const uint32_t bar_afull = bar0 + 8 * 4 * TMA_NSTG;
    const uint32_t bar_aempty = bar_afull + 8, bar_dfull = bar_afull + 16;
    uint32_t *tm_slot = reinterpret_cast<uint32_t *>(smem + SM_BAR + 8 * 4 * TMA_NSTG + 24);
    Harm *hs = reinterpret_cast<Harm *>(smem + SM_HARM);

    if (warp == 0) tmem_alloc(smem_u32(tm_slot), TMEM_COLS);
    for (int h = tid; h < NH; h += 512) hs[h] = a.harm[h];
    if (tid == 0) {
        for (int i = 0; i < 2 * TMA_NSTG; i++) {
            mbar_init(bar_full + 8 * i, 1);
            mbar_init(bar_empty + 8 * i, 4);
        }
        mbar_init(bar_afull, 8);
        mbar_init(bar_aempty, 1);
        mbar_init(bar_dfull, 1);
    }
    {
        uint4 *dst = reinterpret_cast<uint4 *>(smem + SM_B);
        for (int i = tid; i < (2 * BIMG) / 16; i += 512) dst[i] = a.bimg[i];
    }
    fence_proxy_async();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tm_slot;
    const float scale = operand_scale(a.amax, a.gbound);
    const float inv_scale = 1.0f / scale;
    /* each CTA owns a contiguous run of rounds: neighbouring rounds read the
     * same spectrum region */
    const int per_cta = (x.nitems + gridDim.x - 1) / gridDim.x;
    const int item_begin = min(x.nitems, (int)blockIdx.x * per_cta);
    const int item_end = min(x.nitems, item_begin + per_cta);
    const int nround = item_end - item_begin;

    if (warp < 8) {
        /* ---------------- interpolation: set s, TMEM quarter r ---------------- */
        const int s = warp >> 2, r = warp & 3;
        const int hb0 = s ? HB1 : 0, hb1 = s ? NB : HB1;
        const int nhs = 4 * (hb1 - hb0);             /* harmonics of this set */
        const int nseq = nround * nhs;
        const bool leader = (r == 0 && lane == 0);
        const uint32_t stg0 = smem_u32(smem + SM_STG + s * TMA_NSTG * TMA_STG);
        const unsigned char *stgp0 = smem + SM_STG + s * TMA_NSTG * TMA_STG;
        const uint32_t fullb = bar_full + 8 * TMA_NSTG * s, emptyb = bar_empty + 8 * TMA_NSTG * s;
        const uint32_t tl = (uint32_t)(r * 32) << 16;
        const uint32_t abuf0 = tmem + tl + (uint32_t)TM_A, abuf1 = abuf0 + KPAD;
        const int col = col_of_lane(lane), cls = lane >> 4, row = lane & 15;
        int issued = 0;
        bool ok = true;
        if (leader) {
            /* the K padding columns (harmonics past nharms) stay zero */
            for (; issued < min(nseq, TMA_NSTG); issued++)
                tma_issue(a, x, hs, item_begin, hb0, nhs, issued, stg0 + issued * TMA_STG,
                          fullb + 8 * issued);
        }
        if (s == 1) {
#pragma unroll
            for (int c = 2 * NH; c < KPAD; c += 8) {
                tmem_st4(abuf0 + c / 2, 0, 0, 0, 0);
                tmem_st4(abuf0 + AHALF + c / 2, 0, 0, 0, 0);
                tmem_st4(abuf1 + c / 2, 0, 0, 0, 0);
                tmem_st4(abuf1 + AHALF + c / 2, 0, 0, 0, 0);
            }
        }
        int n = 0;
        TPROF_T0(p_all);
        for (int it = 0; it < nround && ok; it++) {
            const int item = item_begin + it;
            const int sup = item / x.rounds_per_super, i0 = 8 * (item % x.rounds_per_super);
            const int ta = i0 + 2 * r;               /* trial indices of A0 and A1 rows */
            const int cabs = 32 * sup + col;
            const int t0 = cabs * x.q + ta;
            unsigned long long fa = 0, fb = 0;
            if (t0 < x.total) fa = a.chunks[chunk_of(a, x, cabs, t0)].filled;
            if (t0 + 1 < x.total) fb = a.chunks[chunk_of(a, x, cabs, t0 + 1)].filled;
            {
                TPROF_T0(p_ae);
                const bool got = it < 1 || mbar_wait(bar_aempty, (it - 1) & 1);
                TPROF_ADD(2, p_ae);
                if (!got) {
                    if (lane == 0) atomicExch(a.err, 1);
                    ok = false;
                    break;
                }
            }
            tc_fence_after();
            for (int hb = hb0; hb < hb1 && ok; hb++) {
                uint32_t hwa[4], lwa[4], hwb[4], lwb[4];
#pragma unroll
                for (int u = 0; u < 4; u++, n++) {
                    const int h = 4 * hb + u + 1;
                    const int stage = n % TMA_NSTG;
                    const unsigned char *stgp = stgp0 + stage * TMA_STG;
                    {
                        TPROF_T0(p_f);
                        if (ok && !mbar_wait(fullb + 8 * stage, (n / TMA_NSTG) & 1)) {
                            if (lane == 0) atomicExch(a.err, 1);
                            ok = false;
                        }
                        TPROF_ADD(1, p_f);
                    }
                    float2 xa = make_float2(0.0f, 0.0f), xb = xa;
                    if (ok) {
                        const Harm &hm = hs[h - 1];
                        const int r0 = roff((uint32_t)i0, (uint32_t)h, (uint32_t)x.q, x.qmag,
                                            hm.carry_res);
                        const int oa = roff((uint32_t)ta, (uint32_t)h, (uint32_t)x.q, x.qmag,
                                            hm.carry_res) - r0;
                        const int ob = roff((uint32_t)(ta + 1), (uint32_t)h, (uint32_t)x.q, x.qmag,
                                            hm.carry_res) - r0;
                        /* 18 bins from the even bin at or below oa (oa <= 3, so in the row) */
                        const float4 *rowa = reinterpret_cast<const float4 *>(
                            stgp + (cls ? TMA_BOX1 : 0) + row * TMA_BOXW * 8 + (oa >> 1) * 16);
                        float2 v[18];
#pragma unroll
                        for (int c = 0; c < 9; c++) {
                            const float4 f = rowa[c];
                            v[2 * c] = make_float2(f.x, f.y);
                            v[2 * c + 1] = make_float2(f.z, f.w);
                        }
                        const float *wa = reinterpret_cast<const float *>(stgp + TMA_WOFF) +
                                          2 * r * TMA_WROW;
                        const float *wb = wa + TMA_WROW;
                        const int pa = oa & 1, db = ob - oa;
                        if (pa == 0) {
                            xa = chain16<0>(v, wa);
                            xb = db ? chain16<1>(v, wb) : chain16<0>(v, wb);
                        } else {
                            xa = chain16<1>(v, wa);
                            xb = db ? chain16<2>(v, wb) : chain16<1>(v, wb);
                        }
                        if (!((fa >> (h - 1)) & 1ULL)) xa = make_float2(0.0f, 0.0f);
                        if (!((fb >> (h - 1)) & 1ULL)) xb = make_float2(0.0f, 0.0f);
                    }
                    __syncwarp();
                    if (lane == 0) mbar_arrive(emptyb + 8 * stage);
                    /* refill the stage of step n-1 (its readers are done by now,
                     * or nearly) with step n-1+NSTG */
                    if (leader && ok && n >= 1 && issued < nseq && issued == n - 1 + TMA_NSTG) {
                        const int ps = (n - 1) % TMA_NSTG;
#ifdef WSK_TMA_PROF
                        const long long p_r = clock64();
                        const bool got_e = mbar_wait(emptyb + 8 * ps, ((n - 1) / TMA_NSTG) & 1);
                        atomicAdd(&g_tma_prof[3], (unsigned long long)(clock64() - p_r));
                        if (!got_e) {
#else
                        if (!mbar_wait(emptyb + 8 * ps, ((n - 1) / TMA_NSTG) & 1)) {
#endif
                            atomicExch(a.err, 1);
                            ok = false;
                        } else {
                            tma_issue(a, x, hs, item_begin, hb0, nhs, issued,
                                      stg0 + ps * TMA_STG, fullb + 8 * ps);
                            issued++;
                        }
                    }
                    split_hl(xa, scale, hwa[u], lwa[u]);
                    split_hl(xb, scale, hwb[u], lwb[u]);
                }
                ok = __shfl_sync(0xffffffffu, (int)ok, 0) != 0;
                tmem_st4(abuf0 + 4 * hb, hwa[0], hwa[1], hwa[2], hwa[3]);
                tmem_st4(abuf0 + AHALF + 4 * hb, lwa[0], lwa[1], lwa[2], lwa[3]);
                tmem_st4(abuf1 + 4 * hb, hwb[0], hwb[1], hwb[2], hwb[3]);
                tmem_st4(abuf1 + AHALF + 4 * hb, lwb[0], lwb[1], lwb[2], lwb[3]);
            }
            asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(bar_afull);
        }
        TPROF_ADD(0, p_all);
        if (!ok && lane == 0) atomicExch(a.err, 1);
        /* drain: every stage this set issued has landed before the CTA ends */
        if (leader) {
            for (int k = n; k < issued; k++)
                mbar_wait(fullb + 8 * (k % TMA_NSTG), (k / TMA_NSTG) & 1);
        }
    } else {
        /* ------------- tensor cores and epilogue (warps 8..15) ------------- */
        const int e = warp - 8;
        const int quarter = e & 3, grp = e >> 2;
        const bool leader = (warp == 8 && lane == 0);
        const uint32_t idesc = (1u << 4) | ((uint32_t)(NPAD >> 3) << 17) |
                               ((uint32_t)(CS_TILE_M >> 4) << 24);
        const uint32_t lbo_b = NPAD * 16;
        const uint32_t b_hi = smem_u32(smem + SM_B), b_lo = b_hi + BIMG;
        const int col = col_of_lane(lane);
        int issued = 0, consumed = 0;
        bool ok = true;
        TPROF_T0(p_all);
        for (int it = 0; it < nround; it++) {
            if (leader && ok) {
#ifdef WSK_TMA_PROF
                const long long p_a = clock64();
                const bool got_a = mbar_wait(bar_afull, it & 1);
                atomicAdd(&g_tma_prof[6], (unsigned long long)(clock64() - p_a));
                if (!got_a) {
#else
                if (!mbar_wait(bar_afull, it & 1)) {
#endif
                    ok = false;
                    atomicExch(a.err, 1);
                } else {
                    tc_fence_after();
#pragma unroll
                    for (int b = 0; b < 2; b++) {
                        const uint32_t a_hi = tmem + (uint32_t)(TM_A + KPAD * b), a_lo = a_hi + AHALF;
                        const uint32_t d = tmem + (uint32_t)(TM_D + D_STRIDE * b);
                        uint32_t acc = 0;
#pragma unroll
                        for (int pass = 0; pass < 3; pass++) {
                            const uint32_t abase = (pass == 1) ? a_lo : a_hi;
                            const uint32_t bbase = (pass == 2) ? b_lo : b_hi;
#pragma unroll
                            for (int k = 0; k < KPAD / 16; k++) {
                                mma_f16_ts(d, abase + (uint32_t)(8 * k),
                                           umma_desc(bbase + (uint32_t)k * 2 * lbo_b, lbo_b, 128),
                                           idesc, acc);
                                acc = 1;
                            }
                        }
                    }
                    mma_commit(bar_aempty);
                    mma_commit(bar_dfull);
                    issued++;
                }
            }
            __syncwarp();
            TPROF_T0(p_d);
            const bool got = mbar_wait(bar_dfull, it & 1);
            const bool all = epi_bar_and(got && ok);
            TPROF_ADD(5, p_d);
            if (!all) {
                if (lane == 0) atomicExch(a.err, 1);
                ok = false;
                break;
            }
            TPROF_T0(p_e);
            consumed++;
            tc_fence_after();
            const int item = item_begin + it;
            const int sup = item / x.rounds_per_super, i0 = 8 * (item % x.rounds_per_super);
            const int cabs = 32 * sup + col;
#pragma unroll 1
            for (int b = 0; b < 2; b++) {
                const int t = cabs * x.q + i0 + 2 * quarter + b;
                const bool valid = t < x.total;
                const int ci = valid ? chunk_of(a, x, cabs, t) : 0;
                const CsChunk &ch = a.chunks[ci];
                const int j = t - (int)ch.i0;
                const uint32_t trow = tmem + (uint32_t)(TM_D + b * D_STRIDE) +
                                      ((uint32_t)(quarter * 32) << 16);
                C::epilogue(grp, trow, ch, a, valid, ci, j, lane, inv_scale);
            }
            TPROF_ADD(7, p_e);
            tc_fence_before();
            epi_bar_and(true);      /* D0 and D1 free for the MMAs of the next round */
        }
        TPROF_ADD(4, p_all);
        /* drain: never free tensor memory under an MMA in flight */
        if (leader) {
            for (int k = consumed; k < issued; k++) mbar_wait(bar_dfull, k & 1);
        }
    }
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, TMEM_COLS);
    }
}

/* Spectrum maximum (cs_amax_kernel's) plus the two staged copies: copy 0 =
 * the spectrum at bin TMA_FRONT, copy 1 = the same shifted down a bin; the
 * zero pads around them are written once when the session is loaded. */
__global__ void tma_prep_kernel(const float2 *__restrict__ amps, int namps,
                                float2 *__restrict__ c0, float2 *__restrict__ c1,
                                unsigned *__restrict__ out)
{
    float mx = 0.0f;
    unsigned bad = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < namps; i += gridDim.x * blockDim.x) {
        const float2 v = amps[i];
        c0[TMA_FRONT + i] = v;
        c1[TMA_FRONT + i - 1] = v;                  /* TMA_FRONT >= 1 */
        const float m = fmaxf(fabsf(v.x), fabsf(v.y));
        if (!(m <= 3.0e38f)) bad = 1;
        mx = fmaxf(mx, m);
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

}  // namespace wsk
