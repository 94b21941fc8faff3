/*
 * The m-tap interpolation of every (trial, harmonic) as tensor-core GEMMs
 * (src/cuda.cu:86-140 computes the same values trial by trial).
 *
 * For harmonic h the trials come in column tiles of q = 2 nh trials that
 * share one phase pattern: trial t = c q + i (pnum 1) starts its window at
 * bin base_h + c h + R_h(i), R_h(i) = floor(i h / q) + [i h mod q >=
 * carry_res_h], and uses weight row t mod P_h = i mod P_h.  So for a band
 * of NB consecutive positions i0 .. i0 + NB - 1 of every column tile
 *
 *   X_h(c q + i) = sum_k Bh[i][k] . amp[base_h + c h + R_h(i0) + k]
 *
 * with one matrix Bh (the band's weights, the rotation by the row's gain
 * folded in: (gr W, -gi W; gi W, gr W) per tap) shared by all column tiles.
 * With 128 column tiles as the MMA's M, the band window (up to 32 bins,
 * Re/Im interleaved) as K and the band's NB trials x {Re, Im} as N, each
 * (harmonic, band) is one 128 x 2NB x K product.
 *
 * Precision: both operands are split into fp16 hi + lo (the window scaled by
 * a power of two from the spectrum maximum, the weights by a power of two
 * fixed per session); D = Ahi Bhi + Alo Bhi + Ahi Blo accumulates in FP32 in
 * tensor memory.  The values carry ~22 significant bits instead of the
 * reference's FP32 FMA chain.
 *
 * Roles (one persistent CTA per SM over units (super-tile of 128 column
 * tiles, harmonic), each unit NBAND steps (h, band)):
 *   warps 0-7   stage the window (fp16 hi/lo, canonical K-major layout with
 *               K chunks padded apart so a row's lanes hit 32 banks; warp w
 *               loads rows w, w + 8, ... one bin a lane) into a ring of NSTG
 *               stages; one thread bulk-copies the band's weight images;
 *   warps 8-19  three sets of four, set d owning accumulator buffer d (steps
 *               k = d mod 3): read it (one TMEM lane quarter a warp),
 *               unscale and store X[h][t] as float2 through a shared-memory
 *               transpose (whole 192-byte row segments a store);
 *   warp 20     one thread issues the MMAs (3 passes x K/16 steps).
 * X is harmonic-major: X[(h - 1) * xstride + t].  wsk::search_pre then runs
 * the transform and the boxcar metrics from X (cs_search_ws.cuh).
 *
 * Status: opt-in (CS_B200_TC_INTERP=1, nharms 60), parity-tested.  Measured
 * at N = 2^23: interp_tc 1.87 ms + search_pre 3.11 ms against 4.67 ms for
 * search_ws, which interpolates in its own warps; the interpolation itself is
 * 2.5x cheaper here, but the metric stage alone, without the interpolation
 * warps overlapping it, and the 7.7 GB round trip of X through HBM cost more
 * than it saves.
 */
#pragma once

namespace tci {

constexpr int NB = 24;                  /* trials of a band (q % NB == 0) */
constexpr int NOUT = 2 * NB;            /* MMA N: (trial, Re/Im) */
constexpr int KMAX = 64;                /* halves of a band window (<= 32 bins) */
constexpr int ROWS = 128;               /* column tiles a unit (MMA M) */
constexpr int NSTG = 2;                 /* shared-memory stages */
constexpr int NSW = 8;                  /* staging warps */
constexpr int ND = 3;                   /* accumulator buffers, one epilogue set each */
constexpr int NEW = 4 * ND;             /* epilogue warps: set d = steps k with k % ND == d */
constexpr int NTHREADS = (NSW + NEW + 1) * 32;
/* A images: K chunks of 8 halves (one 16-byte piece per row) 16 bytes more
 * than the 128 rows apart, so the 8 chunks of one row fall in different
 * banks (the staging threads of a row write them together) */
constexpr int LBO_A = ROWS * 16 + 16;
constexpr int A_BYTES = (KMAX / 8) * LBO_A;       /* one fp16 image */
constexpr int B_BYTES = NOUT * KMAX * 2;
constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
constexpr int DCOLS = 64;               /* TMEM columns a D buffer */
constexpr int TMEM_ALLOC = 256;         /* a power of two >= ND * DCOLS */
static_assert(ND * DCOLS <= TMEM_ALLOC, "tensor memory");
constexpr int BAR_BYTES = 8 * (2 * NSTG + 2 * ND) + 16;
constexpr int MAXBAND = 60 * 5;         /* bands staged in shared memory */
constexpr int TROW = 52;                /* transpose row stride (floats): conflict-free */
constexpr int SMEM_BYTES = NSTG * STAGE_BYTES + BAR_BYTES + 16 * MAXBAND + 4 * 64 +
                           NEW * 32 * TROW * 4;

struct Band {
    int rel;        /* R_h(i0): window start from the column tile's base bin */
    int kpad;       /* window halves, a multiple of 16 (<= KMAX) */
    int boff;       /* first uint4 of the band's hi image; lo follows */
    int i0;         /* first trial position of the band */
};

struct Args {
    const float2 *amps;
    long long namps;
    const unsigned *amax;
    const Band *bands;          /* [nh][nband] */
    const uint4 *bimg;          /* weight images */
    const int *hbase;           /* [nh] base bin: rfloor0 + 1 - m/2 */
    int nh, nband, q;
    long long total;            /* trials */
    long long ncol;             /* column tiles */
    long long nunits;           /* super-tiles x nh */
    float inv_sb;               /* 1 / weight scale */
    float2 *X;
    long long xstride;
    int *err;
};

static __host__ __device__ inline size_t b_offset(int rows, int row, int k)
{
    return (size_t)(k >> 3) * (size_t)rows * 16u + (size_t)(row >> 3) * 128u +
           (size_t)(row & 7) * 16u + (size_t)(k & 7) * 2u;
}

/* The band's weight images arrive by bulk copy, counted on the stage's full
 * barrier (expect_tx first, then the copies). */
static __device__ __forceinline__ void expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.expect_tx.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

static __device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes,
                                                uint32_t bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
                 "[%0], [%1], %2, [%3];" ::"r"(dst), "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

static __device__ __forceinline__ uint32_t pack_h2(float a, float b)
{
    const __half2 h = __floats2half2_rn(a, b);
    return *reinterpret_cast<const uint32_t *>(&h);
}

__global__ void __launch_bounds__(NTHREADS, 1) interp_tc(const Args a)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    unsigned char *bars = smem + NSTG * STAGE_BYTES;
    const uint32_t sfull0 = smem_u32(bars);                 /* [NSTG], 8 staging warps */
    const uint32_t sfree0 = sfull0 + 8 * NSTG;              /* [NSTG], MMA commit */
    const uint32_t dfull0 = sfree0 + 8 * NSTG;              /* [ND], MMA commit */
    const uint32_t dempty0 = dfull0 + 8 * ND;               /* [ND], 4 epilogue warps */
    uint32_t *tm_slot = reinterpret_cast<uint32_t *>(bars + 8 * (2 * NSTG + 2 * ND));
    Band *bands_s = reinterpret_cast<Band *>(bars + BAR_BYTES);
    int *hbase_s = reinterpret_cast<int *>(bars + BAR_BYTES + 16 * MAXBAND);
    for (int i = tid; i < a.nh * a.nband; i += NTHREADS) bands_s[i] = a.bands[i];
    for (int i = tid; i < a.nh; i += NTHREADS) hbase_s[i] = a.hbase[i];
    if (warp == 0) tmem_alloc(smem_u32(tm_slot), TMEM_ALLOC);
    if (tid == 0) {
        for (int i = 0; i < NSTG; i++) {
            mbar_init(sfull0 + 8 * i, NSW);
            mbar_init(sfree0 + 8 * i, 1);
        }
        for (int i = 0; i < ND; i++) {
            mbar_init(dfull0 + 8 * i, 1);
            mbar_init(dempty0 + 8 * i, 4);
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tm_slot;
    const long long grid = gridDim.x;

    if (warp < NSW) {
        /* ------------------------------ staging ------------------------------ */
        const float sA = operand_scale(a.amax, 1.0f);
        long long k = 0;
        bool ok = true;
        for (long long u = blockIdx.x; u < a.nunits && ok; u += grid) {
            const long long st = u / a.nh;
            const int h = (int)(u - st * a.nh) + 1;
            const long long c0 = st * ROWS;                 /* first column tile */
            const long long base = (long long)hbase_s[h - 1] + c0 * h;
            for (int b = 0; b < a.nband; b++, k++) {
                const int s = (int)(k % NSTG);
                if (k >= NSTG &&
                    !__all_sync(0xffffffffu, mbar_wait(sfree0 + 8 * s, (uint32_t)((k / NSTG) - 1) & 1u))) {
                    ok = false;
                    break;
                }
                const Band bd = bands_s[(h - 1) * a.nband + b];
                unsigned char *stg = smem + (size_t)s * STAGE_BYTES;
                unsigned char *ahi = stg, *alo = stg + A_BYTES;
                uint4 *bdst = reinterpret_cast<uint4 *>(stg + 2 * A_BYTES);
                /* window: row c = column tile c0 + c, bins base + c h + rel + j.
                 * Warp w takes rows w, w + NSW, ...; lane j loads bin j of the
                 * row (256 contiguous bytes a row) and writes its fp16 pair
                 * into the row's K chunk j / 4 (the padded chunk stride puts
                 * the 32 lanes in 32 banks).  Every load of the step is issued
                 * before the first store. */
                const int nbin = bd.kpad >> 1;
                constexpr int RPW = ROWS / NSW;                 /* rows a warp */
                float2 x[RPW];
#pragma unroll
                for (int q = 0; q < RPW; q++) {
                    const int c = warp + NSW * q;
                    const long long bin = base + (long long)c * h + bd.rel + lane;
                    x[q] = (lane < nbin && bin >= 0 && bin < a.namps) ? __ldg(a.amps + bin)
                                                                      : make_float2(0.0f, 0.0f);
                }
                /* the band's weight images (hi then lo, NOUT x kpad halves each) */
                if (warp == 0 && lane == 0) {
                    const uint32_t nbytes = (uint32_t)(NOUT * bd.kpad * 2);
                    const uint32_t fb = sfull0 + 8 * s;
                    expect_tx(fb, 2 * nbytes);
                    bulk_g2s(smem_u32(bdst), a.bimg + bd.boff, nbytes, fb);
                    bulk_g2s(smem_u32(bdst) + B_BYTES, a.bimg + bd.boff + nbytes / 16, nbytes, fb);
                }
                if (lane < nbin) {
#pragma unroll
                    for (int q = 0; q < RPW; q++) {
                        const int c = warp + NSW * q;
                        const float vr = x[q].x * sA, vi = x[q].y * sA;
                        const __half2 hh = __floats2half2_rn(vr, vi);
                        const float2 back = __half22float2(hh);
                        const size_t off = (size_t)(lane >> 2) * LBO_A + (size_t)(c >> 3) * 128u +
                                           (size_t)(c & 7) * 16u + (size_t)(lane & 3) * 4u;
                        *reinterpret_cast<uint32_t *>(ahi + off) = *reinterpret_cast<const uint32_t *>(&hh);
                        *reinterpret_cast<uint32_t *>(alo + off) = pack_h2(vr - back.x, vi - back.y);
                    }
                }
                fence_proxy_async();
                __syncwarp();
                if (lane == 0) wsk::mbar_arrive(sfull0 + 8 * s);
            }
        }
        if (!ok && lane == 0) atomicExch(a.err, 1);
    } else if (warp < NSW + NEW) {
        /* ------------------------------ epilogue ----------------------------- */
        const int e = (warp - NSW) & 3;                     /* TMEM lanes 32e.. */
        const int db = (warp - NSW) >> 2;                   /* this set's buffer */
        /* this warp's transpose area: 32 rows x NOUT floats */
        float *tr = reinterpret_cast<float *>(bars + BAR_BYTES + 16 * MAXBAND + 4 * 64) +
                    (size_t)(warp - NSW) * 32 * TROW;
        const float sA = operand_scale(a.amax, 1.0f);
        const float unscale = a.inv_sb / sA;                /* exact: powers of two */
        const long long nsteps = ((a.nunits - blockIdx.x + grid - 1) / grid) * a.nband;
        bool ok = true;
        for (long long k = db; k < nsteps && ok; k += ND) {
            const long long ui = k / a.nband;
            const int b = (int)(k - ui * a.nband);
            const long long u = blockIdx.x + ui * grid;
            const long long st = u / a.nh;
            const int h = (int)(u - st * a.nh) + 1;
            if (!__all_sync(0xffffffffu, mbar_wait(dfull0 + 8 * db, (uint32_t)(k / ND) & 1u))) {
                ok = false;
                break;
            }
            tc_fence_after();
            /* through shared memory, so that a warp's store covers whole
             * row segments (192 B each) instead of 32 separate lines */
            const uint32_t ta = tmem + (uint32_t)(db * DCOLS) + ((uint32_t)(e * 32) << 16);
            {
                float v[32];
                tmem_ld32(ta, v);
#pragma unroll
                for (int p = 0; p < 8; p++)
                    *reinterpret_cast<float4 *>(tr + lane * TROW + 4 * p) =
                        make_float4(v[4 * p] * unscale, v[4 * p + 1] * unscale,
                                    v[4 * p + 2] * unscale, v[4 * p + 3] * unscale);
            }
            {
                float v[16];
                tmem_ld16(ta + 32, v);
#pragma unroll
                for (int p = 0; p < 4; p++)
                    *reinterpret_cast<float4 *>(tr + lane * TROW + 32 + 4 * p) =
                        make_float4(v[4 * p] * unscale, v[4 * p + 1] * unscale,
                                    v[4 * p + 2] * unscale, v[4 * p + 3] * unscale);
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) wsk::mbar_arrive(dempty0 + 8 * db);
            const Band bd = bands_s[(h - 1) * a.nband + b];
            constexpr int CH = NOUT / 4;                /* float4 chunks a row (2 trials each) */
            float2 *xh = a.X + (long long)(h - 1) * a.xstride;
#pragma unroll
            for (int q = 0; q < CH; q++) {
                const int it = lane + 32 * q;           /* (row, chunk) of 32 x CH */
                const int r = it / CH, p = it - r * CH;
                const long long cgr = st * ROWS + e * 32 + r;
                const long long t = cgr * a.q + bd.i0 + 2 * p;
                const float4 w = *reinterpret_cast<const float4 *>(tr + r * TROW + 4 * p);
                if (cgr < a.ncol) {
                    if (t + 1 < a.total) *reinterpret_cast<float4 *>(xh + t) = w;
                    else if (t < a.total) xh[t] = make_float2(w.x, w.y);
                }
            }
            __syncwarp();
        }
        if (!ok && lane == 0) atomicExch(a.err, 1);
    } else if (lane == 0) {
        /* -------------------------------- MMA -------------------------------- */
        const uint32_t idesc = (1u << 4) | ((uint32_t)(NOUT >> 3) << 17) |
                               ((uint32_t)(ROWS >> 4) << 24);
        const uint32_t lbo_a = LBO_A, lbo_b = NOUT * 16;
        long long k = 0, issued = 0;
        bool ok = true;
        for (long long u = blockIdx.x; u < a.nunits && ok; u += grid) {
            const long long st = u / a.nh;
            const int h = (int)(u - st * a.nh) + 1;
            for (int b = 0; b < a.nband; b++, k++) {
                const int s = (int)(k % NSTG), db = (int)(k % ND);
                if (!mbar_wait(sfull0 + 8 * s, (uint32_t)(k / NSTG) & 1u)) { ok = false; break; }
                if (k >= ND && !mbar_wait(dempty0 + 8 * db, (uint32_t)((k / ND) - 1) & 1u)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const Band bd = bands_s[(h - 1) * a.nband + b];
                const uint32_t stg = smem_u32(smem + (size_t)s * STAGE_BYTES);
                const uint32_t ahi = stg, alo = stg + A_BYTES;
                const uint32_t bhi = stg + 2 * A_BYTES, blo = bhi + B_BYTES;
                const uint32_t d = tmem + (uint32_t)(db * DCOLS);
                uint32_t acc = 0;
#pragma unroll
                for (int pass = 0; pass < 3; pass++) {
                    const uint32_t ab = pass == 1 ? alo : ahi;
                    const uint32_t bb = pass == 2 ? blo : bhi;
                    for (int ks = 0; ks < (bd.kpad >> 4); ks++) {
                        mma_f16(d, umma_desc(ab + (uint32_t)ks * 2 * lbo_a, lbo_a, 128),
                                umma_desc(bb + (uint32_t)ks * 2 * lbo_b, lbo_b, 128), idesc, acc);
                        acc = 1;
                    }
                }
                mma_commit(sfree0 + 8 * s);
                mma_commit(dfull0 + 8 * db);
                issued++;
            }
        }
        if (!ok) atomicExch(a.err, 1);
        /* drain: the last commits of each accumulator landed before the
         * tensor memory is released */
        for (long long j = issued > ND ? issued - ND : 0; j < issued; j++)
            mbar_wait(dfull0 + 8 * (int)(j % ND), (uint32_t)(j / ND) & 1u);
    }
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, TMEM_ALLOC);
    }
}

}  // namespace tci
